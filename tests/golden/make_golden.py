"""Write the golden fixtures of tests/golden from seeded scenes and the oracle.

    python tests/golden/make_golden.py

The inputs are taken from chiaro_b200.scenes (seeded ray-cast scenes) and stored
in the C ABI's own form; the outputs are the oracle's (oracle/chiaro_oracle.cpp,
the CPU restatement of crates/chiaro-fusion/src/depth.rs:312-580).
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE.parent))

from chiaro_b200 import scenes  # noqa: E402
from chiaro_b200.depth import output_shape, pack_views  # noqa: E402
from golden import fixture  # noqa: E402
from oracle import oracle  # noqa: E402

SPECS = {"tiny_seed2": ("tiny", 2), "small_seed5": ("small", 5)}


def make(name: str):
    workload, seed = SPECS[name]
    sc = scenes.workload(workload, seed=seed)
    inputs, alignments = sc.inputs(), sc.alignments()
    views, keep = pack_views(inputs, alignments)
    (cols, rows, step), (cc, cr, cs) = output_shape(sc.width, sc.height, sc.options)
    g = {"n_views": np.int64(len(inputs)), "reference_index": np.int64(sc.reference_index),
         "fine_nodes": np.int64(cols * rows), "coarse_nodes": np.int64(cc * cr),
         "labels": np.int64(sc.options.planes + 1),
         "options": np.frombuffer(bytes(sc.options.to_c()), np.uint8).copy()}
    for i, (inp, al) in enumerate(zip(inputs, alignments)):
        v = views[i]
        g[f"luma{i}"] = np.ascontiguousarray(inp.luminance.data, np.float32)
        g[f"view{i}"] = np.array([v.width, v.height, v.has_camera, v.accepted], np.int64)
        g[f"camera{i}"] = np.frombuffer(bytes(v.camera), np.uint8).copy()
        g[f"warp_shape{i}"] = np.array([al.warp.step, al.warp.columns, al.warp.rows], np.int64)
        g[f"warp_points{i}"] = np.ascontiguousarray(al.warp.points, np.float32).reshape(-1)
        g[f"warp_confidence{i}"] = np.ascontiguousarray(al.warp.confidence, np.float32).reshape(-1)
    out = fixture.run(g, oracle.lib().oracle_refine_multiview_depth, extra=(1,))
    g.update(out)
    np.savez_compressed(HERE / f"{name}.npz", **g)
    print(name, (HERE / f"{name}.npz").stat().st_size, "bytes")


if __name__ == "__main__":
    for name in (sys.argv[1:] or fixture.NAMES):
        make(name)
