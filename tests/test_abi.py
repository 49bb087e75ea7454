"""The C ABI library loads and exports every symbol its header declares (CPU).

No compute entry point is called here (there is no GPU); the calls that are
made are pure host functions (options, shapes, version).
"""
import ctypes as C
import re
from pathlib import Path

import numpy as np

from chiaro_b200 import abi, build, runtime
from chiaro_b200.depth import DepthOptions, output_shape

HEADER = Path(__file__).resolve().parent.parent / "include" / "chiaro_depth.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(chiaro_[a-z0-9_]+)\s*\(", text)))


def test_header_declarations_are_bound_and_exported():
    build.build()
    lib = runtime.load_library()
    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
        assert name in runtime.SIGNATURES, f"{name} has no ctypes signature"


def test_struct_layouts_match_the_header(tmp_path):
    """Compile the header with the host C compiler and compare every struct's
    size and field offsets with the ctypes mirror."""
    import subprocess
    structs = {"chiaro_depth_options": abi.DepthOptionsC, "chiaro_camera": abi.CameraC, "chiaro_warp": abi.WarpC,
               "chiaro_view": abi.ViewC, "chiaro_depth_map": abi.DepthMapC, "chiaro_depth_report": abi.DepthReportC,
               "chiaro_depth_debug": abi.DepthDebugC, "chiaro_vignetting": abi.VignettingC,
               "chiaro_sgm_instance": abi.SgmInstanceC, "chiaro_band_options": abi.BandOptionsC,
               "chiaro_band_report": abi.BandReportC, "chiaro_resolution_report": abi.ResolutionReportC,
               "chiaro_align_input": abi.AlignInputC, "chiaro_align_options": abi.AlignOptionsC,
               "chiaro_align_level": abi.AlignLevelC, "chiaro_alignment_report": abi.AlignmentReportC}
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'printf("{cname}.{field} %zu\\n", offsetof({cname}, {field}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    out = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                              text=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(out[cname]) == C.sizeof(py), cname
        for field, _ in py._fields_:
            assert int(out[f"{cname}.{field}"]) == getattr(py, field).offset, (cname, field)


def test_host_side_entry_points():
    lib = runtime.load_library()
    assert lib.chiaro_depth_abi_version() == abi.ABI_VERSION
    o = abi.DepthOptionsC()
    lib.chiaro_depth_options_default(C.byref(o))
    d = DepthOptions()
    assert (o.grid_step, o.near_depth, o.far_depth, o.planes, o.patch_radius) == (8, 500.0, 1e7, 96, 4)
    assert (o.minimum_support, o.best_view_count) == (2, 3)
    assert np.float32(o.minimum_score) == np.float32(d.minimum_score)
    assert lib.chiaro_depth_options_valid(C.byref(o)) == 1
    bad = d.to_c()
    bad.best_view_count = 1
    assert lib.chiaro_depth_options_valid(C.byref(bad)) == 0
    vals = [C.c_uint64() for _ in range(6)]
    assert lib.chiaro_depth_output_shape(4160, 3120, C.byref(o), *[C.byref(v) for v in vals]) == abi.OK
    (cols, rows, step), (cc, cr, cs) = output_shape(4160, 3120, d)
    assert [v.value for v in vals] == [cols, rows, step, cc, cr, cs] == [1041, 781, 4, 521, 391, 8]


def test_invalid_options_map_to_none_without_a_device():
    # validation happens before any device work, so this runs on the CPU box
    from chiaro_b200 import scenes
    from chiaro_b200.depth import pack_views
    lib = runtime.load_library()
    sc = scenes.workload("tiny", seed=1)
    views, keep = pack_views(sc.inputs(), sc.alignments())
    opt = DepthOptions(planes=2).to_c()
    reports = (abi.DepthReportC * 3)()
    status = lib.chiaro_refine_multiview_depth(None, views, 3, 0, C.byref(opt), None, reports, None, None)
    assert status == abi.ERR_ARGUMENT  # a NULL context is rejected before anything else
