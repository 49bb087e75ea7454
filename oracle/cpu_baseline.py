"""Timed CPU baseline of the depth stage on bounded samples (oracle, CPU only).

The reference stage on the full-resolution five-view workload costs minutes of
CPU time, so the baseline runs the oracle's whole stage on a sample of coarse
rows and reports what it measured: SGM cells of the sampled nodes over the
sample's wall time. Nothing is extrapolated.

The sample keeps the reference's threading. build_cost_volume and
measure_direct_depths split all grid rows into one contiguous band per worker
(depth.rs:1204-1206, 729-731); a sample takes the same number of rows from every
band, at the same offset inside each band, so every worker is busy exactly as in
a full run (a few adjacent rows would fall into one worker's band and run on one
thread). The SGM, winner-take-all, filters and per-target decisions run on one
thread, as in the reference, over the sampled rows (oracle_stage_sample).
Successive samples step the offset through the bands, so a run of samples covers
the image from its top edge to its bottom edge.

Test infrastructure: only the benchmark's CPU-baseline leg and its reference arm
call this.
"""
from __future__ import annotations

import ctypes as C
import os
import statistics
import time

import numpy as np

from chiaro_b200.depth import output_shape, pack_views

from . import oracle

STAGES = ("cost_volume", "sgm", "select", "direct", "filters", "decisions")


def worker_bands(rows: int, threads: int):
    """The reference's row bands: (first_row, last_row) per worker (depth.rs:1204-1206)."""
    workers = max(1, min(threads, rows))
    per = -(-rows // workers)
    return [(a, min(a + per, rows)) for a in range(0, rows, per)]


def sample_mask(rows: int, threads: int, offset: int, rows_per_band: int = 1) -> np.ndarray:
    """Coarse rows offset .. offset + rows_per_band - 1 (modulo its length) of every worker band."""
    mask = np.zeros(rows, np.uint8)
    for a, b in worker_bands(rows, threads):
        n = b - a
        for j in range(rows_per_band):
            mask[a + (offset + j) % n] = 1
    return mask


def run_sample(scene, offset: int, threads: int = 0, rows_per_band: int = 1) -> dict:
    """The whole stage on one sample; returns its measured stage times and rate."""
    threads = threads or (os.cpu_count() or 1)
    opt = scene.options
    o = opt.to_c()
    views, keep = pack_views(scene.inputs(), scene.alignments())
    _, (cc, cr, _) = output_shape(scene.width, scene.height, opt)
    mask = sample_mask(cr, threads, offset, rows_per_band)
    seconds = np.zeros(6)
    counts = np.zeros(2, np.uint64)
    t0 = time.perf_counter()
    st = oracle.lib().oracle_stage_sample(views, len(scene.cameras), scene.reference_index, C.byref(o),
                                          mask.ctypes.data_as(C.POINTER(C.c_uint8)), threads,
                                          seconds.ctypes.data_as(C.POINTER(C.c_double)),
                                          counts.ctypes.data_as(C.POINTER(C.c_uint64)))
    wall = time.perf_counter() - t0
    assert st == 0, st
    cells = int(counts[0]) * (opt.planes + 1) * 8
    stage_total = float(seconds.sum())
    return dict(stage_seconds=dict(zip(STAGES, seconds.tolist())), seconds=stage_total, wall_seconds=wall,
                cells=cells, gcells_per_s=cells / stage_total / 1e9, coarse_nodes=int(counts[0]),
                fine_nodes=int(counts[1]), rows=[int(r) for r in np.flatnonzero(mask)], coarse_rows=cr,
                threads=threads, offset=offset)


def run_samples(scene, offsets, threads: int = 0, rows_per_band: int = 1) -> dict:
    """Several samples; the rate is all sampled cells over all measured seconds."""
    runs = [run_sample(scene, k, threads, rows_per_band) for k in offsets]
    cells = sum(r["cells"] for r in runs)
    seconds = sum(r["seconds"] for r in runs)
    rates = [r["gcells_per_s"] for r in runs]
    stage = {s: sum(r["stage_seconds"][s] for r in runs) for s in STAGES}
    first = runs[0]
    bands = len(worker_bands(first["coarse_rows"], first["threads"]))
    return dict(gcells_per_s=cells / seconds / 1e9, cells=cells, seconds=seconds,
                wall_seconds=sum(r["wall_seconds"] for r in runs), samples=len(runs), threads=first["threads"],
                stage_seconds=stage,
                spread={"min_gcells_s": min(rates), "max_gcells_s": max(rates),
                        "stdev_over_mean": (statistics.pstdev(rates) / statistics.mean(rates)) if len(rates) > 1
                        else 0.0},
                sample=(f"whole stage on {rows_per_band} coarse row(s) in each of the {bands} worker bands of the "
                        f"{first['coarse_rows']} coarse rows (offsets {list(offsets)} inside each band, so the "
                        f"samples span the image top to bottom), with the fine rows they seed; cost volume and "
                        f"direct pass on {first['threads']} threads in the reference's row bands, SGM, "
                        f"winner-take-all, filters and per-target decisions on one thread; measured, not "
                        f"extrapolated"))


def run_whole(scene, threads: int = 0) -> dict:
    """The oracle's whole stage on the full workload (for sizes that take seconds)."""
    threads = threads or (os.cpu_count() or 1)
    _, (cc, cr, _) = output_shape(scene.width, scene.height, scene.options)
    t0 = time.perf_counter()
    out = oracle.refine_multiview_depth(scene.inputs(), scene.reference_index, scene.alignments(), scene.options,
                                        threads=threads)
    seconds = time.perf_counter() - t0
    assert out is not None
    cells = cc * cr * (scene.options.planes + 1) * 8
    return dict(gcells_per_s=cells / seconds / 1e9, seconds=seconds, cells=cells, threads=threads,
                sample="the whole stage on the full workload (oracle_refine_multiview_depth), every step")
