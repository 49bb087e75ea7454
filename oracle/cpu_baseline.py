"""Timed CPU baseline of the depth stage on a bounded sample (oracle, CPU only).

The reference stage on the full-resolution five-view workload costs tens of
CPU-minutes (its per-target loop is serial), so the baseline times each stage
of the oracle on a band of rows of the same workload and scales each stage by
the node count it covers:

  * cost volume: ``band`` coarse rows, all host threads (row bands, as
    depth.rs:1204-1206 threads it);
  * SGM and winner-take-all: the full-size volume, one thread (depth.rs runs
    both serially); SGM time does not depend on the cost values, so the volume
    is the band's costs tiled to full size;
  * direct measurement: the matching 2*band fine rows, all host threads, seeded
    by the band's own SGM field;
  * consistency filters and per-target decisions: the fine band, one thread
    (serial in the reference).

The returned estimate is the whole stage's CPU time for the full workload.
Test infrastructure: only the benchmark's CPU-baseline leg and its reference
arm call this.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from chiaro_b200.abi import dptr, fptr, u8ptr
from chiaro_b200.depth import output_shape, pack_views

from . import oracle


def run_sample(scene, band: int = 4, threads: int = 0, row0: int = None) -> dict:
    L = oracle.lib()
    threads = threads or (os.cpu_count() or 1)
    opt = scene.options
    o = opt.to_c()
    inputs, alignments = scene.inputs(), scene.alignments()
    views, keep = pack_views(inputs, alignments)
    n_views = len(inputs)
    ref = scene.reference_index
    (cols, rows, step), (cc, cr, cs) = output_shape(scene.width, scene.height, opt)
    D = opt.planes + 1
    N, M = cc * cr, cols * rows
    a = (cr - band) // 2 if row0 is None else row0
    b = a + band
    times = {}
    # cost volume on the band
    scores = np.zeros(N * D, np.float32)
    costs = np.zeros(N * D, np.float32)
    guidance = np.zeros(N, np.float32)
    tested = np.zeros(N, np.uint8)
    t = time.perf_counter()
    L.oracle_build_cost_volume(views, n_views, ref, C.byref(o), a, b, fptr(scores), fptr(costs), fptr(guidance),
                               u8ptr(tested), threads)
    times["cost_volume"] = (time.perf_counter() - t) * N / (band * cc)
    # SGM + select on the full volume (band tiled)
    sl = slice(a * cc * D, b * cc * D)
    full_costs = np.resize(costs[sl], N * D).astype(np.float32)
    full_scores = np.resize(scores[sl], N * D).astype(np.float32)
    full_guid = np.resize(guidance[a * cc:b * cc], N).astype(np.float32)
    full_tested = np.resize(tested[a * cc:b * cc], N).astype(np.uint8)
    reg = np.empty(N * D, np.float32)
    t = time.perf_counter()
    L.oracle_semi_global_costs(fptr(full_costs), fptr(full_guid), cc, cr, D, fptr(reg))
    times["sgm"] = time.perf_counter() - t
    labels = np.concatenate([[np.nan], np.array(_inverse_depth_samples(opt.near_depth, opt.far_depth,
                                                                       opt.planes))[::-1]])
    has = np.zeros(N, np.uint8)
    depth = np.zeros(N)
    conf = np.zeros(N, np.float32)
    imp = np.zeros(N, np.float32)
    regz = np.zeros(N, np.uint8)
    fill = np.zeros(N, np.uint8)
    t = time.perf_counter()
    L.oracle_select_depths(dptr(labels), D, fptr(full_scores), fptr(reg), u8ptr(full_tested), N, C.byref(o),
                           u8ptr(has), dptr(depth), fptr(conf), fptr(imp), u8ptr(regz), u8ptr(fill))
    times["select"] = time.perf_counter() - t
    # the band's own SGM field seeds the direct pass
    band_costs = np.ascontiguousarray(costs[sl])
    band_reg = np.empty_like(band_costs)
    L.oracle_semi_global_costs(fptr(band_costs), fptr(np.ascontiguousarray(guidance[a * cc:b * cc])), cc, band, D,
                               fptr(band_reg))
    c_has = np.zeros(N, np.uint8)
    c_depth = np.zeros(N)
    c_conf = np.zeros(N, np.float32)
    c_imp = np.zeros(N, np.float32)
    c_reg = np.zeros(N, np.uint8)
    c_fill = np.zeros(N, np.uint8)
    bn = band * cc
    L.oracle_select_depths(dptr(labels), D, fptr(np.ascontiguousarray(scores[sl])), fptr(band_reg),
                           u8ptr(np.ascontiguousarray(tested[a * cc:b * cc])), bn, C.byref(o),
                           u8ptr(c_has[a * cc:]), dptr(c_depth[a * cc:]), fptr(c_conf[a * cc:]),
                           fptr(c_imp[a * cc:]), u8ptr(c_reg[a * cc:]), u8ptr(c_fill[a * cc:]))
    fa, fb = 2 * a, min(rows, 2 * b)
    f_has = np.zeros(M, np.uint8)
    f_depth = np.zeros(M)
    f_conf = np.zeros(M, np.float32)
    f_imp = np.zeros(M, np.float32)
    f_guid = np.zeros(M, np.float32)
    f_tested = np.zeros(M, np.uint8)
    t = time.perf_counter()
    L.oracle_measure_direct_depths(views, n_views, ref, C.byref(o), u8ptr(c_has), dptr(c_depth), fptr(c_conf),
                                   fptr(c_imp), u8ptr(c_reg), fa, fb, u8ptr(f_has), dptr(f_depth), fptr(f_conf),
                                   fptr(f_imp), fptr(f_guid), u8ptr(f_tested), threads)
    fine_band = (fb - fa) * cols
    times["direct"] = (time.perf_counter() - t) * M / fine_band
    # filters on the fine band (its own grid)
    fs = slice(fa * cols, fb * cols)
    bh = np.ascontiguousarray(f_has[fs])
    bd = np.ascontiguousarray(f_depth[fs])
    bc = np.ascontiguousarray(f_conf[fs])
    bg = np.ascontiguousarray(f_guid[fs])
    istep = (1.0 / opt.near_depth - 1.0 / opt.far_depth) / (opt.planes - 1)
    t = time.perf_counter()
    L.oracle_reject_isolated(u8ptr(bh), dptr(bd), fptr(bc), fptr(bg), cols, fb - fa, istep * 2.5)
    L.oracle_reject_small_components(u8ptr(bh), dptr(bd), fptr(bg), cols, fb - fa, istep * 2.5, 24)
    L.oracle_fit_local_planes(u8ptr(bh), dptr(bd), fptr(bc), fptr(bg), cols, fb - fa, istep * 4.0)
    times["filters"] = (time.perf_counter() - t) * M / fine_band
    f_has[fs] = bh
    f_depth[fs] = bd
    kinds = np.zeros(fine_band, np.uint8)
    f_regz = np.zeros(M, np.uint8)
    t = time.perf_counter()
    n_targets = 0
    for tgt in range(n_views):
        if tgt == ref or not alignments[tgt].report.accepted or inputs[tgt].camera is None:
            continue
        n_targets += 1
        L.oracle_target_decisions(views, n_views, ref, tgt, C.byref(o), u8ptr(f_has), dptr(f_depth), fptr(f_conf),
                                  u8ptr(f_regz), fptr(f_guid), fa, fb, u8ptr(kinds))
    times["decisions"] = (time.perf_counter() - t) * M / fine_band
    total = sum(times.values())
    cells = N * D * 8
    return dict(stage_seconds=times, total_seconds=total, cells=cells, gcells_per_s=cells / total / 1e9,
                threads=threads, band_coarse_rows=band, coarse_rows=cr, fine_rows=fb - fa, targets=n_targets,
                sample=(f"coarse rows {a}-{b - 1} of {cr} (cost volume, {threads} threads), fine rows {fa}-{fb - 1} "
                        f"of {rows} (direct pass, {threads} threads; filters and {n_targets} targets' decisions "
                        f"serial), full-size SGM and winner-take-all serial; each stage scaled by node count"))


def _inverse_depth_samples(near, far, count):
    out = np.empty(count)
    oracle.lib().oracle_inverse_depth_samples(near, far, count, dptr(out))
    return out
