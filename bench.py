#!/usr/bin/env python
"""Benchmark of the B200 depth stage (one JSON line on rank 0).

A step is one full pass of the depth stage (refine_multiview_depth,
crates/chiaro-fusion/src/depth.rs:312-580) over the full-resolution five-view
workload: a 4160x3120 reference plus 4 sources, 128 planes over 0.4-50 m,
coarse SGM grid 521x391 (D = 129), direct grid 1041x781. The metric counts
SGM cells (coarse nodes x labels x 8 directions) per second of the whole
stage, so every stage of the step is inside the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm runs with inputs resident in HBM (value) and through the public host
API with pinned host inputs (e2e: one call per frame, its copies and its stage one after the
other), with pageable inputs (e2e_pageable), and as a stream of frames whose copies overlap
the neighbouring frames' stages (e2e_pipelined, chiaro_b200.depth.DepthPipeline). With N > 1 (torchrun) every rank processes
its own replica of the workload (the stage shards by capture; no collective on
the data path): value is the total over ranks, timed as the maximum over ranks.
The reference arm times the CPU oracle (a C++ restatement of the reference's
Rust code): each step is the whole stage on a bounded sample of the same
workload (one coarse row in each of the reference's worker bands, with the
fine rows they seed; the steps step through the bands, top to bottom), or the
whole workload where it takes seconds (two_view). Its value is the SGM cells of
what it processed over the time it took: measured, not extrapolated.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from datetime import timedelta
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "SGM Gcells/s (px·planes·dirs) on 1 B200; learned-band vs full @≥99% agreement"
UNIT = "Gcells/s"
WORKLOAD_TEXT = {
    "five_view": ("five_view: 4160x3120 reference + 4 sources (20-60 mm baselines, <=0.5 deg), 12 slanted planes + "
                  "3 spheres, 128 planes over 0.4-50 m, default DepthOptions; coarse grid step 8 = 521x391 nodes, "
                  "D = 129 labels; direct grid step 4 = 1041x781"),
    "two_view": ("two_view: 1040x780 reference + 1 source (25 mm), 6 slanted planes, 64 planes over 0.4-25 m, "
                 "minimum_support = best_view_count = 1; coarse grid 131x99, D = 65"),
}


def parse_args():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", default="five_view", choices=sorted(WORKLOAD_TEXT))
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--rows-per-band", type=int, default=1,
                   help="coarse rows per worker band in each CPU sample step")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--e2e-steps", type=int, default=0, help="steps of the end-to-end leg (0 = --steps)")
    p.add_argument("--band-eval", type=int, default=8, help="held-out 1040x780 scenes of the band evaluation")
    p.add_argument("--band-eval-full", type=int, default=2,
                   help="held-out full-resolution five-view scenes of the band evaluation")
    p.add_argument("--captures", type=int, default=32, help="captures of the config-4 stream")
    p.add_argument("--no-learned-band", action="store_true")
    p.add_argument("--no-configs", action="store_true", help="skip the per-config sub-objects (two_view, ...)")
    p.add_argument("--profile-case", choices=["stage", "sgm", "bandnet", "coarse"], default=None,
                   help="run only one case's kernels, for an ncu capture (small device footprint): the five-view "
                        "stage (3 warm-up calls and one more), its SGMs (f32 and u16) on a five-view-shaped volume, "
                        "or the band network (a full-resolution proposal and a training step), or the coarse "
                        "search on five_view with the default CTA shape (plain, then the naive band: the cost "
                        "volume at 129, 17 and 25 labels per node)")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(value: float, world: int, device=None) -> float:
    """The maximum of `value` over all ranks (the slowest rank's time); `value` itself on one rank.
    Every rank calls it at the same point (NCCL on the GPUs in the benchmark, gloo in the CPU tests)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, cells_per_step: int, steps: int, seconds: float) -> float:
    """Whole-job Gcells/s: every rank processes its own replica of the workload (weak scaling)."""
    return world * cells_per_step * steps / seconds / 1e9


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        rows = [line.split(",") for line in Path(self.path).read_text().splitlines() if line.count(",") >= 8]
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i] and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs"), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def sgm_traffic():
    """DRAM bytes of one SGM stage call on five_view from the committed ncu capture, or None."""
    import re
    f = ROOT / "profiles" / "sgm_five_view_dram.md"
    if not f.exists():
        return None
    m = re.search(r"traffic_bytes_per_call = (\d+)", f.read_text())
    return int(m.group(1)) if m else None


def correlation_instructions():
    """Warp instructions per launch of the correlation kernels on five_view, from the
    committed ncu capture (profiles/correlation_issue_five_view.md), or {}."""
    import re
    f = ROOT / "profiles" / "correlation_issue_five_view.md"
    if not f.exists():
        return {}
    return {m.group(1): int(m.group(2)) for m in re.finditer(r"warp_instructions ([\w<>]+) = (\d+)", f.read_text())}


def issue_roofline(stage_ms, sm_mhz, cost_threads=None):
    """Instruction-issue fractions of the correlation stages: warp instructions per launch
    (ncu) over the stage's event time at 148 SMs x 4 schedulers x one instruction per cycle.
    cost_threads: the CTA size the autotuner chose for the cost volume (its count differs
    by shape)."""
    counts = correlation_instructions()
    if not counts:
        return None
    peak = 148 * 4 * sm_mhz * 1e6
    cost = f"cost_volume_kernel<{cost_threads}>" if f"cost_volume_kernel<{cost_threads}>" in counts \
        else "cost_volume_kernel"
    # the fine reference patches run right after the tap lattice, inside the cost volume's events
    stages = {"cost_volume": [cost, "patch_sums_kernel"], "direct": ["direct_depth_kernel", "direct_wide_kernel"],
              "decisions": ["target_decision_kernel"]}
    out = {"unit": "warp instructions / s", "peak": peak, "peak_source": f"148 SMs x 4 schedulers at {sm_mhz:.0f} MHz",
           "instructions_source": "profiles/correlation_issue_five_view.md (ncu smsp__inst_executed.sum, one launch)"}
    for stage, kernels in stages.items():
        inst = sum(counts.get(k, 0) for k in kernels)
        if inst and stage_ms.get(stage):
            achieved = inst / (stage_ms[stage] / 1e3)
            out[stage] = {"kernels": kernels, "warp_instructions": inst, "achieved": round(achieved / 1e9, 1),
                          "frac": round(achieved / peak, 4)}
    return out


def stage_bytes(scene):
    """Algorithmic work per step: SGM compulsory bytes and SGM cells."""
    from chiaro_b200.depth import output_shape
    (cols, rows, step), (cc, cr, cs) = output_shape(scene.width, scene.height, scene.options)
    n, d = cc * cr, scene.options.planes + 1
    targets = len(scene.cameras) - 1
    taps = (2 * scene.options.patch_radius + 1) ** 2
    return {"coarse_nodes": n, "labels": d, "fine_nodes": cols * rows, "cells": n * d * 8,
            # read the data-cost volume once, write the aggregate once, guidance per direction
            "sgm_bytes": n * d * 8 + 8 * n * 4,
            # cost build: N * D * V * (2r + 1)^2 taps at 16 FP32 FLOP per tap (3 lerps, 3 moments,
            # coordinate and weight products)
            "cost_taps": n * d * targets * taps, "cost_flop": 16 * n * d * targets * taps}


def run_ours(args, rank, world, local):
    import numpy as np
    import torch
    import torch.distributed as dist

    from chiaro_b200 import build, scenes
    from chiaro_b200.depth import DeviceStage, refine_multiview_depth
    from chiaro_b200.runtime import DepthContext

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(minutes=10), device_id=device)
    build.build()
    scene = scenes.workload(args.workload, seed=args.seed)
    work = stage_bytes(scene)
    ctx = DepthContext(local)
    n = len(scene.cameras)
    M = work["fine_nodes"]
    # planes, warps and outputs resident in HBM: the device-buffer entry point
    stage = DeviceStage(scene.inputs(), scene.reference_index, scene.alignments(), scene.options, context=ctx)
    assert stage.nodes == M

    def step():
        if not stage():
            raise RuntimeError("the stage returned None on the benchmark workload")

    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)  # > 126 MB L2
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    durations, stages = [], []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        step()
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        durations.append(e0.elapsed_time(e1))
        stages.append(ctx.timings())
    torch.cuda.synchronize()
    clk = clocks.stop()
    if world > 1:
        dist.barrier()
    total_ms = float(sum(durations))
    launches = ctx.launches()
    total_ms = max_over_ranks(total_ms, world, device)
    value = whole_job_rate(world, work["cells"], args.steps, total_ms / 1e3)
    stage_ms = {k: statistics.median(s[k] for s in stages) for k in stages[0]}

    # end to end through the public API: pinned host inputs, host outputs
    e2e_steps = args.e2e_steps or args.steps
    inputs = scene.inputs()
    for inp in inputs:
        pinned = torch.empty(inp.luminance.data.size, dtype=torch.float32, pin_memory=True).numpy()
        pinned[:] = inp.luminance.data.reshape(-1)
        inp.luminance.data = pinned.reshape(inp.luminance.height, inp.luminance.width)
    result = None
    for _ in range(max(args.warmup, 2)):  # steady state: the output pool holds two result sets
        result = refine_multiview_depth(inputs, scene.reference_index, scene.alignments(), scene.options,
                                        context=ctx)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2e = []
    for _ in range(e2e_steps):
        alignments = scene.alignments()
        t0 = time.perf_counter()
        result = refine_multiview_depth(inputs, scene.reference_index, alignments, scene.options, context=ctx)
        e2e.append(time.perf_counter() - t0)
        assert result is not None
    e2e_s = max_over_ranks(float(sum(e2e)), world, device)
    targets = sum(1 for i in range(n) if i != scene.reference_index)
    h2d = sum(l.data.nbytes for l in scene.luminance) + sum(w.points.nbytes + w.confidence.nbytes
                                                            for w in scene.warps)
    d2h = M * (8 + 4 + 1) + targets * M * (8 + 4)
    e2e_value = whole_job_rate(world, work["cells"], e2e_steps, e2e_s)
    # the same public call with the scene's own (pageable) numpy planes, as a caller that
    # hands ordinary host vectors makes it
    pageable = scene.inputs()
    for _ in range(max(args.warmup, 2)):
        refine_multiview_depth(pageable, scene.reference_index, scene.alignments(), scene.options, context=ctx)
    e2e_pageable = []
    for _ in range(e2e_steps):
        alignments = scene.alignments()
        t0 = time.perf_counter()
        result = refine_multiview_depth(pageable, scene.reference_index, alignments, scene.options, context=ctx)
        e2e_pageable.append(time.perf_counter() - t0)
        assert result is not None
    e2e_pageable_s = max_over_ranks(float(sum(e2e_pageable)), world, device)
    # a stream of frames through DepthPipeline: each step uploads its frame (planes and warps,
    # pinned) and reads back its outputs, overlapping the neighbouring frames' stages; the
    # timed region holds the first upload and the last read-back
    from chiaro_b200.depth import DepthPipeline
    pipe = DepthPipeline(scene.inputs(), scene.reference_index, scene.alignments(), scene.options, context=ctx)

    def pinned_flat(a):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32).reshape(-1)).pin_memory()

    frame = ([pinned_flat(l.data) for l in scene.luminance], [pinned_flat(w.points) for w in scene.warps],
             [pinned_flat(w.confidence) for w in scene.warps])
    for _ in pipe.run([frame] * max(args.warmup, 2)):
        pass
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    frames_ok = sum(1 for ok, _ in pipe.run([frame] * e2e_steps) if ok)
    pipelined_s = time.perf_counter() - t0
    assert frames_ok == e2e_steps
    pipelined_s = max_over_ranks(pipelined_s, world, device)
    pipelined = {"value": round(whole_job_rate(world, work["cells"], e2e_steps, pipelined_s), 3), "unit": UNIT,
                 "ms_per_step": round(1e3 * pipelined_s / e2e_steps, 3),
                 "h2d_bytes_per_step": int(pipe.bytes_up[-1]), "d2h_bytes_per_step": int(pipe.bytes_down[-1]),
                 "api": "chiaro_b200.depth.DepthPipeline.run (a stream of pinned host frames; each step uploads "
                        "its frame and reads back its outputs while the neighbouring frames' stages run)"}
    del pipe

    configs = {}
    if args.workload == "five_view" and not args.no_configs:
        configs["two_view"] = two_view_config(args, ctx, torch, stream, flush, rank == 0 and world == 1)
    graph = stage_graph(args, torch, stream, flush, stage)
    finest = finest_coarse_grid(args, scene, stage, torch, stream, flush)
    resolution = resolution_warp(args, scene, ctx)
    alignment = global_alignment(args, scene, ctx)
    quantised = quantised_sgm(args, scene, work, ctx, torch, device, stream, flush)
    batched = batched_sgm(args, ctx, torch, device, stream, flush)
    band = None
    if world == 1 and not args.no_learned_band:
        band = learned_band(args, ctx, torch, device)
    if world == 1 and not args.no_configs:
        configs["config2"] = config2_capture(args, ctx, torch, device)
        configs["config4"] = config4_stream(args, ctx, torch, device)

    peaks = measured_peaks()
    sgm_s = stage_ms["sgm"] / 1e3
    achieved = work["sgm_bytes"] / sgm_s / 1e9
    # FP32 peak of the SMs at the clock seen under load: 148 SMs x 128 lanes x 2 FLOP (FMA)
    sm_mhz = clk.get("sm_mhz") or peaks.get("sm_max_mhz") or 1965.0
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    cost_tflops = work["cost_flop"] / (stage_ms["cost_volume"] / 1e3) / 1e12
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (costs, scores) + f64 (geometry, depths)",
        "data": "synthetic (seeded ray-cast scenes, Poisson-Gaussian noise)",
        "config": {"workload": WORKLOAD_TEXT[args.workload], "seed": args.seed,
                   "coarse_nodes": work["coarse_nodes"], "labels": work["labels"],
                   "fine_nodes": work["fine_nodes"], "sgm_cells_per_step": work["cells"],
                   "l2": "flushed between timed steps (256 MiB write on the library stream)",
                   "parallelism": f"replicas x{world} (one capture per GPU, no collective)"},
        "stage_ms": {k: round(v, 4) for k, v in stage_ms.items()},
        "sgm_only_gcells_s": round(work["cells"] / sgm_s / 1e9, 2),
        "roofline": {"kernel": "SGM (sgm_paths_kernel + sgm_sum_kernel, the metric's kernel)", "bound": "hbm",
                     "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": round(achieved / peaks["hbm_gbs"], 4),
                     "traffic": sgm_traffic() if args.workload == "five_view" else None,
                     "traffic_source": "profiles/sgm_five_view_dram.md (ncu dram__bytes_read + write, one call)",
                     "peak_source": peaks["source"], "algorithmic_bytes": work["sgm_bytes"]},
        "stage_graph": graph,
        "finest_coarse_grid": finest,
        "resolution_warp": resolution,
        "global_alignment": alignment,
        "quantised_sgm": dict(quantised, roofline=dict(
            quantised["roofline"], peak=peaks["hbm_gbs"],
            frac=round(quantised["roofline"]["achieved"] / peaks["hbm_gbs"], 4))),
        "batched_sgm": dict(batched, note="SGM of many instances of uneven sizes and label counts: "
                            "per-instance calls (plain) against one persistent batch replayed from a CUDA graph"),
        **({"learned_band": band} if band else {}),
        "issue_roofline": issue_roofline(stage_ms, sm_mhz, ctx.tuning().get((len(scene.cameras) - 1, scene.options.planes + 1,
                                                                          scene.options.patch_radius)))
        if args.workload == "five_view" else None,
        "compute_roofline": {"kernel": "cost_volume_kernel (build_cost_volume, the largest correlation kernel)",
                             "bound": "fp32", "achieved": round(cost_tflops, 2), "peak": round(fp32_peak, 1),
                             "unit": "TFLOP/s", "frac": round(cost_tflops / fp32_peak, 4),
                             "flop_per_tap": 16, "taps": work["cost_taps"],
                             "peak_source": f"148 SMs x 128 FP32 lanes x 2 FLOP at {sm_mhz:.0f} MHz"},
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": round(1e3 * e2e_s / e2e_steps, 3),
                "api": "chiaro_b200.depth.refine_multiview_depth (host buffers, pinned inputs)"},
        "e2e_pageable": {"value": round(whole_job_rate(world, work["cells"], e2e_steps, e2e_pageable_s), 3),
                         "unit": UNIT, "ms_per_step": round(1e3 * e2e_pageable_s / e2e_steps, 3),
                         "api": "chiaro_b200.depth.refine_multiview_depth (host buffers: the scene's own pageable "
                                "numpy planes, as a caller passing ordinary host vectors)"},
        "e2e_pipelined": pipelined,
        **({"configs": configs} if configs else {}),
        "autotune": {"cost_volume_threads_per_node": {f"targets {t}, labels {l}, radius {r}": v
                                                      for (t, l, r), v in ctx.tuning().items()},
                     "note": "CTA size of the cost volume chosen by timing 64-192 threads per node once per bucket "
                             "(every size gives the same bits)"},
        "gpu_launches": launches * args.steps,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import cpu_baseline
        if args.workload == "two_view":
            r = cpu_baseline.run_whole(scene)
            line["cpu_baseline"] = {"value": round(r["gcells_per_s"], 6), "unit": UNIT, "cores": r["threads"],
                                    "kind": "port", "sample": r["sample"], "seconds": round(r["seconds"], 2)}
        else:
            r = cpu_baseline.run_samples(scene, (6, 18), rows_per_band=args.rows_per_band)
            line["cpu_baseline"] = {"value": round(r["gcells_per_s"], 6), "unit": UNIT, "cores": r["threads"],
                                    "kind": "port", "sample": r["sample"], "samples": r["samples"],
                                    "cells": r["cells"], "seconds": round(r["seconds"], 2),
                                    "spread": {k: round(v, 6) for k, v in r["spread"].items()},
                                    "stage_s": {k: round(v, 3) for k, v in r["stage_seconds"].items()}}
        # refine_resolution_warp of every target through the oracle, one host thread as the reference runs it
        from oracle import oracle as oracle_module
        ref = scene.luminance[scene.reference_index]
        t0 = time.perf_counter()
        for t in range(len(scene.cameras)):
            if t != scene.reference_index:
                oracle_module.refine_resolution_warp(ref, scene.luminance[t], scene.warps[t], scene.width,
                                                     scene.height)
        cpu_ms = (time.perf_counter() - t0) * 1e3 / max(1, len(scene.cameras) - 1)
        line["resolution_warp"]["cpu_oracle_ms_per_target"] = round(cpu_ms, 1)
        line["resolution_warp"]["cpu_oracle_threads"] = 1
        # align_module of one target through the oracle (one host thread, as the reference runs a module)
        from chiaro_b200.abi import AlignmentReportC, WarpC
        from chiaro_b200.align import AlignOptions, align_input_c
        inputs = scene.inputs()
        target = next(t for t in range(len(scene.cameras)) if t != scene.reference_index)
        ref_c, keep_r = align_input_c(inputs[scene.reference_index])
        tgt_c, keep_t = align_input_c(inputs[target])
        columns, rows = -(-scene.width // 32) + 1, -(-scene.height // 32) + 1
        points = np.empty(2 * columns * rows, np.float32)
        out = WarpC(capacity=columns * rows, points=points.ctypes.data_as(C.POINTER(C.c_float)))
        gain, report, opt = C.c_float(), AlignmentReportC(), AlignOptions().to_c()
        t0 = time.perf_counter()
        oracle_module.lib().oracle_align_module(C.byref(ref_c), C.byref(tgt_c), 0, C.byref(opt), None, C.byref(out),
                                                C.byref(gain), C.byref(report), None)
        line["global_alignment"]["cpu_oracle_ms_per_target"] = round((time.perf_counter() - t0) * 1e3, 1)
        line["global_alignment"]["cpu_oracle_threads"] = 1
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()
    return line


def resolution_warp(args, scene, ctx):
    """refine_resolution_warp of every target of the workload against the reference module
    (chiaro_refine_resolution_warp: host planes and warps in and out, transfers included),
    wall-clock per call after warm-up, with the bit-exact result's report."""
    from chiaro_b200.resolution import refine_resolution_warp
    ref = scene.luminance[scene.reference_index]
    targets = [t for t in range(len(scene.cameras)) if t != scene.reference_index]
    result = None
    for _ in range(max(args.warmup, 2)):
        for t in targets:
            result = refine_resolution_warp(ref, scene.luminance[t], scene.warps[t], scene.width, scene.height,
                                            context=ctx)
    steps = max(1, min(args.steps, 5))
    t0 = time.perf_counter()
    for _ in range(steps):
        for t in targets:
            result = refine_resolution_warp(ref, scene.luminance[t], scene.warps[t], scene.width, scene.height,
                                            context=ctx)
    ms = (time.perf_counter() - t0) * 1e3 / (steps * len(targets))
    import torch
    planes = [torch.from_numpy(p.data).cuda() for p in scene.luminance]
    for t in targets:  # warm-up of the device-plane form
        refine_resolution_warp(planes[scene.reference_index], planes[t], scene.warps[t], scene.width, scene.height,
                               context=ctx)
    t0 = time.perf_counter()
    for _ in range(steps):
        for t in targets:
            refine_resolution_warp(planes[scene.reference_index], planes[t], scene.warps[t], scene.width,
                                   scene.height, context=ctx)
    device_ms = (time.perf_counter() - t0) * 1e3 / (steps * len(targets))
    del planes
    return {"api": "chiaro_b200.resolution.refine_resolution_warp (host planes and warps)",
            "ms_per_target_device_planes": round(device_ms, 3),
            "plane": [ref.width, ref.height], "control_grid": [result.warp.columns, result.warp.rows],
            "ms_per_target": round(ms, 3), "targets": len(targets),
            "last_report": {k: round(v, 4) for k, v in vars(result.report).items()}}


def global_alignment(args, scene, ctx):
    """align_module of every target of the workload to the reference module
    (chiaro_align_module: host planes in, host warp out, calibrated initialisation),
    wall-clock per call after warm-up, with the last call's report."""
    from chiaro_b200.align import AlignOptions, align_module
    inputs = scene.inputs()
    targets = [t for t in range(len(scene.cameras)) if t != scene.reference_index]
    result = None
    for _ in range(max(args.warmup, 2)):
        for t in targets:
            result = align_module(inputs[scene.reference_index], inputs[t], AlignOptions(), context=ctx)
    steps = max(1, min(args.steps, 3))
    t0 = time.perf_counter()
    for _ in range(steps):
        for t in targets:
            result = align_module(inputs[scene.reference_index], inputs[t], AlignOptions(), context=ctx)
    ms = (time.perf_counter() - t0) * 1e3 / (steps * len(targets))
    r = result.report
    return {"api": "chiaro_b200.align.align_module (host planes, calibrated initialisation)",
            "ms_per_target": round(ms, 3), "targets": len(targets), "status": r.status,
            "levels": [[lv.scale, lv.patches, lv.inliers, round(lv.median_residual_px, 3)] for lv in r.levels],
            "inlier_ratio": round(r.inlier_ratio, 4), "gain": round(result.gain, 4)}


def finest_coarse_grid(args, scene, stage, torch, stream, flush):
    """The workload at grid_step 4: the coarse grid (cost volume and SGM) at the direct grid's
    step, the finest the reference reaches (1041x781 nodes for 4160x3120, four times the
    default's cells). Same inputs, device buffers and timing as the main leg."""
    import dataclasses

    options = dataclasses.replace(scene.options, grid_step=4)
    work = stage_bytes(dataclasses.replace(scene, options=options))
    ctx = stage.ctx

    def step():
        if not stage(options):
            raise RuntimeError("the stage returned None at grid_step 4")

    for _ in range(max(args.warmup, 2)):
        step()
    steps = max(1, min(args.steps, 5))
    total, stages = 0.0, []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        step()
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
        stages.append(ctx.timings())
    ms = total / steps
    return {"grid_step": 4, "coarse_nodes": work["coarse_nodes"], "labels": work["labels"],
            "sgm_cells_per_step": work["cells"], "ms_per_step": round(ms, 3),
            "gcells_s": round(work["cells"] / (ms / 1e3) / 1e9, 3),
            "stage_ms": {k: round(statistics.median(s[k] for s in stages), 4) for k in stages[0]}}


def timed_stage(args, torch, stream, flush, fn, ctx, steps=None):
    """Device time (ms) per call of ``fn`` with the main leg's method (L2 flushed, CUDA
    events on the library's stream) and the median per-stage times."""
    for _ in range(max(args.warmup, 2)):
        fn()
    steps = steps or max(1, args.steps)
    total, stages = 0.0, []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        fn()
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
        stages.append(ctx.timings())
    return total / steps, {k: statistics.median(s[k] for s in stages) for k in stages[0]}


def stage_rooflines(work, ms, stage_ms, sm_mhz):
    """The SGM's HBM fraction and the cost volume's FP32 fraction for one workload."""
    peaks = measured_peaks()
    sgm_gbs = work["sgm_bytes"] / (stage_ms["sgm"] / 1e3) / 1e9
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    cost_tflops = work["cost_flop"] / (stage_ms["cost_volume"] / 1e3) / 1e12
    return {"sgm": {"bound": "hbm", "achieved": round(sgm_gbs, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": round(sgm_gbs / peaks["hbm_gbs"], 4), "algorithmic_bytes": work["sgm_bytes"],
                    "peak_source": peaks["source"]},
            "cost_volume": {"bound": "fp32", "achieved": round(cost_tflops, 3), "peak": round(fp32_peak, 1),
                            "unit": "TFLOP/s", "frac": round(cost_tflops / fp32_peak, 4),
                            "taps": work["cost_taps"], "flop_per_tap": 16}}


def two_view_config(args, ctx, torch, stream, flush, with_cpu):
    """Config 0 (two_view: 1040x780 reference + 1 source at 25 mm, 64 planes): the whole
    stage on device buffers, timed like the main leg, with its SGM and cost-volume
    rooflines, and the oracle's whole stage on the host cores (measured once, whole)."""
    from chiaro_b200 import scenes
    from chiaro_b200.depth import DeviceStage
    scene = scenes.workload("two_view", seed=args.seed)
    work = stage_bytes(scene)
    stage = DeviceStage(scene.inputs(), scene.reference_index, scene.alignments(), scene.options, context=ctx)

    def step():
        if not stage():
            raise RuntimeError("the stage returned None on two_view")

    ms, stage_ms = timed_stage(args, torch, stream, flush, step, ctx)
    sm_mhz = 1965.0
    out = {"workload": WORKLOAD_TEXT["two_view"], "value": round(work["cells"] / (ms / 1e3) / 1e9, 3),
           "unit": UNIT, "ms_per_step": round(ms, 4), "sgm_cells_per_step": work["cells"],
           "coarse_nodes": work["coarse_nodes"], "labels": work["labels"],
           "stage_ms": {k: round(v, 4) for k, v in stage_ms.items()},
           "roofline": stage_rooflines(work, ms, stage_ms, sm_mhz)}
    if with_cpu:
        from oracle import cpu_baseline
        r = cpu_baseline.run_whole(scene)
        out["cpu_baseline"] = {"value": round(r["gcells_per_s"], 6), "unit": UNIT, "cores": r["threads"],
                               "kind": "port", "sample": r["sample"], "seconds": round(r["seconds"], 3)}
    del stage
    return out


def stage_graph(args, torch, stream, flush, stage):
    """The whole stage replayed from its CUDA graph (``DeviceStage(graph=True)``): the first
    call launches, the second captures, the rest replay. The replay's outputs must equal
    the launched stage's bit for bit before it is timed, with the same flush and events as
    the main leg."""
    outputs = [stage.depth, stage.confidence, stage.provenance] + \
        [x for t in stage.targets for x in (stage.points[t], stage.point_confidence[t])]

    def snapshot():
        return [t.clone() for t in outputs]

    stage.graph = False
    stage()
    plain = snapshot()
    stage.graph = True
    try:
        states = []
        for _ in range(3):
            for t in outputs:
                t.zero_()
            stage()
            states.append(stage.graph_state)
        torch.cuda.synchronize()
        identical = all(torch.equal(a.view(torch.uint8), b.view(torch.uint8)) for a, b in zip(plain, snapshot()))
        if not identical or states != [0, 1, 2]:
            return {"error": f"replay differs from the launched stage (states {states})"}
        total = 0.0
        steps = max(1, args.steps)
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            stage()
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
        replayed = stage.graph_state == 2
    finally:
        stage.graph = False
    return {"ms_per_step": round(total / steps, 3), "launches_per_step": stage.ctx.launches(),
            "bit_identical_to_launched": True, "replayed": replayed,
            "note": "one cudaGraphLaunch per call on unchanged views, options and buffers"}


def quantised_sgm(args, scene, work, ctx, torch, device, stream, flush):
    """The quantised u16 SGM (chiaro_sgm_aggregate_u16_device) against the f32 SGM on this
    workload's own cost volume, both timed with CUDA events on the library's stream (L2
    flushed before each step), and the agreement of their winners."""
    import numpy as np

    from chiaro_b200.depth import output_shape, refine_multiview_depth
    (cols, rows, _), (cc, cr, _) = output_shape(scene.width, scene.height, scene.options)
    N, D = cc * cr, scene.options.planes + 1
    dbg = {k: np.zeros(n, t) for k, (n, t) in {"coarse_costs": (N * D, np.float32),
                                                "coarse_guidance": (N, np.float32),
                                                "regularised": (N * D, np.float32),
                                                "coarse_tested": (N, np.uint8)}.items()}
    refine_multiview_depth(scene.inputs(), scene.reference_index, scene.alignments(), scene.options, context=ctx,
                           debug=dbg)
    costs = torch.from_numpy(dbg["coarse_costs"]).to(device)
    guidance = torch.from_numpy(dbg["coarse_guidance"]).to(device)
    out32 = torch.empty(N * D, dtype=torch.float32, device=device)
    best16 = torch.empty(N, dtype=torch.int16, device=device)
    lib = ctx.lib

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        total = 0.0
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            fn()
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
        return total / args.steps

    f32_ms = timed(lambda: ctx.check(lib.chiaro_sgm_aggregate_device(
        ctx.handle, costs.data_ptr(), guidance.data_ptr(), cc, cr, D, out32.data_ptr())))
    u16_ms = timed(lambda: ctx.check(lib.chiaro_sgm_aggregate_u16_device(
        ctx.handle, costs.data_ptr(), guidance.data_ptr(), cc, cr, D, None, best16.data_ptr())))
    best = best16.cpu().numpy().view(np.uint16).astype(np.int64)
    winner32 = 1 + np.argmin(dbg["regularised"].reshape(N, D)[:, 1:], axis=1)
    tested = dbg["coarse_tested"] == 1
    diff = np.abs(best - winner32)[tested]
    u16_bytes = N * D * 4 + 8 * N * 4  # read u16 costs once, write the u16 aggregate once, guidance per direction
    return {"kernel": "sgm_quantise + sgm_u16_paths + sgm_u16_select (chiaro_sgm_aggregate_u16_device)",
            "ms": round(u16_ms, 4), "f32_sgm_ms": round(f32_ms, 4),
            "gcells_s": round(work["cells"] / (u16_ms / 1e3) / 1e9, 2),
            "winner_agreement": {"exact": round(float((diff == 0).mean()), 5),
                                 "within_one_plane": round(float((diff <= 1).mean()), 5),
                                 "tested_nodes": int(tested.sum())},
            "roofline": {"bound": "hbm", "achieved": round(u16_bytes / (u16_ms / 1e3) / 1e9, 1), "unit": "GB/s",
                         "algorithmic_bytes": u16_bytes}}


# Config 2: the reference/source groupings of one capture as SGM instances (raster W x H,
# planes); coarse grid step 8. Config 4: 32 such captures.
GROUPINGS = [(4160, 3120, 128), (4160, 3120, 192), (3120, 2340, 64), (3120, 2340, 128), (2080, 1560, 192),
             (2080, 1560, 64), (2080, 1560, 128), (1560, 1170, 192), (1040, 780, 64), (1040, 780, 128)]


def batched_sgm(args, ctx, torch, device, stream, flush):
    """Configs 2 and 4: the SGM of many instances of uneven sizes and label counts, as plain
    per-instance calls and as one batch (persistent work list, graph replay, autotuned),
    both timed with CUDA events on the library's stream. Costs are seeded synthetic
    volumes of each instance's shape (SGM time does not depend on the values)."""
    from chiaro_b200 import abi
    gen = torch.Generator(device=device)
    gen.manual_seed(args.seed)
    result = {}
    for name, captures in (("config2", 1), ("config4", 32)):
        shapes = []
        for _ in range(captures):
            for w, h, planes in GROUPINGS:
                shapes.append((-(-w // 8) + 1, -(-h // 8) + 1, planes + 1))
        tensors = []
        arr = (abi.SgmInstanceC * len(shapes))()
        for i, (c, r, d) in enumerate(shapes):
            costs = torch.rand(c * r * d, generator=gen, device=device) * 2.25
            guidance = torch.rand(c * r, generator=gen, device=device) * 7.0
            out = torch.empty(c * r * d, device=device)
            tensors += [costs, guidance, out]
            arr[i] = abi.SgmInstanceC(costs.data_ptr(), guidance.data_ptr(), out.data_ptr(), c, r, d)
        cells = sum(c * r * d for c, r, d in shapes) * 8
        nbytes = sum(c * r * d * 8 + 8 * c * r * 4 for c, r, d in shapes)
        lib = ctx.lib

        def plain():
            for i, (c, r, d) in enumerate(shapes):
                ctx.check(lib.chiaro_sgm_aggregate_device(ctx.handle, arr[i].costs, arr[i].guidance, c, r, d,
                                                          arr[i].out))

        def batched():
            ctx.check(lib.chiaro_sgm_aggregate_batch_device(ctx.handle, arr, len(shapes), 0,
                                                            abi.BATCH_GRAPH | abi.BATCH_AUTOTUNE))

        times = {}
        for label, fn in (("plain", plain), ("batched", batched)):
            for _ in range(max(args.warmup, 2)):
                fn()
            total = 0.0
            steps = max(1, min(args.steps, 5))
            for _ in range(steps):
                with torch.cuda.stream(stream):
                    flush.zero_()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                fn()
                with torch.cuda.stream(stream):
                    e1.record(stream)
                e1.synchronize()
                total += e0.elapsed_time(e1)
            times[label] = total / steps
        w, waves, rep = C.c_int(), C.c_int(), C.c_int()
        lib.chiaro_sgm_batch_report(ctx.handle, C.byref(w), C.byref(waves), C.byref(rep))
        result[name] = {"instances": len(shapes), "sgm_cells": cells,
                        "plain_ms": round(times["plain"], 3), "batched_ms": round(times["batched"], 3),
                        "plain_gcells_s": round(cells / times["plain"] / 1e6, 2),
                        "batched_gcells_s": round(cells / times["batched"] / 1e6, 2),
                        "speedup": round(times["plain"] / times["batched"], 3),
                        "warps_per_cta": w.value, "waves": waves.value, "graph_replayed": bool(rep.value),
                        "hbm_achieved_gbs": round(nbytes / times["batched"] / 1e6, 1),
                        "algorithmic_bytes": nbytes}
        del tensors
        torch.cuda.empty_cache()
    return result


WEIGHTS = ROOT / "chiaro_b200" / "weights" / "bandnet.bin"


def band_network(ctx, device):
    """The trained band network (chiaro_b200/weights/bandnet.bin, written by
    chiaro_b200.train_band) and its metadata, or (None, None) without it."""
    from chiaro_b200.bandnet import BandNet
    if not WEIGHTS.exists():
        return None, None
    net = BandNet(ctx, device=device.index or 0)
    meta = net.load(WEIGHTS)
    return net, meta


def learned_band(args, ctx, torch, device):
    """Config 3: the learned-band coarse search (chiaro_coarse_depth_device with the band)
    against the plain search on held-out scenes: the trained network (weights committed
    with their training record) and the naive band, scored by agreement with the plain
    search's winners within one plane over tested nodes, the fallback rate and the time of
    the coarse search (device time, its CUDA events). Scenes: GPU-rendered held-out
    1040x780 five-view-structure scenes and full-resolution five-view scenes, 192 planes."""
    from chiaro_b200 import bandnet, scenes
    from chiaro_b200.depth import DeviceStage
    net, meta = band_network(ctx, device)
    nets = {"learned": net} if net is not None else {}
    out = {"weights": str(WEIGHTS.relative_to(ROOT)) if net is not None else None,
           "training": (meta or {}).get("training"), "training_evaluation": (meta or {}).get("evaluation")}
    for key, name, seeds in (("held_out_1040x780", "band", range(30000, 30000 + args.band_eval)),
                             ("held_out_4160x3120", "five_view", range(31000, 31000 + args.band_eval_full))):
        stages = (DeviceStage(sc.inputs(), 0, sc.alignments(), sc.options, context=ctx)
                  for sc in (scenes.workload(name, seed=s, cache=False, render_device=device,
                                             options=dict(planes=192)) for s in seeds))
        out[key] = dict(bandnet.evaluate_search(stages, nets, 4, 24, 8, 0.5), scenes=len(seeds))
    out["note"] = ("agreement over the plain search's tested nodes; speedup = plain coarse-search time over "
                   "the banded search's (pre-pass, proposal, banded cost volume and SGM, fallback windows)")
    return out


def capture_stages(seed, ctx_for, device, planes=None, surfaces=(12, 3)):
    """DeviceStages of one GPU-rendered 16-module capture's 10 groupings (ctx_for(g) gives
    grouping g's context)."""
    from chiaro_b200 import scenes
    from chiaro_b200.depth import DeviceStage
    groupings = scenes.make_capture(seed, render_device=device, planes=planes, surfaces=surfaces)
    return [DeviceStage(g.inputs(), 0, g.alignments(), g.options, context=ctx_for(i))
            for i, g in enumerate(groupings)], groupings


def config2_capture(args, ctx, torch, device):
    """Config 2: one 16-module capture's 10 reference/source groupings (4160x3120 to
    1040x780, 64/128/192 planes; mid and tele modules behind mirrors) through the whole
    stage: one call per grouping in turn, the same replayed from their CUDA graphs, and all
    groupings at once, each on its own context and stream from its own host thread. Device
    time between events on torch's stream that every context's stream waits on."""
    import threading
    from chiaro_b200.runtime import DepthContext
    contexts = [DepthContext(device.index or 0) for _ in range(10)]
    stages, groupings = capture_stages(args.seed, lambda i: contexts[i], device)
    cells = sum(stage_bytes(g)["cells"] for g in groupings)
    current = torch.cuda.current_stream(device)

    def timed(fn, steps):
        for _ in range(max(args.warmup, 2)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(current)
        for _ in range(steps):
            fn()
        for st in stages:
            current.wait_stream(st.stream)
        e1.record(current)
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    def sequential():
        for st in stages:
            if not st():
                raise RuntimeError("the stage returned None on a capture grouping")

    def concurrent():
        errors = []

        def run(st):
            try:
                st()
            except Exception as e:  # reported below
                errors.append(e)
        threads = [threading.Thread(target=run, args=(st,)) for st in stages]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]

    steps = max(1, min(args.steps, 5))
    seq_ms = timed(sequential, steps)
    conc_ms = timed(concurrent, steps)
    for st in stages:
        st.graph = True
    graph_ms = timed(sequential, steps)
    for st in stages:
        st.graph = False
    per = []
    for st, g in zip(stages, groupings):
        st()
        per.append({"raster": [g.width, g.height], "planes": g.options.planes, "sources": len(g.cameras) - 1,
                    "mirrored": any(c.pose_kind == 1 for c in g.cameras), "stage_ms": st.ctx.timings()["total"]})
    out = {"groupings": len(stages), "sgm_cells_per_capture": cells,
           "sequential_ms": round(seq_ms, 3), "graph_replay_ms": round(graph_ms, 3),
           "concurrent_streams_ms": round(conc_ms, 3),
           "gcells_s": {"sequential": round(cells / seq_ms / 1e6, 3), "graph_replay": round(cells / graph_ms / 1e6, 3),
                        "concurrent_streams": round(cells / conc_ms / 1e6, 3)},
           "per_grouping": per,
           "note": "whole stage per grouping (cost volume, SGM seeding the direct pass, filters, decisions); "
                   "the SGM of each grouping is its own launch"}
    del stages
    for c in contexts:
        c.close()
    torch.cuda.empty_cache()
    return out


def config4_stream(args, ctx, torch, device):
    """Config 4: a stream of seeded 16-module captures (plane counts drawn per grouping from
    {64, 128, 192}, 4-20 slanted planes and 0-5 spheres per capture): the coarse search of
    every grouping in plain form and in learned-band form (the trained network if its
    weights are present, else the naive band), timed per capture (device time of the
    searches; rendering and uploads outside), with captures/s, Gcells/s and the banded
    form's agreement with the plain one."""
    import numpy as np
    from chiaro_b200.coarse import BandOptions, coarse_depth
    net, _ = band_network(ctx, device)
    band = BandOptions(net.params if net is not None else None, 4, 24, 8, 0.5)
    rng = np.random.default_rng(args.seed + 4)
    totals = dict(plain_ms=0.0, banded_ms=0.0, cells=0, tested=0, within_one=0, tiles=0, fallback=0)
    for c in range(args.captures):
        planes = [int(rng.choice([64, 128, 192])) for _ in range(10)]
        surfaces = (int(rng.integers(4, 21)), int(rng.integers(0, 6)))
        stages, groupings = capture_stages(50000 + c, lambda i: ctx, device, planes=planes, surfaces=surfaces)
        if c == 0:  # warm-up on the first capture
            for st in stages:
                coarse_depth(st)
                coarse_depth(st, band)
        for st, g in zip(stages, groupings):
            plain = coarse_depth(st)
            banded = coarse_depth(st, band)
            totals["plain_ms"] += plain.report["ms"]["total"]
            totals["banded_ms"] += banded.report["ms"]["total"]
            totals["cells"] += stage_bytes(g)["cells"]
            tested = plain.tested.cpu().numpy().astype(bool)
            diff = np.abs(banded.winner.cpu().numpy().astype(np.int64) - plain.winner.cpu().numpy())[tested]
            totals["tested"] += int(tested.sum())
            totals["within_one"] += int((diff <= 1).sum())
            totals["tiles"] += banded.report["tiles"]
            totals["fallback"] += banded.report["fallback_tiles"]
        del stages, groupings
    n = args.captures
    return {"captures": n, "groupings_per_capture": 10, "sgm_cells": totals["cells"],
            "band": "learned (committed weights)" if net is not None else "naive (no weights present)",
            "plain": {"ms_per_capture": round(totals["plain_ms"] / n, 3),
                      "captures_per_s": round(1e3 * n / totals["plain_ms"], 3),
                      "gcells_s": round(totals["cells"] / totals["plain_ms"] / 1e6, 3)},
            "banded": {"ms_per_capture": round(totals["banded_ms"] / n, 3),
                       "captures_per_s": round(1e3 * n / totals["banded_ms"], 3),
                       "gcells_s": round(totals["cells"] / totals["banded_ms"] / 1e6, 3),
                       "within_one_plane": round(totals["within_one"] / max(totals["tested"], 1), 5),
                       "fallback_rate": round(totals["fallback"] / max(totals["tiles"], 1), 5)},
            "speedup_banded_vs_plain": round(totals["plain_ms"] / totals["banded_ms"], 3),
            "note": "coarse search (cost volume, SGM, winners) of every grouping; device time from the "
                    "library's CUDA events; the whole stage of a capture is config2"}


def run_reference(args, rank, world):
    """The reference's CPU path (the oracle restatement, all host threads), measured.

    five_view: each step is the whole stage on one sample (one coarse row in each of
    the reference's worker bands and the fine rows they seed, oracle/cpu_baseline.py);
    the timed steps' offsets spread over the bands, so together they cover the image
    from top to bottom. two_view: each step is the whole stage on the whole workload.
    value = SGM cells processed / seconds taken, over the timed steps.
    """
    if rank != 0:
        return None
    from chiaro_b200 import scenes
    from oracle import cpu_baseline

    scene = scenes.workload(args.workload, seed=args.seed)
    work = stage_bytes(scene)
    threads = os.cpu_count() or 1
    if args.workload == "two_view":
        def one(_):
            r = cpu_baseline.run_whole(scene, threads)
            return r["cells"], r["seconds"], r

        offsets = [None] * args.steps
    else:
        from chiaro_b200.depth import output_shape
        _, (_, coarse_rows, _) = output_shape(scene.width, scene.height, scene.options)
        band = min(b - a for a, b in cpu_baseline.worker_bands(coarse_rows, threads))

        def one(offset):
            r = cpu_baseline.run_sample(scene, offset, threads, args.rows_per_band)
            return r["cells"], r["wall_seconds"], r

        offsets = [(i * band) // max(args.steps, 1) for i in range(args.steps)]
    for i in range(args.warmup):
        one(offsets[i % len(offsets)] if offsets else None)
    cells = seconds = 0.0
    rates, last = [], None
    for k in offsets:
        c, t, last = one(k)
        cells += c
        seconds += t
        rates.append(c / t / 1e9)
    value = cells / seconds / 1e9
    sample = last["sample"] if args.workload == "two_view" else (
        f"whole stage on {args.rows_per_band} coarse row(s) in each of the reference's {threads}-worker row bands "
        f"(offsets {offsets[0]}..{offsets[-1]} within the bands, top to bottom over the steps) with the fine rows "
        f"they seed; cost volume and direct pass threaded as the reference threads them, SGM, winner-take-all, "
        f"filters and per-target decisions on one thread; measured, not extrapolated")
    return {
        "metric": METRIC, "value": round(value, 6), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(seconds * 1e3 / args.steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (costs, scores) + f64 (geometry, depths)",
        "data": "synthetic (seeded ray-cast scenes, Poisson-Gaussian noise)",
        "config": {"workload": WORKLOAD_TEXT[args.workload], "seed": args.seed,
                   "sgm_cells_per_step": work["cells"], "sgm_cells_per_timed_step": int(cells / args.steps),
                   "parallelism": f"{threads} host threads (rank 0 only)"},
        "impl": "reference",
        "cpu_baseline": {"value": round(value, 6), "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample,
                         "spread": {"min_gcells_s": round(min(rates), 6), "max_gcells_s": round(max(rates), 6),
                                    "stdev_over_mean": round(statistics.pstdev(rates) / statistics.mean(rates), 4)
                                    if len(rates) > 1 else 0.0},
                         "last_step_stage_s": {k: round(v, 3) for k, v in last.get("stage_seconds", {}).items()}},
        "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def profile_case(args):
    """One case's kernels alone, for an ncu capture of committed code (see --profile-case)."""
    import numpy as np
    import torch
    from chiaro_b200 import build, scenes
    from chiaro_b200.runtime import DepthContext
    build.build()
    device = torch.device("cuda", 0)
    ctx = DepthContext(0)
    if args.profile_case == "stage":
        from chiaro_b200.depth import DeviceStage
        scene = scenes.workload("five_view", seed=args.seed)  # rendered on the host: no torch kernels to skip
        stage = DeviceStage(scene.inputs(), 0, scene.alignments(), scene.options, context=ctx)
        for _ in range(4):
            assert stage()
    elif args.profile_case == "coarse":
        from chiaro_b200.coarse import BandOptions, coarse_depth
        from chiaro_b200.depth import DeviceStage
        ctx.set_autotune(128)  # one shape: the launches are the same on every run
        scene = scenes.workload("five_view", seed=args.seed)
        stage = DeviceStage(scene.inputs(), 0, scene.alignments(), scene.options, context=ctx)
        for _ in range(2):
            coarse_depth(stage)
            coarse_depth(stage, BandOptions(None, 4, 24, 8, 0.5))
    elif args.profile_case == "sgm":
        c, r, d = 521, 391, 129
        g = torch.Generator(device=device)
        g.manual_seed(args.seed)
        costs = torch.rand(c * r * d, generator=g, device=device) * 2.25
        guidance = torch.rand(c * r, generator=g, device=device) * 7.0
        out = torch.empty_like(costs)
        best = torch.empty(c * r, dtype=torch.int16, device=device)
        for _ in range(2):
            ctx.check(ctx.lib.chiaro_sgm_aggregate_device(ctx.handle, costs.data_ptr(), guidance.data_ptr(), c, r, d,
                                                          out.data_ptr()))
            ctx.check(ctx.lib.chiaro_sgm_aggregate_u16_device(ctx.handle, costs.data_ptr(), guidance.data_ptr(), c,
                                                              r, d, None, best.data_ptr()))
    else:
        from chiaro_b200 import bandnet
        from chiaro_b200.coarse import PREPASS_SLOTS
        net, _ = band_network(ctx, device)
        net = net or bandnet.BandNet(ctx, seed=args.seed)
        columns, rows, labels = 521, 391, 193
        rng = np.random.default_rng(args.seed)
        costs = torch.from_numpy(rng.uniform(0, 2.25, (columns * rows, PREPASS_SLOTS)).astype(np.float32)).to(device)
        guidance = torch.from_numpy(rng.uniform(0, 7, columns * rows).astype(np.float32)).to(device)
        for _ in range(2):
            net.propose(costs, guidance, columns, rows, labels, 4, 24, stride=PREPASS_SLOTS)
        sample = bandnet.Sample(costs.reshape(-1), guidance, torch.from_numpy(
            rng.integers(1, labels, columns * rows).astype(np.int32)).to(device),
            torch.ones(columns * rows, dtype=torch.uint8, device=device), columns, rows, labels, PREPASS_SLOTS)
        net.train([sample], 2, 1e-3)
    torch.cuda.synchronize()
    ctx.close()
    print(json.dumps({"profile_case": args.profile_case, "ok": True}))


def main():
    args = parse_args()
    rank, world, local = dist_env()
    if args.profile_case:
        profile_case(args)
        return
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        line = run_ours(args, rank, world, local)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
