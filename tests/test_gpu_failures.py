"""Failures made on the host, through the C ABI (GPU).

Each case makes one call fail in a way the host controls: a union-find retry
bound that runs out, a device-memory cap below what the stage needs, a call
with no views, an output buffer that is too short, a target whose global warp
is undefined everywhere. Each failing call must return its status code (the
reference's ``None`` contract, depth.rs:318-324, for invalid input; an error
code otherwise) and leave the context usable: the next call on the same
context must equal the oracle bit for bit. No case faults, traps or stalls
the GPU: the retry bound ends every loop, and the memory cap refuses before
allocating.
"""
import ctypes as C

import numpy as np
import pytest

from chiaro_b200 import abi, scenes
from chiaro_b200.abi import DepthMapC, DepthReportC, WarpC, dptr, fptr, u8ptr
from chiaro_b200.depth import output_shape, pack_views, refine_multiview_depth

from backends import GpuBackend, OracleBackend

pytestmark = pytest.mark.gpu


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint64) if a.dtype == np.float64 else (a.view(np.uint32) if a.dtype == np.float32 else a)


def _stage_matches_oracle(ctx, scene, alignments=None):
    from oracle import oracle
    al_g = alignments() if alignments else scene.alignments()
    al_o = alignments() if alignments else scene.alignments()
    dmap = refine_multiview_depth(scene.inputs(), 0, al_g, scene.options, context=ctx)
    ref = oracle.refine_multiview_depth(scene.inputs(), 0, al_o, scene.options, threads=4)
    assert dmap is not None and ref is not None
    assert np.array_equal(_bits(dmap.depth), _bits(ref["depth"]))
    assert np.array_equal(dmap.provenance, ref["provenance"])
    for t in range(1, len(scene.cameras)):
        if ref["reports"][t].present:
            assert np.array_equal(_bits(al_g[t].warp.points.reshape(-1)), _bits(ref["points"][t]))
        else:
            assert al_g[t].report.depth is None
    return dmap


@pytest.fixture()
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from chiaro_b200.runtime import DepthContext
    c = DepthContext(0)
    yield c
    c.close()


def _components_case(seed=4, columns=120, rows=90):
    rng = np.random.default_rng(seed)
    n = columns * rows
    has = (rng.random(n) < 0.8).astype(np.uint8)
    depth = 1.0 / (1.0 / rng.choice([800.0, 3000.0], size=n) + rng.normal(0, 1e-6, n))
    guidance = rng.uniform(0, 1.0, n).astype(np.float32)
    return has, depth, guidance


def test_union_retry_bound_reports_a_timeout_and_the_context_recovers(ctx):
    has, depth, guidance = _components_case()
    gpu, cpu = GpuBackend(ctx), OracleBackend()
    ctx.set_union_retry_limit(0)  # no attempt: every join gives up
    before = has.copy()
    status = ctx.lib.chiaro_reject_small_components(ctx.handle, u8ptr(before), dptr(depth), fptr(guidance), 120, 90,
                                                    2.5e-6, 24)
    assert status == abi.ERR_TIMEOUT
    assert b"retries" in ctx.lib.chiaro_depth_last_error(ctx.handle)
    assert np.array_equal(before, has)  # a refused result is not written back
    ctx.set_union_retry_limit(-1)
    expected = cpu.reject_small_components(has, depth, guidance, 120, 90, 2.5e-6, 24)
    assert np.array_equal(gpu.reject_small_components(has, depth, guidance, 120, 90, 2.5e-6, 24), expected)


def test_union_retry_bound_inside_the_stage(ctx):
    scene = scenes.workload("tiny", seed=1)
    ctx.set_union_retry_limit(0)
    with pytest.raises(RuntimeError, match="error 3 "):
        refine_multiview_depth(scene.inputs(), 0, scene.alignments(), scene.options, context=ctx)
    ctx.set_union_retry_limit(-1)
    _stage_matches_oracle(ctx, scene)


def test_memory_cap_refuses_before_allocating_and_the_context_recovers(ctx):
    scene = scenes.workload("tiny", seed=2)
    held = ctx.memory_held()
    ctx.set_memory_limit(held + (1 << 16))  # far below the stage's buffers
    with pytest.raises(RuntimeError, match="memory limit"):
        refine_multiview_depth(scene.inputs(), 0, scene.alignments(), scene.options, context=ctx)
    assert ctx.memory_held() <= held + (1 << 16)
    ctx.set_memory_limit(0)
    _stage_matches_oracle(ctx, scene)
    # a cap above what the stage holds lets the same call run again
    ctx.set_memory_limit(ctx.memory_held())
    _stage_matches_oracle(ctx, scene)
    ctx.set_memory_limit(0)


def _raw_call(ctx, views, n, reference, options, capacity_short=False):
    first = views[0]
    (columns, rows, _), _ = output_shape(int(first.width), int(first.height), options) if n else ((1, 1, 4), None)
    m = columns * rows
    keep = []
    refined = (WarpC * max(n, 1))()
    for i in range(n):
        pts = np.zeros(2 * m, np.float32)
        conf = np.zeros(m, np.float32)
        keep += [pts, conf]
        refined[i].points = fptr(pts)
        refined[i].confidence = fptr(conf)
        refined[i].capacity = m - 1 if capacity_short else m
    depth = np.zeros(m)
    confidence = np.zeros(m, np.float32)
    provenance = np.zeros(m, np.uint8)
    dmap = DepthMapC(capacity=m, depth=dptr(depth), confidence=fptr(confidence), provenance=u8ptr(provenance))
    reports = (DepthReportC * max(n, 1))()
    opt = options.to_c()
    return ctx.lib.chiaro_refine_multiview_depth(ctx.handle, views, n, reference, C.byref(opt), refined, reports,
                                                 C.byref(dmap), None)


def test_refused_inputs_return_their_codes_and_the_context_recovers(ctx):
    scene = scenes.workload("tiny", seed=3)
    views, keep = pack_views(scene.inputs(), scene.alignments())
    # no views: a NULL array is an argument error, an empty one the reference's None
    assert ctx.lib.chiaro_refine_multiview_depth(ctx.handle, None, 0, 0, C.byref(scene.options.to_c()), None, None,
                                                 None, None) == abi.ERR_ARGUMENT
    assert _raw_call(ctx, views, 0, 0, scene.options) == abi.INVALID
    # an output warp one node short
    assert _raw_call(ctx, views, len(scene.cameras), 0, scene.options, capacity_short=True) == abi.ERR_CAPACITY
    _stage_matches_oracle(ctx, scene)


def test_target_with_an_undefined_global_warp(ctx):
    """Every node of target 1's global warp is NaN: Warp::map returns None everywhere
    (align.rs:84-111), so the target scores nothing and the others carry the stage."""
    scene = scenes.workload("tiny", seed=4, n_sources=3)

    def alignments():
        al = scene.alignments()
        al[1].warp.points[:] = np.nan
        return al

    _stage_matches_oracle(ctx, scene, alignments)
