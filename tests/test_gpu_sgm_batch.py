"""The batched SGM (chiaro_sgm_aggregate_batch_device): instances of uneven sizes
and label counts in one persistent launch, each bit for bit equal to the
single-instance SGM (itself bit-exact against the oracle), with waves under a
scratch budget, a replayed CUDA graph and the autotuner."""
import ctypes as C

import numpy as np
import pytest
import torch

from chiaro_b200 import abi

pytestmark = pytest.mark.gpu

SHAPES = [(31, 23, 129), (7, 40, 65), (50, 3, 193), (1, 1, 1), (12, 12, 256), (19, 11, 33), (5, 60, 97)]


def _instances(shapes, seed):
    rng = np.random.default_rng(seed)
    dev = torch.device("cuda", 0)
    items = []
    for columns, rows, labels in shapes:
        n = columns * rows
        costs = rng.uniform(0, 2.25, n * labels).astype(np.float32)
        costs[rng.random(costs.size) < 0.05] = np.float32(2.25)
        guidance = rng.uniform(0, 7, n).astype(np.float32)
        items.append(dict(costs=torch.from_numpy(costs).to(dev), guidance=torch.from_numpy(guidance).to(dev),
                          out=torch.full((n * labels,), np.nan, dtype=torch.float32, device=dev),
                          shape=(columns, rows, labels)))
    arr = (abi.SgmInstanceC * len(items))()
    for i, it in enumerate(items):
        c, r, l = it["shape"]
        arr[i] = abi.SgmInstanceC(it["costs"].data_ptr(), it["guidance"].data_ptr(), it["out"].data_ptr(), c, r, l)
    return items, arr


def _single(ctx, it):
    c, r, l = it["shape"]
    out = torch.empty_like(it["out"])
    ctx.check(ctx.lib.chiaro_sgm_aggregate_device(ctx.handle, it["costs"].data_ptr(), it["guidance"].data_ptr(),
                                                  c, r, l, out.data_ptr()))
    return out.cpu().numpy()


def _check(ctx, items):
    for it in items:
        assert np.array_equal(it["out"].cpu().numpy().view(np.uint32), _single(ctx, it).view(np.uint32)), it["shape"]


def _report(ctx):
    w, waves, rep = C.c_int(), C.c_int(), C.c_int()
    ctx.check(ctx.lib.chiaro_sgm_batch_report(ctx.handle, C.byref(w), C.byref(waves), C.byref(rep)))
    return w.value, waves.value, rep.value


def test_batch_matches_single_instances(gpu_ctx):
    items, arr = _instances(SHAPES, 1)
    gpu_ctx.check(gpu_ctx.lib.chiaro_sgm_aggregate_batch_device(gpu_ctx.handle, arr, len(items), 0, 0))
    _check(gpu_ctx, items)
    assert _report(gpu_ctx)[1] == 1


def test_batch_in_waves_under_a_small_budget(gpu_ctx):
    items, arr = _instances(SHAPES, 2)
    largest = max(8 * ((c * r * l + 63) // 64 * 64) * 4 for c, r, l in SHAPES)
    gpu_ctx.check(gpu_ctx.lib.chiaro_sgm_aggregate_batch_device(gpu_ctx.handle, arr, len(items), largest, 0))
    _check(gpu_ctx, items)
    assert _report(gpu_ctx)[1] > 1
    assert gpu_ctx.lib.chiaro_sgm_aggregate_batch_device(gpu_ctx.handle, arr, len(items), largest // 2,
                                                         0) == abi.ERR_CAPACITY


def test_graph_replay_reads_current_inputs(gpu_ctx):
    items, arr = _instances(SHAPES[:4], 3)
    lib = gpu_ctx.lib
    gpu_ctx.check(lib.chiaro_sgm_aggregate_batch_device(gpu_ctx.handle, arr, len(items), 0, abi.BATCH_GRAPH))
    assert _report(gpu_ctx)[2] == 0
    _check(gpu_ctx, items)
    for it in items:  # new data in the same buffers: the replayed graph must see it
        it["costs"].mul_(0.5).add_(0.3)
        it["out"].fill_(float("nan"))
    gpu_ctx.check(lib.chiaro_sgm_aggregate_batch_device(gpu_ctx.handle, arr, len(items), 0, abi.BATCH_GRAPH))
    assert _report(gpu_ctx)[2] == 1
    _check(gpu_ctx, items)
    # a different batch is captured afresh
    items2, arr2 = _instances(SHAPES[4:], 4)
    gpu_ctx.check(lib.chiaro_sgm_aggregate_batch_device(gpu_ctx.handle, arr2, len(items2), 0, abi.BATCH_GRAPH))
    assert _report(gpu_ctx)[2] == 0
    _check(gpu_ctx, items2)


def test_autotuned_batch_matches(gpu_ctx):
    items, arr = _instances(SHAPES, 5)
    gpu_ctx.check(gpu_ctx.lib.chiaro_sgm_aggregate_batch_device(gpu_ctx.handle, arr, len(items), 0,
                                                                abi.BATCH_AUTOTUNE))
    _check(gpu_ctx, items)
    assert _report(gpu_ctx)[0] in (1, 2, 4, 8)


def test_batch_rejects_bad_instances(gpu_ctx):
    items, arr = _instances(SHAPES[:2], 6)
    bad = (abi.SgmInstanceC * 1)(abi.SgmInstanceC(arr[0].costs, arr[0].guidance, arr[0].out, 4, 4, 300))
    assert gpu_ctx.lib.chiaro_sgm_aggregate_batch_device(gpu_ctx.handle, bad, 1, 0, 0) == abi.ERR_ARGUMENT
    assert gpu_ctx.lib.chiaro_sgm_aggregate_batch_device(gpu_ctx.handle, arr, 2, 0, 8) == abi.ERR_ARGUMENT
