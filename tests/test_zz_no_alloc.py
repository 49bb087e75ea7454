"""The allocation-free components filter against the allocating one (GPU).

chiaro_reject_small_components_noalloc serves callers that cannot allocate
device memory: it takes the caller's device buffers and keeps its union-find
scratch in a static device array. Its result must equal the regular entry
point's bit for bit, including on a second call in a row, which finds the
scratch holding the first call's contents. The file is named to run last.
"""
import ctypes as C

import numpy as np
import pytest

from chiaro_b200 import abi

from backends import GpuBackend

pytestmark = pytest.mark.gpu


def _field(seed, columns, rows):
    rng = np.random.default_rng(seed)
    n = columns * rows
    has = (rng.random(n) < 0.75).astype(np.uint8)
    depth = 1.0 / (1.0 / rng.choice([700.0, 1500.0, 5000.0], size=n) + rng.normal(0, 1.5e-6, n))
    guidance = rng.uniform(0, 1.0, n).astype(np.float32)
    return has, depth, guidance


def test_noalloc_components_match_the_allocating_entry_point(gpu_ctx):
    import torch

    device = torch.device("cuda", gpu_ctx.device)
    lib = gpu_ctx.lib
    reference = GpuBackend(gpu_ctx)
    stream = torch.cuda.current_stream(device)
    tol = 2.5e-6
    # small, large, then small again: the third call finds the large call's parent and
    # size entries beyond its own nodes, and must not read them
    for call, (seed, columns, rows, minimum) in enumerate([(1, 257, 193, 24), (2, 1041, 781, 24),
                                                           (3, 131, 99, 24)]):
        has, depth, guidance = _field(seed, columns, rows)
        expected = reference.reject_small_components(has, depth, guidance, columns, rows, tol, minimum)
        d_has = torch.from_numpy(has).to(device)
        d_depth = torch.from_numpy(depth).to(device)
        d_guid = torch.from_numpy(guidance).to(device)
        d_out = torch.full_like(d_has, 7)
        status = lib.chiaro_reject_small_components_noalloc(
            C.c_void_p(stream.cuda_stream), C.c_void_p(d_has.data_ptr()), C.c_void_p(d_depth.data_ptr()),
            C.c_void_p(d_guid.data_ptr()), columns, rows, tol, minimum, C.c_void_p(d_out.data_ptr()))
        assert status == abi.OK, (call, status)
        torch.cuda.synchronize(device)
        got = d_out.cpu().numpy()
        assert np.array_equal(got, expected), f"call {call}: {(got != expected).sum()} nodes differ"
        assert 0 < expected.sum() < has.sum()  # the filter removed something and kept something


def test_noalloc_components_reject_grids_above_the_stated_maximum(gpu_ctx):
    lib = gpu_ctx.lib
    status = lib.chiaro_reject_small_components_noalloc(None, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1),
                                                        2048, 1024, 1e-6, 24, C.c_void_p(1))
    assert status == abi.ERR_CAPACITY


def test_noalloc_components_minimum_edges(gpu_ctx):
    """minimum_nodes <= 1 removes nothing (depth.rs:941-943): the output is a copy of the
    input. A minimum equal to a component's size keeps that component (the reference
    removes components with fewer nodes than the minimum)."""
    import torch

    device = torch.device("cuda", gpu_ctx.device)
    lib = gpu_ctx.lib
    reference = GpuBackend(gpu_ctx)
    stream = torch.cuda.current_stream(device)
    columns, rows, tol = 64, 48, 2.5e-6
    has, depth, guidance = _field(5, columns, rows)
    d_has = torch.from_numpy(has).to(device)
    d_depth = torch.from_numpy(depth).to(device)
    d_guid = torch.from_numpy(guidance).to(device)
    for minimum in (0, 1, 2, 3, 24):
        d_out = torch.full_like(d_has, 7)
        status = lib.chiaro_reject_small_components_noalloc(
            C.c_void_p(stream.cuda_stream), C.c_void_p(d_has.data_ptr()), C.c_void_p(d_depth.data_ptr()),
            C.c_void_p(d_guid.data_ptr()), columns, rows, tol, minimum, C.c_void_p(d_out.data_ptr()))
        assert status == abi.OK, (minimum, status)
        torch.cuda.synchronize(device)
        got = d_out.cpu().numpy()
        if minimum <= 1:
            assert np.array_equal(got, has), minimum
        else:
            expected = reference.reject_small_components(has, depth, guidance, columns, rows, tol, minimum)
            assert np.array_equal(got, expected), minimum


def test_noalloc_components_refuse_sides_whose_product_wraps(gpu_ctx):
    """2^63 + 1 columns by 2 rows wraps to 2 nodes in 64 bits: refused by each side's
    bound before the product is formed."""
    lib = gpu_ctx.lib
    status = lib.chiaro_reject_small_components_noalloc(None, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1),
                                                        (1 << 63) + 1, 2, 1e-6, 24, C.c_void_p(1))
    assert status == abi.ERR_CAPACITY
