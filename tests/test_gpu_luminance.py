"""Mosaic::luminance_half on the GPU (image.rs:401-428) against the oracle.

Everything before the log (the 2x2 Q6 sum, black/white scaling and the
flat-field mesh gain, calibration.rs:362-379) is f32 arithmetic in the
reference's order and must match the oracle bit for bit: the GPU plane equals
the correctly rounded log of the oracle's argument exactly. The log itself is
the correctly rounded one, while the reference calls the host logf (within 0.82
ulp), so against the oracle's plane the tolerance is 1 ulp, on a small fraction
of pixels.
"""
import ctypes as C

import numpy as np
import pytest

from chiaro_b200 import abi
from chiaro_b200.image import Mosaic, VignettingMesh

pytestmark = pytest.mark.gpu


def _oracle(m: Mosaic):
    from oracle import oracle
    w, h = m.width // 2, m.height // 2
    out = np.zeros(max(w * h, 1), np.float32)
    arg = np.zeros(max(w * h, 1), np.float32)
    gains, cols, rows = None, 0, 0
    if m.vignetting is not None:
        gains = m.vignetting.gains.ctypes.data_as(C.POINTER(C.c_float))
        cols, rows = m.vignetting.columns, m.vignetting.rows
    oracle.lib().oracle_luminance_half_mesh(m.samples.ctypes.data_as(C.POINTER(C.c_uint16)), m.width, m.height,
                                            m.black_q6, m.white_q6, gains, cols, rows,
                                            out.ctypes.data_as(C.POINTER(C.c_float)),
                                            arg.ctypes.data_as(C.POINTER(C.c_float)))
    return out[:w * h], arg[:w * h]


def _mosaic(width, height, seed, mesh=None, black=64 * 64.0, white=4095 * 64.0):
    rng = np.random.default_rng(seed)
    samples = rng.integers(0, 65535, (height, width), dtype=np.uint16)
    samples[rng.random((height, width)) < 0.02] = 0  # below black: linear clamps to 0
    vig = None
    if mesh is not None:
        cols, rows = mesh
        vig = VignettingMesh(cols, rows, rng.uniform(0.8, 1.7, cols * rows))
    return Mosaic(width, height, samples, black, white, vig)


def _check(m: Mosaic, gpu_plane: np.ndarray):
    ref, arg = _oracle(m)
    gpu = np.ascontiguousarray(gpu_plane, np.float32).reshape(-1)
    assert gpu.shape == ref.shape
    if ref.size == 0:
        return 0.0
    exact = np.log(arg.astype(np.float64)).astype(np.float32)
    assert np.array_equal(gpu.view(np.uint32), exact.view(np.uint32)), "pre-log arithmetic differs"
    ulps = np.abs(gpu.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
    assert ulps.max() <= 1
    return float((ulps > 0).mean())


@pytest.mark.parametrize("width,height,mesh", [(2, 2, None), (1, 1, None), (7, 5, None), (64, 48, (2, 2)),
                                               (333, 201, (17, 13)), (1040, 780, (33, 25)),
                                               (4160, 3120, None), (4160, 3120, (65, 49))])
def test_luminance_half_matches_oracle(gpu_ctx, width, height, mesh):
    m = _mosaic(width, height, seed=width * 7 + height, mesh=mesh)
    fraction = _check(m, m.luminance_half(gpu_ctx).data)
    assert fraction < 0.005  # the host logf's misrounded share on this domain is about 0.1%


def test_luminance_half_device_entry(gpu_ctx):
    import torch
    m = _mosaic(1040, 780, seed=5, mesh=(9, 7))
    dev = torch.device("cuda", 0)
    samples = torch.from_numpy(m.samples.reshape(-1).view(np.int16)).to(dev)
    gains = torch.from_numpy(m.vignetting.gains).to(dev)
    out = torch.empty(520 * 390, dtype=torch.float32, device=dev)
    mesh = abi.VignettingC(columns=9, rows=7, gains=C.cast(C.c_void_p(gains.data_ptr()), C.POINTER(C.c_float)))
    gpu_ctx.check(gpu_ctx.lib.chiaro_luminance_half_device(gpu_ctx.handle, samples.data_ptr(), 1040, 780,
                                                           m.black_q6, m.white_q6, C.byref(mesh), out.data_ptr()))
    _check(m, out.cpu().numpy())


def test_luminance_half_rejects_bad_arguments(gpu_ctx):
    lib = gpu_ctx.lib
    out = np.zeros(4, np.float32)
    s = np.zeros(16, np.uint16)
    fp = out.ctypes.data_as(C.POINTER(C.c_float))
    sp = s.ctypes.data_as(C.POINTER(C.c_uint16))
    assert lib.chiaro_luminance_half(gpu_ctx.handle, None, 4, 4, 0.0, 1.0, None, fp) == abi.ERR_ARGUMENT
    mesh = abi.VignettingC(columns=3, rows=3, gains=None)
    assert lib.chiaro_luminance_half(gpu_ctx.handle, sp, 4, 4, 0.0, 1.0, C.byref(mesh), fp) == abi.ERR_ARGUMENT
    odd = s.ctypes.data + 1  # not u16-aligned: refused before any device work
    assert lib.chiaro_luminance_half_device(gpu_ctx.handle, odd, 4, 2, 0.0, 1.0, None,
                                            out.ctypes.data) == abi.ERR_ARGUMENT
