"""refine_resolution_warp on the GPU (chiaro_refine_resolution_warp) against the
oracle's restatement (resolution.rs:232-439): the refined points and confidences
bit for bit and the report exactly, on the reference's own test signal, a
magnified target (Gaussian footprint, radius 5), partly undefined base warps and
a rendered scene's calibrated warps."""
import ctypes as C

import numpy as np
import pytest

from chiaro_b200 import abi, scenes
from chiaro_b200.image import Plane
from chiaro_b200.resolution import refine_resolution_warp, warp_c
from resolution_cases import identity_warp, kat_planes, kat_signal, oracle_refine, warp_map

pytestmark = pytest.mark.gpu


def _same(gpu, cpu):
    assert np.array_equal(gpu.warp.points.view(np.uint32), cpu.warp.points.view(np.uint32))
    assert np.array_equal(gpu.warp.confidence.view(np.uint32), cpu.warp.confidence.view(np.uint32))
    for field in ("verified_fraction", "supported_fraction", "median_correction_px", "mean_confidence"):
        assert np.float32(getattr(gpu.report, field)).view(np.uint32) == \
            np.float32(getattr(cpu.report, field)).view(np.uint32), field


def test_plane_shift_matches_the_oracle(gpu_ctx, oracle_lib):
    reference, target = kat_planes((0.6, -0.35))
    base = identity_warp(512, 384)
    gpu = refine_resolution_warp(reference, target, base, 512, 384, context=gpu_ctx)
    _same(gpu, oracle_refine(oracle_lib, reference, target, base, 512, 384))
    q = warp_map(gpu.warp, 256.0, 192.0)
    assert abs(q[0] - 257.2) < 0.35 and abs(q[1] - 191.3) < 0.35
    assert gpu.report.verified_fraction > 0.5


@pytest.mark.parametrize("scale,shift", [(1.5, (0.4, 0.7)), (1.25, (-1.2, 0.3)), (2.6, (0.0, 0.0))])
def test_magnified_target_matches_the_oracle(gpu_ctx, oracle_lib, scale, shift):
    """base maps the reference raster to a target raster `scale` times larger: the target is
    resampled through the Gaussian footprint (scale > 1.15) and searched over radius 5
    (scale > 1.35)."""
    w, h = 200, 150
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    reference = Plane(w, h, kat_signal(x, y))
    tw, th = int(w * scale), int(h * scale)
    ty, tx = np.mgrid[0:th, 0:tw].astype(np.float32)
    target = Plane(tw, th, kat_signal(tx / np.float32(scale) - np.float32(shift[0]),
                                      ty / np.float32(scale) - np.float32(shift[1])))
    base = identity_warp(2 * w, 2 * h, scale=scale, offset=(0.25, -0.5))
    gpu = refine_resolution_warp(reference, target, base, 2 * w, 2 * h, context=gpu_ctx)
    _same(gpu, oracle_refine(oracle_lib, reference, target, base, 2 * w, 2 * h))
    if scale < 2.0:
        assert gpu.report.verified_fraction > 0.2


def test_partly_undefined_base_warp_matches_the_oracle(gpu_ctx, oracle_lib):
    reference, target = kat_planes((-0.8, 0.45), size=(300, 220))
    width, height = 600, 440
    base = identity_warp(width, height, undefined=lambda px, py: (px > 350) & (py < 200) | (px + py < 100))
    gpu = refine_resolution_warp(reference, target, base, width, height, context=gpu_ctx)
    cpu = oracle_refine(oracle_lib, reference, target, base, width, height)
    _same(gpu, cpu)
    assert np.isnan(gpu.warp.points).any() and gpu.report.verified_fraction > 0.2


@pytest.mark.parametrize("seed", [1, 4])
def test_scene_warps_match_the_oracle(gpu_ctx, oracle_lib, seed):
    sc = scenes.workload("small", seed=seed)
    ref = sc.luminance[sc.reference_index]
    for t in range(len(sc.cameras)):
        if t == sc.reference_index:
            continue
        gpu = refine_resolution_warp(ref, sc.luminance[t], sc.warps[t], sc.width, sc.height, context=gpu_ctx)
        _same(gpu, oracle_refine(oracle_lib, ref, sc.luminance[t], sc.warps[t], sc.width, sc.height))


def test_short_output_is_refused_with_the_grid_shape(gpu_ctx):
    reference, target = kat_planes()
    base = identity_warp(512, 384)
    points = np.empty(8, np.float32)
    out = abi.WarpC(capacity=4, points=points.ctypes.data_as(C.POINTER(C.c_float)))
    report = abi.ResolutionReportC()
    ref, tgt = reference.data, target.data
    base_c = warp_c(base)
    st = gpu_ctx.lib.chiaro_refine_resolution_warp(
        gpu_ctx.handle, ref.ctypes.data_as(C.POINTER(C.c_float)), 256, 192, tgt.ctypes.data_as(C.POINTER(C.c_float)),
        256, 192, C.byref(base_c), 512, 384, C.byref(out), C.byref(report))
    assert st == abi.ERR_CAPACITY and (out.step, out.columns, out.rows) == (32, 17, 13)


def test_device_planes_give_the_same_result(gpu_ctx):
    import torch
    sc = scenes.workload("small", seed=1)
    ref, tgt = sc.luminance[sc.reference_index], sc.luminance[1]
    host = refine_resolution_warp(ref, tgt, sc.warps[1], sc.width, sc.height, context=gpu_ctx)
    device = refine_resolution_warp(torch.from_numpy(ref.data).cuda(), torch.from_numpy(tgt.data).cuda(),
                                    sc.warps[1], sc.width, sc.height, context=gpu_ctx)
    _same(device, host)
