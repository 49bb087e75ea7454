"""The torch ray caster of the benchmark workloads against the numpy one (CPU).

Benchmark captures are rendered with torch (on the GPU there; on the CPU here): its
rays, hit distances and noise-free intensities must be the numpy renderer's, for
canonical, mirrored and orientation-corrected modules with distortion. The capture
generator must give the groupings their raster sizes, plane counts and module kinds.
"""
import numpy as np
import pytest

from chiaro_b200 import scenes


@pytest.mark.parametrize("mirrors,orientation", [(None, None), ({1: True, 2: False}, {2: (0.02, 0.01, -0.01)})])
def test_torch_rays_and_hits_equal_numpy(mirrors, orientation):
    import torch
    sc = scenes.workload("small", seed=4, cache=False, mirrors=mirrors, orientation=orientation)
    tiles = [scenes._noise_tile(np.random.default_rng(4 * 7919 + i)) for i in range(4)]
    gpu_tiles = [torch.as_tensor(t) for t in tiles]
    yy, xx = np.meshgrid(np.arange(0, sc.height, 3.0), np.arange(0, sc.width, 3.0), indexing="ij")
    pix = np.stack([xx.ravel(), yy.ravel()], -1)
    for cam in sc.cameras:
        origin, direction = cam.pixel_to_ray(pix)
        value, distance = scenes._cast(sc.surfaces, tiles, np.asarray(origin[0]), direction)
        t_origin, t_direction = scenes._torch_rays(cam, torch.as_tensor(pix))
        t_value, t_distance = scenes._torch_cast(sc.surfaces, gpu_tiles, t_origin, t_direction)
        assert np.abs(direction - t_direction.numpy()).max() < 1e-12
        assert np.abs(value - t_value.numpy()).max() < 1e-9
        hit = np.isfinite(distance)
        assert np.array_equal(hit, np.isfinite(t_distance.numpy()))
        assert np.abs(distance[hit] - t_distance.numpy()[hit]).max() < 1e-6


def test_capture_groupings():
    groupings = [(320, 240, 24, "wide", 2), (240, 180, 20, "mid", 2), (160, 120, 20, "tele", 3)]
    cap = scenes.make_capture(3, render_device="cpu", groupings=groupings)
    assert [(s.width, s.height, s.options.planes) for s in cap] == [g[:3] for g in groupings]
    for s, g in zip(cap, groupings):
        assert len(s.cameras) == g[4] + 1
        kinds = {c.pose_kind for c in s.cameras}
        assert kinds == ({0} if g[3] == "wide" else {1})
        assert all(c.focal_px == pytest.approx(scenes.FOCAL_MM / scenes.PIXEL_PITCH_MM) for c in s.cameras[:1])
        assert s.luminance[0].data.shape == (g[1] // 2, g[0] // 2)
        assert np.isfinite(s.luminance[0].data).all() and s.luminance[0].data.std() > 0.1
    assert {c.flip for c in cap[1].cameras} == {True, False}
