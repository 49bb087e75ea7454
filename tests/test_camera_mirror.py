"""Mirror poses, image-axis flips and orientation corrections of the camera model (CPU).

The L16's mid and tele modules sit behind fold mirrors: their ResolvedCamera has
a Mirror pose (real_cw, reflect, virtual_center; geometry.rs:86-104), a
flip_img_around_x of Some(true) or Some(false) (geometry.rs:129-136) and may carry
an orientation correction (geometry.rs:111-114). These tests build such cameras
the way the scenes do and check

* the round trip pixel -> ray -> point -> pixel through the oracle, the pattern of
  the reference's distortion test (geometry.rs:367-393) extended to mirror poses;
* that the oracle, the host camera model (numpy) and the device camera code
  (common.cuh, compiled for the host in libchiaro_hostcheck.so) give the same bits
  for pixel_to_ray, project and map_from;
* that a mirror module built to stand in for a canonical one casts the same rays
  (the flip restores the handedness the reflection takes away).
"""
import ctypes as C

import numpy as np
import pytest

from chiaro_b200 import runtime, scenes
from chiaro_b200.abi import dptr
from chiaro_b200.camera import IDENTITY, PolynomialDistortion, ResolvedCamera, reflection, rotation_from_axis_angle


def _cameras():
    """(name, camera, canonical twin or None) for every pose and flip kind."""
    rng = np.random.default_rng(17)
    width, height = 4160, 3120
    f = 3.0 / 0.00112
    k = np.array([[f, 0.0, (width - 1) / 2.0 + 3.5], [0.0, f * 1.0004, (height - 1) / 2.0 - 2.25], [0, 0, 1.0]])
    dist = PolynomialDistortion((2081.5, 1558.0), (3380.0, 3380.0), (0.1138, -0.3495, 0.0004, -0.0002, 0.0934))
    rot = scenes._random_rotation(rng, 0.5)
    centre = np.array([31.0, -17.5, 0.25])
    canonical = scenes._camera(width, height, k, rot, centre, dist)
    out = [("canonical", canonical, None)]
    for flip in (True, False):
        cam = scenes._mirror_camera(width, height, k, rot, centre, flip, rng, dist)
        out.append((f"mirror flip={flip}", cam, canonical))
        cam = scenes._mirror_camera(width, height, k, rot, centre, flip, rng, dist, orientation=(0.03, -0.05, 0.02))
        out.append((f"mirror flip={flip} + orientation", cam, None))
    cam = ResolvedCamera(width=width, height=height, k=k, distortion=dist, rotation_wc=rot,
                         translation_wc=-(rot @ centre),
                         orientation_correction=rotation_from_axis_angle(np.array([0.04, 0.01, -0.02]) * np.pi / 180))
    out.append(("canonical + orientation", cam, None))
    return out


CAMERAS = _cameras()
PIXELS = [(100.0, 100.0), (2080.0, 1560.0), (4100.0, 3000.0), (0.0, 3119.0), (1234.5, 77.25), (4159.0, 0.0)]


@pytest.fixture(scope="module")
def oracle_lib():
    from oracle import oracle
    return oracle.lib()


@pytest.mark.parametrize("name,camera,_", CAMERAS, ids=[c[0] for c in CAMERAS])
def test_pixel_ray_pixel_round_trip_through_the_oracle(oracle_lib, name, camera, _):
    c = camera.to_c()
    for depth in (400.0, 2500.0, 50000.0):
        for px in PIXELS:
            origin, direction, back = np.zeros(3), np.zeros(3), np.zeros(2)
            oracle_lib.oracle_pixel_to_ray(C.byref(c), dptr(np.array(px)), dptr(origin), dptr(direction))
            assert abs(np.linalg.norm(direction) - 1.0) < 1e-12
            point = origin + direction * depth
            assert oracle_lib.oracle_project(C.byref(c), dptr(point), dptr(back)) == 1, (name, px, depth)
            assert abs(back[0] - px[0]) < 1e-6 and abs(back[1] - px[1]) < 1e-6, (name, px, depth, back)


@pytest.mark.parametrize("name,camera,_", CAMERAS, ids=[c[0] for c in CAMERAS])
def test_oracle_and_host_model_agree_bit_for_bit(oracle_lib, name, camera, _):
    c = camera.to_c()
    pix = np.array(PIXELS)
    o_np, d_np = camera.pixel_to_ray(pix)
    for i, px in enumerate(PIXELS):
        origin, direction = np.zeros(3), np.zeros(3)
        oracle_lib.oracle_pixel_to_ray(C.byref(c), dptr(np.array(px)), dptr(origin), dptr(direction))
        assert np.array_equal(origin.view(np.uint64), np.ascontiguousarray(o_np[i]).view(np.uint64)), name
        assert np.array_equal(direction.view(np.uint64), np.ascontiguousarray(d_np[i]).view(np.uint64)), name
    points = o_np + d_np * 1800.0
    proj_np, valid_np = camera.project(points)
    for i in range(len(PIXELS)):
        out = np.zeros(2)
        ok = oracle_lib.oracle_project(C.byref(c), dptr(np.ascontiguousarray(points[i])), dptr(out))
        assert ok == int(valid_np[i]), name
        if ok:
            assert np.array_equal(out.view(np.uint64), np.ascontiguousarray(proj_np[i]).view(np.uint64)), name


def test_device_camera_code_equals_the_oracle_on_mirror_poses(oracle_lib):
    """map_from between every ordered pair of the cameras above, as the kernels compute it
    (common.cuh compiled for the host), against the oracle, bit for bit."""
    hc = runtime.load_hostcheck()
    rng = np.random.default_rng(3)
    checked = 0
    for _, target, _ in CAMERAS:
        for _, reference, _ in CAMERAS:
            t, r = target.to_c(), reference.to_c()
            for _ in range(40):
                pixel = np.array([rng.uniform(-50, 4210), rng.uniform(-50, 3170)])
                depth = float(np.exp(rng.uniform(np.log(300.0), np.log(1e8))))
                a, b = np.zeros(2), np.zeros(2)
                ok_a = oracle_lib.oracle_map_from(C.byref(t), C.byref(r), dptr(pixel), depth, dptr(a))
                ok_b = hc.chiaro_hc_map_from(C.byref(t), C.byref(r), dptr(pixel), depth, dptr(b))
                assert ok_a == ok_b
                if ok_a:
                    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
                    checked += 1
    assert checked > 1200


@pytest.mark.parametrize("name,camera,twin", [c for c in CAMERAS if c[2] is not None], ids=lambda v: str(v)[:24])
def test_mirror_module_casts_the_rays_of_its_canonical_twin(name, camera, twin):
    assert camera.pose_kind == 1 and camera.flip in (True, False)
    pix = np.array(PIXELS)
    o1, d1 = camera.pixel_to_ray(pix)
    o0, d0 = twin.pixel_to_ray(pix)
    assert np.abs(o1 - o0).max() < 1e-11
    assert np.abs(d1 - d0).max() < 1e-13
    # the physical module sits on the far side of the mirror, looking into it
    assert np.linalg.det(camera.real_cw) > 0 and np.linalg.det(camera.reflect) < 0
    p1, v1 = camera.project(o1 + d1 * 3000.0)
    assert v1.all() and np.abs(p1 - pix).max() < 1e-6


def test_reflection_and_axis_angle_follow_the_reference_formulas():
    n = np.array([0.3, -0.5, 0.81])
    r = reflection(n)
    u = n / np.linalg.norm(n)
    assert np.allclose(r, np.eye(3) - 2 * np.outer(u, u), atol=1e-15)
    assert np.array_equal(rotation_from_axis_angle(np.array([0.0, 0.0, 1e-19])), IDENTITY)
    rot = rotation_from_axis_angle(np.array([0.0, 0.0, np.pi / 2]))
    assert np.allclose(rot @ np.array([1.0, 0, 0]), [0, 1.0, 0], atol=1e-15)


def test_mirrored_scene_keeps_the_canonical_scene_and_its_warps():
    """A scene with mirrored modules sees the same surfaces from the same virtual
    positions: its calibrated global warps match the canonical scene's to well under a
    pixel (and exactly where no orientation offset is applied)."""
    base = scenes.workload("tiny", seed=1, cache=False)
    mirrored = scenes.workload("tiny", seed=1, cache=False, mirrors={1: True, 2: False})
    assert [c.pose_kind for c in mirrored.cameras] == [0, 1, 1]
    for t in (1, 2):
        a, b = base.warps[t].points, mirrored.warps[t].points
        finite = np.isfinite(a) & np.isfinite(b)
        assert finite.mean() > 0.9
        assert np.abs(a[finite] - b[finite]).max() < 1e-3
