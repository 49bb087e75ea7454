"""Resolved camera model on the host (numpy, f64).

Mirrors ``ResolvedCamera`` (crates/chiaro-fusion/src/geometry.rs:31-274) and
the small linear algebra of crates/chiaro-fusion/src/math.rs. Every routine is
vectorised over a leading axis of points but keeps the reference's operation
order, so each element rounds exactly as the Rust scalar code does (numpy never
fuses a multiply and an add). The device kernels carry their own copy of this
model; this one serves the host API, synthetic scene rendering and global warp
construction (``Warp.from_fn``).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional, Tuple

import numpy as np

from .abi import CameraC

IDENTITY = np.eye(3, dtype=np.float64)


# ---- math.rs -----------------------------------------------------------------
def determinant(m: np.ndarray) -> float:
    """math.rs:64-68."""
    return (m[0, 0] * (m[1, 1] * m[2, 2] - m[1, 2] * m[2, 1])
            - m[0, 1] * (m[1, 0] * m[2, 2] - m[1, 2] * m[2, 0])
            + m[0, 2] * (m[1, 0] * m[2, 1] - m[1, 1] * m[2, 0]))


def inverse(m: np.ndarray) -> Optional[np.ndarray]:
    """math.rs:70-95 (adjugate over determinant)."""
    m = np.asarray(m, dtype=np.float64)
    det = determinant(m)
    if abs(det) < 1e-300:
        return None
    inv_det = 1.0 / det

    def c(r0, c0, r1, c1):
        return m[r0, c0] * m[r1, c1] - m[r0, c1] * m[r1, c0]

    return np.array([
        [c(1, 1, 2, 2) * inv_det, -c(0, 1, 2, 2) * inv_det, c(0, 1, 1, 2) * inv_det],
        [-c(1, 0, 2, 2) * inv_det, c(0, 0, 2, 2) * inv_det, -c(0, 0, 1, 2) * inv_det],
        [c(1, 0, 2, 1) * inv_det, -c(0, 0, 2, 1) * inv_det, c(0, 0, 1, 1) * inv_det],
    ])


def rotation_about_axis(axis, angle_radians: float) -> np.ndarray:
    """math.rs:98-107 (Rodrigues)."""
    x, y, z = _normalize_one(np.asarray(axis, dtype=np.float64))
    s, c = np.sin(angle_radians), np.cos(angle_radians)
    t = 1.0 - c
    return np.array([
        [t * x * x + c, t * x * y - s * z, t * x * z + s * y],
        [t * x * y + s * z, t * y * y + c, t * y * z - s * x],
        [t * x * z - s * y, t * y * z + s * x, t * z * z + c],
    ])


def rotation_from_axis_angle(vector) -> np.ndarray:
    """math.rs:111-118: rotation by |vector| radians about vector; identity below 1e-18."""
    v = np.asarray(vector, dtype=np.float64)
    angle = float(np.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]))
    if angle < 1e-18:
        return IDENTITY.copy()
    return rotation_about_axis(v, angle)


def reflection(normal) -> np.ndarray:
    """math.rs:120-129: Householder reflection across the plane with unit normal ``normal``."""
    x, y, z = _normalize_one(np.asarray(normal, dtype=np.float64))
    return np.array([
        [1.0 - 2.0 * x * x, -2.0 * x * y, -2.0 * x * z],
        [-2.0 * x * y, 1.0 - 2.0 * y * y, -2.0 * y * z],
        [-2.0 * x * z, -2.0 * y * z, 1.0 - 2.0 * z * z],
    ])


def mirror_pose(real_camera_location, real_camera_orientation_cw, mirror_normal, plane_point):
    """The Mirror pose of ResolvedCamera::new (geometry.rs:86-104) from a mirror's unit
    normal and a point on its plane: (real_cw, reflect, virtual_center), the virtual
    centre being the real centre reflected across the mirror plane."""
    normal = np.asarray(mirror_normal, dtype=np.float64)
    location = np.asarray(real_camera_location, dtype=np.float64)
    plane = np.asarray(plane_point, dtype=np.float64)
    reflect = reflection(normal)
    rel = location - plane
    distance = normal[0] * rel[0] + normal[1] * rel[1] + normal[2] * rel[2]
    virtual_center = location - normal * (2.0 * distance)
    return np.asarray(real_camera_orientation_cw, dtype=np.float64), reflect, virtual_center


def _dot3(a, b):
    # ((a0*b0 + a1*b1) + a2*b2), broadcasting over a leading axis
    return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]


def _mul_vec(m: np.ndarray, v: np.ndarray) -> np.ndarray:
    """mul_vec(m, v) = [dot(m[0], v), dot(m[1], v), dot(m[2], v)] (math.rs:44-46)."""
    return np.stack([_dot3(np.broadcast_to(m[r], v.shape), v) for r in range(3)], axis=-1)


def _normalize(a: np.ndarray) -> np.ndarray:
    """math.rs:39-42: scale by 1/n unless n == 0."""
    n = np.sqrt(_dot3(a, a))
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / n
    out = a * inv[..., None]
    return np.where((n == 0.0)[..., None], a, out)


def _normalize_one(a: np.ndarray) -> np.ndarray:
    return _normalize(a[None])[0]


# ---- geometry.rs ---------------------------------------------------------------
@dataclass
class PolynomialDistortion:
    """PolynomialDistortion (calibration.rs:305-310): Brown k1, k2, p1, p2, k3."""

    center: Tuple[float, float]
    normalization: Tuple[float, float]
    coeffs: Tuple[float, ...]

    def coeff(self, i: int) -> float:
        return float(self.coeffs[i]) if i < len(self.coeffs) else 0.0


def _to_normalized(d: PolynomialDistortion, p: np.ndarray) -> np.ndarray:
    return np.stack([(p[..., 0] - d.center[0]) / d.normalization[0],
                     (p[..., 1] - d.center[1]) / d.normalization[1]], axis=-1)


def _from_normalized(d: PolynomialDistortion, n: np.ndarray) -> np.ndarray:
    return np.stack([n[..., 0] * d.normalization[0] + d.center[0],
                     n[..., 1] * d.normalization[1] + d.center[1]], axis=-1)


def _distort_normalized(d: PolynomialDistortion, xy: np.ndarray) -> np.ndarray:
    """geometry.rs:313-323."""
    k1, k2, p1, p2, k3 = (d.coeff(i) for i in range(5))
    x, y = xy[..., 0], xy[..., 1]
    r2 = x * x + y * y
    radial = 1.0 + k1 * r2 + k2 * r2 * r2 + k3 * r2 * r2 * r2
    return np.stack([x * radial + 2.0 * p1 * x * y + p2 * (r2 + 2.0 * x * x),
                     y * radial + p1 * (r2 + 2.0 * y * y) + 2.0 * p2 * x * y], axis=-1)


def distort(d: PolynomialDistortion, ideal: np.ndarray) -> np.ndarray:
    """geometry.rs:325-330."""
    return _from_normalized(d, _distort_normalized(d, _to_normalized(d, ideal)))


def undistort(d: PolynomialDistortion, pixel: np.ndarray) -> np.ndarray:
    """geometry.rs:334-353: fixed-point inverse, per element early exit."""
    observed = _to_normalized(d, pixel)
    estimate = observed.copy()
    active = np.ones(observed.shape[:-1], dtype=bool)
    for _ in range(20):
        if not active.any():
            break
        distorted = _distort_normalized(d, estimate)
        nxt = np.stack([estimate[..., 0] + (observed[..., 0] - distorted[..., 0]),
                        estimate[..., 1] + (observed[..., 1] - distorted[..., 1])], axis=-1)
        delta = np.fmax(np.abs(nxt[..., 0] - estimate[..., 0]), np.abs(nxt[..., 1] - estimate[..., 1]))
        estimate = np.where(active[..., None], nxt, estimate)
        active = active & ~(delta < 1e-12)
    return _from_normalized(d, estimate)


@dataclass
class ResolvedCamera:
    """ResolvedCamera (geometry.rs:31-62) with a canonical or mirror pose.

    ``flip`` is None, True or False (flip_img_around_x). For a canonical pose
    pass ``rotation_wc`` and ``translation_wc``; for a mirror pose pass
    ``real_cw``, ``reflect`` and ``virtual_center``.
    """

    width: int
    height: int
    k: np.ndarray
    distortion: Optional[PolynomialDistortion] = None
    flip: Optional[bool] = None
    rotation_wc: Optional[np.ndarray] = None
    translation_wc: Optional[np.ndarray] = None
    real_cw: Optional[np.ndarray] = None
    reflect: Optional[np.ndarray] = None
    virtual_center: Optional[np.ndarray] = None
    orientation_correction: np.ndarray = field(default_factory=lambda: IDENTITY.copy())
    name: str = ""

    def __post_init__(self):
        self.k = np.asarray(self.k, dtype=np.float64)
        k_inverse = inverse(self.k)
        if k_inverse is None:
            raise ValueError("singular intrinsic matrix")
        self.k_inverse = k_inverse
        self.orientation_correction = np.asarray(self.orientation_correction, dtype=np.float64)
        if self.rotation_wc is not None:
            self.pose_kind = 0
            self.rotation_wc = np.asarray(self.rotation_wc, dtype=np.float64)
            self.translation_wc = np.asarray(self.translation_wc, dtype=np.float64)
            self.rotation_cw = self.rotation_wc.T.copy()
            # CanonicalPose::center_world (calibration.rs:193-197)
            self.center_c = _mul_vec(self.rotation_cw, self.translation_wc[None])[0] * -1.0
        elif self.real_cw is not None:
            self.pose_kind = 1
            self.real_cw = np.asarray(self.real_cw, dtype=np.float64)
            self.reflect = np.asarray(self.reflect, dtype=np.float64)
            self.virtual_center = np.asarray(self.virtual_center, dtype=np.float64)
        else:
            raise ValueError("camera needs a canonical or a mirror pose")

    @property
    def focal_px(self) -> float:
        return float(self.k[0, 0])

    def center(self) -> np.ndarray:
        return self.center_c if self.pose_kind == 0 else self.virtual_center

    def _reflect_image_axis(self, n: np.ndarray) -> np.ndarray:
        if self.flip is True:
            return np.stack([n[..., 0], -n[..., 1]], axis=-1)
        if self.flip is False:
            return np.stack([-n[..., 0], n[..., 1]], axis=-1)
        return n

    def pixel_to_ray(self, pixel: np.ndarray):
        """geometry.rs:139-166 -> (origin[...,3], direction[...,3])."""
        pixel = np.asarray(pixel, dtype=np.float64)
        ideal = undistort(self.distortion, pixel) if self.distortion is not None else pixel
        ones = np.ones(ideal.shape[:-1])
        direction = _normalize(_mul_vec(self.k_inverse, np.stack([ideal[..., 0], ideal[..., 1], ones], -1)))
        if self.flip is not None:
            xy = self._reflect_image_axis(direction[..., :2])
            direction = _normalize(np.stack([xy[..., 0], xy[..., 1], direction[..., 2]], -1))
        if self.pose_kind == 0:
            origin = np.broadcast_to(self.center_c, direction.shape)
            world = _mul_vec(self.rotation_cw, direction)
        else:
            origin = np.broadcast_to(self.virtual_center, direction.shape)
            world = _mul_vec(self.reflect, _mul_vec(self.real_cw, direction))
        return origin, _normalize(_mul_vec(self.orientation_correction, _normalize(world)))

    def project(self, point: np.ndarray):
        """geometry.rs:172-231 (bounded). Returns (pixel[...,2], valid[...])."""
        point = np.asarray(point, dtype=np.float64)
        if not np.array_equal(self.orientation_correction, IDENTITY):
            c = self.center()
            point = c + _mul_vec(self.orientation_correction.T, point - c)
        if self.pose_kind == 0:
            cam = _mul_vec(self.rotation_wc, point) + self.translation_wc
        else:
            cam = _mul_vec(self.real_cw.T, _mul_vec(self.reflect, point - self.virtual_center))
        valid = ~(cam[..., 2] <= 0.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            normalized = self._reflect_image_axis(
                np.stack([cam[..., 0] / cam[..., 2], cam[..., 1] / cam[..., 2]], -1))
        k = self.k
        ideal = np.stack([k[0, 0] * normalized[..., 0] + k[0, 1] * normalized[..., 1] + k[0, 2],
                          k[1, 1] * normalized[..., 1] + k[1, 2]], -1)
        mx = float(self.width) * 0.5
        my = float(self.height) * 0.5
        outside = ((ideal[..., 0] < -mx) | (ideal[..., 1] < -my)
                   | (ideal[..., 0] > float(self.width) + mx) | (ideal[..., 1] > float(self.height) + my))
        valid = valid & ~outside
        out = distort(self.distortion, ideal) if self.distortion is not None else ideal
        return out, valid

    def map_from(self, reference: "ResolvedCamera", pixel: np.ndarray, depth: float):
        """geometry.rs:237-240: where `reference` pixels land in this camera."""
        origin, direction = reference.pixel_to_ray(pixel)
        return self.project(origin + direction * depth)

    def to_c(self) -> CameraC:
        c = CameraC()
        c.width, c.height = int(self.width), int(self.height)
        c.k[:] = self.k.ravel().tolist()
        c.k_inverse[:] = self.k_inverse.ravel().tolist()
        if self.distortion is not None:
            c.has_distortion = 1
            c.distortion_center[:] = list(self.distortion.center)
            c.distortion_normalization[:] = list(self.distortion.normalization)
            c.distortion_coeffs[:] = [self.distortion.coeff(i) for i in range(5)]
        c.flip = 0 if self.flip is None else (1 if self.flip else 2)
        c.pose_kind = self.pose_kind
        if self.pose_kind == 0:
            c.rotation_wc[:] = self.rotation_wc.ravel().tolist()
            c.rotation_cw[:] = self.rotation_cw.ravel().tolist()
            c.translation_wc[:] = self.translation_wc.tolist()
            c.center[:] = self.center_c.tolist()
        else:
            c.real_cw[:] = self.real_cw.ravel().tolist()
            c.reflect[:] = self.reflect.ravel().tolist()
            c.virtual_center[:] = self.virtual_center.tolist()
        c.orientation_correction[:] = self.orientation_correction.ravel().tolist()
        return c
