"""Seeded synthetic multi-view scenes for the depth stage.

No public dataset is involved: every workload is rendered here from a seed.
A scene is a set of analytic surfaces (a background wall, finite slanted
rectangles and occluding spheres) carrying a band-limited noise texture over
the full 12-bit range. Each module is rendered independently by ray casting
its own pixels (with its own intrinsics, optional Brown distortion, pose and
small rotation), then given Poisson-Gaussian noise (gain 0.5, read sigma 4 DN),
quantised to u16, and converted to the half-resolution log-luminance plane of
``Mosaic::luminance_half`` (crates/chiaro-fusion/src/image.rs:401-428) with
black 0, white 4095 and flat field 1. Global warps are the calibrated
infinity mapping on a 32 px grid, as align.rs:317-324 initialises them.

Named workloads:
  * ``two_view``   – 1040x780 reference + 1 source at a 25 mm baseline, 6
    slanted planes at 0.5-20 m, 64 planes over 0.4-25 m (minimum_support and
    best_view_count set to 1: the reference finds no depth from one source
    with its default of 2).
  * ``five_view``  – 4160x3120 reference + 4 sources at 20-60 mm baselines,
    12 planes + 3 spheres, 128 planes over 0.4-50 m, default options.
  * ``band``       – five_view's structure at 1040x780 (reference + 4 sources, 12 planes +
    3 spheres, 2-6 cm baselines) with 192 planes over 0.4-50 m: the learned band's
    training and evaluation scenes.
  * ``small``      – reduced scenes for parity tests.
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from .align import AlignInput, ModuleAlignment, AlignmentReport, Warp
from .camera import (PolynomialDistortion, ResolvedCamera, mirror_pose, reflection, rotation_about_axis,
                     rotation_from_axis_angle)
from .depth import DepthOptions
from .image import Plane

PIXEL_PITCH_MM = 0.00112   # 1.12 um sensor pitch
FOCAL_MM = 3.0             # f = 3.0 mm lens
FULL_WIDTH = 4160


@dataclass
class Surface:
    kind: str                 # "plane" or "sphere"
    origin: np.ndarray        # plane point / sphere centre (mm)
    normal: np.ndarray        # plane normal (unit)
    axis_u: np.ndarray        # in-plane texture axes (unit)
    axis_v: np.ndarray
    half_u: float = np.inf    # finite rectangle half extents (mm)
    half_v: float = np.inf
    radius: float = 0.0
    texel_mm: float = 1.0
    tex_offset: Tuple[float, float] = (0.0, 0.0)
    tex_index: int = 0


@dataclass
class Scene:
    name: str
    width: int
    height: int
    cameras: List[ResolvedCamera]
    luminance: List[Plane]
    raw: List[np.ndarray]
    warps: List[Warp]
    options: DepthOptions
    reference_index: int = 0
    surfaces: List[Surface] = field(default_factory=list)
    depth_truth: Optional[np.ndarray] = None

    def inputs(self) -> List[AlignInput]:
        return [AlignInput(name=f"M{i}", luminance=self.luminance[i], width=self.width, height=self.height,
                           camera=self.cameras[i], nominal_focal_px=self.cameras[i].focal_px)
                for i in range(len(self.cameras))]

    def alignments(self) -> List[ModuleAlignment]:
        return [ModuleAlignment(name=f"M{i}", warp=Warp(w.step, w.columns, w.rows, w.points.copy(),
                                                         w.confidence.copy()),
                                report=AlignmentReport(camera=f"M{i}", accepted=True))
                for i, w in enumerate(self.warps)]


# ---- texture -------------------------------------------------------------------
def _noise_tile(rng: np.random.Generator, size: int = 512) -> np.ndarray:
    """Band-limited noise tile in [0, 1]: white noise band-passed in the
    Fourier domain (periods of 3-24 texels, 1/f amplitude)."""
    white = rng.standard_normal((size, size))
    f = np.fft.fftfreq(size)
    fr = np.sqrt(f[:, None] ** 2 + f[None, :] ** 2)
    band = ((fr >= 1.0 / 24.0) & (fr <= 1.0 / 3.0)).astype(np.float64)
    with np.errstate(divide="ignore"):
        amp = np.where(fr > 0, 1.0 / np.maximum(fr, 1e-9), 0.0) * band
    tile = np.real(np.fft.ifft2(np.fft.fft2(white) * amp))
    tile -= tile.min()
    tile /= max(tile.max(), 1e-12)
    return tile


def _sample_tile(tile: np.ndarray, u: np.ndarray, v: np.ndarray) -> np.ndarray:
    n = tile.shape[0]
    u0 = np.floor(u)
    v0 = np.floor(v)
    fu = u - u0
    fv = v - v0
    iu = u0.astype(np.int64) % n
    iv = v0.astype(np.int64) % n
    iu1 = (iu + 1) % n
    iv1 = (iv + 1) % n
    top = tile[iv, iu] * (1 - fu) + tile[iv, iu1] * fu
    bot = tile[iv1, iu] * (1 - fu) + tile[iv1, iu1] * fu
    return top * (1 - fv) + bot * fv


# ---- geometry helpers --------------------------------------------------------
def _unit(v):
    v = np.asarray(v, dtype=np.float64)
    return v / np.linalg.norm(v)


def _tangent_axes(normal: np.ndarray):
    a = np.array([1.0, 0.0, 0.0]) if abs(normal[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    u = _unit(np.cross(normal, a))
    v = np.cross(normal, u)
    return u, v


def _intrinsics(width: int, height: int, rng: Optional[np.random.Generator] = None,
                jitter: float = 0.0) -> np.ndarray:
    f = FOCAL_MM / PIXEL_PITCH_MM * width / FULL_WIDTH
    cx, cy = (width - 1) / 2.0, (height - 1) / 2.0
    if rng is not None and jitter > 0:
        f *= 1.0 + rng.uniform(-jitter, jitter)
        cx += rng.uniform(-jitter, jitter) * width
        cy += rng.uniform(-jitter, jitter) * height
    return np.array([[f, 0.0, cx], [0.0, f, cy], [0.0, 0.0, 1.0]])


def _random_rotation(rng: np.random.Generator, max_degrees: float) -> np.ndarray:
    axis = _unit(rng.standard_normal(3))
    return rotation_about_axis(axis, np.deg2rad(rng.uniform(0, max_degrees)))


def _camera(width, height, k, rotation_wc, centre, distortion=None) -> ResolvedCamera:
    t = -(rotation_wc @ centre)
    return ResolvedCamera(width=width, height=height, k=k, distortion=distortion,
                          rotation_wc=rotation_wc, translation_wc=t)


_FLIP_AXIS = {True: np.diag([1.0, -1.0, 1.0]), False: np.diag([-1.0, 1.0, 1.0])}


def _mirror_camera(width, height, k, rotation_wc, centre, flip: bool, rng: np.random.Generator,
                   distortion=None, orientation=None) -> ResolvedCamera:
    """A module behind a 45-degree fold mirror (the L16's mid and tele modules) whose
    virtual camera sits at ``centre`` and looks along ``rotation_wc``.

    The mirror's normal is tilted about 45 degrees from the viewing axis (towards a
    random side), and its plane lies a few millimetres in front of the virtual centre.
    The physical module sits at the virtual centre reflected across that plane and
    looks into the mirror; its orientation real_cw makes reflect . real_cw . F equal the
    virtual camera's camera-to-world rotation, F being the image-axis flip that
    flip_img_around_x restores (geometry.rs:129-136). The pose itself comes from the
    reference's construction (geometry.rs:86-104) through ``mirror_pose``.
    ``orientation`` is an axis-angle offset in degrees (CameraRefinement's
    orientation_offset_degrees, geometry.rs:22-28, applied at geometry.rs:111-114).
    """
    rotation_cw = rotation_wc.T
    axis = rotation_cw[:, 2]
    side = rotation_cw[:, 0] * np.cos(rng.uniform(0, 2 * np.pi)) + rotation_cw[:, 1] * np.sin(rng.uniform(0, 2 * np.pi))
    side = _unit(side - axis * float(side @ axis))
    tilt = np.deg2rad(45.0 + rng.uniform(-3.0, 3.0))
    normal = _unit(-axis * np.cos(tilt) + side * np.sin(tilt))
    plane_point = centre + axis * rng.uniform(4.0, 8.0)
    location = centre - normal * (2.0 * float(normal @ (centre - plane_point)))
    real_cw = reflection(normal) @ rotation_cw @ _FLIP_AXIS[flip]
    real_cw, reflect, virtual_center = mirror_pose(location, real_cw, normal, plane_point)
    oc = np.eye(3) if orientation is None else rotation_from_axis_angle(np.asarray(orientation) * (np.pi / 180.0))
    return ResolvedCamera(width=width, height=height, k=k, distortion=distortion, flip=flip, real_cw=real_cw,
                          reflect=reflect, virtual_center=virtual_center, orientation_correction=oc)


def _random_plane(rng, ref: ResolvedCamera, depth_mm: float, coverage: Tuple[float, float],
                  max_tilt_deg: float, texel_px: float, tex_index: int) -> Surface:
    # centre on a random reference ray, finite rectangle covering part of the view
    px = np.array([[rng.uniform(0.1, 0.9) * ref.width, rng.uniform(0.1, 0.9) * ref.height]])
    o, d = ref.pixel_to_ray(px)
    centre = o[0] + d[0] * depth_mm
    tilt = np.deg2rad(rng.uniform(0, max_tilt_deg))
    az = rng.uniform(0, 2 * np.pi)
    normal = _unit([np.sin(tilt) * np.cos(az), np.sin(tilt) * np.sin(az), -np.cos(tilt)])
    u, v = _tangent_axes(normal)
    fov_mm = depth_mm * ref.width / ref.focal_px
    half_u = 0.5 * fov_mm * rng.uniform(*coverage)
    half_v = 0.5 * fov_mm * rng.uniform(*coverage) * ref.height / ref.width
    texel = depth_mm * texel_px / ref.focal_px
    return Surface("plane", centre, normal, u, v, half_u, half_v, 0.0, texel,
                   (rng.uniform(0, 512), rng.uniform(0, 512)), tex_index)


def _background(rng, ref: ResolvedCamera, depth_mm: float, texel_px: float, tex_index: int) -> Surface:
    tilt = np.deg2rad(rng.uniform(0, 10))
    az = rng.uniform(0, 2 * np.pi)
    normal = _unit([np.sin(tilt) * np.cos(az), np.sin(tilt) * np.sin(az), -np.cos(tilt)])
    u, v = _tangent_axes(normal)
    texel = depth_mm * texel_px / ref.focal_px
    return Surface("plane", np.array([0.0, 0.0, depth_mm]), normal, u, v, np.inf, np.inf, 0.0, texel,
                   (rng.uniform(0, 512), rng.uniform(0, 512)), tex_index)


def _random_sphere(rng, ref: ResolvedCamera, depth_range: Tuple[float, float], texel_px: float,
                   tex_index: int) -> Surface:
    depth = 1.0 / rng.uniform(1.0 / depth_range[1], 1.0 / depth_range[0])
    px = np.array([[rng.uniform(0.15, 0.85) * ref.width, rng.uniform(0.15, 0.85) * ref.height]])
    o, d = ref.pixel_to_ray(px)
    centre = o[0] + d[0] * depth
    fov_mm = depth * ref.width / ref.focal_px
    radius = fov_mm * rng.uniform(0.05, 0.15)
    texel = depth * texel_px / ref.focal_px
    u, v = _tangent_axes(np.array([0.0, 0.0, -1.0]))
    return Surface("sphere", centre, np.array([0.0, 0.0, -1.0]), u, v, np.inf, np.inf, radius, texel,
                   (rng.uniform(0, 512), rng.uniform(0, 512)), tex_index)


def _cast(surfaces: List[Surface], tiles: List[np.ndarray], origin: np.ndarray, direction: np.ndarray):
    """Nearest hit along rays from one centre ``origin`` [3]: (intensity in [0, 1], distance)."""
    n = direction.shape[0]
    best_t = np.full(n, np.inf)
    value = np.zeros(n)
    for s in surfaces:
        if s.kind == "plane":
            denom = direction @ s.normal
            with np.errstate(divide="ignore", invalid="ignore"):
                t = float((s.origin - origin) @ s.normal) / denom
            hit = np.isfinite(t) & (t > 1.0) & (t < best_t)
            if not hit.any():
                continue
            idx = np.flatnonzero(hit)
            th = t[idx]
            dh = direction[idx]
            o_rel = origin - s.origin
            uu = float(o_rel @ s.axis_u) + th * (dh @ s.axis_u)
            vv = float(o_rel @ s.axis_v) + th * (dh @ s.axis_v)
            inside = (np.abs(uu) <= s.half_u) & (np.abs(vv) <= s.half_v)
            idx, th, uu, vv = idx[inside], th[inside], uu[inside], vv[inside]
        else:
            oc = origin - s.origin
            b = direction @ oc
            c = float(oc @ oc) - s.radius * s.radius
            disc = b * b - c
            with np.errstate(invalid="ignore"):
                t = -b - np.sqrt(disc)
            hit = (disc > 0) & (t > 1.0) & (t < best_t)
            if not hit.any():
                continue
            idx = np.flatnonzero(hit)
            th = t[idx]
            rel = _unit_rows(oc + direction[idx] * th[:, None])
            uu = np.arctan2(rel[:, 0], -rel[:, 2]) * s.radius
            vv = np.arcsin(np.clip(rel[:, 1], -1, 1)) * s.radius
        if len(idx):
            value[idx] = _sample_tile(tiles[s.tex_index], uu / s.texel_mm + s.tex_offset[0],
                                      vv / s.texel_mm + s.tex_offset[1])
            best_t[idx] = th
    return value, best_t


def _unit_rows(a):
    return a / np.maximum(np.linalg.norm(a, axis=-1, keepdims=True), 1e-12)


def render_module(camera: ResolvedCamera, surfaces: List[Surface], tiles: List[np.ndarray], seed: int,
                  chunk_rows: int = 64):
    """Ray cast one module: (u16 raster [h, w], per-pixel distance along the ray).

    Row chunks render on a thread pool; each chunk draws its noise from its own
    seed, so the image does not depend on the number of workers.
    """
    h, w = camera.height, camera.width
    raw = np.empty((h, w), dtype=np.uint16)
    depth = np.empty((h, w), dtype=np.float32)
    xs = np.arange(w, dtype=np.float64)

    def chunk(y0: int) -> None:
        y1 = min(h, y0 + chunk_rows)
        yy, xx = np.meshgrid(np.arange(y0, y1, dtype=np.float64), xs, indexing="ij")
        pix = np.stack([xx.ravel(), yy.ravel()], -1)
        o, d = camera.pixel_to_ray(pix)
        val, t = _cast(surfaces, tiles, np.asarray(o[0]), d)
        signal = 4095.0 * (0.04 + 0.92 * val)
        # Poisson-Gaussian noise: gain 0.5 DN per electron, read noise 4 DN
        rng = np.random.default_rng((seed, y0))
        electrons = rng.poisson(signal / 0.5)
        noisy = 0.5 * electrons + rng.normal(0.0, 4.0, size=signal.shape)
        raw[y0:y1] = np.clip(np.rint(noisy), 0, 4095).astype(np.uint16).reshape(y1 - y0, w)
        depth[y0:y1] = t.reshape(y1 - y0, w).astype(np.float32)

    starts = list(range(0, h, chunk_rows))
    workers = min(len(starts), os.cpu_count() or 1, 32)
    if workers <= 1:
        for y0 in starts:
            chunk(y0)
    else:
        from threadpoolctl import threadpool_limits
        with threadpool_limits(1), ThreadPoolExecutor(max_workers=workers) as pool:
            list(pool.map(chunk, starts))
    return raw, depth


# ---- GPU rendering (benchmark workloads) ------------------------------------------
# The same scene model ray cast with torch on a CUDA device, for workloads of many
# full-resolution modules (the batched captures, the band network's training and
# evaluation sets), where the numpy renderer would take minutes. Rays, hits and
# texture follow the numpy path; the noise comes from torch's generator, so an image
# differs from the numpy renderer's for the same seed (neither is a reference output).
def _torch_normalize(v):
    import torch
    n = torch.sqrt((v * v).sum(-1, keepdim=True))
    return torch.where(n == 0, v, v / n)


def _torch_rays(camera: ResolvedCamera, pix):
    """pixel_to_ray (geometry.rs:139-166) on a [n, 2] float64 tensor: (origin [3], directions [n, 3])."""
    import torch
    dev = pix.device
    t64 = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=dev)
    ideal = pix
    d = camera.distortion
    if d is not None:
        centre, norm = t64(d.center), t64(d.normalization)
        k1, k2, p1, p2, k3 = (d.coeff(i) for i in range(5))
        observed = (pix - centre) / norm
        est = observed.clone()
        for _ in range(20):
            x, y = est[:, 0], est[:, 1]
            r2 = x * x + y * y
            radial = 1.0 + k1 * r2 + k2 * r2 * r2 + k3 * r2 * r2 * r2
            dx = x * radial + 2.0 * p1 * x * y + p2 * (r2 + 2.0 * x * x)
            dy = y * radial + p1 * (r2 + 2.0 * y * y) + 2.0 * p2 * x * y
            est = est + (observed - torch.stack([dx, dy], -1))
        ideal = est * norm + centre
    ones = torch.ones(len(pix), dtype=torch.float64, device=dev)
    direction = _torch_normalize(torch.stack([ideal[:, 0], ideal[:, 1], ones], -1) @ t64(camera.k_inverse).T)
    if camera.flip is not None:
        sign = t64([1.0, -1.0, 1.0] if camera.flip else [-1.0, 1.0, 1.0])
        direction = _torch_normalize(direction * sign)
    if camera.pose_kind == 0:
        world = direction @ t64(camera.rotation_cw).T
    else:
        world = direction @ (t64(camera.reflect) @ t64(camera.real_cw)).T
    world = _torch_normalize(_torch_normalize(world) @ t64(camera.orientation_correction).T)
    return t64(camera.center()), world


def _torch_cast(surfaces: List[Surface], tiles, origin, direction):
    """_cast on tensors: (intensity in [0, 1], distance) of the nearest hit along each ray."""
    import torch
    dev = direction.device
    n = direction.shape[0]
    best_t = torch.full((n,), float("inf"), dtype=torch.float64, device=dev)
    value = torch.zeros(n, dtype=torch.float64, device=dev)
    t64 = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=dev)
    for s in surfaces:
        if s.kind == "plane":
            normal = t64(s.normal)
            denom = direction @ normal
            t = float(np.dot(s.origin - origin.cpu().numpy(), s.normal)) / denom
            o_rel = origin - t64(s.origin)
            uu = float(o_rel @ t64(s.axis_u)) + t * (direction @ t64(s.axis_u))
            vv = float(o_rel @ t64(s.axis_v)) + t * (direction @ t64(s.axis_v))
            hit = torch.isfinite(t) & (t > 1.0) & (t < best_t) & (uu.abs() <= s.half_u) & (vv.abs() <= s.half_v)
        else:
            oc = origin - t64(s.origin)
            b = direction @ oc
            c = float(oc @ oc) - s.radius * s.radius
            disc = b * b - c
            t = -b - torch.sqrt(torch.clamp(disc, min=0.0))
            hit = (disc > 0) & (t > 1.0) & (t < best_t)
            rel = _torch_normalize(oc + direction * t[:, None])
            uu = torch.atan2(rel[:, 0], -rel[:, 2]) * s.radius
            vv = torch.asin(torch.clamp(rel[:, 1], -1, 1)) * s.radius
        tile = tiles[s.tex_index]
        size = tile.shape[0]
        u = uu / s.texel_mm + s.tex_offset[0]
        v = vv / s.texel_mm + s.tex_offset[1]
        u0, v0 = torch.floor(u), torch.floor(v)
        fu, fv = u - u0, v - v0
        iu = torch.remainder(torch.nan_to_num(u0, 0.0).long(), size)
        iv = torch.remainder(torch.nan_to_num(v0, 0.0).long(), size)
        iu1, iv1 = (iu + 1) % size, (iv + 1) % size
        top = tile[iv, iu] * (1 - fu) + tile[iv, iu1] * fu
        bottom = tile[iv1, iu] * (1 - fu) + tile[iv1, iu1] * fu
        value = torch.where(hit, top * (1 - fv) + bottom * fv, value)
        best_t = torch.where(hit, t, best_t)
    return value, best_t


def render_module_gpu(camera: ResolvedCamera, surfaces: List[Surface], tiles, seed: int, device,
                      chunk_pixels: int = 1 << 24):
    """Ray cast one module on the GPU: its u16 raster [h, w] as an int32 device tensor. Rows go
    in chunks of about chunk_pixels pixels (a whole full-resolution module in one), so the
    torch ops run on large arrays rather than paying their launch cost per small chunk."""
    import torch
    h, w = camera.height, camera.width
    chunk_rows = max(1, chunk_pixels // w)
    raw = torch.empty((h, w), dtype=torch.int32, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed) & 0x7FFFFFFFFFFFFFFF)
    xs = torch.arange(w, dtype=torch.float64, device=device)
    for y0 in range(0, h, chunk_rows):
        y1 = min(h, y0 + chunk_rows)
        yy = torch.arange(y0, y1, dtype=torch.float64, device=device)
        pix = torch.stack(torch.meshgrid(yy, xs, indexing="ij")[::-1], -1).reshape(-1, 2)
        origin, direction = _torch_rays(camera, pix)
        value, _ = _torch_cast(surfaces, tiles, origin, direction)
        signal = 4095.0 * (0.04 + 0.92 * value)
        electrons = torch.poisson(signal / 0.5, generator=gen)
        noisy = 0.5 * electrons + torch.randn(signal.shape, generator=gen, device=device, dtype=torch.float64) * 4.0
        raw[y0:y1] = torch.clamp(torch.round(noisy), 0, 4095).to(torch.int32).reshape(y1 - y0, w)
    return raw


def luminance_half_gpu(raw, black: float = 0.0, white: float = 4095.0) -> Plane:
    """luminance_half on a device raster (f32 on the GPU; the log is torch's)."""
    import torch
    h, w = raw.shape[0] // 2, raw.shape[1] // 2
    r = raw[: 2 * h, : 2 * w].to(torch.float32)
    s = ((r[0::2, 0::2] + r[0::2, 1::2]) + r[1::2, 0::2]) + r[1::2, 1::2]
    linear = torch.clamp((s * 0.25 - black) / max(white - black, 1.0), min=0.0)
    return Plane(w, h, torch.log(1.0 + 1000.0 * linear).cpu().numpy())


def luminance_half(raw: np.ndarray, black: float = 0.0, white: float = 4095.0) -> Plane:
    """image.rs:401-428 with flat field 1 (f32 arithmetic, host numpy log)."""
    h, w = raw.shape[0] // 2, raw.shape[1] // 2
    r = raw[: 2 * h, : 2 * w].astype(np.float32)
    s = ((r[0::2, 0::2] + r[0::2, 1::2]) + r[1::2, 0::2]) + r[1::2, 1::2]
    rng = np.float32(max(white - black, 1.0))
    linear = np.maximum((s * np.float32(0.25) - np.float32(black)) / rng, np.float32(0.0))
    data = np.log(np.float32(1.0) + np.float32(1000.0) * linear).astype(np.float32)
    return Plane(w, h, data)


def make_scene(name: str, width: int, height: int, n_sources: int, n_planes: int, n_spheres: int,
               depth_range: Tuple[float, float], baseline_range: Tuple[float, float],
               max_rotation_deg: float, options: DepthOptions, seed: int,
               distortion: bool = False, horizontal_only: bool = False, texel_px: float = 3.0,
               mirrors: Optional[Dict[int, bool]] = None,
               orientation: Optional[Dict[int, Tuple[float, float, float]]] = None,
               render_device=None, focal_px: Optional[float] = None) -> Scene:
    """``mirrors`` maps module indices (0 = the reference) to the flip_img_around_x value
    of a module behind a fold mirror (Pose::Mirror); ``orientation`` maps module indices
    to an axis-angle orientation offset in degrees. Both leave the random draws of the
    canonical scene unchanged (their own draws come from a separate generator), so a
    mirrored scene sees the same surfaces from the same virtual positions.
    ``render_device``: a CUDA device to ray cast on (render_module_gpu) instead of numpy.
    ``focal_px``: the modules' focal length in pixels (default: the 3 mm lens scaled to
    the raster width, the same field of view at every size)."""
    rng = np.random.default_rng(seed)
    mirror_rng = np.random.default_rng((seed, 271828))
    mirrors = mirrors or {}
    orientation = orientation or {}
    tiles = [_noise_tile(np.random.default_rng(seed * 7919 + i)) for i in range(4)]
    ref_k = _intrinsics(width, height)
    if focal_px is not None:
        ref_k[0, 0] = ref_k[1, 1] = focal_px
    ref_dist = None
    if distortion:
        ref_dist = PolynomialDistortion(((width - 1) / 2.0, (height - 1) / 2.0), (width * 0.8, width * 0.8),
                                        (0.02, -0.01, 0.0, 0.0, 0.002))
    ref = _camera(width, height, ref_k, np.eye(3), np.zeros(3), ref_dist)
    canonical = [ref]
    for _ in range(n_sources):
        b = rng.uniform(*baseline_range)
        if horizontal_only:
            direction = np.array([1.0, 0.0, 0.0])
        else:
            a = rng.uniform(0, 2 * np.pi)
            direction = np.array([np.cos(a), np.sin(a), 0.0])
        centre = direction * b
        rot = _random_rotation(rng, max_rotation_deg)
        k = _intrinsics(width, height, rng, 0.01) if distortion else ref_k
        if focal_px is not None and distortion:
            k = k.copy()
            k[0, 0] *= focal_px / _intrinsics(width, height)[0, 0]
            k[1, 1] *= focal_px / _intrinsics(width, height)[0, 0]
        dist = None
        if distortion:
            dist = PolynomialDistortion(((width - 1) / 2.0 + rng.uniform(-5, 5), (height - 1) / 2.0 + rng.uniform(-5, 5)),
                                        (width * 0.8, width * 0.8),
                                        (rng.uniform(0.0, 0.04), rng.uniform(-0.02, 0.0), 0.0, 0.0, 0.002))
        canonical.append(_camera(width, height, k, rot, centre, dist))
    cams = []
    for i, cam in enumerate(canonical):
        if i in mirrors or i in orientation:
            centre = cam.center()
            if i in mirrors:
                cam = _mirror_camera(width, height, cam.k, cam.rotation_wc, centre, mirrors[i], mirror_rng,
                                     cam.distortion, orientation.get(i))
            else:
                cam = ResolvedCamera(width=width, height=height, k=cam.k, distortion=cam.distortion,
                                     rotation_wc=cam.rotation_wc, translation_wc=cam.translation_wc,
                                     orientation_correction=rotation_from_axis_angle(
                                         np.asarray(orientation[i]) * (np.pi / 180.0)))
        cams.append(cam)
    ref = cams[0]
    near, far = depth_range
    surfaces = [_background(rng, ref, far, texel_px, 0)]
    for i in range(n_planes - 1):
        d = 1.0 / rng.uniform(1.0 / far, 1.0 / near)
        surfaces.append(_random_plane(rng, ref, d, (0.2, 0.6), 45.0, texel_px, (i + 1) % 4))
    for i in range(n_spheres):
        surfaces.append(_random_sphere(rng, ref, (max(near, 1000.0), min(far, 8000.0)), texel_px, (i + 2) % 4))
    raws, lumas, truth = [], [], None
    gpu_tiles = None
    if render_device is not None:
        import torch
        gpu_tiles = [torch.as_tensor(t, device=render_device) for t in tiles]
    for i, cam in enumerate(cams):
        if gpu_tiles is not None:  # the raster stays on the device; Scene.raw is left empty
            raw = render_module_gpu(cam, surfaces, gpu_tiles, seed * 104729 + i, render_device)
            lumas.append(luminance_half_gpu(raw))
            del raw
            continue
        raw, depth = render_module(cam, surfaces, tiles, seed * 104729 + i)
        raws.append(raw)
        lumas.append(luminance_half(raw))
        if i == 0:
            truth = depth
    warps = [Warp.identity(width, height, 32)]
    for cam in cams[1:]:
        warps.append(Warp.calibrated(ref, cam, width, height, 32))
    return Scene(name, width, height, cams, lumas, raws, warps, options, 0, surfaces, truth)


WORKLOADS: Dict[str, dict] = {
    "two_view": dict(width=1040, height=780, n_sources=1, n_planes=6, n_spheres=0, depth_range=(500.0, 20000.0),
                     baseline_range=(25.0, 25.0), max_rotation_deg=0.3, horizontal_only=True,
                     options=dict(planes=64, near_depth=400.0, far_depth=25000.0, minimum_support=1,
                                  best_view_count=1)),
    "five_view": dict(width=4160, height=3120, n_sources=4, n_planes=12, n_spheres=3,
                      depth_range=(500.0, 20000.0), baseline_range=(20.0, 60.0), max_rotation_deg=0.5,
                      distortion=True, options=dict(planes=128, near_depth=400.0, far_depth=50000.0)),
    "band": dict(width=1040, height=780, n_sources=4, n_planes=12, n_spheres=3, depth_range=(500.0, 20000.0),
                 baseline_range=(20.0, 60.0), max_rotation_deg=0.5, distortion=True,
                 options=dict(planes=192, near_depth=400.0, far_depth=50000.0)),
    "small": dict(width=320, height=240, n_sources=2, n_planes=5, n_spheres=1, depth_range=(500.0, 8000.0),
                  baseline_range=(20.0, 40.0), max_rotation_deg=0.3, distortion=True,
                  options=dict(planes=24, near_depth=400.0, far_depth=20000.0)),
    "tiny": dict(width=160, height=120, n_sources=2, n_planes=4, n_spheres=1, depth_range=(500.0, 6000.0),
                 baseline_range=(20.0, 40.0), max_rotation_deg=0.3, distortion=False,
                 options=dict(planes=16, near_depth=400.0, far_depth=20000.0)),
}

# One synthetic 16-module capture as the depth stage sees it: 10 reference/source
# groupings of 5 wide modules (canonical poses), 5 mid and 6 tele modules (behind fold
# mirrors, alternating flip_img_around_x). Every module is resampled to the wide
# modules' angular pixel size (a common bandwidth: the 3 mm lens at 1.12 um), so a
# grouping's raster is its field of view at that size: 4160x3120 for the wide modules
# down to 1040x780 for the tele ones. (width, height, planes, kind, sources)
CAPTURE_GROUPINGS = [(4160, 3120, 128, "wide", 4), (4160, 3120, 192, "wide", 4), (3120, 2340, 64, "mid", 3),
                     (3120, 2340, 128, "mid", 4), (2080, 1560, 192, "mid", 3), (2080, 1560, 64, "tele", 2),
                     (2080, 1560, 128, "tele", 3), (1560, 1170, 192, "tele", 3), (1040, 780, 64, "tele", 2),
                     (1040, 780, 128, "tele", 3)]


def make_capture(seed: int, render_device=None, planes=None, surfaces: Tuple[int, int] = (12, 3),
                 groupings=CAPTURE_GROUPINGS) -> List[Scene]:
    """The groupings of one seeded capture, each a Scene of its raster size, plane count and
    module kind (mid and tele modules behind mirrors). ``planes`` (optional) replaces each
    grouping's plane count, e.g. drawn per capture; ``surfaces`` = (slanted planes, spheres)."""
    out = []
    for g, (width, height, default_planes, kind, sources) in enumerate(groupings):
        flip = (seed + g) % 2 == 0
        mirrors = {} if kind == "wide" else {i: (flip if i % 2 == 0 else not flip) for i in range(sources + 1)}
        opt = DepthOptions(planes=(planes[g] if planes is not None else default_planes), near_depth=400.0,
                           far_depth=50000.0)
        out.append(make_scene(f"capture{seed}.{g}.{kind}", width, height, sources, surfaces[0], surfaces[1],
                              (500.0, 20000.0), (20.0, 60.0), 0.5, opt, seed * 1000 + g, distortion=True,
                              mirrors=mirrors, render_device=render_device, focal_px=FOCAL_MM / PIXEL_PITCH_MM))
    return out


_CACHE: Dict[tuple, Scene] = {}


def workload(name: str, seed: int = 0, cache: bool = True, **overrides) -> Scene:
    """Render a named workload (see module docstring) from ``seed``."""
    key = (name, seed, repr(sorted(overrides.items())))
    if cache and key in _CACHE:
        return _CACHE[key]
    spec = dict(WORKLOADS[name])
    opt = DepthOptions(**{**spec.pop("options"), **overrides.pop("options", {})})
    spec.update(overrides)
    scene = make_scene(name, options=opt, seed=seed, **spec)
    if cache:
        _CACHE[key] = scene
    return scene
