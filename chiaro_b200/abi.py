"""ctypes mirror of ``include/chiaro_depth.h``.

The structures here are byte-for-byte the C ABI of the depth library: the
Python host layer (``chiaro_b200.depth``) fills them from the Rust-shaped
objects, and a Rust ``-sys`` crate would declare the same ``#[repr(C)]``
structs. Field comments cite the reference type each struct mirrors.
"""
from __future__ import annotations

import ctypes as C

ABI_VERSION = 1

OK = 0
INVALID = 1
ERR_CUDA = 2
ERR_TIMEOUT = 3
ERR_CAPACITY = 4
ERR_ARGUMENT = 5

STATUS_NAMES = {
    OK: "ok",
    INVALID: "invalid input (the reference returns None)",
    ERR_CUDA: "CUDA error",
    ERR_TIMEOUT: "device wait timed out",
    ERR_CAPACITY: "output buffer too small",
    ERR_ARGUMENT: "bad argument",
}

# DepthProvenance (crates/chiaro-fusion/src/depth.rs:115-121)
UNSUPPORTED, GLOBAL, MEASURED, REGULARIZED = 0, 1, 2, 3
# NodeWarp kinds (depth.rs:256-271)
NW_UNDEFINED, NW_GLOBAL, NW_REFINED, NW_OCCLUDED, NW_BOUNDARY = 0, 1, 2, 3, 4


class DepthOptionsC(C.Structure):
    """DepthOptions (depth.rs:39-67)."""

    _fields_ = [
        ("enabled", C.c_int32),
        ("_pad0", C.c_int32),
        ("grid_step", C.c_uint64),
        ("near_depth", C.c_double),
        ("far_depth", C.c_double),
        ("planes", C.c_uint64),
        ("patch_radius", C.c_uint64),
        ("minimum_support", C.c_uint64),
        ("best_view_count", C.c_uint64),
        ("minimum_score", C.c_float),
        ("minimum_margin", C.c_float),
        ("minimum_improvement", C.c_float),
        ("_pad1", C.c_int32),
        ("minimum_neighbour_support", C.c_uint64),
        ("completion_iterations", C.c_uint64),
    ]


class CameraC(C.Structure):
    """ResolvedCamera (geometry.rs:31-62)."""

    _fields_ = [
        ("width", C.c_uint64),
        ("height", C.c_uint64),
        ("k", C.c_double * 9),
        ("k_inverse", C.c_double * 9),
        ("has_distortion", C.c_int32),
        ("flip", C.c_int32),
        ("distortion_center", C.c_double * 2),
        ("distortion_normalization", C.c_double * 2),
        ("distortion_coeffs", C.c_double * 5),
        ("pose_kind", C.c_int32),
        ("_pad0", C.c_int32),
        ("rotation_wc", C.c_double * 9),
        ("rotation_cw", C.c_double * 9),
        ("translation_wc", C.c_double * 3),
        ("center", C.c_double * 3),
        ("real_cw", C.c_double * 9),
        ("reflect", C.c_double * 9),
        ("virtual_center", C.c_double * 3),
        ("orientation_correction", C.c_double * 9),
    ]


class BandOptionsC(C.Structure):
    """chiaro_band_options: the learned-band form of the coarse search."""

    _fields_ = [
        ("params", C.c_void_p),
        ("tile", C.c_uint64),
        ("band", C.c_uint64),
        ("margin", C.c_uint64),
        ("contradicted_fraction", C.c_float),
        ("_pad0", C.c_int32),
    ]


class BandReportC(C.Structure):
    """chiaro_band_report: what a coarse search did."""

    _fields_ = [
        ("tiles", C.c_uint64),
        ("edge_tiles", C.c_uint64),
        ("consistency_tiles", C.c_uint64),
        ("fallback_tiles", C.c_uint64),
        ("windows", C.c_uint64),
        ("window_nodes", C.c_uint64),
        ("ms", C.c_float * 7),
        ("_pad0", C.c_int32),
    ]


class SgmInstanceC(C.Structure):
    """chiaro_sgm_instance: one SGM instance of a batch (device pointers)."""

    _fields_ = [
        ("costs", C.c_void_p),
        ("guidance", C.c_void_p),
        ("out", C.c_void_p),
        ("columns", C.c_uint64),
        ("rows", C.c_uint64),
        ("labels", C.c_uint64),
    ]


BATCH_GRAPH = 1
BATCH_AUTOTUNE = 2


class VignettingC(C.Structure):
    """VignettingMesh (calibration.rs:354-358)."""

    _fields_ = [
        ("columns", C.c_uint64),
        ("rows", C.c_uint64),
        ("gains", C.POINTER(C.c_float)),
    ]


class AlignInputC(C.Structure):
    """AlignInput (align.rs:246-257)."""

    _fields_ = [
        ("luminance", C.POINTER(C.c_float)),
        ("luma_width", C.c_uint64),
        ("luma_height", C.c_uint64),
        ("width", C.c_uint64),
        ("height", C.c_uint64),
        ("has_camera", C.c_int32),
        ("camera", CameraC),
        ("nominal_focal_px", C.c_double),
    ]


class AlignOptionsC(C.Structure):
    """AlignOptions (align.rs:205-243) without the depth options."""

    _fields_ = [
        ("grid_step", C.c_uint64),
        ("patch", C.c_uint64),
        ("coarse_radius", C.c_uint64),
        ("min_score", C.c_float),
        ("inlier_px", C.c_float),
        ("min_inlier_ratio", C.c_float),
        ("refine", C.c_int32),
    ]


ALIGN_MAX_LEVELS = 24


class AlignLevelC(C.Structure):
    _fields_ = [("scale", C.c_uint64), ("patches", C.c_uint64), ("inliers", C.c_uint64),
                ("median_residual_px", C.c_float)]


class AlignmentReportC(C.Structure):
    """The alignment fields of AlignmentReport (align.rs:160-200)."""

    _fields_ = [
        ("initialised_from", C.c_int32),
        ("status", C.c_int32),
        ("accepted", C.c_int32),
        ("coverage", C.c_float),
        ("correction_median_px", C.c_float * 2),
        ("inliers", C.c_uint64),
        ("patches", C.c_uint64),
        ("residual_median_px", C.c_float),
        ("residual_p90_px", C.c_float),
        ("inlier_ratio", C.c_float),
        ("n_levels", C.c_uint64),
        ("levels", AlignLevelC * ALIGN_MAX_LEVELS),
    ]


INITIALISED_FROM = ["reference", None, "calibration", "nominal focal group"]  # 1: the seed's name
ALIGN_STATUS = ["reference", "rejected", "factory model only", "refined", "weak refinement",
                "no correlation support; factory model kept"]


class ResolutionReportC(C.Structure):
    """ResolutionAlignmentReport (resolution.rs:88-100)."""

    _fields_ = [
        ("verified_fraction", C.c_float),
        ("supported_fraction", C.c_float),
        ("median_correction_px", C.c_float),
        ("mean_confidence", C.c_float),
    ]


class WarpC(C.Structure):
    """Warp (align.rs:34-45)."""

    _fields_ = [
        ("step", C.c_uint64),
        ("columns", C.c_uint64),
        ("rows", C.c_uint64),
        ("points", C.POINTER(C.c_float)),
        ("confidence", C.POINTER(C.c_float)),
        ("capacity", C.c_uint64),
    ]


class ViewC(C.Structure):
    """AlignInput (align.rs:246-257) + ModuleAlignment.warp/accepted (align.rs:148-157)."""

    _fields_ = [
        ("luminance", C.POINTER(C.c_float)),
        ("luma_width", C.c_uint64),
        ("luma_height", C.c_uint64),
        ("width", C.c_uint64),
        ("height", C.c_uint64),
        ("has_camera", C.c_int32),
        ("accepted", C.c_int32),
        ("camera", CameraC),
        ("warp", WarpC),
    ]


class DepthMapC(C.Structure):
    """DenseDepthMap (depth.rs:133-141)."""

    _fields_ = [
        ("columns", C.c_uint64),
        ("rows", C.c_uint64),
        ("step", C.c_uint64),
        ("near_depth", C.c_double),
        ("far_depth", C.c_double),
        ("capacity", C.c_uint64),
        ("depth", C.POINTER(C.c_double)),
        ("confidence", C.POINTER(C.c_float)),
        ("provenance", C.POINTER(C.c_uint8)),
    ]


class DepthReportC(C.Structure):
    """DepthAlignmentReport (depth.rs:93-113)."""

    _fields_ = [
        ("present", C.c_int32),
        ("has_median_depth", C.c_int32),
        ("tested_nodes", C.c_uint64),
        ("measured_nodes", C.c_uint64),
        ("regularized_nodes", C.c_uint64),
        ("fallback_nodes", C.c_uint64),
        ("refined_nodes", C.c_uint64),
        ("occluded_nodes", C.c_uint64),
        ("boundary_nodes", C.c_uint64),
        ("reconstructed_fraction", C.c_float),
        ("refined_fraction", C.c_float),
        ("occluded_fraction", C.c_float),
        ("has_median_score_improvement", C.c_int32),
        ("median_depth", C.c_double),
        ("median_score_improvement", C.c_float),
        ("_pad0", C.c_int32),
    ]


_DEBUG_FIELDS = [
    ("coarse_scores", C.c_float),
    ("coarse_costs", C.c_float),
    ("coarse_guidance", C.c_float),
    ("coarse_tested", C.c_uint8),
    ("regularised", C.c_float),
    ("coarse_has", C.c_uint8),
    ("coarse_depth", C.c_double),
    ("coarse_confidence", C.c_float),
    ("coarse_improvement", C.c_float),
    ("coarse_regularized", C.c_uint8),
    ("coarse_fillable", C.c_uint8),
    ("direct_has", C.c_uint8),
    ("direct_depth", C.c_double),
    ("direct_confidence", C.c_float),
    ("direct_improvement", C.c_float),
    ("direct_regularized", C.c_uint8),
    ("direct_guidance", C.c_float),
    ("direct_tested", C.c_uint8),
    ("isolated_has", C.c_uint8),
    ("component_has", C.c_uint8),
    ("fitted_depth", C.c_double),
    ("decision_kind", C.c_uint8),
]


class DepthDebugC(C.Structure):
    """Intermediate-stage capture buffers (all optional)."""

    _fields_ = [(name, C.POINTER(t)) for name, t in _DEBUG_FIELDS]


DEBUG_FIELD_TYPES = dict(_DEBUG_FIELDS)


def fptr(a):
    """Pointer to a contiguous numpy float32 array."""
    return a.ctypes.data_as(C.POINTER(C.c_float))


def dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def u8ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def u16ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint16))


def sizeptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_size_t))
