"""Loading of the CUDA library and the per-thread device context.

The library is ``chiaro_b200/_build/libchiaro_depth.so`` (built in-tree by
``chiaro_b200.build``). Loading fails loudly when it is missing: the depth
stage has no CPU fallback.
"""
from __future__ import annotations

import collections
import ctypes as C
import threading
import weakref
from pathlib import Path
from typing import Optional

import numpy as np

from . import abi
from .abi import (DepthDebugC, DepthMapC, DepthOptionsC, DepthReportC, ViewC, WarpC)
from .build import HOSTCHECK, LIB

P = C.POINTER

# name -> (restype, argtypes); mirrors include/chiaro_depth.h
SIGNATURES = {
    "chiaro_depth_abi_version": (C.c_int, []),
    "chiaro_depth_ctx_create": (C.c_int, [C.c_int, P(C.c_void_p)]),
    "chiaro_depth_ctx_destroy": (None, [C.c_void_p]),
    "chiaro_depth_last_error": (C.c_char_p, [C.c_void_p]),
    "chiaro_depth_options_default": (None, [P(DepthOptionsC)]),
    "chiaro_depth_options_valid": (C.c_int, [P(DepthOptionsC)]),
    "chiaro_depth_output_shape": (C.c_int, [C.c_uint64, C.c_uint64, P(DepthOptionsC), P(C.c_uint64),
                                            P(C.c_uint64), P(C.c_uint64), P(C.c_uint64), P(C.c_uint64),
                                            P(C.c_uint64)]),
    "chiaro_refine_multiview_depth": (C.c_int, [C.c_void_p, P(ViewC), C.c_size_t, C.c_size_t, P(DepthOptionsC),
                                                P(WarpC), P(DepthReportC), P(DepthMapC), P(DepthDebugC)]),
    "chiaro_refine_multiview_depth_device": (C.c_int, [C.c_void_p, P(ViewC), C.c_size_t, C.c_size_t,
                                                       P(DepthOptionsC), P(WarpC), P(DepthReportC), P(DepthMapC)]),
    "chiaro_depth_last_timings": (C.c_int, [C.c_void_p, P(C.c_float), C.c_int]),
    "chiaro_depth_last_launches": (C.c_int, [C.c_void_p]),
    "chiaro_depth_ctx_stream": (C.c_void_p, [C.c_void_p]),
    "chiaro_sgm_aggregate_u16": (C.c_int, [C.c_void_p, P(C.c_float), P(C.c_float), C.c_uint64, C.c_uint64,
                                           C.c_uint64, P(C.c_uint16), P(C.c_uint16)]),
    "chiaro_sgm_aggregate_u16_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64,
                                                  C.c_uint64, C.c_void_p, C.c_void_p]),
    "chiaro_sgm_aggregate_batch_device": (C.c_int, [C.c_void_p, P(abi.SgmInstanceC), C.c_uint64, C.c_uint64,
                                                    C.c_int]),
    "chiaro_sgm_batch_report": (C.c_int, [C.c_void_p, P(C.c_int), P(C.c_int), P(C.c_int)]),
    "chiaro_sgm_banded_report": (C.c_int, [C.c_void_p, P(C.c_int)]),
    "chiaro_warp_sample_device": (C.c_int, [C.c_void_p, P(abi.WarpC), C.c_void_p, C.c_uint64, C.c_void_p,
                                            C.c_void_p]),
    "chiaro_depth_sample_nearest_device": (C.c_int, [C.c_void_p, P(abi.DepthMapC), C.c_void_p, C.c_uint64,
                                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "chiaro_depth_set_stage_graph": (C.c_int, [C.c_void_p, C.c_int32]),
    "chiaro_depth_stage_graph_state": (C.c_int, [C.c_void_p]),
    "chiaro_depth_set_union_retry_limit": (C.c_int, [C.c_void_p, C.c_int32]),
    "chiaro_depth_set_memory_limit": (C.c_int, [C.c_void_p, C.c_uint64]),
    "chiaro_depth_memory_held": (C.c_uint64, [C.c_void_p]),
    "chiaro_depth_set_autotune": (C.c_int, [C.c_void_p, C.c_int32]),
    "chiaro_depth_tuning": (C.c_int, [C.c_void_p, P(C.c_uint64), P(C.c_int32), C.c_int]),
    "chiaro_align_options_default": (None, [P(abi.AlignOptionsC)]),
    "chiaro_align_module": (C.c_int, [C.c_void_p, P(abi.AlignInputC), P(abi.AlignInputC), C.c_int32,
                                      P(abi.AlignOptionsC), P(abi.WarpC), P(abi.WarpC), P(C.c_float),
                                      P(abi.AlignmentReportC)]),
    "chiaro_refine_resolution_warp_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p,
                                                       C.c_uint64, C.c_uint64, P(abi.WarpC), C.c_uint64,
                                                       C.c_uint64, P(abi.WarpC), P(abi.ResolutionReportC)]),
    "chiaro_refine_resolution_warp": (C.c_int, [C.c_void_p, P(C.c_float), C.c_uint64, C.c_uint64, P(C.c_float),
                                                C.c_uint64, C.c_uint64, P(abi.WarpC), C.c_uint64, C.c_uint64,
                                                P(abi.WarpC), P(abi.ResolutionReportC)]),
    "chiaro_sgm_banded": (C.c_int, [C.c_void_p, P(C.c_float), P(C.c_float), C.c_uint64, C.c_uint64, C.c_uint64,
                                    P(C.c_int32), C.c_uint64, C.c_uint64, C.c_uint64, P(C.c_int32), P(C.c_uint8)]),
    "chiaro_sgm_banded_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64,
                                           C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p]),
    "chiaro_bandnet_parameter_count": (C.c_uint64, []),
    "chiaro_bandnet_propose_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                                C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64,
                                                C.c_void_p, C.c_void_p]),
    "chiaro_bandnet_train_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                              C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64,
                                              C.c_float, P(C.c_float)]),
    "chiaro_bandnet_gradient_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64,
                                                 C.c_uint64, C.c_void_p, P(C.c_float)]),
    "chiaro_coarse_depth_device": (C.c_int, [C.c_void_p, P(ViewC), C.c_size_t, C.c_size_t, P(DepthOptionsC),
                                             P(abi.BandOptionsC), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             P(abi.BandReportC)]),
    "chiaro_band_prepass_device": (C.c_int, [C.c_void_p, P(ViewC), C.c_size_t, C.c_size_t, P(DepthOptionsC),
                                             C.c_void_p, C.c_void_p, C.c_void_p]),
    "chiaro_host_alloc": (C.c_int, [C.c_uint64, P(C.c_void_p)]),
    "chiaro_host_free": (None, [C.c_void_p]),
    "chiaro_luminance_half": (C.c_int, [C.c_void_p, P(C.c_uint16), C.c_uint64, C.c_uint64, C.c_float, C.c_float,
                                        P(abi.VignettingC), P(C.c_float)]),
    "chiaro_luminance_half_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_float,
                                               C.c_float, P(abi.VignettingC), C.c_void_p]),
    "chiaro_sgm_aggregate": (C.c_int, [C.c_void_p, P(C.c_float), P(C.c_float), C.c_uint64, C.c_uint64, C.c_uint64,
                                       P(C.c_float)]),
    "chiaro_sgm_aggregate_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64,
                                              C.c_uint64, C.c_void_p]),
    "chiaro_select_depths": (C.c_int, [C.c_void_p, P(C.c_double), C.c_uint64, P(C.c_float), P(C.c_float),
                                       P(C.c_uint8), C.c_uint64, P(DepthOptionsC), P(C.c_uint8), P(C.c_double),
                                       P(C.c_float), P(C.c_float), P(C.c_uint8), P(C.c_uint8)]),
    "chiaro_reject_isolated": (C.c_int, [C.c_void_p, P(C.c_uint8), P(C.c_double), P(C.c_float), P(C.c_float),
                                         C.c_uint64, C.c_uint64, C.c_double]),
    "chiaro_reject_small_components": (C.c_int, [C.c_void_p, P(C.c_uint8), P(C.c_double), P(C.c_float),
                                                 C.c_uint64, C.c_uint64, C.c_double, C.c_uint64]),
    "chiaro_fit_local_planes": (C.c_int, [C.c_void_p, P(C.c_uint8), P(C.c_double), P(C.c_float), P(C.c_float),
                                          C.c_uint64, C.c_uint64, C.c_double]),
    "chiaro_warp_decisions_filter": (C.c_int, [C.c_void_p, P(C.c_uint8), P(C.c_float), P(C.c_float),
                                               P(C.c_uint8), P(C.c_float), C.c_uint64, C.c_uint64, C.c_int,
                                               C.c_int]),
    "chiaro_reject_small_components_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                         C.c_uint64, C.c_uint64, C.c_double, C.c_uint64,
                                                         C.c_void_p]),
}

HOSTCHECK_SIGNATURES = {
    "chiaro_hc_exp_f32": (C.c_float, [C.c_float]),
    "chiaro_hc_exp_f64": (C.c_double, [C.c_double]),
    "chiaro_hc_expf_mismatches": (C.c_uint64, [C.c_uint32, C.c_uint32, C.c_int, P(C.c_uint32)]),
    "chiaro_hc_exp_mismatches": (C.c_uint64, [C.c_uint32, C.c_uint32, C.c_double, P(C.c_uint32)]),
    "chiaro_hc_floor_mismatches": (C.c_uint64, [C.c_uint32, C.c_uint32]),
    "chiaro_hc_smalldiv_mismatches": (C.c_uint64, []),
    "chiaro_hc_aggregate_mismatches": (C.c_uint64, [C.c_uint64, C.c_uint64]),
    "chiaro_hc_plane_sample": (C.c_float, [P(C.c_float), C.c_int, C.c_int, C.c_float, C.c_float, P(C.c_int)]),
    "chiaro_hc_warp_map": (C.c_int, [P(C.c_float), C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                     P(C.c_float)]),
    "chiaro_hc_map_from": (C.c_int, [P(abi.CameraC), P(abi.CameraC), P(C.c_double), C.c_double, P(C.c_double)]),
}

_lib = None
_hostcheck = None
_lock = threading.Lock()
_local = threading.local()


def _bind(lib, table):
    for name, (res, args) in table.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def library_path() -> Path:
    return LIB


def load_library():
    """Load libchiaro_depth.so (raising if it has not been built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB.exists():
                raise RuntimeError(f"{LIB} is missing: build it with `python -m chiaro_b200.build` "
                                   "(the depth stage has no CPU fallback)")
            _lib = _bind(C.CDLL(str(LIB)), SIGNATURES)
            if _lib.chiaro_depth_abi_version() != abi.ABI_VERSION:
                raise RuntimeError("libchiaro_depth.so ABI version mismatch")
    return _lib


def load_hostcheck():
    global _hostcheck
    with _lock:
        if _hostcheck is None:
            if not HOSTCHECK.exists():
                raise RuntimeError(f"{HOSTCHECK} is missing: run `python -m chiaro_b200.build`")
            _hostcheck = _bind(C.CDLL(str(HOSTCHECK)), HOSTCHECK_SIGNATURES)
    return _hostcheck


class DepthContext:
    """One CUDA device context of the library (own stream and buffers)."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        status = self.lib.chiaro_depth_ctx_create(device, C.byref(h))
        if status != abi.OK:
            raise RuntimeError(f"chiaro_depth_ctx_create(device={device}) failed: {abi.STATUS_NAMES.get(status)}")
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            self.lib.chiaro_depth_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, status: int):
        if status != abi.OK:
            msg = self.lib.chiaro_depth_last_error(self.handle) or b""
            raise RuntimeError(f"depth library error {status} ({abi.STATUS_NAMES.get(status, '?')}): "
                               f"{msg.decode(errors='replace')}")

    def timings(self) -> dict:
        ms = (C.c_float * 7)()
        n = self.lib.chiaro_depth_last_timings(self.handle, ms, 7)
        names = ["cost_volume", "sgm", "select", "direct", "filters", "decisions", "total"]
        return {names[i]: float(ms[i]) for i in range(n)}

    def launches(self) -> int:
        return int(self.lib.chiaro_depth_last_launches(self.handle))

    def stream_handle(self) -> int:
        return int(self.lib.chiaro_depth_ctx_stream(self.handle) or 0)

    def set_union_retry_limit(self, retries: int = -1) -> None:
        """Bound the union-find joins' attempts (negative: the node count plus one, which
        cannot run out; 0: every join gives up at once)."""
        self.check(self.lib.chiaro_depth_set_union_retry_limit(self.handle, int(retries)))

    def set_memory_limit(self, nbytes: int = 0) -> None:
        """Cap the device memory the context's buffers may hold (0: no cap)."""
        self.check(self.lib.chiaro_depth_set_memory_limit(self.handle, int(nbytes)))

    def memory_held(self) -> int:
        return int(self.lib.chiaro_depth_memory_held(self.handle))

    def set_autotune(self, mode) -> None:
        """Launch shapes of the cost volume: True/1 autotune (the default), False/0 the default
        shape, or a CTA size (64, 96, 128, 160, 192) for every launch."""
        self.check(self.lib.chiaro_depth_set_autotune(self.handle, int(mode)))

    def tuning(self) -> dict:
        """The autotuner's choices: {(targets, labels scored, radius): threads per node CTA}."""
        n = int(self.lib.chiaro_depth_tuning(self.handle, None, None, 0))
        keys = (C.c_uint64 * max(n, 1))()
        threads = (C.c_int32 * max(n, 1))()
        n = int(self.lib.chiaro_depth_tuning(self.handle, keys, threads, n))
        return {(int(k) >> 24, (int(k) >> 8) & 0xFFFF, int(k) & 0xFF): int(t) for k, t in zip(keys[:n], threads[:n])}

    def make_debug(self, arrays: dict) -> DepthDebugC:
        dbg = DepthDebugC()
        for name, arr in arrays.items():
            setattr(dbg, name, arr.ctypes.data_as(C.POINTER(abi.DEBUG_FIELD_TYPES[name])))
        return dbg


class _PinnedBlock:
    """One page-locked host buffer lent to numpy arrays; back to the pool when they are gone."""

    def __init__(self, pool, ptr: int, nbytes: int, shape, dtype):
        shape = (int(shape),) if np.isscalar(shape) else tuple(int(s) for s in shape)
        self.__array_interface__ = {"data": (ptr, False), "shape": shape,
                                    "typestr": np.dtype(dtype).str, "version": 3}
        weakref.finalize(self, pool._release, ptr, nbytes)


class PinnedPool:
    """A caching pool of page-locked host buffers (chiaro_host_alloc), keyed by size.

    ``empty(shape, dtype)`` returns a numpy array backed by pinned memory; when the
    array and every view of it are garbage-collected, the buffer returns to the pool
    for the next call, so a steady loop of stage calls pins its output memory once.
    The return path takes no lock (a finalizer may run inside any allocation, the
    pool's own included): it appends to a deque that ``empty`` drains.
    """

    def __init__(self, lib):
        self.lib = lib
        self.free = {}
        self.returned = collections.deque()
        self.lock = threading.Lock()

    def empty(self, shape, dtype) -> np.ndarray:
        nbytes = max(int(np.prod(shape)) * np.dtype(dtype).itemsize, 1)
        ptr = None
        with self.lock:
            while self.returned:
                size, p = self.returned.popleft()
                self.free.setdefault(size, []).append(p)
            stack = self.free.get(nbytes)
            if stack:
                ptr = stack.pop()
        if ptr is None:
            p = C.c_void_p()
            if self.lib.chiaro_host_alloc(nbytes, C.byref(p)) != abi.OK or not p.value:
                return np.empty(shape, dtype)  # pinning refused: pageable memory still works
            ptr = p.value
        return np.asarray(_PinnedBlock(self, ptr, nbytes, shape, dtype))

    def _release(self, ptr: int, nbytes: int):
        self.returned.append((nbytes, ptr))


_pinned: Optional[PinnedPool] = None


def pinned_pool() -> PinnedPool:
    global _pinned
    lib = load_library()  # takes _lock itself
    with _lock:
        if _pinned is None:
            _pinned = PinnedPool(lib)
    return _pinned


def default_context(device: Optional[int] = None) -> DepthContext:
    """The calling thread's context (one per host thread, as the library requires)."""
    ctx = getattr(_local, "ctx", None)
    if ctx is None or (device is not None and ctx.device != device):
        ctx = DepthContext(0 if device is None else device)
        _local.ctx = ctx
    return ctx
