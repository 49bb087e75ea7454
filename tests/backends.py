"""Two implementations of the stage's array operators behind one interface.

``OracleBackend`` calls the CPU oracle; ``GpuBackend`` calls the CUDA library
through its C ABI. The known-answer tests and the parity tests run the same
cases through both.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from chiaro_b200 import abi
from chiaro_b200.abi import dptr, fptr, u8ptr


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _u8(a):
    return np.ascontiguousarray(a, dtype=np.uint8)


class OracleBackend:
    name = "oracle"

    def __init__(self):
        from oracle import oracle
        self.o = oracle
        self.L = oracle.lib()

    def sgm(self, costs, guidance, columns, rows, labels):
        return self.o.semi_global_costs(costs, guidance, columns, rows, labels)

    def select_depths(self, labels, scores, regularised, tested, options):
        labels, scores, regularised, tested = _f64(labels), _f32(scores), _f32(regularised), _u8(tested)
        n = len(tested)
        out = dict(has=np.zeros(n, np.uint8), depth=np.zeros(n), confidence=np.zeros(n, np.float32),
                   improvement=np.zeros(n, np.float32), regularized=np.zeros(n, np.uint8),
                   fillable=np.zeros(n, np.uint8))
        opt = options.to_c()
        self.L.oracle_select_depths(dptr(labels), len(labels), fptr(scores), fptr(regularised), u8ptr(tested), n,
                                    C.byref(opt), u8ptr(out["has"]), dptr(out["depth"]), fptr(out["confidence"]),
                                    fptr(out["improvement"]), u8ptr(out["regularized"]), u8ptr(out["fillable"]))
        return out

    def reject_isolated(self, has, depth, confidence, guidance, columns, rows, tol):
        has = _u8(has).copy()
        self.L.oracle_reject_isolated(u8ptr(has), dptr(_f64(depth)), fptr(_f32(confidence)), fptr(_f32(guidance)),
                                      columns, rows, tol)
        return has

    def reject_small_components(self, has, depth, guidance, columns, rows, tol, minimum):
        has = _u8(has).copy()
        self.L.oracle_reject_small_components(u8ptr(has), dptr(_f64(depth)), fptr(_f32(guidance)), columns, rows,
                                              tol, minimum)
        return has

    def fit_local_planes(self, has, depth, confidence, guidance, columns, rows, tol):
        depth = _f64(depth).copy()
        self.L.oracle_fit_local_planes(u8ptr(_u8(has)), dptr(depth), fptr(_f32(confidence)), fptr(_f32(guidance)),
                                       columns, rows, tol)
        return depth

    def warp_filter(self, kind, glob, point, measured, guidance, columns, rows, consensus=True, boundaries=True):
        kind, glob, point = _u8(kind).copy(), _f32(glob).copy(), _f32(point).copy()
        self.L.oracle_warp_decisions_filter(u8ptr(kind), fptr(glob), fptr(point), u8ptr(_u8(measured)),
                                            fptr(_f32(guidance)), columns, rows, int(consensus), int(boundaries))
        return kind, glob, point


class GpuBackend:
    name = "gpu"

    def __init__(self, ctx):
        self.ctx = ctx
        self.L = ctx.lib

    def sgm(self, costs, guidance, columns, rows, labels):
        costs, guidance = _f32(costs), _f32(guidance)
        out = np.empty(columns * rows * labels, dtype=np.float32)
        self.ctx.check(self.L.chiaro_sgm_aggregate(self.ctx.handle, fptr(costs), fptr(guidance), columns, rows,
                                                   labels, fptr(out)))
        return out

    def select_depths(self, labels, scores, regularised, tested, options):
        labels, scores, regularised, tested = _f64(labels), _f32(scores), _f32(regularised), _u8(tested)
        n = len(tested)
        out = dict(has=np.zeros(n, np.uint8), depth=np.zeros(n), confidence=np.zeros(n, np.float32),
                   improvement=np.zeros(n, np.float32), regularized=np.zeros(n, np.uint8),
                   fillable=np.zeros(n, np.uint8))
        opt = options.to_c()
        self.ctx.check(self.L.chiaro_select_depths(
            self.ctx.handle, dptr(labels), len(labels), fptr(scores), fptr(regularised), u8ptr(tested), n,
            C.byref(opt), u8ptr(out["has"]), dptr(out["depth"]), fptr(out["confidence"]),
            fptr(out["improvement"]), u8ptr(out["regularized"]), u8ptr(out["fillable"])))
        return out

    def reject_isolated(self, has, depth, confidence, guidance, columns, rows, tol):
        has = _u8(has).copy()
        self.ctx.check(self.L.chiaro_reject_isolated(self.ctx.handle, u8ptr(has), dptr(_f64(depth)),
                                                     fptr(_f32(confidence)), fptr(_f32(guidance)), columns, rows,
                                                     tol))
        return has

    def reject_small_components(self, has, depth, guidance, columns, rows, tol, minimum):
        has = _u8(has).copy()
        self.ctx.check(self.L.chiaro_reject_small_components(self.ctx.handle, u8ptr(has), dptr(_f64(depth)),
                                                             fptr(_f32(guidance)), columns, rows, tol, minimum))
        return has

    def fit_local_planes(self, has, depth, confidence, guidance, columns, rows, tol):
        depth = _f64(depth).copy()
        self.ctx.check(self.L.chiaro_fit_local_planes(self.ctx.handle, u8ptr(_u8(has)), dptr(depth),
                                                      fptr(_f32(confidence)), fptr(_f32(guidance)), columns, rows,
                                                      tol))
        return depth

    def warp_filter(self, kind, glob, point, measured, guidance, columns, rows, consensus=True, boundaries=True):
        kind, glob, point = _u8(kind).copy(), _f32(glob).copy(), _f32(point).copy()
        self.ctx.check(self.L.chiaro_warp_decisions_filter(self.ctx.handle, u8ptr(kind), fptr(glob), fptr(point),
                                                           u8ptr(_u8(measured)), fptr(_f32(guidance)), columns,
                                                           rows, int(consensus), int(boundaries)))
        return kind, glob, point
