"""ORACLE — test infrastructure only.

ctypes binding of the CPU restatement (oracle/src). Imported only by the
tests, by ``__graft_entry__.smoke()`` as the checker, and by the CPU-baseline
leg of ``bench.py``. The product library never loads it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_u8p = ctypes.POINTER(ctypes.c_uint8)
_i32p = ctypes.POINTER(ctypes.c_int32)
_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)


def build() -> str:
    """Compile the restatement (make, in-tree) and return the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_create.restype = ctypes.c_void_p
        L.oracle_create.argtypes = [ctypes.c_int]
        L.oracle_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_set_reference.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_int, ctypes.c_int, _u8p]
        L.oracle_run.argtypes = [ctypes.c_void_p, _u8p, _u8p, _i32p, _f32p, ctypes.c_int, _f32p,
                                 ctypes.c_int, _f64p]
        L.oracle_run_capture.argtypes = [ctypes.c_void_p, _u8p, _u8p, _i32p, _f32p, ctypes.c_int,
                                         _f32p, ctypes.c_int, _f64p, _f32p, _i32p, ctypes.c_int]
        L.oracle_prepare.argtypes = [_u8p, ctypes.c_int, ctypes.c_int, _u8p, _f32p, _f32p, _f32p]
        L.oracle_pool.argtypes = [_u8p, ctypes.c_int, ctypes.c_int, _u8p, ctypes.c_int, ctypes.c_int,
                                  _i32p, _i32p, _f32p, _f64p]
        L.oracle_solve_nodes.argtypes = [ctypes.c_int, _u8p, _u8p, ctypes.c_int, ctypes.c_int, _u8p,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         _i32p, _f32p, _i32p, _f32p, _i32p]
        L.oracle_median_vsg.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        _f32p, _f32p, _u8p, _f32p]
        L.oracle_vsg_window_node_count.argtypes = [ctypes.c_int, ctypes.c_int]
        L.oracle_corpus.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, _f32p, ctypes.c_int]
        L.oracle_ff_inputs.argtypes = [ctypes.c_int, _u8p, _u8p]
        _lib = L
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


class Oracle:
    """One reference cache (ReferenceCache) of the restatement."""

    def __init__(self, fp64: bool = False):
        self._h = lib().oracle_create(1 if fp64 else 0)

    def close(self):
        if self._h:
            lib().oracle_destroy(self._h)
            self._h = None

    __del__ = close

    def set_reference(self, gray: np.ndarray, mask: np.ndarray | None = None) -> int:
        gray = np.ascontiguousarray(gray, np.uint8)
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        return lib().oracle_set_reference(self._h, _p(gray, _u8p), gray.shape[1], gray.shape[0], _p(m, _u8p))

    def run(self, deformed: np.ndarray, params, capacity: int | None = None, mask=None, model_h=None,
            metrics_len: int = 24, capture: bool = False):
        d = np.ascontiguousarray(deformed, np.uint8)
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        p = np.asarray(params, np.int32)
        gw, gh = max(p[2] // max(p[4], 1), 1), max(p[3] // max(p[4], 1), 1)
        if capacity is None:
            capacity = int(gw * gh * 8)
        out = np.zeros(max(capacity, 1), np.float32)
        met = np.zeros(max(metrics_len, 1), np.float32)
        H = None if model_h is None else np.ascontiguousarray(model_h, np.float64).reshape(9)
        if not capture:
            rc = lib().oracle_run(self._h, _p(d, _u8p), _p(m, _u8p), _p(p, _i32p), _p(out, _f32p),
                                  capacity, _p(met, _f32p), metrics_len, _p(H, _f64p))
            pts = out[: max(rc, 0) * 8].reshape(-1, 8).copy()
            return rc, pts, met[:metrics_len].copy()
        n = int(gw * gh) + 16
        gf = np.zeros((n, 7), np.float32)
        gi = np.zeros((n, 4), np.int32)
        rc = lib().oracle_run_capture(self._h, _p(d, _u8p), _p(m, _u8p), _p(p, _i32p), _p(out, _f32p),
                                      capacity, _p(met, _f32p), metrics_len, _p(H, _f64p),
                                      _p(gf, _f32p), _p(gi, _i32p), n)
        pts = out[: max(rc, 0) * 8].reshape(-1, 8).copy()
        return rc, pts, met[:metrics_len].copy(), gf, gi


def prepare(gray, mask=None):
    gray = np.ascontiguousarray(gray, np.uint8)
    h, w = gray.shape
    I = np.zeros((h, w), np.float32)
    gx = np.zeros((h, w), np.float32)
    gy = np.zeros((h, w), np.float32)
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    lib().oracle_prepare(_p(gray, _u8p), w, h, _p(m, _u8p), _p(I, _f32p), _p(gx, _f32p), _p(gy, _f32p))
    return I, gx, gy


def pool(gray, xy, dim, mask=None):
    gray = np.ascontiguousarray(gray, np.uint8)
    h, w = gray.shape
    xy = np.ascontiguousarray(xy, np.int32).reshape(-1, 2)
    n = xy.shape[0]
    valid = np.zeros(n, np.int32)
    ms = np.zeros((n, 2), np.float32)
    H = np.zeros((n, 21), np.float64)
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    lib().oracle_pool(_p(gray, _u8p), w, h, _p(m, _u8p), dim, n, _p(xy, _i32p), _p(valid, _i32p),
                      _p(ms, _f32p), _p(H, _f64p))
    return valid, ms, H


def solve_nodes(ref, dfm, xy, guess, mode, dim, lm=True, six=False, mask=None, fp64=False):
    ref = np.ascontiguousarray(ref, np.uint8)
    dfm = np.ascontiguousarray(dfm, np.uint8)
    h, w = ref.shape
    xy = np.ascontiguousarray(xy, np.int32).reshape(-1, 2)
    n = xy.shape[0]
    guess = np.ascontiguousarray(guess, np.float32).reshape(n, 6)
    mode = np.ascontiguousarray(np.broadcast_to(np.asarray(mode, np.int32), (n,)))
    fout = np.zeros((n, 7), np.float32)
    iout = np.zeros((n, 6), np.int32)
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    lib().oracle_solve_nodes(1 if fp64 else 0, _p(ref, _u8p), _p(dfm, _u8p), w, h, _p(m, _u8p), dim,
                             1 if lm else 0, 1 if six else 0, n, _p(xy, _i32p), _p(guess, _f32p),
                             _p(mode, _i32p), _p(fout, _f32p), _p(iout, _i32p))
    return fout, iout


def median_vsg(u, v, valid, step, window):
    gh, gw = u.shape
    u = np.ascontiguousarray(u, np.float32)
    v = np.ascontiguousarray(v, np.float32)
    val = np.ascontiguousarray(valid, np.uint8).copy()
    strain = np.zeros((gh, gw, 3), np.float32)
    rej = lib().oracle_median_vsg(gw, gh, step, window, _p(u, _f32p), _p(v, _f32p), _p(val, _u8p),
                                  _p(strain, _f32p))
    return rej, val, strain


def vsg_window_node_count(step, window):
    return lib().oracle_vsg_window_node_count(step, window)


def corpus(use6: bool, fp64: bool = False):
    n = 1024
    ixy = np.zeros((n, 3), np.int32)
    vals = np.zeros((n, 7), np.float32)
    cnt = lib().oracle_corpus(1 if use6 else 0, 1 if fp64 else 0, _p(ixy, _i32p), _p(vals, _f32p), n)
    return ixy[:cnt].copy(), vals[:cnt].copy()


def ff_inputs(scenario: int):
    ref = np.zeros((320, 320), np.uint8)
    dfm = np.zeros((320, 320), np.uint8)
    lib().oracle_ff_inputs(scenario, _p(ref, _u8p), _p(dfm, _u8p))
    return ref, dfm
