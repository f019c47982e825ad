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
# The same restatement built with the reference's own compiler flags: timed as
# the CPU baseline, never used to check results bit for bit.
_REFFLAGS_PATH = os.path.join(_HERE, "_build", "liboracle_refflags.so")
_SYNTH_PATH = os.path.join(_HERE, "_build", "liboracle_synth.so")
_lib = None
_libs = {}

_u8p = ctypes.POINTER(ctypes.c_uint8)
_i32p = ctypes.POINTER(ctypes.c_int32)
_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)


def build() -> str:
    """Compile the restatement (make, in-tree) and return the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib(kind: str = "contract"):
    """The restatement library: kind "contract" (the checker, strict IEEE
    arithmetic mirroring the device) or "reference_flags" (the timing build)."""
    global _lib
    if kind == "contract" and _lib is not None:
        return _lib
    if kind in _libs:
        return _libs[kind]
    path = {"contract": _LIB_PATH, "reference_flags": _REFFLAGS_PATH}[kind]
    if True:
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.oracle_create.restype = ctypes.c_void_p
        L.oracle_create.argtypes = [ctypes.c_int]
        L.oracle_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_set_reference.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_int, ctypes.c_int, _u8p]
        L.oracle_run.argtypes = [ctypes.c_void_p, _u8p, _u8p, _i32p, _f32p, ctypes.c_int, _f32p,
                                 ctypes.c_int, _f64p]
        L.oracle_run_guided.argtypes = [ctypes.c_void_p, _u8p, _u8p, _i32p, _f32p, ctypes.c_int, _f32p,
                                        ctypes.c_int, _f64p, _f32p, ctypes.c_int]
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
        L.oracle_inc_create.restype = ctypes.c_void_p
        L.oracle_inc_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_inc_init.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_int, ctypes.c_int, _u8p, _i32p, ctypes.c_int]
        L.oracle_inc_process.argtypes = [ctypes.c_void_p, _u8p, _f32p, ctypes.c_int, _f32p, ctypes.c_int, _i32p]
        field = [ctypes.c_int] * 5 + [_f32p] * 7 + [_u8p]
        L.oracle_inc_sample.argtypes = field + [ctypes.c_float, ctypes.c_float, _f32p]
        L.oracle_inc_fit.argtypes = field + [ctypes.c_float, ctypes.c_float, ctypes.c_float, _f32p]
        L.oracle_inc_anchor_need.argtypes = field + [ctypes.c_float, ctypes.c_float, ctypes.c_int]
        L.oracle_inc_node_field.argtypes = [ctypes.c_int, ctypes.c_int, _f32p, _f32p, _f32p, _u8p, _u8p]
        L.oracle_inc_warp_mask.argtypes = [_u8p, ctypes.c_int, ctypes.c_int] + [ctypes.c_int] * 5 + \
            [_f32p, _f32p, _u8p, ctypes.c_int, _u8p]
        L.oracle_inc_match.argtypes = [_u8p, _u8p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                       ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float, _f32p]
        _libs[kind] = L
        if kind == "contract":
            _lib = L
    return L


def synth_path() -> str:
    """Path of the oracle-side build of the seeded speckle generator (the same
    C ABI as the package's synth library), for a CPU-only caller that loads no
    library of the package."""
    if not os.path.exists(_SYNTH_PATH):
        build()
    return _SYNTH_PATH


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


class Oracle:
    """One reference cache (ReferenceCache) of the restatement."""

    def __init__(self, fp64: bool = False, kind: str = "contract"):
        self._L = lib(kind)
        self._h = self._L.oracle_create(1 if fp64 else 0)

    def close(self):
        if getattr(self, "_h", None):
            self._L.oracle_destroy(self._h)
            self._h = None

    __del__ = close

    def set_reference(self, gray: np.ndarray, mask: np.ndarray | None = None) -> int:
        gray = np.ascontiguousarray(gray, np.uint8)
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        return self._L.oracle_set_reference(self._h, _p(gray, _u8p), gray.shape[1], gray.shape[0], _p(m, _u8p))

    def run(self, deformed: np.ndarray, params, capacity: int | None = None, mask=None, model_h=None,
            metrics_len: int = 24, capture: bool = False, anchor_uv=None):
        """run_full_field. anchor_uv ([n][2] float32, NaN for none): per
        anchor-lattice node displacement guesses under model_h."""
        d = np.ascontiguousarray(deformed, np.uint8)
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        p = np.asarray(params, np.int32)
        gw, gh = max(p[2] // max(p[4], 1), 1), max(p[3] // max(p[4], 1), 1)
        if capacity is None:
            capacity = int(gw * gh * 8)
        out = np.zeros(max(capacity, 1), np.float32)
        met = np.zeros(max(metrics_len, 1), np.float32)
        H = None if model_h is None else np.ascontiguousarray(model_h, np.float64).reshape(9)
        if anchor_uv is not None:
            g = np.ascontiguousarray(anchor_uv, np.float32).reshape(-1, 2)
            rc = self._L.oracle_run_guided(self._h, _p(d, _u8p), _p(m, _u8p), _p(p, _i32p), _p(out, _f32p),
                                           capacity, _p(met, _f32p), metrics_len, _p(H, _f64p), _p(g, _f32p),
                                           g.shape[0])
            pts = out[: max(rc, 0) * 8].reshape(-1, 8).copy()
            return rc, pts, met[:metrics_len].copy()
        if not capture:
            rc = self._L.oracle_run(self._h, _p(d, _u8p), _p(m, _u8p), _p(p, _i32p), _p(out, _f32p),
                                  capacity, _p(met, _f32p), metrics_len, _p(H, _f64p))
            pts = out[: max(rc, 0) * 8].reshape(-1, 8).copy()
            return rc, pts, met[:metrics_len].copy()
        n = int(gw * gh) + 16
        gf = np.zeros((n, 7), np.float32)
        gi = np.zeros((n, 4), np.int32)
        rc = self._L.oracle_run_capture(self._h, _p(d, _u8p), _p(m, _u8p), _p(p, _i32p), _p(out, _f32p),
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


# ------------------------------------------------------------------ incremental
class IncrementalOracle:
    """The incremental session over the restatement (oracle/src/incremental.hpp)."""

    def __init__(self):
        self._h = lib().oracle_inc_create()

    def close(self):
        if self._h:
            lib().oracle_inc_destroy(self._h)
            self._h = None

    __del__ = close

    def init(self, ref, params, update_interval: int, mask=None) -> int:
        g = np.ascontiguousarray(ref, np.uint8)
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        p = np.asarray(params, np.int32)
        return lib().oracle_inc_init(self._h, _p(g, _u8p), g.shape[1], g.shape[0], _p(m, _u8p), _p(p, _i32p),
                                     update_interval)

    def process(self, frame, capacity: int, metrics_len: int = 24):
        d = np.ascontiguousarray(frame, np.uint8)
        out = np.zeros(max(capacity, 1), np.float32)
        met = np.zeros(max(metrics_len, 1), np.float32)
        info = np.zeros(6, np.int32)
        rc = lib().oracle_inc_process(self._h, _p(d, _u8p), _p(out, _f32p), capacity, _p(met, _f32p), metrics_len,
                                      _p(info, _i32p))
        return rc, out[: max(rc, 0) * 8].reshape(-1, 8).copy(), met[:metrics_len].copy(), info


class NodeField:
    """A lattice for the incremental math entries: (gw, gh, rx, ry, step) and per-node arrays."""

    def __init__(self, gw, gh, rx, ry, step):
        self.geom = (gw, gh, rx, ry, step)
        n = gw * gh
        self.u, self.v = np.zeros(n, np.float32), np.zeros(n, np.float32)
        self.ux, self.uy = np.zeros(n, np.float32), np.zeros(n, np.float32)
        self.vx, self.vy = np.zeros(n, np.float32), np.zeros(n, np.float32)
        self.corr = np.zeros(n, np.float32)
        self.valid = np.ones(n, np.uint8)

    def node(self, i, j):
        gw, gh, rx, ry, step = self.geom
        return float(rx + i * step), float(ry + j * step)

    def _args(self):
        return list(self.geom) + [_p(a, _f32p) for a in (self.u, self.v, self.ux, self.uy, self.vx, self.vy,
                                                          self.corr)] + [_p(self.valid, _u8p)]


def inc_sample(f: NodeField, x, y):
    r = np.zeros(4, np.float32)
    ok = lib().oracle_inc_sample(*f._args(), x, y, _p(r, _f32p))
    return bool(ok), float(r[0]), float(r[1]), float(r[2]), bool(r[3])


def inc_fit(f: NodeField, x, y, radius):
    r = np.zeros(3, np.float32)
    ok = lib().oracle_inc_fit(*f._args(), x, y, radius, _p(r, _f32p))
    return bool(ok), float(r[0]), float(r[1]), float(r[2])


def inc_anchor_need(f: NodeField, x, y, subset):
    return ["drop", "refresh", "keep"][lib().oracle_inc_anchor_need(*f._args(), x, y, subset)]


def inc_node_field(u, v, corr, solved):
    gh, gw = u.shape
    out = np.zeros(gw * gh, np.uint8)
    arrs = [np.ascontiguousarray(a, np.float32).ravel() for a in (u, v, corr)]
    s = np.ascontiguousarray(solved, np.uint8).ravel()
    rej = lib().oracle_inc_node_field(gw, gh, _p(arrs[0], _f32p), _p(arrs[1], _f32p), _p(arrs[2], _f32p),
                                      _p(s, _u8p), _p(out, _u8p))
    return out.reshape(gh, gw), rej


def inc_warp_mask(mask0, geom, U, V, valid, margin):
    m = np.ascontiguousarray(mask0, np.uint8)
    H, W = m.shape
    out = np.zeros_like(m)
    U = np.ascontiguousarray(U, np.float32).ravel()
    V = np.ascontiguousarray(V, np.float32).ravel()
    valid = np.ascontiguousarray(valid, np.uint8).ravel()
    lib().oracle_inc_warp_mask(_p(m, _u8p), W, H, *geom, _p(U, _f32p), _p(V, _f32p), _p(valid, _u8p), margin,
                               _p(out, _u8p))
    return out


def inc_match(ref, dfm, x, y, subset, gx, gy, max_shift):
    """make_anchor on ref at (x, y) and match_anchor on dfm. Returns (rc, x, y, corr, ax, ay, dx, dy); rc -1
    when no anchor is cut."""
    r = np.ascontiguousarray(ref, np.uint8)
    d = np.ascontiguousarray(dfm, np.uint8)
    out = np.full(7, -1.0, np.float32)
    rc = lib().oracle_inc_match(_p(r, _u8p), _p(d, _u8p), r.shape[1], r.shape[0], x, y, subset, gx, gy, max_shift,
                                _p(out, _f32p))
    return (rc,) + tuple(float(v) for v in out)
