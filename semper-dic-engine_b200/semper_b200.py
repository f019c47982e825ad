"""Python binding of libsemper_b200.so (ctypes) and of the speckle generator.

The engine is the C ABI of include/semper_c.h; the stage entries are the
kernel-level C ABI of include/semper_dic_cuda.h, here driven with torch device
tensors. Nothing in this module computes on the CPU: a missing library, or a
machine without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# The full library (C ABI, extensions, stage ABI, C++ API). libsemper_c.so is
# the same code exporting only the reference's eleven C-ABI symbols.
LIB_PATH = os.path.join(HERE, "lib", "libsemper_b200.so")
C_LIB_PATH = os.path.join(HERE, "lib", "libsemper_c.so")
SYNTH_PATH = os.path.join(HERE, "lib", "libsemper_synth.so")

_u8p = ctypes.POINTER(ctypes.c_uint8)
_i32p = ctypes.POINTER(ctypes.c_int32)
_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p

SEMPER_ERR_ROI, SEMPER_ERR_INIT, SEMPER_ERR_STRAIN_WINDOW, SEMPER_ERR_SEED, SEMPER_ERR_CANCELLED = -2, -3, -4, -5, -99
INIT_AUTO_SEARCH, INIT_NO_SEARCH, INIT_NO_SIMPLEX = 0, 1, 2

TASK_DT = np.dtype([("node", "<i4"), ("cx", "<i4"), ("cy", "<i4"), ("mode", "<i4"), ("g", "<f4", (6,))])
RESULT_DT = np.dtype([("p", "<f4", (7,)), ("status", "<i4"), ("iters", "<i4"), ("trigger_iters", "<i4"),
                      ("invalid_ref", "<i4"), ("flags", "<i4")])
assert TASK_DT.itemsize == 40 and RESULT_DT.itemsize == 48

C_SYMBOLS = ["semper_cancel", "semper_create", "semper_destroy", "semper_incremental_cancel",
             "semper_incremental_create", "semper_incremental_destroy", "semper_incremental_init",
             "semper_incremental_process", "semper_run", "semper_set_reference", "semper_version"]
EXT_SYMBOLS = ["semper_b200_last_timings", "semper_b200_run_device", "semper_b200_set_global_model",
               "semper_b200_stream", "semper_b200_set_global_motion", "semper_b200_last_global_motion",
               "semper_b200_batch_create", "semper_b200_batch_destroy", "semper_b200_batch_run",
               "semper_b200_batch_last_error", "semper_b200_incremental_profile", "semper_b200_fast_pass_shape",
               "semper_b200_set_tma_wait_limit", "semper_b200_last_tma_timeout",
               "semper_b200_proposal_create", "semper_b200_proposal_destroy", "semper_b200_proposal_param_count",
               "semper_b200_proposal_set_params", "semper_b200_proposal_get_params", "semper_b200_proposal_forward",
               "semper_b200_proposal_gradients", "semper_b200_proposal_synth", "semper_b200_proposal_train",
               "semper_b200_proposal_predict_warped",
               "semper_b200_set_proposal", "semper_b200_last_learned", "semper_b200_learned_guesses",
               "semper_b200_inc_batch_create", "semper_b200_inc_batch_destroy", "semper_b200_inc_batch_init",
               "semper_b200_inc_batch_process", "semper_b200_batch_create_on", "semper_b200_inc_batch_create_on"]
DIC_SYMBOLS = ["dic_cuda_image_prep", "dic_cuda_grid_scan", "dic_cuda_hessian_pool", "dic_cuda_solve",
               "dic_cuda_solve_scratch_bytes",
               "dic_cuda_median_pass", "dic_cuda_clear_failed", "dic_cuda_vsg", "dic_cuda_pack_scratch_bytes",
               "dic_cuda_pack"]


class SemperParams(ctypes.Structure):
    _fields_ = [("rect_x", ctypes.c_int32), ("rect_y", ctypes.c_int32), ("rect_w", ctypes.c_int32),
                ("rect_h", ctypes.c_int32), ("step", ctypes.c_int32), ("subset_size", ctypes.c_int32),
                ("strain_window", ctypes.c_int32), ("use_6x6_interpolator", ctypes.c_int32)]


class IncrementalInfo(ctypes.Structure):
    _fields_ = [("reference_frame", ctypes.c_int32), ("reference_updated", ctypes.c_int32),
                ("tracked_points", ctypes.c_int32), ("frame0_points", ctypes.c_int32),
                ("taylor_fallbacks", ctypes.c_int32), ("lost_this_frame", ctypes.c_int32)]


class IncFrame(ctypes.Structure):
    """semper_b200_inc_frame (include/semper_b200_ext.h)."""


class BatchJob(ctypes.Structure):
    """semper_b200_job (include/semper_b200_ext.h)."""
    _fields_ = [("reference", ctypes.c_void_p), ("deformed", ctypes.c_void_p), ("mask", ctypes.c_void_p),
                ("width", ctypes.c_int32), ("height", ctypes.c_int32), ("params", SemperParams),
                ("out", ctypes.c_void_p), ("out_capacity", ctypes.c_int32), ("metrics", ctypes.c_void_p),
                ("metrics_len", ctypes.c_int32), ("result", ctypes.c_int32)]


IncFrame._fields_ = [("sequence", ctypes.c_int32), ("frame", ctypes.c_void_p), ("out", ctypes.c_void_p),
                     ("out_capacity", ctypes.c_int32), ("metrics", ctypes.c_void_p), ("metrics_len", ctypes.c_int32),
                     ("info", IncrementalInfo), ("result", ctypes.c_int32)]

PROGRESS_CB = ctypes.CFUNCTYPE(None, ctypes.c_int, ctypes.c_void_p)

_lib = None
_synth = None


def build() -> None:
    """Compile the library in-tree (make; nvcc for sm_100a)."""
    subprocess.run(["make", "-s", "-j8", "-C", HERE], check=True)


def lib():
    """The loaded libsemper_c.so (raises if it is absent and cannot be built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.semper_create.restype = _vp
        L.semper_destroy.argtypes = [_vp]
        L.semper_set_reference.argtypes = [_vp, _u8p, ctypes.c_size_t, _u8p, ctypes.c_size_t, ctypes.c_int,
                                           ctypes.c_int]
        L.semper_run.argtypes = [_vp, _u8p, ctypes.c_size_t, _u8p, ctypes.c_size_t, ctypes.POINTER(SemperParams),
                                 _f32p, ctypes.c_int, _f32p, ctypes.c_int, PROGRESS_CB, _vp]
        L.semper_cancel.argtypes = [_vp]
        L.semper_version.restype = ctypes.c_char_p
        L.semper_incremental_create.restype = _vp
        L.semper_incremental_destroy.argtypes = [_vp]
        L.semper_incremental_init.argtypes = [_vp, _u8p, ctypes.c_size_t, _u8p, ctypes.c_size_t, ctypes.c_int,
                                              ctypes.c_int, ctypes.POINTER(SemperParams), ctypes.c_int32]
        L.semper_incremental_process.argtypes = [_vp, _u8p, ctypes.c_size_t, _f32p, ctypes.c_int, _f32p,
                                                 ctypes.c_int, ctypes.POINTER(IncrementalInfo), PROGRESS_CB, _vp]
        L.semper_incremental_cancel.argtypes = [_vp]
        L.semper_b200_run_device.argtypes = [_vp, _vp, ctypes.POINTER(SemperParams), _vp, ctypes.c_int, _f32p,
                                             ctypes.c_int]
        L.semper_b200_stream.argtypes = [_vp]
        L.semper_b200_stream.restype = _vp
        L.semper_b200_last_timings.argtypes = [_vp, _f32p, ctypes.POINTER(ctypes.c_longlong)]
        L.semper_b200_set_global_model.argtypes = [_vp, _f64p]
        L.semper_b200_fast_pass_shape.argtypes = [_vp, ctypes.c_int, ctypes.c_int]
        L.semper_b200_set_global_motion.argtypes = [_vp, ctypes.c_int]
        L.semper_b200_proposal_create.argtypes = [ctypes.c_int32]
        L.semper_b200_proposal_create.restype = _vp
        L.semper_b200_proposal_destroy.argtypes = [_vp]
        L.semper_b200_proposal_param_count.restype = ctypes.c_int64
        L.semper_b200_proposal_set_params.argtypes = [_vp, _f32p, ctypes.c_int64]
        L.semper_b200_proposal_get_params.argtypes = [_vp, _f32p, ctypes.c_int64]
        L.semper_b200_proposal_forward.argtypes = [_vp, _f32p, ctypes.c_int32, _f32p]
        L.semper_b200_proposal_gradients.argtypes = [_vp, _f32p, _f32p, ctypes.c_int32, _f32p, _f32p]
        L.semper_b200_proposal_synth.argtypes = [_vp, _u8p, ctypes.c_int32, ctypes.c_int32, _f32p, ctypes.c_uint64,
                                                 ctypes.c_int32, _f32p, _f32p]
        L.semper_b200_proposal_train.argtypes = [_vp, _u8p, ctypes.c_int32, ctypes.c_int32, _f32p, ctypes.c_int32,
                                                 ctypes.c_int32, ctypes.c_float, ctypes.c_uint64, _f32p]
        L.semper_b200_proposal_predict_warped.argtypes = [_vp, _u8p, _u8p, ctypes.c_int32, ctypes.c_int32, _f32p,
                                                          ctypes.c_int32, ctypes.c_int32, _f32p]
        L.semper_b200_set_proposal.argtypes = [_vp, _vp, ctypes.c_int]
        L.semper_b200_learned_guesses.argtypes = [_vp, _f32p, ctypes.c_int32]
        L.semper_b200_last_learned.argtypes = [_vp, _f64p]
        L.semper_b200_set_tma_wait_limit.argtypes = [_vp, ctypes.c_int]
        L.semper_b200_last_tma_timeout.argtypes = [_vp]
        L.semper_b200_batch_create.argtypes = [ctypes.c_int32]
        L.semper_b200_batch_create.restype = _vp
        L.semper_b200_batch_destroy.argtypes = [_vp]
        L.semper_b200_batch_run.argtypes = [_vp, ctypes.POINTER(BatchJob), ctypes.c_int32]
        L.semper_b200_incremental_profile.argtypes = [_vp, _f64p]
        L.semper_b200_inc_batch_create.argtypes = [ctypes.c_int32]
        L.semper_b200_inc_batch_create.restype = _vp
        L.semper_b200_inc_batch_create_on.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32]
        L.semper_b200_inc_batch_create_on.restype = _vp
        L.semper_b200_batch_create_on.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32]
        L.semper_b200_batch_create_on.restype = _vp
        L.semper_b200_inc_batch_destroy.argtypes = [_vp]
        L.semper_b200_inc_batch_init.argtypes = [_vp, ctypes.c_int32, _u8p, _u8p, ctypes.c_int32, ctypes.c_int32,
                                                 ctypes.POINTER(SemperParams), ctypes.c_int32]
        L.semper_b200_inc_batch_process.argtypes = [_vp, ctypes.POINTER(IncFrame), ctypes.c_int32]
        L.semper_b200_batch_last_error.argtypes = [_vp]
        L.semper_b200_batch_last_error.restype = ctypes.c_char_p
        L.semper_b200_last_global_motion.argtypes = [_vp, _f64p]
        L.dic_cuda_image_prep.argtypes = [_vp] * 2 + [ctypes.c_int] * 3 + [_vp] * 4
        L.dic_cuda_grid_scan.argtypes = [_vp] + [ctypes.c_int] * 8 + [_vp, _vp, _vp]
        L.dic_cuda_hessian_pool.argtypes = [_vp] * 3 + [ctypes.c_int] * 3 + [_vp] + [ctypes.c_int] * 7 + [_vp] * 5
        L.dic_cuda_solve.argtypes = [_vp] * 4 + [ctypes.c_int] * 3 + [_vp] * 3 + [ctypes.c_int] * 3 + \
            [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp]
        L.dic_cuda_solve_scratch_bytes.argtypes = [ctypes.c_int]
        L.dic_cuda_solve_scratch_bytes.restype = ctypes.c_size_t
        L.dic_cuda_median_pass.argtypes = [ctypes.c_int] * 2 + [_vp] * 6
        L.dic_cuda_clear_failed.argtypes = [ctypes.c_int, _vp, _vp, _vp]
        L.dic_cuda_vsg.argtypes = [ctypes.c_int] * 4 + [_vp] * 7
        L.dic_cuda_pack_scratch_bytes.argtypes = [ctypes.c_int]
        L.dic_cuda_pack_scratch_bytes.restype = ctypes.c_size_t
        L.dic_cuda_pack.argtypes = [ctypes.c_int] * 6 + [_vp] * 9 + [ctypes.c_size_t, _vp]
        _lib = L
    return _lib


def use_synth_library(path: str) -> None:
    """Generate speckle with another build of the same generator (same C ABI),
    e.g. the checker's own copy for a CPU-only caller; before the first use."""
    global SYNTH_PATH, _synth
    if _synth is not None:
        raise RuntimeError("the speckle generator is already loaded")
    SYNTH_PATH = path


def synth_lib():
    global _synth
    if _synth is None:
        if not os.path.exists(SYNTH_PATH):
            build()
        S = ctypes.CDLL(SYNTH_PATH)
        S.synth_speckle.argtypes = [_u8p, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, _f64p, ctypes.c_double, ctypes.c_uint64]
        S.synth_speckle.restype = ctypes.c_int
        S.synth_displacement.argtypes = [_f64p, ctypes.c_int, _f64p, _f64p, _f64p, _f64p]
        _synth = S
    return _synth


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def params(rect, step, subset, window, six=False) -> SemperParams:
    x, y, w, h = rect
    return SemperParams(x, y, w, h, step, subset, window, 1 if six else 0)


class Engine:
    """semper_engine: one reference cache on the GPU (semper_create ...)."""

    def __init__(self):
        self._h = lib().semper_create()
        if not self._h:
            raise RuntimeError("semper_create failed (no usable CUDA device?)")

    def close(self):
        h = getattr(self, "_h", None)
        self._h = None
        if h and _lib is not None:  # at interpreter exit the library may be gone already
            _lib.semper_destroy(h)

    __del__ = close

    def set_reference(self, gray: np.ndarray, mask: np.ndarray | None = None) -> int:
        g = np.ascontiguousarray(gray, np.uint8)
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        return lib().semper_set_reference(self._h, _p(g, _u8p), g.size, _p(m, _u8p), 0 if m is None else m.size,
                                          g.shape[1], g.shape[0])

    def set_reference_bytes(self, data: bytes, width: int, height: int) -> int:
        """semper_set_reference with a raw buffer as the reference's decoding
        takes it (width*height gray bytes, or 4*width*height RGBA)."""
        buf = np.frombuffer(data, np.uint8)
        return lib().semper_set_reference(self._h, _p(buf, _u8p), buf.size, None, 0, width, height)

    def run(self, deformed: np.ndarray, prm: SemperParams, capacity: int | None = None, mask=None,
            metrics_len: int = 24, progress=None, out: np.ndarray | None = None, copy: bool = True):
        """semper_run. `out` (float32, >= capacity) may be a caller buffer,
        e.g. pinned memory; the returned points are a copy, or with copy False
        a view of `out` (valid until `out` is reused)."""
        d = np.ascontiguousarray(deformed, np.uint8)
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        if capacity is None:
            capacity = max(prm.rect_w // max(prm.step, 1), 1) * max(prm.rect_h // max(prm.step, 1), 1) * 8
        if out is None:
            out = np.zeros(max(capacity, 1), np.float32)
        met = np.zeros(max(metrics_len, 1), np.float32)
        cb = PROGRESS_CB(progress) if progress else PROGRESS_CB()
        rc = lib().semper_run(self._h, _p(d, _u8p), d.size, _p(m, _u8p), 0 if m is None else m.size,
                              ctypes.byref(prm), _p(out, _f32p), capacity, _p(met, _f32p), metrics_len, cb, None)
        pts = out[: max(rc, 0) * 8].reshape(-1, 8)
        return rc, pts.copy() if copy else pts, met[:metrics_len].copy()

    def cancel(self):
        lib().semper_cancel(self._h)

    def run_device(self, d_def, prm: SemperParams, d_out, capacity: int, metrics_len: int = 24):
        """semper_b200_run_device: deformed frame and output are device tensors."""
        met = np.zeros(max(metrics_len, 1), np.float32)
        rc = lib().semper_b200_run_device(self._h, ctypes.c_void_p(d_def.data_ptr()), ctypes.byref(prm),
                                          ctypes.c_void_p(d_out.data_ptr()), capacity, _p(met, _f32p), metrics_len)
        return rc, met[:metrics_len].copy()

    def stream_handle(self) -> int:
        return lib().semper_b200_stream(self._h) or 0

    def last_timings(self):
        t = np.zeros(8, np.float32)
        c = (ctypes.c_longlong * 5)()
        lib().semper_b200_last_timings(self._h, _p(t, _f32p), c)
        names = ["prep", "pool", "seed", "mesh", "path_a", "path_b", "strain", "total"]
        counts = ["icgn_iters", "pixel_iters", "path_a_tasks", "path_a_pixel_iters", "launches"]
        return dict(zip(names, map(float, t))), dict(zip(counts, map(int, c)))

    def fast_pass_shape(self, subset_size: int, six: bool = False) -> int:
        """The Path A fast pass's shape the autotuner kept: 0 reference read
        from the planes, 1 staged in shared memory, -1 not decided yet."""
        return lib().semper_b200_fast_pass_shape(self._h, subset_size, 1 if six else 0)

    def set_global_model(self, H=None) -> int:
        Hm = None if H is None else np.ascontiguousarray(H, np.float64).reshape(9)
        return lib().semper_b200_set_global_model(self._h, _p(Hm, _f64p))

    def set_proposal(self, net, learned=True) -> int:
        """Learned seeding from `net` (a Proposal, kept alive by this engine).
        learned: True or 1, the proposal first; "rescue" or 2, the
        global-motion estimate first and the proposal only where it fails;
        False or 0, off."""
        self._proposal = net
        mode = 2 if learned == "rescue" else int(learned)
        return lib().semper_b200_set_proposal(self._h, None if net is None else net._h, mode)

    def last_learned(self) -> dict:
        o = np.zeros(18, np.float64)
        lib().semper_b200_last_learned(self._h, _p(o, _f64p))
        return {"ran": bool(o[0]), "proposed": bool(o[1]), "kept": bool(o[2]), "pairs": int(o[3]),
                "inliers": int(o[4]), "anchors": int(o[5]), "err_mean_px": float(o[6]), "err_max_px": float(o[7]),
                "ms": float(o[8]), "H": o[9:18].reshape(3, 3).copy()}

    def learned_guesses(self) -> np.ndarray:
        """[n][2] displacement guesses per anchor-lattice node of the last
        learned seeding (NaN where none; empty when it did not run)."""
        n = lib().semper_b200_learned_guesses(self._h, None, 0)
        out = np.zeros((max(n, 0), 2), np.float32)
        if n > 0:
            lib().semper_b200_learned_guesses(self._h, _p(out, _f32p), 2 * n)
        return out

    def set_tma_wait_limit(self, polls: int) -> int:
        return lib().semper_b200_set_tma_wait_limit(self._h, polls)

    def last_tma_timeout(self) -> int:
        return lib().semper_b200_last_tma_timeout(self._h)

    def set_global_motion(self, on: bool) -> int:
        return lib().semper_b200_set_global_motion(self._h, 1 if on else 0)

    def last_global_motion(self) -> dict:
        """The similarity the last run estimated (semper_b200_last_global_motion)."""
        o = np.zeros(18, np.float64)
        lib().semper_b200_last_global_motion(self._h, _p(o, _f64p))
        return {"locked": bool(o[0]), "theta": o[1], "scale": o[2], "t": (o[3], o[4]), "centre": (o[5], o[6]),
                "peaks": (o[7], o[8]), "H": o[9:].reshape(3, 3).copy()}


# The proposal network's trained weights (train_proposal.py), shipped with the package.
PROPOSAL_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "proposal.npy")


class Proposal:
    """The learned seed proposal network (semper_b200_proposal_*): two 64x64
    patches -> the affine map between them, on BF16 tensor-core kernels."""

    def __init__(self, max_batch: int = 256):
        self._h = lib().semper_b200_proposal_create(max_batch)
        if not self._h:
            raise RuntimeError("semper_b200_proposal_create failed")
        self.max_batch = max_batch

    @classmethod
    def trained(cls, max_batch: int = 256, path: str | None = None) -> "Proposal":
        """A network with the shipped trained weights (or those at `path`)."""
        net = cls(max_batch)
        net.set_params(np.load(path or PROPOSAL_WEIGHTS))
        return net

    def close(self):
        h = getattr(self, "_h", None)
        self._h = None
        if h and _lib is not None:
            _lib.semper_b200_proposal_destroy(h)

    __del__ = close

    @staticmethod
    def param_count() -> int:
        return int(lib().semper_b200_proposal_param_count())

    def set_params(self, flat: np.ndarray):
        f = np.ascontiguousarray(flat, np.float32)
        _ck(lib().semper_b200_proposal_set_params(self._h, _p(f, _f32p), f.size), "proposal params")

    def get_params(self) -> np.ndarray:
        f = np.zeros(self.param_count(), np.float32)
        _ck(lib().semper_b200_proposal_get_params(self._h, _p(f, _f32p), f.size), "proposal params")
        return f

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        out = np.zeros((x.shape[0], 6), np.float32)
        _ck(lib().semper_b200_proposal_forward(self._h, _p(x, _f32p), x.shape[0], _p(out, _f32p)), "forward")
        return out

    def gradients(self, x: np.ndarray, target: np.ndarray):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(target, np.float32)
        g = np.zeros(self.param_count(), np.float32)
        loss = np.zeros(1, np.float32)
        _ck(lib().semper_b200_proposal_gradients(self._h, _p(x, _f32p), _p(t, _f32p), x.shape[0], _p(g, _f32p),
                                                 _p(loss, _f32p)), "gradients")
        return float(loss[0]), g

    def synth(self, speckle: np.ndarray, cfg, seed: int, batch: int):
        s = np.ascontiguousarray(speckle, np.uint8)
        c = np.asarray(cfg, np.float32)
        x = np.zeros((batch, 64, 64, 2), np.float32)
        t = np.zeros((batch, 6), np.float32)
        _ck(lib().semper_b200_proposal_synth(self._h, _p(s, _u8p), s.shape[1], s.shape[0], _p(c, _f32p), seed, batch,
                                             _p(x, _f32p), _p(t, _f32p)), "synth")
        return x, t

    def train(self, speckle: np.ndarray, cfg, steps: int, batch: int, lr: float, seed: int) -> np.ndarray:
        s = np.ascontiguousarray(speckle, np.uint8)
        c = np.asarray(cfg, np.float32)
        losses = np.zeros(max(steps, 1), np.float32)
        _ck(lib().semper_b200_proposal_train(self._h, _p(s, _u8p), s.shape[1], s.shape[0], _p(c, _f32p), steps, batch,
                                             lr, seed, _p(losses, _f32p)), "train")
        return losses[:steps]

    def predict_warped(self, ref: np.ndarray, dfm: np.ndarray, maps: np.ndarray, f: int) -> np.ndarray:
        """Residual maps [K, 6] for pairs cut from two u8 frames, the second
        patch of each sampled through maps[k] = (cx, cy, a00, a01, a10, a11,
        bx, by) (semper_b200_proposal_predict_warped)."""
        r = np.ascontiguousarray(ref, np.uint8)
        d = np.ascontiguousarray(dfm, np.uint8)
        m = np.ascontiguousarray(maps, np.float32).reshape(-1, 8)
        out = np.zeros((m.shape[0], 6), np.float32)
        _ck(lib().semper_b200_proposal_predict_warped(self._h, _p(r, _u8p), _p(d, _u8p), r.shape[1], r.shape[0],
                                                      _p(m, _f32p), m.shape[0], f, _p(out, _f32p)), "predict_warped")
        return out


class Batch:
    """semper_b200_batch: independent pairs solved concurrently."""

    def __init__(self, workers: int = 8, devices=None):
        """devices: GPU ordinals the workers spread over (None: the current one)."""
        if devices:
            dv = (ctypes.c_int32 * len(devices))(*devices)
            self._h = lib().semper_b200_batch_create_on(workers, dv, len(devices))
        else:
            self._h = lib().semper_b200_batch_create(workers)
        if not self._h:
            raise RuntimeError("semper_b200_batch_create failed")

    def close(self):
        h = getattr(self, "_h", None)
        self._h = None
        if h and _lib is not None:  # at interpreter exit the library may be gone already
            _lib.semper_b200_batch_destroy(h)

    __del__ = close

    def run(self, jobs, metrics_len: int = 24):
        """jobs: dicts with ref, dfm, prm and optionally mask and capacity.
        Returns one (rc, points, metrics) per job, in the jobs' order."""
        keep, arr = [], (BatchJob * max(len(jobs), 1))()
        outs = []
        for k, j in enumerate(jobs):
            ref = np.ascontiguousarray(j["ref"], np.uint8)
            dfm = np.ascontiguousarray(j["dfm"], np.uint8)
            m = j.get("mask")
            m = None if m is None else np.ascontiguousarray(m, np.uint8)
            prm = j["prm"]
            cap = j.get("capacity")
            if cap is None:
                cap = max(prm.rect_w // max(prm.step, 1), 1) * max(prm.rect_h // max(prm.step, 1), 1) * 8
            # fresh per call and written by the library up to the point count,
            # so neither zeroed nor copied on the way out
            out = np.empty(max(cap, 1), np.float32)
            met = np.zeros(max(metrics_len, 1), np.float32)
            keep += [ref, dfm, m, out, met]
            outs.append((out, met))
            b = arr[k]
            b.reference, b.deformed = ref.ctypes.data, dfm.ctypes.data
            b.mask = None if m is None else m.ctypes.data
            b.height, b.width = ref.shape
            b.params = prm
            b.out, b.out_capacity = out.ctypes.data, cap
            b.metrics, b.metrics_len = met.ctypes.data, metrics_len
            b.result = 0
        rc = lib().semper_b200_batch_run(self._h, arr, len(jobs))
        if rc != 0:
            raise RuntimeError(f"semper_b200_batch_run returned {rc}")
        self.last_error = (lib().semper_b200_batch_last_error(self._h) or b"").decode()
        res = []
        for k, (out, met) in enumerate(outs):
            r = arr[k].result
            res.append((r, out[: max(r, 0) * 8].reshape(-1, 8), met[:metrics_len]))
        return res


def job_cost(prm) -> int:
    """A job's relative solve cost for sharding: grid nodes x subset pixels."""
    return (prm.rect_w // prm.step) * (prm.rect_h // prm.step) * prm.subset_size * prm.subset_size


def shard(costs, rank: int, world: int) -> list:
    """The indices of `costs` that rank `rank` of `world` takes: largest cost
    first, each to the least-loaded rank (the lowest rank on a tie). Every
    rank computes the same assignment, so the shards cover every index exactly
    once with no exchange between ranks."""
    if world <= 1:
        return list(range(len(costs)))
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0] * world
    mine = []
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += costs[i]
        if r == rank:
            mine.append(i)
    return sorted(mine)


def batch_job_params(n: int = 256, seed: int = 0, min_side: int = 256, max_side: int = 2048):
    """The params (and whether a mask comes with each) of batch_jobs(n, seed,
    ...) without generating any frame: [(params, has_mask)]."""
    return [(j["prm"], j["has_mask"]) for j in batch_jobs(n, seed, min_side, max_side, frames=False)]


def batch_jobs(n: int = 256, seed: int = 0, min_side: int = 256, max_side: int = 2048, only=None,
               frames: bool = True):
    """The batched uneven workload: n independent pairs, side ~ U{min_side..
    max_side} (square frames of seeded speckle as cfg0), each under its own
    affine warp (|rotation| <= 10 deg, stretch <= 3 % per axis, translation
    <= 8 px, about the frame centre) with noise sigma 1, and its own random
    circular holes in the mask (1-3 discs removing a fraction ~ U[0, 0.4] of
    the frame); per pair subset ~ {15, 21, 31, 41}, step ~ {4, 8},
    strain window = subset, the whole frame as ROI. `only`: the job indices
    to build (a shard; every job is drawn the same either way), in index
    order; `frames` False skips the frames and masks (params only)."""
    rng = np.random.default_rng(9000 + seed)
    keep = None if only is None else set(only)
    jobs = []
    for k in range(n):
        side = int(rng.integers(min_side, max_side + 1))
        th = np.radians(rng.uniform(-10.0, 10.0))
        sx, sy = 1.0 + rng.uniform(-0.03, 0.03), 1.0 + rng.uniform(-0.03, 0.03)
        c, s_ = np.cos(th), np.sin(th)
        a = (c * sx - 1.0, -s_ * sy, s_ * sx, c * sy - 1.0)
        t = rng.uniform(-8.0, 8.0, 2)
        warp = warp_block(cx=side / 2, cy=side / 2, u0=t[0], v0=t[1], a=a)
        frac = rng.uniform(0.0, 0.4)
        nd = int(rng.integers(1, 4))
        mask = None
        build = frames and (keep is None or k in keep)
        if frac > 0.0:
            mask = np.full((side, side), 255, np.uint8) if build else None
            r = side * np.sqrt(frac / (nd * np.pi))
            for _ in range(nd):
                cx_, cy_ = rng.uniform(0, side, 2)
                if not build:
                    continue
                x0, x1 = max(int(cx_ - r), 0), min(int(cx_ + r) + 2, side)
                y0, y1 = max(int(cy_ - r), 0), min(int(cy_ + r) + 2, side)
                yy, xx = np.mgrid[y0:y1, x0:x1]
                sub = mask[y0:y1, x0:x1]
                sub[(xx - cx_) ** 2 + (yy - cy_) ** 2 < r * r] = 0
        subset = int(rng.choice([15, 21, 31, 41]))
        step = int(rng.choice([4, 8]))
        prm = params((0, 0, side, side), step, subset, subset)
        if not frames:
            jobs.append({"prm": prm, "warp": warp, "index": k, "has_mask": frac > 0.0})
            continue
        if keep is not None and k not in keep:
            continue
        ref = speckle(side, side, 10000 + 17 * seed + k)
        dfm = speckle(side, side, 10000 + 17 * seed + k, warp, 1.0, 20000 + k)
        jobs.append({"ref": ref, "dfm": dfm, "mask": mask, "prm": prm, "warp": warp, "index": k})
    return jobs


class Incremental:
    """semper_incremental: a frame sequence against a moving reference."""

    def __init__(self):
        self._h = lib().semper_incremental_create()
        if not self._h:
            raise RuntimeError("semper_incremental_create failed")

    def close(self):
        h = getattr(self, "_h", None)
        self._h = None
        if h and _lib is not None:  # at interpreter exit the library may be gone already
            _lib.semper_incremental_destroy(h)

    __del__ = close

    def init(self, ref, prm: SemperParams, update_interval: int, mask=None) -> int:
        g = np.ascontiguousarray(ref, np.uint8)
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        return lib().semper_incremental_init(self._h, _p(g, _u8p), g.size, _p(m, _u8p),
                                             0 if m is None else m.size, g.shape[1], g.shape[0],
                                             ctypes.byref(prm), update_interval)

    def process(self, frame, capacity: int, metrics_len: int = 24, progress=None):
        d = np.ascontiguousarray(frame, np.uint8)
        out = np.zeros(max(capacity, 1), np.float32)
        met = np.zeros(max(metrics_len, 1), np.float32)
        info = IncrementalInfo()
        cb = PROGRESS_CB(progress) if progress else PROGRESS_CB()
        rc = lib().semper_incremental_process(self._h, _p(d, _u8p), d.size, _p(out, _f32p), capacity,
                                              _p(met, _f32p), metrics_len, ctypes.byref(info), cb, None)
        return rc, out[: max(rc, 0) * 8].reshape(-1, 8).copy(), met[:metrics_len].copy(), info

    def cancel(self):
        lib().semper_incremental_cancel(self._h)

    def profile(self) -> dict:
        """Where the last process() call spent its time (semper_b200_incremental_profile)."""
        o = np.zeros(16, np.float64)
        lib().semper_b200_incremental_profile(self._h, _p(o, _f64p))
        keys = ["total", "run", "match", "warp_mask", "adopt", "pack", "matches", "runs",
                "prep", "pool", "seed", "mesh", "path_a", "path_b", "strain", "solve_total"]
        return dict(zip(keys, map(float, o)))


class IncrementalBatch:
    """semper_b200_inc_batch: several frame sequences advanced together, one
    session each, their solves interleaved on the device."""

    def __init__(self, sequences: int, devices=None):
        """devices: GPU ordinals the sessions spread over (None: the current one)."""
        if devices:
            dv = (ctypes.c_int32 * len(devices))(*devices)
            self._h = lib().semper_b200_inc_batch_create_on(sequences, dv, len(devices))
        else:
            self._h = lib().semper_b200_inc_batch_create(sequences)
        if not self._h:
            raise RuntimeError("semper_b200_inc_batch_create failed")
        self.sequences = sequences

    def close(self):
        h = getattr(self, "_h", None)
        self._h = None
        if h and _lib is not None:  # at interpreter exit the library may be gone already
            _lib.semper_b200_inc_batch_destroy(h)

    __del__ = close

    def init(self, seq: int, ref, prm: SemperParams, update_interval: int, mask=None) -> int:
        g = np.ascontiguousarray(ref, np.uint8)
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        return lib().semper_b200_inc_batch_init(self._h, seq, _p(g, _u8p), _p(m, _u8p), g.shape[1], g.shape[0],
                                                ctypes.byref(prm), update_interval)

    def process(self, frames: dict, capacity: int, metrics_len: int = 24):
        """frames: {sequence: frame}. Returns {sequence: (rc, points, metrics, info)}."""
        seqs = sorted(frames)
        arr = (IncFrame * len(seqs))()
        keep = []
        for i, q in enumerate(seqs):
            d = np.ascontiguousarray(frames[q], np.uint8)
            out = np.empty(max(capacity, 1), np.float32)  # fresh per call: returned as views
            met = np.zeros(max(metrics_len, 1), np.float32)
            keep.append((d, out, met))
            arr[i].sequence = q
            arr[i].frame = d.ctypes.data
            arr[i].out = out.ctypes.data
            arr[i].out_capacity = capacity
            arr[i].metrics = met.ctypes.data
            arr[i].metrics_len = metrics_len
        rc = lib().semper_b200_inc_batch_process(self._h, arr, len(seqs))
        if rc != 0:
            raise RuntimeError(f"semper_b200_inc_batch_process returned {rc}")
        res = {}
        for i, q in enumerate(seqs):
            r = arr[i].result
            _, out, met = keep[i]
            info = IncrementalInfo()
            ctypes.memmove(ctypes.byref(info), ctypes.byref(arr[i].info), ctypes.sizeof(IncrementalInfo))
            res[q] = (r, out[: max(r, 0) * 8].reshape(-1, 8), met[:metrics_len], info)
        return res


def version() -> str:
    return lib().semper_version().decode()


# --------------------------------------------------------------- synthetic speckle
def warp_block(cx=0.0, cy=0.0, u0=0.0, v0=0.0, a=(0.0, 0.0, 0.0, 0.0), su=0.0, Lu=0.0, sv=0.0, Lv=0.0,
               modes=()) -> np.ndarray:
    """The synth_speckle warp parameter block (see csrc/synth/speckle.cpp)."""
    flat = [cx, cy, u0, v0, *a, su, Lu, sv, Lv, float(len(modes))]
    for m in modes:
        flat.extend(m)
    return np.asarray(flat, np.float64)


def speckle(w, h, seed, warp=None, noise=0.0, noise_seed=0, density=0.02, sigma=(1.5, 3.0), amp=(180.0, 220.0),
            background=30.0) -> np.ndarray:
    """One frame of the seeded Gaussian-blob speckle, optionally warped."""
    out = np.zeros((h, w), np.uint8)
    W = None if warp is None else np.ascontiguousarray(warp, np.float64)
    rc = synth_lib().synth_speckle(_p(out, _u8p), w, h, seed, density, sigma[0], sigma[1], amp[0], amp[1],
                                   background, _p(W, _f64p), noise, noise_seed)
    if rc != 0:
        raise RuntimeError("synth_speckle failed")
    return out


def displacement(warp, X, Y):
    X = np.ascontiguousarray(X, np.float64).ravel()
    Y = np.ascontiguousarray(Y, np.float64).ravel()
    u = np.zeros_like(X)
    v = np.zeros_like(X)
    W = np.ascontiguousarray(warp, np.float64)
    synth_lib().synth_displacement(_p(W, _f64p), X.size, _p(X, _f64p), _p(Y, _f64p), _p(u, _f64p), _p(v, _f64p))
    return u, v


def config_pair(cfg: int, size: int | None = None, pair: int = 0):
    """(reference, deformed, params, warp) of a benchmark configuration.

    cfg 0: 512^2, translation (0.4, -0.25), noise 1, step 10, subset 21, window 21.
    cfg 1: 4096^2, u = 0.005 x + 2 sin(2 pi y / 256), v = -0.003 y + 1.5 sin(2 pi x / 384),
           noise 2, step 4, subset 31, window 31.
    cfg 4-plain: 4096^2 at the learned-seed comparison's solve settings (step 8,
           subset 41, window 41) under the cfg-1 field (the large-motion warp
           needs a global front end; see the proposal network).
    `size` overrides the image edge (same field, same settings) for small cases.
    """
    if cfg == 0:
        n = size or 512
        warp = warp_block(u0=0.4, v0=-0.25)
        prm = params((0, 0, n, n), 10, 21, 21)
        noise = 1.0
    elif cfg == 1:
        n = size or 4096
        warp = warp_block(a=(0.005, 0.0, 0.0, -0.003), su=2.0, Lu=256.0, sv=1.5, Lv=384.0)
        prm = params((0, 0, n, n), 4, 31, 31)
        noise = 2.0
    elif cfg == 4:
        n = size or 4096
        warp = warp_block(a=(0.005, 0.0, 0.0, -0.003), su=2.0, Lu=256.0, sv=1.5, Lv=384.0)
        prm = params((0, 0, n, n), 8, 41, 41)
        noise = 2.0
    else:
        raise ValueError(cfg)
    ref = speckle(n, n, 1000 + pair)
    dfm = speckle(n, n, 1000 + pair, warp, noise, 2000 + 1)
    return ref, dfm, prm, warp


def large_motion_pair(size: int | None = None, pair: int = 0, angle_deg: float | None = None,
                      shift: tuple | None = None, grf_px: float = 5.0, grf_len: float = 300.0, modes: int = 16):
    """(reference, deformed, params, warp, similarity) of the large-deformation
    workload: 4096^2 speckle under a rigid rotation ~ U[0, 180) deg about the
    image centre and a translation of up to 60 px, plus a smooth random
    displacement field of amplitude `grf_px` (per component a sum of `modes`
    cosines with wavevectors ~ N(0, grf_len^-2) per axis, a Gaussian
    covariance of length grf_len, and random phases, scaled so that the
    field's largest magnitude over the frame, sampled every 16 px, is
    grf_px), noise sigma 2; step 8, subset 41, window 41.
    The rect is the centred square whose every subset stays inside the
    deformed frame at any rotation (side (n/2 - 105) sqrt 2, rounded down to
    the step: 105 px cover the 60 px translation, the random field, half a
    subset and the interpolation border), so that the anchor lattice can keep
    a global model (at least 90% of its anchors solved).
    `similarity` = (angle rad, tx, ty) of the rigid part."""
    n = size or 4096
    rng = np.random.default_rng(7000 + pair)
    th = np.radians(rng.uniform(0.0, 180.0) if angle_deg is None else angle_deg)
    if shift is None:
        r, phi = 60.0 * np.sqrt(rng.uniform()), rng.uniform(0.0, 2 * np.pi)
        shift = (r * np.cos(phi), r * np.sin(phi))
    a = (np.cos(th) - 1.0, -np.sin(th), np.sin(th), np.cos(th) - 1.0)
    md = []
    if grf_px != 0.0:
        for c in range(2 * modes):
            k = rng.normal(0.0, 1.0 / grf_len, 2)
            md.append([k[0], k[1], 1.0 if c % 2 == 0 else 0.0, 1.0 if c % 2 == 1 else 0.0,
                       rng.uniform(0.0, 2 * np.pi)])
        g = np.arange(0.0, n, 16.0)
        X, Y = np.meshgrid(g, g)
        u, v = displacement(warp_block(modes=md), X, Y)
        scale = grf_px / float(np.max(np.hypot(u, v)))
        for m in md:
            m[2] *= scale
            m[3] *= scale
    warp = warp_block(cx=n / 2, cy=n / 2, u0=shift[0], v0=shift[1], a=a, modes=[tuple(m) for m in md])
    side = int((n / 2 - 105) * np.sqrt(2.0)) // 8 * 8
    x0 = (n - side) // 2
    prm = params((x0, x0, side, side), 8, 41, 41)
    ref = speckle(n, n, 4000 + pair)
    dfm = speckle(n, n, 4000 + pair, warp, 2.0, 5000 + pair)
    return ref, dfm, prm, warp, (float(th), float(shift[0]), float(shift[1]))


# --------------------------------------------------------------- kernel-level stages (torch device tensors)
def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ck(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed with CUDA error {rc}")


def pitch_of(width: int) -> int:
    """Row pitch (elements) of the float planes: rows padded to 16 bytes."""
    return (width + 3) & ~3


def image_prep(px, mask=None):
    """Float planes (I, gx, gy) of an 8-bit image, rows pitched to 16 bytes:
    tensors of shape (h, pitch); columns >= w are zero."""
    import torch

    h, w = px.shape
    P = pitch_of(w)
    I = torch.empty((h, P), dtype=torch.float32, device=px.device)
    gx = torch.empty_like(I)
    gy = torch.empty_like(I)
    _ck(lib().dic_cuda_image_prep(_ptr(px), _ptr(mask), w, h, P, _ptr(I), _ptr(gx), _ptr(gy), _stream()),
        "image_prep")
    return I, gx, gy


def grid_scan(mask, w, h, grid, rect, step, subset):
    import torch

    gw, gh = grid
    skip = torch.empty(gh * gw, dtype=torch.uint8, device="cuda")
    nv = torch.zeros(1, dtype=torch.int32, device="cuda")
    _ck(lib().dic_cuda_grid_scan(_ptr(mask), w, h, gw, gh, rect[0], rect[1], step, subset, _ptr(skip), _ptr(nv),
                                 _stream()), "grid_scan")
    return skip, nv


def hessian_pool(planes, width, skip, grid, rect, step, subset, lm=True):
    import torch

    I, gx, gy = planes
    h, P = I.shape
    gw, gh = grid
    n = gw * gh
    valid = torch.empty(n, dtype=torch.uint8, device="cuda")
    ms = torch.empty((n, 2), dtype=torch.float32, device="cuda")
    H = torch.empty((n, 21), dtype=torch.float64, device="cuda")
    Hs = torch.empty((n, 21), dtype=torch.float64, device="cuda")
    _ck(lib().dic_cuda_hessian_pool(_ptr(I), _ptr(gx), _ptr(gy), width, h, P, _ptr(skip), gw, gh, rect[0], rect[1],
                                    step, subset, 1 if lm else 0, _ptr(valid), _ptr(ms), _ptr(H), _ptr(Hs),
                                    _stream()), "hessian_pool")
    return valid, ms, H, Hs


def solve(ref_planes, def_I, width, pool, subset, tasks: np.ndarray, lm=True, six=False, blocks=0):
    """tasks: TASK_DT array (node indexes into pool). Returns RESULT_DT array."""
    import torch

    rI, rgx, rgy = ref_planes
    valid, ms, _H, Hs = pool
    h, P = rI.shape
    n = len(tasks)
    tbytes = torch.from_numpy(np.ascontiguousarray(tasks).view(np.uint8).copy()).cuda()
    res = torch.zeros(n * RESULT_DT.itemsize, dtype=torch.uint8, device="cuda")
    scratch = torch.empty(lib().dic_cuda_solve_scratch_bytes(n), dtype=torch.uint8, device="cuda")
    _ck(lib().dic_cuda_solve(_ptr(rI), _ptr(rgx), _ptr(rgy), _ptr(def_I), width, h, P, _ptr(valid), _ptr(ms),
                             _ptr(Hs), subset, 1 if lm else 0, 1 if six else 0, _ptr(tbytes), n, _ptr(res),
                             _ptr(scratch), blocks, _stream()), "solve")
    torch.cuda.synchronize()
    return res.cpu().numpy().view(RESULT_DT).copy()


def median_vsg(u, v, valid, step, window):
    """Median test (up to 5 passes) then VSG on device tensors; returns
    (rejected, valid', exx, eyy, exy)."""
    import torch

    gh, gw = u.shape
    ok = valid.clone()
    fail = torch.zeros_like(ok)
    nf = torch.zeros(1, dtype=torch.int32, device="cuda")
    rejected = 0
    for _ in range(5):
        nf.zero_()
        _ck(lib().dic_cuda_median_pass(gw, gh, _ptr(u), _ptr(v), _ptr(ok), _ptr(fail), _ptr(nf), _stream()), "median")
        k = int(nf.item())
        if k == 0:
            break
        _ck(lib().dic_cuda_clear_failed(gw * gh, _ptr(ok), _ptr(fail), _stream()), "clear")
        rejected += k
    exx = torch.empty_like(u)
    eyy = torch.empty_like(u)
    exy = torch.empty_like(u)
    _ck(lib().dic_cuda_vsg(gw, gh, step, window, _ptr(u), _ptr(v), _ptr(ok), _ptr(exx), _ptr(eyy), _ptr(exy),
                           _stream()), "vsg")
    torch.cuda.synchronize()
    return rejected, ok, exx, eyy, exy
