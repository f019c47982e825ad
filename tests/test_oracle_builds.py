"""The CPU restatement's two builds and the checker's copy of the speckle
generator.

The timing build (the reference's compiler flags, multiply-adds unfused as the
reference computes them) is the CPU baseline of the benchmark; it must solve
the same grid to the same field as the checker build, within float rounding.
The checker's copy of the generator must give the package generator's bytes.
"""
import ctypes

import numpy as np

import semper_b200 as sb


def test_reference_flags_build_matches_checker(oracle_lib):
    ref, dfm, prm, _ = sb.config_pair(0, size=384)
    p = [0, 0, 384, 384, prm.step, prm.subset_size, prm.strain_window, 0]
    out = []
    for kind in ("contract", "reference_flags"):
        o = oracle_lib.Oracle(False, kind=kind)
        o.set_reference(ref)
        out.append(o.run(dfm, p))
    (ra, pa, ma), (rb, pb, mb) = out
    assert ra == rb > 900
    assert np.array_equal(pa[:, :2], pb[:, :2])
    assert np.abs(pa[:, 2:4] - pb[:, 2:4]).max() <= 1e-3
    assert np.abs(pa[:, 4:7] - pb[:, 4:7]).max() <= 1e-4


def test_checker_speckle_generator_matches_package(oracle_lib):
    a = sb.speckle(200, 180, 77, sb.warp_block(cx=100, cy=90, u0=1.5, v0=-2.0, a=(0.01, 0.0, 0.0, -0.02)), 1.0, 5)
    S = ctypes.CDLL(oracle_lib.synth_path())
    u8p, f64p = ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_double)
    S.synth_speckle.argtypes = [u8p, ctypes.c_int, ctypes.c_int, ctypes.c_uint64] + [ctypes.c_double] * 6 + \
        [f64p, ctypes.c_double, ctypes.c_uint64]
    b = np.zeros_like(a)
    W = np.ascontiguousarray(sb.warp_block(cx=100, cy=90, u0=1.5, v0=-2.0, a=(0.01, 0.0, 0.0, -0.02)))
    assert S.synth_speckle(b.ctypes.data_as(u8p), 200, 180, 77, 0.02, 1.5, 3.0, 180.0, 220.0, 30.0,
                           W.ctypes.data_as(f64p), 1.0, 5) == 0
    assert np.array_equal(a, b)
