"""The C++ API (include/semper/pipeline.hpp, incremental.hpp) on the GPU,
called from a C++ program built here against libsemper_b200.so, against the
C ABI on the same inputs:
  * run_full_field with an ROI mask of another size, passed as a strided view:
    the library resizes it by nearest neighbour (full_field_solver.cpp:
    191-194), so the points equal semper_run's with OpenCV's resize of the
    mask (tests/golden/boundary_fixtures.npz), bit for bit; a request on the
    caller's token inside an open CancelScope ends the solve with kCancelled;
  * IncrementalSession::process_frame, frame by frame, equals
    semper_incremental_process;
  * a raw RGBA reference equals its gray form converted as OpenCV does.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle
import semper_b200 as sb

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIX = os.path.join(REPO, "tests", "golden", "boundary_fixtures.npz")


@pytest.fixture(scope="module")
def caller(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cxx") / "api_check")
    lib_dir = os.path.dirname(sb.LIB_PATH)
    sb.lib()
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(REPO, "include"),
                    os.path.join(REPO, "tests", "cpp", "api_check.cpp"), "-o", out, "-L", lib_dir, "-lsemper_b200",
                    f"-Wl,-rpath,{lib_dir}"], check=True)
    return out


def _records(path):
    raw = open(path, "rb").read()
    out, i = [], 0
    while i < len(raw):
        rc, n = np.frombuffer(raw, np.int32, 2, i)
        i += 8
        pts = np.frombuffer(raw, np.float32, n, i).reshape(-1, 8).copy()
        i += 4 * n
        out.append((int(rc), pts))
    return out


PRM = [0, 0, 320, 320, 12, 21, 48]


def test_run_full_field_resized_strided_mask_equals_c_abi(caller, tmp_path):
    f = np.load(FIX)
    ref, dfm = oracle.ff_inputs(1)
    small = f["mask_small"]
    h, w = small.shape
    strided = np.zeros((h, w + 7), np.uint8)
    strided[:, :w] = small
    for name, arr in (("ref", ref), ("def", dfm), ("mask", strided)):
        np.ascontiguousarray(arr).tofile(tmp_path / f"{name}.raw")
    res = tmp_path / "out.bin"
    r = subprocess.run([caller, "full", "320", "320", str(tmp_path / "ref.raw"), str(tmp_path / "def.raw"),
                        str(tmp_path / "mask.raw"), str(w), str(h), str(w + 7)] + [str(v) for v in PRM] + [str(res)],
                       capture_output=True, text=True, check=True)
    recs = _records(res)
    mask320 = f["mask_320"]
    e = sb.Engine()
    assert e.set_reference(ref, mask320) == 0
    rc, pts, _ = e.run(dfm, sb.params(tuple(PRM[:4]), PRM[4], PRM[5], PRM[6]), mask=mask320)
    assert rc > 100
    assert recs[0][0] == rc and np.array_equal(recs[0][1], pts)
    assert recs[1][0] == rc and np.array_equal(recs[1][1], pts)
    assert recs[2][0] == sb.SEMPER_ERR_CANCELLED
    assert "progress 100" in r.stdout


def test_incremental_session_equals_c_abi(caller, tmp_path):
    n = 320
    ref = sb.speckle(n, n, 61)
    frames = []
    for t in range(1, 5):
        w = sb.warp_block(cx=n / 2, cy=n / 2, u0=0.8 * t, v0=0.4 * t, a=(0.003 * t, 0.0, 0.0, -0.002 * t))
        frames.append(sb.speckle(n, n, 61, w, 1.0, 500 + t))
    ref.tofile(tmp_path / "ref.raw")
    paths = []
    for k, fr in enumerate(frames):
        p = tmp_path / f"f{k}.raw"
        fr.tofile(p)
        paths.append(str(p))
    prm = [16, 16, 288, 288, 8, 21, 21]
    res = tmp_path / "inc.bin"
    subprocess.run([caller, "inc", str(n), str(n), str(tmp_path / "ref.raw")] + [str(v) for v in prm] +
                   ["2", str(res)] + paths, check=True, capture_output=True, text=True)
    recs = _records(res)
    inc = sb.Incremental()
    assert inc.init(ref, sb.params(tuple(prm[:4]), prm[4], prm[5], prm[6]), 2) == 0
    for (rc, pts), fr in zip(recs, frames):
        drc, dpts, _, _ = inc.process(fr, 36 * 36 * 8)
        assert rc == drc > 500 and np.array_equal(pts, dpts)


def test_raw_rgba_reference_equals_opencv_gray():
    """semper_set_reference with a raw RGBA buffer solves as with the gray
    image OpenCV's RGBA2GRAY makes of it (the fixed-point rule the boundary
    fixture pins, applied here in numpy)."""
    ref, dfm = oracle.ff_inputs(0)
    rng = np.random.default_rng(9)
    # RGBA frames whose luma follows the reference: G carries the image, R and
    # B are noise the conversion mixes in
    rgba = np.zeros(ref.shape + (4,), np.uint8)
    rgba[..., 0] = rng.integers(0, 256, ref.shape)
    rgba[..., 2] = rng.integers(0, 256, ref.shape)
    rgba[..., 1] = ref
    rgba[..., 3] = 255
    R, G, B = [rgba[..., c].astype(np.int64) for c in range(3)]
    gray = ((9798 * R + 19235 * G + 3735 * B + (1 << 14)) >> 15).astype(np.uint8)
    prm = sb.params(tuple(PRM[:4]), PRM[4], PRM[5], PRM[6])
    a, b = sb.Engine(), sb.Engine()
    assert a.set_reference_bytes(rgba.tobytes(), 320, 320) == 0
    assert b.set_reference(gray) == 0
    ra, pa, _ = a.run(dfm, prm)
    rb, pb, _ = b.run(dfm, prm)
    assert ra == rb and np.array_equal(pa, pb)
