"""The boundary's raw-image conversions against OpenCV's own results
(tests/golden/boundary_fixtures.npz, made by make_boundary_fixtures.py with
cv2): the raw-RGBA gray conversion of the reference's decoding
(src/io/image_codec.cpp:141-152) and the nearest-neighbour resize of an ROI
mask of another size (src/pipeline/full_field_solver.cpp:191-194). The
conversions are host code (csrc/host/gray.hpp), compiled here into a small
checker; no GPU is needed."""
import os
import subprocess

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIX = os.path.join(REPO, "tests", "golden", "boundary_fixtures.npz")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("gray") / "gray_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(REPO, "semper-dic-engine_b200", "csrc", "host"),
                    os.path.join(REPO, "tests", "cpp", "gray_check.cpp"), "-o", out], check=True)
    return out


def test_rgba_to_gray_matches_opencv(checker, tmp_path):
    f = np.load(FIX)
    rgba = np.ascontiguousarray(f["rgba"])
    src, dst = tmp_path / "rgba.raw", tmp_path / "gray.raw"
    rgba.tofile(src)
    subprocess.run([checker, "luma", str(src), str(rgba.shape[0] * rgba.shape[1]), str(dst)], check=True)
    got = np.fromfile(dst, np.uint8).reshape(rgba.shape[:2])
    assert np.array_equal(got, f["gray"])


def test_rgba_to_gray_every_color(checker, tmp_path):
    """All 2^24 RGB triples against the fixed-point rule the fixture pins
    (9798 R + 19235 G + 3735 B + 2^14) >> 15, restated here in numpy."""
    r = np.arange(256, dtype=np.int64)
    R, G, B = [x.ravel() for x in np.meshgrid(r, r, r, indexing="ij")]
    rgba = np.stack([R, G, B, np.zeros_like(R)], 1).astype(np.uint8)
    src, dst = tmp_path / "all.raw", tmp_path / "all_gray.raw"
    rgba.tofile(src)
    subprocess.run([checker, "luma", str(src), str(R.size), str(dst)], check=True)
    got = np.fromfile(dst, np.uint8)
    want = ((9798 * R + 19235 * G + 3735 * B + (1 << 14)) >> 15).astype(np.uint8)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("name,stride_pad", [("mask_small", 0), ("mask_strided_src", 13)])
def test_mask_resize_matches_opencv(checker, tmp_path, name, stride_pad):
    f = np.load(FIX)
    m = f[name]
    h, w = m.shape
    buf = np.zeros((h, w + stride_pad), np.uint8)
    buf[:, :w] = m
    src, dst = tmp_path / "m.raw", tmp_path / "m320.raw"
    buf.tofile(src)
    subprocess.run([checker, "resize", str(src), str(w), str(h), str(w + stride_pad), "320", "320", str(dst)],
                   check=True)
    got = np.fromfile(dst, np.uint8).reshape(320, 320)
    want = f["mask_320" if name == "mask_small" else "mask_strided_320"]
    assert np.array_equal(got, want)
