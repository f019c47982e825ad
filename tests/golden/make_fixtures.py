"""Regenerate the golden fixtures under tests/golden/ from the reference tree.

Run here, where the reference checkout and OpenCV's Python module exist:

    python tests/golden/make_fixtures.py /path/to/reference
    SEMPER_REFERENCE=/path/to/reference python tests/golden/make_fixtures.py

It writes
  golden_corpus_bicubic.npz, golden_corpus_keys6x6.npz
      the reference's GoldenCorpus records (tests/fixtures/golden_corpus.bin.*,
      written by tests/integration/test_golden_corpus.cpp:104-114): per point
      x, y, status and u, v, ux, uy, vx, vy, ZNSSD.
  full_field_golden.npz
      the reference's FullFieldGolden runs (tests/fixtures/full_field_golden.bin,
      written by tests/integration/test_full_field_golden.cpp:147-162): per
      scenario the return code, metrics slots 0-8, 16, 19-23, the packed points,
      and the global-motion homography the reference's AKAZE front end finds on
      the regenerated inputs (src/pipeline/akaze_features.cpp:122-182 with
      src/pipeline/full_field_anchors.cpp:204-279 scale order), computed with
      OpenCV's own AKAZE / BFMatcher / findHomography so the restatement can be
      fed the model the reference used.
The binary fixtures are data the reference's tests produced; nothing here
copies reference source.
"""
from __future__ import annotations

import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))

CORPUS_DT = np.dtype([("x", "<i4"), ("y", "<i4"), ("status", "<i4"), ("u", "<f4"), ("v", "<f4"),
                      ("ux", "<f4"), ("uy", "<f4"), ("vx", "<f4"), ("vy", "<f4"), ("corr", "<f4")])
FF_SLOTS = np.array([0, 1, 2, 3, 4, 5, 6, 7, 8, 16, 19, 20, 21, 22, 23], np.int32)


def read_corpus(path):
    d = open(path, "rb").read()
    n = struct.unpack("<I", d[:4])[0]
    return np.frombuffer(d[4:4 + n * CORPUS_DT.itemsize], dtype=CORPUS_DT)


def read_ff(path):
    d = open(path, "rb").read()
    n = struct.unpack("<I", d[:4])[0]
    off = 4
    runs = []
    for _ in range(n):
        code = struct.unpack("<i", d[off:off + 4])[0]
        off += 4
        counts = np.frombuffer(d[off:off + 60], "<f4").copy()
        off += 60
        npf = struct.unpack("<I", d[off:off + 4])[0]
        off += 4
        pts = np.frombuffer(d[off:off + 4 * npf], "<f4").reshape(-1, 8).copy()
        off += 4 * npf
        runs.append((code, counts, pts))
    return runs


def akaze_model(ref, dfm, roi):
    """The reference's L0 global model: AKAZE over the ROI padded by 40/scale px
    at 0.25x, 0.5x, 1x (INTER_AREA), Lowe ratio 0.75, RANSAC 3 px; the first
    scale with >= 25 inliers, else the best with >= 10."""
    import cv2

    H_img, W_img = ref.shape
    best = None
    for scale in (0.25, 0.5, 1.0):
        pad = int(40.0 / scale)
        x0, y0 = max(roi[0] - pad, 0), max(roi[1] - pad, 0)
        x1, y1 = min(roi[0] + roi[2] + pad, W_img), min(roi[1] + roi[3] + pad, H_img)
        if round((x1 - x0) * scale) < 16 or round((y1 - y0) * scale) < 16:
            continue
        ak = cv2.AKAZE_create()

        def det(img):
            small = cv2.resize(img[y0:y1, x0:x1], None, fx=scale, fy=scale, interpolation=cv2.INTER_AREA)
            return ak.detectAndCompute(small, None)

        k1, d1 = det(ref)
        k2, d2 = det(dfm)
        if d1 is None or d2 is None or len(k2) == 0:
            continue
        p1, p2 = [], []
        for m in cv2.BFMatcher(cv2.NORM_HAMMING).knnMatch(d1, d2, k=2):
            if len(m) != 2 or not (m[0].distance < 0.75 * m[1].distance):
                continue
            p1.append(k1[m[0].queryIdx].pt)
            p2.append(k2[m[0].trainIdx].pt)
        if len(p1) < 10:
            continue
        H, inl = cv2.findHomography(np.float32(p1), np.float32(p2), cv2.RANSAC, 3.0)
        if H is None or int(inl.sum()) < 10:
            continue
        T = np.array([[scale, 0, -scale * x0], [0, scale, -scale * y0], [0, 0, 1]])
        Ti = np.array([[1 / scale, 0, x0], [0, 1 / scale, y0], [0, 0, 1]])
        cand = (Ti @ H @ T, int(inl.sum()), scale)
        if best is None or cand[1] > best[1]:
            best = cand
        if cand[1] >= 25:
            break
    return best


def main(ref_root):
    fx = os.path.join(ref_root, "tests", "fixtures")
    for suf in ("bicubic", "keys6x6"):
        a = read_corpus(os.path.join(fx, "golden_corpus.bin." + suf))
        np.savez_compressed(os.path.join(HERE, f"golden_corpus_{suf}.npz"), records=a)
    runs = read_ff(os.path.join(fx, "full_field_golden.bin"))
    import oracle

    models = []
    for s in range(len(runs)):
        ref, dfm = oracle.ff_inputs(s)
        m = akaze_model(ref, dfm, (0, 0, 320, 320))
        models.append(m[0] if m is not None else np.full((3, 3), np.nan))
    np.savez_compressed(
        os.path.join(HERE, "full_field_golden.npz"),
        codes=np.array([r[0] for r in runs], np.int32),
        counts=np.stack([r[1] for r in runs]),
        slots=FF_SLOTS,
        points0=runs[0][2], points1=runs[1][2],
        models=np.stack(models),
    )
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SEMPER_REFERENCE")
    if not root:
        sys.exit("usage: make_fixtures.py <reference checkout>  (or set SEMPER_REFERENCE)")
    main(root)
