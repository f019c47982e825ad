"""Golden data for the boundary's raw-image conversions, made with OpenCV's
own Python module (the reference converts with OpenCV: cvtColor RGBA2GRAY in
src/io/image_codec.cpp:141-152, resize INTER_NEAREST in
src/pipeline/full_field_solver.cpp:191-194).

    python tests/golden/make_boundary_fixtures.py

writes tests/golden/boundary_fixtures.npz:
  rgba, gray          a seeded 64x48 RGBA frame and cv2's RGBA2GRAY of it
  mask_small          a seeded 0/255 mask of 97 x 71 with two discs
  mask_320            cv2.resize(mask_small, (320, 320), INTER_NEAREST)
  mask_strided_src    a 200 x 150 mask, and mask_strided_320 its resize
"""
import os

import cv2
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def discs(w, h, seed):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    m = np.full((h, w), 255, np.uint8)
    for _ in range(2):
        cx, cy, r = rng.uniform(0, w), rng.uniform(0, h), rng.uniform(0.1, 0.25) * min(w, h)
        m[(xx - cx) ** 2 + (yy - cy) ** 2 < r * r] = 0
    return m


def main():
    rng = np.random.default_rng(2024)
    rgba = rng.integers(0, 256, (48, 64, 4), dtype=np.uint8)
    gray = cv2.cvtColor(rgba, cv2.COLOR_RGBA2GRAY)
    small = discs(97, 71, 5)
    big = discs(200, 150, 6)
    np.savez_compressed(os.path.join(HERE, "boundary_fixtures.npz"), rgba=rgba, gray=gray, mask_small=small,
                        mask_320=cv2.resize(small, (320, 320), interpolation=cv2.INTER_NEAREST),
                        mask_strided_src=big,
                        mask_strided_320=cv2.resize(big, (320, 320), interpolation=cv2.INTER_NEAREST))
    print("wrote", os.path.join(HERE, "boundary_fixtures.npz"), "with OpenCV", cv2.__version__)


if __name__ == "__main__":
    main()
