"""Input scenarios shared by the CPU and GPU tests.

`lattice_masked_pair` builds a pair on which the anchor lattice cannot seed
and the central-tendency fallback (Path C, src/pipeline/full_field_path_c.cpp:27-156)
must: an ROI mask removes one pixel at every lattice node, so every lattice
node's subset is masked and skipped (full_field_solver.cpp's grid scan skips a
node whose subset holds a masked pixel), the lattice accepts nothing, the
routing sees no seed (quality NONE, no published anchor), and Path C's search
from the grid centre finds the translation. The nodes between the lattice
nodes keep full subsets (step 12 > half a subset of 21), and the flood of
Path B then covers them.
"""
import math

import numpy as np

import semper_b200 as sb


def lattice_count(n, stride):
    """Lattice indices on an axis of n nodes: 0, s, 2s, ... and the last node
    (src/pipeline/full_field_anchors.cpp:64-69)."""
    c = (n + stride - 1) // stride
    if (c - 1) * stride != n - 1:
        c += 1
    return c


def lattice_indices(n, stride):
    idx = list(range(0, n, stride))
    if idx[-1] != n - 1:
        idx.append(n - 1)
    return idx


def plan_anchor_lattice(gw, gh, target=256):
    """The lattice strides (sx, sy) of plan_anchor_lattice
    (src/pipeline/full_field_anchors.cpp:73-119): an isotropic stride aiming
    at `target` nodes, each axis clamped to keep 3 indices, then widened back
    inside the budget."""
    stride = max(1, int(math.floor(math.sqrt(gw * gh / float(target)) + 0.5)))
    budget = lattice_count(gw, stride) * lattice_count(gh, stride)
    sx = sy = stride
    while sx > 1 and lattice_count(gw, sx) < 3:
        sx -= 1
    while sy > 1 and lattice_count(gh, sy) < 3:
        sy -= 1
    while lattice_count(gw, sx) * lattice_count(gh, sy) > budget:
        grow_x = lattice_count(gw, sx + 1) >= 3
        grow_y = lattice_count(gh, sy + 1) >= 3
        if not grow_x and not grow_y:
            break
        if grow_x and (not grow_y or lattice_count(gw, sx) >= lattice_count(gh, sy)):
            sx += 1
        else:
            sy += 1
    return sx, sy


def lattice_masked_pair(n=768, step=12, subset=21, window=49):
    """(reference, deformed, mask, params): 768^2 speckle under a translation
    of (2.3, -1.7) px with a small stretch, noise sigma 1 on the deformed
    frame, and a mask with one pixel off at every anchor-lattice node."""
    warp = sb.warp_block(u0=2.3, v0=-1.7, a=(0.002, 0.0, 0.0, -0.001))
    ref = sb.speckle(n, n, 4242)
    dfm = sb.speckle(n, n, 4242, warp, 1.0, 77)
    gw = n // step  # nodes at 0, step, ... < n on the full-frame rect
    sx, sy = plan_anchor_lattice(gw, gw)
    mask = np.full((n, n), 255, np.uint8)
    for gy in lattice_indices(gw, sy):
        for gx in lattice_indices(gw, sx):
            mask[gy * step, gx * step] = 0
    return ref, dfm, mask, sb.params((0, 0, n, n), step, subset, window)
