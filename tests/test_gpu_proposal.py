"""The learned seed proposal network's device kernels (BF16 tensor-core
convolutions and MLP, FP32 accumulation) against the numpy restatement of the
same network (oracle/proposal.py): forward outputs and every parameter's
gradient; then training on device-made synthetic pairs lowers the loss.

The device and the restatement round the same values to bfloat16; their FP32
sums run in different orders, and a sum that lands next to a bfloat16 rounding
boundary can round the other way, so the comparison is relative, per tensor:
1 % for outputs and gradients."""
import numpy as np
import pytest

import proposal as P
import semper_b200 as sb

pytestmark = pytest.mark.gpu

# max rotation (rad), max stretch, max shear, max shift (px), noise, box factor
CFG = [2 * np.pi, 0.03, 0.02, 48.0, 2.0, 4]


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / (np.linalg.norm(b) + 1e-30))


@pytest.fixture(scope="module")
def speckle():
    return sb.speckle(1536, 1536, 77)


def test_forward_and_gradients_match_restatement(speckle):
    net = sb.Proposal(64)
    rng = np.random.default_rng(4)
    p = P.init_params(5)
    for n in p:
        if n.startswith("b"):
            p[n] = (rng.standard_normal(p[n].shape) * 0.05).astype(np.float32)
    p["w6"] = (rng.standard_normal(p["w6"].shape) * 0.05).astype(np.float32)
    net.set_params(P.flatten(p))
    assert np.array_equal(net.get_params(), P.flatten(p))
    x, t = net.synth(speckle, CFG, seed=3, batch=48)
    assert np.isfinite(x).all() and np.abs(x.reshape(48, -1, 2).mean(1)).max() < 0.05
    out = net.forward(x)
    ref, cache = P.forward(p, x)
    assert _rel(out, ref) < 1e-2
    loss, g = net.gradients(x, t)
    rloss, go = P.loss_and_grad(ref, t)
    assert abs(loss - rloss) <= 1e-2 * rloss
    gref = P.backward(p, cache, go)
    gdev = P.unflatten(g)
    for name in P.param_names():
        assert _rel(gdev[name], gref[name]) < 1e-2, name


# the small-residual refinement setting (box factor 2, rotation up to 15 deg,
# shift up to 24 px), where a few hundred steps already learn the translation
CFG_FINE = [np.radians(15.0), 0.03, 0.02, 24.0, 2.0, 2]


def test_training_lowers_the_loss(speckle):
    net = sb.Proposal(64)
    losses = net.train(speckle, CFG_FINE, steps=400, batch=64, lr=1e-3, seed=11)
    assert np.isfinite(losses).all()
    first, last = losses[:20].mean(), losses[-20:].mean()
    print(f"loss {first:.1f} -> {last:.1f} (patch px^2)")
    assert last < 0.7 * first


def test_shipped_weights_accuracy(speckle):
    """The trained weights shipped with the package, on held-out synthetic
    pairs of each refinement stage: median shift error (full-resolution px)
    and rotation error (deg)."""
    net = sb.Proposal(256)
    net.set_params(np.load(sb.PROPOSAL_WEIGHTS))
    for cfg, shift_px, rot_deg in (([2 * np.pi, 0.03, 0.02, 48.0, 2.0, 4], 40.0, 20.0),
                                   ([np.radians(15.0), 0.03, 0.02, 24.0, 2.0, 2], 4.0, 3.0),
                                   ([np.radians(8.0), 0.03, 0.02, 10.0, 2.0, 1], 2.0, 3.0)):
        x, t = net.synth(speckle, cfg, seed=901, batch=256)
        o = net.forward(x)
        rot = lambda a: np.degrees(np.arctan2(a[:, 2] - a[:, 1], 2.0 + a[:, 0] + a[:, 3]))
        dr = np.abs((rot(o) - rot(t) + 180.0) % 360.0 - 180.0)
        dt = cfg[5] * 16.0 * np.hypot(o[:, 4] - t[:, 4], o[:, 5] - t[:, 5])
        print(f"f={cfg[5]}: shift median {np.median(dt):.2f} px, rotation median {np.median(dr):.2f} deg")
        assert np.median(dt) < shift_px and np.median(dr) < rot_deg
