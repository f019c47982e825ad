"""Learned seeding on the device (Engine::run with a proposal network): the
network's global model and per-anchor guesses, the anchor lattice judging the
model by the reference's keep rule (full_field_anchors.cpp:122-168, 204-279),
and the global-motion estimate as the fallback.

Parity: everything after the network is the reference's pipeline, so the
oracle, given the model and the anchor guesses the device's network produced,
must return the device's field bit for bit. Gain: on the large-deformation
workload (rotation up to 180 deg, translation up to 60 px, a 5 px random
field) the lattice alone (the reference's AUTO_SEARCH: a +-15 px scan and the
2-DOF Simplex) finds nothing, while learned seeding recovers the whole field
at the accuracy of a seeding from the true motion."""
import numpy as np
import pytest

import oracle as O
import semper_b200 as sb

pytestmark = pytest.mark.gpu


def _plist(prm):
    return [prm.rect_x, prm.rect_y, prm.rect_w, prm.rect_h, prm.step, prm.subset_size, prm.strain_window,
            prm.use_6x6_interpolator]


@pytest.fixture(scope="module")
def net():
    return sb.Proposal.trained()


@pytest.fixture(scope="module", params=[0, 3])
def pair(request):
    return request.param, sb.large_motion_pair(pair=request.param)


def test_learned_seeding_parity_with_oracle(net, pair):
    k, (ref, dfm, prm, warp, sim) = pair
    eng = sb.Engine()
    assert eng.set_reference(ref) == 0
    assert eng.set_proposal(net, True) == 0
    rc, pts, met = eng.run(dfm, prm)
    L = eng.last_learned()
    g = eng.learned_guesses()
    print(f"pair {k}: rc {rc}, kept {L['kept']}, inliers {L['inliers']}, guesses {np.isfinite(g[:, 0]).sum()}, "
          f"network {L['ms']:.2f} ms, model vs anchors mean {L['err_mean_px']:.2f} max {L['err_max_px']:.2f} px")
    assert L["ran"] and L["proposed"] and L["kept"]
    assert rc > 0 and np.isfinite(g).all()
    o = O.Oracle()
    assert o.set_reference(ref) == 0
    rc2, pts2, met2 = o.run(dfm, _plist(prm), model_h=L["H"], anchor_uv=g)
    assert rc2 == rc
    assert np.array_equal(pts, pts2)
    assert np.array_equal(met[:8], met2[:8])


def test_learned_seeding_gain(net, pair):
    """Learned against the lattice alone and against the global-motion estimate."""
    k, (ref, dfm, prm, warp, sim) = pair
    res = {}
    for mode in ("learned", "global", "lattice"):
        eng = sb.Engine()
        assert eng.set_reference(ref) == 0
        if mode == "learned":
            eng.set_proposal(net, True)
        if mode != "global":
            eng.set_global_motion(False)
        rc, pts, met = eng.run(dfm, prm)
        t, _ = eng.last_timings()
        rms = None
        if rc > 0:
            u, v = sb.displacement(warp, pts[:, 0], pts[:, 1])
            rms = float(np.sqrt(np.mean((pts[:, 2] - u) ** 2 + (pts[:, 3] - v) ** 2)))
        res[mode] = (rc, rms, t["seed"])
        print(f"pair {k} {mode}: points {rc}, rms vs true field {rms}, seeding {t['seed']:.2f} ms")
    n_grid = (prm.rect_w // prm.step) * (prm.rect_h // prm.step)
    assert res["lattice"][0] <= 0  # nothing found by the lattice alone
    assert res["learned"][0] >= 0.95 * n_grid
    assert res["learned"][1] < 0.01
    if res["global"][0] > 0:
        assert res["learned"][0] >= res["global"][0]


def test_rescue_order_matches_the_seeding_it_takes(net, pair):
    """The rescue order (the global-motion estimate first, the proposal only
    where the lattice rejects the estimate's model): on pair 0, whose estimate
    the lattice keeps, the field of the estimate alone, with the network never
    run; on pair 3, whose estimate is off by pixels and rejected, the field of
    the proposal-first seeding, bit for bit."""
    k, (ref, dfm, prm, warp, sim) = pair
    out = {}
    for mode in ("rescue", "learned", "global"):
        eng = sb.Engine()
        assert eng.set_reference(ref) == 0
        if mode != "global":
            assert eng.set_proposal(net, "rescue" if mode == "rescue" else True) == 0
        rc, pts, met = eng.run(dfm, prm)
        out[mode] = (rc, pts, met, eng.last_learned())
    rc, pts, met, L = out["rescue"]
    other = out["global"] if k == 0 else out["learned"]
    assert rc == other[0] > 0
    assert np.array_equal(pts, other[1])
    assert np.array_equal(met[:8], other[2][:8])
    assert L["ran"] == (k == 3)
    if k == 3:
        assert L["kept"] and out["global"][0] <= 0
