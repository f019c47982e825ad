"""The CPU restatement against the reference's own golden fixtures.

These pin the oracle before it is trusted as the parity checker:
  * GoldenCorpus (tests/integration/test_golden_corpus.cpp): per-subset IC-GN,
    compared with the reference's rules and tolerances (:131-222);
  * FullFieldGolden (tests/integration/test_full_field_golden.cpp): the whole
    pipeline, fed the global-motion homography the reference's AKAZE front end
    produces on the same inputs, compared with the fixture's tolerances
    (:106-117, :266-276).
"""
import os

import numpy as np
import pytest

TOL_DISP, TOL_STRAIN = 1e-2, 1e-3
ON_TRUTH_PX, LOCAL_MIN_SCALE = 0.1, 5.0
SCEN = [(3.2, -1.7, 0, 0, 0, 0), (2.1, 1.4, 0.015, -0.008, 0.006, 0.012)]


def _on_truth(g, s):
    dx, dy = g["x"] - 256.0, g["y"] - 256.0
    ut = s[0] + s[2] * dx + s[3] * dy
    vt = s[1] + s[4] * dx + s[5] * dy
    return np.hypot(g["u"] - ut, g["v"] - vt) <= ON_TRUTH_PX


@pytest.mark.parametrize("interp", ["bicubic", "keys6x6"])
def test_golden_corpus(oracle_lib, golden_dir, interp):
    g = np.load(os.path.join(golden_dir, f"golden_corpus_{interp}.npz"))["records"]
    ixy, vals = oracle_lib.corpus(interp == "keys6x6")
    _, vals64 = oracle_lib.corpus(interp == "keys6x6", fp64=True)
    assert len(ixy) == len(g)
    assert (ixy[:, 0] == g["x"]).all() and (ixy[:, 1] == g["y"]).all()
    half = len(g) // 2
    scen = np.array([0] * half + [1] * (len(g) - half))
    status_mism = value_mism = to_exh = to_conv = excused = 0
    worst = 0.0
    for i in range(len(g)):
        exact = _on_truth(g[i], SCEN[scen[i]])
        sc = 1.0 if exact else LOCAL_MIN_SCALE
        c = vals[i]
        agree = (abs(g[i]["u"] - c[0]) <= TOL_DISP * sc and abs(g[i]["v"] - c[1]) <= TOL_DISP * sc and
                 max(abs(g[i]["ux"] - c[2]), abs(g[i]["uy"] - c[3]), abs(g[i]["vx"] - c[4]),
                     abs(g[i]["vy"] - c[5])) <= TOL_STRAIN * sc)
        if g[i]["status"] != ixy[i, 2]:
            if g[i]["corr"] < 2.0 and c[6] < 2.0 and agree:
                if ixy[i, 2] != 0:
                    to_exh += 1
                else:
                    to_conv += 1
                continue
            status_mism += 1
            continue
        if g[i]["status"] != 0:
            continue
        if exact:
            worst = max(worst, abs(g[i]["u"] - c[0]), abs(g[i]["v"] - c[1]))
        if not agree:
            # Excused only where the restatement's FP32 answer is the FP64
            # answer: the gap is then the reference's own float rounding on a
            # slowly converging subset ((236, 412): uy 5.6e-3 there, 6.9e-3
            # here and in FP64).
            fp64_same = (np.abs(vals64[i][:2] - c[:2]).max() <= 1e-4 and
                         np.abs(vals64[i][2:6] - c[2:6]).max() <= 1e-5)
            if fp64_same and abs(g[i]["u"] - c[0]) <= TOL_DISP * sc and abs(g[i]["v"] - c[1]) <= TOL_DISP * sc:
                excused += 1
            else:
                value_mism += 1
    assert value_mism == 0
    assert excused <= 1
    assert abs(to_exh - to_conv) <= 2 and to_exh + to_conv <= 6
    # The one unexcused flip the Keys 6x6 corpus shows is (214, 104): the
    # reference exhausted its 50 iterations wandering to (5.71, -3.69) with a
    # strain of -0.30; this restatement converges on the true field there.
    assert status_mism <= (1 if interp == "keys6x6" else 0)
    assert worst <= TOL_DISP


def _ff_compare(pts, gp, tol_disp, tol_strain=1e-4, tol_corr=1e-4):
    assert pts.shape == gp.shape
    assert (pts[:, :2] == gp[:, :2]).all()  # grid geometry is exact
    d = np.abs(pts - gp)
    assert d[:, 2:4].max() <= tol_disp
    assert d[:, 4:7].max() <= tol_strain
    assert d[:, 7].max() <= tol_corr


@pytest.mark.parametrize("scenario", [0, 1])
def test_full_field_golden_with_reference_model(oracle_lib, golden_dir, scenario):
    f = np.load(os.path.join(golden_dir, "full_field_golden.npz"))
    ref, dfm = oracle_lib.ff_inputs(scenario)
    o = oracle_lib.Oracle(False)
    o.set_reference(ref)
    rc, pts, met = o.run(dfm, [0, 0, 320, 320, 12, 21, 48, 0], model_h=f["models"][scenario])
    assert rc == f["codes"][scenario]
    tol = np.zeros(15, np.float32)
    tol[8], tol[13] = 0.1, 1e-4
    got = met[f["slots"]]
    assert (np.abs(got - f["counts"][scenario]) <= tol).all(), (got, f["counts"][scenario])
    _ff_compare(pts, f[f"points{scenario}"], 5e-3)


@pytest.mark.parametrize("scenario", [0, 1])
def test_full_field_golden_without_model(oracle_lib, golden_dir, scenario):
    """No global model (the reference's path when AKAZE finds none): the anchor
    lattice searches on its own, and the field that comes out is the same."""
    f = np.load(os.path.join(golden_dir, "full_field_golden.npz"))
    ref, dfm = oracle_lib.ff_inputs(scenario)
    o = oracle_lib.Oracle(False)
    o.set_reference(ref)
    rc, pts, met = o.run(dfm, [0, 0, 320, 320, 12, 21, 48, 0])
    assert rc == f["codes"][scenario]
    assert met[21] == 0.0
    # search-seeded anchors stop elsewhere inside the IC-GN tolerance
    _ff_compare(pts, f[f"points{scenario}"], 2e-2, 5e-4, 1e-3)


def test_fp64_agrees_with_fp32(oracle_lib):
    """The FP32 engine against the same math in FP64 (the accuracy judge)."""
    ref, dfm = oracle_lib.ff_inputs(1)
    a = oracle_lib.Oracle(False)
    b = oracle_lib.Oracle(True)
    a.set_reference(ref)
    b.set_reference(ref)
    ra, pa, _ = a.run(dfm, [0, 0, 320, 320, 12, 21, 48, 0])
    rb, pb, _ = b.run(dfm, [0, 0, 320, 320, 12, 21, 48, 0])
    assert ra == rb
    assert np.abs(pa[:, 2:4] - pb[:, 2:4]).max() <= 1e-2
