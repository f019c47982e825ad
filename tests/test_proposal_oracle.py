"""The proposal network's CPU restatement (oracle/proposal.py) checked
against itself by central finite differences, in float64 with the bfloat16
rounding switched off: its backward pass, the checker of the device's
gradients, gives the derivative of its forward pass."""
import numpy as np
import pytest

import proposal as P


@pytest.fixture
def exact(monkeypatch):
    monkeypatch.setattr(P, "bf16", lambda a: np.asarray(a, np.float64))
    return P


def test_gradients_match_finite_differences(exact):
    rng = np.random.default_rng(1)
    p = {k: v.astype(np.float64) for k, v in exact.init_params(3).items()}
    for k in p:
        if k.startswith("b"):
            p[k] = rng.standard_normal(p[k].shape) * 0.1
    p["w6"] = rng.standard_normal(p["w6"].shape) * 0.1
    x = rng.standard_normal((2, 64, 64, 2))
    tgt = rng.standard_normal((2, 6)) * 0.1

    def loss(q):
        out, _ = exact.forward(q, x)
        return exact.loss_and_grad(out, tgt)[0]

    out, cache = exact.forward(p, x)
    _, go = exact.loss_and_grad(out, tgt)
    g = exact.backward(p, cache, go)
    for name in ["w0", "b0", "w2", "b3", "w4", "w5", "b5", "w6", "b6"]:
        flat = p[name].reshape(-1)
        for i in rng.integers(0, flat.size, 3):
            old = flat[i]
            flat[i] = old + 1e-5
            lp = loss(p)
            flat[i] = old - 1e-5
            lm = loss(p)
            flat[i] = old
            fd = (lp - lm) / 2e-5
            an = g[name].reshape(-1)[i]
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)), (name, i, fd, an)


def test_flat_layout_round_trip():
    p = P.init_params(0)
    flat = P.flatten(p)
    q = P.unflatten(flat)
    assert all(np.array_equal(p[n], q[n]) for n in P.param_names())
    assert flat.size == 2 * 16 * 9 + 16 + 16 * 32 * 9 + 32 + 32 * 64 * 9 + 64 + 64 * 128 * 9 + 128 + \
        128 * 128 * 9 + 128 + 512 * 128 + 128 + 128 * 6 + 6
