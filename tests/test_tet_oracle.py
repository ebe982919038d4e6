"""The oracle's restatement of the learned tetrahedron proposal: its
negative log-likelihood gradient against finite differences (BF16 rounding
off, FP64), and the vMF density normalisation."""
import numpy as np
import pytest

from oracle import binding as orc


@pytest.fixture
def exact_fp64():
    orc.load().orc_mlp_set_bf16(0)
    yield
    orc.load().orc_mlp_set_bf16(1)


def random_problem(seed, n=6):
    rng = np.random.default_rng(seed)
    w = (rng.normal(size=6288) * 0.2).astype(np.float32)
    x = rng.normal(size=(n, 16)).astype(np.float32)
    x[:, 13:] = 0.0
    s = rng.normal(size=(n, 4, 3))
    s /= np.linalg.norm(s, axis=-1, keepdims=True)
    return w, x, s.reshape(n, 12).astype(np.float32)


def test_gradient_matches_finite_differences(exact_fp64):
    w, x, s = random_problem(1)
    g, loss = orc.mlp_gradient(w, x, s)
    rng = np.random.default_rng(7)
    picks = rng.choice(np.arange(6288), size=60, replace=False)
    for i in picks:
        if 13 * 64 <= i < 16 * 64:  # weights of the zero-padded inputs
            continue
        h = 1e-2 * max(1.0, abs(float(w[i])))
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        h_eff = (float(wp[i]) - float(wm[i])) / 2.0
        lp = orc.mlp_gradient(wp, x, s)[1]
        lm = orc.mlp_gradient(wm, x, s)[1]
        fd = (lp - lm) / (2 * h_eff)
        assert fd == pytest.approx(g[i], rel=2e-3, abs=2e-3 * (1 + abs(g).max() * 1e-3)), i


def test_vmf_density_normalised():
    # log f = log k - log(2 pi) - log(1 - e^{-2k}) + k (mu.x - 1) integrates to 1 on S^2
    for kap in (0.05, 1.0, 20.0, 300.0):
        c = np.linspace(-1, 1, 200001)
        f = kap / (2 * np.pi * -np.expm1(-2 * kap)) * np.exp(kap * (c - 1.0))
        integral = 2 * np.pi * np.trapezoid(f, c)
        assert integral == pytest.approx(1.0, rel=1e-4)
