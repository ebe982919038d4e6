"""Known answers that pin the oracle (and through it the engine) to the
physics and to the reference's energy convention."""
import json
import os

import numpy as np
import pytest

from cudacode_b200.engine import System
from oracle.binding import Oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def set_spins(o, L, vec_fn, R=1):
    sh = o.spin_shape()
    a = np.zeros(sh, dtype=np.float32)
    for s in range(16):
        a[:, s, :, :3] = vec_fn(s)
    o.set_spins(a)


def test_reference_total_energy_convention():
    """E_reference (TotalEnergy, spin-1/2 S^2=1/4, couplings_const with
    J1=J2=J) == E_engine / 4 on seeded configurations."""
    cases = json.load(open(os.path.join(GOLDEN, "reference_energy.json")))["cases"]
    for c in cases:
        L = c["L"]
        v = np.array(c["spins"], dtype=np.float32)  # plane-major (site*L^3 + cell)
        o = Oracle([System(L=L, temperatures=[1.0], J1=c["J"])], fp64=True)
        a = np.zeros(o.spin_shape(), dtype=np.float32)
        a[0, :, :, :3] = v.reshape(16, L ** 3, 3)
        o.set_spins(a)
        e, _ = o.observables()
        assert e[0] / 4.0 == pytest.approx(c["energy_reference_units"], rel=1e-12, abs=1e-12)


@pytest.mark.parametrize("L", [2, 3, 4])
def test_ferromagnet_energy(L):
    o = Oracle([System(L=L, temperatures=[1.0], J1=1.0)])
    set_spins(o, L, lambda s: (0.0, 0.0, 1.0))
    e, m = o.observables()
    N = 16 * L ** 3
    assert e[0] == pytest.approx(3.0 * N)
    assert m[0] == pytest.approx([0.0, 0.0, N])


@pytest.mark.parametrize("L", [2, 4])
def test_all_in_all_out_energy(L):
    # each spin along its local <111> axis: zero total spin on every tetrahedron
    axes = np.array([[-1, -1, -1], [1, 1, -1], [-1, 1, 1], [1, -1, 1]], dtype=np.float64)
    axes /= np.sqrt(3.0)
    o = Oracle([System(L=L, temperatures=[1.0], J1=1.0)], fp64=True)
    set_spins(o, L, lambda s: axes[s % 4])
    e, m = o.observables()
    assert e[0] == pytest.approx(-16 * L ** 3, rel=1e-6)
    assert np.abs(m[0]).max() < 1e-3


def test_over_relaxation_conserves_energy_and_norm():
    o = Oracle([System(L=3, temperatures=[0.5, 1.0], J1=1.0, J2=0.05, J3=0.03)], seed=7)
    o.init_random()
    e0, _ = o.observables()
    o.overrelax_sweep(5)
    e1, _ = o.observables()
    assert np.allclose(e0, e1, atol=1e-3)
    s = o.get_spins()
    n = np.linalg.norm(s[..., :3], axis=-1)
    assert np.abs(n - 1).max() < 1e-5


def test_high_temperature_series():
    """E/N = -J^2/T + O(1/T^3) for the classical Heisenberg pyrochlore."""
    T = 10.0
    o = Oracle([System(L=3, temperatures=[T], J1=1.0)], seed=3, fp64=True)
    o.init_random()
    o.tune_cone(0.5, 10, 5)
    es = []
    for _ in range(400):
        o.metropolis_sweep(1)
        o.overrelax_sweep(1)
        es.append(o.observables()[0][0] / (16 * 27))
    es = np.array(es[50:])
    # series: -1/T (1 - ...) ; allow the O(1/T^3) term and statistical error
    assert abs(es.mean() - (-1.0 / T)) < 0.01


def test_fp32_oracle_deterministic():
    def run():
        o = Oracle([System(L=3, temperatures=[0.3, 0.6], J1=1.0)], seed=99)
        o.init_random()
        o.set_cone(np.array([0.5, 0.0], dtype=np.float32))
        o.metropolis_sweep(3)
        o.overrelax_sweep(2)
        return o.get_spins()
    a, b = run(), run()
    assert np.array_equal(a, b)


def test_structure_factor_ferromagnet_and_sum_rule():
    L = 2
    o = Oracle([System(L=L, temperatures=[1.0])], fp64=True)
    set_spins(o, L, lambda s: (0.0, 1.0, 0.0))
    sq = o.structure_factor(G=4, stride=1)
    N = 16 * L ** 3
    # q = 0 carries |M|^2 / N = N; other q of the cubic grid with all four
    # FCC corners in phase vanish unless a reciprocal-lattice vector of the FCC
    assert sq[2, 2, 2] == pytest.approx(N)
    assert (sq >= -1e-9).all()


def test_structure_factor_sum_rule_over_full_zone():
    """sum over the L^3 wave vectors of one cubic zone, times the 64 basis
    translations of the extended zone (stride 1, G = 4L covers 4 zones per
    axis), equals sum_i |S_i|^2 * (4L)^3 / N-normalisation: the Parseval
    identity for a lattice with basis on the 4L grid."""
    L = 2
    o = Oracle([System(L=L, temperatures=[1.0])], fp64=True, seed=3)
    o.init_random()
    G = 4 * L
    sq = o.structure_factor(G=G, stride=1)
    # positions are multiples of a/4: on the (4L)^3 grid the DFT is unitary,
    # sum_q |F(q)|^2 = (4L)^3 sum_i |S_i|^2, and S = |F|^2 / N.
    N = 16 * L ** 3
    s = o.get_spins64()[..., :3]
    assert sq.sum() == pytest.approx((4 * L) ** 3 * (s ** 2).sum() / N, rel=1e-9)
