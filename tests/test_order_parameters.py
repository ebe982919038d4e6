"""Order parameters (the reference's Measurement, Pyrochlore.cu:526-641, and
Math.cu:335-541: irreps, quadrupole, monopole density, |Sz|, Ising map).

CPU: the oracle against golden values evaluated from the reference's own
expressions (tests/golden/make_golden.py), and known answers of the
all-in-all-out state. GPU: the engine against the oracle."""
import json
import os

import numpy as np
import pytest

from cudacode_b200.engine import Engine, System, geometric_ladder
from oracle.binding import Oracle

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                     "reference_order.json")))
AXES = np.array([[1, 1, 1], [-1, -1, 1], [1, -1, -1], [-1, 1, -1]], dtype=np.float64)


def load(o, L, v):
    a = np.zeros(o.spin_shape(), dtype=np.float32)
    a[0, :, :, :3] = np.asarray(v, dtype=np.float32).reshape(16, L ** 3, 3)
    o.set_spins(a)


@pytest.mark.parametrize("fp64", [False, True])
def test_oracle_matches_the_reference_order_parameters(fp64):
    for c in GOLDEN["cases"]:
        L = c["L"]
        o = Oracle([System(L=L, temperatures=[1.0])], fp64=fp64)
        load(o, L, c["spins"])
        np.testing.assert_allclose(o.order_parameters()[0], c["order"], rtol=1e-12, atol=1e-10)
        np.testing.assert_array_equal(o.ising_configuration(0), c["ising"])


def test_all_in_all_out_known_answers():
    L = 3
    N = 16 * L ** 3
    o = Oracle([System(L=L, temperatures=[1.0])], fp64=True)
    v = np.zeros((16, L ** 3, 3))
    for s in range(16):
        v[s] = AXES[s & 3] / np.sqrt(3.0)
    load(o, L, v.reshape(-1, 3))
    q = o.order_parameters()[0]
    assert q[0] == pytest.approx(N, rel=1e-6)          # A2
    np.testing.assert_allclose(q[1:12], 0.0, atol=1e-4)
    np.testing.assert_allclose(q[12:18], 0.0, atol=1e-4)  # isotropic on average
    assert q[18] == pytest.approx(L ** 3 * 4 * np.sqrt(3.0), rel=1e-6)
    assert q[19] == pytest.approx(N, rel=1e-6)
    assert np.all(o.ising_configuration(0) == 0)


@pytest.mark.gpu
def test_engine_matches_oracle():
    temps = geometric_ladder(0.1, 1.0, 5)
    systems = [System(L=6, temperatures=temps), System(L=9, temperatures=temps, J2=0.05)]
    e, o = Engine(systems, seed=31), Oracle(systems, seed=31)
    e.init_random()
    o.init_random()
    for _ in range(2):
        for s in range(2):
            np.testing.assert_allclose(e.order_parameters(s), o.order_parameters(s),
                                       rtol=1e-11, atol=1e-9)
            for r in (0, len(temps) - 1):
                np.testing.assert_array_equal(e.ising_configuration(r, s),
                                              o.ising_configuration(r, s))
        e.cycle(1, 2, True, 3)
        o.cycle(1, 2, True, 3)


@pytest.mark.gpu
def test_engine_matches_the_reference_golden():
    for c in GOLDEN["cases"]:
        L = c["L"]
        e = Engine([System(L=L, temperatures=[1.0])], seed=1)
        a = np.zeros(e.spin_shape(), dtype=np.float32)
        a[0, :, :, :3] = np.asarray(c["spins"], dtype=np.float32).reshape(16, L ** 3, 3)
        e.set_spins(a)
        np.testing.assert_allclose(e.order_parameters()[0], c["order"], rtol=1e-12, atol=1e-10)
        np.testing.assert_array_equal(e.ising_configuration(0), c["ising"])
