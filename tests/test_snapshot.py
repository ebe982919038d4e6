"""Measurement snapshots (pyro_snapshot, PYRO_OPT_MEASURE_SNAPSHOT): the
measurement calls read a copy of the state taken between cycles, on the
context's measurement stream, while later cycles run. What they return
equals a synchronous measurement of the same state in an identical context,
and the Monte Carlo chain is unchanged by the snapshot."""
import numpy as np
import pytest

from cudacode_b200.engine import Engine, PyroError, System, geometric_ladder

pytestmark = pytest.mark.gpu


def measurements(e):
    E, M = e.last_observables()
    return {"E": E, "M": M, "T": e.temperatures_of_replicas(), "perm": e.permutation(),
            "op": e.order_parameters(), "sub": e.sublattice_magnetisation(),
            "sq": e.structure_factor(8, 1), "ising": e.ising_configuration(2)}


@pytest.mark.parametrize("cycle_kernel", [0, 2])
def test_snapshot_measurements_equal_synchronous_ones_and_keep_the_chain(cycle_kernel):
    s = System(L=8, temperatures=geometric_ladder(0.1, 1.5, 6))
    a, b = Engine([s], seed=13), Engine([s], seed=13)
    for e in (a, b):
        e.set_option(e.OPT_CYCLE_KERNEL, cycle_kernel)
        e.init_random()
        e.cycle(1, 3, True, 3)
    want = measurements(b)
    a.snapshot()
    a.cycle(1, 3, True, 4)  # queued behind the snapshot's copy
    a.set_option(a.OPT_MEASURE_SNAPSHOT, 1)
    assert a.get_option(a.OPT_MEASURE_SNAPSHOT) == 1
    got = measurements(a)
    a.set_option(a.OPT_MEASURE_SNAPSHOT, 0)
    for k in want:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    b.cycle(1, 3, True, 4)
    assert np.array_equal(a.get_spins(), b.get_spins())
    assert np.array_equal(a.permutation(), b.permutation())
    # a second snapshot replaces the first
    a.snapshot()
    a.set_option(a.OPT_MEASURE_SNAPSHOT, 1)
    np.testing.assert_array_equal(a.order_parameters(), b.order_parameters())
    a.set_option(a.OPT_MEASURE_SNAPSHOT, 0)


def test_snapshot_mode_needs_a_snapshot():
    e = Engine([System(L=4, temperatures=[0.5, 1.0])], seed=2)
    with pytest.raises(PyroError):
        e.set_option(e.OPT_MEASURE_SNAPSHOT, 1)
    with pytest.raises(PyroError):
        e.set_option(e.OPT_MEASURE_SNAPSHOT, 2)
