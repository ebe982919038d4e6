"""The stream-ordered host copies (pyro_set_cone_async,
pyro_last_observables_async): a driver that queues every step's cone upload,
cycle and energy read before synchronising gets the same chain and the same
per-step energies as the synchronous calls; pageable buffers and the
snapshot mode are refused."""
import numpy as np
import pytest
import torch

from cudacode_b200.engine import Engine, PyroError, System, geometric_ladder

pytestmark = pytest.mark.gpu

PYRO_ERR_ARG, PYRO_ERR_STATE = -1, -6


def make(seed=7):
    temps = geometric_ladder(0.05, 1.5, 6)
    e = Engine([System(L=8, temperatures=temps, J2=0.03)], seed=seed)
    e.init_random()
    return e, len(temps)


def test_queued_steps_equal_synchronous_steps():
    steps = 5
    cones = [np.linspace(-0.5 + 0.1 * k, 0.8, 6).astype(np.float32) for k in range(steps)]
    a, n = make()
    ref_e = []
    for k in range(steps):
        a.set_cone(cones[k])
        a.cycle(1, 2, True, 1)
        ref_e.append(a.last_observables()[0])
    b, _ = make()
    pinned = [torch.from_numpy(c).pin_memory() for c in cones]
    e_h = torch.empty((steps, n), dtype=torch.float64).pin_memory()
    m_h = torch.empty((steps, n, 3), dtype=torch.float64).pin_memory()
    for k in range(steps):
        b.set_cone_async(pinned[k].numpy())
        b.cycle(1, 2, True, 1)
        b.last_observables_async(e_h[k].numpy(), m_h[k].numpy())
    b.synchronize()
    for k in range(steps):
        np.testing.assert_array_equal(e_h[k].numpy(), ref_e[k])
    assert np.array_equal(a.get_spins(), b.get_spins())
    assert np.array_equal(a.permutation(), b.permutation())
    np.testing.assert_array_equal(m_h[-1].numpy(), a.last_observables()[1])


def test_pageable_buffers_and_snapshot_mode_are_refused():
    e, n = make()
    with pytest.raises(PyroError) as err:
        e.set_cone_async(np.full(n, 0.3, dtype=np.float32))
    assert err.value.code == PYRO_ERR_ARG
    bad = torch.full((n,), 1.5, dtype=torch.float32).pin_memory()
    with pytest.raises(PyroError) as err:
        e.set_cone_async(bad.numpy())
    assert err.value.code == PYRO_ERR_ARG
    e.cycle(1, 1, True, 1)
    with pytest.raises(PyroError) as err:
        e.last_observables_async(np.empty(n, dtype=np.float64))
    assert err.value.code == PYRO_ERR_ARG
    e.snapshot()
    e.set_option(e.OPT_MEASURE_SNAPSHOT, 1)
    out = torch.empty(n, dtype=torch.float64).pin_memory()
    with pytest.raises(PyroError) as err:
        e.last_observables_async(out.numpy())
    assert err.value.code == PYRO_ERR_STATE
