"""GPU parity at the sizes the benchmark runs: the engine (through the C-ABI)
against the host oracle on the same seeds, bit for bit.

* L = 32 with the kernel schedule that the parallel-tempering benchmark
  times (J1 per-pass kernels on replica groups of 2 dealt to 4 concurrent
  chains, Metropolis one site per thread, over-relaxation one cell per
  thread, programmatic dependent launch, energies fused into each group's
  last pass), 100 sweeps as 20 cycles of 1 Metropolis + 4 over-relaxation
  sweeps with replica exchange; and a shard of 8 replicas at the top of the
  64-temperature ladder, whose Philox keys are the global replica numbers.
* L = 64 with J2 = J3 = 0.05 (16-colour passes, compile-time-offset kernel,
  replica groups), 10 sweeps.
* The 256-system batched configuration (8.7 GB of spins), whose last systems
  lie beyond 4 GiB of spin memory, 2 sweeps; the oracle runs only the last
  two systems, keyed like the engine's.
"""
import numpy as np
import pytest

from cudacode_b200.engine import Engine, System, geometric_ladder
from oracle.binding import Oracle

pytestmark = pytest.mark.gpu

E_RTOL, E_ATOL = 1e-12, 1e-9


def grouped_schedule(e, group=2, chains=4, site_mode=1):
    e.set_option(e.OPT_CYCLE_KERNEL, 0)
    e.set_option(e.OPT_REPLICA_GROUP, group)
    e.set_option(e.OPT_CHAINS, chains)
    e.set_option(e.OPT_J1_SITE_MODE, site_mode)
    e.set_option(e.OPT_PDL, 1)
    e.set_option(e.OPT_FUSED_OBS, 1)


def test_L32_benchmark_schedule_100_sweeps_bit_exact():
    temps = geometric_ladder(0.02, 2.0, 8)
    s = System(L=32, temperatures=temps)
    e = Engine([s], seed=12346)
    o = Oracle([s], seed=12346)
    grouped_schedule(e)
    e.init_random()
    o.init_random()
    cones = np.linspace(-0.8, 0.9, 8).astype(np.float32)
    e.set_cone(cones)
    o.set_cone(cones)
    e.cycle(1, 4, True, 20)
    o.cycle(1, 4, True, 20)
    a, b = e.get_spins(), o.get_spins()
    assert np.abs(a - b).max() <= 1e-5
    assert np.array_equal(a, b), "bit-exact contract"
    assert np.array_equal(e.permutation(), o.permutation())
    assert np.array_equal(e.acceptance()[0], o.acceptance()[0])
    E0, M0 = e.last_observables()
    E1, M1 = o.observables()
    np.testing.assert_allclose(E0, E1, rtol=E_RTOL, atol=E_ATOL)
    np.testing.assert_allclose(M0, M1, rtol=E_RTOL, atol=E_ATOL)
    assert e.sweep_count() == 100


def test_L32_shard_of_the_64_ladder_bit_exact():
    temps = geometric_ladder(0.02, 2.0, 64)
    s = System(L=32, temperatures=temps, n_replicas=8, replica_offset=56)
    e = Engine([s], seed=777)
    o = Oracle([s], seed=777)
    grouped_schedule(e)
    e.init_random()
    o.init_random()
    cones = np.linspace(-0.9, 0.95, 64).astype(np.float32)
    e.set_cone(cones)
    o.set_cone(cones)
    e.cycle(1, 4, False, 4)
    o.cycle(1, 4, False, 4)
    assert np.array_equal(e.get_spins(), o.get_spins())
    assert np.array_equal(e.acceptance()[0], o.acceptance()[0])


def test_L64_further_neighbours_grouped_bit_exact():
    s = System(L=64, temperatures=[0.03, 1.0], J2=0.05, J3=0.05)
    e = Engine([s], seed=4321, renorm_every=5)
    o = Oracle([s], seed=4321, renorm_every=5)
    e.set_option(e.OPT_FAR_KERNEL, 1)
    e.set_option(e.OPT_GROUP_MB, 40)
    e.set_option(e.OPT_CHAINS, 2)
    assert e.info()["n_colours"] == 16
    e.init_random()
    o.init_random()
    cones = np.array([0.6, -0.3], dtype=np.float32)
    e.set_cone(cones)
    o.set_cone(cones)
    e.cycle(1, 1, False, 5)
    o.cycle(1, 1, False, 5)
    assert np.array_equal(e.get_spins(), o.get_spins())
    assert np.array_equal(e.acceptance()[0], o.acceptance()[0])
    E0, _ = e.last_observables()
    E1, _ = o.observables()
    np.testing.assert_allclose(E0, E1, rtol=E_RTOL, atol=E_ATOL)


def batched_systems():
    """The 256 uneven systems of the batched benchmark workload."""
    rng = np.random.default_rng(12345 + 3)
    systems = []
    for _ in range(256):
        L = int(rng.choice([8, 12, 16, 20, 24]))
        nT = int(rng.integers(16, 33))
        j2, j3 = rng.uniform(-0.1, 0.1, 2)
        systems.append(System(L=L, temperatures=geometric_ladder(0.05, 1.5, nT), J2=float(j2),
                              J3=float(j3)))
    return systems


def test_batched_context_beyond_4GiB_last_systems_bit_exact():
    systems = batched_systems()
    spin_bytes = sum(16 * s.n_sites * len(s.temperatures) for s in systems)
    assert spin_bytes > 4 * 2 ** 30
    first_last = sum(16 * s.n_sites * len(s.temperatures) for s in systems[:-2])
    assert first_last > 4 * 2 ** 30  # the two systems checked start beyond 4 GiB
    e = Engine(systems, seed=12348, renorm_every=2)
    e.set_option(e.OPT_FAR_KERNEL, 1)
    e.set_option(e.OPT_GROUP_MB, 40)
    e.set_option(e.OPT_CHAINS, 2)
    e.init_random()
    cones = [np.linspace(-0.5, 0.8, len(s.temperatures)).astype(np.float32) for s in systems]
    for k in range(len(systems)):
        e.set_cone(cones[k], k)
    e.cycle(1, 1, False, 1)
    # The oracle holds only the last two systems. Philox keys are (temperature
    # base of the system + replica); the first of the two gets its engine key
    # through a shard of a ladder padded with the temperatures before it.
    a, b = systems[-2], systems[-1]
    before = sum(len(s.temperatures) for s in systems[:-2])
    pad = [1.0] * before
    oa = System(L=a.L, temperatures=pad + list(a.temperatures), J2=a.J2, J3=a.J3,
                n_replicas=len(a.temperatures), replica_offset=before)
    o = Oracle([oa, b], seed=12348, renorm_every=2)
    o.init_random()
    o.set_cone(np.concatenate([np.zeros(before, np.float32), cones[-2]]), 0)
    o.set_cone(cones[-1], 1)
    o.metropolis_sweep(1)
    o.overrelax_sweep(1)
    for ko, ke in ((0, len(systems) - 2), (1, len(systems) - 1)):
        assert np.array_equal(e.get_spins(ke), o.get_spins(ko)), ke
    e.close()
