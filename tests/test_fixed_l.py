"""The fixed-L per-pass kernels (isotropic J1 systems with L = 16 or 32,
cell decode by shifts, neighbour planes as compile-time offsets) against the
run-time-L kernels and the host oracle, bit for bit: every Metropolis /
over-relaxation form (cell or site per thread), replica groups on chains,
the fused last pass with its FP64 energies, renormalisation and a replica
shard whose Philox keys are global replica numbers.
"""
import numpy as np
import pytest

from cudacode_b200.engine import Engine, System, geometric_ladder
from oracle.binding import Oracle

pytestmark = pytest.mark.gpu


def run(system, seed, fixed, site_mode, group, chains, cycles, renorm=0, fused=1):
    e = Engine([system], seed=seed, renorm_every=renorm)
    assert e.get_option(e.OPT_J1_FIXED_L) == 1  # the default
    e.set_option(e.OPT_J1_FIXED_L, fixed)
    e.set_option(e.OPT_CYCLE_KERNEL, 0)
    e.set_option(e.OPT_J1_SITE_MODE, site_mode)
    e.set_option(e.OPT_REPLICA_GROUP, group)
    e.set_option(e.OPT_CHAINS, chains)
    e.set_option(e.OPT_FUSED_OBS, fused)
    e.init_random()
    n = len(system.temperatures) if system.n_replicas is None else system.n_replicas
    e.set_cone(np.linspace(-0.7, 0.9, len(system.temperatures)).astype(np.float32))
    e.cycle(1, 3, True, cycles)
    out = (e.get_spins(), e.permutation(), e.acceptance()[0], e.last_observables())
    e.close()
    return out, n


@pytest.mark.parametrize("L", [16, 32])
@pytest.mark.parametrize("site_mode", [0, 1, 2, 3])
def test_fixed_equals_runtime_forms(L, site_mode):
    s = System(L=L, temperatures=geometric_ladder(0.05, 1.5, 4))
    (a, pa, aa, (ea, ma)), _ = run(s, 91, 1, site_mode, 2, 2, 3)
    (b, pb, ab, (eb, mb)), _ = run(s, 91, 0, site_mode, 2, 2, 3)
    assert np.array_equal(a, b)
    assert np.array_equal(pa, pb)
    assert np.array_equal(aa, ab)
    np.testing.assert_allclose(ea, eb, rtol=1e-13, atol=1e-10)
    np.testing.assert_allclose(ma, mb, rtol=1e-13, atol=1e-10)


@pytest.mark.parametrize("fused", [0, 1])
def test_fixed_L16_against_oracle_with_renormalisation(fused):
    temps = geometric_ladder(0.04, 2.0, 6)
    s = System(L=16, temperatures=temps)
    seed = 4242
    e = Engine([s], seed=seed, renorm_every=3)
    e.set_option(e.OPT_CYCLE_KERNEL, 0)
    e.set_option(e.OPT_REPLICA_GROUP, 4)
    e.set_option(e.OPT_CHAINS, 2)
    e.set_option(e.OPT_FUSED_OBS, fused)
    o = Oracle([s], seed=seed, renorm_every=3)
    e.init_random()
    o.init_random()
    cones = np.linspace(-0.8, 0.95, len(temps)).astype(np.float32)
    e.set_cone(cones)
    o.set_cone(cones)
    e.cycle(2, 3, True, 4)
    o.cycle(2, 3, True, 4)
    assert np.array_equal(e.get_spins(), o.get_spins()), "bit-exact contract"
    assert np.array_equal(e.permutation(), o.permutation())
    assert np.array_equal(e.acceptance()[0], o.acceptance()[0])
    E0, M0 = e.last_observables()
    E1, M1 = o.observables()
    np.testing.assert_allclose(E0, E1, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(M0, M1, rtol=1e-12, atol=1e-9)


def test_fixed_L32_shard_against_oracle():
    temps = geometric_ladder(0.02, 2.0, 16)
    s = System(L=32, temperatures=temps, n_replicas=3, replica_offset=11)
    e = Engine([s], seed=99)
    o = Oracle([s], seed=99)
    e.set_option(e.OPT_REPLICA_GROUP, 1)
    e.set_option(e.OPT_CHAINS, 3)
    e.init_random()
    o.init_random()
    cones = np.linspace(-0.9, 0.9, len(temps)).astype(np.float32)
    e.set_cone(cones)
    o.set_cone(cones)
    e.cycle(1, 2, False, 2)
    o.cycle(1, 2, False, 2)
    assert np.array_equal(e.get_spins(), o.get_spins())
    assert np.array_equal(e.acceptance()[0], o.acceptance()[0])


@pytest.mark.parametrize("L,cluster", [(16, 16), (16, 4), (32, 16), (32, 8), (32, 2)])
def test_fixed_cluster_cycle_against_oracle(L, cluster):
    """The cluster-resident cycle kernel with the fixed-L cell form (loads
    through L1 between cluster barriers), chained with exchanges."""
    temps = geometric_ladder(0.03, 1.8, 5)
    s = System(L=L, temperatures=temps)
    e = Engine([s], seed=2024 + L, renorm_every=4)
    e.set_option(e.OPT_CYCLE_KERNEL, 1)
    e.set_option(e.OPT_CLUSTER_SIZE, cluster)
    assert e.get_option(e.OPT_CYCLE_KERNEL) == 1
    o = Oracle([s], seed=2024 + L, renorm_every=4)
    e.init_random()
    o.init_random()
    cones = np.linspace(-0.6, 0.9, len(temps)).astype(np.float32)
    e.set_cone(cones)
    o.set_cone(cones)
    e.cycle(1, 4, True, 3)
    o.cycle(1, 4, True, 3)
    assert np.array_equal(e.get_spins(), o.get_spins()), "bit-exact contract"
    assert np.array_equal(e.permutation(), o.permutation())
    assert np.array_equal(e.acceptance()[0], o.acceptance()[0])
    E0, M0 = e.last_observables()
    E1, M1 = o.observables()
    np.testing.assert_allclose(E0, E1, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(M0, M1, rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("stagger", [2, 4, 9])
def test_staggered_chains_give_the_same_chain(stagger):
    """Odd chains starting after their partner's first passes change only
    the timing: spins, permutation and energies as with simultaneous chains
    and as the oracle's."""
    temps = geometric_ladder(0.03, 1.5, 8)
    s = System(L=16, temperatures=temps)
    e = Engine([s], seed=606)
    o = Oracle([s], seed=606)
    e.set_option(e.OPT_REPLICA_GROUP, 1)
    e.set_option(e.OPT_CHAINS, 4)
    e.set_option(e.OPT_CHAIN_STAGGER, stagger)
    assert e.get_option(e.OPT_CHAIN_STAGGER) == stagger
    e.init_random()
    o.init_random()
    cones = np.linspace(-0.7, 0.9, len(temps)).astype(np.float32)
    e.set_cone(cones)
    o.set_cone(cones)
    e.cycle(1, 3, True, 3)
    o.cycle(1, 3, True, 3)
    assert np.array_equal(e.get_spins(), o.get_spins())
    assert np.array_equal(e.permutation(), o.permutation())
    np.testing.assert_allclose(e.last_observables()[0], o.observables()[0], rtol=1e-12, atol=1e-9)
