"""GPU parity: the CUDA engine (through the C-ABI) against the host oracle on
the same seeded inputs. The update arithmetic is specified bit-for-bit
(include/pyro_math.h), so per-spin agreement is expected to be exact; the
asserted bound is the 1e-5 per component over the first 100 sweeps that the
engine promises. FP64 observables differ only by summation order: rel 1e-12."""
import numpy as np
import pytest

from cudacode_b200.engine import Engine, PyroError, System, geometric_ladder
from oracle.binding import Oracle

pytestmark = pytest.mark.gpu

SPIN_TOL = 1e-5


def pair(systems, seed=2024, renorm_every=0):
    e = Engine(systems, seed=seed, renorm_every=renorm_every)
    o = Oracle(systems, seed=seed, renorm_every=renorm_every)
    return e, o


def assert_spins_equal(e, o, n_sys=1):
    for k in range(n_sys):
        a, b = e.get_spins(k), o.get_spins(k)
        diff = np.abs(a - b).max()
        assert diff <= SPIN_TOL, (k, diff)
    return diff


def test_init_random_bit_exact():
    systems = [System(L=4, temperatures=[0.5, 1.0]), System(L=3, temperatures=[1.0], J2=0.1)]
    e, o = pair(systems)
    e.init_random()
    o.init_random()
    for k in range(2):
        assert np.array_equal(e.get_spins(k), o.get_spins(k))
    n = np.linalg.norm(e.get_spins(0)[..., :3], axis=-1)
    assert np.abs(n - 1).max() < 1e-6


@pytest.mark.parametrize("L,R", [(4, 1), (8, 3)])
def test_plain_sweeps_100_per_spin(L, R):
    temps = geometric_ladder(0.1, 2.0, R)
    e, o = pair([System(L=L, temperatures=temps)], renorm_every=7)
    e.init_random()
    o.init_random()
    cones = np.linspace(-0.5, 0.9, R).astype(np.float32)
    e.set_cone(cones)
    o.set_cone(cones)
    for k in range(20):  # 20 x (1 M + 4 OR) = 100 sweeps
        e.metropolis_sweep(1)
        o.metropolis_sweep(1)
        e.overrelax_sweep(4)
        o.overrelax_sweep(4)
    a, b = e.get_spins(), o.get_spins()
    assert np.abs(a - b).max() <= SPIN_TOL
    assert np.array_equal(a, b), "bit-exact contract"
    acc_e, prop_e = e.acceptance()
    acc_o, prop_o = o.acceptance()
    assert np.array_equal(acc_e, acc_o) and np.array_equal(prop_e, prop_o)
    assert e.sweep_count() == o.sweep_count() == 100


@pytest.mark.parametrize("far", [0, 1])
def test_further_neighbour_sixteen_colours(far):
    s = System(L=4, temperatures=[0.2, 0.7], J1=1.0, J2=-0.08, J3=0.06, J3b=0.03)
    e, o = pair([s])
    e.set_option(e.OPT_FAR_KERNEL, far)
    assert e.info()["n_colours"] == 16
    e.init_random()
    o.init_random()
    c = np.array([0.3, -0.2], dtype=np.float32)
    e.set_cone(c)
    o.set_cone(c)
    for _ in range(10):
        e.metropolis_sweep(1)
        o.metropolis_sweep(1)
        e.overrelax_sweep(2)
        o.overrelax_sweep(2)
    assert np.array_equal(e.get_spins(), o.get_spins())


def test_batched_uneven_systems():
    rng = np.random.default_rng(5)
    systems = []
    for L in (3, 4, 5, 4):
        nT = int(rng.integers(2, 5))
        j2, j3 = rng.uniform(-0.1, 0.1, 2) if L != 5 else (0.0, 0.0)
        systems.append(System(L=L, temperatures=geometric_ladder(0.05, 1.5, nT), J2=j2, J3=j3))
    e, o = pair(systems, renorm_every=5)
    e.init_random()
    o.init_random()
    for k, s in enumerate(systems):
        c = np.linspace(0.0, 0.8, len(s.temperatures)).astype(np.float32)
        e.set_cone(c, k)
        o.set_cone(c, k)
    for _ in range(6):
        e.metropolis_sweep(1)
        o.metropolis_sweep(1)
        e.overrelax_sweep(2)
        o.overrelax_sweep(2)
    for k in range(len(systems)):
        assert np.array_equal(e.get_spins(k), o.get_spins(k)), k


def test_observables_fp64():
    s = System(L=6, temperatures=[0.3, 0.9, 2.0], J2=0.05, J3=-0.04)
    e, o = pair([s])
    e.init_random()
    o.init_random()
    e.metropolis_sweep(3)
    o.metropolis_sweep(3)
    E1, M1 = e.observables()
    E2, M2 = o.observables()
    np.testing.assert_allclose(E1, E2, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(M1, M2, rtol=1e-12, atol=1e-9)


def test_parallel_tempering_swaps_match():
    temps = geometric_ladder(0.05, 2.0, 8)
    e, o = pair([System(L=4, temperatures=temps)])
    e.init_random()
    o.init_random()
    total = 0
    for k in range(12):
        e.metropolis_sweep(1)
        o.metropolis_sweep(1)
        e.overrelax_sweep(1)
        o.overrelax_sweep(1)
        n1 = e.pt_swap(-1)
        n2 = o.pt_swap(-1)
        assert n1 == n2
        total += n1
        assert np.array_equal(e.permutation(), o.permutation())
    assert total > 0
    assert np.array_equal(e.get_spins(), o.get_spins())
    T = e.temperatures_of_replicas()
    assert sorted(T) == pytest.approx(temps)


def test_graph_cycle_matches_oracle():
    temps = geometric_ladder(0.02, 2.0, 6)
    e, o = pair([System(L=4, temperatures=temps)], renorm_every=10)
    e.init_random()
    o.init_random()
    c = np.linspace(-1.0, 0.95, 6).astype(np.float32)
    e.set_cone(c)
    o.set_cone(c)
    e.enable_history(64)
    e.cycle(1, 4, True, 20)
    h_o = o.cycle(1, 4, True, 20, record=True)
    assert np.array_equal(e.get_spins(), o.get_spins())
    assert np.array_equal(e.permutation(), o.permutation())
    h_e = e.history()
    assert h_e.shape == (20, 6)
    np.testing.assert_allclose(h_e, h_o, rtol=1e-12, atol=1e-9)
    assert e.sweep_count() == 100


def test_tune_cone_matches_oracle():
    temps = [0.1, 0.5, 3.0]
    e, o = pair([System(L=4, temperatures=temps)])
    e.init_random()
    o.init_random()
    e.tune_cone(0.5, 8, 3, 1)
    o.tune_cone(0.5, 8, 3, 1)
    assert np.array_equal(e.get_cone(), o.get_cone())
    assert np.array_equal(e.get_spins(), o.get_spins())


def test_sharded_contexts_equal_unsharded():
    torch = pytest.importorskip("torch")
    temps = geometric_ladder(0.05, 1.0, 6)
    full = Engine([System(L=4, temperatures=temps)], seed=77)
    halves = [Engine([System(L=4, temperatures=temps, n_replicas=3, replica_offset=3 * r)], seed=77)
              for r in range(2)]
    full.init_random()
    for h in halves:
        h.init_random()
    e_all = torch.zeros(6, dtype=torch.float64, device="cuda")
    for k in range(6):
        full.cycle(1, 2, False, 1)
        full.pt_swap(-1)
        for r, h in enumerate(halves):
            h.cycle(1, 2, False, 1)
            h.observables_device(e_all.data_ptr() + 8 * 3 * r)
            h.synchronize()
        for h in halves:
            h.pt_swap_global(e_all.data_ptr(), -1)
        for h in halves:
            assert np.array_equal(h.permutation(), full.permutation())
    f = full.get_spins()
    for r, h in enumerate(halves):
        assert np.array_equal(h.get_spins(), f[3 * r:3 * r + 3])


def test_determinism_two_runs():
    def run():
        e = Engine([System(L=5, temperatures=[0.2, 0.4])], seed=11)
        e.init_random()
        e.tune_cone(0.5, 3, 2)
        e.cycle(1, 3, True, 5)
        return e.get_spins(), e.observables()[0]
    (a, ea), (b, eb) = run(), run()
    assert np.array_equal(a, b) and np.array_equal(ea, eb)


def test_errors_are_reported():
    with pytest.raises(PyroError):
        Engine([System(L=1, temperatures=[1.0])])
    with pytest.raises(PyroError):
        Engine([System(L=4, temperatures=[1.0, 0.5])])  # not increasing
    e = Engine([System(L=4, temperatures=[1.0, 2.0])])
    with pytest.raises(PyroError):
        e.set_cone(np.array([2.0, 0.0], dtype=np.float32))
    with pytest.raises(PyroError):
        e.metropolis_sweep(-1)
    sh = Engine([System(L=4, temperatures=[1.0, 2.0], n_replicas=1)])
    with pytest.raises(PyroError):
        sh.pt_swap()
    with pytest.raises(PyroError):
        sh.cycle(1, 1, True, 1)


def test_check_spins_flags_planted_nan():
    e = Engine([System(L=3, temperatures=[1.0])])
    e.init_random()
    assert e.check_spins() == -1
    s = e.get_spins()
    s[0, 5, 7, 1] = np.nan
    e.set_spins(s)
    assert e.check_spins() == 5 * 27 + 7


@pytest.mark.parametrize("specialised,site_mode", [(0, 0), (1, 0), (1, 1), (1, 2), (1, 3)])
def test_j1_kernel_variants_bit_exact(specialised, site_mode):
    temps = geometric_ladder(0.05, 1.0, 3)
    e, o = pair([System(L=6, temperatures=temps)], renorm_every=3)
    e.set_option(e.OPT_J1_KERNEL, specialised)
    e.set_option(e.OPT_J1_SITE_MODE, site_mode)
    e.init_random()
    o.init_random()
    c = np.array([0.6, 0.1, -0.7], dtype=np.float32)
    e.set_cone(c)
    o.set_cone(c)
    for _ in range(5):
        e.metropolis_sweep(1)
        o.metropolis_sweep(1)
        e.overrelax_sweep(3)
        o.overrelax_sweep(3)
    assert np.array_equal(e.get_spins(), o.get_spins())
    E1, M1 = e.observables()
    E2, M2 = o.observables()
    np.testing.assert_allclose(E1, E2, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(M1, M2, rtol=1e-12, atol=1e-9)
    a1, _ = e.acceptance()
    a2, _ = o.acceptance()
    assert np.array_equal(a1, a2)


def test_mixed_j1_and_further_neighbour_systems():
    systems = [System(L=4, temperatures=[0.3, 0.8]),
               System(L=3, temperatures=[0.5, 1.0, 2.0], J2=0.04, J3=-0.02),
               System(L=5, temperatures=[1.0])]
    e, o = pair(systems, renorm_every=4)
    e.init_random()
    o.init_random()
    e.cycle(1, 3, True, 4)
    o.cycle(1, 3, True, 4)
    for k in range(3):
        assert np.array_equal(e.get_spins(k), o.get_spins(k)), k
        np.testing.assert_allclose(e.observables(k)[0], o.observables(k)[0], rtol=1e-12)
        assert np.array_equal(e.permutation(k), o.permutation(k))


@pytest.mark.parametrize("cs", [16, 8, 4, 2])
def test_cluster_cycle_kernel_bit_exact(cs):
    temps = geometric_ladder(0.03, 1.5, 5)
    e, o = pair([System(L=8, temperatures=temps)], renorm_every=6)
    e.set_option(e.OPT_CYCLE_KERNEL, 1)
    e.set_option(e.OPT_CLUSTER_SIZE, cs)
    e.init_random()
    o.init_random()
    c = np.linspace(-0.9, 0.9, 5).astype(np.float32)
    e.set_cone(c)
    o.set_cone(c)
    e.enable_history(16)
    e.cycle(1, 4, True, 6)
    h = o.cycle(1, 4, True, 6, record=True)
    assert np.array_equal(e.get_spins(), o.get_spins())
    assert np.array_equal(e.permutation(), o.permutation())
    np.testing.assert_allclose(e.history(), h, rtol=1e-12, atol=1e-9)
    e.metropolis_sweep(2)
    o.metropolis_sweep(2)
    e.overrelax_sweep(3)
    o.overrelax_sweep(3)
    assert np.array_equal(e.get_spins(), o.get_spins())
    assert np.array_equal(e.acceptance()[0], o.acceptance()[0])
    assert e.get_option(e.OPT_CYCLE_KERNEL) == 1
    assert e.get_option(e.OPT_CLUSTER_SIZE) <= cs


@pytest.mark.parametrize("group,chains", [(1, 1), (2, 1), (3, 1), (1, 2), (2, 4)])
def test_replica_groups_bit_exact(group, chains):
    temps = geometric_ladder(0.05, 1.0, 5)
    e, o = pair([System(L=6, temperatures=temps)], renorm_every=3)
    e.set_option(e.OPT_REPLICA_GROUP, group)
    e.set_option(e.OPT_CHAINS, chains)
    e.init_random()
    o.init_random()
    e.cycle(1, 3, True, 4)
    o.cycle(1, 3, True, 4)
    assert np.array_equal(e.get_spins(), o.get_spins())
    assert np.array_equal(e.permutation(), o.permutation())


@pytest.mark.parametrize("mb,chains", [(1, 1), (1, 2), (3, 3)])
def test_generic_groups_bit_exact(mb, chains):
    rng = np.random.default_rng(3)
    systems = [System(L=L, temperatures=geometric_ladder(0.05, 1.5, nt), J2=float(j2), J3=float(j3))
               for L, nt, (j2, j3) in [(4, 5, rng.uniform(-0.1, 0.1, 2)), (5, 3, (0.05, 0.02)),
                                       (3, 4, (-0.03, 0.06))]]
    systems.append(System(L=4, temperatures=[0.2, 0.5, 1.0]))  # J1 system in the same context
    e, o = pair(systems, renorm_every=4)
    e.set_option(e.OPT_GROUP_MB, mb)
    e.set_option(e.OPT_CHAINS, chains)
    e.set_option(e.OPT_REPLICA_GROUP, 2)
    e.init_random()
    o.init_random()
    e.cycle(1, 3, True, 3)
    o.cycle(1, 3, True, 3)
    for k in range(len(systems)):
        assert np.array_equal(e.get_spins(k), o.get_spins(k)), k
        assert np.array_equal(e.permutation(k), o.permutation(k)), k


def test_autotune_keeps_results_exact():
    temps = geometric_ladder(0.05, 1.0, 4)
    e, o = pair([System(L=8, temperatures=temps)])
    e.init_random()
    o.init_random()
    chosen = e.autotune(1, 2, 2)
    assert chosen >= 0
    # every variant ran 1 + 2 cycles of (1 M + 2 OR + swap); replay the same count on the oracle
    n_cycles = e.sweep_count() // 3
    o.cycle(1, 2, True, n_cycles)
    assert np.array_equal(e.get_spins(), o.get_spins())
    assert np.array_equal(e.permutation(), o.permutation())


@pytest.mark.parametrize("L,G,stride,replica", [(4, 8, 1, -1), (4, 16, 1, 0), (6, 6, 4, 1),
                                               (3, 12, 1, -1),
                                               (8, 4, 1, -1),    # fold period 8 >= G: no residues
                                               (5, 10, 3, -1),   # stride coprime with L, residues
                                               (8, 6, 2, 0),     # fold period 4 < G
                                               (12, 8, 3, 2)])   # fold period 4, one replica
def test_structure_factor_matches_direct_sum(L, G, stride, replica):
    s = System(L=L, temperatures=[0.2, 0.6, 1.4], J2=0.05 if L == 3 else 0.0)
    e, o = pair([s])
    e.init_random()
    o.init_random()
    e.cycle(1, 2, True, 3)
    o.cycle(1, 2, True, 3)
    a = e.structure_factor(G, stride, replica)
    b = o.structure_factor(G, stride, replica)
    np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-9)
    if stride == 1 and G == 4 * L:
        spins = e.get_spins()[..., :3].astype(np.float64)
        sel = spins if replica < 0 else spins[replica:replica + 1]
        assert a.sum() == pytest.approx((4 * L) ** 3 * (sel ** 2).sum() / (16 * L ** 3) /
                                        sel.shape[0], rel=1e-9)


@pytest.mark.parametrize("L,J2,J3", [(4, 0.0, 0.0), (8, 0.0, 0.0), (5, 0.06, -0.04), (3, 0.0, 0.0),
                                     (6, 0.0, 0.0), (7, 0.0, 0.0)])
def test_shared_memory_cycles_bit_exact(L, J2, J3):
    temps = geometric_ladder(0.1, 1.0, 3)
    e, o = pair([System(L=L, temperatures=temps, J2=J2, J3=J3)], renorm_every=4)
    assert e.get_option(e.OPT_SMEM_KERNEL) == 1
    e.init_random()
    o.init_random()
    c = np.array([0.7, 0.2, -0.6], dtype=np.float32)
    e.set_cone(c)
    o.set_cone(c)
    e.enable_history(32)
    e.cycle(1, 5, False, 7)
    h = o.cycle(1, 5, False, 7, record=True)
    assert np.array_equal(e.get_spins(), o.get_spins())
    assert np.array_equal(e.acceptance()[0], o.acceptance()[0])
    np.testing.assert_allclose(e.history(), h, rtol=1e-12, atol=1e-9)
    assert e.sweep_count() == 42
    # the next call continues the same chain on the other kernels
    e.set_option(e.OPT_SMEM_KERNEL, 0)
    e.cycle(1, 5, False, 2)
    o.cycle(1, 5, False, 2)
    assert np.array_equal(e.get_spins(), o.get_spins())


@pytest.mark.parametrize("pdl, site_mode", [(0, 1), (1, 1), (1, 0), (1, 3)])
def test_programmatic_dependent_launch_keeps_the_chain(pdl, site_mode):
    temps = geometric_ladder(0.1, 1.5, 8)
    s = System(L=9, temperatures=temps)
    e, o = pair([s])
    e.set_option(e.OPT_PDL, pdl)
    e.set_option(e.OPT_J1_SITE_MODE, site_mode)
    e.set_option(e.OPT_REPLICA_GROUP, 2)
    e.set_option(e.OPT_CHAINS, 3)
    assert e.get_option(e.OPT_PDL) == pdl
    e.init_random()
    o.init_random()
    e.cycle(1, 4, True, 6)
    o.cycle(1, 4, True, 6)
    assert np.array_equal(e.get_spins(), o.get_spins())
    assert np.array_equal(e.permutation(), o.permutation())


@pytest.mark.parametrize("L", [6, 12])  # shared-memory cycles (L <= 8) and per-pass cycles
def test_sharded_backend_reuses_the_cycle_energies(L):
    """The sharded driver's engine backend takes the energies that the cycle
    computed (pyro_last_observables_device) instead of recomputing them; two
    shards in one process, their all-gather emulated by concatenation,
    reproduce the unsharded run bit for bit."""
    torch = pytest.importorskip("torch")
    from cudacode_b200.distributed import EngineBackend
    temps = geometric_ladder(0.05, 1.0, 6)
    full = Engine([System(L=L, temperatures=temps)], seed=91)
    shards = [Engine([System(L=L, temperatures=temps, n_replicas=3, replica_offset=3 * r)],
                     seed=91) for r in range(2)]
    full.init_random()
    backends = []
    for s in shards:
        s.init_random()
        backends.append(EngineBackend(s, torch.device("cuda")))
    for _ in range(5):
        full.cycle(1, 2, False, 1)
        full.pt_swap(-1)
        for b in backends:
            b.sweeps(1, 2)
        e_all = torch.cat([b.local_energies().clone() for b in backends])
        e_full, _ = full.observables()
        assert np.array_equal(e_all.cpu().numpy(), e_full) or \
            np.allclose(e_all.cpu().numpy(), e_full, rtol=1e-12)
        for b in backends:
            b.swap_global(e_all, -1)
        for s in shards:
            assert np.array_equal(s.permutation(), full.permutation())
    f = full.get_spins()
    for r, s in enumerate(shards):
        assert np.array_equal(s.get_spins(), f[3 * r:3 * r + 3])


@pytest.mark.parametrize("L, swap, group", [(9, True, 0), (9, True, 2), (6, False, 0)])
def test_last_observables_are_the_cycle_energies(L, swap, group):
    s = System(L=L, temperatures=geometric_ladder(0.1, 1.0, 4))
    e = Engine([s], seed=5)
    e.set_option(e.OPT_REPLICA_GROUP, group)
    e.init_random()
    e.cycle(1, 2, swap, 3)
    E0, M0 = e.last_observables()
    E1, M1 = e.observables()
    np.testing.assert_allclose(E0, E1, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(M0, M1.reshape(-1, 3), rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("L,n_metro,n_or,site_mode,group,chains",
                         [(6, 1, 3, 1, 2, 2), (5, 2, 0, 0, 3, 1), (8, 1, 1, 0, 4, 3)])
def test_energies_from_the_last_pass(L, n_metro, n_or, site_mode, group, chains):
    """The energies and magnetisations a replica group's last colour pass
    computes (fused) equal a separate lattice-wide evaluation to FP64
    rounding, and the chain (spins, exchange decisions) equals the one with
    the separate observables kernel and the oracle's."""
    temps = geometric_ladder(0.05, 1.0, 7)
    runs = []
    for fused in (1, 0):
        e, o = pair([System(L=L, temperatures=temps)], renorm_every=3)
        e.set_option(e.OPT_REPLICA_GROUP, group)
        e.set_option(e.OPT_CHAINS, chains)
        e.set_option(e.OPT_J1_SITE_MODE, site_mode)
        e.set_option(e.OPT_FUSED_OBS, fused)
        assert e.get_option(e.OPT_FUSED_OBS) == fused
        e.init_random()
        o.init_random()
        e.cycle(n_metro, n_or, True, 4)
        o.cycle(n_metro, n_or, True, 4)
        assert np.array_equal(e.get_spins(), o.get_spins())
        assert np.array_equal(e.permutation(), o.permutation())
        E0, M0 = e.last_observables()
        E1, M1 = e.observables()
        np.testing.assert_allclose(E0, E1, rtol=1e-12, atol=1e-9)
        np.testing.assert_allclose(M0, M1.reshape(-1, 3), rtol=1e-12, atol=1e-9)
        runs.append((e.get_spins(), E0))
    assert np.array_equal(runs[0][0], runs[1][0])
    np.testing.assert_allclose(runs[0][1], runs[1][1], rtol=1e-12, atol=1e-9)


def test_option_and_proposal_values_are_checked():
    e = Engine([System(L=4, temperatures=[0.5, 1.0])])
    for opt in (e.OPT_TET_GROUPED, e.OPT_FUSED_OBS, e.OPT_PDL):
        with pytest.raises(PyroError):
            e.set_option(opt, 2)
        with pytest.raises(PyroError):
            e.set_option(opt, -1)
    with pytest.raises(PyroError):  # the learned move is not initialised yet
        e.tet_set_proposal(1)
    with pytest.raises(PyroError):
        e.cycle_tet(1, 1, 1, True, 1)
    e.tet_init(seed=1)
    for bad in (-1, 2):
        with pytest.raises(PyroError):
            e.tet_set_proposal(bad)
    e.tet_set_proposal(0)
    e.tet_set_proposal(1)


def test_spins_in_the_reference_layout():
    """pyro_set/get_spins_planar use the reference's layout: per replica the
    x, y and z planes of 16 L^3 values (site index s L^3 + cell)."""
    s = System(L=3, temperatures=[0.5, 1.0, 2.0])
    e = Engine([s], seed=4)
    e.init_random()
    f4 = e.get_spins()                        # [R][16][L^3][4]
    planes = e.get_spins_planar()             # [R][3][16 L^3]
    R = f4.shape[0]
    expect = f4[..., :3].reshape(R, 16 * 27, 3).transpose(0, 2, 1)
    assert np.array_equal(planes, expect.astype(np.float64))
    rng = np.random.default_rng(2)
    v = rng.normal(size=(R, 3, 16 * 27))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    e.set_spins_planar(v)
    back = e.get_spins()
    assert np.array_equal(back[..., :3].reshape(R, 16 * 27, 3),
                          v.transpose(0, 2, 1).astype(np.float32))
    assert np.all(back[..., 3] == 0.0)
    with pytest.raises(ValueError):
        e.set_spins_planar(v[:, :2])


def test_a_subset_of_systems_with_the_full_sets_keys_reproduces_their_chains():
    """One rank's share of independent systems: a context holding systems 1
    and 3 of a batch, with the Philox keys they have in the whole batch
    (pyro_set_system_keys), reproduces their chains bit for bit."""
    from cudacode_b200.distributed import system_keys
    systems = [System(L=L, temperatures=geometric_ladder(0.1, 1.5, n), J2=j2)
               for L, n, j2 in [(4, 3, 0.0), (5, 4, 0.05), (6, 2, 0.0), (8, 3, 0.0)]]
    full = Engine(systems, seed=31)
    full.init_random()
    full.cycle(1, 3, True, 5)
    keys = system_keys(systems)
    part = Engine([systems[1], systems[3]], seed=31)
    for j, gi in enumerate((1, 3)):
        part.set_system_keys(j, *keys[gi])
    part.init_random()
    part.cycle(1, 3, True, 5)
    for j, gi in enumerate((1, 3)):
        assert np.array_equal(part.get_spins(j), full.get_spins(gi)), gi
        assert np.array_equal(part.permutation(j), full.permutation(gi)), gi
