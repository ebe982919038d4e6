"""GPU checks of the learned tetrahedron proposal: the tensor-core forward
pass and the training gradient against the oracle's FP64 restatement (same
BF16 rounding points), detailed balance of the MH-corrected move against the
plain chain, and maximum-likelihood training lowering the loss."""
import numpy as np
import pytest

from cudacode_b200.engine import Engine, PyroError, System, geometric_ladder
from oracle import binding as orc
from oracle.binding import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tensor_memory", [1, 0])
@pytest.mark.parametrize("n", [1, 128, 300, 5000])
def test_forward_matches_oracle(tensor_memory, n):
    """Both forward kernels (tcgen05 with tensor-memory accumulators, and
    mma.sync) against the FP64 restatement with the same BF16 rounding
    points; ragged row counts included."""
    e = Engine([System(L=4, temperatures=[0.2, 0.5])], seed=3)
    e.tet_init(seed=11)
    e.tet_set_forward(tensor_memory)
    rng = np.random.default_rng(0)
    w = (rng.normal(size=6288) * 0.2).astype(np.float32)
    w[13 * 64:16 * 64] = 0.0
    e.tet_set_weights(w)
    x = rng.normal(size=(n, 16)).astype(np.float32)
    x[:, 13:] = 0.0
    got = e.tet_forward(x)
    want = orc.mlp_forward(w, x)
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err < 2e-3, err


def test_tensor_memory_forward_agrees_with_mma_sync():
    e = Engine([System(L=4, temperatures=[0.2, 0.5])], seed=3)
    e.tet_init(seed=5)
    rng = np.random.default_rng(2)
    x = rng.normal(size=(4096, 16)).astype(np.float32)
    x[:, 13:] = 0.0
    e.tet_set_forward(1)
    a = e.tet_forward(x)
    b = e.tet_forward(x)
    e.tet_set_forward(0)
    c = e.tet_forward(x)
    np.testing.assert_array_equal(a, b)  # deterministic
    assert np.abs(a - c).max() / np.abs(c).max() < 2e-3


def test_gradient_matches_oracle():
    e = Engine([System(L=4, temperatures=[0.2, 0.5])], seed=3)
    e.tet_init(seed=12)
    rng = np.random.default_rng(1)
    w = (rng.normal(size=6288) * 0.15).astype(np.float32)
    w[13 * 64:16 * 64] = 0.0
    e.tet_set_weights(w)
    n = 517  # not a multiple of the 128-sample CTA tile
    x = rng.normal(size=(n, 16)).astype(np.float32)
    x[:, 13:] = 0.0
    s = rng.normal(size=(n, 4, 3))
    s /= np.linalg.norm(s, axis=-1, keepdims=True)
    s = s.reshape(n, 12).astype(np.float32)
    g, loss = e.tet_gradient(x, s)
    g_ref, loss_ref = orc.mlp_gradient(w, x, s)
    assert loss == pytest.approx(loss_ref, rel=1e-3)
    rel = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    cos = float(g @ g_ref / (np.linalg.norm(g) * np.linalg.norm(g_ref)))
    assert rel < 1e-2 and cos > 0.9999, (rel, cos)


def test_collected_features_match_oracle():
    s = System(L=4, temperatures=[0.3, 0.9])
    e = Engine([s], seed=5)
    o = Oracle([s], seed=5)
    e.init_random()
    o.init_random()
    e.tet_init(seed=1, sample_capacity=4 * 2 * 64)
    assert e.tet_collect(stride=1) == 4 * 2 * 64
    f, t = e.tet_samples(4 * 2 * 64)
    f = f.reshape(4, 2, 64, 16)
    t = t.reshape(4, 2, 64, 12)
    for corner in range(4):
        for r in range(2):
            fo, so = o.tet_features(r, corner)
            np.testing.assert_allclose(f[corner, r], fo, rtol=1e-6, atol=1e-6)
            assert np.array_equal(t[corner, r], so)


def chain_energy(e, n_burn, n_meas, step):
    for _ in range(n_burn):
        step()
    es = []
    for _ in range(n_meas):
        step()
        es.append(e.observables()[0])
    return np.array(es)


def mean_and_error(x):
    """Mean and its standard error from batch means (20 batches)."""
    b = x[: len(x) // 20 * 20].reshape(20, -1).mean(axis=1)
    return b.mean(), b.std(ddof=1) / np.sqrt(20)


@pytest.mark.parametrize("form,proposal", [(2, 1), (3, 1), (2, 0), (0, 1)])
def test_learned_move_preserves_the_boltzmann_distribution(form, proposal):
    """Tetrahedron moves alone (untrained network) and the plain method,
    both started from the same equilibrated spins, sample the same energy
    distribution: detailed balance of the MH test (form 3: the network on
    tcgen05; proposal 1: site 3 from its exact conditional, 0: four network
    vMFs)."""
    temps = [0.4, 1.2]
    s = System(L=4, temperatures=temps)
    plain = Engine([s], seed=21)
    plain.init_random()
    plain.tune_cone(0.5, 10, 5)
    for _ in range(300):
        plain.metropolis_sweep(1)
        plain.overrelax_sweep(1)
    start = plain.get_spins()
    e_plain = chain_energy(plain, 0, 2000, lambda: plain.metropolis_sweep(1))
    tet = Engine([s], seed=22)
    tet.set_spins(start)
    tet.tet_init(seed=5)
    tet.tet_set_kernel(form)
    tet.tet_set_proposal(proposal)
    e_tet = chain_energy(tet, 100, 2000, lambda: tet.tet_sweep(1))
    acc, prop = tet.tet_acceptance()
    assert (acc > 0).all()
    for k in range(2):
        m1, s1 = mean_and_error(e_plain[:, k])
        m2, s2 = mean_and_error(e_tet[:, k])
        assert abs(m1 - m2) < 4.0 * np.hypot(s1, s2) + 1e-9, (k, m1, s1, m2, s2)


def test_training_lowers_the_loss_and_raises_acceptance():
    s = System(L=6, temperatures=geometric_ladder(0.05, 0.5, 4))
    e = Engine([s], seed=8)
    e.init_random()
    e.tune_cone(0.5, 10, 5, 2)
    e.tet_init(seed=3, sample_capacity=200_000)
    for _ in range(20):
        e.cycle(1, 4, True, 5)
        e.tet_collect(stride=1)
    first = e.tet_train(1, batch=4096, lr=2e-3)
    e.tet_reset_acceptance()
    e.tet_sweep(5)
    a0, p0 = e.tet_acceptance()
    last = e.tet_train(600, batch=4096, lr=2e-3)
    assert last < first - 1.0, (first, last)
    e.tet_reset_acceptance()
    e.tet_sweep(5)
    a1, p1 = e.tet_acceptance()
    assert (a1 / p1).mean() > (a0 / p0).mean(), (a0 / p0, a1 / p1)
    # drawing site 3 from its exact conditional accepts more often than the
    # network's fourth vMF (same network, same states)
    saved = e.get_spins()
    e.tet_set_proposal(0)
    e.tet_reset_acceptance()
    e.tet_sweep(5)
    a2, p2 = e.tet_acceptance()
    e.set_spins(saved)
    e.tet_set_proposal(1)
    assert (a1 / p1).mean() > (a2 / p2).mean(), (a1 / p1, a2 / p2)
    # the trained move alone still samples the plain chain's distribution:
    # replica perm[t] holds temperature slot t in `e`; the plain chain gets
    # the same configurations with replica t at slot t.
    start = e.get_spins()
    perm = e.permutation()
    plain = Engine([s], seed=9)
    plain.set_spins(start[perm])
    plain.set_cone(e.get_cone())
    plain_E = chain_energy(plain, 50, 4000, lambda: (plain.metropolis_sweep(1),
                                                     plain.overrelax_sweep(2)))
    tet_E = chain_energy(e, 50, 4000, lambda: e.tet_sweep(1))
    assert np.array_equal(perm, e.permutation())  # no exchanges in either chain
    for t in range(4):
        m1, s1 = mean_and_error(plain_E[:, t])
        m2, s2 = mean_and_error(tet_E[:, perm[t]])
        assert abs(m1 - m2) < 4.0 * np.hypot(s1, s2) + 1e-6, (t, m1, s1, m2, s2)


def test_learned_move_requires_j1_only():
    e = Engine([System(L=3, temperatures=[1.0], J2=0.1)])
    with pytest.raises(PyroError):
        e.tet_init()


@pytest.mark.parametrize("L,proposal", [(4, 1), (7, 1), (16, 1), (7, 0)])
def test_cluster_and_per_pass_tet_kernels_agree(L, proposal):
    s = System(L=L, temperatures=[0.1, 0.3, 0.9])
    runs = []
    for cluster in (0, 1, 2):
        e = Engine([s], seed=41)
        e.init_random()
        e.tet_init(seed=2)
        e.tet_set_kernel(cluster)
        e.tet_set_proposal(proposal)
        e.tet_sweep(3)
        e.cycle_tet(1, 1, 2, True, 2)
        runs.append((e.get_spins(), e.tet_acceptance()[0], e.permutation()))
    for k in (1, 2):
        assert np.array_equal(runs[0][0], runs[k][0])
        assert np.array_equal(runs[0][1], runs[k][1])
        assert np.array_equal(runs[0][2], runs[k][2])


@pytest.mark.parametrize("L", [4, 7])
def test_tensor_memory_move_matches_the_mma_sync_move_closely(L):
    """Form 3 evaluates the same network on tcgen05; its accumulations round
    differently, so the chains are not bit-identical, but one sweep from the
    same state accepts almost the same moves and all spins stay unit."""
    s = System(L=L, temperatures=[0.1, 0.3, 0.9])
    runs = []
    for form in (0, 3):
        e = Engine([s], seed=41)
        e.init_random()
        e.tet_init(seed=2)
        e.tet_set_kernel(form)
        e.tet_sweep(1)
        acc, prop = e.tet_acceptance()
        runs.append((e.get_spins(), acc, prop))
    a, b = runs[0][0], runs[1][0]
    same = np.all(a == b, axis=-1)
    assert same.mean() > 0.99
    n = np.linalg.norm(b[..., :3], axis=-1)
    assert np.abs(n - 1).max() < 1e-4
    assert np.abs(runs[0][1].astype(np.int64) - runs[1][1].astype(np.int64)).max() <= \
        max(2, int(0.01 * runs[0][2][0]))


@pytest.mark.parametrize("form,group,chains", [(2, 2, 3), (2, 3, 2), (0, 1, 4), (1, 2, 2),
                                               (3, 4, 2)])
def test_learned_sweeps_in_replica_groups_match_ungrouped(form, group, chains):
    """Learned sweeps run inside the replica groups (each group's after its
    plain sweeps, on its chain) give the same chain, bit for bit, as the
    learned sweeps over all replicas after every group's plain sweeps."""
    systems = [System(L=5, temperatures=geometric_ladder(0.05, 0.5, 7)),
               System(L=4, temperatures=[0.1, 0.3, 0.9], J2=0.05),
               System(L=6, temperatures=[0.08, 0.2])]
    runs = []
    for grouped in (0, 1):
        e = Engine(systems, seed=43)
        e.init_random()
        e.tet_init(seed=4)
        e.tet_set_kernel(form)
        e.set_option(e.OPT_REPLICA_GROUP, group)
        e.set_option(e.OPT_CHAINS, chains)
        e.set_option(e.OPT_TET_GROUPED, grouped)
        assert e.get_option(e.OPT_TET_GROUPED) == grouped
        e.cycle_tet(1, 1, 1, True, 3)
        e.cycle_tet(0, 1, 2, True, 2)
        e.cycle(1, 2, True, 1)
        runs.append([(e.get_spins(k), e.tet_acceptance(k)[0], e.permutation(k),
                      *e.last_observables(k)) for k in range(len(systems))])
    for k in range(len(systems)):
        for a, b in zip(runs[0][k], runs[1][k]):
            assert np.array_equal(a, b), k
