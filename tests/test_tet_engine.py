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


OFF_B3 = 6288 - 16  # output biases: per site (mu_x, mu_y, mu_z, log kappa)


@pytest.mark.parametrize("closure,form,T,corner,log_kappa,both", [
    (1, 0, 0.05, 0, [5.5, 1.0, -3.5, 2.0], False),   # sharp and flat vMFs, cold: rejections
    (0, 0, 1.0, 2, [-3.5, -3.5, -3.5, -3.5], True),  # near-uniform proposals, four network vMFs
    (1, 3, 0.5, 3, [-3.0, -3.0, -3.0, 0.0], True),   # tcgen05 network form
    (1, 0, 2.0, 1, [0.5, -3.5, -3.5, -3.5], True)])
def test_learned_move_matches_the_fp64_restatement(closure, form, T, corner, log_kappa, both):
    """One traced pass of the learned move, tetrahedron by tetrahedron,
    against the oracle's FP64 restatement (orc_tet_move_check): the spins and
    external fields it read, its network outputs (BF16 network, to 3% of
    their scale), its vMF draws (the FP64 inverse-CDF draws from the same
    Philox words, to 2e-4), its log Metropolis-Hastings ratio (the FP64
    ratio with both proposal densities and their normalisations, to the
    FP32 rounding of its terms), its test uniform (exact), its decision
    (equal wherever log u is not within the rounding band of log r), its
    beta (the replica's temperature), and the spins it left."""
    L, R, seed = 6, 3, 91
    temps = geometric_ladder(T, 4 * T, R)
    s = System(L=L, temperatures=temps)
    e = Engine([s], seed=seed)
    e.init_random()
    e.cycle(1, 2, True, 2)
    e.tet_init(seed=4)
    w = e.tet_weights()
    w[OFF_B3 + np.array([3, 7, 11, 15])] = log_kappa  # output biases of the four log kappas
    e.tet_set_weights(w)
    e.tet_set_proposal(closure)
    e.tet_sweep(2)  # the traced pass uses counter value 2
    before = e.get_spins()
    rec = e.tet_trace_pass(corner, form)
    after = e.get_spins()
    L3 = L ** 3
    t_of_rep = e.temperatures_of_replicas()
    np.testing.assert_array_equal(rec[:, 0, 55], (1.0 / t_of_rep).astype(np.float32))
    o = Oracle([s], seed=seed)
    o.set_spins(before)
    rec2 = rec.reshape(R * L3, 56)
    for r in range(R):
        feats, spins = o.tet_features(r, corner)
        np.testing.assert_array_equal(rec[r, :, 0:12], spins)
        np.testing.assert_allclose(rec[r, :, 12:24], 3.0 * feats[:, :12], atol=2e-6)
        feats[:, 12] = np.log(rec[r, 0, 55]) / 3.0  # beta of the replica (the oracle's is unswapped)
        net = orc.mlp_forward(w, feats)
        assert np.abs(rec[r, :, 24:40] - net).max() <= 3e-2 * np.abs(net).max()
    rep = np.repeat(np.arange(R), L3)
    cell = np.tile(np.arange(L3), R)
    chk = orc.tet_move_check(rec2, rep, cell, corner, L3, seed, 2, 1.0, closure)
    assert np.abs(rec2[:, 40:52] - chk[:, 5:17]).max() <= 2e-4
    assert np.abs(np.linalg.norm(rec2[:, 40:52].reshape(-1, 4, 3), axis=-1) - 1).max() < 1e-5
    np.testing.assert_array_equal(rec2[:, 54].astype(np.float64), chk[:, 1])
    # tolerance: FP32 rounding of the ratio's terms
    beta = rec2[:, 55].astype(np.float64)
    kap = np.exp(np.clip(rec2[:, 24:40].reshape(-1, 4, 4)[:, :, 3], -4, 6)).sum(axis=1)
    hmag = np.linalg.norm(rec2[:, 12:24].reshape(-1, 4, 3), axis=-1).sum(axis=1)
    scale = 2 * beta * (6 + hmag) + 2 * kap + (4 * beta * (3 + hmag) if closure else 0)
    tol = 4e-6 * scale + 1e-5
    dev = np.abs(rec2[:, 52] - chk[:, 0])
    assert np.all(dev <= tol), (dev.max(), np.argmax(dev - tol))
    u = rec2[:, 54].astype(np.float64)
    clear = np.abs(np.log(u) - chk[:, 0]) > tol
    assert clear.mean() > 0.99
    np.testing.assert_array_equal(rec2[clear, 53], chk[clear, 2])
    acc = rec2[:, 53] > 0.5
    if both:
        assert 0 < acc.sum() < len(acc)  # both outcomes occur
    a = after[:, 4 * corner:4 * corner + 4, :, :3].transpose(0, 2, 1, 3).reshape(R * L3, 12)
    b = before[:, 4 * corner:4 * corner + 4, :, :3].transpose(0, 2, 1, 3).reshape(R * L3, 12)
    np.testing.assert_array_equal(a[acc], rec2[acc, 40:52])
    np.testing.assert_array_equal(a[~acc], b[~acc])
