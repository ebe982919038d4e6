"""GPU parity of the work-queue cycle kernel (PYRO_OPT_CYCLE_KERNEL = 2):
one launch per J1 system per cycle, items (pass, chunk, replica) that wait
on per-chunk progress counters of the previous pass. Its chains must equal
the host oracle's bit for bit in every form (site / cell per pass type),
replica grouping, sweep mix and lattice size, including sizes whose last
chunk is partial and lattices with fewer chunks than one dependency window;
its energies (the observables pass) equal a separate evaluation to FP64
rounding. A dependency wait that runs out (a planted item that never
reports, with a short poll limit) ends the cycle with PYRO_ERR_TIMEOUT and
leaves a context that continues correctly after a checkpoint restore."""
import numpy as np
import pytest

from cudacode_b200.engine import Engine, PyroError, System, geometric_ladder
from oracle.binding import Oracle

pytestmark = pytest.mark.gpu

PYRO_ERR_TIMEOUT = -3


def pair(systems, seed=77, renorm_every=0):
    return (Engine(systems, seed=seed, renorm_every=renorm_every),
            Oracle(systems, seed=seed, renorm_every=renorm_every))


def wave(e, forms=3, group=0):
    e.set_option(e.OPT_CYCLE_KERNEL, 2)
    e.set_option(e.OPT_J1_SITE_MODE, forms)
    e.set_option(e.OPT_REPLICA_GROUP, group)
    assert e.get_option(e.OPT_CYCLE_KERNEL) == 2


@pytest.mark.parametrize("L,R,forms,group,n_metro,n_or", [
    (6, 5, 3, 0, 1, 3),     # one chunk per replica: every item waits on the whole replica
    (8, 4, 3, 2, 1, 4),     # two chunks per replica
    (12, 6, 3, 4, 1, 4),    # L^3 = 1728: partial last chunk
    (12, 6, 1, 4, 2, 2),    # Metropolis site form, over-relaxation cell form
    (16, 4, 0, 3, 1, 2),    # both cell form, uneven last group
    (16, 4, 2, 0, 3, 0),    # Metropolis only (cell form)
    (20, 3, 3, 1, 0, 3),    # over-relaxation only, groups of one replica
])
def test_wave_kernel_bit_exact(L, R, forms, group, n_metro, n_or):
    temps = geometric_ladder(0.05, 1.5, R)
    e, o = pair([System(L=L, temperatures=temps)], renorm_every=3)
    wave(e, forms, group)
    e.init_random()
    o.init_random()
    cones = np.linspace(-0.7, 0.9, R).astype(np.float32)
    e.set_cone(cones)
    o.set_cone(cones)
    e.enable_history(8)
    e.cycle(n_metro, n_or, True, 4)
    h = o.cycle(n_metro, n_or, True, 4, record=True)
    assert np.array_equal(e.get_spins(), o.get_spins())
    assert np.array_equal(e.permutation(), o.permutation())
    assert np.array_equal(e.acceptance()[0], o.acceptance()[0])
    np.testing.assert_allclose(e.history(), h, rtol=1e-12, atol=1e-9)
    E0, M0 = e.last_observables()
    E1, M1 = o.observables()
    np.testing.assert_allclose(E0, E1, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(M0, M1, rtol=1e-12, atol=1e-9)
    # the other calls keep the chain on the per-pass kernels
    e.metropolis_sweep(1)
    o.metropolis_sweep(1)
    assert np.array_equal(e.get_spins(), o.get_spins())


def test_wave_kernel_with_generic_systems_in_the_context():
    systems = [System(L=8, temperatures=geometric_ladder(0.1, 1.0, 3)),
               System(L=5, temperatures=geometric_ladder(0.1, 1.0, 4), J2=0.07, J3=-0.03),
               System(L=10, temperatures=geometric_ladder(0.2, 2.0, 2))]
    e, o = pair(systems, seed=5, renorm_every=4)
    wave(e, 3, 2)
    e.set_option(e.OPT_GROUP_MB, 1)
    e.init_random()
    o.init_random()
    e.cycle(1, 2, True, 3)
    o.cycle(1, 2, True, 3)
    for k in range(3):
        assert np.array_equal(e.get_spins(k), o.get_spins(k)), k
        assert np.array_equal(e.permutation(k), o.permutation(k)), k
        np.testing.assert_allclose(e.last_observables(k)[0], o.observables(k)[0], rtol=1e-12,
                                   atol=1e-9)


def test_wave_kernel_shard_keys():
    temps = geometric_ladder(0.02, 2.0, 16)
    s = System(L=9, temperatures=temps, n_replicas=5, replica_offset=11)
    e, o = pair([s], seed=8)
    wave(e, 1, 2)
    e.init_random()
    o.init_random()
    e.cycle(1, 4, False, 3)
    o.cycle(1, 4, False, 3)
    assert np.array_equal(e.get_spins(), o.get_spins())


def test_wave_wait_that_runs_out_reports_timeout_and_the_context_recovers(tmp_path):
    temps = geometric_ladder(0.1, 1.0, 4)
    s = System(L=8, temperatures=temps)
    e, o = pair([s], seed=19)
    wave(e, 3, 2)
    e.init_random()
    o.init_random()
    e.cycle(1, 2, True, 2)
    o.cycle(1, 2, True, 2)
    ck = str(tmp_path / "before.ck")
    e.save_checkpoint(ck)
    # item 3 (a pass-0 item of the first group) never reports completion:
    # the items of pass 1 that need its chunk give up after 4096 polls
    e.set_option(e.OPT_WAVE_STALL, 3)
    e.cycle(1, 2, True, 1)
    with pytest.raises(PyroError) as err:
        e.synchronize()
    assert err.value.code == PYRO_ERR_TIMEOUT
    e.synchronize()  # the condition was cleared
    e.set_option(e.OPT_WAVE_STALL, -1)
    e.load_checkpoint(ck)
    e.cycle(1, 2, True, 3)
    o.cycle(1, 2, True, 3)
    assert np.array_equal(e.get_spins(), o.get_spins())
    assert np.array_equal(e.permutation(), o.permutation())


@pytest.mark.parametrize("L,R,forms,group,in_flight,n_metro,n_or", [
    (12, 6, 3, 2, 4, 1, 4),    # the benchmark's cycle shape, partial last chunk
    (16, 5, 1, 2, 2, 1, 3),    # cell-form over-relaxation, uneven last group
    (8, 7, 0, 3, 8, 2, 1),     # both cell form, more groups in flight than passes allow
    (20, 4, 3, 1, 3, 3, 0),    # Metropolis only, groups of one replica
    (9, 3, 2, 4, 2, 0, 2),     # over-relaxation only, one group
])
def test_skewed_launches_bit_exact(L, R, forms, group, in_flight, n_metro, n_or):
    temps = geometric_ladder(0.05, 1.5, R)
    e, o = pair([System(L=L, temperatures=temps)], renorm_every=3)
    e.set_option(e.OPT_CYCLE_KERNEL, 3)
    e.set_option(e.OPT_J1_SITE_MODE, forms)
    e.set_option(e.OPT_REPLICA_GROUP, group)
    e.set_option(e.OPT_CHAINS, in_flight)
    e.init_random()
    o.init_random()
    cones = np.linspace(-0.6, 0.8, R).astype(np.float32)
    e.set_cone(cones)
    o.set_cone(cones)
    e.enable_history(8)
    e.cycle(n_metro, n_or, True, 4)
    h = o.cycle(n_metro, n_or, True, 4, record=True)
    assert np.array_equal(e.get_spins(), o.get_spins())
    assert np.array_equal(e.permutation(), o.permutation())
    assert np.array_equal(e.acceptance()[0], o.acceptance()[0])
    np.testing.assert_allclose(e.history(), h, rtol=1e-12, atol=1e-9)
    E0, M0 = e.last_observables()
    E1, M1 = o.observables()
    np.testing.assert_allclose(E0, E1, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(M0, M1, rtol=1e-12, atol=1e-9)


def batched_16_colour(n=5, seed=3):
    rng = np.random.default_rng(seed)
    systems = []
    for i in range(n):
        L = int(rng.choice([4, 6, 9, 12, 16]))
        R = int(rng.integers(2, 5))
        systems.append(System(L=L, temperatures=geometric_ladder(0.05, 1.5, R),
                              J2=float(rng.uniform(-0.1, 0.1)), J3=float(rng.uniform(-0.1, 0.1))))
    return systems


@pytest.mark.parametrize("group_mb,n_metro,n_or", [(0, 1, 2), (1, 1, 3), (3, 2, 1), (0, 0, 2)])
def test_work_queue_of_16_colour_systems_bit_exact(group_mb, n_metro, n_or):
    """The batched 16-colour systems as one work-queue launch per cycle:
    uneven L (one chunk per replica up to 16 chunks with a dependency window
    narrower than the replica), groups of about group_mb MB, against the
    oracle bit for bit."""
    systems = batched_16_colour()
    e, o = pair(systems, seed=31, renorm_every=3)
    e.set_option(e.OPT_CYCLE_KERNEL, 2)
    e.set_option(e.OPT_GROUP_MB, group_mb)
    e.init_random()
    o.init_random()
    for k, sy in enumerate(systems):
        c = np.linspace(-0.6, 0.8, len(sy.temperatures)).astype(np.float32)
        e.set_cone(c, k)
        o.set_cone(c, k)
    e.cycle(n_metro, n_or, True, 3)
    o.cycle(n_metro, n_or, True, 3)
    for k in range(len(systems)):
        assert np.array_equal(e.get_spins(k), o.get_spins(k)), k
        assert np.array_equal(e.permutation(k), o.permutation(k)), k
        assert np.array_equal(e.acceptance(k)[0], o.acceptance(k)[0]), k
        np.testing.assert_allclose(e.last_observables(k)[0], o.observables(k)[0], rtol=1e-12,
                                   atol=1e-9)


def test_work_queue_skips_contexts_with_bond_matrix_systems():
    """An anisotropic system off the nearest-neighbour path keeps the 16-colour
    systems on their per-pass kernels: same chains."""
    systems = batched_16_colour(3, seed=9)
    e, o = pair(systems, seed=4)
    sym = np.array([[0.1, 0.02, 0.0], [0.02, -0.05, 0.01], [0.0, 0.01, 0.03]])
    A = np.tile(np.eye(3), (4, 4, 1, 1)) + sym
    e.set_exchange(A, system=1)
    o.set_exchange(A, system=1)
    e.set_option(e.OPT_CYCLE_KERNEL, 2)
    e.init_random()
    o.init_random()
    e.cycle(1, 1, True, 2)
    o.cycle(1, 1, True, 2)
    for k in range(len(systems)):
        assert np.array_equal(e.get_spins(k), o.get_spins(k)), k


def test_work_queue_of_16_colour_systems_wait_that_runs_out(tmp_path):
    systems = batched_16_colour(3, seed=12)
    e, o = pair(systems, seed=23)
    e.set_option(e.OPT_CYCLE_KERNEL, 2)
    e.init_random()
    o.init_random()
    e.cycle(1, 1, True, 1)
    o.cycle(1, 1, True, 1)
    ck = str(tmp_path / "before.ck")
    e.save_checkpoint(ck)
    # item 1 (a pass-0 item) never reports completion: the pass-1 items that
    # need its chunk give up after 4096 polls
    e.set_option(e.OPT_WAVE_STALL, 1)
    e.cycle(1, 1, True, 1)
    with pytest.raises(PyroError) as err:
        e.synchronize()
    assert err.value.code == PYRO_ERR_TIMEOUT
    e.synchronize()
    e.set_option(e.OPT_WAVE_STALL, -1)
    e.load_checkpoint(ck)
    e.cycle(1, 1, True, 2)
    o.cycle(1, 1, True, 2)
    for k in range(len(systems)):
        assert np.array_equal(e.get_spins(k), o.get_spins(k)), k
