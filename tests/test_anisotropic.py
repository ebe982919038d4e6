"""The anisotropic model: bond-dependent nearest-neighbour exchange and a
Zeeman field (the reference's couplings_const, Pyrochlore.cu:169-184, and
InitializeMagneticField, Pyrochlore.cu:414-450, entering TotalEnergy,
Pyrochlore.cu:468-523).

CPU: the builders against the reference's literal tables, the oracle's
energy against the reference's TotalEnergy on seeded configurations, single
spins in a field against the Langevin function, and energy conservation of
over-relaxation. GPU: the engine bit for bit against the oracle on every
kernel path that runs such a system, mixed with isotropic systems, and the
checks of the C-ABI (bad matrices, checkpoints, the learned move)."""
import json
import math
import os

import numpy as np
import pytest

from cudacode_b200.engine import (Engine, PyroError, System, geometric_ladder,
                                  reference_exchange, reference_field)
from oracle.binding import Oracle

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                     "reference_anisotropic.json")))
DEFAULTS = (-0.09 / 0.29, -0.22 / 0.29, -1.00, 0.0)  # Pyrochlore.cu:138-141


def reference_couplings(J):
    """couplings_const at (J1..J4): linear in J, from the golden basis."""
    basis = np.array(GOLDEN["couplings_basis"])  # (4 J's, 4, 4, 9)
    return np.tensordot(np.asarray(J, dtype=np.float64), basis, axes=1).reshape(4, 4, 3, 3)


def case_field(fi):
    if fi is None:
        return None
    c = GOLDEN["fields"][fi]
    return reference_field(c["gxy"], c["gz"], c["B"])


def test_reference_exchange_matches_couplings_const():
    rng = np.random.default_rng(3)
    for J in [DEFAULTS, (1.0, 2.0, 3.0, 4.0)] + [tuple(rng.normal(size=4)) for _ in range(4)]:
        A = reference_exchange(*J)
        C = reference_couplings(J)
        for a in range(4):
            assert np.all(A[a, a] == 0.0)
            for b in range(4):
                if a != b:
                    np.testing.assert_allclose(A[a, b], -0.25 * C[a, b], rtol=0, atol=1e-15)
                    np.testing.assert_array_equal(A[a, b], A[b, a].T)


def test_reference_field_matches_initialize_magnetic_field():
    for c in GOLDEN["fields"]:
        f = reference_field(c["gxy"], c["gz"], c["B"])
        F = np.array(c["field_on_site"]).reshape(4, 3)
        np.testing.assert_allclose(f, 0.5 * F, rtol=1e-13, atol=1e-16)


@pytest.mark.parametrize("fp64", [True, False])
def test_oracle_energy_equals_reference_total_energy(fp64):
    for c in GOLDEN["cases"]:
        L = c["L"]
        o = Oracle([System(L=L, temperatures=[1.0], J1=0.0)], fp64=fp64)
        o.set_exchange(reference_exchange(*c["J"]), case_field(c["field_case"]))
        a = np.zeros(o.spin_shape(), dtype=np.float32)
        a[0, :, :, :3] = np.array(c["spins"], dtype=np.float32).reshape(16, L ** 3, 3)
        o.set_spins(a)
        e, _ = o.observables()
        # the reference's spin-1/2 factor is folded into the matrices and fields
        assert e[0] == pytest.approx(c["energy_reference_units"], rel=1e-12, abs=1e-12)


def test_isotropic_matrices_give_the_heisenberg_energy():
    rng = np.random.default_rng(1)
    A = np.zeros((4, 4, 3, 3))
    for a in range(4):
        for b in range(4):
            if a != b:
                A[a, b] = 0.7 * np.eye(3)
    o_iso = Oracle([System(L=3, temperatures=[1.0], J1=0.7, J2=0.1)], fp64=True)
    o_mat = Oracle([System(L=3, temperatures=[1.0], J1=0.0, J2=0.1)], fp64=True)
    o_mat.set_exchange(A)
    v = rng.normal(size=o_iso.spin_shape())
    v[..., :3] /= np.linalg.norm(v[..., :3], axis=-1, keepdims=True)
    v[..., 3] = 0.0
    for o in (o_iso, o_mat):
        o.set_spins(v.astype(np.float32))
    assert o_mat.observables()[0][0] == pytest.approx(o_iso.observables()[0][0], rel=1e-12)


def langevin(x):
    return 1.0 / math.tanh(x) - 1.0 / x


def test_spins_in_a_field_follow_the_langevin_function():
    # No exchange: every spin feels only its sublattice's field f_b, so
    # <f_b/|f_b| . S> = coth(beta |f_b|) - 1 / (beta |f_b|).
    rng = np.random.default_rng(11)
    f = rng.normal(size=(4, 3))
    f *= (np.array([0.5, 1.0, 1.5, 2.0]) / np.linalg.norm(f, axis=1))[:, None]
    temps = [0.4, 1.0, 2.5]
    o = Oracle([System(L=2, temperatures=temps, J1=0.0)], seed=5)
    o.set_exchange(np.zeros((4, 4, 3, 3)), f)
    o.init_random()
    o.tune_cone(0.5, 12, 10)
    o.cycle(1, 1, False, 200)
    fhat = f / np.linalg.norm(f, axis=1, keepdims=True)
    acc = np.zeros((len(temps), 4))
    n = 300
    for _ in range(n):
        o.cycle(1, 1, False, 4)
        s = o.get_spins()[..., :3].astype(np.float64)  # (R, 16, L^3, 3); replica r at T[r]
        for b in range(4):
            sites = s[:, b::4]  # sites b, 4 + b, 8 + b, 12 + b
            acc[:, b] += np.einsum("rsck,k->r", sites, fhat[b]) / (4 * 8)
    got = acc / n
    for t, T in enumerate(temps):
        for b in range(4):
            want = langevin(np.linalg.norm(f[b]) / T)
            assert got[t, b] == pytest.approx(want, abs=0.02), (T, b)


def test_overrelaxation_conserves_the_anisotropic_energy():
    o = Oracle([System(L=3, temperatures=[0.5, 1.0], J1=0.0)], seed=2)
    o.set_exchange(reference_exchange(0.4, -0.3, 0.2, 0.35), 5.0 * case_field(1))
    o.init_random()
    e0, _ = o.observables()
    o.overrelax_sweep(10)
    e1, _ = o.observables()
    np.testing.assert_allclose(e1, e0, rtol=2e-5, atol=2e-4)


# ---------------------------------------------------------------- GPU ---

def pair(systems, seed=7):
    return Engine(systems, seed=seed), Oracle(systems, seed=seed)


def set_both(e, o, A, f, system=0):
    e.set_exchange(A, f, system)
    o.set_exchange(A, f, system)


@pytest.mark.gpu
@pytest.mark.parametrize("L, J, field, J2", [
    (3, DEFAULTS, True, 0.0),
    (4, (0.4, -0.3, 0.2, 0.35), True, 0.0),
    (4, DEFAULTS, False, 0.05),      # 16 colours (J2, J3 shells stay isotropic)
    (10, (0.4, -0.3, 0.2, 0.35), True, 0.0),  # beyond the shared-memory kernel
])
def test_engine_matches_oracle_bit_for_bit(L, J, field, J2):
    sysd = System(L=L, temperatures=geometric_ladder(0.1, 1.0, 4), J1=0.0, J2=J2, J3=0.5 * J2)
    e, o = pair([sysd])
    f = 10.0 * reference_field(1.0, 2.0, [0.3, -0.4, 1.0]) if field else None
    set_both(e, o, reference_exchange(*J), f)
    e.init_random()
    o.init_random()
    cone = np.array([0.2, 0.4, 0.6, 0.8], dtype=np.float32)
    e.set_cone(cone)
    o.set_cone(cone)
    e.metropolis_sweep(3)
    e.overrelax_sweep(2)
    o.metropolis_sweep(3)
    o.overrelax_sweep(2)
    np.testing.assert_array_equal(e.get_spins(), o.get_spins())
    np.testing.assert_array_equal(e.acceptance()[0], o.acceptance()[0])
    # captured cycles with exchange, then cycles without (shared-memory kernel for L <= 8)
    e.cycle(1, 2, True, 3)
    o.cycle(1, 2, True, 3)
    e.cycle(1, 1, False, 2)
    o.cycle(1, 1, False, 2)
    np.testing.assert_array_equal(e.get_spins(), o.get_spins())
    np.testing.assert_array_equal(e.permutation(), o.permutation())
    E, M = e.observables()
    Eo, Mo = o.observables()
    np.testing.assert_allclose(E, Eo, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(M, Mo, rtol=1e-12, atol=1e-9)


@pytest.mark.gpu
def test_mixed_with_isotropic_systems_and_back():
    temps = geometric_ladder(0.2, 1.5, 4)
    systems = [System(L=4, temperatures=temps, J1=1.0), System(L=3, temperatures=temps, J1=0.0)]
    e, o = pair(systems, seed=9)
    set_both(e, o, reference_exchange(*DEFAULTS), reference_field(1.0, 1.0, [0, 0, 3.0]), 1)
    assert e.get_exchange(0) is None
    A, f = e.get_exchange(1)
    np.testing.assert_array_equal(A, reference_exchange(*DEFAULTS))
    e.init_random()
    o.init_random()
    for run in (lambda x: x.cycle(1, 2, True, 4), lambda x: (x.metropolis_sweep(1),
                                                             x.overrelax_sweep(1))):
        run(e)
        run(o)
        for s in (0, 1):
            np.testing.assert_array_equal(e.get_spins(s), o.get_spins(s))
    # back to isotropic J1 = 0: only the (zero) further shells remain
    e.set_exchange(None, system=1)
    o.set_exchange(None, system=1)
    assert e.get_exchange(1) is None
    e.cycle(1, 1, True, 2)
    o.cycle(1, 1, True, 2)
    for s in (0, 1):
        np.testing.assert_array_equal(e.get_spins(s), o.get_spins(s))


@pytest.mark.gpu
def test_exchange_arguments_and_state(tmp_path):
    sysd = System(L=3, temperatures=[0.5, 1.0], J1=0.0)
    e = Engine([sysd], seed=1)
    A = reference_exchange(*DEFAULTS)
    bad = A.copy()
    bad[0, 1, 0, 2] += 0.1  # no longer the transpose of A[1][0]
    with pytest.raises(PyroError):
        e.set_exchange(bad)
    with pytest.raises(PyroError):
        e.set_exchange(A, system=1)
    e.set_exchange(A, reference_field(1.0, 1.0, [0, 0, 1.0]))
    # the learned move needs an isotropic J1-only system
    with pytest.raises(PyroError):
        e.tet_init(seed=1)
    e.init_random()
    e.cycle(1, 1, True, 2)
    path = str(tmp_path / "ck.bin")
    e.save_checkpoint(path)
    e2 = Engine([sysd], seed=1)
    e2.set_exchange(A, reference_field(1.0, 1.0, [0, 0, 1.0]))
    e2.load_checkpoint(path)
    np.testing.assert_array_equal(e2.get_spins(), e.get_spins())
    e3 = Engine([sysd], seed=1)  # isotropic: the checkpoint does not fit
    with pytest.raises(PyroError):
        e3.load_checkpoint(path)


@pytest.mark.gpu
@pytest.mark.parametrize("options", [
    {"J1_KERNEL": 0},                       # generic colour-pass kernel
    {"J1_SITE_MODE": 0},                    # cell per thread, both sweeps
    {"J1_SITE_MODE": 3},                    # site per thread, both sweeps
    {"REPLICA_GROUP": 2, "CHAINS": 2},      # L2-resident groups on two graph branches
    {"CYCLE_KERNEL": 1},                    # isotropic-only kernel: falls back to per-pass
    {"CYCLE_KERNEL": 2, "J1_SITE_MODE": 3, "REPLICA_GROUP": 2},  # work-queue kernel, site form
    {"CYCLE_KERNEL": 2, "J1_SITE_MODE": 1},                     # work queue, cell-form OR
])
def test_kernel_variants_agree_with_the_oracle(options):
    temps = geometric_ladder(0.1, 1.2, 6)
    systems = [System(L=10, temperatures=temps, J1=0.0), System(L=9, temperatures=temps, J1=1.0)]
    e, o = pair(systems, seed=21)
    set_both(e, o, reference_exchange(0.4, -0.3, 0.2, 0.35),
             10.0 * reference_field(2.4, 0.3, [0.0, 0.0, 1.0]), 0)
    for name, value in options.items():
        e.set_option(getattr(Engine, "OPT_" + name), value)
    e.init_random()
    o.init_random()
    e.cycle(1, 3, True, 3)
    o.cycle(1, 3, True, 3)
    for s in (0, 1):
        np.testing.assert_array_equal(e.get_spins(s), o.get_spins(s))
    np.testing.assert_allclose(e.observables(0)[0], o.observables(0)[0], rtol=1e-12)


@pytest.mark.gpu
def test_autotuned_schedule_agrees_with_the_oracle():
    temps = geometric_ladder(0.1, 1.2, 8)
    sysd = System(L=12, temperatures=temps, J1=0.0)
    A, f = reference_exchange(*DEFAULTS), reference_field(1.0, 1.0, [0.0, 0.0, 2.0])
    tuner = Engine([sysd], seed=4)
    tuner.set_exchange(A, f)
    tuner.init_random()
    tuner.autotune(1, 4, 1)
    names = ["J1_KERNEL", "CYCLE_KERNEL", "CLUSTER_SIZE", "J1_SITE_MODE", "REPLICA_GROUP",
             "CHAINS", "GROUP_MB", "FAR_KERNEL"]
    chosen = {n: tuner.get_option(getattr(Engine, "OPT_" + n)) for n in names}
    e, o = pair([sysd], seed=4)
    set_both(e, o, A, f)
    for n, v in chosen.items():
        e.set_option(getattr(Engine, "OPT_" + n), v)
    e.init_random()
    o.init_random()
    e.cycle(1, 4, True, 4)
    o.cycle(1, 4, True, 4)
    np.testing.assert_array_equal(e.get_spins(), o.get_spins())


def test_reference_gtensor_matches_magnetization_gpu():
    from cudacode_b200.engine import reference_gtensor
    for c in GOLDEN["fields"]:
        np.testing.assert_allclose(reference_gtensor(c["gxy"], c["gz"]),
                                   np.array(c["magnetization_g"]), rtol=1e-14, atol=1e-15)


@pytest.mark.gpu
def test_sublattice_magnetisation_matches_the_spins():
    temps = geometric_ladder(0.2, 1.0, 3)
    e = Engine([System(L=5, temperatures=temps), System(L=4, temperatures=temps, J1=0.0)], seed=3)
    e.set_exchange(reference_exchange(*DEFAULTS), system=1)
    e.init_random()
    e.cycle(1, 1, True, 2)
    for s in (0, 1):
        got = e.sublattice_magnetisation(s)
        sp = e.get_spins(s)[..., :3].astype(np.float64)  # (R, 16, L^3, 3)
        want = np.stack([sp[:, b::4].sum(axis=(1, 2)) for b in range(4)], axis=1)
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-9)
        _, M = e.observables(s)
        np.testing.assert_allclose(got.sum(axis=1), M.reshape(-1, 3), rtol=1e-12, atol=1e-9)
