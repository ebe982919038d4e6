"""Long-run observables of the FP32 engine against an FP64 host run.

The engine (FP32 spins, FP64 reductions) and the oracle in FP64 mode (FP64
spins, fields and updates, libm functions) run independent chains of the
same model; energy per site, specific heat and S(q) must agree within their
statistical errors (the spec asks for 2 sigma; the asserts allow 3 sigma
so that the test does not fail by chance, and the largest deviation is
printed)."""
import numpy as np
import pytest

from cudacode_b200 import stats
from cudacode_b200.engine import Engine, System
from oracle.binding import Oracle

pytestmark = pytest.mark.gpu

L, TEMPS, CYCLES, SNAP_EVERY = 4, [0.3, 1.0], 12000, 100


def batch_mean_error(x, n_batches=20):
    b = np.asarray(x)[: len(x) // n_batches * n_batches].reshape(n_batches, -1)
    means = b.mean(axis=1)
    return means.mean(), means.std(ddof=1) / np.sqrt(n_batches)


def batch_heat(e, T, n, n_batches=20):
    b = np.asarray(e)[: len(e) // n_batches * n_batches].reshape(n_batches, -1)
    c = b.var(axis=1) / (n * T * T)
    return c.mean(), c.std(ddof=1) / np.sqrt(n_batches)


def run_chain(obj, is_engine):
    cones = np.array([0.4, -0.3], dtype=np.float32)
    obj.set_cone(cones)
    obj.init_random()
    if is_engine:
        obj.cycle(1, 2, False, 2000)
        obj.enable_history(SNAP_EVERY)
    else:
        obj.cycle(1, 2, False, 2000)
    es, sqs = [], []
    for _ in range(CYCLES // SNAP_EVERY):
        if is_engine:
            obj.cycle(1, 2, False, SNAP_EVERY)
            es.append(obj.history())
        else:
            es.append(obj.cycle(1, 2, False, SNAP_EVERY, record=True))
        sqs.append(np.stack([obj.structure_factor(4, 2, replica=r) for r in range(2)]))
    return np.concatenate(es), np.stack(sqs)


def test_fp32_engine_matches_fp64_host_run():
    s = System(L=L, temperatures=TEMPS)
    n = s.n_sites
    e32, sq32 = run_chain(Engine([s], seed=101), True)
    e64, sq64 = run_chain(Oracle([s], seed=202, fp64=True, threads=4), False)
    worst = 0.0
    for t, T in enumerate(TEMPS):
        m1, d1 = stats.mean_error(e32[:, t] / n)
        m2, d2 = stats.mean_error(e64[:, t] / n)
        z = abs(m1 - m2) / np.hypot(d1, d2)
        worst = max(worst, z)
        assert z < 3.0, ("E", T, m1, d1, m2, d2)
        c1, dc1 = batch_heat(e32[:, t], T, n)
        c2, dc2 = batch_heat(e64[:, t], T, n)
        z = abs(c1 - c2) / np.hypot(dc1, dc2)
        worst = max(worst, z)
        assert z < 3.0, ("C", T, c1, dc1, c2, dc2)
        for q in [(2, 2, 3), (2, 3, 3), (3, 3, 3), (2, 2, 2)]:
            a, da = batch_mean_error(sq32[:, t][(slice(None),) + q])
            b, db = batch_mean_error(sq64[:, t][(slice(None),) + q])
            if da + db == 0:
                continue
            z = abs(a - b) / np.hypot(da, db)
            worst = max(worst, z)
            assert z < 3.0, ("S(q)", T, q, a, da, b, db)
    print(f"largest deviation: {worst:.2f} sigma")


def test_anisotropic_model_matches_fp64_host_run():
    """The reference's J1-J4 model with a field: energy and specific heat of
    the FP32 engine against an independent FP64 host chain (the matrix and
    field paths of both)."""
    from cudacode_b200.engine import reference_exchange, reference_field
    A = reference_exchange(0.4, -0.3, 0.2, 0.35)
    f = 3.0 * reference_field(2.4, 0.3, [0.3, -0.2, 1.0])
    temps = [0.08, 0.3]
    s = System(L=L, temperatures=temps, J1=0.0)
    n = s.n_sites

    def chain(obj, is_engine):
        obj.set_exchange(A, f)
        obj.set_cone(np.array([0.5, -0.2], dtype=np.float32))
        obj.init_random()
        obj.cycle(1, 2, False, 2000)
        if is_engine:
            obj.enable_history(CYCLES)
            obj.cycle(1, 2, False, CYCLES)
            return obj.history()
        return obj.cycle(1, 2, False, CYCLES, record=True)

    e32 = chain(Engine([s], seed=303), True)
    e64 = chain(Oracle([s], seed=404, fp64=True, threads=4), False)
    worst = 0.0
    for t, T in enumerate(temps):
        m1, d1 = stats.mean_error(e32[:, t] / n)
        m2, d2 = stats.mean_error(e64[:, t] / n)
        z = abs(m1 - m2) / np.hypot(d1, d2)
        worst = max(worst, z)
        assert z < 3.0, ("E", T, m1, d1, m2, d2)
        c1, dc1 = batch_heat(e32[:, t], T, n)
        c2, dc2 = batch_heat(e64[:, t], T, n)
        z = abs(c1 - c2) / np.hypot(dc1, dc2)
        worst = max(worst, z)
        assert z < 3.0, ("C", T, c1, dc1, c2, dc2)
    print(f"largest deviation: {worst:.2f} sigma")
