"""pyro_observables_noalloc: the entry point for callers that cannot allocate
device memory (memory pools or arenas that own the GPU's memory, frameworks
that forbid allocation once their buffers are sized). It keeps its scratch in
a fixed static array inside the library instead of calling cudaMalloc.

The GPU test calls it through the C-ABI on spins copied out of an engine
context and checks its energies and magnetisations, on two calls in a row,
against the context's own observables (pyro_observables) and against the host
oracle's FP64 observables of the same spins, within the FP64 tolerance used
by the other parity tests. The CPU tests check that requests larger than the
static array and misaligned pointers are refused before anything reaches the
GPU. This file is named to run last, so that a run stopping at the first
failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from cudacode_b200.engine import Engine, System, geometric_ladder, load_library

RTOL, ATOL = 1e-12, 1e-9


def noalloc_fn():
    lib = load_library()
    fn = lib.pyro_observables_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                   C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
    return fn


def make_system(L, R, J):
    return System(L=L, temperatures=geometric_ladder(0.1, 1.5, R), J1=J[0], J2=J[1], J3=J[2],
                  J3b=J[3])


@pytest.mark.gpu
@pytest.mark.parametrize("L,R,J", [(8, 3, (1.0, 0.0, 0.0, 0.0)),
                                   (5, 2, (1.0, 0.07, -0.05, 0.02))])
def test_noalloc_matches_context_and_oracle_twice(L, R, J):
    torch = pytest.importorskip("torch")
    from oracle.binding import Oracle

    fn = noalloc_fn()
    eng = Engine([make_system(L, R, J)], seed=31 + L)
    eng.init_random()
    eng.metropolis_sweep(2)
    eng.overrelax_sweep(2)
    e_ctx, m_ctx = eng.observables()
    orc = Oracle([make_system(L, R, J)], seed=31 + L)
    orc.set_spins(eng.get_spins())
    e_orc, m_orc = orc.observables()
    spins = torch.empty(R * 16 * L ** 3 * 4, dtype=torch.float32, device="cuda")
    eng.get_spins_device(spins.data_ptr())
    eng.synchronize()
    for call in range(2):
        e = torch.full((R,), float("nan"), dtype=torch.float64, device="cuda")
        m = torch.full((R, 3), float("nan"), dtype=torch.float64, device="cuda")
        rc = fn(spins.data_ptr(), L, R, J[0], J[1], J[2], J[3], e.data_ptr(), m.data_ptr(), None)
        assert rc == 0, rc
        torch.cuda.synchronize()
        for e_ref, m_ref in ((e_ctx, m_ctx), (e_orc, m_orc)):
            np.testing.assert_allclose(e.cpu().numpy(), e_ref, rtol=RTOL, atol=ATOL)
            np.testing.assert_allclose(m.cpu().numpy(), m_ref, rtol=RTOL, atol=ATOL)
    orc.close()
    eng.close()


def test_noalloc_rejects_requests_beyond_its_scratch():
    fn = noalloc_fn()
    # L = 64 needs 2048 partial sums per replica; 40 replicas exceed 65536.
    dummy = C.c_void_p(256)
    rc = fn(dummy, 64, 40, 1.0, 0.0, 0.0, 0.0, dummy, None, None)
    assert rc == -1


@pytest.mark.parametrize("spins,energy,mag", [(256 + 8, 256, None), (256 + 4, 256, None),
                                              (256, 256 + 4, None), (256, 256, 256 + 2)])
def test_noalloc_rejects_misaligned_pointers(spins, energy, mag):
    # Refused on the host before any CUDA call: the addresses are never read.
    fn = noalloc_fn()
    rc = fn(C.c_void_p(spins), 4, 1, 1.0, 0.0, 0.0, 0.0, C.c_void_p(energy),
            None if mag is None else C.c_void_p(mag), None)
    assert rc == -1
