"""Sharded parallel tempering over world_size-2 gloo ranks on the CPU.

The host-side exchange protocol (replica sharding, all_gather of the FP64
energies, identical Philox-driven exchange on every rank) is tested with the
oracle standing in for the engine: the two half-ladder ranks must reproduce
the unsharded run of the whole ladder bit for bit, spins and temperature
labels. A planted mistake (one rank contributing its energies in the wrong
replica order) must break it."""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cudacode_b200.distributed import ShardedPT, shard
from cudacode_b200.engine import System, geometric_ladder

L, N_T, SEED, CYCLES = 3, 6, 99, 12


class OracleBackend:
    """CPU stand-in for the engine (test infrastructure)."""

    def __init__(self, oracle, scrambled=False):
        self.o = oracle
        self.scrambled = scrambled

    def sweeps(self, n_metro, n_or):
        self.o.metropolis_sweep(n_metro)
        self.o.overrelax_sweep(n_or)

    def local_energies(self):
        e = torch.from_numpy(self.o.observables()[0].copy())
        if self.scrambled:  # planted mistake: local energies in reversed replica order
            e = e.flip(0).contiguous()
        return e

    def swap_global(self, all_energies, parity):
        self.o.pt_swap_global(all_energies.numpy(), parity)


class FakeEngine:
    """Host stand-in for cudacode_b200.engine.Engine with exactly the calls
    that EngineBackend makes (energies passed by pointer, as the engine's
    device calls take them), backed by the oracle (test infrastructure)."""

    def __init__(self, oracle, system, reversed_energies=False):
        self.o = oracle
        self.systems = [system]
        self.reversed_energies = reversed_energies
        self._e = None

    def stream_handle(self):
        return 0

    def cycle(self, n_metro, n_or, do_swap, n_cycles):
        assert not do_swap and n_cycles == 1
        self.o.metropolis_sweep(n_metro)
        self.o.overrelax_sweep(n_or)
        self._e = np.ascontiguousarray(self.o.observables()[0])  # the cycle's own energies

    def last_observables_device(self, e_ptr, m_ptr=0, system=0):
        e = self._e[::-1].copy() if self.reversed_energies else self._e  # planted mistake
        ctypes.memmove(e_ptr, e.ctypes.data, e.nbytes)

    def pt_swap_global(self, e_all_ptr, parity=-1, system=0):
        n = len(self.systems[0].temperatures)
        e = np.ctypeslib.as_array((ctypes.c_double * n).from_address(e_all_ptr)).copy()
        self.o.pt_swap_global(e, parity)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_rank(rank, world, port, out_dir, scrambled, engine_backend=False):
    from oracle.binding import Oracle

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    temps = geometric_ladder(0.1, 2.0, N_T)
    off, cnt = shard(N_T, world, rank)
    o = Oracle([System(L=L, temperatures=temps, n_replicas=cnt, replica_offset=off)], seed=SEED,
               threads=1)
    o.init_random()
    o.set_cone(np.linspace(-0.5, 0.8, N_T).astype(np.float32))
    if engine_backend:  # the engine's backend class over a host stand-in of the engine
        from cudacode_b200.distributed import EngineBackend
        system = System(L=L, temperatures=temps, n_replicas=cnt, replica_offset=off)
        backend = EngineBackend(FakeEngine(o, system, reversed_energies=scrambled and rank == 1),
                                torch.device("cpu"))
    else:
        backend = OracleBackend(o, scrambled=scrambled and rank == 1)
    pt = ShardedPT(backend, N_T)
    for _ in range(CYCLES):
        pt.cycle(1, 2)
    np.save(os.path.join(out_dir, f"spins{rank}.npy"), o.get_spins())
    np.save(os.path.join(out_dir, f"perm{rank}.npy"), o.permutation())
    dist.barrier()
    dist.destroy_process_group()


def reference_run():
    from oracle.binding import Oracle

    temps = geometric_ladder(0.1, 2.0, N_T)
    o = Oracle([System(L=L, temperatures=temps)], seed=SEED, threads=1)
    o.init_random()
    o.set_cone(np.linspace(-0.5, 0.8, N_T).astype(np.float32))
    for _ in range(CYCLES):
        o.metropolis_sweep(1)
        o.overrelax_sweep(2)
        e, _ = o.observables()
        o.pt_swap_global(e, -1)
    return o.get_spins(), o.permutation()


def launch(tmp_path, scrambled, engine_backend=False):
    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=run_rank, args=(r, 2, port, str(tmp_path), scrambled,
                                                engine_backend)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    spins = np.concatenate([np.load(tmp_path / f"spins{r}.npy") for r in range(2)])
    perms = [np.load(tmp_path / f"perm{r}.npy") for r in range(2)]
    return spins, perms


def test_shard_blocks():
    assert [shard(6, 2, r) for r in range(2)] == [(0, 3), (3, 3)]
    assert [shard(7, 3, r) for r in range(3)] == [(0, 3), (3, 2), (5, 2)]
    with pytest.raises(ValueError):
        shard(1, 2, 0)


def test_two_ranks_reproduce_the_unsharded_ladder(tmp_path):
    spins, perms = launch(tmp_path, scrambled=False)
    ref_spins, ref_perm = reference_run()
    assert np.array_equal(perms[0], perms[1])
    assert np.array_equal(perms[0], ref_perm)
    assert np.array_equal(spins, ref_spins)
    assert not np.array_equal(ref_perm, np.arange(N_T))  # some exchanges happened


def test_planted_energy_order_mistake_is_detected(tmp_path):
    spins, perms = launch(tmp_path, scrambled=True)
    ref_spins, ref_perm = reference_run()
    assert not (np.array_equal(perms[0], ref_perm) and np.array_equal(spins, ref_spins))


def test_engine_backend_ordering_over_two_ranks(tmp_path):
    """EngineBackend (energies of the cycle copied by pointer, gathered,
    handed to the global exchange) over two gloo ranks, with a host stand-in
    for the engine: the unsharded ladder bit for bit; a rank that hands over
    its energies in the wrong order is detected."""
    spins, perms = launch(tmp_path, scrambled=False, engine_backend=True)
    ref_spins, ref_perm = reference_run()
    assert np.array_equal(perms[0], perms[1])
    assert np.array_equal(perms[0], ref_perm)
    assert np.array_equal(spins, ref_spins)
    spins, perms = launch(tmp_path, scrambled=True, engine_backend=True)
    assert not (np.array_equal(perms[0], ref_perm) and np.array_equal(spins, ref_spins))


BATCH = [(3, 4, 0.0), (4, 3, 0.05), (3, 2, -0.04), (5, 2, 0.0), (4, 5, 0.02)]  # L, temps, J2


def batch_systems():
    return [System(L=L, temperatures=geometric_ladder(0.1, 1.5, n), J2=j2)
            for L, n, j2 in BATCH]


def run_system_rank(rank, world, port, out_dir):
    from cudacode_b200.distributed import gather_system_results, make_system_shard
    from oracle.binding import Oracle

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    systems = batch_systems()
    o, local = make_system_shard(systems, world, rank, seed=SEED,
                                 factory=lambda s: Oracle(s, seed=SEED, threads=1))
    o.init_random()
    o.cycle(1, 2, True, CYCLES)
    mine = {gi: (o.get_spins(j), o.permutation(j)) for j, gi in enumerate(local)}
    allres = gather_system_results(mine, len(systems))
    if rank == 0:
        np.save(os.path.join(out_dir, "batch.npy"),
                np.array([np.concatenate([r[0].ravel(), r[1].astype(np.float32)])
                          for r in allres], dtype=object), allow_pickle=True)
    dist.barrier()
    dist.destroy_process_group()


def test_deal_systems_balances_and_covers():
    from cudacode_b200.distributed import deal_systems
    sizes = [5, 1, 4, 4, 2, 7, 3]
    parts = [deal_systems(sizes, 3, r) for r in range(3)]
    assert sorted(sum(parts, [])) == list(range(7))
    loads = [sum(sizes[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(sizes)
    with pytest.raises(ValueError):
        deal_systems([1], 2, 0)


def test_systems_dealt_over_two_ranks_reproduce_the_whole_batch(tmp_path):
    """Independent systems shared out over two gloo ranks, each rank one
    context with the full set's Philox keys and no collective until the
    final gather: every system's spins and permutation equal the
    single-context run's bit for bit."""
    from oracle.binding import Oracle

    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=run_system_rank, args=(r, 2, port, str(tmp_path)))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    got = np.load(tmp_path / "batch.npy", allow_pickle=True)
    o = Oracle(batch_systems(), seed=SEED, threads=1)
    o.init_random()
    o.cycle(1, 2, True, CYCLES)
    for i in range(len(BATCH)):
        want = np.concatenate([o.get_spins(i).ravel(), o.permutation(i).astype(np.float32)])
        assert np.array_equal(got[i], want), i
