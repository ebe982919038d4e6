"""Parallel tempering across GPUs: one process per GPU, replicas sharded.

Each rank holds a contiguous block of the configurations of one global
temperature ladder (``System(n_replicas=R, replica_offset=rank * R)``). A
cycle is: the local sweeps (no exchange), the FP64 energies of the local
replicas, an ``all_gather`` of those energies (8 bytes per replica, over
NCCL on GPUs), and the exchange step applied identically on every rank from
the gathered vector (``pyro_pt_swap_global``: Philox-driven, so no decision
has to be broadcast). Spins never leave their GPU; only temperature labels
move. Because Philox keys use the global replica index, a sharded run
reproduces the single-GPU run of the same ladder.

Replaces the reference's multi-GPU layer: one pthread per GPU with
host-staged energy reductions and a host-side swap (MonteCarlo.cu:15-245,
TrySwapingTemperatures MonteCarlo.cu:105-172).

The driver only needs an object with ``sweeps(n_metro, n_or)``,
``local_energies() -> tensor`` and ``swap_global(all_energies, parity)``;
:class:`EngineBackend` binds it to the CUDA engine.

Many independent systems (the batched configuration) shard whole systems
instead: :func:`deal_systems` gives each rank a set of systems of about equal
work, every rank runs its own engine with its own exchanges and no
collective, and :func:`gather_system_results` collects per-system results on
every rank at the end, in the global system order.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch
import torch.distributed as dist

from .engine import Engine, System


def shard(n_total: int, world: int, rank: int) -> tuple[int, int]:
    """(offset, count) of the replicas held by `rank`; blocks differ by <= 1."""
    if n_total < world:
        raise ValueError(f"{n_total} replicas cannot be spread over {world} ranks")
    base, extra = divmod(n_total, world)
    count = base + (1 if rank < extra else 0)
    offset = rank * base + min(rank, extra)
    return offset, count


class EngineBackend:
    """The CUDA engine as a sharded-PT backend (energies stay on the GPU).

    The engine queues on its own stream and the collective on torch's
    current stream; each hand-over makes the receiving stream wait for the
    other (no host synchronisation). On a CPU device (a host stand-in for
    the engine, used by the tests) the calls are synchronous and there is
    nothing to order."""

    def __init__(self, engine: Engine, device: torch.device):
        self.engine = engine
        self.device = device
        self.n_local = engine.systems[0].replicas()
        self._e = torch.zeros(self.n_local, dtype=torch.float64, device=device)

    def _engine_stream(self) -> torch.cuda.Stream:
        h = self.engine.stream_handle()
        if h == 0:
            return torch.cuda.default_stream(self.device)
        return torch.cuda.ExternalStream(h, device=self.device)

    def sweeps(self, n_metro: int, n_or: int) -> None:
        self.engine.cycle(n_metro, n_or, False, 1)

    def local_energies(self) -> torch.Tensor:
        # the cycle computed them at its end: copy, do not recompute
        self.engine.last_observables_device(self._e.data_ptr())
        if self.device.type == "cuda":
            torch.cuda.current_stream(self.device).wait_stream(self._engine_stream())
        return self._e

    def swap_global(self, all_energies: torch.Tensor, parity: int) -> None:
        if self.device.type == "cuda":
            self._engine_stream().wait_stream(torch.cuda.current_stream(self.device))
        self.engine.pt_swap_global(all_energies.data_ptr(), parity)


@dataclass
class ShardedPT:
    backend: object
    n_total: int
    group: object = None

    def __post_init__(self):
        self.world = dist.get_world_size(self.group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(self.group) if dist.is_initialized() else 0
        self.offset, self.count = shard(self.n_total, self.world, self.rank)
        counts = [shard(self.n_total, self.world, r)[1] for r in range(self.world)]
        if len(set(counts)) != 1:
            raise ValueError("all_gather needs equal shards: choose replicas divisible by ranks")

    def cycle(self, n_metro: int, n_or: int, parity: int = -1) -> torch.Tensor:
        """One cycle; returns the gathered energies (global replica order)."""
        self.backend.sweeps(n_metro, n_or)
        e_local = self.backend.local_energies()
        if self.world > 1:
            e_all = torch.empty(self.n_total, dtype=e_local.dtype, device=e_local.device)
            dist.all_gather_into_tensor(e_all, e_local.contiguous(), group=self.group)
        else:
            e_all = e_local
        self.backend.swap_global(e_all, parity)
        return e_all


def make_engine_shard(L: int, temperatures, world: int, rank: int, seed: int, device: int,
                      **couplings) -> Engine:
    """Engine holding this rank's block of the global ladder."""
    offset, count = shard(len(temperatures), world, rank)
    return Engine([System(L=L, temperatures=list(temperatures), n_replicas=count,
                          replica_offset=offset, **couplings)], seed=seed, device=device)


def deal_systems(sizes, world: int, rank: int) -> list[int]:
    """Indices of the systems held by `rank`: greedy by decreasing size
    (sites x replicas) onto the least loaded rank, ties to the lowest rank,
    so the ranks' work differs by at most one system. The same on every rank."""
    if len(sizes) < world:
        raise ValueError(f"{len(sizes)} systems cannot be spread over {world} ranks")
    load = [0] * world
    owner = [0] * len(sizes)
    for i in sorted(range(len(sizes)), key=lambda i: (-sizes[i], i)):
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += sizes[i]
    return [i for i in range(len(sizes)) if owner[i] == rank]


def gather_system_results(local: dict, n_systems: int, group=None) -> list:
    """{global system index: result} of every rank -> list over all systems
    (on every rank; one object gather at the end of a run)."""
    if not dist.is_initialized():
        out = [None] * n_systems
        for i, v in local.items():
            out[i] = v
        return out
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, local, group=group)
    out = [None] * n_systems
    for part in parts:
        for i, v in part.items():
            out[i] = v
    return out


def system_keys(systems) -> list[tuple[int, int]]:
    """(key_base, swap_key) of every system in the full set: the Philox keys
    each has in a context holding all of them."""
    keys, base = [], 0
    for i, sy in enumerate(systems):
        keys.append((base, i))
        base += len(sy.temperatures)
    return keys


def make_system_shard(systems, world: int, rank: int, seed: int, device: int = 0,
                      factory=None, **kwargs):
    """This rank's share of independent systems (deal_systems) in one context
    whose Philox keys are those of the full set, so each system's chain is
    the one an unsharded run gives. Returns (context, global indices).
    `factory` builds the context (default: the CUDA engine)."""
    sizes = [sy.n_sites * sy.replicas() for sy in systems]
    local = deal_systems(sizes, world, rank)
    make = factory or (lambda sys_list: Engine(sys_list, seed=seed, device=device, **kwargs))
    ctx = make([systems[i] for i in local])
    keys = system_keys(systems)
    for j, gi in enumerate(local):
        ctx.set_system_keys(j, *keys[gi])
    return ctx, local
