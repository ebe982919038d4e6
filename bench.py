"""Benchmark: parallel-tempering Monte Carlo of the pyrochlore Heisenberg
antiferromagnet, L=32 (524,288 sites), 64 replicas on a geometric ladder
T in [0.02, 2.0], 1 cone-Metropolis + 4 over-relaxation sweeps per exchange
attempt, FP64 energies and swap test. One step = one such cycle over all
replicas; metric = spin updates per nanosecond (whole job).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Under torchrun (N > 1) every rank holds 64 replicas of one global ladder of
64 N temperatures; energies are all-gathered over NCCL each cycle and every
rank applies the identical exchange (weak scaling).

``--impl reference`` times the reference algorithm's CPU implementation (the
C++/OpenMP port in oracle/, the reference itself does not build) on the host
cores for the same workload, on a bounded sample of replicas per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L = 32
R_PER_GPU = 64
T_MIN, T_MAX = 0.02, 2.0
N_METRO, N_OR = 1, 4
SEED = 12345 + 1
METRIC = "spin-updates/ns"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
BYTES_PER_UPDATE_PASS = 80  # float4 spins, J1 4-colour pass: 16 N/4 own + 48 N/4 nbr + 16 N/4 write


def set_workload(l: int, replicas: int) -> None:
    global L, R_PER_GPU
    L, R_PER_GPU = l, replicas


TRAFFIC_PROFILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles",
                               "or_pass_L32_R64_streaming.md")


def profiled_traffic():
    """DRAM bytes (read + write) per launch of the over-relaxation pass, from
    the committed ncu summary of this workload (line 'traffic_bytes_per_launch: N')."""
    try:
        with open(TRAFFIC_PROFILE) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def hbm_peak():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """Samples the SM clock and the clock-event (throttle) reasons during a
    region: through NVML every 20 ms when the NVML binding is importable
    (read-only queries), else through `nvidia-smi -lms 100`. The sampler is
    running before the region starts."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()
        self.lines: list[str] = []
        self.samples: list[tuple[float, float, set]] = []

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.dev)
            self.nvml = (pynvml, h)
            bits = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap}
            mx = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))

            def poll():
                while True:
                    sm = float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                    r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((sm, mx, {n for n, b in bits.items() if r & b}))
                    if self.stop.wait(0.02):
                        return

            self.t = threading.Thread(target=poll, daemon=True)
            self.t.start()
            while not self.samples and self.t.is_alive():
                time.sleep(0.001)
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 3.0:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.nvml:
            self.stop.set()
            self.t.join(timeout=2)
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        for s_mhz, m_mhz, rs in self.samples:
            sm.append(s_mhz)
            mx = m_mhz
            reasons |= rs
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(self.NAMES, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml" if self.samples else "nvidia-smi"}


KERNEL_OPTIONS = ("J1_KERNEL", "CYCLE_KERNEL", "CLUSTER_SIZE", "J1_SITE_MODE", "REPLICA_GROUP",
                  "CHAINS", "PDL", "FUSED_OBS", "J1_FIXED_L", "CHAIN_STAGGER")


def cpu_baseline_and_parity(kernel_options: dict, cycles: int = 6):
    """The cpu_baseline leg at the benchmark's own workload: the oracle port
    runs `cycles` whole cycles (1 M + 4 OR sweeps, FP64 energies, exchange)
    of all replicas of the L=32 ladder on every host core, timed; a fresh
    engine context with the kernel schedule that was timed runs the same
    cycles from the same seed, and its spins, permutation and energies are
    checked against the oracle's (bit for bit; energies to FP64 rounding)."""
    from cudacode_b200.engine import Engine, System, geometric_ladder
    from oracle.binding import Oracle

    temps = geometric_ladder(T_MIN, T_MAX, R_PER_GPU)
    sysd = System(L=L, temperatures=temps)
    cones = np.full(R_PER_GPU, 0.3, dtype=np.float32)
    o = Oracle([sysd], seed=SEED, threads=os.cpu_count())
    o.init_random()
    o.set_cone(cones)
    t0 = time.perf_counter()
    o.cycle(N_METRO, N_OR, True, cycles)
    dt = time.perf_counter() - t0
    n_threads = o.lib.orc_set_threads(0)
    updates = R_PER_GPU * 16 * L ** 3 * (N_METRO + N_OR) * cycles
    cpu = {"value": updates / (dt * 1e9), "unit": "updates/ns", "cores": n_threads, "kind": "port",
           "sample": f"all {R_PER_GPU} replicas, {cycles} cycles ({dt:.1f} s)"}
    e = Engine([sysd], seed=SEED)
    for name, value in kernel_options.items():
        e.set_option(getattr(Engine, "OPT_" + name), value)
    e.init_random()
    e.set_cone(cones)
    e.cycle(N_METRO, N_OR, True, cycles)
    a, b = e.get_spins(), o.get_spins()
    E0, _ = e.last_observables()
    E1, _ = o.observables()
    exact = bool(np.array_equal(a, b) and np.array_equal(e.permutation(), o.permutation()))
    e_ok = bool(np.allclose(E0, E1, rtol=1e-12, atol=1e-9))
    parity = {"check": "bit-exact" if exact and e_ok else "MISMATCH",
              "what": f"the timed kernel schedule on a fresh context of the same workload and seed, "
                      f"{cycles} cycles, all {R_PER_GPU} replicas, against the oracle: spins and "
                      f"exchange permutation bit for bit, FP64 energies to rel 1e-12",
              "max_spin_diff": float(np.abs(a - b).max()),
              "max_energy_rel_diff": float(np.max(np.abs(E0 - E1) / np.maximum(np.abs(E1), 1.0)))}
    e.close()
    o.close()
    return cpu, parity


def cpu_baseline_sample(threads: int | None = None, replicas: int = 16, cycles: int = 25):
    """The reference algorithm's CPU path (oracle port) on a bounded sample."""
    from cudacode_b200.engine import System, geometric_ladder
    from oracle.binding import Oracle

    temps = geometric_ladder(T_MIN, T_MAX, R_PER_GPU)
    o = Oracle([System(L=L, temperatures=temps, n_replicas=replicas)], seed=SEED,
               threads=threads or os.cpu_count())
    o.init_random()
    o.set_cone(np.full(R_PER_GPU, 0.3, dtype=np.float32))
    o.metropolis_sweep(1)  # warm caches / threads
    t0 = time.perf_counter()
    for _ in range(cycles):
        o.metropolis_sweep(N_METRO)
        o.overrelax_sweep(N_OR)
        o.observables()
    dt = time.perf_counter() - t0
    updates = replicas * 16 * L ** 3 * (N_METRO + N_OR) * cycles
    n_threads = o.lib.orc_set_threads(0)
    return updates / (dt * 1e9), n_threads, dt, f"{replicas} of {R_PER_GPU} replicas, {cycles} cycles"


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    vals = []
    n_threads = None
    for _ in range(args.warmup):
        cpu_baseline_sample(replicas=4, cycles=1)
    for _ in range(args.steps):
        v, n_threads, dt, sample = cpu_baseline_sample(replicas=4, cycles=1)
        vals.append(v)
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "updates/ns",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (random unit spins from Philox seed)",
        "config": workload_config(args.gpus),
        "cpu_baseline": {"value": value, "unit": "updates/ns", "cores": n_threads, "kind": "port",
                         "sample": "per step: 4 of 64 replicas of L=32, 1 cycle (1 M + 4 OR "
                                   "sweeps + FP64 energies)"},
        "e2e": {"value": value, "unit": "updates/ns", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(n_gpus):
    return {"workload": f"pyrochlore Heisenberg AFM PT: L={L} ({16 * L ** 3:,} sites), J1=1, "
                        f"{R_PER_GPU} replicas per GPU on a geometric ladder T in [0.02, 2.0], "
                        "1 Metropolis + 4 over-relaxation sweeps + FP64 energies + swap per step",
            "L": L, "replicas_per_gpu": R_PER_GPU, "global_replicas": R_PER_GPU * n_gpus,
            "sweeps_per_step": N_METRO + N_OR, "parallelism": f"replicas sharded over {n_gpus} GPU",
            "l2": f"inputs larger than L2 ({R_PER_GPU * 16 * L ** 3 * 16 / 1e6:.0f} MB of spins "
                  "per GPU > 126 MB)"}


def _timed(stream, fn):
    import torch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / 1e3


def run_small(args):
    """L=4 (1,024 sites), J1=1, T=0.5, one replica, cone tuned to 50%
    acceptance, cycle = 1 Metropolis + 5 over-relaxation sweeps, 10^4 cycles,
    on the GPU (shared-memory kernel) and on the host (oracle port, all host
    cores); energy per site compared within 2 sigma."""
    import torch

    from cudacode_b200 import stats
    from cudacode_b200.engine import Engine, System
    from oracle.binding import Oracle

    cycles = 10_000
    s = System(L=4, temperatures=[0.5])
    eng = Engine([s], seed=SEED + 1)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    eng.init_random()
    eng.tune_cone(0.5, 30, 20, 5)
    eng.cycle(1, 5, False, 1000)
    eng.enable_history(cycles)
    sec = _timed(stream, lambda: eng.cycle(1, 5, False, cycles))
    eng.reset_acceptance()
    eng.metropolis_sweep(200)
    acc, prop = eng.acceptance()
    h = eng.history()[:, 0] / 1024
    o = Oracle([s], seed=SEED + 1, threads=os.cpu_count())
    o.init_random()
    o.tune_cone(0.5, 30, 20, 5)
    o.cycle(1, 5, False, 1000)
    t0 = time.perf_counter()
    ho = o.cycle(1, 5, False, cycles, record=True)[:, 0] / 1024
    host_s = time.perf_counter() - t0
    updates = 1024 * 6 * cycles
    m1, e1 = stats.mean_error(h)
    m2, e2 = stats.mean_error(ho)
    print(json.dumps({
        "metric": "spin-updates/ns", "workload": "small", "value": updates / (sec * 1e9),
        "unit": "updates/ns", "host_value": updates / (host_s * 1e9), "host_cores": os.cpu_count(),
        "gpu_seconds": sec, "host_seconds": host_s, "acceptance": float(acc[0] / prop[0]),
        "E_per_site_gpu": [m1, e1], "E_per_site_host": [m2, e2],
        "agreement_sigma": abs(m1 - m2) / np.hypot(e1, e2),
        "config": {"workload": "L=4 (1,024 sites) J1=1 T=0.5, 1 replica, 1 Metropolis + 5 "
                               "over-relaxation sweeps per cycle, 10^4 cycles",
                   "kernel": "shared-memory-resident cycles (one launch)"}}), flush=True)
    return 0


def run_batched(args):
    """256 systems, L uniform in {8,12,16,20,24}, 16-32 replicas each on its
    own geometric ladder in [0.05, 1.5], J1=1 and J2, J3 uniform in
    [-0.1, 0.1] (16-colour schedule); cycle = 1 Metropolis + 4 over-relaxation
    sweeps + FP64 energies + exchange, one CUDA graph for all systems."""
    import torch

    from cudacode_b200.engine import Engine, System, geometric_ladder

    rng = np.random.default_rng(12345 + 3)
    systems = []
    for _ in range(args.systems):
        Ls = int(rng.choice([8, 12, 16, 20, 24]))
        nT = int(rng.integers(16, 33))
        j2, j3 = rng.uniform(-0.1, 0.1, 2)
        systems.append(System(L=Ls, temperatures=geometric_ladder(0.05, 1.5, nT), J2=float(j2),
                              J3=float(j3)))
    eng = Engine(systems, seed=SEED + 2)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    eng.init_random()
    for k, sy in enumerate(systems):
        eng.set_cone(np.full(len(sy.temperatures), 0.3, dtype=np.float32), k)
    if args.kernel == "wave":
        # the work-queue launch over every system (one per cycle)
        eng.set_option(eng.OPT_CYCLE_KERNEL, 2)
        eng.set_option(eng.OPT_GROUP_MB, args.group_mb or 0)
        choice = None
    else:
        choice = eng.autotune(1, 4, 2)
    eng.cycle(1, 4, True, args.warmup)
    steps = args.steps if args.steps != 300 else 20
    sec = _timed(stream, lambda: eng.cycle(1, 4, True, steps))
    spins = sum(len(sy.temperatures) * sy.n_sites for sy in systems)
    updates = spins * 5 * steps
    roofline = far_roofline(eng, stream, spins, choice_schedule(eng), updates / (sec * 1e9))
    print(json.dumps({
        "metric": "spin-updates/ns", "workload": "batched", "value": updates / (sec * 1e9),
        "unit": "updates/ns", "ms_per_step": 1e3 * sec / steps, "steps": steps,
        "spins": spins, "systems": args.systems, "autotune_choice": choice,
        "roofline": roofline,
        "config": {"workload": "256 systems, L in {8,12,16,20,24}, 16-32 replicas each, ladders "
                               "in [0.05, 1.5], J2, J3 in [-0.1, 0.1], 1 M + 4 OR + exchange"}}),
          flush=True)
    return 0


def choice_schedule(eng):
    """True when the chosen schedule keeps replica groups in L2 across a cycle."""
    return eng.get_option(eng.OPT_GROUP_MB) > 0 or eng.get_option(eng.OPT_REPLICA_GROUP) > 0


def far_roofline(eng, stream, spins, l2_resident, value):
    """Roofline of the 16-colour over-relaxation pass (compile-time-offset
    kernel) streaming from HBM: 272 algorithmic bytes per update (the replica
    read once, one site plane written, per pass of 1/16 of the sites), timed
    over whole sweeps with replica groups switched off; plus the HBM bytes of
    the schedule that was timed."""
    eng.set_option(eng.OPT_GROUP_MB, 0)
    eng.set_option(eng.OPT_REPLICA_GROUP, 0)
    eng.set_option(eng.OPT_CHAINS, 1)
    eng.overrelax_sweep(1)
    or_s = _timed(stream, lambda: eng.overrelax_sweep(2)) / 2
    achieved = 272 * spins / or_s / 1e9  # per sweep: 16 passes x 272 B x N/16 updates
    peak, kind = hbm_peak()
    sched_bytes = 32.0 / 5 if l2_resident else 272.0
    return {"bound": "hbm", "kernel": "far_pass_kernel<site, over-relaxation>, one launch per "
                                      "colour pass over all replicas, streaming from HBM",
            "bytes_per_update": 272, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": kind, "ms_per_launch": 1e3 * or_s / 16,
            "traffic": None,
            "schedule": {"l2_resident_groups": l2_resident, "hbm_bytes_per_update": sched_bytes,
                         "achieved": value * sched_bytes, "frac": value * sched_bytes / peak}}


def run_large(args):
    """L=64 (4,194,304 sites), J1=1, J2=J3=0.05, 32 replicas on a geometric
    ladder in [0.03, 1.0], renormalised every 100 sweeps; cycles of 1
    Metropolis + 4 over-relaxation sweeps + FP64 energies + exchange; S(q) on
    a 32^3 grid; FP64-oracle error of E, M and S(q) over the first 100 sweeps
    of one replica."""
    import torch

    from cudacode_b200.engine import Engine, System, geometric_ladder
    from oracle.binding import Oracle

    temps = geometric_ladder(0.03, 1.0, 32)
    s = System(L=64, temperatures=temps, J2=0.05, J3=0.05)
    eng = Engine([s], seed=SEED + 4, renorm_every=100)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    eng.init_random()
    eng.set_cone(np.full(32, 0.3, dtype=np.float32))
    choice = eng.autotune(1, 4, 1)
    eng.cycle(1, 4, True, args.warmup)
    steps = args.steps if args.steps != 300 else 10
    sec = _timed(stream, lambda: eng.cycle(1, 4, True, steps))
    updates = 32 * s.n_sites * 5 * steps
    roofline = far_roofline(eng, stream, 32 * s.n_sites, choice_schedule(eng), updates / (sec * 1e9))
    sq_s = _timed(stream, lambda: eng.structure_factor(32, 4))
    # precision accounting: replica 0 of a 1-replica L=64 system, first 100
    # sweeps, GPU FP32 vs the host FP64 oracle from the same initial spins
    one = System(L=64, temperatures=[0.1], J2=0.05, J3=0.05)
    g1 = Engine([one], seed=SEED + 5, renorm_every=100)
    g1.init_random()
    g1.set_cone(np.array([0.5], dtype=np.float32))
    o64 = Oracle([one], seed=SEED + 5, renorm_every=100, fp64=True, threads=os.cpu_count())
    o64.set_spins(g1.get_spins())
    o64.set_cone(np.array([0.5], dtype=np.float32))
    errs = []
    for k in range(1, 101):
        g1.metropolis_sweep(1) if k % 5 == 1 else g1.overrelax_sweep(1)
        o64.metropolis_sweep(1) if k % 5 == 1 else o64.overrelax_sweep(1)
        if k in (1, 5, 10, 25, 50, 100):
            e_g, m_g = g1.observables()
            e_o, m_o = o64.observables()
            rec = {"sweep": k, "E_rel": float(abs(e_g[0] - e_o[0]) / abs(e_o[0])),
                   "M_abs_per_site": float(np.abs(m_g - m_o).max() / one.n_sites)}
            if k in (1, 100):
                sg = g1.structure_factor(4, 32)
                so = o64.structure_factor(4, 32)
                rec["Sq_rel"] = float(np.abs(sg - so).max() / np.abs(so).max())
            errs.append(dict(rec,
                             max_spin_diff=float(np.abs(g1.get_spins() -
                                                        o64.get_spins64().astype(np.float32)).max())))
    print(json.dumps({
        "metric": "spin-updates/ns", "workload": "large", "value": updates / (sec * 1e9),
        "unit": "updates/ns", "ms_per_step": 1e3 * sec / steps, "steps": steps,
        "structure_factor_32cubed_ms": 1e3 * sq_s, "autotune_choice": choice,
        "roofline": roofline,
        "fp64_error_first_100_sweeps": errs,
        "config": {"workload": "L=64, J1=1, J2=J3=0.05, 32 replicas in [0.03, 1.0], renormalise "
                               "every 100 sweeps, 1 M + 4 OR + exchange; S(q) 32^3, stride 4"}}),
          flush=True)
    return 0


def run_aniso(args):
    """The reference's anisotropic model (bond matrices of J1..J4 at the
    reference's default couplings, g-tensor Zeeman field of B = 1 T along
    [001], gxy = 2.4, gz = 0.3): L=32, 64 replicas on a geometric ladder in
    [0.02, 2.0], cycles of 1 Metropolis + 4 over-relaxation sweeps + FP64
    energies + exchange; host baseline: the oracle port on 4 replicas."""
    import time

    import torch

    from cudacode_b200.engine import (Engine, System, geometric_ladder, reference_exchange,
                                      reference_field)
    from oracle.binding import Oracle

    J = (-0.09 / 0.29, -0.22 / 0.29, -1.00, 0.0)
    A = reference_exchange(*J)
    f = reference_field(2.4, 0.3, [0.0, 0.0, 1.0])
    temps = geometric_ladder(0.02, 2.0, 64)
    s = System(L=32, temperatures=temps, J1=0.0)
    eng = Engine([s], seed=SEED + 6)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    eng.set_exchange(A, f)
    eng.init_random()
    eng.set_cone(np.full(64, 0.3, dtype=np.float32))
    choice = eng.autotune(1, 4, 1)
    eng.cycle(1, 4, True, max(3, args.warmup))
    steps = args.steps if args.steps != 300 else 100
    sec = _timed(stream, lambda: eng.cycle(1, 4, True, steps))
    updates = 64 * s.n_sites * 5 * steps
    # host: the oracle port on 4 of the replicas, all cores
    host = System(L=32, temperatures=temps[:4], J1=0.0)
    o = Oracle([host], seed=SEED + 6, threads=os.cpu_count())
    o.set_exchange(A, f)
    o.init_random()
    o.set_cone(np.full(4, 0.3, dtype=np.float32))
    t0 = time.perf_counter()
    o.cycle(1, 4, True, 3)
    host_s = time.perf_counter() - t0
    host_rate = 4 * host.n_sites * 5 * 3 / (host_s * 1e9)
    print(json.dumps({
        "metric": "spin-updates/ns", "workload": "aniso", "value": updates / (sec * 1e9),
        "unit": "updates/ns", "ms_per_step": 1e3 * sec / steps, "steps": steps,
        "autotune_choice": choice,
        "cpu_baseline": {"value": host_rate, "unit": "updates/ns", "cores": os.cpu_count(),
                         "kind": "port", "sample": "4 replicas x 3 cycles"},
        "config": {"workload": "anisotropic J1-J4 model at the reference's default couplings "
                               "(-0.09/0.29, -0.22/0.29, -1, 0) with a 1 T [001] field (gxy 2.4, "
                               "gz 0.3): L=32, 64 replicas in [0.02, 2.0], 1 M + 4 OR + "
                               "exchange"}}), flush=True)
    return 0


def run_learned(args):
    """Energy ESS/s at T=0.05 of the learned method (plain PT cycles with
    learned tetrahedron sweeps, at its best schedule) against the plain PT
    cycle of the benchmark (1 Metropolis + 4 over-relaxation sweeps per
    exchange) and against the plain method at its own best schedule
    (`ratio_vs_plain_best_schedule`), at L=16, 8 temperatures on a geometric
    ladder in [0.05, 0.5].
    The network is trained on the GPU on ~10^6 tetrahedra from the plain
    chains first. Device time by CUDA events; tau_int by Sokal windowing."""
    import torch

    from cudacode_b200 import stats
    from cudacode_b200.engine import Engine, System, geometric_ladder

    Ll, nT = 16, 8
    temps = geometric_ladder(0.05, 0.5, nT)
    cycles = args.steps if args.steps != 300 else 20000
    eng = Engine([System(L=Ll, temperatures=temps)], seed=SEED + 3)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    eng.init_random()
    eng.tune_cone(0.5, 20, 5, 4)
    eng.cycle(1, 4, True, 2000)
    eng.tet_init(seed=7, sample_capacity=1 << 20)
    n_samples = 0
    while n_samples < (1 << 20):
        eng.cycle(1, 4, True, 25)
        n_samples += eng.tet_collect(1)
    t0 = time.perf_counter()
    loss0 = eng.tet_train(1, 4096, 2e-3)
    loss = eng.tet_train(1500, 4096, 2e-3)
    loss = eng.tet_train(4500, 4096, 5e-4)
    loss = eng.tet_train(3000, 4096, 2e-4)
    train_s = time.perf_counter() - t0
    choice = eng.autotune(1, 4, 5)

    def measure(n_tet, n_metro=1, n_or=4):
        eng.enable_history(cycles)
        eng.tet_reset_acceptance()
        run = (lambda k: eng.cycle(n_metro, n_or, True, k)) if n_tet == 0 else \
            (lambda k: eng.cycle_tet(n_metro, n_or, n_tet, True, k))
        run(args.warmup)
        eng.enable_history(cycles)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        run(cycles)
        b.record(stream)
        torch.cuda.synchronize()
        sec = a.elapsed_time(b) / 1e3
        h = eng.history()
        taus = [stats.tau_int(h[:, t]) for t in range(nT)]
        ess_s = [len(h) / (2 * tau) / sec for tau in taus]
        means = [stats.mean_error(h[:, t]) for t in range(nT)]
        acc, prop = eng.tet_acceptance()
        return {"schedule": {"metropolis": n_metro, "overrelax": n_or, "tetrahedron": n_tet},
                "seconds": sec, "us_per_cycle": 1e6 * sec / cycles, "tau_int": taus,
                "ess_per_s": ess_s,
                "E_per_site": [(m / (16 * Ll ** 3), e / (16 * Ll ** 3)) for m, e in means],
                "tet_acceptance": (acc / np.maximum(prop, 1)).tolist() if n_tet else None}

    # Schedules are chosen on one set of chains and the ratio is measured on
    # fresh, longer chains of the two winners (no selection bias); the plain
    # method gets its own best schedule.
    plain_runs = [measure(0, m, o) for m, o in
                  ((1, 4), (1, 0), (1, 1), (1, 2), (2, 0), (2, 1), (2, 4), (3, 0), (3, 1),
                   (4, 0), (4, 1))]
    schedules = [measure(t, m, o) for t, m, o in
                 ((1, 1, 4), (1, 1, 1), (1, 1, 0), (1, 0, 0), (1, 0, 1), (2, 0, 0), (2, 0, 1),
                  (1, 2, 0), (1, 1, 2), (1, 2, 1), (3, 0, 0), (2, 1, 0), (3, 1, 0))]
    best_plain = max(plain_runs, key=lambda r: r["ess_per_s"][0])["schedule"]
    best_learned = max(schedules, key=lambda r: r["ess_per_s"][0])["schedule"]
    final_cycles = 3 * cycles

    def remeasure(sch):
        nonlocal cycles
        keep, cycles = cycles, final_cycles
        try:
            return measure(sch["tetrahedron"], sch["metropolis"], sch["overrelax"])
        finally:
            cycles = keep

    standard = {"metropolis": 1, "overrelax": 4, "tetrahedron": 0}
    plain = remeasure(standard)  # the plain PT cycle of the benchmark (1 M + 4 OR)
    plain_best = plain if best_plain == standard else remeasure(best_plain)
    learned = remeasure(best_learned)
    # the same schedule with all four sites from the network's vMFs
    eng.tet_set_proposal(0)
    learned_product = remeasure(best_learned)
    eng.tet_set_proposal(1)
    ratio = learned["ess_per_s"][0] / plain["ess_per_s"][0]
    ratio_best = learned["ess_per_s"][0] / plain_best["ess_per_s"][0]
    agree = [abs(p[0] - q[0]) / max(np.hypot(p[1], q[1]), 1e-30)
             for p, q in zip(plain["E_per_site"], learned["E_per_site"])]
    line = {"metric": "energy ESS/s learned-proposal vs plain at T=0.05", "value": ratio,
            "unit": "x", "higher_is_better": True, "n_gpus": 1, "steps": cycles,
            "warmup": args.warmup, "dtype": "f32 spins, bf16 MLP",
            "data": "synthetic (random unit spins from Philox seed)",
            "config": {"workload": "learned tetrahedron proposal: L=16 (65,536 sites), J1=1 AFM, "
                                   "8 temperatures geometric in [0.05, 0.5]; learned method at its "
                                   "best schedule (chosen on separate chains) vs the plain 1 M + "
                                   "4 OR cycle; ratio_vs_plain_best_schedule: vs the plain "
                                   "method's own best schedule",
                       "training_samples": n_samples,
                       "train_seconds": train_s, "loss_first": loss0, "loss_last": loss},
            "kernels_autotune_choice": choice,
            "plain": plain, "learned": learned,
            "learned_product_proposal": {k: learned_product[k] for k in
                                         ("us_per_cycle", "tau_int", "ess_per_s",
                                          "tet_acceptance")},
            "ratio_vs_plain_best_schedule": ratio_best, "plain_best": plain_best,
            "selection_cycles": cycles, "final_cycles": final_cycles,
            "plain_schedules": [{"schedule": r["schedule"], "us_per_cycle": r["us_per_cycle"],
                                 "tau_int_T0.05": r["tau_int"][0],
                                 "ess_per_s_T0.05": r["ess_per_s"][0]} for r in plain_runs],
            "learned_schedules": [{"schedule": r["schedule"], "us_per_cycle": r["us_per_cycle"],
                                   "tau_int_T0.05": r["tau_int"][0],
                                   "ess_per_s_T0.05": r["ess_per_s"][0]} for r in schedules],
            "energy_agreement_sigma": agree}
    print(json.dumps(line), flush=True)
    return 0


def learned_leg(cycles: int = 60000, warmup: int = 2000) -> dict:
    """The second half of the metric, compact: energy ESS/s at T=0.05 of the
    learned method against the plain method, each at a fixed schedule chosen
    beforehand by the full learned workload (`--workload learned`): plain
    3 Metropolis + 1 over-relaxation sweeps per exchange (the plain method's
    best), learned 2 tetrahedron sweeps per exchange. L=16 (65,536 sites),
    8 temperatures geometric in [0.05, 0.5]; the network trained on the GPU
    on 2^20 tetrahedra from the plain chains; chains of `cycles` exchange
    cycles each, device time by CUDA events, tau_int by Sokal windowing."""
    import torch

    from cudacode_b200 import stats
    from cudacode_b200.engine import Engine, System, geometric_ladder

    Ll, nT = 16, 8
    temps = geometric_ladder(0.05, 0.5, nT)
    eng = Engine([System(L=Ll, temperatures=temps)], seed=SEED + 3)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    eng.init_random()
    eng.tune_cone(0.5, 20, 5, 1)
    eng.cycle(3, 1, True, warmup)
    eng.tet_init(seed=7, sample_capacity=1 << 20)
    n_samples = 0
    while n_samples < (1 << 20):
        eng.cycle(3, 1, True, 25)
        n_samples += eng.tet_collect(1)
    t0 = time.perf_counter()
    eng.tet_train(1500, 4096, 2e-3)
    eng.tet_train(4500, 4096, 5e-4)
    loss = eng.tet_train(3000, 4096, 2e-4)
    train_s = time.perf_counter() - t0
    choice = eng.autotune(3, 1, 5)
    n = 16 * Ll ** 3

    def chain(n_metro, n_or, n_tet):
        run = (lambda k: eng.cycle(n_metro, n_or, True, k)) if n_tet == 0 else \
            (lambda k: eng.cycle_tet(n_metro, n_or, n_tet, True, k))
        run(warmup)
        eng.enable_history(cycles)
        eng.tet_reset_acceptance()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        run(cycles)
        b.record(stream)
        torch.cuda.synchronize()
        sec = a.elapsed_time(b) / 1e3
        h = eng.history()
        tau = stats.tau_int(h[:, 0])
        means = [stats.mean_error(h[:, t] / n) for t in range(nT)]
        out = {"schedule": {"metropolis": n_metro, "overrelax": n_or, "tetrahedron": n_tet},
               "us_per_cycle": 1e6 * sec / cycles, "tau_int_T0.05": tau,
               "ess_per_s_T0.05": cycles / (2 * tau) / sec, "E_per_site": means}
        if n_tet:
            acc, prop = eng.tet_acceptance()
            out["tet_acceptance_T0.05"] = float(acc[0] / max(prop[0], 1))
        return out

    plain = chain(3, 1, 0)
    # the learned cycle at its own best replica grouping (the autotuner times
    # plain cycles only): a few groupings timed on untimed warm-up cycles;
    # every grouping gives the same chain
    tet_timing = {}
    for group, chains in ((0, 1), (8, 1), (4, 2), (2, 4), (1, 8), (2, 2)):
        eng.set_option(eng.OPT_REPLICA_GROUP, group)
        eng.set_option(eng.OPT_CHAINS, chains)
        eng.cycle_tet(0, 0, 2, True, 20)
        torch.cuda.synchronize()
        tet_timing[(group, chains)] = _timed(stream, lambda: eng.cycle_tet(0, 0, 2, True, 200))
    tet_best = min(tet_timing, key=tet_timing.get)
    eng.set_option(eng.OPT_REPLICA_GROUP, tet_best[0])
    eng.set_option(eng.OPT_CHAINS, tet_best[1])
    learned = chain(0, 0, 2)
    learned["replica_group_chains"] = list(tet_best)
    learned["groupings_us_per_cycle"] = {f"{g}x{c}": 1e6 * t / 200 for (g, c), t in tet_timing.items()}
    agree = [abs(p[0] - q[0]) / max(float(np.hypot(p[1], q[1])), 1e-30)
             for p, q in zip(plain["E_per_site"], learned["E_per_site"])]
    eng.close()
    return {"metric": "energy ESS/s at T=0.05, learned proposal vs the plain method at its best "
                      "schedule",
            "ratio_vs_plain_best_schedule": learned["ess_per_s_T0.05"] / plain["ess_per_s_T0.05"],
            "plain": plain, "learned": learned, "cycles_per_chain": cycles,
            "energy_agreement_sigma_max": max(agree),
            "config": {"workload": "L=16 (65,536 sites), J1=1 AFM, 8 temperatures geometric in "
                                   "[0.05, 0.5]", "training_samples": n_samples,
                       "train_seconds": train_s, "loss_last": loss,
                       "autotune_choice_plain": choice}}


STEP_PROFILE = os.path.join(ROOT, "profiles", "pt_step_L32_R64_instructions.md")


def profiled_step(kernel_desc: dict):
    """Per-update figures of one step of the timed kernels, from the committed
    ncu summary (blocks of lines 'schedule: k=v ...', then
    'warp_instructions_per_update: X', 'l2_bytes_per_update: Y',
    'l2_peak_gbs: Z'); None when no block is of the timed kernels."""
    keys = ("warp_instructions_per_update", "l2_bytes_per_update", "l2_peak_gbs")
    try:
        blocks = []
        with open(STEP_PROFILE) as f:
            for line in f:
                if line.startswith("schedule:"):
                    sched = dict(kv.split("=") for kv in line.split(":", 1)[1].split())
                    blocks.append((sched, {}))
                elif blocks:
                    for key in keys:
                        if line.startswith(key + ":"):
                            blocks[-1][1][key] = float(line.split(":", 1)[1])
        for sched, vals in blocks:
            if len(vals) == len(keys) and all(str(kernel_desc.get(k)) == v
                                              for k, v in sched.items()):
                return vals
    except (OSError, ValueError):
        pass
    return None


def relaunch_under_torchrun(args) -> int | None:
    """`--gpus N` (N > 1) outside torchrun runs this script again as N ranks
    through torch.distributed.run (one process per GPU, 127.0.0.1
    rendezvous); under torchrun, WORLD_SIZE must equal N."""
    world = os.environ.get("WORLD_SIZE")
    if world is None:
        if args.gpus <= 1:
            return None
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
               f"--nproc-per-node={args.gpus}", "--master-addr", "127.0.0.1",
               "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]
        return subprocess.call(cmd)
    if int(world) != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}", file=sys.stderr)
        return 2
    return None


def run_dry(args) -> int:
    """Launcher check without a GPU: the ranks meet over gloo, and rank 0
    prints the line's n_gpus (the world size)."""
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("gloo", timeout=timedelta(seconds=60))
        t = __import__("torch").tensor([rank])
        dist.all_reduce(t)
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"dry_run": True, "n_gpus": world, "gpus_arg": args.gpus}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned-proposal ESS/s leg of the default line")
    ap.add_argument("--dry-run", action="store_true",
                    help="check the launcher only: ranks meet over gloo, no GPU work")
    ap.add_argument("--L", type=int, default=L, help="lattice size (profiling cases)")
    ap.add_argument("--replicas", type=int, default=R_PER_GPU, help="replicas per GPU")
    ap.add_argument("--workload", default="pt",
                    choices=["pt", "learned", "small", "batched", "large", "aniso"],
                    help="pt: the parallel-tempering benchmark (default); learned: energy "
                         "ESS/s of the learned tetrahedron proposal vs the plain method; "
                         "small: L=4 on the GPU and on the host; batched: 256 uneven "
                         "systems; large: L=64 with J2/J3, S(q) and FP64 error accounting; "
                         "aniso: the reference's anisotropic J1-J4 model with a field")
    ap.add_argument("--kernel", default="auto",
                    choices=["auto", "pass", "cluster", "grouped", "wave"],
                    help="auto: autotuner picks; pass: one launch per colour pass; "
                         "cluster: cluster-resident cycle kernel; grouped: per-pass kernels "
                         "over replica groups (--group) on concurrent chains (--chains); "
                         "wave: the work-queue cycle kernel over replica groups (--group), "
                         "pass forms --site-mode")
    ap.add_argument("--group", type=int, default=4)
    ap.add_argument("--chains", type=int, default=2)
    ap.add_argument("--site-mode", type=int, default=None,
                    help="J1 pass forms (bit 0 Metropolis, bit 1 over-relaxation one site "
                         "per thread) for --kernel grouped / wave (wave default 3)")
    ap.add_argument("--systems", type=int, default=256,
                    help="--workload batched: number of systems (256 in the configuration)")
    ap.add_argument("--group-mb", type=int, default=None,
                    help="--workload batched --kernel wave: MB of spins per work-queue group "
                         "(0: one group)")
    ap.add_argument("--cluster-size", type=int, default=None,
                    help="CTAs per cluster of --kernel cluster (default: the engine's)")
    ap.add_argument("--stagger", type=int, default=None,
                    help="--kernel grouped: each odd chain starts after the preceding chain's first "
                         "N passes")
    ap.add_argument("--fixed-l", type=int, default=1, choices=[0, 1],
                    help="1: per-pass J1 kernels compiled for L = 16 / 32 (default); "
                         "0: the run-time-L kernels")
    args = ap.parse_args()
    rc = relaunch_under_torchrun(args)
    if rc is not None:
        return rc
    if args.dry_run:
        return run_dry(args)
    if args.workload == "learned":
        return run_learned(args)
    if args.workload == "small":
        return run_small(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "large":
        return run_large(args)
    if args.workload == "aniso":
        return run_aniso(args)
    set_workload(args.L, args.replicas)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    from cudacode_b200.engine import Engine, System, geometric_ladder

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        # the communicator's INIT lines name the ranks that joined
        os.environ.setdefault("NCCL_DEBUG", "INFO")
        os.environ.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    n_gpus = world

    temps = geometric_ladder(T_MIN, T_MAX, R_PER_GPU * n_gpus)
    sysd = System(L=L, temperatures=temps, n_replicas=R_PER_GPU, replica_offset=R_PER_GPU * rank)
    eng = Engine([sysd], seed=SEED, device=local)
    stream = torch.cuda.Stream(device=local)
    eng.set_stream(stream.cuda_stream)
    eng.init_random()
    cones = np.full(len(temps), 0.3, dtype=np.float32)
    eng.set_cone(cones)
    variant = None
    eng.set_option(eng.OPT_J1_FIXED_L, args.fixed_l)
    if args.kernel == "auto":
        # the autotuner's cycles are untimed warm-up Monte Carlo steps; on a
        # shard (one of several ranks) it runs them without the local
        # exchange, and each rank keeps its own fastest variant (every
        # variant gives the same chain)
        variant = eng.autotune(N_METRO, N_OR, 16)
    else:
        eng.set_option(eng.OPT_CYCLE_KERNEL, {"cluster": 1, "wave": 2}.get(args.kernel, 0))
        if args.kernel == "cluster" and args.cluster_size is not None:
            eng.set_option(eng.OPT_CLUSTER_SIZE, args.cluster_size)
        if args.kernel in ("grouped", "wave"):
            eng.set_option(eng.OPT_REPLICA_GROUP, args.group)
        if args.kernel == "grouped":
            eng.set_option(eng.OPT_CHAINS, args.chains)
        if args.kernel == "wave":
            eng.set_option(eng.OPT_J1_SITE_MODE, 3 if args.site_mode is None else args.site_mode)
        elif args.kernel == "grouped" and args.site_mode is not None:
            eng.set_option(eng.OPT_J1_SITE_MODE, args.site_mode)
        if args.kernel == "grouped" and args.stagger is not None:
            eng.set_option(eng.OPT_CHAIN_STAGGER, args.stagger)
    options = {n: eng.get_option(getattr(Engine, "OPT_" + n)) for n in KERNEL_OPTIONS}
    kernel_desc = {"cycle_kernel": options["CYCLE_KERNEL"],
                   "cluster_size": options["CLUSTER_SIZE"],
                   "j1_kernel": options["J1_KERNEL"],
                   "replica_group": options["REPLICA_GROUP"],
                   "chains": options["CHAINS"],
                   "j1_site_mode": options["J1_SITE_MODE"],
                   "j1_fixed_l": options["J1_FIXED_L"],
                   "chain_stagger": options["CHAIN_STAGGER"], "autotune_choice": variant}
    if world > 1:
        from cudacode_b200.distributed import EngineBackend, ShardedPT
        pt = ShardedPT(EngineBackend(eng, torch.device(f"cuda:{local}")), R_PER_GPU * n_gpus)

    def step():
        if world == 1:
            eng.cycle(N_METRO, N_OR, True, 1)
        else:
            with torch.cuda.stream(stream):
                pt.cycle(N_METRO, N_OR)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            torch.cuda.synchronize()
            launches0 = eng.launch_count()
            start.record(stream)
            for _ in range(args.steps):
                step()
            stop.record(stream)
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            launches_timed = eng.launch_count() - launches0
        eng.synchronize()  # raises if a bounded device wait ran out
        ms = start.elapsed_time(stop)
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    updates = R_PER_GPU * n_gpus * 16 * L ** 3 * (N_METRO + N_OR) * args.steps
    value = updates / (ms * 1e6)
    clocks = clk.summary()

    peak, peak_kind = hbm_peak()
    # End to end through the C-ABI with host buffers: each step uploads the cone
    # widths from pinned host memory, runs the cycle, and copies the FP64
    # energies and magnetisations it computed to pinned host memory; the
    # copies are queued on the engine's stream (pyro_set_cone_async,
    # pyro_last_observables_async), so step k + 1 is queued while step k
    # runs, and the wall clock ends when every step's results are on the host.
    e2e_steps = 0 if args.no_e2e else max(40, args.steps)
    n_loc = R_PER_GPU
    cones_h = torch.from_numpy(cones).pin_memory()
    e_h = torch.empty((max(e2e_steps, 1), n_loc), dtype=torch.float64).pin_memory()
    m_h = torch.empty((max(e2e_steps, 1), n_loc, 3), dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        eng.set_cone_async(cones_h.numpy())
        step()
        eng.last_observables_async(e_h[k].numpy(), m_h[k].numpy())  # this step's results
    eng.synchronize()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if e2e_steps and not np.all(np.isfinite(e_h.numpy())):
        raise RuntimeError("e2e: non-finite energies")
    e2e_value = (R_PER_GPU * n_gpus * 16 * L ** 3 * (N_METRO + N_OR) * e2e_steps / (e2e_s * 1e9)
                 if e2e_steps else None)
    if world > 1 and e2e_value is not None:
        t = torch.tensor([e2e_value], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        e2e_value = float(t.item()) * 1.0

    # Roofline of the timed step. With the work-queue kernel (or replica
    # groups) a replica stays in L2 for all 20 passes of its cycle, so the
    # step's algorithmic HBM bytes are one read and one write of every spin
    # per cycle: 32 B per 5 updates. The binding block reports the step's
    # instruction-issue fraction (warp instructions per update from the
    # committed ncu summary, times the updates, over 4 schedulers x the SMs x
    # the sampled SM clock x the time) and its L2 fraction (L2 bytes per
    # update from the same summary over the L2 peak).
    l2_resident = (kernel_desc["replica_group"] > 0 or kernel_desc["cycle_kernel"] > 0)
    sched_bytes = 32.0 / (N_METRO + N_OR) if l2_resident else float(BYTES_PER_UPDATE_PASS)
    step_ms = ms / args.steps
    step_updates = R_PER_GPU * 16 * L ** 3 * (N_METRO + N_OR)  # per GPU
    achieved = step_updates * sched_bytes / (step_ms * 1e-3) / 1e9
    wave = kernel_desc["cycle_kernel"] == 2
    prof = profiled_step(kernel_desc) if (L, R_PER_GPU) == (32, 64) else None
    props = torch.cuda.get_device_properties(local)
    binding = None
    if prof and clocks.get("sm_mhz"):
        issue_slots = props.multi_processor_count * 4 * clocks["sm_mhz"] * 1e6 * step_ms * 1e-3
        ipu = prof["warp_instructions_per_update"]
        l2_gbs = step_updates * prof["l2_bytes_per_update"] / (step_ms * 1e-3) / 1e9
        binding = {
            "resource": "the chains of dependent colour-pass launches (neither instruction "
                        "issue nor L2 bandwidth saturates)",
            "issue": {"warp_instructions_per_update": ipu,
                      "frac": ipu * step_updates / issue_slots,
                      "sm_mhz": clocks["sm_mhz"], "sms": props.multi_processor_count},
            "l2": {"bytes_per_update": prof["l2_bytes_per_update"], "achieved_gbs": l2_gbs,
                   "peak_gbs": prof["l2_peak_gbs"], "frac": l2_gbs / prof["l2_peak_gbs"]},
            "source": "profiles/pt_step_L32_R64_instructions.md (ncu smsp__inst_executed.sum "
                      "over one step's launches; lts__t_bytes.sum per launch)"}

    # The streaming form of the same passes, for comparison: one launch per
    # colour pass over all replicas, 80 algorithmic bytes per update.
    pass_updates = R_PER_GPU * 16 * L ** 3 // 4
    or_ms = None
    if world == 1:
        eng.set_option(eng.OPT_CYCLE_KERNEL, 0)
        eng.set_option(eng.OPT_REPLICA_GROUP, 0)
        eng.set_option(eng.OPT_CHAINS, 1)
        n_or_timed = 20
        with torch.cuda.stream(stream):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            eng.overrelax_sweep(2)
            a.record(stream)
            eng.overrelax_sweep(n_or_timed)
            b.record(stream)
            torch.cuda.synchronize()
            or_ms = a.elapsed_time(b) / (n_or_timed * 4)  # per colour pass
    stream_gbs = pass_updates * BYTES_PER_UPDATE_PASS / (or_ms * 1e-3) / 1e9 if or_ms else None
    eng.close()

    cpu, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, parity = cpu_baseline_and_parity(options)
    learned = None
    if rank == 0 and world == 1 and not args.no_learned:
        learned = learned_leg()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "updates/ns", "n_gpus": n_gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (random unit spins from Philox seed)",
            "config": dict(workload_config(n_gpus), kernels=kernel_desc),
            "roofline": {
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "kernel": ("j1_wave_kernel: the step's sweeps and energies in one work-queue "
                           "launch (plus a 33 KB memset and the exchange kernel)" if wave else
                           "the step's per-pass J1 kernels over replica groups" if l2_resident
                           else "j1_pass_kernel, one launch per colour pass"),
                "bytes_per_update": sched_bytes, "updates_per_launch": step_updates,
                "ms_per_launch": step_ms,
                "traffic": None,
                "binding": binding,
                "note": ("HBM is not the bound of this schedule: each replica group stays in L2 "
                         "for its cycle, so HBM sees one read and one write per spin per cycle; "
                         "binding gives the step's instruction-issue and L2 fractions"
                         if l2_resident else "every pass streams the lattice from HBM"),
                "streaming_pass": {
                    "what": "j1_pass_kernel<colour, over-relaxation> streaming from HBM, one "
                            "launch per colour pass over all replicas (not the timed schedule)",
                    "bytes_per_update": BYTES_PER_UPDATE_PASS, "updates_per_launch": pass_updates,
                    "ms_per_launch": or_ms, "achieved": stream_gbs,
                    "frac": stream_gbs / peak if stream_gbs else None,
                    "traffic": profiled_traffic() if (L, R_PER_GPU) == (32, 64) else None}},
            "cpu_baseline": cpu,
            "parity": parity,
            "learned": learned,
            "e2e": {"value": e2e_value, "unit": "updates/ns",
                    "h2d_bytes_per_step": 4 * len(temps),
                    "d2h_bytes_per_step": 8 * R_PER_GPU + 24 * R_PER_GPU},
            "gpu_launches": launches_timed,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
