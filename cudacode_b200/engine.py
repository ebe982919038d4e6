"""Python binding of the C-ABI in ``include/pyro.h`` (ctypes).

The engine runs only on the GPU: loading fails loudly when ``libpyro.so`` is
missing, and every call raises :class:`PyroError` when the library returns a
negative status. Host arrays are numpy arrays owned by the caller.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libpyro.so")

PYRO_OK = 0
ERRORS = {
    -1: "PYRO_ERR_ARG",
    -2: "PYRO_ERR_CUDA",
    -3: "PYRO_ERR_TIMEOUT",
    -4: "PYRO_ERR_NAN",
    -5: "PYRO_ERR_IO",
    -6: "PYRO_ERR_STATE",
    -7: "PYRO_ERR_NOMEM",
}


class PyroError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


class SystemDesc(C.Structure):
    _fields_ = [
        ("L", C.c_int),
        ("n_replicas", C.c_int),
        ("replica_offset", C.c_int),
        ("n_temperatures", C.c_int),
        ("temperatures", C.POINTER(C.c_double)),
        ("J1", C.c_double),
        ("J2", C.c_double),
        ("J3", C.c_double),
        ("J3b", C.c_double),
    ]


class Config(C.Structure):
    _fields_ = [
        ("n_systems", C.c_int),
        ("systems", C.POINTER(SystemDesc)),
        ("seed", C.c_uint64),
        ("device", C.c_int),
        ("renorm_every", C.c_int),
    ]


_lib = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Loads libpyro.so (built in-tree by ``python -m cudacode_b200.build``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -m cudacode_b200.build`; "
            "the engine has no CPU fallback")
    lib = C.CDLL(path)
    P = C.c_void_p
    i, d, f = C.c_int, C.c_double, C.c_float
    pd, pf, pi = C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_int)
    pu64 = C.POINTER(C.c_uint64)
    sig = {
        "pyro_create": (i, [C.POINTER(Config), C.POINTER(P)]),
        "pyro_destroy": (i, [P]),
        "pyro_last_error": (C.c_char_p, [P]),
        "pyro_version": (i, []),
        "pyro_neighbour_table": (i, [i, pi]),
        "pyro_set_option": (i, [P, i, i]),
        "pyro_get_option": (i, [P, i, pi]),
        "pyro_autotune": (i, [P, i, i, i, pi]),
        "pyro_set_stream": (i, [P, P]),
        "pyro_get_stream": (P, [P]),
        "pyro_synchronize": (i, [P]),
        "pyro_snapshot": (i, [P]),
        "pyro_set_system_keys": (i, [P, i, i, i]),
        "pyro_system_info": (i, [P, i, pi, pi, pi, pi]),
        "pyro_init_random": (i, [P]),
        "pyro_set_spins": (i, [P, i, pf]),
        "pyro_get_spins": (i, [P, i, pf]),
        "pyro_set_spins_planar": (i, [P, i, pd]),
        "pyro_get_spins_planar": (i, [P, i, pd]),
        "pyro_set_spins_device": (i, [P, i, P]),
        "pyro_get_spins_device": (i, [P, i, P]),
        "pyro_metropolis_sweep": (i, [P, i]),
        "pyro_overrelax_sweep": (i, [P, i]),
        "pyro_set_cone": (i, [P, i, pf]),
        "pyro_get_cone": (i, [P, i, pf]),
        "pyro_get_acceptance": (i, [P, i, pu64, pu64]),
        "pyro_reset_acceptance": (i, [P]),
        "pyro_tune_cone": (i, [P, d, i, i, i]),
        "pyro_observables": (i, [P, i, pd, pd]),
        "pyro_observables_device": (i, [P, i, P, P]),
        "pyro_get_temperatures": (i, [P, i, pd]),
        "pyro_get_permutation": (i, [P, i, pi]),
        "pyro_pt_swap": (i, [P, i, pi]),
        "pyro_pt_swap_global": (i, [P, i, P, i]),
        "pyro_get_swap_stats": (i, [P, i, pu64, pu64]),
        "pyro_cycle": (i, [P, i, i, i, i]),
        "pyro_enable_history": (i, [P, i]),
        "pyro_get_history": (i, [P, i, pd, pi]),
        "pyro_get_sweep_count": (i, [P, pu64]),
        "pyro_get_launch_count": (i, [P, pu64]),
        "pyro_check_spins": (i, [P, f, C.POINTER(C.c_longlong)]),
        "pyro_structure_factor": (i, [P, i, i, i, i, pd]),
        "pyro_tet_init": (i, [P, C.c_uint64, C.c_longlong]),
        "pyro_tet_set_weights": (i, [P, pf, i]),
        "pyro_tet_get_weights": (i, [P, pf, i]),
        "pyro_tet_sweep": (i, [P, i]),
        "pyro_tet_trace_pass": (i, [P, i, i, i, pf]),
        "pyro_tet_set_kernel": (i, [P, i]),
        "pyro_tet_set_proposal": (i, [P, i]),
        "pyro_tet_acceptance": (i, [P, i, pu64, pu64]),
        "pyro_tet_reset_acceptance": (i, [P]),
        "pyro_tet_collect": (i, [P, i, i, C.POINTER(C.c_longlong)]),
        "pyro_tet_samples": (i, [P, pf, pf, C.c_longlong, C.POINTER(C.c_longlong)]),
        "pyro_tet_train": (i, [P, i, i, f, pd]),
        "pyro_tet_forward": (i, [P, pf, i, pf]),
        "pyro_tet_forward_device": (i, [P, C.c_void_p, i, C.c_void_p]),
        "pyro_last_observables_device": (i, [P, i, C.c_void_p, C.c_void_p]),
        "pyro_set_cone_async": (i, [P, i, C.c_void_p]),
        "pyro_last_observables_async": (i, [P, i, C.c_void_p, C.c_void_p]),
        "pyro_last_observables": (i, [P, i, pd, pd]),
        "pyro_tet_set_forward": (i, [P, i]),
        "pyro_tet_gradient": (i, [P, pf, pf, i, pf, pd]),
        "pyro_cycle_tet": (i, [P, i, i, i, i, i]),
        "pyro_save_checkpoint": (i, [P, C.c_char_p]),
        "pyro_load_checkpoint": (i, [P, C.c_char_p]),
        "pyro_save_configurations": (i, [P, i, C.c_char_p, i]),
        "pyro_read_configurations": (i, [P, i, C.c_char_p, i]),
        "pyro_set_exchange": (i, [P, i, pd, pd]),
        "pyro_get_exchange": (i, [P, i, pd, pd, pi]),
        "pyro_reference_exchange": (i, [d, d, d, d, pd]),
        "pyro_reference_field": (i, [d, d, pd, pd]),
        "pyro_reference_gtensor": (i, [d, d, pd]),
        "pyro_sublattice_magnetisation": (i, [P, i, pd]),
        "pyro_order_parameters": (i, [P, i, pd]),
        "pyro_ising_configuration": (i, [P, i, i, pi]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


@dataclass
class System:
    """One pyrochlore lattice: L^3 cubic cells (16 L^3 sites) and a ladder."""

    L: int
    temperatures: Sequence[float]
    J1: float = 1.0
    J2: float = 0.0
    J3: float = 0.0
    J3b: float = 0.0
    n_replicas: int | None = None  # default: the whole ladder
    replica_offset: int = 0

    @property
    def n_sites(self) -> int:
        return 16 * self.L ** 3

    @property
    def n_colours(self) -> int:
        return 16 if (self.J2 or self.J3 or self.J3b) else 4

    def replicas(self) -> int:
        return len(self.temperatures) if self.n_replicas is None else self.n_replicas


def neighbour_table(site: int) -> np.ndarray:
    """(30, 4) array of (dx, dy, dz, target site) for cubic-cell site `site`."""
    lib = load_library()
    out = np.empty(120, dtype=np.int32)
    rc = lib.pyro_neighbour_table(site, _ptr(out, C.c_int))
    if rc != PYRO_OK:
        raise PyroError(rc, "pyro_neighbour_table")
    return out.reshape(30, 4)


def reference_exchange(J1: float, J2: float, J3: float, J4: float) -> np.ndarray:
    """Bond matrices (4, 4, 3, 3) of the reference's J1..J4 model in this
    engine's convention (energies and temperatures as the reference's)."""
    out = np.empty(144, dtype=np.float64)
    rc = load_library().pyro_reference_exchange(J1, J2, J3, J4, _ptr(out, C.c_double))
    if rc != PYRO_OK:
        raise PyroError(rc, "pyro_reference_exchange")
    return out.reshape(4, 4, 3, 3)


def reference_field(gxy: float, gz: float, B) -> np.ndarray:
    """Site fields (4, 3) of a field B (tesla) with the reference's g-tensors."""
    b = np.ascontiguousarray(B, dtype=np.float64).reshape(3)
    out = np.empty(12, dtype=np.float64)
    rc = load_library().pyro_reference_field(gxy, gz, _ptr(b, C.c_double), _ptr(out, C.c_double))
    if rc != PYRO_OK:
        raise PyroError(rc, "pyro_reference_field")
    return out.reshape(4, 3)


def reference_gtensor(gxy: float, gz: float) -> np.ndarray:
    """g-tensors (4, 3, 3) of the four sublattices."""
    out = np.empty(36, dtype=np.float64)
    rc = load_library().pyro_reference_gtensor(gxy, gz, _ptr(out, C.c_double))
    if rc != PYRO_OK:
        raise PyroError(rc, "pyro_reference_gtensor")
    return out.reshape(4, 3, 3)


def geometric_ladder(t_min: float, t_max: float, n: int) -> list[float]:
    if n == 1:
        return [float(t_min)]
    r = (t_max / t_min) ** (1.0 / (n - 1))
    return [float(t_min * r ** k) for k in range(n)]


class Engine:
    """One GPU context over one or more systems (``pyro_ctx``)."""

    def __init__(self, systems: Sequence[System], seed: int = 12345, device: int = 0,
                 renorm_every: int = 0):
        self.lib = load_library()
        self.systems = list(systems)
        self._temps = [np.ascontiguousarray(s.temperatures, dtype=np.float64) for s in systems]
        descs = (SystemDesc * len(systems))()
        for k, s in enumerate(systems):
            descs[k].L = s.L
            descs[k].n_replicas = s.replicas()
            descs[k].replica_offset = s.replica_offset
            descs[k].n_temperatures = len(s.temperatures)
            descs[k].temperatures = _ptr(self._temps[k], C.c_double)
            descs[k].J1, descs[k].J2, descs[k].J3, descs[k].J3b = s.J1, s.J2, s.J3, s.J3b
        cfg = Config(len(systems), descs, seed, device, renorm_every)
        h = C.c_void_p()
        rc = self.lib.pyro_create(C.byref(cfg), C.byref(h))
        if rc != PYRO_OK:
            raise PyroError(rc, "pyro_create failed (see stderr)")
        self.ctx = h
        self.seed = seed

    # -- plumbing ---------------------------------------------------------
    def _ck(self, rc: int) -> int:
        if rc < 0:
            raise PyroError(rc, self.lib.pyro_last_error(self.ctx).decode())
        return rc

    def close(self) -> None:
        if getattr(self, "ctx", None):
            self.lib.pyro_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    OPT_J1_KERNEL = 1
    OPT_CYCLE_KERNEL = 2
    OPT_CLUSTER_SIZE = 3
    OPT_J1_SITE_MODE = 4
    OPT_SMEM_KERNEL = 5
    OPT_REPLICA_GROUP = 6
    OPT_CHAINS = 7
    OPT_GROUP_MB = 8
    OPT_FAR_KERNEL = 9
    OPT_PDL = 10
    OPT_TET_GROUPED = 11
    OPT_FUSED_OBS = 12
    OPT_WAVE_STALL = 13
    OPT_MEASURE_SNAPSHOT = 14
    OPT_J1_FIXED_L = 15
    OPT_CHAIN_STAGGER = 16

    def set_option(self, option: int, value: int) -> None:
        self._ck(self.lib.pyro_set_option(self.ctx, option, value))

    def get_option(self, option: int) -> int:
        v = C.c_int()
        self._ck(self.lib.pyro_get_option(self.ctx, option, C.byref(v)))
        return v.value

    def autotune(self, n_metro: int = 1, n_or: int = 4, cycles: int = 3) -> int:
        """Times the kernel variants on real cycles and keeps the fastest."""
        v = C.c_int()
        self._ck(self.lib.pyro_autotune(self.ctx, n_metro, n_or, cycles, C.byref(v)))
        return v.value

    def set_stream(self, stream_handle: int) -> None:
        self._ck(self.lib.pyro_set_stream(self.ctx, C.c_void_p(stream_handle)))

    def stream_handle(self) -> int:
        """The cudaStream_t the context queues its work on (as an integer)."""
        return int(self.lib.pyro_get_stream(self.ctx) or 0)

    def synchronize(self) -> None:
        self._ck(self.lib.pyro_synchronize(self.ctx))

    def set_system_keys(self, system: int, key_base: int, swap_key: int) -> None:
        """Philox keys of a system (pyro_set_system_keys)."""
        self._ck(self.lib.pyro_set_system_keys(self.ctx, system, key_base, swap_key))

    def snapshot(self) -> None:
        """Queues a measurement snapshot (pyro_snapshot)."""
        self._ck(self.lib.pyro_snapshot(self.ctx))

    def info(self, system: int = 0) -> dict:
        L, n, r, c = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        self._ck(self.lib.pyro_system_info(self.ctx, system, C.byref(L), C.byref(n), C.byref(r),
                                           C.byref(c)))
        return {"L": L.value, "n_sites": n.value, "n_replicas": r.value, "n_colours": c.value}

    # -- spins ------------------------------------------------------------
    def init_random(self) -> None:
        self._ck(self.lib.pyro_init_random(self.ctx))

    def spin_shape(self, system: int = 0) -> tuple:
        s = self.systems[system]
        return (s.replicas(), 16, s.L ** 3, 4)

    def get_spins(self, system: int = 0) -> np.ndarray:
        out = np.empty(self.spin_shape(system), dtype=np.float32)
        self._ck(self.lib.pyro_get_spins(self.ctx, system, _ptr(out, C.c_float)))
        return out

    def set_spins(self, spins: np.ndarray, system: int = 0) -> None:
        a = np.ascontiguousarray(spins, dtype=np.float32)
        if a.size != int(np.prod(self.spin_shape(system))):
            raise ValueError(f"expected {self.spin_shape(system)} spins, got {a.shape}")
        self._ck(self.lib.pyro_set_spins(self.ctx, system, _ptr(a, C.c_float)))

    def get_spins_planar(self, system: int = 0) -> np.ndarray:
        """Spins in the reference's layout: [replica][x, y, z][16 L^3], FP64."""
        R, n = self.spin_shape(system)[0], int(np.prod(self.spin_shape(system)[1:-1]))
        out = np.empty((R, 3, n), dtype=np.float64)
        self._ck(self.lib.pyro_get_spins_planar(self.ctx, system, _ptr(out, C.c_double)))
        return out

    def set_spins_planar(self, planes: np.ndarray, system: int = 0) -> None:
        R, n = self.spin_shape(system)[0], int(np.prod(self.spin_shape(system)[1:-1]))
        a = np.ascontiguousarray(planes, dtype=np.float64)
        if a.size != R * 3 * n:
            raise ValueError(f"expected {(R, 3, n)} values, got {a.shape}")
        self._ck(self.lib.pyro_set_spins_planar(self.ctx, system, _ptr(a, C.c_double)))

    def set_spins_device(self, ptr: int, system: int = 0) -> None:
        self._ck(self.lib.pyro_set_spins_device(self.ctx, system, C.c_void_p(ptr)))

    def get_spins_device(self, ptr: int, system: int = 0) -> None:
        self._ck(self.lib.pyro_get_spins_device(self.ctx, system, C.c_void_p(ptr)))

    def check_spins(self, tol: float = 1e-3) -> int:
        bad = C.c_longlong(-1)
        rc = self.lib.pyro_check_spins(self.ctx, tol, C.byref(bad))
        if rc == -4:
            return bad.value
        self._ck(rc)
        return -1

    # -- sweeps -----------------------------------------------------------
    def metropolis_sweep(self, n: int = 1) -> None:
        self._ck(self.lib.pyro_metropolis_sweep(self.ctx, n))

    def overrelax_sweep(self, n: int = 1) -> None:
        self._ck(self.lib.pyro_overrelax_sweep(self.ctx, n))

    def cycle(self, n_metro: int, n_or: int, do_swap: bool = True, n_cycles: int = 1) -> None:
        self._ck(self.lib.pyro_cycle(self.ctx, n_metro, n_or, int(bool(do_swap)), n_cycles))

    def launch_count(self) -> int:
        v = C.c_uint64()
        self._ck(self.lib.pyro_get_launch_count(self.ctx, C.byref(v)))
        return v.value

    def sweep_count(self) -> int:
        v = C.c_uint64()
        self._ck(self.lib.pyro_get_sweep_count(self.ctx, C.byref(v)))
        return v.value

    # -- anisotropic exchange ----------------------------------------------
    def set_exchange(self, exchange, field=None, system: int = 0) -> None:
        """Bond matrices (4, 4, 3, 3) and site fields (4, 3) of a system;
        exchange=None returns it to isotropic J1."""
        if exchange is None:
            self._ck(self.lib.pyro_set_exchange(self.ctx, system, None, None))
            return
        a = np.ascontiguousarray(exchange, dtype=np.float64).reshape(144)
        f = None if field is None else np.ascontiguousarray(field, dtype=np.float64).reshape(12)
        self._ck(self.lib.pyro_set_exchange(self.ctx, system, _ptr(a, C.c_double),
                                            None if f is None else _ptr(f, C.c_double)))

    def get_exchange(self, system: int = 0):
        """(matrices, fields) as set, or None for an isotropic system."""
        a = np.empty(144, dtype=np.float64)
        f = np.empty(12, dtype=np.float64)
        is_set = C.c_int()
        self._ck(self.lib.pyro_get_exchange(self.ctx, system, _ptr(a, C.c_double),
                                            _ptr(f, C.c_double), C.byref(is_set)))
        return (a.reshape(4, 4, 3, 3), f.reshape(4, 3)) if is_set.value else None

    def sublattice_magnetisation(self, system: int = 0) -> np.ndarray:
        """(replicas, 4, 3) FP64 magnetisation of each sublattice, replica order."""
        out = np.empty(self.systems[system].replicas() * 12, dtype=np.float64)
        self._ck(self.lib.pyro_sublattice_magnetisation(self.ctx, system, _ptr(out, C.c_double)))
        return out.reshape(-1, 4, 3)

    def order_parameters(self, system: int = 0) -> np.ndarray:
        """(replicas, 20) FP64 order parameters, replica order: 12 irrep
        components, 6 quadrupole sums, monopole density, |Sz| sum."""
        out = np.empty(self.systems[system].replicas() * 20, dtype=np.float64)
        self._ck(self.lib.pyro_order_parameters(self.ctx, system, _ptr(out, C.c_double)))
        return out.reshape(-1, 20)

    def ising_configuration(self, replica: int, system: int = 0) -> np.ndarray:
        """(L^3,) int32 masks: bit 4 t + b set where a_b . S < 0."""
        out = np.empty(self.systems[system].L ** 3, dtype=np.int32)
        self._ck(self.lib.pyro_ising_configuration(self.ctx, system, replica,
                                                   _ptr(out, C.c_int)))
        return out

    # -- cone -------------------------------------------------------------
    def set_cone(self, cosmax, system: int = 0) -> None:
        a = np.ascontiguousarray(cosmax, dtype=np.float32)
        self._ck(self.lib.pyro_set_cone(self.ctx, system, _ptr(a, C.c_float)))

    def get_cone(self, system: int = 0) -> np.ndarray:
        out = np.empty(len(self.systems[system].temperatures), dtype=np.float32)
        self._ck(self.lib.pyro_get_cone(self.ctx, system, _ptr(out, C.c_float)))
        return out

    def acceptance(self, system: int = 0) -> tuple[np.ndarray, np.ndarray]:
        n = len(self.systems[system].temperatures)
        acc = np.zeros(n, dtype=np.uint64)
        prop = np.zeros(n, dtype=np.uint64)
        self._ck(self.lib.pyro_get_acceptance(self.ctx, system, _ptr(acc, C.c_uint64),
                                              _ptr(prop, C.c_uint64)))
        return acc, prop

    def reset_acceptance(self) -> None:
        self._ck(self.lib.pyro_reset_acceptance(self.ctx))

    def tune_cone(self, target: float = 0.5, iterations: int = 20, sweeps: int = 10,
                  n_or: int = 0) -> None:
        self._ck(self.lib.pyro_tune_cone(self.ctx, target, iterations, sweeps, n_or))

    # -- observables and exchange ----------------------------------------
    def observables(self, system: int = 0) -> tuple[np.ndarray, np.ndarray]:
        r = self.systems[system].replicas()
        e = np.empty(r, dtype=np.float64)
        m = np.empty((r, 3), dtype=np.float64)
        self._ck(self.lib.pyro_observables(self.ctx, system, _ptr(e, C.c_double),
                                           _ptr(m, C.c_double)))
        return e, m

    def last_observables(self, system: int = 0) -> tuple[np.ndarray, np.ndarray]:
        """FP64 energies and magnetisations the last cycle computed (no recompute)."""
        n = self.systems[system].replicas()
        e = np.empty(n, dtype=np.float64)
        m = np.empty((n, 3), dtype=np.float64)
        self._ck(self.lib.pyro_last_observables(self.ctx, system, _ptr(e, C.c_double),
                                                _ptr(m, C.c_double)))
        return e, m

    def set_cone_async(self, pinned_cosmax, system: int = 0) -> None:
        """Queue the cone widths from pinned host memory (a float32 array of
        the system's temperatures, e.g. a pinned torch tensor's numpy view);
        it must stay unchanged until synchronize() returns."""
        a = pinned_cosmax
        if a.dtype != np.float32 or not a.flags["C_CONTIGUOUS"]:
            raise ValueError("set_cone_async: a contiguous float32 array is needed")
        self._ck(self.lib.pyro_set_cone_async(self.ctx, system, a.ctypes.data))

    def last_observables_async(self, pinned_energy, pinned_mag=None, system: int = 0) -> None:
        """Queue the copy of the last cycle's energies (and magnetisations) to
        pinned host arrays (float64, n and (n, 3)); read them after
        synchronize()."""
        for a in (pinned_energy, pinned_mag):
            if a is not None and (a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]):
                raise ValueError("last_observables_async: contiguous float64 arrays are needed")
        self._ck(self.lib.pyro_last_observables_async(
            self.ctx, system, pinned_energy.ctypes.data,
            None if pinned_mag is None else pinned_mag.ctypes.data))

    def last_observables_device(self, e_ptr: int, m_ptr: int = 0, system: int = 0) -> None:
        """Energies (and magnetisations) of the last cycle, without recomputing."""
        self._ck(self.lib.pyro_last_observables_device(self.ctx, system, e_ptr or None,
                                                       m_ptr or None))

    def observables_device(self, e_ptr: int, m_ptr: int = 0, system: int = 0) -> None:
        self._ck(self.lib.pyro_observables_device(self.ctx, system, C.c_void_p(e_ptr),
                                                  C.c_void_p(m_ptr or None)))

    def temperatures_of_replicas(self, system: int = 0) -> np.ndarray:
        out = np.empty(len(self.systems[system].temperatures), dtype=np.float64)
        self._ck(self.lib.pyro_get_temperatures(self.ctx, system, _ptr(out, C.c_double)))
        return out

    def permutation(self, system: int = 0) -> np.ndarray:
        out = np.empty(len(self.systems[system].temperatures), dtype=np.int32)
        self._ck(self.lib.pyro_get_permutation(self.ctx, system, _ptr(out, C.c_int)))
        return out

    def pt_swap(self, parity: int = -1) -> int:
        n = C.c_int()
        self._ck(self.lib.pyro_pt_swap(self.ctx, parity, C.byref(n)))
        return n.value

    def pt_swap_global(self, e_all_ptr: int, parity: int = -1, system: int = 0) -> None:
        self._ck(self.lib.pyro_pt_swap_global(self.ctx, system, C.c_void_p(e_all_ptr), parity))

    def swap_stats(self, system: int = 0) -> tuple[np.ndarray, np.ndarray]:
        n = len(self.systems[system].temperatures)
        a = np.zeros(n, dtype=np.uint64)
        t = np.zeros(n, dtype=np.uint64)
        self._ck(self.lib.pyro_get_swap_stats(self.ctx, system, _ptr(a, C.c_uint64),
                                              _ptr(t, C.c_uint64)))
        return a, t

    def enable_history(self, capacity: int) -> None:
        self._ck(self.lib.pyro_enable_history(self.ctx, capacity))
        self._history_cap = capacity

    def history(self, system: int = 0) -> np.ndarray:
        """Energy of every temperature slot per recorded cycle, oldest first."""
        nT = len(self.systems[system].temperatures)
        cap = getattr(self, "_history_cap", 0)
        if cap <= 0:
            raise PyroError(-6, "history not enabled")
        out = np.empty((cap, nT), dtype=np.float64)
        n = C.c_int()
        self._ck(self.lib.pyro_get_history(self.ctx, system, _ptr(out, C.c_double), C.byref(n)))
        return out[: n.value].copy()

    def structure_factor(self, G: int, stride: int = 1, replica: int = -1,
                         system: int = 0) -> np.ndarray:
        out = np.empty((G, G, G), dtype=np.float64)
        self._ck(self.lib.pyro_structure_factor(self.ctx, system, replica, G, stride,
                                                _ptr(out, C.c_double)))
        return out

    # -- checkpoint / configuration files ---------------------------------
    def save_checkpoint(self, path: str) -> None:
        self._ck(self.lib.pyro_save_checkpoint(self.ctx, os.fsencode(path)))

    def load_checkpoint(self, path: str) -> None:
        self._ck(self.lib.pyro_load_checkpoint(self.ctx, os.fsencode(path)))

    def save_configurations(self, prefix: str, append: bool = False, system: int = 0) -> None:
        self._ck(self.lib.pyro_save_configurations(self.ctx, system, os.fsencode(prefix),
                                                   int(append)))

    def read_configurations(self, prefix: str, repetition: int = 0, system: int = 0) -> None:
        self._ck(self.lib.pyro_read_configurations(self.ctx, system, os.fsencode(prefix),
                                                   repetition))

    # -- learned tetrahedron proposal -------------------------------------
    N_MLP_PARAMS = 6288

    def tet_init(self, seed: int = 1, sample_capacity: int = 0) -> None:
        self._ck(self.lib.pyro_tet_init(self.ctx, seed, sample_capacity))

    def tet_weights(self) -> np.ndarray:
        w = np.empty(self.N_MLP_PARAMS, dtype=np.float32)
        self._ck(self.lib.pyro_tet_get_weights(self.ctx, _ptr(w, C.c_float), w.size))
        return w

    def tet_set_weights(self, w) -> None:
        a = np.ascontiguousarray(w, dtype=np.float32)
        self._ck(self.lib.pyro_tet_set_weights(self.ctx, _ptr(a, C.c_float), a.size))

    def tet_set_kernel(self, cluster: int) -> None:
        self._ck(self.lib.pyro_tet_set_kernel(self.ctx, cluster))

    def tet_set_proposal(self, kind: int) -> None:
        """1 (default): site 3 of each tetrahedron from its exact conditional
        given the proposed sites 0-2; 0: all four from the network's vMFs."""
        self._ck(self.lib.pyro_tet_set_proposal(self.ctx, kind))

    def tet_sweep(self, n: int = 1) -> None:
        self._ck(self.lib.pyro_tet_sweep(self.ctx, n))

    TET_TRACE_FLOATS = 56

    def tet_trace_pass(self, corner: int, form: int = 0, system: int = 0) -> np.ndarray:
        """One learned pass over corner `corner` with per-tetrahedron records
        [n_rep][L^3][56] (see pyro_tet_trace_pass)."""
        s = self.systems[system]
        out = np.empty((s.replicas(), s.L ** 3, self.TET_TRACE_FLOATS), dtype=np.float32)
        self._ck(self.lib.pyro_tet_trace_pass(self.ctx, system, corner, form,
                                              _ptr(out, C.c_float)))
        return out

    def tet_acceptance(self, system: int = 0):
        n = len(self.systems[system].temperatures)
        a = np.zeros(n, dtype=np.uint64)
        p = np.zeros(n, dtype=np.uint64)
        self._ck(self.lib.pyro_tet_acceptance(self.ctx, system, _ptr(a, C.c_uint64),
                                              _ptr(p, C.c_uint64)))
        return a, p

    def tet_reset_acceptance(self) -> None:
        self._ck(self.lib.pyro_tet_reset_acceptance(self.ctx))

    def tet_collect(self, stride: int = 1, system: int = 0) -> int:
        n = C.c_longlong()
        self._ck(self.lib.pyro_tet_collect(self.ctx, system, stride, C.byref(n)))
        return n.value

    def tet_samples(self, max_n: int):
        f = np.empty((max_n, 16), dtype=np.float32)
        t = np.empty((max_n, 12), dtype=np.float32)
        n = C.c_longlong()
        self._ck(self.lib.pyro_tet_samples(self.ctx, _ptr(f, C.c_float), _ptr(t, C.c_float), max_n,
                                           C.byref(n)))
        return f[: n.value], t[: n.value]

    def tet_train(self, steps: int, batch: int = 4096, lr: float = 1e-3) -> float:
        loss = C.c_double()
        self._ck(self.lib.pyro_tet_train(self.ctx, steps, batch, lr, C.byref(loss)))
        return loss.value

    def tet_forward(self, feats) -> np.ndarray:
        x = np.ascontiguousarray(feats, dtype=np.float32)
        out = np.empty((x.shape[0], 16), dtype=np.float32)
        self._ck(self.lib.pyro_tet_forward(self.ctx, _ptr(x, C.c_float), x.shape[0],
                                           _ptr(out, C.c_float)))
        return out

    def tet_set_forward(self, tensor_memory: int) -> None:
        """Batched forward kernel: 1 tcgen05 (default), 0 mma.sync."""
        self._ck(self.lib.pyro_tet_set_forward(self.ctx, tensor_memory))

    def tet_forward_device(self, feats_ptr: int, n: int, out_ptr: int) -> None:
        self._ck(self.lib.pyro_tet_forward_device(self.ctx, feats_ptr, n, out_ptr))

    def tet_gradient(self, feats, targets):
        x = np.ascontiguousarray(feats, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        g = np.empty(self.N_MLP_PARAMS, dtype=np.float32)
        loss = C.c_double()
        self._ck(self.lib.pyro_tet_gradient(self.ctx, _ptr(x, C.c_float), _ptr(t, C.c_float),
                                            x.shape[0], _ptr(g, C.c_float), C.byref(loss)))
        return g, loss.value

    def cycle_tet(self, n_metro: int, n_or: int, n_tet: int, do_swap: bool = True,
                  n_cycles: int = 1) -> None:
        self._ck(self.lib.pyro_cycle_tet(self.ctx, n_metro, n_or, n_tet, int(bool(do_swap)),
                                         n_cycles))
