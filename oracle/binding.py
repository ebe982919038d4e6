"""ctypes binding of oracle/liboracle.so (test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    src = os.path.join(HERE, "oracle.cpp")
    if not os.path.exists(LIB) or (os.path.exists(src) and
                                   os.path.getmtime(src) > os.path.getmtime(LIB)):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    lib = C.CDLL(LIB)
    P, i, d, f = C.c_void_p, C.c_int, C.c_double, C.c_float
    pi, pd, pf = C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_float)
    pu32, pu64 = C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)
    sig = {
        "orc_create": (P, [i, pi, pi, pi, pi, pd, pd, C.c_uint64, i, i]),
        "orc_destroy": (None, [P]),
        "orc_set_threads": (i, [i]),
        "orc_init_random": (None, [P]),
        "orc_n_spins": (C.c_longlong, [P, i]),
        "orc_set_spins": (None, [P, i, pf]),
        "orc_get_spins": (None, [P, i, pf]),
        "orc_get_spins64": (None, [P, i, pd]),
        "orc_metropolis_sweep": (None, [P, i]),
        "orc_overrelax_sweep": (None, [P, i]),
        "orc_set_cone": (None, [P, i, pf]),
        "orc_set_exchange": (None, [P, i, pd, pd]),
        "orc_order_parameters": (None, [P, i, pd]),
        "orc_ising_configuration": (None, [P, i, i, pi]),
        "orc_get_cone": (None, [P, i, pf]),
        "orc_get_acceptance": (None, [P, i, pu64, pu64]),
        "orc_reset_acceptance": (None, [P]),
        "orc_tune_cone": (None, [P, d, i, i, i]),
        "orc_observables": (None, [P, i, pd, pd]),
        "orc_pt_swap": (i, [P, i]),
        "orc_pt_swap_global": (i, [P, i, pd, i]),
        "orc_cycle": (None, [P, i, i, i, i, pd]),
        "orc_get_permutation": (None, [P, i, pi]),
        "orc_get_swap_stats": (None, [P, i, pu64, pu64]),
        "orc_sweep_count": (C.c_uint64, [P]),
        "orc_structure_factor": (None, [P, i, i, i, i, pd]),
        "orc_mlp_param_count": (i, []),
        "orc_mlp_set_bf16": (None, [i]),
        "orc_mlp_forward": (None, [pf, pf, i, pd]),
        "orc_mlp_gradient": (None, [pf, pf, pf, i, pd, pd]),
        "orc_tet_features": (None, [P, i, i, i, pf, pf]),
        "orc_set_system_keys": (None, [P, i, i, i]),
        "orc_tet_move_check": (None, [pf, i, pi, pi, i, i, C.c_uint64, C.c_uint64, d, i, pd]),
        "orc_neighbours": (None, [i, pi]),
        "orc_philox": (None, [pu32, pu32, pu32]),
        "orc_expf": (f, [f]),
        "orc_logf": (f, [f]),
        "orc_sincospif": (None, [f, pf, pf]),
        "orc_exp64": (d, [d]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class Oracle:
    """Same systems/seed semantics as cudacode_b200.engine.Engine."""

    def __init__(self, systems: Sequence, seed: int = 12345, renorm_every: int = 0,
                 fp64: bool = False, threads: int = 0):
        self.lib = load()
        if threads:
            self.lib.orc_set_threads(threads)
        self.systems = list(systems)
        n = len(systems)
        L = np.array([s.L for s in systems], dtype=np.int32)
        R = np.array([s.replicas() for s in systems], dtype=np.int32)
        off = np.array([s.replica_offset for s in systems], dtype=np.int32)
        nT = np.array([len(s.temperatures) for s in systems], dtype=np.int32)
        T = np.concatenate([np.asarray(s.temperatures, dtype=np.float64) for s in systems])
        J = np.array([[s.J1, s.J2, s.J3, s.J3b] for s in systems], dtype=np.float64).ravel()
        self.h = self.lib.orc_create(n, _p(L, C.c_int), _p(R, C.c_int), _p(off, C.c_int),
                                     _p(nT, C.c_int), _p(T, C.c_double), _p(J, C.c_double),
                                     seed, renorm_every, int(fp64))
        self.total_temps = int(nT.sum())
        self.temp_base = np.concatenate([[0], np.cumsum(nT)[:-1]]).astype(int)

    def close(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def spin_shape(self, system=0):
        s = self.systems[system]
        return (s.replicas(), 16, s.L ** 3, 4)

    def init_random(self):
        self.lib.orc_init_random(self.h)

    def set_system_keys(self, system, key_base, swap_key):
        self.lib.orc_set_system_keys(self.h, system, key_base, swap_key)

    def get_spins(self, system=0):
        out = np.empty(self.spin_shape(system), dtype=np.float32)
        self.lib.orc_get_spins(self.h, system, _p(out, C.c_float))
        return out

    def get_spins64(self, system=0):
        out = np.empty(self.spin_shape(system), dtype=np.float64)
        self.lib.orc_get_spins64(self.h, system, _p(out, C.c_double))
        return out

    def set_spins(self, spins, system=0):
        a = np.ascontiguousarray(spins, dtype=np.float32)
        assert a.size == int(np.prod(self.spin_shape(system)))
        self.lib.orc_set_spins(self.h, system, _p(a, C.c_float))

    def metropolis_sweep(self, n=1):
        self.lib.orc_metropolis_sweep(self.h, n)

    def overrelax_sweep(self, n=1):
        self.lib.orc_overrelax_sweep(self.h, n)

    def set_exchange(self, exchange, field=None, system=0):
        """Bond matrices (4 x 4 x 3 x 3) and site fields (4 x 3) of a system."""
        if exchange is None:
            self.lib.orc_set_exchange(self.h, system, None, None)
            return
        a = np.ascontiguousarray(exchange, dtype=np.float64).reshape(144)
        f = None if field is None else np.ascontiguousarray(field, dtype=np.float64).reshape(12)
        self.lib.orc_set_exchange(self.h, system, _p(a, C.c_double),
                                  None if f is None else _p(f, C.c_double))

    def order_parameters(self, system=0):
        out = np.zeros((self.systems[system].replicas(), 20))
        self.lib.orc_order_parameters(self.h, system, _p(out, C.c_double))
        return out

    def ising_configuration(self, replica, system=0):
        out = np.zeros(self.systems[system].L ** 3, dtype=np.int32)
        self.lib.orc_ising_configuration(self.h, system, replica, _p(out, C.c_int))
        return out

    def set_cone(self, c, system=0):
        a = np.ascontiguousarray(c, dtype=np.float32)
        self.lib.orc_set_cone(self.h, system, _p(a, C.c_float))

    def get_cone(self, system=0):
        out = np.empty(len(self.systems[system].temperatures), dtype=np.float32)
        self.lib.orc_get_cone(self.h, system, _p(out, C.c_float))
        return out

    def acceptance(self, system=0):
        n = len(self.systems[system].temperatures)
        a = np.zeros(n, dtype=np.uint64)
        p = np.zeros(n, dtype=np.uint64)
        self.lib.orc_get_acceptance(self.h, system, _p(a, C.c_uint64), _p(p, C.c_uint64))
        return a, p

    def reset_acceptance(self):
        self.lib.orc_reset_acceptance(self.h)

    def tune_cone(self, target=0.5, iterations=20, sweeps=10, n_or=0):
        self.lib.orc_tune_cone(self.h, target, iterations, sweeps, n_or)

    def observables(self, system=0):
        r = self.systems[system].replicas()
        e = np.empty(r)
        m = np.empty((r, 3))
        self.lib.orc_observables(self.h, system, _p(e, C.c_double), _p(m, C.c_double))
        return e, m

    def pt_swap(self, parity=-1):
        return self.lib.orc_pt_swap(self.h, parity)

    def pt_swap_global(self, e_all, parity=-1, system=0):
        a = np.ascontiguousarray(e_all, dtype=np.float64)
        return self.lib.orc_pt_swap_global(self.h, system, _p(a, C.c_double), parity)

    def cycle(self, n_metro, n_or, do_swap=True, n_cycles=1, record=False):
        hist = np.zeros((n_cycles, self.total_temps)) if record else None
        self.lib.orc_cycle(self.h, n_metro, n_or, int(do_swap), n_cycles,
                           _p(hist, C.c_double) if record else None)
        return hist

    def permutation(self, system=0):
        out = np.empty(len(self.systems[system].temperatures), dtype=np.int32)
        self.lib.orc_get_permutation(self.h, system, _p(out, C.c_int))
        return out

    def swap_stats(self, system=0):
        n = len(self.systems[system].temperatures)
        a = np.zeros(n, dtype=np.uint64)
        t = np.zeros(n, dtype=np.uint64)
        self.lib.orc_get_swap_stats(self.h, system, _p(a, C.c_uint64), _p(t, C.c_uint64))
        return a, t

    def structure_factor(self, G, stride=1, replica=-1, system=0):
        out = np.empty((G, G, G))
        self.lib.orc_structure_factor(self.h, system, replica, G, stride, _p(out, C.c_double))
        return out

    def tet_features(self, replica, corner, system=0):
        L3 = self.systems[system].L ** 3
        f = np.empty((L3, 16), dtype=np.float32)
        s = np.empty((L3, 12), dtype=np.float32)
        self.lib.orc_tet_features(self.h, system, replica, corner, _p(f, C.c_float), _p(s, C.c_float))
        return f, s

    def sweep_count(self):
        return int(self.lib.orc_sweep_count(self.h))


def neighbours(s: int) -> np.ndarray:
    out = np.empty(120, dtype=np.int32)
    load().orc_neighbours(s, _p(out, C.c_int))
    return out.reshape(30, 4)


def philox(ctr, key) -> np.ndarray:
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    out = np.empty(4, dtype=np.uint32)
    load().orc_philox(_p(c, C.c_uint32), _p(k, C.c_uint32), _p(out, C.c_uint32))
    return out


def expf(x: float) -> float:
    return load().orc_expf(x)


def logf(x: float) -> float:
    return load().orc_logf(x)


def sincospif(a: float):
    s, c = C.c_float(), C.c_float()
    load().orc_sincospif(a, C.byref(s), C.byref(c))
    return s.value, c.value


def exp64(x: float) -> float:
    return load().orc_exp64(x)


def mlp_forward(weights, feats):
    w = np.ascontiguousarray(weights, dtype=np.float32)
    x = np.ascontiguousarray(feats, dtype=np.float32)
    out = np.empty((x.shape[0], 16))
    load().orc_mlp_forward(_p(w, C.c_float), _p(x, C.c_float), x.shape[0], _p(out, C.c_double))
    return out


def mlp_gradient(weights, feats, targets):
    w = np.ascontiguousarray(weights, dtype=np.float32)
    x = np.ascontiguousarray(feats, dtype=np.float32)
    t = np.ascontiguousarray(targets, dtype=np.float32)
    g = np.empty(load().orc_mlp_param_count())
    loss = C.c_double()
    load().orc_mlp_gradient(_p(w, C.c_float), _p(x, C.c_float), _p(t, C.c_float), x.shape[0],
                            _p(g, C.c_double), C.byref(loss))
    return g, loss.value


def tet_move_check(records, rep_key, cell, corner, L3, seed, sweep, J1, closure):
    """FP64 restatement of the learned move for trace records (n, 56): per
    record log r, test uniform, decision, log q ratio, dE and the FP64 vMF
    draws (12) from the move's Philox words; array (n, 17)."""
    rec = np.ascontiguousarray(records, dtype=np.float32).reshape(-1, 56)
    n = rec.shape[0]
    rk = np.ascontiguousarray(rep_key, dtype=np.int32).reshape(n)
    ce = np.ascontiguousarray(cell, dtype=np.int32).reshape(n)
    out = np.empty((n, 17))
    load().orc_tet_move_check(_p(rec, C.c_float), n, _p(rk, C.c_int), _p(ce, C.c_int), corner, L3,
                              seed, sweep, J1, int(closure), _p(out, C.c_double))
    return out
