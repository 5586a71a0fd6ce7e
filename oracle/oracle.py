"""ctypes front end of the CPU oracle (oracle/ccd_oracle.c) — TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.
Parity of this oracle is pinned against dumps of the reference itself (tests/golden/).
"""
import ctypes
import os

import numpy as np

from .build import build_oracle

_lib = None
vp = ctypes.c_void_p
u64 = ctypes.c_uint64
i64 = ctypes.c_int64
dbl = ctypes.c_double
PD = ctypes.POINTER(ctypes.c_double)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libccdoracle.so")
        if not os.path.exists(path):
            build_oracle()
        L = ctypes.CDLL(path)
        L.oracle_create.argtypes = [vp]
        L.oracle_create.restype = vp
        L.oracle_free.argtypes = [vp]
        L.oracle_free.restype = None
        L.oracle_t2_size.argtypes = [vp]
        L.oracle_t2_size.restype = u64
        for f in ("oracle_calc_t2diff_p2_p1hh", "oracle_calc_t2diff_h2pp_h1",
                  "oracle_calc_t2diff_phhp", "oracle_calc_t2diff_pphh",
                  "oracle_map_from_distributed", "oracle_map_to_distributed", "oracle_reset"):
            getattr(L, f).argtypes = [vp]
            getattr(L, f).restype = None
        L.oracle_calc_t2_pphh.argtypes = [vp, dbl]
        L.oracle_calc_t2_pphh.restype = dbl
        L.oracle_step.argtypes = [vp, dbl]
        L.oracle_step.restype = dbl
        L.oracle_set_t2.argtypes = [vp, PD]
        L.oracle_set_t2.restype = None
        L.oracle_get_t2.argtypes = [vp, PD]
        L.oracle_get_t2.restype = None
        L.oracle_solve.argtypes = [vp, dbl, i64, dbl, PD, PD]
        L.oracle_solve.restype = i64
        L.oracle_read_chain.argtypes = [vp, ctypes.c_int, PD]
        L.oracle_read_chain.restype = u64
        L.oracle_fnv1a.argtypes = [vp, u64]
        L.oracle_fnv1a.restype = u64
        _lib = L
    return _lib


def fnv1a(arr):
    a = np.ascontiguousarray(arr)
    return int(lib().oracle_fnv1a(a.ctypes.data_as(vp), a.nbytes))


class Oracle:
    """CPU restatement of the reference CCD loop over a System's problem."""

    def __init__(self, system):
        self.system = system  # keeps the problem's host memory alive
        self._s = lib().oracle_create(ctypes.cast(system.problem, vp))
        if not self._s:
            raise MemoryError("oracle_create failed")
        self.n_t2 = int(lib().oracle_t2_size(self._s))

    def close(self):
        if self._s:
            lib().oracle_free(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self):
        lib().oracle_reset(self._s)

    def step(self, mixing=0.5):
        return float(lib().oracle_step(self._s, mixing))

    def solve(self, tol=1e-8, max_iters=100, mixing=0.5):
        energies = np.zeros(max_iters + 2)
        e = ctypes.c_double()
        n = lib().oracle_solve(self._s, tol, max_iters, mixing,
                               energies.ctypes.data_as(PD), ctypes.byref(e))
        return float(e.value), int(n), energies[:n].copy()

    def t2(self):
        out = np.zeros(self.n_t2)
        lib().oracle_get_t2(self._s, out.ctypes.data_as(PD))
        return out

    def set_t2(self, t2):
        t2 = np.ascontiguousarray(t2, dtype=np.float64)
        assert t2.size == self.n_t2
        lib().oracle_set_t2(self._s, t2.ctypes.data_as(PD))

    def chain(self, chain_id):
        n = lib().oracle_read_chain(self._s, chain_id, None)
        out = np.zeros(n)
        lib().oracle_read_chain(self._s, chain_id, out.ctypes.data_as(PD))
        return out

    # Stage entry points (calc.cpp / Chain.hpp names).
    def calc_t2diff_p2_p1hh(self): lib().oracle_calc_t2diff_p2_p1hh(self._s)
    def calc_t2diff_h2pp_h1(self): lib().oracle_calc_t2diff_h2pp_h1(self._s)
    def calc_t2diff_phhp(self): lib().oracle_calc_t2diff_phhp(self._s)
    def calc_t2diff_pphh(self): lib().oracle_calc_t2diff_pphh(self._s)
    def map_from_distributed(self): lib().oracle_map_from_distributed(self._s)
    def calc_t2_pphh(self, mixing=0.5): return float(lib().oracle_calc_t2_pphh(self._s, mixing))
    def map_to_distributed(self): lib().oracle_map_to_distributed(self._s)
