"""ORACLE - test infrastructure.  Python binding of the CPU restatement
(oracle/librw_oracle.so, built by ``make -C oracle``).  Used only by tests/,
__graft_entry__.smoke() and bench.py's CPU baseline, as the checker."""
from __future__ import annotations

import ctypes as ct
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from retainwall_code_b200 import _abi  # noqa: E402

STAGES = {"begin_step": 0, "neighbor_search_p": 1, "neighbor_search_c": 2, "rigid_body_update": 3, "adami": 4,
          "find_corner": 5, "shepard": 6, "interaction": 7, "predictor": 8, "corrector": 9, "end_step": 10}

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "librw_oracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle`")
        L = ct.CDLL(path)
        L.orc_create.restype = ct.c_void_p
        L.orc_create.argtypes = [ct.POINTER(_abi.Case), ct.c_int, ct.c_int]
        L.orc_destroy.argtypes = [ct.c_void_p]
        L.orc_stage.argtypes = [ct.c_void_p, ct.c_int]
        L.orc_step.argtypes = [ct.c_void_p, ct.c_int]
        L.orc_get_array.argtypes = [ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_size_t]
        L.orc_set_array.argtypes = [ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_size_t]
        L.orc_set_counters.argtypes = [ct.c_void_p, ct.c_double, ct.c_int, ct.c_int, ct.c_int]
        L.orc_set_option.argtypes = [ct.c_void_p, ct.c_int, ct.c_double]
        L.orc_get_info.argtypes = [ct.c_void_p, ct.POINTER(_abi.Info)]
        L.orc_wall_force.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p, ct.POINTER(ct.c_double)]
        dp = ct.POINTER(ct.c_double)
        L.orc_hypo_cs.argtypes = [ct.c_int, ct.c_double, ct.c_double, dp, dp, dp, dp, dp]
        L.orc_hypo_basic.argtypes = [ct.c_int, ct.c_double, dp, dp, dp, dp]
        L.orc_dp.argtypes = [ct.c_int, ct.c_int, ct.c_double, dp, dp, dp, dp, ct.POINTER(ct.c_int)]
        L.orc_kernel_w.restype = ct.c_double
        L.orc_kernel_w.argtypes = [ct.c_int, ct.c_double, ct.c_double]
        L.orc_kernel_f.restype = ct.c_double
        L.orc_kernel_f.argtypes = [ct.c_int, ct.c_double, ct.c_double]
        _lib = L
    return _lib


class Oracle:
    """CPU restatement of one case; same array names/layouts as the product's C ABI."""

    def __init__(self, case, precision: int = 4, threads: int = 0):
        keep: list = []
        c = _abi.case_struct(case, keep)
        self._h = lib().orc_create(ct.byref(c), precision, threads)
        self.precision = precision

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stage(self, name: str) -> None:
        assert lib().orc_stage(self._h, STAGES[name]) == 0

    def step(self, n: int = 1) -> None:
        assert lib().orc_step(self._h, n) == 0

    def info(self) -> _abi.Info:
        inf = _abi.Info()
        lib().orc_get_info(self._h, ct.byref(inf))
        return inf

    def get(self, name: str) -> np.ndarray:
        rows, cols, dt = _abi.array_spec(name, self.info())
        a = np.zeros((rows, cols), dt) if cols > 1 else np.zeros(rows, dt)
        rc = lib().orc_get_array(self._h, _abi.ARRAYS[name], a.ctypes.data, a.nbytes)
        assert rc == 0, (name, rc)
        return a

    def set(self, name: str, a: np.ndarray) -> None:
        rows, cols, dt = _abi.array_spec(name, self.info())
        a = np.ascontiguousarray(a, dtype=dt)
        rc = lib().orc_set_array(self._h, _abi.ARRAYS[name], a.ctypes.data, a.nbytes)
        assert rc == 0, (name, rc)

    def set_counters(self, time: float, step: int, npm: int, np_delete_m: int) -> None:
        lib().orc_set_counters(self._h, time, step, npm, np_delete_m)

    def set_option(self, opt: int, value: float) -> None:
        assert lib().orc_set_option(self._h, opt, value) == 0

    def wall_force(self, mode: int = 0, wall_id: int = 10, strip=None) -> np.ndarray:
        out = (ct.c_double * 3)()
        sp = None
        if strip is not None:
            sa = (ct.c_double * 3)(*strip)
            sp = ct.cast(sa, ct.c_void_p)
        lib().orc_wall_force(self._h, mode, wall_id, sp, out)
        return np.array(out[:])


def hypo_cs(precision, dt, density, omega4, rate6, sigma6, par15):
    f = lambda a: np.ascontiguousarray(a, np.float64)
    om, rt, sg, pr = f(omega4), f(rate6), f(sigma6).copy(), f(par15)
    m = ct.c_double(0)
    P = lambda a: a.ctypes.data_as(ct.POINTER(ct.c_double))
    lib().orc_hypo_cs(precision, dt, density, P(om), P(rt), P(sg), P(pr), ct.byref(m))
    return sg, m.value


def hypo_basic(precision, dt, omega4, rate6, sigma6, par15):
    f = lambda a: np.ascontiguousarray(a, np.float64)
    om, rt, sg, pr = f(omega4), f(rate6), f(sigma6).copy(), f(par15)
    P = lambda a: a.ctypes.data_as(ct.POINTER(ct.c_double))
    lib().orc_hypo_basic(precision, dt, P(om), P(rt), P(sg), P(pr))
    return sg


def dp(precision, dt, omega4, rate6, sigma6, par15, mui=False):
    """Drucker-Prager (mui=False; returns (stress, yield flag)) or mu(I)-DP (mui=True;
    returns (stress, 0)) stress update."""
    f = lambda a: np.ascontiguousarray(a, np.float64)
    om, rt, sg, pr = f(omega4), f(rate6), f(sigma6).copy(), f(par15)
    y = ct.c_int(0)
    P = lambda a: a.ctypes.data_as(ct.POINTER(ct.c_double))
    lib().orc_dp(precision, 1 if mui else 0, dt, P(om), P(rt), P(sg), P(pr), ct.byref(y))
    return sg, y.value
