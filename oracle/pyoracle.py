"""ctypes access to the oracle (the CPU checker) — test infrastructure only.

Two libraries:
  oracle/liboracle_fv.so        the restatement in oracle/fv_oracle.c (built by `make -C oracle`)
  oracle/_ref/libdrnum_ref.so   the reference's own sources (built by oracle/build_ref.sh),
                                present only where the reference sources were available

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker; the drnum_b200 package never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_int, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle_fv.so")
REF_LIB = os.path.join(HERE, "_ref", "libdrnum_ref.so")

_P = POINTER(c_double)


def build_oracle() -> str:
    src = os.path.join(HERE, "fv_oracle.c")
    if not os.path.exists(ORACLE_LIB) or os.path.getmtime(src) > os.path.getmtime(ORACLE_LIB):
        subprocess.run(["make", "-s", "-C", HERE, "liboracle_fv.so"], check=True)
    return ORACLE_LIB


_orc = None
_ref = None


def oracle_lib():
    global _orc
    if _orc is None:
        lib = ctypes.CDLL(build_oracle())
        lib.dno_run.restype = c_int
        lib.dno_run.argtypes = [c_int, c_int, c_int, POINTER(c_int), c_double, c_double, c_double,
                                _P, c_void_p, c_int, c_double, _P, c_int]
        lib.dno_residual.restype = c_int
        lib.dno_residual.argtypes = [c_int, c_int, c_int, POINTER(c_int), c_double, c_double, c_double, _P, _P]
        _orc = lib
    return _orc


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("compiled reference not found: run oracle/build_ref.sh")
        lib = ctypes.CDLL(REF_LIB)
        lib.dnref_run.restype = c_int
        lib.dnref_run.argtypes = [c_int, c_int, c_int, POINTER(c_int), c_double, c_double, c_double,
                                  _P, c_void_p, c_int, c_double, _P, c_int, c_int, _P, _P]
        lib.dnref_real_size.restype = c_int
        _ref = lib
    return _ref


def _per(periodic):
    return (c_int * 3)(*(1 if p else 0 for p in periodic))


def oracle_run(U0, h, dt, steps, alpha=(0.25, 0.5, 1.0), periodic=(True, True, True), active=None):
    """Runs the C restatement; returns the state after `steps` RK steps."""
    U = np.ascontiguousarray(U0, dtype=np.float64).copy()
    _, ni, nj, nk = U.shape
    hx, hy, hz = (h, h, h) if np.isscalar(h) else h
    al = np.ascontiguousarray(alpha, dtype=np.float64)
    act = None
    if active is not None:
        act = np.ascontiguousarray(active, dtype=np.uint8)
    rc = oracle_lib().dno_run(ni, nj, nk, _per(periodic), hx, hy, hz, U.ctypes.data_as(_P),
                              act.ctypes.data if act is not None else None,
                              int(steps), float(dt), al.ctypes.data_as(_P), len(al))
    if rc != 0:
        raise RuntimeError(f"oracle failed: {rc}")
    return U


def oracle_residual(U0, h, periodic=(True, True, True)):
    U = np.ascontiguousarray(U0, dtype=np.float64)
    _, ni, nj, nk = U.shape
    hx, hy, hz = (h, h, h) if np.isscalar(h) else h
    res = np.empty_like(U)
    rc = oracle_lib().dno_residual(ni, nj, nk, _per(periodic), hx, hy, hz, U.ctypes.data_as(_P), res.ctypes.data_as(_P))
    if rc != 0:
        raise RuntimeError(f"oracle failed: {rc}")
    return res


def ref_run(U0, h, dt, steps, alpha=(0.25, 0.5, 1.0), periodic=(True, True, True), active=None, threads=1):
    """Runs the compiled reference; returns (state, seconds of the RK loop)."""
    U = np.ascontiguousarray(U0, dtype=np.float64)
    _, ni, nj, nk = U.shape
    hx, hy, hz = (h, h, h) if np.isscalar(h) else h
    out = np.empty_like(U)
    al = np.ascontiguousarray(alpha, dtype=np.float64)
    sec = c_double()
    act = None
    if active is not None:
        act = np.ascontiguousarray(active, dtype=np.uint8)
    rc = ref_lib().dnref_run(ni, nj, nk, _per(periodic), hx, hy, hz, U.ctypes.data_as(_P),
                             act.ctypes.data if act is not None else None, int(steps), float(dt),
                             al.ctypes.data_as(_P), len(al), int(threads), out.ctypes.data_as(_P),
                             ctypes.byref(sec))
    if rc != 0:
        raise RuntimeError(f"reference run failed: {rc}")
    return out, sec.value


class RefSession:
    """A persistent reference run (compiled reference library) for timing."""

    def __init__(self, U0, h, alpha=(0.25, 0.5, 1.0), periodic=(True, True, True), threads=0):
        lib = ref_lib()
        lib.dnref_session_create.restype = c_void_p
        lib.dnref_session_create.argtypes = [c_int, c_int, c_int, POINTER(c_int), c_double, c_double, c_double,
                                             _P, _P, c_int, c_int]
        lib.dnref_session_step.restype = c_double
        lib.dnref_session_step.argtypes = [c_void_p, c_int, c_double]
        lib.dnref_session_destroy.restype = None
        lib.dnref_session_destroy.argtypes = [c_void_p]
        lib.dnref_max_threads.restype = c_int
        self.lib = lib
        U = np.ascontiguousarray(U0, dtype=np.float64)
        _, ni, nj, nk = U.shape
        hx, hy, hz = (h, h, h) if np.isscalar(h) else h
        al = np.ascontiguousarray(alpha, dtype=np.float64)
        self.s = lib.dnref_session_create(ni, nj, nk, _per(periodic), hx, hy, hz, U.ctypes.data_as(_P),
                                          al.ctypes.data_as(_P), len(al), int(threads))
        if not self.s:
            raise RuntimeError("reference session creation failed")
        self.threads = lib.dnref_max_threads()

    def step(self, steps, dt):
        return self.lib.dnref_session_step(self.s, int(steps), float(dt))

    def close(self):
        if self.s:
            self.lib.dnref_session_destroy(self.s)
            self.s = None

    def __del__(self):
        self.close()
