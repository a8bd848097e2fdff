"""ctypes wrapper of oracle/_ref/libdrnum_refapp.so: a DrNUM application
built from the reference's own PatchGrid / CartesianPatch / RungeKutta
(rungekutta.cpp:27-42) that drives drnum_b200 through the C++ binding
include/drnum_b200_iterator.h (B200_CartesianIterator, B200_LevelSetBC).
Test infrastructure: oracle/build_ref.sh builds the library."""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "..", "oracle", "_ref", "libdrnum_refapp.so")
RK3 = (0.25, 0.5, 1.0)
_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB)
        L.refapp_run_single.restype = c_int
        L.refapp_run_single.argtypes = [c_int, c_int, c_int, c_int, POINTER(c_int), c_double, c_double, c_double,
                                        c_void_p, c_void_p, c_int, c_double, c_void_p, c_int, c_char_p, c_int]
        L.refapp_run_grid.restype = c_int
        L.refapp_run_grid.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                      c_void_p, c_int, c_double, c_void_p, c_int, c_void_p, c_void_p, c_int, c_int,
                                      c_double, c_char_p, c_int]
        _lib = L
    return _lib


class AppError(RuntimeError):
    pass


def run_single(U0, h, dt, steps, periodic=(True, True, True), active=None, scheme=0, alpha=RK3):
    """One patch advanced `steps` RK steps by the reference's RungeKutta over
    B200_CartesianIterator; returns field 0."""
    U = np.ascontiguousarray(U0, dtype=np.float64).copy()
    _, ni, nj, nk = U.shape
    hx, hy, hz = (h, h, h) if np.isscalar(h) else h
    per = (c_int * 3)(*(1 if p else 0 for p in periodic))
    act = None if active is None else np.ascontiguousarray(active, dtype=np.uint8)
    al = np.ascontiguousarray(alpha, dtype=np.float64)
    err = ctypes.create_string_buffer(512)
    rc = lib().refapp_run_single(int(scheme), ni, nj, nk, per, hx, hy, hz, U.ctypes.data,
                                 None if act is None else act.ctypes.data, int(steps), float(dt), al.ctypes.data,
                                 len(al), err, 512)
    if rc != 0:
        raise AppError(f"application run failed ({rc}): {err.value.decode()}")
    return U


def run_grid(patches, states, dt, steps, bcs=None, inactive=None, G=None, ls=(3, 0, 0.1), alpha=RK3):
    """A patch grid (layout dicts) built by the reference's PatchGrid, its
    donor tables from PatchGrid::computeDependencies, advanced by RungeKutta
    over B200_CartesianIterator (B200_LevelSetBC as post-operation with G).
    bcs = {patch: {side: (kind, params, table)}}.  Returns the states."""
    np_ = len(patches)
    n = np.ascontiguousarray([p["n"] for p in patches], dtype=np.int32)
    o = np.ascontiguousarray([p["origin"] for p in patches], dtype=np.float64)
    L = np.ascontiguousarray([p["length"] for p in patches], dtype=np.float64)
    sk = np.ascontiguousarray([p["seek"] for p in patches], dtype=np.int32)
    kinds = np.zeros((np_, 6), dtype=np.int32)
    params = np.zeros((np_, 6, 5))
    tables = (c_void_p * (6 * np_))()
    keep = []
    for p, sides in (bcs or {}).items():
        for side, (kind, par, tab) in sides.items():
            kinds[p, side] = int(kind)
            if par is not None:
                params[p, side] = par
            if tab is not None:
                t = np.ascontiguousarray(tab, dtype=np.float64)
                keep.append(t)
                tables[6 * p + side] = t.ctypes.data
    outs = [np.ascontiguousarray(s, dtype=np.float64).copy() for s in states]
    sp = (c_void_p * np_)(*[s.ctypes.data for s in outs])
    ina = None if inactive is None else np.ascontiguousarray(inactive, dtype=np.int32)
    gp = None
    if G is not None:
        gs = [None if g is None else np.ascontiguousarray(g, dtype=np.float64) for g in G]
        keep += [g for g in gs if g is not None]
        gp = (c_void_p * np_)(*[None if g is None else g.ctypes.data for g in gs])
    al = np.ascontiguousarray(alpha, dtype=np.float64)
    err = ctypes.create_string_buffer(512)
    rc = lib().refapp_run_grid(np_, n.ctypes.data, o.ctypes.data, L.ctypes.data, sk.ctypes.data, kinds.ctypes.data,
                               params.ctypes.data, tables, sp, int(steps), float(dt), al.ctypes.data, len(al),
                               None if ina is None else ina.ctypes.data, gp, int(ls[0]), int(ls[1]), float(ls[2]),
                               err, 512)
    if rc != 0:
        raise AppError(f"application run failed ({rc}): {err.value.decode()}")
    return outs
