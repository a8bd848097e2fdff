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
import math
import os
import subprocess
from ctypes import POINTER, c_double, c_int, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle_fv.so")
REF_LIB = os.path.join(HERE, "_ref", "libdrnum_ref.so")
# the reference in its shipped single precision (`real` = float, drnum.h:43)
REF_LIB_F32 = os.path.join(HERE, "_ref", "libdrnum_ref_f32.so")

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
        lib.dnref_run_scheme.restype = c_int
        lib.dnref_run_scheme.argtypes = [c_int] + lib.dnref_run.argtypes
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


def oracle_residual_bc(U0, h, bcs, periodic=(False, False, False)):
    """Residual with patch-face fluxes: bcs = {side: (kind, params, table)}
    for sides 0..5 (x-min, x-max, y-min, y-max, z-min, z-max)."""
    lib = oracle_lib()
    lib.dno_residual_bc.restype = c_int
    lib.dno_residual_bc.argtypes = [c_int, c_int, c_int, POINTER(c_int), c_double, c_double, c_double,
                                    POINTER(c_int), _P, POINTER(_P), _P, _P]
    U = np.ascontiguousarray(U0, dtype=np.float64)
    _, ni, nj, nk = U.shape
    hx, hy, hz = (h, h, h) if np.isscalar(h) else h
    kinds = (c_int * 6)()
    ff = np.zeros(30)
    tabs = (_P * 6)()
    keep = []
    for side, (kind, params, table) in (bcs or {}).items():
        kinds[side] = int(kind)
        if params is not None:
            ff[5 * side:5 * side + 5] = params
        if table is not None:
            t = np.ascontiguousarray(table, dtype=np.float64)
            keep.append(t)
            tabs[side] = t.ctypes.data_as(_P)
    res = np.empty_like(U)
    rc = lib.dno_residual_bc(ni, nj, nk, _per(periodic), hx, hy, hz, kinds, ff.ctypes.data_as(_P), tabs,
                             U.ctypes.data_as(_P), res.ctypes.data_as(_P))
    if rc != 0:
        raise RuntimeError(f"oracle failed: {rc}")
    return res


def oracle_residual(U0, h, periodic=(True, True, True)):
    U = np.ascontiguousarray(U0, dtype=np.float64)
    _, ni, nj, nk = U.shape
    hx, hy, hz = (h, h, h) if np.isscalar(h) else h
    res = np.empty_like(U)
    rc = oracle_lib().dno_residual(ni, nj, nk, _per(periodic), hx, hy, hz, U.ctypes.data_as(_P), res.ctypes.data_as(_P))
    if rc != 0:
        raise RuntimeError(f"oracle failed: {rc}")
    return res


def ref_run(U0, h, dt, steps, alpha=(0.25, 0.5, 1.0), periodic=(True, True, True), active=None, threads=1,
            scheme=0):
    """Runs the compiled reference; returns (state, seconds of the RK loop).
    scheme: the Euler flux, numbered as DN_FLUX_* (0 AusmPlus, 2 VanLeer, 3 Roe)."""
    U = np.ascontiguousarray(U0, dtype=np.float64)
    _, ni, nj, nk = U.shape
    hx, hy, hz = (h, h, h) if np.isscalar(h) else h
    out = np.empty_like(U)
    al = np.ascontiguousarray(alpha, dtype=np.float64)
    sec = c_double()
    act = None
    if active is not None:
        act = np.ascontiguousarray(active, dtype=np.uint8)
    rc = ref_lib().dnref_run_scheme(int(scheme), ni, nj, nk, _per(periodic), hx, hy, hz, U.ctypes.data_as(_P),
                                    act.ctypes.data if act is not None else None, int(steps), float(dt),
                                    al.ctypes.data_as(_P), len(al), int(threads), out.ctypes.data_as(_P),
                                    ctypes.byref(sec))
    if rc != 0:
        raise RuntimeError(f"reference run failed: {rc}")
    return out, sec.value


_ref32 = None


def ref_f32_available() -> bool:
    return os.path.exists(REF_LIB_F32)


class RefSession:
    """A persistent reference run (compiled reference library) for timing.
    precision "f64": the FP64 build (the parity checker); "f32": the
    reference's shipped single-precision build.  The periodic axes carry two
    ghost layers per side: the iterator computes (n+4) cells along each of
    them (`computed_cells`)."""

    def __init__(self, U0, h, alpha=(0.25, 0.5, 1.0), periodic=(True, True, True), threads=0, precision="f64"):
        global _ref32
        if precision == "f32":
            if _ref32 is None:
                if not ref_f32_available():
                    raise RuntimeError("single-precision reference not found: run oracle/build_ref.sh")
                _ref32 = ctypes.CDLL(REF_LIB_F32)
            lib = _ref32
        else:
            lib = ref_lib()
        lib.dnref_real_size.restype = c_int
        self.real_bytes = lib.dnref_real_size()
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
        self.computed_cells = int(np.prod([x + (4 if p else 0) for x, p in zip((ni, nj, nk), periodic)]))

    def step(self, steps, dt):
        return self.lib.dnref_session_step(self.s, int(steps), float(dt))

    def close(self):
        if self.s:
            self.lib.dnref_session_destroy(self.s)
            self.s = None

    def __del__(self):
        self.close()


# ------------------------------------------------------------------ patch grids

def _grid_arrays(patches):
    """patches: list of dicts with n (3), origin (3), length (3), seek (6)."""
    n = np.ascontiguousarray([p["n"] for p in patches], dtype=np.int32).ravel()
    o = np.ascontiguousarray([p["origin"] for p in patches], dtype=np.float64).ravel()
    L = np.ascontiguousarray([p["length"] for p in patches], dtype=np.float64).ravel()
    s = np.ascontiguousarray([p["seek"] for p in patches], dtype=np.int32).ravel()
    return n, o, L, s


class RefGrid:
    """The reference's PatchGrid over axis-aligned Cartesian patches (compiled
    reference library): donor tables from PatchGrid::computeDependencies and
    RK steps with Patch::accessDonorDataDirect after every stage."""

    def __init__(self, patches, add_protect=0, threads=1, num_vars=5, grid_file=None, scale=1.0):
        """patches: layout dicts; or grid_file (a path relative to the
        working directory) read by the reference's PatchGrid::readGrid."""
        lib = ref_lib()
        lib.dnref_grid_read.restype = c_void_p
        lib.dnref_grid_read.argtypes = [ctypes.c_char_p, c_double, c_int, c_int]
        lib.dnref_grid_num_patches.restype = c_int
        lib.dnref_grid_num_patches.argtypes = [c_void_p]
        lib.dnref_grid_patch_info.restype = c_int
        lib.dnref_grid_patch_info.argtypes = [c_void_p, c_int, c_void_p, _P, _P, ctypes.c_char_p, c_int]
        lib.dnref_grid_create_nv.restype = c_void_p
        lib.dnref_grid_create_nv.argtypes = [c_int, POINTER(c_int), _P, _P, POINTER(c_int), c_int, c_int, c_int]
        lib.dnref_grid_levelset.restype = c_int
        lib.dnref_grid_levelset.argtypes = [c_void_p, POINTER(_P), c_int, c_int, c_double]
        lib.dnref_grid_levelset_layer.restype = c_int
        lib.dnref_grid_levelset_layer.argtypes = [c_void_p, c_int, c_int, c_int, c_void_p] + [c_void_p] * 5
        lib.dnref_grid_tables.restype = c_int
        lib.dnref_grid_tables.argtypes = [c_void_p, c_int] + [c_void_p] * 8
        for nm in ("dnref_grid_set_state", "dnref_grid_get_state"):
            getattr(lib, nm).restype = c_int
            getattr(lib, nm).argtypes = [c_void_p, c_int, _P]
        lib.dnref_grid_copy_donor_data.restype = c_int
        lib.dnref_grid_copy_donor_data.argtypes = [c_void_p, c_int]
        lib.dnref_grid_run.restype = c_int
        lib.dnref_grid_run.argtypes = [c_void_p, c_int, c_double, _P, c_int, _P]
        lib.dnref_grid_run_scheme.restype = c_int
        lib.dnref_grid_run_scheme.argtypes = [c_void_p, c_int, c_int, c_double, _P, c_int, _P]
        lib.dnref_grid_destroy.restype = None
        lib.dnref_grid_destroy.argtypes = [c_void_p]
        self.lib = lib
        self.patches = patches
        if grid_file is not None:
            self.h = lib.dnref_grid_read(str(grid_file).encode(), float(scale), int(add_protect), int(threads))
            if not self.h:
                raise RuntimeError("reference grid read failed")
            return
        n, o, L, s = _grid_arrays(patches)
        self.h = lib.dnref_grid_create_nv(len(patches), n.ctypes.data_as(POINTER(c_int)), o.ctypes.data_as(_P),
                                          L.ctypes.data_as(_P), s.ctypes.data_as(POINTER(c_int)),
                                          int(add_protect), int(threads), int(num_vars))
        if not self.h:
            raise RuntimeError("reference grid creation failed")

    def num_patches(self):
        return self.lib.dnref_grid_num_patches(self.h)

    def patch_info(self, p):
        """(cells, reference point, spacing, solver-code string) of patch p."""
        n = np.zeros(3, np.int64)
        o = np.zeros(3)
        d = np.zeros(3)
        buf = ctypes.create_string_buffer(4096)
        if self.lib.dnref_grid_patch_info(self.h, p, n.ctypes.data, o.ctypes.data_as(_P), d.ctypes.data_as(_P),
                                          buf, len(buf)) != 0:
            raise RuntimeError("patch_info failed")
        return n, o, d, buf.value.decode()

    def tables(self, p):
        counts = np.zeros(4, dtype=np.int64)
        rc = self.lib.dnref_grid_tables(self.h, p, counts.ctypes.data, None, None, None, None, None, None, None)
        if rc != 0:
            raise RuntimeError(f"reference tables failed: {rc}")
        t = {"rec_unique": np.zeros(counts[0], np.uint64), "donor_patch": np.zeros(counts[1], np.int32),
             "num_receivers": np.zeros(counts[1], np.int64), "stride": np.zeros(counts[1], np.int32),
             "rec_concat": np.zeros(counts[2], np.uint64), "donor_idx": np.zeros(counts[3], np.uint64),
             "weight": np.zeros(counts[3], np.float64)}
        rc = self.lib.dnref_grid_tables(self.h, p, counts.ctypes.data, t["rec_unique"].ctypes.data,
                                        t["donor_patch"].ctypes.data, t["num_receivers"].ctypes.data,
                                        t["stride"].ctypes.data, t["rec_concat"].ctypes.data,
                                        t["donor_idx"].ctypes.data, t["weight"].ctypes.data)
        if rc != 0:
            raise RuntimeError(f"reference tables failed: {rc}")
        t["counts"] = counts
        return t

    def set_bc(self, p, side, kind, params=None, table=None):
        self.lib.dnref_grid_set_bc.restype = c_int
        self.lib.dnref_grid_set_bc.argtypes = [c_void_p, c_int, c_int, c_int, _P, _P]
        pa = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
        ta = None if table is None else np.ascontiguousarray(table, dtype=np.float64)
        rc = self.lib.dnref_grid_set_bc(self.h, p, side, kind, None if pa is None else pa.ctypes.data_as(_P),
                                        None if ta is None else ta.ctypes.data_as(_P))
        if rc != 0:
            raise RuntimeError(f"reference set_bc failed: {rc}")

    def levelset(self, G, num_inner, num_outer, min_inner_rel_dist):
        """G: list per patch of [ni][nj][nk] level-set values or None (the
        grid must have num_vars=6)."""
        keep = [None if g is None else np.ascontiguousarray(g, dtype=np.float64) for g in G]
        arr = (_P * len(keep))(*[None if g is None else g.ctypes.data_as(_P) for g in keep])
        rc = self.lib.dnref_grid_levelset(self.h, arr, int(num_inner), int(num_outer), float(min_inner_rel_dist))
        if rc != 0:
            raise RuntimeError(f"reference level set failed: {rc}")

    def levelset_layer(self, p, inner, layer):
        n = ctypes.c_longlong()
        rc = self.lib.dnref_grid_levelset_layer(self.h, p, inner, layer, ctypes.addressof(n), None, None, None,
                                                None, None)
        if rc != 0:
            raise RuntimeError(f"reference level-set layer failed: {rc}")
        m = n.value
        d = {"cells": np.zeros(m, np.uint64), "g": np.zeros(m), "grad": np.zeros((m, 3)),
             "donors": np.zeros((m, 8), np.uint64), "weights": np.zeros((m, 8))}
        self.lib.dnref_grid_levelset_layer(self.h, p, inner, layer, ctypes.addressof(n), d["cells"].ctypes.data,
                                           d["g"].ctypes.data, d["grad"].ctypes.data, d["donors"].ctypes.data,
                                           d["weights"].ctypes.data)
        return d

    def set_state(self, p, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        if self.lib.dnref_grid_set_state(self.h, p, U.ctypes.data_as(_P)) != 0:
            raise RuntimeError("set_state failed")

    def get_state(self, p):
        n = self.patches[p]["n"]
        U = np.empty((5, n[0], n[1], n[2]))
        if self.lib.dnref_grid_get_state(self.h, p, U.ctypes.data_as(_P)) != 0:
            raise RuntimeError("get_state failed")
        return U

    def copy_donor_data(self, field=0):
        if self.lib.dnref_grid_copy_donor_data(self.h, field) != 0:
            raise RuntimeError("copy_donor_data failed")

    def deactivate(self, p, inactive=True):
        """Patch p left out of the following runs' stages (the iterator's
        deactivatePatch, iterators/patchiterator.h:127-133)."""
        self.lib.dnref_grid_deactivate.restype = c_int
        self.lib.dnref_grid_deactivate.argtypes = [c_void_p, c_int, c_int]
        if self.lib.dnref_grid_deactivate(self.h, int(p), int(bool(inactive))) != 0:
            raise RuntimeError("deactivate failed")

    def run(self, steps, dt, alpha=(0.25, 0.5, 1.0), scheme=0):
        al = np.ascontiguousarray(alpha, dtype=np.float64)
        sec = c_double()
        rc = self.lib.dnref_grid_run_scheme(self.h, int(scheme), int(steps), float(dt), al.ctypes.data_as(_P),
                                            len(al), ctypes.byref(sec))
        if rc != 0:
            raise RuntimeError(f"reference grid run failed: {rc}")
        return sec.value

    def close(self):
        if self.h:
            self.lib.dnref_grid_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def oracle_donor_copy(states, tables):
    """Donor copy (Patch::accessDonorDataDirect, patch.cpp:573-653) over the
    state list, in place: each receiving cell = sum over donor patches (table
    order) of the donor's sum over contributions of U_donor * w."""
    for r, t in enumerate(tables):
        nu = len(t["rec_unique"])
        if nu == 0:
            continue
        Ur = states[r].reshape(5, -1)
        acc = {}
        rc = 0
        wi = 0
        for q, d in enumerate(t["donor_patch"]):
            m, s = int(t["num_receivers"][q]), int(t["stride"][q])
            cells = t["rec_concat"][rc:rc + m].astype(np.int64)
            idx = t["donor_idx"][wi:wi + m * s].astype(np.int64).reshape(m, s)
            w = t["weight"][wi:wi + m * s].reshape(m, s)
            Ud = states[int(d)].reshape(5, -1)
            inter = np.zeros((5, m))
            for k in range(s):
                inter = inter + Ud[:, idx[:, k]] * w[:, k]
            for j, c in enumerate(cells):
                acc.setdefault(int(c), []).append(inter[:, j])
            rc += m
            wi += m * s
        for c, parts in acc.items():
            a = np.zeros(5)
            for x in parts:
                a = a + x
            Ur[:, c] = a


def oracle_levelset_bc(states, layers):
    """Slip-wall mirror condition (CPU_LevelSetObjectBC<LSOBCCompressibleEulerOp>,
    cpu_levelsetobjectbc.h:58-90, lsobccompressibleeulerop.h:49-144) in place:
    layers[p] = list of inner layer dicts (cells, grad, donors, weights) or None.
    Pass 1 gathers every layer cell's mirror state, pass 2 writes the cells."""
    acc = {}
    for p, L in enumerate(layers):
        if not L:
            continue
        U = states[p].reshape(5, -1)
        for li, d in enumerate(L):
            a = np.zeros((5, len(d["cells"])))
            for t in range(8):
                idx = d["donors"][:, t].astype(np.int64)
                a = a + d["weights"][:, t] * U[:, idx]
            acc[(p, li)] = a
    relax, eps = 0.5, 1.e-6
    for p, L in enumerate(layers):
        if not L:
            continue
        U = states[p].reshape(5, -1)
        for li, d in enumerate(L):
            a = acc[(p, li)]
            c = d["cells"].astype(np.int64)
            gx, gy, gz = d["grad"][:, 0], d["grad"][:, 1], d["grad"][:, 2]
            n = a[1] * gx + a[2] * gy + a[3] * gz
            for m, g in ((1, gx), (2, gy), (3, gz)):
                cur = U[m, c]
                hard = a[m] - 2. * n * g
                damp = np.abs(cur - hard) / (np.abs(cur) + eps)
                damp = np.where(damp > (1. - relax), 1. - relax, damp)
                U[m, c] = (1. - damp) * hard + damp * cur
            U[0, c] = a[0]
            U[4, c] = a[4]


def oracle_grid_run(states, spacings, tables, dt, steps, alpha=(0.25, 0.5, 1.0), bcs=None, layers=None):
    """RK steps of a patch grid with the C restatement of the residual
    (closed patch faces, with the patch-face fluxes of bcs[p] = {side: (kind,
    params, table)}) and the numpy donor copy, in the order of
    RungeKutta::operator() (rungekutta.cpp:27-42).  Returns new states."""
    U = [np.ascontiguousarray(s, dtype=np.float64).copy() for s in states]
    for _ in range(steps):
        oracle_donor_copy(U, tables)
        Un = [u.copy() for u in U]
        for q, a in enumerate(alpha):
            if q > 0:
                oracle_donor_copy(U, tables)   # repeats the last copy unless a post-operation changed donors
            for p, u in enumerate(U):
                hx, hy, hz = spacings[p]
                res = oracle_residual_bc(u, (hx, hy, hz), (bcs or {}).get(p, {}))
                pf = (a * dt) / (hx * hy * hz)
                U[p] = Un[p] + pf * res
            oracle_donor_copy(U, tables)
            if layers is not None:
                oracle_levelset_bc(U, layers)
    return U


def oracle_flow_stats(U, dt, dx):
    """The reference applications' output-step diagnostics of one patch
    (drnumBaseFlowDemo/main.h:255-284; PerfectGas::conservativeToPrimitive,
    perfectgas.h:84-93, with R = 287.2, gamma = 1.4, cv = 717.5): CFL_max
    over the cells of max(|u|, |u+a|, |u-a|) * dt / dx, and the density
    range started from 1000 and 0.  numpy evaluates each operation in FP64
    with IEEE rounding and no contraction, in the reference's order."""
    R, gamma, cv = 287.2, 1.4, 717.5
    U = np.asarray(U, dtype=np.float64).reshape(5, -1)
    ir = 1.0 / U[0]
    u, v, w = U[1] * ir, U[2] * ir, U[3] * ir
    T = (U[4] * ir - 0.5 * ((u * u + v * v) + w * w)) / cv
    a = np.sqrt((gamma * R) * T)
    cfl = max(0.0, float(np.max(np.abs(u) * dt / dx)), float(np.max(np.abs(u + a) * dt / dx)),
              float(np.max(np.abs(u - a) * dt / dx)))
    return cfl, min(1000.0, float(U[0].min())), max(0.0, float(U[0].max()))


# --------------------------------------------- the reference's GPU level-set path

def oracle_levelset_gpu_setup(G, h):
    """GPU_CartesianLevelSetBC's set-up (gpu_cartesianlevelsetbc.h:106-125,
    129-229) on one patch: the G < 0 cells (deactivated) and the inside cells
    (no G >= 0 cell in the edge-limited two-cell box) with the neighbours the
    inside-cell kernel averages and their weights |d . grad G| / |d| (:414-487),
    grad G as GPU_CartesianLevelSetBC::grad (:78-93).  Raises where the
    reference stops with a BUG (:170-179)."""
    G = np.asarray(G, dtype=np.float64)
    imax, jmax, kmax = G.shape
    hx, hy, hz = (h, h, h) if np.isscalar(h) else h
    idx, idy, idz = 1.0 / hx, 1.0 / hy, 1.0 / hz
    below, inside = [], []
    for i in range(imax):
        for j in range(jmax):
            for k in range(kmax):
                if not G[i, j, k] < 0:
                    continue
                below.append((i * jmax + j) * kmax + k)
                ext = True
                i0, i1, j0, j1, k0, k1 = -2, 2, -2, 2, -2, 2
                if i < 2: i0 += 2 - i
                if i == imax - 1: i1 = 0
                if i == imax - 2: i1 = 1
                if j < 2: j0 += 2 - j
                if j == jmax - 1: j1 = 0
                if j == jmax - 2: j1 = 1
                if k < 2: k0 += 2 - k
                if k == kmax - 1: k1 = 0
                if k == kmax - 2: k1 = 1
                for di in range(i0, i1 + 1):
                    for dj in range(j0, j1 + 1):
                        for dk in range(k0, k1 + 1):
                            if di == 0 and dj == 0 and dk == 0:
                                continue
                            a, b, c = i + 2 * di, j + 2 * dj, k + 2 * dk
                            if min(a, b, c) < 0 or a >= imax or b >= jmax or c >= kmax:
                                raise ValueError(f"G < 0 cell {(i, j, k)} too close to the patch edge")
                            if G[i + di, j + dj, k + dk] >= 0:
                                ext = False
                                break
                if not ext:
                    continue
                if i < 2: i0 = 0
                if i >= imax - 2: i1 = 0
                if j < 2: j0 = 0
                if j >= jmax - 2: j1 = 0
                if k < 2: k0 = 0
                if k >= kmax - 2: k1 = 0
                g = lambda a, b, c: float(G[a, b, c])
                if i == 0: gx = idx * (g(i + 1, j, k) - g(i, j, k))
                elif i == imax - 1: gx = idx * (g(i, j, k) - g(i - 1, j, k))
                else: gx = 0.5 * idx * (g(i + 1, j, k) - g(i - 1, j, k))
                if j == 0: gy = idy * (g(i, j + 1, k) - g(i, j, k))
                elif j == jmax - 1: gy = idy * (g(i, j, k) - g(i, j - 1, k))
                else: gy = 0.5 * idy * (g(i, j + 1, k) - g(i, j - 1, k))
                if k == 0: gz = idz * (g(i, j, k + 1) - g(i, j, k))
                elif k == kmax - 1: gz = idz * (g(i, j, k) - g(i, j, k - 1))
                else: gz = 0.5 * idz * (g(i, j, k + 1) - g(i, j, k - 1))
                nbr, w = [], []
                for di in range(i0, i1 + 1):
                    for dj in range(j0, j1 + 1):
                        for dk in range(k0, k1 + 1):
                            if di == 0 and dj == 0 and dk == 0:
                                continue
                            gn = g(i + di, j + dj, k + dk)
                            if gn >= 0 or gn > g(i, j, k):
                                ddx, ddy, ddz = float(di) * hx, float(dj) * hy, float(dk) * hz
                                nbr.append(((i + di) * jmax + j + dj) * kmax + k + dk)
                                w.append(abs(ddx * gx + ddy * gy + ddz * gz) / math.sqrt(ddx * ddx + ddy * ddy + ddz * ddz))
                inside.append(((i * jmax + j) * kmax + k, nbr, w))
    return below, inside


def oracle_levelset_gpu_apply(U, Un, setup, receivers=()):
    """GPU_CartesianLevelSetBC::operator() after a stage (in place on U):
    the deactivated cells hold the step-start state Un, as the reference's
    GPU advance kernel leaves inactive cells (gpu_cartesianiterator.h:199-205),
    except cells a donor copy writes (`receivers`); then every inside cell
    with neighbours takes their weighted mean, all read before any is written
    (the reference writes field 2 and copies it back)."""
    below, inside = setup
    u = U.reshape(5, -1)
    un = Un.reshape(5, -1)
    rec = set(int(x) for x in receivers)
    for c in below:
        if c not in rec:
            u[:, c] = un[:, c]
    out = []
    for c, nbr, w in inside:
        if not nbr:
            continue
        var = np.zeros(5)
        total = 0.0
        for n, wt in zip(nbr, w):
            total += wt
            var = var + wt * u[:, n]
        out.append((c, var / total))
    for c, v in out:
        if not np.isfinite(v).all():
            raise FloatingPointError("inside-cell average not finite")
        u[:, c] = v
