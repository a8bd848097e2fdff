"""The reference's GPU level-set path (GPU_CartesianLevelSetBC with
CompressibleLsSlip-style inside cells): G < 0 cells deactivated and held at
the step-start state, inside cells replaced by the weighted mean of their
neighbours of larger G after every stage.  FP64 bitwise against the numpy
restatement oracle/pyoracle.py::oracle_levelset_gpu_*; FP32 bulk within
tolerance of FP64."""
import ctypes

import numpy as np
import pytest

import pyoracle
from drnum_b200 import _lib, cases
from drnum_b200._lib import DN_ERR_ARG, DN_FP32, DN_FP64
from drnum_b200.api import AusmPlus, B200CartesianIterator, CartesianPatch

N, H = 24, 1.0 / 24


def _case():
    U0 = cases.random_state(N, N, N, seed=5, amp=0.01, mach=0.3)
    patch = dict(n=(N, N, N), origin=(0.0, 0.0, 0.0), length=(1.0, 1.0, 1.0), seek=(0, 0, 0, 0, 0, 0))
    G = cases.sphere_sdf(patch, (0.5, 0.47, 0.52), 0.3)
    dt = cases.cfl_dt(U0, H, 0.5)
    return U0, G, dt


def _oracle(U0, G, dt, steps, alphas=cases.RK3_ALPHA):
    setup = pyoracle.oracle_levelset_gpu_setup(G, H)
    active = G >= 0
    U = U0.copy()
    for _ in range(steps):
        Un = U.copy()
        for a in alphas:
            res = pyoracle.oracle_residual_bc(U, H, {}, periodic=(False, False, False))
            pf = (a * dt) / (H * H * H)
            U = np.where(active[None], Un + pf * res, U)
            pyoracle.oracle_levelset_gpu_apply(U, Un, setup)
    return U, setup


def _gpu(U0, G, dt, steps, precision):
    p = CartesianPatch(N, N, N, spacing=(H, H, H), periodic=(False, False, False))
    p.setField(0, U0)
    it = B200CartesianIterator(AusmPlus(), 0, precision)
    it.addPatch(p)
    it.updateDevice(fields=(0,))
    lib = _lib.load()
    Gc = np.ascontiguousarray(G)
    _lib.check(it.ctx, lib.dn_patch_set_levelset_gpu(it.ctx, 0, Gc.ctypes.data))
    counts = np.zeros(3, dtype=np.int64)
    _lib.check(it.ctx, lib.dn_patch_levelset_gpu_counts(it.ctx, 0, counts.ctypes.data))
    for _ in range(steps):
        it.rkStep(dt, cases.RK3_ALPHA)
    it.updateHost(fields=(0,))
    it.close()
    return p.getField(0).copy(), counts


pytestmark = pytest.mark.gpu


def test_gpu_levelset_path_fp64_bitwise_vs_restatement():
    U0, G, dt = _case()
    want, (below, inside) = _oracle(U0, G, dt, 3)
    assert len(inside) > 0 and any(n for _, n, _ in inside)
    got, counts = _gpu(U0, G, dt, 3, DN_FP64)
    assert list(counts) == [len(below), len(inside), sum(len(n) for _, n, _ in inside)]
    assert np.array_equal(got, want), np.abs(got - want).max()


def test_gpu_levelset_path_fp32_tracks_fp64():
    U0, G, dt = _case()
    a, _ = _gpu(U0, G, dt, 3, DN_FP64)
    b, _ = _gpu(U0, G, dt, 3, DN_FP32)
    d = np.abs(b[0] - a[0]) / cases.RHO_INF
    assert np.sqrt((d ** 2).mean()) < 1e-5 and d.max() < 1e-4, d.max()


def test_gpu_levelset_path_refuses_cells_near_the_edge():
    # a G < 0 cell one cell from the edge: the reference's set-up stops with a BUG
    U0, _, _ = _case()
    G = np.ones((N, N, N))
    G[1, 10, 10] = -1.0
    p = CartesianPatch(N, N, N, spacing=(H, H, H), periodic=(False, False, False))
    p.setField(0, U0)
    it = B200CartesianIterator(AusmPlus(), 0, DN_FP64)
    it.addPatch(p)
    lib = _lib.load()
    Gc = np.ascontiguousarray(G)
    assert lib.dn_patch_set_levelset_gpu(it.ctx, 0, Gc.ctypes.data) == DN_ERR_ARG
    it.close()
