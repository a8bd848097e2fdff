"""Parity of the CUDA stage kernels (through the C ABI) with the reference
outputs and the oracle.

FP64: bit-exact against the reference library's own outputs (golden
fixtures) and against the oracle restatement on further shapes.
FP32 bulk: relative L2 / L-infinity error against the FP64 oracle within the
stated tolerances, and exact conservation on periodic patches.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import cases_def
import pyoracle
from drnum_b200 import cases
from drnum_b200._lib import DN_FP32, DN_FP64, DnError
from drnum_b200.api import AusmPlus, B200CartesianIterator, CartesianPatch, RungeKutta

pytestmark = pytest.mark.gpu

# FP32 bulk tolerances against the FP64 oracle (relative to the free-stream
# magnitude of each variable), after the stated number of steps
F32_L2_TOL = 2e-6
F32_LINF_TOL = 5e-5


def run_gpu(U0, h, dt, steps, periodic=(True, True, True), active=None, precision=DN_FP64,
            alpha=cases.RK3_ALPHA, use_compute=False):
    _, ni, nj, nk = U0.shape
    patch = CartesianPatch(ni, nj, nk, spacing=(h, h, h), periodic=periodic)
    patch.setField(0, U0)
    if active is not None:
        patch.active[...] = active
    it = B200CartesianIterator(AusmPlus(), 0, precision)
    it.addPatch(patch)
    it.updateDevice(fields=(0,))
    if use_compute:
        for _ in range(steps):
            it.copyField(0, 1)
            for a in alpha:
                it.compute(a * dt)
    else:
        rk = RungeKutta()
        for a in alpha:
            rk.addAlpha(a)
        rk.addIterator(it)
        for _ in range(steps):
            rk(dt)
    it.updateHost(fields=(0,))
    sums = it.conservationSums()
    it.close()
    return patch.getField(0).copy(), sums


def load_golden(golden_dir, name):
    z = np.load(os.path.join(golden_dir, f"{name}.npz"))
    active = z["active"] if z["active"].size else None
    return z, active


@pytest.mark.parametrize("name", cases_def.FULL)
def test_fp64_bitwise_vs_reference_fixtures(golden_dir, name):
    z, active = load_golden(golden_dir, name)
    out, _ = run_gpu(z["U0"], float(z["h"]), float(z["dt"]), int(z["steps"]),
                     tuple(bool(p) for p in z["periodic"]), active)
    assert np.array_equal(out, z["out"]), f"max abs diff {np.abs(out - z['out']).max()}"


def test_fp64_cfg1_64cube_100_steps_bitwise(golden_dir):
    meta = json.load(open(os.path.join(golden_dir, "digests.json")))["cfg1_64_100"]
    c = cases_def.build("cfg1_64_100")
    out, _ = run_gpu(np.ascontiguousarray(c["U0"]), c["h"], c["dt"], c["steps"])
    assert hashlib.sha256(np.ascontiguousarray(out).tobytes()).hexdigest() == meta["output_sha256"]


@pytest.mark.parametrize("shape,periodic,steps", [
    ((37, 29, 45), (True, True, True), 3),       # ragged against the 4x32 / 8x32 tiles
    ((70, 5, 33), (True, False, True), 2),        # several i-chunks, thin closed y
    ((16, 40, 3), (False, True, False), 3),       # tiny closed k (first-order everywhere)
    ((2, 9, 11), (False, True, True), 2),         # i <= 2: no x faces (cartesianiterator.h:149)
    ((24, 24, 24), (False, False, False), 4),     # closed box
])
def test_fp64_bitwise_vs_oracle(shape, periodic, steps):
    U0 = cases.random_state(*shape, seed=11, amp=0.02, mach=0.5)
    h = 1.0 / 32
    dt = cases.cfl_dt(U0, h, 0.5)
    ref = pyoracle.oracle_run(U0, h, dt, steps, periodic=periodic)
    out, _ = run_gpu(U0, h, dt, steps, periodic)
    assert np.array_equal(out, ref), f"max abs diff {np.abs(out - ref).max()}"


def test_fp64_stagewise_api_equals_fused_step():
    U0, h, dt = cases.periodic_box(24)
    a, _ = run_gpu(U0, h, dt, 3)
    b, _ = run_gpu(U0, h, dt, 3, use_compute=True)
    assert np.array_equal(a, b)


def test_fp64_residual_single_stage_matches_oracle():
    U0 = cases.random_state(13, 17, 19, seed=5, amp=0.03, mach=0.7)
    h = 1.0 / 20
    res = pyoracle.oracle_residual(U0, h)
    factor = 1e-7
    out, _ = run_gpu(U0, h, factor, 1, alpha=(1.0,))
    expect = U0 + (factor / (h * h * h)) * res
    assert np.array_equal(out, expect)


def rel_errors(a, b):
    scale = np.array([cases.RHO_INF, cases.RHO_INF * cases.A_INF, cases.RHO_INF * cases.A_INF,
                      cases.RHO_INF * cases.A_INF, cases.RHO_INF * cases.GAS_CV * cases.T_INF])
    d = (a - b) / scale[:, None, None, None]
    return np.sqrt((d ** 2).reshape(5, -1).mean(1)), np.abs(d).reshape(5, -1).max(1)


def test_fp32_error_and_exact_conservation_vortex_48():
    U0, h, dt = cases.periodic_box(48)
    steps = 50
    ref = pyoracle.oracle_run(U0, h, dt, steps)
    out, sums = run_gpu(U0, h, dt, steps, precision=DN_FP32)
    l2, linf = rel_errors(out, ref)
    assert l2.max() < F32_L2_TOL, l2
    assert linf.max() < F32_LINF_TOL, linf
    # exact conservation: the FP64 sums equal those of the quantised initial state
    _, s0 = run_gpu(U0, h, dt, 0, precision=DN_FP32)
    assert np.array_equal(sums, s0), sums - s0


def test_fp32_closed_and_masked_against_oracle():
    U0 = cases.random_state(20, 18, 22, seed=9, amp=0.01, mach=0.4)
    h = 1.0 / 32
    dt = cases.cfl_dt(U0, h, 0.5)
    act = (np.random.default_rng(3).random((20, 18, 22)) > 0.1).astype(np.uint8)
    ref = pyoracle.oracle_run(U0, h, dt, 5, periodic=(False, True, False), active=act)
    out, _ = run_gpu(U0, h, dt, 5, (False, True, False), act, precision=DN_FP32)
    l2, linf = rel_errors(out, ref)
    assert l2.max() < F32_L2_TOL and linf.max() < F32_LINF_TOL, (l2, linf)
    frozen = act == 0
    # inactive cells keep their start value exactly (as stored on the device)
    start, _ = run_gpu(U0, h, dt, 0, (False, True, False), act, precision=DN_FP32)
    assert np.array_equal(out[:, frozen], start[:, frozen])


def test_upload_download_roundtrip():
    U0 = cases.random_state(9, 10, 11, seed=1)
    for prec in (DN_FP64, DN_FP32):
        out, _ = run_gpu(U0, 0.1, 0.0, 0, precision=prec)
        if prec == DN_FP64:
            assert np.array_equal(out, U0)
        else:
            # quantisation error is at most half a quantum of the variable
            # (quantum <= 2^-24 * magnitude scale, which is below 1.2x max|U_v|)
            for v in range(5):
                scale = np.abs(U0[v]).max() if v in (0, 4) else 2 * np.abs(U0[1:4]).max() + 1e3
                assert np.abs(out[v] - U0[v]).max() <= scale * 2.0 ** -24, v


@pytest.mark.parametrize("prec", [DN_FP64, DN_FP32])
def test_async_transfer_pipeline_equals_synchronous_calls(prec):
    # upload k+1 / stages k+1 / download k overlapping through the async
    # calls give the same bits as the synchronous calls, every step
    import ctypes
    import torch
    from drnum_b200 import _lib
    U0, h, dt = cases.periodic_box(24)
    ht = torch.float64 if prec == DN_FP64 else torch.float32
    nt = np.float64 if prec == DN_FP64 else np.float32
    ptr = _lib.dptr if prec == DN_FP64 else _lib.fptr
    up_sync = "dn_patch_upload" if prec == DN_FP64 else "dn_patch_upload_f32"
    dn_sync = "dn_patch_download" if prec == DN_FP64 else "dn_patch_download_f32"
    alpha = np.ascontiguousarray(cases.RK3_ALPHA, dtype=np.float64)
    results = []
    for mode in ("sync", "async"):
        patch = CartesianPatch(24, 24, 24, spacing=(h, h, h))
        it = B200CartesianIterator(AusmPlus(), 0, prec)
        it.addPatch(patch)
        lib, ctx = it.lib, it.ctx
        hin = [torch.empty(U0.shape, dtype=ht, pin_memory=True).numpy() for _ in range(2)]
        hout = [torch.empty(U0.shape, dtype=ht, pin_memory=True).numpy() for _ in range(4)]
        for b in hin:
            b[...] = U0.astype(nt)
        for k in range(4):
            # step k starts from input (k % 2); the inputs hold the same state
            if mode == "sync":
                _lib.check(ctx, getattr(lib, up_sync)(ctx, 0, 0, ptr(hin[k % 2])))
                _lib.check(ctx, lib.dn_rk_step(ctx, dt, _lib.dptr(alpha), 3))
                _lib.check(ctx, getattr(lib, dn_sync)(ctx, 0, 0, ptr(hout[k])))
            else:
                _lib.check(ctx, getattr(lib, up_sync + "_async")(ctx, 0, 0, ptr(hin[k % 2])))
                _lib.check(ctx, lib.dn_rk_step(ctx, dt, _lib.dptr(alpha), 3))
                _lib.check(ctx, getattr(lib, dn_sync + "_async")(ctx, 0, 0, ptr(hout[k])))
        _lib.check(ctx, lib.dn_sync(ctx))
        results.append([o.copy() for o in hout])
        it.close()
    for k in range(4):
        assert np.array_equal(results[0][k], results[1][k]), k
        assert np.array_equal(results[1][k], results[1][0]), k
    assert not np.array_equal(results[0][0], U0.astype(nt))


def test_field_difference_matches_numpy():
    U0, h, dt = cases.periodic_box(16)
    patch = CartesianPatch(16, 16, 16, spacing=(h, h, h))
    patch.setField(0, U0)
    it = B200CartesianIterator(AusmPlus(), 0, DN_FP64)
    it.addPatch(patch)
    it.updateDevice(fields=(0,))
    it.rkStep(dt, cases.RK3_ALPHA)
    it.updateHost(fields=(0, 1))
    mx, l2 = it.computeVariableDifference(0, 0, 0, 1, 0)
    d = patch.getField(1)[0] - patch.getField(0)[0]
    assert np.isclose(mx, np.abs(d).max(), rtol=1e-12)
    assert np.isclose(l2, np.sqrt((d ** 2).sum()), rtol=1e-12)
    it.close()


def test_errors_are_reported_not_fatal():
    it = B200CartesianIterator(AusmPlus(), 0, DN_FP64)
    with pytest.raises(DnError):
        it.addPatch(CartesianPatch(2, 8, 8, spacing=(0.1, 0.1, 0.1), periodic=(True, True, True)))
    with pytest.raises(DnError):
        it.addPatch(CartesianPatch(8, 8, 8, spacing=(0.0, 0.1, 0.1)))
    with pytest.raises(DnError):
        it.rkStep(float("nan"), cases.RK3_ALPHA)
    it.close()
