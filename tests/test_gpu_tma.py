"""The two ways the stage kernels stage their planes give identical bits:
TMA box loads, and cell-by-cell asynchronous copies (with wrapped or
clamped cells) for the tiles TMA cannot serve.  With
DN_FX_NO_TMA=1 every tile copies cell by cell; the results must not
change, on periodic, closed and mixed patches, with inactive cells, and
with the per-stage residual and conservation sums."""
import os

import numpy as np
import pytest

from drnum_b200 import cases
from drnum_b200._lib import DN_FP32, DN_FP64
from drnum_b200.api import AusmPlus, B200CartesianIterator, CartesianPatch

pytestmark = pytest.mark.gpu


def run_fx32(U0, h, dt, steps, periodic, active=None, no_tma=False, precision=DN_FP32):
    old = os.environ.get("DN_FX_NO_TMA")
    os.environ["DN_FX_NO_TMA"] = "1" if no_tma else "0"
    try:
        _, ni, nj, nk = U0.shape
        p = CartesianPatch(ni, nj, nk, spacing=(h, h, h), periodic=periodic)
        p.setField(0, U0)
        if active is not None:
            p.active[...] = active
        it = B200CartesianIterator(AusmPlus(), 0, precision)
        it.addPatch(p)
        it.updateDevice(fields=(0,))
        for _ in range(steps):
            it.rkStep(dt, cases.RK3_ALPHA)
        it.updateHost(fields=(0,))
        sums = it.conservationSums()
        want = 0 if no_tma or (precision == DN_FP64 and nk % 2) else 1
        assert it.tmaPatchCount() == want
        it.close()
        return p.getField(0).copy(), sums
    finally:
        if old is None:
            del os.environ["DN_FX_NO_TMA"]
        else:
            os.environ["DN_FX_NO_TMA"] = old


@pytest.mark.parametrize("shape,periodic", [
    ((40, 64, 64), (True, True, True)),      # 4 x 4 tiles: 4 interior
    ((24, 72, 80), (False, False, False)),   # closed on every axis
    ((20, 50, 68), (True, False, True)),     # ragged tiles, mixed axes
    ((16, 36, 36), (False, True, False)),    # the smallest patch with an interior tile
    ((18, 40, 37), (True, True, True)),      # nk % 4 != 0: padded rows, periodic seams
    ((12, 35, 42), (False, False, False)),   # padded rows, closed
    ((10, 19, 5), (True, False, True)),      # one ragged k tile of 5 cells in rows of 8
])
def test_tma_staging_equals_cell_copies(shape, periodic):
    ni, nj, nk = shape
    U0 = cases.random_state(ni, nj, nk, seed=ni + nj + nk, amp=0.03, mach=0.4)
    h = 1.0 / 32
    dt = cases.cfl_dt(U0, h, 0.5)
    a, sa = run_fx32(U0, h, dt, 3, periodic)
    b, sb = run_fx32(U0, h, dt, 3, periodic, no_tma=True)
    assert np.array_equal(a, b)
    assert np.array_equal(np.asarray(sa), np.asarray(sb))
    assert not np.array_equal(a, U0)


def test_tma_staging_with_inactive_cells_and_vortex_box():
    U0, h, dt = cases.periodic_box(48)
    rng = np.random.default_rng(5)
    active = (rng.random((48, 48, 48)) > 0.1).astype(np.uint8)
    a, _ = run_fx32(U0, h, dt, 4, (True, True, True), active)
    b, _ = run_fx32(U0, h, dt, 4, (True, True, True), active, no_tma=True)
    assert np.array_equal(a, b)


def run_workload_fx32(name, scale, steps, no_tma, shapes=None):
    from drnum_b200 import _lib, workloads
    old = os.environ.get("DN_FX_NO_TMA")
    os.environ["DN_FX_NO_TMA"] = "1" if no_tma else "0"
    try:
        case = workloads.build(name, scale)
        _, objs = workloads.make_grid(case)
        it = workloads.make_iterator(objs, DN_FP32)
        it.setOption(_lib.DN_OPT_BATCHED, 1)
        if shapes is not None:
            for p in range(len(objs)):
                it.setTile(p, shapes[p % len(shapes)])
        for _ in range(steps):
            it.rkStep(case["dt"], cases.RK3_ALPHA)
        it.updateHost(fields=(0,))
        out = [o.getField(0).copy() for o in objs]
        # every FP32 patch (rows padded to 16 bytes) is staged by TMA unless it is turned off
        assert it.tmaPatchCount() == (0 if no_tma else len(objs))
        it.close()
        return out
    finally:
        if old is None:
            del os.environ["DN_FX_NO_TMA"]
        else:
            os.environ["DN_FX_NO_TMA"] = old


@pytest.mark.parametrize("name,scale,shapes", [
    ("sphere", 0.25, None),          # closed patches, level-set wall
    ("tiled", 0.25, [0, 1]),         # 8 uneven patches, both tile shapes
    ("jet", 0.125, [1]),             # far field and inflow faces
])
def test_batched_tma_staging_equals_cell_copies(name, scale, shapes):
    a = run_workload_fx32(name, scale, 3, False, shapes)
    b = run_workload_fx32(name, scale, 3, True, shapes)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("shape,periodic", [
    ((24, 40, 72), (True, True, True)),      # 4 x 32 tiles: interior, seam and ragged
    ((20, 18, 40), (False, False, False)),   # closed: every tile by TMA, zero-filled halo
    ((16, 22, 66), (False, True, True)),
    ((12, 20, 37), (True, True, True)),      # odd nk: no TMA map, both runs copy cell by cell
])
def test_fp64_tma_staging_equals_cell_copies(shape, periodic):
    ni, nj, nk = shape
    U0 = cases.random_state(ni, nj, nk, seed=3 * ni + nk, amp=0.03, mach=0.4)
    h = 1.0 / 32
    dt = cases.cfl_dt(U0, h, 0.5)
    a, sa = run_fx32(U0, h, dt, 2, periodic, precision=DN_FP64)
    b, sb = run_fx32(U0, h, dt, 2, periodic, no_tma=True, precision=DN_FP64)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, U0)
