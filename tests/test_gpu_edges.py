"""Edge cases of the device path: size limits, the fixed-point range, thin
and degenerate axes in FP32, inactive cells in FP32, an empty level-set
wall.  Every failure is a returned status; the context stays usable."""
import numpy as np
import pytest

import cases_def
from drnum_b200 import cases
from drnum_b200._lib import DN_ERR_RANGE, DN_FP32, DN_FP64, DnError
from drnum_b200.api import AusmPlus, B200CartesianIterator, CartesianPatch

pytestmark = pytest.mark.gpu


def test_fp32_patch_over_the_offset_limit_is_refused_before_allocation():
    it = B200CartesianIterator(AusmPlus(), 0, DN_FP32)
    with pytest.raises(DnError) as e:
        it.addPatch(CartesianPatch(1024, 1024, 420, spacing=(1e-3,) * 3))   # 5 * cells >= 2^31
    assert "2^31" in str(e.value)
    # still usable
    U0, h, dt = cases.periodic_box(16)
    p = CartesianPatch(16, 16, 16, spacing=(h, h, h))
    p.setField(0, U0)
    it.addPatch(p)
    it.updateDevice(fields=(0,))
    it.rkStep(dt, cases.RK3_ALPHA)
    it.close()


def test_fp32_state_outside_the_offset_range_is_reported():
    U0, h, dt = cases.periodic_box(16)
    it = B200CartesianIterator(AusmPlus(), 0, DN_FP32)
    p = CartesianPatch(16, 16, 16, spacing=(h, h, h))
    it.addPatch(p)
    base = U0.reshape(5, -1).mean(axis=1)
    # a range a thousand times too small for the state: the upload must fail
    it.setBase(0, base, np.abs(U0.reshape(5, -1) - base[:, None]).max(axis=1) / 1000 + 1e-30)
    p.setField(0, U0)
    with pytest.raises(DnError) as e:
        it.updateDevice(fields=(0,))
    assert e.value.code == DN_ERR_RANGE
    # with a range that covers the state (and, for the momenta, the pressure
    # flux) the same context works afterwards
    scale = np.array([U0[0].max(), 1.0, 1.0, 1.0, U0[4].max()])
    scale[1:4] = (U0[0] * (np.abs(U0[1] / U0[0]) + cases.A_INF)).max()
    it.setBase(0, base, 4 * scale)
    it.updateDevice(fields=(0,))
    it.rkStep(dt, cases.RK3_ALPHA)
    it.updateHost(fields=(0,))
    assert np.isfinite(p.getField(0)).all()
    # a momentum range far below the pressure flux scale is reported, not wrapped
    it.setBase(0, base, np.array([4 * scale[0], 1e-3, 1e-3, 1e-3, 4 * scale[4]]))
    p.setField(0, np.broadcast_to(base[:, None, None, None], U0.shape).copy())
    it.updateDevice(fields=(0,))
    with pytest.raises(DnError) as e:
        it.rkStep(dt, cases.RK3_ALPHA)
        it.sync()
    assert e.value.code == DN_ERR_RANGE
    it.close()


def test_fp32_stage_leaving_the_offset_range_is_reported_and_recoverable():
    U0, h, dt = cases.periodic_box(16)
    it = B200CartesianIterator(AusmPlus(), 0, DN_FP32)
    p = CartesianPatch(16, 16, 16, spacing=(h, h, h))
    it.addPatch(p)
    base = U0.reshape(5, -1).mean(axis=1)
    dev = np.abs(U0.reshape(5, -1) - base[:, None]).max(axis=1)
    it.setBase(0, base, dev * 1.0001 + 1e-30)      # the state just fits, a large step does not
    p.setField(0, U0)
    it.updateDevice(fields=(0,))
    with pytest.raises(DnError) as e:
        for _ in range(3):
            it.rkStep(200 * dt, cases.RK3_ALPHA)
            it.sync()
    assert e.value.code == DN_ERR_RANGE
    assert "offset" in str(e.value)
    base_ok = np.abs(U0.reshape(5, -1)).max(axis=1)
    base_ok[1:4] = (U0[0] * (np.abs(U0[1] / U0[0]) + cases.A_INF)).max()
    it.setBase(0, base, 4 * base_ok)
    it.updateDevice(fields=(0,))
    it.rkStep(dt, cases.RK3_ALPHA)
    it.sync()
    it.close()


@pytest.mark.parametrize("name", ["flat_8x2x9", "column_1x1x10", "thin_3x5x4"])
def test_fp32_thin_axes_track_fp64(golden_dir, name):
    import os
    z = np.load(os.path.join(golden_dir, f"{name}.npz"))
    periodic = tuple(bool(x) for x in z["periodic"])
    _, ni, nj, nk = z["U0"].shape
    outs = {}
    for prec in (DN_FP64, DN_FP32):
        p = CartesianPatch(ni, nj, nk, spacing=(float(z["h"]),) * 3, periodic=periodic)
        p.setField(0, z["U0"])
        it = B200CartesianIterator(AusmPlus(), 0, prec)
        it.addPatch(p)
        it.updateDevice(fields=(0,))
        for _ in range(int(z["steps"])):
            it.rkStep(float(z["dt"]), cases.RK3_ALPHA)
        it.updateHost(fields=(0,))
        it.close()
        outs[prec] = p.getField(0).copy()
    assert np.array_equal(outs[DN_FP64], z["out"])
    d = np.abs(outs[DN_FP32][0] - outs[DN_FP64][0]) / cases.RHO_INF
    assert np.sqrt((d ** 2).mean()) < 1e-5 and d.max() < 1e-4, d.max()


def test_fp32_inactive_cells_keep_their_state_exactly():
    U0 = cases.random_state(12, 10, 9, seed=21, amp=0.02, mach=0.3)
    h = 1.0 / 16
    dt = cases.cfl_dt(U0, h, 0.5)
    p = CartesianPatch(12, 10, 9, spacing=(h, h, h))
    p.setField(0, U0)
    rng = np.random.default_rng(3)
    p.active[...] = (rng.random((12, 10, 9)) > 0.2).astype(np.uint8)
    it = B200CartesianIterator(AusmPlus(), 0, DN_FP32)
    it.addPatch(p)
    it.updateDevice(fields=(0,))
    it.updateHost(fields=(0,))
    stored = p.getField(0).copy()            # the state as the fixed-point storage holds it
    for _ in range(3):
        it.rkStep(dt, cases.RK3_ALPHA)
    it.updateHost(fields=(0,))
    it.close()
    out = p.getField(0)
    off = p.active == 0
    assert np.array_equal(out[:, off], stored[:, off])
    assert not np.array_equal(out[:, ~off], stored[:, ~off])


@pytest.mark.parametrize("prec", [DN_FP64, DN_FP32])
def test_level_set_wall_outside_the_patch_changes_nothing(prec):
    U0, h, dt = cases.periodic_box(16)
    outs = []
    for wall in (False, True):
        p = CartesianPatch(16, 16, 16, spacing=(h, h, h))
        p.setField(0, U0)
        if wall:
            # a sphere far away: G > 0 everywhere, no layer cells
            desc = dict(n=(16, 16, 16), origin=(0.0, 0.0, 0.0), length=(1.0, 1.0, 1.0))
            p.setLevelSet(cases.sphere_sdf(desc, (5.0, 5.0, 5.0), 0.1), 3, 0, 0.1)
        it = B200CartesianIterator(AusmPlus(), 0, prec)
        it.addPatch(p)
        it.updateDevice(fields=(0,))
        if wall:
            it.setLevelSets()
            assert sum(len(layer["cells"]) for layer in it.levelSetLayers(0)["inner"]) == 0
        for _ in range(2):
            it.rkStep(dt, cases.RK3_ALPHA)
        it.updateHost(fields=(0,))
        it.close()
        outs.append(p.getField(0).copy())
    assert np.array_equal(outs[0], outs[1])


def test_fp32_residual_sum_beyond_int32_is_reported():
    """Six neighbours flow into one cell, advanced with an oversized step:
    each of the cell's six mass faces stays below the per-face limit of 2^30
    quanta, but their sum lies between 3 * 2^30 and 4 * 2^30, which an int32
    sum would wrap back into the valid offset range.  The stage must report
    that the offset left its range."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
    import pyoracle
    n, h, c = 8, 1.0 / 8, 4
    U0 = np.zeros((5, n, n, n))
    U0[0] = cases.RHO_INF
    U0[4] = cases.P_INF / (cases.GAS_GAMMA - 1.0)
    V = 0.3 * cases.A_INF
    for ax in range(3):
        for side in (-1, 1):
            idx = [c, c, c]
            idx[ax] += side
            U0[1 + ax][tuple(idx)] = -side * V * cases.RHO_INF   # towards the centre cell
            U0[4][tuple(idx)] += 0.5 * cases.RHO_INF * V * V
    # mass change of the centre cell per unit dt of one forward-Euler stage (FP64 oracle)
    dM = pyoracle.oracle_run(U0, h, 1.0, 1, alpha=(1.0,))[0, c, c, c] - U0[0, c, c, c]
    assert dM > 0
    base = U0.reshape(5, -1).mean(axis=1)
    # momenta and energy get wide ranges: their faces stay far below the limits
    scale = np.array([4 * cases.RHO_INF, 1e6, 1e6, 1e6, 1e12])
    q0 = 2.0 ** np.ceil(np.log2(scale[0] / 2 ** 30))
    dt = 3.5 * 2 ** 30 * q0 / dM               # the centre's mass update: 3.5 * 2^30 quanta
    assert 3.5 * 2 ** 30 / 6 < 2 ** 30         # so no single (symmetric) face reaches the limit
    p = CartesianPatch(n, n, n, spacing=(h, h, h))
    p.setField(0, U0)
    it = B200CartesianIterator(AusmPlus(), 0, DN_FP32)
    it.addPatch(p)
    it.setBase(0, base, scale)
    it.updateDevice(fields=(0,))
    with pytest.raises(DnError) as e:
        it.rkStep(dt, (1.0,))
        it.sync()
    assert e.value.code == DN_ERR_RANGE
    assert "offset left its range" in str(e.value)
    it.close()
