"""The generic flux-functor stage (include/drnum_b200_functor.cuh): the
built-in VanLeer and Roe schemes bit for bit against the reference's own
functors (golden fixtures from the compiled reference), AUSM+ through the
functor kernel bit for bit against the specialised kernel and the
reference, the patch-face kinds, graph replay, and a caller-written functor
installed with dn_set_stage_function."""
import ctypes
import os

import numpy as np
import pytest

import cases_def
from drnum_b200 import _lib, cases
from drnum_b200._lib import DN_FP32, DN_FP64, DnError
from drnum_b200.api import AusmPlus, B200CartesianIterator, CartesianPatch, Roe, RungeKutta, VanLeer
from test_gpu_grid import make_grid

pytestmark = pytest.mark.gpu

SCHEME_OPS = {"vanleer": VanLeer, "roe": Roe}
EXAMPLE_LIB = os.path.join(os.path.dirname(_lib.LIB_PATH), "examples", "libdn_example_stage.so")


def run(U0, h, dt, steps, periodic, active, op, graph=False, stagewise=False):
    _, ni, nj, nk = U0.shape
    patch = CartesianPatch(ni, nj, nk, spacing=(h, h, h), periodic=periodic)
    patch.setField(0, U0)
    if active is not None:
        patch.active[...] = active
    it = B200CartesianIterator(op, 0, DN_FP64)
    it.addPatch(patch)
    it.updateDevice(fields=(0,))
    it.setOption(_lib.DN_OPT_GRAPH, 1 if graph else 0)
    if stagewise:
        for _ in range(steps):
            it.copyField(0, 1)
            for a in cases.RK3_ALPHA:
                it.compute(a * dt)
    else:
        for _ in range(steps):
            it.rkStep(dt, cases.RK3_ALPHA)
    it.updateHost(fields=(0,))
    it.close()
    return patch.getField(0).copy()


def fixture(golden_dir, name):
    z = np.load(os.path.join(golden_dir, f"{name}.npz"))
    active = z["active"] if z["active"].size else None
    return z, active, tuple(bool(p) for p in z["periodic"])


@pytest.mark.parametrize("sname", sorted(cases_def.SCHEMES))
@pytest.mark.parametrize("name", cases_def.SCHEME_CASES)
def test_scheme_bitwise_vs_reference_fixtures(golden_dir, sname, name):
    z, active, periodic = fixture(golden_dir, f"scheme_{sname}_{name}")
    out = run(z["U0"], float(z["h"]), float(z["dt"]), int(z["steps"]), periodic, active, SCHEME_OPS[sname]())
    assert np.array_equal(out, z["out"]), (sname, name, np.abs(out - z["out"]).max())


@pytest.mark.parametrize("name", cases_def.FULL)
def test_ausmplus_through_functor_kernel_bitwise(golden_dir, name):
    z, active, periodic = fixture(golden_dir, name)
    out = run(z["U0"], float(z["h"]), float(z["dt"]), int(z["steps"]), periodic, active, AusmPlus(functor=True))
    assert np.array_equal(out, z["out"]), (name, np.abs(out - z["out"]).max())


@pytest.mark.parametrize("sname", sorted(cases_def.SCHEMES))
def test_scheme_grid_with_every_patch_face_kind(golden_dir, sname):
    z = np.load(os.path.join(golden_dir, f"grid_bc_box_{sname}.npz"))
    it, objs, _, dt, steps = make_grid("bc_box", DN_FP64, op=SCHEME_OPS[sname]())
    for _ in range(steps):
        it.rkStep(dt, cases.RK3_ALPHA)
    it.updateHost(fields=(0,))
    it.close()
    for p, cp in enumerate(objs):
        ref = z[f"p{p}_out"]
        assert np.array_equal(cp.getField(0), ref), (sname, p, np.abs(cp.getField(0) - ref).max())


@pytest.mark.parametrize("sname", sorted(cases_def.SCHEMES))
def test_scheme_graph_and_stagewise_equal_fused(golden_dir, sname):
    z, active, periodic = fixture(golden_dir, f"scheme_{sname}_vortex_16")
    args = (z["U0"], float(z["h"]), float(z["dt"]), int(z["steps"]), periodic, active, SCHEME_OPS[sname]())
    ref = z["out"]
    assert np.array_equal(run(*args, graph=True), ref)
    assert np.array_equal(run(*args, stagewise=True), ref)


def test_scheme_needs_fp64():
    with pytest.raises(DnError):
        B200CartesianIterator(VanLeer(), 0, DN_FP32)
    it = B200CartesianIterator(AusmPlus(), 0, DN_FP32)
    with pytest.raises(DnError):
        it.setFluxScheme(Roe())
    it.close()


def rusanov_numpy(U0, h, dt, steps, alpha=cases.RK3_ALPHA):
    """First-order Rusanov flux on a periodic patch, RK as the reference's
    RungeKutta (numpy, for the example stage function)."""
    R, gam, cv = 287.2, 1.4, 717.5

    def flux(U, d):
        ir = 1.0 / U[0]
        vel = U[1:4] * ir
        T = (U[4] * ir - 0.5 * (vel ** 2).sum(axis=0)) / cv
        p = U[0] * R * T
        un = vel[d]
        F = np.empty_like(U)
        F[0] = U[0] * un
        for c in range(3):
            F[1 + c] = U[1 + c] * un + (p if c == d else 0.0)
        F[4] = (U[4] + p) * un
        return F, np.abs(un) + np.sqrt(gam * R * T)

    def residual(U):
        res = np.zeros_like(U)
        for d in range(3):
            UL = np.roll(U, 1, axis=1 + d)       # cell below the face
            FL, sl = flux(UL, d)
            FR, sr = flux(U, d)
            Ff = h * h * (0.5 * (FL + FR) - 0.5 * np.maximum(sl, sr) * (U - UL))
            res += Ff - np.roll(Ff, -1, axis=1 + d)
        return res

    U = U0.copy()
    for _ in range(steps):
        Un = U.copy()
        for a in alpha:
            U = Un + a * dt / h ** 3 * residual(U)
    return U


def test_user_stage_function_example():
    assert os.path.exists(EXAMPLE_LIB), "example stage library missing: run python -m drnum_b200.build"
    ex = ctypes.CDLL(EXAMPLE_LIB)
    fn = ctypes.cast(ex.dn_example_rusanov_stage, ctypes.c_void_p).value
    U0 = cases.random_state(8, 6, 7, seed=11, amp=0.02, mach=0.4)
    h = 1.0 / 16
    dt = cases.cfl_dt(U0, h, 0.4)
    steps = 2
    patch = CartesianPatch(8, 6, 7, spacing=(h, h, h), periodic=(True, True, True))
    patch.setField(0, U0)
    it = B200CartesianIterator(AusmPlus(), 0, DN_FP64)
    it.addPatch(patch)
    it.updateDevice(fields=(0,))
    calls = ctypes.c_longlong(0)
    it.setStageFunction(fn, ctypes.addressof(calls))
    for _ in range(steps):
        it.rkStep(dt, cases.RK3_ALPHA)
    it.updateHost(fields=(0,))
    assert calls.value == 3 * steps
    out = patch.getField(0).copy()
    ref = rusanov_numpy(U0, h, dt, steps)
    scale = np.abs(U0).reshape(5, -1).max(axis=1)[:, None, None, None]
    assert np.abs(out - ref).max() / 1.0 < 1e-11 * max(1.0, float(scale.max()))
    assert (np.abs(out - ref) / scale).max() < 1e-12
    # None restores the built-in scheme
    it.setStageFunction(None)
    it.rkStep(dt, cases.RK3_ALPHA)
    it.close()


# ---------------------------------------------------------- the reference's own functors
REF_PLUGIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                          "libref_functor_stage.so")
needs_ref_plugin = pytest.mark.skipif(not os.path.exists(REF_PLUGIN),
                                      reason="reference functor plugin (oracle/build_ref.sh) not built")


def run_stage_fn(z, fn_name):
    lib = ctypes.CDLL(REF_PLUGIN)
    fn = ctypes.cast(getattr(lib, fn_name), ctypes.c_void_p).value
    U0 = z["U0"]
    _, ni, nj, nk = U0.shape
    h = float(z["h"])
    patch = CartesianPatch(ni, nj, nk, spacing=(h, h, h), periodic=tuple(bool(p) for p in z["periodic"]))
    patch.setField(0, U0)
    if z["active"].size:
        patch.active[...] = z["active"]
    it = B200CartesianIterator(AusmPlus(), 0, DN_FP64)
    it.addPatch(patch)
    it.updateDevice(fields=(0,))
    it.setStageFunction(fn)
    for _ in range(int(z["steps"])):
        it.rkStep(float(z["dt"]), cases.RK3_ALPHA)
    it.updateHost(fields=(0,))
    it.close()
    return patch.getField(0).copy()


@needs_ref_plugin
@pytest.mark.parametrize("name", cases_def.SCHEME_CASES)
def test_reference_vanleer_functor_compiled_for_the_device_is_bitwise(golden_dir, name):
    # DrNUM's own VanLeer<5, Upwind2<5, VanAlbada>, PerfectGas> source, compiled
    # against the device patch view, on the generic stage
    z = np.load(os.path.join(golden_dir, f"scheme_vanleer_{name}.npz"))
    out = run_stage_fn(z, "dnref_stage_vanleer")
    assert np.array_equal(out, z["out"]), (name, np.abs(out - z["out"]).max())


@needs_ref_plugin
@pytest.mark.parametrize("name", cases_def.VISC_CASES)
def test_reference_viscous_jet_functors_compiled_for_the_device(golden_dir, name):
    # VanLeer + CompressibleViscFlux (the field fluxes of the jet application):
    # the viscosity law calls pow, whose device and host versions may differ in
    # the last bit, so the bound is the reference's 1e-12 relative to each
    # variable's magnitude instead of bit equality
    z = np.load(os.path.join(golden_dir, f"visc_{name}.npz"))
    out = run_stage_fn(z, "dnref_stage_vanleer_visc")
    scale = np.abs(z["out"]).reshape(5, -1).max(axis=1)[:, None, None, None]
    rel = (np.abs(out - z["out"]) / scale).max()
    assert rel < 1e-12, (name, rel)
    # and the viscous terms are really there: the inviscid functor differs
    inviscid = run_stage_fn(z, "dnref_stage_vanleer")
    assert (np.abs(inviscid - z["out"]) / scale).max() > 1e-9


@needs_ref_plugin
@pytest.mark.parametrize("name", cases_def.SMAG_CASES)
def test_reference_smagorinsky_baseflow_functors_compiled_for_the_device(golden_dir, name):
    # Roe + CompressibleSmagorinskyFlux<5, 2400> (the field fluxes of the
    # base-flow application): the eddy viscosity takes a square root and the
    # viscosity law calls pow, so the bound is 1e-12 relative to each
    # variable's magnitude, as for the jet functors
    z = np.load(os.path.join(golden_dir, f"smag_{name}.npz"))
    out = run_stage_fn(z, "dnref_stage_roe_smag")
    scale = np.abs(z["out"]).reshape(5, -1).max(axis=1)[:, None, None, None]
    rel = (np.abs(out - z["out"]) / scale).max()
    assert rel < 1e-12, (name, rel)
    inviscid = run_stage_fn(z, "dnref_stage_roe")
    assert (np.abs(inviscid - z["out"]) / scale).max() > 1e-9
