"""A DrNUM application, unchanged in its run() structure, on drnum_b200: the
reference's own PatchGrid, computeDependencies and RungeKutta drive the
library through the C++ binding include/drnum_b200_iterator.h
(B200_CartesianIterator in place of GPU_CartesianIterator, B200_LevelSetBC in
place of CPU_LevelSetObjectBC).  FP64 results must equal the reference's
golden fixtures bit for bit."""
import hashlib
import json
import os

import numpy as np
import pytest

import cases_def
import pyoracle
import refapp
from drnum_b200 import cases

needs_app = pytest.mark.skipif(not refapp.available(), reason="oracle/_ref/libdrnum_refapp.so not built")


def _fixture(golden_dir, name):
    return np.load(os.path.join(golden_dir, f"{name}.npz"))


@needs_app
def test_binding_reports_errors_instead_of_exiting():
    # without a usable GPU the context cannot be created: the binding throws,
    # the application gets the library's message (the reference would exit)
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    U0, h, dt = cases.periodic_box(8)
    with pytest.raises(refapp.AppError) as e:
        refapp.run_single(U0, h, dt, 1)
    assert "drnum_b200" in str(e.value)


@pytest.mark.gpu
@needs_app
def test_cfg1_64cube_100_steps_through_reference_rungekutta(golden_dir):
    meta = json.load(open(os.path.join(golden_dir, "digests.json")))["cfg1_64_100"]
    c = cases_def.build("cfg1_64_100")
    out = refapp.run_single(np.ascontiguousarray(c["U0"]), c["h"], c["dt"], c["steps"])
    assert hashlib.sha256(np.ascontiguousarray(out).tobytes()).hexdigest() == meta["output_sha256"]


@pytest.mark.gpu
@needs_app
@pytest.mark.parametrize("name", cases_def.FULL)
def test_single_patch_fixtures_through_reference_rungekutta(golden_dir, name):
    z = _fixture(golden_dir, name)
    active = z["active"] if z["active"].size else None
    out = refapp.run_single(z["U0"], float(z["h"]), float(z["dt"]), int(z["steps"]),
                            tuple(bool(p) for p in z["periodic"]), active)
    assert np.array_equal(out, z["out"]), (name, np.abs(out - z["out"]).max())


@pytest.mark.gpu
@needs_app
@pytest.mark.parametrize("sname", sorted(cases_def.SCHEMES))
@pytest.mark.parametrize("name", ["vortex_16", "closed_10x7x12"])
def test_vanleer_and_roe_functors_through_reference_rungekutta(golden_dir, sname, name):
    z = _fixture(golden_dir, f"scheme_{sname}_{name}")
    active = z["active"] if z["active"].size else None
    out = refapp.run_single(z["U0"], float(z["h"]), float(z["dt"]), int(z["steps"]),
                            tuple(bool(p) for p in z["periodic"]), active, scheme=cases_def.SCHEMES[sname])
    assert np.array_equal(out, z["out"]), (sname, name, np.abs(out - z["out"]).max())


@pytest.mark.gpu
@needs_app
@pytest.mark.parametrize("name", sorted(cases_def.GRID_STEPS))
def test_patch_grids_through_reference_rungekutta(golden_dir, name):
    # octant grids, the jet grid (far field + inflow), the box with every
    # boundary kind, the sphere walls (B200_LevelSetBC post-operation)
    z = _fixture(golden_dir, f"grid_{name}")
    patches, states, _, dt, steps = cases_def.grid_case(name)
    G = cases_def.grid_levelset(name)
    ls = (cases_def.LS_INNER, cases_def.LS_OUTER, cases_def.LS_MIN_REL)
    outs = refapp.run_grid(patches, states, dt, steps, cases_def.grid_bcs(name), G=G, ls=ls)
    for p in range(len(patches)):
        assert np.array_equal(outs[p], z[f"p{p}_out"]), (name, p, np.abs(outs[p] - z[f"p{p}_out"]).max())


@pytest.mark.gpu
@needs_app
@pytest.mark.skipif(not pyoracle.ref_available(), reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("off", [1, 5])
def test_deactivated_patch_equals_reference_iterator(off):
    # PatchIterator::deactivatePatch: the patch is left out of every stage,
    # donor copies still write its receiving cells; against the reference's
    # CPU iterator with the same patch deactivated
    patches, states, _, dt, _ = cases_def.grid_case("octants_8")
    steps = 3
    ref = pyoracle.RefGrid(patches)
    for p, U in enumerate(states):
        ref.set_state(p, U)
    ref.deactivate(off)
    ref.run(steps, dt)
    want = [ref.get_state(p) for p in range(len(patches))]
    ref.close()
    inactive = [1 if p == off else 0 for p in range(len(patches))]
    outs = refapp.run_grid(patches, states, dt, steps, inactive=inactive)
    for p in range(len(patches)):
        assert np.array_equal(outs[p], want[p]), (off, p, np.abs(outs[p] - want[p]).max())
    assert not np.array_equal(outs[off], states[off])       # its receiving cells moved


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_compute_of_a_patch_subset(precision):
    # PatchIterator::compute(factor, patches): the listed patches advance as in
    # computeAll, the others keep their state
    from test_gpu_grid import make_grid
    sub = [0, 2, 5]
    full, objs_f, _, dt, _ = make_grid("octants_8", precision)
    part, objs_p, _, _, _ = make_grid("octants_8", precision)
    part.updateHost(fields=(0,))
    before = [o.getField(0).copy() for o in objs_p]
    for it in (full, part):
        it.copyField(0, 1)
    full.compute(0.25 * dt)
    part.compute(0.25 * dt, sub)
    full.updateHost(fields=(0,))
    part.updateHost(fields=(0,))
    for p in range(len(objs_f)):
        want = objs_f[p].getField(0) if p in sub else before[p]
        assert np.array_equal(objs_p[p].getField(0), want), p
    for it in (full, part):
        it.close()
