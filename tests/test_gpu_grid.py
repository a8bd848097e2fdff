"""Multi-patch (overlap) path on the GPU through the C ABI: donor tables on
the context, the donor copy kernel and RK steps of a dual-resolution grid,
against the reference's own outputs (tests/golden/grid_*.npz) and the oracle."""
import ctypes
import os

import numpy as np
import pytest

import cases_def
import pyoracle
from drnum_b200 import _lib, cases
from drnum_b200._lib import DN_FP32, DN_FP64
from drnum_b200.api import (AusmPlus, B200CartesianIterator, B200LevelSetObjectBC, CartesianPatch, PatchGrid,
                            RungeKutta)

pytestmark = pytest.mark.gpu

TABLE_KEYS = ("rec_unique", "donor_patch", "num_receivers", "stride", "rec_concat", "donor_idx", "weight")
# FP32 bulk against FP64 on the grid: relative to the free-stream scale
F32_GRID_L2_TOL = 1e-5
F32_GRID_LINF_TOL = 1e-4


def _fixture(golden_dir, name):
    return np.load(os.path.join(golden_dir, f"grid_{name}.npz"))


def make_grid_objects(name, states=None):
    """The host patches of a grid case (fields, boundary fluxes, level sets)
    with their donor tables computed: (patches, dt, steps)."""
    patches, st0, spacings, dt, steps = cases_def.grid_case(name)
    states = st0 if states is None else states
    grid = PatchGrid()
    objs = []
    bcs = cases_def.grid_bcs(name) or {}
    G = cases_def.grid_levelset(name)
    for q, (p, U) in enumerate(zip(patches, states)):
        cp = CartesianPatch(*p["n"], lengths=p["length"], origin=p["origin"], periodic=(False, False, False),
                            seek=p["seek"])
        cp.setField(0, U)
        for side, (kind, params, table) in bcs.get(q, {}).items():
            cp.setBoundary(side, kind, params, table)
        if G is not None:
            cp.setLevelSet(G[q], cases_def.LS_INNER, cases_def.LS_OUTER, cases_def.LS_MIN_REL)
        grid.insertPatch(cp)
        objs.append(cp)
    grid.computeDependencies()
    return objs, dt, steps


def make_grid(name, precision, states=None, op=None, shadows=None):
    patches, st0, spacings, dt, steps = cases_def.grid_case(name)
    states = st0 if states is None else states
    grid = PatchGrid()
    objs = []
    bcs = cases_def.grid_bcs(name) or {}
    G = cases_def.grid_levelset(name)
    for q, (p, U) in enumerate(zip(patches, states)):
        cp = CartesianPatch(*p["n"], lengths=p["length"], origin=p["origin"], periodic=(False, False, False),
                            seek=p["seek"])
        cp.setField(0, U)
        for side, (kind, params, table) in bcs.get(q, {}).items():
            cp.setBoundary(side, kind, params, table)
        if G is not None:
            cp.setLevelSet(G[q], cases_def.LS_INNER, cases_def.LS_OUTER, cases_def.LS_MIN_REL)
        grid.insertPatch(cp)
        objs.append(cp)
    grid.computeDependencies()
    it = B200CartesianIterator(op if op is not None else AusmPlus(), 0, precision)
    for q, cp in enumerate(objs):
        it.addPatch(cp, shadow=bool(shadows and shadows[q]))
    it.updateDevice(fields=(0,))
    return it, objs, grid, dt, steps


@pytest.mark.parametrize("name", sorted(cases_def.GRID_STEPS))
def test_grid_fp64_bitwise_vs_reference(golden_dir, name):
    z = _fixture(golden_dir, name)
    it, objs, _, dt, steps = make_grid(name, DN_FP64)
    for _ in range(steps):
        it.rkStep(dt, cases.RK3_ALPHA)
    it.updateHost(fields=(0,))
    it.close()
    for p, cp in enumerate(objs):
        ref = z[f"p{p}_out"]
        assert np.array_equal(cp.getField(0), ref), (name, p, np.abs(cp.getField(0) - ref).max())


def test_context_tables_equal_reference(golden_dir):
    z = _fixture(golden_dir, "octants_ragged")
    it, objs, _, _, _ = make_grid("octants_ragged", DN_FP64)
    assert it.computeDependencies() == 0          # rebuilt on the context from the patch descriptions
    for p in range(len(objs)):
        t = it.donorTables(p)
        for k in TABLE_KEYS:
            a, b = t[k], z[f"p{p}_{k}"]
            if a.dtype == np.float64:
                a, b = a.view(np.uint64), b.view(np.uint64)
            assert np.array_equal(a, b), (p, k)
    it.close()


def test_donor_copy_matches_oracle():
    patches, _, _, _, _ = cases_def.grid_case("octants_8")
    rng = np.random.default_rng(7)
    states = [cases.random_state(*p["n"], seed=int(rng.integers(1 << 30)), amp=0.02) for p in patches]
    it, objs, grid, _, _ = make_grid("octants_8", DN_FP64, states)
    it.copyDonorData(0)
    it.updateHost(fields=(0,))
    it.close()
    expect = [s.copy() for s in states]
    pyoracle.oracle_donor_copy(expect, grid.tables)
    for p, cp in enumerate(objs):
        assert np.array_equal(cp.getField(0), expect[p]), p


def test_grid_stagewise_api_equals_fused_step(golden_dir):
    name = "octants_8"
    z = _fixture(golden_dir, name)
    it, objs, _, dt, steps = make_grid(name, DN_FP64)
    rk = RungeKutta()
    for a in cases.RK3_ALPHA:
        rk.addAlpha(a)
    rk.addIterator(it)
    rk.addPostOperation(lambda: None)    # forces the reference's stage-by-stage sequence
    for _ in range(steps):
        rk(dt)
    it.updateHost(fields=(0,))
    it.close()
    for p, cp in enumerate(objs):
        assert np.array_equal(cp.getField(0), z[f"p{p}_out"]), p


@pytest.mark.parametrize("name,steps", [("octants_ragged", 6), ("octants_jet", 30), ("sphere_pair", 30)])
def test_grid_fp32_against_fp64(name, steps):
    out = {}
    for prec in (DN_FP64, DN_FP32):
        it, objs, _, dt, _ = make_grid(name, prec)
        for _ in range(steps):
            it.rkStep(dt, cases.RK3_ALPHA)
        it.updateHost(fields=(0,))
        it.close()
        out[prec] = [cp.getField(0).copy() for cp in objs]
    scale = np.array([cases.RHO_INF, cases.RHO_INF * cases.A_INF, cases.RHO_INF * cases.A_INF,
                      cases.RHO_INF * cases.A_INF, cases.RHO_INF * cases.A_INF ** 2])[:, None, None, None]
    for a, b in zip(out[DN_FP32], out[DN_FP64]):
        d = (a - b) / scale
        l2 = np.sqrt((d ** 2).reshape(5, -1).mean(1))
        assert l2.max() < F32_GRID_L2_TOL, l2
        assert np.abs(d).max() < F32_GRID_LINF_TOL


def test_set_donors_rejects_invalid_tables(golden_dir):
    z = _fixture(golden_dir, "pair_x")
    patches = cases_def.grid_layout("pair_x")
    it = B200CartesianIterator(AusmPlus(), 0, DN_FP64)
    for p in patches:
        it.addPatch(CartesianPatch(*p["n"], lengths=p["length"], origin=p["origin"],
                                   periodic=(False, False, False), seek=p["seek"]))
    lib, ctx = it.lib, it.ctx

    def call(t):
        counts = np.ascontiguousarray(t["counts"], dtype=np.int64)
        arrs = [np.ascontiguousarray(t[k]) for k in TABLE_KEYS]
        types = [c for _, _, c, _ in _lib.DONOR_FIELDS]
        return lib.dn_patch_set_donors(ctx, 0, _lib.ptr(counts, ctypes.c_int64),
                                       *[_lib.ptr(a, ct) for a, ct in zip(arrs, types)])

    good = {k: z[f"p0_{k}"].copy() for k in TABLE_KEYS + ("counts",)}
    assert call(good) == _lib.DN_OK
    bad = {k: v.copy() for k, v in good.items()}
    bad["donor_patch"][0] = 0                      # a patch cannot be its own donor
    assert call(bad) == _lib.DN_ERR_ARG
    bad = {k: v.copy() for k, v in good.items()}
    bad["donor_idx"][0] = 10 ** 9                  # donor cell outside the donor patch
    assert call(bad) == _lib.DN_ERR_ARG
    bad = {k: v.copy() for k, v in good.items()}
    bad["rec_unique"] = bad["rec_unique"][::-1].copy()   # not ascending
    assert call(bad) == _lib.DN_ERR_ARG
    it.close()


def test_boundary_kinds_rejected_where_invalid():
    it = B200CartesianIterator(AusmPlus(), 0, DN_FP64)
    pid = it.addPatch(CartesianPatch(6, 6, 6, lengths=(1.0, 1.0, 1.0), periodic=(True, False, False)))
    lib, ctx = it.lib, it.ctx
    ff = np.array([1e5, 300.0, 10.0, 0.0, 0.0])
    assert lib.dn_patch_set_bc(ctx, pid, 0, _lib.DN_BC_FARFIELD, _lib.dptr(ff), None) == _lib.DN_ERR_ARG  # periodic axis
    assert lib.dn_patch_set_bc(ctx, pid, 2, 7, None, None) == _lib.DN_ERR_ARG                        # unknown kind
    assert lib.dn_patch_set_bc(ctx, pid, 6, _lib.DN_BC_SLIP, None, None) == _lib.DN_ERR_ARG           # no side 6
    assert lib.dn_patch_set_bc(ctx, pid, 2, _lib.DN_BC_INFLOW, None, None) == _lib.DN_ERR_ARG         # table missing
    bad = ff.copy()
    bad[1] = -1.0
    assert lib.dn_patch_set_bc(ctx, pid, 2, _lib.DN_BC_FARFIELD, _lib.dptr(bad), None) == _lib.DN_ERR_ARG
    assert lib.dn_patch_set_bc(ctx, pid, 3, _lib.DN_BC_FARFIELD, _lib.dptr(ff), None) == _lib.DN_OK
    it.close()


@pytest.mark.parametrize("name", sorted(cases_def.LEVELSET))
def test_context_levelset_layers_equal_reference(golden_dir, name):
    z = _fixture(golden_dir, name)
    it, objs, _, _, _ = make_grid(name, DN_FP64)
    for p in range(len(objs)):
        L = it.levelSetLayers(p)
        for layer in range(cases_def.LS_INNER):
            for k in ("cells", "g", "grad", "donors", "weights"):
                a, b = L["inner"][layer][k], z[f"p{p}_ls{layer}_{k}"]
                if a.dtype == np.float64:
                    a, b = a.view(np.uint64), b.view(np.uint64)
                assert np.array_equal(a, b), (name, p, layer, k)
    it.close()


def test_levelset_stagewise_post_operation_equals_fused_step(golden_dir):
    name = "sphere_pair"
    z = _fixture(golden_dir, name)
    it, objs, _, dt, steps = make_grid(name, DN_FP64)
    rk = RungeKutta()
    for a in cases.RK3_ALPHA:
        rk.addAlpha(a)
    rk.addIterator(it)
    rk.addPostOperation(B200LevelSetObjectBC(it))
    for _ in range(steps):
        rk(dt)
    it.updateHost(fields=(0,))
    it.close()
    for p, cp in enumerate(objs):
        assert np.array_equal(cp.getField(0), z[f"p{p}_out"]), p


@pytest.mark.parametrize("precision", [DN_FP64, DN_FP32])
@pytest.mark.parametrize("graph", [0, 1])
def test_step_start_donor_copy_left_out_only_while_current(precision, graph):
    """A step starts with a donor copy (rungekutta.cpp:30) unless the step-
    start buffer's receiving cells already hold it: the last step ended with
    a donor copy into that buffer and nothing has written it since.  An
    upload into field 0, or an upload into field 1 copied into field 0,
    makes the next step copy again, bit for bit like a fresh context."""
    name = "octants_8"
    patches = cases_def.grid_case(name)[0]
    garbage = [cases.random_state(*p["n"], seed=100 + q, amp=0.03) for q, p in enumerate(patches)]
    alpha = np.ascontiguousarray(cases.RK3_ALPHA, dtype=np.float64)

    def upload(it, field, states):
        for q, U in enumerate(states):
            a = np.ascontiguousarray(U, dtype=np.float64)
            _lib.check(it.ctx, it.lib.dn_patch_upload(it.ctx, q, field, _lib.dptr(a)))

    def fresh_step(states):
        # (the first upload fixes the FP32-bulk base and quantum of every patch)
        it, objs, _, dt, _ = make_grid(name, precision)
        it.setOption(_lib.DN_OPT_GRAPH, graph)
        upload(it, 0, states)
        it.rkStep(dt, alpha)
        out = [it.downloadField(q, 0) for q in range(len(objs))]
        it.close()
        return out

    expect = fresh_step(garbage)
    for route in ("upload", "copy"):
        it, objs, _, dt, _ = make_grid(name, precision)
        it.setOption(_lib.DN_OPT_GRAPH, graph)
        n = [it.launchCount()]
        for _ in range(3):
            it.rkStep(dt, alpha)
            n.append(it.launchCount())
        per_step = np.diff(n)
        assert per_step[1] == per_step[0] - 1 and per_step[2] == per_step[1], per_step
        if route == "upload":
            upload(it, 0, garbage)
        else:
            upload(it, 1, garbage)
            it.copyField(1, 0)
        it.rkStep(dt, alpha)
        got = [it.downloadField(q, 0) for q in range(len(objs))]
        it.close()
        for q, (a, b) in enumerate(zip(got, expect)):
            assert np.array_equal(a, b), (route, q)


def test_step_start_donor_copy_kept_when_donors_include_receiving_cells(golden_dir):
    # tables in which a donor cell of patch 1 is a receiving cell of patch 0:
    # a repeated donor copy would read what the last one wrote, so every
    # step keeps its step-start copy (with the reference's tables it is left
    # out from the second step on)
    z = _fixture(golden_dir, "pair_x")
    patches = cases_def.grid_layout("pair_x")
    alpha = np.ascontiguousarray(cases.RK3_ALPHA, dtype=np.float64)

    def launches_per_step(chain):
        it = B200CartesianIterator(AusmPlus(), 0, DN_FP64)
        for p in patches:
            cp = CartesianPatch(*p["n"], lengths=p["length"], origin=p["origin"],
                                periodic=(False, False, False), seek=p["seek"])
            cp.setField(0, cases.uniform_state([p], mach=0.3)[0])
            it.addPatch(cp)
        for q in range(2):
            t = {k: z[f"p{q}_{k}"].copy() for k in TABLE_KEYS + ("counts",)}
            if chain and q == 1:
                assert int(t["donor_patch"][0]) == 0
                t["donor_idx"][0] = z["p0_rec_unique"][0]
            it.setDonorTablesOf(q, t)
        it.updateDevice(fields=(0,))
        n = [it.launchCount()]
        for _ in range(3):
            it.rkStep(1e-6, alpha)
            n.append(it.launchCount())
        it.close()
        return np.diff(n)

    plain = launches_per_step(False)
    assert plain[1] == plain[0] - 1 and plain[2] == plain[1], plain
    chained = launches_per_step(True)
    assert chained[0] == chained[1] == chained[2] == plain[0], chained


@pytest.mark.parametrize("precision", [DN_FP64, DN_FP32])
@pytest.mark.parametrize("graph", [0, 1])
def test_donor_copies_after_a_wall_away_from_the_overlap_left_out(precision, graph):
    # the reduced sphere workload: the level-set wall writes no donor and no
    # receiving cell, so the donor copies that follow it (before the next
    # stage and at the next step's start) would rewrite the same bits and are
    # left out; the reference's stage-by-stage sequence with the wall as a
    # post-operation (every copy made) gives the same result
    from drnum_b200 import workloads
    case = workloads.build("sphere", 0.25)
    alpha = np.ascontiguousarray(cases.RK3_ALPHA, dtype=np.float64)

    def fused():
        _, objs = workloads.make_grid(case)
        it = workloads.make_iterator(objs, precision, 0)
        it.setOption(_lib.DN_OPT_GRAPH, graph)
        n = [it.launchCount()]
        for _ in range(3):
            it.rkStep(case["dt"], alpha)
            n.append(it.launchCount())
        out = [it.downloadField(q, 0) for q in range(len(objs))]
        it.close()
        return out, np.diff(n)

    def stagewise():
        _, objs = workloads.make_grid(case)
        it = workloads.make_iterator(objs, precision, 0)
        rk = RungeKutta()
        for a in cases.RK3_ALPHA:
            rk.addAlpha(a)
        rk.addIterator(it)
        rk.addPostOperation(B200LevelSetObjectBC(it))
        n = [it.launchCount()]
        for _ in range(3):
            rk(case["dt"])
            n.append(it.launchCount())
        out = [it.downloadField(q, 0) for q in range(len(objs))]
        it.close()
        return out, np.diff(n)

    a, na = fused()
    b, nb = stagewise()
    for q, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x, y), q
    # per step the stage-by-stage sequence makes 6 donor copies (one before
    # and one after every stage); the fused step 4 in its first step (the
    # step-start copy, one after every stage) and 3 from then on
    assert na[0] == nb[0] - 2 and na[1] == na[2] == nb[1] - 3, (na, nb)
