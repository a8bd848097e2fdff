"""Overlap set-up (donor tables) and the oracle's multi-patch step against the
reference (CPU only).

The fixtures tests/golden/grid_*.npz hold the reference's own donor tables
(PatchGrid::computeDependencies, patchgrid.cpp:119-268) and, for the octant
grids, its multi-patch RK steps; they are generated from the compiled
reference by tests/golden/make_golden.py --grids.
"""
import ctypes
import os

import numpy as np
import pytest

import cases_def
import pyoracle
from drnum_b200 import _lib, cases

TABLE_KEYS = ("rec_unique", "donor_patch", "num_receivers", "stride", "rec_concat", "donor_idx", "weight")


def _descs(patches, add_protect=0):
    arr = (_lib.dn_patch_desc * len(patches))()
    for d, p in zip(arr, patches):
        d.ni, d.nj, d.nk = p["n"]
        for a in range(3):
            d.face[a] = _lib.DN_FACE_CLOSED
            d.origin[a] = p["origin"][a]
            d.length[a] = p["length"][a]
        for a in range(6):
            d.seek[a] = p["seek"][a]
        d.add_protect = add_protect
    return arr


def build_tables(patches, add_protect=0):
    lib = _lib.load()
    h = ctypes.c_void_p()
    nd = ctypes.c_int64()
    rc = lib.dn_overlap_build(_descs(patches, add_protect), len(patches), ctypes.byref(h), ctypes.byref(nd))
    assert rc == _lib.DN_OK
    try:
        return [_lib.read_donor_tables(lib.dn_overlap_counts, lib.dn_overlap_get, h, p)
                for p in range(len(patches))], nd.value
    finally:
        lib.dn_overlap_destroy(h)


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype == np.float64:
        return np.array_equal(a.view(np.uint64), b.view(np.uint64))   # bit for bit
    return np.array_equal(a, b)


def _fixture(golden_dir, name):
    return np.load(os.path.join(golden_dir, f"grid_{name}.npz"))


@pytest.mark.parametrize("name", cases_def.GRID_TABLES)
def test_donor_tables_equal_reference_fixtures(golden_dir, name):
    z = _fixture(golden_dir, name)
    patches = cases_def.grid_layout(name)
    mine, _ = build_tables(patches, cases_def.GRID_ADD_PROTECT.get(name, 0))
    for p in range(len(patches)):
        for k in TABLE_KEYS + ("counts",):
            assert _same(mine[p][k], z[f"p{p}_{k}"]), (name, p, k)


@pytest.mark.skipif(not pyoracle.ref_available(), reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("seed", [11, 12, 13])
def test_donor_tables_equal_live_reference(seed):
    rng = np.random.default_rng(seed)
    patches = []
    for p in range(5):
        n = tuple(int(x) for x in rng.integers(8, 16, 3))
        h = float(rng.choice([0.1, 0.05, 0.025]))
        seek = tuple(int(x) for x in rng.integers(0, 3, 6))
        patches.append(dict(n=n, origin=tuple(float(x) for x in rng.uniform(0, 0.5, 3)),
                            length=tuple(h * x for x in n), seek=seek))
    ref = pyoracle.RefGrid(patches, 0)
    mine, _ = build_tables(patches)
    for p in range(len(patches)):
        t = ref.tables(p)
        for k in TABLE_KEYS:
            assert _same(mine[p][k], t[k]), (seed, p, k)


@pytest.mark.parametrize("name", ["octants_8", "octants_ragged"])
def test_octant_grids_leave_no_seek_cell_without_donor(name):
    _, nd = build_tables(cases_def.grid_layout(name))
    assert nd == 0


@pytest.mark.parametrize("name", sorted(cases_def.GRID_STEPS))
def test_oracle_grid_steps_equal_reference(golden_dir, name):
    z = _fixture(golden_dir, name)
    patches, states, spacings, dt, steps = cases_def.grid_case(name)
    assert float(z["dt"]) == dt and int(z["steps"]) == steps
    tables = [{k: z[f"p{p}_{k}"] for k in TABLE_KEYS} for p in range(len(patches))]
    layers = _ls_tables(z, name, len(patches)) if name in cases_def.LEVELSET else None
    out = pyoracle.oracle_grid_run(states, spacings, tables, dt, steps, cases_def.ALPHA, cases_def.grid_bcs(name),
                                   layers)
    for p in range(len(patches)):
        assert np.array_equal(out[p], z[f"p{p}_out"]), (name, p, np.abs(out[p] - z[f"p{p}_out"]).max())


def test_oracle_donor_copy_detects_planted_weight_error(golden_dir):
    # a weight changed in the oracle's tables changes the interpolated cells
    z = _fixture(golden_dir, "octants_8")
    patches, states, _, _, _ = cases_def.grid_case("octants_8")
    tables = [{k: z[f"p{p}_{k}"].copy() for k in TABLE_KEYS} for p in range(len(patches))]
    a = [s.copy() for s in states]
    pyoracle.oracle_donor_copy(a, tables)
    tables[0]["weight"][0] *= 1.0 + 1e-9
    b = [s.copy() for s in states]
    pyoracle.oracle_donor_copy(b, tables)
    assert not np.array_equal(a[0], b[0])


def test_degenerate_donor_zone_is_reported():
    # a donor zone one cell wide: the reference stops with a BUG
    # (cartesianpatch.cpp:1146-1151); the set-up returns an error instead
    patches = [dict(n=(6, 6, 6), origin=(0.0, 0.0, 0.0), length=(0.6, 0.6, 0.6), seek=(2, 2, 2, 2, 2, 2)),
               dict(n=(6, 6, 6), origin=(0.15, 0.15, 0.15), length=(0.6, 0.6, 0.6), seek=(2, 2, 2, 2, 2, 2))]
    lib = _lib.load()
    h = ctypes.c_void_p()
    rc = lib.dn_overlap_build(_descs(patches, 1), 2, ctypes.byref(h), None)
    assert rc == _lib.DN_ERR_ARG and not h.value


def test_overlap_build_rejects_invalid_layouts():
    lib = _lib.load()
    h = ctypes.c_void_p()
    bad = [dict(n=(4, 4, 4), origin=(0.0, 0.0, 0.0), length=(0.4, 0.4, 0.4), seek=(3, 3, 0, 0, 0, 0))]
    assert lib.dn_overlap_build(_descs(bad), 1, ctypes.byref(h), None) == _lib.DN_ERR_ARG
    assert lib.dn_overlap_build(None, 1, ctypes.byref(h), None) == _lib.DN_ERR_ARG
    assert lib.dn_overlap_build(_descs(bad), 0, ctypes.byref(h), None) == _lib.DN_ERR_ARG
    assert lib.dn_overlap_counts(None, 0, None) == _lib.DN_ERR_ARG


# ------------------------------------------------------------------ level sets

LS_KEYS = ("cells", "g", "grad", "donors", "weights")


def classify(patch, G, num_inner, num_outer, min_rel):
    lib = _lib.load()
    h = ctypes.c_void_p()
    rc = lib.dn_levelset_classify(ctypes.byref(_descs([patch])[0]), _lib.dptr(np.ascontiguousarray(G)),
                                  num_inner, num_outer, min_rel, ctypes.byref(h))
    assert rc == _lib.DN_OK
    try:
        return _lib.read_levelset_layers(lib.dn_lslayers_count, lib.dn_lslayers_get, h, (), num_inner, num_outer)
    finally:
        lib.dn_lslayers_destroy(h)


@pytest.mark.parametrize("name", sorted(cases_def.LEVELSET))
def test_levelset_layers_equal_reference_fixtures(golden_dir, name):
    z = _fixture(golden_dir, name)
    patches = cases_def.grid_layout(name)
    for p, G in enumerate(cases_def.grid_levelset(name)):
        L = classify(patches[p], G, cases_def.LS_INNER, cases_def.LS_OUTER, cases_def.LS_MIN_REL)
        for layer in range(cases_def.LS_INNER):
            for k in LS_KEYS:
                assert _same(L["inner"][layer][k], z[f"p{p}_ls{layer}_{k}"]), (name, p, layer, k)


@pytest.mark.skipif(not pyoracle.ref_available(), reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("seed", [21, 22, 23, 24])
def test_levelset_layers_equal_live_reference(seed):
    # random spheres, layer counts, replacement distances, inner and outer layers
    rng = np.random.default_rng(seed)
    n = tuple(int(x) for x in rng.integers(12, 20, 3))
    patch = dict(n=n, origin=(0.0, 0.0, 0.0), length=tuple(x / 16 for x in n), seek=(0, 0, 0, 0, 0, 0))
    centre = tuple(float(x) for x in rng.uniform(0.3, 0.5, 3))
    G = cases.sphere_sdf(patch, centre, float(rng.uniform(0.15, 0.3)), fp32=bool(seed % 2))
    ni, no, mr = int(rng.integers(1, 4)), int(rng.integers(0, 3)), float(rng.choice([0.0, 0.1, 0.4]))
    ref = pyoracle.RefGrid([patch], num_vars=6)
    ref.levelset([G], ni, no, mr)
    mine = classify(patch, G, ni, no, mr)
    for inner, num in ((1, ni), (0, no)):
        for layer in range(num):
            r = ref.levelset_layer(0, inner, layer)
            m = mine["inner" if inner else "outer"][layer]
            for k in LS_KEYS:
                if not inner and k in ("donors", "weights"):
                    continue
                assert _same(m[k], r[k]), (seed, inner, layer, k)


def test_levelset_classify_rejects_invalid_input():
    lib = _lib.load()
    patch = dict(n=(8, 8, 8), origin=(0.0, 0.0, 0.0), length=(0.5, 0.5, 0.5), seek=(0, 0, 0, 0, 0, 0))
    G = cases.sphere_sdf(patch, (0.25, 0.25, 0.25), 0.1)
    h = ctypes.c_void_p()
    d = _descs([patch])[0]
    assert lib.dn_levelset_classify(ctypes.byref(d), None, 3, 0, 0.1, ctypes.byref(h)) == _lib.DN_ERR_ARG
    assert lib.dn_levelset_classify(ctypes.byref(d), _lib.dptr(G), 0, 0, 0.1, ctypes.byref(h)) == _lib.DN_ERR_ARG
    assert lib.dn_levelset_classify(ctypes.byref(d), _lib.dptr(G), -1, 0, 0.0, ctypes.byref(h)) == _lib.DN_ERR_ARG


def _ls_tables(z, name, num_patches):
    out = []
    for p in range(num_patches):
        if f"p{p}_ls0_cells" not in z:
            out.append(None)
            continue
        out.append([{k: z[f"p{p}_ls{layer}_{k}"] for k in LS_KEYS} for layer in range(cases_def.LS_INNER)])
    return out


def test_overlap_setup_result_independent_of_thread_count(monkeypatch):
    # receiving patches are spread over host threads; the tables must not
    # depend on how many
    patches = cases.tiled_grid(slots=(3, 3, 2), seed=5)
    monkeypatch.setenv("DN_SETUP_THREADS", "1")
    one, nd1 = build_tables(patches)
    monkeypatch.setenv("DN_SETUP_THREADS", "5")
    many, nd5 = build_tables(patches)
    assert nd1 == nd5 == 0
    for a, b in zip(one, many):
        for k in TABLE_KEYS:
            assert _same(a[k], b[k]), k


# ------------------------------------------------- full-size benchmark layouts

@pytest.mark.skipif(not pyoracle.ref_available(), reason="compiled reference (oracle/_ref) not built")
def test_levelset_classification_full_size_sphere_group_equals_reference():
    # the level-set wall workload at its stated size: 256 x 128 x 128 cells in
    # two overlapping patches, sphere r = 0.08 at (0.3, 0.5, 0.5) as an FP32
    # distance field, 3 inner layers, min_inner_rel_dist 0.1: cell lists,
    # distances, gradients, mirror donors and weights bit for bit
    from drnum_b200 import workloads
    case = workloads.build("sphere")
    G, ni, no, mr = case["levelset"]
    assert [p["n"] for p in case["patches"]] == [(131, 128, 128), (131, 128, 128)]
    ref = pyoracle.RefGrid(case["patches"], num_vars=6)
    ref.levelset(G, ni, no, mr)
    total = 0
    for p, patch in enumerate(case["patches"]):
        mine = classify(patch, G[p], ni, no, mr)
        for layer in range(ni):
            r = ref.levelset_layer(p, 1, layer)
            m = mine["inner"][layer]
            total += len(m["cells"])
            for k in LS_KEYS:
                assert _same(m[k], r[k]), (p, layer, k)
    assert total > 1000
    ref.close()


@pytest.mark.skipif(not pyoracle.ref_available(), reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("name", ["jet", "tiled"])
def test_donor_tables_full_size_workloads_equal_reference(name):
    # the donor tables of the dual-resolution jet (8 patches, 10.9 M cells)
    # and of the 512-patch uneven grid (69.8 M cells) at their stated sizes,
    # against the reference's PatchGrid::computeDependencies, bit for bit
    from drnum_b200 import workloads
    patches = workloads.build(name)["patches"]
    mine, nd = build_tables(patches)
    assert nd == 0
    ref = pyoracle.RefGrid(patches, 0, threads=0)
    for p in range(len(patches)):
        t = ref.tables(p)
        for k in TABLE_KEYS:
            assert _same(mine[p][k], t[k]), (name, p, k)
    ref.close()
