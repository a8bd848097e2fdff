"""Batched stage launch, CUDA-graph replay and the tile autotuner on the GPU:
every form must give the same bits as the per-patch launches."""
import numpy as np
import pytest

import cases_def
from drnum_b200 import _lib, cases
from drnum_b200._lib import DN_FP32, DN_FP64, DN_OPT_BATCHED, DN_OPT_GRAPH
from test_gpu_grid import make_grid

pytestmark = pytest.mark.gpu


def _run(name, precision, steps, batched=1, graph=0, shapes=None, autotune=False, dt_scale=None):
    it, objs, _, dt, _ = make_grid(name, precision)
    it.setOption(DN_OPT_BATCHED, batched)
    it.setOption(DN_OPT_GRAPH, graph)
    if shapes is not None:
        for p in range(len(objs)):
            it.setTile(p, shapes[p % len(shapes)])
    if autotune:
        cost = it.autotune()
        assert np.all(cost > 0)
    for s in range(steps):
        d = dt * (dt_scale[s] if dt_scale else 1.0)
        it.rkStep(d, cases.RK3_ALPHA)
    it.updateHost(fields=(0,))
    launches = it.launchCount()
    it.close()
    return [cp.getField(0).copy() for cp in objs], launches


@pytest.mark.parametrize("precision", [DN_FP64, DN_FP32])
@pytest.mark.parametrize("name", ["octants_jet", "sphere_pair"])
def test_batched_equals_per_patch(name, precision):
    a, _ = _run(name, precision, 4, batched=0)
    b, _ = _run(name, precision, 4, batched=1)
    c, _ = _run(name, precision, 4, batched=1, shapes=[1, 0])
    for x, y, z in zip(a, b, c):
        assert np.array_equal(x, y) and np.array_equal(x, z)


@pytest.mark.parametrize("precision", [DN_FP64, DN_FP32])
def test_graph_replay_equals_launches(precision):
    # 7 steps: every buffer rotation is replayed at least twice; dt changes once
    scale = [1, 1, 1, 1, 0.5, 0.5, 1]
    a, la = _run("sphere_pair", precision, 7, graph=0, dt_scale=scale)
    b, lb = _run("sphere_pair", precision, 7, graph=1, dt_scale=scale)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert la == lb     # the graph replays exactly the kernels the plain path launches


def test_autotuned_shapes_give_the_same_result(tmp_path):
    a, _ = _run("octants_jet", DN_FP32, 3)
    b, _ = _run("octants_jet", DN_FP32, 3, autotune=True)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_autotune_cache_is_reused(tmp_path):
    path = tmp_path / "tune.txt"
    it, objs, _, _, _ = make_grid("octants_8", DN_FP64)
    c1 = it.autotune(path)
    c2 = it.autotune(path)                 # read back, no new measurement
    it.close()
    assert np.array_equal(c1, c2)
    assert len(path.read_text().strip().splitlines()) == 1


@pytest.mark.parametrize("precision", [DN_FP64, DN_FP32])
def test_runs_are_deterministic(precision):
    # the same case twice on fresh contexts: bit-identical states (owner-computes
    # residuals, no atomics on the state, fixed summation orders)
    a, _ = _run("bc_box", precision, 5, graph=1)
    b, _ = _run("bc_box", precision, 5, graph=1)
    c, _ = _run("octants_jet", precision, 3)
    d, _ = _run("octants_jet", precision, 3)
    for x, y in zip(a + c, b + d):
        assert np.array_equal(x, y)


def test_single_patch_chunk_autotune_changes_no_result():
    # the plane-chunk length the autotuner picks for a single-patch FP32
    # launch changes the CTA decomposition, not a bit of the result
    from drnum_b200.api import AusmPlus, B200CartesianIterator, CartesianPatch
    U0, h, dt = cases.periodic_box(48)
    outs = []
    for tune in (False, True):
        p = CartesianPatch(48, 48, 48, spacing=(h, h, h))
        p.setField(0, U0)
        it = B200CartesianIterator(AusmPlus(), 0, DN_FP32)
        it.addPatch(p)
        it.updateDevice(fields=(0,))
        if tune:
            it.autotune()
        for _ in range(3):
            it.rkStep(dt, cases.RK3_ALPHA)
        it.updateHost(fields=(0,))
        outs.append(p.getField(0).copy())
        it.close()
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("name", ["octants_jet", "sphere_pair"])
def test_batched_schedules_give_the_same_result(name):
    # one CTA per work item (items of 8 or 24 planes) and persistent CTAs
    # over balanced item ranges (1, 2 or 4 waves, every tile shape), FP32
    # bulk: the same bits as the per-patch launches
    def run(waves, min_planes, shapes=None):
        it, objs, _, dt, _ = make_grid(name, DN_FP32)
        it.setOption(_lib.DN_OPT_BATCH_WAVES, waves)
        it.setOption(_lib.DN_OPT_BATCH_MIN_PLANES, min_planes)
        if shapes is not None:
            for p in range(len(objs)):
                it.setTile(p, shapes[p % len(shapes)])
        for _ in range(3):
            it.rkStep(dt, cases.RK3_ALPHA)
        it.updateHost(fields=(0,))
        it.close()
        return [cp.getField(0).copy() for cp in objs]

    ref, _ = _run(name, DN_FP32, 3, batched=0)
    for waves, min_planes, shapes in [(0, 8, None), (0, 24, [2]), (1, 8, [2, 1]), (2, 8, [0]), (4, 8, [1, 2, 0])]:
        got = run(waves, min_planes, shapes)
        for x, y in zip(ref, got):
            assert np.array_equal(x, y), (waves, min_planes, shapes)


def test_schedule_options_are_checked():
    it, _, _, _, _ = make_grid("octants_jet", DN_FP32)
    lib = it.lib
    assert lib.dn_set_option(it.ctx, _lib.DN_OPT_BATCH_WAVES, -1) == _lib.DN_ERR_ARG
    assert lib.dn_set_option(it.ctx, _lib.DN_OPT_BATCH_MIN_PLANES, 0) == _lib.DN_ERR_ARG
    assert lib.dn_set_option(it.ctx, _lib.DN_OPT_BATCH_WAVES, 3) == _lib.DN_OK
    it.close()


@pytest.mark.parametrize("precision", [DN_FP64, DN_FP32])
@pytest.mark.parametrize("name", ["jet", "tiled"])
def test_donor_table_forms_give_the_same_result(name, precision):
    # interpolation patterns (the default) and per-contribution tables on
    # the dual-resolution jet (cells with donors in two or three patches)
    # and the uneven grid (zero weights), reduced: the same bits
    from drnum_b200 import workloads
    case = workloads.build(name, 0.25)

    def run(form):
        _, objs = workloads.make_grid(case)
        it = workloads.make_iterator(objs, precision, 0)
        it.setOption(_lib.DN_OPT_DONOR_TABLES, form)
        for _ in range(2):
            it.rkStep(case["dt"], cases.RK3_ALPHA)
        out = [it.downloadField(q, 0) for q in range(len(objs))]
        it.close()
        return out

    a, b = run(0), run(1)
    for q, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x, y), q


def test_donor_table_option_is_checked():
    it, _, _, _, _ = make_grid("octants_8", DN_FP32)
    assert it.lib.dn_set_option(it.ctx, _lib.DN_OPT_DONOR_TABLES, 2) == _lib.DN_ERR_ARG
    assert it.lib.dn_set_option(it.ctx, _lib.DN_OPT_DONOR_TABLES, 1) == _lib.DN_OK
    it.close()


@pytest.mark.parametrize("name", ["tiled", "jet"])
def test_batched_workload_equals_per_patch(name):
    # reduced workloads, FP32 bulk (ragged tiles, patch faces, overlaps):
    # the batched launches give the bits of one launch per patch
    from drnum_b200 import workloads
    case = workloads.build(name, 0.25)

    def run(batched, shape=None):
        _, objs = workloads.make_grid(case)
        it = workloads.make_iterator(objs, DN_FP32, 0)
        it.setOption(DN_OPT_BATCHED, batched)
        if shape is not None:
            # 16 x 32 tiles: the batched launches cover short remainders of
            # closed axes with 16 x 16 and 8 x 32 tiles
            for q in range(len(objs)):
                it.setTile(q, shape)
        for _ in range(2):
            it.rkStep(case["dt"], cases.RK3_ALPHA)
        out = [it.downloadField(q, 0) for q in range(len(objs))]
        it.close()
        return out

    a, b, c = run(0), run(1), run(1, 2)
    for q, (x, y, z) in enumerate(zip(a, b, c)):
        assert np.array_equal(x, y) and np.array_equal(x, z), q
