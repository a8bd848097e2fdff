"""The multi-patch benchmark workloads: layouts are consistent on the CPU,
and on the GPU the FP32 bulk form tracks plain FP64 at reduced scale."""
import numpy as np
import pytest

from drnum_b200 import _lib, cases, workloads
from test_overlap import build_tables


@pytest.mark.parametrize("name", workloads.NAMES)
def test_workload_layouts_have_donors_for_every_seek_cell(name):
    case = workloads.build(name, scale=0.25)
    _, no_donor = build_tables(case["patches"])
    assert no_donor == 0
    assert len(case["states"]) == len(case["patches"])
    for p, U in zip(case["patches"], case["states"]):
        assert U.shape == (5,) + tuple(p["n"]) and np.isfinite(U).all()


def test_tiled_workload_full_size_layout():
    # 512 patches; per-axis extents drawn from the even numbers of 16..96
    # cells at the fine spacing (refinement 2), half as many at refinement 1
    patches = cases.tiled_grid()
    cells = sum(int(np.prod(p["n"])) for p in patches)
    assert len(patches) == 512 and 60e6 < cells < 80e6
    assert {p["refinement"] for p in patches} == {1, 2}
    for p in patches:
        inner = [p["n"][a] - 2 * ((p["seek"][2 * a] > 0) + (p["seek"][2 * a + 1] > 0)) for a in range(3)]
        for x in inner:
            assert 16 <= x * (3 - p["refinement"]) <= 96 and x * (3 - p["refinement"]) % 2 == 0, (p, x)


def test_jet_workload_full_size_layout():
    # core 192 x 96 x 96 at h; seven patches at 2h of 64..128 cells per axis,
    # their 3-cell overlaps included
    patches = workloads.build("jet")["patches"]
    assert len(patches) == 8 and patches[0]["n"] == (192, 96, 96)
    h = patches[0]["length"][0] / 192
    for p in patches[1:]:
        assert abs(p["length"][0] / p["n"][0] - 2 * h) < 1e-15
        assert all(64 <= x <= 128 for x in p["n"]), p
    cells = sum(int(np.prod(p["n"])) for p in patches)
    assert 10e6 < cells < 13e6


@pytest.mark.gpu
@pytest.mark.parametrize("name", workloads.NAMES)
def test_workload_fp32_tracks_fp64(name):
    case = workloads.build(name, scale=0.25)
    grid, objs = workloads.make_grid(case)
    its = {prec: workloads.make_iterator(objs, prec) for prec in (_lib.DN_FP32, _lib.DN_FP64)}
    for it in its.values():
        it.setOption(_lib.DN_OPT_GRAPH, 1)
        for _ in range(10):
            it.rkStep(case["dt"], cases.RK3_ALPHA)
        it.sync()
    for q in range(len(objs)):
        a = its[_lib.DN_FP32].downloadField(q)
        b = its[_lib.DN_FP64].downloadField(q)
        assert np.isfinite(b).all()
        d = np.abs(a[0] - b[0]) / cases.RHO_INF
        assert np.sqrt((d ** 2).mean()) < 1e-5 and d.max() < 1e-4, (name, q, d.max())
    for it in its.values():
        it.close()
