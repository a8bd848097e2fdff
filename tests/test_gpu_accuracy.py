"""Accuracy of the FP32 bulk form against plain FP64 on the full-size
periodic workload (256^3 cells, 1000 RK steps): the density error bound and
the conservation of the FP64 sums."""
import numpy as np
import pytest

from drnum_b200 import cases
from drnum_b200._lib import DN_FP32, DN_FP64, DN_OPT_GRAPH
from drnum_b200.api import AusmPlus, B200CartesianIterator, CartesianPatch

pytestmark = pytest.mark.gpu

N = 256
STEPS = 1000
RHO_L2_TOL = 1e-5          # relative to the free-stream density
DRIFT_TOL = 1e-10          # relative drift of the FP64 conservation sums


def test_fp32_density_error_and_drift_after_1000_steps_256cube():
    U0, h, dt = cases.periodic_box(N)
    out, sums = {}, {}
    for prec in (DN_FP64, DN_FP32):
        patch = CartesianPatch(N, N, N, spacing=(h, h, h), num_fields=1)
        patch.setField(0, U0)
        it = B200CartesianIterator(AusmPlus(), 0, prec)
        it.addPatch(patch)
        it.updateDevice(fields=(0,))
        it.setOption(DN_OPT_GRAPH, 1)
        s0 = it.conservationSums()
        for _ in range(STEPS):
            it.rkStep(dt, cases.RK3_ALPHA)
        it.sync()
        sums[prec] = (s0, it.conservationSums())
        out[prec] = it.downloadField(0)
        it.close()
    drho = (out[DN_FP32][0] - out[DN_FP64][0]) / cases.RHO_INF
    l2 = float(np.sqrt(np.mean(drho ** 2)))
    assert l2 <= RHO_L2_TOL, l2
    s0, s1 = sums[DN_FP32]
    for v in (0, 1, 4):    # mass, x momentum, energy (the y/z momenta sum to ~0)
        assert abs(s1[v] - s0[v]) <= DRIFT_TOL * abs(s0[v]), (v, s0[v], s1[v])
