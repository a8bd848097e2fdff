"""The applications' output-step diagnostics on the device (dn_flow_stats):
CFL number and density range equal the reference's FP64 loop, restated in
numpy by the oracle, on the state the device holds."""
import numpy as np
import pytest

import pyoracle
from drnum_b200 import cases
from drnum_b200._lib import DN_FP32, DN_FP64
from drnum_b200.api import AusmPlus, B200CartesianIterator, CartesianPatch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [DN_FP64, DN_FP32])
def test_flow_stats_equal_the_reference_loop(prec):
    shapes = [(20, 18, 33), (9, 40, 16)]
    its_states = []
    it = B200CartesianIterator(AusmPlus(), 0, prec)
    patches = []
    for q, (ni, nj, nk) in enumerate(shapes):
        U0 = cases.random_state(ni, nj, nk, seed=11 + q, amp=0.05, mach=0.6)
        h = 1.0 / (24 + 8 * q)
        p = CartesianPatch(ni, nj, nk, spacing=(h, 0.7 * h, 1.3 * h), periodic=(True, True, True))
        p.setField(0, U0)
        it.addPatch(p)
        patches.append((p, h))
    it.updateDevice(fields=(0,))
    dt = 2.5e-5
    for _ in range(2):
        it.rkStep(dt, cases.RK3_ALPHA)
    it.updateHost(fields=(0,))
    want = [0.0, 1000.0, 0.0]
    for q, (p, h) in enumerate(patches):
        got = it.flowStats(0, dt, [q])
        ref = pyoracle.oracle_flow_stats(p.getField(0), dt, h)
        assert got == ref, (q, got, ref)
        want = [max(want[0], ref[0]), min(want[1], ref[1]), max(want[2], ref[2])]
    assert it.flowStats(0, dt) == tuple(want)
    assert 0.0 < want[0] < 1.0 and want[1] < want[2]
    it.close()
