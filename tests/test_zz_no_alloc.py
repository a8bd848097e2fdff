"""The allocation-free sums entry point (dn_field_sums_noalloc) against the
context-based dn_conservation_sums, through the C ABI.

dn_field_sums_noalloc serves callers that cannot allocate device memory
(their device memory is reserved up front or owned by another pool); here the
caller's field lives in a buffer the test allocates itself.  Collected last
so that a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from drnum_b200 import _lib, cases
from drnum_b200._lib import DN_ERR_RANGE, DN_FP64, DN_OK
from drnum_b200.api import AusmPlus, B200CartesianIterator, CartesianPatch

pytestmark = pytest.mark.gpu

N = 40


def _context_state_and_sums(steps):
    U0, h, dt = cases.periodic_box(N)
    patch = CartesianPatch(N, N, N, spacing=(h, h, h))
    patch.setField(0, U0)
    it = B200CartesianIterator(AusmPlus(), 0, DN_FP64)
    it.addPatch(patch)
    it.updateDevice(fields=(0,))
    for _ in range(steps):
        it.rkStep(dt, cases.RK3_ALPHA)
    it.updateHost(fields=(0,))
    sums = it.conservationSums()
    it.close()
    return patch.getField(0).copy(), sums, h ** 3


def test_noalloc_sums_match_context_sums_on_two_calls():
    import torch
    lib = _lib.load()
    for call, steps in enumerate((1, 3)):
        U, expected, dV = _context_state_and_sums(steps)
        field = torch.from_numpy(np.ascontiguousarray(U)).to("cuda:0")   # the caller's own buffer
        torch.cuda.synchronize()
        out = np.zeros(5)
        rc = lib.dn_field_sums_noalloc(ctypes.c_void_p(field.data_ptr()), N ** 3, dV, _lib.dptr(out), None)
        assert rc == DN_OK, f"call {call}: status {rc}"
        scale = np.abs(U).reshape(5, -1).sum(1) * dV
        assert np.all(np.abs(out - expected) <= 1e-12 * scale), (call, out - expected)


def test_noalloc_rejects_fields_beyond_its_fixed_scratch():
    import torch
    lib = _lib.load()
    field = torch.zeros(5 * 8, dtype=torch.float64, device="cuda:0")
    out = np.zeros(5)
    # 2^27 + 1 cells exceed the fixed scratch; rejected before any launch
    rc = lib.dn_field_sums_noalloc(ctypes.c_void_p(field.data_ptr()), (1 << 27) + 1, 1.0, _lib.dptr(out), None)
    assert rc == DN_ERR_RANGE
