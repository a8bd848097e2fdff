"""The oracle restatement (oracle/fv_oracle.c) against the reference's own
outputs (tests/golden/, generated from the compiled reference library)."""
import hashlib
import json
import os

import numpy as np
import pytest

import cases_def
import pyoracle


def _load(golden_dir, name):
    z = np.load(os.path.join(golden_dir, f"{name}.npz"))
    active = z["active"] if z["active"].size else None
    return z, active


@pytest.mark.parametrize("name", cases_def.FULL)
def test_oracle_matches_reference_bitwise(golden_dir, name):
    z, active = _load(golden_dir, name)
    out = pyoracle.oracle_run(z["U0"], float(z["h"]), float(z["dt"]), int(z["steps"]), tuple(z["alpha"]),
                              tuple(bool(p) for p in z["periodic"]), active)
    assert np.array_equal(out, z["out"]), f"max diff {np.abs(out - z['out']).max()}"


def test_fixture_inputs_regenerate(golden_dir):
    # the case generator still produces the stored inputs
    for name in cases_def.FULL:
        z, _ = _load(golden_dir, name)
        c = cases_def.build(name)
        assert np.array_equal(np.asarray(c["U0"]), z["U0"]), name


def test_oracle_cfg1_64cube_100_steps_digest(golden_dir):
    meta = json.load(open(os.path.join(golden_dir, "digests.json")))["cfg1_64_100"]
    c = cases_def.build("cfg1_64_100")
    U0 = np.ascontiguousarray(c["U0"], dtype=np.float64)
    assert hashlib.sha256(U0.tobytes()).hexdigest() == meta["input_sha256"]
    out = pyoracle.oracle_run(U0, c["h"], c["dt"], c["steps"], cases_def.ALPHA, c["periodic"])
    assert hashlib.sha256(out.tobytes()).hexdigest() == meta["output_sha256"]


def test_oracle_detects_planted_error(golden_dir):
    # a mistake planted in the oracle's input shows up in the comparison
    z, active = _load(golden_dir, "rough_8")
    U0 = z["U0"].copy()
    U0[4, 3, 3, 3] *= 1.0 + 1e-12
    out = pyoracle.oracle_run(U0, float(z["h"]), float(z["dt"]), int(z["steps"]), tuple(z["alpha"]),
                              tuple(bool(p) for p in z["periodic"]), active)
    assert not np.array_equal(out, z["out"])


def test_oracle_conserves_on_periodic_box():
    c = cases_def.build("vortex_16")
    out = pyoracle.oracle_run(c["U0"], c["h"], c["dt"], 3)
    s0 = c["U0"].reshape(5, -1).sum(1)
    s1 = out.reshape(5, -1).sum(1)
    assert np.allclose(s0, s1, rtol=1e-13, atol=1e-9)
