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


@pytest.mark.skipif(not pyoracle.ref_available(), reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("sname", sorted(cases_def.SCHEMES))
def test_scheme_fixtures_reproduce_from_reference(golden_dir, sname):
    # the VanLeer / Roe fixtures are the compiled reference's own outputs,
    # and their inputs still come from the case generator
    for name in cases_def.SCHEME_CASES:
        z, active = _load(golden_dir, f"scheme_{sname}_{name}")
        c = cases_def.build(name)
        assert np.array_equal(np.asarray(c["U0"]), z["U0"]), name
        out, _ = pyoracle.ref_run(z["U0"], float(z["h"]), float(z["dt"]), int(z["steps"]), tuple(z["alpha"]),
                                  tuple(bool(p) for p in z["periodic"]), active, threads=1,
                                  scheme=int(z["scheme"]))
        assert np.array_equal(out, z["out"]), (sname, name)


@pytest.mark.skipif(not pyoracle.ref_available(), reason="compiled reference (oracle/_ref) not built")
def test_schemes_differ_from_each_other(golden_dir):
    # the scheme switch of the reference driver reaches the flux: the three
    # schemes give different states on the same input
    outs = [_load(golden_dir, f"scheme_{s}_vortex_16")[0]["out"] for s in sorted(cases_def.SCHEMES)]
    outs.append(_load(golden_dir, "vortex_16")[0]["out"])
    for a in range(len(outs)):
        for b in range(a + 1, len(outs)):
            assert not np.array_equal(outs[a], outs[b])


@pytest.mark.skipif(not pyoracle.ref_available(), reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("prefix", sorted(cases_def.VISCOUS_SETS))
def test_viscous_fixtures_reproduce_and_carry_their_viscous_terms(golden_dir, prefix):
    # the viscous fixtures (VanLeer + CompressibleViscFlux, Roe +
    # CompressibleSmagorinskyFlux) are the compiled reference's own outputs,
    # and differ from the same Euler flux without the viscous part
    inviscid = {cases_def.VISC_SCHEME: cases_def.SCHEMES["vanleer"], cases_def.SMAG_SCHEME: cases_def.SCHEMES["roe"]}
    scheme, names = cases_def.VISCOUS_SETS[prefix]
    for name in names:
        z, active = _load(golden_dir, f"{prefix}_{name}")
        assert int(z["scheme"]) == scheme
        args = (z["U0"], float(z["h"]), float(z["dt"]), int(z["steps"]), tuple(z["alpha"]),
                tuple(bool(p) for p in z["periodic"]), active)
        out, _ = pyoracle.ref_run(*args, threads=1, scheme=scheme)
        assert np.array_equal(out, z["out"]), (prefix, name)
        euler, _ = pyoracle.ref_run(*args, threads=1, scheme=inviscid[scheme])
        scale = np.abs(z["out"]).reshape(5, -1).max(axis=1)[:, None, None, None]
        assert (np.abs(euler - z["out"]) / scale).max() > 1e-9, (prefix, name)
