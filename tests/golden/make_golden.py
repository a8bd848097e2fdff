"""Generates the golden fixtures of tests/golden/ from the reference itself.

    python tests/golden/make_golden.py              # single-patch fixtures + grids
    python tests/golden/make_golden.py --grids      # grids only
    python tests/golden/make_golden.py --schemes    # VanLeer / Roe / viscous fixtures
    python tests/golden/make_golden.py --viscous smag   # one viscous set (visc, smag)
    python tests/golden/make_golden.py --cases a,b  # the named single-patch fixtures only

Needs oracle/_ref/libdrnum_ref.so, i.e. the reference DrNUM library compiled
(FP64) from its own sources by oracle/build_ref.sh.  Each fixture stores the
input state, the case parameters and the reference's output after the given
number of RK steps (one OpenMP thread: the reference's canonical accumulation
order).  The 64^3 x 100-step case stores SHA-256 digests and sums instead of
the 10 MB field.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

import pyoracle  # noqa: E402
import cases_def  # noqa: E402


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def main(only=None):
    assert pyoracle.ref_lib().dnref_real_size() == 8
    for name in cases_def.FULL:
        if only is not None and name not in only:
            continue
        c = cases_def.build(name)
        out, sec = pyoracle.ref_run(c["U0"], c["h"], c["dt"], c["steps"], cases_def.ALPHA,
                                    c["periodic"], c["active"], threads=1)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), U0=c["U0"], out=out, h=c["h"], dt=c["dt"],
                            steps=c["steps"], periodic=np.array(c["periodic"], dtype=np.int8),
                            active=c["active"] if c["active"] is not None else np.ones(0, np.uint8),
                            alpha=np.array(cases_def.ALPHA))
        print(f"{name}: {sec:.3f} s")
    if only is not None:
        return
    meta = {}
    for name in cases_def.DIGEST:
        c = cases_def.build(name)
        out, sec = pyoracle.ref_run(c["U0"], c["h"], c["dt"], c["steps"], cases_def.ALPHA,
                                    c["periodic"], c["active"], threads=1)
        meta[name] = dict(input_sha256=digest(c["U0"]), output_sha256=digest(out),
                          sums=[float(x) for x in out.reshape(5, -1).sum(axis=1)],
                          rho_sample=[float(x) for x in out[0].reshape(-1)[::4099]],
                          h=c["h"], dt=c["dt"], steps=c["steps"], seconds=sec)
        print(f"{name}: {sec:.3f} s")
    with open(os.path.join(HERE, "digests.json"), "w") as f:
        json.dump(meta, f, indent=1)
    make_grids()


def make_grids():
    """Donor tables of the reference's PatchGrid::computeDependencies for the
    grid layouts, and the reference's multi-patch RK steps (RungeKutta +
    CartesianIterator + Patch::accessDonorDataDirect) for the octant grids."""
    for name in cases_def.GRID_TABLES:
        patches = cases_def.grid_layout(name)
        G = cases_def.grid_levelset(name)
        g = pyoracle.RefGrid(patches, cases_def.GRID_ADD_PROTECT.get(name, 0), threads=1,
                             num_vars=6 if G is not None else 5)
        arrays = {}
        for p in range(len(patches)):
            t = g.tables(p)
            for k, v in t.items():
                arrays[f"p{p}_{k}"] = v
        if G is not None:
            g.levelset(G, cases_def.LS_INNER, cases_def.LS_OUTER, cases_def.LS_MIN_REL)
            for p in range(len(patches)):
                for layer in range(cases_def.LS_INNER):
                    for k, v in g.levelset_layer(p, 1, layer).items():
                        arrays[f"p{p}_ls{layer}_{k}"] = v
        bcs = cases_def.grid_bcs(name) or {}
        for p, sides in bcs.items():
            for side, (kind, params, table) in sides.items():
                g.set_bc(p, side, kind, params, table)
        if name in cases_def.GRID_STEPS:
            _, states, _, dt, steps = cases_def.grid_case(name)
            for p, U in enumerate(states):
                g.set_state(p, U)
            g.run(steps, dt, cases_def.ALPHA)
            for p in range(len(patches)):
                arrays[f"p{p}_out"] = g.get_state(p)
            arrays["dt"] = np.array(dt)
            arrays["steps"] = np.array(steps)
        g.close()
        arrays["num_patches"] = np.array(len(patches))
        np.savez_compressed(os.path.join(HERE, f"grid_{name}.npz"), **arrays)
        print(f"grid_{name}: {len(patches)} patches")


def make_schemes():
    """The reference's CartesianIterator with its VanLeer and Roe functors
    (Upwind2<VanAlbada>, PerfectGas) on the single-patch cases, and on the
    bc_box grid with every patch-face kind."""
    for sname, scheme in cases_def.SCHEMES.items():
        for name in cases_def.SCHEME_CASES:
            c = cases_def.build(name)
            out, sec = pyoracle.ref_run(c["U0"], c["h"], c["dt"], c["steps"], cases_def.ALPHA,
                                        c["periodic"], c["active"], threads=1, scheme=scheme)
            np.savez_compressed(os.path.join(HERE, f"scheme_{sname}_{name}.npz"), U0=c["U0"], out=out, h=c["h"],
                                dt=c["dt"], steps=c["steps"], periodic=np.array(c["periodic"], dtype=np.int8),
                                active=c["active"] if c["active"] is not None else np.ones(0, np.uint8),
                                alpha=np.array(cases_def.ALPHA), scheme=np.array(scheme))
            print(f"scheme_{sname}_{name}: {sec:.3f} s")
        gname = "bc_box"
        patches, states, _, dt, steps = cases_def.grid_case(gname)
        g = pyoracle.RefGrid(patches, 0, threads=1)
        for p, sides in (cases_def.grid_bcs(gname) or {}).items():
            for side, (kind, params, table) in sides.items():
                g.set_bc(p, side, kind, params, table)
        for p, U in enumerate(states):
            g.set_state(p, U)
        g.run(steps, dt, cases_def.ALPHA, scheme=scheme)
        arrays = {f"p{p}_out": g.get_state(p) for p in range(len(patches))}
        g.close()
        arrays.update(dt=np.array(dt), steps=np.array(steps), scheme=np.array(scheme),
                      num_patches=np.array(len(patches)))
        np.savez_compressed(os.path.join(HERE, f"grid_{gname}_{sname}.npz"), **arrays)
        print(f"grid_{gname}_{sname}")
    make_viscous()


def make_viscous(only=None):
    """The reference's viscous functor sets (VanLeer + CompressibleViscFlux,
    Roe + CompressibleSmagorinskyFlux) on their single-patch cases."""
    for prefix, (scheme, names) in cases_def.VISCOUS_SETS.items():
        if only and prefix not in only:
            continue
        for name in names:
            c = cases_def.build(name)
            out, sec = pyoracle.ref_run(c["U0"], c["h"], c["dt"], c["steps"], cases_def.ALPHA, c["periodic"],
                                        c["active"], threads=1, scheme=scheme)
            np.savez_compressed(os.path.join(HERE, f"{prefix}_{name}.npz"), U0=c["U0"], out=out, h=c["h"],
                                dt=c["dt"], steps=c["steps"], periodic=np.array(c["periodic"], dtype=np.int8),
                                active=np.ones(0, np.uint8), alpha=np.array(cases_def.ALPHA),
                                scheme=np.array(scheme))
            print(f"{prefix}_{name}: {sec:.3f} s")


if __name__ == "__main__":
    if "--grids" in sys.argv:
        make_grids()
    elif "--schemes" in sys.argv:
        make_schemes()
    elif "--viscous" in sys.argv:
        make_viscous(set(sys.argv[sys.argv.index("--viscous") + 1].split(",")))
    elif "--cases" in sys.argv:
        main(only=set(sys.argv[sys.argv.index("--cases") + 1].split(",")))
    else:
        main()
