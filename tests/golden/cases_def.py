"""Definitions of the golden cases (shared by the generator and the tests).

Each case is a seeded input state, a spacing, a time step, a step count and
per-axis periodicity; the expected output comes from the reference library
itself (compiled FP64 from its own sources, one OpenMP thread).
"""
from __future__ import annotations

import numpy as np

from drnum_b200 import cases

ALPHA = cases.RK3_ALPHA


def build(name):
    """Returns dict(U0, h, dt, steps, periodic, active) for a case name."""
    if name == "rough_8":
        U = cases.random_state(8, 8, 8, seed=2, amp=0.05, mach=0.6)
        h = 1.0 / 16
        return dict(U0=U, h=h, dt=cases.cfl_dt(U, h, 0.4), steps=2, periodic=(True, True, True), active=None)
    if name == "ragged_12x10x9":
        U = cases.random_state(12, 10, 9, seed=1, amp=0.01, mach=0.3)
        h = 1.0 / 16
        return dict(U0=U, h=h, dt=cases.cfl_dt(U, h, 0.5), steps=3, periodic=(True, True, True), active=None)
    if name == "vortex_16":
        U, h, dt = cases.periodic_box(16)
        return dict(U0=U, h=h, dt=dt, steps=5, periodic=(True, True, True), active=None)
    if name == "closed_10x7x12":
        U = cases.random_state(10, 7, 12, seed=3, amp=0.02, mach=0.5)
        h = 1.0 / 16
        return dict(U0=U, h=h, dt=cases.cfl_dt(U, h, 0.5), steps=3, periodic=(False, True, False), active=None)
    if name == "masked_9":
        U = cases.random_state(9, 9, 9, seed=4, amp=0.02, mach=0.3)
        h = 1.0 / 16
        rng = np.random.default_rng(5)
        act = (rng.random((9, 9, 9)) > 0.15).astype(np.uint8)
        return dict(U0=U, h=h, dt=cases.cfl_dt(U, h, 0.5), steps=2, periodic=(True, False, True), active=act)
    if name == "thin_3x5x4":
        U = cases.random_state(3, 5, 4, seed=6, amp=0.02, mach=0.3)
        h = 1.0 / 16
        return dict(U0=U, h=h, dt=cases.cfl_dt(U, h, 0.5), steps=2, periodic=(False, False, False), active=None)
    if name == "cfg1_64_100":
        U, h, dt = cases.periodic_box(64)
        return dict(U0=U, h=h, dt=dt, steps=100, periodic=(True, True, True), active=None)
    raise KeyError(name)


# full-field fixtures (small); the 64^3 x 100 case stores a digest
FULL = ["rough_8", "ragged_12x10x9", "vortex_16", "closed_10x7x12", "masked_9", "thin_3x5x4"]
DIGEST = ["cfg1_64_100"]


# ------------------------------------------------------------------ patch grids

def grid_layout(name):
    """Patch layouts of the donor-table fixtures (list of patch dicts)."""
    if name == "pair_x":
        return [dict(n=(12, 8, 8), origin=(0.0, 0.0, 0.0), length=(1.2, 0.8, 0.8), seek=(0, 2, 0, 0, 0, 0)),
                dict(n=(12, 8, 8), origin=(0.8, 0.0, 0.0), length=(1.2, 0.8, 0.8), seek=(2, 0, 0, 0, 0, 0))]
    if name == "embedded":
        return [dict(n=(10, 10, 10), origin=(0.0, 0.0, 0.0), length=(1.0, 1.0, 1.0), seek=(2, 2, 2, 2, 2, 2)),
                dict(n=(16, 16, 16), origin=(0.3, 0.27, 0.31), length=(0.4, 0.4, 0.4), seek=(2, 2, 2, 2, 2, 2))]
    if name in ("random6", "random6_prot1"):
        rng = np.random.default_rng(3)
        out = []
        for p in range(6):
            n = tuple(int(x) for x in rng.integers(6, 14, 3))
            if name == "random6_prot1":
                n = tuple(max(x, 9) for x in n)
            h = [0.1, 0.05][p % 2]
            out.append(dict(n=n, origin=tuple(float(x) for x in rng.uniform(0, 0.6, 3)),
                            length=tuple(h * x for x in n), seek=(2, 2, 2, 2, 2, 2)))
        return out
    if name == "octants_8":
        return cases.octant_grid(nf=(8, 8, 8), h=1.0 / 16, overlap=3, seek=2)
    if name == "octants_ragged":
        return cases.octant_grid(nf=(12, 8, 10), h=1.0 / 24, overlap=4, seek=2)
    raise KeyError(name)


GRID_ADD_PROTECT = {"random6_prot1": 1}
# layouts whose donor tables are fixtures; the octant grids also store RK steps
GRID_TABLES = ["pair_x", "embedded", "random6", "random6_prot1", "octants_8", "octants_ragged"]
GRID_STEPS = {"octants_8": 3, "octants_ragged": 2}


def grid_case(name):
    """Layout, initial states, spacings and time step of a stepped grid case."""
    patches = grid_layout(name)
    states = cases.grid_state(patches)
    dt = cases.grid_dt(patches, states)
    spacings = [tuple(p["length"][a] / p["n"][a] for a in range(3)) for p in patches]
    return patches, states, spacings, dt, GRID_STEPS[name]
