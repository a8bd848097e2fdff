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
    if name == "flat_8x2x9":
        # a closed axis of two cells: no faces along it (cartesianiterator.h:160)
        U = cases.random_state(8, 2, 9, seed=8, amp=0.02, mach=0.4)
        h = 1.0 / 16
        return dict(U0=U, h=h, dt=cases.cfl_dt(U, h, 0.5), steps=2, periodic=(True, False, True), active=None)
    if name == "column_1x1x10":
        # two closed axes of one cell: a 1-D problem along k
        U = cases.random_state(1, 1, 10, seed=9, amp=0.02, mach=0.4)
        h = 1.0 / 16
        return dict(U0=U, h=h, dt=cases.cfl_dt(U, h, 0.5), steps=3, periodic=(False, False, True), active=None)
    if name == "transonic_10":
        # Mach ~1 with strong perturbations: faces on both sides of |M| = 1
        # (van Leer's supersonic branches, Roe's sonic entropy modification)
        U = cases.random_state(10, 10, 10, seed=7, amp=0.08, mach=1.0)
        h = 1.0 / 16
        return dict(U0=U, h=h, dt=cases.cfl_dt(U, h, 0.4), steps=2, periodic=(True, True, True), active=None)
    if name == "micro_12":
        # micrometre cells: the viscous stresses are about 1 % of the pressure
        # fluxes, so the viscous functor shows in every cell
        U = cases.random_state(12, 12, 12, seed=12, amp=0.02, mach=0.3)
        h = 2e-6
        return dict(U0=U, h=h, dt=cases.cfl_dt(U, h, 0.4), steps=3, periodic=(True, True, True), active=None)
    if name == "micro_closed_10x8x9":
        U = cases.random_state(10, 8, 9, seed=13, amp=0.02, mach=0.3)
        h = 2e-6
        return dict(U0=U, h=h, dt=cases.cfl_dt(U, h, 0.4), steps=3, periodic=(False, True, False), active=None)
    if name == "cfg1_64_100":
        U, h, dt = cases.periodic_box(64)
        return dict(U0=U, h=h, dt=dt, steps=100, periodic=(True, True, True), active=None)
    raise KeyError(name)


# full-field fixtures (small); the 64^3 x 100 case stores a digest
FULL = ["rough_8", "ragged_12x10x9", "vortex_16", "closed_10x7x12", "masked_9", "thin_3x5x4", "flat_8x2x9",
        "column_1x1x10"]
DIGEST = ["cfg1_64_100"]

# Euler flux schemes of the generic functor path (numbered as DN_FLUX_*) and
# the single-patch cases each is pinned on; the bc_box grid is pinned too
SCHEMES = {"vanleer": 2, "roe": 3}
SCHEME_CASES = ["vortex_16", "closed_10x7x12", "masked_9", "thin_3x5x4", "transonic_10"]

# the reference's own VanLeer + CompressibleViscFlux functors (the field
# fluxes of its jet application), compiled for the device against the
# generic functor stage (oracle/ref_functor_stage.cu), pinned on these cases
VISC_SCHEME = 4
VISC_CASES = ["micro_12", "micro_closed_10x8x9", "vortex_16"]

# the reference's own Roe + CompressibleSmagorinskyFlux<5, 2400> functors (the
# field fluxes of its base-flow application), pinned the same way
SMAG_SCHEME = 5
SMAG_CASES = ["micro_12", "micro_closed_10x8x9", "vortex_16"]

# fixture prefix -> (reference scheme number, cases) of the viscous functor sets
VISCOUS_SETS = {"visc": (VISC_SCHEME, VISC_CASES), "smag": (SMAG_SCHEME, SMAG_CASES)}


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
    if name == "octants_jet":
        return grid_layout("octants_8")
    if name == "bc_box":
        return [dict(n=(10, 8, 9), origin=(0.0, 0.0, 0.0), length=(1.0, 0.8, 0.9), seek=(0, 0, 0, 0, 0, 0))]
    if name == "sphere_box":
        return [dict(n=(20, 16, 16), origin=(0.0, 0.0, 0.0), length=(1.25, 1.0, 1.0), seek=(0, 0, 0, 0, 0, 0))]
    if name == "sphere_pair":
        return [dict(n=(14, 16, 16), origin=(0.0, 0.0, 0.0), length=(0.875, 1.0, 1.0), seek=(0, 2, 0, 0, 0, 0)),
                dict(n=(14, 16, 16), origin=(0.5, 0.0, 0.0), length=(0.875, 1.0, 1.0), seek=(2, 0, 0, 0, 0, 0))]
    raise KeyError(name)


GRID_ADD_PROTECT = {"random6_prot1": 1}
# layouts whose donor tables are fixtures; the octant grids also store RK steps
GRID_TABLES = ["pair_x", "embedded", "random6", "random6_prot1", "octants_8", "octants_ragged", "octants_jet",
               "bc_box", "sphere_box", "sphere_pair"]
GRID_STEPS = {"octants_8": 3, "octants_ragged": 2, "octants_jet": 3, "bc_box": 3, "sphere_box": 3, "sphere_pair": 3}
# level-set walls: name -> (centre, radius); 3 inner layers, no outer layer,
# min_inner_rel_dist 0.1 (testBlockObjects/main.h:384-388), FP32 distance field
LEVELSET = {"sphere_box": ((0.4, 0.5, 0.5), 0.2), "sphere_pair": ((0.6, 0.5, 0.5), 0.2)}
LS_INNER, LS_OUTER, LS_MIN_REL = 3, 0, 0.1


def grid_levelset(name):
    """Per-patch level-set fields of a grid case (None without a wall)."""
    if name not in LEVELSET:
        return None
    centre, radius = LEVELSET[name]
    return [cases.sphere_sdf(p, centre, radius) for p in grid_layout(name)]


def grid_case(name):
    """Layout, initial states, spacings and time step of a stepped grid case."""
    patches = grid_layout(name)
    if name == "bc_box":
        states = cases.grid_state(patches, centre=(0.45, 0.4, 0.45))
    elif name in LEVELSET:
        states = cases.uniform_state(patches, mach=0.5)
    else:
        states = cases.grid_state(patches)
    dt = cases.grid_dt(patches, states)
    spacings = [tuple(p["length"][a] / p["n"][a] for a in range(3)) for p in patches]
    return patches, states, spacings, dt, GRID_STEPS[name]


# grids with patch-face fluxes: layout name -> boundary conditions
def grid_bcs(name):
    if name in LEVELSET:
        return cases.outer_farfield_bcs(grid_layout(name), (cases.P_INF, cases.T_INF, 0.5 * cases.A_INF, 0.0, 0.0))
    if name == "octants_jet":
        return cases.jet_bcs(grid_layout("octants_8"), radius=0.12, noise=1e-3)
    if name == "bc_box":
        patch = grid_layout("bc_box")[0]
        t = cases.jet_table(patch, 0.6 * cases.A_INF, 0.9 * cases.T_INF, radius=0.2, u_far=0.1 * cases.A_INF,
                            p_jet=1.05 * cases.P_INF, noise=1e-2)
        far_a = (cases.P_INF, cases.T_INF, 0.3 * cases.A_INF, 0.05 * cases.A_INF, 0.0)
        far_b = (0.95 * cases.P_INF, 1.1 * cases.T_INF, 0.0, -1.2 * cases.A_INF, 0.1 * cases.A_INF)
        return {0: {0: (cases.BC_INFLOW, None, t), 1: (cases.BC_FARFIELD, far_a, None),
                    2: (cases.BC_SLIP, None, None), 3: (cases.BC_FARFIELD, far_b, None),
                    4: (cases.BC_SLIP, None, None), 5: (cases.BC_ZERO, None, None)}}
    return None
