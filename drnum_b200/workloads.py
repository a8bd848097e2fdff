"""The multi-patch benchmark workloads, built through the reference-style API.

    jet     dual-resolution jet: a 192 x 96 x 96 core patch at h nested at the
            inlet of a box tiled by seven patches at 2h (64 to 128 cells per
            axis, their 3-cell overlaps included), Mach 0.8 top-hat jet (radius 0.05, seeded
            1e-3 white noise) on the core's x-min face, far field at rest
            elsewhere
    sphere  level-set wall: 256 x 128 x 128 cells over [0, 2] x [0, 1]^2 in two
            overlapping patches, free stream at Mach 0.5, a sphere of radius
            0.08 at (0.3, 0.5, 0.5) as an FP32 signed-distance field with the
            slip-wall mirror condition (3 inner layers, min_inner_rel_dist 0.1)
    tiled   uneven batched grid: 8 x 8 x 8 patches with per-axis extents drawn
            from U{16..96} (seeded), refinement 1 and 2 in a checkerboard,
            2-cell overlaps, one seeded isentropic vortex per patch on a Mach
            0.4 stream, far field outside

Every state is synthetic and seeded; the reference ships no cases.
"""
from __future__ import annotations

import numpy as np

from . import cases
from ._lib import DN_FP32, DN_FP64
from .api import AusmPlus, B200CartesianIterator, CartesianPatch, PatchGrid

NAMES = ("jet", "sphere", "tiled")


def build(name, scale=1.0):
    """Returns dict(patches, states, bcs, levelset, dt, description).
    scale < 1 shrinks the case (for tests)."""
    if name == "jet":
        core = tuple(max(8, int(round(x * scale)) // 4 * 4) for x in (192, 96, 96))
        # the seven coarse patches span 64 (x halves) and 128 (y, z halves)
        # cells including their 3-cell overlaps: the box is twice that less
        # the overlap (122 x 250 x 250 cells at full size)
        nx, ny = (max(12, int(round(x * scale / 4)) * 4) for x in (64, 128))
        box = (2 * (nx - 3), 2 * (ny - 3), 2 * (ny - 3))
        patches = cases.jet_grid(core=core, box=box)
        states = cases.uniform_state(patches, mach=0.0)
        bcs = cases.jet_bcs(patches, radius=0.05, noise=1e-3, seed=1234)
        h = 0.5 / box[0]
        dt = 0.5 * h / ((0.8 + 1.0) * cases.A_INF)
        desc = (f"dual-resolution jet: 8 overlapping patches, core {core[0]}x{core[1]}x{core[2]} at h=1/{2 * box[0]} "
                f"nested at the inlet of a {box[0]}x{box[1]}x{box[2]}-cell box at 2h tiled by seven patches of "
                f"{nx}-{ny} cells per axis (3-cell overlaps included), Mach 0.8 top-hat jet r=0.05 + 1e-3 seeded "
                "noise, far field at rest")
        return dict(patches=patches, states=states, bcs=bcs, levelset=None, dt=dt, description=desc)
    if name == "sphere":
        n = tuple(max(16, int(round(x * scale)) // 2 * 2) for x in (256, 128, 128))
        patches = cases.sphere_group(n=n)
        states = cases.uniform_state(patches, mach=0.5)
        ff = (cases.P_INF, cases.T_INF, 0.5 * cases.A_INF, 0.0, 0.0)
        bcs = cases.outer_farfield_bcs(patches, ff)
        G = [cases.sphere_sdf(p, (0.3, 0.5, 0.5), 0.08) for p in patches]
        h = 2.0 / n[0]
        dt = 0.5 * h / (1.5 * cases.A_INF)
        desc = (f"level-set sphere wall: {n[0]}x{n[1]}x{n[2]} cells over [0,2]x[0,1]^2 in 2 overlapping patches, "
                "Mach 0.5, sphere r=0.08 at (0.3,0.5,0.5) as FP32 SDF, slip mirror BC (3 inner layers)")
        return dict(patches=patches, states=states, bcs=bcs, levelset=(G, 3, 0, 0.1), dt=dt, description=desc)
    if name == "tiled":
        slots = tuple(max(2, int(round(8 * scale))) for _ in range(3))
        patches = cases.tiled_grid(slots=slots)
        states = cases.tiled_state(patches)
        ff = (cases.P_INF, cases.T_INF, 0.4 * cases.A_INF, 0.0, 0.0)
        bcs = cases.outer_farfield_bcs(patches, ff)
        h = min(min(p["length"][a] / p["n"][a] for a in range(3)) for p in patches)
        dt = 0.4 * h / (1.6 * cases.A_INF)
        cells = sum(int(np.prod(p["n"])) for p in patches)
        desc = (f"uneven batched grid: {len(patches)} patches ({cells / 1e6:.1f} M cells), per-axis extents drawn "
                "from U{16..96} (seed 42), half at refinement 1 and half at refinement 2, tiled box with 2-cell "
                "overlaps, one seeded isentropic vortex (strength 3-6, radius 4 coarse cells) per patch on Mach 0.4 "
                "flow, far field outside")
        return dict(patches=patches, states=states, bcs=bcs, levelset=None, dt=dt, description=desc)
    raise KeyError(name)


def make_grid(case):
    """PatchGrid with the workload's patches (one host field each), boundary
    fluxes and level sets; donor tables computed.  Returns (grid, patches)."""
    grid = PatchGrid()
    objs = []
    for q, (p, U) in enumerate(zip(case["patches"], case["states"])):
        cp = CartesianPatch(*p["n"], lengths=p["length"], origin=p["origin"], periodic=(False, False, False),
                            seek=p["seek"], num_fields=1)
        cp.setField(0, U)
        for side, (kind, params, table) in case["bcs"].get(q, {}).items():
            cp.setBoundary(side, kind, params, table)
        if case["levelset"] is not None:
            G, ni, no, mr = case["levelset"]
            cp.setLevelSet(G[q], ni, no, mr)
        grid.insertPatch(cp)
        objs.append(cp)
    grid.computeDependencies()
    return grid, objs


def make_iterator(objs, precision, device=0):
    """B200CartesianIterator over the patches of make_grid, state uploaded."""
    it = B200CartesianIterator(AusmPlus(), device, precision)
    for cp in objs:
        it.addPatch(cp)
    it.updateDevice(fields=(0,))
    return it


__all__ = ["NAMES", "build", "make_grid", "make_iterator", "DN_FP32", "DN_FP64"]
