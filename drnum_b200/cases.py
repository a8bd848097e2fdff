"""Seeded synthetic initial states of the benchmark workloads (FP64, host).

All states are conservative variables [rho, rho u, rho v, rho w, rho E] laid
out [5][ni][nj][nk] (k fastest), built with the reference's gas model:
PerfectGas::primitiveToConservative (perfectgas.h:58-66), R = 287.2,
gamma = 1.4, cv = 717.5.  The reference ships no cases, so these are the
stand-ins for its workloads; every generator is deterministic.
"""
from __future__ import annotations

import math

import numpy as np

GAS_R = 287.2
GAS_GAMMA = 1.4
GAS_CV = 717.5

P_INF = 1.0e5
T_INF = 300.0
RHO_INF = P_INF / (GAS_R * T_INF)
A_INF = math.sqrt(GAS_GAMMA * GAS_R * T_INF)

RK3_ALPHA = (0.25, 0.5, 1.0)   # drnumJetDemo/main.h:131-133


def prim_to_cons(p, T, u, v, w):
    """PerfectGas::primitiveToConservative(p, T, u, v, w) (perfectgas.h:58-66)."""
    r = p / (GAS_R * T)
    out = np.empty((5,) + np.shape(r))
    out[0] = r
    out[1] = r * u
    out[2] = r * v
    out[3] = r * w
    out[4] = r * (GAS_CV * T + 0.5 * (u * u + v * v + w * w))
    return out


def cons_to_prim(U):
    """PerfectGas::conservativeToPrimitive (perfectgas.h:84-93): p, T, u, v, w."""
    r = U[0]
    u, v, w = U[1] / r, U[2] / r, U[3] / r
    T = (U[4] / r - 0.5 * (u * u + v * v + w * w)) / GAS_CV
    p = r * GAS_R * T
    return p, T, u, v, w


def cell_centres(n, h, origin=0.0):
    return origin + (np.arange(n) + 0.5) * h


def vortex_pulse(ni, nj, nk, lengths=(1.0, 1.0, 1.0), mach=0.3, beta=5.0, radius=0.1,
                 pulse_amp=1e-2, pulse_width=0.05, centre=None):
    """Uniform flow along x at `mach`, an isentropic vortex (axis along z,
    strength beta, radius `radius`, centred) and a Gaussian density pulse
    at constant pressure, on a periodic box of `lengths`.

    Vortex (Yee-type, velocities in units of a_inf, radius-normalised r):
        du = -beta/(2 pi) * y' * exp((1 - r^2)/2),  dv = +beta/(2 pi) * x' * exp((1 - r^2)/2)
        T/T_inf = 1 - (gamma-1) beta^2 / (8 gamma pi^2) * exp(1 - r^2),  rho ~ T^(1/(gamma-1))
    Pulse: rho *= 1 + pulse_amp * exp(-|x - c|^2 / pulse_width^2) at fixed p.
    """
    Lx, Ly, Lz = lengths
    hx, hy, hz = Lx / ni, Ly / nj, Lz / nk
    if centre is None:
        centre = (0.5 * Lx, 0.5 * Ly, 0.5 * Lz)
    x = cell_centres(ni, hx)[:, None, None]
    y = cell_centres(nj, hy)[None, :, None]
    z = cell_centres(nk, hz)[None, None, :]
    xr = (x - centre[0]) / radius
    yr = (y - centre[1]) / radius
    r2 = xr * xr + yr * yr
    e = np.exp(0.5 * (1.0 - r2))
    k = beta / (2.0 * math.pi)
    u = mach * A_INF - k * yr * e * A_INF
    v = k * xr * e * A_INF
    w = np.zeros_like(u)
    Tn = 1.0 - (GAS_GAMMA - 1.0) * beta * beta / (8.0 * GAS_GAMMA * math.pi ** 2) * e * e
    T = T_INF * Tn
    rho = RHO_INF * Tn ** (1.0 / (GAS_GAMMA - 1.0))
    p = rho * GAS_R * T
    d2 = (x - centre[0]) ** 2 + (y - centre[1]) ** 2 + (z - centre[2]) ** 2
    rho = rho * (1.0 + pulse_amp * np.exp(-d2 / pulse_width ** 2))
    T = p / (rho * GAS_R)
    shape = (ni, nj, nk)
    return prim_to_cons(np.broadcast_to(p, shape), np.broadcast_to(T, shape),
                        np.broadcast_to(u, shape), np.broadcast_to(v, shape), np.broadcast_to(w, shape))


def random_state(ni, nj, nk, seed=0, amp=0.05, mach=0.4):
    """A rough seeded state (white-noise perturbations of every primitive) that
    drives the limiter and the sub/supersonic AUSM+ branches everywhere."""
    rng = np.random.default_rng(seed)
    shape = (ni, nj, nk)
    p = P_INF * (1.0 + amp * rng.standard_normal(shape))
    T = T_INF * (1.0 + amp * rng.standard_normal(shape))
    u = A_INF * (mach + 10 * amp * rng.standard_normal(shape))
    v = A_INF * (10 * amp * rng.standard_normal(shape))
    w = A_INF * (10 * amp * rng.standard_normal(shape))
    return prim_to_cons(p, T, u, v, w)


def cfl_dt(U, dx, cfl=0.5):
    """dt = cfl * dx / max(|u| + a) over the state (drnumJetDemo/main.h:108-111
    style characteristic speed with the cell-wise velocity magnitude)."""
    p, T, u, v, w = cons_to_prim(U)
    a = np.sqrt(GAS_GAMMA * GAS_R * T)
    s = np.sqrt(u * u + v * v + w * w) + a
    return cfl * dx / float(s.max())


def periodic_box(n, steps_hint=None):
    """The single periodic patch workload of n^3 cells on the unit cube:
    returns (U0, h, dt)."""
    h = 1.0 / n
    U = vortex_pulse(n, n, n)
    dt = cfl_dt(U, h, 0.5)
    return U, h, dt


# ------------------------------------------------------------------ patch grids
#
# A grid is a list of axis-aligned patches, each a dict with
#   n (cells per axis), origin, length (extent per axis), seek (6 layers:
#   imin imax jmin jmax kmin kmax; 0 on a side without a neighbour).

def patch_centres(p):
    """Cell-centre coordinates (x, y, z) of a patch, inertial frame, as
    broadcastable arrays (CartesianPatch::xyzCell, cartesianpatch.h:267-273)."""
    h = [p["length"][a] / p["n"][a] for a in range(3)]
    xs = [p["origin"][a] + (0.5 * h[a] + np.arange(p["n"][a]) * h[a]) for a in range(3)]
    return xs[0][:, None, None], xs[1][None, :, None], xs[2][None, None, :]


def octant_grid(nf=(8, 8, 8), h=1.0 / 16, overlap=3, seek=2):
    """Dual-resolution 2x2x2 box: the octant at the origin is one patch at
    spacing h with nf cells per axis, the seven other octants are patches at
    spacing 2h.  Every patch reaches `overlap` of its own cells across each
    interior interface and receives data in `seek` layers there; the box
    faces carry no seek layers."""
    X = [nf[a] * h for a in range(3)]
    patches = []
    for oc in range(8):
        bits = ((oc >> 2) & 1, (oc >> 1) & 1, oc & 1)
        fine = oc == 0
        hh = h if fine else 2.0 * h
        n, origin, sk = [], [], []
        for a in range(3):
            cells = nf[a] if fine else nf[a] // 2
            n.append(cells + overlap)
            if bits[a] == 0:      # lower octant: interior side is the upper one
                origin.append(0.0)
                sk += [0, seek]
            else:
                origin.append(X[a] - overlap * hh)
                sk += [seek, 0]
        patches.append(dict(n=tuple(n), origin=tuple(origin), length=tuple(n[a] * hh for a in range(3)),
                            seek=tuple(sk)))
    return patches


def grid_state(patches, mach=0.3, beta=5.0, radius=0.1, centre=(0.25, 0.25, 0.25), pulse_amp=1e-2,
               pulse_width=0.05):
    """The vortex-and-pulse field of vortex_pulse evaluated at every patch's
    own cell centres (overlapping patches agree where they overlap)."""
    out = []
    for p in patches:
        x, y, z = patch_centres(p)
        xr = (x - centre[0]) / radius
        yr = (y - centre[1]) / radius
        e = np.exp(0.5 * (1.0 - (xr * xr + yr * yr)))
        k = beta / (2.0 * math.pi)
        shape = tuple(p["n"])
        u = np.broadcast_to(mach * A_INF - k * yr * e * A_INF, shape)
        v = np.broadcast_to(k * xr * e * A_INF, shape)
        w = np.zeros(shape)
        Tn = np.broadcast_to(1.0 - (GAS_GAMMA - 1.0) * beta * beta / (8.0 * GAS_GAMMA * math.pi ** 2) * e * e, shape)
        rho = RHO_INF * Tn ** (1.0 / (GAS_GAMMA - 1.0))
        pr = rho * GAS_R * T_INF * Tn
        d2 = (x - centre[0]) ** 2 + (y - centre[1]) ** 2 + (z - centre[2]) ** 2
        rho = rho * (1.0 + pulse_amp * np.exp(-d2 / pulse_width ** 2))
        T = pr / (rho * GAS_R)
        out.append(np.ascontiguousarray(prim_to_cons(pr, T, u, v, w)))
    return out


def grid_dt(patches, states, cfl=0.5):
    """One global time step: cfl * min over patches of h / max(|u| + a)."""
    return min(cfl_dt(U, min(p["length"][a] / p["n"][a] for a in range(3)), cfl) for p, U in zip(patches, states))


# ------------------------------------------------------------ patch-face fluxes
#
# Boundary conditions of a grid: {patch: {side: (kind, params, table)}} with
# side 0..5 = x-min, x-max, y-min, y-max, z-min, z-max and kind as DN_BC_*
# (0 zero flux, 1 far field with params p, T, u, v, w, 2 slip wall, 3 face
# table [faces][5] = p (NaN: boundary cell), T, u, v, w).

BC_ZERO, BC_FARFIELD, BC_SLIP, BC_INFLOW = 0, 1, 2, 3


def iterator_face_coords(n, h):
    """Face-centre coordinates along one axis of a patch side as the
    reference's wall loops produce them: start at h/2 and add h per face
    (cartesianiterator.h:193-207)."""
    out = np.empty(n)
    c = 0.5 * h
    for q in range(n):
        out[q] = c
        c += h
    return out


def jet_table(patch, u_jet, T_jet, radius, u_far=0.0, T_far=T_INF, p_jet=None, noise=0.0, seed=1234):
    """Face table of a top-hat jet on the x-min side of `patch`, the state
    JetFlux::xWallM prescribes (applications/drnumJetDemo/jetflux.h:165-191):
    inside radius (around the side's centre, patch coordinates) u = u_jet,
    T = T_jet and p = p_jet or the boundary cell's; outside u = u_far,
    T = T_far, p from the boundary cell.  `noise` adds seeded white noise of
    that relative amplitude (times u_jet) to the jet's u, v, w."""
    ni, nj, nk = patch["n"]
    dy, dz = patch["length"][1] / nj, patch["length"][2] / nk
    y, z = iterator_face_coords(nj, dy), iterator_face_coords(nk, dz)
    y0, z0 = 0.5 * nj * dy, 0.5 * nk * dz
    rr = (y[:, None] - y0) ** 2 + (z[None, :] - z0) ** 2
    inside = rr < radius * radius
    rng = np.random.default_rng(seed)
    t = np.empty((nj, nk, 5))
    t[..., 0] = np.nan
    t[..., 1] = np.where(inside, T_jet, T_far)
    t[..., 2] = np.where(inside, u_jet, u_far)
    t[..., 3] = 0.0
    t[..., 4] = 0.0
    if p_jet is not None:
        t[..., 0] = np.where(inside, p_jet, np.nan)
    if noise:
        pert = noise * u_jet * rng.uniform(-1.0, 1.0, (nj, nk, 3))
        t[..., 2:5] += np.where(inside[..., None], pert, 0.0)
    return t.reshape(-1, 5)


def outer_farfield_bcs(patches, state=(P_INF, T_INF, 0.0, 0.0, 0.0)):
    """Far field on every side of every patch that has no seek layers."""
    return {p: {side: (BC_FARFIELD, tuple(state), None) for side in range(6) if patch["seek"][side] == 0}
            for p, patch in enumerate(patches)}


def jet_bcs(patches, core=0, mach_jet=0.8, radius=0.05, noise=1e-3, seed=1234):
    """Far field at rest on the outer sides and a top-hat jet of Mach
    `mach_jet` on the x-min side of patch `core`."""
    bcs = outer_farfield_bcs(patches)
    bcs[core][0] = (BC_INFLOW, None, jet_table(patches[core], mach_jet * A_INF, T_INF, radius, noise=noise,
                                               seed=seed))
    return bcs


# ------------------------------------------------------------------ level sets

def sphere_sdf(patch, centre, radius, fp32=True):
    """Signed distance |x - c| - R of a sphere at every cell centre of a
    patch (SphereLevelSet::calcDistance, spherelevelset.cpp:21-32), optionally
    rounded to FP32 (the FP32 signed-distance field of the wall workload)."""
    x, y, z = patch_centres(patch)
    dx, dy, dz = x - centre[0], y - centre[1], z - centre[2]
    g = np.sqrt(dx * dx + dy * dy + dz * dz) - radius
    g = np.broadcast_to(g, tuple(patch["n"]))
    return np.ascontiguousarray(g.astype(np.float32).astype(np.float64) if fp32 else g)


def uniform_state(patches, mach=0.5, p=P_INF, T=T_INF):
    """Free stream at `mach` along x on every patch."""
    out = []
    for q in patches:
        shape = tuple(q["n"])
        out.append(np.ascontiguousarray(prim_to_cons(np.full(shape, p), np.full(shape, T),
                                                     np.full(shape, mach * A_INF), np.zeros(shape),
                                                     np.zeros(shape))))
    return out


# ------------------------------------------------------- benchmark workloads

def jet_grid(core=(192, 96, 96), box=(128, 256, 256), overlap=3, seek=2):
    """Dual-resolution jet workload: a core patch of `core` cells at spacing
    h and seven patches at 2h around it.  The seven tile a box of `box`
    cells at 2h (x length 1, so h = 1 / (2 box[0])): 2 x 2 x 2 blocks split
    at half the box on each axis, the two blocks of the upper (y, z) quadrant
    merged along x, so every side spans box/2 or box cells.  The core starts
    at the box's x-min face, centred in y and z, where the jet enters; it is
    nested in the coarse patches and receives data in `seek` layers on its
    five other faces.  Coarse patches reach `overlap` of their own cells
    across each interface between them, with `seek` layers there; the box
    faces carry none."""
    H = 1.0 / box[0]                 # coarse spacing 2h
    h = 0.5 * H
    half = [box[a] // 2 for a in range(3)]
    cy, cz = 0.5 * box[1] * H, 0.5 * box[2] * H
    patches = [dict(n=tuple(core), origin=(0.0, cy - 0.5 * core[1] * h, cz - 0.5 * core[2] * h),
                    length=tuple(core[a] * h for a in range(3)), seek=(0, seek, seek, seek, seek, seek))]
    for b in range(2):
        for c in range(2):
            xs = [(0, box[0])] if (b, c) == (1, 1) else [(0, half[0]), (half[0], box[0])]
            for x0, x1 in xs:
                lo = [x0, b * half[1], c * half[2]]
                hi = [x1, (b + 1) * half[1], (c + 1) * half[2]]
                n, origin, sk = [], [], []
                for a in range(3):
                    lo_in, hi_in = lo[a] > 0, hi[a] < box[a]
                    n.append(hi[a] - lo[a] + overlap * (int(lo_in) + int(hi_in)))
                    origin.append((lo[a] - (overlap if lo_in else 0)) * H)
                    sk += [seek if lo_in else 0, seek if hi_in else 0]
                patches.append(dict(n=tuple(n), origin=tuple(origin), length=tuple(n[a] * H for a in range(3)),
                                    seek=tuple(sk)))
    return patches


def sphere_group(n=(256, 128, 128), L=1.0, overlap=3):
    """Level-set wall workload: a patch group of n cells over [0, 2L] x [0, L]
    x [0, L] split into two patches along x that overlap by `overlap` cells
    on each side of the cut (seek layers 2)."""
    h = 2.0 * L / n[0]
    half = n[0] // 2
    a = dict(n=(half + overlap, n[1], n[2]), origin=(0.0, 0.0, 0.0),
             length=((half + overlap) * h, n[1] * h, n[2] * h), seek=(0, 2, 0, 0, 0, 0))
    b = dict(n=(n[0] - half + overlap, n[1], n[2]), origin=((half - overlap) * h, 0.0, 0.0),
             length=((n[0] - half + overlap) * h, n[1] * h, n[2] * h), seek=(2, 0, 0, 0, 0, 0))
    return [a, b]


def tiled_grid(slots=(8, 8, 8), extent=(16, 96), h=1.0 / 256, overlap=2, seed=42):
    """Uneven batched workload: a box of slots[0] x slots[1] x slots[2]
    patches.  The extent of each slot row along each axis is drawn uniformly
    from the even numbers of `extent` cells of spacing h (seed); patches
    alternate between refinement 2 (spacing h: the drawn count of cells) and
    refinement 1 (spacing 2h: half of it) in a checkerboard.  Every patch
    reaches `overlap` of its own cells across each interior interface, with
    2 seek layers there."""
    rng = np.random.default_rng(seed)
    ext = [rng.integers(extent[0] // 2, extent[1] // 2 + 1, slots[a]) for a in range(3)]   # in cells of 2h
    H = 2.0 * h
    starts = [np.concatenate(([0], np.cumsum(ext[a])[:-1])) * H for a in range(3)]
    patches = []
    for a in range(slots[0]):
        for b in range(slots[1]):
            for c in range(slots[2]):
                r = 2 if (a + b + c) % 2 else 1
                hh = H / r
                idx = (a, b, c)
                n, origin, sk = [], [], []
                for ax in range(3):
                    lo_in = idx[ax] > 0
                    hi_in = idx[ax] < slots[ax] - 1
                    cells = int(ext[ax][idx[ax]]) * r
                    n.append(cells + overlap * (int(lo_in) + int(hi_in)))
                    origin.append(float(starts[ax][idx[ax]]) - (overlap * hh if lo_in else 0.0))
                    sk += [2 if lo_in else 0, 2 if hi_in else 0]
                patches.append(dict(n=tuple(n), origin=tuple(origin), length=tuple(n[q] * hh for q in range(3)),
                                    seek=tuple(sk), refinement=r))
    return patches


def vortex_field(patch, mach, centre, beta, radius):
    """Isentropic vortex (axis z) of strength beta on uniform flow at `mach`
    along x, at the patch's cell centres."""
    x, y, z = patch_centres(patch)
    xr = (x - centre[0]) / radius
    yr = (y - centre[1]) / radius
    e = np.exp(0.5 * (1.0 - (xr * xr + yr * yr)))
    k = beta / (2.0 * math.pi)
    shape = tuple(patch["n"])
    u = np.broadcast_to(mach * A_INF - k * yr * e * A_INF, shape)
    v = np.broadcast_to(k * xr * e * A_INF, shape)
    Tn = np.broadcast_to(1.0 - (GAS_GAMMA - 1.0) * beta * beta / (8.0 * GAS_GAMMA * math.pi ** 2) * e * e, shape)
    rho = RHO_INF * Tn ** (1.0 / (GAS_GAMMA - 1.0))
    p = rho * GAS_R * T_INF * Tn
    return np.ascontiguousarray(prim_to_cons(p, T_INF * Tn, u, v, np.zeros(shape)))


def tiled_state(patches, mach=0.4, seed=42, radius_cells=4.0, h=1.0 / 256, cutoff=4.0):
    """One seeded vortex per patch (axis z, centre in the middle 40 % of the
    patch, strength 3..6, radius `radius_cells` coarse cells of 2h, damped
    along z over the same radius, exactly zero beyond `cutoff` radii) on a
    common uniform flow.  The vortices superpose into one global field
    (velocity perturbations add, temperature factors multiply) evaluated at
    every patch's own cell centres, so overlapping patches agree."""
    rng = np.random.default_rng(seed + 1)
    R = radius_cells * 2.0 * h
    vort = []
    for p in patches:
        lo = np.array(p["origin"])
        L = np.array(p["length"])
        vort.append((lo + L * rng.uniform(0.3, 0.7, 3), float(rng.uniform(3.0, 6.0))))
    centres = np.array([c for c, _ in vort])
    reach = cutoff * R
    out = []
    for p in patches:
        lo = np.array(p["origin"])
        hi = lo + np.array(p["length"])
        xs = [p["origin"][a] + (np.arange(p["n"][a]) + 0.5) * (p["length"][a] / p["n"][a]) for a in range(3)]
        shape = tuple(p["n"])
        du = np.zeros(shape)
        dv = np.zeros(shape)
        Tn = np.ones(shape)
        near = np.all((centres > lo - reach) & (centres < hi + reach), axis=1)
        for q in np.nonzero(near)[0]:
            c, beta = vort[q]
            sl = []
            for a in range(3):                        # sub-box within reach of the centre
                i0 = int(np.searchsorted(xs[a], c[a] - reach))
                i1 = int(np.searchsorted(xs[a], c[a] + reach))
                sl.append(slice(i0, i1))
            if any(t.start >= t.stop for t in sl):
                continue
            x = xs[0][sl[0]][:, None, None]
            y = xs[1][sl[1]][None, :, None]
            z = xs[2][sl[2]][None, None, :]
            xr, yr, zr = (x - c[0]) / R, (y - c[1]) / R, (z - c[2]) / R
            r2 = xr * xr + yr * yr + zr * zr
            e = np.exp(0.5 * (1.0 - (xr * xr + yr * yr))) * np.exp(-0.5 * zr * zr) * (r2 < cutoff * cutoff)
            k = beta / (2.0 * math.pi)
            sub = (sl[0], sl[1], sl[2])
            du[sub] = du[sub] - k * yr * e * A_INF
            dv[sub] = dv[sub] + k * xr * e * A_INF
            Tn[sub] = Tn[sub] * (1.0 - (GAS_GAMMA - 1.0) * beta * beta / (8.0 * GAS_GAMMA * math.pi ** 2) * e * e)
        rho = RHO_INF * Tn ** (1.0 / (GAS_GAMMA - 1.0))
        pr = rho * GAS_R * T_INF * Tn
        u = mach * A_INF + du
        out.append(np.ascontiguousarray(prim_to_cons(pr, T_INF * Tn, u, dv, np.zeros(shape))))
    return out
