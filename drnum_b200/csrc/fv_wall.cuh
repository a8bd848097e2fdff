// Patch-face (wall) fluxes of a stage: the flux functor's x/y/zWall{M,P}
// called for the outer faces of a non-periodic patch axis
// (iterators/cartesianiterator.h:190-308, gpu_cartesianiterator.h:117-186).
//
// Each face uses the first-order state of its own boundary cell (the
// reference's Upwind2 projection drops to first order at the patch edge,
// reconstruction/upwind2.h:39-42) and is added to that cell's residual after
// all interior faces, in the reference's order x-min, x-max, y-min, y-max,
// z-min, z-max, with + on min sides and - on max sides.  Axes of two cells or
// fewer get no wall flux (cartesianiterator.h:193,212,...).
//
// Kinds:
//   zero flux    a functor whose wall methods add nothing
//   far field    CompressibleFarfieldFlux (fluxes/compressiblefarfieldflux.h:26-181)
//   slip wall    CompressibleSlipFlux (fluxes/compressibleslipflux.h:34-98): pressure only
//   inflow       a prescribed face state (u, v, w, T and optionally p) per face, the
//                JetFlux::xWallM form of applications/drnumJetDemo/jetflux.h:158-192;
//                p from the boundary cell where the table's p is NaN
#pragma once

#include "fv_numerics.cuh"

namespace dn {

enum WallKind : int { kWallZero = 0, kWallFarfield = 1, kWallSlip = 2, kWallInflow = 3 };

struct WallBC {
  int any;                // 0: every side has zero flux
  int kind[6];            // per side: x-min, x-max, y-min, y-max, z-min, z-max
  double ff[6][6];        // far field per side: p0, T0, u0, v0, w0, a0 (primitive, from the
                          // conservative far-field state, perfectgas.h:84-93)
  const double* table[6]; // inflow per side: [faces][5] = p (NaN: boundary cell), T, u, v, w;
                          // x sides: face j*nk+k, y sides: i*nk+k, z sides: i*nj+j
};

constexpr double kGasCp = 1004.5;   // PerfectGas::cp (perfectgas.h:33)

// Primitive state of a conservative state (PerfectGas::conservativeToPrimitive,
// perfectgas.h:84-93; COMPR_VARS, compressibleflux.h:26-38).
template <typename T>
__device__ __forceinline__ void wall_prim(const T U[5], T& p, T& Tt, T& u, T& v, T& w)
{
  const T ir = T(1.0) / U[0];
  u = U[1] * ir;
  v = U[2] * ir;
  w = U[3] * ir;
  Tt = (U[4] * ir - T(0.5) * (u * u + v * v + w * w)) / T(Gas::cv);
  p = U[0] * T(Gas::R) * Tt;
}

// Flux through a face of axis AXIS from the face state (p, T, u, v, w): the
// common tail of CompressibleFarfieldFlux and JetFlux::xWallM.
template <int AXIS, typename T>
__device__ __forceinline__ void wall_state_flux(T A, T p, T Tt, T u, T v, T w, T F[5])
{
  const T un = AXIS == 0 ? u : (AXIS == 1 ? v : w);
  F[0] = A * p / (T(Gas::R) * Tt) * un;
  F[1] = F[0] * u;
  F[2] = F[0] * v;
  F[3] = F[0] * w;
  if (AXIS == 0) F[1] = F[1] + A * p;
  if (AXIS == 1) F[2] = F[2] + A * p;
  if (AXIS == 2) F[3] = F[3] + A * p;
  F[4] = F[0] * (T(kGasCp) * Tt + T(0.5) * (u * u + v * v + w * w));
}

// Wall flux of side `side` (2 * AXIS + 1 on the max side) for a boundary cell
// with state U; `face` indexes the side's inflow table.  Returns false for a
// zero-flux side (nothing to add).
template <int AXIS, typename T>
__device__ __forceinline__ bool wall_flux(const WallBC& bc, int side, int face, const T U[5], T A, T F[5])
{
  const int kind = bc.kind[side];
  if (kind == kWallZero) return false;
  const bool plus = side & 1;
  T p1, T1, u1, v1, w1;
  wall_prim(U, p1, T1, u1, v1, w1);
  if (kind == kWallSlip) {
    F[0] = T(0); F[1] = T(0); F[2] = T(0); F[3] = T(0); F[4] = T(0);
    F[1 + AXIS] = A * p1;
    return true;
  }
  if (kind == kWallInflow) {
    const double* e = bc.table[side] + (size_t)face * 5;
    const T p = (e[0] == e[0]) ? (T)e[0] : p1;    // NaN: pressure of the boundary cell
    wall_state_flux<AXIS>(A, p, (T)e[1], (T)e[2], (T)e[3], (T)e[4], F);
    return true;
  }
  // far field: face state from the sign and size of the mean inward Mach number
  const double* f = bc.ff[side];
  const T p0 = (T)f[0], T0 = (T)f[1], u0 = (T)f[2], v0 = (T)f[3], w0 = (T)f[4], a0 = (T)f[5];
  const T a1 = dn_sqrt(T(Gas::gamma) * T(Gas::R) * T1);
  const T un0 = AXIS == 0 ? u0 : (AXIS == 1 ? v0 : w0);
  const T un1 = AXIS == 0 ? u1 : (AXIS == 1 ? v1 : w1);
  const T M0 = plus ? -(un0 / a0) : un0 / a0;
  const T M1 = plus ? -(un1 / a1) : un1 / a1;
  const T M = T(0.5) * (M0 + M1);
  T p, Tt, u, v, w;
  if (M >= T(0)) {
    p = M >= T(1) ? p0 : p1;               // supersonic / subsonic inflow
    Tt = T0; u = u0; v = v0; w = w0;
  } else {
    // outflow: the reference's test `M <= 1` holds for every M < 0, so the
    // whole face state comes from the boundary cell
    p = p1; Tt = T1; u = u1; v = v1; w = w1;
  }
  wall_state_flux<AXIS>(A, p, Tt, u, v, w, F);
  return true;
}

// Adds the wall fluxes of a boundary cell (i, j, k) to its residual r in the
// reference's order; F_to_r converts a flux to the residual's type.  yz =
// false: the x sides only (a caller that has placed the y and z sides
// elsewhere).
template <typename T, typename R, typename Conv>
__device__ __forceinline__ void add_wall_fluxes(const WallBC& bc, int ni, int nj, int nk, int per_x, int per_y,
                                                int per_z, int i, int j, int k, const T U[5], T Ax, T Ay, T Az,
                                                R r[5], Conv F_to_r, bool yz = true)
{
  T F[5];
  if (!per_x && ni > 2) {
    if (i == 0 && wall_flux<0>(bc, 0, j * nk + k, U, Ax, F)) {
      #pragma unroll
      for (int v = 0; v < 5; ++v) r[v] += F_to_r(v, F[v]);
    }
    if (i == ni - 1 && wall_flux<0>(bc, 1, j * nk + k, U, Ax, F)) {
      #pragma unroll
      for (int v = 0; v < 5; ++v) r[v] -= F_to_r(v, F[v]);
    }
  }
  if (!yz) return;
  if (!per_y && nj > 2) {
    if (j == 0 && wall_flux<1>(bc, 2, i * nk + k, U, Ay, F)) {
      #pragma unroll
      for (int v = 0; v < 5; ++v) r[v] += F_to_r(v, F[v]);
    }
    if (j == nj - 1 && wall_flux<1>(bc, 3, i * nk + k, U, Ay, F)) {
      #pragma unroll
      for (int v = 0; v < 5; ++v) r[v] -= F_to_r(v, F[v]);
    }
  }
  if (!per_z && nk > 2) {
    if (k == 0 && wall_flux<2>(bc, 4, i * nj + j, U, Az, F)) {
      #pragma unroll
      for (int v = 0; v < 5; ++v) r[v] += F_to_r(v, F[v]);
    }
    if (k == nk - 1 && wall_flux<2>(bc, 5, i * nj + j, U, Az, F)) {
      #pragma unroll
      for (int v = 0; v < 5; ++v) r[v] -= F_to_r(v, F[v]);
    }
  }
}

} // namespace dn
