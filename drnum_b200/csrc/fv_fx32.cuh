// FP32 bulk stage kernel with fixed-point storage ("FX32").
//
// Same scheme as the reference (Upwind2 MUSCL on conservative variables with
// the van Albada limiter, AUSM+ flux, low-storage RK update; see
// fv_numerics.cuh for the reference citations) evaluated in FP32, with
// storage and accumulation arranged for bandwidth and exact conservation:
//
// Storage.  A patch holds per variable v an FP64 base B_v and a power-of-two
// quantum q_v; a cell stores the int32 offset o with U = B_v + q_v * o.  The
// quantum is 2^-30 of four times the variable's magnitude scale, far below
// the FP32 spacing of U, so storage adds no visible rounding.
//
// Update.  Each face flux F (FP32) is scaled by (factor/dV)/q_v and rounded
// once to an integer number of quanta; the two cells of the face add the
// same integer with opposite signs and the cell update o_new = o_n + sum of
// its six face integers is exact.  The per-variable totals over a periodic
// patch are therefore conserved exactly and their FP64 sums are exact.
//
// Reconstruction.  For the van Albada limiter the reference's two face-side
// states of a cell (upwind2.h:29-52 with vanalbada.h:28-33, evaluated once
// per face side, i.e. two limiter calls and four divisions per cell and
// direction) are U_c + s and U_c - s with the same slope
//     s = 1/2 * a*b*(a+b) / (a^2 + b^2),  a = U_c - U_{c-1},  b = U_{c+1} - U_c
// (phi(r) a / 2 with r = b/a, phi = (r^2+r)/(r^2+1), and phi(1/r) = phi(r)/r for
// the opposite side), so one division per cell, direction and variable gives
// both states.  s = 0 where c-1 or c+1 lies outside a closed patch (the
// reference's first-order fallback, upwind2.h:39-42).
//
// Element offsets are 32-bit: the host limits an FX32 patch to 5*ni*nj*kp <
// 2^31, kp being the row pitch along k (nk rounded up to a multiple of 4, so
// that every row starts on a 16-byte boundary, as TMA boxes need).
//
// Faces on tile and chunk borders are evaluated by both neighbouring CTAs;
// conservation needs both evaluations to give the same integer, so the
// translation unit is compiled without implicit multiply-add contraction
// (every FMA is written out with fmaf) and identical inputs always produce
// identical bits.
//
// Data flow per CTA: a TJ x TK tile of (j, k) columns marches along i.  Each
// plane of the stencil state (int32) with a two-cell halo in j and k is
// loaded into a shared-memory staging plane one iteration before its first
// use, by one TMA box load where the halo lies inside the patch, else cell
// by cell with cp.async (wrapped or clamped cells), and dequantised from
// there once into a three-plane FP32 ring; f(n) of the own cells arrives the
// same way.  x faces are evaluated per thread along its own column (the
// left state of the next face stays in registers); y and z face states and
// face integers are exchanged through shared memory.
#pragma once

#include <cstdint>
#include "fv_numerics.cuh"
#include "fv_wall.cuh"
#include "fv_tma.cuh"

namespace dn {

struct FxParams {
  float Ax, Ay, Az;
  float base[5];        // B_v rounded to FP32
  float quantum[5];     // q_v
  float face_scale[5];  // (factor/dV)/q_v
};

struct FxGeom {
  int ni, nj, nk;
  int kp;                // row pitch along k in elements (nk rounded up to a multiple of 4)
  int per_x, per_y, per_z;
  int i_chunk;
};

struct FxArgs {
  const int32_t* in;     // f(k-1) offsets, [5][ni][nj][nk]
  const int32_t* un;     // f(n) offsets (own cell)
  int32_t* out;          // f(k) offsets
  const uint8_t* active; // NULL = all active
  int* err;
  unsigned long long* err_info;
  FxGeom g;
  FxParams p;
  WallBC wall;           // patch-face fluxes of the non-periodic axes
};

constexpr int kFxLimit = 1 << 30;   // |o| must stay below this

// Primitive face-side state (COMPRESSIBLE_*_VARS): density, velocity,
// pressure, speed of sound and total enthalpy.  p = rho R T with
// T = (rE/rho - |u|^2/2)/cv, written as p = (R/cv) (rE - rho|u|^2/2).
struct Prim {
  float r, u, v, w, p, a, H;
};

__device__ __forceinline__ Prim fx_prim(float r, float ru, float rv, float rw, float rE)
{
  constexpr float R_over_cv = (float)(Gas::R / Gas::cv);
  constexpr float gam = (float)Gas::gamma;
  Prim s;
  const float ir = __fdividef(1.0f, r);
  s.r = r;
  s.u = ru * ir;
  s.v = rv * ir;
  s.w = rw * ir;
  const float ke2 = fmaf(rw, s.w, fmaf(rv, s.v, ru * s.u));   // rho |u|^2
  s.p = R_over_cv * fmaf(-0.5f, ke2, rE);
  const float p_ir = s.p * ir;
  s.a = sqrtf(gam * p_ir);
  s.H = fmaf(rE, ir, p_ir);                                    // (rho E + p) / rho
  return s;
}

// AUSM+ split Mach number and pressure polynomials of one face side
// (compressibleflux.h:46-75) in closed form:
//   s = +1:  M4 = 1/4 (M+1)^2 (1 + 1/2 (M-1)^2),  P5 = 1/4 (M+1)^2 ((2-M) + 3/4 M (M-1)^2)
//   s = -1:  M4 = -1/4 (M-1)^2 (1 + 1/2 (M+1)^2), P5 = 1/4 (M-1)^2 ((2+M) - 3/4 M (M+1)^2)
// for |M| < 1; for |M| >= 1, M4 = M1 = (M + s|M|)/2 and P5 = M1/M, which is
// exactly 1 when s*M > 0 and 0 otherwise (no division needed).
template <int S>
__device__ __forceinline__ void fx_split(float M, float& m4, float& p5)
{
  const float ap = M + 1.0f, am = M - 1.0f;
  const float ap2 = ap * ap, am2 = am * am;
  float sub_m4, sub_p5, sup_m4, sup_p5;
  if (S > 0) {
    sub_m4 = 0.25f * ap2 * fmaf(0.5f, am2, 1.0f);
    sub_p5 = 0.25f * ap2 * fmaf(0.75f * M, am2, 2.0f - M);
    sup_m4 = fmaxf(M, 0.0f);
    sup_p5 = M > 0.0f ? 1.0f : 0.0f;
  } else {
    sub_m4 = -0.25f * am2 * fmaf(0.5f, ap2, 1.0f);
    sub_p5 = 0.25f * am2 * fmaf(-0.75f * M, ap2, 2.0f + M);
    sup_m4 = fminf(M, 0.0f);
    sup_p5 = M < 0.0f ? 1.0f : 0.0f;
  }
  const bool sup = fabsf(M) >= 1.0f;
  m4 = sup ? sup_m4 : sub_m4;
  p5 = sup ? sup_p5 : sub_p5;
}

// AUSM+ flux (ausmplus.h:39-106) between face sides L and R, normal DIR.
// The reference's convective part h0 (phi_L + phi_R) - g0 (phi_R - phi_L)
// with h0 = f0/2, g0 = |f0|/2 is the upwind form max(f0, 0) phi_L +
// min(f0, 0) phi_R, evaluated here with one multiply-add per variable.
template <int DIR>
__device__ __forceinline__ void fx_ausm(const Prim& L, const Prim& R, float A, float F[5])
{
  const float unl = DIR == 0 ? L.u : (DIR == 1 ? L.v : L.w);
  const float unr = DIR == 0 ? R.u : (DIR == 1 ? R.v : R.w);
  const float a = 0.5f * (L.a + R.a);
  const float ia = __fdividef(1.0f, a);
  const float Ml = unl * ia, Mr = unr * ia;
  float m4l, p5l, m4r, p5r;
  fx_split<1>(Ml, m4l, p5l);
  fx_split<-1>(Mr, m4r, p5r);
  const float M = m4l + m4r;
  const float Mp = fmaxf(M, 0.0f);
  const float Mm = fminf(M, 0.0f);
  const float p = fmaf(p5l, L.p, p5r * R.p);
  const float f0 = a * A * fmaf(L.r, Mp, R.r * Mm);
  const float cp = fmaxf(f0, 0.0f);
  const float cm = fminf(f0, 0.0f);
  const float Ap = A * p;
  F[0] = f0;
  F[1] = DIR == 0 ? fmaf(cp, L.u, fmaf(cm, R.u, Ap)) : fmaf(cp, L.u, cm * R.u);
  F[2] = DIR == 1 ? fmaf(cp, L.v, fmaf(cm, R.v, Ap)) : fmaf(cp, L.v, cm * R.v);
  F[3] = DIR == 2 ? fmaf(cp, L.w, fmaf(cm, R.w, Ap)) : fmaf(cp, L.w, cm * R.w);
  F[4] = fmaf(cp, L.H, cm * R.H);
}

// Twice the van Albada slope shared by both face-side states of a cell,
// 2 s = a b (a + b) / (a^2 + b^2); the face states are U +- 0.5 * (2 s), one
// multiply-add each.  The denominator carries 1e-30, far below any nonzero
// a^2 + b^2 of offsets of at least one quantum, so that a = b = 0 gives 0
// without a test.
__device__ __forceinline__ float fx_slope(float a, float b)
{
  const float den = fmaf(a, a, fmaf(b, b, 1e-30f));
  return a * b * (a + b) * __fdividef(1.0f, den);
}

// ---------------------------------------------------------------------------
// Paired y/z evaluation.  Lane x of a pair carries a y-direction quantity of
// a cell, lane y the z-direction one; the halo cells and faces of the two
// directions share a thread, which halves the work of the threads that
// handle the tile's halo.  Every y and z slope and face of the kernel, own or
// halo, goes through these functions, so a face evaluated by two CTAs rounds
// identically.  (The packed f32x2 instructions of sm_100 measured no faster
// here than two scalar ones: the kernel is not FP32-pipe bound.)
__device__ __forceinline__ float2 v2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return make_float2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c)
{
  return make_float2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y));
}
__device__ __forceinline__ float2 rcp2(float2 a) { return make_float2(__fdividef(1.0f, a.x), __fdividef(1.0f, a.y)); }
__device__ __forceinline__ float2 max0(float2 a) { return make_float2(fmaxf(a.x, 0.0f), fmaxf(a.y, 0.0f)); }
__device__ __forceinline__ float2 min0(float2 a) { return make_float2(fminf(a.x, 0.0f), fminf(a.y, 0.0f)); }

struct Prim2 {
  float2 r, u, v, w, p, a, H;
};

__device__ __forceinline__ Prim2 fx_prim2(float2 r, float2 ru, float2 rv, float2 rw, float2 rE)
{
  constexpr float R_over_cv = (float)(Gas::R / Gas::cv);
  constexpr float gam = (float)Gas::gamma;
  Prim2 s;
  const float2 ir = rcp2(r);
  s.r = r;
  s.u = mul2(ru, ir);
  s.v = mul2(rv, ir);
  s.w = mul2(rw, ir);
  const float2 ke2 = fma2(rw, s.w, fma2(rv, s.v, mul2(ru, s.u)));
  s.p = mul2(v2(R_over_cv), fma2(v2(-0.5f), ke2, rE));
  const float2 p_ir = mul2(s.p, ir);
  const float2 t = mul2(v2(gam), p_ir);
  s.a = make_float2(sqrtf(t.x), sqrtf(t.y));
  s.H = fma2(rE, ir, p_ir);
  return s;
}

// fx_split for a pair of Mach numbers (both lanes on the same side S)
template <int S>
__device__ __forceinline__ void fx_split2(float2 M, float2& m4, float2& p5)
{
  const float2 ap = add2(M, v2(1.0f)), am = sub2(M, v2(1.0f));
  const float2 ap2 = mul2(ap, ap), am2 = mul2(am, am);
  float2 sub_m4, sub_p5;
  if (S > 0) {
    const float2 t = mul2(v2(0.25f), ap2);
    sub_m4 = mul2(t, fma2(v2(0.5f), am2, v2(1.0f)));
    sub_p5 = mul2(t, fma2(mul2(v2(0.75f), M), am2, sub2(v2(2.0f), M)));
  } else {
    const float2 t = mul2(v2(0.25f), am2);
    sub_m4 = mul2(v2(-1.0f), mul2(t, fma2(v2(0.5f), ap2, v2(1.0f))));
    sub_p5 = mul2(t, fma2(mul2(v2(-0.75f), M), ap2, add2(v2(2.0f), M)));
  }
  const bool supx = fabsf(M.x) >= 1.0f, supy = fabsf(M.y) >= 1.0f;
  if (S > 0) {
    m4.x = supx ? fmaxf(M.x, 0.0f) : sub_m4.x;
    m4.y = supy ? fmaxf(M.y, 0.0f) : sub_m4.y;
    p5.x = supx ? (M.x > 0.0f ? 1.0f : 0.0f) : sub_p5.x;
    p5.y = supy ? (M.y > 0.0f ? 1.0f : 0.0f) : sub_p5.y;
  } else {
    m4.x = supx ? fminf(M.x, 0.0f) : sub_m4.x;
    m4.y = supy ? fminf(M.y, 0.0f) : sub_m4.y;
    p5.x = supx ? (M.x < 0.0f ? 1.0f : 0.0f) : sub_p5.x;
    p5.y = supy ? (M.y < 0.0f ? 1.0f : 0.0f) : sub_p5.y;
  }
}

// fx_ausm for a y face (lane x, normal y) and a z face (lane y, normal z);
// A = (Ay, Az)
__device__ __forceinline__ void fx_ausm2(const Prim2& L, const Prim2& R, float2 A, float2 F[5])
{
  const float2 unl = make_float2(L.v.x, L.w.y);
  const float2 unr = make_float2(R.v.x, R.w.y);
  const float2 a = mul2(v2(0.5f), add2(L.a, R.a));
  const float2 ia = rcp2(a);
  float2 m4l, p5l, m4r, p5r;
  fx_split2<1>(mul2(unl, ia), m4l, p5l);
  fx_split2<-1>(mul2(unr, ia), m4r, p5r);
  const float2 M = add2(m4l, m4r);
  const float2 p = fma2(p5l, L.p, mul2(p5r, R.p));
  const float2 f0 = mul2(mul2(a, A), fma2(L.r, max0(M), mul2(R.r, min0(M))));
  const float2 cp = max0(f0), cm = min0(f0);
  const float2 Ap = mul2(A, p);
  F[0] = f0;
  F[1] = fma2(cp, L.u, mul2(cm, R.u));
  F[2] = fma2(cp, L.v, fma2(cm, R.v, make_float2(Ap.x, 0.0f)));
  F[3] = fma2(cp, L.w, fma2(cm, R.w, make_float2(0.0f, Ap.y)));
  F[4] = fma2(cp, L.H, mul2(cm, R.H));
}

// fx_slope (twice the van Albada slope) of a pair of (a, b) differences
__device__ __forceinline__ float2 fx_slope2(float2 a, float2 b)
{
  const float2 den = fma2(a, a, fma2(b, b, v2(1e-30f)));
  return mul2(mul2(mul2(a, b), add2(a, b)), rcp2(den));
}

// Cell whose state stands at index x of an axis: the wrapped cell on a
// periodic axis, the nearest edge cell outside a closed one.  Copying the
// edge cell outward makes the van Albada slope of an edge cell exactly zero
// (one of its differences vanishes), which is the reference's first-order
// reconstruction at a closed patch edge (upwind2.h:39-42), with no test.
// A face flux in whole quanta.  A face of 2^30 quanta or more (a single
// face moving the offset by the whole representable range) or a flux that is
// not finite would saturate or vanish in the int32 conversion; it is flagged
// instead of passing silently.
__device__ __forceinline__ int fx_quant(float x, bool& bad)
{
  bad |= !(fabsf(x) < 1073741824.0f);
  return __float2int_rn(x);
}

__device__ __forceinline__ int fx_index(int x, int n, int per)
{
  if (per) {
    x %= n;
    return x < 0 ? x + n : x;
  }
  return x < 0 ? 0 : (x >= n ? n - 1 : x);
}

__device__ __forceinline__ bool fx_face_exists(int x, int n, int per)
{
  if (n <= 2) return false;
  return per ? true : (x >= 1 && x <= n - 1);
}

// Shared memory of a CTA.  Every array starts on a 128-byte boundary and is
// laid out so that a warp's accesses hit distinct banks: the plane ring
// stores rows in interleaved pairs ([row/2][col][row%2]), since a warp of a
// 16-wide tile spans two rows; the z arrays keep own columns at stride TK
// and park the one extra (halo) column of each row in the bank the own
// columns leave free.  The staging area holds the next plane as stored
// (int32) until it is dequantised into the ring: a main box of rows j0-2 ..
// j0+TJ+1 and columns k0-4 .. k0+TK+3 (plain rows; the column origin k0-4
// keeps a TMA box on a 16-byte boundary), and, for tiles at the seam of a
// periodic axis, the wrapped columns (k side box, 4 wide), the wrapped rows
// (j side box, 2 high) and their corner.
template <int TJ, int TK>
struct FxSmem {
  static constexpr int PJ = TJ + 4;
  static constexpr int PK = TK + 4;
  static constexpr int SK = TK + 8;              // main box row: columns k0-4 .. k0+TK+3
  static constexpr int NW = TJ * TK / 32;        // warps of a CTA
  // Side boxes only for 16-wide tiles: with them the 32-wide tile's shared
  // memory would leave room for two CTAs per SM instead of three (its
  // tiles at a periodic seam copy cell by cell).
  static constexpr bool SEAMS = TK <= 16;
  static constexpr int up128(int n) { return (n + 31) / 32 * 32; }   // int32 count to 128 bytes
  static constexpr int ST_M = 0;                                   // main box [5][PJ][SK]
  static constexpr int ST_K = ST_M + up128(5 * PJ * SK);           // k side box [5][PJ][4]
  static constexpr int ST_J = ST_K + (SEAMS ? up128(5 * PJ * 4) : 0);   // j side box [5][2][SK]
  static constexpr int ST_C = ST_J + (SEAMS ? up128(5 * 2 * SK) : 0);   // corner box [5][2][4]
  static constexpr int ST_N = ST_C + (SEAMS ? up128(5 * 2 * 4) : 0);
  alignas(128) float plane[3][5][PJ / 2][PK][2]; // dequantised state, ring over planes i .. i+2
  alignas(128) int stage[ST_N];                  // plane i+3 as stored, on its way into the ring
  alignas(128) int un[5][TJ][TK];                // f(n) of the own cells of the current plane
  alignas(128) float sy[5][TJ + 1][TK];          // y: left state of the face above row jj-1 (row -1 .. TJ-1)
  alignas(128) float sy_top[5][TK];              // y: right state of the face below row TJ (halo)
  alignas(128) float szL[5][TJ][TK];             // z: left state of the face above col kk (own columns)
  alignas(128) float szH[5][NW][32];             // z: left state of the face above col -1 (halo), see zh_slot
  alignas(128) float sz_top[5][TJ];              // z: right state of the face below col TK (halo)
  alignas(128) int qy[5][TJ + 1][TK];            // y face integers, face below row jj
  alignas(128) int qzL[5][TJ][TK];               // z face integers, face below col kk (own columns)
  alignas(128) int qzT[5][NW][32];               // z face integers, face below col TK (halo), see zt_slot
  alignas(8) uint64_t bar[2];                    // mbarriers of the TMA loads: staging plane, f(n)
};

// bank-free slots of the per-row halo values of the z arrays
template <int TK> __device__ __forceinline__ int zh_slot(int row) { return (row * TK + TK - 1) & 31; }
template <int TK> __device__ __forceinline__ int zt_slot(int row) { return (row * TK) & 31; }
template <int TK> __device__ __forceinline__ int z_warp(int row) { return (row * TK) >> 5; }

__device__ __forceinline__ void fx_cp_async4(void* smem, const void* gmem)
{
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" :: "r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void fx_cp_async_commit()
{
  asm volatile("cp.async.commit_group;" ::: "memory");
}

template <int N>
__device__ __forceinline__ void fx_cp_async_wait()
{
  asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory");
}

// Is the tile "full": every own column inside the patch and, on closed j/k
// axes, two more rows/columns of cells on both sides, so that every y/z
// slope and face of the tile exists?  Such tiles (almost all of a large
// patch) run a form of the tile function without the per-thread edge tests.
template <int TJ, int TK>
__device__ __forceinline__ bool fx_tile_full(const FxGeom& g, int j0, int k0)
{
  const bool fy = (j0 + TJ <= g.nj) && (g.per_y || (j0 >= 2 && j0 + TJ + 2 <= g.nj));
  const bool fz = (k0 + TK <= g.nk) && (g.per_z || (k0 >= 2 && k0 + TK + 2 <= g.nk));
  return fy && fz;
}

// Device error bit of a TMA transfer that did not complete within the
// bounded wait.
constexpr int kFxErrTma = 32;

// Tensor maps of the stage input of a patch, one per box: main (TK+8 x
// TJ+4), k side (4 x TJ+4), j side (TK+8 x 2), corner (4 x 2), each x 1
// plane x 5 variables.
constexpr int kFxMapMain = 0, kFxMapK = 1, kFxMapJ = 2, kFxMapC = 3, kFxMaps = 4;

// Where a tile's halo along one axis comes from when its planes are staged
// by TMA: 0 inside the patch or clamped (closed axis), 1 wrapped below the
// first cell, 2 wrapped above the last cell; -1 not stageable by TMA (a
// periodic axis whose tile needs both ends, or a ragged tile at the seam).
__device__ __forceinline__ int fx_seam(int t0, int T, int n, int per)
{
  if (!per || (t0 >= 2 && t0 + T + 2 <= n)) return 0;
  if (t0 == 0 && n >= T + 2) return 1;
  if (t0 >= 2 && t0 + T == n) return 2;
  return -1;
}

// One tile of one patch: columns (j0 .. j0+TJ-1, k0 .. k0+TK-1), planes i0 .. i1-1.
// tm_in: the kFxMaps tensor maps of the stage input, tm_un: the map of f(n)
// (box TK x TJ x 1 x 5), or null.  With maps, a tile stages its planes by
// TMA box loads unless fx_seam excludes it; closed-axis cells outside the
// patch then read the edge cell's slot of the main box, and the cells across
// the seam of a periodic axis come from the side boxes.  Other tiles copy
// cell by cell.
template <int TJ, int TK, bool FULL>
__device__ __forceinline__ void fx_stage_tile_impl(const FxArgs& a, const CUtensorMap* tm_in,
                                                   const CUtensorMap* tm_un, int j0, int k0, int i0, int i1)
{
  constexpr int NT = TJ * TK;
  constexpr int PJ = TJ + 4, PK = TK + 4;
  constexpr int NP = PJ * PK;                     // positions of a plane tile (per variable)
  constexpr int PPT = (NP + NT - 1) / NT;         // positions per thread
  using Smem = FxSmem<TJ, TK>;
  constexpr int SK = Smem::SK;
  extern __shared__ __align__(128) unsigned char fx_smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(fx_smem_raw);

  const FxGeom& g = a.g;
  const FxParams& P = a.p;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * TK + tx;
  const int j = j0 + ty, k = k0 + tx;
  const bool own = FULL || ((j < g.nj) && (k < g.nk));
  const int njk = g.nj * g.kp;                    // plane stride (rows of kp elements)
  const size_t nc = (size_t)g.ni * njk;           // variable stride
  // TMA boxes start at x = k0-4 (main; a multiple of 4 int32 since TK is),
  // k0 (f(n)), and nk-4 or 0 (k side box): the first seam tile of a periodic
  // k axis needs nk % 4 == 0 for its side box (the last one has k0+TK = nk,
  // a multiple of 4 already); box cells beyond the patch are zero-filled and
  // never read; destinations 128-byte aligned
  const int seam_j = fx_seam(j0, TJ, g.nj, g.per_y);
  const int seam_k = fx_seam(k0, TK, g.nk, g.per_z);
  const bool tma = tm_in != nullptr && seam_j >= 0 && seam_k >= 0 && (Smem::SEAMS || (seam_j | seam_k) == 0) &&
                   (seam_k != 1 || (g.nk & 3) == 0) &&
                   ((smem_u32(&sm.stage[0]) | smem_u32(&sm.un[0][0][0])) & 127) == 0;

  // plane element (jj, kk) of variable v in ring slot sl (rows interleaved in pairs)
  auto PL = [&](int sl, int v, int jj, int kk) -> float& { return sm.plane[sl][v][jj >> 1][kk][jj & 1]; };

  // per-thread plane positions e = tid + m*NT in ring order [row/2][col][row%2]:
  // in-plane offset j*nk + k of the (wrapped, or on closed axes clamped)
  // column, and where the position's cell lies in the staging area: offset
  // of variable 0 and the stride between variables of its box (cell copies
  // fill the main box position by position)
  int32_t poff[PPT];
  int32_t soff[PPT];
  int32_t svar[PPT];
  #pragma unroll
  for (int m = 0; m < PPT; ++m) {
    const int e = tid + m * NT;
    poff[m] = -1;
    soff[m] = 0;
    svar[m] = PJ * SK;
    if (e < NP) {
      const int jj = (e / (2 * PK)) * 2 + (e & 1);
      const int kk = (e % (2 * PK)) >> 1;
      const int jg = j0 - 2 + jj, kg = k0 - 2 + kk;
      poff[m] = fx_index(jg, g.nj, g.per_y) * g.kp + fx_index(kg, g.nk, g.per_z);
      soff[m] = Smem::ST_M + jj * SK + kk + 2;
      if (tma) {
        // row: in the main box (clamped on a closed axis) or across the seam
        const bool jside = g.per_y && (jg < 0 || jg >= g.nj);
        const int jr = jside ? (jg < 0 ? jg + 2 : jg - g.nj) : (g.per_y ? jg : min(max(jg, 0), g.nj - 1)) - (j0 - 2);
        const bool kside = g.per_z && (kg < 0 || kg >= g.nk);
        const int kr = kside ? (kg < 0 ? kg + 4 : kg - g.nk) : (g.per_z ? kg : min(max(kg, 0), g.nk - 1)) - (k0 - 4);
        if (jside) {
          soff[m] = (kside ? Smem::ST_C + jr * 4 : Smem::ST_J + jr * SK) + kr;
          svar[m] = kside ? 2 * 4 : 2 * SK;
        } else {
          soff[m] = (kside ? Smem::ST_K + jr * 4 : Smem::ST_M + jr * SK) + kr;
          svar[m] = kside ? PJ * 4 : PJ * SK;
        }
      }
    }
  }

  // plane ip of the stage input, copied cell by cell (cp.async) as int32
  // into ring slot sl, then dequantised there in place by the copying thread
  auto issue_ring = [&](int sl, int ip) {
    int* dst = reinterpret_cast<int*>(&sm.plane[sl][0][0][0][0]);
    const int32_t* src = a.in + (size_t)fx_index(ip, g.ni, g.per_x) * njk;
    #pragma unroll
    for (int v = 0; v < 5; ++v) {
      #pragma unroll
      for (int m = 0; m < PPT; ++m) {
        const int e = tid + m * NT;
        if (e < NP) fx_cp_async4(dst + v * NP + e, src + (size_t)v * nc + poff[m]);
      }
    }
  };
  auto dequant_ring = [&](int sl) {
    float* f = &sm.plane[sl][0][0][0][0];
    const int* q = reinterpret_cast<const int*>(f);
    #pragma unroll
    for (int v = 0; v < 5; ++v) {
      #pragma unroll
      for (int m = 0; m < PPT; ++m) {
        const int e = tid + m * NT;
        if (e < NP) f[v * NP + e] = fmaf(P.quantum[v], (float)q[v * NP + e], P.base[v]);
      }
    }
  };
  // plane ip into the staging plane, cell by cell (tiles without TMA)
  auto issue_stage = [&](int ip) {
    int* dst = &sm.stage[0];
    const int32_t* src = a.in + (size_t)fx_index(ip, g.ni, g.per_x) * njk;
    #pragma unroll
    for (int v = 0; v < 5; ++v) {
      #pragma unroll
      for (int m = 0; m < PPT; ++m) {
        const int e = tid + m * NT;
        if (e < NP) fx_cp_async4(dst + soff[m] + v * svar[m], src + (size_t)v * nc + poff[m]);
      }
    }
  };
  // the staging area, dequantised into ring slot sl
  auto dequant_stage = [&](int sl) {
    float* f = &sm.plane[sl][0][0][0][0];
    const int* q = &sm.stage[0];
    #pragma unroll
    for (int v = 0; v < 5; ++v) {
      #pragma unroll
      for (int m = 0; m < PPT; ++m) {
        const int e = tid + m * NT;
        if (e < NP) f[v * NP + e] = fmaf(P.quantum[v], (float)q[soff[m] + v * svar[m]], P.base[v]);
      }
    }
  };
  // f(n) of the own cell, plane ip, cell by cell (tiles without TMA)
  auto fetch_un = [&](int ip) {
    if (own) {
      const int c = ip * njk + j * g.kp + k;
      #pragma unroll
      for (int v = 0; v < 5; ++v) fx_cp_async4(&sm.un[v][ty][tx], a.un + (size_t)v * nc + c);
    }
  };
  // TMA loads of f(n) of plane ip and, if wanted, of stage-input plane ip+3
  // (one thread; the barrier before it ended every read of both buffers)
  auto issue_tma = [&](int ip, bool plane_too) {
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&sm.bar[1], 5u * TJ * TK * 4u);
    tma_load_4d(&sm.un[0][0][0], tm_un, &sm.bar[1], k0, j0, ip, 0);
    if (plane_too) {
      const int pl = fx_index(ip + 3, g.ni, g.per_x);
      const int xs = seam_k == 1 ? g.nk - 4 : 0;     // k side box: the wrapped columns
      const int ys = seam_j == 1 ? g.nj - 2 : 0;     // j side box: the wrapped rows
      const unsigned bytes = 5u * 4u * (PJ * SK + (seam_k ? PJ * 4 : 0) + (seam_j ? 2 * SK : 0) +
                                        (seam_j && seam_k ? 2 * 4 : 0));
      mbar_arrive_expect_tx(&sm.bar[0], bytes);
      tma_load_4d(&sm.stage[Smem::ST_M], tm_in + kFxMapMain, &sm.bar[0], k0 - 4, j0 - 2, pl, 0);
      if (seam_k) tma_load_4d(&sm.stage[Smem::ST_K], tm_in + kFxMapK, &sm.bar[0], xs, j0 - 2, pl, 0);
      if (seam_j) tma_load_4d(&sm.stage[Smem::ST_J], tm_in + kFxMapJ, &sm.bar[0], k0 - 4, ys, pl, 0);
      if (seam_j && seam_k) tma_load_4d(&sm.stage[Smem::ST_C], tm_in + kFxMapC, &sm.bar[0], xs, ys, pl, 0);
    }
  };

  if (tma && tid == 0) {
    mbar_init(&sm.bar[0], 1);
    mbar_init(&sm.bar[1], 1);
    mbar_init_fence();
  }

  // prologue: planes i0 .. i0+2 in the ring (the barrier below also
  // publishes the mbarrier initialisation)
  for (int q = 0; q <= 2; ++q) issue_ring(q, i0 + q);
  fx_cp_async_commit();
  fx_cp_async_wait<0>();
  for (int q = 0; q <= 2; ++q) dequant_ring(q);
  __syncthreads();

  // x direction registers: left state of the face above the current cell,
  // the downwind difference of the current cell, and the lower face integers
  bool fbad = false;     // a face flux left the fixed-point range (fx_quant)
  bool tbad = false;     // a TMA wait ran out
  Prim xleft;
  float xb[5];           // U_{i+1} - U_i of the own column (becomes a of cell i+1)
  int qx_lo[5];
  {
    // slope of cell i0 (needs i0-1, i0, i0+1) and the face below i0; planes
    // i0-1 and i0-2 of the own column come straight from the stage input
    const int64_t col = (int64_t)j * g.kp + k;
    const int iw1 = fx_index(i0 - 1, g.ni, g.per_x);
    float Ul[5], Sp[5], Sm[5];
    float U0[5];
    #pragma unroll
    for (int v = 0; v < 5; ++v) {
      const float um = own ? fmaf(P.quantum[v], (float)__ldg(a.in + (int64_t)v * nc + (int64_t)iw1 * njk + col), P.base[v])
                           : 0.0f;
      const float uc = PL(0, v, ty + 2, tx + 2);
      const float up = PL(1, v, ty + 2, tx + 2);
      const float s = fx_slope(uc - um, up - uc);
      U0[v] = uc;
      Sp[v] = fmaf(s, 0.5f, uc);
      Sm[v] = fmaf(s, -0.5f, uc);
      xb[v] = up - uc;
      Ul[v] = um;
    }
    xleft = fx_prim(Sp[0], Sp[1], Sp[2], Sp[3], Sp[4]);
    // face below i0: left state from cell i0-1 (slope needs i0-2)
    const bool ex = own && fx_face_exists(i0, g.ni, g.per_x);
    if (ex) {
      const int iw2 = fx_index(i0 - 2, g.ni, g.per_x);
      float Lm[5];
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        const float umm = fmaf(P.quantum[v], (float)__ldg(a.in + (int64_t)v * nc + (int64_t)iw2 * njk + col), P.base[v]);
        Lm[v] = fmaf(fx_slope(Ul[v] - umm, U0[v] - Ul[v]), 0.5f, Ul[v]);
      }
      float F[5];
      fx_ausm<0>(fx_prim(Lm[0], Lm[1], Lm[2], Lm[3], Lm[4]), fx_prim(Sm[0], Sm[1], Sm[2], Sm[3], Sm[4]), P.Ax, F);
      #pragma unroll
      for (int v = 0; v < 5; ++v) qx_lo[v] = fx_quant(F[v] * P.face_scale[v], fbad);
    } else {
      #pragma unroll
      for (int v = 0; v < 5; ++v) qx_lo[v] = 0;
    }
  }

  int s0 = 0, sp1 = 1, sp2 = 2;       // ring slots of planes i, i+1, i+2
  unsigned ph_plane = 0, ph_un = 0;   // parities of the next TMA completions
  for (int i = i0; i < i1; ++i) {
    const bool more = i + 3 <= i1 + 1;  // plane i+3 is read by a later iteration

    // ---------------- y and z face states of plane i
    float2 yzm[5];   // right states of the y (lane x) and z (lane y) faces below the own cell
    {
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        const float2 uc = v2(PL(s0, v, ty + 2, tx + 2));
        const float2 ul = make_float2(PL(s0, v, ty + 1, tx + 2), PL(s0, v, ty + 2, tx + 1));
        const float2 uh = make_float2(PL(s0, v, ty + 3, tx + 2), PL(s0, v, ty + 2, tx + 3));
        const float2 s = fx_slope2(sub2(uc, ul), sub2(uh, uc));
        const float2 up = fma2(s, v2(0.5f), uc);
        sm.sy[v][ty + 1][tx] = up.x;
        sm.szL[v][ty][tx] = up.y;
        yzm[v] = fma2(s, v2(-0.5f), uc);
      }
    }
    // halo cells, y and z in pairs: y rows -1 (left state) and TJ (right
    // state), z cols -1 and TK
    for (int h = tid; h < 2 * (TK > TJ ? TK : TJ); h += NT) {
      const bool hy = h < 2 * TK, hz = h < 2 * TJ;
      const int kky = h % TK;
      const bool topy = h >= TK;
      const int jjy = topy ? TJ : -1;                 // tile-relative row of the y cell
      const int jjz = h % TJ;
      const bool topz = h >= TJ;
      const int kkz = topz ? TK : -1;                 // tile-relative col of the z cell
      // a lane without a cell evaluates the other lane's cell and stores nothing
      const int ry = hy ? jjy + 2 : jjz + 2, cy = hy ? kky + 2 : kkz + 2;
      const int rz = hz ? jjz + 2 : jjy + 2, cz = hz ? kkz + 2 : kky + 2;
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        const float2 uc = make_float2(PL(s0, v, ry, cy), PL(s0, v, rz, cz));
        const float2 ul = make_float2(PL(s0, v, ry - 1, cy), PL(s0, v, rz, cz - 1));
        const float2 uh = make_float2(PL(s0, v, ry + 1, cy), PL(s0, v, rz, cz + 1));
        const float2 s = fx_slope2(sub2(uc, ul), sub2(uh, uc));
        const float2 up = fma2(s, v2(0.5f), uc), dn = fma2(s, v2(-0.5f), uc);
        if (hy) {
          if (topy) sm.sy_top[v][kky] = dn.x;
          else sm.sy[v][0][kky] = up.x;
        }
        if (hz) {
          if (topz) sm.sz_top[v][jjz] = dn.y;
          else sm.szH[v][z_warp<TK>(jjz)][zh_slot<TK>(jjz)] = up.y;
        }
      }
    }
    __syncthreads();

    // every read of the staging plane (dequantised at the end of the last
    // iteration) and of f(n) (the last update) preceded this barrier: load
    // f(n) of plane i and stage-input plane i+3 into them
    if (tma) {
      if (tid == 0) issue_tma(i, more);
    } else {
      fetch_un(i);
      fx_cp_async_commit();
      if (more) issue_stage(i + 3);
      fx_cp_async_commit();
    }

    // ---------------- y and z faces below the own cell (+ the top halo faces)
    {
      // the face below row j is needed even when row j itself lies beyond a
      // periodic patch (it is the wrapped face above the last row)
      const bool exy = FULL || (k < g.nk && fx_face_exists(j, g.nj, g.per_y) && (g.per_y || j < g.nj));
      const bool exz = FULL || (j < g.nj && fx_face_exists(k, g.nk, g.per_z) && (g.per_z || k < g.nk));
      float2 L[5];
      #pragma unroll
      for (int v = 0; v < 5; ++v)
        L[v] = make_float2(sm.sy[v][ty][tx], tx > 0 ? sm.szL[v][ty][tx - 1] : sm.szH[v][z_warp<TK>(ty)][zh_slot<TK>(ty)]);
      float2 F[5];
      fx_ausm2(fx_prim2(L[0], L[1], L[2], L[3], L[4]), fx_prim2(yzm[0], yzm[1], yzm[2], yzm[3], yzm[4]),
               make_float2(P.Ay, P.Az), F);
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        const float2 q = mul2(F[v], v2(P.face_scale[v]));
        sm.qy[v][ty][tx] = exy ? fx_quant(q.x, fbad) : 0;
        sm.qzL[v][ty][tx] = exz ? fx_quant(q.y, fbad) : 0;
      }
    }
    // halo faces, y and z in pairs: below halo row TJ (col kk = h) and below
    // halo col TK (row jj = h)
    // (on the second warp: the first one did the halo slopes of this plane)
    for (int h = (tid + NT - 32) % NT; h < (TK > TJ ? TK : TJ); h += NT) {
      const bool hy = h < TK, hz = h < TJ;
      bool exy = hy, exz = hz;
      if (!FULL) {
        const int jf = j0 + TJ, kf = k0 + h;
        exy = exy && kf < g.nk && fx_face_exists(jf, g.nj, g.per_y) && (g.per_y || jf < g.nj);
        const int jz = j0 + h, kz = k0 + TK;
        exz = exz && jz < g.nj && fx_face_exists(kz, g.nk, g.per_z) && (g.per_z || kz < g.nk);
      }
      // a lane without a face evaluates the other lane's face and stores nothing
      const int ky = hy ? h : 0, jz = hz ? h : 0;
      float2 L[5], R[5];
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        L[v] = make_float2(sm.sy[v][TJ][ky], sm.szL[v][jz][TK - 1]);
        R[v] = make_float2(sm.sy_top[v][ky], sm.sz_top[v][jz]);
      }
      float2 F[5];
      fx_ausm2(fx_prim2(L[0], L[1], L[2], L[3], L[4]), fx_prim2(R[0], R[1], R[2], R[3], R[4]),
               make_float2(P.Ay, P.Az), F);
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        const float2 q = mul2(F[v], v2(P.face_scale[v]));
        if (hy) sm.qy[v][TJ][h] = exy ? fx_quant(q.x, fbad) : 0;
        if (hz) sm.qzT[v][z_warp<TK>(h)][zt_slot<TK>(h)] = exz ? fx_quant(q.y, fbad) : 0;
      }
    }
    // ---------------- x: face above cell i (between i and i+1)
    int qx_hi[5];
    {
      const bool ex = own && fx_face_exists(i + 1, g.ni, g.per_x);
      float Sm[5], Sp[5];
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        const float uc = PL(sp1, v, ty + 2, tx + 2);
        const float up = PL(sp2, v, ty + 2, tx + 2);
        const float b = up - uc;
        const float s = fx_slope(xb[v], b);
        Sm[v] = fmaf(s, -0.5f, uc);
        Sp[v] = fmaf(s, 0.5f, uc);
        xb[v] = b;
      }
      if (ex) {
        float F[5];
        fx_ausm<0>(xleft, fx_prim(Sm[0], Sm[1], Sm[2], Sm[3], Sm[4]), P.Ax, F);
        #pragma unroll
        for (int v = 0; v < 5; ++v) qx_hi[v] = fx_quant(F[v] * P.face_scale[v], fbad);
      } else {
        #pragma unroll
        for (int v = 0; v < 5; ++v) qx_hi[v] = 0;
      }
      xleft = fx_prim(Sp[0], Sp[1], Sp[2], Sp[3], Sp[4]);
    }

    __syncthreads();

    // ---------------- residual and update of the own cell
    // f(n) of plane i has arrived (the staging copy may stay in flight)
    if (tma) {
      tbad |= !mbar_wait(&sm.bar[1], ph_un);
      ph_un ^= 1u;
    } else {
      fx_cp_async_wait<1>();
    }
    if (own) {
      const int c = i * njk + j * g.kp + k;       // 5*ni*nj*kp < 2^31 (host check)
      const int ncv = (int)nc;
      const bool act = a.active ? (a.active[c] != 0) : true;
      int bad = 0;
      int res[5];
      #pragma unroll
      for (int v = 0; v < 5; ++v)
        res[v] = qx_lo[v] + sm.qy[v][ty][tx] + sm.qzL[v][ty][tx]
               - (tx < TK - 1 ? sm.qzL[v][ty][tx + 1] : sm.qzT[v][z_warp<TK>(ty)][zt_slot<TK>(ty)])
               - sm.qy[v][ty + 1][tx] - qx_hi[v];
      if (a.wall.any && (i == 0 || i == g.ni - 1 || j == 0 || j == g.nj - 1 || k == 0 || k == g.nk - 1)) {
        // the cell's state, re-read from the stage input: the ring slot of
        // plane i receives plane i+3 below, with no barrier in between
        float uc[5];
        #pragma unroll
        for (int v = 0; v < 5; ++v) uc[v] = fmaf(P.quantum[v], (float)a.in[v * ncv + c], P.base[v]);
        add_wall_fluxes(a.wall, g.ni, g.nj, g.nk, g.per_x, g.per_y, g.per_z, i, j, k, uc, P.Ax, P.Ay, P.Az, res,
                        [&](int v, float F) { return fx_quant(F * P.face_scale[v], fbad); });
      }
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        int32_t o;
        if (act) {
          const int r = res[v];
          const int un = sm.un[v][ty][tx];
          // |un| < 2^30 and |r| < 2^30 (face integers are bounded by the
          // exact range of the update), so the int32 sum cannot overflow
          const int on = un + r;
          if (on >= kFxLimit || on <= -kFxLimit) {
            bad |= 1;
            if (a.err_info && atomicCAS(&a.err_info[0], ~0ull, (unsigned long long)c) == ~0ull) {
              a.err_info[1] = (unsigned long long)v;
              a.err_info[2] = (unsigned long long)__double_as_longlong((double)un);
              a.err_info[3] = (unsigned long long)__double_as_longlong((double)r);
            }
          }
          o = on;
        } else {
          o = a.in[v * ncv + c];
        }
        a.out[v * ncv + c] = o;
      }
      if (bad && a.err) atomicOr(a.err, bad);
    }
    #pragma unroll
    for (int v = 0; v < 5; ++v) {
      qx_lo[v] = qx_hi[v];
    }

    // ---------------- ring: plane i (last read before this iteration's
    // first barrier) gives its slot to plane i+3, dequantised from the
    // staging plane; the next iteration's first barrier publishes it
    if (more) {
      if (tma) {
        tbad |= !mbar_wait(&sm.bar[0], ph_plane);
        ph_plane ^= 1u;
      } else {
        fx_cp_async_wait<0>();
      }
      dequant_stage(s0);
    }
    const int t = s0;
    s0 = sp1;
    sp1 = sp2;
    sp2 = t;
  }
  if (fbad && a.err) atomicOr(a.err, 16);
  if (tbad && a.err) atomicOr(a.err, kFxErrTma);
}

template <int TJ, int TK>
__device__ __forceinline__ void fx_stage_tile(const FxArgs& a, const CUtensorMap* tm_in, const CUtensorMap* tm_un,
                                              int j0, int k0, int i0, int i1)
{
  if (fx_tile_full<TJ, TK>(a.g, j0, k0)) fx_stage_tile_impl<TJ, TK, true>(a, tm_in, tm_un, j0, k0, i0, i1);
  else fx_stage_tile_impl<TJ, TK, false>(a, tm_in, tm_un, j0, k0, i0, i1);
}

// Resident CTAs per SM the register allocation is sized for: three
// 256-thread CTAs (80 registers, 55-58 KB shared memory each) measured 26 %
// faster than two on the 256^3 patch.
#ifndef DN_FX_MIN_BLOCKS
#define DN_FX_MIN_BLOCKS 3
#endif

// Parameters of the single-patch launch: the stage arguments and the tensor
// maps of the stage input and of f(n) (valid when tma != 0).
struct FxLaunch {
  CUtensorMap tm_in[kFxMaps];
  CUtensorMap tm_un;
  FxArgs a;
  int tma;
};

// One patch per launch: grid (k tiles, j tiles, i chunks).
template <int TJ, int TK>
__global__ void __launch_bounds__(TJ * TK, DN_FX_MIN_BLOCKS)
fx_stage_kernel(const __grid_constant__ FxLaunch L)
{
  const int i0 = blockIdx.z * L.a.g.i_chunk;
  fx_stage_tile<TJ, TK>(L.a, L.tma ? L.tm_in : nullptr, L.tma ? &L.tm_un : nullptr, blockIdx.y * TJ,
                        blockIdx.x * TK, i0, min(L.a.g.ni, i0 + L.a.g.i_chunk));
}

} // namespace dn
