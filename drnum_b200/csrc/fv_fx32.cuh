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
// (every FMA is written out) and identical inputs always produce identical
// bits.
//
// Work decomposition.  A thread owns two neighbouring cells of a row, (j, k)
// and (j, k+1) with k even, and evaluates everything of the pair with the
// packed FP32 instructions of sm_100 (__ffma2_rn, __fmul2_rn, __fadd2_rn: one
// instruction for both cells): the kernel is bound by instruction issue, not
// by memory bandwidth or the FP32 pipes, so halving the arithmetic
// instructions is what speeds it up.  A CTA owns a TJ x TK tile of (j, k)
// columns and marches along i through a range of planes.  Each plane of the
// stencil state (int32) with a two-cell halo in j and k is loaded into a
// shared-memory staging plane one iteration before its first use, by TMA box
// loads where the halo lies inside the patch or across a periodic seam, else
// cell by cell with cp.async, and dequantised from there once into a
// three-plane FP32 ring; f(n) of the own cells arrives the same way.  Per
// plane:
//   A  slopes of the own pair in y and z (and of the tile's halo rows and
//      columns); the face-side states the neighbours need go to shared memory
//   B  y and z faces below the own cells (the z face between the two cells
//      of a pair never leaves the thread) and the x face above them, along
//      the thread's own column (the left state of the next x face stays in
//      registers); face integers go to shared memory
//   C  residual and update of the own cells, then the plane three ahead is
//      dequantised into the ring slot this plane leaves.
#pragma once

#include <cstdint>
#include "fv_numerics.cuh"
#include "fv_wall.cuh"
#include "fv_tma.cuh"

namespace dn {

// Stage parameters, each held twice (as the pair arithmetic consumes them:
// one 64-bit constant load per use).
struct FxParams {
  float2 A[3];          // face areas of the x, y and z faces
  float2 base[5];       // B_v rounded to FP32
  float2 quantum[5];    // q_v
  float2 face_scale[5]; // (factor/dV)/q_v
};

// The parameters of a stage with RK factor alpha*dt of a patch with spacings
// (dx, dy, dz) and fixed-point base and quantum (the single-patch launch and
// the batched kernel both call this, so their parameters are identical).
__host__ __device__ inline void fx_set_params(FxParams& p, double dx, double dy, double dz, double factor,
                                              const double* base, const double* quantum)
{
  const float ax = (float)(dy * dz), ay = (float)(dx * dz), az = (float)(dx * dy);
  p.A[0] = make_float2(ax, ax);
  p.A[1] = make_float2(ay, ay);
  p.A[2] = make_float2(az, az);
  const double pf = factor / (dx * dy * dz);
  for (int v = 0; v < 5; ++v) {
    const float b = (float)base[v], q = (float)quantum[v], f = (float)(pf / quantum[v]);
    p.base[v] = make_float2(b, b);
    p.quantum[v] = make_float2(q, q);
    p.face_scale[v] = make_float2(f, f);
  }
}

struct FxGeom {
  int ni, nj, nk;
  int kp;                // row pitch along k in elements (nk rounded up to a multiple of 4)
  int per_x, per_y, per_z;
  int i_chunk;
};

struct FxArgs {
  const int32_t* in;     // f(k-1) offsets, [5][ni][nj][kp]
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

// Face integers of at most this magnitude keep any cell's residual (at most
// six faces) inside int32: 6 * 1.25 * 2^28 < 2^31.  While every face of a
// CTA's plane stays below it the residuals are summed in 32 bits; otherwise
// that plane sums them in 64 bits.  Either way the result is exact.
constexpr float kFxNarrowFace = 335544320.0f;    // 1.25 * 2^28
constexpr float kFxFaceLimit = 1073741824.0f;    // 2^30: a face this large is an error

// ---------------------------------------------------------------------------
// Packed pair arithmetic: lane x belongs to the cell (or face) at k, lane y
// to the one at k+1.
__device__ __forceinline__ float2 v2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b as one packed multiply-add, b * (-1) + a (the product is exact, so
// the result is the correctly rounded difference)
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 rcp2(float2 a) { return make_float2(__fdividef(1.0f, a.x), __fdividef(1.0f, a.y)); }
__device__ __forceinline__ float2 sqrt2(float2 a) { return make_float2(sqrtf(a.x), sqrtf(a.y)); }
__device__ __forceinline__ float2 max0(float2 a) { return make_float2(fmaxf(a.x, 0.0f), fmaxf(a.y, 0.0f)); }
__device__ __forceinline__ float2 min0(float2 a) { return make_float2(fminf(a.x, 0.0f), fminf(a.y, 0.0f)); }

// Primitive face-side state (COMPRESSIBLE_*_VARS) of a pair: density,
// velocity, pressure, speed of sound and total enthalpy.  p = rho R T with
// T = (rE/rho - |u|^2/2)/cv, written as p = (R/cv) (rE - rho|u|^2/2).
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
  const float2 ke2 = fma2(rw, s.w, fma2(rv, s.v, mul2(ru, s.u)));   // rho |u|^2
  s.p = mul2(v2(R_over_cv), fma2(v2(-0.5f), ke2, rE));
  const float2 p_ir = mul2(s.p, ir);
  s.a = sqrt2(mul2(v2(gam), p_ir));
  s.H = fma2(rE, ir, p_ir);                                          // (rho E + p) / rho
  return s;
}

// AUSM+ split Mach number and pressure polynomials of one face side
// (compressibleflux.h:46-75) for a pair of Mach numbers, side S = +1 (left)
// or -1 (right).  With z = (1 + S M)/2 clamped to [0, 1] both sides share
// one form:
//   |M4| = z^2 (1 + 2 (z-1)^2),   P5 = z^2 (3 - 2z + 3 (2z-1) (z-1)^2),
// which for |M| < 1 is the reference's 1/4 (M+S)^2 (1 + 1/2 (M-S)^2) and
// 1/4 (M+S)^2 ((2 - S M) + 3/4 S M (M-S)^2); the clamp makes P5 exactly 1
// (S M >= 1) or 0 (S M <= -1) as the reference's M1/M ratio is, and M4
// becomes M1 = (M + S|M|)/2 with the added term max(M-1, 0) (S = +1) or
// min(M+1, 0) (S = -1).
template <int S>
__device__ __forceinline__ void fx_split2(float2 M, float2& m4, float2& p5)
{
  const float2 z = make_float2(__saturatef(fmaf(0.5f * S, M.x, 0.5f)), __saturatef(fmaf(0.5f * S, M.y, 0.5f)));
  const float2 zm1 = add2(z, v2(-1.0f));
  const float2 w = mul2(zm1, zm1);
  const float2 z2 = mul2(z, z);
  const float2 mag = mul2(z2, fma2(v2(2.0f), w, v2(1.0f)));
  const float2 t = fma2(v2(2.0f), z, v2(-1.0f));
  p5 = mul2(z2, fma2(mul2(v2(3.0f), t), w, fma2(v2(-2.0f), z, v2(3.0f))));
  if (S > 0) {
    m4 = add2(mag, max0(add2(M, v2(-1.0f))));
  } else {
    m4 = sub2(min0(add2(M, v2(1.0f))), mag);
  }
}

// AUSM+ flux (ausmplus.h:39-106) of a pair of faces with normal DIR between
// face sides L and R.  The reference's convective part h0 (phi_L + phi_R) -
// g0 (phi_R - phi_L) with h0 = f0/2, g0 = |f0|/2 is the upwind form
// max(f0, 0) phi_L + min(f0, 0) phi_R.
template <int DIR>
__device__ __forceinline__ void fx_ausm2(const Prim2& L, const Prim2& R, float2 A, float2 F[5])
{
  const float2 unl = DIR == 0 ? L.u : (DIR == 1 ? L.v : L.w);
  const float2 unr = DIR == 0 ? R.u : (DIR == 1 ? R.v : R.w);
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
  F[1] = DIR == 0 ? fma2(cp, L.u, fma2(cm, R.u, Ap)) : fma2(cp, L.u, mul2(cm, R.u));
  F[2] = DIR == 1 ? fma2(cp, L.v, fma2(cm, R.v, Ap)) : fma2(cp, L.v, mul2(cm, R.v));
  F[3] = DIR == 2 ? fma2(cp, L.w, fma2(cm, R.w, Ap)) : fma2(cp, L.w, mul2(cm, R.w));
  F[4] = fma2(cp, L.H, mul2(cm, R.H));
}

// Twice the van Albada slope shared by both face-side states of a cell,
// 2 s = a b (a + b) / (a^2 + b^2), for a pair; the face states are
// U +- 0.5 * (2 s).  The denominator carries 1e-30, far below any nonzero
// a^2 + b^2 of offsets of at least one quantum, so that a = b = 0 gives 0
// without a test.
__device__ __forceinline__ float2 fx_slope2(float2 a, float2 b)
{
  const float2 den = fma2(a, a, fma2(b, b, v2(1e-30f)));
  return mul2(mul2(mul2(a, b), add2(a, b)), rcp2(den));
}

// Range of the face fluxes (in quanta) a thread has converted: the largest
// magnitude, NaN once a flux is not finite (PTX max.NaN, three inputs; the
// absolute values fold into the operands).
struct FaceRange {
  float hi = 0.0f;
  __device__ __forceinline__ void add2(float a, float b)
  {
    asm("max.NaN.f32 %0, %1, %2, %3;" : "=f"(hi) : "f"(hi), "f"(fabsf(a)), "f"(fabsf(b)));
  }
  __device__ __forceinline__ void add(const FaceRange& o)
  {
    asm("max.NaN.f32 %0, %1, %2;" : "=f"(hi) : "f"(hi), "f"(o.hi));
  }
  // largest magnitude (NaN if any flux was not finite)
  __device__ __forceinline__ float mag() const { return hi; }
};

// A pair of face fluxes in whole quanta, recorded in r.  A face of 2^30
// quanta or more (a single face moving the offset by the whole
// representable range) would saturate in the int32 conversion; the caller
// flags it instead of passing it on.
__device__ __forceinline__ int2 fx_quant2(float2 x, FaceRange& r)
{
  r.add2(x.x, x.y);
  return make_int2(__float2int_rn(x.x), __float2int_rn(x.y));
}

// A single face flux in whole quanta (patch-face fluxes), recorded in r.
__device__ __forceinline__ int fx_quant1(float x, FaceRange& r)
{
  r.add2(x, x);
  return __float2int_rn(x);
}

// Patch-face flux of side `side` (axis AXIS) of a boundary cell with FP32
// state U, in whole quanta (0 for a zero-flux side), recorded in r.  Placed
// in the face arrays where the missing interior face would be, a min side's
// flux counts as the face below the cell and a max side's as the face above
// it, so the residual adds it with the reference's signs (+ min, - max).
template <int AXIS>
__device__ __forceinline__ void fx_wall_quanta(const WallBC& bc, int side, int face, const float U[5], float A,
                                               const float2* face_scale, FaceRange& r, int q[5])
{
  float F[5];
  const bool on = wall_flux<AXIS>(bc, side, face, U, A, F);
  #pragma unroll
  for (int v = 0; v < 5; ++v) q[v] = on ? fx_quant1(F[v] * face_scale[v].x, r) : 0;
}

// Cell whose state stands at index x of an axis: the wrapped cell on a
// periodic axis, the nearest edge cell outside a closed one.  Copying the
// edge cell outward makes the van Albada slope of an edge cell exactly zero
// (one of its differences vanishes), which is the reference's first-order
// reconstruction at a closed patch edge (upwind2.h:39-42), with no test.
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

// Resident CTAs per SM the register allocation is sized for: two 256-thread
// or three 128-thread CTAs (the shared memory of the tile allows no more).
template <int NT>
struct FxOccupancy {
  static constexpr int min_blocks = NT >= 256 ? 2 : 3;
};

// Shared memory of a CTA.  Every array starts on a 128-byte boundary.  The
// staging area holds the next plane as stored (int32) until it is
// dequantised into the ring: a main box of rows j0-2 .. j0+TJ+1 and columns
// k0-4 .. k0+TK+3 (the column origin k0-4 keeps a TMA box on a 16-byte
// boundary), and, for tiles at the seam of a periodic axis, the wrapped
// columns (k side box, 4 wide), the wrapped rows (j side box, 2 high) and
// their corner.  Pairs are read and written as 8-byte words: a half-warp
// then covers one row of a 32-wide tile, 32 consecutive banks.
template <int TJ, int TK>
struct FxSmem {
  static constexpr int PJ = TJ + 4;              // ring rows j0-2 .. j0+TJ+1
  static constexpr int PK = TK + 4;              // ring columns k0-2 .. k0+TK+1
  static constexpr int SK = TK + 8;              // main box row: columns k0-4 .. k0+TK+3
  static constexpr int TP = TK / 2;              // pairs (threads) per row
  static constexpr int NT = TJ * TP;             // threads of a CTA
  static constexpr int up128(int n) { return (n + 31) / 32 * 32; }   // int32 count to 128 bytes
  static constexpr int ST_M = 0;                                   // main box [5][PJ][SK]
  static constexpr int ST_K = ST_M + up128(5 * PJ * SK);           // k side box [5][PJ][4]
  static constexpr int ST_J = ST_K + up128(5 * PJ * 4);            // j side box [5][2][SK]
  static constexpr int ST_C = ST_J + up128(5 * 2 * SK);            // corner box [5][2][4]
  static constexpr int ST_N = ST_C + up128(5 * 2 * 4);
  alignas(128) float plane[3][5][PJ][PK];        // dequantised state, ring over planes i .. i+2
  alignas(128) int stage[ST_N];                  // plane i+3 as stored, on its way into the ring
  alignas(128) int un[5][TJ][TK];                // f(n) of the own cells of the current plane
  alignas(128) float sy[5][TJ + 1][TK];          // y: left state of the face below row jj (jj = 0 .. TJ)
  alignas(128) float sy_top[5][TK];              // y: right state of the face below halo row TJ
  alignas(128) float szp[5][TJ][TP + 1];         // z: left state of the face below column 2p (p = 0 .. TP)
  alignas(128) float sz_top[5][TJ];              // z: right state of the face below halo column TK
  alignas(128) int qy[5][TJ + 1][TK];            // y face integers, face below row jj
  alignas(128) int2 qz[5][TJ][TP + 1];           // z face integers below columns 2p and 2p+1
  alignas(8) uint64_t bar[2];                    // mbarriers of the TMA loads: staging plane, f(n)
  int wide[2];                                   // a face of the plane reached kFxNarrowFace
};

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

// Is every own cell of the tile inside the patch?  Such tiles that are not
// full lie next to a closed patch face: their faces on that patch face do
// not exist and their halo there repeats the edge cell, but every thread
// owns both cells of its pair.
template <int TJ, int TK>
__device__ __forceinline__ bool fx_tile_inside(const FxGeom& g, int j0, int k0)
{
  return j0 + TJ <= g.nj && k0 + TK <= g.nk;
}

// Forms of the tile function: tiles that reach beyond the patch (every test
// per cell), tiles inside the patch next to a closed face (face masks per
// thread, clamped halo pairs), full tiles (no test).
constexpr int kFxEdge = 0, kFxInside = 1, kFxFull = 2;

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

// Where ring position (row jj, column c) of a tile reads its cell in the
// staging area: offset of variable 0 (*soff) and stride between variables
// (*svar).  Cell copies fill the main box position by position; TMA boxes
// hold the main box plus the side boxes of a periodic seam, and on a closed
// axis the cells outside the patch read the edge cell's slot of the box.
template <int TJ, int TK>
__device__ __forceinline__ void fx_stage_slot(const FxGeom& g, bool tma, int j0, int k0, int jj, int c, int* soff,
                                              int* svar)
{
  using Smem = FxSmem<TJ, TK>;
  constexpr int PJ = Smem::PJ, SK = Smem::SK;
  *soff = Smem::ST_M + jj * SK + c + 2;
  *svar = PJ * SK;
  if (!tma) return;
  const int jg = j0 - 2 + jj, kg = k0 - 2 + c;
  const bool jside = g.per_y && (jg < 0 || jg >= g.nj);
  const int jr = jside ? (jg < 0 ? jg + 2 : jg - g.nj) : (g.per_y ? jg : min(max(jg, 0), g.nj - 1)) - (j0 - 2);
  const bool kside = g.per_z && (kg < 0 || kg >= g.nk);
  const int kr = kside ? (kg < 0 ? kg + 4 : kg - g.nk) : (g.per_z ? kg : min(max(kg, 0), g.nk - 1)) - (k0 - 4);
  if (jside) {
    *soff = (kside ? Smem::ST_C + jr * 4 : Smem::ST_J + jr * SK) + kr;
    *svar = kside ? 2 * 4 : 2 * SK;
  } else {
    *soff = (kside ? Smem::ST_K + jr * 4 : Smem::ST_M + jr * SK) + kr;
    *svar = kside ? PJ * 4 : PJ * SK;
  }
}

// One tile of one patch: columns (j0 .. j0+TJ-1, k0 .. k0+TK-1), planes i0 .. i1-1.
// tm_in: the kFxMaps tensor maps of the stage input, tm_un: the map of f(n)
// (box TK x TJ x 1 x 5), or null.  With maps, a tile stages its planes by
// TMA box loads unless fx_seam excludes it; other tiles copy cell by cell.
// MODE kFxFull tiles (fx_tile_full) skip every edge test, and their ring
// positions come in adjacent pairs in every staging form (no clamping; a
// periodic seam falls between pairs), so they dequantise pairwise.  MODE
// kFxInside tiles (fx_tile_inside) dequantise pairwise too: a pair whose two
// positions clamp to one edge cell of a closed k axis reads that cell twice.
// NEXT: the CTA takes another work item after this one (persistent CTAs):
// the tile then ends with a barrier and retires its mbarriers, and returns
// false (in every thread) when a TMA wait ran out, as a transfer may still
// be writing shared memory and the CTA must take no further item.  WALLS =
// false: the patch has no patch-face fluxes (a.wall.any == 0), and their
// code is left out.
template <int TJ, int TK, int MODE, bool NEXT = false, bool WALLS = true>
__device__ __forceinline__ bool fx_stage_tile_impl(const FxArgs& a, const CUtensorMap* tm_in,
                                                   const CUtensorMap* tm_un, int j0, int k0, int i0, int i1)
{
  using Smem = FxSmem<TJ, TK>;
  constexpr int PJ = Smem::PJ, PK = Smem::PK, SK = Smem::SK, TP = Smem::TP, NT = Smem::NT;
  constexpr int NP = PJ * PK;                     // positions of a plane tile (per variable)
  constexpr int PPT = (NP + NT - 1) / NT;         // positions per thread
  constexpr int NPP = PJ * (PK / 2);              // position pairs of a plane tile
  constexpr int PPT2 = (NPP + NT - 1) / NT;       // position pairs per thread
  static_assert(TK % 4 == 0 && TJ % 2 == 0 && TP <= 32 && TJ / 2 <= 32 && NT >= 64 && TK + TJ <= NT,
                "tile shape");
  constexpr bool FULL = MODE == kFxFull;
  constexpr bool PAIRS = MODE != kFxEdge;         // own pairs inside the patch, pairwise dequantisation
  extern __shared__ __align__(128) unsigned char fx_smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(fx_smem_raw);

  const FxGeom& g = a.g;
  const FxParams& P = a.p;
  const int tp = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * TP + tp;
  const int kk = 2 * tp;                          // tile column of the pair's first cell
  const int j = j0 + ty, ka = k0 + kk, kb = ka + 1;
  // inside tiles place the y and z patch-face fluxes of their boundary cells
  // in the face arrays, in the slot of the missing face, during the slope
  // phase (their state is in the ring then); the face phase leaves those
  // slots alone and the residual sums them like interior faces.  The slots
  // are written and read by the same thread.
  const bool yz_walls = WALLS && MODE == kFxInside && a.wall.any;
  const bool w_ymin = yz_walls && j == 0 && !g.per_y && g.nj > 2;
  const bool w_ymax = yz_walls && j == g.nj - 1 && !g.per_y && g.nj > 2;
  const bool w_zmin = yz_walls && ka == 0 && !g.per_z && g.nk > 2;
  const bool w_zmax = yz_walls && kb == g.nk - 1 && !g.per_z && g.nk > 2;
  const bool own_a = PAIRS || ((j < g.nj) && (ka < g.nk));
  const bool own_b = PAIRS || ((j < g.nj) && (kb < g.nk));
  const int njk = g.nj * g.kp;                    // plane stride (rows of kp elements)
  const int nc = g.ni * njk;                      // variable stride (5 * nc < 2^31, host check)
  // TMA boxes start at x = k0-4 (main; a multiple of 4 int32 since TK is),
  // k0 (f(n)), and nk-4 or 0 (k side box): the first seam tile of a periodic
  // k axis needs nk % 4 == 0 for its side box (the last one has k0+TK = nk,
  // a multiple of 4 already); box cells beyond the patch are zero-filled and
  // never read; destinations 128-byte aligned
  const int seam_j = fx_seam(j0, TJ, g.nj, g.per_y);
  const int seam_k = fx_seam(k0, TK, g.nk, g.per_z);
  const bool tma = tm_in != nullptr && seam_j >= 0 && seam_k >= 0 && (seam_k != 1 || (g.nk & 3) == 0) &&
                   ((smem_u32(&sm.stage[0]) | smem_u32(&sm.un[0][0][0])) & 127) == 0;

  auto PL2 = [&](int sl, int v, int jj, int c) -> float2& {
    return *reinterpret_cast<float2*>(&sm.plane[sl][v][jj][c]);
  };
  // the own pair's ring position (row ty+2, column kk+2) in slot 0,
  // variable 0; a slot's own pair of variable v, dj rows and dk columns away,
  // is then (base + v*VS + dj*PK + dk) with compile-time offsets
  constexpr int VS = PJ * PK, SS = 5 * VS;
  const float* const ring_me = &sm.plane[0][0][ty + 2][kk + 2];
  auto RP = [&](const float* base, int v, int dj, int dk) -> float2 {
    return *reinterpret_cast<const float2*>(base + v * VS + dj * PK + dk);
  };

  // per-thread staging positions: single positions e = tid + m*NT in ring
  // order [row][column] with the in-plane offset j*kp + k of their (wrapped
  // or clamped) cell for cell copies; the edge form also keeps their
  // staging slots, the pair forms the staging slots of position pairs (bit
  // m of `dup`: pair m reads one clamped edge cell for both positions)
  int32_t poff[PPT];
  int32_t soff[PAIRS ? PPT2 : PPT];
  int32_t svar[PAIRS ? PPT2 : PPT];
  unsigned dup = 0;
  #pragma unroll
  for (int m = 0; m < PPT; ++m) {
    const int e = tid + m * NT;
    poff[m] = -1;
    if (e < NP) {
      const int jj = e / PK, c = e % PK;
      poff[m] = fx_index(j0 - 2 + jj, g.nj, g.per_y) * g.kp + fx_index(k0 - 2 + c, g.nk, g.per_z);
      if (!PAIRS) fx_stage_slot<TJ, TK>(g, tma, j0, k0, jj, c, &soff[m], &svar[m]);
    }
  }
  if (PAIRS) {
    #pragma unroll
    for (int m = 0; m < PPT2; ++m) {
      const int e = tid + m * NT;
      soff[m] = 0;
      svar[m] = 0;
      if (e < NPP) {
        const int jj = e / (PK / 2), c = 2 * (e % (PK / 2));
        fx_stage_slot<TJ, TK>(g, tma, j0, k0, jj, c, &soff[m], &svar[m]);
        if (MODE == kFxInside) {
          // the second position reads the same slot (a clamped edge cell) or the next one
          int s1, v1;
          fx_stage_slot<TJ, TK>(g, tma, j0, k0, jj, c + 1, &s1, &v1);
          if (s1 == soff[m]) dup |= 1u << m;
        }
      }
    }
  }

  // plane ip of the stage input, copied cell by cell (cp.async) as int32
  // into ring slot sl, then dequantised there in place by the copying thread
  auto issue_ring = [&](int sl, int ip) {
    int* dst = reinterpret_cast<int*>(&sm.plane[sl][0][0][0]);
    const int32_t* src = a.in + fx_index(ip, g.ni, g.per_x) * njk;
    #pragma unroll
    for (int v = 0; v < 5; ++v) {
      #pragma unroll
      for (int m = 0; m < PPT; ++m) {
        const int e = tid + m * NT;
        if (e < NP) fx_cp_async4(dst + v * NP + e, src + v * nc + poff[m]);
      }
    }
  };
  auto dequant_ring = [&](int sl) {
    float* f = &sm.plane[sl][0][0][0];
    const int* q = reinterpret_cast<const int*>(f);
    #pragma unroll
    for (int v = 0; v < 5; ++v) {
      #pragma unroll
      for (int m = 0; m < PPT; ++m) {
        const int e = tid + m * NT;
        if (e < NP) f[v * NP + e] = fmaf(P.quantum[v].x, (float)q[v * NP + e], P.base[v].x);
      }
    }
  };
  // plane ip into the staging plane's main box, cell by cell (tiles without TMA)
  auto issue_stage = [&](int ip) {
    int* dst = &sm.stage[Smem::ST_M];
    const int32_t* src = a.in + fx_index(ip, g.ni, g.per_x) * njk;
    #pragma unroll
    for (int v = 0; v < 5; ++v) {
      #pragma unroll
      for (int m = 0; m < PPT; ++m) {
        const int e = tid + m * NT;
        if (e < NP) fx_cp_async4(dst + v * (PJ * SK) + (e / PK) * SK + e % PK + 2, src + v * nc + poff[m]);
      }
    }
  };
  // the staging area, dequantised into ring slot sl
  auto dequant_stage = [&](int sl) {
    const int* q = &sm.stage[0];
    if (PAIRS) {
      // pair e of a ring slot starts at float 2e of its variable's plane;
      // a pair of two positions starts on an even slot (8-byte aligned), a
      // clamped pair reads its one cell from the aligned word holding it
      float2* f = reinterpret_cast<float2*>(&sm.plane[sl][0][0][0]);
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        #pragma unroll
        for (int m = 0; m < PPT2; ++m) {
          const int e = tid + m * NT;
          if (e < NPP) {
            int2 o = *reinterpret_cast<const int2*>(q + (soff[m] & ~1) + v * svar[m]);
            if (MODE == kFxInside && ((dup >> m) & 1u)) {
              const int x = (soff[m] & 1) ? o.y : o.x;
              o = make_int2(x, x);
            }
            f[v * NPP + e] = fma2(P.quantum[v], make_float2((float)o.x, (float)o.y), P.base[v]);
          }
        }
      }
    } else {
      float* f = &sm.plane[sl][0][0][0];
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        #pragma unroll
        for (int m = 0; m < PPT; ++m) {
          const int e = tid + m * NT;
          if (e < NP) f[v * NP + e] = fmaf(P.quantum[v].x, (float)q[soff[m] + v * svar[m]], P.base[v].x);
        }
      }
    }
  };
  // f(n) of the own cells, plane ip, cell by cell (tiles without TMA)
  auto fetch_un = [&](int ip) {
    const int c = ip * njk + j * g.kp + ka;
    #pragma unroll
    for (int v = 0; v < 5; ++v) {
      if (own_a) fx_cp_async4(&sm.un[v][ty][kk], a.un + v * nc + c);
      if (own_b) fx_cp_async4(&sm.un[v][ty][kk + 1], a.un + v * nc + c + 1);
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

  if (tid == 0) {
    if (tma) {
      mbar_init(&sm.bar[0], 1);
      mbar_init(&sm.bar[1], 1);
      mbar_init_fence();
    }
    sm.wide[0] = 0;
    sm.wide[1] = 0;
  }

  // prologue: planes i0 .. i0+2 in the ring (the barrier below also
  // publishes the mbarrier initialisation and the cleared flags)
  for (int q = 0; q <= 2; ++q) issue_ring(q, i0 + q);
  fx_cp_async_commit();
  fx_cp_async_wait<0>();
  for (int q = 0; q <= 2; ++q) dequant_ring(q);
  __syncthreads();

  // x direction registers: prim of the left state of the face above the
  // current cells, the downwind difference and the state of the next plane,
  // and the lower face integers
  FaceRange fmag;        // face fluxes in quanta of the current plane
  FaceRange xmag;        // the same of the x faces below the current cells (the last plane's upper ones)
  bool fbad = false;     // a face flux reached 2^30 quanta or was not finite
  bool tbad = false;     // a TMA wait ran out
  Prim2 xleft;
  float2 xb[5];          // U_{i+1} - U_i of the own pair (becomes a of cell i+1)
  int2 qx_lo[5];
  {
    // slope of cell i0 (needs i0-1, i0, i0+1) and the face below i0; planes
    // i0-1 and i0-2 of the own column come straight from the stage input
    // (read as a pair when the first cell is inside: the second of a partial
    // pair lies in the row padding)
    const int col = j * g.kp + ka;
    const int iw1 = fx_index(i0 - 1, g.ni, g.per_x);
    float2 Ul[5], Sp[5], Sm[5], U0[5];
    #pragma unroll
    for (int v = 0; v < 5; ++v) {
      float2 um = v2(0.0f);
      if (own_a) {
        const int2 o = __ldg(reinterpret_cast<const int2*>(a.in + v * nc + iw1 * njk + col));
        um = fma2(P.quantum[v], make_float2((float)o.x, (float)o.y), P.base[v]);
      }
      const float2 uc = PL2(0, v, ty + 2, kk + 2);
      const float2 up = PL2(1, v, ty + 2, kk + 2);
      const float2 s = fx_slope2(sub2(uc, um), sub2(up, uc));
      U0[v] = uc;
      Sp[v] = fma2(s, v2(0.5f), uc);
      Sm[v] = fma2(s, v2(-0.5f), uc);
      xb[v] = sub2(up, uc);
      Ul[v] = um;
    }
    xleft = fx_prim2(Sp[0], Sp[1], Sp[2], Sp[3], Sp[4]);
    // face below i0: left state from cell i0-1 (slope needs i0-2)
    if (own_a && fx_face_exists(i0, g.ni, g.per_x)) {
      const int iw2 = fx_index(i0 - 2, g.ni, g.per_x);
      float2 Lm[5];
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        const int2 o = __ldg(reinterpret_cast<const int2*>(a.in + v * nc + iw2 * njk + col));
        const float2 umm = fma2(P.quantum[v], make_float2((float)o.x, (float)o.y), P.base[v]);
        Lm[v] = fma2(fx_slope2(sub2(Ul[v], umm), sub2(U0[v], Ul[v])), v2(0.5f), Ul[v]);
      }
      float2 F[5];
      fx_ausm2<0>(fx_prim2(Lm[0], Lm[1], Lm[2], Lm[3], Lm[4]), fx_prim2(Sm[0], Sm[1], Sm[2], Sm[3], Sm[4]), P.A[0],
                  F);
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        qx_lo[v] = fx_quant2(mul2(F[v], P.face_scale[v]), xmag);
        if (!own_b) qx_lo[v].y = 0;
      }
    } else {
      #pragma unroll
      for (int v = 0; v < 5; ++v) qx_lo[v] = make_int2(0, 0);
    }
  }

  int s0 = 0, sp1 = 1, sp2 = 2;       // ring slots of planes i, i+1, i+2
  unsigned ph_plane = 0, ph_un = 0;   // parities of the next TMA completions
  int par = 0;                        // plane parity: slot of sm.wide
  for (int i = i0; i < i1; ++i) {
    const bool more = i + 3 <= i1 + 1;  // plane i+3 is read by a later iteration

    // ---------------- A: y and z slopes of plane i
    float2 ym[5];    // right states of the y faces below the own pair
    float2 zm[5];    // right states of the z faces below the own pair
    float zpx[5];    // left state of the z face between the pair's cells
    const float* const r0 = ring_me + s0 * SS;
    #pragma unroll
    for (int v = 0; v < 5; ++v) {
      const float2 C = RP(r0, v, 0, 0);
      {
        const float2 lo = RP(r0, v, -1, 0), hi = RP(r0, v, 1, 0);
        const float2 s = fx_slope2(sub2(C, lo), sub2(hi, C));
        *reinterpret_cast<float2*>(&sm.sy[v][ty + 1][kk]) = fma2(s, v2(0.5f), C);
        ym[v] = fma2(s, v2(-0.5f), C);
      }
      {
        const float zl = RP(r0, v, 0, -2).y, zh = RP(r0, v, 0, 2).x;
        const float d1 = C.y - C.x;
        const float2 s = fx_slope2(make_float2(C.x - zl, d1), make_float2(d1, zh - C.y));
        const float2 zp = fma2(s, v2(0.5f), C);
        zm[v] = fma2(s, v2(-0.5f), C);
        zpx[v] = zp.x;
        sm.szp[v][ty][tp + 1] = zp.y;
      }
    }
    // halo slopes (first warps): y rows -1 (left states) and TJ (right
    // states) in column pairs; z columns -1 (left state, lane x) and TK
    // (right state, lane y) of a row
    if (tid < TK + TJ) {
      if (tid < TK) {
        const bool top = tid >= TP;
        const int c = 2 * (tid % TP);
        const int r = top ? TJ + 2 : 1;             // ring row of the halo cell
        #pragma unroll
        for (int v = 0; v < 5; ++v) {
          const float2 C = PL2(s0, v, r, c + 2);
          const float2 s = fx_slope2(sub2(C, PL2(s0, v, r - 1, c + 2)), sub2(PL2(s0, v, r + 1, c + 2), C));
          if (top) *reinterpret_cast<float2*>(&sm.sy_top[v][c]) = fma2(s, v2(-0.5f), C);
          else *reinterpret_cast<float2*>(&sm.sy[v][0][c]) = fma2(s, v2(0.5f), C);
        }
      } else {
        const int jj = tid - TK;
        #pragma unroll
        for (int v = 0; v < 5; ++v) {
          const float* row = &sm.plane[s0][v][jj + 2][0];
          const float2 C = make_float2(row[1], row[TK + 2]);
          const float2 s = fx_slope2(sub2(C, make_float2(row[0], row[TK + 1])),
                                     sub2(make_float2(row[2], row[TK + 3]), C));
          sm.szp[v][jj][0] = fmaf(s.x, 0.5f, C.x);
          sm.sz_top[v][jj] = fmaf(s.y, -0.5f, C.y);
        }
      }
    }
    FaceRange wmag_yz;   // y and z patch-face fluxes of the own cells
    if (w_ymin || w_ymax || w_zmin || w_zmax) {
      float Ua[5], Ub[5];
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        const float2 u = RP(r0, v, 0, 0);
        Ua[v] = u.x;
        Ub[v] = u.y;
      }
      int qa[5], qb[5];
      if (w_ymin || w_ymax) {
        const int side = w_ymin ? 2 : 3;
        fx_wall_quanta<1>(a.wall, side, i * g.nk + ka, Ua, P.A[1].x, P.face_scale, wmag_yz, qa);
        fx_wall_quanta<1>(a.wall, side, i * g.nk + kb, Ub, P.A[1].x, P.face_scale, wmag_yz, qb);
        #pragma unroll
        for (int v = 0; v < 5; ++v)
          *reinterpret_cast<int2*>(&sm.qy[v][w_ymin ? ty : ty + 1][kk]) = make_int2(qa[v], qb[v]);
      }
      if (w_zmin) {
        fx_wall_quanta<2>(a.wall, 4, i * g.nj + j, Ua, P.A[2].x, P.face_scale, wmag_yz, qa);
        #pragma unroll
        for (int v = 0; v < 5; ++v) sm.qz[v][ty][tp].x = qa[v];
      }
      if (w_zmax) {
        fx_wall_quanta<2>(a.wall, 5, i * g.nj + j, Ub, P.A[2].x, P.face_scale, wmag_yz, qb);
        #pragma unroll
        for (int v = 0; v < 5; ++v) sm.qz[v][ty][tp + 1].x = qb[v];
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
    if (tid == 0) sm.wide[par ^ 1] = 0;   // flag of the next plane (its last reader passed the barrier)
    fmag = xmag;                          // the x faces below the own cells count for this plane too
    fmag.add(wmag_yz);

    // ---------------- B: faces
    // y faces below the own pair; the face below row j is needed even when
    // row j itself lies beyond a periodic patch (it is the wrapped face above
    // the last row)
    {
      float2 L[5];
      #pragma unroll
      for (int v = 0; v < 5; ++v) L[v] = *reinterpret_cast<const float2*>(&sm.sy[v][ty][kk]);
      float2 F[5];
      fx_ausm2<1>(fx_prim2(L[0], L[1], L[2], L[3], L[4]), fx_prim2(ym[0], ym[1], ym[2], ym[3], ym[4]), P.A[1], F);
      bool exa = true, exb = true;
      if (!FULL) {
        const bool ey = fx_face_exists(j, g.nj, g.per_y) && (PAIRS || g.per_y || j < g.nj);
        exa = ey && (PAIRS || ka < g.nk);
        exb = ey && (PAIRS || kb < g.nk);
      }
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        int2 q = fx_quant2(mul2(F[v], P.face_scale[v]), fmag);
        if (!exa) q.x = 0;
        if (!exb) q.y = 0;
        if (!w_ymin) *reinterpret_cast<int2*>(&sm.qy[v][ty][kk]) = q;   // else: the patch face, placed before
      }
    }
    // z faces below the pair's two cells
    {
      float2 L[5];
      #pragma unroll
      for (int v = 0; v < 5; ++v) L[v] = make_float2(sm.szp[v][ty][tp], zpx[v]);
      float2 F[5];
      fx_ausm2<2>(fx_prim2(L[0], L[1], L[2], L[3], L[4]), fx_prim2(zm[0], zm[1], zm[2], zm[3], zm[4]), P.A[2], F);
      bool exa = true, exb = true;
      if (!FULL) {
        const bool rowin = PAIRS || j < g.nj;
        exa = rowin && fx_face_exists(ka, g.nk, g.per_z) && (PAIRS || g.per_z || ka < g.nk);
        exb = rowin && fx_face_exists(kb, g.nk, g.per_z) && (PAIRS || g.per_z || kb < g.nk);
      }
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        int2 q = fx_quant2(mul2(F[v], P.face_scale[v]), fmag);
        if (!exa) q.x = 0;
        if (!exb) q.y = 0;
        if (w_zmin) sm.qz[v][ty][tp].y = q.y;   // .x: the patch face, placed before
        else sm.qz[v][ty][tp] = q;
      }
    }
    // halo faces: below halo row TJ in column pairs (second-to-last warp)
    // and below halo column TK for rows jj and jj + TJ/2 (last warp)
    {
      const int h = tid - (NT - 64);
      if (h >= 0 && h < TP) {
        const int c = 2 * h;
        float2 L[5], R[5];
        #pragma unroll
        for (int v = 0; v < 5; ++v) {
          L[v] = *reinterpret_cast<const float2*>(&sm.sy[v][TJ][c]);
          R[v] = *reinterpret_cast<const float2*>(&sm.sy_top[v][c]);
        }
        float2 F[5];
        fx_ausm2<1>(fx_prim2(L[0], L[1], L[2], L[3], L[4]), fx_prim2(R[0], R[1], R[2], R[3], R[4]), P.A[1], F);
        bool exa = true, exb = true;
        if (!FULL) {
          const int jf = j0 + TJ;
          const bool ey = fx_face_exists(jf, g.nj, g.per_y) && (g.per_y || jf < g.nj);
          exa = ey && (PAIRS || k0 + c < g.nk);
          exb = ey && (PAIRS || k0 + c + 1 < g.nk);
        }
        // (the last row's patch face, if any, is placed by its own cells)
        const bool keep = yz_walls && j0 + TJ == g.nj && !g.per_y && g.nj > 2;
        #pragma unroll
        for (int v = 0; v < 5; ++v) {
          int2 q = fx_quant2(mul2(F[v], P.face_scale[v]), fmag);
          if (!exa) q.x = 0;
          if (!exb) q.y = 0;
          if (!keep) *reinterpret_cast<int2*>(&sm.qy[v][TJ][c]) = q;
        }
      } else if (h >= 32 && h < 32 + TJ / 2) {
        const int ja = h - 32, jb = ja + TJ / 2;
        float2 L[5], R[5];
        #pragma unroll
        for (int v = 0; v < 5; ++v) {
          L[v] = make_float2(sm.szp[v][ja][TP], sm.szp[v][jb][TP]);
          R[v] = make_float2(sm.sz_top[v][ja], sm.sz_top[v][jb]);
        }
        float2 F[5];
        fx_ausm2<2>(fx_prim2(L[0], L[1], L[2], L[3], L[4]), fx_prim2(R[0], R[1], R[2], R[3], R[4]), P.A[2], F);
        bool exa = true, exb = true;
        if (!FULL) {
          const int kz = k0 + TK;
          const bool ez = fx_face_exists(kz, g.nk, g.per_z) && (g.per_z || kz < g.nk);
          exa = ez && (PAIRS || j0 + ja < g.nj);
          exb = ez && (PAIRS || j0 + jb < g.nj);
        }
        // (the last column's patch face, if any, is placed by its own cells)
        const bool keep = yz_walls && k0 + TK == g.nk && !g.per_z && g.nk > 2;
        #pragma unroll
        for (int v = 0; v < 5; ++v) {
          const int2 q = fx_quant2(mul2(F[v], P.face_scale[v]), fmag);
          if (!keep) {
            sm.qz[v][ja][TP].x = exa ? q.x : 0;
            sm.qz[v][jb][TP].x = exb ? q.y : 0;
          }
        }
      }
    }
    // x: face above cell i (between i and i+1), along the own column
    int2 qx_hi[5];
    {
      float2 Sm[5], Sp[5];
      const float* const r1 = ring_me + sp1 * SS;
      const float* const r2 = ring_me + sp2 * SS;
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        const float2 uc = RP(r1, v, 0, 0);
        const float2 up = RP(r2, v, 0, 0);
        const float2 b = sub2(up, uc);
        const float2 s = fx_slope2(xb[v], b);
        Sm[v] = fma2(s, v2(-0.5f), uc);
        Sp[v] = fma2(s, v2(0.5f), uc);
        xb[v] = b;
      }
      const bool ex = fx_face_exists(i + 1, g.ni, g.per_x);
      float2 F[5];
      fx_ausm2<0>(xleft, fx_prim2(Sm[0], Sm[1], Sm[2], Sm[3], Sm[4]), P.A[0], F);
      xmag = FaceRange();
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        qx_hi[v] = fx_quant2(mul2(F[v], P.face_scale[v]), xmag);
        if (!ex || !own_a) qx_hi[v].x = 0;
        if (!ex || !own_b) qx_hi[v].y = 0;
      }
      fmag.add(xmag);
      xleft = fx_prim2(Sp[0], Sp[1], Sp[2], Sp[3], Sp[4]);
    }
    // faces of 2^30 quanta or more, or not finite, are errors; faces beyond
    // the narrow bound make the plane sum its residuals in 64 bits
    const float m = fmag.mag();
    fbad |= !(m < kFxFaceLimit);
    if (!(m < kFxNarrowFace)) sm.wide[par] = 1;

    __syncthreads();

    // ---------------- C: residual and update of the own cells
    // f(n) of plane i has arrived (the staging copy may stay in flight)
    if (tma) {
      tbad |= !mbar_wait(&sm.bar[1], ph_un);
      ph_un ^= 1u;
    } else {
      fx_cp_async_wait<1>();
    }
    if (own_a) {
      const int c = i * njk + j * g.kp + ka;      // even: rows start on 16-byte boundaries
      const bool wide = sm.wide[par] != 0;
      bool act_a = true, act_b = own_b;
      if (a.active) {
        act_a = a.active[c] != 0;
        act_b = act_b && a.active[c + 1] != 0;
      }
      // patch-face fluxes of boundary cells: whole quanta like the interior
      // faces (a wall face replaces the cell's missing interior face, so a
      // cell still sums six faces)
      // (inside tiles: the y and z sides are in the face arrays already)
      const bool any_wall = WALLS && a.wall.any;
      const bool x_only = MODE == kFxInside;
      const bool edge_i = any_wall && (i == 0 || i == g.ni - 1);
      const bool edge_ijk = edge_i || (any_wall && !x_only && (j == 0 || j == g.nj - 1));
      const bool wall_a = x_only ? edge_i : any_wall && (edge_ijk || ka == 0 || ka == g.nk - 1);
      const bool wall_b = own_b && (x_only ? edge_i : any_wall && (edge_ijk || kb == g.nk - 1));
      long long wa[5] = {0, 0, 0, 0, 0}, wb[5] = {0, 0, 0, 0, 0};
      FaceRange wmag;
      if (wall_a || wall_b) {
        #pragma unroll
        for (int q = 0; q < 2; ++q) {
          if (q == 0 ? !wall_a : !wall_b) continue;
          // the cell's state, re-read from the stage input: the ring slot of
          // plane i receives plane i+3 below, with no barrier in between
          float uc[5];
          #pragma unroll
          for (int v = 0; v < 5; ++v) uc[v] = fmaf(P.quantum[v].x, (float)a.in[v * nc + c + q], P.base[v].x);
          add_wall_fluxes(a.wall, g.ni, g.nj, g.nk, g.per_x, g.per_y, g.per_z, i, j, ka + q, uc, P.A[0].x, P.A[1].x,
                          P.A[2].x, q == 0 ? wa : wb,
                          [&](int v, float F) { return fx_quant1(F * P.face_scale[v].x, wmag); }, !x_only);
        }
        fbad |= !(wmag.mag() < kFxFaceLimit);
      }
      int2 o[5];
      if (!wide && wmag.mag() < kFxNarrowFace) {
        // every face of the plane and every wall face of the pair below
        // kFxNarrowFace: |residual| < 2^31 fits int32, and |un + residual| <
        // 3 * 2^30, so the wrapped 32-bit sum lies in (-2^30, 2^30) exactly
        // when the true one does
        #pragma unroll
        for (int v = 0; v < 5; ++v) {
          const int2 ylo = *reinterpret_cast<const int2*>(&sm.qy[v][ty][kk]);
          const int2 yhi = *reinterpret_cast<const int2*>(&sm.qy[v][ty + 1][kk]);
          const int2 zlo = sm.qz[v][ty][tp];
          const int zhi = sm.qz[v][ty][tp + 1].x;
          const int2 un = *reinterpret_cast<const int2*>(&sm.un[v][ty][kk]);
          const unsigned ra = (unsigned)qx_lo[v].x - (unsigned)qx_hi[v].x + (unsigned)ylo.x - (unsigned)yhi.x +
                              (unsigned)zlo.x - (unsigned)zlo.y + (unsigned)wa[v];
          const unsigned rb = (unsigned)qx_lo[v].y - (unsigned)qx_hi[v].y + (unsigned)ylo.y - (unsigned)yhi.y +
                              (unsigned)zlo.y - (unsigned)zhi + (unsigned)wb[v];
          o[v].x = (int)((unsigned)un.x + ra);
          o[v].y = (int)((unsigned)un.y + rb);
        }
      } else {
        // 64-bit residuals: a face of the plane or of the pair's walls
        // beyond the narrow bound
        #pragma unroll
        for (int v = 0; v < 5; ++v) {
          const int2 ylo = *reinterpret_cast<const int2*>(&sm.qy[v][ty][kk]);
          const int2 yhi = *reinterpret_cast<const int2*>(&sm.qy[v][ty + 1][kk]);
          const int2 zlo = sm.qz[v][ty][tp];
          const int zhi = sm.qz[v][ty][tp + 1].x;
          const int2 un = *reinterpret_cast<const int2*>(&sm.un[v][ty][kk]);
          const long long ra = (long long)qx_lo[v].x - qx_hi[v].x + ylo.x - yhi.x + zlo.x - zlo.y + wa[v];
          const long long rb = (long long)qx_lo[v].y - qx_hi[v].y + ylo.y - yhi.y + zlo.y - zhi + wb[v];
          const long long oa = (long long)un.x + ra, ob = (long long)un.y + rb;
          // results outside the range are clamped to its edge and flagged below
          o[v].x = (int)(oa >= kFxLimit ? kFxLimit : (oa <= -kFxLimit ? -kFxLimit : oa));
          o[v].y = (int)(ob >= kFxLimit ? kFxLimit : (ob <= -kFxLimit ? -kFxLimit : ob));
        }
      }
      // offsets outside (-kFxLimit, kFxLimit): bit 2v (cell a) or 2v+1
      // (cell b) of `bad`, without a branch per variable
      unsigned bad = 0;
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        if (!act_a) o[v].x = a.in[v * nc + c];
        if (!act_b) o[v].y = own_b ? a.in[v * nc + c + 1] : 0;
        const bool ba = act_a && (unsigned)o[v].x + (unsigned)(kFxLimit - 1) > 2u * (unsigned)(kFxLimit - 1);
        const bool bb = act_b && (unsigned)o[v].y + (unsigned)(kFxLimit - 1) > 2u * (unsigned)(kFxLimit - 1);
        bad |= (ba ? 1u : 0u) << (2 * v);
        bad |= (bb ? 2u : 0u) << (2 * v);
        if (own_b) *reinterpret_cast<int2*>(a.out + v * nc + c) = o[v];
        else a.out[v * nc + c] = o[v].x;
      }
      if (bad) {
        // the first failing (variable, cell) of this pair is recorded
        const int bit = __ffs(bad) - 1, v = bit >> 1, q = bit & 1;
        const int2 un = *reinterpret_cast<const int2*>(&sm.un[v][ty][kk]);
        const int u = q == 0 ? un.x : un.y;
        int ov = o[0].x;
        #pragma unroll
        for (int w = 0; w < 5; ++w) if (w == v) ov = q == 0 ? o[w].x : o[w].y;
        if (a.err_info && atomicCAS(&a.err_info[0], ~0ull, (unsigned long long)(c + q)) == ~0ull) {
          a.err_info[1] = (unsigned long long)v;
          a.err_info[2] = (unsigned long long)__double_as_longlong((double)u);
          a.err_info[3] = (unsigned long long)__double_as_longlong((double)((long long)ov - u));
        }
        if (a.err) atomicOr(a.err, 1);
      }
    }
    #pragma unroll
    for (int v = 0; v < 5; ++v) qx_lo[v] = qx_hi[v];

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
    par ^= 1;
  }
  if (fbad && a.err) atomicOr(a.err, 16);
  if (tbad && a.err) atomicOr(a.err, kFxErrTma);
  if (!NEXT) return true;
  // every transfer the tile issued has completed unless a wait ran out: the
  // mbarriers are then retired for the next work item's initialisation
  const bool any_tbad = __syncthreads_or(tbad) != 0;
  if (tma && tid == 0 && !any_tbad) {
    mbar_inval(&sm.bar[0]);
    mbar_inval(&sm.bar[1]);
  }
  return !any_tbad;
}

template <int TJ, int TK, bool WALLS>
__device__ __forceinline__ void fx_stage_tile(const FxArgs& a, const CUtensorMap* tm_in, const CUtensorMap* tm_un,
                                              int j0, int k0, int i0, int i1)
{
  if (fx_tile_full<TJ, TK>(a.g, j0, k0))
    fx_stage_tile_impl<TJ, TK, kFxFull, false, WALLS>(a, tm_in, tm_un, j0, k0, i0, i1);
  else if (fx_tile_inside<TJ, TK>(a.g, j0, k0))
    fx_stage_tile_impl<TJ, TK, kFxInside, false, WALLS>(a, tm_in, tm_un, j0, k0, i0, i1);
  else fx_stage_tile_impl<TJ, TK, kFxEdge, false, WALLS>(a, tm_in, tm_un, j0, k0, i0, i1);
}

// Parameters of the single-patch launch: the stage arguments and the tensor
// maps of the stage input and of f(n) (valid when tma != 0).
struct FxLaunch {
  CUtensorMap tm_in[kFxMaps];
  CUtensorMap tm_un;
  FxArgs a;
  int tma;
};

// One patch per launch: grid (k tiles, j tiles, i chunks), block (TK/2, TJ);
// WALLS: the patch has patch-face fluxes.
template <int TJ, int TK, bool WALLS>
__global__ void __launch_bounds__(TJ * TK / 2, FxOccupancy<TJ * TK / 2>::min_blocks)
fx_stage_kernel(const __grid_constant__ FxLaunch L)
{
  const int i0 = blockIdx.z * L.a.g.i_chunk;
  fx_stage_tile<TJ, TK, WALLS>(L.a, L.tma ? L.tm_in : nullptr, L.tma ? &L.tm_un : nullptr, blockIdx.y * TJ,
                               blockIdx.x * TK, i0, min(L.a.g.ni, i0 + L.a.g.i_chunk));
}

} // namespace dn
