// Fused RK-stage kernel for one Cartesian patch: residual (all x, y and z
// face fluxes) and update f_out = f_n + factor/dV * Res(f_in) in one launch.
//
// Replaces the reference's per-stage sequence of a residual memset plus ten
// launches (six colour-split flux kernels, three boundary kernels, advance;
// iterators/gpu_cartesianiterator.h:54-304) that read-modify-write a residual
// field in HBM.  Here:
//   - a CTA owns a TJ x TK tile of (j, k) columns (k fastest, coalesced) and
//     marches along i through a chunk of planes;
//   - each plane of the stencil state is staged once in shared memory with a
//     two-cell halo in j and k, in a ring of three planes (i .. i+2; the own
//     column of plane i-1 is kept in registers); plane i+2 is loaded while
//     the y and z faces of plane i are evaluated: by one TMA box load where
//     no periodic seam crosses the tile's halo, else cell by cell with
//     cp.async;
//   - every face flux is evaluated exactly once: x faces per thread along its
//     own column (the upper face of cell i is kept in registers as the lower
//     face of cell i+1), y and z faces of the current plane into shared
//     memory;
//   - the residual is summed per cell in registers in the reference's order
//     (+Fx_lo +Fy_lo +Fz_lo -Fz_hi -Fy_hi -Fx_hi, the order the single-thread
//     CPU iterator produces, cartesianiterator.h:115-188), no atomics;
//   - the update is written once; inactive cells copy their input
//     (cartesianiterator.h:315, gpu_cartesianiterator.h:199-201).
//
// The storage/arithmetic form is a policy:
//   Policy::Store   element type in HBM
//   Policy::Real    arithmetic type
//   Policy::load(v, x)           stored value -> arithmetic value
//   Policy::face(v, F)           face flux -> value summed into the residual
//   Policy::update(v, un, r)     new stored value from stored f_n and residual
#pragma once

#include <cstdint>
#include "fv_numerics.cuh"
#include "fv_wall.cuh"
#include "fv_tma.cuh"

namespace dn {

struct StageGeom {
  int ni, nj, nk;
  int per_x, per_y, per_z;   // 1 = periodic wrap, 0 = closed
  int i_chunk;               // planes per CTA along i
};

template <class Policy>
struct StageArgs {
  const typename Policy::Store* in;   // stencil state f(k-1), [5][ni][nj][nk]
  const typename Policy::Store* un;   // step-start state f(n), own cell only
  typename Policy::Store* out;        // f(k)
  const uint8_t* active;              // per cell, NULL = all active
  int* err;                           // device error word (bit flags)
  unsigned long long* err_info;       // first failing cell: [cell, var, bits(un), bits(r)]
  StageGeom g;
  typename Policy::Params p;
  WallBC wall;                        // patch-face fluxes of the non-periodic axes
};

// index along an axis with periodic wrap; returns -1 if outside a closed axis
__device__ __forceinline__ int axis_idx(int x, int n, int per)
{
  if (per) {
    x %= n;
    return x < 0 ? x + n : x;
  }
  return (x < 0 || x >= n) ? -1 : x;
}

// does the face below cell index x (between x-1 and x) exist?
__device__ __forceinline__ bool face_exists(int x, int n, int per)
{
  if (n <= 2) return false;               // cartesianiterator.h:149,160,171
  return per ? true : (x >= 1 && x <= n - 1);
}

// is cell index x inside the axis (or wrapped)?
__device__ __forceinline__ bool cell_ok(int x, int n, int per)
{
  return per ? true : (x >= 0 && x < n);
}

template <class Policy, int TJ, int TK>
struct StageSmem {
  using Real = typename Policy::Real;
  using FaceT = typename Policy::FaceT;
  static constexpr int PJ = TJ + 4;
  static constexpr int PK = TK + 4;
  alignas(128) Real plane[3][5][PJ][PK];   // planes i .. i+2 (plane i-1 of the own column is kept in registers)
  FaceT fy[5][TJ + 1][TK];
  FaceT fz[5][TJ][TK + 1];
  alignas(8) uint64_t bar;                 // mbarrier of the TMA plane loads
};

// Plane ip into ring slot `slot` cell by cell: cp.async of the cells inside
// the patch (wrapped on periodic axes), zero for cells outside a closed one
// (never read).  The caller commits and waits.
template <class Policy, int TJ, int TK>
__device__ __forceinline__ void load_plane_async(StageSmem<Policy, TJ, TK>& sm, int slot,
                                                 const typename Policy::Store* __restrict__ in,
                                                 const StageGeom& g, int i, int j0, int k0)
{
  static_assert(sizeof(typename Policy::Store) == 8 && sizeof(typename Policy::Real) == 8,
                "cell copies move the stored 8-byte value unchanged");
  constexpr int PJ = TJ + 4, PK = TK + 4;
  const size_t nc = (size_t)g.ni * g.nj * g.nk;
  const int tid = threadIdx.y * TK + threadIdx.x;
  for (int e = tid; e < 5 * PJ * PK; e += TJ * TK) {
    const int v = e / (PJ * PK);
    const int rem = e - v * (PJ * PK);
    const int jj = rem / PK;
    const int kk = rem - jj * PK;
    const int j = axis_idx(j0 - 2 + jj, g.nj, g.per_y);
    const int k = axis_idx(k0 - 2 + kk, g.nk, g.per_z);
    typename Policy::Real* dst = &sm.plane[slot][v][jj][kk];
    if (j >= 0 && k >= 0) {
      const unsigned sa = smem_u32(dst);
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;"
                   :: "r"(sa), "l"(in + v * nc + ((size_t)i * g.nj + j) * g.nk + k) : "memory");
    } else {
      *dst = typename Policy::Real(0);
    }
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

template <class Policy, int TJ, int TK>
__device__ __forceinline__ void load_plane(StageSmem<Policy, TJ, TK>& sm, int slot,
                                           const typename Policy::Store* __restrict__ in,
                                           const typename Policy::Params& pp,
                                           const StageGeom& g, int ip, int j0, int k0)
{
  using Real = typename Policy::Real;
  constexpr int PJ = TJ + 4, PK = TK + 4;
  const int i = axis_idx(ip, g.ni, g.per_x);
  if (i < 0) return;                      // plane outside a closed patch: never read
  const size_t nc = (size_t)g.ni * g.nj * g.nk;
  const int tid = threadIdx.y * TK + threadIdx.x;
  for (int e = tid; e < 5 * PJ * PK; e += TJ * TK) {
    const int v = e / (PJ * PK);
    const int rem = e - v * (PJ * PK);
    const int jj = rem / PK;
    const int kk = rem - jj * PK;
    const int j = axis_idx(j0 - 2 + jj, g.nj, g.per_y);
    const int k = axis_idx(k0 - 2 + kk, g.nk, g.per_z);
    Real val = Real(0);
    if (j >= 0 && k >= 0) {
      val = Policy::load(pp, v, in[v * nc + ((size_t)i * g.nj + j) * g.nk + k]);
    }
    sm.plane[slot][v][jj][kk] = val;
  }
}

// One tile of one patch: columns (j0 .. j0+TJ-1, k0 .. k0+TK-1), planes i0 .. i1-1.
// tm: tensor map of the stage input with box (TK+4, TJ+4, 1, 5), or null.
template <class Policy, int TJ, int TK>
__device__ __forceinline__ void fv_stage_tile(const StageArgs<Policy>& a, const CUtensorMap* tm, int j0, int k0,
                                              int i0, int i1)
{
  using Real = typename Policy::Real;
  using FaceT = typename Policy::FaceT;
  using Smem = StageSmem<Policy, TJ, TK>;
  extern __shared__ __align__(128) unsigned char dn_smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(dn_smem_raw);

  const StageGeom& g = a.g;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int j = j0 + ty, k = k0 + tx;
  const bool own = (j < g.nj) && (k < g.nk);
  const size_t nc = (size_t)g.ni * g.nj * g.nk;
  const Real Ax = a.p.Ax, Ay = a.p.Ay, Az = a.p.Az;
  const int tid = ty * TK + tx;
  // TMA plane loads where no periodic seam crosses the tile's halo (on a
  // closed axis the box cells outside the patch are zero-filled, as the
  // cell copies write them); the box starts at column k0-2, a multiple of 2
  // elements (16 bytes) since TK is even
  constexpr unsigned kPlaneBytes = 5u * (TJ + 4) * (TK + 4) * sizeof(Real);
  const bool tma = tm != nullptr && (!g.per_y || (j0 >= 2 && j0 + TJ + 2 <= g.nj)) &&
                   (!g.per_z || (k0 >= 2 && k0 + TK + 2 <= g.nk)) && (smem_u32(&sm.plane[0][0][0][0]) & 127) == 0;
  if (tma && tid == 0) {
    mbar_init(&sm.bar, 1);
    mbar_init_fence();
  }
  unsigned phase = 0;
  bool tbad = false;

  // a three-plane ring, slot of plane p = p mod 3, rotated by hand: sa, sb,
  // sc hold planes i-1, i, i+1 at the top of iteration i
  int sa = (i0 + 2) % 3, sb = i0 % 3, sc = (i0 + 1) % 3;
  // prologue: planes i0-1 .. i0+1 and the x face below cell i0; the own
  // column of plane i0-2 comes straight from memory
  for (int q = -1; q <= 1; ++q) load_plane<Policy, TJ, TK>(sm, (i0 + q + 3) % 3, a.in, a.p, g, i0 + q, j0, k0);
  __syncthreads();

  FaceT fx_lo[5];
  {
    const bool ex = face_exists(i0, g.ni, g.per_x);
    if (ex && own) {
      Real vl[5], vr[5], F[5];
      const bool sl = cell_ok(i0 - 2, g.ni, g.per_x);
      const bool sr = cell_ok(i0 + 1, g.ni, g.per_x);
      const int im2 = axis_idx(i0 - 2, g.ni, g.per_x);
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        const Real um2 = sl ? Policy::load(a.p, v, a.in[v * nc + ((size_t)im2 * g.nj + j) * g.nk + k]) : Real(0);
        const Real um1 = sm.plane[sa][v][ty + 2][tx + 2];
        const Real up0 = sm.plane[sb][v][ty + 2][tx + 2];
        const Real up1 = sm.plane[sc][v][ty + 2][tx + 2];
        vl[v] = upwind2_left(um2, um1, up0, sl);
        vr[v] = upwind2_right(um1, up0, up1, sr);
      }
      ausm_plus<0>(face_side(vl), face_side(vr), Ax, F);
      #pragma unroll
      for (int v = 0; v < 5; ++v) fx_lo[v] = Policy::face(a.p, v, F[v]);
    } else {
      #pragma unroll
      for (int v = 0; v < 5; ++v) fx_lo[v] = FaceT(0);
    }
  }

  for (int i = i0; i < i1; ++i) {
    // plane i+2 replaces plane i-1 in the ring; the own column of plane i-1
    // (the x face above cell i reads it) moves to registers first
    Real xm1[5];
    #pragma unroll
    for (int v = 0; v < 5; ++v) xm1[v] = sm.plane[sa][v][ty + 2][tx + 2];
    __syncthreads();
    // plane i+2 into the freed slot, arriving while the y and z faces of
    // plane i are evaluated (a plane outside a closed patch is never read)
    const int ip2 = axis_idx(i + 2, g.ni, g.per_x);
    if (ip2 >= 0) {
      if (tma) {
        if (tid == 0) {
          fence_proxy_async_smem();
          mbar_arrive_expect_tx(&sm.bar, kPlaneBytes);
          tma_load_4d(&sm.plane[sa][0][0][0], tm, &sm.bar, k0 - 2, j0 - 2, ip2, 0);
        }
      } else {
        load_plane_async<Policy, TJ, TK>(sm, sa, a.in, g, ip2, j0, k0);
      }
    }
    const int s0 = sb, sp1 = sc, sp2 = sa;

    // y faces of plane i: face at row jj (0..TJ) lies below cell j0+jj
    // (the items beyond one per thread, the faces below halo row TJ, fall to
    // the last warp, and those of the z loop below to the one before it, so
    // that no warp evaluates more than one extra face per plane)
    for (int f = (ty * TK + tx + 32) % (TJ * TK); f < (TJ + 1) * TK; f += TJ * TK) {
      const int jj = f / TK, kk = f - jj * TK;
      const int jf = j0 + jj, kf = k0 + kk;
      FaceT out[5];
      const bool ex = face_exists(jf, g.nj, g.per_y) && kf < g.nk && (g.per_y || jf < g.nj);
      if (ex) {
        Real vl[5], vr[5], F[5];
        const bool sl = cell_ok(jf - 2, g.nj, g.per_y);
        const bool sr = cell_ok(jf + 1, g.nj, g.per_y);
        #pragma unroll
        for (int v = 0; v < 5; ++v) {
          const Real um2 = sm.plane[s0][v][jj][kk + 2];
          const Real um1 = sm.plane[s0][v][jj + 1][kk + 2];
          const Real up0 = sm.plane[s0][v][jj + 2][kk + 2];
          const Real up1 = sm.plane[s0][v][jj + 3][kk + 2];
          vl[v] = upwind2_left(um2, um1, up0, sl);
          vr[v] = upwind2_right(um1, up0, up1, sr);
        }
        ausm_plus<1>(face_side(vl), face_side(vr), Ay, F);
        #pragma unroll
        for (int v = 0; v < 5; ++v) out[v] = Policy::face(a.p, v, F[v]);
      } else {
        #pragma unroll
        for (int v = 0; v < 5; ++v) out[v] = FaceT(0);
      }
      #pragma unroll
      for (int v = 0; v < 5; ++v) sm.fy[v][jj][kk] = out[v];
    }

    // z faces of plane i: face at column kk (0..TK) lies below cell k0+kk
    for (int f = (ty * TK + tx + 64) % (TJ * TK); f < TJ * (TK + 1); f += TJ * TK) {
      const int jj = f / (TK + 1), kk = f - jj * (TK + 1);
      const int jf = j0 + jj, kf = k0 + kk;
      FaceT out[5];
      const bool ex = face_exists(kf, g.nk, g.per_z) && jf < g.nj && (g.per_z || kf < g.nk);
      if (ex) {
        Real vl[5], vr[5], F[5];
        const bool sl = cell_ok(kf - 2, g.nk, g.per_z);
        const bool sr = cell_ok(kf + 1, g.nk, g.per_z);
        #pragma unroll
        for (int v = 0; v < 5; ++v) {
          const Real um2 = sm.plane[s0][v][jj + 2][kk];
          const Real um1 = sm.plane[s0][v][jj + 2][kk + 1];
          const Real up0 = sm.plane[s0][v][jj + 2][kk + 2];
          const Real up1 = sm.plane[s0][v][jj + 2][kk + 3];
          vl[v] = upwind2_left(um2, um1, up0, sl);
          vr[v] = upwind2_right(um1, up0, up1, sr);
        }
        ausm_plus<2>(face_side(vl), face_side(vr), Az, F);
        #pragma unroll
        for (int v = 0; v < 5; ++v) out[v] = Policy::face(a.p, v, F[v]);
      } else {
        #pragma unroll
        for (int v = 0; v < 5; ++v) out[v] = FaceT(0);
      }
      #pragma unroll
      for (int v = 0; v < 5; ++v) sm.fz[v][jj][kk] = out[v];
    }
    // plane i+2 has arrived (this thread's copies, or the TMA box); the
    // barrier publishes it and the y and z faces
    if (ip2 >= 0) {
      if (tma) {
        tbad |= !mbar_wait(&sm.bar, phase);
        phase ^= 1u;
      } else {
        asm volatile("cp.async.wait_group 0;" ::: "memory");
      }
    }
    __syncthreads();

    // x face above cell i (between i and i+1), own column
    FaceT fx_hi[5];
    {

      const bool ex = face_exists(i + 1, g.ni, g.per_x);
      if (ex && own) {
        Real vl[5], vr[5], F[5];
        const bool sl = cell_ok(i - 1, g.ni, g.per_x);
        const bool sr = cell_ok(i + 2, g.ni, g.per_x);
        #pragma unroll
        for (int v = 0; v < 5; ++v) {
          const Real um2 = xm1[v];
          const Real um1 = sm.plane[s0][v][ty + 2][tx + 2];
          const Real up0 = sm.plane[sp1][v][ty + 2][tx + 2];
          const Real up1 = sm.plane[sp2][v][ty + 2][tx + 2];
          vl[v] = upwind2_left(um2, um1, up0, sl);
          vr[v] = upwind2_right(um1, up0, up1, sr);
        }
        ausm_plus<0>(face_side(vl), face_side(vr), Ax, F);
        #pragma unroll
        for (int v = 0; v < 5; ++v) fx_hi[v] = Policy::face(a.p, v, F[v]);
      } else {
        #pragma unroll
        for (int v = 0; v < 5; ++v) fx_hi[v] = FaceT(0);
      }
    }


    if (own) {
      const size_t c = ((size_t)i * g.nj + j) * g.nk + k;
      const bool act = a.active ? (a.active[c] != 0) : true;
      int bad = 0;
      FaceT res[5];
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        FaceT r = fx_lo[v];
        r += sm.fy[v][ty][tx];
        r += sm.fz[v][ty][tx];
        r -= sm.fz[v][ty][tx + 1];
        r -= sm.fy[v][ty + 1][tx];
        r -= fx_hi[v];
        res[v] = r;
      }
      if (a.wall.any && (i == 0 || i == g.ni - 1 || j == 0 || j == g.nj - 1 || k == 0 || k == g.nk - 1)) {
        Real U[5];
        #pragma unroll
        for (int v = 0; v < 5; ++v) U[v] = sm.plane[s0][v][ty + 2][tx + 2];
        add_wall_fluxes(a.wall, g.ni, g.nj, g.nk, g.per_x, g.per_y, g.per_z, i, j, k, U, Ax, Ay, Az, res,
                        [&](int v, Real F) { return Policy::face(a.p, v, F); });
      }
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        const int bad_before = bad;
        const FaceT r = res[v];
        typename Policy::Store o;
        if (act) {
          o = Policy::update(a.p, v, a.un[v * nc + c], r, bad);
        } else {
          o = a.in[v * nc + c];
        }
        a.out[v * nc + c] = o;
        if (bad != bad_before && a.err_info &&
            atomicCAS(&a.err_info[0], ~0ull, (unsigned long long)c) == ~0ull) {
          a.err_info[1] = (unsigned long long)v;
          a.err_info[2] = (unsigned long long)__double_as_longlong((double)a.un[v * nc + c]);
          a.err_info[3] = (unsigned long long)__double_as_longlong((double)r);
        }
      }
      if (bad && a.err) atomicOr(a.err, bad);
    }
    #pragma unroll
    for (int v = 0; v < 5; ++v) fx_lo[v] = fx_hi[v];
    sa = sb;
    sb = sc;
    sc = sp2;
  }
  if (tbad && a.err) atomicOr(a.err, 32);
}

// Parameters of the single-patch launch: the stage arguments and the tensor
// map of the stage input (valid when tma != 0).
template <class Policy>
struct StageLaunch {
  CUtensorMap tm;
  StageArgs<Policy> a;
  int tma;
};

// One patch per launch: grid (k tiles, j tiles, i chunks).
template <class Policy, int TJ, int TK>
__global__ void __launch_bounds__(TJ * TK)
fv_stage_kernel(const __grid_constant__ StageLaunch<Policy> L)
{
  const int i0 = blockIdx.z * L.a.g.i_chunk;
  fv_stage_tile<Policy, TJ, TK>(L.a, L.tma ? &L.tm : nullptr, blockIdx.y * TJ, blockIdx.x * TK, i0,
                                min(L.a.g.ni, i0 + L.a.g.i_chunk));
}

} // namespace dn
