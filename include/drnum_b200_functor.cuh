/* drnum_b200_functor.cuh -- generic flux-functor stage for CUDA C++ callers.
 *
 * The reference iterates a flux functor OP over the faces of a patch
 * (GPU_CartesianIterator<DIM, OP>, iterators/gpu_cartesianiterator.h:54-304,
 * and the CPU CartesianIterator<DIM, OP>, iterators/cartesianiterator.h:
 * 87-325).  OP is duck-typed:
 *
 *   template <typename PATCH> __device__ void xField(PATCH* patch,
 *       size_t i, size_t j, size_t k, double x, double y, double z,
 *       double A, double* flux);        // face between i-1 and i, flux += ...
 *   ... yField, zField (faces below j, below k), and the patch-face methods
 *   xWallM, xWallP, yWallM, yWallP, zWallM, zWallP with the same signature.
 *
 * dn::launch_functor_stage<OP>(L, op) runs one RK stage of one patch with
 * such a functor as ONE fused kernel: every face is evaluated once per CTA
 * (x faces carried in registers along each thread's column, y and z faces
 * exchanged through shared memory), the residual of a cell is summed in
 * registers in the order the reference's single-thread CPU iterator
 * produces (+x_lo +y_lo +z_lo -z_hi -y_hi -x_hi, then the patch faces x-min,
 * x-max, y-min, y-max, z-min, z-max; cartesianiterator.h:115-308), and
 * out = un + factor/dV * residual is written once (inactive cells copy
 * their input, cartesianiterator.h:311-320).  Compiled without FMA
 * contraction (nvcc -fmad=false) and given a functor whose arithmetic
 * follows the reference's, the result equals the reference CPU iterator bit
 * for bit.
 *
 * The PATCH a functor sees is dn::FunctorPatch, a device view of the stage
 * input with the accessors the reference's functors and reconstructions call
 * (f, getVar, checkRange, index, isSplitFace, sizeI/J/K, dx/dy/dz, ...).
 * Inside the stage kernel the view reads from a shared-memory copy of the
 * CTA's tile: planes i-1 .. i+2 of the current plane i with a two-cell halo
 * in j and k, copied asynchronously one plane ahead (the stencils of the
 * reference's reconstructions and viscous gradients stay inside it); reads
 * outside that window go to global memory.
 * Periodic axes wrap indices (size_t arithmetic that went below zero wraps
 * too), so a functor needs no ghost layers; closed axes behave as the
 * reference's patch edges (checkRange false outside).  Field 0 is the stage
 * input, the only field a flux functor reads.
 *
 * Coordinates passed to the functor are cell centres 0.5*d + n*d
 * (gpu_cartesianiterator.h:58-62); wall calls get the reference CPU
 * iterator's arguments (face index 0 or n on the wall axis).
 *
 * Install a stage function that calls launch_functor_stage with
 * dn_set_stage_function (drnum_b200.h) to run it inside dn_rk_step. */
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include "drnum_b200.h"

namespace dn {

/* device view of one patch's stage input */
class FunctorPatch
{
public:
  const double* m_In = nullptr;
  const unsigned char* m_Active = nullptr;
  size_t m_N[3] = {0, 0, 0};
  int m_Per[3] = {0, 0, 0};
  double m_D[3] = {1, 1, 1};
  size_t m_NC = 0;
  int m_Id = 0;
  /* shared-memory window (set by the stage kernel, null elsewhere): planes
     m_P0 .. m_P0+3 in ring slots m_S0, m_S0+1, ... (mod kSlots), rows
     m_J0 .. m_J0+m_WJ-1, columns m_K0 .. m_K0+m_WK-1, [slot][var][row][col] */
  static constexpr int kSlots = 5;
  const double* m_Tile = nullptr;
  long long m_P0 = 0, m_J0 = 0, m_K0 = 0;
  int m_S0 = 0, m_WJ = 0, m_WK = 0;

  __device__ __forceinline__ size_t sizeI() const { return m_N[0]; }
  __device__ __forceinline__ size_t sizeJ() const { return m_N[1]; }
  __device__ __forceinline__ size_t sizeK() const { return m_N[2]; }
  __device__ __forceinline__ size_t sizeL() const { return m_NC; }
  __device__ __forceinline__ size_t numVariables() const { return 5; }
  __device__ __forceinline__ double dx() const { return m_D[0]; }
  __device__ __forceinline__ double dy() const { return m_D[1]; }
  __device__ __forceinline__ double dz() const { return m_D[2]; }
  __device__ __forceinline__ double idx() const { return 1.0/m_D[0]; }
  __device__ __forceinline__ double idy() const { return 1.0/m_D[1]; }
  __device__ __forceinline__ double idz() const { return 1.0/m_D[2]; }
  __device__ __forceinline__ double dV() const { return m_D[0]*m_D[1]*m_D[2]; }
  __device__ __forceinline__ int getIndex() const { return m_Id; }

  /* index along axis a, wrapped on a periodic axis; -1 outside a closed one */
  __device__ __forceinline__ long long axis(int a, size_t x) const
  {
    long long s = (long long)x;
    const long long n = (long long)m_N[a];
    if (m_Per[a]) {
      // stencils reach a few cells past the patch: one fold, a remainder
      // only for indices further out
      if (s < 0) s += n;
      else if (s >= n) s -= n;
      if (s < 0 || s >= n) {
        s %= n;
        if (s < 0) s += n;
      }
      return s;
    }
    return (s < 0 || s >= n) ? -1 : s;
  }
  __device__ __forceinline__ bool checkRange(size_t i, size_t j, size_t k) const
  {
    return axis(0, i) >= 0 && axis(1, j) >= 0 && axis(2, k) >= 0;
  }
  __device__ __forceinline__ size_t index(size_t i, size_t j, size_t k) const
  {
    return ((size_t)axis(0, i)*m_N[1] + (size_t)axis(1, j))*m_N[2] + (size_t)axis(2, k);
  }
  __device__ __forceinline__ bool isSplitFace(size_t, size_t) const { return false; }
  __device__ __forceinline__ bool isActive(size_t i, size_t j, size_t k) const
  {
    return m_Active ? m_Active[index(i, j, k)] != 0 : true;
  }
  /* f(field, var, i, j, k) of the stage input (field is ignored: flux
     functors read field 0) */
  __device__ __forceinline__ double f(size_t, size_t var, size_t i, size_t j, size_t k) const
  {
    if (m_Tile) {
      /* indices that went below zero wrapped as size_t; as signed values
         they address the halo, which holds the wrapped cells */
      const long long dp = (long long)i - m_P0, dj = (long long)j - m_J0, dk = (long long)k - m_K0;
      if ((unsigned long long)dp < 4ull && (unsigned long long)dj < (unsigned long long)m_WJ &&
          (unsigned long long)dk < (unsigned long long)m_WK) {
        int sl = m_S0 + (int)dp;
        if (sl >= kSlots) sl -= kSlots;
        return m_Tile[(((size_t)sl*5 + var)*m_WJ + (size_t)dj)*m_WK + (size_t)dk];
      }
    }
    return f_global(var, i, j, k);
  }
  /* the read outside the shared-memory window, kept out of line: the
     functors call f() at dozens of sites, and inlining the index folding
     at each of them filled the instruction cache */
  __device__ __noinline__ double f_global(size_t var, size_t i, size_t j, size_t k) const
  {
    return __ldg(m_In + var*m_NC + index(i, j, k));
  }
  __device__ __forceinline__ void getVar(size_t field, size_t i, size_t j, size_t k, double* var) const
  {
    for (size_t v = 0; v < 5; ++v) var[v] = f(field, v, i, j, k);
  }
  template <typename DIMT>
  __device__ __forceinline__ void getVar(DIMT, size_t field, size_t i, size_t j, size_t k, double* var) const
  {
    getVar(field, i, j, k, var);
  }
  /* Gradient along axis A at cell (i, j, k): central difference, one-sided
     where a neighbour lies outside a closed axis (the difference is then
     taken to the cell itself with the doubled factor), as
     CartesianPatch::getXGrad/getYGrad/getZGrad (cartesianpatch_common.h:
     188-312, whose y form alone returns zero on an axis of two cells or
     fewer); the viscous functors read their transverse gradients here. */
  template <int A>
  __device__ __forceinline__ void grad(size_t field, size_t i, size_t j, size_t k, double* g) const
  {
    if (A == 1 && m_N[1] <= 2) {
      for (int v = 0; v < 5; ++v) g[v] = 0;
      return;
    }
    const size_t c[3] = {i, j, k};
    double D = 0.5/m_D[A];
    size_t n1 = c[A] - 1, n2 = c[A] + 1;
    if (axis(A, n1) < 0) { n1 = c[A]; D *= 2; }
    if (axis(A, n2) < 0) { n2 = c[A]; D *= 2; }
    size_t a1[3] = {i, j, k}, a2[3] = {i, j, k};
    a1[A] = n1;
    a2[A] = n2;
    double v1[5];
    getVar(field, a2[0], a2[1], a2[2], g);
    getVar(field, a1[0], a1[1], a1[2], v1);
    for (int v = 0; v < 5; ++v) {
      g[v] -= v1[v];
      g[v] *= D;
    }
  }
  template <typename DIMT>
  __device__ __forceinline__ void getXGrad(DIMT, size_t field, size_t i, size_t j, size_t k, double* g) const
  { grad<0>(field, i, j, k, g); }
  template <typename DIMT>
  __device__ __forceinline__ void getYGrad(DIMT, size_t field, size_t i, size_t j, size_t k, double* g) const
  { grad<1>(field, i, j, k, g); }
  template <typename DIMT>
  __device__ __forceinline__ void getZGrad(DIMT, size_t field, size_t i, size_t j, size_t k, double* g) const
  { grad<2>(field, i, j, k, g); }
};

namespace functor_detail {

__device__ __forceinline__ bool face_exists(int x, int n, int per)
{
  if (n <= 2) return false;                  /* cartesianiterator.h:149,160,171 */
  return per ? true : (x >= 1 && x <= n - 1);
}

template <int TJ, int TK>
struct Smem {
  static constexpr int PJ = TJ + 4, PK = TK + 4;
  double plane[FunctorPatch::kSlots][5][PJ][PK];   /* ring of planes, rows j0-2.., columns k0-2.. */
  double fy[5][TJ + 1][TK];                  /* face below row jj of the tile */
  double fz[5][TJ][TK + 1];                  /* face below column kk */
};

/* ring slot of plane p >= -1 */
__device__ __forceinline__ int ring_slot(int p) { return (p + FunctorPatch::kSlots) % FunctorPatch::kSlots; }

/* Plane p of the stage input into its ring slot, cell by cell with cp.async:
   cells inside the patch (wrapped on periodic axes), zero for cells outside
   a closed one.  Commits one copy group. */
template <int TJ, int TK>
__device__ __forceinline__ void load_plane(Smem<TJ, TK>& sm, const FunctorPatch& P, int p, int j0, int k0)
{
  constexpr int PJ = TJ + 4, PK = TK + 4;
  const int sl = ring_slot(p);
  const long long ip = P.axis(0, (size_t)(long long)p);
  const int tid = threadIdx.y * TK + threadIdx.x;
  for (int e = tid; e < 5 * PJ * PK; e += TJ * TK) {
    const int v = e / (PJ * PK);
    const int rem = e - v * (PJ * PK);
    const int jj = rem / PK, kk = rem - jj * PK;
    const long long jg = P.axis(1, (size_t)(long long)(j0 - 2 + jj));
    const long long kg = P.axis(2, (size_t)(long long)(k0 - 2 + kk));
    double* dst = &sm.plane[sl][v][jj][kk];
    if (ip >= 0 && jg >= 0 && kg >= 0) {
      const double* src = P.m_In + v*P.m_NC + ((size_t)ip*P.m_N[1] + (size_t)jg)*P.m_N[2] + (size_t)kg;
      const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"(sa), "l"(src) : "memory");
    } else {
      *dst = 0.0;
    }
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

struct Args {
  FunctorPatch view;
  const double* un;
  double* out;
  double pf;                                 /* factor / dV */
  int i_chunk;
};

template <class OP, int TJ, int TK>
__global__ void __launch_bounds__(TJ * TK, 2)
functor_stage_kernel(const Args a, OP op)
{
  extern __shared__ __align__(16) unsigned char functor_smem_raw[];
  Smem<TJ, TK>& sm = *reinterpret_cast<Smem<TJ, TK>*>(functor_smem_raw);
  FunctorPatch P = a.view;
  const int ni = (int)P.m_N[0], nj = (int)P.m_N[1], nk = (int)P.m_N[2];
  const int px = P.m_Per[0], py = P.m_Per[1], pz = P.m_Per[2];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int j0 = blockIdx.y * TJ, k0 = blockIdx.x * TK;
  const int i0 = blockIdx.z * a.i_chunk;
  const int i1 = min(ni, i0 + a.i_chunk);
  const int j = j0 + ty, k = k0 + tx;
  const bool own = j < nj && k < nk;
  const double dx = P.m_D[0], dy = P.m_D[1], dz = P.m_D[2];
  const double Ax = dy*dz, Ay = dx*dz, Az = dx*dy;   /* cartesianiterator.h:96-98 */
  const double yc = 0.5*dy + j*dy, zc = 0.5*dz + k*dz;

  /* planes i0-1 .. i0+2 into the ring; the first x face (below i0) reads
     plane i0-2 from global memory */
  for (int p = i0 - 1; p <= i0 + 2; ++p) load_plane<TJ, TK>(sm, P, p, j0, k0);
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  P.m_Tile = &sm.plane[0][0][0][0];
  P.m_J0 = j0 - 2;
  P.m_K0 = k0 - 2;
  P.m_WJ = TJ + 4;
  P.m_WK = TK + 4;
  P.m_P0 = i0 - 1;
  P.m_S0 = ring_slot(i0 - 1);

  double flo[5];
  if (own && face_exists(i0, ni, px)) {
    double F[5] = {0, 0, 0, 0, 0};
    op.xField(&P, (size_t)i0, (size_t)j, (size_t)k, 0.5*dx + i0*dx, yc, zc, Ax, F);
    for (int v = 0; v < 5; ++v) flo[v] = F[v];
  } else {
    for (int v = 0; v < 5; ++v) flo[v] = 0.0;
  }

  for (int i = i0; i < i1; ++i) {
    /* plane i+3 into the slot of plane i-2 (last read in the previous
       iteration, before its final barrier); the window moves to i-1 .. i+2 */
    if (i + 3 <= i1 + 1) load_plane<TJ, TK>(sm, P, i + 3, j0, k0);
    P.m_P0 = i - 1;
    P.m_S0 = ring_slot(i - 1);
    const double xc = 0.5*dx + i*dx;
    double fhi[5];
    if (own && face_exists(i + 1, ni, px)) {
      double F[5] = {0, 0, 0, 0, 0};
      op.xField(&P, (size_t)(i + 1), (size_t)j, (size_t)k, 0.5*dx + (i + 1)*dx, yc, zc, Ax, F);
      for (int v = 0; v < 5; ++v) fhi[v] = F[v];
    } else {
      for (int v = 0; v < 5; ++v) fhi[v] = 0.0;
    }
    // y and z faces below the own cell; the faces below the halo row TJ and
    // the halo column TK go to the last two warps, so that no warp
    // evaluates more than one extra face per plane
    auto y_face = [&](int jj, int kk) {
      const int jf = j0 + jj, kf = k0 + kk;
      double F[5] = {0, 0, 0, 0, 0};
      if (kf < nk && face_exists(jf, nj, py) && (py || jf < nj))
        op.yField(&P, (size_t)i, (size_t)jf, (size_t)kf, xc, 0.5*dy + jf*dy, 0.5*dz + kf*dz, Ay, F);
      for (int v = 0; v < 5; ++v) sm.fy[v][jj][kk] = F[v];
    };
    auto z_face = [&](int jj, int kk) {
      const int jf = j0 + jj, kf = k0 + kk;
      double F[5] = {0, 0, 0, 0, 0};
      if (jf < nj && face_exists(kf, nk, pz) && (pz || kf < nk))
        op.zField(&P, (size_t)i, (size_t)jf, (size_t)kf, xc, 0.5*dy + jf*dy, 0.5*dz + kf*dz, Az, F);
      for (int v = 0; v < 5; ++v) sm.fz[v][jj][kk] = F[v];
    };
    y_face(ty, tx);
    z_face(ty, tx);
    {
      constexpr int NW = TJ * TK / 32;
      const int warp = (ty * TK + tx) >> 5, lane = (ty * TK + tx) & 31;
      if (warp == NW - 1)
        for (int kk = lane; kk < TK; kk += 32) y_face(TJ, kk);
      if (warp == (NW >= 2 ? NW - 2 : 0))
        for (int jj = lane; jj < TJ; jj += 32) z_face(jj, TK);
    }
    __syncthreads();
    if (own) {
      double r[5];
      for (int v = 0; v < 5; ++v) {
        double s = flo[v];
        s += sm.fy[v][ty][tx];
        s += sm.fz[v][ty][tx];
        s -= sm.fz[v][ty][tx + 1];
        s -= sm.fy[v][ty + 1][tx];
        s -= fhi[v];
        r[v] = s;
      }
      /* patch faces of closed axes (cartesianiterator.h:190-308) */
      if (!px && ni > 2 && (i == 0 || i == ni - 1)) {
        double F[5] = {0, 0, 0, 0, 0};
        if (i == 0) {
          op.xWallM(&P, (size_t)0, (size_t)j, (size_t)k, 0.5*dx, yc, zc, Ax, F);
          for (int v = 0; v < 5; ++v) r[v] += F[v];
        }
        if (i == ni - 1) {
          for (int v = 0; v < 5; ++v) F[v] = 0;
          op.xWallP(&P, (size_t)ni, (size_t)j, (size_t)k, 0.5*dx + ni*dx, yc, zc, Ax, F);
          for (int v = 0; v < 5; ++v) r[v] -= F[v];
        }
      }
      if (!py && nj > 2 && (j == 0 || j == nj - 1)) {
        double F[5] = {0, 0, 0, 0, 0};
        if (j == 0) {
          op.yWallM(&P, (size_t)i, (size_t)0, (size_t)k, xc, 0.5*dy, zc, Ay, F);
          for (int v = 0; v < 5; ++v) r[v] += F[v];
        }
        if (j == nj - 1) {
          for (int v = 0; v < 5; ++v) F[v] = 0;
          op.yWallP(&P, (size_t)i, (size_t)nj, (size_t)k, xc, 0.5*dy + nj*dy, zc, Ay, F);
          for (int v = 0; v < 5; ++v) r[v] -= F[v];
        }
      }
      if (!pz && nk > 2 && (k == 0 || k == nk - 1)) {
        double F[5] = {0, 0, 0, 0, 0};
        if (k == 0) {
          op.zWallM(&P, (size_t)i, (size_t)j, (size_t)0, xc, yc, 0.5*dz, Az, F);
          for (int v = 0; v < 5; ++v) r[v] += F[v];
        }
        if (k == nk - 1) {
          for (int v = 0; v < 5; ++v) F[v] = 0;
          op.zWallP(&P, (size_t)i, (size_t)j, (size_t)nk, xc, yc, 0.5*dz + nk*dz, Az, F);
          for (int v = 0; v < 5; ++v) r[v] -= F[v];
        }
      }
      const size_t c = ((size_t)i*nj + j)*nk + k;
      const bool act = P.m_Active ? P.m_Active[c] != 0 : true;
      for (int v = 0; v < 5; ++v) {
        const size_t e = v*P.m_NC + c;
        a.out[e] = act ? a.un[e] + a.pf*r[v] : P.m_In[e];
      }
    }
    for (int v = 0; v < 5; ++v) flo[v] = fhi[v];
    /* plane i+3 has arrived; the barrier publishes it and ends the reads of
       the face arrays and of plane i-1 */
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
  }
}

} // namespace functor_detail

/* Launches one stage of patch L->patch with functor op on L->stream.
 * Returns the launch's cudaError_t. */
template <class OP, int TJ = 8, int TK = 32>
cudaError_t launch_functor_stage(const dn_stage_launch* L, const OP& op)
{
  functor_detail::Args a;
  a.view.m_In = L->in;
  a.view.m_Active = L->active;
  a.view.m_N[0] = (size_t)L->ni; a.view.m_N[1] = (size_t)L->nj; a.view.m_N[2] = (size_t)L->nk;
  for (int d = 0; d < 3; ++d) a.view.m_Per[d] = L->periodic[d];
  a.view.m_D[0] = L->dx; a.view.m_D[1] = L->dy; a.view.m_D[2] = L->dz;
  a.view.m_NC = (size_t)L->ni * L->nj * L->nk;
  a.view.m_Id = L->patch;
  a.un = L->un;
  a.out = L->out;
  a.pf = L->factor / (L->dx * L->dy * L->dz);   /* cartesianiterator.h:311 */
  const int tk = (L->nk + TK - 1) / TK, tj = (L->nj + TJ - 1) / TJ;
  /* plane ranges: about four CTAs per SM in total */
  const long long want = 4LL * (L->num_sms > 0 ? L->num_sms : 148);
  long long chunks = want / ((long long)tk * tj);
  if (chunks < 1) chunks = 1;
  if (chunks > L->ni) chunks = L->ni;
  a.i_chunk = (int)((L->ni + chunks - 1) / chunks);
  const dim3 grid(tk, tj, (L->ni + a.i_chunk - 1) / a.i_chunk);
  const dim3 block(TK, TJ);
  auto kern = functor_detail::functor_stage_kernel<OP, TJ, TK>;
  const int smem = (int)sizeof(functor_detail::Smem<TJ, TK>);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  kern<<<grid, block, smem, (cudaStream_t)L->stream>>>(a, op);
  return cudaGetLastError();
}

} // namespace dn
