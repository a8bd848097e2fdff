// Level-set slip-wall boundary condition (CPU_LevelSetObjectBC::operator(),
// cpu_levelsetobjectbc.h:58-90, with LSOBCCompressibleEulerOp,
// lsobccompressibleeulerop.h:49-144).
//
// The reference runs two passes over the inner layer cells: `access`
// interpolates each cell's mirror-point state into the abuse field, then
// `operateInner` writes the cell: density and energy from the mirror state,
// the momentum reflected at the wall normal and relaxed (relax 0.5).  Here
// the two passes are two launches with one thread per layer cell and a
// compact scratch of 5 values per layer cell instead of a whole abuse field.
// Built with -fmad=false: the FP64 form rounds like the reference's CPU
// path.  The GPU level-set path's average (further below) is evaluated the
// same way, without contraction (the reference's own nvcc build of that
// kernel may fuse `var += weight * value` into an FMA).
#include "dn_lsbc.cuh"
#include "fv_fx32.cuh"

namespace dn {

namespace {

constexpr int kLsThreads = 128;

template <bool FX>
__device__ __forceinline__ double load_u(const LsPlan& p, int pr, int buf, int v, int64_t c)
{
  const int64_t nc = p.nc[pr];
  if (FX) {
    const int32_t* f = static_cast<const int32_t*>(p.bufs[pr * 3 + buf]);
    return p.base[pr * 5 + v] + p.quantum[pr * 5 + v] * (double)f[v * nc + c];
  }
  const double* f = static_cast<const double*>(p.bufs[pr * 3 + buf]);
  return f[v * nc + c];
}

template <bool FX>
__global__ void __launch_bounds__(kLsThreads)
k_ls_access(const LsPlan p, int buf)
{
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= p.n) return;
  const int pr = p.patch[q];
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int s = 0; s < 8; ++s) {
    const int64_t d = p.donor[(size_t)q * 8 + s];
    const double w = p.w[(size_t)q * 8 + s];
    #pragma unroll
    for (int v = 0; v < 5; ++v) acc[v] += w * load_u<FX>(p, pr, buf, v, d);
  }
  #pragma unroll
  for (int v = 0; v < 5; ++v) p.acc[(size_t)q * 5 + v] = acc[v];
}

template <bool FX>
__global__ void __launch_bounds__(kLsThreads)
k_ls_operate(const LsPlan p, int buf, int* err)
{
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= p.n) return;
  const int pr = p.patch[q];
  const int64_t c = p.cell[q];
  const double* a = p.acc + (size_t)q * 5;
  const double gxn = p.grad[(size_t)q * 3 + 0], gyn = p.grad[(size_t)q * 3 + 1], gzn = p.grad[(size_t)q * 3 + 2];
  const double relax = 0.5;
  const double eps = 1.e-6;
  // normal projection of the mirror momentum; reflected ("hard") momentum
  const double rho_uvw_n = a[1] * gxn + a[2] * gyn + a[3] * gzn;
  const double g[3] = {gxn, gyn, gzn};
  double out[5];
  out[0] = a[0];
  out[4] = a[4];
  #pragma unroll
  for (int m = 0; m < 3; ++m) {
    const double cur = load_u<FX>(p, pr, buf, 1 + m, c);
    const double hard = a[1 + m] - 2. * rho_uvw_n * g[m];
    const double diff = cur - hard;
    double damp = fabs(diff) / (fabs(cur) + eps);
    if (damp > (1. - relax)) damp = 1. - relax;
    out[1 + m] = (1. - damp) * hard + damp * cur;
  }
  const int64_t nc = p.nc[pr];
  if (FX) {
    int32_t* f = static_cast<int32_t*>(p.bufs[pr * 3 + buf]);
    int bad = 0;
    #pragma unroll
    for (int v = 0; v < 5; ++v) {
      double o = rint((out[v] - p.base[pr * 5 + v]) / p.quantum[pr * 5 + v]);
      if (!(fabs(o) < (double)kFxLimit)) {
        bad = 8;
        o = 0.0;
      }
      f[v * nc + c] = (int32_t)o;
    }
    if (bad && err) atomicOr(err, bad);
  } else {
    double* f = static_cast<double*>(p.bufs[pr * 3 + buf]);
    #pragma unroll
    for (int v = 0; v < 5; ++v) f[v * nc + c] = out[v];
  }
}

template <bool FX>
__global__ void __launch_bounds__(kLsThreads)
k_lsg_reset(const LsPlan p, int buf, int step_buf)
{
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= p.n_reset) return;
  const int pr = p.reset_patch[q];
  const int64_t c = p.reset_cell[q], nc = p.nc[pr];
  if (FX) {
    const int32_t* s = static_cast<const int32_t*>(p.bufs[pr * 3 + step_buf]);
    int32_t* f = static_cast<int32_t*>(p.bufs[pr * 3 + buf]);
    #pragma unroll
    for (int v = 0; v < 5; ++v) f[v * nc + c] = s[v * nc + c];
  } else {
    const double* s = static_cast<const double*>(p.bufs[pr * 3 + step_buf]);
    double* f = static_cast<double*>(p.bufs[pr * 3 + buf]);
    #pragma unroll
    for (int v = 0; v < 5; ++v) f[v * nc + c] = s[v * nc + c];
  }
}

// GPU_CartesianLevelSetInsideCellsBC_kernel (gpu_cartesianlevelsetbc.h:414-487):
// var += weight * neighbour in the neighbours' order, then var / total weight
template <bool FX>
__global__ void __launch_bounds__(kLsThreads)
k_lsg_gather(const LsPlan p, int buf)
{
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= p.n_avg) return;
  const int64_t b = p.avg_start[q], e = p.avg_start[q + 1];
  if (b == e) return;
  const int pr = p.avg_patch[q];
  double var[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  double total = 0.0;
  for (int64_t m = b; m < e; ++m) {
    const double w = p.avg_w[m];
    const int64_t d = p.avg_nbr[m];
    total += w;
    #pragma unroll
    for (int v = 0; v < 5; ++v) var[v] += w * load_u<FX>(p, pr, buf, v, d);
  }
  #pragma unroll
  for (int v = 0; v < 5; ++v) p.avg_acc[(size_t)q * 5 + v] = var[v] / total;
}

template <bool FX>
__global__ void __launch_bounds__(kLsThreads)
k_lsg_write(const LsPlan p, int buf, int* err)
{
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= p.n_avg) return;
  if (p.avg_start[q] == p.avg_start[q + 1]) return;
  const int pr = p.avg_patch[q];
  const int64_t c = p.avg_cell[q], nc = p.nc[pr];
  const double* a = p.avg_acc + (size_t)q * 5;
  int bad = 0;
  if (FX) {
    int32_t* f = static_cast<int32_t*>(p.bufs[pr * 3 + buf]);
    #pragma unroll
    for (int v = 0; v < 5; ++v) {
      double o = rint((a[v] - p.base[pr * 5 + v]) / p.quantum[pr * 5 + v]);
      if (a[v] != a[v]) {
        bad |= kErrLsAverage;
        o = 0.0;
      } else if (!(fabs(o) < (double)kFxLimit)) {
        bad |= 8;
        o = 0.0;
      }
      f[v * nc + c] = (int32_t)o;
    }
  } else {
    double* f = static_cast<double*>(p.bufs[pr * 3 + buf]);
    #pragma unroll
    for (int v = 0; v < 5; ++v) {
      if (a[v] != a[v]) bad |= kErrLsAverage;
      f[v * nc + c] = a[v];
    }
  }
  if (bad && err) atomicOr(err, bad);
}

} // namespace

cudaError_t launch_levelset_gpu(const LsPlan& p, int buf, int step_buf, bool fixed_point, int* err, cudaStream_t st)
{
  if (p.n_reset > 0) {
    const int blocks = (p.n_reset + kLsThreads - 1) / kLsThreads;
    if (fixed_point) k_lsg_reset<true><<<blocks, kLsThreads, 0, st>>>(p, buf, step_buf);
    else k_lsg_reset<false><<<blocks, kLsThreads, 0, st>>>(p, buf, step_buf);
  }
  if (p.n_avg > 0) {
    const int blocks = (p.n_avg + kLsThreads - 1) / kLsThreads;
    if (fixed_point) {
      k_lsg_gather<true><<<blocks, kLsThreads, 0, st>>>(p, buf);
      k_lsg_write<true><<<blocks, kLsThreads, 0, st>>>(p, buf, err);
    } else {
      k_lsg_gather<false><<<blocks, kLsThreads, 0, st>>>(p, buf);
      k_lsg_write<false><<<blocks, kLsThreads, 0, st>>>(p, buf, err);
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_levelset_bc(const LsPlan& p, int buf, bool fixed_point, int* err, cudaStream_t st)
{
  if (p.n <= 0) return cudaSuccess;
  const int blocks = (p.n + kLsThreads - 1) / kLsThreads;
  if (fixed_point) {
    k_ls_access<true><<<blocks, kLsThreads, 0, st>>>(p, buf);
    k_ls_operate<true><<<blocks, kLsThreads, 0, st>>>(p, buf, err);
  } else {
    k_ls_access<false><<<blocks, kLsThreads, 0, st>>>(p, buf);
    k_ls_operate<false><<<blocks, kLsThreads, 0, st>>>(p, buf, err);
  }
  return cudaGetLastError();
}

} // namespace dn
