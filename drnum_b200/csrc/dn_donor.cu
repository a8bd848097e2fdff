// Donor copy kernels (Patch::accessDonorDataDirect, patch.cpp:573-653;
// GPU_PatchIterator_kernelCopyDonorData, gpu_patchiterator.h:141-188).
//
// The reference zeroes every receiving cell and then runs one pass (CPU) or
// one launch (GPU) per donor patch that adds that donor's weighted sum.
// Here one thread owns one receiving cell and walks its donor groups in
// table order, so a single launch serves all patches, nothing is zeroed in
// HBM and there are no atomics.  Built with -fmad=false: the FP64 form
// rounds like the reference CPU loop (product, then sum, per contribution;
// donor sums added to a zero-initialised accumulator).
#include "dn_donor.cuh"
#include "fv_fx32.cuh"

namespace dn {

namespace {

constexpr int kDonorThreads = 256;

// table entries in the plan's width (NARROW: the 32-bit copies)
template <bool NARROW> __device__ __forceinline__ int64_t rv_cell_at(const DonorPlan& p, int r)
{ return NARROW ? (int64_t)p.rv_cell32[r] : p.rv_cell[r]; }
template <bool NARROW> __device__ __forceinline__ int64_t gp_wi_at(const DonorPlan& p, int g)
{ return NARROW ? (int64_t)p.gp_wi32[g] : p.gp_wi[g]; }
template <bool NARROW> __device__ __forceinline__ int64_t idx_at(const DonorPlan& p, int64_t e)
{ return NARROW ? (int64_t)p.idx32[e] : p.idx[e]; }

template <bool NARROW>
__global__ void __launch_bounds__(kDonorThreads)
k_donor_copy_f64(const DonorPlan p, int buf)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= p.n_recv) return;
  const int pr = p.rv_patch[r];
  const int64_t cell = rv_cell_at<NARROW>(p, r);
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int g = p.rv_grp[r]; g < p.rv_grp[r + 1]; ++g) {
    const int pd = p.gp_donor[g];
    const double* src = static_cast<const double*>(p.bufs[pd * 3 + buf]);
    const int64_t ncd = p.nc[pd];
    const int64_t w0 = gp_wi_at<NARROW>(p, g);
    double inter[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int s = 0; s < p.gp_stride[g]; ++s) {
      const int64_t c = idx_at<NARROW>(p, w0 + s);
      const double w = p.w[w0 + s];
      #pragma unroll
      for (int v = 0; v < 5; ++v) inter[v] += src[v * ncd + c] * w;
    }
    #pragma unroll
    for (int v = 0; v < 5; ++v) acc[v] += inter[v];
  }
  double* dst = static_cast<double*>(p.bufs[pr * 3 + buf]);
  const int64_t ncr = p.nc[pr];
  #pragma unroll
  for (int v = 0; v < 5; ++v) dst[v * ncr + cell] = acc[v];
}

template <bool NARROW>
__global__ void __launch_bounds__(kDonorThreads)
k_donor_copy_fx32(const DonorPlan p, int buf, int* err)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= p.n_recv) return;
  const int pr = p.rv_patch[r];
  const int64_t cell = rv_cell_at<NARROW>(p, r);
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int g = p.rv_grp[r]; g < p.rv_grp[r + 1]; ++g) {
    const int pd = p.gp_donor[g];
    const int32_t* src = static_cast<const int32_t*>(p.bufs[pd * 3 + buf]);
    const int64_t ncd = p.nc[pd];
    const int64_t w0 = gp_wi_at<NARROW>(p, g);
    double inter[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int s = 0; s < p.gp_stride[g]; ++s) {
      const int64_t c = idx_at<NARROW>(p, w0 + s);
      const double w = p.w[w0 + s];
      #pragma unroll
      for (int v = 0; v < 5; ++v) {
        const double u = p.base[pd * 5 + v] + p.quantum[pd * 5 + v] * (double)src[v * ncd + c];
        inter[v] += u * w;
      }
    }
    #pragma unroll
    for (int v = 0; v < 5; ++v) acc[v] += inter[v];
  }
  int32_t* dst = static_cast<int32_t*>(p.bufs[pr * 3 + buf]);
  const int64_t ncr = p.nc[pr];
  int bad = 0;
  #pragma unroll
  for (int v = 0; v < 5; ++v) {
    double o = rint((acc[v] - p.base[pr * 5 + v]) / p.quantum[pr * 5 + v]);
    if (!(fabs(o) < (double)kFxLimit)) {   // out of the receiving patch's offset range (or NaN)
      bad = 4;
      o = 0.0;
    }
    dst[v * ncr + cell] = (int32_t)o;
  }
  if (bad && err) atomicOr(err, bad);
}

int blocks_for(int n) { return (n + kDonorThreads - 1) / kDonorThreads; }

} // namespace

cudaError_t launch_donor_copy_f64(const DonorPlan& p, int buf, cudaStream_t st)
{
  if (p.n_recv <= 0) return cudaSuccess;
  if (p.narrow) k_donor_copy_f64<true><<<blocks_for(p.n_recv), kDonorThreads, 0, st>>>(p, buf);
  else k_donor_copy_f64<false><<<blocks_for(p.n_recv), kDonorThreads, 0, st>>>(p, buf);
  return cudaGetLastError();
}

cudaError_t launch_donor_copy_fx32(const DonorPlan& p, int buf, int* err, cudaStream_t st)
{
  if (p.n_recv <= 0) return cudaSuccess;
  if (p.narrow) k_donor_copy_fx32<true><<<blocks_for(p.n_recv), kDonorThreads, 0, st>>>(p, buf, err);
  else k_donor_copy_fx32<false><<<blocks_for(p.n_recv), kDonorThreads, 0, st>>>(p, buf, err);
  return cudaGetLastError();
}

} // namespace dn
