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

#include <atomic>

namespace dn {

namespace {

constexpr int kDonorThreads = 256;

// Donor value of variable v at device cell c: FP64 fields as stored, FP32
// bulk offsets dequantised in FP64 (base + quantum * offset).
template <bool FX> struct DonorField;
template <> struct DonorField<false> {
  const double* f;
  using raw = double;
  __device__ __forceinline__ DonorField(const DonorPlan& p, int pd, int buf)
      : f(static_cast<const double*>(p.bufs[pd * 3 + buf])) {}
  __device__ __forceinline__ raw load(int64_t i) const { return f[i]; }
  __device__ __forceinline__ double value(const DonorPlan&, int, int, raw x) const { return x; }
};
template <> struct DonorField<true> {
  const int32_t* f;
  using raw = int32_t;
  __device__ __forceinline__ DonorField(const DonorPlan& p, int pd, int buf)
      : f(static_cast<const int32_t*>(p.bufs[pd * 3 + buf])) {}
  __device__ __forceinline__ raw load(int64_t i) const { return f[i]; }
  __device__ __forceinline__ double value(const DonorPlan& p, int pd, int v, raw x) const
  { return p.base[pd * 5 + v] + p.quantum[pd * 5 + v] * (double)x; }
};

// Writes the accumulated sums to receiving cell `cell` of patch pr.
template <bool FX>
__device__ __forceinline__ void store_recv(const DonorPlan& p, int buf, int pr, int64_t cell, const double acc[5],
                                           int* err)
{
  const int64_t ncr = p.nc[pr];
  if (!FX) {
    double* dst = static_cast<double*>(p.bufs[pr * 3 + buf]);
    #pragma unroll
    for (int v = 0; v < 5; ++v) dst[v * ncr + cell] = acc[v];
    return;
  }
  int32_t* dst = static_cast<int32_t*>(p.bufs[pr * 3 + buf]);
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

// Adds the weighted donor sum of one pattern-form group to acc.
// Contributions are taken BLK at a time: the donor loads of a block are all
// issued before the first product, so a group waits for one memory round
// trip per block instead of one per contribution.  Products and sums keep
// the table order.
template <bool FX, int BLK>
__device__ __forceinline__ void add_group(const DonorPlan& p, int buf, uint4 gr, double acc[5])
{
  const int pd = (int)gr.w;
  const int s0 = (int)gr.y, n = (int)gr.z;
  const int64_t ncd = p.nc[pd];
  const int64_t c0 = (int64_t)gr.x;
  const DonorField<FX> src(p, pd, buf);
  double inter[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int b = 0; b < n; b += BLK) {
    int64_t cc[BLK];
    double w[BLK];
    typename DonorField<FX>::raw x[BLK][5];
    #pragma unroll
    for (int s = 0; s < BLK; ++s) {
      if (b + s < n) {
        cc[s] = c0 + p.pt_off[s0 + b + s];
        w[s] = p.pt_w[s0 + b + s];
      }
    }
    #pragma unroll
    for (int s = 0; s < BLK; ++s) {
      if (b + s < n) {
        #pragma unroll
        for (int v = 0; v < 5; ++v) x[s][v] = src.load(v * ncd + cc[s]);
      }
    }
    #pragma unroll
    for (int s = 0; s < BLK; ++s) {
      if (b + s < n) {
        #pragma unroll
        for (int v = 0; v < 5; ++v) inter[v] += src.value(p, pd, v, x[s][v]) * w[s];
      }
    }
  }
  #pragma unroll
  for (int v = 0; v < 5; ++v) acc[v] += inter[v];
}

// Pattern form: a thread takes receiving cells r, r + stride, ... (stride
// = all threads of the launch) and loads the next cell's table entries
// before it gathers the current cell's donors, so the table loads of one
// cell overlap the donor loads of the one before.
template <bool FX, int BLK>
__global__ void __launch_bounds__(kDonorThreads, 2)
k_donor_copy_pat(const DonorPlan p, int buf, int* err)
{
  const int stride = gridDim.x * blockDim.x;
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= p.n_recv) return;
  int pr = p.rv_patch[r];
  uint32_t cell = p.rv_cell32[r];
  uint4 gr = p.gp_pat[r];
  int g = 0, g1 = 0;
  if (p.rv_more) {
    g = p.rv_more[r];
    g1 = p.rv_more[r + 1];
  }
  for (;;) {
    const int rn = r + stride;
    const bool more = rn < p.n_recv;
    int pr_n = 0, gn = 0, g1n = 0;
    uint32_t cell_n = 0;
    uint4 gr_n = make_uint4(0u, 0u, 0u, 0u);
    if (more) {
      pr_n = p.rv_patch[rn];
      cell_n = p.rv_cell32[rn];
      gr_n = p.gp_pat[rn];
      if (p.rv_more) {
        gn = p.rv_more[rn];
        g1n = p.rv_more[rn + 1];
      }
    }
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (;;) {
      add_group<FX, BLK>(p, buf, gr, acc);
      if (g >= g1) break;
      gr = p.gp_pat[g++];
    }
    store_recv<FX>(p, buf, pr, (int64_t)cell, acc, err);
    if (!more) break;
    r = rn;
    pr = pr_n;
    cell = cell_n;
    gr = gr_n;
    g = gn;
    g1 = g1n;
  }
}

// Wide form: 64-bit donor cells and contribution offsets.
template <bool FX>
__global__ void __launch_bounds__(kDonorThreads)
k_donor_copy_wide(const DonorPlan p, int buf, int* err)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= p.n_recv) return;
  const int pr = p.rv_patch[r];
  const int64_t cell = p.rv_cell[r];
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int g = p.rv_grp[r]; g < p.rv_grp[r + 1]; ++g) {
    const int pd = p.gp_donor[g];
    const DonorField<FX> src(p, pd, buf);
    const int64_t ncd = p.nc[pd];
    const int64_t w0 = p.gp_wi[g];
    double inter[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int s = 0; s < p.gp_stride[g]; ++s) {
      const int64_t c = p.idx[w0 + s];
      const double w = p.w[w0 + s];
      #pragma unroll
      for (int v = 0; v < 5; ++v) inter[v] += src.value(p, pd, v, src.load(v * ncd + c)) * w;
    }
    #pragma unroll
    for (int v = 0; v < 5; ++v) acc[v] += inter[v];
  }
  store_recv<FX>(p, buf, pr, cell, acc, err);
}

int blocks_for(int n) { return (n + kDonorThreads - 1) / kDonorThreads; }

// Grid of the pattern form: the CTAs that are resident at once (each
// thread then walks several receiving cells), at most one per 256 cells.
template <bool FX, int BLK>
int pattern_blocks(int n)
{
  // per device, computed once (threads that race here store the same value)
  static std::atomic<int> per_device[64];
  int dev = 0;
  cudaGetDevice(&dev);
  std::atomic<int>& slot = per_device[dev & 63];
  int cap = slot.load(std::memory_order_relaxed);
  if (cap <= 0) {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_donor_copy_pat<FX, BLK>, kDonorThreads, 0);
    cap = sms * (per_sm > 0 ? per_sm : 1);
    if (cap <= 0) cap = 1;
    slot.store(cap, std::memory_order_relaxed);
  }
  const int b = blocks_for(n);
  return b < cap ? b : cap;
}

} // namespace

cudaError_t launch_donor_copy_f64(const DonorPlan& p, int buf, cudaStream_t st)
{
  if (p.n_recv <= 0) return cudaSuccess;
  if (p.patterned) k_donor_copy_pat<false, 4><<<pattern_blocks<false, 4>(p.n_recv), kDonorThreads, 0, st>>>(p, buf, nullptr);
  else k_donor_copy_wide<false><<<blocks_for(p.n_recv), kDonorThreads, 0, st>>>(p, buf, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_donor_copy_fx32(const DonorPlan& p, int buf, int* err, cudaStream_t st)
{
  if (p.n_recv <= 0) return cudaSuccess;
  if (p.patterned) k_donor_copy_pat<true, 4><<<pattern_blocks<true, 4>(p.n_recv), kDonorThreads, 0, st>>>(p, buf, err);
  else k_donor_copy_wide<true><<<blocks_for(p.n_recv), kDonorThreads, 0, st>>>(p, buf, err);
  return cudaGetLastError();
}

} // namespace dn
