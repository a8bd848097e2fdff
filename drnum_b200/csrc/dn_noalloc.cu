// Allocation-free conservation sums of a caller-owned FP64 field.
//
// Some callers cannot allocate device memory: a solver that reserves all of
// its device memory once at start-up and forbids allocation inside the time
// loop, or a host framework whose device memory comes from its own pool.
// For them dn_field_sums_noalloc computes the same five FP64 sums as
// dn_conservation_sums without any cudaMalloc/cudaFree: its per-block partial
// sums live in a file-scope device array of fixed size.
//
// Rules of use:
//  * the array holds partials for at most kNoAllocMaxBlocks blocks of
//    kNoAllocCellsPerBlock cells, so a field is limited to 2^27 cells;
//    larger fields are rejected with DN_ERR_RANGE;
//  * every block overwrites its own slot and every call rewrites the totals,
//    so nothing needs clearing (the array keeps the last call's contents);
//  * all calls share the one array per device: calls whose kernels overlap
//    on the GPU (different streams, or different host threads) race and must
//    be serialised by the caller;
//  * the first call on a device, with that device current, resolves the
//    device address of the array (cudaGetSymbolAddress); make that first
//    call before any stream capture on that device.  The address is kept
//    for the life of the process: after a cudaDeviceReset of that device it
//    is stale, so do not call this function on a device that was reset;
//  * the field is an unpadded FP64 array [5][ncells] (the layout of an FP64
//    context's buffers and of DrNUM's host fields); the int32 fixed-point
//    buffers of an FP32-bulk context, whose rows are padded, cannot be
//    passed.
#include "drnum_b200.h"

#include <cuda_runtime.h>
#include <mutex>

namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxBlocks = 8192;
constexpr long long kNoAllocCellsPerBlock = 16384;
constexpr long long kNoAllocMaxCells = (long long)kNoAllocMaxBlocks * kNoAllocCellsPerBlock;   // 2^27
constexpr int kMaxDevices = 64;

// 8192 blocks x 5 variables partial sums, then the 5 totals (8 slots):
// 327,744 B (about 320 KiB) per device, held until exit
static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxBlocks * 5 + 8];

std::mutex g_setup_mutex;
double* g_partials_ptr[kMaxDevices] = {};

__global__ void __launch_bounds__(kNoAllocThreads)
k_sums_noalloc(const double* __restrict__ f, long long nc, double* __restrict__ partials)
{
  __shared__ double red[5][kNoAllocThreads];
  const long long c0 = (long long)blockIdx.x * kNoAllocCellsPerBlock;
  const long long c1 = c0 + kNoAllocCellsPerBlock < nc ? c0 + kNoAllocCellsPerBlock : nc;
  double acc[5] = {0, 0, 0, 0, 0};
  for (long long c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
    #pragma unroll
    for (int v = 0; v < 5; ++v) acc[v] += f[v * nc + c];
  }
  #pragma unroll
  for (int v = 0; v < 5; ++v) red[v][threadIdx.x] = acc[v];
  __syncthreads();
  for (int s = kNoAllocThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      #pragma unroll
      for (int v = 0; v < 5; ++v) red[v][threadIdx.x] += red[v][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x < 5) partials[blockIdx.x * 5 + threadIdx.x] = red[threadIdx.x][0];
}

// Sums the partials of each variable in block order (one thread per
// variable, fixed order) into the totals slots after the partials.
__global__ void k_sums_noalloc_finish(double* __restrict__ partials, int blocks)
{
  const int v = threadIdx.x;
  if (v >= 5) return;
  double t = 0.0;
  for (int b = 0; b < blocks; ++b) t += partials[b * 5 + v];
  partials[kNoAllocMaxBlocks * 5 + v] = t;
}

// Device address of the scratch array on the current device (resolved once).
int partials_on_current_device(double** out)
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return DN_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_partials_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) return DN_ERR_CUDA;
    g_partials_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_partials_ptr[dev];
  return DN_OK;
}

} // namespace

extern "C" int dn_field_sums_noalloc(const double* field, int64_t ncells, double dV, double out[5], void* stream)
{
  if (!field || !out || ncells < 1) return DN_ERR_ARG;
  if (ncells > kNoAllocMaxCells) return DN_ERR_RANGE;   // more cells than the fixed scratch covers
  double* partials = nullptr;
  int s = partials_on_current_device(&partials);
  if (s != DN_OK) return s;
  const int blocks = (int)((ncells + kNoAllocCellsPerBlock - 1) / kNoAllocCellsPerBlock);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // each launch's own status (cudaGetLastError would also return, and clear,
  // an unrelated error left by an earlier launch of the caller)
  long long nc = (long long)ncells;
  void* sum_args[] = {(void*)&field, (void*)&nc, (void*)&partials};
  if (cudaLaunchKernel((const void*)k_sums_noalloc, dim3(blocks), dim3(kNoAllocThreads), sum_args, 0, st) !=
      cudaSuccess)
    return DN_ERR_CUDA;
  int nb = blocks;
  void* fin_args[] = {(void*)&partials, (void*)&nb};
  if (cudaLaunchKernel((const void*)k_sums_noalloc_finish, dim3(1), dim3(32), fin_args, 0, st) != cudaSuccess)
    return DN_ERR_CUDA;
  double tot[5];
  if (cudaMemcpyAsync(tot, partials + kNoAllocMaxBlocks * 5, sizeof(tot), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return DN_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return DN_ERR_CUDA;
  for (int v = 0; v < 5; ++v) out[v] = tot[v] * dV;
  return DN_OK;
}
