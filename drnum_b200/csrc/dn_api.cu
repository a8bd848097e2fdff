// C ABI of drnum_b200 (declared in include/drnum_b200.h): contexts, patches,
// host <-> device transfers, RK stepping and FP64 reductions.
//
// A context owns, per patch, three physical field buffers and an optional
// active mask.  Logical fields 0/1/2 (current state / step-start state /
// scratch, as in the reference applications) map onto the physical buffers
// through a permutation, so an RK step never copies a field: stage s reads
// the previous stage's output (or the step-start state) and writes the other
// buffer, and the step-start state stays untouched as field 1
// (rungekutta.cpp:27-42 copies field 0 into field 1 instead).
#include "drnum_b200.h"
#include "fv_launch.h"
#include "fv_fx32.cuh"
#include "dn_donor.cuh"
#include "dn_overlap.h"
#include "dn_levelset.h"
#include "dn_lsbc.cuh"
#include "fv_batch.cuh"
#include "fv_schemes.cuh"
#include "dn_gridio.h"
#include <nvtx3/nvToolsExt.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

// NVTX range over a scope: the library's host-side phases appear by name in
// Nsight timelines (no cost unless a tool is attached)
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

struct DnPatch {
  dn_patch_desc d;
  size_t nc = 0;                            // cells, ni*nj*nk
  int kp = 0;                               // row pitch along k in elements: FX32 nk rounded up to a
                                            // multiple of 4 (16-byte rows for TMA boxes), FP64 nk
  size_t ncp = 0;                           // device elements per variable, ni*nj*kp
  int i_chunk = 0;                          // FX32 single-patch launch: planes per CTA (0: default)
  void* buf[3] = {nullptr, nullptr, nullptr};
  uint8_t* active = nullptr;
  double base[5] = {0, 0, 0, 0, 0};
  double quantum[5] = {1, 1, 1, 1, 1};
  bool base_set = false;
  dn::WallBC wall{};                        // device view (table pointers are device memory)
  bool owned = true;                        // false: a shadow of a patch another rank advances
  bool patch_active = true;                 // false: left out of stages, its state carried over
  // compact shadow (dn_patch_add_shadow): another rank's patch of which this
  // context holds only `held` (ascending cell indices, the donor cells its
  // own patches read), stored [var][held position]; ncp = held.size()
  bool compact = false;
  std::vector<uint64_t> held;
};

// Device offset of cell index c = (i*nj + j)*nk + k in the patch's rows of kp elements.
inline uint64_t pad_cell(const DnPatch& p, uint64_t c)
{
  const uint64_t nk = (uint64_t)p.d.nk;
  return (c / nk) * (uint64_t)p.kp + c % nk;
}

// Device offset of cell c: its padded row position, or for a compact shadow
// its position among the held cells (false where the shadow does not hold it).
inline bool dev_cell(const DnPatch& p, uint64_t c, uint64_t* out)
{
  if (!p.compact) {
    *out = pad_cell(p, c);
    return true;
  }
  auto it = std::lower_bound(p.held.begin(), p.held.end(), c);
  if (it == p.held.end() || *it != c) return false;
  *out = (uint64_t)(it - p.held.begin());
  return true;
}

} // namespace

// A captured RK step and what it was captured for.
struct GraphEntry {
  int A = 0, X = 0, Y = 0, n = 0;
  double dt = 0, alpha[16] = {};
  bool skip0 = false;                  // the step-start donor copy left out (its buffer was current)
  cudaGraphExec_t exec = nullptr;
  int64_t launches = 0;
  int fresh_after = -1;                // the context's donor_fresh once the step has run
  bool same(const GraphEntry& o) const
  {
    if (A != o.A || X != o.X || Y != o.Y || n != o.n || skip0 != o.skip0 || std::memcmp(&dt, &o.dt, sizeof dt))
      return false;
    return std::memcmp(alpha, o.alpha, sizeof(double) * n) == 0;
  }
};

struct dn_ctx {
  int device = 0;
  int precision = DN_FP64;
  int num_sms = 148;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  std::vector<DnPatch> patches;
  int fmap[3] = {0, 1, 2};
  std::string err;
  int* d_err = nullptr;
  unsigned long long* d_err_info = nullptr;   // [cell, var, bits(f_n), bits(residual)] of the first failure
  void* staging = nullptr;
  size_t staging_bytes = 0;
  double* d_partials = nullptr;
  size_t partials_cap = 0;
  int64_t launches = 0;
  // donor tables (host) and their device form
  std::vector<dn::DonorTables> tables;
  bool plan_dirty = true;
  std::vector<void*> plan_mem;
  dn::DonorPlan plan{};
  // physical buffer whose receiving cells hold the donor copy of its own
  // donor cells under the current plan (-1: none known), valid while the
  // case generation is donor_fresh_gen; plan_chained: some donor cell is a
  // receiving cell, so a donor copy is not idempotent
  int donor_fresh = -1;
  int64_t donor_fresh_gen = -1;
  bool plan_chained = false;
  // the level-set wall writes a donor or a receiving cell of the plan (its
  // post-operation then makes the buffer's donor copy stale)
  bool ls_touches_donors = true;
  bool donor_wide = false;                    // DN_OPT_DONOR_TABLES = 1
  // level-set layers per patch and their device form
  std::vector<dn::LevelSetLayers> ls;
  std::vector<char> ls_on;
  std::vector<dn::LevelSetGpu> lsg;           // the reference's GPU level-set path, per patch
  std::vector<char> lsg_on;
  bool ls_dirty = true;
  std::vector<void*> ls_mem;
  dn::LsPlan ls_plan{};
  // batched stage launch: per-patch tile shape, patch records and work lists
  bool batched = true;
  std::vector<int> shape;
  bool batch_dirty = true;
  void* d_records = nullptr;
  void* d_maps = nullptr;                     // batched: dn::BatchMaps per tile shape and patch
  // work items per tile form (dn::kFxEdge, kFxInside, kFxFull; FP64: all in
  // [kFxEdge]) and tile shape
  void* d_items[3][dn::kNumShapes] = {};
  int n_items[3][dn::kNumShapes] = {};
  void* d_groups[3][dn::kNumShapes] = {};     // FX32: item ranges of the persistent CTAs
  int n_groups[3][dn::kNumShapes] = {};
  // schedule of a batched stage (autotuned): batch_waves > 0 (FX32 only)
  // deals the work to that many waves of persistent CTAs; 0 launches one
  // CTA per work item, items of at least batch_min_planes planes
  int batch_min_planes = 8;
  int batch_waves = 2;
  cudaStream_t s_aux = nullptr;               // second branch of a batched stage (inside and edge tiles)
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // CUDA graphs of whole RK steps; any change of the case bumps generation
  bool use_graph = false;
  std::vector<GraphEntry> graphs;
  cudaStream_t graph_stream = nullptr;
  int64_t generation = 0;
  int64_t graph_generation = -1;
  // asynchronous host transfers: a copy-in and a copy-out stream with two
  // staging buffers each, and a conversion stream for downloads, ordered
  // against the context's stream by events
  cudaStream_t s_in = nullptr, s_out = nullptr, s_conv = nullptr;
  void* st_in[2] = {nullptr, nullptr};
  size_t st_in_bytes[2] = {0, 0};
  void* st_out[2] = {nullptr, nullptr};
  size_t st_out_bytes[2] = {0, 0};
  cudaEvent_t ev_in_done[2] = {nullptr, nullptr}, ev_in_free[2] = {nullptr, nullptr};
  bool ev_in_free_set[2] = {false, false};
  cudaEvent_t ev_main = nullptr;
  cudaEvent_t ev_out_read[2] = {nullptr, nullptr}, ev_d2h_done[2] = {nullptr, nullptr};
  bool ev_d2h_done_set[2] = {false, false};
  unsigned in_seq = 0, out_seq = 0;
  // exchange hook of a sharded grid: called before every donor copy, with
  // exch_phys the physical buffer about to receive the copy
  dn_exchange_fn exch_fn = nullptr;
  void* exch_user = nullptr;
  int exch_phys = -1;
  // FP64 flux scheme (DN_FLUX_*) or a user stage function replacing it
  int scheme = DN_FLUX_AUSMPLUS;
  dn_stage_fn stage_fn = nullptr;
  void* stage_user = nullptr;
};

#ifndef DN_FX_WAVE_CTAS
#define DN_FX_WAVE_CTAS 2   // CTAs per SM counted in a wave when sizing FX32 plane ranges
#endif

namespace {

constexpr int kSumThreads = 256;
constexpr int kSumBlocks = 1184;   // 8 per SM on 148 SMs; fixed => deterministic order

int fail(dn_ctx* c, int code, const char* fmt, ...)
{
  if (c) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    c->err = buf;
  }
  return code;
}

int cuda_fail(dn_ctx* c, cudaError_t e, const char* what)
{
  return fail(c, DN_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

size_t elem_size(const dn_ctx* c) { return c->precision == DN_FP64 ? sizeof(double) : sizeof(float); }

int set_device(dn_ctx* c)
{
  cudaError_t e = cudaSetDevice(c->device);
  return e == cudaSuccess ? DN_OK : cuda_fail(c, e, "cudaSetDevice");
}

int ensure_staging(dn_ctx* c, size_t bytes)
{
  if (c->staging_bytes >= bytes) return DN_OK;
  if (c->staging) cudaFree(c->staging);
  c->staging = nullptr;
  c->staging_bytes = 0;
  cudaError_t e = cudaMalloc(&c->staging, bytes);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc(staging)");
  c->staging_bytes = bytes;
  return DN_OK;
}

int check_patch(dn_ctx* c, int id)
{
  if (!c) return DN_ERR_ARG;
  if (id < 0 || id >= (int)c->patches.size()) return fail(c, DN_ERR_ARG, "invalid patch id %d", id);
  return DN_OK;
}

// Entry points that read or write a patch's whole state refuse a compact
// shadow: it holds only the donor cells of another rank's patch.
int check_whole(dn_ctx* c, int id)
{
  int s = check_patch(c, id);
  if (s) return s;
  if (c->patches[id].compact)
    return fail(c, DN_ERR_STATE, "patch %d is a compact shadow (another rank's patch; only its donor cells are held)", id);
  return DN_OK;
}

int check_field(dn_ctx* c, int f)
{
  if (f < 0 || f > 2) return fail(c, DN_ERR_ARG, "invalid field %d (0..2)", f);
  return DN_OK;
}

// ---------------------------------------------------------------- kernels

struct QParams {
  double base[5];
  double inv_q[5];
  double q[5];
};

// Host layout [v][i][j][k] (element e) <-> device rows of kp elements:
// e = row*nk + k  ->  row*kp + k (rows never straddle variables).
template <typename Src>
__global__ void k_quantize(const Src* __restrict__ src, int32_t* __restrict__ dst, size_t nc, int nk, int kp,
                           QParams qp, int* err)
{
  const size_t n = 5 * nc;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int v = (int)(e / nc);
    double o = rint(((double)src[e] - qp.base[v]) * qp.inv_q[v]);
    if (!(fabs(o) < (double)dn::kFxLimit)) {
      atomicOr(err, 2);
      o = 0.0;
    }
    size_t d = e;
    if (kp != nk) {                       // padded rows
      const size_t row = e / (size_t)nk;
      d = row * (size_t)kp + (e - row * (size_t)nk);
    }
    dst[d] = (int32_t)o;
  }
}

template <typename Dst>
__global__ void k_dequantize(const int32_t* __restrict__ src, Dst* __restrict__ dst, size_t nc, int nk, int kp,
                             QParams qp)
{
  const size_t n = 5 * nc;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int v = (int)(e / nc);
    size_t d = e;
    if (kp != nk) {                       // padded rows
      const size_t row = e / (size_t)nk;
      d = row * (size_t)kp + (e - row * (size_t)nk);
    }
    dst[e] = (Dst)(qp.base[v] + qp.q[v] * (double)src[d]);
  }
}

template <typename Src, typename Dst>
__global__ void k_convert(const Src* __restrict__ src, Dst* __restrict__ dst, size_t n)
{
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    dst[e] = (Dst)src[e];
}

// Per-block FP64 partial sums of the five variables over one field; each
// block covers a fixed contiguous range and reduces it in a fixed tree order,
// so the result does not depend on scheduling.
template <typename T>
__global__ void __launch_bounds__(kSumThreads)
k_partial_sums(const T* __restrict__ f, size_t nc, double* __restrict__ partials)
{
  __shared__ double red[5][kSumThreads];
  const size_t per = (nc + gridDim.x - 1) / gridDim.x;
  const size_t c0 = blockIdx.x * per;
  const size_t c1 = c0 + per < nc ? c0 + per : nc;
  double acc[5] = {0, 0, 0, 0, 0};
  for (size_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
    #pragma unroll
    for (int v = 0; v < 5; ++v) acc[v] += (double)f[v * nc + c];
  }
  #pragma unroll
  for (int v = 0; v < 5; ++v) red[v][threadIdx.x] = acc[v];
  __syncthreads();
  for (int s = kSumThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      #pragma unroll
      for (int v = 0; v < 5; ++v) red[v][threadIdx.x] += red[v][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x < 5) partials[blockIdx.x * 5 + threadIdx.x] = red[threadIdx.x][0];
}

// Exact per-block sums of int32 offsets (int64 accumulation, fixed order).
__global__ void __launch_bounds__(kSumThreads)
k_partial_sums_i32(const int32_t* __restrict__ f, size_t nc, long long* __restrict__ partials)
{
  __shared__ long long red[5][kSumThreads];
  const size_t per = (nc + gridDim.x - 1) / gridDim.x;
  const size_t c0 = blockIdx.x * per;
  const size_t c1 = c0 + per < nc ? c0 + per : nc;
  long long acc[5] = {0, 0, 0, 0, 0};
  for (size_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
    #pragma unroll
    for (int v = 0; v < 5; ++v) acc[v] += f[v * nc + c];
  }
  #pragma unroll
  for (int v = 0; v < 5; ++v) red[v][threadIdx.x] = acc[v];
  __syncthreads();
  for (int s = kSumThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      #pragma unroll
      for (int v = 0; v < 5; ++v) red[v][threadIdx.x] += red[v][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x < 5) partials[blockIdx.x * 5 + threadIdx.x] = red[threadIdx.x][0];
}

// Flow diagnostics of the reference applications' output step
// (drnumBaseFlowDemo/main.h:255-284, drnumBasicAero/main.h:608-637): per
// cell PerfectGas::conservativeToPrimitive (perfectgas.h:84-93),
// a = sqrt(gamma R T), CFL = max(|u|, |u+a|, |u-a|) dt / dx, and the density
// range.  Written with round-to-nearest intrinsics (no contraction), so each
// cell's values equal the reference's FP64 loop and the extrema are exact.
// Per-block partials: [cfl_max, rho_min, rho_max].
template <typename T>
__global__ void __launch_bounds__(kSumThreads)
k_flow_stats(const T* __restrict__ f, size_t nc, int nk, int kp, QParams q, int quantized, double dt, double dx,
             double* __restrict__ partials)
{
  __shared__ double s_cfl[kSumThreads], s_rmin[kSumThreads], s_rmax[kSumThreads];
  const size_t per = (nc + gridDim.x - 1) / gridDim.x;
  const size_t c0 = blockIdx.x * per;
  const size_t c1 = c0 + per < nc ? c0 + per : nc;
  double cfl = 0.0, rmin = 1000.0, rmax = 0.0;   // the applications' start values
  for (size_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
    if (kp != nk && (int)(c % (size_t)kp) >= nk) continue;   // row padding
    double var[5];
    #pragma unroll
    for (int v = 0; v < 5; ++v) {
      const double x = (double)f[v * nc + c];
      var[v] = quantized ? __dadd_rn(q.base[v], __dmul_rn(q.q[v], x)) : x;
    }
    rmin = fmin(var[0], rmin);
    rmax = fmax(var[0], rmax);
    const double ir = __ddiv_rn(1.0, var[0]);
    const double u = __dmul_rn(var[1], ir), v = __dmul_rn(var[2], ir), w = __dmul_rn(var[3], ir);
    const double ke = __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w));
    const double T = __ddiv_rn(__dsub_rn(__dmul_rn(var[4], ir), __dmul_rn(0.5, ke)), dn::Gas::cv);
    const double a = __dsqrt_rn(__dmul_rn(__dmul_rn(dn::Gas::gamma, dn::Gas::R), T));
    cfl = fmax(cfl, __ddiv_rn(__dmul_rn(fabs(u), dt), dx));
    cfl = fmax(cfl, __ddiv_rn(__dmul_rn(fabs(__dadd_rn(u, a)), dt), dx));
    cfl = fmax(cfl, __ddiv_rn(__dmul_rn(fabs(__dsub_rn(u, a)), dt), dx));
  }
  s_cfl[threadIdx.x] = cfl;
  s_rmin[threadIdx.x] = rmin;
  s_rmax[threadIdx.x] = rmax;
  __syncthreads();
  for (int st = kSumThreads / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) {
      s_cfl[threadIdx.x] = fmax(s_cfl[threadIdx.x], s_cfl[threadIdx.x + st]);
      s_rmin[threadIdx.x] = fmin(s_rmin[threadIdx.x], s_rmin[threadIdx.x + st]);
      s_rmax[threadIdx.x] = fmax(s_rmax[threadIdx.x], s_rmax[threadIdx.x + st]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partials[blockIdx.x * 3] = s_cfl[0];
    partials[blockIdx.x * 3 + 1] = s_rmin[0];
    partials[blockIdx.x * 3 + 2] = s_rmax[0];
  }
}

// max and sum of squared differences of two variables (Patch::computeVariableDifference)
template <typename T>
__global__ void __launch_bounds__(kSumThreads)
k_diff(const T* __restrict__ a, const T* __restrict__ b, size_t nc, QParams qa, int va, QParams qb, int vb,
       int quantized, double* __restrict__ partials)
{
  __shared__ double smax[kSumThreads];
  __shared__ double ssum[kSumThreads];
  const size_t per = (nc + gridDim.x - 1) / gridDim.x;
  const size_t c0 = blockIdx.x * per;
  const size_t c1 = c0 + per < nc ? c0 + per : nc;
  double mx = 0, sm = 0;
  for (size_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
    double x = (double)a[c], y = (double)b[c];
    if (quantized) {
      x = qa.base[va] + qa.q[va] * x;
      y = qb.base[vb] + qb.q[vb] * y;
    }
    const double d = (y - x) * (y - x);
    mx = d > mx ? d : mx;
    sm += d;
  }
  smax[threadIdx.x] = mx;
  ssum[threadIdx.x] = sm;
  __syncthreads();
  for (int s = kSumThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      smax[threadIdx.x] = smax[threadIdx.x] > smax[threadIdx.x + s] ? smax[threadIdx.x] : smax[threadIdx.x + s];
      ssum[threadIdx.x] += ssum[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partials[blockIdx.x * 2] = smax[0];
    partials[blockIdx.x * 2 + 1] = ssum[0];
  }
}

int grid_for(size_t n)
{
  size_t g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return (int)g;
}

QParams qparams(const DnPatch& p)
{
  QParams q;
  for (int v = 0; v < 5; ++v) {
    q.base[v] = p.base[v];
    q.q[v] = p.quantum[v];
    q.inv_q[v] = 1.0 / p.quantum[v];
  }
  return q;
}

int ensure_partials(dn_ctx* c, size_t n)
{
  if (c->partials_cap >= n) return DN_OK;
  if (c->d_partials) cudaFree(c->d_partials);
  c->d_partials = nullptr;
  c->partials_cap = 0;
  cudaError_t e = cudaMalloc(&c->d_partials, n * sizeof(double));
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc(partials)");
  c->partials_cap = n;
  return DN_OK;
}

int read_device_error(dn_ctx* c)
{
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "device error word");
  if (h != 0) {
    unsigned long long info[4] = {0, 0, 0, 0};
    cudaMemcpyAsync(info, c->d_err_info, sizeof(info), cudaMemcpyDeviceToHost, c->stream);
    cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
    cudaMemsetAsync(c->d_err_info, 0xff, 4 * sizeof(unsigned long long), c->stream);
    cudaStreamSynchronize(c->stream);
    double un, r;
    std::memcpy(&un, &info[2], sizeof(double));
    std::memcpy(&r, &info[3], sizeof(double));
    if (h & 1)
      return fail(c, DN_ERR_RANGE, "fixed-point offset left its range (|o| >= 2^30) during a stage "
                  "(first at cell %llu var %llu: f_n offset %.9g, residual %.9g quanta)", info[0], info[1], un, r);
    if (h & 2) return fail(c, DN_ERR_RANGE, "uploaded state outside the FP32 offset range of the patch base/quantum");
    if (h & 4) return fail(c, DN_ERR_RANGE, "an interpolated receiving cell left the offset range of its patch");
    if (h & 8) return fail(c, DN_ERR_RANGE, "a level-set wall cell left the offset range of its patch");
    if (h & 16) return fail(c, DN_ERR_RANGE, "a face flux of a stage was not finite or reached 2^30 offset quanta "
                            "(the state or its fluxes left the fixed-point range of the patch)");
    if (h & 32) return fail(c, DN_ERR_DEVICE, "a TMA transfer of a stage did not complete within its bounded wait");
    if (h & dn::kErrLsAverage)
      return fail(c, DN_ERR_DEVICE, "an inside-cell average of the GPU level-set path was not finite "
                  "(the reference's kernel traps there)");
    return fail(c, DN_ERR_DEVICE, "device error word 0x%x", h);
  }
  return DN_OK;
}

// Derives base and quantum from a host state: base = mean per variable;
// quantum = 2^ceil(log2(4 M_v / 2^30)) with M_v the magnitude scale of the
// variable (max |rho|, max rho*(|u|+a) for all three momenta, max |rho E|):
// offsets up to 4 M_v stay inside the int32 range used (|o| < 2^30) and the
// resolution, about 4e-9 M_v, is far below the FP32 spacing of U.
template <typename T>
void derive_base(DnPatch& p, const T* h)
{
  const size_t nc = p.nc;
  double sum[5] = {0, 0, 0, 0, 0};
  double mr = 0, mm = 0, me = 0;
  for (size_t c = 0; c < nc; ++c) {
    const double r = h[c], ru = h[nc + c], rv = h[2 * nc + c], rw = h[3 * nc + c], rE = h[4 * nc + c];
    sum[0] += r; sum[1] += ru; sum[2] += rv; sum[3] += rw; sum[4] += rE;
    const double ar = std::fabs(r);
    mr = ar > mr ? ar : mr;
    me = std::fabs(rE) > me ? std::fabs(rE) : me;
    if (r > 0) {
      const double u = ru / r, v = rv / r, w = rw / r;
      const double q2 = u * u + v * v + w * w;
      const double T_ = (rE / r - 0.5 * q2) / 717.5;
      const double a = T_ > 0 ? std::sqrt(1.4 * 287.2 * T_) : 0.0;
      const double m = r * (std::sqrt(q2) + a);
      mm = m > mm ? m : mm;
    }
  }
  const double M[5] = {mr, mm, mm, mm, me};
  for (int v = 0; v < 5; ++v) {
    p.base[v] = sum[v] / (double)nc;
    double Mv = M[v] > 0 ? M[v] : 1.0;
    p.quantum[v] = std::ldexp(1.0, (int)std::ceil(std::log2(4.0 * Mv / (double)dn::kFxLimit)));
  }
  p.base_set = true;
}

// ------------------------------------------------------------ donor plan

void free_plan(dn_ctx* c)
{
  for (void* m : c->plan_mem) cudaFree(m);
  c->plan_mem.clear();
  c->plan = dn::DonorPlan{};
}

template <typename T>
int plan_upload(dn_ctx* c, const std::vector<T>& h, const T** out)
{
  *out = nullptr;
  if (h.empty()) return DN_OK;
  void* d = nullptr;
  cudaError_t e = cudaMalloc(&d, h.size() * sizeof(T));
  if (e != cudaSuccess) return fail(c, DN_ERR_NOMEM, "cudaMalloc(donor plan)");
  c->plan_mem.push_back(d);
  e = cudaMemcpyAsync(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "donor plan upload");
  *out = static_cast<const T*>(d);
  return DN_OK;
}

bool has_donors(const dn_ctx* c)
{
  for (const auto& t : c->tables) if (!t.rec_unique.empty()) return true;
  return false;
}

// Regroups the per-patch tables by receiving cell (groups in donor order)
// and uploads them with the per-patch buffer table.
bool levelset_touches_donors(const dn_ctx* c);

int build_plan(dn_ctx* c)
{
  free_plan(c);
  c->donor_fresh = -1;
  const size_t np = c->patches.size();
  std::vector<int32_t> rv_patch, rv_grp(1, 0), gp_donor, gp_stride;
  std::vector<int64_t> rv_cell, gp_wi, idx, nc(np);
  std::vector<double> w, base(np * 5), quantum(np * 5);
  std::vector<void*> bufs(np * 3);
  for (size_t r = 0; r < np; ++r) {
    const DnPatch& P = c->patches[r];
    nc[r] = (int64_t)P.ncp;
    for (int b = 0; b < 3; ++b) bufs[r * 3 + b] = P.buf[b];
    for (int v = 0; v < 5; ++v) { base[r * 5 + v] = P.base[v]; quantum[r * 5 + v] = P.quantum[v]; }
    if (r >= c->tables.size() || !P.owned) continue;
    const dn::DonorTables& T = c->tables[r];
    const size_t nu = T.rec_unique.size();
    if (nu == 0) continue;
    // groups of this patch in (donor, receiver) order, then listed per receiving cell
    std::vector<int32_t> ld, ls;
    std::vector<int64_t> lw;
    std::vector<std::vector<size_t>> groups(nu);
    const int64_t wi_base = (int64_t)idx.size();
    size_t rc_off = 0;
    int64_t wi_off = 0;
    for (size_t q = 0; q < T.donor_patch.size(); ++q) {
      for (int64_t ll = 0; ll < T.num_receivers[q]; ++ll) {
        const uint64_t cell = T.rec_concat[rc_off + (size_t)ll];
        const size_t u = (size_t)(std::lower_bound(T.rec_unique.begin(), T.rec_unique.end(), cell) - T.rec_unique.begin());
        groups[u].push_back(ld.size());
        ld.push_back(T.donor_patch[q]);
        ls.push_back(T.stride[q]);
        lw.push_back(wi_base + wi_off + ll * T.stride[q]);
      }
      rc_off += (size_t)T.num_receivers[q];
      wi_off += T.num_receivers[q] * T.stride[q];
    }
    // donor cells at their device offsets (rows of kp elements, or the held
    // position in a compact shadow)
    {
      size_t o = 0;
      for (size_t q = 0; q < T.donor_patch.size(); ++q) {
        const DnPatch& D = c->patches[(size_t)T.donor_patch[q]];
        const size_t m = (size_t)(T.num_receivers[q] * T.stride[q]);
        for (size_t e = 0; e < m; ++e) {
          uint64_t dc;
          if (!dev_cell(D, T.donor_idx[o + e], &dc)) {
            free_plan(c);
            return fail(c, DN_ERR_STATE, "donor cell %llu of patch %d is not held by its compact shadow "
                        "(dn_shadow_alloc with the exchange that delivers it)",
                        (unsigned long long)T.donor_idx[o + e], T.donor_patch[q]);
          }
          idx.push_back((int64_t)dc);
        }
        o += m;
      }
    }
    w.insert(w.end(), T.weight.begin(), T.weight.end());
    for (size_t u = 0; u < nu; ++u) {
      rv_patch.push_back((int32_t)r);
      rv_cell.push_back((int64_t)pad_cell(P, T.rec_unique[u]));
      for (size_t g : groups[u]) {
        gp_donor.push_back(ld[g]);
        gp_stride.push_back(ls[g]);
        gp_wi.push_back(lw[g]);
      }
      rv_grp.push_back((int32_t)gp_donor.size());
    }
  }
  if (rv_patch.size() >= (size_t)INT32_MAX || gp_donor.size() >= (size_t)INT32_MAX)
    return fail(c, DN_ERR_RANGE, "too many receiving cells or donor groups for one donor plan");
  // a donor cell that is also a receiving cell (of the plan) would make a
  // repeated donor copy read what the last one wrote
  {
    std::vector<std::vector<bool>> recv(np);
    for (size_t r = 0; r < np && r < c->tables.size(); ++r) {
      const DnPatch& P = c->patches[r];
      if (!P.owned || c->tables[r].rec_unique.empty()) continue;
      recv[r].assign((size_t)P.d.ni * P.d.nj * P.d.nk, false);
      for (uint64_t u : c->tables[r].rec_unique) if (u < recv[r].size()) recv[r][u] = true;
    }
    bool chained = false;
    for (size_t r = 0; r < np && r < c->tables.size() && !chained; ++r) {
      if (!c->patches[r].owned) continue;
      const dn::DonorTables& T = c->tables[r];
      size_t o = 0;
      for (size_t q = 0; q < T.donor_patch.size() && !chained; ++q) {
        const std::vector<bool>& R = recv[(size_t)T.donor_patch[q]];
        const size_t m = (size_t)(T.num_receivers[q] * T.stride[q]);
        if (!R.empty()) {
          for (size_t e = 0; e < m; ++e) {
            const uint64_t d = T.donor_idx[o + e];
            if (d < R.size() && R[d]) { chained = true; break; }
          }
        }
        o += m;
      }
    }
    c->plan_chained = chained;
  }
  c->ls_touches_donors = levelset_touches_donors(c);
  // pattern form: every group as (first donor cell, first pattern entry,
  // entries, donor patch); the pattern entries (offsets from the first
  // donor cell, weights) listed once for all groups that share them.  A
  // cell's first group sits at the cell's index, further groups after all
  // first ones.  FP32-bulk plans leave zero weights out: a donor value is
  // always finite there, and adding +-0 to a sum that starts at +0 never
  // changes it.
  auto fits32 = [](const std::vector<int64_t>& v) {
    for (int64_t x : v) if (x < 0 || x > (int64_t)UINT32_MAX) return false;
    return true;
  };
  const size_t n_recv = rv_patch.size();
  bool patterned = !c->donor_wide && fits32(rv_cell) && fits32(idx);
  std::vector<uint4> gp_pat;
  std::vector<int32_t> rv_more, pt_off;
  std::vector<double> pt_w;
  if (patterned) {
    const bool drop_zero = c->precision != DN_FP64;
    std::unordered_map<std::string, int32_t> starts;
    std::string key, last_key;
    int32_t last_start = 0;
    bool any_more = false;
    for (size_t r = 0; r < n_recv; ++r) any_more = any_more || rv_grp[r + 1] - rv_grp[r] > 1;
    gp_pat.resize(n_recv, make_uint4(0u, 0u, 0u, 0u));
    if (any_more) rv_more.assign(n_recv + 1, 0);
    auto pattern_of = [&](size_t g, uint4* out) {
      const int64_t w0 = gp_wi[g], n = gp_stride[g];
      const int64_t c0 = n > 0 ? idx[(size_t)w0] : 0;
      key.clear();
      for (int64_t q = 0; q < n; ++q) {
        const double ws = w[(size_t)(w0 + q)];
        if (drop_zero && ws == 0.0) continue;
        const int64_t d = idx[(size_t)(w0 + q)] - c0;
        if (d < INT32_MIN || d > INT32_MAX) return false;
        const int32_t d32 = (int32_t)d;
        key.append(reinterpret_cast<const char*>(&d32), sizeof(d32));
        key.append(reinterpret_cast<const char*>(&ws), sizeof(ws));
      }
      const size_t entries = key.size() / (sizeof(int32_t) + sizeof(double));
      int32_t start = last_start;
      if (key != last_key) {
        auto it = starts.find(key);
        if (it != starts.end()) {
          start = it->second;
        } else {
          if (pt_off.size() + entries >= (size_t)INT32_MAX) return false;
          start = (int32_t)pt_off.size();
          starts.emplace(key, start);
          for (size_t o = 0; o < key.size(); o += sizeof(int32_t) + sizeof(double)) {
            int32_t d32;
            double ws;
            std::memcpy(&d32, key.data() + o, sizeof(d32));
            std::memcpy(&ws, key.data() + o + sizeof(d32), sizeof(ws));
            pt_off.push_back(d32);
            pt_w.push_back(ws);
          }
        }
        last_key = key;
        last_start = start;
      }
      *out = make_uint4((unsigned)c0, (unsigned)start, (unsigned)entries, (unsigned)gp_donor[g]);
      return true;
    };
    for (size_t r = 0; r < n_recv && patterned; ++r) {
      const size_t g0 = (size_t)rv_grp[r], g1 = (size_t)rv_grp[r + 1];
      if (g1 == g0) gp_pat[r] = make_uint4(0u, 0u, 0u, (unsigned)rv_patch[r]);   // no donor: sums to zero
      else patterned = pattern_of(g0, &gp_pat[r]);
      if (any_more) rv_more[r] = (int32_t)gp_pat.size();
      for (size_t g = g0 + 1; g < g1 && patterned; ++g) {
        uint4 e;
        patterned = pattern_of(g, &e);
        gp_pat.push_back(e);
      }
    }
    if (any_more) rv_more[n_recv] = (int32_t)gp_pat.size();
  }
  int s;
  dn::DonorPlan& P = c->plan;
  P.n_recv = (int32_t)rv_patch.size();
  P.patterned = patterned ? 1 : 0;
  if ((s = plan_upload(c, rv_patch, &P.rv_patch)) || (s = plan_upload(c, nc, &P.nc)) ||
      (s = plan_upload(c, base, &P.base)) || (s = plan_upload(c, quantum, &P.quantum))) {
    free_plan(c);
    return s;
  }
  if (patterned) {
    const std::vector<uint32_t> rc(rv_cell.begin(), rv_cell.end());
    if ((s = plan_upload(c, rc, &P.rv_cell32)) || (s = plan_upload(c, gp_pat, &P.gp_pat)) ||
        (s = plan_upload(c, rv_more, &P.rv_more)) || (s = plan_upload(c, pt_off, &P.pt_off)) ||
        (s = plan_upload(c, pt_w, &P.pt_w))) {
      free_plan(c);
      return s;
    }
  } else if ((s = plan_upload(c, rv_grp, &P.rv_grp)) || (s = plan_upload(c, rv_cell, &P.rv_cell)) ||
             (s = plan_upload(c, gp_donor, &P.gp_donor)) || (s = plan_upload(c, gp_stride, &P.gp_stride)) ||
             (s = plan_upload(c, gp_wi, &P.gp_wi)) || (s = plan_upload(c, idx, &P.idx)) ||
             (s = plan_upload(c, w, &P.w))) {
    free_plan(c);
    return s;
  }
  if ((s = plan_upload(c, bufs, &P.bufs))) { free_plan(c); return s; }
  c->plan_dirty = false;
  return DN_OK;
}

// ------------------------------------------------------- level-set plan

void free_ls_plan(dn_ctx* c)
{
  for (void* m : c->ls_mem) cudaFree(m);
  c->ls_mem.clear();
  c->ls_plan = dn::LsPlan{};
}

template <typename T>
int ls_upload(dn_ctx* c, const std::vector<T>& h, const T** out)
{
  *out = nullptr;
  if (h.empty()) return DN_OK;
  void* d = nullptr;
  cudaError_t e = cudaMalloc(&d, h.size() * sizeof(T));
  if (e != cudaSuccess) return fail(c, DN_ERR_NOMEM, "cudaMalloc(level-set plan)");
  c->ls_mem.push_back(d);
  e = cudaMemcpyAsync(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "level-set plan upload");
  *out = static_cast<const T*>(d);
  return DN_OK;
}

// Flattens the inner layer cells of all patches with a level set (patch,
// layer, cell order, as LevelSetObjectBC::transferCellLayerData,
// levelsetobjectbc.cpp:38-134) and uploads them.
// Whether a cell the level-set wall writes (inner layer cells, and the GPU
// path's reset and inside cells) is a donor or a receiving cell of an owned
// patch's donor tables (host cell indices).
bool levelset_touches_donors(const dn_ctx* c)
{
  const size_t np = c->patches.size();
  std::vector<std::vector<bool>> used(np);
  auto mark = [&](size_t p, uint64_t cell) {
    const DnPatch& P = c->patches[p];
    if (used[p].empty()) used[p].assign((size_t)P.d.ni * P.d.nj * P.d.nk, false);
    if (cell < used[p].size()) used[p][cell] = true;
  };
  for (size_t r = 0; r < np && r < c->tables.size(); ++r) {
    if (!c->patches[r].owned) continue;
    const dn::DonorTables& T = c->tables[r];
    for (uint64_t u : T.rec_unique) mark(r, u);
    size_t o = 0;
    for (size_t q = 0; q < T.donor_patch.size(); ++q) {
      const size_t m = (size_t)(T.num_receivers[q] * T.stride[q]);
      for (size_t e = 0; e < m; ++e) mark((size_t)T.donor_patch[q], T.donor_idx[o + e]);
      o += m;
    }
  }
  auto hit = [&](size_t p, uint64_t cell) { return !used[p].empty() && cell < used[p].size() && used[p][cell]; };
  for (size_t r = 0; r < np; ++r) {
    if (!c->patches[r].owned) continue;
    if (r < c->ls.size() && c->ls_on[r]) {
      for (const auto& layer : c->ls[r].inner)
        for (const dn::LayerCell& lc : layer) if (hit(r, lc.cell)) return true;
    }
    if (r < c->lsg.size() && c->lsg_on[r]) {
      for (uint64_t cb : c->lsg[r].below) if (hit(r, cb)) return true;
      for (const dn::LsInsideCell& ic : c->lsg[r].inside) if (hit(r, ic.cell)) return true;
    }
  }
  return false;
}

int build_ls_plan(dn_ctx* c)
{
  free_ls_plan(c);
  c->ls_touches_donors = levelset_touches_donors(c);
  const size_t np = c->patches.size();
  std::vector<int32_t> patch;
  std::vector<int64_t> cell, donor, nc(np);
  std::vector<double> grad, w, base(np * 5), quantum(np * 5);
  std::vector<void*> bufs(np * 3);
  for (size_t r = 0; r < np; ++r) {
    const DnPatch& P = c->patches[r];
    nc[r] = (int64_t)P.ncp;
    for (int b = 0; b < 3; ++b) bufs[r * 3 + b] = P.buf[b];
    for (int v = 0; v < 5; ++v) { base[r * 5 + v] = P.base[v]; quantum[r * 5 + v] = P.quantum[v]; }
    if (r >= c->ls.size() || !c->ls_on[r] || !P.owned) continue;
    for (const auto& layer : c->ls[r].inner) {
      for (const dn::LayerCell& lc : layer) {
        patch.push_back((int32_t)r);
        cell.push_back((int64_t)pad_cell(P, lc.cell));
        for (int a = 0; a < 3; ++a) grad.push_back(lc.grad[a]);
        for (int q = 0; q < 8; ++q) { donor.push_back((int64_t)pad_cell(P, lc.donor[q])); w.push_back(lc.weight[q]); }
      }
    }
  }
  // the GPU level-set path: deactivated cells that no donor copy writes, and
  // the inside cells with their neighbours
  std::vector<int32_t> rpatch, apatch;
  std::vector<int64_t> rcell, acell, astart(1, 0), anbr;
  std::vector<double> aw;
  for (size_t r = 0; r < np && r < c->lsg.size(); ++r) {
    const DnPatch& P = c->patches[r];
    if (!c->lsg_on[r] || !P.owned) continue;
    const std::vector<uint64_t>* rec = r < c->tables.size() ? &c->tables[r].rec_unique : nullptr;
    for (uint64_t cb : c->lsg[r].below) {
      if (rec && std::binary_search(rec->begin(), rec->end(), cb)) continue;
      rpatch.push_back((int32_t)r);
      rcell.push_back((int64_t)pad_cell(P, cb));
    }
    for (const dn::LsInsideCell& ic : c->lsg[r].inside) {
      apatch.push_back((int32_t)r);
      acell.push_back((int64_t)pad_cell(P, ic.cell));
      for (size_t m = 0; m < ic.nbr.size(); ++m) {
        anbr.push_back((int64_t)pad_cell(P, ic.nbr[m]));
        aw.push_back(ic.w[m]);
      }
      astart.push_back((int64_t)anbr.size());
    }
  }
  if (patch.size() >= (size_t)INT32_MAX || rpatch.size() >= (size_t)INT32_MAX || apatch.size() >= (size_t)INT32_MAX)
    return fail(c, DN_ERR_RANGE, "too many level-set cells");
  dn::LsPlan& L = c->ls_plan;
  L.n = (int32_t)patch.size();
  L.n_reset = (int32_t)rpatch.size();
  L.n_avg = (int32_t)apatch.size();
  int s;
  if ((s = ls_upload(c, patch, &L.patch)) || (s = ls_upload(c, cell, &L.cell)) || (s = ls_upload(c, grad, &L.grad)) ||
      (s = ls_upload(c, donor, &L.donor)) || (s = ls_upload(c, w, &L.w)) || (s = ls_upload(c, nc, &L.nc)) ||
      (s = ls_upload(c, base, &L.base)) || (s = ls_upload(c, quantum, &L.quantum)) ||
      (s = ls_upload(c, bufs, &L.bufs)) || (s = ls_upload(c, rpatch, &L.reset_patch)) ||
      (s = ls_upload(c, rcell, &L.reset_cell)) || (s = ls_upload(c, apatch, &L.avg_patch)) ||
      (s = ls_upload(c, acell, &L.avg_cell)) || (L.n_avg > 0 && (s = ls_upload(c, astart, &L.avg_start))) ||
      (s = ls_upload(c, anbr, &L.avg_nbr)) || (s = ls_upload(c, aw, &L.avg_w))) {
    free_ls_plan(c);
    return s;
  }
  for (int q = 0; q < 2; ++q) {
    const size_t n = q == 0 ? (size_t)L.n : (size_t)L.n_avg;
    if (n == 0) continue;
    void* d = nullptr;
    cudaError_t e = cudaMalloc(&d, n * 5 * sizeof(double));
    if (e != cudaSuccess) { free_ls_plan(c); return fail(c, DN_ERR_NOMEM, "cudaMalloc(level-set scratch)"); }
    c->ls_mem.push_back(d);
    (q == 0 ? L.acc : L.avg_acc) = static_cast<double*>(d);
  }
  c->ls_dirty = false;
  return DN_OK;
}

void donor_stale(dn_ctx* c, int b);

// Level-set wall conditions on physical buffer `b` of every patch (step_b:
// the step-start state, which the GPU level-set path resets its
// deactivated cells to).
int levelset_bc(dn_ctx* c, int b, int step_b)
{
  NvtxRange nvtx("dn level-set wall");
  bool any = false, any_gpu = false;
  for (char on : c->ls_on) any = any || on;
  for (char on : c->lsg_on) any_gpu = any_gpu || on;
  if (!any && !any_gpu) return DN_OK;
  int s;
  if (c->ls_dirty && (s = build_ls_plan(c))) return s;
  if (c->ls_touches_donors) donor_stale(c, b);
  const dn::LsPlan& L = c->ls_plan;
  cudaError_t e = cudaSuccess;
  if (any && L.n > 0) {
    e = dn::launch_levelset_bc(L, b, c->precision != DN_FP64, c->d_err, c->stream);
    c->launches += 2;
  }
  if (e == cudaSuccess && any_gpu) {
    e = dn::launch_levelset_gpu(L, b, step_b, c->precision != DN_FP64, c->d_err, c->stream);
    c->launches += (L.n_reset > 0 ? 1 : 0) + (L.n_avg > 0 ? 2 : 0);
  }
  if (e != cudaSuccess) return cuda_fail(c, e, "level-set boundary launch");
  return DN_OK;
}

// Physical buffer b is written by something other than a donor copy (b < 0:
// any buffer): its receiving cells may no longer match its donor cells.
void donor_stale(dn_ctx* c, int b)
{
  if (b < 0 || c->donor_fresh == b) c->donor_fresh = -1;
}

// Buffer b's receiving cells hold the donor copy of its current donor cells
// under the current plan, so a donor copy into b would rewrite the same
// values.  Never for a sharded grid (other ranks change donor cells) or a
// plan whose donor cells include receiving cells.
bool donor_current(const dn_ctx* c, int b)
{
  return b >= 0 && c->donor_fresh == b && c->donor_fresh_gen == c->generation && !c->plan_dirty &&
         !c->plan_chained && !c->exch_fn;
}

// Donor copy into physical buffer `b` of every patch, preceded by the
// exchange hook where one is set (every rank of a sharded grid exchanges
// before every donor copy, whether or not its own patches receive).
int donor_copy(dn_ctx* c, int b)
{
  NvtxRange nvtx("dn donor copy");
  int s;
  if (c->exch_fn) {
    c->exch_phys = b;
    const int rc = c->exch_fn(c->exch_user);
    c->exch_phys = -1;
    if (rc) return fail(c, rc < 0 ? rc : DN_ERR_ARG, "exchange hook returned %d", rc);
  }
  if (!has_donors(c)) return DN_OK;
  if (c->plan_dirty && (s = build_plan(c))) return s;
  cudaError_t e = c->precision == DN_FP64 ? dn::launch_donor_copy_f64(c->plan, b, c->stream)
                                          : dn::launch_donor_copy_fx32(c->plan, b, c->d_err, c->stream);
  c->launches++;
  if (e != cudaSuccess) return cuda_fail(c, e, "donor copy launch");
  c->donor_fresh = c->exch_fn ? -1 : b;
  c->donor_fresh_gen = c->generation;
  return DN_OK;
}

// ------------------------------------------------------------ RK step

bool any_levelset(const dn_ctx* c)
{
  for (char on : c->ls_on) if (on) return true;
  for (char on : c->lsg_on) if (on) return true;
  return false;
}

int stage_all(dn_ctx* c, int in_b, int un_b, int out_b, double factor);

// Exchange of donor cells between ranks: gather into / scatter from a
// [var][item] buffer of the storage type (patch buffer table and cell
// counts are the donor plan's).
template <typename T>
__global__ void k_exchange_pack(void* const* bufs, const int64_t* nc, int phys, const int32_t* patch,
                                const uint64_t* cell, int64_t n, T* out)
{
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int p = patch[t];
    const T* f = static_cast<const T*>(bufs[(size_t)p * 3 + phys]);
    const int64_t m = nc[p], c = (int64_t)cell[t];
    #pragma unroll
    for (int v = 0; v < 5; ++v) out[v * n + t] = f[v * m + c];
  }
}

template <typename T>
__global__ void k_exchange_unpack(void* const* bufs, const int64_t* nc, int phys, const int32_t* patch,
                                  const uint64_t* cell, int64_t n, const T* in)
{
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int p = patch[t];
    T* f = static_cast<T*>(bufs[(size_t)p * 3 + phys]);
    const int64_t m = nc[p], c = (int64_t)cell[t];
    #pragma unroll
    for (int v = 0; v < 5; ++v) f[v * m + c] = in[v * n + t];
  }
}

// Launches of one RK step (RungeKutta::operator(), rungekutta.cpp:27-42)
// from step-start buffer A through the other two buffers X, Y.
int rk_step_enqueue(dn_ctx* c, double dt, const double* alpha, int n_alpha, int A, int X, int Y)
{
  int in = A;
  int st;
  // copyDonorData(0) before the step-start copy (rungekutta.cpp:30); the
  // copy before each later stage (:34-36) repeats the previous stage's, so
  // it is skipped unless a post-operation (the level-set wall) may have
  // changed donor cells since
  // (a sharded grid never skips it: a level-set wall on another rank may
  // have changed donor cells this rank reads)
  // (the step-start copy is also left out when A's receiving cells already
  // hold it: the last step ended with a donor copy into A and nothing has
  // written A since; a repeated copy would write the same bits)
  const bool post_op = any_levelset(c) || c->exch_fn != nullptr;
  if (!donor_current(c, A) && (st = donor_copy(c, A))) return st;
  for (int s = 0; s < n_alpha; ++s) {
    const int out = (s & 1) ? Y : X;
    const double factor = alpha[s] * dt;   // (*i)*dt, rungekutta.cpp:37
    if (s > 0 && post_op && !donor_current(c, in) && (st = donor_copy(c, in))) return st;
    if ((st = stage_all(c, in, A, out, factor))) return st;
    if ((st = donor_copy(c, out))) return st;   // copyDonorData(0) after the stage (:38)
    if ((st = levelset_bc(c, out, A))) return st;   // runPostOperations() (:39)
    in = out;
  }
  return DN_OK;
}

void free_graphs(dn_ctx* c)
{
  for (auto& gc : c->graphs) if (gc.exec) cudaGraphExecDestroy(gc.exec);
  c->graphs.clear();
}

int build_batch(dn_ctx* c);
int build_plan(dn_ctx* c);
int build_ls_plan(dn_ctx* c);

// The step as a CUDA graph: captured once per (buffer rotation, dt, alphas)
// and replayed; everything that allocates (tables, work lists) is built
// before the capture.
int rk_step_graph(dn_ctx* c, double dt, const double* alpha, int n_alpha, int A, int X, int Y)
{
  int st;
  if (c->batched && c->batch_dirty && (st = build_batch(c))) return st;
  if (has_donors(c) && c->plan_dirty && (st = build_plan(c))) return st;
  if (any_levelset(c) && c->ls_dirty && (st = build_ls_plan(c))) return st;
  if (c->graph_stream != c->stream || c->graph_generation != c->generation) {
    free_graphs(c);
    c->graph_stream = c->stream;
    c->graph_generation = c->generation;
  }
  GraphEntry key;
  key.A = A; key.X = X; key.Y = Y; key.dt = dt; key.n = n_alpha;
  key.skip0 = donor_current(c, A);
  for (int q = 0; q < n_alpha; ++q) key.alpha[q] = alpha[q];
  GraphEntry* hit = nullptr;
  for (auto& gc : c->graphs) if (gc.same(key)) hit = &gc;
  if (!hit) {
    if (c->graphs.size() >= 6) free_graphs(c);
    cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return cuda_fail(c, e, "begin graph capture");
    const int64_t l0 = c->launches;
    st = rk_step_enqueue(c, dt, alpha, n_alpha, A, X, Y);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(c->stream, &g);
    if (st) { if (g) cudaGraphDestroy(g); return st; }
    if (e != cudaSuccess) return cuda_fail(c, e, "end graph capture");
    key.launches = c->launches - l0;
    key.fresh_after = c->donor_fresh;
    c->launches = l0;
    e = cudaGraphInstantiate(&key.exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(c, e, "graph instantiate");
    c->graphs.push_back(key);
    hit = &c->graphs.back();
  }
  cudaError_t e = cudaGraphLaunch(hit->exec, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "graph launch");
  c->launches += hit->launches;
  c->donor_fresh = hit->fresh_after;
  c->donor_fresh_gen = c->generation;
  return DN_OK;
}

// ------------------------------------------------------------ batched stage

void free_batch(dn_ctx* c)
{
  if (c->d_records) cudaFree(c->d_records);
  c->d_records = nullptr;
  if (c->d_maps) cudaFree(c->d_maps);
  c->d_maps = nullptr;
  for (int f = 0; f < 3; ++f) {
    for (int q = 0; q < dn::kNumShapes; ++q) {
      if (c->d_items[f][q]) cudaFree(c->d_items[f][q]);
      c->d_items[f][q] = nullptr;
      c->n_items[f][q] = 0;
      if (c->d_groups[f][q]) cudaFree(c->d_groups[f][q]);
      c->d_groups[f][q] = nullptr;
      c->n_groups[f][q] = 0;
    }
  }
}

// Default tile shape of a patch: the one that wastes fewer k lanes (k is
// the coalesced axis; ties go to the wider tile), 16 rows where the patch
// has that many.
int default_shape(const DnPatch& p)
{
  const int nk = p.d.nk;
  const double e32 = (double)nk / (double)(((nk + 31) / 32) * 32);
  const double e16 = (double)nk / (double)(((nk + 15) / 16) * 16);
  if (e16 > e32 + 1e-12) return 1;
  return p.d.nj >= 16 ? 2 : 0;
}

// Work items of persistent CTAs: the column runs (patch, column tile, all
// planes) of one launch are cut along i and dealt in order to at most
// `slots` CTAs (one wave) so that every CTA gets about the same number of
// planes, each item charged kProlog planes for its prologue (three planes
// staged and dequantised before the first update).  A CTA's items follow
// one another along the runs; no piece is shorter than kMinPiece planes
// where its run is longer.  The share per CTA starts at the even split and
// grows by 1 % until the deal fits the wave.  Returns the items and the
// group offsets (groups.size() - 1 CTAs).
constexpr double kProlog = 3.0;
constexpr int kMinPiece = 4;

void deal_greedy(const std::vector<dn::WorkItem>& runs, double target, std::vector<dn::WorkItem>& items,
                 std::vector<int>& groups)
{
  items.clear();
  groups.assign(1, 0);
  double acc = 0;
  for (const auto& r : runs) {
    int i = r.i0;
    while (i < r.i1) {
      if (acc > 0 && acc + kProlog + kMinPiece > target) {   // this CTA is full
        groups.push_back((int)items.size());
        acc = 0;
      }
      acc += kProlog;
      int take = std::max((int)std::ceil(target - acc), kMinPiece);
      take = std::min(take, r.i1 - i);
      if (r.i1 - i - take > 0 && r.i1 - i - take < kMinPiece) take = r.i1 - i;   // no short leftover
      items.push_back(dn::WorkItem{r.patch, r.j0, r.k0, i, i + take});
      acc += take;
      i += take;
    }
  }
  groups.push_back((int)items.size());
}

void deal_runs(const std::vector<dn::WorkItem>& runs, int slots, std::vector<dn::WorkItem>& items,
               std::vector<int>& groups)
{
  long planes = 0;
  for (const auto& r : runs) planes += r.i1 - r.i0;
  const long want = std::max(1L, std::min<long>(slots, planes / (2 * kMinPiece)));
  double target = ((double)planes + kProlog * (double)want) / (double)want;
  for (int k = 0; k < 400; ++k) {
    deal_greedy(runs, target, items, groups);
    if ((long)groups.size() - 1 <= want) return;
    target *= 1.01;
  }
}

// Column tiles (j0, k0, tile shape) of a patch whose batched tile shape is
// `shape`.  An FP32-bulk patch with 16 x 32 tiles covers a remainder on a
// closed axis with narrower tiles: a last column of at most 16 cells with
// 16 x 16 tiles, a last band of at most 8 rows with 8 x 32 tiles (its corner
// with a 16 x 16 tile).  They leave fewer idle lanes than 16 x 32 tiles
// reaching beyond the patch; every cell is computed the same way in any
// tile, so the bits do not change.
struct TileRef {
  int j0, k0, shape;
};

void patch_tiles(const dn_ctx* c, const DnPatch& P, int shape, std::vector<TileRef>& out)
{
  out.clear();
  const bool fp64 = c->precision == DN_FP64;
  int tj, tk;
  dn::shape_tile(fp64, shape, &tj, &tk);
  const int nj = P.d.nj, nk = P.d.nk;
  int njm = nj, nkm = nk;          // the extents the main shape covers
  bool kr = false, jr = false;
  if (!fp64 && shape == 2) {
    const int krem = nk % 32, jrem = nj % 16;
    kr = P.d.face[2] != DN_FACE_PERIODIC && nk > 32 && krem > 0 && krem <= 16;
    jr = P.d.face[1] != DN_FACE_PERIODIC && nj > 16 && jrem > 0 && jrem <= 8;
    if (kr) nkm = nk - krem;
    if (jr) njm = nj - jrem;
  }
  for (int j0 = 0; j0 < njm; j0 += tj)
    for (int k0 = 0; k0 < nkm; k0 += tk) out.push_back(TileRef{j0, k0, shape});
  if (kr)
    for (int j0 = 0; j0 < njm; j0 += 16) out.push_back(TileRef{j0, nkm, 1});
  if (jr) {
    for (int k0 = 0; k0 < nkm; k0 += 32) out.push_back(TileRef{njm, k0, 0});
    if (kr) out.push_back(TileRef{njm, nkm, 1});
  }
}

// Patch records and work items (patch, column tile, plane range) of every
// patch, grouped by tile form and shape.  FX32: each launch is one wave of
// persistent CTAs over balanced groups of items (deal_runs).  FP64: plane
// ranges sized so that the launch holds about four waves of CTAs.
int build_batch(dn_ctx* c)
{
  free_batch(c);
  const size_t np = c->patches.size();
  if (np == 0) { c->batch_dirty = false; return DN_OK; }
  const bool fp64 = c->precision == DN_FP64;
  std::vector<dn::BatchPatch> rec(np);
  // tensor maps per tile shape and patch: maps[shape * np + patch]
  std::vector<dn::BatchMaps> maps(np * dn::kNumShapes);
  std::vector<std::vector<TileRef>> ptiles(np);
  long tiles = 0;
  for (size_t q = 0; q < np; ++q) {
    const DnPatch& P = c->patches[q];
    dn::BatchPatch& r = rec[q];
    std::memset(&r, 0, sizeof(r));
    for (int b = 0; b < 3; ++b) r.buf[b] = P.buf[b];
    r.active = P.active;
    r.ni = P.d.ni; r.nj = P.d.nj; r.nk = P.d.nk; r.kp = P.kp;
    r.per_x = P.d.face[0] == DN_FACE_PERIODIC;
    r.per_y = P.d.face[1] == DN_FACE_PERIODIC;
    r.per_z = P.d.face[2] == DN_FACE_PERIODIC;
    r.dx = P.d.dx; r.dy = P.d.dy; r.dz = P.d.dz;
    for (int v = 0; v < 5; ++v) { r.base[v] = P.base[v]; r.quantum[v] = P.quantum[v]; }
    r.wall = P.wall;
    patch_tiles(c, P, c->shape[q], ptiles[q]);
    bool used[dn::kNumShapes] = {};
    for (const TileRef& t : ptiles[q]) used[t.shape] = true;
    if (P.owned && P.patch_active) tiles += (long)ptiles[q].size();
    // shadows are never staged: no tensor maps
    r.tma = P.owned ? 1 : 0;
    for (int sh = 0; sh < dn::kNumShapes && r.tma; ++sh) {
      if (!used[sh]) continue;
      int tj, tk;
      dn::shape_tile(fp64, sh, &tj, &tk);
      dn::BatchMaps& M = maps[(size_t)sh * np + q];
      if (!fp64) {
        dn::FxGeom g{};
        g.ni = P.d.ni; g.nj = P.d.nj; g.nk = P.d.nk; g.kp = P.kp;
        for (int b = 0; b < 3 && r.tma; ++b)
          r.tma = dn::encode_stage_maps(M.in[b], &M.un[b], (const int32_t*)P.buf[b], (const int32_t*)P.buf[b], g,
                                        tj, tk) ? 1 : 0;
      } else {
        for (int b = 0; b < 3 && r.tma; ++b)
          r.tma = dn::encode_stage_map_f64(&M.in[b][0], (const double*)P.buf[b], P.d.ni, P.d.nj, P.d.nk, tj, tk)
                      ? 1 : 0;
      }
    }
  }
  if (tiles == 0) {
    // no owned patch (a rank whose share of the grid is empty): nothing to launch
    c->batch_dirty = false;
    return DN_OK;
  }
  const long want = (long)c->num_sms * 2 * 4;
  long chunks = (want + tiles - 1) / tiles;
  if (chunks < 1) chunks = 1;
  // FX32 items go to one list per tile form: full tiles (every y/z slope
  // and face exists: no edge test), tiles inside the patch next to a closed
  // face (per-thread face masks), tiles that reach beyond the patch; a
  // launch per form keeps one code path per kernel
  std::vector<dn::WorkItem> items[3][dn::kNumShapes];
  std::vector<int> groups[3][dn::kNumShapes];
  for (size_t q = 0; q < np; ++q) {
    const DnPatch& P = c->patches[q];
    if (!P.owned || !P.patch_active) continue;
    const bool per_y = P.d.face[1] == DN_FACE_PERIODIC, per_z = P.d.face[2] == DN_FACE_PERIODIC;
    // persistent CTAs: one run of all planes per column tile, cut by
    // deal_runs below
    const bool persistent = !fp64 && c->batch_waves > 0;
    long ic = (P.d.ni + chunks - 1) / chunks;
    if (ic < c->batch_min_planes) ic = c->batch_min_planes;   // amortise each item's 3-plane prologue
    if (ic > P.d.ni || persistent) ic = P.d.ni;
    for (int i0 = 0; i0 < P.d.ni; i0 += (int)ic)
      for (const TileRef& t : ptiles[q]) {
        int tj, tk;
        dn::shape_tile(fp64, t.shape, &tj, &tk);
        const int j0 = t.j0, k0 = t.k0;
        const bool fy = (j0 + tj <= P.d.nj) && (per_y || (j0 >= 2 && j0 + tj + 2 <= P.d.nj));
        const bool fz = (k0 + tk <= P.d.nk) && (per_z || (k0 >= 2 && k0 + tk + 2 <= P.d.nk));
        const bool inside = j0 + tj <= P.d.nj && k0 + tk <= P.d.nk;
        const int form = fp64 ? dn::kFxEdge : (fy && fz) ? dn::kFxFull : inside ? dn::kFxInside : dn::kFxEdge;
        items[form][t.shape].push_back(dn::WorkItem{(int)q, j0, k0, i0, std::min(P.d.ni, i0 + (int)ic)});
      }
  }
  if (!fp64 && c->batch_waves > 0) {
    for (int f = 0; f < 3; ++f) {
      for (int q = 0; q < dn::kNumShapes; ++q) {
        if (items[f][q].empty()) continue;
        int occ = 0;
        cudaError_t e = dn::fx32_batched_occupancy(q, f, &occ);
        if (e != cudaSuccess) return cuda_fail(c, e, "batched stage occupancy");
        const std::vector<dn::WorkItem> runs = items[f][q];
        deal_runs(runs, c->num_sms * std::max(1, occ) * c->batch_waves, items[f][q], groups[f][q]);
      }
    }
  }
  cudaError_t e = cudaMalloc(&c->d_records, np * sizeof(dn::BatchPatch));
  if (e != cudaSuccess) return fail(c, DN_ERR_NOMEM, "cudaMalloc(patch records)");
  e = cudaMemcpyAsync(c->d_records, rec.data(), np * sizeof(dn::BatchPatch), cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "patch record upload");
  if (!maps.empty()) {
    e = cudaMalloc(&c->d_maps, maps.size() * sizeof(dn::BatchMaps));
    if (e != cudaSuccess) return fail(c, DN_ERR_NOMEM, "cudaMalloc(tensor maps)");
    e = cudaMemcpyAsync(c->d_maps, maps.data(), maps.size() * sizeof(dn::BatchMaps), cudaMemcpyHostToDevice,
                        c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "tensor map upload");
  }
  for (int f = 0; f < 3; ++f) {
    for (int q = 0; q < dn::kNumShapes; ++q) {
      const std::vector<dn::WorkItem>& it = items[f][q];
      if (it.empty()) continue;
      if (it.size() > (size_t)INT32_MAX) return fail(c, DN_ERR_RANGE, "too many work items");
      e = cudaMalloc(&c->d_items[f][q], it.size() * sizeof(dn::WorkItem));
      if (e != cudaSuccess) return fail(c, DN_ERR_NOMEM, "cudaMalloc(work items)");
      e = cudaMemcpyAsync(c->d_items[f][q], it.data(), it.size() * sizeof(dn::WorkItem), cudaMemcpyHostToDevice,
                          c->stream);
      if (e != cudaSuccess) return cuda_fail(c, e, "work item upload");
      c->n_items[f][q] = (int)it.size();
      const std::vector<int>& gr = groups[f][q];
      if (!gr.empty()) {
        e = cudaMalloc(&c->d_groups[f][q], gr.size() * sizeof(int));
        if (e != cudaSuccess) return fail(c, DN_ERR_NOMEM, "cudaMalloc(work groups)");
        e = cudaMemcpyAsync(c->d_groups[f][q], gr.data(), gr.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) return cuda_fail(c, e, "work group upload");
        c->n_groups[f][q] = (int)gr.size() - 1;
      }
    }
  }
  e = cudaStreamSynchronize(c->stream);   // host vectors go out of scope
  if (e != cudaSuccess) return cuda_fail(c, e, "batch upload");
  c->batch_dirty = false;
  return DN_OK;
}

int stage_patch(dn_ctx* c, DnPatch& p, int in_b, int un_b, int out_b, double factor);

// An inactive (or unlisted) patch's state carried from buffer in_b into out_b.
int carry_patch(dn_ctx* c, DnPatch& p, int in_b, int out_b)
{
  if (in_b == out_b) return DN_OK;
  cudaError_t e = cudaMemcpyAsync(p.buf[out_b], p.buf[in_b], 5 * p.ncp * elem_size(c), cudaMemcpyDeviceToDevice,
                                  c->stream);
  return e == cudaSuccess ? DN_OK : cuda_fail(c, e, "inactive patch copy");
}

// One RK stage of every active patch: in_b -> out_b with step-start state
// un_b; inactive patches carry their state into out_b.
int stage_all(dn_ctx* c, int in_b, int un_b, int out_b, double factor)
{
  NvtxRange nvtx("dn stage");
  donor_stale(c, out_b);
  int s;
  for (auto& p : c->patches) {
    if (p.owned && !p.patch_active && (s = carry_patch(c, p, in_b, out_b))) return s;
  }
  // a single patch keeps its parameters in the kernel's constant bank (the
  // batched form reads them from shared memory); the results are identical.
  // Flux functors (another scheme or a user stage function) run per patch.
  const bool functor = c->precision == DN_FP64 && (c->scheme != DN_FLUX_AUSMPLUS || c->stage_fn);
  if (!c->batched || c->patches.size() == 1 || functor) {
    for (auto& p : c->patches) {
      if (!p.owned || !p.patch_active) continue;
      s = stage_patch(c, p, in_b, un_b, out_b, factor);
      if (s) return s;
    }
    return DN_OK;
  }
  if (c->batch_dirty && (s = build_batch(c))) return s;
  // full-tile launches on the context's stream, inside- and edge-tile
  // launches on a second branch forked from it and joined after (they write
  // disjoint tiles), so the forms overlap instead of queueing behind each
  // other
  bool any_edge = false, any_full = false;
  for (int q = 0; q < dn::kNumShapes; ++q) {
    any_edge = any_edge || c->n_items[dn::kFxEdge][q] > 0 || c->n_items[dn::kFxInside][q] > 0;
    any_full = any_full || c->n_items[dn::kFxFull][q] > 0;
  }
  const bool fork = any_edge && any_full;
  cudaError_t e = cudaSuccess;
  if (fork) {
    if (!c->s_aux) {
      e = cudaStreamCreateWithFlags(&c->s_aux, cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
      if (e != cudaSuccess) return cuda_fail(c, e, "stage branch stream");
    }
    e = cudaEventRecord(c->ev_fork, c->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->s_aux, c->ev_fork, 0);
    if (e != cudaSuccess) return cuda_fail(c, e, "stage branch fork");
  }
  for (int f = dn::kFxFull; f >= dn::kFxEdge; --f) {
    cudaStream_t st = (fork && f != dn::kFxFull) ? c->s_aux : c->stream;
    for (int q = 0; q < dn::kNumShapes; ++q) {
      if (!c->n_items[f][q]) continue;
      dn::Batch b;
      b.patches = static_cast<const dn::BatchPatch*>(c->d_records);
      b.maps = c->d_maps ? static_cast<const dn::BatchMaps*>(c->d_maps) + (size_t)q * c->patches.size() : nullptr;
      b.items = static_cast<const dn::WorkItem*>(c->d_items[f][q]);
      b.n_items = c->n_items[f][q];
      b.groups = static_cast<const int*>(c->d_groups[f][q]);
      b.n_groups = c->n_groups[f][q];
      b.in_b = in_b; b.un_b = un_b; b.out_b = out_b;
      b.factor = factor;
      b.err = c->d_err;
      b.err_info = c->d_err_info;
      e = c->precision == DN_FP64 ? dn::launch_stage_f64_batched(b, q, st)
                                  : dn::launch_stage_fx32_batched(b, q, f, st);
      c->launches++;
      if (e != cudaSuccess) return cuda_fail(c, e, "batched stage launch");
    }
  }
  if (fork) {
    e = cudaEventRecord(c->ev_join, c->s_aux);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, c->ev_join, 0);
    if (e != cudaSuccess) return cuda_fail(c, e, "stage branch join");
  }
  return DN_OK;
}

int stage_patch(dn_ctx* c, DnPatch& p, int in_b, int un_b, int out_b, double factor)
{
  const double dx = p.d.dx, dy = p.d.dy, dz = p.d.dz;
  const double dV = dx * dy * dz;
  const double pf = factor / dV;
  dn::StageGeom g;
  g.ni = p.d.ni; g.nj = p.d.nj; g.nk = p.d.nk;
  g.per_x = p.d.face[0] == DN_FACE_PERIODIC;
  g.per_y = p.d.face[1] == DN_FACE_PERIODIC;
  g.per_z = p.d.face[2] == DN_FACE_PERIODIC;
  cudaError_t e;
  if (c->precision == DN_FP64 && (c->scheme != DN_FLUX_AUSMPLUS || c->stage_fn)) {
    dn_stage_launch L;
    L.patch = (int)(&p - c->patches.data());
    L.in = (const double*)p.buf[in_b];
    L.un = (const double*)p.buf[un_b];
    L.out = (double*)p.buf[out_b];
    L.active = p.active;
    L.ni = g.ni; L.nj = g.nj; L.nk = g.nk;
    L.periodic[0] = g.per_x; L.periodic[1] = g.per_y; L.periodic[2] = g.per_z;
    L.dx = dx; L.dy = dy; L.dz = dz;
    L.factor = factor;
    L.stream = (void*)c->stream;
    L.num_sms = c->num_sms;
    c->launches++;
    if (c->stage_fn) {
      const int rc = c->stage_fn(c->stage_user, &L);
      if (rc) return fail(c, rc < 0 ? rc : DN_ERR_ARG, "user stage function returned %d for patch %d", rc, L.patch);
      return DN_OK;
    }
    e = dn::launch_scheme_stage(c->scheme, &L, p.wall);
    if (e != cudaSuccess) return cuda_fail(c, e, "functor stage launch");
    return DN_OK;
  } else if (c->precision == DN_FP64) {
    dn::StageArgs<dn::PolicyF64> a;
    a.in = (const double*)p.buf[in_b];
    a.un = (const double*)p.buf[un_b];
    a.out = (double*)p.buf[out_b];
    a.active = p.active;
    a.err = c->d_err;
    a.err_info = c->d_err_info;
    g.i_chunk = dn::default_i_chunk(g.ni, g.nj, g.nk, 4, 32, c->num_sms, 3);
    a.g = g;
    a.p.Ax = dy * dz; a.p.Ay = dx * dz; a.p.Az = dx * dy; a.p.pf = pf;
    a.wall = p.wall;
    e = dn::launch_stage_f64(a, dn::StageShape{4, 32, g.i_chunk}, c->stream);
  } else {
    dn::FxArgs a;
    a.in = (const int32_t*)p.buf[in_b];
    a.un = (const int32_t*)p.buf[un_b];
    a.out = (int32_t*)p.buf[out_b];
    a.active = p.active;
    a.err = c->d_err;
    a.err_info = c->d_err_info;
    int tj, tk;
    dn::fx32_tile(&tj, &tk);
    a.g.ni = g.ni; a.g.nj = g.nj; a.g.nk = g.nk; a.g.kp = p.kp;
    a.g.per_x = g.per_x; a.g.per_y = g.per_y; a.g.per_z = g.per_z;
    a.g.i_chunk = p.i_chunk > 0 ? std::min(p.i_chunk, g.ni)
                                : dn::default_i_chunk(g.ni, g.nj, g.nk, tj, tk, c->num_sms, DN_FX_WAVE_CTAS);
    dn::fx_set_params(a.p, dx, dy, dz, factor, p.base, p.quantum);
    a.wall = p.wall;
    e = dn::launch_stage_fx32(a, c->stream);
  }
  c->launches++;
  if (e != cudaSuccess) return cuda_fail(c, e, "stage kernel launch");
  return DN_OK;
}

// Upload into a compact shadow: the FP32-bulk base and quantum derived from
// the whole host state (as its owner derives them), then the held cells,
// gathered on the host.
template <typename H>
int upload_shadow(dn_ctx* c, DnPatch& p, int field, const H* host)
{
  if (c->precision == DN_FP32 && !p.base_set) {
    derive_base(p, host);
    c->plan_dirty = true;
    c->ls_dirty = true;
    c->batch_dirty = true;
    c->generation++;
  }
  const size_t m = p.held.size();
  if (m == 0) return DN_OK;
  std::vector<H> g(5 * m);
  for (int v = 0; v < 5; ++v)
    for (size_t t = 0; t < m; ++t) g[(size_t)v * m + t] = host[(size_t)v * p.nc + p.held[t]];
  int s;
  if ((s = ensure_staging(c, g.size() * sizeof(H)))) return s;
  cudaError_t e = cudaMemcpyAsync(c->staging, g.data(), g.size() * sizeof(H), cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "shadow upload copy");
  void* dst = p.buf[c->fmap[field]];
  if (c->precision == DN_FP64) {
    k_convert<H, double><<<grid_for(5 * m), 256, 0, c->stream>>>((const H*)c->staging, (double*)dst, 5 * m);
  } else {
    // held positions are consecutive: rows of m cells, pitch m
    k_quantize<H><<<grid_for(5 * m), 256, 0, c->stream>>>((const H*)c->staging, (int32_t*)dst, m, (int)m, (int)m,
                                                       qparams(p), c->d_err);
  }
  c->launches++;
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(c, e, "shadow upload conversion");
  e = cudaStreamSynchronize(c->stream);     // the gathered host vector goes out of scope
  if (e != cudaSuccess) return cuda_fail(c, e, "shadow upload");
  return read_device_error(c);
}

template <typename H>
int upload_impl(dn_ctx* c, int id, int field, const H* host)
{
  NvtxRange nvtx("dn upload");
  int s = check_patch(c, id);
  if (s) return s;
  if ((s = check_field(c, field))) return s;
  if (!host) return fail(c, DN_ERR_ARG, "host pointer is NULL");
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  donor_stale(c, c->fmap[field]);
  DnPatch& p = c->patches[id];
  if (p.compact) return upload_shadow(c, p, field, host);
  void* dst = p.buf[c->fmap[field]];
  const size_t n = 5 * p.nc;
  cudaError_t e;
  if (c->precision == DN_FP64 && sizeof(H) == sizeof(double)) {
    e = cudaMemcpyAsync(dst, host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "upload copy");
    return DN_OK;
  }
  if (c->precision == DN_FP32 && !p.base_set) {
    derive_base(p, host);
    c->plan_dirty = true;
    c->ls_dirty = true;
    c->batch_dirty = true;
    c->generation++;
  }
  if ((s = ensure_staging(c, n * sizeof(H)))) return s;
  e = cudaMemcpyAsync(c->staging, host, n * sizeof(H), cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "upload copy");
  if (c->precision == DN_FP64) {
    k_convert<H, double><<<grid_for(n), 256, 0, c->stream>>>((const H*)c->staging, (double*)dst, n);
  } else {
    k_quantize<H><<<grid_for(n), 256, 0, c->stream>>>((const H*)c->staging, (int32_t*)dst, p.nc, p.d.nk, p.kp,
                                                   qparams(p), c->d_err);
  }
  c->launches++;
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(c, e, "upload conversion");
  if (c->precision == DN_FP32) return read_device_error(c);
  return DN_OK;
}

template <typename H>
int download_impl(dn_ctx* c, int id, int field, H* host)
{
  NvtxRange nvtx("dn download");
  int s = check_whole(c, id);
  if (s) return s;
  if ((s = check_field(c, field))) return s;
  if (!host) return fail(c, DN_ERR_ARG, "host pointer is NULL");
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  DnPatch& p = c->patches[id];
  const void* src = p.buf[c->fmap[field]];
  const size_t n = 5 * p.nc;
  cudaError_t e;
  if (c->precision == DN_FP64 && sizeof(H) == sizeof(double)) {
    e = cudaMemcpyAsync(host, src, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  } else {
    if ((s = ensure_staging(c, n * sizeof(H)))) return s;
    if (c->precision == DN_FP64) {
      k_convert<double, H><<<grid_for(n), 256, 0, c->stream>>>((const double*)src, (H*)c->staging, n);
    } else {
      k_dequantize<H><<<grid_for(n), 256, 0, c->stream>>>((const int32_t*)src, (H*)c->staging, p.nc, p.d.nk,
                                                     p.kp, qparams(p));
    }
    c->launches++;
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "download conversion");
    e = cudaMemcpyAsync(host, c->staging, n * sizeof(H), cudaMemcpyDeviceToHost, c->stream);
  }
  if (e != cudaSuccess) return cuda_fail(c, e, "download copy");
  e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "download sync");
  return read_device_error(c);
}

int ensure_async(dn_ctx* c)
{
  if (c->s_in) return DN_OK;
  bool ok = cudaStreamCreateWithFlags(&c->s_in, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&c->s_out, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&c->s_conv, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&c->ev_main, cudaEventDisableTiming) == cudaSuccess;
  for (int b = 0; b < 2 && ok; ++b)
    ok = cudaEventCreateWithFlags(&c->ev_in_done[b], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&c->ev_in_free[b], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&c->ev_out_read[b], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&c->ev_d2h_done[b], cudaEventDisableTiming) == cudaSuccess;
  return ok ? DN_OK : fail(c, DN_ERR_CUDA, "cannot create the transfer streams");
}

int ensure_buffer(dn_ctx* c, void*& buf, size_t& cap, size_t bytes)
{
  if (cap >= bytes) return DN_OK;
  if (buf) cudaFree(buf);
  buf = nullptr;
  cap = 0;
  cudaError_t e = cudaMalloc(&buf, bytes);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc(transfer staging)");
  cap = bytes;
  return DN_OK;
}

// Upload through the copy-in stream: host -> staging[b] on s_in, then the
// conversion into the field on the context's stream once the copy is done.
// Staging[b] is refilled only after the conversion that read it.
template <typename H>
int upload_async_impl(dn_ctx* c, int id, int field, const H* host)
{
  NvtxRange nvtx("dn upload (async)");
  int s = check_whole(c, id);
  if (s) return s;
  if ((s = check_field(c, field))) return s;
  if (!host) return fail(c, DN_ERR_ARG, "host pointer is NULL");
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  if ((s = ensure_async(c))) return s;
  donor_stale(c, c->fmap[field]);
  DnPatch& p = c->patches[id];
  if (c->precision == DN_FP32 && !p.base_set) {
    derive_base(p, host);
    c->plan_dirty = true;
    c->ls_dirty = true;
    c->batch_dirty = true;
    c->generation++;
  }
  const int b = (int)(c->in_seq++ & 1);
  const size_t n = 5 * p.nc;
  if ((s = ensure_buffer(c, c->st_in[b], c->st_in_bytes[b], n * sizeof(H)))) return s;
  cudaError_t e = cudaSuccess;
  if (c->ev_in_free_set[b]) e = cudaStreamWaitEvent(c->s_in, c->ev_in_free[b], 0);
  if (e == cudaSuccess) e = cudaMemcpyAsync(c->st_in[b], host, n * sizeof(H), cudaMemcpyHostToDevice, c->s_in);
  if (e == cudaSuccess) e = cudaEventRecord(c->ev_in_done[b], c->s_in);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, c->ev_in_done[b], 0);
  if (e != cudaSuccess) return cuda_fail(c, e, "asynchronous upload copy");
  void* dst = p.buf[c->fmap[field]];
  if (c->precision == DN_FP64) {
    k_convert<H, double><<<grid_for(n), 256, 0, c->stream>>>((const H*)c->st_in[b], (double*)dst, n);
  } else {
    k_quantize<H><<<grid_for(n), 256, 0, c->stream>>>((const H*)c->st_in[b], (int32_t*)dst, p.nc, p.d.nk, p.kp,
                                                   qparams(p), c->d_err);
  }
  c->launches++;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaEventRecord(c->ev_in_free[b], c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "asynchronous upload conversion");
  c->ev_in_free_set[b] = true;
  return DN_OK;
}

// Download: once the context's stream reached this point, the field is
// converted into staging[b] on the conversion stream (after the previous
// copy out of staging[b] has finished); the context's stream waits for that
// conversion only, and the copy to the host runs on s_out.  A conversion
// never queues behind an earlier host copy, so the copies of consecutive
// downloads run back to back while the stages continue.
template <typename H>
int download_async_impl(dn_ctx* c, int id, int field, H* host)
{
  NvtxRange nvtx("dn download (async)");
  int s = check_whole(c, id);
  if (s) return s;
  if ((s = check_field(c, field))) return s;
  if (!host) return fail(c, DN_ERR_ARG, "host pointer is NULL");
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  if ((s = ensure_async(c))) return s;
  DnPatch& p = c->patches[id];
  const int b = (int)(c->out_seq++ & 1);
  const size_t n = 5 * p.nc;
  if ((s = ensure_buffer(c, c->st_out[b], c->st_out_bytes[b], n * sizeof(H)))) return s;
  cudaError_t e = cudaEventRecord(c->ev_main, c->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c->s_conv, c->ev_main, 0);
  if (e == cudaSuccess && c->ev_d2h_done_set[b]) e = cudaStreamWaitEvent(c->s_conv, c->ev_d2h_done[b], 0);
  if (e != cudaSuccess) return cuda_fail(c, e, "asynchronous download ordering");
  const void* src = p.buf[c->fmap[field]];
  if (c->precision == DN_FP64) {
    k_convert<double, H><<<grid_for(n), 256, 0, c->s_conv>>>((const double*)src, (H*)c->st_out[b], n);
  } else {
    k_dequantize<H><<<grid_for(n), 256, 0, c->s_conv>>>((const int32_t*)src, (H*)c->st_out[b], p.nc, p.d.nk,
                                                      p.kp, qparams(p));
  }
  c->launches++;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaEventRecord(c->ev_out_read[b], c->s_conv);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, c->ev_out_read[b], 0);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c->s_out, c->ev_out_read[b], 0);
  if (e == cudaSuccess) e = cudaMemcpyAsync(host, c->st_out[b], n * sizeof(H), cudaMemcpyDeviceToHost, c->s_out);
  if (e == cudaSuccess) e = cudaEventRecord(c->ev_d2h_done[b], c->s_out);
  if (e != cudaSuccess) return cuda_fail(c, e, "asynchronous download copy");
  c->ev_d2h_done_set[b] = true;
  return DN_OK;
}

} // namespace

extern "C" {

int dn_ctx_create(int device, int precision, dn_ctx** out)
{
  if (!out) return DN_ERR_ARG;
  *out = nullptr;
  if (precision != DN_FP64 && precision != DN_FP32) return DN_ERR_ARG;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return DN_ERR_CUDA;
  dn_ctx* c = new dn_ctx();
  c->device = device;
  c->precision = precision;
  if (set_device(c) != DN_OK) { delete c; return DN_ERR_CUDA; }
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) { delete c; return DN_ERR_CUDA; }
  c->stream = c->own;
  if (cudaMalloc(&c->d_err, sizeof(int)) != cudaSuccess) { cudaStreamDestroy(c->own); delete c; return DN_ERR_NOMEM; }
  if (cudaMalloc(&c->d_err_info, 4 * sizeof(unsigned long long)) != cudaSuccess) {
    cudaFree(c->d_err); cudaStreamDestroy(c->own); delete c; return DN_ERR_NOMEM;
  }
  cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
  cudaMemsetAsync(c->d_err_info, 0xff, 4 * sizeof(unsigned long long), c->stream);
  *out = c;
  return DN_OK;
}

int dn_ctx_destroy(dn_ctx* c)
{
  if (!c) return DN_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (auto& p : c->patches) {
    for (int b = 0; b < 3; ++b) if (p.buf[b]) cudaFree(p.buf[b]);
    if (p.active) cudaFree(p.active);
    for (int sd = 0; sd < 6; ++sd) if (p.wall.table[sd]) cudaFree((void*)p.wall.table[sd]);
  }
  free_graphs(c);
  free_plan(c);
  free_ls_plan(c);
  free_batch(c);
  if (c->staging) cudaFree(c->staging);
  if (c->s_in) cudaStreamSynchronize(c->s_in);
  if (c->s_conv) cudaStreamSynchronize(c->s_conv);
  if (c->s_out) cudaStreamSynchronize(c->s_out);
  for (int b = 0; b < 2; ++b) {
    if (c->st_in[b]) cudaFree(c->st_in[b]);
    if (c->st_out[b]) cudaFree(c->st_out[b]);
    if (c->ev_in_done[b]) cudaEventDestroy(c->ev_in_done[b]);
    if (c->ev_in_free[b]) cudaEventDestroy(c->ev_in_free[b]);
    if (c->ev_out_read[b]) cudaEventDestroy(c->ev_out_read[b]);
    if (c->ev_d2h_done[b]) cudaEventDestroy(c->ev_d2h_done[b]);
  }
  if (c->ev_main) cudaEventDestroy(c->ev_main);
  if (c->s_aux) cudaStreamSynchronize(c->s_aux);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->s_aux) cudaStreamDestroy(c->s_aux);
  if (c->s_in) cudaStreamDestroy(c->s_in);
  if (c->s_conv) cudaStreamDestroy(c->s_conv);
  if (c->s_out) cudaStreamDestroy(c->s_out);
  if (c->d_partials) cudaFree(c->d_partials);
  if (c->d_err) cudaFree(c->d_err);
  if (c->d_err_info) cudaFree(c->d_err_info);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
  return DN_OK;
}

int dn_last_error(const dn_ctx* c, char* buf, size_t n)
{
  if (!c || !buf || n == 0) return DN_ERR_ARG;
  std::strncpy(buf, c->err.c_str(), n - 1);
  buf[n - 1] = 0;
  return DN_OK;
}

int dn_set_stream(dn_ctx* c, void* stream)
{
  if (!c) return DN_ERR_ARG;
  c->stream = stream ? (cudaStream_t)stream : c->own;
  return DN_OK;
}

namespace {

int add_patch(dn_ctx* c, const dn_patch_desc* d, int* id, bool compact)
{
  if (!c || !d || !id) return DN_ERR_ARG;
  if (d->ni < 1 || d->nj < 1 || d->nk < 1) return fail(c, DN_ERR_ARG, "patch size must be positive");
  for (int a = 0; a < 3; ++a) {
    if (d->face[a] != DN_FACE_PERIODIC && d->face[a] != DN_FACE_CLOSED)
      return fail(c, DN_ERR_ARG, "face kind of axis %d is not DN_FACE_PERIODIC or DN_FACE_CLOSED", a);
    const int n = a == 0 ? d->ni : (a == 1 ? d->nj : d->nk);
    if (d->face[a] == DN_FACE_PERIODIC && n < 3)
      return fail(c, DN_ERR_ARG, "periodic axis %d needs at least 3 cells", a);
  }
  dn_patch_desc dd = *d;
  const int nn[3] = {d->ni, d->nj, d->nk};
  double* sp[3] = {&dd.dx, &dd.dy, &dd.dz};
  for (int a = 0; a < 3; ++a) {
    if (d->length[a] > 0) *sp[a] = d->length[a] / nn[a];   // CartesianPatch::computeDeltas
    if (!(*sp[a] > 0) || !std::isfinite(*sp[a])) return fail(c, DN_ERR_ARG, "cell spacing of axis %d must be positive", a);
    if (!std::isfinite(d->origin[a])) return fail(c, DN_ERR_ARG, "origin must be finite");
    if (d->seek[2 * a] < 0 || d->seek[2 * a + 1] < 0 || d->add_protect < 0 ||
        d->seek[2 * a] + d->seek[2 * a + 1] + 2 * d->add_protect > nn[a])
      return fail(c, DN_ERR_ARG, "seek/protect layers of axis %d exceed the patch", a);
    if (d->face[a] == DN_FACE_PERIODIC && (d->seek[2 * a] || d->seek[2 * a + 1]))
      return fail(c, DN_ERR_ARG, "a periodic axis (%d) cannot have seek layers", a);
  }
  const size_t nc = (size_t)d->ni * d->nj * d->nk;
  if (nc > ((size_t)1 << 40)) return fail(c, DN_ERR_ARG, "patch too large");
  // FX32 rows padded to a multiple of 4 int32 (16 bytes): every row of every
  // patch can then be staged by TMA boxes
  const int kp = c->precision == DN_FP32 ? (d->nk + 3) / 4 * 4 : d->nk;
  const size_t ncp = (size_t)d->ni * d->nj * kp;
  if (c->precision == DN_FP32 && 5 * ncp >= ((size_t)1 << 31))
    return fail(c, DN_ERR_ARG, "FP32 patch limited to 5*ni*nj*nk < 2^31 (32-bit element offsets; nk rounded up to "
                "a multiple of 4)");
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  DnPatch p;
  p.d = dd;
  p.nc = nc;
  p.kp = kp;
  p.ncp = compact ? 0 : ncp;
  p.compact = compact;
  p.owned = !compact;
  const size_t bytes = 5 * p.ncp * elem_size(c);
  for (int b = 0; b < 3 && bytes; ++b) {
    cudaError_t e = cudaMalloc(&p.buf[b], bytes);
    if (e != cudaSuccess) {
      for (int q = 0; q < b; ++q) cudaFree(p.buf[q]);
      return fail(c, DN_ERR_NOMEM, "cudaMalloc of %zu bytes for a patch field failed", bytes);
    }
    cudaMemsetAsync(p.buf[b], 0, bytes, c->stream);
  }
  c->patches.push_back(p);
  c->tables.resize(c->patches.size());
  c->ls.resize(c->patches.size());
  c->ls_on.resize(c->patches.size(), 0);
  c->lsg.resize(c->patches.size());
  c->lsg_on.resize(c->patches.size(), 0);
  c->shape.push_back(default_shape(c->patches.back()));
  c->plan_dirty = true;
  c->ls_dirty = true;
  c->batch_dirty = true;
  c->generation++;
  *id = (int)c->patches.size() - 1;
  return DN_OK;
}

} // namespace

int dn_patch_add(dn_ctx* c, const dn_patch_desc* d, int* id) { return add_patch(c, d, id, false); }

int dn_patch_add_shadow(dn_ctx* c, const dn_patch_desc* d, int* id) { return add_patch(c, d, id, true); }

int dn_patch_device_cells(dn_ctx* c, int id, int64_t* cells)
{
  int s = check_patch(c, id);
  if (s) return s;
  if (!cells) return fail(c, DN_ERR_ARG, "output pointer is NULL");
  *cells = (int64_t)c->patches[id].ncp;
  return DN_OK;
}

int dn_patch_set_base(dn_ctx* c, int id, const double base[5], const double range[5])
{
  int s = check_patch(c, id);
  if (s) return s;
  if (!base || !range) return fail(c, DN_ERR_ARG, "base and range are required");
  DnPatch& p = c->patches[id];
  for (int v = 0; v < 5; ++v) {
    if (!std::isfinite(base[v]) || !(range[v] > 0) || !std::isfinite(range[v]))
      return fail(c, DN_ERR_ARG, "base/range of variable %d invalid", v);
  }
  for (int v = 0; v < 5; ++v) {
    p.base[v] = base[v];
    p.quantum[v] = std::ldexp(1.0, (int)std::ceil(std::log2(range[v] / (double)dn::kFxLimit)));
  }
  p.base_set = true;
  c->plan_dirty = true;
  c->ls_dirty = true;
  c->batch_dirty = true;
  c->generation++;
  return DN_OK;
}

int dn_patch_upload(dn_ctx* c, int id, int field, const double* host) { return upload_impl(c, id, field, host); }
int dn_patch_upload_f32(dn_ctx* c, int id, int field, const float* host) { return upload_impl(c, id, field, host); }
int dn_patch_download(dn_ctx* c, int id, int field, double* host) { return download_impl(c, id, field, host); }
int dn_patch_download_f32(dn_ctx* c, int id, int field, float* host) { return download_impl(c, id, field, host); }
int dn_patch_upload_async(dn_ctx* c, int id, int field, const double* host) { return upload_async_impl(c, id, field, host); }
int dn_patch_upload_f32_async(dn_ctx* c, int id, int field, const float* host) { return upload_async_impl(c, id, field, host); }
int dn_patch_download_async(dn_ctx* c, int id, int field, double* host) { return download_async_impl(c, id, field, host); }
int dn_patch_download_f32_async(dn_ctx* c, int id, int field, float* host) { return download_async_impl(c, id, field, host); }

int dn_patch_set_active(dn_ctx* c, int id, const uint8_t* mask)
{
  int s = (mask ? check_whole : check_patch)(c, id);
  if (s) return s;
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  DnPatch& p = c->patches[id];
  c->batch_dirty = true;
  c->generation++;
  if (!mask) {
    if (p.active) {
      cudaStreamSynchronize(c->stream);
      cudaFree(p.active);
    }
    p.active = nullptr;
    return DN_OK;
  }
  cudaError_t e;
  if (!p.active) {
    e = cudaMalloc(&p.active, p.ncp);
    if (e != cudaSuccess) return fail(c, DN_ERR_NOMEM, "cudaMalloc(active mask)");
    e = cudaMemsetAsync(p.active, 1, p.ncp, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "active mask");
  }
  // rows of nk flags into rows of kp (the padding stays set, never read)
  e = cudaMemcpy2DAsync(p.active, (size_t)p.kp, mask, (size_t)p.d.nk, (size_t)p.d.nk, (size_t)p.d.ni * p.d.nj,
                        cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "active mask upload");
  return DN_OK;
}

int dn_copy_field(dn_ctx* c, int i_src, int i_dst)
{
  if (!c) return DN_ERR_ARG;
  int s;
  if ((s = check_field(c, i_src)) || (s = check_field(c, i_dst))) return s;
  if (i_src == i_dst) return DN_OK;
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  donor_stale(c, c->fmap[i_dst]);
  for (auto& p : c->patches) {
    if (p.ncp == 0) continue;               // a compact shadow that holds no cell
    cudaError_t e = cudaMemcpyAsync(p.buf[c->fmap[i_dst]], p.buf[c->fmap[i_src]], 5 * p.ncp * elem_size(c),
                                    cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "copyField");
  }
  return DN_OK;
}

int dn_compute(dn_ctx* c, double factor)
{
  if (!c) return DN_ERR_ARG;
  if (!std::isfinite(factor)) return fail(c, DN_ERR_ARG, "factor is not finite");
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  int s = stage_all(c, c->fmap[0], c->fmap[1], c->fmap[2], factor);
  if (s) return s;
  std::swap(c->fmap[0], c->fmap[2]);
  return DN_OK;
}

int dn_compute_patches(dn_ctx* c, double factor, const int32_t* ids, int n)
{
  if (!c) return DN_ERR_ARG;
  if (n < 0 || (n > 0 && !ids)) return fail(c, DN_ERR_ARG, "invalid patch list");
  if (!std::isfinite(factor)) return fail(c, DN_ERR_ARG, "factor is not finite");
  std::vector<char> listed(c->patches.size(), 0);
  for (int q = 0; q < n; ++q) {
    if (ids[q] < 0 || ids[q] >= (int)c->patches.size()) return fail(c, DN_ERR_ARG, "invalid patch id %d", ids[q]);
    if (listed[ids[q]]) return fail(c, DN_ERR_ARG, "patch %d listed twice", ids[q]);
    listed[ids[q]] = 1;
  }
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  NvtxRange nvtx("dn stage (patch list)");
  const int in_b = c->fmap[0], un_b = c->fmap[1], out_b = c->fmap[2];
  donor_stale(c, out_b);
  int s;
  for (size_t q = 0; q < c->patches.size(); ++q) {
    DnPatch& p = c->patches[q];
    if (!p.owned) continue;
    s = (listed[q] && p.patch_active) ? stage_patch(c, p, in_b, un_b, out_b, factor) : carry_patch(c, p, in_b, out_b);
    if (s) return s;
  }
  std::swap(c->fmap[0], c->fmap[2]);
  return DN_OK;
}

int dn_patch_activate(dn_ctx* c, int id, int active)
{
  int s = check_patch(c, id);
  if (s) return s;
  if (c->patches[id].patch_active != (active != 0)) {
    c->patches[id].patch_active = active != 0;
    c->batch_dirty = true;
    c->generation++;
  }
  return DN_OK;
}

int dn_rk_step(dn_ctx* c, double dt, const double* alpha, int n_alpha)
{
  if (!c) return DN_ERR_ARG;
  NvtxRange nvtx("dn_rk_step");
  if (!alpha || n_alpha < 1 || n_alpha > 16) return fail(c, DN_ERR_ARG, "need 1..16 RK stage coefficients");
  if (!std::isfinite(dt)) return fail(c, DN_ERR_ARG, "dt is not finite");
  for (int q = 0; q < n_alpha; ++q) if (!std::isfinite(alpha[q])) return fail(c, DN_ERR_ARG, "alpha not finite");
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  // A = step-start state, X/Y = the two other buffers
  const int A = c->fmap[0], X = c->fmap[2], Y = c->fmap[1];
  int st;
  // a step with an exchange hook runs its launches directly: the hook's
  // transfers belong to the caller's library, not to a captured graph
  if (c->use_graph && !c->exch_fn) st = rk_step_graph(c, dt, alpha, n_alpha, A, X, Y);
  else st = rk_step_enqueue(c, dt, alpha, n_alpha, A, X, Y);
  if (st) return st;
  const int last = ((n_alpha - 1) & 1) ? Y : X;
  c->fmap[0] = last;
  c->fmap[1] = A;
  c->fmap[2] = (last == X) ? Y : X;
  return DN_OK;
}

int dn_sync(dn_ctx* c)
{
  if (!c) return DN_ERR_ARG;
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  cudaError_t e = cudaSuccess;
  if (c->s_in) e = cudaStreamSynchronize(c->s_in);
  if (e == cudaSuccess && c->s_conv) e = cudaStreamSynchronize(c->s_conv);
  if (e == cudaSuccess && c->s_out) e = cudaStreamSynchronize(c->s_out);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "stream synchronize");
  return read_device_error(c);
}

int dn_conservation_sums(dn_ctx* c, double out[5])
{
  if (!c || !out) return DN_ERR_ARG;
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  int s;
  if ((s = ensure_partials(c, (size_t)kSumBlocks * 5))) return s;
  std::vector<double> h((size_t)kSumBlocks * 5);
  std::vector<long long> hi((size_t)kSumBlocks * 5);
  double tot[5] = {0, 0, 0, 0, 0};
  for (auto& p : c->patches) {
    if (!p.owned) continue;
    const void* f = p.buf[c->fmap[0]];
    cudaError_t e;
    const double dV = p.d.dx * p.d.dy * p.d.dz;
    if (c->precision == DN_FP64) {
      k_partial_sums<double><<<kSumBlocks, kSumThreads, 0, c->stream>>>((const double*)f, p.ncp, c->d_partials);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), c->d_partials, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    } else {
      // the row padding holds zero offsets: it adds nothing
      k_partial_sums_i32<<<kSumBlocks, kSumThreads, 0, c->stream>>>((const int32_t*)f, p.ncp, (long long*)c->d_partials);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaMemcpyAsync(hi.data(), c->d_partials, hi.size() * sizeof(long long), cudaMemcpyDeviceToHost, c->stream);
    }
    c->launches++;
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "conservation sums");
    for (int v = 0; v < 5; ++v) {
      double pv;
      if (c->precision == DN_FP64) {
        double ps = 0;
        for (int b = 0; b < kSumBlocks; ++b) ps += h[(size_t)b * 5 + v];
        pv = ps;
      } else {
        long long ps = 0;   // exact
        for (int b = 0; b < kSumBlocks; ++b) ps += hi[(size_t)b * 5 + v];
        pv = (double)p.nc * p.base[v] + p.quantum[v] * (double)ps;
      }
      tot[v] += pv * dV;
    }
  }
  for (int v = 0; v < 5; ++v) out[v] = tot[v];
  return read_device_error(c);
}

int dn_field_difference(dn_ctx* c, int id, int f1, int v1, int f2, int v2, double* max_norm, double* l2_norm)
{
  int s = check_whole(c, id);
  if (s) return s;
  if ((s = check_field(c, f1)) || (s = check_field(c, f2))) return s;
  if (v1 < 0 || v1 > 4 || v2 < 0 || v2 > 4) return fail(c, DN_ERR_ARG, "variable index out of range");
  if (!max_norm || !l2_norm) return DN_ERR_ARG;
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  if ((s = ensure_partials(c, (size_t)kSumBlocks * 2))) return s;
  DnPatch& p = c->patches[id];
  QParams q = qparams(p);
  if (c->precision == DN_FP64) {
    const double* a = (const double*)p.buf[c->fmap[f1]] + (size_t)v1 * p.ncp;
    const double* b = (const double*)p.buf[c->fmap[f2]] + (size_t)v2 * p.ncp;
    k_diff<double><<<kSumBlocks, kSumThreads, 0, c->stream>>>(a, b, p.ncp, q, v1, q, v2, 0, c->d_partials);
  } else {
    // the row padding holds zero offsets in every field: its differences are 0
    const int32_t* a = (const int32_t*)p.buf[c->fmap[f1]] + (size_t)v1 * p.ncp;
    const int32_t* b = (const int32_t*)p.buf[c->fmap[f2]] + (size_t)v2 * p.ncp;
    k_diff<int32_t><<<kSumBlocks, kSumThreads, 0, c->stream>>>(a, b, p.ncp, q, v1, q, v2, 1, c->d_partials);
  }
  c->launches++;
  std::vector<double> h((size_t)kSumBlocks * 2);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), c->d_partials, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "field difference");
  double mx = 0, sm = 0;
  for (int b = 0; b < kSumBlocks; ++b) {
    mx = h[(size_t)b * 2] > mx ? h[(size_t)b * 2] : mx;
    sm += h[(size_t)b * 2 + 1];
  }
  *max_norm = std::sqrt(mx);
  *l2_norm = std::sqrt(sm);
  return DN_OK;
}

int dn_flow_stats(dn_ctx* c, int id, int field, double dt, double out[3])
{
  int s = check_whole(c, id);
  if (s) return s;
  if ((s = check_field(c, field))) return s;
  if (!out) return fail(c, DN_ERR_ARG, "output pointer is NULL");
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  if ((s = ensure_partials(c, (size_t)kSumBlocks * 3))) return s;
  DnPatch& p = c->patches[id];
  QParams q = qparams(p);
  const void* f = p.buf[c->fmap[field]];
  if (c->precision == DN_FP64)
    k_flow_stats<double><<<kSumBlocks, kSumThreads, 0, c->stream>>>((const double*)f, p.ncp, p.d.nk, p.kp, q, 0, dt,
                                                                   p.d.dx, c->d_partials);
  else
    k_flow_stats<int32_t><<<kSumBlocks, kSumThreads, 0, c->stream>>>((const int32_t*)f, p.ncp, p.d.nk, p.kp, q, 1, dt,
                                                                    p.d.dx, c->d_partials);
  c->launches++;
  std::vector<double> h((size_t)kSumBlocks * 3);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), c->d_partials, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "flow statistics");
  double cfl = 0.0, rmin = 1000.0, rmax = 0.0;
  for (int b = 0; b < kSumBlocks; ++b) {
    cfl = std::max(cfl, h[(size_t)b * 3]);
    rmin = std::min(rmin, h[(size_t)b * 3 + 1]);
    rmax = std::max(rmax, h[(size_t)b * 3 + 2]);
  }
  out[0] = cfl;
  out[1] = rmin;
  out[2] = rmax;
  return read_device_error(c);
}

int dn_patch_set_bc(dn_ctx* c, int id, int side, int kind, const double* params, const double* table)
{
  int s = check_patch(c, id);
  if (s) return s;
  if (side < 0 || side > 5) return fail(c, DN_ERR_ARG, "side %d is not 0..5", side);
  DnPatch& P = c->patches[id];
  const int axis = side / 2;
  if (P.d.face[axis] == DN_FACE_PERIODIC) return fail(c, DN_ERR_ARG, "axis %d of patch %d is periodic", axis, id);
  if (kind != DN_BC_ZERO_FLUX && kind != DN_BC_FARFIELD && kind != DN_BC_SLIP && kind != DN_BC_INFLOW)
    return fail(c, DN_ERR_ARG, "unknown boundary kind %d", kind);
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  if (kind == DN_BC_FARFIELD) {
    if (!params) return fail(c, DN_ERR_ARG, "far field needs p, T, u, v, w");
    for (int q = 0; q < 5; ++q) if (!std::isfinite(params[q])) return fail(c, DN_ERR_ARG, "far-field value not finite");
    if (!(params[0] > 0) || !(params[1] > 0)) return fail(c, DN_ERR_ARG, "far-field p and T must be positive");
    // CompressibleFarfieldFlux::setFarfield stores the conservative state
    // (perfectgas.h:58-66); its wall methods convert it back (perfectgas.h:84-93)
    const double pp = params[0], T = params[1], u = params[2], v = params[3], w = params[4];
    const double R = 287.2, cv = 717.5, gamma = 1.4;
    double var[5];
    var[0] = pp / (R * T);
    var[1] = var[0] * u;
    var[2] = var[0] * v;
    var[3] = var[0] * w;
    var[4] = var[0] * (cv * T + 0.5 * (u * u + v * v + w * w));
    const double ir = 1.0 / var[0];
    const double u0 = var[1] * ir, v0 = var[2] * ir, w0 = var[3] * ir;
    const double T0 = (var[4] * ir - 0.5 * (u0 * u0 + v0 * v0 + w0 * w0)) / cv;
    const double p0 = var[0] * R * T0;
    double* f = P.wall.ff[side];
    f[0] = p0; f[1] = T0; f[2] = u0; f[3] = v0; f[4] = w0;
    f[5] = std::sqrt(gamma * R * T0);
  }
  if (P.wall.table[side]) {
    cudaStreamSynchronize(c->stream);
    cudaFree((void*)P.wall.table[side]);
    P.wall.table[side] = nullptr;
  }
  if (kind == DN_BC_INFLOW) {
    if (!table) return fail(c, DN_ERR_ARG, "inflow needs a face table");
    const size_t na = axis == 0 ? (size_t)P.d.nj * P.d.nk : (axis == 1 ? (size_t)P.d.ni * P.d.nk : (size_t)P.d.ni * P.d.nj);
    for (size_t q = 0; q < na; ++q) {
      const double* e = table + 5 * q;
      if (!(e[1] > 0) || !std::isfinite(e[1]) || !std::isfinite(e[2]) || !std::isfinite(e[3]) ||
          !std::isfinite(e[4]) || (e[0] == e[0] && !(e[0] > 0)))
        return fail(c, DN_ERR_ARG, "inflow face %zu: invalid state", q);
    }
    void* d = nullptr;
    cudaError_t e = cudaMalloc(&d, na * 5 * sizeof(double));
    if (e != cudaSuccess) return fail(c, DN_ERR_NOMEM, "cudaMalloc(inflow table)");
    e = cudaMemcpyAsync(d, table, na * 5 * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { cudaFree(d); return cuda_fail(c, e, "inflow table upload"); }
    P.wall.table[side] = static_cast<const double*>(d);
  }
  P.wall.kind[side] = kind;
  P.wall.any = 0;
  for (int q = 0; q < 6; ++q) if (P.wall.kind[q] != DN_BC_ZERO_FLUX) P.wall.any = 1;
  c->batch_dirty = true;
  c->generation++;
  return DN_OK;
}

int dn_grid_compute_dependencies(dn_ctx* c, int64_t* no_donor)
{
  NvtxRange nvtx("dn overlap set-up");
  if (!c) return DN_ERR_ARG;
  std::vector<dn::OverlapPatch> ops;
  for (const DnPatch& p : c->patches) ops.push_back(dn::overlap_patch(p.d));
  std::vector<dn::DonorTables> t;
  std::string err;
  if (!dn::build_overlap(ops, t, err)) return fail(c, DN_ERR_ARG, "%s", err.c_str());
  int64_t nd = 0;
  for (const auto& x : t) nd += x.no_donor;
  c->tables.swap(t);
  c->plan_dirty = true;
  c->ls_dirty = true;
  c->batch_dirty = true;
  c->generation++;
  if (no_donor) *no_donor = nd;
  return DN_OK;
}

int dn_patch_donor_counts(dn_ctx* c, int id, int64_t counts[4])
{
  int s = check_patch(c, id);
  if (s) return s;
  if (!counts) return fail(c, DN_ERR_ARG, "counts is NULL");
  const dn::DonorTables& t = c->tables[id];
  counts[0] = (int64_t)t.rec_unique.size();
  counts[1] = (int64_t)t.donor_patch.size();
  counts[2] = (int64_t)t.rec_concat.size();
  counts[3] = (int64_t)t.donor_idx.size();
  return DN_OK;
}

int dn_patch_get_donors(dn_ctx* c, int id, uint64_t* rec_unique, int32_t* donor_patch, int64_t* num_receivers,
                        int32_t* stride, uint64_t* rec_concat, uint64_t* donor_idx, double* weight)
{
  int s = check_patch(c, id);
  if (s) return s;
  const dn::DonorTables& t = c->tables[id];
  if ((!rec_unique && !t.rec_unique.empty()) || (!rec_concat && !t.rec_concat.empty()) ||
      (!donor_idx && !t.donor_idx.empty()) || (!weight && !t.weight.empty()) ||
      (!t.donor_patch.empty() && (!donor_patch || !num_receivers || !stride)))
    return fail(c, DN_ERR_ARG, "an output array is NULL");
  std::copy(t.rec_unique.begin(), t.rec_unique.end(), rec_unique);
  std::copy(t.donor_patch.begin(), t.donor_patch.end(), donor_patch);
  std::copy(t.num_receivers.begin(), t.num_receivers.end(), num_receivers);
  std::copy(t.stride.begin(), t.stride.end(), stride);
  std::copy(t.rec_concat.begin(), t.rec_concat.end(), rec_concat);
  std::copy(t.donor_idx.begin(), t.donor_idx.end(), donor_idx);
  std::copy(t.weight.begin(), t.weight.end(), weight);
  return DN_OK;
}

int dn_patch_set_donors(dn_ctx* c, int id, const int64_t counts[4], const uint64_t* rec_unique,
                        const int32_t* donor_patch, const int64_t* num_receivers, const int32_t* stride,
                        const uint64_t* rec_concat, const uint64_t* donor_idx, const double* weight)
{
  int s = check_patch(c, id);
  if (s) return s;
  if (!counts) return fail(c, DN_ERR_ARG, "counts is NULL");
  for (int q = 0; q < 4; ++q) if (counts[q] < 0) return fail(c, DN_ERR_ARG, "negative table size");
  if ((counts[0] && !rec_unique) || (counts[1] && (!donor_patch || !num_receivers || !stride)) ||
      (counts[2] && !rec_concat) || (counts[3] && (!donor_idx || !weight)))
    return fail(c, DN_ERR_ARG, "a table array is NULL");
  const size_t nc = c->patches[id].nc;
  dn::DonorTables t;
  t.rec_unique.assign(rec_unique, rec_unique + counts[0]);
  for (size_t u = 0; u < t.rec_unique.size(); ++u) {
    if (t.rec_unique[u] >= nc || (u > 0 && t.rec_unique[u] <= t.rec_unique[u - 1]))
      return fail(c, DN_ERR_ARG, "receiving cells must be ascending cell indices of the patch");
  }
  int64_t nrec = 0, nwi = 0;
  for (int64_t q = 0; q < counts[1]; ++q) {
    if (donor_patch[q] < 0 || donor_patch[q] >= (int)c->patches.size() || donor_patch[q] == id)
      return fail(c, DN_ERR_ARG, "donor %lld: invalid donor patch %d", (long long)q, donor_patch[q]);
    if (num_receivers[q] < 0 || stride[q] < 1) return fail(c, DN_ERR_ARG, "donor %lld: invalid size", (long long)q);
    nrec += num_receivers[q];
    nwi += num_receivers[q] * stride[q];
  }
  if (nrec != counts[2] || nwi != counts[3]) return fail(c, DN_ERR_ARG, "table sizes do not add up");
  t.donor_patch.assign(donor_patch, donor_patch + counts[1]);
  t.num_receivers.assign(num_receivers, num_receivers + counts[1]);
  t.stride.assign(stride, stride + counts[1]);
  t.rec_concat.assign(rec_concat, rec_concat + counts[2]);
  for (uint64_t cell : t.rec_concat) {
    if (!std::binary_search(t.rec_unique.begin(), t.rec_unique.end(), cell))
      return fail(c, DN_ERR_ARG, "concatenated receiving cell %llu is not a receiving cell", (unsigned long long)cell);
  }
  t.donor_idx.assign(donor_idx, donor_idx + counts[3]);
  t.weight.assign(weight, weight + counts[3]);
  int64_t off = 0;
  for (int64_t q = 0; q < counts[1]; ++q) {
    const size_t ncd = c->patches[donor_patch[q]].nc;
    for (int64_t e = 0; e < num_receivers[q] * stride[q]; ++e) {
      if (t.donor_idx[(size_t)(off + e)] >= ncd) return fail(c, DN_ERR_ARG, "donor cell index out of range");
      if (!std::isfinite(t.weight[(size_t)(off + e)])) return fail(c, DN_ERR_ARG, "donor weight not finite");
    }
    off += num_receivers[q] * stride[q];
  }
  c->tables[id] = std::move(t);
  c->plan_dirty = true;
  c->ls_dirty = true;
  c->batch_dirty = true;
  c->generation++;
  return DN_OK;
}

int dn_patch_set_levelset(dn_ctx* c, int id, const double* G, int num_inner_layers, int num_outer_layers,
                          double min_inner_rel_dist)
{
  int s = (G ? check_whole : check_patch)(c, id);
  if (s) return s;
  if (!G) {
    c->ls_on[id] = 0;
    c->ls[id] = dn::LevelSetLayers();
    c->ls_dirty = true;
    c->generation++;
    return DN_OK;
  }
  if (!(min_inner_rel_dist <= 0) && !std::isfinite(min_inner_rel_dist))
    return fail(c, DN_ERR_ARG, "min_inner_rel_dist must be finite");
  for (size_t l = 0; l < c->patches[id].nc; ++l)
    if (!std::isfinite(G[l])) return fail(c, DN_ERR_ARG, "level-set value of cell %zu is not finite", l);
  dn::LevelSetLayers L;
  std::string err;
  if (!dn::classify_levelset(dn::overlap_patch(c->patches[id].d), G, num_inner_layers, num_outer_layers,
                             min_inner_rel_dist, L, err))
    return fail(c, DN_ERR_ARG, "%s", err.c_str());
  c->ls[id] = std::move(L);
  c->ls_on[id] = 1;
  c->lsg_on[id] = 0;
  c->lsg[id] = dn::LevelSetGpu();
  c->ls_dirty = true;
  c->generation++;
  return DN_OK;
}

int dn_patch_set_levelset_layers(dn_ctx* c, int id, int num_inner_layers, const int64_t* counts,
                                 const uint64_t* cells, const double* g, const double* grad, const uint64_t* donors,
                                 const double* weights)
{
  int s = (num_inner_layers > 0 ? check_whole : check_patch)(c, id);
  if (s) return s;
  if (num_inner_layers < 0 || (num_inner_layers > 0 && !counts)) return fail(c, DN_ERR_ARG, "invalid layer counts");
  int64_t total = 0;
  for (int l = 0; l < num_inner_layers; ++l) {
    if (counts[l] < 0) return fail(c, DN_ERR_ARG, "negative layer count");
    total += counts[l];
  }
  if (total > 0 && !(cells && g && grad && donors && weights)) return fail(c, DN_ERR_ARG, "layer arrays missing");
  const uint64_t nc = c->patches[id].nc;
  dn::LevelSetLayers L;
  L.inner.resize(num_inner_layers);
  int64_t q = 0;
  for (int l = 0; l < num_inner_layers; ++l) {
    for (int64_t e = 0; e < counts[l]; ++e, ++q) {
      dn::LayerCell lc;
      lc.cell = cells[q];
      lc.g = g[q];
      for (int a = 0; a < 3; ++a) lc.grad[a] = grad[3 * q + a];
      for (int t = 0; t < 8; ++t) {
        lc.donor[t] = donors[8 * q + t];
        lc.weight[t] = weights[8 * q + t];
        if (lc.donor[t] >= nc) return fail(c, DN_ERR_ARG, "mirror donor %llu outside patch %d",
                                           (unsigned long long)lc.donor[t], id);
      }
      if (lc.cell >= nc) return fail(c, DN_ERR_ARG, "layer cell %llu outside patch %d", (unsigned long long)lc.cell, id);
      L.inner[l].push_back(lc);
    }
  }
  c->ls[id] = std::move(L);
  c->ls_on[id] = num_inner_layers > 0 ? 1 : 0;
  c->ls_dirty = true;
  c->generation++;
  return DN_OK;
}

int dn_patch_set_levelset_gpu(dn_ctx* c, int id, const double* G)
{
  int s = (G ? check_whole : check_patch)(c, id);
  if (s) return s;
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  DnPatch& P = c->patches[id];
  if (!G) {
    c->lsg_on[id] = 0;
    c->lsg[id] = dn::LevelSetGpu();
    c->ls_dirty = true;
    c->generation++;
    return DN_OK;
  }
  for (size_t l = 0; l < P.nc; ++l)
    if (!std::isfinite(G[l])) return fail(c, DN_ERR_ARG, "level-set value of cell %zu is not finite", l);
  dn::LevelSetGpu L;
  std::string err;
  if (!dn::classify_levelset_gpu(dn::overlap_patch(P.d), G, L, err)) return fail(c, DN_ERR_ARG, "%s", err.c_str());
  // deactivate the G < 0 cells (GPU_CartesianLevelSetBC's constructor),
  // keeping cells the patch's mask already deactivated
  std::vector<uint8_t> mask(P.nc, 1);
  if (P.active) {
    std::vector<uint8_t> dev(P.ncp);
    cudaError_t e = cudaMemcpyAsync(dev.data(), P.active, P.ncp, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "active mask download");
    for (size_t l = 0; l < P.nc; ++l) mask[l] = dev[pad_cell(P, l)];
  }
  for (uint64_t l : L.below) mask[l] = 0;
  if ((s = dn_patch_set_active(c, id, mask.data()))) return s;
  c->lsg[id] = std::move(L);
  c->lsg_on[id] = 1;
  c->ls_on[id] = 0;
  c->ls[id] = dn::LevelSetLayers();
  c->ls_dirty = true;
  c->generation++;
  return DN_OK;
}

int dn_patch_levelset_gpu_counts(dn_ctx* c, int id, int64_t counts[3])
{
  int s = check_patch(c, id);
  if (s) return s;
  if (!counts) return fail(c, DN_ERR_ARG, "counts is NULL");
  counts[0] = (int64_t)c->lsg[id].below.size();
  counts[1] = (int64_t)c->lsg[id].inside.size();
  int64_t nb = 0;
  for (const auto& ic : c->lsg[id].inside) nb += (int64_t)ic.nbr.size();
  counts[2] = nb;
  return DN_OK;
}

int dn_patch_levelset_count(dn_ctx* c, int id, int inner, int layer, int64_t* n)
{
  int s = check_patch(c, id);
  if (s) return s;
  if (!n) return fail(c, DN_ERR_ARG, "n is NULL");
  const auto& lists = inner ? c->ls[id].inner : c->ls[id].outer;
  if (layer < 0 || layer >= (int)lists.size()) return fail(c, DN_ERR_ARG, "layer %d does not exist", layer);
  *n = (int64_t)lists[layer].size();
  return DN_OK;
}

int dn_patch_levelset_get(dn_ctx* c, int id, int inner, int layer, uint64_t* cells, double* g, double* grad,
                          uint64_t* donors, double* weights)
{
  int s = check_patch(c, id);
  if (s) return s;
  const auto& lists = inner ? c->ls[id].inner : c->ls[id].outer;
  if (layer < 0 || layer >= (int)lists.size()) return fail(c, DN_ERR_ARG, "layer %d does not exist", layer);
  size_t q = 0;
  for (const dn::LayerCell& lc : lists[layer]) {
    if (cells) cells[q] = lc.cell;
    if (g) g[q] = lc.g;
    for (int a = 0; a < 3; ++a) if (grad) grad[3 * q + a] = lc.grad[a];
    for (int t = 0; t < 8; ++t) {
      if (donors) donors[8 * q + t] = lc.donor[t];
      if (weights) weights[8 * q + t] = lc.weight[t];
    }
    ++q;
  }
  return DN_OK;
}

int dn_apply_levelset_bc(dn_ctx* c, int field)
{
  if (!c) return DN_ERR_ARG;
  int s;
  if ((s = check_field(c, field))) return s;
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  return levelset_bc(c, c->fmap[field], c->fmap[1]);
}

int dn_copy_donor_data(dn_ctx* c, int field)
{
  if (!c) return DN_ERR_ARG;
  int s;
  if ((s = check_field(c, field))) return s;
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  return donor_copy(c, c->fmap[field]);
}

int dn_set_option(dn_ctx* c, int option, int value)
{
  if (!c) return DN_ERR_ARG;
  if (option == DN_OPT_BATCHED) {
    c->batched = value != 0;
    c->generation++;
    return DN_OK;
  }
  if (option == DN_OPT_GRAPH) {
    c->use_graph = value != 0;
    return DN_OK;
  }
  if (option == DN_OPT_BATCH_WAVES || option == DN_OPT_BATCH_MIN_PLANES) {
    if (value < (option == DN_OPT_BATCH_WAVES ? 0 : 1) || value > 64)
      return fail(c, DN_ERR_ARG, "schedule option %d out of range: %d", option, value);
    (option == DN_OPT_BATCH_WAVES ? c->batch_waves : c->batch_min_planes) = value;
    c->batch_dirty = true;
    c->generation++;
    return DN_OK;
  }
  if (option == DN_OPT_DONOR_TABLES) {
    if (value < 0 || value > 1) return fail(c, DN_ERR_ARG, "donor table option out of range: %d", value);
    c->donor_wide = value == 1;
    c->plan_dirty = true;
    c->generation++;
    return DN_OK;
  }
  return fail(c, DN_ERR_ARG, "unknown option %d", option);
}

int dn_patch_set_owned(dn_ctx* c, int id, int owned)
{
  int s = check_patch(c, id);
  if (s) return s;
  if (c->patches[id].compact) {
    if (owned) return fail(c, DN_ERR_STATE, "patch %d is a compact shadow and stays another rank's", id);
    return DN_OK;
  }
  c->patches[id].owned = owned != 0;
  c->plan_dirty = true;
  c->ls_dirty = true;
  c->batch_dirty = true;
  c->generation++;
  return DN_OK;
}

int dn_exchange_build_ctx(dn_ctx* c, const int32_t* owner, int rank, int world, dn_exchange** out)
{
  if (!c || !owner || !out) return DN_ERR_ARG;
  *out = nullptr;
  std::vector<dn::DonorTables> tables(c->tables);
  tables.resize(c->patches.size());
  dn_exchange* e = new dn_exchange();
  std::string err;
  if (!dn::build_exchange(tables, owner, rank, world, e->ex, err)) {
    delete e;
    return fail(c, DN_ERR_ARG, "%s", err.c_str());
  }
  *out = e;
  return DN_OK;
}

int dn_shadow_alloc(dn_ctx* c, dn_exchange* e)
{
  if (!c || !e) return DN_ERR_ARG;
  const dn::Exchange& x = e->ex;
  if (x.device >= 0)
    return fail(c, DN_ERR_STATE, "allocate the shadows before the exchange's first pack or unpack");
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  // the cells each compact shadow receives, over all peers
  std::vector<std::vector<uint64_t>> held(c->patches.size());
  for (int q = 0; q < x.world; ++q) {
    for (size_t t = 0; t < x.recv_patch[q].size(); ++t) {
      const int32_t p = x.recv_patch[q][t];
      if (p < 0 || p >= (int)c->patches.size()) return fail(c, DN_ERR_ARG, "exchange names patch %d", p);
      held[(size_t)p].push_back(x.recv_cell[q][t]);
    }
  }
  for (size_t p = 0; p < c->patches.size(); ++p) {
    DnPatch& P = c->patches[p];
    if (!P.compact) continue;
    std::vector<uint64_t>& h = held[p];
    std::sort(h.begin(), h.end());
    h.erase(std::unique(h.begin(), h.end()), h.end());
    if (!h.empty() && h.back() >= P.nc) return fail(c, DN_ERR_ARG, "exchange cell outside patch %zu", p);
    for (int b = 0; b < 3; ++b) {
      if (P.buf[b]) cudaFree(P.buf[b]);
      P.buf[b] = nullptr;
    }
    P.held.swap(h);
    P.ncp = P.held.size();
    const size_t bytes = 5 * P.ncp * elem_size(c);
    for (int b = 0; b < 3 && bytes; ++b) {
      cudaError_t er = cudaMalloc(&P.buf[b], bytes);
      if (er != cudaSuccess) return fail(c, DN_ERR_NOMEM, "cudaMalloc of %zu bytes for a shadow field failed", bytes);
      er = cudaMemsetAsync(P.buf[b], 0, bytes, c->stream);
      if (er != cudaSuccess) return cuda_fail(c, er, "shadow field clear");
    }
  }
  c->plan_dirty = true;
  c->ls_dirty = true;
  c->batch_dirty = true;
  c->generation++;
  return DN_OK;
}

int dn_exchange_destroy(dn_exchange* e)
{
  if (!e) return DN_OK;
  if (e->ex.device >= 0) {
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(e->ex.device);
    for (void* p : e->ex.dev) cudaFree(p);
    cudaSetDevice(cur);
  }
  delete e;
  return DN_OK;
}

namespace {

// device copies of the exchange lists: [peer][send_patch, send_cell, recv_patch, recv_cell]
int exchange_device_lists(dn_ctx* c, dn_exchange* e)
{
  dn::Exchange& x = e->ex;
  if (x.device >= 0) {
    if (x.device != c->device) return fail(c, DN_ERR_ARG, "exchange lists live on device %d, context on %d", x.device, c->device);
    return DN_OK;
  }
  for (int q = 0; q < x.world; ++q) {
    for (size_t t = 0; t < x.send_patch[q].size(); ++t)
      if (c->patches[(size_t)x.send_patch[q][t]].compact)
        return fail(c, DN_ERR_STATE, "the exchange sends from patch %d, a compact shadow of this context",
                    x.send_patch[q][t]);
  }
  // cells at their device offsets (rows of kp elements; held positions in
  // compact shadows)
  std::vector<std::vector<uint64_t>> sc(x.world), rc(x.world);
  for (int q = 0; q < x.world; ++q) {
    sc[q].resize(x.send_cell[q].size());
    rc[q].resize(x.recv_cell[q].size());
    for (size_t t = 0; t < sc[q].size(); ++t)
      sc[q][t] = pad_cell(c->patches[(size_t)x.send_patch[q][t]], x.send_cell[q][t]);
    for (size_t t = 0; t < rc[q].size(); ++t) {
      if (!dev_cell(c->patches[(size_t)x.recv_patch[q][t]], x.recv_cell[q][t], &rc[q][t]))
        return fail(c, DN_ERR_STATE, "cell %llu of patch %d is received but not held by its compact shadow "
                    "(dn_shadow_alloc with this exchange first)", (unsigned long long)x.recv_cell[q][t],
                    x.recv_patch[q][t]);
    }
  }
  x.dev.assign((size_t)x.world * 4, nullptr);
  x.device = c->device;
  for (int q = 0; q < x.world; ++q) {
    const void* src[4] = {x.send_patch[q].data(), sc[q].data(), x.recv_patch[q].data(), rc[q].data()};
    const size_t bytes[4] = {x.send_patch[q].size() * 4, x.send_cell[q].size() * 8, x.recv_patch[q].size() * 4,
                             x.recv_cell[q].size() * 8};
    for (int a = 0; a < 4; ++a) {
      if (!bytes[a]) continue;
      void* d = nullptr;
      if (cudaMalloc(&d, bytes[a]) != cudaSuccess) return fail(c, DN_ERR_NOMEM, "cudaMalloc(exchange lists)");
      x.dev[(size_t)q * 4 + a] = d;
      cudaError_t er = cudaMemcpy(d, src[a], bytes[a], cudaMemcpyHostToDevice);
      if (er != cudaSuccess) return cuda_fail(c, er, "exchange list upload");
    }
  }
  return DN_OK;
}

int exchange_move(dn_ctx* c, dn_exchange* e, int field, int peer, void* buf, bool pack)
{
  NvtxRange nvtx("dn exchange");
  if (!c || !e) return DN_ERR_ARG;
  int s;
  if (field == DN_FIELD_DONOR_COPY) {
    if (c->exch_phys < 0) return fail(c, DN_ERR_STATE, "DN_FIELD_DONOR_COPY is valid only inside the exchange hook");
  } else if ((s = check_field(c, field))) {
    return s;
  }
  if (peer < 0 || peer >= e->ex.world || peer == e->ex.rank) return fail(c, DN_ERR_ARG, "peer %d is not another rank", peer);
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  if (c->plan_dirty && (s = build_plan(c))) return s;
  if ((s = exchange_device_lists(c, e))) return s;
  const dn::Exchange& x = e->ex;
  const int64_t n = (int64_t)(pack ? x.send_cell[peer].size() : x.recv_cell[peer].size());
  if (n == 0) return DN_OK;
  if (!buf) return fail(c, DN_ERR_ARG, "exchange buffer is NULL");
  const int32_t* patch = static_cast<const int32_t*>(x.dev[(size_t)peer * 4 + (pack ? 0 : 2)]);
  const uint64_t* cell = static_cast<const uint64_t*>(x.dev[(size_t)peer * 4 + (pack ? 1 : 3)]);
  void* const* bufs = c->plan.bufs;
  const int phys = field == DN_FIELD_DONOR_COPY ? c->exch_phys : c->fmap[field];
  if (!pack) donor_stale(c, phys);
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)c->num_sms * 8);
  if (c->precision == DN_FP64) {
    if (pack) k_exchange_pack<double><<<blocks, 256, 0, c->stream>>>(bufs, c->plan.nc, phys, patch, cell, n, (double*)buf);
    else k_exchange_unpack<double><<<blocks, 256, 0, c->stream>>>(bufs, c->plan.nc, phys, patch, cell, n, (const double*)buf);
  } else {
    if (pack) k_exchange_pack<int32_t><<<blocks, 256, 0, c->stream>>>(bufs, c->plan.nc, phys, patch, cell, n, (int32_t*)buf);
    else k_exchange_unpack<int32_t><<<blocks, 256, 0, c->stream>>>(bufs, c->plan.nc, phys, patch, cell, n, (const int32_t*)buf);
  }
  c->launches++;
  cudaError_t er = cudaGetLastError();
  if (er != cudaSuccess) return cuda_fail(c, er, pack ? "exchange pack" : "exchange unpack");
  return DN_OK;
}

} // namespace

int dn_exchange_pack(dn_ctx* c, dn_exchange* e, int field, int peer, void* buf)
{
  return exchange_move(c, e, field, peer, buf, true);
}

int dn_exchange_unpack(dn_ctx* c, dn_exchange* e, int field, int peer, const void* buf)
{
  return exchange_move(c, e, field, peer, const_cast<void*>(buf), false);
}

int dn_write_data(dn_ctx* c, int field, const char* base, double time, int count)
{
  if (!c) return DN_ERR_ARG;
  if (!base) return fail(c, DN_ERR_ARG, "base file name is NULL");
  int s;
  if ((s = check_field(c, field))) return s;
  std::string bytes;
  dn::dnd_header(bytes, 8, time);
  std::vector<double> h;
  for (size_t q = 0; q < c->patches.size(); ++q) {
    h.resize(5 * c->patches[q].nc);
    if ((s = download_impl(c, (int)q, field, h.data()))) return s;
    dn::dnd_values(bytes, 8, h.data(), h.size());
  }
  const std::string name = dn::dnd_file_name(base, count);
  if (!dn::dnd_write_file(name, bytes)) return fail(c, DN_ERR_ARG, "cannot write %s", name.c_str());
  return DN_OK;
}

int dn_read_data(dn_ctx* c, int field, const char* file_name, double* time)
{
  if (!c) return DN_ERR_ARG;
  if (!file_name) return fail(c, DN_ERR_ARG, "file name is NULL");
  int s;
  if ((s = check_field(c, field))) return s;
  std::string name(file_name);
  if (name.size() < 4 || name.compare(name.size() - 4, 4, ".dnd") != 0) name += ".dnd";
  std::string bytes;
  if (!dn::dnd_read_file(name, bytes)) return fail(c, DN_ERR_ARG, "cannot read %s", name.c_str());
  int prec;
  double t;
  size_t off;
  if (!dn::dnd_parse_header(bytes, &prec, &t, &off)) return fail(c, DN_ERR_ARG, "%s: truncated header", name.c_str());
  size_t total = 0;
  for (auto& p : c->patches) total += 5 * p.nc;
  if (bytes.size() != off + total * (size_t)prec)
    return fail(c, DN_ERR_ARG, "%s holds %zu bytes of values, the context's patches need %zu", name.c_str(),
                bytes.size() - off, total * (size_t)prec);
  std::vector<double> h;
  for (size_t q = 0; q < c->patches.size(); ++q) {
    h.resize(5 * c->patches[q].nc);
    dn::dnd_get_values(bytes, off, prec, h.data(), h.size());
    off += h.size() * (size_t)prec;
    if ((s = upload_impl(c, (int)q, field, h.data()))) return s;
  }
  if (time) *time = t;
  return DN_OK;
}

int dn_set_flux_scheme(dn_ctx* c, int scheme)
{
  if (!c) return DN_ERR_ARG;
  if (scheme < DN_FLUX_AUSMPLUS || scheme > DN_FLUX_ROE) return fail(c, DN_ERR_ARG, "unknown flux scheme %d", scheme);
  if (scheme != DN_FLUX_AUSMPLUS && c->precision != DN_FP64)
    return fail(c, DN_ERR_ARG, "flux scheme %d needs an FP64 context (FP32 runs AUSM+ only)", scheme);
  c->scheme = scheme;
  c->generation++;
  return DN_OK;
}

int dn_set_exchange_hook(dn_ctx* c, dn_exchange_fn fn, void* user)
{
  if (!c) return DN_ERR_ARG;
  c->exch_fn = fn;
  c->exch_user = user;
  c->generation++;
  return DN_OK;
}

int dn_set_stage_function(dn_ctx* c, dn_stage_fn fn, void* user)
{
  if (!c) return DN_ERR_ARG;
  if (fn && c->precision != DN_FP64) return fail(c, DN_ERR_ARG, "user stage functions need an FP64 context");
  c->stage_fn = fn;
  c->stage_user = user;
  c->generation++;
  return DN_OK;
}

int dn_patch_set_tile(dn_ctx* c, int id, int shape)
{
  int s = check_patch(c, id);
  if (s) return s;
  if (shape < 0 || shape >= dn::kNumShapes) return fail(c, DN_ERR_ARG, "tile shape %d is not 0..%d", shape, dn::kNumShapes - 1);
  c->shape[id] = shape;
  c->batch_dirty = true;
  c->generation++;
  return DN_OK;
}

namespace {

// padded cells a patch occupies with tile shape `shape`
double padded_cells(const dn_ctx* c, const DnPatch& p, int shape)
{
  std::vector<TileRef> t;
  patch_tiles(c, p, shape, t);
  double cells = 0;
  for (const TileRef& r : t) {
    int tj, tk;
    dn::shape_tile(c->precision == DN_FP64, r.shape, &tj, &tk);
    cells += (double)tj * (double)tk;
  }
  return (double)p.d.ni * cells;
}

std::string device_name(int dev)
{
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return "unknown";
  return prop.name;
}

// cache lines: "<device>|<precision>|<shapes>|<cost shape 0>|<cost shape 1>|..."
bool read_tune_cache(const char* path, const std::string& dev, int precision, double cost[dn::kNumShapes])
{
  if (!path) return false;
  FILE* f = std::fopen(path, "r");
  if (!f) return false;
  char line[1024];
  bool found = false;
  while (std::fgets(line, sizeof line, f)) {
    char name[256];
    int prec, ns, pos = 0;
    if (std::sscanf(line, "%255[^|]|%d|%d%n", name, &prec, &ns, &pos) != 3 || dev != name || prec != precision ||
        ns != dn::kNumShapes)
      continue;
    double c[dn::kNumShapes];
    const char* q = line + pos;
    int got = 0;
    for (int k = 0; k < dn::kNumShapes; ++k) {
      int m = 0;
      if (std::sscanf(q, "|%lf%n", &c[k], &m) != 1) break;
      q += m;
      ++got;
    }
    if (got != dn::kNumShapes) continue;
    for (int k = 0; k < dn::kNumShapes; ++k) cost[k] = c[k];
    found = true;
  }
  std::fclose(f);
  return found;
}

void write_tune_cache(const char* path, const std::string& dev, int precision, const double cost[dn::kNumShapes])
{
  if (!path) return;
  FILE* f = std::fopen(path, "a");
  if (!f) return;
  std::fprintf(f, "%s|%d|%d", dev.c_str(), precision, dn::kNumShapes);
  for (int k = 0; k < dn::kNumShapes; ++k) std::fprintf(f, "|%.17g", cost[k]);
  std::fprintf(f, "\n");
  std::fclose(f);
}

} // namespace

int dn_autotune(dn_ctx* c, const char* cache_path, double cost_out[DN_NUM_TILE_SHAPES])
{
  NvtxRange nvtx("dn autotune");
  if (!c) return DN_ERR_ARG;
  if (c->patches.empty()) return fail(c, DN_ERR_STATE, "no patches to tune for");
  if (set_device(c) != DN_OK) return DN_ERR_CUDA;
  donor_stale(c, -1);
  const std::string dev = device_name(c->device);
  static_assert(DN_NUM_TILE_SHAPES == dn::kNumShapes, "tile shape count");
  double cost[dn::kNumShapes] = {};
  if (!read_tune_cache(cache_path, dev, c->precision, cost)) {
    // measure each tile shape on the case itself: one stage of every patch
    // into the scratch field (field 2), factor 0
    const std::vector<int> saved = c->shape;
    const bool saved_batched = c->batched;
    c->batched = true;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int st = DN_OK;
    for (int sh = 0; sh < dn::kNumShapes && st == DN_OK; ++sh) {
      double padded = 0;
      for (size_t q = 0; q < c->patches.size(); ++q) {
        c->shape[q] = sh;
        if (c->patches[q].owned && c->patches[q].patch_active) padded += padded_cells(c, c->patches[q], sh);
      }
      c->batch_dirty = true;
      const int reps = 5;
      for (int r = 0; r < 2 + reps && st == DN_OK; ++r) {
        if (r == 2) cudaEventRecord(e0, c->stream);
        st = stage_all(c, c->fmap[0], c->fmap[1], c->fmap[2], 0.0);
      }
      cudaEventRecord(e1, c->stream);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      cost[sh] = (double)ms * 1e6 / reps / padded;      // ns per padded cell and stage
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->batched = saved_batched;
    c->shape = saved;
    if (st != DN_OK) { c->batch_dirty = true; c->generation++; return st; }
    int s2 = read_device_error(c);
    if (s2 != DN_OK) return s2;
    write_tune_cache(cache_path, dev, c->precision, cost);
  }
  // FX32 stages that run the single-patch kernel (one patch, or batching
  // off): the plane-chunk length of its CTAs, measured among a few
  // candidates on the patch itself (one stage into the scratch field,
  // factor 0; the chunking changes no result)
  if (c->precision == DN_FP32 && (c->patches.size() == 1 || !c->batched)) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (size_t q = 0; q < c->patches.size(); ++q) {
      DnPatch& P = c->patches[q];
      if (!P.owned) continue;
      int tj, tk;
      dn::fx32_tile(&tj, &tk);
      const int def = dn::default_i_chunk(P.d.ni, P.d.nj, P.d.nk, tj, tk, c->num_sms, DN_FX_WAVE_CTAS);
      const int cand[6] = {def, 16, 24, 32, 48, 64};
      int best = def;
      double best_ms = 1e300;
      for (int k = 0; k < 6; ++k) {
        if (cand[k] > P.d.ni || (k > 0 && cand[k] == def)) continue;
        P.i_chunk = cand[k];
        int st = DN_OK;
        for (int r = 0; r < 7 && st == DN_OK; ++r) {
          if (r == 2) cudaEventRecord(e0, c->stream);
          st = stage_patch(c, P, c->fmap[0], c->fmap[1], c->fmap[2], 0.0);
        }
        cudaEventRecord(e1, c->stream);
        cudaEventSynchronize(e1);
        if (st != DN_OK) { P.i_chunk = 0; cudaEventDestroy(e0); cudaEventDestroy(e1); return st; }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) { best_ms = ms; best = cand[k]; }
      }
      P.i_chunk = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int s3 = read_device_error(c);
    if (s3 != DN_OK) return s3;
  }
  for (size_t q = 0; q < c->patches.size(); ++q) {
    int best = 0;
    double best_t = cost[0] * padded_cells(c, c->patches[q], 0);
    for (int sh = 1; sh < dn::kNumShapes; ++sh) {
      const double t = cost[sh] * padded_cells(c, c->patches[q], sh);
      if (t < best_t) { best_t = t; best = sh; }
    }
    c->shape[q] = best;
  }
  c->batch_dirty = true;
  c->generation++;
  // batched stages: the schedule of the work items, measured among a few
  // candidates with the shapes just chosen (one stage of every patch into
  // the scratch field, factor 0; the schedule changes no result): FP64 the
  // shortest plane range of an item; FX32 that, or instead the waves of
  // persistent CTAs (fewer waves save prologues, more let the hardware even
  // out tiles of unequal cost, one CTA per item keeps neighbouring columns
  // on the same planes at the same time)
  if (c->batched && c->patches.size() > 1) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const bool fp64 = c->precision == DN_FP64;
    // (waves, shortest item): persistent waves for FP32 bulk, or one CTA per item
    const int cand64[5][2] = {{0, 8}, {0, 16}, {0, 24}, {0, 32}, {0, 48}};
    const int cand32[8][2] = {{0, 8}, {0, 16}, {0, 24}, {0, 32}, {0, 48}, {1, 8}, {2, 8}, {4, 8}};
    const int n_cand = fp64 ? 5 : 8;
    int best_w = c->batch_waves, best_p = c->batch_min_planes;
    double best_ms = 1e300;
    int st = DN_OK;
    for (int k = 0; k < n_cand && st == DN_OK; ++k) {
      c->batch_waves = fp64 ? cand64[k][0] : cand32[k][0];
      c->batch_min_planes = fp64 ? cand64[k][1] : cand32[k][1];
      c->batch_dirty = true;
      for (int r = 0; r < 5 && st == DN_OK; ++r) {
        if (r == 2) cudaEventRecord(e0, c->stream);
        st = stage_all(c, c->fmap[0], c->fmap[1], c->fmap[2], 0.0);
      }
      cudaEventRecord(e1, c->stream);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (st == DN_OK && ms < best_ms) { best_ms = ms; best_w = c->batch_waves; best_p = c->batch_min_planes; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->batch_waves = best_w;
    c->batch_min_planes = best_p;
    c->batch_dirty = true;
    c->generation++;
    if (st != DN_OK) return st;
    int s4 = read_device_error(c);
    if (s4 != DN_OK) return s4;
  }
  if (cost_out) {
    for (int k = 0; k < dn::kNumShapes; ++k) cost_out[k] = cost[k];
  }
  return DN_OK;
}

int dn_launch_count(const dn_ctx* c, int64_t* count)
{
  if (!c || !count) return DN_ERR_ARG;
  *count = c->launches;
  return DN_OK;
}

int dn_tma_patch_count(dn_ctx* c, int64_t* count)
{
  if (!c || !count) return DN_ERR_ARG;
  int64_t n = 0;
  for (const DnPatch& P : c->patches) {
    if (P.compact) continue;
    int tj, tk;
    dn::shape_tile(c->precision == DN_FP64, 0, &tj, &tk);
    bool ok;
    if (c->precision == DN_FP64) {
      CUtensorMap m;
      ok = dn::encode_stage_map_f64(&m, (const double*)P.buf[0], P.d.ni, P.d.nj, P.d.nk, tj, tk);
    } else {
      dn::FxGeom g{};
      g.ni = P.d.ni; g.nj = P.d.nj; g.nk = P.d.nk; g.kp = P.kp;
      CUtensorMap mi[dn::kFxMaps], mu;
      ok = dn::encode_stage_maps(mi, &mu, (const int32_t*)P.buf[0], (const int32_t*)P.buf[0], g, tj, tk);
    }
    n += ok ? 1 : 0;
  }
  *count = n;
  return DN_OK;
}

} // extern "C"
