// FP64 stage kernel instantiation.  Built with -fmad=false: together with the
// operation order of fv_numerics.cuh this reproduces the reference CPU
// iterator (compiled with -ffp-contract=off) bit for bit.
#include <cstring>
#include "fv_launch.h"
#include "fv_tma_host.h"
#include "fv_batch.cuh"

namespace dn {

namespace {
constexpr int F64_TJ = 4;
constexpr int F64_TK = 32;
}

bool encode_stage_map_f64(CUtensorMap* tm, const double* in, int ni, int nj, int nk, int tj, int tk)
{
  if (tma_disabled()) return false;
  return encode_patch_field_map(tm, in, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, ni, nj, nk, nk, tk + 4, tj + 4);
}

cudaError_t launch_stage_f64(const StageArgs<PolicyF64>& a, const StageShape& s, cudaStream_t st)
{
  using Smem = StageSmem<PolicyF64, F64_TJ, F64_TK>;
  auto kern = fv_stage_kernel<PolicyF64, F64_TJ, F64_TK>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
  if (e != cudaSuccess) return e;
  (void)s;
  StageLaunch<PolicyF64> L;
  std::memset(&L, 0, sizeof L);
  L.a = a;
  L.tma = encode_stage_map_f64(&L.tm, a.in, a.g.ni, a.g.nj, a.g.nk, F64_TJ, F64_TK);
  dim3 block(F64_TK, F64_TJ, 1);
  dim3 grid((a.g.nk + F64_TK - 1) / F64_TK, (a.g.nj + F64_TJ - 1) / F64_TJ,
            (a.g.ni + a.g.i_chunk - 1) / a.g.i_chunk);
  kern<<<grid, block, sizeof(Smem), st>>>(L);
  return cudaGetLastError();
}

namespace {
template <int TJ, int TK>
cudaError_t launch_f64_batched(const Batch& b, cudaStream_t st)
{
  using Smem = StageSmem<PolicyF64, TJ, TK>;
  auto kern = fv_stage_batched_f64<TJ, TK>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
  if (e != cudaSuccess) return e;
  kern<<<b.n_items, dim3(TK, TJ, 1), sizeof(Smem), st>>>(b);
  return cudaGetLastError();
}
} // namespace

cudaError_t launch_stage_f64_batched(const Batch& b, int shape, cudaStream_t st)
{
  if (b.n_items <= 0) return cudaSuccess;
  if (shape == 0) return launch_f64_batched<4, 32>(b, st);
  if (shape == 1) return launch_f64_batched<8, 16>(b, st);
  return launch_f64_batched<8, 32>(b, st);
}

} // namespace dn
