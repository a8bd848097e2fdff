// FP64 stage kernel instantiation.  Built with -fmad=false: together with the
// operation order of fv_numerics.cuh this reproduces the reference CPU
// iterator (compiled with -ffp-contract=off) bit for bit.
#include "fv_launch.h"

namespace dn {

namespace {
constexpr int F64_TJ = 4;
constexpr int F64_TK = 32;
}

cudaError_t launch_stage_f64(const StageArgs<PolicyF64>& a, const StageShape& s, cudaStream_t st)
{
  using Smem = StageSmem<PolicyF64, F64_TJ, F64_TK>;
  auto kern = fv_stage_kernel<PolicyF64, F64_TJ, F64_TK>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
  if (e != cudaSuccess) return e;
  (void)s;
  dim3 block(F64_TK, F64_TJ, 1);
  dim3 grid((a.g.nk + F64_TK - 1) / F64_TK, (a.g.nj + F64_TJ - 1) / F64_TJ,
            (a.g.ni + a.g.i_chunk - 1) / a.g.i_chunk);
  kern<<<grid, block, sizeof(Smem), st>>>(a);
  return cudaGetLastError();
}

} // namespace dn
