// FP32 bulk stage kernel instantiation (grid-quantised offset storage).
#include "fv_launch.h"

namespace dn {

namespace {
constexpr int F32_TJ = 8;
constexpr int F32_TK = 32;
}

cudaError_t launch_stage_f32q(const StageArgs<PolicyF32Q>& a, const StageShape& s, cudaStream_t st)
{
  using Smem = StageSmem<PolicyF32Q, F32_TJ, F32_TK>;
  auto kern = fv_stage_kernel<PolicyF32Q, F32_TJ, F32_TK>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
  if (e != cudaSuccess) return e;
  (void)s;
  dim3 block(F32_TK, F32_TJ, 1);
  dim3 grid((a.g.nk + F32_TK - 1) / F32_TK, (a.g.nj + F32_TJ - 1) / F32_TJ,
            (a.g.ni + a.g.i_chunk - 1) / a.g.i_chunk);
  kern<<<grid, block, sizeof(Smem), st>>>(a);
  return cudaGetLastError();
}

int default_i_chunk(int ni, int nj, int nk, int tj, int tk, int num_sms, int ctas_per_sm)
{
  const long tiles = (long)((nj + tj - 1) / tj) * ((nk + tk - 1) / tk);
  const long want = (long)num_sms * ctas_per_sm * 4;   // about four waves
  long chunks = (want + tiles - 1) / tiles;
  if (chunks < 1) chunks = 1;
  long ic = (ni + chunks - 1) / chunks;
  if (ic < 8) ic = 8;                                   // amortise the 4-plane prologue
  if (ic > ni) ic = ni;
  return (int)ic;
}

} // namespace dn
