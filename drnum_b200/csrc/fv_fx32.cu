// FX32 (FP32 bulk, fixed-point storage) stage kernel instantiation.
#include "fv_launch.h"
#include "fv_fx32.cuh"
#include "fv_batch.cuh"

namespace dn {

namespace {
#ifndef DN_FX_TJ
#define DN_FX_TJ 16
#endif
#ifndef DN_FX_TK
#define DN_FX_TK 16
#endif
constexpr int FX_TJ = DN_FX_TJ;   // tile of the single-patch launch (j x k)
constexpr int FX_TK = DN_FX_TK;
}

cudaError_t launch_stage_fx32(const FxArgs& a, cudaStream_t st)
{
  using Smem = FxSmem<FX_TJ, FX_TK>;
  auto kern = fx_stage_kernel<FX_TJ, FX_TK>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
  if (e != cudaSuccess) return e;
  dim3 block(FX_TK, FX_TJ, 1);
  dim3 grid((a.g.nk + FX_TK - 1) / FX_TK, (a.g.nj + FX_TJ - 1) / FX_TJ,
            (a.g.ni + a.g.i_chunk - 1) / a.g.i_chunk);
  kern<<<grid, block, sizeof(Smem), st>>>(a);
  return cudaGetLastError();
}

void fx32_tile(int* tj, int* tk) { *tj = FX_TJ; *tk = FX_TK; }

namespace {
template <int TJ, int TK>
cudaError_t launch_fx_batched(const Batch& b, cudaStream_t st)
{
  using Smem = FxSmem<TJ, TK>;
  auto kern = fx_stage_batched<TJ, TK>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
  if (e != cudaSuccess) return e;
  kern<<<b.n_items, dim3(TK, TJ, 1), sizeof(Smem), st>>>(b);
  return cudaGetLastError();
}
} // namespace

cudaError_t launch_stage_fx32_batched(const Batch& b, int shape, cudaStream_t st)
{
  if (b.n_items <= 0) return cudaSuccess;
  return shape == 0 ? launch_fx_batched<8, 32>(b, st) : launch_fx_batched<16, 16>(b, st);
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
