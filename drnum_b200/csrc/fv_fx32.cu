// FX32 (FP32 bulk, fixed-point storage) stage kernel instantiation.
#include <cstdlib>
#include <cstring>
#include "fv_launch.h"
#include "fv_tma_host.h"
#include "fv_fx32.cuh"
#include "fv_batch.cuh"

namespace dn {

namespace {
#ifndef DN_FX_TJ
#define DN_FX_TJ 16
#endif
#ifndef DN_FX_TK
#define DN_FX_TK 32
#endif
constexpr int FX_TJ = DN_FX_TJ;   // tile of the single-patch launch (j x k)
constexpr int FX_TK = DN_FX_TK;
}

namespace {

bool encode_field_map(CUtensorMap* m, const int32_t* base, const FxGeom& g, unsigned bk, unsigned bj)
{
  return encode_patch_field_map(m, base, CU_TENSOR_MAP_DATA_TYPE_INT32, 4, g.ni, g.nj, g.nk, g.kp, bk, bj);
}

} // namespace

bool encode_stage_maps(CUtensorMap* tm_in, CUtensorMap* tm_un, const int32_t* in, const int32_t* un, const FxGeom& g,
                       int tj, int tk)
{
  // TMA staging when the rows are 16-byte strided and the fields 16-byte
  // aligned (checked by encode_patch_field_map)
  if (tma_disabled()) return false;
  const unsigned bj = tj + 4, bk = tk + 8;
  return encode_field_map(&tm_in[kFxMapMain], in, g, bk, bj) && encode_field_map(&tm_in[kFxMapK], in, g, 4, bj) &&
         encode_field_map(&tm_in[kFxMapJ], in, g, bk, 2) && encode_field_map(&tm_in[kFxMapC], in, g, 4, 2) &&
         encode_field_map(tm_un, un, g, tk, tj);
}

cudaError_t launch_stage_fx32(const FxArgs& a, cudaStream_t st)
{
  using Smem = FxSmem<FX_TJ, FX_TK>;
  auto kern = a.wall.any ? fx_stage_kernel<FX_TJ, FX_TK, true> : fx_stage_kernel<FX_TJ, FX_TK, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
  if (e != cudaSuccess) return e;
  FxLaunch L;
  std::memset(&L, 0, sizeof L);
  L.a = a;
  L.tma = encode_stage_maps(L.tm_in, &L.tm_un, a.in, a.un, a.g, FX_TJ, FX_TK);
  dim3 block(FX_TK / 2, FX_TJ, 1);
  dim3 grid((a.g.nk + FX_TK - 1) / FX_TK, (a.g.nj + FX_TJ - 1) / FX_TJ,
            (a.g.ni + a.g.i_chunk - 1) / a.g.i_chunk);
  kern<<<grid, block, sizeof(Smem), st>>>(L);
  return cudaGetLastError();
}

void fx32_tile(int* tj, int* tk) { *tj = FX_TJ; *tk = FX_TK; }

namespace {
template <int TJ, int TK, int MODE>
cudaError_t launch_fx_batched(const Batch& b, cudaStream_t st)
{
  using Smem = FxSmem<TJ, TK>;
  auto kern = b.groups ? fx_stage_batched_persistent<TJ, TK, MODE> : fx_stage_batched<TJ, TK, MODE>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
  if (e != cudaSuccess) return e;
  kern<<<b.groups ? b.n_groups : b.n_items, dim3(TK / 2, TJ, 1), sizeof(Smem), st>>>(b);
  return cudaGetLastError();
}

template <int MODE>
cudaError_t launch_fx_batched_shape(const Batch& b, int shape, cudaStream_t st)
{
  if (shape == 0) return launch_fx_batched<8, 32, MODE>(b, st);
  if (shape == 1) return launch_fx_batched<16, 16, MODE>(b, st);
  return launch_fx_batched<16, 32, MODE>(b, st);
}

template <int TJ, int TK, int MODE>
cudaError_t occupancy_of(int* blocks)
{
  using Smem = FxSmem<TJ, TK>;
  auto kern = fx_stage_batched_persistent<TJ, TK, MODE>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, kern, TJ * TK / 2, sizeof(Smem));
}

template <int MODE>
cudaError_t occupancy_shape(int shape, int* blocks)
{
  if (shape == 0) return occupancy_of<8, 32, MODE>(blocks);
  if (shape == 1) return occupancy_of<16, 16, MODE>(blocks);
  return occupancy_of<16, 32, MODE>(blocks);
}
} // namespace

cudaError_t fx32_batched_occupancy(int shape, int form, int* blocks)
{
  if (form == kFxFull) return occupancy_shape<kFxFull>(shape, blocks);
  if (form == kFxInside) return occupancy_shape<kFxInside>(shape, blocks);
  return occupancy_shape<kFxEdge>(shape, blocks);
}

cudaError_t launch_stage_fx32_batched(const Batch& b, int shape, int form, cudaStream_t st)
{
  if (b.n_items <= 0) return cudaSuccess;
  if (form == kFxFull) return launch_fx_batched_shape<kFxFull>(b, shape, st);
  if (form == kFxInside) return launch_fx_batched_shape<kFxInside>(b, shape, st);
  return launch_fx_batched_shape<kFxEdge>(b, shape, st);
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
