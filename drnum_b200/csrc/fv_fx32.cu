// FX32 (FP32 bulk, fixed-point storage) stage kernel instantiation.
#include <cstdlib>
#include <cstring>
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

namespace {

// cuTensorMapEncodeTiled of the driver, reached through the runtime's entry
// point query (no link-time dependency on the driver library)
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_tiled()
{
  static const EncodeTiled fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeTiled) nullptr;
    return reinterpret_cast<EncodeTiled>(p);
  }();
  return fn;
}

// Tensor map of one field of a patch, [5][ni][nj][nk] int32, with box
// (bk, bj, 1, 5).  The caller has checked nk % 4 == 0 (16-byte row stride)
// and the 16-byte alignment of the base.
bool encode_field_map(CUtensorMap* m, const int32_t* base, const FxGeom& g, unsigned bk, unsigned bj)
{
  const EncodeTiled enc = encode_tiled();
  if (!enc) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)g.nk, (cuuint64_t)g.nj, (cuuint64_t)g.ni, 5};
  const cuuint64_t strides[3] = {(cuuint64_t)g.nk * 4, (cuuint64_t)g.nj * g.nk * 4, (cuuint64_t)g.ni * g.nj * g.nk * 4};
  const cuuint32_t box[4] = {bk, bj, 1, 5};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_INT32, 4, const_cast<int32_t*>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

} // namespace

bool encode_stage_maps(CUtensorMap* tm_in, CUtensorMap* tm_un, const int32_t* in, const int32_t* un, const FxGeom& g,
                       int tj, int tk)
{
  // TMA staging when the rows are 16-byte strided and the fields 16-byte
  // aligned; with DN_FX_NO_TMA=1 in the environment every tile copies cell
  // by cell (the two give identical results)
  const char* nt = std::getenv("DN_FX_NO_TMA");
  if (nt && nt[0] == '1') return false;
  if (((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(un)) & 15) != 0 || g.nk % 4 != 0) return false;
  const unsigned bj = tj + 4, bk = tk + 8;
  return encode_field_map(&tm_in[kFxMapMain], in, g, bk, bj) && encode_field_map(&tm_in[kFxMapK], in, g, 4, bj) &&
         encode_field_map(&tm_in[kFxMapJ], in, g, bk, 2) && encode_field_map(&tm_in[kFxMapC], in, g, 4, 2) &&
         encode_field_map(tm_un, un, g, tk, tj);
}

cudaError_t launch_stage_fx32(const FxArgs& a, cudaStream_t st)
{
  using Smem = FxSmem<FX_TJ, FX_TK>;
  auto kern = fx_stage_kernel<FX_TJ, FX_TK>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
  if (e != cudaSuccess) return e;
  FxLaunch L;
  std::memset(&L, 0, sizeof L);
  L.a = a;
  L.tma = encode_stage_maps(L.tm_in, &L.tm_un, a.in, a.un, a.g, FX_TJ, FX_TK);
  dim3 block(FX_TK, FX_TJ, 1);
  dim3 grid((a.g.nk + FX_TK - 1) / FX_TK, (a.g.nj + FX_TJ - 1) / FX_TJ,
            (a.g.ni + a.g.i_chunk - 1) / a.g.i_chunk);
  kern<<<grid, block, sizeof(Smem), st>>>(L);
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
