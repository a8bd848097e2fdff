// Host side of the TMA staging: tensor maps of patch fields, encoded with
// the driver's cuTensorMapEncodeTiled (reached through the runtime's entry
// point query, so the library has no link-time dependency on the driver).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdlib>

namespace dn {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_tiled_fn()
{
  static const EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeTiledFn) nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// DN_FX_NO_TMA=1 in the environment turns TMA staging off (every tile then
// copies cell by cell; the results are identical)
inline bool tma_disabled()
{
  const char* v = std::getenv("DN_FX_NO_TMA");
  return v && v[0] == '1';
}

// Tensor map of one field of a patch, [5][ni][nj][nk] elements of `elem`
// bytes stored in rows of kp >= nk elements, with box (bk, bj, 1, 5).  False
// unless the rows are 16-byte strided and the base is 16-byte aligned, or
// when the driver refuses.
inline bool encode_patch_field_map(CUtensorMap* m, const void* base, CUtensorMapDataType type, unsigned elem,
                                   int ni, int nj, int nk, int kp, unsigned bk, unsigned bj)
{
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || ((uint64_t)kp * elem) % 16 != 0 || kp < nk) return false;
  const EncodeTiledFn enc = encode_tiled_fn();
  if (!enc) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)nk, (cuuint64_t)nj, (cuuint64_t)ni, 5};
  const cuuint64_t strides[3] = {(cuuint64_t)kp * elem, (cuuint64_t)nj * kp * elem, (cuuint64_t)ni * nj * kp * elem};
  const cuuint32_t box[4] = {bk, bj, 1, 5};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return enc(m, type, 4, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

} // namespace dn
