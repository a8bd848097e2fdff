// Host-side launchers of the fused stage kernels (one translation unit per
// arithmetic form so each gets its own floating-point compile flags).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "fv_policies.cuh"
#include "fv_stage.cuh"

namespace dn {

// Tile and chunk shape of one launch.
struct StageShape {
  int tj, tk;      // CTA tile in j and k (threads = tj*tk)
  int i_chunk;     // planes per CTA along i
};

cudaError_t launch_stage_f64(const StageArgs<PolicyF64>& a, const StageShape& s, cudaStream_t st);
// Tensor map of an FP64 stage input for tj x tk tiles (box tk+4 x tj+4 x 1 x
// 5); false when the patch does not allow it (rows not 16-byte strided,
// unaligned field) or DN_FX_NO_TMA=1 is set.
bool encode_stage_map_f64(CUtensorMap* tm, const double* in, int ni, int nj, int nk, int tj, int tk);

struct FxArgs;
struct FxGeom;
cudaError_t launch_stage_fx32(const FxArgs& a, cudaStream_t st);
void fx32_tile(int* tj, int* tk);
// Tensor maps for TMA staging of an FX32 stage with tj x tk tiles: the
// kFxMaps boxes of the stage input `in` and the box of f(n) `un`; false when
// the patch does not allow them (rows not 16-byte strided, unaligned fields)
// or DN_FX_NO_TMA=1 is set.
bool encode_stage_maps(CUtensorMap* tm_in, CUtensorMap* tm_un, const int32_t* in, const int32_t* un, const FxGeom& g,
                       int tj, int tk);

// Batched launches over a work list (fv_batch.cuh).  Tile shapes (j x k):
//   FX32: 0 = 8 x 32, 1 = 16 x 16, 2 = 16 x 32;  FP64: 0 = 4 x 32, 1 = 8 x 16, 2 = 8 x 32.
struct Batch;
constexpr int kNumShapes = 3;
// full: every item's tile is full (fx_tile_full), run by the tile form
// without edge tests
// form: kFxEdge, kFxInside or kFxFull (the tile form of every item of b)
cudaError_t launch_stage_fx32_batched(const Batch& b, int shape, int form, cudaStream_t st);
// resident CTAs per SM of the batched FX32 kernel of a tile shape and form
cudaError_t fx32_batched_occupancy(int shape, int form, int* blocks);
cudaError_t launch_stage_f64_batched(const Batch& b, int shape, cudaStream_t st);
inline void shape_tile(bool fp64, int shape, int* tj, int* tk)
{
  *tk = shape == 1 ? 16 : 32;
  if (fp64) *tj = shape == 0 ? 4 : 8;
  else *tj = shape == 0 ? 8 : 16;
}

// Chooses the i-chunk so that the grid holds enough CTAs to fill the GPU.
int default_i_chunk(int ni, int nj, int nk, int tj, int tk, int num_sms, int ctas_per_sm);

} // namespace dn
