// Device form of the level-set slip-wall boundary condition of all patches
// of a context, and its launcher.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace dn {

// Inner layer cells of all patches (device pointers), in the reference's
// order (patch, layer, cell).
struct LsPlan {
  int32_t n;                  // layer cells over all patches
  const int32_t* patch;       // patch per layer cell
  const int64_t* cell;        // cell index in its patch
  const double* grad;         // [n][3] normalised level-set gradient
  const int64_t* donor;       // [n][8] mirror-point donors (same patch)
  const double* w;            // [n][8] mirror-point weights
  double* acc;                // [n][5] scratch: interpolated mirror state
  void* const* bufs;          // [num_patches * 3] physical field buffers
  const int64_t* nc;          // [num_patches]
  const double* base;         // [num_patches * 5] FP32-bulk base state
  const double* quantum;      // [num_patches * 5]
};

// CPU_LevelSetObjectBC<LSOBCCompressibleEulerOp>::operator() on physical
// buffer `buf`: gather every cell's mirror state, then overwrite the cell
// (two launches: the gather of one cell may read another layer cell).
cudaError_t launch_levelset_bc(const LsPlan& p, int buf, bool fixed_point, int* err, cudaStream_t st);

} // namespace dn
