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
  // the reference's GPU level-set path (GPU_CartesianLevelSetBC): the
  // deactivated (G < 0) cells that no donor copy writes, reset to the
  // step-start state as the GPU iterator's advance kernel leaves inactive
  // cells (gpu_cartesianiterator.h:199-205), and the inside cells with their
  // averaged neighbours (CSR) and weights
  int32_t n_reset;
  const int32_t* reset_patch;
  const int64_t* reset_cell;
  int32_t n_avg;
  const int32_t* avg_patch;
  const int64_t* avg_cell;
  const int64_t* avg_start;   // [n_avg + 1]
  const int64_t* avg_nbr;
  const double* avg_w;
  double* avg_acc;            // [n_avg][5] scratch: the averaged state
};

// Device error bit of a level-set average that is not finite (the
// reference's inside-cell kernel traps there, gpu_cartesianlevelsetbc.h:478-481).
constexpr int kErrLsAverage = 64;

// CPU_LevelSetObjectBC<LSOBCCompressibleEulerOp>::operator() on physical
// buffer `buf`: gather every cell's mirror state, then overwrite the cell
// (two launches: the gather of one cell may read another layer cell).
cudaError_t launch_levelset_bc(const LsPlan& p, int buf, bool fixed_point, int* err, cudaStream_t st);

// GPU_CartesianLevelSetBC::operator() (gpu_cartesianlevelsetbc.h:491-527) on
// physical buffer `buf`, with step_buf holding the step-start state: the
// deactivated cells are reset to it, then every inside cell with neighbours
// is replaced by their weighted mean (gathered first, written second, like
// the reference's field-2 copy).  Its boundary-cell kernel writes nothing
// and is not run.
cudaError_t launch_levelset_gpu(const LsPlan& p, int buf, int step_buf, bool fixed_point, int* err, cudaStream_t st);

} // namespace dn
