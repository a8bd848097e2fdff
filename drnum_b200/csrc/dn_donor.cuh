// Device form of the donor tables of all patches of a context, and the
// launchers of the donor copy (receiving cell <- weighted donor cells).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace dn {

// All receiving cells of all patches, each with its contributions grouped
// by donor patch in table order (device pointers).
//
// Two forms.  The pattern form (patterned != 0; every device cell offset
// below 2^32) stores a group as its donor patch, its first donor cell and
// the position of its contributions in a table of interpolation patterns
// (the other contributions' offsets from the first donor cell, and the
// weights).  Overlapping Cartesian patches repeat a few thousand stencils
// over millions of receiving cells, so the pattern table stays in cache
// and a receiving cell streams 24 B of tables.  A cell's first group is
// group r of the cell's own index; the groups after it, where a cell has
// donors in several patches, follow in table order at rv_more[r] ..
// rv_more[r+1]-1 (rv_more NULL: no cell has more than one).  The wide form
// keeps every contribution's 64-bit donor cell and weight.
struct DonorPlan {
  int32_t n_recv;             // unique receiving cells over all patches
  const int32_t* rv_patch;    // receiving patch per receiving cell
  int patterned;
  // pattern form
  const uint32_t* rv_cell32;  // cell index (device offset) in the receiving patch
  const uint4* gp_pat;        // per group: (first donor cell, first pattern entry, entries, donor patch)
  const int32_t* rv_more;     // [n_recv + 1] the groups after the first, or NULL
  const int32_t* pt_off;      // pattern entries: donor cell less the group's first
  const double* pt_w;         // pattern entries: weight
  // wide form
  const int32_t* rv_grp;      // [n_recv + 1] CSR offsets into the groups
  const int64_t* rv_cell;
  const int32_t* gp_donor;    // donor patch per group
  const int32_t* gp_stride;   // contributions per group
  const int64_t* gp_wi;       // first contribution of the group in idx/w
  const int64_t* idx;         // donor cell (device offset) per contribution
  const double* w;            // weight per contribution
  void* const* bufs;          // [num_patches * 3] physical field buffers
  const int64_t* nc;          // [num_patches] cells per patch
  const double* base;         // [num_patches * 5] FP32-bulk base state
  const double* quantum;      // [num_patches * 5] FP32-bulk quantum
};

// FP64 fields: recv = sum over donor patches of (sum over contributions of
// donor * weight), with the reference's rounding order.
cudaError_t launch_donor_copy_f64(const DonorPlan& p, int buf, cudaStream_t st);

// int32 fixed-point fields (FP32 bulk): donors dequantised and summed in
// FP64 with the FP64 weights, result quantised to the receiving patch.
cudaError_t launch_donor_copy_fx32(const DonorPlan& p, int buf, int* err, cudaStream_t st);

} // namespace dn
