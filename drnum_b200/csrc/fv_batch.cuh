// Batched stage launch: every patch of a context advances in one launch per
// RK stage (per tile shape), each CTA taking one work item (patch, column
// tile, range of planes) from a work list.  Replaces the reference's serial
// per-patch loop of 10 launches and 10 synchronisations
// (gpu_cartesianiterator.h:218-304), which leaves a B200 idle on small patches.
//
// The CTA copies its patch's record into shared memory, derives the stage
// parameters exactly as the single-patch launch does on the host, and runs
// the same tile function; results are therefore bitwise identical to the
// per-patch launches.
#pragma once

#include <cstdint>
#include "fv_policies.cuh"
#include "fv_stage.cuh"
#include "fv_fx32.cuh"

namespace dn {

// Per-patch record of the batched launch (device memory).
struct BatchPatch {
  void* buf[3];                 // physical field buffers
  const uint8_t* active;        // NULL = all active
  int ni, nj, nk;
  int kp;                       // row pitch along k (FX32: nk rounded up to a multiple of 4; FP64: nk)
  int per_x, per_y, per_z;
  int tma;                      // FX32: the patch's entry of Batch::maps is valid
  double dx, dy, dz;
  double base[5], quantum[5];   // FP32-bulk fixed-point base and quantum
  WallBC wall;
};

struct WorkItem {
  int patch, j0, k0, i0, i1;
};

// Tensor maps of a patch for its tile shape, per physical buffer.  FX32:
// the staging boxes of a stage input (in[b][0 .. kFxMaps-1]) and the box of
// f(n) (un[b]).  FP64: the plane box (TK+4 x TJ+4 x 1 x 5) in in[b][0].
struct BatchMaps {
  CUtensorMap in[3][kFxMaps];
  CUtensorMap un[3];
};

struct Batch {
  const BatchPatch* patches;
  const BatchMaps* maps;        // FX32: per patch, or NULL
  const WorkItem* items;
  int n_items;
  // FX32: the items of persistent CTA b are items[groups[b] ..
  // groups[b+1]-1], taken in order (NULL: one CTA per item); n_groups CTAs
  const int* groups;
  int n_groups;
  int in_b, un_b, out_b;        // physical buffers: stage input, step start, output
  double factor;                // alpha * dt
  int* err;
  unsigned long long* err_info;
};

// Cooperative copy of a patch record into shared memory.
__device__ __forceinline__ void load_patch_record(BatchPatch& dst, const BatchPatch* src)
{
  const int nt = blockDim.x * blockDim.y;
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
  uint32_t* d = reinterpret_cast<uint32_t*>(&dst);
  for (int w = t; w < (int)(sizeof(BatchPatch) / 4); w += nt) d[w] = s[w];
}

// MODE (kFxEdge, kFxInside, kFxFull): the tile form every item of the
// launch runs; the host sorts the items by form (fx_tile_full,
// fx_tile_inside), and the device re-checks each tile and falls back to the
// edge form.  One form per kernel keeps one code path per launch: several
// forms in one kernel made them compete for the instruction cache of an SM
// running tiles of many patches (13-17 % slower on the jet and sphere
// workloads).
// Stage arguments of work item w in shared memory (thread 0; the caller
// synchronises).
__device__ __forceinline__ void fx_item_args(FxArgs& args, const BatchPatch& rec, const Batch& b, const WorkItem& w)
{
  args.in = static_cast<const int32_t*>(rec.buf[b.in_b]);
  args.un = static_cast<const int32_t*>(rec.buf[b.un_b]);
  args.out = static_cast<int32_t*>(rec.buf[b.out_b]);
  args.active = rec.active;
  args.err = b.err;
  args.err_info = b.err_info;
  args.g.ni = rec.ni; args.g.nj = rec.nj; args.g.nk = rec.nk; args.g.kp = rec.kp;
  args.g.per_x = rec.per_x; args.g.per_y = rec.per_y; args.g.per_z = rec.per_z;
  args.g.i_chunk = w.i1 - w.i0;
  fx_set_params(args.p, rec.dx, rec.dy, rec.dz, b.factor, rec.base, rec.quantum);
  args.wall = rec.wall;
}

// The tile form MODE (falling back to the edge form where the tile does not
// qualify) of one work item; NEXT as fx_stage_tile_impl.
template <int TJ, int TK, int MODE, bool NEXT>
__device__ __forceinline__ bool fx_item(const FxArgs& args, const BatchPatch& rec, const Batch& b, const WorkItem& w)
{
  const BatchMaps* M = (b.maps && rec.tma) ? b.maps + w.patch : nullptr;
  const CUtensorMap* tm_in = M ? M->in[b.in_b] : nullptr;
  const CUtensorMap* tm_un = M ? &M->un[b.un_b] : nullptr;
  if (MODE == kFxFull && fx_tile_full<TJ, TK>(args.g, w.j0, w.k0))
    return fx_stage_tile_impl<TJ, TK, kFxFull, NEXT>(args, tm_in, tm_un, w.j0, w.k0, w.i0, w.i1);
  if (MODE == kFxInside && fx_tile_inside<TJ, TK>(args.g, w.j0, w.k0))
    return fx_stage_tile_impl<TJ, TK, kFxInside, NEXT>(args, tm_in, tm_un, w.j0, w.k0, w.i0, w.i1);
  return fx_stage_tile_impl<TJ, TK, kFxEdge, NEXT>(args, tm_in, tm_un, w.j0, w.k0, w.i0, w.i1);
}

// One CTA per work item.
template <int TJ, int TK, int MODE>
__global__ void __launch_bounds__(TJ * TK / 2, FxOccupancy<TJ * TK / 2>::min_blocks)
fx_stage_batched(const Batch b)
{
  __shared__ __align__(16) BatchPatch rec;
  __shared__ __align__(16) FxArgs args;
  const WorkItem w = b.items[blockIdx.x];
  load_patch_record(rec, b.patches + w.patch);
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) fx_item_args(args, rec, b, w);
  __syncthreads();
  fx_item<TJ, TK, MODE, false>(args, rec, b, w);
}

// Persistent CTAs: CTA b takes the items groups[b] .. groups[b+1]-1 in
// order.  The host deals the work so that one or a few waves of CTAs hold it
// with equal planes per CTA and a CTA's items follow one another along i
// (one prologue per item, no tail of short items).
template <int TJ, int TK, int MODE>
__global__ void __launch_bounds__(TJ * TK / 2, FxOccupancy<TJ * TK / 2>::min_blocks)
fx_stage_batched_persistent(const Batch b)
{
  __shared__ __align__(16) BatchPatch rec;
  __shared__ __align__(16) FxArgs args;
  const int w_begin = b.groups[blockIdx.x], w_end = b.groups[blockIdx.x + 1];
  int loaded = -1;                              // patch whose record is in shared memory
  for (int wi = w_begin; wi < w_end; ++wi) {
    // (every thread is past the previous item's closing barrier)
    const WorkItem w = b.items[wi];
    if (w.patch != loaded) {
      load_patch_record(rec, b.patches + w.patch);
      loaded = w.patch;
    }
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) fx_item_args(args, rec, b, w);
    __syncthreads();
    if (!fx_item<TJ, TK, MODE, true>(args, rec, b, w)) return;   // a transfer may still be landing
  }
}

template <int TJ, int TK>
__global__ void __launch_bounds__(TJ * TK)
fv_stage_batched_f64(const Batch b)
{
  __shared__ __align__(16) BatchPatch rec;
  __shared__ __align__(16) StageArgs<PolicyF64> args;
  const WorkItem w = b.items[blockIdx.x];
  load_patch_record(rec, b.patches + w.patch);
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    args.in = static_cast<const double*>(rec.buf[b.in_b]);
    args.un = static_cast<const double*>(rec.buf[b.un_b]);
    args.out = static_cast<double*>(rec.buf[b.out_b]);
    args.active = rec.active;
    args.err = b.err;
    args.err_info = b.err_info;
    args.g.ni = rec.ni; args.g.nj = rec.nj; args.g.nk = rec.nk;
    args.g.per_x = rec.per_x; args.g.per_y = rec.per_y; args.g.per_z = rec.per_z;
    args.g.i_chunk = w.i1 - w.i0;
    args.p.Ax = rec.dy * rec.dz;
    args.p.Ay = rec.dx * rec.dz;
    args.p.Az = rec.dx * rec.dy;
    args.p.pf = b.factor / (rec.dx * rec.dy * rec.dz);
    args.wall = rec.wall;
  }
  __syncthreads();
  const BatchMaps* M = (b.maps && rec.tma) ? b.maps + w.patch : nullptr;
  fv_stage_tile<PolicyF64, TJ, TK>(args, M ? &M->in[b.in_b][0] : nullptr, w.j0, w.k0, w.i0, w.i1);
}

} // namespace dn
