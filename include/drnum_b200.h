/*
 * drnum_b200 — C ABI of the B200 (sm_100a) implementation of DrNUM's
 * per-patch explicit finite-volume step.
 *
 * The reference drives its GPU path through C++ templates and one argument-
 * less FFI seam (applications/ * /main.cpp:25-30 calling extern "C" GPU_main()).
 * This header replaces the operator API that run() uses underneath that seam:
 *
 *   reference (file:line)                                   replaced by
 *   ------------------------------------------------------  -----------------------------
 *   GPU_PatchIterator ctor, cudaSetDevice                    dn_ctx_create
 *     (iterators/gpu_patchiterator.h:57-83)
 *   GPU_PatchIterator::addPatch / GPU_Patch ctor             dn_patch_add
 *     (gpu_patchiterator.h:86-95, gpu_patch.h:43-129)
 *   PatchIterator::updateDevice / updateHost                 dn_patch_upload[_f32],
 *     (patchiterator.h:43-44, gpu_patchiterator.h:106-126)   dn_patch_download[_f32]
 *   Patch::deactivate / m_Active (patch_common.h:502-504)    dn_patch_set_active
 *   PatchIterator::copyField (patchiterator.h:97-103)        dn_copy_field
 *   PatchIterator::computeAll / compute                      dn_compute, dn_compute_patches
 *     (patchiterator.h:50,80-87, gpu_cartesianiterator.h:218-304)
 *   PatchIterator::activatePatch / deactivatePatch           dn_patch_activate
 *     (patchiterator.h:56-57,119-133)
 *   RungeKutta::operator()(dt) (rungekutta.cpp:27-42)        dn_rk_step
 *   Patch::computeVariableDifference (patch.cpp:733-746)     dn_field_difference
 *   the applications' CFL / density diagnostics              dn_flow_stats
 *     (drnumBaseFlowDemo/main.h:255-284)
 *   PatchGrid::computeDependencies (patchgrid.cpp:119-268)   dn_grid_compute_dependencies
 *   PatchIterator::copyDonorData (patchiterator.h:106-111)   dn_copy_donor_data
 *   LevelSetObject + CPU_LevelSetObjectBC                    dn_patch_set_levelset,
 *     (levelsetobject.cpp:44-388, cpu_levelsetobjectbc.h)    dn_apply_levelset_bc
 *
 * Conventions
 *   - Every call returns an int status: DN_OK (0) or a negative DN_ERR_*.
 *     Nothing exits, aborts or traps; dn_last_error() gives the message.
 *   - Host arrays of a patch are laid out [var][i][j][k], k fastest, exactly
 *     like Patch::getField (patch_common.h:72-95, cartesianpatch_common.h:61).
 *   - Work is issued on the context's CUDA stream (dn_set_stream) and is
 *     stream-ordered; calls that return host data synchronise that stream.
 *   - Fields: 0 = current state, 1 = state at the start of the last RK step,
 *     2 = scratch, as in the reference applications (setNumberOfFields(3)).
 */
#ifndef DRNUM_B200_H
#define DRNUM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DN_OK             0
#define DN_ERR_ARG       -1   /* invalid argument */
#define DN_ERR_CUDA      -2   /* CUDA runtime error */
#define DN_ERR_STATE     -3   /* call not valid in the current state */
#define DN_ERR_NOMEM     -4   /* device or host allocation failed */
#define DN_ERR_RANGE     -5   /* value outside the representable range */
#define DN_ERR_DEVICE    -6   /* a kernel reported an error (see message) */

/* Arithmetic/storage form of a context. */
#define DN_FP64           0   /* plain FP64 path, operation order of the reference CPU iterator */
#define DN_FP32           1   /* FP32 bulk path with FP64 base state and FP64 sums */

/* Patch-face treatment per axis. */
#define DN_FACE_PERIODIC  0   /* index wrap (periodic patch) */
#define DN_FACE_CLOSED    1   /* first-order reconstruction at the edge, zero face flux */

/* Flux through an outer face of a non-periodic patch axis (the flux
 * functor's x/y/zWall{M,P}, iterators/cartesianiterator.h:190-308). */
#define DN_BC_ZERO_FLUX   0   /* wall methods that add nothing */
#define DN_BC_FARFIELD    1   /* CompressibleFarfieldFlux (fluxes/compressiblefarfieldflux.h:26-181) */
#define DN_BC_SLIP        2   /* CompressibleSlipFlux (fluxes/compressibleslipflux.h:34-98) */
#define DN_BC_INFLOW      3   /* prescribed face state per face, the JetFlux::xWallM form
                                 (applications/drnumJetDemo/jetflux.h:158-192) */

typedef struct dn_ctx dn_ctx;

/* Geometry of one axis-aligned Cartesian patch (CartesianPatch::readFromFile,
 * cartesianpatch.cpp:98-133: origin, NI NJ NK, seek layers per side, lengths). */
typedef struct dn_patch_desc {
  int32_t ni, nj, nk;      /* cells per axis */
  int32_t face[3];         /* DN_FACE_* for the x, y and z axis */
  double  dx, dy, dz;      /* cell spacing; ignored on an axis whose length[] is > 0 */
  double  origin[3];       /* lower corner in inertial coordinates */
  double  length[3];       /* patch extent per axis; if > 0 the spacing is length/n, exactly
                              as CartesianPatch::computeDeltas (cartesianpatch.cpp:160-165) */
  int32_t seek[6];         /* receiving (seek) layers at imin, imax, jmin, jmax, kmin, kmax;
                              0 = none (CartesianPatch::setSeekExceptions, cartesianpatch.cpp:146-157) */
  int32_t add_protect;     /* additional protected layers next to the seek layers
                              (PatchGrid::setNumAddProtectLayers, patchgrid.cpp:87-90) */
} dn_patch_desc;

/* Creates a context on CUDA device `device` with precision DN_FP64 or DN_FP32.
 * Replaces: GPU_PatchIterator ctor (iterators/gpu_patchiterator.h:57-83). */
int dn_ctx_create(int device, int precision, dn_ctx** out);

/* Frees all device memory of the context.  NULL is accepted. */
int dn_ctx_destroy(dn_ctx* ctx);

/* Copies the last error message (NUL-terminated, truncated to n bytes). */
int dn_last_error(const dn_ctx* ctx, char* buf, size_t n);

/* Makes subsequent work of the context run on `stream` (a cudaStream_t, or
 * NULL for the context's own stream). */
int dn_set_stream(dn_ctx* ctx, void* stream);

/* Adds a patch; allocates its three fields on the device (the active mask
 * on the first dn_patch_set_active).  FP32-bulk fields are stored in rows
 * padded to a multiple of 4 cells (16 bytes) along k, invisible through the
 * API; such a patch is limited to 5*ni*nj*nk' < 2^31 with nk' = nk rounded
 * up to a multiple of 4 (32-bit element offsets, DN_ERR_ARG otherwise).
 * Replaces: GPU_PatchIterator::addPatch + GPU_Patch ctor
 * (iterators/gpu_patchiterator.h:86-95, gpu_patch.h:43-129). */
int dn_patch_add(dn_ctx* ctx, const dn_patch_desc* desc, int* patch_id);

/* Boundary flux of side `side` (0 x-min, 1 x-max, 2 y-min, 3 y-max, 4 z-min,
 * 5 z-max) of a non-periodic axis; every side starts as DN_BC_ZERO_FLUX.
 *   DN_BC_FARFIELD: params = far-field p, T, u, v, w
 *                   (CompressibleFarfieldFlux::setFarfield, compressiblefarfieldflux.h:87-90)
 *   DN_BC_INFLOW:   table = per face {p, T, u, v, w}; p = NaN takes the boundary
 *                   cell's pressure.  Faces ordered j*nk+k (x sides), i*nk+k (y sides),
 *                   i*nj+j (z sides).  The table is copied.
 * The face flux uses the boundary cell's own state and is added to its
 * residual after the interior faces, as the reference's iterator does. */
int dn_patch_set_bc(dn_ctx* ctx, int patch_id, int side, int kind, const double* params, const double* table);

/* DN_FP32 only: FP64 base state the FP32 offsets are stored against, and the
 * per-variable offset quantum is derived from `range` (the largest expected
 * |U - base| per variable, which for the momenta must also cover the scale
 * of the pressure flux, rho*(|u| + a)).  Optional; dn_patch_upload derives
 * both from the uploaded data when this was not called (range = 4 x max
 * |rho|, rho*(|u| + a), |rho E|).  A state or face flux outside the range is
 * reported as DN_ERR_RANGE, never wrapped. */
int dn_patch_set_base(dn_ctx* ctx, int patch_id, const double base[5], const double range[5]);

/* Host -> device copy of field `field` of one patch, [5][ni][nj][nk].
 * Replaces: PatchIterator::updateDevice (gpu_patchiterator.h:114-126). */
int dn_patch_upload(dn_ctx* ctx, int patch_id, int field, const double* host);
int dn_patch_upload_f32(dn_ctx* ctx, int patch_id, int field, const float* host);

/* Device -> host copy of field `field` of one patch, [5][ni][nj][nk].
 * Replaces: PatchIterator::updateHost (gpu_patchiterator.h:106-111). */
int dn_patch_download(dn_ctx* ctx, int patch_id, int field, double* host);
int dn_patch_download_f32(dn_ctx* ctx, int patch_id, int field, float* host);

/* Asynchronous forms of the four calls above: they return once the work is
 * enqueued, and the host buffer must stay untouched (and, for the copy to
 * overlap, pinned) until dn_sync.  Uploads copy on a copy-in stream and
 * downloads on a copy-out stream, each through two device staging buffers;
 * events keep them in order with the context's stream (an upload's
 * conversion into the field waits for its copy, a download reads the field
 * where the context's stream stood when it was called, and later work on the
 * field waits for that read only).  So the download of step k, the upload of
 * step k+1 and the stages of step k+1 overlap on the two copy engines and the
 * SMs.  No reference counterpart (updateHost/updateDevice are synchronous,
 * gpu_patchiterator.h:106-126); errors of the conversions surface at
 * dn_sync. */
int dn_patch_upload_async(dn_ctx* ctx, int patch_id, int field, const double* host);
int dn_patch_upload_f32_async(dn_ctx* ctx, int patch_id, int field, const float* host);
int dn_patch_download_async(dn_ctx* ctx, int patch_id, int field, double* host);
int dn_patch_download_f32_async(dn_ctx* ctx, int patch_id, int field, float* host);

/* Sets the active mask (1 = active, 0 = frozen) of a patch; NULL = all active.
 * Replaces: Patch::activate/deactivate (patch_common.h:502-504). */
int dn_patch_set_active(dn_ctx* ctx, int patch_id, const uint8_t* mask);

/* Copies field i_src to field i_dst on every patch.
 * Replaces: PatchIterator::copyField (patchiterator.h:97-103). */
int dn_copy_field(dn_ctx* ctx, int i_src, int i_dst);

/* One RK stage on every patch: f0 = f1 + factor/dV * Res(f0) on active cells.
 * Replaces: PatchIterator::computeAll -> GPU_CartesianIterator::compute
 * (patchiterator.h:80-87, gpu_cartesianiterator.h:218-304). */
int dn_compute(dn_ctx* ctx, double factor);

/* One RK stage of the listed patches only (ids, n of them; each once),
 * skipping inactive ones: every other patch keeps its field 0 (the stage's
 * output buffer receives a copy of its input).  DN_ERR_ARG for an id out of
 * range or listed twice.
 * Replaces: PatchIterator::compute(factor, patches) (patchiterator.h:50;
 * the reference's CPU iterator, cartesianiterator.h:87-93, walks the list). */
int dn_compute_patches(dn_ctx* ctx, double factor, const int32_t* patches, int n);

/* Takes a patch out of (active = 0) or back into (1) every later stage of
 * dn_compute, dn_compute_patches and dn_rk_step: an inactive patch keeps
 * its state (its output buffers receive copies of the input), while donor
 * copies and the level-set wall still write its receiving cells, as the
 * reference's copyDonorData does for every patch.  Patches start active.
 * Replaces: PatchIterator::activatePatch / deactivatePatch
 * (patchiterator.h:56-57,119-133), read by the stage loop of
 * GPU_CartesianIterator::compute (gpu_cartesianiterator.h:226). */
int dn_patch_activate(dn_ctx* ctx, int patch, int active);

/* One full low-storage RK time step with stage factors alpha[0..n-1]*dt,
 * without the field 0 -> 1 copy (field 1 holds the step-start state after
 * the call, as after the reference's step).  With donor tables it runs the
 * reference's sequence: donor copy, then per stage compute + donor copy
 * (+ the level-set wall, and a donor copy before every later stage).  A
 * donor copy into a buffer whose receiving cells already hold it (nothing
 * but a donor copy has written the buffer since, under the same tables,
 * and no donor cell is a receiving cell) is left out: it would write the
 * same values.  Sharded contexts (an exchange hook) make every copy.
 * Replaces: RungeKutta::operator()(dt) (rungekutta.cpp:27-42). */
int dn_rk_step(dn_ctx* ctx, double dt, const double* alpha, int n_alpha);

/* Blocks until all work of the context has finished. */
int dn_sync(dn_ctx* ctx);

/* FP64 sums over all cells of all patches of field 0: mass, x/y/z momentum,
 * total energy (sum of U * dV).  Synchronises the context's stream. */
int dn_conservation_sums(dn_ctx* ctx, double out[5]);

/* Max-norm and L2-norm of field1(var1) - field2(var2) of one patch.
 * Replaces: Patch::computeVariableDifference (patch.cpp:733-746). */
int dn_field_difference(dn_ctx* ctx, int patch_id, int i_field1, int i_var1,
                        int i_field2, int i_var2, double* max_norm, double* l2_norm);

/* Diagnostics of one patch's field as the reference applications compute
 * them at each output step: out[0] = max over cells of max(|u|, |u+a|,
 * |u-a|) * dt / dx (the CFL number of time step dt), out[1] = min(1000,
 * min rho), out[2] = max(0, max rho); per cell in FP64 with the reference's
 * operation order, so the values equal the reference's loop.
 * Replaces: the loop of drnumBaseFlowDemo/main.h:255-284 and
 * drnumBasicAero/main.h:608-637 over a host copy of the field. */
int dn_flow_stats(dn_ctx* ctx, int patch_id, int i_field, double dt, double out[3]);

/* Builds the donor tables of every patch from the patches' geometry and seek
 * and protection layers: receiving cells, donor patches, 8-point trilinear
 * donor stencils and weights, multi-donor averaging and padding.  Indices and
 * FP64 weights equal the reference's.  *no_donor (may be NULL) receives the
 * number of seek cells that found no donor; they are dropped, as the
 * reference does after its warning (patch.cpp:370-395).
 * Replaces: PatchGrid::computeDependencies(true) (patchgrid.cpp:119-268),
 * Patch::finalizeDependencies / buildDonorTransferData (patch.cpp:319-465,128-218). */
int dn_grid_compute_dependencies(dn_ctx* ctx, int64_t* no_donor);

/* Sizes of a patch's donor tables: counts[0] unique receiving cells,
 * counts[1] donor patches, counts[2] concatenated receiving cells,
 * counts[3] concatenated contributions (Patch::getNumReceivingCellsUnique,
 * getNumDonorPatches, getNumReceivingCellsConcat, getNumDonorWIConcat,
 * patch_common.h:132-150). */
int dn_patch_donor_counts(dn_ctx* ctx, int patch_id, int64_t counts[4]);

/* Copies a patch's donor tables out, in the reference's direct-transfer
 * layout (patch.cpp:128-218): rec_unique[counts[0]]; per donor
 * donor_patch/num_receivers/stride[counts[1]]; rec_concat[counts[2]];
 * donor_idx/weight[counts[3]]. */
int dn_patch_get_donors(dn_ctx* ctx, int patch_id, uint64_t* rec_unique, int32_t* donor_patch,
                        int64_t* num_receivers, int32_t* stride, uint64_t* rec_concat,
                        uint64_t* donor_idx, double* weight);

/* Sets a patch's donor tables built elsewhere (for example by the
 * reference's PatchGrid), same layout as dn_patch_get_donors.  Donor patches
 * are context patch ids.  Replaces: GPU_Patch's donor-table upload and
 * updateDonorPointers (gpu_patch.h:43-129,142-173). */
int dn_patch_set_donors(dn_ctx* ctx, int patch_id, const int64_t counts[4], const uint64_t* rec_unique,
                        const int32_t* donor_patch, const int64_t* num_receivers, const int32_t* stride,
                        const uint64_t* rec_concat, const uint64_t* donor_idx, const double* weight);

/* Host-only form of dn_grid_compute_dependencies: builds the donor tables of
 * np patch descriptions without a context or a GPU (patch ids are positions
 * in `patches`).  Read them with dn_overlap_counts / dn_overlap_get (same
 * layout as dn_patch_get_donors), hand them to a context with
 * dn_patch_set_donors, free them with dn_overlap_destroy.
 * Replaces: PatchGrid::computeDependencies(true) (patchgrid.cpp:119-268). */
typedef struct dn_overlap dn_overlap;
int dn_overlap_build(const dn_patch_desc* patches, int np, dn_overlap** out, int64_t* no_donor);
int dn_overlap_counts(const dn_overlap* ov, int patch_id, int64_t counts[4]);
int dn_overlap_get(const dn_overlap* ov, int patch_id, uint64_t* rec_unique, int32_t* donor_patch,
                   int64_t* num_receivers, int32_t* stride, uint64_t* rec_concat,
                   uint64_t* donor_idx, double* weight);
int dn_overlap_destroy(dn_overlap* ov);

/* Donor copy into field `field` of every patch: each receiving cell gets
 * the weighted sum of its donor cells (per donor patch in table order, then
 * summed over donor patches).  Patches are axis-aligned, so no vector
 * rotation applies.  Replaces: PatchIterator::copyDonorData
 * (patchiterator.h:106-111) -> Patch::accessDonorDataDirect (patch.cpp:573-653),
 * GPU_PatchIterator::copyDonorData (gpu_patchiterator.h:190-233). */
int dn_copy_donor_data(dn_ctx* ctx, int field);

/* Level-set slip wall of one patch: classifies the cell layers next to the
 * zero level of the signed-distance field G ([ni][nj][nk], host, FP64 values;
 * an FP32 field is passed widened) and, from then on, applies the slip-wall
 * mirror condition to the inner layers after every RK stage (after the
 * donor copy, as a post-operation).  num_inner_layers/num_outer_layers and
 * min_inner_rel_dist as LevelSetObject's constructor; G = NULL removes the
 * wall.  The layer lists equal the reference's.
 * Replaces: LevelSetObject::update/extractBCellLayers (levelsetobject.cpp:44-388),
 * LevelSetObjectBC::transferCellLayerData (levelsetobjectbc.cpp:38-134) and
 * CPU_LevelSetObjectBC<LSOBCCompressibleEulerOp> (cpu_levelsetobjectbc.h:58-90,
 * lsobccompressibleeulerop.h:49-144). */
int dn_patch_set_levelset(dn_ctx* ctx, int patch_id, const double* G, int num_inner_layers,
                          int num_outer_layers, double min_inner_rel_dist);

/* A patch's level-set wall from layers classified elsewhere (for example by
 * the reference's LevelSetObject::extractBCellLayers): num_inner_layers inner
 * (G < 0) layers of counts[layer] cells, concatenated in layer order: cell
 * index, G, normalised gradient [n][3], mirror-point donors and weights
 * [n][8] (the layout of dn_patch_levelset_get).  From then on the slip-wall
 * mirror condition runs on them as after dn_patch_set_levelset.
 * Replaces: LevelSetObjectBC::transferCellLayerData (levelsetobjectbc.cpp:38-134)
 * reading LevelSetObject::getInnerCellsLayers (levelsetobject.h:128). */
int dn_patch_set_levelset_layers(dn_ctx* ctx, int patch_id, int num_inner_layers, const int64_t* counts,
                                 const uint64_t* cells, const double* g, const double* grad, const uint64_t* donors,
                                 const double* weights);

/* The level-set wall of the reference's GPU path instead, for applications
 * that use GPU_CartesianLevelSetBC<DIM, NUM_LS, StoredLevelSet,
 * CompressibleLsSlip> (e.g. drnumBasicAero): every cell with G < 0 is
 * deactivated (gpu_cartesianlevelsetbc.h:106-125; cells the patch's mask
 * already deactivated stay so) and, like the reference's GPU iterator
 * (gpu_cartesianiterator.h:199-205), holds the step-start state through the
 * stages unless a donor copy writes it; after every stage each "inside" cell
 * (G < 0 with no G >= 0 cell in its two-cell box) takes the weighted mean of
 * its box cells of larger G, weight |d . grad G| / |d|
 * (gpu_cartesianlevelsetbc.h:129-229,414-487).  The reference's boundary-cell
 * kernel writes nothing (:316-411) and has no counterpart.  A mean that is not
 * finite is reported as DN_ERR_DEVICE where the reference traps.  Returns
 * DN_ERR_ARG where the reference stops with a BUG (a G < 0 cell within two
 * cells of the patch edge, :170-179).  Replaces the patch's other level-set
 * wall; G = NULL removes it (the cells stay deactivated: dn_patch_set_active
 * restores the mask). */
int dn_patch_set_levelset_gpu(dn_ctx* ctx, int patch_id, const double* G);

/* Sizes of a patch's GPU level-set path: counts[0] deactivated cells,
 * counts[1] inside cells, counts[2] averaged neighbour entries. */
int dn_patch_levelset_gpu_counts(dn_ctx* ctx, int patch_id, int64_t counts[3]);

/* Size and contents of one layer of a patch's level-set classification
 * (inner = 1: G < 0 layers, 0: outer layers), in the reference's order:
 * cell index, G, normalised gradient [n][3], mirror-point donors and weights
 * [n][8] (inner layers; outer layers carry zeros).  Any output may be NULL.
 * Replaces: LevelSetObject::getInnerCellsLayers/getOuterCellsLayers
 * (levelsetobject.h:128-131), LSLayerDataExtrapol (lslayerdataextrapol.h:19-34). */
int dn_patch_levelset_count(dn_ctx* ctx, int patch_id, int inner, int layer, int64_t* n);
int dn_patch_levelset_get(dn_ctx* ctx, int patch_id, int inner, int layer, uint64_t* cells, double* g,
                          double* grad, uint64_t* donors, double* weights);

/* The level-set wall condition alone, on field `field` of every patch with a
 * level set.  Replaces: CPU_LevelSetObjectBC::operator() (cpu_levelsetobjectbc.h:58-90). */
int dn_apply_levelset_bc(dn_ctx* ctx, int field);

/* Host-only form of the classification (no context, no GPU): the layers of
 * one patch description.  Read with dn_lslayers_count/dn_lslayers_get (same
 * layout as dn_patch_levelset_get), free with dn_lslayers_destroy. */
typedef struct dn_lslayers dn_lslayers;
int dn_levelset_classify(const dn_patch_desc* patch, const double* G, int num_inner_layers,
                         int num_outer_layers, double min_inner_rel_dist, dn_lslayers** out);
int dn_lslayers_count(const dn_lslayers* ls, int inner, int layer, int64_t* n);
int dn_lslayers_get(const dn_lslayers* ls, int inner, int layer, uint64_t* cells, double* g, double* grad,
                    uint64_t* donors, double* weights);
int dn_lslayers_destroy(dn_lslayers* ls);

/* Context options.
 *   DN_OPT_BATCHED (default 1): one launch per RK stage and tile shape over a
 *     work list of (patch, column tile, plane range) items of all patches;
 *     0 = one launch per patch.  Results are identical.
 *   DN_OPT_GRAPH (default 0): dn_rk_step captures the whole step (stages,
 *     donor copies, level-set wall) as a CUDA graph once per buffer rotation,
 *     dt and alphas, and replays it.
 *   DN_OPT_BATCH_WAVES (FP32 bulk, default 2): > 0 deals each batched launch's
 *     work to that many waves of persistent CTAs with equal planes per CTA;
 *     0 launches one CTA per work item.  dn_autotune measures the choices.
 *   DN_OPT_BATCH_MIN_PLANES (default 8): shortest plane range of a work item
 *     when one CTA takes one item.
 *   DN_OPT_DONOR_TABLES (default 0): device form of the donor tables.  0 =
 *     interpolation patterns (each group as donor patch, first donor cell and
 *     a shared entry of offsets and weights) wherever every device cell
 *     offset fits 32 bits, else per-contribution 64-bit tables; 1 = always
 *     the per-contribution tables.
 *   The schedule and table options change no result.
 * No reference counterpart (the reference launches 10 kernels per patch and
 * stage, each followed by a device synchronisation, gpu_cartesianiterator.h:218-304). */
#define DN_OPT_BATCHED    0
#define DN_OPT_GRAPH      1
#define DN_OPT_BATCH_WAVES      2
#define DN_OPT_BATCH_MIN_PLANES 3
#define DN_OPT_DONOR_TABLES     4
int dn_set_option(dn_ctx* ctx, int option, int value);

/* Tile shape of a patch in the batched launch (j x k): 0 = 8 x 32 (FP64
 * 4 x 32), 1 = 16 x 16 (FP64 8 x 16), 2 = 16 x 32 (FP64 8 x 32).  The default
 * wastes the fewest k lanes and takes the 16-row tile where the patch has
 * at least 16 rows. */
#define DN_NUM_TILE_SHAPES 3
int dn_patch_set_tile(dn_ctx* ctx, int patch_id, int shape);

/* Autotuner: measures each tile shape's cost per padded cell on the
 * context's own patches (one stage into the scratch field 2, which it
 * overwrites), then gives every patch the shape of least predicted time.
 * cache_path (may be NULL) holds measured costs per device and precision and
 * is reused on the next call; cost_out[DN_NUM_TILE_SHAPES] (may be NULL) returns them in ns per
 * padded cell and stage.  FP32-bulk stages that run one patch per launch (a
 * single patch, or batching off) also get the plane-chunk length of their
 * CTAs, measured among a few candidates on the patch itself; batched stages
 * of several patches get the shortest plane range of a work item the same
 * way.  None of the choices changes a result.  No reference counterpart. */
int dn_autotune(dn_ctx* ctx, const char* cache_path, double cost_out[DN_NUM_TILE_SHAPES]);

/* Flux scheme of the stage of an FP64 context; replaces the OP template
 * argument of GPU_CartesianIterator<DIM, OP> (gpu_cartesianiterator.h:37)
 * for the schemes DrNUM's applications instantiate.  All use the Upwind2
 * reconstruction with the van Albada limiter and the patch-face fluxes of
 * dn_patch_set_bc:
 *   DN_FLUX_AUSMPLUS   AusmPlus (fluxes/ausmplus.h), the specialised fused
 *                      kernels (default; the only scheme of DN_FP32)
 *   DN_FLUX_AUSMPLUS_FUNCTOR  the same flux through the generic functor
 *                      kernel (bitwise equal to DN_FLUX_AUSMPLUS)
 *   DN_FLUX_VANLEER    VanLeer (fluxes/vanleer.h)
 *   DN_FLUX_ROE        Roe with its entropy fix (fluxes/roe.h)
 * DN_ERR_ARG for an unknown scheme or a non-default scheme on DN_FP32. */
#define DN_FLUX_AUSMPLUS          0
#define DN_FLUX_AUSMPLUS_FUNCTOR  1
#define DN_FLUX_VANLEER           2
#define DN_FLUX_ROE               3
int dn_set_flux_scheme(dn_ctx* ctx, int scheme);

/* A user stage function: one RK stage of one patch, launched by the caller's
 * own code (typically dn::launch_functor_stage<OP> of drnum_b200_functor.cuh
 * with the caller's flux functor, the analogue of instantiating
 * GPU_CartesianIterator<DIM, OP> with an application functor,
 * gpu_cartesianiterator.h:37 with e.g. applications/drnumJetDemo/jetflux.h).
 * It must enqueue its work on L->stream and return 0, or a negative value
 * that dn_rk_step / dn_compute pass on.  It computes
 *   out = un + factor/dV * residual(in)   (inactive cells: out = in)
 * for the patch's ni x nj x nk cells, [5][ni][nj][nk] FP64 arrays. */
typedef struct dn_stage_launch {
  int patch;                  /* patch id */
  const double* in;           /* stage input f(k-1) (device) */
  const double* un;           /* step-start state f(n) (device) */
  double* out;                /* stage output f(k) (device) */
  const unsigned char* active;/* per cell, NULL = all active (device) */
  int ni, nj, nk;
  int periodic[3];            /* 1 = index wrap on that axis */
  double dx, dy, dz;
  double factor;              /* alpha * dt */
  void* stream;               /* cudaStream_t */
  int num_sms;
} dn_stage_launch;
typedef int (*dn_stage_fn)(void* user, const dn_stage_launch* L);

/* Installs a user stage function for every patch of an FP64 context (NULL
 * restores the built-in scheme).  It runs inside dn_compute / dn_rk_step in
 * place of the built-in stage launch, one call per patch and stage, and is
 * captured into the step's CUDA graph with DN_OPT_GRAPH.  DN_ERR_ARG on an
 * FP32 context. */
int dn_set_stage_function(dn_ctx* ctx, dn_stage_fn fn, void* user);

/* Patch-grid files.  dn_grid_read parses a grid file as PatchGrid::readGrid
 * (patchgrid.cpp:479-557, CartesianPatch::readFromFile, cartesianpatch.cpp:
 * 98-133): blocks "<type> <comment> { ... }" up to type 0; type 1001 holds
 * the reference point, base vectors i and j, IO scale, Ni Nj Nk, the six
 * seek-layer counts, the lengths and solver codes.  Reference point and
 * lengths are scaled by IO scale * `scale`.  Patches come back as
 * descriptors (closed faces, seek counts in seek[6]) and their solver-code
 * string (normalised as CodeString::buildFrom, codestring.cpp:43-100).
 * Axis-aligned patches only: other base vectors, unknown block types or a
 * malformed block give DN_ERR_ARG.  dn_grid_write writes descriptors in the
 * layout of the reference's grid generator (Python/drnum.py:199-244);
 * codes may be NULL. */
typedef struct dn_gridfile dn_gridfile;
int dn_grid_read(const char* path, double scale, dn_gridfile** out);
int dn_gridfile_count(const dn_gridfile* g, int* n);
int dn_gridfile_patch(const dn_gridfile* g, int index, dn_patch_desc* desc, char* codes, size_t n_codes);
int dn_gridfile_destroy(dn_gridfile* g);
int dn_grid_write(const char* path, int n, const dn_patch_desc* patches, const char* const* codes);

/* Restart files.  dn_write_data writes field `field` of every patch of the
 * context to <base>_<count, 6 digits>.dnd as PatchGrid::writeData
 * (patchgrid.cpp:559-578): Qt QDataStream big-endian int32 precision (8),
 * the time as a double, then each patch's [5][ni][nj][nk] values, patches
 * in context order.  dn_read_data reads such a file (".dnd" is appended if
 * missing; precision 4 files are read too) into field `field` and returns
 * its time, as PatchGrid::readData (patchgrid.cpp:580-611); a file whose
 * size does not match the context's patches gives DN_ERR_ARG. */
int dn_write_data(dn_ctx* ctx, int field, const char* base_file_name, double time, int count);
int dn_read_data(dn_ctx* ctx, int field, const char* file_name, double* time);

/* Patch grids sharded over ranks (one process per GPU).  The reference runs
 * every patch of a grid in one process and its donor copy reads other
 * patches directly (Patch::accessDonorDataDirect, patch.cpp:573-653).  Here
 * each rank adds every patch of the grid to its context, owns some
 * (dn_patch_set_owned; default: all) and keeps the others as shadows: stages,
 * donor copies into receiving cells and the level-set wall run on owned
 * patches only, and conservation sums cover owned patches only.  Before each
 * donor copy a rank sends the owners' donor cells its peers read and
 * receives those it reads into its shadows; the donor copy then runs on
 * local memory and gives the same bits as a single context.
 *   dn_exchange_build (host only, from dn_overlap_build's tables) and
 *   dn_exchange_build_ctx (from the context's tables): the exchange lists of
 *     `rank` given owner[num_patches]; (patch, cell) pairs per peer, unique
 *     and ascending, so both ranks of a pair derive the same order;
 *   dn_exchange_counts / _get: the lists of one peer;
 *   dn_exchange_pack / _unpack: gather the send cells of field `field` into,
 *     or scatter the receive cells from, a device buffer of 5 x n elements
 *     [var][item] of the context's storage type (8-byte double for DN_FP64,
 *     4-byte int32 offsets for DN_FP32, whose shadows share the owner's base
 *     and quantum), enqueued on the context's stream.
 * Moving the buffers between ranks is the caller's (NCCL send/recv;
 * drnum_b200/shard.py).
 *
 * Memory that scales with the rank's share: a rank adds the patches it owns
 * with dn_patch_add and every other patch with dn_patch_add_shadow (no field
 * memory), sets the donor tables, builds the exchange and then calls
 * dn_shadow_alloc, which gives each compact shadow field memory for exactly
 * the cells the exchange delivers to it, [var][position among the received
 * cells in ascending order].  Device memory is then the owned patches plus
 * the donor cells their receiving cells read, not the whole grid.  A compact
 * shadow refuses the calls that need its whole state (downloads,
 * asynchronous uploads, active masks, level sets, flow statistics, field
 * differences, restart files: DN_ERR_STATE); dn_patch_upload on it derives
 * the FP32-bulk base and quantum from the whole host state, as its owner does,
 * and copies the held cells.  dn_shadow_alloc must precede the exchange's
 * first pack or unpack.  dn_patch_device_cells gives the cells per variable
 * a patch holds on the device (rows padded for FP32 bulk).
 * The reference has no counterpart (one process holds the whole grid). */
typedef struct dn_exchange dn_exchange;
int dn_patch_set_owned(dn_ctx* ctx, int patch_id, int owned);
int dn_patch_add_shadow(dn_ctx* ctx, const dn_patch_desc* desc, int* patch_id);
int dn_shadow_alloc(dn_ctx* ctx, dn_exchange* ex);
int dn_patch_device_cells(dn_ctx* ctx, int patch_id, int64_t* cells);
int dn_exchange_build(const dn_overlap* ov, const int32_t* owner, int rank, int world, dn_exchange** out);
int dn_exchange_build_ctx(dn_ctx* ctx, const int32_t* owner, int rank, int world, dn_exchange** out);
int dn_exchange_counts(const dn_exchange* ex, int peer, int64_t* n_send, int64_t* n_recv);
int dn_exchange_get(const dn_exchange* ex, int peer, int32_t* send_patch, uint64_t* send_cell, int32_t* recv_patch,
                    uint64_t* recv_cell);
/* Exchange hook: fn(user) is called on the host before every donor copy the
 * context makes (dn_rk_step, dn_copy_donor_data), also where this rank's
 * patches receive nothing, with the copy's launches not yet enqueued; inside
 * it, dn_exchange_pack / _unpack with field DN_FIELD_DONOR_COPY address the
 * buffer the copy is about to read and fill.  A sharded rank moves its donor
 * cells there (pack, send/recv on the context's stream, unpack), so that
 * dn_rk_step runs the whole step in one call with the fields rotated in
 * place.  With a hook, dn_rk_step never captures a graph and never skips
 * the donor copy before a stage.  A nonzero return fails the calling
 * function with that code.  fn NULL removes the hook. */
#define DN_FIELD_DONOR_COPY (-1)
typedef int (*dn_exchange_fn)(void* user);
int dn_set_exchange_hook(dn_ctx* ctx, dn_exchange_fn fn, void* user);
int dn_exchange_pack(dn_ctx* ctx, dn_exchange* ex, int field, int peer, void* dev_buf);
int dn_exchange_unpack(dn_ctx* ctx, dn_exchange* ex, int field, int peer, const void* dev_buf);
int dn_exchange_destroy(dn_exchange* ex);

/* Number of device kernel launches the context has issued so far. */
int dn_launch_count(const dn_ctx* ctx, int64_t* count);

/* Number of the context's patches whose stage planes are staged by TMA box
 * loads (FP32 bulk: every patch, its rows padded to 16 bytes; FP64: patches
 * with an even nk), 0 with DN_FX_NO_TMA=1 in the environment.  The other
 * patches stage cell by cell; the results are identical. */
int dn_tma_patch_count(dn_ctx* ctx, int64_t* count);

/* No counterpart in the reference.  The FP64 sums of dn_conservation_sums
 * (sum of U * dV per variable) over a caller-owned device field
 * [5][ncells] (FP64), for callers that cannot allocate device memory, such as
 * a solver that reserves all device memory at start-up or a host framework
 * that owns the device memory pool.  Allocates nothing: the per-block partial
 * sums live in a fixed 320 KiB device array inside the library, which limits
 * the field to 2^27 cells (larger fields return DN_ERR_RANGE).  `out` is a
 * host array; the call synchronises `stream` (a cudaStream_t, NULL = legacy
 * default stream).  All calls on a device share that array: calls that
 * overlap on the GPU race.  The first call on a device (with it current)
 * resolves the array's device address; make it before any stream capture.
 * That address is kept for the life of the process and is stale after a
 * cudaDeviceReset of the device: do not call this on a device that was
 * reset.  The field must be unpadded FP64 [5][ncells] (an FP64 context's
 * buffers, DrNUM's host layout); the padded int32 fixed-point buffers of an
 * FP32-bulk context cannot be passed. */
int dn_field_sums_noalloc(const double* field, int64_t ncells, double dV, double out[5], void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DRNUM_B200_H */
