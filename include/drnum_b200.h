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
 *   PatchIterator::computeAll / compute                      dn_compute
 *     (patchiterator.h:80-87, gpu_cartesianiterator.h:218-304)
 *   RungeKutta::operator()(dt) (rungekutta.cpp:27-42)        dn_rk_step
 *   Patch::computeVariableDifference (patch.cpp:733-746)     dn_field_difference
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

typedef struct dn_ctx dn_ctx;

/* Geometry of one Cartesian patch (CartesianPatch: sizeI/J/K, dx/dy/dz, origin). */
typedef struct dn_patch_desc {
  int32_t ni, nj, nk;      /* cells per axis */
  int32_t face[3];         /* DN_FACE_* for the x, y and z axis */
  double  dx, dy, dz;      /* cell spacing, as CartesianPatch::computeDeltas (cartesianpatch.cpp:160-165) */
  double  origin[3];       /* lower corner in inertial coordinates */
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

/* Adds a patch; allocates its three fields and active mask on the device.
 * Replaces: GPU_PatchIterator::addPatch + GPU_Patch ctor
 * (iterators/gpu_patchiterator.h:86-95, gpu_patch.h:43-129). */
int dn_patch_add(dn_ctx* ctx, const dn_patch_desc* desc, int* patch_id);

/* DN_FP32 only: FP64 base state the FP32 offsets are stored against, and the
 * per-variable offset quantum is derived from `range` (the largest expected
 * |U - base| per variable).  Optional; dn_patch_upload derives both from the
 * uploaded data when this was not called. */
int dn_patch_set_base(dn_ctx* ctx, int patch_id, const double base[5], const double range[5]);

/* Host -> device copy of field `field` of one patch, [5][ni][nj][nk].
 * Replaces: PatchIterator::updateDevice (gpu_patchiterator.h:114-126). */
int dn_patch_upload(dn_ctx* ctx, int patch_id, int field, const double* host);
int dn_patch_upload_f32(dn_ctx* ctx, int patch_id, int field, const float* host);

/* Device -> host copy of field `field` of one patch, [5][ni][nj][nk].
 * Replaces: PatchIterator::updateHost (gpu_patchiterator.h:106-111). */
int dn_patch_download(dn_ctx* ctx, int patch_id, int field, double* host);
int dn_patch_download_f32(dn_ctx* ctx, int patch_id, int field, float* host);

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

/* One full low-storage RK time step with stage factors alpha[0..n-1]*dt,
 * without the field 0 -> 1 copy (field 1 holds the step-start state after
 * the call, as after the reference's step).
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

/* Number of device kernel launches the context has issued so far. */
int dn_launch_count(const dn_ctx* ctx, int64_t* count);

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
 * resolves the array's device address; make it before any stream capture. */
int dn_field_sums_noalloc(const double* field, int64_t ncells, double dV, double out[5], void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DRNUM_B200_H */
