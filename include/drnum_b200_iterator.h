/*
 * drnum_b200_iterator.h — DrNUM's iterator API on drnum_b200 (header-only C++).
 *
 * A DrNUM application keeps its run(): PatchGrid set-up, RungeKutta loop,
 * post-operations.  It uses B200_CartesianIterator<5, OP> where it used
 * GPU_CartesianIterator<5, OP> (iterators/gpu_cartesianiterator.h:29-40) and
 * B200_LevelSetBC where it used CPU_LevelSetObjectBC<LSOBCCompressibleEulerOp>
 * (cpu_levelsetobjectbc.h:58-90).  The class derives from the reference's
 * PatchIterator (iterators/patchiterator.h:28-69), so RungeKutta /
 * TimeIntegration (rungekutta.cpp:27-42, timeintegration.cpp:28-55) drive it
 * through the same virtuals they drive the reference's iterators with:
 *
 *   PatchIterator virtual          drnum_b200 call
 *   addPatch(Patch*)               dn_patch_add (CartesianPatch geometry)
 *   updateDevice / updateHost      dn_patch_upload / dn_patch_download of fields 0 and 1
 *                                  (field 2 is the stages' scratch on both sides);
 *                                  inactive cells (Patch::deactivate) as dn_patch_set_active
 *   compute(factor, patches)       dn_compute, or dn_compute_patches for a subset;
 *                                  activatePatch/deactivatePatch flags (read here,
 *                                  at compute time, like gpu_cartesianiterator.h:226)
 *                                  become dn_patch_activate
 *   copyField(src, dst)            dn_copy_field
 *   copyDonorData(field)           dn_copy_donor_data, with the donor tables the
 *                                  reference's PatchGrid::computeDependencies built
 *                                  (handed over on first use, dn_patch_set_donors)
 *
 * The flux functor OP selects the scheme: AusmPlus<5, Upwind2<5, VanAlbada>,
 * PerfectGas> runs the fused AUSM+ stage (FP64 build: the plain FP64 path,
 * bitwise equal to the reference's CPU iterator; float build: the FP32-bulk
 * path), VanLeer and Roe with the same reconstruction the FP64 functor stage
 * (DN_FLUX_VANLEER, DN_FLUX_ROE).  The functor's patch-face fluxes
 * (x/y/zWall{M,P}) are given per patch side with setBoundary (DN_BC_* kinds:
 * far field, slip wall, prescribed inflow state as JetFlux::xWallM).
 * Periodic axes (the reference's CartesianCyclicCopy post-operation,
 * cartesiancycliccopy.h:51-69) are patch properties here: setPeriodic before
 * addPatch.
 *
 * Errors: the reference prints and exits (BUG / ERROR, drnum.h:109-128);
 * here a failing call throws std::runtime_error with the library's message.
 *
 * Needs the reference's include tree (src/drnumlib on the include path) and
 * libdrnum_b200.so at link time.
 */
#ifndef DRNUM_B200_ITERATOR_H
#define DRNUM_B200_ITERATOR_H

#include "drnum_b200.h"

#include "iterators/patchiterator.h"
#include "cartesianpatch.h"
#include "genericoperation.h"
#include "levelsetobject.h"
#include "lslayerdataextrapol.h"
#include "perfectgas.h"
#include "fluxes/ausmplus.h"
#include "fluxes/vanleer.h"
#include "fluxes/roe.h"
#include "reconstruction/upwind2.h"
#include "reconstruction/vanalbada.h"

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

/* Scheme of a flux functor type: -1 for functors the library does not
 * carry (they run through dn_set_stage_function and the device functor
 * header include/drnum_b200_functor.cuh instead). */
template <typename OP> struct B200FluxScheme { static const int value = -1; };
template <> struct B200FluxScheme<AusmPlus<5, Upwind2<5, VanAlbada>, PerfectGas> > { static const int value = DN_FLUX_AUSMPLUS; };
template <> struct B200FluxScheme<VanLeer<5, Upwind2<5, VanAlbada>, PerfectGas> > { static const int value = DN_FLUX_VANLEER; };
template <> struct B200FluxScheme<Roe<5, Upwind2<5, VanAlbada>, PerfectGas> > { static const int value = DN_FLUX_ROE; };

template <unsigned int DIM, typename OP>
class B200_CartesianIterator : public PatchIterator
{
public:
  /* As GPU_CartesianIterator<DIM, OP>(OP op, int cuda_device, size_t
   * thread_limit) (gpu_cartesianiterator.h:37); the thread limit has no
   * counterpart (the library sizes its launches itself).  The precision
   * follows `real`: FP64 for the double build, FP32 bulk for float. */
  B200_CartesianIterator(OP, int cuda_device = 0, size_t = 0)
  {
    static_assert(DIM == 5, "drnum_b200 carries the five compressible Euler variables");
    check(nullptr, dn_ctx_create(cuda_device, sizeof(real) == 8 ? DN_FP64 : DN_FP32, &m_Ctx));
    const int scheme = B200FluxScheme<OP>::value;
    if (scheme < 0) fail("flux functor without a drnum_b200 scheme: use dn_set_stage_function");
    if (scheme != DN_FLUX_AUSMPLUS) check(m_Ctx, dn_set_flux_scheme(m_Ctx, scheme));
  }

  ~B200_CartesianIterator() { dn_ctx_destroy(m_Ctx); }
  B200_CartesianIterator(const B200_CartesianIterator&) = delete;
  B200_CartesianIterator& operator=(const B200_CartesianIterator&) = delete;

  dn_ctx* context() { return m_Ctx; }

  /* Axes of the patches added after this call that are periodic. */
  void setPeriodic(bool x, bool y, bool z)
  {
    m_Face[0] = x ? DN_FACE_PERIODIC : DN_FACE_CLOSED;
    m_Face[1] = y ? DN_FACE_PERIODIC : DN_FACE_CLOSED;
    m_Face[2] = z ? DN_FACE_PERIODIC : DN_FACE_CLOSED;
  }

  virtual void addPatch(Patch* patch)
  {
    CartesianPatch* cp = dynamic_cast<CartesianPatch*>(patch);
    if (!cp) fail("B200_CartesianIterator takes Cartesian patches");
    if (cp->numVariables() < DIM) fail("a patch needs at least five variables");
    dn_patch_desc d = {};
    d.ni = int32_t(cp->sizeI());
    d.nj = int32_t(cp->sizeJ());
    d.nk = int32_t(cp->sizeK());
    for (int a = 0; a < 3; ++a) d.face[a] = m_Face[a];
    d.dx = cp->dx();
    d.dy = cp->dy();
    d.dz = cp->dz();
    int id = -1;
    check(m_Ctx, dn_patch_add(m_Ctx, &d, &id));
    PatchIterator::addPatch(patch);
    m_Cartesian.push_back(cp);
    m_Active.push_back(1);
    m_Masked.push_back(0);
    m_DonorsSet = false;
  }

  /* Flux through side `side` (0 x-min .. 5 z-max) of patch i_patch: the
   * functor's wall method there.  kind DN_BC_*; params/table as
   * dn_patch_set_bc. */
  void setBoundary(size_t i_patch, int side, int kind, const double* params = nullptr, const double* table = nullptr)
  {
    check(m_Ctx, dn_patch_set_bc(m_Ctx, int(i_patch), side, kind, params, table));
  }

  /* GPU_PatchIterator::updateDevice (gpu_patchiterator.h:114-126): fields
   * 0 and 1 of every patch to the device (field 2 is stage scratch). */
  virtual void updateDevice()
  {
    for (size_t p = 0; p < numPatches(); ++p) {
      for (size_t f = 0; f < fields(p); ++f) upload(p, f);
      uploadActive(p);
    }
    setDonors();
  }

  /* GPU_PatchIterator::updateHost (gpu_patchiterator.h:106-111). */
  virtual void updateHost()
  {
    for (size_t p = 0; p < numPatches(); ++p) {
      for (size_t f = 0; f < fields(p); ++f) download(p, f);
    }
  }

  virtual void compute(real factor, const vector<size_t>& patches)
  {
    setDonors();
    for (size_t p = 0; p < numPatches(); ++p) {
      const int a = patchActive(p) ? 1 : 0;
      if (a != m_Active[p]) {
        check(m_Ctx, dn_patch_activate(m_Ctx, int(p), a));
        m_Active[p] = a;
      }
    }
    bool all = patches.size() == numPatches();
    for (size_t q = 0; all && q < patches.size(); ++q) all = patches[q] == q;
    if (all) {
      check(m_Ctx, dn_compute(m_Ctx, double(factor)));
      return;
    }
    std::vector<int32_t> ids(patches.begin(), patches.end());
    check(m_Ctx, dn_compute_patches(m_Ctx, double(factor), ids.data(), int(ids.size())));
  }

  virtual void copyField(size_t i_src, size_t i_dst)
  {
    check(m_Ctx, dn_copy_field(m_Ctx, int(i_src), int(i_dst)));
  }

  virtual void copyDonorData(size_t i_field)
  {
    setDonors();
    check(m_Ctx, dn_copy_donor_data(m_Ctx, int(i_field)));
  }

  /* Waits for the queued device work and reports device-side errors. */
  void sync() { check(m_Ctx, dn_sync(m_Ctx)); }

  static void check(dn_ctx* c, int status)
  {
    if (status == DN_OK) return;
    char msg[512] = {0};
    if (c) dn_last_error(c, msg, sizeof msg);
    throw std::runtime_error(std::string("drnum_b200: ") + (msg[0] ? msg : "error ") +
                             (msg[0] ? "" : std::to_string(status)));
  }

private:
  dn_ctx* m_Ctx = nullptr;
  int m_Face[3] = {DN_FACE_CLOSED, DN_FACE_CLOSED, DN_FACE_CLOSED};
  vector<CartesianPatch*> m_Cartesian;
  vector<int> m_Active;            // activity flags as last handed to the library
  vector<int> m_Masked;            // patches whose cell mask was handed over
  bool m_DonorsSet = false;

  static void fail(const char* what) { throw std::runtime_error(std::string("drnum_b200: ") + what); }

  size_t fields(size_t p) { return m_Cartesian[p]->numFields() < 2 ? m_Cartesian[p]->numFields() : 2; }

  // the first five variables of field f (the variable-major layout of
  // Patch::getField makes them one contiguous block)
  void upload(size_t p, size_t f)
  {
    real* h = m_Cartesian[p]->getField(f);
    if (sizeof(real) == 8) check(m_Ctx, dn_patch_upload(m_Ctx, int(p), int(f), reinterpret_cast<const double*>(h)));
    else check(m_Ctx, dn_patch_upload_f32(m_Ctx, int(p), int(f), reinterpret_cast<const float*>(h)));
  }

  // the patch's per-cell activity (Patch::getActive, patch_common.h:127-130),
  // handed over once a cell is inactive (or was)
  void uploadActive(size_t p)
  {
    CartesianPatch* P = m_Cartesian[p];
    const size_t nc = P->sizeI() * P->sizeJ() * P->sizeK();
    const bool* a = P->getActive();
    bool all = true;
    for (size_t c = 0; all && c < nc; ++c) all = a[c];
    if (all && !m_Masked[p]) return;
    std::vector<uint8_t> mask(nc);
    for (size_t c = 0; c < nc; ++c) mask[c] = a[c] ? 1 : 0;
    check(m_Ctx, dn_patch_set_active(m_Ctx, int(p), mask.data()));
    m_Masked[p] = 1;
  }

  void download(size_t p, size_t f)
  {
    real* h = m_Cartesian[p]->getField(f);
    if (sizeof(real) == 8) check(m_Ctx, dn_patch_download(m_Ctx, int(p), int(f), reinterpret_cast<double*>(h)));
    else check(m_Ctx, dn_patch_download_f32(m_Ctx, int(p), int(f), reinterpret_cast<float*>(h)));
  }

  // The donor tables PatchGrid::computeDependencies left in the patches
  // (Patch::buildDonorTransferData, patch.cpp:128-218), once: donor_t::data
  // (the donor's field 0) names the donor patch.  Axis-aligned patches only
  // (the donor copy applies no vector rotation).
  void setDonors()
  {
    if (m_DonorsSet) return;
    for (size_t p = 0; p < numPatches(); ++p) {
      CartesianPatch* P = m_Cartesian[p];
      const int64_t counts[4] = {int64_t(P->getNumReceivingCellsUnique()), int64_t(P->getNumDonorPatches()),
                                 int64_t(P->getNumReceivingCellsConcat()), int64_t(P->getNumDonorWIConcat())};
      if (counts[1] == 0) continue;
      std::vector<int32_t> donor(counts[1]), stride(counts[1]);
      std::vector<int64_t> nrec(counts[1]);
      for (int64_t d = 0; d < counts[1]; ++d) {
        const donor_t& t = P->getDonors()[d];
        donor[d] = -1;
        for (size_t q = 0; q < numPatches(); ++q)
          if (m_Cartesian[q]->getField(0) == t.data) donor[d] = int32_t(q);
        if (donor[d] < 0) fail("a donor patch is not part of this iterator");
        if (!(t.axx == 1 && t.ayy == 1 && t.azz == 1 && t.axy == 0 && t.axz == 0 && t.ayx == 0 && t.ayz == 0 &&
              t.azx == 0 && t.azy == 0))
          fail("rotated donor patches are not supported");
        nrec[d] = int64_t(t.num_receiver_cells);
        stride[d] = int32_t(t.stride);
      }
      std::vector<uint64_t> ru(P->getReceivingCellIndicesUnique(), P->getReceivingCellIndicesUnique() + counts[0]);
      std::vector<uint64_t> rc(P->getReceivingCellIndicesConcat(), P->getReceivingCellIndicesConcat() + counts[2]);
      std::vector<uint64_t> di(P->getDonorIndexConcat(), P->getDonorIndexConcat() + counts[3]);
      std::vector<double> w(P->getDonorWeightConcat(), P->getDonorWeightConcat() + counts[3]);
      check(m_Ctx, dn_patch_set_donors(m_Ctx, int(p), counts, ru.data(), donor.data(), nrec.data(), stride.data(),
                                       rc.data(), di.data(), w.data()));
    }
    m_DonorsSet = true;
  }
};

/* The slip-wall level-set condition as a post-operation, in place of
 * CPU_LevelSetObjectBC<LSOBCCompressibleEulerOp>(field, levelset_object, ...)
 * (cpu_levelsetobjectbc.h:58-90): it takes the application's LevelSetObject
 * (levelsetobject.cpp:24-388) after extractBCellLayers and hands its inner
 * layers (cells, G, gradient, mirror donors and weights, as
 * LevelSetObjectBC::transferCellLayerData reads them, levelsetobjectbc.cpp:38-134)
 * to the library once; operator() applies the mirror condition to field 0 of
 * every patch of the iterator. */
template <unsigned int DIM, typename OP>
class B200_LevelSetBC : public GenericOperation
{
public:
  B200_LevelSetBC(B200_CartesianIterator<DIM, OP>& it, LevelSetObject* levelset_object) : m_It(it)
  {
    PatchGrid* grid = levelset_object->getPatchGrid();
    vector<vector<vector<LSLayerDataExtrapol> > >& L = levelset_object->getInnerCellsLayers();
    for (size_t p = 0; p < it.numPatches(); ++p) {
      size_t q = 0;   // the patch's index in the level-set object's grid
      while (q < grid->getNumPatches() && grid->getPatch(q) != it.getPatch(p)) ++q;
      if (q == grid->getNumPatches() || q >= L.size()) continue;
      std::vector<int64_t> counts;
      std::vector<uint64_t> cells, donors;
      std::vector<double> g, grad, weights;
      for (size_t layer = 0; layer < L[q].size(); ++layer) {
        counts.push_back(int64_t(L[q][layer].size()));
        for (const LSLayerDataExtrapol& c : L[q][layer]) {
          cells.push_back(c.m_Cell);
          g.push_back(c.m_G);
          grad.push_back(c.m_Gx);
          grad.push_back(c.m_Gy);
          grad.push_back(c.m_Gz);
          for (int t = 0; t < 8; ++t) {
            donors.push_back(c.m_MirrorDonor[t]);
            weights.push_back(c.m_MirrorWeight[t]);
          }
        }
      }
      B200_CartesianIterator<DIM, OP>::check(
          it.context(), dn_patch_set_levelset_layers(it.context(), int(p), int(counts.size()), counts.data(),
                                                     cells.data(), g.data(), grad.data(), donors.data(),
                                                     weights.data()));
    }
  }

  virtual void operator()()
  {
    B200_CartesianIterator<DIM, OP>::check(m_It.context(), dn_apply_levelset_bc(m_It.context(), 0));
  }

private:
  B200_CartesianIterator<DIM, OP>& m_It;
};

#endif /* DRNUM_B200_ITERATOR_H */
