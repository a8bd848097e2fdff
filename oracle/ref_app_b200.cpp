// A DrNUM application driving drnum_b200 through the C++ binding
// include/drnum_b200_iterator.h: the reference's own PatchGrid,
// CartesianPatch, PatchGrid::computeDependencies and RungeKutta
// (rungekutta.cpp:27-42), with B200_CartesianIterator in place of
// GPU_CartesianIterator and B200_LevelSetBC in place of
// CPU_LevelSetObjectBC<LSOBCCompressibleEulerOp>.
// Test infrastructure only: built by oracle/build_ref.sh against the
// reference's sources, linked with the compiled reference
// (oracle/_ref/libdrnum_ref.so) and with libdrnum_b200.so; the GPU tests
// call the two extern "C" entry points below and compare the results with
// the golden fixtures.

#include "patchgrid.h"
#include "cartesianpatch.h"
#include "rungekutta.h"
#include "levelsetobject.h"
#include "drnum_b200_iterator.h"

#include <cstring>
#include <exception>
#include <sstream>
#include <string>
#include <vector>

namespace {

typedef AusmPlus<5, Upwind2<5, VanAlbada>, PerfectGas> AppAusm;
typedef VanLeer<5, Upwind2<5, VanAlbada>, PerfectGas> AppVanLeer;
typedef Roe<5, Upwind2<5, VanAlbada>, PerfectGas> AppRoe;

// A patch as the grid-file reader sees it (CartesianPatch::readFromFile,
// cartesianpatch.cpp:98-133): origin, base vectors, IO scale, cells, seek
// layers, lengths, solver codes.
CartesianPatch* appPatch(PatchGrid& grid, const double o[3], const int n[3], const int seek[6], const double L[3])
{
  std::ostringstream s;
  s.precision(17);
  s << o[0] << " " << o[1] << " " << o[2] << "  1 0 0  0 1 0  1  " << n[0] << " " << n[1] << " " << n[2] << "  ";
  for (int a = 0; a < 6; ++a) s << seek[a] << " ";
  s << " " << L[0] << " " << L[1] << " " << L[2] << "  0 0 0 0 0 0 0";
  CartesianPatch* p = new CartesianPatch(&grid);
  p->setIndex(grid.insertPatch(p));
  std::istringstream iss(s.str());
  p->readFromFile(iss, 1.0);
  return p;
}

void copyError(const std::exception& e, char* err, int len)
{
  if (err && len > 0) {
    std::strncpy(err, e.what(), size_t(len) - 1);
    err[len - 1] = 0;
  }
}

template <typename OP>
void runSingle(int ni, int nj, int nk, const int* periodic, double hx, double hy, double hz, double* U,
               const unsigned char* active, int steps, double dt, const double* alpha, int n_alpha)
{
  PatchGrid grid;
  grid.setNumberOfFields(3);
  grid.setNumberOfVariables(5);
  grid.defineVectorVar(1);
  const double o[3] = {0, 0, 0}, L[3] = {ni * hx, nj * hy, nk * hz};
  const int n[3] = {ni, nj, nk}, seek[6] = {0, 0, 0, 0, 0, 0};
  CartesianPatch* patch = appPatch(grid, o, n, seek, L);
  const size_t nc = size_t(ni) * nj * nk;
  std::memcpy(patch->getField(0), U, 5 * nc * sizeof(double));
  if (active) {
    for (size_t c = 0; c < nc; ++c) if (!active[c]) patch->getActive()[c] = false;   // Patch::deactivate(c)
  }
  B200_CartesianIterator<5, OP> it(OP(), 0);
  it.setPeriodic(periodic[0] != 0, periodic[1] != 0, periodic[2] != 0);
  it.addPatch(patch);
  it.updateDevice();
  RungeKutta rk;
  for (int q = 0; q < n_alpha; ++q) rk.addAlpha(alpha[q]);
  rk.addIterator(&it);
  for (int s = 0; s < steps; ++s) rk(dt);
  it.updateHost();
  it.sync();
  std::memcpy(U, patch->getField(0), 5 * nc * sizeof(double));
}

} // namespace

extern "C" {

// One patch of ni x nj x nk cells of spacing (hx, hy, hz), periodic axes as
// flagged, advanced `steps` RK steps by the reference's RungeKutta over
// B200_CartesianIterator<5, OP>; scheme 0 AusmPlus, 2 VanLeer, 3 Roe (with
// Upwind2<5, VanAlbada>).  U: [5][ni][nj][nk], in and out; active: one byte
// per cell (0 = Patch::deactivate), or NULL.  Returns 0, or -1 with the
// message in err.
int refapp_run_single(int scheme, int ni, int nj, int nk, const int* periodic, double hx, double hy, double hz,
                      double* U, const unsigned char* active, int steps, double dt, const double* alpha, int n_alpha,
                      char* err, int errlen)
{
  if (sizeof(real) != 8) return -2;
  try {
    if (scheme == 2) runSingle<AppVanLeer>(ni, nj, nk, periodic, hx, hy, hz, U, active, steps, dt, alpha, n_alpha);
    else if (scheme == 3) runSingle<AppRoe>(ni, nj, nk, periodic, hx, hy, hz, U, active, steps, dt, alpha, n_alpha);
    else runSingle<AppAusm>(ni, nj, nk, periodic, hx, hy, hz, U, active, steps, dt, alpha, n_alpha);
  } catch (const std::exception& e) {
    copyError(e, err, errlen);
    return -1;
  }
  return 0;
}

// A patch grid: np patches (n, origin, length [np][3], seek [np][6]) in a
// PatchGrid with the reference's dependencies (computeDependencies(true), 2
// seek layers, padded direct transfer); per patch side a boundary kind
// (DN_BC_*), far-field parameters [np][6][5] and inflow tables (np*6
// pointers, NULL where none); states[np] hold [5][cells] in and out.
// inactive[np] (or NULL) deactivates patches (PatchIterator::deactivatePatch);
// G[np] (or NULL) adds the level-set slip wall: the distance field in
// variable 5, the reference's LevelSetObject over it and B200_LevelSetBC as
// the post-operation.  Advanced `steps`
// steps by RungeKutta.  Returns 0, or -1 with the message in err.
int refapp_run_grid(int np, const int* n, const double* origin, const double* length, const int* seek,
                    const int* bc_kind, const double* bc_params, const double* const* bc_tables,
                    double* const* states, int steps, double dt, const double* alpha, int n_alpha,
                    const int* inactive, const double* const* G, int ls_inner, int ls_outer, double ls_min_rel,
                    char* err, int errlen)
{
  if (sizeof(real) != 8 || np < 1) return -2;
  try {
    PatchGrid grid;
    grid.setNumberOfFields(3);
    grid.setNumberOfVariables(G ? 6 : 5);
    grid.defineVectorVar(1);
    grid.setInterpolateData();
    grid.setNumSeekLayers(2);
    grid.setNumAddProtectLayers(0);
    grid.setTransferType("padded_direct");
    std::vector<CartesianPatch*> patches;
    for (int p = 0; p < np; ++p) patches.push_back(appPatch(grid, origin + 3 * p, n + 3 * p, seek + 6 * p, length + 3 * p));
    grid.computeDependencies(true);
    for (int p = 0; p < np; ++p) {
      const size_t nc = size_t(n[3 * p]) * n[3 * p + 1] * n[3 * p + 2];
      real* f = patches[p]->getField(0);
      std::memcpy(f, states[p], 5 * nc * sizeof(double));
      if (G) {
        for (size_t c = 0; c < nc; ++c) f[5 * nc + c] = G[p] ? G[p][c] : 1.0;
      }
    }
    B200_CartesianIterator<5, AppAusm> it(AppAusm(), 0);
    for (int p = 0; p < np; ++p) it.addPatch(patches[p]);
    for (int p = 0; p < np; ++p) {
      for (int side = 0; side < 6; ++side) {
        const int kind = bc_kind[6 * p + side];
        if (kind == DN_BC_ZERO_FLUX) continue;
        it.setBoundary(size_t(p), side, kind, bc_params + 5 * (6 * p + side), bc_tables[6 * p + side]);
      }
      if (inactive && inactive[p]) it.deactivatePatch(size_t(p));
    }
    it.updateDevice();
    RungeKutta rk;
    for (int q = 0; q < n_alpha; ++q) rk.addAlpha(alpha[q]);
    rk.addIterator(&it);
    // the level-set wall as the applications set it up: a LevelSetObject on
    // the grid's variable 5 (testBlockObjects/main.h:384-388), its layers,
    // and the boundary condition over them as a post-operation
    LevelSetObject* lso = nullptr;
    B200_LevelSetBC<5, AppAusm>* wall = nullptr;
    if (G) {
      lso = new LevelSetObject(nullptr, &grid, 0, 5, size_t(ls_inner), size_t(ls_outer), ls_min_rel, -1.);
      lso->extractBCellLayers();
      wall = new B200_LevelSetBC<5, AppAusm>(it, lso);
      rk.addPostOperation(wall);
    }
    for (int s = 0; s < steps; ++s) rk(dt);
    it.updateHost();
    it.sync();
    delete wall;
    delete lso;
    for (int p = 0; p < np; ++p) {
      const size_t nc = size_t(n[3 * p]) * n[3 * p + 1] * n[3 * p + 2];
      std::memcpy(states[p], patches[p]->getField(0), 5 * nc * sizeof(double));
    }
  } catch (const std::exception& e) {
    copyError(e, err, errlen);
    return -1;
  }
  return 0;
}

} // extern "C"
