// Driver for the compiled reference DrNUM library (FP64), used as the checker
// that pins this repository's oracle restatement and as the CPU baseline.
// Test infrastructure only: it links the reference's own sources (built by
// oracle/build_ref.sh into oracle/_ref/) and exposes a few extern "C" entry
// points that run the reference code paths on caller-provided inputs.
//
// Everything numerical below is done by the reference's own classes:
//   CartesianPatch / PatchGrid           (cartesianpatch.cpp, patchgrid.cpp, patch.cpp)
//   CartesianIterator<5, OP>             (iterators/cartesianiterator.h:87-325)
//   AusmPlus<5, Upwind2<5, VanAlbada>, PerfectGas>  (fluxes/ausmplus.h:39-106)
//   VanLeer / Roe with the same reconstruction        (fluxes/vanleer.h, fluxes/roe.h)
//   RungeKutta                           (rungekutta.cpp:27-42)
// The only pieces written here are harness glue: a periodic ghost-layer copy
// post-operation (the reference has only a k-axis GPU version,
// cartesiancycliccopy.h:51-69) and zero patch-face fluxes, because the
// periodic ghosts overwrite every outer cell anyway.

#include "patchgrid.h"
#include "cartesianpatch.h"
#include "rungekutta.h"
#include "genericoperation.h"
#include "perfectgas.h"
#include "fluxes/ausmplus.h"
#include "fluxes/vanleer.h"
#include "fluxes/roe.h"
#include "fluxes/compressibleviscflux.h"
#include "fluxes/compressiblesmagorinskyflux.h"
#include "fluxes/compressiblefarfieldflux.h"
#include "fluxes/compressibleslipflux.h"
#include "reconstruction/upwind1.h"
#include "reconstruction/upwind2.h"
#include "reconstruction/vanalbada.h"
#include "iterators/cartesianiterator.h"
#include "levelsetobject.h"
#include "cpu_levelsetobjectbc.h"
#include "lsobccompressibleeulerop.h"

#include <chrono>
#include <sstream>
#include <string>
#include <vector>
#include <cstring>
#include <unistd.h>

// utilities.cpp is not compiled (it needs Qt's file classes); this restates
// the one function the compiled sources use (utilities.cpp:95-106).
bool checkVector(vec3_t V)
{
  for (int i = 0; i < 3; i++) {
    if (std::isnan(V[i])) return false;
    if (std::isinf(V[i])) return false;
  }
  return true;
}

namespace {

typedef AusmPlus<5, Upwind2<5, VanAlbada>, PerfectGas> RefAusm;
typedef VanLeer<5, Upwind2<5, VanAlbada>, PerfectGas> RefVanLeer;
typedef Roe<5, Upwind2<5, VanAlbada>, PerfectGas> RefRoe;
typedef CompressibleViscFlux<5, PerfectGas> RefVisc;

// The field fluxes of the jet application's JetFlux: the Euler flux, then
// the viscous flux (applications/drnumJetDemo/jetflux.h:101-114).
struct RefVanLeerVisc
{
  RefVanLeer m_Euler;
  RefVisc m_Visc;
  template <typename P> void xField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.xField(p, i, j, k, x, y, z, A, f); m_Visc.xField(p, i, j, k, x, y, z, A, f); }
  template <typename P> void yField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.yField(p, i, j, k, x, y, z, A, f); m_Visc.yField(p, i, j, k, x, y, z, A, f); }
  template <typename P> void zField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.zField(p, i, j, k, x, y, z, A, f); m_Visc.zField(p, i, j, k, x, y, z, A, f); }
};

// The field fluxes of the base-flow application's BaseFlowFlux: Roe, then the
// Smagorinsky flux with C_s = 0.24 (applications/drnumBaseFlowDemo/
// baseflowflux.h:26-27).
typedef CompressibleSmagorinskyFlux<5, 2400, PerfectGas> RefSmag;
struct RefRoeSmag
{
  RefRoe m_Euler;
  RefSmag m_Visc;
  template <typename P> void xField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.xField(p, i, j, k, x, y, z, A, f); m_Visc.xField(p, i, j, k, x, y, z, A, f); }
  template <typename P> void yField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.yField(p, i, j, k, x, y, z, A, f); m_Visc.yField(p, i, j, k, x, y, z, A, f); }
  template <typename P> void zField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.zField(p, i, j, k, x, y, z, A, f); m_Visc.zField(p, i, j, k, x, y, z, A, f); }
};

// Flux functor with one of the reference's Euler field fluxes and zero
// patch-face fluxes (the ghost layers of periodic axes overwrite the outer
// cells; closed axes are walls with no flux).
template <class E>
struct PeriodicFluxT
{
  E m_Ausm;
  template <typename P> void xField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Ausm.xField(p, i, j, k, x, y, z, A, f); }
  template <typename P> void yField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Ausm.yField(p, i, j, k, x, y, z, A, f); }
  template <typename P> void zField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Ausm.zField(p, i, j, k, x, y, z, A, f); }
  template <typename P> void xWallM(P*, size_t, size_t, size_t, real, real, real, real, real*) {}
  template <typename P> void xWallP(P*, size_t, size_t, size_t, real, real, real, real, real*) {}
  template <typename P> void yWallM(P*, size_t, size_t, size_t, real, real, real, real, real*) {}
  template <typename P> void yWallP(P*, size_t, size_t, size_t, real, real, real, real, real*) {}
  template <typename P> void zWallM(P*, size_t, size_t, size_t, real, real, real, real, real*) {}
  template <typename P> void zWallP(P*, size_t, size_t, size_t, real, real, real, real, real*) {}
};
typedef PeriodicFluxT<RefAusm> PeriodicFlux;

// Patch-face fluxes per patch and side (x-min, x-max, y-min, y-max, z-min,
// z-max): 0 none, 1 the reference's CompressibleFarfieldFlux, 2 its
// CompressibleSlipFlux, 3 a prescribed face state per face (the flux of the
// jet application's JetFlux::xWallM, applications/drnumJetDemo/jetflux.h:
// 165-191, restated here because that class lives in an application).
typedef CompressibleFarfieldFlux<5, Upwind1<5>, PerfectGas> RefFarfield;
typedef CompressibleSlipFlux<5, Upwind1<5>, PerfectGas> RefSlip;

struct SideConfig
{
  int kind[6] = {0, 0, 0, 0, 0, 0};
  RefFarfield farfield[6];
  std::vector<double> table[6];
};

struct GridBC
{
  std::vector<SideConfig> patches;
};

template <class E>
struct SideFluxT
{
  E m_Ausm;
  RefSlip m_Slip;
  GridBC* m_BC = nullptr;

  template <typename P> void xField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Ausm.xField(p, i, j, k, x, y, z, A, f); }
  template <typename P> void yField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Ausm.yField(p, i, j, k, x, y, z, A, f); }
  template <typename P> void zField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Ausm.zField(p, i, j, k, x, y, z, A, f); }

  template <typename P> SideConfig* cfg(P* p)
  {
    if (!m_BC || p->getIndex() >= m_BC->patches.size()) return nullptr;
    return &m_BC->patches[p->getIndex()];
  }

  // prescribed face state: boundary cell (ic, jc, kc), face entry e
  template <typename P> void inflow(P* p, int dir, size_t ic, size_t jc, size_t kc, const double* e, real A, real* flux)
  {
    dim_t<5> dim;
    real var[5];
    real pp, T, u, v, w;
    p->getVar(dim, 0, ic, jc, kc, var);
    PerfectGas::conservativeToPrimitive(var, pp, T, u, v, w);
    if (e[0] == e[0]) pp = e[0];
    T = e[1]; u = e[2]; v = e[3]; w = e[4];
    real un = dir == 0 ? u : (dir == 1 ? v : w);
    flux[0] = A*pp/(PerfectGas::R()*T)*un;
    flux[1] = flux[0]*u;
    flux[2] = flux[0]*v;
    flux[3] = flux[0]*w;
    if (dir == 0) flux[1] = flux[0]*u + A*pp;
    if (dir == 1) flux[2] = flux[0]*v + A*pp;
    if (dir == 2) flux[3] = flux[0]*w + A*pp;
    flux[4] = flux[0]*(PerfectGas::cp()*T + 0.5*(u*u + v*v + w*w));
  }

#define DN_SIDE(NAME, SIDE, DIR, IC, JC, KC, FACE)                                                     \
  template <typename P> void NAME(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) \
  {                                                                                                  \
    SideConfig* c = cfg(p);                                                                          \
    if (!c) return;                                                                                  \
    switch (c->kind[SIDE]) {                                                                         \
      case 1: c->farfield[SIDE].NAME(p, i, j, k, x, y, z, A, f); break;                              \
      case 2: m_Slip.NAME(p, i, j, k, x, y, z, A, f); break;                                         \
      case 3: inflow(p, DIR, IC, JC, KC, &c->table[SIDE][5*(FACE)], A, f); break;                    \
      default: break;                                                                                \
    }                                                                                                \
  }
  DN_SIDE(xWallM, 0, 0, i, j, k, j*p->sizeK() + k)
  DN_SIDE(xWallP, 1, 0, i - 1, j, k, j*p->sizeK() + k)
  DN_SIDE(yWallM, 2, 1, i, j, k, i*p->sizeK() + k)
  DN_SIDE(yWallP, 3, 1, i, j - 1, k, i*p->sizeK() + k)
  DN_SIDE(zWallM, 4, 2, i, j, k, i*p->sizeJ() + j)
  DN_SIDE(zWallP, 5, 2, i, j, k - 1, i*p->sizeJ() + j)
#undef DN_SIDE
};
typedef SideFluxT<RefAusm> SideFlux;

// Periodic ghost copy, field 0, for the axes flagged periodic; each such axis
// carries G ghost layers per side (ghosted size N = n + 2G).
struct PeriodicGhostCopy : public GenericOperation
{
  CartesianPatch* m_P;
  size_t m_G[3];
  PeriodicGhostCopy(CartesianPatch* p, const size_t g[3]) : m_P(p) { for (int a = 0; a < 3; ++a) m_G[a] = g[a]; }
  virtual void operator()()
  {
    CartesianPatch* p = m_P;
    const size_t NI = p->sizeI(), NJ = p->sizeJ(), NK = p->sizeK();
    const size_t ni = NI - 2*m_G[0], nj = NJ - 2*m_G[1], nk = NK - 2*m_G[2];
    for (size_t v = 0; v < 5; ++v) {
      for (size_t g = 0; g < m_G[0]; ++g) {
        for (size_t j = 0; j < NJ; ++j) for (size_t k = 0; k < NK; ++k) {
          p->f(0, v, g, j, k)                = p->f(0, v, g + ni, j, k);
          p->f(0, v, NI - m_G[0] + g, j, k)  = p->f(0, v, m_G[0] + g, j, k);
        }
      }
      for (size_t g = 0; g < m_G[1]; ++g) {
        for (size_t i = 0; i < NI; ++i) for (size_t k = 0; k < NK; ++k) {
          p->f(0, v, i, g, k)                = p->f(0, v, i, g + nj, k);
          p->f(0, v, i, NJ - m_G[1] + g, k)  = p->f(0, v, i, m_G[1] + g, k);
        }
      }
      for (size_t g = 0; g < m_G[2]; ++g) {
        for (size_t i = 0; i < NI; ++i) for (size_t j = 0; j < NJ; ++j) {
          p->f(0, v, i, j, g)                = p->f(0, v, i, j, g + nk);
          p->f(0, v, i, j, NK - m_G[2] + g)  = p->f(0, v, i, j, m_G[2] + g);
        }
      }
    }
  }
};

std::string patchText(double x0, double y0, double z0, size_t ni, size_t nj, size_t nk,
                      const size_t seek[6], double lx, double ly, double lz)
{
  std::ostringstream s;
  s.precision(17);
  s << x0 << " " << y0 << " " << z0 << "  1 0 0  0 1 0  1  "
    << ni << " " << nj << " " << nk << "  "
    << seek[0] << " " << seek[1] << " " << seek[2] << " " << seek[3] << " " << seek[4] << " " << seek[5] << "  "
    << lx << " " << ly << " " << lz << "  0 0 0 0 0 0 0";
  return s.str();
}

CartesianPatch* addPatch(PatchGrid& grid, const std::string& text)
{
  CartesianPatch* p = new CartesianPatch(&grid);
  size_t index = grid.insertPatch(p);
  p->setIndex(index);
  std::istringstream iss(text);
  p->readFromFile(iss, 1.0);
  return p;
}

} // namespace

extern "C" {

// Runs `steps` RK steps (alpha[0..n_alpha-1]) of the reference CPU iterator
// on one patch of ni x nj x nk cells of spacing (hx, hy, hz).  Axes flagged in
// periodic[3] are periodic (two ghost layers refreshed after every stage, as a
// post-operation); the other axes are closed (the reference's own first-order
// edge reconstruction, zero patch-face flux).  active may be NULL.
// init/out: [5][ni][nj][nk] conservative variables (k fastest).
// Returns 0 on success; *seconds = steady_clock time of the RK loop only.
extern "C++" {
template <class E>
int run_impl(int ni, int nj, int nk, const int* periodic, double hx, double hy, double hz,
             const double* init, const unsigned char* active, int steps, double dt,
             const double* alpha, int n_alpha, int threads, double* out, double* seconds)
{
  if (sizeof(real) != 8) return -1;
  if (ni < 1 || nj < 1 || nk < 1 || n_alpha < 1) return -2;
  size_t G[3];
  for (int a = 0; a < 3; ++a) G[a] = (periodic && periodic[a]) ? 2 : 0;
  const size_t NI = ni + 2*G[0], NJ = nj + 2*G[1], NK = nk + 2*G[2];
#ifdef OPEN_MP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  PatchGrid grid;
  grid.setNumberOfFields(3);
  grid.setNumberOfVariables(5);
  grid.defineVectorVar(1);
  size_t seek[6] = {0, 0, 0, 0, 0, 0};
  CartesianPatch* p = addPatch(grid, patchText(0, 0, 0, NI, NJ, NK, seek, NI*hx, NJ*hy, NK*hz));
  const size_t n = size_t(ni)*nj*nk;
  for (size_t v = 0; v < 5; ++v)
    for (size_t i = 0; i < size_t(ni); ++i)
      for (size_t j = 0; j < size_t(nj); ++j)
        for (size_t k = 0; k < size_t(nk); ++k)
          p->f(0, v, i + G[0], j + G[1], k + G[2]) = init[v*n + (i*nj + j)*nk + k];
  if (active) {
    for (size_t i = 0; i < size_t(ni); ++i)
      for (size_t j = 0; j < size_t(nj); ++j)
        for (size_t k = 0; k < size_t(nk); ++k)
          if (!active[(i*nj + j)*nk + k]) p->deactivate(i + G[0], j + G[1], k + G[2]);
  }
  PeriodicGhostCopy ghosts(p, G);
  ghosts();

  PeriodicFluxT<E> flux;
  CartesianIterator<5, PeriodicFluxT<E>> iterator(flux);
  iterator.addPatch(p);
  RungeKutta rk;
  for (int a = 0; a < n_alpha; ++a) rk.addAlpha(alpha[a]);
  rk.addIterator(&iterator);
  rk.addPostOperation(&ghosts);

  auto t0 = std::chrono::steady_clock::now();
  for (int s = 0; s < steps; ++s) rk(dt);
  auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();

  for (size_t v = 0; v < 5; ++v)
    for (size_t i = 0; i < size_t(ni); ++i)
      for (size_t j = 0; j < size_t(nj); ++j)
        for (size_t k = 0; k < size_t(nk); ++k)
          out[v*n + (i*nj + j)*nk + k] = p->f(0, v, i + G[0], j + G[1], k + G[2]);
  return 0;
}

} // extern "C++"

int dnref_run(int ni, int nj, int nk, const int* periodic, double hx, double hy, double hz,
              const double* init, const unsigned char* active, int steps, double dt,
              const double* alpha, int n_alpha, int threads, double* out, double* seconds)
{
  return run_impl<RefAusm>(ni, nj, nk, periodic, hx, hy, hz, init, active, steps, dt, alpha, n_alpha, threads,
                           out, seconds);
}

// dnref_run with the Euler flux `scheme`: 0 AusmPlus, 2 VanLeer, 3 Roe (the
// numbering of DN_FLUX_*; all with Upwind2<5, VanAlbada> and PerfectGas), and
// 4 VanLeer plus CompressibleViscFlux, 5 Roe plus CompressibleSmagorinskyFlux.
int dnref_run_scheme(int scheme, int ni, int nj, int nk, const int* periodic, double hx, double hy, double hz,
                     const double* init, const unsigned char* active, int steps, double dt,
                     const double* alpha, int n_alpha, int threads, double* out, double* seconds)
{
  switch (scheme) {
    case 0: case 1:
      return run_impl<RefAusm>(ni, nj, nk, periodic, hx, hy, hz, init, active, steps, dt, alpha, n_alpha, threads,
                               out, seconds);
    case 2:
      return run_impl<RefVanLeer>(ni, nj, nk, periodic, hx, hy, hz, init, active, steps, dt, alpha, n_alpha,
                                  threads, out, seconds);
    case 3:
      return run_impl<RefRoe>(ni, nj, nk, periodic, hx, hy, hz, init, active, steps, dt, alpha, n_alpha, threads,
                              out, seconds);
    case 4:
      return run_impl<RefVanLeerVisc>(ni, nj, nk, periodic, hx, hy, hz, init, active, steps, dt, alpha, n_alpha,
                                      threads, out, seconds);
    case 5:
      return run_impl<RefRoeSmag>(ni, nj, nk, periodic, hx, hy, hz, init, active, steps, dt, alpha, n_alpha,
                                  threads, out, seconds);
    default:
      return -3;
  }
}

int dnref_real_size() { return int(sizeof(real)); }

// A persistent single-patch run for timing: set up once, step repeatedly.
struct DnRefSession
{
  PatchGrid grid;
  CartesianPatch* patch = nullptr;
  PeriodicGhostCopy* ghosts = nullptr;
  CartesianIterator<5, PeriodicFlux>* iterator = nullptr;
  RungeKutta rk;
  size_t G[3];
};

// The state is converted to `real` cell by cell, so a session also runs in
// the reference's single-precision build (libdrnum_ref_f32.so).
void* dnref_session_create(int ni, int nj, int nk, const int* periodic, double hx, double hy, double hz,
                           const double* init, const double* alpha, int n_alpha, int threads)
{
  if (ni < 1 || nj < 1 || nk < 1 || n_alpha < 1) return nullptr;
#ifdef OPEN_MP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  DnRefSession* s = new DnRefSession();
  for (int a = 0; a < 3; ++a) s->G[a] = (periodic && periodic[a]) ? 2 : 0;
  const size_t NI = ni + 2*s->G[0], NJ = nj + 2*s->G[1], NK = nk + 2*s->G[2];
  s->grid.setNumberOfFields(3);
  s->grid.setNumberOfVariables(5);
  s->grid.defineVectorVar(1);
  size_t seek[6] = {0, 0, 0, 0, 0, 0};
  s->patch = addPatch(s->grid, patchText(0, 0, 0, NI, NJ, NK, seek, NI*hx, NJ*hy, NK*hz));
  const size_t n = size_t(ni)*nj*nk;
  for (size_t v = 0; v < 5; ++v)
    for (size_t i = 0; i < size_t(ni); ++i)
      for (size_t j = 0; j < size_t(nj); ++j)
        for (size_t k = 0; k < size_t(nk); ++k)
          s->patch->f(0, v, i + s->G[0], j + s->G[1], k + s->G[2]) = init[v*n + (i*nj + j)*nk + k];
  s->ghosts = new PeriodicGhostCopy(s->patch, s->G);
  (*s->ghosts)();
  PeriodicFlux flux;
  s->iterator = new CartesianIterator<5, PeriodicFlux>(flux);
  s->iterator->addPatch(s->patch);
  for (int a = 0; a < n_alpha; ++a) s->rk.addAlpha(alpha[a]);
  s->rk.addIterator(s->iterator);
  s->rk.addPostOperation(s->ghosts);
  return s;
}

// Runs `steps` RK steps; returns the steady_clock seconds of RungeKutta::operator() only.
double dnref_session_step(void* session, int steps, double dt)
{
  DnRefSession* s = (DnRefSession*)session;
  auto t0 = std::chrono::steady_clock::now();
  for (int i = 0; i < steps; ++i) s->rk(dt);
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

void dnref_session_destroy(void* session)
{
  DnRefSession* s = (DnRefSession*)session;
  if (!s) return;
  delete s->iterator;
  delete s->ghosts;
  delete s;
}

int dnref_max_threads()
{
#ifdef OPEN_MP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// ---------------------------------------------------------------- patch grids
// A grid of axis-aligned Cartesian patches with overlap interpolation: the
// reference's PatchGrid::computeDependencies builds the donor tables, and
// RungeKutta + CartesianIterator + Patch::accessDonorDataDirect step it.
// Patch faces carry zero flux (closed); receiving cells are overwritten by
// the donor copy after every stage.
void* dnref_grid_create_nv(int np, const int* n, const double* origin, const double* length, const int* seek,
                           int add_protect, int threads, int num_vars);

struct DnRefGrid
{
  PatchGrid grid;
  std::vector<CartesianPatch*> patches;
  GridBC bc;
  LevelSetObject* lso = nullptr;
  CPU_LevelSetObjectBC<LSOBCCompressibleEulerOp>* lsbc = nullptr;
  std::vector<char> inactive;   // patches the runs deactivate (PatchIterator::deactivatePatch)
};

// n[3*np], origin[3*np], length[3*np], seek[6*np] (imin imax jmin jmax kmin kmax)
void* dnref_grid_create(int np, const int* n, const double* origin, const double* length, const int* seek,
                        int add_protect, int threads)
{
  return dnref_grid_create_nv(np, n, origin, length, seek, add_protect, threads, 5);
}

// As dnref_grid_create with num_vars variables per cell (6 keeps the level-set
// field G in variable 5, as the test application does, testBlockObjects/main.h:384-388).
void* dnref_grid_create_nv(int np, const int* n, const double* origin, const double* length, const int* seek,
                           int add_protect, int threads, int num_vars)
{
  if (sizeof(real) != 8 || np < 1) return nullptr;
#ifdef OPEN_MP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  DnRefGrid* g = new DnRefGrid();
  g->grid.setNumberOfFields(3);
  g->grid.setNumberOfVariables(size_t(num_vars));
  g->grid.defineVectorVar(1);
  g->grid.setInterpolateData();
  g->grid.setNumSeekLayers(2);
  g->grid.setNumAddProtectLayers(size_t(add_protect));
  g->grid.setTransferType("padded_direct");
  for (int p = 0; p < np; ++p) {
    size_t sk[6];
    for (int a = 0; a < 6; ++a) sk[a] = size_t(seek[6*p + a]);
    g->patches.push_back(addPatch(g->grid, patchText(origin[3*p], origin[3*p+1], origin[3*p+2],
                                                     n[3*p], n[3*p+1], n[3*p+2], sk,
                                                     length[3*p], length[3*p+1], length[3*p+2])));
  }
  g->grid.computeDependencies(true);
  g->bc.patches.resize(g->patches.size());
  return g;
}

// A grid read from a grid file by the reference's PatchGrid::readGrid
// (patchgrid.cpp:479-557; `relpath` is relative to the working directory, as
// readGrid takes it), set up like dnref_grid_create and with its
// dependencies computed.
void* dnref_grid_read(const char* relpath, double scale, int add_protect, int threads)
{
  if (sizeof(real) != 8 || !relpath) return nullptr;
#ifdef OPEN_MP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  DnRefGrid* g = new DnRefGrid();
  g->grid.setNumberOfFields(3);
  g->grid.setNumberOfVariables(5);
  g->grid.defineVectorVar(1);
  g->grid.setInterpolateData();
  g->grid.setNumSeekLayers(2);
  g->grid.setNumAddProtectLayers(size_t(add_protect));
  g->grid.setTransferType("padded_direct");
  g->grid.readGrid(relpath, scale);
  for (size_t p = 0; p < g->grid.getNumPatches(); ++p)
    g->patches.push_back(dynamic_cast<CartesianPatch*>(g->grid.getPatch(p)));
  g->grid.computeDependencies(true);
  g->bc.patches.resize(g->patches.size());
  return g;
}

int dnref_grid_num_patches(void* handle)
{
  DnRefGrid* g = (DnRefGrid*)handle;
  return g ? int(g->patches.size()) : -1;
}

// Cells, reference point, spacing and solver-code string of patch p.
int dnref_grid_patch_info(void* handle, int p, long long* n, double* origin, double* delta, char* codes, int len)
{
  DnRefGrid* g = (DnRefGrid*)handle;
  if (!g || p < 0 || p >= int(g->patches.size())) return -1;
  CartesianPatch* P = g->patches[p];
  n[0] = (long long)P->sizeI(); n[1] = (long long)P->sizeJ(); n[2] = (long long)P->sizeK();
  origin[0] = P->xo(); origin[1] = P->yo(); origin[2] = P->zo();
  delta[0] = P->dx(); delta[1] = P->dy(); delta[2] = P->dz();
  std::string c = P->accessSolverCodes();
  if (codes && len > 0) std::snprintf(codes, size_t(len), "%s", c.c_str());
  return 0;
}

// Patch-face flux of side `side` of patch p: kind 0 none, 1 far field
// (params p, T, u, v, w), 2 slip wall, 3 face table ([faces][5] p or NaN, T,
// u, v, w; x sides j*nk+k, y sides i*nk+k, z sides i*nj+j).
int dnref_grid_set_bc(void* handle, int p, int side, int kind, const double* params, const double* table)
{
  DnRefGrid* g = (DnRefGrid*)handle;
  if (!g || p < 0 || p >= int(g->patches.size()) || side < 0 || side > 5 || kind < 0 || kind > 3) return -1;
  SideConfig& c = g->bc.patches[p];
  c.kind[side] = kind;
  if (kind == 1) c.farfield[side].setFarfield(params[0], params[1], params[2], params[3], params[4]);
  if (kind == 3) {
    CartesianPatch* P = g->patches[p];
    const int axis = side / 2;
    const size_t n = axis == 0 ? P->sizeJ()*P->sizeK() : (axis == 1 ? P->sizeI()*P->sizeK() : P->sizeI()*P->sizeJ());
    c.table[side].assign(table, table + 5*n);
  }
  return 0;
}

// Donor tables of patch p.  counts[4] = {unique receiving cells, donor
// patches, concatenated receiving cells, concatenated contributions}; the
// arrays may be NULL (counts only).  donor_patch/num_receivers/stride have
// one entry per donor patch.
int dnref_grid_tables(void* handle, int p, long long* counts, unsigned long long* rec_unique,
                      int* donor_patch, long long* num_receivers, int* stride, unsigned long long* rec_concat,
                      unsigned long long* donor_idx, double* weight)
{
  DnRefGrid* g = (DnRefGrid*)handle;
  if (!g || p < 0 || p >= int(g->patches.size())) return -1;
  CartesianPatch* P = g->patches[p];
  counts[0] = (long long)P->getNumReceivingCellsUnique();
  counts[1] = (long long)P->getNumDonorPatches();
  counts[2] = (long long)P->getNumReceivingCellsConcat();
  counts[3] = (long long)P->getNumDonorWIConcat();
  if (!rec_unique) return 0;
  for (size_t i = 0; i < P->getNumReceivingCellsUnique(); ++i) rec_unique[i] = P->getReceivingCellIndicesUnique()[i];
  for (size_t i = 0; i < P->getNumReceivingCellsConcat(); ++i) rec_concat[i] = P->getReceivingCellIndicesConcat()[i];
  for (size_t i = 0; i < P->getNumDonorWIConcat(); ++i) {
    donor_idx[i] = P->getDonorIndexConcat()[i];
    weight[i] = P->getDonorWeightConcat()[i];
  }
  for (size_t d = 0; d < P->getNumDonorPatches(); ++d) {
    const donor_t& dn = P->getDonors()[d];
    int idx = -1;
    for (size_t q = 0; q < g->patches.size(); ++q) if (g->patches[q]->getField(0) == dn.data) idx = int(q);
    donor_patch[d] = idx;
    num_receivers[d] = (long long)dn.num_receiver_cells;
    stride[d] = int(dn.stride);
    const bool identity = dn.axx == 1 && dn.ayy == 1 && dn.azz == 1 && dn.axy == 0 && dn.axz == 0 &&
                          dn.ayx == 0 && dn.ayz == 0 && dn.azx == 0 && dn.azy == 0;
    if (!identity) return -2;   // axis-aligned patches only
  }
  return 0;
}

// Level-set slip wall: G per patch (NULL entries: no wall, G = 1) into
// variable 5 of field 0, the reference's LevelSetObject classification
// (extractBCellLayers) and CPU_LevelSetObjectBC<LSOBCCompressibleEulerOp>
// with abuse field 2 as a post-operation of every stage.  Needs num_vars 6.
int dnref_grid_levelset(void* handle, const double* const* G, int num_inner, int num_outer, double min_inner_rel_dist)
{
  DnRefGrid* g = (DnRefGrid*)handle;
  if (!g || g->patches.empty() || g->patches[0]->numVariables() < 6) return -1;
  for (size_t p = 0; p < g->patches.size(); ++p) {
    CartesianPatch* P = g->patches[p];
    real* var = P->getVariable(0, 5);
    for (size_t c = 0; c < P->variableSize(); ++c) var[c] = G[p] ? G[p][c] : 1.0;
  }
  g->lso = new LevelSetObject(nullptr, &g->grid, 0, 5, size_t(num_inner), size_t(num_outer), min_inner_rel_dist, -1.);
  g->lso->extractBCellLayers();
  LSOBCCompressibleEulerOp op;
  g->lsbc = new CPU_LevelSetObjectBC<LSOBCCompressibleEulerOp>(0, g->lso, 2, op);
  g->lsbc->transferCellLayerData();
  return 0;
}

// One layer of patch p's classification: *n cells; arrays may be NULL.
int dnref_grid_levelset_layer(void* handle, int p, int inner, int layer, long long* n, unsigned long long* cells,
                              double* gv, double* grad, unsigned long long* donors, double* weights)
{
  DnRefGrid* g = (DnRefGrid*)handle;
  if (!g || !g->lso || p < 0 || p >= int(g->patches.size())) return -1;
  vector<vector<vector<LSLayerDataExtrapol> > >& L =
      inner ? g->lso->getInnerCellsLayers() : g->lso->getOuterCellsLayers();
  if (layer < 0 || layer >= int(L[p].size())) return -2;
  const vector<LSLayerDataExtrapol>& cl = L[p][layer];
  *n = (long long)cl.size();
  for (size_t q = 0; q < cl.size(); ++q) {
    if (cells) cells[q] = cl[q].m_Cell;
    if (gv) gv[q] = cl[q].m_G;
    if (grad) { grad[3*q] = cl[q].m_Gx; grad[3*q + 1] = cl[q].m_Gy; grad[3*q + 2] = cl[q].m_Gz; }
    for (int t = 0; t < 8; ++t) {
      if (donors) donors[8*q + t] = inner ? cl[q].m_MirrorDonor[t] : 0;
      if (weights) weights[8*q + t] = inner ? cl[q].m_MirrorWeight[t] : 0.;
    }
  }
  return 0;
}

// Field 0 of patch p, [5][ni][nj][nk].
int dnref_grid_set_state(void* handle, int p, const double* U)
{
  DnRefGrid* g = (DnRefGrid*)handle;
  if (!g || p < 0 || p >= int(g->patches.size())) return -1;
  CartesianPatch* P = g->patches[p];
  const size_t n = P->sizeI()*P->sizeJ()*P->sizeK();
  for (size_t v = 0; v < 5; ++v)
    for (size_t c = 0; c < n; ++c) P->getVariable(0, v)[c] = U[v*n + c];
  return 0;
}

int dnref_grid_get_state(void* handle, int p, double* U)
{
  DnRefGrid* g = (DnRefGrid*)handle;
  if (!g || p < 0 || p >= int(g->patches.size())) return -1;
  CartesianPatch* P = g->patches[p];
  const size_t n = P->sizeI()*P->sizeJ()*P->sizeK();
  for (size_t v = 0; v < 5; ++v)
    for (size_t c = 0; c < n; ++c) U[v*n + c] = P->getVariable(0, v)[c];
  return 0;
}

// Donor copy into field `field` of every patch (PatchIterator::copyDonorData).
int dnref_grid_copy_donor_data(void* handle, int field)
{
  DnRefGrid* g = (DnRefGrid*)handle;
  if (!g) return -1;
  for (size_t p = 0; p < g->patches.size(); ++p) g->patches[p]->accessDonorDataDirect(size_t(field));
  return 0;
}

extern "C++" {
template <class E>
int grid_run_impl(DnRefGrid* g, int steps, double dt, const double* alpha, int n_alpha, double* seconds)
{
  SideFluxT<E> flux;
  flux.m_BC = &g->bc;
  CartesianIterator<5, SideFluxT<E>> iterator(flux);
  for (size_t p = 0; p < g->patches.size(); ++p) iterator.addPatch(g->patches[p]);
  for (size_t p = 0; p < g->inactive.size(); ++p) if (g->inactive[p]) iterator.deactivatePatch(p);
  RungeKutta rk;
  for (int a = 0; a < n_alpha; ++a) rk.addAlpha(alpha[a]);
  rk.addIterator(&iterator);
  if (g->lsbc) rk.addPostOperation(g->lsbc);
  auto t0 = std::chrono::steady_clock::now();
  for (int s = 0; s < steps; ++s) rk(dt);
  auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  return 0;
}
} // extern "C++"

// Marks patch p inactive (1) or active (0) for the following runs: the
// iterator's deactivatePatch (iterators/patchiterator.h:127-133).
int dnref_grid_deactivate(void* handle, int p, int inactive)
{
  DnRefGrid* g = (DnRefGrid*)handle;
  if (!g || p < 0 || p >= int(g->patches.size())) return -1;
  g->inactive.resize(g->patches.size(), 0);
  g->inactive[p] = char(inactive != 0);
  return 0;
}

// `steps` RK steps of all patches with the Euler flux `scheme` (as in
// dnref_run_scheme); *seconds = time of RungeKutta::operator() only.
int dnref_grid_run_scheme(void* handle, int scheme, int steps, double dt, const double* alpha, int n_alpha,
                          double* seconds)
{
  DnRefGrid* g = (DnRefGrid*)handle;
  if (!g || n_alpha < 1) return -1;
  switch (scheme) {
    case 0: case 1: return grid_run_impl<RefAusm>(g, steps, dt, alpha, n_alpha, seconds);
    case 2: return grid_run_impl<RefVanLeer>(g, steps, dt, alpha, n_alpha, seconds);
    case 3: return grid_run_impl<RefRoe>(g, steps, dt, alpha, n_alpha, seconds);
    default: return -3;
  }
}

// `steps` RK steps of all patches (AUSM+); *seconds = time of RungeKutta::operator() only.
int dnref_grid_run(void* handle, int steps, double dt, const double* alpha, int n_alpha, double* seconds)
{
  return dnref_grid_run_scheme(handle, 0, steps, dt, alpha, n_alpha, seconds);
}

void dnref_grid_destroy(void* handle)
{
  delete (DnRefGrid*)handle;
}

} // extern "C"
