// The reference's own flux functors, compiled for the device against the
// generic functor stage of this repository (include/drnum_b200_functor.cuh).
// Test infrastructure only: built by oracle/build_ref.sh into oracle/_ref/
// from the reference's headers where they lie, it shows that an application
// functor written against DrNUM's patch interface runs unchanged on the
// B200 stage.  Exports stage functions for dn_set_stage_function:
//   dnref_stage_vanleer       VanLeer<5, Upwind2<5, VanAlbada>, PerfectGas>
//                             (fluxes/vanleer.h)
//   dnref_stage_vanleer_visc  the same plus CompressibleViscFlux<5, PerfectGas>
//                             (fluxes/compressibleviscflux.h), the field fluxes of
//                             the jet application's JetFlux (applications/
//                             drnumJetDemo/jetflux.h:23-24, 101-114)
//   dnref_stage_roe           Roe<5, Upwind2<5, VanAlbada>, PerfectGas> (fluxes/roe.h)
//   dnref_stage_roe_smag      the same plus CompressibleSmagorinskyFlux<5, 2400,
//                             PerfectGas> (fluxes/compressiblesmagorinskyflux.h),
//                             the field fluxes of the base-flow application's
//                             BaseFlowFlux (applications/drnumBaseFlowDemo/
//                             baseflowflux.h:26-27)
// Patch faces carry no flux (the periodic and closed cases of the tests).
#include "drnum.h"
#include "perfectgas.h"
#include "reconstruction/upwind2.h"
#include "reconstruction/vanalbada.h"
#include "fluxes/vanleer.h"
#include "fluxes/roe.h"
#include "fluxes/compressibleviscflux.h"
#include "fluxes/compressiblesmagorinskyflux.h"
#include "drnum_b200_functor.cuh"

namespace {

typedef VanLeer<5, Upwind2<5, VanAlbada>, PerfectGas> RefVanLeer;
typedef CompressibleViscFlux<5, PerfectGas> RefVisc;
typedef Roe<5, Upwind2<5, VanAlbada>, PerfectGas> RefRoe;
typedef CompressibleSmagorinskyFlux<5, 2400, PerfectGas> RefSmag;

#define DNREF_NO_WALL(NAME) \
  template <typename P> __device__ void NAME(P*, size_t, size_t, size_t, real, real, real, real, real*) {}

struct VanLeerOnly
{
  RefVanLeer m_Euler;
  template <typename P> __device__ void xField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.xField(p, i, j, k, x, y, z, A, f); }
  template <typename P> __device__ void yField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.yField(p, i, j, k, x, y, z, A, f); }
  template <typename P> __device__ void zField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.zField(p, i, j, k, x, y, z, A, f); }
  DNREF_NO_WALL(xWallM) DNREF_NO_WALL(xWallP) DNREF_NO_WALL(yWallM) DNREF_NO_WALL(yWallP)
  DNREF_NO_WALL(zWallM) DNREF_NO_WALL(zWallP)
};

// JetFlux::xField order: Euler flux, then the viscous flux (jetflux.h:101-114)
struct VanLeerVisc
{
  RefVanLeer m_Euler;
  RefVisc m_Visc;
  template <typename P> __device__ void xField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.xField(p, i, j, k, x, y, z, A, f); m_Visc.xField(p, i, j, k, x, y, z, A, f); }
  template <typename P> __device__ void yField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.yField(p, i, j, k, x, y, z, A, f); m_Visc.yField(p, i, j, k, x, y, z, A, f); }
  template <typename P> __device__ void zField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.zField(p, i, j, k, x, y, z, A, f); m_Visc.zField(p, i, j, k, x, y, z, A, f); }
  DNREF_NO_WALL(xWallM) DNREF_NO_WALL(xWallP) DNREF_NO_WALL(yWallM) DNREF_NO_WALL(yWallP)
  DNREF_NO_WALL(zWallM) DNREF_NO_WALL(zWallP)
};

struct RoeOnly
{
  RefRoe m_Euler;
  template <typename P> __device__ void xField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.xField(p, i, j, k, x, y, z, A, f); }
  template <typename P> __device__ void yField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.yField(p, i, j, k, x, y, z, A, f); }
  template <typename P> __device__ void zField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.zField(p, i, j, k, x, y, z, A, f); }
  DNREF_NO_WALL(xWallM) DNREF_NO_WALL(xWallP) DNREF_NO_WALL(yWallM) DNREF_NO_WALL(yWallP)
  DNREF_NO_WALL(zWallM) DNREF_NO_WALL(zWallP)
};

// BaseFlowFlux::xField order: Euler flux, then the Smagorinsky flux
struct RoeSmag
{
  RefRoe m_Euler;
  RefSmag m_Visc;
  template <typename P> __device__ void xField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.xField(p, i, j, k, x, y, z, A, f); m_Visc.xField(p, i, j, k, x, y, z, A, f); }
  template <typename P> __device__ void yField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.yField(p, i, j, k, x, y, z, A, f); m_Visc.yField(p, i, j, k, x, y, z, A, f); }
  template <typename P> __device__ void zField(P* p, size_t i, size_t j, size_t k, real x, real y, real z, real A, real* f) { m_Euler.zField(p, i, j, k, x, y, z, A, f); m_Visc.zField(p, i, j, k, x, y, z, A, f); }
  DNREF_NO_WALL(xWallM) DNREF_NO_WALL(xWallP) DNREF_NO_WALL(yWallM) DNREF_NO_WALL(yWallP)
  DNREF_NO_WALL(zWallM) DNREF_NO_WALL(zWallP)
};

} // namespace

extern "C" int dnref_stage_vanleer(void*, const dn_stage_launch* L)
{
  return dn::launch_functor_stage(L, VanLeerOnly()) == cudaSuccess ? 0 : -2;
}

extern "C" int dnref_stage_vanleer_visc(void*, const dn_stage_launch* L)
{
  return dn::launch_functor_stage(L, VanLeerVisc()) == cudaSuccess ? 0 : -2;
}

extern "C" int dnref_stage_roe(void*, const dn_stage_launch* L)
{
  return dn::launch_functor_stage(L, RoeOnly()) == cudaSuccess ? 0 : -2;
}

extern "C" int dnref_stage_roe_smag(void*, const dn_stage_launch* L)
{
  return dn::launch_functor_stage(L, RoeSmag()) == cudaSuccess ? 0 : -2;
}
