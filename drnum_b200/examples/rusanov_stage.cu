// Example of a caller-written flux functor on the generic functor stage
// (include/drnum_b200_functor.cuh): a first-order Rusanov (local
// Lax-Friedrichs) flux with zero-flux patch faces, installed into a context
// with dn_set_stage_function.  It plays the part of an application functor
// such as the jet demo's JetFlux (applications/drnumJetDemo/jetflux.h), which
// the reference passes as the OP of GPU_CartesianIterator<5, OP>.
//
// Build (done by python -m drnum_b200.build):
//   nvcc -gencode arch=compute_100a,code=sm_100a -fmad=false -shared -Xcompiler -fPIC \
//        -I include rusanov_stage.cu -o libdn_example_stage.so
#include "drnum_b200_functor.cuh"

namespace {

struct RusanovFirstOrder
{
  static constexpr double R = 287.2, gamma = 1.4, cv = 717.5;

  // physical flux along axis d and the largest wave speed of one state
  __device__ static double flux_and_speed(const double U[5], int d, double F[5])
  {
    const double ir = 1.0/U[0];
    const double vel[3] = {U[1]*ir, U[2]*ir, U[3]*ir};
    const double T = (U[4]*ir - 0.5*(vel[0]*vel[0] + vel[1]*vel[1] + vel[2]*vel[2]))/cv;
    const double p = U[0]*R*T;
    const double un = vel[d];
    F[0] = U[0]*un;
    for (int c = 0; c < 3; ++c) F[1 + c] = U[1 + c]*un + (c == d ? p : 0.0);
    F[4] = (U[4] + p)*un;
    return fabs(un) + sqrt(gamma*R*T);
  }

  template <int D, class P>
  __device__ void face(P* p, size_t i, size_t j, size_t k, double A, double* flux) const
  {
    double UL[5], UR[5], FL[5], FR[5];
    p->getVar(0, D == 0 ? i - 1 : i, D == 1 ? j - 1 : j, D == 2 ? k - 1 : k, UL);
    p->getVar(0, i, j, k, UR);
    const double sl = flux_and_speed(UL, D, FL), sr = flux_and_speed(UR, D, FR);
    const double s = sl > sr ? sl : sr;
    for (int v = 0; v < 5; ++v) flux[v] += A*(0.5*(FL[v] + FR[v]) - 0.5*s*(UR[v] - UL[v]));
  }

  template <class P> __device__ void xField(P* p, size_t i, size_t j, size_t k, double, double, double, double A, double* f) const { face<0>(p, i, j, k, A, f); }
  template <class P> __device__ void yField(P* p, size_t i, size_t j, size_t k, double, double, double, double A, double* f) const { face<1>(p, i, j, k, A, f); }
  template <class P> __device__ void zField(P* p, size_t i, size_t j, size_t k, double, double, double, double A, double* f) const { face<2>(p, i, j, k, A, f); }
  template <class P> __device__ void xWallM(P*, size_t, size_t, size_t, double, double, double, double, double*) const {}
  template <class P> __device__ void xWallP(P*, size_t, size_t, size_t, double, double, double, double, double*) const {}
  template <class P> __device__ void yWallM(P*, size_t, size_t, size_t, double, double, double, double, double*) const {}
  template <class P> __device__ void yWallP(P*, size_t, size_t, size_t, double, double, double, double, double*) const {}
  template <class P> __device__ void zWallM(P*, size_t, size_t, size_t, double, double, double, double, double*) const {}
  template <class P> __device__ void zWallP(P*, size_t, size_t, size_t, double, double, double, double, double*) const {}
};

} // namespace

extern "C" int dn_example_rusanov_stage(void* user, const dn_stage_launch* L)
{
  if (user) ++*static_cast<long long*>(user);   // optional call counter
  return dn::launch_functor_stage(L, RusanovFirstOrder{}) == cudaSuccess ? 0 : -2;
}
