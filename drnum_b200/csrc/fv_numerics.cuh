// Face numerics of DrNUM's Euler path: MUSCL Upwind2 reconstruction on
// conservative variables with the van Albada limiter, conversion to
// primitives, and the AUSM+ face flux.  Written as device functions that a
// stage kernel evaluates once per face.
//
// The expression order follows the reference term by term so that the FP64
// instantiation, compiled without FMA contraction, reproduces the reference
// CPU iterator bit for bit:
//   nonZero                      drnum.h:256-263
//   VanAlbada::lim               reconstruction/vanalbada.h:28-33
//   Upwind2::project             reconstruction/upwind2.h:29-52
//   COMPRESSIBLE_*_VARS          fluxes/compressibleflux.h:236-271
//   M1, M2, M4, P5               fluxes/compressibleflux.h:46-75
//   AusmPlus::x/y/zField         fluxes/ausmplus.h:39-106
//   PerfectGas constants         perfectgas.h:31-34 (R = 287.2, gamma = 1.4,
//                                cv = 717.5; kept as given, cp - cv != R)
#pragma once

namespace dn {

struct Gas {
  static constexpr double R = 287.2;
  static constexpr double gamma = 1.4;
  static constexpr double cv = 717.5;
};

template <typename T> __device__ __forceinline__ T dn_abs(T x);
template <> __device__ __forceinline__ double dn_abs<double>(double x) { return fabs(x); }
template <> __device__ __forceinline__ float dn_abs<float>(float x) { return fabsf(x); }

template <typename T> __device__ __forceinline__ T dn_sqrt(T x);
template <> __device__ __forceinline__ double dn_sqrt<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float dn_sqrt<float>(float x) { return sqrtf(x); }

// nonZero(x, eps): drnum.h:256-263
template <typename T>
__device__ __forceinline__ T non_zero(T x, T eps)
{
  if (x < T(0)) {
    return (-eps < x) ? -eps : x;
  }
  return (eps > x) ? eps : x;
}

// VanAlbada::lim(delta1, delta2): vanalbada.h:28-33
template <typename T>
__device__ __forceinline__ T van_albada(T d1, T d2)
{
  T r = d2 / non_zero(d1, T(1e-10));
  return (r*r + r) / (r*r + T(1));
}

// AUSM polynomials, compressibleflux.h:46-75; s is +1 or -1.
template <typename T> __device__ __forceinline__ T ausm_m1(T M, T s) { return T(0.5)*(M + s*dn_abs(M)); }
template <typename T> __device__ __forceinline__ T ausm_m2(T M, T s) { T q = M + s; return T(0.25)*s*(q*q); }
template <typename T>
__device__ __forceinline__ T ausm_m4(T M, T s)
{
  if (dn_abs(M) >= T(1)) return ausm_m1(M, s);
  return ausm_m2(M, s)*(T(1) - T(2)*s*ausm_m2(M, -s));
}
template <typename T>
__device__ __forceinline__ T ausm_p5(T M, T s)
{
  if (dn_abs(M) >= T(1)) return ausm_m1(M, s)/M;
  return ausm_m2(M, s)*((T(2)*s - M) - T(3)*s*M*ausm_m2(M, -s));
}

// Upwind2 left/right state of one face along one axis.
//   um2, um1 | up0, up1   (cells c-2, c-1 | c, c+1 along the axis)
// Left state  = project(c1 = c-1, c2 = c,   c0 = c-2)
// Right state = project(c1 = c,   c2 = c-1, c0 = c+1)
// second_l / second_r are false where c0 is outside a closed patch
// (upwind2.h:39-42: the state stays first order).
template <typename T>
__device__ __forceinline__ T upwind2_left(T um2, T um1, T up0, bool second)
{
  T var = um1;
  if (second) {
    T delta01 = um1 - um2;
    T delta12 = up0 - um1;
    var += T(0.5)*van_albada(delta01, delta12)*delta01;
  }
  return var;
}
template <typename T>
__device__ __forceinline__ T upwind2_right(T um1, T up0, T up1, bool second)
{
  T var = up0;
  if (second) {
    T delta01 = up0 - up1;
    T delta12 = um1 - up0;
    var += T(0.5)*van_albada(delta01, delta12)*delta01;
  }
  return var;
}

// Conservative -> primitive conversion of one face side
// (COMPRESSIBLE_LEFT_VARS / _RIGHT_VARS, compressibleflux.h:236-271).
template <typename T>
struct FaceSide {
  T r, u, v, w, p, a, H;
};

template <typename T>
__device__ __forceinline__ FaceSide<T> face_side(const T var[5])
{
  FaceSide<T> s;
  T r  = var[0];
  T ir = T(1.0)/r;
  T ru = var[1];
  T rv = var[2];
  T rw = var[3];
  T u  = ru*ir;
  T v  = rv*ir;
  T w  = rw*ir;
  T rE = var[4];
  T Tt = (rE*ir - T(0.5)*(u*u + v*v + w*w))/T(Gas::cv);
  T p  = r*T(Gas::R)*Tt;
  T a  = dn_sqrt(T(Gas::gamma)*T(Gas::R)*Tt);
  T H  = (rE + p)/r;
  s.r = r; s.u = u; s.v = v; s.w = w; s.p = p; s.a = a; s.H = H;
  return s;
}

// AusmPlus face flux through a face of area A with normal along axis DIR
// (0 = x, 1 = y, 2 = z), ausmplus.h:39-106.  flux[0..4] is overwritten.
template <int DIR, typename T>
__device__ __forceinline__ void ausm_plus(const FaceSide<T>& L, const FaceSide<T>& Rs, T A, T flux[5])
{
  const T un_l = DIR == 0 ? L.u : (DIR == 1 ? L.v : L.w);
  const T un_r = DIR == 0 ? Rs.u : (DIR == 1 ? Rs.v : Rs.w);
  T a  = T(0.5)*(L.a + Rs.a);
  T M  = ausm_m4(un_l/a, T(1)) + ausm_m4(un_r/a, T(-1));
  T Mp = T(0.5)*(M + dn_abs(M));
  T Mm = T(0.5)*(M - dn_abs(M));
  T p  = ausm_p5(un_l/a, T(1))*L.p + ausm_p5(un_r/a, T(-1))*Rs.p;
  T f0 = a*A*(L.r*Mp + Rs.r*Mm);
  T h0 = T(0.5)*f0;
  T g0 = T(0.5)*dn_abs(f0);
  flux[0] = f0;
  if (DIR == 0) flux[1] = h0*(L.u + Rs.u) + A*p - g0*(Rs.u - L.u);
  else          flux[1] = h0*(L.u + Rs.u)       - g0*(Rs.u - L.u);
  if (DIR == 1) flux[2] = h0*(L.v + Rs.v) + A*p - g0*(Rs.v - L.v);
  else          flux[2] = h0*(L.v + Rs.v)       - g0*(Rs.v - L.v);
  if (DIR == 2) flux[3] = h0*(L.w + Rs.w) + A*p - g0*(Rs.w - L.w);
  else          flux[3] = h0*(L.w + Rs.w)       - g0*(Rs.w - L.w);
  flux[4] = h0*(L.H + Rs.H) - g0*(Rs.H - L.H);
}

} // namespace dn
