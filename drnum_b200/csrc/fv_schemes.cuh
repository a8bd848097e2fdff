// Euler flux schemes of DrNUM's applications as flux functors for the
// generic functor stage (drnum_b200_functor.cuh), FP64, with the reference's
// operation order so that the translation unit (built with -fmad=false)
// reproduces the reference CPU iterator bit for bit:
//   Upwind2<5, VanAlbada>::project   reconstruction/upwind2.h:29-52
//   COMPRESSIBLE_*_VARS, *_PROJ*      fluxes/compressibleflux.h:236-298
//   AusmPlus                          fluxes/ausmplus.h:39-106
//   VanLeer                           fluxes/vanleer.h:36-196
//   Roe                               fluxes/roe.h:46-660
// Each scheme is written once for the three face normals (DIR = 0, 1, 2);
// where the reference's three copies differ in the grouping of a product,
// the difference is kept (noted at the place).
//
// SchemeFlux<E> combines a scheme with the patch-face fluxes of
// dn_patch_set_bc (far field, slip wall, prescribed inflow; fv_wall.cuh).
#pragma once

#include "drnum_b200_functor.cuh"
#include "fv_numerics.cuh"
#include "fv_wall.cuh"

namespace dn {

// Upwind2 reconstruction with the van Albada limiter on a functor patch:
// the state of cell 1 extrapolated towards cell 2, second order where cell
// 0 = 2*c1 - c2 and cell 2 exist (upwind2.h:39-42).
struct Upwind2VanAlbada {
  template <class P>
  __device__ __forceinline__ void project(P* p, double* var, size_t field, size_t i1, size_t j1, size_t k1,
                                          size_t i2, size_t j2, size_t k2) const
  {
    for (int v = 0; v < 5; ++v) var[v] = p->f(field, v, i1, j1, k1);
    const size_t i0 = 2*i1 - i2, j0 = 2*j1 - j2, k0 = 2*k1 - k2;
    if (p->checkRange(i0, j0, k0) && p->checkRange(i2, j2, k2) &&
        !p->isSplitFace(p->index(i0, j0, k0), p->index(i1, j1, k1))) {
      for (int v = 0; v < 5; ++v) {
        const double f1 = p->f(field, v, i1, j1, k1);
        const double delta01 = f1 - p->f(field, v, i0, j0, k0);
        const double delta12 = p->f(field, v, i2, j2, k2) - f1;
        var[v] += 0.5*van_albada(delta01, delta12)*delta01;
      }
    }
  }
};

// Left (cell below the face) and right (cell of the face index) states of
// the face below (i, j, k) along DIR.
template <int DIR, class P>
__device__ __forceinline__ void face_states(P* p, size_t i, size_t j, size_t k, double vl[5], double vr[5])
{
  Upwind2VanAlbada rec;
  const size_t im = DIR == 0 ? i - 1 : i, jm = DIR == 1 ? j - 1 : j, km = DIR == 2 ? k - 1 : k;
  rec.project(p, vl, 0, im, jm, km, i, j, k);
  rec.project(p, vr, 0, i, j, k, im, jm, km);
}

// Conservative and primitive quantities of a face side
// (COMPRESSIBLE_LEFT_VARS / _RIGHT_VARS, compressibleflux.h:236-271).
struct SideVars {
  double r, ir, ru, rv, rw, u, v, w, rE, T, p, a, H;
  __device__ __forceinline__ double vel(int d) const { return d == 0 ? u : (d == 1 ? v : w); }
  __device__ __forceinline__ double mom(int d) const { return d == 0 ? ru : (d == 1 ? rv : rw); }
};

__device__ __forceinline__ SideVars side_vars(const double var[5])
{
  SideVars s;
  s.r = var[0];
  s.ir = 1.0/s.r;
  s.ru = var[1];
  s.rv = var[2];
  s.rw = var[3];
  s.u = s.ru*s.ir;
  s.v = s.rv*s.ir;
  s.w = s.rw*s.ir;
  s.rE = var[4];
  s.T = (s.rE*s.ir - 0.5*(s.u*s.u + s.v*s.v + s.w*s.w))/Gas::cv;
  s.p = s.r*Gas::R*s.T;
  s.a = sqrt(Gas::gamma*Gas::R*s.T);
  s.H = (s.rE + s.p)/s.r;
  return s;
}

// ---------------------------------------------------------------- AUSM+
struct AusmPlusScheme {
  template <int DIR, class P>
  __device__ __forceinline__ void field(P* p, size_t i, size_t j, size_t k, double A, double* flux) const
  {
    double vl[5], vr[5], F[5];
    face_states<DIR>(p, i, j, k, vl, vr);
    ausm_plus<DIR>(face_side(vl), face_side(vr), A, F);
    for (int v = 0; v < 5; ++v) flux[v] += F[v];
  }
};

// ---------------------------------------------------------------- van Leer
// Flux-vector splitting: the left side contributes its supersonic flux for
// M >= 1 and the split flux for -1 < M < 1, the right side likewise for
// M <= -1 and -1 < M < 1 (vanleer.h:36-89 per direction).
struct VanLeerScheme {
  template <int DIR>
  __device__ __forceinline__ static void side(const SideVars& s, int sgn, double F[5])
  {
    const double un = s.vel(DIR);
    const double M = un/s.a;
    for (int v = 0; v < 5; ++v) F[v] = 0;
    const bool super = sgn > 0 ? (M >= 1) : (M <= -1);
    const bool sub = sgn > 0 ? (M > -1) : (M < 1);
    if (super) {
      F[0] = s.r*un;
      for (int d = 0; d < 3; ++d) F[1 + d] = d == DIR ? un*s.mom(d) + s.p : un*s.mom(d);
      F[4] = un*(s.rE + s.p);
    } else if (sub) {
      if (sgn > 0) F[0] = 0.25*s.a*s.r*(M + 1)*(M + 1);
      else         F[0] = -0.25*s.a*s.r*(M - 1)*(M - 1);
      for (int d = 0; d < 3; ++d) {
        if (d == DIR) F[1 + d] = F[0]*(un + s.p/(s.a*s.r)*(sgn > 0 ? (-M + 2) : (-M - 2)));
        else          F[1 + d] = F[0]*s.vel(d);
      }
      F[4] = F[0]/s.r*(s.rE + s.p);
    }
  }

  template <int DIR, class P>
  __device__ __forceinline__ void field(P* p, size_t i, size_t j, size_t k, double A, double* flux) const
  {
    double vl[5], vr[5], Fl[5], Fr[5];
    face_states<DIR>(p, i, j, k, vl, vr);
    side<DIR>(side_vars(vl), +1, Fl);
    side<DIR>(side_vars(vr), -1, Fr);
    for (int v = 0; v < 5; ++v) flux[v] += A*(Fr[v] + Fl[v]);
  }
};

// ---------------------------------------------------------------- Roe
// Roe-averaged upwind flux with the reference's entropy modification of the
// acoustic eigenvalue (roe.h:46-248 per direction): for a non-positive
// contact eigenvalue the flux is F(W_r) - A+ (W_r - W_l) through the last
// eigenvector, otherwise F(W_l) + A- (W_r - W_l) through the first.
struct RoeScheme {
  // products of the reference: u/v/w momenta times the other velocities
  __device__ __forceinline__ static double cross(const SideVars& s, int c, int d)
  {
    const int a = c < d ? c : d, b = c < d ? d : c;
    return (a == 0 ? s.ru : s.rv) * (b == 1 ? s.v : s.w);   // ru*v, ru*w, rv*w
  }

  template <int DIR>
  __device__ __forceinline__ static void side_flux(const SideVars& s, double pp, double A, double F[5])
  {
    const double ep = s.rE + pp;
    F[0] = s.mom(DIR)*A;
    for (int d = 0; d < 3; ++d) F[1 + d] = d == DIR ? (s.mom(d)*s.vel(d) + pp)*A : cross(s, d, DIR)*A;
    // the z copy of the reference writes ep*(w*A) (roe.h:538), x and y (ep*u)*A
    F[4] = DIR == 2 ? ep*(s.vel(DIR)*A) : ep*s.vel(DIR)*A;
  }

  template <int DIR, class P>
  __device__ __forceinline__ void field(P* p, size_t i, size_t j, size_t k, double A, double* flux) const
  {
    double vl[5], vr[5];
    face_states<DIR>(p, i, j, k, vl, vr);
    const SideVars L = side_vars(vl), R = side_vars(vr);
    double fl[5] = {0, 0, 0, 0, 0};

    const double gam = 0.5*(Gas::gamma + Gas::gamma);
    const double gam1 = gam - 1.0;
    const double coef1 = sqrt(L.r);
    const double coef2 = sqrt(R.r);
    const double isomme = 1.0/(coef1 + coef2);
    const double h_l = (gam*L.rE*L.ir) - (.5*gam1)*(L.u*L.u + L.v*L.v + L.w*L.w);
    const double h_r = (gam*R.rE*R.ir) - (.5*gam1)*(R.u*R.u + R.v*R.v + R.w*R.w);
    double ave[3];
    ave[0] = (coef1*L.u + coef2*R.u)*isomme;
    ave[1] = (coef1*L.v + coef2*R.v)*isomme;
    ave[2] = (coef1*L.w + coef2*R.w)*isomme;
    const double h_ave = (coef1*h_l + coef2*h_r)*isomme;

    double scal = ave[DIR]*A;
    const double iA = 1.0/A;
    const double q2 = ave[0]*ave[0] + ave[1]*ave[1] + ave[2]*ave[2];
    double c = gam1*(h_ave - 0.5*q2);
    if (c < 1e-6) c = 1e-6;
    c = sqrt(c);
    const double c2 = c*A;
    double eig1 = scal - c2;
    const double eig2 = scal;
    double eig3 = scal + c2;

    const double dU[5] = {R.r - L.r, R.ru - L.ru, R.rv - L.rv, R.rw - L.rw, R.rE - L.rE};
    const double p_r = gam1*(R.rE - 0.5*(R.ru*R.ru + R.rv*R.rv + R.rw*R.rw)*R.ir);
    const double p_l = gam1*(L.rE - 0.5*(L.ru*L.ru + L.rv*L.rv + L.rw*L.rw)*L.ir);
    if (eig2 <= 0.0) {
      side_flux<DIR>(R, p_r, A, fl);
      const double lambda_l = L.vel(DIR)*A + A*sqrt(gam*p_l*L.ir);
      const double lambda_r = R.vel(DIR)*A + A*sqrt(gam*p_r*R.ir);
      if ((lambda_l < 0.) && (lambda_r > 0.)) eig3 = lambda_r*(eig3 - lambda_l)/(lambda_r - lambda_l);
      if (eig3 > 0.0) {
        scal = scal*iA;
        const double hn = A*iA;
        const double usc = 1.0/c;
        const double t = gam1*usc;
        double av[5], b[5];
        av[0] = usc;
        for (int d = 0; d < 3; ++d) av[1 + d] = d == DIR ? ave[d]*usc + hn : ave[d]*usc;
        av[4] = 0.5*q2*usc + 2.5*c + scal;
        b[0] = 0.5*(0.5*t*q2 - scal);
        for (int d = 0; d < 3; ++d) b[1 + d] = d == DIR ? 0.5*(hn - t*ave[d]) : -0.5*t*ave[d];
        b[4] = 0.5*t;
        const double alpha = eig3*(b[0]*dU[0] + b[1]*dU[1] + b[2]*dU[2] + b[3]*dU[3] + b[4]*dU[4]);
        for (int v = 0; v < 5; ++v) fl[v] -= av[v]*alpha;
      }
    }
    if (eig2 > 0.0) {
      side_flux<DIR>(L, p_l, A, fl);
      const double lambda_l = L.vel(DIR)*A - A*sqrt(gam*p_l*L.ir);
      const double lambda_r = R.vel(DIR)*A - A*sqrt(gam*p_r*R.ir);
      if ((lambda_l < 0.) && (lambda_r > 0.)) eig1 = lambda_l*(lambda_r - eig1)/(lambda_r - lambda_l);
      if (eig1 < 0.0) {
        scal = scal*iA;
        const double hn = A*iA;
        const double usc = 1.0/c;
        const double t = gam1*usc;
        double av[5], b[5];
        av[0] = usc;
        for (int d = 0; d < 3; ++d) av[1 + d] = d == DIR ? ave[d]*usc - hn : ave[d]*usc;
        av[4] = 0.5*q2*usc + 2.5*c - scal;
        b[0] = 0.5*(0.5*t*q2 + scal);
        for (int d = 0; d < 3; ++d) b[1 + d] = d == DIR ? -0.5*(hn + t*ave[d]) : -0.5*(t*ave[d]);
        b[4] = 0.5*t;
        const double alpha = eig1*(b[0]*dU[0] + b[1]*dU[1] + b[2]*dU[2] + b[3]*dU[3] + b[4]*dU[4]);
        for (int v = 0; v < 5; ++v) fl[v] += av[v]*alpha;
      }
    }
    for (int v = 0; v < 5; ++v) flux[v] += fl[v];
  }
};

// ---------------------------------------------------------------- scheme + patch faces
template <class E>
struct SchemeFlux {
  E euler;
  WallBC wall;

  template <class P> __device__ void xField(P* p, size_t i, size_t j, size_t k, double, double, double, double A, double* f) const
  { euler.template field<0>(p, i, j, k, A, f); }
  template <class P> __device__ void yField(P* p, size_t i, size_t j, size_t k, double, double, double, double A, double* f) const
  { euler.template field<1>(p, i, j, k, A, f); }
  template <class P> __device__ void zField(P* p, size_t i, size_t j, size_t k, double, double, double, double A, double* f) const
  { euler.template field<2>(p, i, j, k, A, f); }

  // patch face `side` of boundary cell (ic, jc, kc); `face` indexes the
  // side's inflow table
  template <int AXIS, class P>
  __device__ __forceinline__ void side(P* p, int s, int face, size_t ic, size_t jc, size_t kc, double A, double* f) const
  {
    double U[5], F[5];
    p->getVar(0, ic, jc, kc, U);
    if (wall_flux<AXIS>(wall, s, face, U, A, F))
      for (int v = 0; v < 5; ++v) f[v] += F[v];
  }
  template <class P> __device__ void xWallM(P* p, size_t i, size_t j, size_t k, double, double, double, double A, double* f) const
  { side<0>(p, 0, (int)(j*p->sizeK() + k), i, j, k, A, f); }
  template <class P> __device__ void xWallP(P* p, size_t i, size_t j, size_t k, double, double, double, double A, double* f) const
  { side<0>(p, 1, (int)(j*p->sizeK() + k), i - 1, j, k, A, f); }
  template <class P> __device__ void yWallM(P* p, size_t i, size_t j, size_t k, double, double, double, double A, double* f) const
  { side<1>(p, 2, (int)(i*p->sizeK() + k), i, j, k, A, f); }
  template <class P> __device__ void yWallP(P* p, size_t i, size_t j, size_t k, double, double, double, double A, double* f) const
  { side<1>(p, 3, (int)(i*p->sizeK() + k), i, j - 1, k, A, f); }
  template <class P> __device__ void zWallM(P* p, size_t i, size_t j, size_t k, double, double, double, double A, double* f) const
  { side<2>(p, 4, (int)(i*p->sizeJ() + j), i, j, k, A, f); }
  template <class P> __device__ void zWallP(P* p, size_t i, size_t j, size_t k, double, double, double, double A, double* f) const
  { side<2>(p, 5, (int)(i*p->sizeJ() + j), i, j, k - 1, A, f); }
};

// one stage of one FP64 patch with a built-in scheme (DN_FLUX_*)
cudaError_t launch_scheme_stage(int scheme, const dn_stage_launch* L, const WallBC& wall);

} // namespace dn
