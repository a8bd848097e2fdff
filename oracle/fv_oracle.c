/*
 * ORACLE — CPU restatement of DrNUM's per-patch explicit finite-volume step.
 *
 * Test infrastructure only.  This file is the checker that the CUDA path of
 * drnum_b200 is compared against; the product never links or calls it.
 * Parity of this restatement is pinned against the reference library itself
 * (compiled from its own sources by oracle/build_ref.sh) through the committed
 * fixtures under tests/golden/.
 *
 * It evaluates, in FP64 and in the reference's exact operation order
 * (compile with -ffp-contract=off):
 *   - Upwind2<5, VanAlbada>::project   reconstruction/upwind2.h:29-52
 *   - VanAlbada::lim                   reconstruction/vanalbada.h:28-33
 *   - nonZero                          drnum.h:256-263
 *   - COMPRESSIBLE_LEFT/RIGHT_VARS     fluxes/compressibleflux.h:236-298
 *   - M1/M2/M4/P5                      fluxes/compressibleflux.h:46-75
 *   - AusmPlus::x/y/zField             fluxes/ausmplus.h:39-106
 *   - CartesianIterator::compute       iterators/cartesianiterator.h:87-325
 *     (face loop order i, j, k; x, y, z faces; res[lo] -= F, res[hi] += F;
 *      update f0 = f1 + factor/dV * res on active cells)
 *   - RungeKutta::operator()           rungekutta.cpp:27-42
 *   - PerfectGas constants             perfectgas.h:31-34
 *
 * Patch faces are either periodic (index wrap, identical to the reference run
 * with two ghost layers that are refreshed after every stage) or closed
 * (reconstruction drops to first order where the upwind-upwind cell is out of
 * range, upwind2.h:39-42, and the patch-face flux is zero).
 *
 * Storage: [var][i][j][k], k fastest (cartesianpatch_common.h:61,153).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#define GAS_R 287.2      /* perfectgas.h:31 */
#define GAS_GAMMA 1.4    /* perfectgas.h:32 */
#define GAS_CV 717.5     /* perfectgas.h:34 */
#define LIM_EPS 1e-10    /* GLOBAL_EPS, drnum.h:70 */

static double sqr(double x) { return x*x; }

/* drnum.h:256-263 */
static double non_zero(double x, double eps)
{
  if (x < 0) {
    return (-eps < x) ? -eps : x;   /* min(-eps, x) */
  }
  return (eps > x) ? eps : x;       /* max(eps, x) */
}

/* vanalbada.h:28-33 */
static double van_albada(double d1, double d2)
{
  double r = d2/non_zero(d1, LIM_EPS);
  return (sqr(r) + r)/(sqr(r) + 1);
}

/* compressibleflux.h:46-75 */
static double m1(double M, double s) { return 0.5*(M + s*fabs(M)); }
static double m2(double M, double s) { return 0.25*s*sqr(M + s); }
static double m4(double M, double s)
{
  if (fabs(M) >= 1) return m1(M, s);
  return m2(M, s)*(1 - 2*s*m2(M, -s));
}
static double p5(double M, double s)
{
  if (fabs(M) >= 1) return m1(M, s)/M;
  return m2(M, s)*((2*s - M) - 3*s*M*m2(M, -s));
}

typedef struct {
  int ni, nj, nk;
  int periodic[3];          /* per axis: 1 = periodic wrap, 0 = closed */
  double dx, dy, dz;
  /* patch-face fluxes of closed axes, per side x-min, x-max, y-min, y-max,
   * z-min, z-max: 0 zero flux, 1 far field, 2 slip wall, 3 inflow table */
  int bc[6];
  double ff[6][5];          /* far field p, T, u, v, w */
  const double* table[6];   /* inflow: per face p (NaN: boundary cell), T, u, v, w */
} dno_patch;

static size_t cell(const dno_patch* p, long i, long j, long k)
{
  return ((size_t)i*p->nj + (size_t)j)*p->nk + (size_t)k;
}

/* wrap or flag an index along one axis; returns -1 when out of range */
static long axis_index(long i, int n, int periodic)
{
  if (periodic) {
    i %= n;
    if (i < 0) i += n;
    return i;
  }
  return (i < 0 || i >= n) ? -1 : i;
}

/* Upwind2<5, VanAlbada>::project for the face-side whose cell is c1 and whose
 * downwind neighbour is c2 (upwind2.h:29-52); c0 = 2*c1 - c2.  When c0 is out
 * of range (closed face) the state stays first order. */
static void project(const double* f, size_t nc, size_t c0, int c0_ok,
                    size_t c1, size_t c2, double var[5])
{
  for (int v = 0; v < 5; ++v) var[v] = f[v*nc + c1];
  if (c0_ok) {
    for (int v = 0; v < 5; ++v) {
      double delta01 = f[v*nc + c1] - f[v*nc + c0];
      double delta12 = f[v*nc + c2] - f[v*nc + c1];
      var[v] += 0.5*van_albada(delta01, delta12)*delta01;
    }
  }
}

/* AusmPlus face flux (ausmplus.h:39-106) for direction dir (0=x,1=y,2=z)
 * between the left state var_l and the right state var_r, face area A. */
static void ausm_flux(int dir, const double var_l[5], const double var_r[5],
                      double A, double flux[5])
{
  /* COMPRESSIBLE_LEFT_VARS */
  double r_l  = var_l[0];
  double ir_l = 1.0/r_l;
  double ru_l = var_l[1];
  double rv_l = var_l[2];
  double rw_l = var_l[3];
  double u_l  = ru_l*ir_l;
  double v_l  = rv_l*ir_l;
  double w_l  = rw_l*ir_l;
  double rE_l = var_l[4];
  double T_l  = (rE_l*ir_l - 0.5*(u_l*u_l + v_l*v_l + w_l*w_l))/GAS_CV;
  double p_l  = r_l*GAS_R*T_l;
  double a_l  = sqrt(GAS_GAMMA*GAS_R*T_l);
  double H_l  = (rE_l + p_l)/r_l;
  /* COMPRESSIBLE_RIGHT_VARS */
  double r_r  = var_r[0];
  double ir_r = 1.0/r_r;
  double ru_r = var_r[1];
  double rv_r = var_r[2];
  double rw_r = var_r[3];
  double u_r  = ru_r*ir_r;
  double v_r  = rv_r*ir_r;
  double w_r  = rw_r*ir_r;
  double rE_r = var_r[4];
  double T_r  = (rE_r*ir_r - 0.5*(u_r*u_r + v_r*v_r + w_r*w_r))/GAS_CV;
  double p_r  = r_r*GAS_R*T_r;
  double a_r  = sqrt(GAS_GAMMA*GAS_R*T_r);
  double H_r  = (rE_r + p_r)/r_r;

  double un_l = dir == 0 ? u_l : (dir == 1 ? v_l : w_l);
  double un_r = dir == 0 ? u_r : (dir == 1 ? v_r : w_r);

  double a  = 0.5*(a_l + a_r);
  double M  = m4(un_l/a, 1) + m4(un_r/a, -1);
  double Mp = 0.5*(M + fabs(M));
  double Mm = 0.5*(M - fabs(M));
  double p  = p5(un_l/a, 1)*p_l + p5(un_r/a, -1)*p_r;

  double f0 = 0.0 + a*A*(r_l*Mp + r_r*Mm);
  double pu = dir == 0 ? A*p : 0.0;
  double pv = dir == 1 ? A*p : 0.0;
  double pw = dir == 2 ? A*p : 0.0;
  /* the pressure term is added only in the normal-momentum row; in the
   * others the reference expression has no "+ A*p" term at all */
  flux[0] = f0;
  flux[1] = 0.0 + (dir == 0 ? 0.5*f0*(u_l + u_r) + pu - 0.5*fabs(f0)*(u_r - u_l)
                            : 0.5*f0*(u_l + u_r)      - 0.5*fabs(f0)*(u_r - u_l));
  flux[2] = 0.0 + (dir == 1 ? 0.5*f0*(v_l + v_r) + pv - 0.5*fabs(f0)*(v_r - v_l)
                            : 0.5*f0*(v_l + v_r)      - 0.5*fabs(f0)*(v_r - v_l));
  flux[3] = 0.0 + (dir == 2 ? 0.5*f0*(w_l + w_r) + pw - 0.5*fabs(f0)*(w_r - w_l)
                            : 0.5*f0*(w_l + w_r)      - 0.5*fabs(f0)*(w_r - w_l));
  flux[4] = 0.0 + (0.5*f0*(H_l + H_r) - 0.5*fabs(f0)*(H_r - H_l));
}

/* Flux through the lower face of cell (i,j,k) in direction dir, i.e. between
 * cell c-e_dir and c (the face handled when the reference's loop visits c,
 * cartesianiterator.h:148-179).  Returns 0 when the face does not exist. */
static int face_flux(const dno_patch* p, const double* f, int dir,
                     long i, long j, long k, double flux[5])
{
  const size_t nc = (size_t)p->ni*p->nj*p->nk;
  long d[3] = {0, 0, 0};
  d[dir] = 1;
  int n[3] = {p->ni, p->nj, p->nk};
  long c[3] = {i, j, k};
  /* cells along the axis: m2 = c-2e, m1 = c-e, c, p1 = c+e */
  long idx_m1[3], idx_m2[3], idx_p1[3];
  int ok_m1 = 1, ok_m2 = 1, ok_p1 = 1;
  for (int a = 0; a < 3; ++a) {
    long xm1 = axis_index(c[a] - d[a], n[a], p->periodic[a]);
    long xm2 = axis_index(c[a] - 2*d[a], n[a], p->periodic[a]);
    long xp1 = axis_index(c[a] + d[a], n[a], p->periodic[a]);
    if (xm1 < 0) ok_m1 = 0;
    if (xm2 < 0) ok_m2 = 0;
    if (xp1 < 0) ok_p1 = 0;
    idx_m1[a] = xm1; idx_m2[a] = xm2; idx_p1[a] = xp1;
  }
  if (!ok_m1) return 0;
  /* the reference skips the x-faces when NI <= 2 (cartesianiterator.h:149) */
  if (n[dir] <= 2) return 0;
  size_t cc  = cell(p, i, j, k);
  size_t cm1 = cell(p, idx_m1[0], idx_m1[1], idx_m1[2]);
  size_t cm2 = ok_m2 ? cell(p, idx_m2[0], idx_m2[1], idx_m2[2]) : 0;
  size_t cp1 = ok_p1 ? cell(p, idx_p1[0], idx_p1[1], idx_p1[2]) : 0;
  double var_l[5], var_r[5];
  project(f, nc, cm2, ok_m2, cm1, cc, var_l);   /* COMPRESSIBLE_LEFT_PROJ  */
  project(f, nc, cp1, ok_p1, cc, cm1, var_r);   /* COMPRESSIBLE_RIGHT_PROJ */
  double A = dir == 0 ? p->dy*p->dz : (dir == 1 ? p->dx*p->dz : p->dx*p->dy);
  ausm_flux(dir, var_l, var_r, A, flux);
  return 1;
}

/*
 * Residual of CartesianIterator::compute (cartesianiterator.h:107-188).
 * With a single thread the reference's face loop (i, j, k ascending; x, y, z
 * faces; res[lo] -= F, res[hi] += F) accumulates into every interior cell in
 * the order +Fx(lo) +Fy(lo) +Fz(lo) -Fz(hi) -Fy(hi) -Fx(hi).  The faces are
 * evaluated once each here and summed per cell in that order, which also
 * holds for the wrapped faces of a periodic patch (the reference runs those
 * on a ghosted patch whose ghosts are refreshed after every stage).
 */
#define GAS_CP 1004.5     /* perfectgas.h:33 */

/* PerfectGas::conservativeToPrimitive, perfectgas.h:84-93 (also COMPR_VARS,
 * compressibleflux.h:26-38) */
static void cons_to_prim(const double* var, double* p, double* T, double* u, double* v, double* w)
{
  double ir = 1.0/var[0];
  *u = var[1]*ir;
  *v = var[2]*ir;
  *w = var[3]*ir;
  *T = (var[4]*ir - 0.5*(*u * *u + *v * *v + *w * *w))/GAS_CV;
  *p = var[0]*GAS_R * *T;
}

/* face-state flux, compressiblefarfieldflux.h:100-105 and jetflux.h:186-190 */
static void state_flux(int dir, double A, double p, double T, double u, double v, double w, double* flux)
{
  double un = dir == 0 ? u : (dir == 1 ? v : w);
  flux[0] = A*p/(GAS_R*T)*un;
  flux[1] = flux[0]*u + (dir == 0 ? A*p : 0.0);
  flux[2] = flux[0]*v + (dir == 1 ? A*p : 0.0);
  flux[3] = flux[0]*w + (dir == 2 ? A*p : 0.0);
  if (dir != 0) flux[1] = flux[0]*u;
  if (dir != 1) flux[2] = flux[0]*v;
  if (dir != 2) flux[3] = flux[0]*w;
  flux[4] = flux[0]*(GAS_CP*T + 0.5*(u*u + v*v + w*w));
}

/* Wall flux of one side for boundary-cell state var (first order: the
 * Upwind2 projection at the patch edge, upwind2.h:39-42).  Returns 0 for a
 * zero-flux side.
 *   far field: CompressibleFarfieldFlux::x/y/zWall{M,P}, compressiblefarfieldflux.h:26-181
 *   slip:      CompressibleSlipFlux, compressibleslipflux.h:34-98
 *   inflow:    JetFlux::xWallM, jetflux.h:158-192 (state from a face table) */
static int wall_flux(const dno_patch* p, int side, size_t face, const double* var, double A, double* flux)
{
  int kind = p->bc[side];
  int dir = side/2, plus = side & 1;
  double p1, T1, u1, v1, w1;
  if (kind == 0) return 0;
  cons_to_prim(var, &p1, &T1, &u1, &v1, &w1);
  if (kind == 2) {
    for (int v = 0; v < 5; ++v) flux[v] = 0;
    flux[1 + dir] += A*p1;
    return 1;
  }
  if (kind == 3) {
    const double* e = p->table[side] + 5*face;
    double pp = (e[0] == e[0]) ? e[0] : p1;
    state_flux(dir, A, pp, e[1], e[2], e[3], e[4], flux);
    return 1;
  }
  /* far field: setFarfield stores the conservative state (perfectgas.h:58-66) */
  double m[5], p0, T0, u0, v0, w0;
  const double* q = p->ff[side];
  m[0] = q[0]/(GAS_R*q[1]);
  m[1] = m[0]*q[2];
  m[2] = m[0]*q[3];
  m[3] = m[0]*q[4];
  m[4] = m[0]*(GAS_CV*q[1] + 0.5*(q[2]*q[2] + q[3]*q[3] + q[4]*q[4]));
  cons_to_prim(m, &p0, &T0, &u0, &v0, &w0);
  double a0 = sqrt(GAS_GAMMA*GAS_R*T0);
  double a1 = sqrt(GAS_GAMMA*GAS_R*T1);
  double un0 = dir == 0 ? u0 : (dir == 1 ? v0 : w0);
  double un1 = dir == 0 ? u1 : (dir == 1 ? v1 : w1);
  double M0 = plus ? -(un0/a0) : un0/a0;
  double M1 = plus ? -(un1/a1) : un1/a1;
  double M = 0.5*(M0 + M1);
  if (M >= 0) {
    state_flux(dir, A, M >= 1 ? p0 : p1, T0, u0, v0, w0, flux);
  } else {
    state_flux(dir, A, p1, T1, u1, v1, w1, flux);   /* `M <= 1` always holds here */
  }
  return 1;
}

/* Wall loops of cartesianiterator.h:190-308: x-min (+), x-max (-), y-min,
 * y-max, z-min, z-max, each over its whole side, after the interior faces. */
static void add_walls(const dno_patch* p, const double* f, double* res)
{
  const size_t nc = (size_t)p->ni*p->nj*p->nk;
  const int n[3] = {p->ni, p->nj, p->nk};
  const double A[3] = {p->dy*p->dz, p->dx*p->dz, p->dx*p->dy};
  for (int side = 0; side < 6; ++side) {
    int dir = side/2, plus = side & 1;
    if (p->periodic[dir] || n[dir] <= 2 || p->bc[side] == 0) continue;
    int a = dir == 0 ? 1 : 0, b = dir == 2 ? 1 : 2;     /* the two axes spanning the side */
    for (long ia = 0; ia < n[a]; ++ia)
      for (long ib = 0; ib < n[b]; ++ib) {
        long c[3];
        c[dir] = plus ? n[dir] - 1 : 0;
        c[a] = ia;
        c[b] = ib;
        size_t cc = cell(p, c[0], c[1], c[2]);
        double var[5], flux[5];
        for (int v = 0; v < 5; ++v) var[v] = f[v*nc + cc];
        if (!wall_flux(p, side, (size_t)ia*n[b] + ib, var, A[dir], flux)) continue;
        for (int v = 0; v < 5; ++v) {
          if (plus) res[v*nc + cc] -= flux[v];
          else res[v*nc + cc] += flux[v];
        }
      }
  }
}

static void residual_canonical(const dno_patch* p, const double* f, double* res,
                               double* fx, double* fy, double* fz)
{
  const size_t nc = (size_t)p->ni*p->nj*p->nk;
  double* F[3] = {fx, fy, fz};
  for (int dir = 0; dir < 3; ++dir) {
    for (long i = 0; i < p->ni; ++i)
      for (long j = 0; j < p->nj; ++j)
        for (long k = 0; k < p->nk; ++k) {
          double flux[5];
          size_t cc = cell(p, i, j, k);
          int ok = face_flux(p, f, dir, i, j, k, flux);
          for (int v = 0; v < 5; ++v) F[dir][v*nc + cc] = ok ? flux[v] : 0.0;
        }
  }
  for (long i = 0; i < p->ni; ++i)
    for (long j = 0; j < p->nj; ++j)
      for (long k = 0; k < p->nk; ++k) {
        size_t cc = cell(p, i, j, k);
        long hi[3];
        int ok_hi[3];
        long c[3] = {i, j, k};
        int n[3] = {p->ni, p->nj, p->nk};
        size_t chi[3];
        for (int dir = 0; dir < 3; ++dir) {
          long cp[3] = {c[0], c[1], c[2]};
          hi[dir] = axis_index(c[dir] + 1, n[dir], p->periodic[dir]);
          ok_hi[dir] = hi[dir] >= 0;
          cp[dir] = ok_hi[dir] ? hi[dir] : 0;
          chi[dir] = cell(p, cp[0], cp[1], cp[2]);
        }
        for (int v = 0; v < 5; ++v) {
          double r = 0.0;
          r += F[0][v*nc + cc];
          r += F[1][v*nc + cc];
          r += F[2][v*nc + cc];
          if (ok_hi[2]) r -= F[2][v*nc + chi[2]];
          if (ok_hi[1]) r -= F[1][v*nc + chi[1]];
          if (ok_hi[0]) r -= F[0][v*nc + chi[0]];
          res[v*nc + cc] = r;
        }
      }
  add_walls(p, f, res);
}

/*
 * One RK stage on all active cells: f0 = f1 + (alpha*dt)/dV * res(f0)
 * (cartesianiterator.h:310-322; factor = alpha*dt, rungekutta.cpp:37).
 */
static void stage(const dno_patch* p, double* f0, const double* f1,
                  const uint8_t* active, double factor, double* work)
{
  const size_t nc = (size_t)p->ni*p->nj*p->nk;
  double* res = work;
  residual_canonical(p, f0, res, work + 5*nc, work + 10*nc, work + 15*nc);
  double dV = p->dx*p->dy*p->dz;
  double patch_factor = factor/dV;
  for (size_t c = 0; c < nc; ++c) {
    if (active && !active[c]) continue;
    for (int v = 0; v < 5; ++v) {
      f0[v*nc + c] = f1[v*nc + c] + patch_factor*res[v*nc + c];
    }
  }
}

/*
 * Runs `steps` time steps of the low-storage RK scheme with n_alpha stages on
 * one patch.  state: [5][ni][nj][nk] in/out.  periodic: 3 flags.  active may be
 * NULL (all active).  Returns 0, or a negative error code.
 */
int dno_run(int ni, int nj, int nk, const int* periodic,
            double dx, double dy, double dz,
            double* state, const uint8_t* active,
            int steps, double dt, const double* alpha, int n_alpha)
{
  if (ni < 1 || nj < 1 || nk < 1 || n_alpha < 1 || !state || !alpha) return -1;
  dno_patch p;
  memset(&p, 0, sizeof p);
  p.ni = ni; p.nj = nj; p.nk = nk;
  p.periodic[0] = periodic ? periodic[0] : 1;
  p.periodic[1] = periodic ? periodic[1] : 1;
  p.periodic[2] = periodic ? periodic[2] : 1;
  p.dx = dx; p.dy = dy; p.dz = dz;
  const size_t nc = (size_t)ni*nj*nk;
  double* f1 = (double*)malloc(5*nc*sizeof(double));
  double* work = (double*)malloc(20*nc*sizeof(double));
  if (!f1 || !work) { free(f1); free(work); return -2; }
  for (int s = 0; s < steps; ++s) {
    memcpy(f1, state, 5*nc*sizeof(double));           /* copyField(0, 1) */
    for (int a = 0; a < n_alpha; ++a) {
      stage(&p, state, f1, active, alpha[a]*dt, work);
    }
  }
  free(f1);
  free(work);
  return 0;
}

/* One residual evaluation (the right-hand side before the factor/dV scaling). */
int dno_residual(int ni, int nj, int nk, const int* periodic,
                 double dx, double dy, double dz,
                 const double* state, double* res)
{
  dno_patch p;
  memset(&p, 0, sizeof p);
  p.ni = ni; p.nj = nj; p.nk = nk;
  p.periodic[0] = periodic ? periodic[0] : 1;
  p.periodic[1] = periodic ? periodic[1] : 1;
  p.periodic[2] = periodic ? periodic[2] : 1;
  p.dx = dx; p.dy = dy; p.dz = dz;
  const size_t nc = (size_t)ni*nj*nk;
  double* work = (double*)malloc(15*nc*sizeof(double));
  if (!work) return -2;
  residual_canonical(&p, state, res, work, work + 5*nc, work + 10*nc);
  free(work);
  return 0;
}

/* One residual evaluation with patch-face fluxes on the closed axes:
 * bc[6] kinds (0 zero flux, 1 far field, 2 slip, 3 inflow), ff[6*5] far-field
 * p, T, u, v, w per side, tables[6] inflow face tables (or NULL). */
int dno_residual_bc(int ni, int nj, int nk, const int* periodic,
                    double dx, double dy, double dz,
                    const int* bc, const double* ff, const double* const* tables,
                    const double* state, double* res)
{
  dno_patch p;
  memset(&p, 0, sizeof p);
  p.ni = ni; p.nj = nj; p.nk = nk;
  for (int a = 0; a < 3; ++a) p.periodic[a] = periodic ? periodic[a] : 1;
  p.dx = dx; p.dy = dy; p.dz = dz;
  for (int sd = 0; sd < 6; ++sd) {
    p.bc[sd] = bc ? bc[sd] : 0;
    for (int q = 0; q < 5; ++q) p.ff[sd][q] = ff ? ff[5*sd + q] : 0.0;
    p.table[sd] = tables ? tables[sd] : NULL;
    if (p.bc[sd] == 3 && !p.table[sd]) return -3;
  }
  const size_t nc = (size_t)ni*nj*nk;
  double* work = (double*)malloc(15*nc*sizeof(double));
  if (!work) return -2;
  residual_canonical(&p, state, res, work, work + 5*nc, work + 10*nc);
  free(work);
  return 0;
}
