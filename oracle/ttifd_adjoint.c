/*
 * ttifd_adjoint.c -- CPU reference of the adjoint-state gradient, in double
 * precision (TEST INFRASTRUCTURE: the checker of the device gradient, never
 * part of the product path).
 *
 * The reference (wavetomo/TTI-FDModeling) has no adjoint. This file states the
 * discrete adjoint of its coordinate-rotation time step
 * (src/main/sufdmod2dTTIelastic/sufdmod2dTTIelastic_coordinate_rotation.c:
 * velocity update :614-672, stress update :804-845, free surface :847-863,
 * stress source :865-886, receivers isoelastic.c:103-144) and of its
 * stiffness build (:497-537), the same for the tensor-rotation formulation
 * (sufdmod2dTTIelastic_tensor_rotation.c: tau update and sigma = R tau
 * :799-851, stiffness :498-519), and for the Bond-transformation
 * formulation (sufdmod2dTTIelastic_bond_transformation.c: velocity update
 * :654-703, stress update :836-873, stiffness :492-541 and its free-surface
 * rewrite :543-568), so that
 *   J = 1/2 sum over recorded samples (d - dobs)^2
 * has gradients with respect to vp, epsilon, delta and theta (degrees) at
 * every padded cell. Conventions: vs and rho are held fixed; the MEAL arrays
 * coef1, coef2 and Beta are frozen (given, from the float setup of a
 * reference model); stiffness uses vp/Beta, vs/Beta, rho*Beta (meal.c:450-490).
 * Sources: the stress source (stype 1, :865-886) and the velocity sources
 * (stype 2-8, :674-802), which add to v after the velocity update. The
 * source tables do not depend on the model, so the model gradient has the same
 * adjoint for every stype; the source-wavelet gradient reads lambda_v between
 * the stress-half and velocity-half adjoints. A velocity source window can
 * reach cells the velocity update never writes (the image rows above a free
 * surface, the outer rim); v there only accumulates source samples, so its
 * adjoint only accumulates the transposed stress stencils. The forward
 * states are all kept in memory (small test grids).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "ttifd_adjoint.h"

#define NH 5
static const double RSGC[5] = {1.24362739770907f, -0.114021164233934f, 0.0272965993810630f, -0.00699199493927320f,
                               0.00132022981661381f};

struct adj_ctx {
  int nz, nx, nt, E, Nz, Nx, izs, fs, mt, seistype, nts, stype;
  double dx, dz, dt, scalar;
  size_t Np;
  /* frozen MEAL */
  double *coef1, *coef2, *beta;
  /* model and derived arrays */
  double *vp, *vs, *rho, *eps, *delta, *theta;  /* as given (padded) */
  double *c11, *c13, *c33, *c55, *sn, *cs, *snv, *csv, *ir;
  int bond, tensor;     /* Bond transformation / tensor rotation instead of coordinate rotation */
  double *c15, *c35;    /* Bond only */
  /* geometry */
  int nsrc, *sx, *sz;
  double *src; /* [nsrc][nt] */
  int nrec[3], *rx[3], *rz[3];
};

#define A2(a, ix, iz) ((a)[(size_t)(ix) * (size_t)c->Nz + (size_t)(iz)])

static double *dalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

adj_ctx *adj_create(int nz, int nx, int nt, double dx, double dz, double dt, int ealThick, int freesurface, int mt,
                    int seistype, double scalar)
{
  adj_ctx *c = (adj_ctx *)calloc(1, sizeof(adj_ctx));
  c->nz = nz;
  c->nx = nx;
  c->nt = nt;
  c->E = ealThick + NH;
  c->Nz = nz + 2 * c->E;
  c->Nx = nx + 2 * c->E;
  c->izs = freesurface ? c->E : NH;
  c->fs = freesurface;
  c->mt = mt;
  c->seistype = seistype;
  c->nts = (nt - 1) / mt + 1;
  c->dx = dx;
  c->dz = dz;
  c->dt = dt;
  c->scalar = scalar;
  c->stype = 1;
  c->Np = (size_t)c->Nz * c->Nx;
  double **arrs[] = {&c->coef1, &c->coef2, &c->beta, &c->vp,  &c->vs,  &c->rho, &c->eps, &c->delta, &c->theta, &c->c11,
                     &c->c13,   &c->c33,   &c->c55,  &c->sn,  &c->cs,  &c->snv, &c->csv, &c->ir,    &c->c15,   &c->c35};
  for (size_t k = 0; k < sizeof arrs / sizeof arrs[0]; ++k) *arrs[k] = dalloc(c->Np);
  return c;
}

void adj_destroy(adj_ctx *c)
{
  if (!c) return;
  double *arrs[] = {c->coef1, c->coef2, c->beta, c->vp,  c->vs,  c->rho, c->eps, c->delta, c->theta, c->c11,
                    c->c13,   c->c33,   c->c55,  c->sn,  c->cs,  c->snv, c->csv, c->ir,    c->c15,   c->c35};
  for (size_t k = 0; k < sizeof arrs / sizeof arrs[0]; ++k) free(arrs[k]);
  free(c->sx);
  free(c->sz);
  free(c->src);
  for (int k = 0; k < 3; ++k) {
    free(c->rx[k]);
    free(c->rz[k]);
  }
  free(c);
}

void adj_grid(const adj_ctx *c, int *Nz, int *Nx, int *nts)
{
  *Nz = c->Nz;
  *Nx = c->Nx;
  *nts = c->nts;
}

void adj_set_formulation(adj_ctx *c, int variant)
{
  c->tensor = variant == 1;
  c->bond = variant == 2;
}

void adj_set_stype(adj_ctx *c, int stype) { c->stype = stype; }

/* Bond rotation of the VTI moduli (bond:492-541): c11 c13 c15 c33 c35 c55 */
static void bond_moduli(double C11, double C13, double C33, double C55, double th, double out[6])
{
  const double s2 = sin(th) * sin(th), c2 = cos(th) * cos(th), s4 = s2 * s2, c4 = c2 * c2;
  const double s2t = sin(2.0 * th), c2t = cos(2.0 * th), s22 = s2t * s2t, c22 = c2t * c2t;
  out[0] = C11 * c4 + C33 * s4 + (0.5 * C13 + C55) * s22;
  out[1] = (0.25 * (C11 + C33) - C55) * s22 + C13 * (s4 + c4);
  out[2] = 0.5 * (-C11 * c2 + C33 * s2 + (C13 + 2.0 * C55) * c2t) * s2t;
  out[3] = C11 * s4 + C33 * c4 + (0.5 * C13 + C55) * s22;
  out[4] = 0.5 * (-C11 * s2 + C33 * c2 - (C13 + 2.0 * C55) * c2t) * s2t;
  out[5] = 0.25 * (C11 + C33 - 2.0 * C13) * s22 + C55 * c22;
}

/* Bond free-surface row (bond:543-568): the moduli a = (c11 c13 c15 c33 c35 c55)
 * are replaced by an effective c11 (returned) and zeros; dc[k] = d c11'/d a[k]. */
static double bond_fs_c11(const double a[6], double dc[6])
{
  const double a11 = a[0], a13 = a[1], a15 = a[2], a33 = a[3], a35 = a[4], a55 = a[5];
  const double N = a13 * a55 - a15 * a35, D = a33 * a55 - a35 * a35;
  double n35 = -N / D;
  int fallback = !isfinite(n35);
  if (fallback) n35 = -a13 / a33;
  if (!isfinite(n35)) n35 = 0.0;
  const double M = a13 * n35 - a15 * a33, Q = a33 * a55 - n35 * n35, n55 = M / Q;
  for (int v = 0; v < 6; ++v) {  /* one-hot forward derivatives */
    const double d11 = v == 0, d13 = v == 1, d15 = v == 2, d33 = v == 3, d35 = v == 4, d55 = v == 5;
    double dn35;
    if (!fallback) {
      const double dN = d13 * a55 + a13 * d55 - d15 * a35 - a15 * d35, dD = d33 * a55 + a33 * d55 - 2.0 * a35 * d35;
      dn35 = -(dN * D - N * dD) / (D * D);
    } else {
      dn35 = isfinite(-a13 / a33) ? -(d13 * a33 - a13 * d33) / (a33 * a33) : 0.0;
    }
    const double dM = d13 * n35 + a13 * dn35 - d15 * a33 - a15 * d33;
    const double dQ = d33 * a55 + a33 * d55 - 2.0 * n35 * dn35;
    const double dn55 = (dM * Q - M * dQ) / (Q * Q);
    dc[v] = d11 - d13 * n35 - a13 * dn35 + d15 * n55 + a15 * dn55;
  }
  return a11 - a13 * n35 + a15 * n55;
}

/* derivatives of bond_moduli: d[m][0..5] = d(c11..c55)/d(C11, C13, C33, theta)[m] */
static void bond_moduli_grad(double C11, double C13, double C33, double C55, double th, double d[4][6])
{
  const double s2 = sin(th) * sin(th), c2 = cos(th) * cos(th), s4 = s2 * s2, c4 = c2 * c2;
  const double s2t = sin(2.0 * th), c2t = cos(2.0 * th), s22 = s2t * s2t;
  const double ds2 = s2t, dc2 = -s2t, ds4 = 2.0 * s2 * s2t, dc4 = -2.0 * c2 * s2t;
  const double ds2t = 2.0 * c2t, dc2t = -2.0 * s2t, ds22 = 4.0 * s2t * c2t, dc22 = -ds22;
  const double d11[6] = {c4, 0.25 * s22, -0.5 * c2 * s2t, s4, -0.5 * s2 * s2t, 0.25 * s22};
  const double d13[6] = {0.5 * s22, s4 + c4, 0.5 * c2t * s2t, 0.5 * s22, -0.5 * c2t * s2t, -0.5 * s22};
  const double d33[6] = {s4, 0.25 * s22, 0.5 * s2 * s2t, c4, 0.5 * c2 * s2t, 0.25 * s22};
  const double A = C13 + 2.0 * C55;
  const double dth[6] = {
      C11 * dc4 + C33 * ds4 + (0.5 * C13 + C55) * ds22,
      (0.25 * (C11 + C33) - C55) * ds22 + C13 * (ds4 + dc4),
      0.5 * ((-C11 * dc2 + C33 * ds2 + A * dc2t) * s2t + (-C11 * c2 + C33 * s2 + A * c2t) * ds2t),
      C11 * ds4 + C33 * dc4 + (0.5 * C13 + C55) * ds22,
      0.5 * ((-C11 * ds2 + C33 * dc2 - A * dc2t) * s2t + (-C11 * s2 + C33 * c2 - A * c2t) * ds2t),
      0.25 * (C11 + C33 - 2.0 * C13) * ds22 + C55 * dc22};
  for (int k = 0; k < 6; ++k) {
    d[0][k] = d11[k];
    d[1][k] = d13[k];
    d[2][k] = d33[k];
    d[3][k] = dth[k];
  }
}

void adj_set_meal(adj_ctx *c, const float *coef1, const float *coef2, const float *beta)
{
  for (size_t i = 0; i < c->Np; ++i) {
    c->coef1[i] = coef1[i];
    c->coef2[i] = coef2[i];
    c->beta[i] = beta[i];
  }
}

/* stiffness and angles (coord:497-537) from the model in double */
void adj_set_model(adj_ctx *c, const double *vp, const double *vs, const double *rho, const double *eps,
                   const double *delta, const double *theta)
{
  const size_t Np = c->Np;
  memcpy(c->vp, vp, Np * sizeof(double));
  memcpy(c->vs, vs, Np * sizeof(double));
  memcpy(c->rho, rho, Np * sizeof(double));
  memcpy(c->eps, eps, Np * sizeof(double));
  memcpy(c->delta, delta, Np * sizeof(double));
  memcpy(c->theta, theta, Np * sizeof(double));
  for (size_t i = 0; i < Np; ++i) {
    const double B = c->beta[i];
    const double p = vp[i] / B, s = vs[i] / B, r = rho[i] * B;
    const double f = 1.0 - (s / p) * (s / p);
    c->c11[i] = r * p * p * (1.0 + 2.0 * eps[i]);
    c->c13[i] = r * (p * p * sqrt(f * (f + 2.0 * delta[i])) - s * s);
    c->c33[i] = r * p * p;
    c->c55[i] = r * s * s;
    const double th = c->scalar * theta[i] / 180.0 * M_PI;
    if (c->bond) {
      double m[6];
      bond_moduli(c->c11[i], c->c13[i], c->c33[i], c->c55[i], th, m);
      c->c11[i] = m[0];
      c->c13[i] = m[1];
      c->c15[i] = m[2];
      c->c33[i] = m[3];
      c->c35[i] = m[4];
      c->c55[i] = m[5];
      if (c->fs && (int)(i % (size_t)c->Nz) == c->E) {  /* the free-surface row */
        double dc[6];
        c->c11[i] = bond_fs_c11(m, dc);
        c->c13[i] = c->c15[i] = c->c33[i] = c->c35[i] = c->c55[i] = 0.0;
      }
    }
    c->sn[i] = sin(th);
    c->cs[i] = cos(th);
  }
  for (int ix = 0; ix < c->Nx; ++ix)
    for (int iz = 0; iz < c->Nz; ++iz) {
      const int inner = ix < c->Nx - 1 && iz < c->Nz - 1;
#define RB(x, z) (A2(c->rho, x, z) * A2(c->beta, x, z))
      if (inner) {
        A2(c->ir, ix, iz) = 4.0 / (RB(ix, iz) + RB(ix + 1, iz) + RB(ix, iz + 1) + RB(ix + 1, iz + 1));
        A2(c->snv, ix, iz) =
            0.25 * (A2(c->sn, ix, iz) + A2(c->sn, ix + 1, iz) + A2(c->sn, ix, iz + 1) + A2(c->sn, ix + 1, iz + 1));
        A2(c->csv, ix, iz) =
            0.25 * (A2(c->cs, ix, iz) + A2(c->cs, ix + 1, iz) + A2(c->cs, ix, iz + 1) + A2(c->cs, ix + 1, iz + 1));
      } else {
        A2(c->ir, ix, iz) = 1.0 / RB(ix, iz);
        A2(c->snv, ix, iz) = A2(c->sn, ix, iz);
        A2(c->csv, ix, iz) = A2(c->cs, ix, iz);
      }
#undef RB
    }
}

void adj_set_source(adj_ctx *c, int n, const int *sx, const int *sz, const double *w)
{
  free(c->sx);
  free(c->sz);
  free(c->src);
  c->nsrc = n;
  c->sx = (int *)malloc(sizeof(int) * (n ? n : 1));
  c->sz = (int *)malloc(sizeof(int) * (n ? n : 1));
  c->src = dalloc((size_t)n * c->nt);
  memcpy(c->sx, sx, sizeof(int) * n);
  memcpy(c->sz, sz, sizeof(int) * n);
  memcpy(c->src, w, sizeof(double) * (size_t)n * c->nt);
}

void adj_set_receivers(adj_ctx *c, int kind, int n, const int *gx, const int *gz)
{
  free(c->rx[kind]);
  free(c->rz[kind]);
  c->nrec[kind] = n;
  c->rx[kind] = (int *)malloc(sizeof(int) * (n ? n : 1));
  c->rz[kind] = (int *)malloc(sizeof(int) * (n ? n : 1));
  memcpy(c->rx[kind], gx, sizeof(int) * n);
  memcpy(c->rz[kind], gz, sizeof(int) * n);
}

/* ---------------------------------------------------------------- stencils */
/* velocity-node pair (coord:621-630) and stress-node pair (coord:811-816) */
static void dv(const adj_ctx *c, const double *a, int ix, int iz, double *d1, double *d2)
{
  double s1 = 0.0, s2 = 0.0;
  for (int k = 1; k <= NH; ++k) {
    s1 += RSGC[k - 1] * (A2(a, ix + k, iz + k) - A2(a, ix - k + 1, iz - k + 1));
    s2 += RSGC[k - 1] * (A2(a, ix + k, iz - k + 1) - A2(a, ix - k + 1, iz + k));
  }
  *d1 = s1;
  *d2 = s2;
}

static void ds(const adj_ctx *c, const double *a, int ix, int iz, double *d1, double *d2)
{
  double s1 = 0.0, s2 = 0.0;
  for (int k = 1; k <= NH; ++k) {
    s1 += RSGC[k - 1] * (A2(a, ix + k - 1, iz + k - 1) - A2(a, ix - k, iz - k));
    s2 += RSGC[k - 1] * (A2(a, ix + k - 1, iz - k) - A2(a, ix - k, iz + k - 1));
  }
  *d1 = s1;
  *d2 = s2;
}

/* the velocity-node pair with cells outside the grid read as zero */
static double at0(const adj_ctx *c, const double *a, int ix, int iz)
{
  return ix < 0 || ix >= c->Nx || iz < 0 || iz >= c->Nz ? 0.0 : A2(a, ix, iz);
}

static void dv_rim(const adj_ctx *c, const double *a, int ix, int iz, double *d1, double *d2)
{
  double s1 = 0.0, s2 = 0.0;
  for (int k = 1; k <= NH; ++k) {
    s1 += RSGC[k - 1] * (at0(c, a, ix + k, iz + k) - at0(c, a, ix - k + 1, iz - k + 1));
    s2 += RSGC[k - 1] * (at0(c, a, ix + k, iz - k + 1) - at0(c, a, ix - k + 1, iz + k));
  }
  *d1 = s1;
  *d2 = s2;
}

static double src_weight(const adj_ctx *c, int a, int b)
{
  const double alpha = log(0.8) / (c->dx * c->dx + c->dz * c->dz);
  const double rx = a * c->dx, rz = b * c->dz;
  return exp(alpha * (rx * rx + rz * rz)) / (c->dx * c->dz) * c->dt;
}

/* cells and weights of velocity source n (stype 2-8, coord:674-802):
 * vx[cell] += wx src(t), vz[cell] += wz src(t). stype 4 is stype 2 followed by
 * stype 3 on the same window; stype 8 touches four cells without a window.
 * Returns the number of cells (at most 121). */
static int vsrc_cells(const adj_ctx *c, int n, int *cx, int *cz, double *wx, double *wz)
{
  const int x0 = c->sx[n] + c->E, z0 = c->sz[n] + c->E;
  int m = 0;
  if (c->stype == 8) {
    static const int ox[4] = {0, -1, -1, 0}, oz[4] = {0, 0, -1, -1};
    static const double sgx[4] = {-1.0, -1.0, 1.0, 1.0}, sgz[4] = {1.0, -1.0, -1.0, 1.0};
    const double q = 0.125 * sqrt(2.0);
    for (int k = 0; k < 4; ++k, ++m) {
      cx[m] = x0 + ox[k];
      cz[m] = z0 + oz[k];
      wx[m] = sgx[k] * q;
      wz[m] = sgz[k] * q;
    }
    return m;
  }
  const double alpha = log(0.8) / (c->dx * c->dx + c->dz * c->dz);
  for (int a = -NH; a <= NH; ++a)
    for (int b = -NH; b <= NH; ++b) {
      const int ix = x0 + a, iz = z0 + b;
      if (ix < 0 || ix >= c->Nx || iz < 0 || iz >= c->Nz) continue;
      const double w = src_weight(c, a, b), kx = 2.0 * alpha * a * c->dx * w, kz = 2.0 * alpha * b * c->dz * w;
      double x = 0.0, z = 0.0;
      if (c->stype == 2 || c->stype == 4) {  /* divergence force */
        x += kx;
        z += kz;
      }
      if (c->stype == 3 || c->stype == 4) {  /* curl force */
        x -= kz;
        z += kx;
      }
      if (c->stype == 5) x = w;  /* horizontal point force */
      if (c->stype == 6) z = w;  /* vertical point force */
      if (c->stype == 7) x = z = 0.5 * sqrt(2.0) * w;  /* tilted point force */
      cx[m] = ix;
      cz[m] = iz;
      wx[m] = x;
      wz[m] = z;
      ++m;
    }
  return m;
}

/* ---------------------------------------------------------------- forward */
typedef struct {
  double *vx, *vz, *sxx, *szz, *sxz, *txx, *tzz, *txz;  /* tau: tensor rotation only */
} state;

static void velocity_half(const adj_ctx *c, state *u)
{
  const double hx = 0.5 / c->dx, hz = 0.5 / c->dz;
  for (int ix = NH; ix < c->Nx - NH; ++ix)
    for (int iz = c->izs; iz < c->Nz - NH; ++iz) {
      double a1, a2, b1, b2, e1, e2;
      dv(c, u->sxx, ix, iz, &a1, &a2);
      dv(c, u->szz, ix, iz, &b1, &b2);
      dv(c, u->sxz, ix, iz, &e1, &e2);
      const double sxx_x = hx * (a1 + a2), sxx_z = hx * (a1 - a2); /* coord:633 uses 1/dx */
      const double szz_x = hx * (b1 + b2), szz_z = hz * (b1 - b2);
      const double sxz_x = hx * (e1 + e2), sxz_z = hz * (e1 - e2);
      const size_t i = (size_t)ix * c->Nz + iz;
      const double cv = c->csv[i], sv = c->snv[i], br = c->coef2[i] * c->ir[i];
      if (c->bond || c->tensor) {
        u->vx[i] = c->coef1[i] * u->vx[i] + br * (sxx_x + sxz_z);
        u->vz[i] = c->coef1[i] * u->vz[i] + br * (sxz_x + szz_z);
      } else {
        u->vx[i] = c->coef1[i] * u->vx[i] + br * (cv * sxx_x - sv * sxx_z + sv * sxz_x + cv * sxz_z);
        u->vz[i] = c->coef1[i] * u->vz[i] + br * (cv * sxz_x - sv * sxz_z + sv * szz_x + cv * szz_z);
      }
    }
}

static void stress_half(const adj_ctx *c, state *u)
{
  const double hx = 0.5 / c->dx, hz = 0.5 / c->dz;
  for (int ix = NH; ix < c->Nx - NH; ++ix)
    for (int iz = c->izs; iz < c->Nz - NH; ++iz) {
      double a1, a2, b1, b2;
      ds(c, u->vx, ix, iz, &a1, &a2);
      ds(c, u->vz, ix, iz, &b1, &b2);
      double vxx = hx * (a1 + a2), vxz = hz * (a1 - a2), vzx = hx * (b1 + b2), vzz = hz * (b1 - b2);
      const size_t i = (size_t)ix * c->Nz + iz;
      const double a = c->coef1[i], b = c->coef2[i];
      if (c->bond) {
        const double sh = vzx + vxz;
        u->sxx[i] = a * u->sxx[i] + b * (c->c11[i] * vxx + c->c13[i] * vzz + c->c15[i] * sh);
        u->szz[i] = a * u->szz[i] + b * (c->c13[i] * vxx + c->c33[i] * vzz + c->c35[i] * sh);
        u->sxz[i] = a * u->sxz[i] + b * (c->c15[i] * vxx + c->c35[i] * vzz + c->c55[i] * sh);
        continue;
      }
      const double s = c->sn[i], co = c->cs[i];
      if (c->tensor) {  /* rotated strain rates, Hooke on tau, sigma = R tau (tensor:826-851) */
        const double s2 = s * s, c2 = co * co, st = 2.0 * s * co, sh = vxz + vzx;
        const double exx = c2 * vxx + s2 * vzz - 0.5 * st * sh, ezz = s2 * vxx + c2 * vzz + 0.5 * st * sh;
        const double exz = st * (vxx - vzz) + (c2 - s2) * sh;
        const double nxx = a * u->txx[i] + b * (c->c11[i] * exx + c->c13[i] * ezz);
        const double nzz = a * u->tzz[i] + b * (c->c13[i] * exx + c->c33[i] * ezz);
        const double nxz = a * u->txz[i] + b * c->c55[i] * exz;
        u->txx[i] = nxx;
        u->tzz[i] = nzz;
        u->txz[i] = nxz;
        u->sxx[i] = c2 * nxx + s2 * nzz + st * nxz;
        u->szz[i] = s2 * nxx + c2 * nzz - st * nxz;
        u->sxz[i] = -0.5 * st * (nxx - nzz) + (c2 - s2) * nxz;
        continue;
      }
      const double rxx = co * vxx - s * vxz, rxz = s * vxx + co * vxz;
      const double rzx = co * vzx - s * vzz, rzz = s * vzx + co * vzz;
      u->sxx[i] = a * u->sxx[i] + b * (c->c11[i] * rxx + c->c13[i] * rzz);
      u->szz[i] = a * u->szz[i] + b * (c->c13[i] * rxx + c->c33[i] * rzz);
      u->sxz[i] = a * u->sxz[i] + b * c->c55[i] * (rzx + rxz);
    }
}

static void free_surface(const adj_ctx *c, state *u)
{
  const int s = c->izs;
  for (int ix = NH; ix < c->Nx - NH; ++ix) {
    A2(u->sxz, ix, s) = 0.0;
    A2(u->szz, ix, s) = 0.0;
    for (int k = 1; k <= NH; ++k) {
      A2(u->sxx, ix, s - k) = 2.0 * A2(u->sxx, ix, s) - A2(u->sxx, ix, s + k);
      A2(u->szz, ix, s - k) = -A2(u->szz, ix, s + k);
      A2(u->sxz, ix, s - k) = -A2(u->sxz, ix, s + k);
    }
  }
}

static void velocity_source(const adj_ctx *c, state *u, int it)
{
  int cx[121], cz[121];
  double wx[121], wz[121];
  for (int n = 0; n < c->nsrc; ++n) {
    const double w = c->src[(size_t)n * c->nt + it];
    const int m = vsrc_cells(c, n, cx, cz, wx, wz);
    for (int q = 0; q < m; ++q) {
      A2(u->vx, cx[q], cz[q]) += wx[q] * w;
      A2(u->vz, cx[q], cz[q]) += wz[q] * w;
    }
  }
}

static void stress_source(const adj_ctx *c, state *u, int it)
{
  if (c->stype != 1) return;
  for (int n = 0; n < c->nsrc; ++n) {
    const int x0 = c->sx[n] + c->E, z0 = c->sz[n] + c->E;
    const double w = c->src[(size_t)n * c->nt + it];
    for (int a = -NH; a <= NH; ++a)
      for (int b = -NH; b <= NH; ++b) {
        const int ix = x0 + a, iz = z0 + b;
        if (ix < 0 || ix >= c->Nx || iz < 0 || iz >= c->Nz) continue;
        const double k = 0.5 * src_weight(c, a, b) * w;
        A2(u->sxx, ix, iz) += k;
        A2(u->szz, ix, iz) += k;
        if (c->tensor) {
          A2(u->txx, ix, iz) += k;
          A2(u->tzz, ix, iz) += k;
        }
      }
  }
}

static int want(const adj_ctx *c, int k)
{
  return k < 2 ? (c->seistype == 1 || c->seistype == 3) : (c->seistype == 2 || c->seistype == 3);
}

static void record(const adj_ctx *c, const state *u, int it, double *rec[3])
{
  if (c->seistype <= 0 || it % c->mt != 0) return;
  const int j = it / c->mt;
  for (int k = 0; k < 3; ++k) {
    if (!want(c, k) || !rec[k]) continue;
    for (int t = 0; t < c->nrec[k]; ++t) {
      const int x = c->rx[k][t] + c->E, z = c->rz[k][t] + c->E;
      double v;
      if (k == 0) v = A2(u->vx, x, z);
      else if (k == 1) v = A2(u->vz, x, z);
      else v = 0.5 * (A2(u->sxx, x, z) + A2(u->szz, x, z));
      rec[k][(size_t)t * c->nts + j] = v;
    }
  }
}

static state state_alloc(size_t n)
{
  state s = {dalloc(n), dalloc(n), dalloc(n), dalloc(n), dalloc(n), dalloc(n), dalloc(n), dalloc(n)};
  return s;
}

static void state_free(state *s)
{
  free(s->vx);
  free(s->vz);
  free(s->sxx);
  free(s->szz);
  free(s->sxz);
  free(s->txx);
  free(s->tzz);
  free(s->txz);
}

/* one step; `keep` (may be NULL) receives (v after the velocity half, sigma
 * and tau before the stress half), the states the adjoint step reads */
static void step(const adj_ctx *c, state *u, int it, double *rec[3], state *keep)
{
  velocity_half(c, u);
  if (c->stype >= 2) velocity_source(c, u, it);
  if (keep) {
    memcpy(keep->vx, u->vx, c->Np * sizeof(double));
    memcpy(keep->vz, u->vz, c->Np * sizeof(double));
    memcpy(keep->sxx, u->sxx, c->Np * sizeof(double));
    memcpy(keep->szz, u->szz, c->Np * sizeof(double));
    memcpy(keep->sxz, u->sxz, c->Np * sizeof(double));
    memcpy(keep->txx, u->txx, c->Np * sizeof(double));
    memcpy(keep->tzz, u->tzz, c->Np * sizeof(double));
    memcpy(keep->txz, u->txz, c->Np * sizeof(double));
  }
  stress_half(c, u);
  if (c->fs) free_surface(c, u);
  stress_source(c, u, it);
  record(c, u, it, rec);
}

void adj_forward(adj_ctx *c, double *rec[3])
{
  state u = state_alloc(c->Np);
  for (int it = 0; it < c->nt; ++it) step(c, &u, it, rec, NULL);
  state_free(&u);
}

/* ---------------------------------------------------------------- adjoint */
double adj_gradient(adj_ctx *c, const double *dobs[3], double *g_vp, double *g_eps, double *g_delta,
                    double *g_theta, double *g_src)
{
  const size_t Np = c->Np;
  const int Nz = c->Nz, Nx = c->Nx, izs = c->izs;
  const double hx = 0.5 / c->dx, hz = 0.5 / c->dz;
  double *rec[3] = {NULL, NULL, NULL};
  for (int k = 0; k < 3; ++k)
    if (want(c, k) && c->nrec[k] > 0) rec[k] = dalloc((size_t)c->nrec[k] * c->nts);
  /* forward, keeping every step's (v_new, sigma_old) */
  state *keep = (state *)malloc(sizeof(state) * c->nt);
  state u = state_alloc(Np);
  for (int it = 0; it < c->nt; ++it) {
    keep[it] = state_alloc(Np);
    step(c, &u, it, rec, &keep[it]);
  }
  state_free(&u);
  /* residuals and misfit */
  double J = 0.0;
  for (int k = 0; k < 3; ++k) {
    if (!rec[k]) continue;
    for (size_t q = 0; q < (size_t)c->nrec[k] * c->nts; ++q) {
      rec[k][q] -= dobs[k][q];
      J += 0.5 * rec[k][q] * rec[k][q];
    }
  }
  /* adjoint state and work arrays */
  state L = state_alloc(Np);
  double *T[6];
  for (int k = 0; k < 6; ++k) T[k] = dalloc(Np);
  double *gc11 = dalloc(Np), *gc13 = dalloc(Np), *gc33 = dalloc(Np), *gc55 = dalloc(Np), *gth = dalloc(Np);
  double *gsv = dalloc(Np), *gcv = dalloc(Np), *gc15 = dalloc(Np), *gc35 = dalloc(Np);
  if (g_src) memset(g_src, 0, sizeof(double) * (size_t)c->nsrc * c->nt);
  for (int it = c->nt - 1; it >= 0; --it) {
    const state *f = &keep[it];
    /* residual injection (adjoint of record) */
    if (c->seistype > 0 && it % c->mt == 0) {
      const int j = it / c->mt;
      for (int k = 0; k < 3; ++k) {
        if (!rec[k]) continue;
        for (int t = 0; t < c->nrec[k]; ++t) {
          const int x = c->rx[k][t] + c->E, z = c->rz[k][t] + c->E;
          const double r = rec[k][(size_t)t * c->nts + j];
          if (k == 0) A2(L.vx, x, z) += r;
          else if (k == 1) A2(L.vz, x, z) += r;
          else {
            A2(L.sxx, x, z) += 0.5 * r;
            A2(L.szz, x, z) += 0.5 * r;
          }
        }
      }
    }
    /* source-wavelet gradient (adjoint of the stress source) */
    if (g_src && c->stype == 1)
      for (int n = 0; n < c->nsrc; ++n) {
        const int x0 = c->sx[n] + c->E, z0 = c->sz[n] + c->E;
        double acc = 0.0;
        for (int a = -NH; a <= NH; ++a)
          for (int b = -NH; b <= NH; ++b) {
            const int ix = x0 + a, iz = z0 + b;
            if (ix < 0 || ix >= Nx || iz < 0 || iz >= Nz) continue;
            acc += 0.5 * src_weight(c, a, b) * (A2(L.sxx, ix, iz) + A2(L.szz, ix, iz));
            if (c->tensor) acc += 0.5 * src_weight(c, a, b) * (A2(L.txx, ix, iz) + A2(L.tzz, ix, iz));
          }
        g_src[(size_t)n * c->nt + it] = acc;
      }
    /* adjoint of the free surface */
    if (c->fs)
      for (int ix = NH; ix < Nx - NH; ++ix) {
        for (int k = 1; k <= NH; ++k) {
          A2(L.sxx, ix, izs) += 2.0 * A2(L.sxx, ix, izs - k);
          A2(L.sxx, ix, izs + k) -= A2(L.sxx, ix, izs - k);
          A2(L.sxx, ix, izs - k) = 0.0;
          A2(L.szz, ix, izs + k) -= A2(L.szz, ix, izs - k);
          A2(L.szz, ix, izs - k) = 0.0;
          A2(L.sxz, ix, izs + k) -= A2(L.sxz, ix, izs - k);
          A2(L.sxz, ix, izs - k) = 0.0;
        }
        A2(L.sxz, ix, izs) = 0.0;
        A2(L.szz, ix, izs) = 0.0;
      }
    /* adjoint of the stress half: gradient terms, then T = d(sigma)/d(strain)^T lambda */
    for (int k = 0; k < 4; ++k) memset(T[k], 0, Np * sizeof(double));
    for (int ix = NH; ix < Nx - NH; ++ix)
      for (int iz = izs; iz < Nz - NH; ++iz) {
        const size_t i = (size_t)ix * Nz + iz;
        double a1, a2, b1, b2;
        ds(c, f->vx, ix, iz, &a1, &a2);
        ds(c, f->vz, ix, iz, &b1, &b2);
        const double vxx = hx * (a1 + a2), vxz = hz * (a1 - a2), vzx = hx * (b1 + b2), vzz = hz * (b1 - b2);
        const double la = L.sxx[i], lb = L.szz[i], le = L.sxz[i], b = c->coef2[i];
        if (c->bond) {  /* sigma = H (vxx, vzz, vzx + vxz), H symmetric with c15, c35 */
          const double sh = vzx + vxz;
          gc11[i] += b * la * vxx;
          gc13[i] += b * (la * vzz + lb * vxx);
          gc15[i] += b * (la * sh + le * vxx);
          gc33[i] += b * lb * vzz;
          gc35[i] += b * (lb * sh + le * vzz);
          gc55[i] += b * le * sh;
          const double Lxx = b * (c->c11[i] * la + c->c13[i] * lb + c->c15[i] * le);
          const double Lzz = b * (c->c13[i] * la + c->c33[i] * lb + c->c35[i] * le);
          const double Lsh = b * (c->c15[i] * la + c->c35[i] * lb + c->c55[i] * le);
          T[0][i] = Lxx;
          T[1][i] = Lsh;
          T[2][i] = Lsh;
          T[3][i] = Lzz;
          L.sxx[i] *= c->coef1[i];
          L.szz[i] *= c->coef1[i];
          L.sxz[i] *= c->coef1[i];
          continue;
        }
        const double s = c->sn[i], co = c->cs[i];
        if (c->tensor) {
          /* forward: n = coef1 tau + coef2 H e(theta, v); tau' = n; sigma' = R(theta) n */
          const double s2 = s * s, c2 = co * co, st = 2.0 * s * co, cd = c2 - s2, sh = vxz + vzx;
          const double exx = c2 * vxx + s2 * vzz - 0.5 * st * sh, ezz = s2 * vxx + c2 * vzz + 0.5 * st * sh;
          const double exz = st * (vxx - vzz) + cd * sh;
          const double c11 = c->c11[i], c13 = c->c13[i], c33 = c->c33[i], c55 = c->c55[i], a = c->coef1[i];
          const double nxx = a * f->txx[i] + b * (c11 * exx + c13 * ezz);
          const double nzz = a * f->tzz[i] + b * (c13 * exx + c33 * ezz);
          const double nxz = a * f->txz[i] + b * c55 * exz;
          /* lambda_n = lambda_tau' + R^T lambda_sigma' */
          const double lxx = L.txx[i] + c2 * la + s2 * lb - 0.5 * st * le;
          const double lzz = L.tzz[i] + s2 * la + c2 * lb + 0.5 * st * le;
          const double lxz = L.txz[i] + st * la - st * lb + cd * le;
          gc11[i] += b * lxx * exx;
          gc13[i] += b * (lxx * ezz + lzz * exx);
          gc33[i] += b * lzz * ezz;
          gc55[i] += b * lxz * exz;
          /* theta: through the strain rotation and through R */
          const double dexx = st * (vzz - vxx) - cd * sh, dexz = 2.0 * cd * (vxx - vzz) - 2.0 * st * sh;
          const double dnxx = b * (c11 * dexx - c13 * dexx), dnzz = b * (c13 * dexx - c33 * dexx);
          const double dnxz = b * c55 * dexz;
          const double rxx_ = -st * nxx + st * nzz + 2.0 * cd * nxz, rzz_ = -rxx_;
          const double rxz_ = -cd * (nxx - nzz) - 2.0 * st * nxz;
          gth[i] += lxx * dnxx + lzz * dnzz + lxz * dnxz + la * rxx_ + lb * rzz_ + le * rxz_;
          /* lambda of the strain rates, then of the velocity derivatives */
          const double Lexx = b * (c11 * lxx + c13 * lzz), Lezz = b * (c13 * lxx + c33 * lzz), Lexz = b * c55 * lxz;
          const double Lsh = -0.5 * st * Lexx + 0.5 * st * Lezz + cd * Lexz;
          T[0][i] = c2 * Lexx + s2 * Lezz + st * Lexz;
          T[1][i] = Lsh;
          T[2][i] = Lsh;
          T[3][i] = s2 * Lexx + c2 * Lezz - st * Lexz;
          L.txx[i] = a * lxx;
          L.tzz[i] = a * lzz;
          L.txz[i] = a * lxz;
          L.sxx[i] = L.szz[i] = L.sxz[i] = 0.0;  /* sigma is overwritten by R tau */
          continue;
        }
        const double rxx = co * vxx - s * vxz, rxz = s * vxx + co * vxz;
        const double rzx = co * vzx - s * vzz, rzz = s * vzx + co * vzz;
        const double c11 = c->c11[i], c13 = c->c13[i], c33 = c->c33[i], c55 = c->c55[i];
        gc11[i] += b * la * rxx;
        gc13[i] += b * (la * rzz + lb * rxx);
        gc33[i] += b * lb * rzz;
        gc55[i] += b * le * (rzx + rxz);
        gth[i] += b * (la * (-c11 * rxz + c13 * rzx) + lb * (-c13 * rxz + c33 * rzx) + le * c55 * (rxx - rzz));
        const double Lxx = b * (c11 * la + c13 * lb), Lzz = b * (c13 * la + c33 * lb), Lq = b * c55 * le;
        T[0][i] = co * Lxx + s * Lq;   /* d/d vxx */
        T[1][i] = -s * Lxx + co * Lq;  /* d/d vxz */
        T[2][i] = co * Lq + s * Lzz;   /* d/d vzx */
        T[3][i] = -s * Lq + co * Lzz;  /* d/d vzz */
        L.sxx[i] *= c->coef1[i];
        L.szz[i] *= c->coef1[i];
        L.sxz[i] *= c->coef1[i];
      }
    /* transposed stress stencils onto the velocity nodes: minus the velocity-node pair */
    for (int ix = NH; ix < Nx - NH; ++ix)
      for (int iz = izs; iz < Nz - NH; ++iz) {
        const size_t i = (size_t)ix * Nz + iz;
        double p1, p2, q1, q2, r1, r2, s1, s2;
        dv(c, T[0], ix, iz, &p1, &p2);
        dv(c, T[1], ix, iz, &q1, &q2);
        dv(c, T[2], ix, iz, &r1, &r2);
        dv(c, T[3], ix, iz, &s1, &s2);
        L.vx[i] -= hx * (p1 + p2) + hz * (q1 - q2);
        L.vz[i] -= hx * (r1 + r2) + hz * (s1 - s2);
      }
    if (c->stype >= 2) {
      /* velocity cells outside the update (image rows, rim): v there holds the
       * injected samples, so lambda_v only accumulates the transposed stencils */
      for (int ix = 0; ix < Nx; ++ix)
        for (int iz = 0; iz < Nz; ++iz) {
          if (ix >= NH && ix < Nx - NH && iz >= izs && iz < Nz - NH) continue;
          double p1, p2, q1, q2, r1, r2, s1, s2;
          dv_rim(c, T[0], ix, iz, &p1, &p2);
          dv_rim(c, T[1], ix, iz, &q1, &q2);
          dv_rim(c, T[2], ix, iz, &r1, &r2);
          dv_rim(c, T[3], ix, iz, &s1, &s2);
          A2(L.vx, ix, iz) -= hx * (p1 + p2) + hz * (q1 - q2);
          A2(L.vz, ix, iz) -= hx * (r1 + r2) + hz * (s1 - s2);
        }
      /* source-wavelet gradient (adjoint of the velocity sources) */
      if (g_src) {
        int cx[121], cz[121];
        double wx[121], wz[121];
        for (int n = 0; n < c->nsrc; ++n) {
          const int m = vsrc_cells(c, n, cx, cz, wx, wz);
          double acc = 0.0;
          for (int q = 0; q < m; ++q) acc += wx[q] * A2(L.vx, cx[q], cz[q]) + wz[q] * A2(L.vz, cx[q], cz[q]);
          g_src[(size_t)n * c->nt + it] = acc;
        }
      }
    }
    /* adjoint of the velocity half */
    for (int k = 0; k < 6; ++k) memset(T[k], 0, Np * sizeof(double));
    for (int ix = NH; ix < Nx - NH; ++ix)
      for (int iz = izs; iz < Nz - NH; ++iz) {
        const size_t i = (size_t)ix * Nz + iz;
        double a1, a2, b1, b2, e1, e2;
        dv(c, f->sxx, ix, iz, &a1, &a2);
        dv(c, f->szz, ix, iz, &b1, &b2);
        dv(c, f->sxz, ix, iz, &e1, &e2);
        const double sxx_x = hx * (a1 + a2), sxx_z = hx * (a1 - a2);
        const double szz_x = hx * (b1 + b2), szz_z = hz * (b1 - b2);
        const double sxz_x = hx * (e1 + e2), sxz_z = hz * (e1 - e2);
        const double br = c->coef2[i] * c->ir[i];
        const double Fx = br * L.vx[i], Fz = br * L.vz[i];
        /* coordinate: rotation by theta_v; Bond: fx = sxx_x + sxz_z, fz = sxz_x + szz_z */
        const int norot = c->bond || c->tensor;
        const double cv = norot ? 1.0 : c->csv[i], sv = norot ? 0.0 : c->snv[i];
        if (!norot) {
          gsv[i] += Fx * (-sxx_z + sxz_x) + Fz * (-sxz_z + szz_x);
          gcv[i] += Fx * (sxx_x + sxz_z) + Fz * (sxz_x + szz_z);
        }
        const double Axx_x = cv * Fx, Axx_z = -sv * Fx;
        const double Axz_x = sv * Fx + cv * Fz, Axz_z = cv * Fx - sv * Fz;
        const double Azz_x = sv * Fz, Azz_z = cv * Fz;
        T[0][i] = hx * (Axx_x + Axx_z); /* sxx: both derivatives scaled by 1/dx */
        T[1][i] = hx * (Axx_x - Axx_z);
        T[2][i] = hx * Azz_x + hz * Azz_z;
        T[3][i] = hx * Azz_x - hz * Azz_z;
        T[4][i] = hx * Axz_x + hz * Axz_z;
        T[5][i] = hx * Axz_x - hz * Axz_z;
        L.vx[i] *= c->coef1[i];
        L.vz[i] *= c->coef1[i];
      }
    /* transposed velocity stencils onto the stress nodes: minus the stress-node pair
     * (rows above izStart included: the free-surface image reads them) */
    const int z_lo = c->fs ? izs - NH : izs;
    for (int ix = NH; ix < Nx - NH; ++ix)
      for (int iz = z_lo; iz < Nz - NH; ++iz) {
        const size_t i = (size_t)ix * Nz + iz;
        /* sigma_xx: d1 pair of T0 plus d2 pair of T1 (likewise for zz, xz) */
        double p1, p2, q1, q2, r1, r2, unused;
        ds(c, T[0], ix, iz, &p1, &unused);
        ds(c, T[1], ix, iz, &unused, &p2);
        ds(c, T[2], ix, iz, &q1, &unused);
        ds(c, T[3], ix, iz, &unused, &q2);
        ds(c, T[4], ix, iz, &r1, &unused);
        ds(c, T[5], ix, iz, &unused, &r2);
        L.sxx[i] -= p1 + p2;
        L.szz[i] -= q1 + q2;
        L.sxz[i] -= r1 + r2;
      }
  }
  /* chain rule: stiffness -> (vp, eps, delta); angles -> theta (degrees) */
  const double rad = c->scalar * M_PI / 180.0;
  for (int ix = 0; ix < Nx; ++ix)
    for (int iz = 0; iz < Nz; ++iz) {
      const size_t i = (size_t)ix * Nz + iz;
      const double B = c->beta[i];
      const double p = c->vp[i] / B, s = c->vs[i] / B, r = c->rho[i] * B;
      const double f = 1.0 - (s / p) * (s / p), e = c->eps[i], d = c->delta[i];
      const double q = sqrt(f * (f + 2.0 * d));
      const double dc11_dp = 2.0 * r * p * (1.0 + 2.0 * e), dc33_dp = 2.0 * r * p;
      const double dc13_dp = r * (2.0 * p * q + p * p * (f + d) / q * 2.0 * s * s / (p * p * p));
      double G11 = gc11[i], G13 = gc13[i], G33 = gc33[i];  /* gradients of the VTI moduli */
      if (c->bond) {
        const double th = c->scalar * c->theta[i] / 180.0 * M_PI;
        const double C11 = r * p * p * (1.0 + 2.0 * e), C13 = r * (p * p * q - s * s), C33 = r * p * p,
                     C55 = r * s * s;
        double dm[4][6];
        bond_moduli_grad(C11, C13, C33, C55, th, dm);
        double gm[6] = {gc11[i], gc13[i], gc15[i], gc33[i], gc35[i], gc55[i]};
        if (c->fs && iz == c->E) {  /* only the effective c11 acts on the free-surface row */
          double m[6], dc[6];
          bond_moduli(C11, C13, C33, C55, th, m);
          bond_fs_c11(m, dc);
          const double g = gc11[i];
          for (int k = 0; k < 6; ++k) gm[k] = g * dc[k];
        }
        G11 = G13 = G33 = 0.0;
        double gt = 0.0;
        for (int k = 0; k < 6; ++k) {
          G11 += gm[k] * dm[0][k];
          G13 += gm[k] * dm[1][k];
          G33 += gm[k] * dm[2][k];
          gt += gm[k] * dm[3][k];
        }
        g_theta[i] = gt * rad;
      }
      g_vp[i] = (G11 * dc11_dp + G13 * dc13_dp + G33 * dc33_dp) / B;
      g_eps[i] = G11 * 2.0 * r * p * p;
      g_delta[i] = G13 * r * p * p * f / q;
      if (c->tensor) g_theta[i] = gth[i] * rad;  /* no rotation at the velocity node */
      if (c->bond || c->tensor) continue;
      /* theta at the stress node, plus the velocity-node averages that read it */
      double gt = gth[i];
      const double sn = c->sn[i], cs = c->cs[i];
      for (int a = 0; a <= 1; ++a)
        for (int b = 0; b <= 1; ++b) {
          const int vx = ix - a, vz = iz - b;
          if (vx < 0 || vz < 0) continue;
          const int inner = vx < Nx - 1 && vz < Nz - 1;
          if (!inner && (a || b)) continue;
          const double w = inner ? 0.25 : 1.0;
          const size_t j = (size_t)vx * Nz + vz;
          gt += w * (gsv[j] * cs - gcv[j] * sn);
        }
      g_theta[i] = gt * rad;
    }
  for (int it = 0; it < c->nt; ++it) state_free(&keep[it]);
  free(keep);
  state_free(&L);
  for (int k = 0; k < 6; ++k) free(T[k]);
  free(gc11);
  free(gc13);
  free(gc33);
  free(gc55);
  free(gth);
  free(gsv);
  free(gc15);
  free(gc35);
  free(gcv);
  for (int k = 0; k < 3; ++k) free(rec[k]);
  return J;
}
