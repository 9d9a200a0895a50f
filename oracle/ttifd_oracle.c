/*
 * CPU restatement of the reference's 2D TTI elastic RSG modelling loop.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the oracle the CUDA library is
 * checked against; it is never linked into the product. It restates, cell by
 * cell and with the reference's floating-point expression order (so that a
 * gcc -ffp-contract=off build reproduces the reference's own build bit for
 * bit), the following reference code (paths relative to the reference root;
 * coord = src/main/sufdmod2dTTIelastic/sufdmod2dTTIelastic_coordinate_rotation.c,
 * tensor = ..._tensor_rotation.c, bond = ..._bond_transformation.c):
 *
 *   RSG coefficients            coord:468-474
 *   stability limit             src/lib/fdmod/stable.c:217-246
 *   MEAL damping / scaling      src/lib/absorbc/meal.c:23-29, 51-201
 *   MEAL FD coefficients        src/lib/absorbc/meal.c:450-502 (order 1)
 *   stiffness build             coord:497-537, tensor:498-535, bond:492-541
 *   Bond free-surface rewrite   bond:543-568
 *   velocity update             coord:614-672, tensor:617-666, bond:654-703
 *   velocity sources stype 2-8  coord:674-802
 *   stress update               coord:804-845, tensor:799-851, bond:836-873
 *   free surface                coord:847-863
 *   stress source stype 1       coord:865-886, tensor:871-895
 *   receivers                   src/lib/fdmod/isoelastic.c:103-144
 *   snapshots                   src/lib/fdmod/isoelastic.c:240-289, snapshot.c:28-39
 *   energy                      coord:898-924
 *   model padding               src/lib/absorbc/padmod.c:33-59
 *   vp->vs, vp->rho defaults    src/lib/rockmod/modparconvert.c:42-58, 128-141
 *   Ricker wavelet              src/lib/wavelet/wavelet.c:81-99
 */
#include "ttifd_oracle.h"

#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef ORC_PI
#define ORC_PI 3.14159265358979323846
#endif

enum { NHALF = 5 }; /* half length of the 10th-order RSG operator (coord:309) */

/* least-squares RSG coefficients, coord:468-469 */
static const float RSG[NHALF] = {1.24362739770907f, -0.114021164233934f, 0.0272965993810630f,
                                 -0.00699199493927320f, 0.00132022981661381f};

struct orc_ctx {
  tti_config cfg;
  int E, Nz, Nx, izStart;
  size_t Np;
  int have_model;
  float *par[TTI_P_COUNT];
  float *fld[8];
  int nsrc;
  int *sx, *sz;
  float *src; /* [nsrc][nt] */
  int nrec[3];
  int *rx[3], *rz[3];
  float *rec[3]; /* [ntrace][nts] */
  int nts;
  float *ek, *ep;
  int step_index; /* number of steps taken since reset */
  char msg[512];
};

static int fail(orc_ctx *c, int code, const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(c->msg, sizeof c->msg, fmt, ap);
  va_end(ap);
  return code;
}

#define AT(a, ix, iz) ((a)[(size_t)(ix) * (size_t)Nz + (size_t)(iz)])

/* ------------------------------------------------------------------ */
/* free-standing helpers                                               */
/* ------------------------------------------------------------------ */

/* padmod.c:33-59: replicate the edge rows into the top/bottom rims of the
 * interior columns, then whole edge columns into the left/right rims. */
void orc_pad_model(float *mod, int Nx, int Nz, int nlayer)
{
  for (int ix = nlayer; ix < Nx - nlayer; ++ix) {
    float top = AT(mod, ix, nlayer), bot = AT(mod, ix, Nz - nlayer - 1);
    for (int k = 1; k <= nlayer; ++k) {
      AT(mod, ix, nlayer - k) = top;
      AT(mod, ix, Nz - nlayer - 1 + k) = bot;
    }
  }
  for (int k = 1; k <= nlayer; ++k)
    for (int iz = 0; iz < Nz; ++iz) {
      AT(mod, nlayer - k, iz) = AT(mod, nlayer, iz);
      AT(mod, Nx - nlayer - 1 + k, iz) = AT(mod, Nx - nlayer - 1, iz);
    }
}

/* modparconvert.c:42-58 */
void orc_vp2vs(const float *vp, float *vs, int n)
{
  for (int i = 0; i < n; ++i) vs[i] = vp[i] <= 1500.0 ? 0.0f : (float)(0.577350269189626 * vp[i]);
}

/* modparconvert.c:128-141 (Gardner) */
void orc_vp2rho_gardner(const float *vp, float *rho, int n)
{
  for (int i = 0; i < n; ++i) rho[i] = vp[i] <= 1500.0 ? 1000.0f : (float)(1741.0 * pow(vp[i] / 1000.0, 0.25));
}

/* stable.c:217-246: dt_max = 1 / (vp_max sqrt((1/dx^2 + 1/dz^2) (C1 + C3 + C5))) */
double orc_dt_max(const float *vp, int Nx, int Nz, float dx, float dz)
{
  double vmax = FLT_MIN;
  size_t n = (size_t)Nx * (size_t)Nz;
  for (size_t i = 0; i < n; ++i) vmax = fmaxf(vp[i], (float)vmax);
  double csum = 0.0f;
  for (int k = 0; k < NHALF; k += 2) csum += RSG[k] * pow(-1.0, 1.0 * k);
  return 1.0f / (vmax * sqrt((1.0 / (dx * dx) + 1.0 / (dz * dz)) * csum));
}

/* wavelet.c:81-99 */
void orc_ricker(float *src, float A, float fpeak, float delay, float dt, int nt)
{
  const float pi = 3.141592654f;
  for (int it = 0; it < nt; ++it) {
    float t = it * dt - delay;
    src[it] = t <= delay ? A * (1.0f - 2.0f * powf(pi * fpeak * t, 2.0f)) * expf(-1.0f * powf(pi * fpeak * t, 2.0f))
                         : 0.0f;
  }
  if (nt > 0) src[0] = 0.0f;
}

/* ------------------------------------------------------------------ */
/* context                                                             */
/* ------------------------------------------------------------------ */
orc_ctx *orc_create(const tti_config *cfg)
{
  orc_ctx *c = (orc_ctx *)calloc(1, sizeof *c);
  if (!c) return NULL;
  c->cfg = *cfg;
  c->E = cfg->ealThick + NHALF;
  c->Nz = cfg->nz + 2 * c->E;
  c->Nx = cfg->nx + 2 * c->E;
  c->Np = (size_t)c->Nz * (size_t)c->Nx;
  c->izStart = cfg->freesurface == 0 ? NHALF : c->E;
  c->nts = cfg->mt > 0 ? (cfg->nt - 1) / cfg->mt + 1 : 0;
  for (int f = 0; f < 8; ++f) c->fld[f] = (float *)calloc(c->Np, sizeof(float));
  for (int p = 0; p < TTI_P_COUNT; ++p) c->par[p] = (float *)calloc(c->Np, sizeof(float));
  c->ek = (float *)calloc(cfg->nt > 0 ? cfg->nt : 1, sizeof(float));
  c->ep = (float *)calloc(cfg->nt > 0 ? cfg->nt : 1, sizeof(float));
  return c;
}

void orc_destroy(orc_ctx *c)
{
  if (!c) return;
  for (int f = 0; f < 8; ++f) free(c->fld[f]);
  for (int p = 0; p < TTI_P_COUNT; ++p) free(c->par[p]);
  for (int k = 0; k < 3; ++k) {
    free(c->rx[k]);
    free(c->rz[k]);
    free(c->rec[k]);
  }
  free(c->sx);
  free(c->sz);
  free(c->src);
  free(c->ek);
  free(c->ep);
  free(c);
}

const char *orc_last_error(const orc_ctx *c) { return c ? c->msg : "null context"; }

int orc_grid(const orc_ctx *c, int *Nz, int *Nx, int *E)
{
  *Nz = c->Nz;
  *Nx = c->Nx;
  *E = c->E;
  return TTI_OK;
}

/* ------------------------------------------------------------------ */
/* setup: MEAL (meal.c:51-201, 450-502) and stiffness                  */
/* ------------------------------------------------------------------ */

/* meal.c:23-29 */
static float meal_weight(float alpha, int l, int nlayer)
{
  float d = (0.1f * l) / (0.1f * nlayer);
  return expf(logf(2.0f) * powf(d, alpha)) - 1.0f;
}

static void meal_profile(orc_ctx *c, const float *vp, const float *vs)
{
  const tti_config *g = &c->cfg;
  const int Nz = c->Nz, Nx = c->Nx, nl = c->E;
  const float pd = 2, PPWfd = 10.0f;
  const float Rcoef = powf(10.0f, -1.0f * ((log10f(nl) - 1.0f) / (log10f(2.0f))) - 3.0f - 0.5f * pd);
  const float thx = nl * g->dx, thz = nl * g->dz;
  const float alpha = g->eal_alpha == -1.0f ? 2.5f : g->eal_alpha;
  const int izs = g->freesurface == 0 ? 0 : nl;
  float *D = c->par[TTI_P_D], *Beta = c->par[TTI_P_BETA];
#pragma omp parallel for
  for (int ix = 0; ix < Nx; ++ix) {
    for (int iz = 0; iz < Nz; ++iz) {
      float v = AT(vp, ix, iz);
      float Vs = AT(vs, ix, iz) == 0.0f ? v / sqrtf(3.0f) : AT(vs, ix, iz);
      float Dx = 0.0f, Dz = 0.0f, Bx = 1.0f, Bz = 1.0f;
      int lz = 0, lx = 0;
      if (g->freesurface == 0 && iz < nl) lz = nl - iz;  /* top rim */
      if (iz >= Nz - nl) lz = iz - (Nz - nl - 1);        /* bottom rim */
      if (iz >= izs && ix < nl) lx = nl - ix;            /* left rim */
      if (iz >= izs && ix >= Nx - nl) lx = ix - (Nx - nl - 1); /* right rim */
      if (lz) {
        float w = meal_weight(alpha, lz, nl);
        float d0 = -1.0f * (1.0f + pd) * v * logf(Rcoef) / (2.0f * thz);
        float beta = 2.0f * (Vs / (g->dz * g->fpeak)) / PPWfd;
        Dz = d0 * w;
        Bz = 1.0f + (beta - 1.0f) * w;
      }
      if (lx) {
        float w = meal_weight(alpha, lx, nl);
        float d0 = -1.0f * (1.0f + pd) * v * logf(Rcoef) / (2.0f * thx);
        float beta = 2.0f * (Vs / (g->dx * g->fpeak)) / PPWfd;
        Dx = d0 * w;
        Bx = 1.0f + (beta - 1.0f) * w;
      }
      AT(D, ix, iz) = sqrtf(powf(Dx, 2.0f) + powf(Dz, 2.0f));
      AT(Beta, ix, iz) = sqrtf(powf(Bx - 1.0f, 2.0f) + powf(Bz - 1.0f, 2.0f)) + 1.0f;
    }
  }
}

int orc_upload_model(orc_ctx *c, const float *vp0, const float *vs0, const float *rho0, const float *eps,
                     const float *delta, const float *theta0)
{
  const tti_config *g = &c->cfg;
  const int Nz = c->Nz, Nx = c->Nx;
  const size_t Np = c->Np;
  double dtmax = orc_dt_max(vp0, Nx, Nz, g->dx, g->dz);
  if (g->dt > dtmax)
    return fail(c, TTI_ERR_UNSTABLE,
                "the finite differenct scheme is unstable! the time step size must smaller than %5.5f!", dtmax);
  float *vp = c->par[TTI_P_VP], *vs = c->par[TTI_P_VS], *rho = c->par[TTI_P_RHO];
  memcpy(vp, vp0, Np * sizeof(float));
  memcpy(vs, vs0, Np * sizeof(float));
  memcpy(rho, rho0, Np * sizeof(float));
  meal_profile(c, vp, vs);
  float *D = c->par[TTI_P_D], *Beta = c->par[TTI_P_BETA];
  float *coef1 = c->par[TTI_P_COEF1], *coef2 = c->par[TTI_P_COEF2];
  /* meal.c:450-490, order 1 */
  for (size_t i = 0; i < Np; ++i) {
    vp[i] /= Beta[i];
    vs[i] /= Beta[i];
    rho[i] *= Beta[i];
    D[i] /= Beta[i];
    coef1[i] = (1.0 - 0.5 * g->dt * D[i]) / (1.0 + 0.5 * g->dt * D[i]);
    coef2[i] = g->dt / (1.0 + 0.5 * g->dt * D[i]);
  }
  float *th = (float *)malloc(Np * sizeof(float));
  /* per-cell stiffness, coord:497-515 / tensor:500-519 / bond:493-526 */
#pragma omp parallel for
  for (size_t i = 0; i < Np; ++i) {
    double f = 1.0 - pow(vs[i] / vp[i], 2.0);
    th[i] = g->scalar * theta0[i] / 180.0 * ORC_PI;
    if (g->variant == TTI_BOND) {
      double C11 = rho[i] * vp[i] * vp[i] * (1.0 + 2.0 * eps[i]);
      double C13 = rho[i] * (vp[i] * vp[i] * sqrt(f * (f + 2.0 * delta[i])) - vs[i] * vs[i]);
      double C33 = rho[i] * vp[i] * vp[i];
      double C55 = rho[i] * vs[i] * vs[i];
      double s2 = sin(th[i]) * sin(th[i]), c2 = cos(th[i]) * cos(th[i]);
      double s4 = s2 * s2, c4 = c2 * c2;
      double s2t = sin(2.0 * th[i]), c2t = cos(2.0 * th[i]);
      double s22 = s2t * s2t, c22 = c2t * c2t;
      c->par[TTI_P_C11][i] = C11 * c4 + C33 * s4 + (0.5 * C13 + C55) * s22;
      c->par[TTI_P_C13][i] = (0.25 * (C11 + C33) - C55) * s22 + C13 * (s4 + c4);
      c->par[TTI_P_C15][i] = 0.5 * (-1.0 * C11 * c2 + C33 * s2 + (C13 + 2.0 * C55) * c2t) * s2t;
      c->par[TTI_P_C33][i] = C11 * s4 + C33 * c4 + (0.5 * C13 + C55) * s22;
      c->par[TTI_P_C35][i] = 0.5 * (-1.0 * C11 * s2 + C33 * c2 - (C13 + 2.0 * C55) * c2t) * s2t;
      c->par[TTI_P_C55][i] = 0.25 * (C11 + C33 - 2.0 * C13) * s22 + C55 * c22;
    } else {
      c->par[TTI_P_C11][i] = rho[i] * vp[i] * vp[i] * (1.0 + 2.0 * eps[i]);
      c->par[TTI_P_C13][i] = rho[i] * (vp[i] * vp[i] * sqrt(f * (f + 2.0 * delta[i])) - vs[i] * vs[i]);
      c->par[TTI_P_C33][i] = rho[i] * vp[i] * vp[i];
      c->par[TTI_P_C55][i] = rho[i] * vs[i] * vs[i];
      if (g->variant == TTI_COORDINATE) {
        c->par[TTI_P_SIN][i] = sin(th[i]);
        c->par[TTI_P_COS][i] = cos(th[i]);
      } else {
        c->par[TTI_P_SIN2][i] = sin(th[i]) * sin(th[i]);
        c->par[TTI_P_COS2][i] = cos(th[i]) * cos(th[i]);
        c->par[TTI_P_SIN_2T][i] = sin(2.0 * th[i]);
      }
    }
  }
  free(th);
  /* buoyancy and theta averaged onto the velocity node (ix+1/2, iz+1/2);
   * the last row and column keep the stress-node value (coord:516-537) */
  float *ir = c->par[TTI_P_INVRHO];
  const float *s = c->par[TTI_P_SIN], *co = c->par[TTI_P_COS];
#pragma omp parallel for
  for (int ix = 0; ix < Nx; ++ix)
    for (int iz = 0; iz < Nz; ++iz) {
      int inner = ix < Nx - 1 && iz < Nz - 1;
      if (inner) {
        AT(ir, ix, iz) = 4.0 / (AT(rho, ix, iz) + AT(rho, ix + 1, iz) + AT(rho, ix, iz + 1) + AT(rho, ix + 1, iz + 1));
      } else {
        AT(ir, ix, iz) = 1.0 / AT(rho, ix, iz);
      }
      if (g->variant == TTI_COORDINATE) {
        if (inner) {
          AT(c->par[TTI_P_SIN_V], ix, iz) =
              0.25 * (AT(s, ix, iz) + AT(s, ix + 1, iz) + AT(s, ix, iz + 1) + AT(s, ix + 1, iz + 1));
          AT(c->par[TTI_P_COS_V], ix, iz) =
              0.25 * (AT(co, ix, iz) + AT(co, ix + 1, iz) + AT(co, ix, iz + 1) + AT(co, ix + 1, iz + 1));
        } else {
          AT(c->par[TTI_P_SIN_V], ix, iz) = AT(s, ix, iz);
          AT(c->par[TTI_P_COS_V], ix, iz) = AT(co, ix, iz);
        }
      }
    }
  /* bond:543-568: the free-surface row gets an effective c11 and the other
   * moduli vanish; c35 is replaced first and c55 uses the new c35 */
  if (g->variant == TTI_BOND && g->freesurface == 1) {
    float *c11 = c->par[TTI_P_C11], *c13 = c->par[TTI_P_C13], *c15 = c->par[TTI_P_C15];
    float *c33 = c->par[TTI_P_C33], *c35 = c->par[TTI_P_C35], *c55 = c->par[TTI_P_C55];
    const int iz = c->E;
    for (int ix = 0; ix < Nx; ++ix) {
      float a13 = AT(c13, ix, iz), a15 = AT(c15, ix, iz), a33 = AT(c33, ix, iz);
      float a35 = AT(c35, ix, iz), a55 = AT(c55, ix, iz);
      float n35 = -(a13 * a55 - a15 * a35) / (a33 * a55 - a35 * a35);
      float n55 = (a13 * n35 - a15 * a33) / (a33 * a55 - n35 * n35);
      if (isnan(n35) || isinf(n35)) n35 = -a13 / a33;
      if (isnan(n35) || isinf(n35)) n35 = 0.0f;
      AT(c11, ix, iz) = AT(c11, ix, iz) - a13 * n35 + a15 * n55;
      AT(c13, ix, iz) = AT(c15, ix, iz) = AT(c33, ix, iz) = AT(c35, ix, iz) = AT(c55, ix, iz) = 0.0f;
    }
  }
  c->have_model = 1;
  return TTI_OK;
}

int orc_fetch_param(orc_ctx *c, int which, float *out)
{
  if (which < 0 || which >= TTI_P_COUNT) return fail(c, TTI_ERR_ARG, "bad param id %d", which);
  memcpy(out, c->par[which], c->Np * sizeof(float));
  return TTI_OK;
}

/* ------------------------------------------------------------------ */
/* geometry                                                            */
/* ------------------------------------------------------------------ */
int orc_set_source(orc_ctx *c, int ntrace, const int *posx, const int *posz, const float *src)
{
  for (int i = 0; i < ntrace; ++i) {
    if (posz[i] < 0 || posz[i] > c->cfg.nz)
      return fail(c, TTI_ERR_RANGE, "the position of source in 1st dimension (%d) must be between 0 and %d!", posz[i],
                  c->cfg.nz);
    if (posx[i] < 0 || posx[i] > c->cfg.nx)
      return fail(c, TTI_ERR_RANGE, "the position of source in 2nd dimension (%d) must be between 0 and %d!", posx[i],
                  c->cfg.nx);
  }
  free(c->sx);
  free(c->sz);
  free(c->src);
  c->nsrc = ntrace;
  c->sx = (int *)malloc(sizeof(int) * (ntrace ? ntrace : 1));
  c->sz = (int *)malloc(sizeof(int) * (ntrace ? ntrace : 1));
  c->src = (float *)malloc(sizeof(float) * (size_t)(ntrace ? ntrace : 1) * c->cfg.nt);
  memcpy(c->sx, posx, sizeof(int) * ntrace);
  memcpy(c->sz, posz, sizeof(int) * ntrace);
  memcpy(c->src, src, sizeof(float) * (size_t)ntrace * c->cfg.nt);
  return TTI_OK;
}

int orc_set_receivers(orc_ctx *c, int kind, int ntrace, const int *posx, const int *posz)
{
  if (kind < 0 || kind > 2) return fail(c, TTI_ERR_ARG, "bad receiver kind %d", kind);
  for (int i = 0; i < ntrace; ++i) {
    if (posz[i] < 0 || posz[i] > c->cfg.nz)
      return fail(c, TTI_ERR_RANGE, "the position of receiver in 1st dimension (%d) must be between 0 and %d!",
                  posz[i], c->cfg.nz);
    if (posx[i] < 0 || posx[i] > c->cfg.nx)
      return fail(c, TTI_ERR_RANGE, "the position of receiver in 2nd dimension (%d) must be between 0 and %d!",
                  posx[i], c->cfg.nx);
  }
  free(c->rx[kind]);
  free(c->rz[kind]);
  free(c->rec[kind]);
  c->nrec[kind] = ntrace;
  c->rx[kind] = (int *)malloc(sizeof(int) * (ntrace ? ntrace : 1));
  c->rz[kind] = (int *)malloc(sizeof(int) * (ntrace ? ntrace : 1));
  c->rec[kind] = (float *)calloc((size_t)(ntrace ? ntrace : 1) * c->nts, sizeof(float));
  memcpy(c->rx[kind], posx, sizeof(int) * ntrace);
  memcpy(c->rz[kind], posz, sizeof(int) * ntrace);
  return TTI_OK;
}

int orc_reset(orc_ctx *c)
{
  for (int f = 0; f < 8; ++f) memset(c->fld[f], 0, c->Np * sizeof(float));
  for (int k = 0; k < 3; ++k)
    if (c->rec[k]) memset(c->rec[k], 0, sizeof(float) * (size_t)c->nrec[k] * c->nts);
  memset(c->ek, 0, sizeof(float) * c->cfg.nt);
  memset(c->ep, 0, sizeof(float) * c->cfg.nt);
  c->step_index = 0;
  return TTI_OK;
}

int orc_current_it(const orc_ctx *c)
{
  return c->cfg.mode == 2 ? c->cfg.nt - 1 - c->step_index : c->step_index;
}

/* ------------------------------------------------------------------ */
/* the RSG derivative pairs                                            */
/* ------------------------------------------------------------------ */

/* Velocity node (ix+1/2, iz+1/2) from stress nodes, coord:621-630:
 *   d1 = sum_k C_k (a[x+k][z+k]   - a[x-k+1][z-k+1])   (main diagonal)
 *   d2 = sum_k C_k (a[x+k][z-k+1] - a[x-k+1][z+k])     (anti-diagonal) */
static inline void diag_at_v(const float *a, int Nz, int ix, int iz, float *d1, float *d2)
{
  float s1 = RSG[0] * (AT(a, ix + 1, iz + 1) - AT(a, ix, iz));
  float s2 = RSG[0] * (AT(a, ix + 1, iz) - AT(a, ix, iz + 1));
  for (int k = 2; k <= NHALF; ++k) {
    s1 = s1 + RSG[k - 1] * (AT(a, ix + k, iz + k) - AT(a, ix - k + 1, iz - k + 1));
    s2 = s2 + RSG[k - 1] * (AT(a, ix + k, iz - k + 1) - AT(a, ix - k + 1, iz + k));
  }
  *d1 = s1;
  *d2 = s2;
}

/* Stress node (ix, iz) from velocity nodes, coord:811-816:
 *   d1 = sum_k C_k (a[x+k-1][z+k-1] - a[x-k][z-k])
 *   d2 = sum_k C_k (a[x+k-1][z-k]   - a[x-k][z+k-1]) */
static inline void diag_at_s(const float *a, int Nz, int ix, int iz, float *d1, float *d2)
{
  float s1 = RSG[0] * (AT(a, ix, iz) - AT(a, ix - 1, iz - 1));
  float s2 = RSG[0] * (AT(a, ix, iz - 1) - AT(a, ix - 1, iz));
  for (int k = 2; k <= NHALF; ++k) {
    s1 = s1 + RSG[k - 1] * (AT(a, ix + k - 1, iz + k - 1) - AT(a, ix - k, iz - k));
    s2 = s2 + RSG[k - 1] * (AT(a, ix + k - 1, iz - k) - AT(a, ix - k, iz + k - 1));
  }
  *d1 = s1;
  *d2 = s2;
}

/* ------------------------------------------------------------------ */
/* one time step                                                       */
/* ------------------------------------------------------------------ */
static void velocity_update(orc_ctx *c)
{
  const tti_config *g = &c->cfg;
  const int Nz = c->Nz, Nx = c->Nx, z0 = c->izStart;
  const float invdx = 1.0 / g->dx, invdz = 1.0 / g->dz;
  float *vx = c->fld[TTI_F_VX], *vz = c->fld[TTI_F_VZ];
  const float *sxx = c->fld[TTI_F_SXX], *szz = c->fld[TTI_F_SZZ], *sxz = c->fld[TTI_F_SXZ];
  float **P = c->par;
#pragma omp parallel for
  for (int ix = NHALF; ix < Nx - NHALF; ++ix)
    for (int iz = z0; iz < Nz - NHALF; ++iz) {
      float d1, d2;
      size_t i = (size_t)ix * Nz + iz;
      diag_at_v(sxx, Nz, ix, iz, &d1, &d2);
      float sxx_x = 0.5f * (d1 + d2) * invdx;
      float sxx_z = 0.5f * (d1 - d2) * invdx; /* coord:633 uses invdx */
      diag_at_v(szz, Nz, ix, iz, &d1, &d2);
      float szz_x = 0.5f * (d1 + d2) * invdx;
      float szz_z = 0.5f * (d1 - d2) * invdz;
      diag_at_v(sxz, Nz, ix, iz, &d1, &d2);
      float sxz_x = 0.5f * (d1 + d2) * invdx;
      float sxz_z = 0.5f * (d1 - d2) * invdz;
      float a = P[TTI_P_COEF1][i], b = P[TTI_P_COEF2][i], r = P[TTI_P_INVRHO][i];
      if (g->variant == TTI_COORDINATE) {
        float cv = P[TTI_P_COS_V][i], sv = P[TTI_P_SIN_V][i];
        vx[i] = a * vx[i] + b * r * (cv * sxx_x - sv * sxx_z + sv * sxz_x + cv * sxz_z);
        vz[i] = a * vz[i] + b * r * (cv * sxz_x - sv * sxz_z + sv * szz_x + cv * szz_z);
      } else {
        vx[i] = a * vx[i] + b * r * (sxx_x + sxz_z);
        vz[i] = a * vz[i] + b * r * (sxz_x + szz_z);
      }
    }
}

static void stress_update(orc_ctx *c)
{
  const tti_config *g = &c->cfg;
  const int Nz = c->Nz, Nx = c->Nx, z0 = c->izStart;
  const float invdx = 1.0 / g->dx, invdz = 1.0 / g->dz;
  const float *vx = c->fld[TTI_F_VX], *vz = c->fld[TTI_F_VZ];
  float *sxx = c->fld[TTI_F_SXX], *szz = c->fld[TTI_F_SZZ], *sxz = c->fld[TTI_F_SXZ];
  float *txx = c->fld[TTI_F_TXX], *tzz = c->fld[TTI_F_TZZ], *txz = c->fld[TTI_F_TXZ];
  float **P = c->par;
#pragma omp parallel for
  for (int ix = NHALF; ix < Nx - NHALF; ++ix)
    for (int iz = z0; iz < Nz - NHALF; ++iz) {
      float d1, d2;
      size_t i = (size_t)ix * Nz + iz;
      diag_at_s(vx, Nz, ix, iz, &d1, &d2);
      float vxx = 0.5f * (d1 + d2) * invdx, vxz = 0.5f * (d1 - d2) * invdz;
      diag_at_s(vz, Nz, ix, iz, &d1, &d2);
      float vzx = 0.5f * (d1 + d2) * invdx, vzz = 0.5f * (d1 - d2) * invdz;
      float a = P[TTI_P_COEF1][i], b = P[TTI_P_COEF2][i];
      float c11 = P[TTI_P_C11][i], c13 = P[TTI_P_C13][i], c33 = P[TTI_P_C33][i], c55 = P[TTI_P_C55][i];
      if (g->variant == TTI_COORDINATE) {
        /* rotate the gradient into the symmetry frame, coord:821-837 */
        float s = P[TTI_P_SIN][i], co = P[TTI_P_COS][i];
        float r = s * vxx + co * vxz;
        vxx = co * vxx - s * vxz;
        vxz = r;
        r = s * vzx + co * vzz;
        vzx = co * vzx - s * vzz;
        vzz = r;
        sxx[i] = a * sxx[i] + b * (c11 * vxx + c13 * vzz);
        szz[i] = a * szz[i] + b * (c13 * vxx + c33 * vzz);
        sxz[i] = a * sxz[i] + b * c55 * (vzx + vxz);
      } else if (g->variant == TTI_TENSOR) {
        /* rotated strain rates, Hooke on tau, then sigma = R tau (tensor:826-851) */
        float s2 = P[TTI_P_SIN2][i], c2 = P[TTI_P_COS2][i], st = P[TTI_P_SIN_2T][i];
        float exx = c2 * vxx + s2 * vzz - 0.5f * st * (vxz + vzx);
        float ezz = s2 * vxx + c2 * vzz + 0.5f * st * (vxz + vzx);
        float exz = st * (vxx - vzz) + (c2 - s2) * (vxz + vzx);
        float nxx = a * txx[i] + b * (c11 * exx + c13 * ezz);
        float nzz = a * tzz[i] + b * (c13 * exx + c33 * ezz);
        float nxz = a * txz[i] + b * c55 * exz;
        txx[i] = nxx;
        tzz[i] = nzz;
        txz[i] = nxz;
        sxx[i] = c2 * nxx + s2 * nzz + st * nxz;
        szz[i] = s2 * nxx + c2 * nzz - st * nxz;
        sxz[i] = -0.5f * st * (nxx - nzz) + (c2 - s2) * nxz;
      } else {
        float c15 = P[TTI_P_C15][i], c35 = P[TTI_P_C35][i];
        sxx[i] = a * sxx[i] + b * (c11 * vxx + c13 * vzz + c15 * (vzx + vxz));
        szz[i] = a * szz[i] + b * (c13 * vxx + c33 * vzz + c35 * (vzx + vxz));
        sxz[i] = a * sxz[i] + b * (c15 * vxx + c35 * vzz + c55 * (vzx + vxz));
      }
    }
}

/* coord:847-863: stress image about row izStart */
static void free_surface(orc_ctx *c)
{
  const int Nz = c->Nz, Nx = c->Nx, s = c->izStart;
  float *sxx = c->fld[TTI_F_SXX], *szz = c->fld[TTI_F_SZZ], *sxz = c->fld[TTI_F_SXZ];
  for (int ix = NHALF; ix < Nx - NHALF; ++ix) {
    AT(sxz, ix, s) = 0.0f;
    AT(szz, ix, s) = 0.0f;
    for (int k = 1; k <= NHALF; ++k) {
      AT(sxx, ix, s - k) = 2.0f * AT(sxx, ix, s) - AT(sxx, ix, s + k);
      AT(szz, ix, s - k) = -AT(szz, ix, s + k);
      AT(sxz, ix, s - k) = -AT(sxz, ix, s + k);
    }
  }
}

/* Gaussian-smoothed point sources (coord:674-802 and 865-886):
 * weight = exp(alpha r^2) dt/(dx dz), alpha = ln 0.8 / (dx^2 + dz^2),
 * applied over the 11 x 11 cells around each source. `stage` 0 applies the
 * velocity sources (after the velocity update), 1 the stress source. */
static void apply_sources(orc_ctx *c, int it, int stage)
{
  const tti_config *g = &c->cfg;
  const int Nz = c->Nz, Nx = c->Nx, E = c->E, st = g->stype;
  const float invdx = 1.0 / g->dx, invdz = 1.0 / g->dz;
  const float alpha = logf(0.8f) / (g->dx * g->dx + g->dz * g->dz);
  float *vx = c->fld[TTI_F_VX], *vz = c->fld[TTI_F_VZ];
  if (stage == 0 && st == 8) {
    const float q = 0.125f * sqrtf(2.0f);
    for (int s = 0; s < c->nsrc; ++s) {
      int x = c->sx[s] + E, z = c->sz[s] + E;
      float a = c->src[(size_t)s * g->nt + it];
      AT(vx, x, z) -= q * a;
      AT(vz, x, z) += q * a;
      AT(vx, x - 1, z) -= q * a;
      AT(vz, x - 1, z) -= q * a;
      AT(vx, x - 1, z - 1) += q * a;
      AT(vz, x - 1, z - 1) -= q * a;
      AT(vx, x, z - 1) += q * a;
      AT(vz, x, z - 1) += q * a;
    }
    return;
  }
  /* pass list: the divergence pass runs over all sources before the curl
   * pass, as the reference's two separate blocks do for stype 4 */
  int passes[2], np = 0;
  if (stage == 0) {
    if (st == 2 || st == 4) passes[np++] = 2;
    if (st == 3 || st == 4) passes[np++] = 3;
    if (st == 5 || st == 6 || st == 7) passes[np++] = st;
  } else if (st == 1) {
    passes[np++] = 1;
  }
  for (int p = 0; p < np; ++p) {
    int kind = passes[p];
    for (int s = 0; s < c->nsrc; ++s) {
      int x0 = c->sx[s] + E, z0 = c->sz[s] + E;
      float a = c->src[(size_t)s * g->nt + it];
      int xa = x0 - NHALF > 0 ? x0 - NHALF : 0, xb = x0 + NHALF < Nx - 1 ? x0 + NHALF : Nx - 1;
      int za = z0 - NHALF > 0 ? z0 - NHALF : 0, zb = z0 + NHALF < Nz - 1 ? z0 + NHALF : Nz - 1;
      for (int ix = xa; ix <= xb; ++ix) {
        float rx = (ix - x0) * g->dx;
        for (int iz = za; iz <= zb; ++iz) {
          float rz = (iz - z0) * g->dz;
          float w = expf(alpha * (rx * rx + rz * rz)) * invdx * invdz * g->dt;
          switch (kind) {
          case 1:
            AT(c->fld[TTI_F_SXX], ix, iz) += 0.5f * w * a;
            AT(c->fld[TTI_F_SZZ], ix, iz) += 0.5f * w * a;
            if (g->variant == TTI_TENSOR) {
              AT(c->fld[TTI_F_TXX], ix, iz) += 0.5f * w * a;
              AT(c->fld[TTI_F_TZZ], ix, iz) += 0.5f * w * a;
            }
            break;
          case 2:
            AT(vx, ix, iz) += 2.0f * alpha * rx * w * a;
            AT(vz, ix, iz) += 2.0f * alpha * rz * w * a;
            break;
          case 3:
            AT(vx, ix, iz) -= 2.0f * alpha * rz * w * a;
            AT(vz, ix, iz) += 2.0f * alpha * rx * w * a;
            break;
          case 5:
            AT(vx, ix, iz) += w * a;
            break;
          case 6:
            AT(vz, ix, iz) += w * a;
            break;
          case 7:
            AT(vx, ix, iz) += 0.5f * sqrtf(2.0f) * w * a;
            AT(vz, ix, iz) += 0.5f * sqrtf(2.0f) * w * a;
            break;
          }
        }
      }
    }
  }
}

/* isoelastic.c:103-144 */
static void record(orc_ctx *c, int it)
{
  const tti_config *g = &c->cfg;
  const int Nz = c->Nz, E = c->E;
  if (g->seistype <= 0 || it % g->mt != 0) return;
  int irec = it / g->mt;
  int want_v = g->seistype == 1 || g->seistype == 3, want_p = g->seistype == 2 || g->seistype == 3;
  for (int k = 0; k < 3; ++k) {
    if ((k < 2 && !want_v) || (k == 2 && !want_p)) continue;
    for (int t = 0; t < c->nrec[k]; ++t) {
      int x = c->rx[k][t] + E, z = c->rz[k][t] + E;
      float val;
      if (k == TTI_REC_VX) val = AT(c->fld[TTI_F_VX], x, z);
      else if (k == TTI_REC_VZ) val = AT(c->fld[TTI_F_VZ], x, z);
      else val = 0.5f * (AT(c->fld[TTI_F_SXX], x, z) + AT(c->fld[TTI_F_SZZ], x, z));
      c->rec[k][(size_t)t * c->nts + irec] = val;
    }
  }
}

/* coord:898-924 (isotropic energy diagnostic over the physical area) */
static void energy(orc_ctx *c, int it)
{
  const tti_config *g = &c->cfg;
  const int Nz = c->Nz, E = c->E;
  float **P = c->par, **F = c->fld;
  double ek = 0.0, ep = 0.0;
  for (int ix = 0; ix < g->nx; ++ix)
    for (int iz = 0; iz < g->nz; ++iz) {
      size_t i = (size_t)(ix + E) * Nz + (iz + E);
      float r = P[TTI_P_INVRHO][i], c11 = P[TTI_P_C11][i], c55 = P[TTI_P_C55][i];
      float sx = F[TTI_F_SXX][i], sz = F[TTI_F_SZZ][i], sq = F[TTI_F_SXZ][i];
      ek += powf(F[TTI_F_VX][i], 2.0f) / r + powf(F[TTI_F_VZ][i], 2.0f) / r;
      ep += 0.25f * (((c11 + 2.0f * c55) * sx - c11 * sz) * sx + (c11 * sx - (c11 + 2.0f * c55) * sz) * sz) /
                (c55 * (c11 + c55)) +
            sq * sq / c55;
    }
  c->ek[it] = 0.5f * (float)ek * g->dx * g->dz;
  c->ep[it] = 0.5f * (float)ep * g->dx * g->dz;
}

int orc_step(orc_ctx *c, int nsteps)
{
  if (!c->have_model) return fail(c, TTI_ERR_STATE, "model not uploaded");
  for (int n = 0; n < nsteps; ++n) {
    if (c->step_index >= c->cfg.nt) return fail(c, TTI_ERR_STATE, "time loop already finished");
    int it = orc_current_it(c);
    velocity_update(c);
    apply_sources(c, it, 0);
    stress_update(c);
    if (c->cfg.freesurface == 1) free_surface(c);
    apply_sources(c, it, 1);
    record(c, it);
    if (c->cfg.energy == 1) energy(c, it);
    c->step_index++;
  }
  return TTI_OK;
}

int orc_fetch_traces(orc_ctx *c, int kind, float *out)
{
  if (kind < 0 || kind > 2 || !c->rec[kind]) return fail(c, TTI_ERR_ARG, "no receivers of kind %d", kind);
  memcpy(out, c->rec[kind], sizeof(float) * (size_t)c->nrec[kind] * c->nts);
  return TTI_OK;
}

int orc_fetch_field(orc_ctx *c, int which, float *out)
{
  if (which < 0 || which >= 8) return fail(c, TTI_ERR_ARG, "bad field %d", which);
  memcpy(out, c->fld[which], c->Np * sizeof(float));
  return TTI_OK;
}

int orc_fetch_energy(orc_ctx *c, float *ek, float *ep)
{
  memcpy(ek, c->ek, sizeof(float) * c->cfg.nt);
  memcpy(ep, c->ep, sizeof(float) * c->cfg.nt);
  return TTI_OK;
}

/* isoelastic.c:240-289 / snapshot.c:28-39: kind 1/4/6 = vx, 2/5/7 = vz,
 * 3 = p = (sxx + szz)/2; savew = 0 keeps the physical nz x nx area */
int orc_snapshot(orc_ctx *c, int kind, float *out)
{
  const int Nz = c->Nz, Nx = c->Nx, E = c->E, sw = c->cfg.savew;
  int x0 = sw == 0 ? E : 0, x1 = sw == 0 ? Nx - E : Nx;
  int z0 = sw == 0 ? E : 0, z1 = sw == 0 ? Nz - E : Nz;
  size_t o = 0;
  for (int ix = x0; ix < x1; ++ix)
    for (int iz = z0; iz < z1; ++iz) {
      float v;
      if (kind == 3) v = 0.5f * (AT(c->fld[TTI_F_SXX], ix, iz) + AT(c->fld[TTI_F_SZZ], ix, iz));
      else if (kind == 1 || kind == 4 || kind == 6) v = AT(c->fld[TTI_F_VX], ix, iz);
      else v = AT(c->fld[TTI_F_VZ], ix, iz);
      out[o++] = v;
    }
  return TTI_OK;
}
