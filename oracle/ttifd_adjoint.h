/*
 * ttifd_adjoint.h -- double-precision CPU reference of the adjoint-state
 * gradient (test infrastructure only; see ttifd_adjoint.c).
 */
#ifndef TTIFD_ADJOINT_H
#define TTIFD_ADJOINT_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct adj_ctx adj_ctx;

adj_ctx *adj_create(int nz, int nx, int nt, double dx, double dz, double dt, int ealThick, int freesurface, int mt,
                    int seistype, double scalar);
void adj_destroy(adj_ctx *c);
void adj_grid(const adj_ctx *c, int *Nz, int *Nx, int *nts);
/* 0: coordinate rotation (default), 1: tensor rotation, 2: Bond transformation
 * (without free surface). Before adj_set_model. */
void adj_set_formulation(adj_ctx *c, int variant);
/* frozen MEAL arrays, padded [Nx][Nz] */
void adj_set_meal(adj_ctx *c, const float *coef1, const float *coef2, const float *beta);
/* padded [Nx][Nz] model (theta in degrees); builds the coordinate-rotation stiffness */
void adj_set_model(adj_ctx *c, const double *vp, const double *vs, const double *rho, const double *eps,
                   const double *delta, const double *theta);
/* source type: 1 stress source (default), 2-8 velocity sources */
void adj_set_stype(adj_ctx *c, int stype);
/* sources of the set stype; positions in physical cells, w is [n][nt] */
void adj_set_source(adj_ctx *c, int n, const int *sx, const int *sz, const double *w);
void adj_set_receivers(adj_ctx *c, int kind, int n, const int *gx, const int *gz);
/* traces [ntrace][nts] per recorded component (NULL entries skipped) */
void adj_forward(adj_ctx *c, double *rec[3]);
/* J = 1/2 sum (d - dobs)^2 and its gradients per padded cell; g_src (may be
 * NULL) receives dJ/d(source samples), [nsrc][nt] */
double adj_gradient(adj_ctx *c, const double *dobs[3], double *g_vp, double *g_eps, double *g_delta,
                    double *g_theta, double *g_src);

#ifdef __cplusplus
}
#endif
#endif
