/* CPU restatement of the reference's 2D TTI elastic RSG time loop.
 *
 * TEST INFRASTRUCTURE ONLY -- the checker for the CUDA library, never part
 * of the product. Called from tests/ (ctypes), __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg only. Mirrors include/ttifd.h with an orc_
 * prefix so a parity test runs the same calls on both sides. */
#ifndef TTIFD_ORACLE_H
#define TTIFD_ORACLE_H

#include "../include/ttifd.h"

typedef struct orc_ctx orc_ctx;

orc_ctx *orc_create(const tti_config *cfg);
void orc_destroy(orc_ctx *c);
const char *orc_last_error(const orc_ctx *c);
int orc_grid(const orc_ctx *c, int *Nz, int *Nx, int *E);
int orc_upload_model(orc_ctx *c, const float *vp, const float *vs, const float *rho, const float *eps,
                     const float *delta, const float *theta);
int orc_fetch_param(orc_ctx *c, int which, float *out);
int orc_set_source(orc_ctx *c, int ntrace, const int *posx, const int *posz, const float *src);
int orc_set_receivers(orc_ctx *c, int kind, int ntrace, const int *posx, const int *posz);
int orc_reset(orc_ctx *c);
int orc_step(orc_ctx *c, int nsteps);
int orc_current_it(const orc_ctx *c);
int orc_fetch_traces(orc_ctx *c, int kind, float *out);
int orc_fetch_field(orc_ctx *c, int which, float *out);
int orc_fetch_energy(orc_ctx *c, float *ek, float *ep);
/* Body of the snapshot file of `kind` (1..7) for the current wavefield. */
int orc_snapshot(orc_ctx *c, int kind, float *out);

/* free-standing restatements of library helpers */
void orc_pad_model(float *mod, int Nx, int Nz, int nlayer);
void orc_vp2vs(const float *vp, float *vs, int n);
void orc_vp2rho_gardner(const float *vp, float *rho, int n);
double orc_dt_max(const float *vp, int Nx, int Nz, float dx, float dz);
void orc_ricker(float *src, float A, float fpeak, float delay, float dt, int nt);

#endif
