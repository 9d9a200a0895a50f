// Kernel launch wrappers shared by the C-ABI layer (api.cu).
#pragma once

#include "ttifd_internal.cuh"

namespace ttifd {

// ---------------- setup ----------------
struct SetupIn {
  const float *vp, *vs, *rho, *eps, *delta, *theta;  // padded raw model, [Nx][pitch]
  int pitch;                                         // floats per column (Nz: as uploaded)
};
struct SetupOut {
  float *D, *Beta, *coef1, *coef2, *vp, *vs, *rho, *invrho;
  float *c11, *c13, *c15, *c33, *c35, *c55;
  float *sn, *cs, *snv, *csv, *s2, *c2, *s2t;
};
// Scalars of the MEAL profile computed on the host with the host libm
// (exactly as meal.c evaluates them): w[l] = absorbWeight(alpha, l, E).
struct MealConst {
  const float *w;  // device, [E + 1]
  float logR;      // logf(Rcoef)
  float two_thx, two_thz;   // 2 * E * dx, 2 * E * dz
  float dx_fpeak, dz_fpeak; // dx * fpeak, dz * fpeak
  float sqrt3;              // sqrtf(3)
  float dt;
};
void launch_setup(const Grid &g, const SetupIn &in, const SetupOut &out, const MealConst &mc, int variant,
                  float scalar, int freesurface, cudaStream_t st);
// Expands `na` dense physical [nx][nz] arrays (nz * nx floats apart) into
// dense padded [Nx][Nz] arrays (Nz * Nx floats apart), the E-wide rims filled
// as padModel2d fills them on the host.
void launch_expand_physical(const float *phys, float *pad, int na, int nz, int nx, int E, cudaStream_t st);

// ---------------- per-step ----------------
// Source weight tables over the 11 x 11 window (offset (a, b) at a*11+b,
// a = ix - isx + 5, b = iz - isz + 5), precomputed on the host in the
// reference's float expression order (coord:674-886).
struct SourceTables {
  float k1[121];  // 0.5 w          (stype 1, on sxx/szz)
  float kx[121];  // 2 alpha rx w   (stype 2/3)
  float kz[121];  // 2 alpha rz w
  float k5[121];  // w              (stype 5/6)
  float k7[121];  // 0.5 sqrt2 w    (stype 7)
  float q8;       // 0.125 sqrt2    (stype 8)
};

struct StepArgs {
  Grid g;
  Fields f;
  Params p;
  float invdx, invdz;
  int variant;
  bool exact;
};

void launch_velocity(const StepArgs &a, cudaStream_t st);
void launch_stress(const StepArgs &a, cudaStream_t st);
void launch_free_surface(const StepArgs &a, cudaStream_t st);
// stage 0: velocity sources (stype 2..8), stage 1: stress source (stype 1)
void launch_sources(const StepArgs &a, const SourceSet &s, const SourceTables *tab, int stype, int stage, int it,
                    cudaStream_t st);
void launch_receivers(const StepArgs &a, const ReceiverSet &r, int seistype, int irec, int *flag, cudaStream_t st);
void launch_energy(const StepArgs &a, int nz, int nx, double *out2, cudaStream_t st);
// free surface + stress source (stype 1) + receiver samples, one thread per column
struct PostArgs {
  int freesurface, stype, tensor, it, irec;
  SourceSet src;
  float k1[121];
  const int *colptr[3], *rz[3], *rid[3];  // receivers grouped by column (null: component off)
  float *rec[3];
  int nrec[3];
  int *flag;
};
void launch_post(const StepArgs &a, const PostArgs &p, cudaStream_t st);

// ---------------- batched (many instances per launch) ----------------
// Per-instance arguments in device memory; the time index comes from the
// shared step counter `step` (it = step, or nt - 1 - step for mode 2), and an
// instance whose nt has been reached does nothing.
struct BatchPost {
  Grid g;
  Fields f;
  PostArgs p;  // it / irec unused
  int nt, mode2, mt, rec_on;
};
struct BatchSrc {
  Grid g;
  Fields f;
  SourceSet s;
  const SourceTables *tab;  // device
  int variant, stype, nt, mode2;
};
void launch_post_batch(const BatchPost *d, int n, int maxNx, const int *step, cudaStream_t st);
void launch_sources_batch(const BatchSrc *d, int n, const int *step, cudaStream_t st);
void launch_advance(int *step, cudaStream_t st);
// dst[f][0..n) = src[f][0..n), f < 5 (n a multiple of 4, 16-byte aligned arrays)
// the first nf (<= 5) of the arrays src[] into dst[], n floats each, one launch
void launch_copy5(float *const *src, float *const *dst, int nf, size_t n, cudaStream_t st);
// out[r - r0][t] = in[t][r] for t < nts, r0 <= r < r0 + nr (in has n columns)
void launch_transpose(const float *in, float *out, int nts, int n, int r0, int nr, cudaStream_t st);
// Pack a snapshot (kind 1..7) of the physical (savew = 0) or padded area
// into a dense [nx_out][nz_out] buffer.
void launch_snapshot(const StepArgs &a, int kind, int savew, float *dst, cudaStream_t st);

// C-ABI helpers shared by the entry points in other translation units
StepArgs handle_step_args(const tti_handle *h);
void handle_source_tables(const tti_handle *h, SourceTables *t);
int handle_check_flag(tti_handle *h);
// one time step; `keep` (5 device arrays or null) receives vx vz sxx szz sxz
// between the velocity sources and the stress update
int handle_step(tti_handle *h, const SourceTables &tab, float *const *keep);  // keep: 8 pointers or null
// Fields of one kept step of the gradient (the arrays `keep` of handle_step
// points at). Tiled kernels: the strain rates vxx vxz vzx vzz, then for the
// coordinate rotation the stress derivative combinations P Q R S (8 fields),
// for the tensor rotation txx tzz txz before the stress half (7), for Bond
// nothing more (4). Per-cell kernels: vx vz after the velocity half and the
// stresses (tensor: tau) before the stress half (5).
int keep_fields(const tti_handle *h);
// frees the gradient's device memory of h (adjoint.cu)
void grad_release(tti_handle *h);
int create_handle(tti_handle **out, const tti_config *cfg, int device, const tti_handle *share, bool force_tiled);
int handle_error(tti_handle *h, int code, const char *msg);

}  // namespace ttifd
