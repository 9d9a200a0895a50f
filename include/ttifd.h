/*
 * ttifd.h -- C ABI of the B200 time-stepping library for 2D TTI elastic
 * modelling on a rotated staggered grid (RSG).
 *
 * Each entry point replaces a region of the reference drivers'
 * main() (wavetomo/TTI-FDModeling):
 *   src/main/sufdmod2dTTIelastic/sufdmod2dTTIelastic_coordinate_rotation.c
 *   src/main/sufdmod2dTTIelastic/sufdmod2dTTIelastic_tensor_rotation.c
 *   src/main/sufdmod2dTTIelastic/sufdmod2dTTIelastic_bond_transformation.c
 * (cited below as coord:, tensor:, bond: with line numbers). The caller keeps
 * getpar, the model file reads, padModel2d, read2dsource / read2dreceiver and
 * traces2d_output; everything from the stability check to the end of the time
 * loop runs on the GPU behind these calls.
 *
 * Conventions
 *  - Plain C types only. Every function returns an int status (TTI_OK = 0);
 *    tti_last_error() gives the message. Callers that want the reference's
 *    behaviour print it with err() and exit(1).
 *  - Grids: Nz = nz + 2E, Nx = nx + 2E with E = ealThick + 5 (the reference
 *    adds N = 5 to ealThick, coord:309-312). Host arrays are [Nx][Nz] FP32,
 *    z fastest (the layout of CWP alloc2float(Nz, Nx); pass arr[0]).
 *  - One handle = one shot on one device, one CUDA stream, one host thread.
 *  - Host buffers are owned by the caller and copied; device memory is owned
 *    by the handle.
 */
#ifndef TTIFD_H
#define TTIFD_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define TTI_OK 0
#define TTI_ERR_ARG 1       /* invalid argument or configuration            */
#define TTI_ERR_UNSTABLE 2  /* dt above the RSG stability limit (stable.c:217-246) */
#define TTI_ERR_RANGE 3     /* source / receiver position out of the model (obsinfo.c:69-80, 206-218) */
#define TTI_ERR_CUDA 4      /* CUDA runtime error                           */
#define TTI_ERR_NOMEM 5     /* device allocation failed                     */
#define TTI_ERR_NONFINITE 6 /* NaN/Inf watchdog tripped in the wavefield    */
#define TTI_ERR_STATE 7     /* call out of order (e.g. run before upload)   */
#define TTI_ERR_CALLBACK 8  /* a host callback returned nonzero             */

/* ---- formulations (the three reference drivers) ---- */
#define TTI_COORDINATE 0 /* coordinate rotation, coord:611-926 */
#define TTI_TENSOR 1     /* tensor rotation,     tensor:614-935 */
#define TTI_BOND 2       /* Bond transformation, bond:651-954 */

/* ---- receiver components (elastic2dReceiver, isoelastic.c:103-144) ---- */
#define TTI_REC_VX 0
#define TTI_REC_VZ 1
#define TTI_REC_P 2

/* ---- wavefield ids for tti_fetch_field ---- */
#define TTI_F_VX 0
#define TTI_F_VZ 1
#define TTI_F_SXX 2
#define TTI_F_SZZ 3
#define TTI_F_SXZ 4
#define TTI_F_TXX 5 /* tensor formulation only */
#define TTI_F_TZZ 6
#define TTI_F_TXZ 7

/* ---- precomputed per-cell arrays for tti_fetch_param (the setup dumps
 *      D_/Beta_/coef1_/coef2_/invrho_/c*_%05d_%05d.bin, coord:480-557) ---- */
#define TTI_P_D 0
#define TTI_P_BETA 1
#define TTI_P_COEF1 2
#define TTI_P_COEF2 3
#define TTI_P_INVRHO 4
#define TTI_P_C11 5
#define TTI_P_C13 6
#define TTI_P_C15 7 /* Bond only */
#define TTI_P_C33 8
#define TTI_P_C35 9 /* Bond only */
#define TTI_P_C55 10
#define TTI_P_SIN 11   /* coordinate: sin(theta) at stress nodes */
#define TTI_P_COS 12   /* coordinate: cos(theta) at stress nodes */
#define TTI_P_SIN_V 13 /* coordinate: sin(theta) averaged to velocity nodes */
#define TTI_P_COS_V 14 /* coordinate: cos(theta) averaged to velocity nodes */
#define TTI_P_SIN2 15  /* tensor: sin^2(theta) */
#define TTI_P_COS2 16  /* tensor: cos^2(theta) */
#define TTI_P_SIN_2T 17 /* tensor: sin(2 theta) */
#define TTI_P_VP 18    /* vp after the MEAL rescale vp/Beta (meal.c:454-460) */
#define TTI_P_VS 19    /* vs after vs/Beta */
#define TTI_P_RHO 20   /* rho after rho*Beta */
#define TTI_P_COUNT 21

/* Run configuration: the getpar keys of the reference drivers (coord:134-294). */
typedef struct tti_config {
  int variant;      /* TTI_COORDINATE / TTI_TENSOR / TTI_BOND */
  int nz, nx, nt;   /* physical grid and time samples */
  float dx, dz, dt; /* sampling (m, m, s) */
  int ealThick;     /* absorbing layers as given on the command line (default 30) */
  float eal_alpha;  /* MEAL weight exponent, -1 = default 2.5 (meal.c:74-77) */
  int freesurface;  /* 1 = stress-image free surface at z = E */
  float fpeak;      /* peak frequency used by MEAL's Beta */
  float scalar;     /* factor applied to theta (degrees) */
  int stype;        /* source type 1..8 */
  int seistype;     /* 0 none, 1 vx+vz, 2 p, 3 all */
  int mt;           /* receiver decimation in time */
  int wsave;        /* snapshot kind 0..5 */
  int savew;        /* 0: physical area only, 1: whole padded grid */
  int snap_sample;  /* snapshot every snap_sample steps (it % snap_sample == 0) */
  int mode;         /* 1: it = 0..nt-1, 2: it = nt-1..0 (coord:611) */
  int energy;       /* 1: record Ek/Ep per step (coord:898-924) */
} tti_config;

typedef struct tti_handle tti_handle;

/* Snapshot sink: called on the host thread at every it % snap_sample == 0.
 * `kind` is 1 (vx), 2 (vz), 3 (p), 4 (vxp), 5 (vzp), 6 (vxs), 7 (vzs),
 * matching the file names of elastic2dSnapshot (isoelastic.c:240-289).
 * `data` is nx_out records of nz_out floats (the raw-binary file body).
 * Return 0 to continue, nonzero to abort the run with TTI_ERR_CALLBACK. */
typedef int (*tti_snapshot_fn)(void *user, int it, int kind, const float *data, int nz_out, int nx_out);

/* Creates a handle on CUDA device `device`; validates cfg. Replaces the
 * allocation block coord:295-344 (device side). */
int tti_create(tti_handle **out, const tti_config *cfg, int device);
int tti_destroy(tti_handle *h);
/* Last error message of h (or of the last failed tti_create when h is NULL). */
const char *tti_last_error(const tti_handle *h);
/* Padded grid sizes and E = ealThick + 5. */
int tti_grid(const tti_handle *h, int *Nz, int *Nx, int *E);

/* Uploads the padded model ([Nx][Nz], after padModel2d) and precomputes on the
 * device: stability check (coord:476, stable.c:217-246), MEAL D/Beta
 * (coord:478, meal.c:51-201), MEAL FD coefficients with the vp/vs/rho rescale
 * (coord:479, meal.c:450-502) and the stiffness build of the selected
 * formulation (coord:497-537, tensor:498-535, bond:492-568 incl. the
 * free-surface stiffness rewrite). vs/rho must be given (defaults are the
 * caller's, coord:362-415). */
int tti_upload_model(tti_handle *h, const float *vp, const float *vs, const float *rho, const float *epsilon,
                     const float *delta, const float *theta);
/* The same from the physical model ([nx][nz], as the model files hold it,
 * before padModel2d): the arrays cross the host link unpadded and the rims
 * are filled on the device as padModel2d (padmod.c:33-59) fills them on the
 * host, every rim cell taking the value of the nearest physical cell, so the
 * result is tti_upload_model's on the padded arrays, bit for bit. On a
 * 1126 x 7872 model it moves 12 % fewer bytes. */
int tti_upload_model_physical(tti_handle *h, const float *vp, const float *vs, const float *rho,
                              const float *epsilon, const float *delta, const float *theta);
/* Copies one precomputed array ([Nx][Nz]) to host memory (setup dumps). */
int tti_fetch_param(tti_handle *h, int which, float *out);

/* Source geometry and wavelets, as read2dsource returns them
 * (obsinfo.c:34-87): positions in cells of the physical grid,
 * src is [ntrace][nt]. Replaces the Source2D argument of the loop. */
int tti_set_source(tti_handle *h, int ntrace, const int *posx, const int *posz, const float *src);
/* Receiver line for one component (read2dreceiver, obsinfo.c:175-230). */
int tti_set_receivers(tti_handle *h, int kind, int ntrace, const int *posx, const int *posz);

/* Runs the whole time loop (coord:611-926): zero wavefields, nt steps,
 * snapshots through `snap` (may be NULL), receivers, energy. */
int tti_run(tti_handle *h, tti_snapshot_fn snap, void *user);
/* Page-locked host memory for the caller's arrays (no counterpart in the
 * reference, which keeps everything in host memory). tti_upload_model from
 * six such arrays, tti_fetch_traces into one and tti_run's snapshots into a
 * buffer given to tti_set_snapshot_buffer move in one copy each at the host
 * link's rate; with pageable arrays the library stages those copies through
 * its own page-locked chunks. Page-locking is slow (about 0.4 ms per MB): take
 * the buffers once and reuse them shot after shot. tti_host_free releases a
 * buffer of tti_host_alloc (TTI_ERR_ARG for any other pointer). */
int tti_host_alloc(size_t bytes, void **ptr);
int tti_host_free(void *ptr);
/* Host buffer of `floats` floats into which tti_run delivers its snapshots
 * (NULL: the library's own buffer), kind q of a snapshot step at q x nz_out x
 * nx_out, so it needs (kinds of wsave) x nz_out x nx_out floats (TTI_ERR_ARG
 * when smaller, TTI_ERR_STATE when wsave writes none). When it is page-locked
 * (tti_host_alloc) the copy of a snapshot to the host runs on a second stream
 * while the time steps go on, and the callbacks of a snapshot step run later:
 * at the next snapshot step or at the end of tti_run, in step order, with
 * `data` pointing into this buffer (valid until the callback returns). A
 * nonzero return still ends the run with TTI_ERR_CALLBACK. With a pageable
 * buffer snapshots are delivered at their step, as without one. The buffer
 * must outlive every tti_run of h that uses it. */
int tti_set_snapshot_buffer(tti_handle *h, float *host, size_t floats);
/* Lower-level stepping: zero the wavefields / advance `nsteps` steps from the
 * current step index without snapshots. tti_run = reset + all steps. */
int tti_reset(tti_handle *h);
int tti_step(tti_handle *h, int nsteps);
/* Device time in ms of the last tti_run / tti_step call (CUDA events). */
int tti_elapsed_ms(const tti_handle *h, float *ms);
/* Measurement aid (no counterpart in the reference, which only prints the
 * loop wall time, coord:927-930): advances `nsteps` steps like tti_step with
 * CUDA events on the handle's stream around each phase and returns the total
 * device ms per phase: ms[0] the velocity update, ms[1] the stress update,
 * ms[2] everything else (sources, free surface, receivers, energy). */
int tti_profile_steps(tti_handle *h, int nsteps, float ms[3]);
/* Number of kernels this handle has launched since tti_create. */
int tti_kernel_launches(const tti_handle *h, long long *n);

/* Snapshot of the current wavefield without allocating device memory (no
 * counterpart in the reference). For callers whose GPU memory must not grow
 * at the point of the call: a host application whose device memory is
 * budgeted by another framework's pool, or code that runs while another
 * stream of the process is being captured into a CUDA graph (a device
 * allocation there is refused and spoils that capture). `kind` as for
 * tti_snapshot_fn; `out` receives nx_out records of nz_out floats.
 * The field is packed in a static device array of 16 Mi floats (64 MiB per
 * GPU); larger snapshots fail with TTI_ERR_ARG. With CUDA's default lazy
 * module loading, the FIRST call on a device loads the library's snapshot
 * module and so commits those 64 MiB (and resolves the array's device
 * address); later calls allocate nothing, and the array is held until the
 * process exits. Make that first call early (before a memory budget is fixed
 * and before any stream capture starts). Calls share the array: calls whose
 * GPU work overlaps race. The call copies to pageable memory and synchronises
 * the handle's stream, so it returns TTI_ERR_STATE when that stream is being
 * captured; captures of other streams (any capture mode, this thread or
 * another) are left intact. */
int tti_snapshot_static(tti_handle *h, int kind, float *out);
/* The CUDA stream (a cudaStream_t) on which all of h's device work is
 * ordered, for callers that order their own work after it (no counterpart in
 * the reference). */
int tti_get_stream(const tti_handle *h, void **stream);

/* Recorded traces of one component, [ntrace][(nt-1)/mt+1] (Receiver2D.recv). */
int tti_fetch_traces(tti_handle *h, int kind, float *out);
/* Current wavefield ([Nx][Nz]). */
int tti_fetch_field(tti_handle *h, int which, float *out);
/* Energy per step (energy = 1): Ek[nt], Ep[nt] (coord:898-924, 942-968). */
int tti_fetch_energy(tti_handle *h, float *ek, float *ep);

/* ---- Adjoint-state gradient ---------------------------------------------------
 * The reference has no adjoint; these entry points add one for all three
 * formulations (for Bond through its free-surface stiffness rewrite,
 * bond:543-568, too) and every source type: the source tables do not depend
 * on the model, so stype only changes the forward replay and the source
 * gradient. Misfit
 *   J = 1/2 sum over the recorded samples of (d - dobs)^2
 * (the components seistype records). tti_grad_run cuts the loop into
 * `ncheck` segments: a forward pass saves the state at each segment start
 * (the checkpoints) and keeps the last segment's states, then the discrete
 * adjoint runs backwards, recomputing each earlier segment from its
 * checkpoint. Memory: ncheck - 1 checkpoints of a full state (5 fields,
 * tensor 8) and ceil(nt / ncheck) kept steps of 8 fields (coordinate), 7
 * (tensor) or 4 (Bond) on the default kernels, 5 on the per-cell kernels;
 * ncheck = 1 keeps every step and recomputes nothing. The shot's gradient is
 * ADDED to the handle's sums (so several
 * shots accumulate; tti_grad_zero clears them). Conventions: vs and rho are
 * held fixed; the MEAL arrays coef1, coef2, Beta stay those of the uploaded
 * model. Gradients are per padded cell, [Nx][Nz], theta in degrees. */
#define TTI_G_VP 0
#define TTI_G_EPS 1
#define TTI_G_DELTA 2
#define TTI_G_THETA 3
/* Observed traces of one recorded component, [ntrace][(nt-1)/mt+1]. */
int tti_grad_set_observed(tti_handle *h, int kind, const float *dobs);
int tti_grad_zero(tti_handle *h);
/* tti_elapsed_ms afterwards gives the device time of the whole run. */
int tti_grad_run(tti_handle *h, int ncheck, double *misfit);
/* The same gradient under binomial checkpointing (Revolve: Griewank and
 * Walther, ACM TOMS 26(1), 2000). The nt steps are cut into macro-steps of
 * `keep_steps` steps; the adjoint of a macro-step runs right after a forward
 * recomputation of it that keeps its steps (keep_steps kept steps in memory),
 * and the states at macro-step starts live in `snapshots` full-state slots
 * placed by the binomial rule, which minimises the macro-steps advanced for
 * that memory. Memory: snapshots full states + keep_steps kept steps. The
 * result is bit-identical to tti_grad_run's. keep_steps = 1 is classic
 * Revolve; snapshots >= nt / keep_steps - 1 recomputes every macro-step once. */
int tti_grad_run_binomial(tti_handle *h, int snapshots, int keep_steps, double *misfit);
/* Macro-steps the binomial schedule advances (recording passes excluded) to
 * reverse `macro_steps` of them with `snapshots` slots; host only, no device. */
long long tti_grad_schedule_cost(int macro_steps, int snapshots);
/* Chooses (snapshots, keep_steps) for tti_grad_run_binomial on h so that the
 * checkpoint slots and kept steps fit in budget_bytes of device memory with
 * the fewest forward steps (*forward_steps, may be NULL: advances plus one
 * recording pass). TTI_ERR_NOMEM when not even one kept step fits. Host only. */
int tti_grad_plan(const tti_handle *h, double budget_bytes, int *snapshots, int *keep_steps,
                  long long *forward_steps);
int tti_grad_fetch(tti_handle *h, int which, float *out);
/* dJ/d(source samples) of the last run, [nsrc][nt]: the stress source
 * (stype 1) reads the adjoint stresses after the residual injection; the
 * velocity sources (stype 2-8, coord:674-802) read the adjoint velocities
 * between the stress-half and velocity-half adjoints, with the window cells
 * outside the velocity update accumulating their own adjoint. */
int tti_grad_fetch_source(tti_handle *h, float *out);
/* Device pointers of the 7 gradient sums (c11, c13, c33, c55, theta at the
 * stress node, sin/cos theta at the velocity node), each `count` floats of
 * [Nx][pitch] layout: a multi-GPU caller all-reduces them in place (the chain
 * rule in tti_grad_fetch is linear in them). */
int tti_grad_accumulators(tti_handle *h, float **dev, size_t *count, size_t *pitch);

/* ---- Batched execution ------------------------------------------------------
 * Many shots (and many models, of different sizes and nt) advanced together:
 * each half-step is one launch over every instance's tiles, and the time loop
 * runs as replays of a CUDA graph of several steps. The reference runs one shot
 * per program invocation (the time loop of coord:611-926); these entry points
 * replace N such invocations. Instances record traces only (wsave = 0,
 * energy = 0); all models use the same formulation.
 *
 * cfg[m] describes model m; model_of[i] (NULL: all 0) names the model of
 * instance i. Instance handles (tti_batch_instance) are ordinary handles owned
 * by the batch: tti_set_source, tti_set_receivers and tti_fetch_traces work on
 * them as on a single shot. The instances of a model share its parameter
 * arrays, uploaded once with tti_batch_upload_model. */
typedef struct tti_batch tti_batch;
int tti_batch_create(tti_batch **b, int nmodels, const tti_config *cfg, int ninst, const int *model_of,
                     int device);
int tti_batch_destroy(tti_batch *b);
const char *tti_batch_last_error(const tti_batch *b);
tti_handle *tti_batch_instance(tti_batch *b, int i);
int tti_batch_upload_model(tti_batch *b, int m, const float *vp, const float *vs, const float *rho,
                           const float *epsilon, const float *delta, const float *theta);
/* Schedule: the shots of a model run tile by tile in groups of `group`
 * (0: all of them, so each parameter tile is read from HBM once per step;
 * 1: shot after shot), and the loop replays a CUDA graph of `graph_steps`
 * steps (0: no graph). */
int tti_batch_set_order(tti_batch *b, int group, int graph_steps);
/* Grid of the batched half-step launches: 0 = one CTA per (instance, tile)
 * work item, 1 = persistent (one resident wave of CTAs walks the work table).
 * Both give the same bits. */
int tti_batch_set_schedule(tti_batch *b, int persistent);
/* The schedule in use (any output may be NULL). */
int tti_batch_get_schedule(const tti_batch *b, int *group, int *graph_steps, int *persistent);
/* Times every group size in {all, 1, 4, 16} (those below the shot count)
 * with and without a graph of 20 steps, with one CTA per work item and with a
 * persistent grid, each over nsteps steps (at least one graph replay, at most
 * the longest instance's nt) in two rounds, keeps the fastest and resets the
 * batch. Outputs (may be NULL): the choice and its ms per step; the grid
 * chosen is read with tti_batch_get_schedule. */
int tti_batch_autotune(tti_batch *b, int nsteps, int *group, int *graph_steps, float *ms_per_step);
/* Zeroes every instance and rebuilds the launch tables from the current
 * sources and receivers. */
int tti_batch_reset(tti_batch *b);
/* Advances every instance nsteps (an instance past its own nt stays idle). */
int tti_batch_step(tti_batch *b, int nsteps);
/* reset + step(max nt): every instance from it = 0 to its own nt. */
int tti_batch_run(tti_batch *b);
int tti_batch_elapsed_ms(const tti_batch *b, float *ms);
/* Gradients of all instances at once: each instance (with its source,
 * receivers and tti_grad_set_observed traces) runs tti_grad_run_binomial
 * with the given schedule from its own host thread on its own stream, so the
 * shots' kernels overlap on the device, and the instances of a model share
 * its parameter arrays. Afterwards the sums of a model's instances are added
 * into its first instance (tti_grad_fetch there gives the model's gradient
 * over those shots) and the other instances' sums are cleared.
 * tti_batch_elapsed_ms gives the wall time of the whole call. misfits
 * (may be NULL) receives each instance's J. The reference has no gradient;
 * this replaces one adjoint run per shot. */
int tti_batch_grad_run(tti_batch *b, int snapshots, int keep_steps, double *misfits);
int tti_batch_kernel_launches(const tti_batch *b, long long *n);

#ifdef __cplusplus
}
#endif
#endif
