/*
 * Drop-in replacement of the reference programs
 *   sufdmod2dTTIelastic_coordinate_rotation   (TTI_PROGRAM_VARIANT "coordinate_rotation")
 *   sufdmod2dTTIelastic_tensor_rotation       ("tensor_rotation")
 *   sufdmod2dTTIelastic_bond_transformation   ("bond_transformation")
 * Same getpar keys and defaults (coord:134-294), same input files, same output
 * files and names (setup dumps coord:480-557, vs_/rho_ defaults :365-398,
 * snapshots isoelastic.c:240-289, SU traces traces.c:146-196, energy text
 * files :942-968), same timing lines on stdout (:930, :1007) and exit status 1
 * with a message on the same error conditions. The time loop runs on the GPU
 * through the C ABI of include/ttifd.h.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "hostio.h"
#include "ttifd.h"

#ifndef TTI_PROGRAM_VARIANT
#define TTI_PROGRAM_VARIANT "coordinate_rotation"
#endif

static double now_s(void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static int variant_id(void)
{
  if (strcmp(TTI_PROGRAM_VARIANT, "tensor_rotation") == 0) return TTI_TENSOR;
  if (strcmp(TTI_PROGRAM_VARIANT, "bond_transformation") == 0) return TTI_BOND;
  return TTI_COORDINATE;
}

static const char *usage =
    " SUFDMOD2DTTIELASTIC (" TTI_PROGRAM_VARIANT ", B200) nz= nx= nt= dx= dz= dt= fpeak= ...\n"
    " Rotated staggered grid finite-difference modelling of the 2D first-order elastic wave\n"
    " equation in TTI media, time loop on the GPU.\n"
    " Required: dz dx dt nz nx nt fpeak vpfile epsilonfile deltafile thetafile sourcefile\n"
    " Optional: vsfile rhofile scalar(1) stype(1) recposfile seistype(0) mt(1) ealThick(30)\n"
    "           eal_alpha(2.5) freesurface(0) mode(1) energy(0) savew(0) wsave(1)\n"
    "           snap_sample(500/(dt*1000)) fx(0) fz(0) shotID(1) snap_prefix(snap)\n"
    "           trace_prefix(traces) device(0)\n";

typedef struct {
  const char *prefix;
  int nz, nx;
  float dt;
} snap_ctx;

static const char *snap_name(int kind)
{
  static const char *n[] = {"", "vx", "vz", "p", "vxp", "vzp", "vxs", "vzs"};
  return kind >= 1 && kind <= 7 ? n[kind] : "x";
}

/* elastic2dSnapshot file naming: %s_<kind>_%05d_%05d_%05dms.bin with the time
 * (int)(1000 * it * dt) evaluated in float (isoelastic.c:252-285) */
static int write_snapshot(void *user, int it, int kind, const float *data, int nz_out, int nx_out)
{
  const snap_ctx *s = (const snap_ctx *)user;
  char fn[512];
  snprintf(fn, sizeof fn, "%s_%s_%05d_%05d_%05dms.bin", s->prefix, snap_name(kind), nz_out, nx_out,
           (int)(1000 * it * s->dt));
  hio_write_floats(fn, data, (size_t)nz_out * nx_out);
  return 0;
}

/* traces2d_output / putraces_2d (traces.c:36-72, 146-196) */
static void write_traces(const char *prefix, const char *comp, int shotID, int nts, int ntr, float dt_rec, float fx,
                         float fz, float dx, float dz, int sx, int sz, const int *gx, const int *gz, const float *rec)
{
  char fn[512];
  snprintf(fn, sizeof fn, "%s_%s_%04d_%05d_%05d_%05.2fms.su", prefix, comp, shotID, nts, ntr, dt_rec * 1000.0f);
  FILE *fp = fopen(fn, "wb");
  if (!fp) hio_err("efopen: cannot open %s", fn);
  unsigned char h[HIO_SU_HDR];
  memset(h, 0, sizeof h);
  hio_put_i32(h, HIO_TRACL, 1);
  hio_put_u16(h, HIO_NS, nts);
  hio_put_u16(h, HIO_DT, (unsigned short)(dt_rec * 1000000));
  hio_put_i32(h, HIO_NTR, ntr);
  hio_put_i16(h, HIO_SCALEL, -1000);
  hio_put_i16(h, HIO_SCALCO, -1000);
  hio_put_f32(h, HIO_F1, 0.0f);
  hio_put_f32(h, HIO_D1, dt_rec);
  hio_put_i32(h, HIO_FLDR, shotID);
  const int hsx = hio_scalar_write(fx + sx * dx, -1000);
  hio_put_i32(h, HIO_SX, hsx);
  hio_put_i32(h, HIO_SDEL, hio_scalar_write(fz + sz * dz, -1000));
  for (int t = 0; t < ntr; ++t) {
    hio_put_i32(h, HIO_TRACR, t + 1);
    hio_put_i16(h, HIO_TRID, gx[t]);
    const int hgx = hio_scalar_write(fx + gx[t] * dx, -1000);
    hio_put_i32(h, HIO_GX, hgx);
    hio_put_i32(h, HIO_GDEL, hio_scalar_write(fz + gz[t] * dz, -1000));
    hio_put_i32(h, HIO_OFFSET, hgx - hsx);
    hio_put_i32(h, HIO_CDP, (int)(0.5f * (hgx + hsx)));
    hio_write_trace(fp, h, rec + (size_t)t * nts, nts);
  }
  fclose(fp);
}

static void check(tti_handle *h, int rc)
{
  if (rc != TTI_OK) hio_err("<error>: %s", tti_last_error(h));
}

static void dump_param(tti_handle *h, int id, const char *name, float *buf, int Nz, int Nx)
{
  char fn[256];
  check(h, tti_fetch_param(h, id, buf));
  snprintf(fn, sizeof fn, "%s_%05d_%05d.bin", name, Nz, Nx);
  hio_write_floats(fn, buf, (size_t)Nz * Nx);
}

/* read2dreceiver (obsinfo.c:175-230): trace 1 gx, trace 2 gz, in cells */
static int read_receivers(const char *path, int nx, int nz, int **gx, int **gz)
{
  hio_trace *t;
  int n = hio_read_su(path, &t);
  if (n < 0) hio_err("<error>: failed to open recposfile (%s)!", path);
  if (n < 2) hio_err("<error>: failed to get traces in recposfile (%s)!", path);
  if (t[0].ns != t[1].ns)
    hio_err("<error>: the number of Group coordinate's samples are not match, Group X coordinate : %d, Group Z "
            "coordinate : %d.",
            t[0].ns, t[1].ns);
  int ntr = t[0].ns;
  *gx = (int *)malloc(sizeof(int) * (ntr ? ntr : 1));
  *gz = (int *)malloc(sizeof(int) * (ntr ? ntr : 1));
  for (int i = 0; i < ntr; ++i) {
    (*gz)[i] = (int)t[1].data[i];
    if ((*gz)[i] < 0 || (*gz)[i] > nz)
      hio_err("<error>: the position of receiver in 1st dimension (%d) must be between 0 and %d!", (*gz)[i], nz);
    (*gx)[i] = (int)t[0].data[i];
    if ((*gx)[i] < 0 || (*gx)[i] > nx)
      hio_err("<error>: the position of receiver in 2nd dimension (%d) must be between 0 and %d!", (*gx)[i], nx);
  }
  hio_warn("the number of traces is %d!", ntr);
  hio_free_traces(t, n);
  return ntr;
}

int main(int argc, char **argv)
{
  hio_initargs(argc, argv);
  if (argc == 1) {
    fputs(usage, stderr);
    return 1;
  }
  const double t_total0 = now_s();
  int nz, nx, nt, freesurface, ealThick, mode, savew, wsave, stype, seistype, mt, snap_sample, shotID, energy, device;
  float dx, dz, dt, fx, fz, scalar, fpeak, eal_alpha;
  char *vpfile = NULL, *vsfile = NULL, *rhofile = NULL, *thetafile = NULL, *epsilonfile = NULL, *deltafile = NULL;
  char *sourcefile = NULL, *recposfile = NULL, *trace_prefix = "traces", *snap_prefix = "snap";

  if (!hio_getfloat("dx", &dx)) hio_err("<error>: must specify sampling interval in 1st dimension!");
  if (!hio_getfloat("dz", &dz)) hio_err("<error>: must specify sampling interval in 2nd dimension!");
  if (!hio_getfloat("dt", &dt)) hio_err("<error>: must specify sampling interval in time dimension!");
  if (!hio_getfloat("fx", &fx)) fx = 0.0f;
  if (!hio_getfloat("fz", &fz)) fz = 0.0f;
  if (!hio_getfloat("scalar", &scalar)) scalar = 1.0f;
  if (!hio_getfloat("fpeak", &fpeak)) hio_err("<error>: must specify peak frequency of source wavelet!");
  if (!hio_getfloat("eal_alpha", &eal_alpha)) eal_alpha = -1.0f;
  if (!hio_getint("nz", &nz)) hio_err("<error>: must specify the number of samples in 1st dimension!");
  if (!hio_getint("nx", &nx)) hio_err("<error>: must specify the number of samples in 2nd dimension!!");
  if (!hio_getint("nt", &nt)) hio_err("<error>: must specify the number of samples in time dimension!!");
  if (!hio_getint("freesurface", &freesurface)) freesurface = 0;
  if (!hio_getint("ealThick", &ealThick)) ealThick = 30;
  if (!hio_getint("mode", &mode)) mode = 1;
  if (!hio_getint("savew", &savew)) savew = 0;
  if (!hio_getint("wsave", &wsave)) wsave = 1;
  if (!hio_getint("stype", &stype)) stype = 1;
  if (!hio_getint("seistype", &seistype)) seistype = 0; /* coord:220-225 (the doc says 1) */
  if (!hio_getint("mt", &mt)) mt = 1;
  if (!hio_getint("snap_sample", &snap_sample)) snap_sample = 500 / (dt * 1000);
  if (!hio_getint("shotID", &shotID)) shotID = 1;
  if (!hio_getint("energy", &energy)) energy = 0;
  if (!hio_getint("device", &device)) device = 0;
  if (!hio_getstring("vpfile", &vpfile)) hio_err("<error>: must specify P-wave velocity!");
  if (!hio_getstring("vsfile", &vsfile))
    hio_warn("<warning>: didn't specify S-wave velocity! The program will set S-wave velocity as vp / sqrt(3)!");
  if (!hio_getstring("rhofile", &rhofile))
    hio_warn("<warning>: didn't specify density file! The program will set density as 310 * pow(vp, 0.25)!");
  if (!hio_getstring("epsilonfile", &epsilonfile)) hio_err("<error>: must specify Thomsen parameter (epsilon) file!");
  if (!hio_getstring("deltafile", &deltafile)) hio_err("<error>: must specify Thomsen parameter (delta) file!");
  if (!hio_getstring("thetafile", &thetafile)) hio_err("<error>: must specify dip angle (theta) file!");
  if (!hio_getstring("sourcefile", &sourcefile)) hio_err("<error>: must specify sourcefile!");
  if (!hio_getstring("recposfile", &recposfile)) hio_warn("<warning>: didn't specify receiver_p position file!");
  hio_getstring("snap_prefix", &snap_prefix);
  hio_getstring("trace_prefix", &trace_prefix);

  tti_config cfg = {variant_id(), nz, nx, nt, dx, dz, dt, ealThick, eal_alpha, freesurface, fpeak, scalar,
                    stype, seistype, mt, wsave, savew, snap_sample, mode, energy};
  tti_handle *h = NULL;
  if (tti_create(&h, &cfg, device) != TTI_OK) hio_err("<error>: %s", tti_last_error(NULL));
  int Nz, Nx, E;
  tti_grid(h, &Nz, &Nx, &E);
  const size_t Np = (size_t)Nz * Nx;

  /* ---- model (coord:345-461) ---- */
  float *m[6];
  for (int k = 0; k < 6; ++k) m[k] = (float *)calloc(Np, sizeof(float));
  float *vp = m[0], *vs = m[1], *rho = m[2], *eps = m[3], *dlt = m[4], *th = m[5];
  char fn[512];
  hio_read_model(vpfile, vp, nz, nx, E, Nz);
  if (vsfile == NULL) { /* vp2vs, modparconvert.c:42-58, on the whole array before padding */
    for (size_t i = 0; i < Np; ++i) vs[i] = vp[i] <= 1500.0 ? 0.0f : (float)(0.577350269189626 * vp[i]);
    snprintf(fn, sizeof fn, "vs_%05d_%05d.bin", nz, nx);
    FILE *fp = fopen(fn, "wb");
    for (int ix = 0; ix < nx && fp; ++ix) fwrite(vs + (size_t)(ix + E) * Nz + E, sizeof(float), nz, fp);
    if (fp) fclose(fp);
  } else {
    hio_read_model(vsfile, vs, nz, nx, E, Nz);
  }
  if (rhofile == NULL) { /* Gardner, modparconvert.c:128-141 */
    for (size_t i = 0; i < Np; ++i) rho[i] = vp[i] <= 1500.0 ? 1000.0f : (float)(1741.0 * pow(vp[i] / 1000.0, 0.25));
    snprintf(fn, sizeof fn, "rho_%05d_%05d.bin", nz, nx);
    FILE *fp = fopen(fn, "wb");
    for (int ix = 0; ix < nx && fp; ++ix) fwrite(rho + (size_t)(ix + E) * Nz + E, sizeof(float), nz, fp);
    if (fp) fclose(fp);
  } else {
    hio_read_model(rhofile, rho, nz, nx, E, Nz);
  }
  hio_read_model(epsilonfile, eps, nz, nx, E, Nz);
  hio_read_model(deltafile, dlt, nz, nx, E, Nz);
  hio_read_model(thetafile, th, nz, nx, E, Nz);
  /* padModel2d (padmod.c:33-59): rims of the interior columns, then full columns */
  for (int k = 0; k < 6; ++k) {
    float *a = m[k];
    for (int ix = E; ix < Nx - E; ++ix)
      for (int l = 1; l <= E; ++l) {
        a[(size_t)ix * Nz + E - l] = a[(size_t)ix * Nz + E];
        a[(size_t)ix * Nz + Nz - E - 1 + l] = a[(size_t)ix * Nz + Nz - E - 1];
      }
    for (int l = 1; l <= E; ++l) {
      memcpy(a + (size_t)(E - l) * Nz, a + (size_t)E * Nz, sizeof(float) * Nz);
      memcpy(a + (size_t)(Nx - E - 1 + l) * Nz, a + (size_t)(Nx - E - 1) * Nz, sizeof(float) * Nz);
    }
  }

  /* ---- stability, MEAL, stiffness on the device (coord:476-537) ---- */
  check(h, tti_upload_model(h, vp, vs, rho, eps, dlt, th));
  float *buf = m[0]; /* reuse the host vp buffer for the dumps */
  dump_param(h, TTI_P_D, "D", buf, Nz, Nx);
  dump_param(h, TTI_P_BETA, "Beta", buf, Nz, Nx);
  dump_param(h, TTI_P_COEF1, "coef1", buf, Nz, Nx);
  dump_param(h, TTI_P_COEF2, "coef2", buf, Nz, Nx);
  dump_param(h, TTI_P_INVRHO, "invrho", buf, Nz, Nx);
  dump_param(h, TTI_P_C11, "c11", buf, Nz, Nx);
  dump_param(h, TTI_P_C13, "c13", buf, Nz, Nx);
  if (cfg.variant == TTI_BOND) dump_param(h, TTI_P_C15, "c15", buf, Nz, Nx);
  dump_param(h, TTI_P_C33, "c33", buf, Nz, Nx);
  if (cfg.variant == TTI_BOND) dump_param(h, TTI_P_C35, "c35", buf, Nz, Nx);
  dump_param(h, TTI_P_C55, "c55", buf, Nz, Nx);
  for (int k = 0; k < 6; ++k) free(m[k]);

  /* ---- source (read2dsource, obsinfo.c:34-87) ---- */
  hio_trace *st;
  int nst = hio_read_su(sourcefile, &st);
  if (nst < 0) hio_err("efopen: cannot open %s", sourcefile);
  if (nst == 0) hio_err("<error>: no trace in sourcefile (%s)!", sourcefile);
  const int nsrc = hio_get_i32(st[0].h, HIO_NTR);
  hio_warn("<warning>: the number of trace is %d in sourcefile (%s)!", nsrc, sourcefile);
  if (nst > nsrc) hio_err("<error>: the number of traces in sourcefile (%s) is out of %d!", sourcefile, nsrc);
  int *sx = (int *)calloc(nsrc > 0 ? nsrc : 1, sizeof(int)), *sz = (int *)calloc(nsrc > 0 ? nsrc : 1, sizeof(int));
  float *src = (float *)calloc((size_t)(nsrc > 0 ? nsrc : 1) * nt, sizeof(float));
  for (int i = 0; i < nst; ++i) {
    sz[i] = hio_scalar_read((float)hio_get_i32(st[i].h, HIO_SDEPTH), hio_get_i16(st[i].h, HIO_SCALEL));
    if (sz[i] < 0 || sz[i] > nz)
      hio_err("<error>: the position of source in 1st dimension (%d) must be between 0 and %d!", sz[i], nz);
    sx[i] = hio_scalar_read((float)hio_get_i32(st[i].h, HIO_SX), hio_get_i16(st[i].h, HIO_SCALCO));
    if (sx[i] < 0 || sx[i] > nx)
      hio_err("<error>: the position of source in 2nd dimension (%d) must be between 0 and %d!", sx[i], nx);
    hio_resample(st[i].ns, hio_get_u16(st[i].h, HIO_DT) / 1000000.0f, hio_get_f32(st[i].h, HIO_F1), st[i].data, nt, dt,
                 src + (size_t)i * nt);
  }
  check(h, tti_set_source(h, nsrc, sx, sz, src));

  /* ---- receivers ---- */
  int nrec = 0, *gx = NULL, *gz = NULL;
  if (seistype > 0) {
    if (!recposfile) hio_err("<error>: failed to open recposfile ((null))!");
    nrec = read_receivers(recposfile, nx, nz, &gx, &gz);
    if (seistype == 1 || seistype == 3) {
      check(h, tti_set_receivers(h, TTI_REC_VX, nrec, gx, gz));
      check(h, tti_set_receivers(h, TTI_REC_VZ, nrec, gx, gz));
    }
    if (seistype == 2 || seistype == 3) check(h, tti_set_receivers(h, TTI_REC_P, nrec, gx, gz));
  }

  fprintf(stderr, "%s: Input Parameters:\n", argv[0]);
  fprintf(stderr, "%s: nx = %d, nz = %d, nt = %d\n", argv[0], nx, nz, nt);
  fprintf(stderr, "%s: Nx = %d, Nz = %d\n", argv[0], Nx, Nz);
  fprintf(stderr, "%s: dx = %6.5f, dz = %6.5f, dt = %6.5f\n", argv[0], dx, dz, dt);

  /* ---- time loop on the GPU ---- */
  snap_ctx sc = {snap_prefix, nz, nx, dt};
  const double t0 = now_s();
  int rc = tti_run(h, wsave > 0 ? write_snapshot : NULL, &sc);
  if (rc == TTI_ERR_NONFINITE) hio_warn("<warning>: %s", tti_last_error(h));
  else check(h, rc);
  fprintf(stderr, "\n");
  fprintf(stdout, "Finite difference modeling takes %lf s.\n", now_s() - t0);

  /* ---- traces ---- */
  const int nts = (nt - 1) / mt + 1;
  const float dt_rec = mt * dt;
  if (seistype > 0 && nrec > 0) {
    float *rec = (float *)malloc(sizeof(float) * (size_t)nrec * nts);
    if (seistype == 1 || seistype == 3) {
      check(h, tti_fetch_traces(h, TTI_REC_VX, rec));
      write_traces(trace_prefix, "vx", shotID, nts, nrec, dt_rec, fx, fz, dx, dz, sx[0], sz[0], gx, gz, rec);
      check(h, tti_fetch_traces(h, TTI_REC_VZ, rec));
      write_traces(trace_prefix, "vz", shotID, nts, nrec, dt_rec, fx, fz, dx, dz, sx[0], sz[0], gx, gz, rec);
    }
    if (seistype == 2 || seistype == 3) {
      check(h, tti_fetch_traces(h, TTI_REC_P, rec));
      write_traces(trace_prefix, "p", shotID, nts, nrec, dt_rec, fx, fz, dx, dz, sx[0], sz[0], gx, gz, rec);
    }
    free(rec);
  }
  /* ---- energy (coord:942-968) ---- */
  if (energy == 1) {
    float *ek = (float *)malloc(sizeof(float) * nt), *ep = (float *)malloc(sizeof(float) * nt);
    check(h, tti_fetch_energy(h, ek, ep));
    FILE *f1 = fopen("src.txt", "w"), *f2 = fopen("Eng.txt", "w"), *f3 = fopen("Ek.txt", "w"),
         *f4 = fopen("Ep.txt", "w");
    for (int it = 0; it < nt; ++it) {
      if (f1) fprintf(f1, "%10.5e\n", nsrc > 0 ? src[it] : 0.0f);
      if (f2) fprintf(f2, "%10.5e\n", ek[it] + ep[it]);
      if (f3) fprintf(f3, "%10.5e\n", ek[it]);
      if (f4) fprintf(f4, "%10.5e\n", ep[it]);
    }
    if (f1) fclose(f1);
    if (f2) fclose(f2);
    if (f3) fclose(f3);
    if (f4) fclose(f4);
    free(ek);
    free(ep);
  }
  tti_destroy(h);
  hio_free_traces(st, nst);
  free(sx);
  free(sz);
  free(src);
  free(gx);
  free(gz);
  fprintf(stdout, "Total time takes %lf s.\n", now_s() - t_total0);
  return 0;
}
