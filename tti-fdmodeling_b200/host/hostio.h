/* Host-side I/O of the drop-in programs: getpar-style arguments, SU traces,
 * raw FP32 model and snapshot files. Formats and conventions follow the
 * reference (see hostio.c); the implementation is this project's own. */
#ifndef TTIFD_HOSTIO_H
#define TTIFD_HOSTIO_H

#include <stddef.h>
#include <stdio.h>

/* ---- getpar: `key=value` command-line arguments, last occurrence wins ---- */
void hio_initargs(int argc, char **argv);
int hio_getint(const char *key, int *v);
int hio_getfloat(const char *key, float *v);
int hio_getstring(const char *key, char **v);
/* message on stderr and exit(1), as SU's err() (the reference's failure mode) */
void hio_err(const char *fmt, ...);
void hio_warn(const char *fmt, ...);

/* ---- SU traces: 240-byte SEG-Y/SU header + ns native floats ---- */
#define HIO_SU_HDR 240
typedef struct {
  unsigned char h[HIO_SU_HDR];
  int ns;
  float *data; /* ns samples (owned) */
} hio_trace;

/* byte offsets of the header fields the programs use */
enum {
  HIO_TRACL = 0, HIO_TRACR = 4, HIO_FLDR = 8, HIO_CDP = 20, HIO_TRID = 28, HIO_OFFSET = 36, HIO_SDEPTH = 48,
  HIO_GDEL = 52, HIO_SDEL = 56, HIO_SCALEL = 68, HIO_SCALCO = 70, HIO_SX = 72, HIO_GX = 80, HIO_NS = 114,
  HIO_DT = 116, HIO_D1 = 180, HIO_F1 = 184, HIO_NTR = 204
};
int hio_get_i32(const unsigned char *h, int off);
int hio_get_i16(const unsigned char *h, int off);
int hio_get_u16(const unsigned char *h, int off);
float hio_get_f32(const unsigned char *h, int off);
void hio_put_i32(unsigned char *h, int off, int v);
void hio_put_i16(unsigned char *h, int off, int v);
void hio_put_u16(unsigned char *h, int off, int v);
void hio_put_f32(unsigned char *h, int off, float v);

/* reads all traces of an SU file; returns count (exits on a malformed file) */
int hio_read_su(const char *path, hio_trace **out);
void hio_free_traces(hio_trace *t, int n);
void hio_write_trace(FILE *fp, const unsigned char *hdr, const float *data, int ns);

/* src/lib/supro/head.c:37-60 coordinate scalar convention */
int hio_scalar_read(float key, int scalar);
int hio_scalar_write(float key, int scalar);

/* resamples one trace (ns samples at dxin, first at fxin) onto t = it*dt,
 * it < nt; samples on the grid are copied, outside the trace is zero */
void hio_resample(int ns, float dxin, float fxin, const float *in, int nt, float dt, float *out);

/* raw FP32 files */
void hio_read_model(const char *path, float *padded, int nz, int nx, int E, int Nz);
void hio_write_floats(const char *path, const float *a, size_t n);

#endif
