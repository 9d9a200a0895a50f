/* Host I/O for the drop-in programs. Conventions kept from the reference:
 *  - getpar keys as `key=value` arguments (SU getpar; the last occurrence
 *    wins, as the demo scripts pass `scalar=-1` twice, demo/test_bp01.sh:46-57);
 *  - err(): message and exit status 1 (every reference error path);
 *  - SU traces (src/lib/fdmod/obsinfo.c, traces.c): 240-byte header in the
 *    SEG-Y rev.0 byte positions plus the SU fields d1/f1/ntr, native byte
 *    order, followed by ns floats;
 *  - model files: nx records of nz floats, read into the interior of the
 *    padded [Nx][Nz] array (coord:356-359).
 */
#include "hostio.h"

#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static int g_argc;
static char **g_argv;

void hio_initargs(int argc, char **argv)
{
  g_argc = argc;
  g_argv = argv;
}

static const char *value_of(const char *key)
{
  size_t n = strlen(key);
  const char *v = NULL;
  for (int i = 1; i < g_argc; ++i)
    if (strncmp(g_argv[i], key, n) == 0 && g_argv[i][n] == '=') v = g_argv[i] + n + 1;
  return v;
}

int hio_getint(const char *key, int *v)
{
  const char *s = value_of(key);
  if (!s) return 0;
  *v = (int)strtol(s, NULL, 10);
  return 1;
}

int hio_getfloat(const char *key, float *v)
{
  const char *s = value_of(key);
  if (!s) return 0;
  *v = (float)strtod(s, NULL);
  return 1;
}

int hio_getstring(const char *key, char **v)
{
  const char *s = value_of(key);
  if (!s) return 0;
  *v = (char *)s;
  return 1;
}

static void vmsg(const char *fmt, va_list ap)
{
  fprintf(stderr, "%s: ", g_argv && g_argv[0] ? g_argv[0] : "ttifd");
  vfprintf(stderr, fmt, ap);
  fprintf(stderr, "\n");
}

void hio_err(const char *fmt, ...)
{
  va_list ap;
  fflush(stdout);
  va_start(ap, fmt);
  vmsg(fmt, ap);
  va_end(ap);
  exit(1);
}

void hio_warn(const char *fmt, ...)
{
  if (getenv("TTIFD_QUIET")) return;
  va_list ap;
  va_start(ap, fmt);
  vmsg(fmt, ap);
  va_end(ap);
}

/* ---------------- header fields ---------------- */
int hio_get_i32(const unsigned char *h, int off)
{
  int32_t v;
  memcpy(&v, h + off, 4);
  return v;
}
int hio_get_i16(const unsigned char *h, int off)
{
  int16_t v;
  memcpy(&v, h + off, 2);
  return v;
}
int hio_get_u16(const unsigned char *h, int off)
{
  uint16_t v;
  memcpy(&v, h + off, 2);
  return v;
}
float hio_get_f32(const unsigned char *h, int off)
{
  float v;
  memcpy(&v, h + off, 4);
  return v;
}
void hio_put_i32(unsigned char *h, int off, int v)
{
  int32_t x = v;
  memcpy(h + off, &x, 4);
}
void hio_put_i16(unsigned char *h, int off, int v)
{
  int16_t x = (int16_t)v;
  memcpy(h + off, &x, 2);
}
void hio_put_u16(unsigned char *h, int off, int v)
{
  uint16_t x = (uint16_t)v;
  memcpy(h + off, &x, 2);
}
void hio_put_f32(unsigned char *h, int off, float v) { memcpy(h + off, &v, 4); }

/* ---------------- SU files ---------------- */
int hio_read_su(const char *path, hio_trace **out)
{
  FILE *fp = fopen(path, "rb");
  if (!fp) return -1;
  int n = 0, cap = 4;
  hio_trace *t = (hio_trace *)malloc(sizeof *t * cap);
  for (;;) {
    unsigned char h[HIO_SU_HDR];
    size_t got = fread(h, 1, HIO_SU_HDR, fp);
    if (got == 0) break;
    if (got != HIO_SU_HDR) hio_err("<error>: truncated SU header in %s", path);
    int ns = hio_get_u16(h, HIO_NS);
    float *d = (float *)malloc(sizeof(float) * (ns ? ns : 1));
    if (fread(d, sizeof(float), ns, fp) != (size_t)ns) hio_err("<error>: truncated SU trace in %s", path);
    if (n == cap) t = (hio_trace *)realloc(t, sizeof *t * (cap *= 2));
    memcpy(t[n].h, h, HIO_SU_HDR);
    t[n].ns = ns;
    t[n].data = d;
    ++n;
  }
  fclose(fp);
  *out = t;
  return n;
}

void hio_free_traces(hio_trace *t, int n)
{
  for (int i = 0; i < n; ++i) free(t[i].data);
  free(t);
}

void hio_write_trace(FILE *fp, const unsigned char *hdr, const float *data, int ns)
{
  if (fwrite(hdr, 1, HIO_SU_HDR, fp) != HIO_SU_HDR || fwrite(data, sizeof(float), ns, fp) != (size_t)ns)
    hio_err("<error>: failed to write SU trace");
}

/* head.c:37-51: value = key * 10^(sign(scalar) * log10|scalar|), truncated */
int hio_scalar_read(float key, int scalar)
{
  if (scalar == 0) hio_err("<error> : scalar must not be %d!", scalar);
  int e = (int)((scalar < 0 ? -1.0 : 1.0) * log10((double)abs(scalar)));
  return (int)(key * pow(10.0, e));
}

int hio_scalar_write(float key, int scalar) { return hio_scalar_read(key, -scalar); }

/* The reference resamples the source trace with SU's ints8r onto
 * t = it*dt (obsinfo.c:82). When the trace is sampled on the modelling grid
 * (the case sumksrc2d produces) that returns the samples themselves; outside
 * the trace it returns 0. Off-grid traces use an 8-point Hann-windowed sinc. */
void hio_resample(int ns, float dxin, float fxin, const float *in, int nt, float dt, float *out)
{
  int warned = 0;
  for (int it = 0; it < nt; ++it) {
    float t = it * dt;
    double p = ((double)t - (double)fxin) / (double)dxin;
    double r = floor(p + 0.5);
    if (fabs(p - r) <= 1.0e-4) {
      long i = (long)r;
      out[it] = (i >= 0 && i < ns) ? in[i] : 0.0f;
      continue;
    }
    if (!warned) {
      warned = 1;
      hio_warn("<warning>: source trace is not sampled on the modelling time grid; resampling with a windowed sinc");
    }
    long i0 = (long)floor(p);
    double frac = p - i0, acc = 0.0;
    for (int k = -3; k <= 4; ++k) {
      double x = k - frac;
      double s = fabs(x) < 1e-12 ? 1.0 : sin(M_PI * x) / (M_PI * x);
      double w = 0.5 * (1.0 + cos(M_PI * x / 4.5));
      long i = i0 + k;
      acc += s * w * ((i >= 0 && i < ns) ? in[i] : 0.0);
    }
    out[it] = (float)acc;
  }
}

void hio_read_model(const char *path, float *padded, int nz, int nx, int E, int Nz)
{
  FILE *fp = fopen(path, "rb");
  if (!fp) hio_err("<error>: fail to open file: %s!", path);
  for (int ix = 0; ix < nx; ++ix) {
    size_t got = fread(padded + (size_t)(ix + E) * Nz + E, sizeof(float), nz, fp);
    if (got != (size_t)nz) hio_err("<error>: short read in %s", path);
  }
  fclose(fp);
}

void hio_write_floats(const char *path, const float *a, size_t n)
{
  FILE *fp = fopen(path, "wb");
  if (!fp) hio_err("<error>: cannot open %s for writing", path);
  if (fwrite(a, sizeof(float), n, fp) != n) hio_err("<error>: write error on %s", path);
  fclose(fp);
}
