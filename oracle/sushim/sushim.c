/* Self-written implementation of the small Seismic Unix / CWP subset that the
 * reference's hot-path C sources call (getpar, err/warn, checked I/O,
 * contiguous allocators, SU trace read/write, ints8r).
 *
 * TEST INFRASTRUCTURE ONLY: linked into the oracle build of the reference
 * (oracle/_ref/). Seismic Unix is not installed here and not vendored by the
 * reference (its Makefiles link -lsu -lpar -lcwp from $CWPROOT), so this
 * follows SU's documented behaviour:
 *   - getpar: command-line `key=value` pairs, the last occurrence wins;
 *   - err(): message on stderr, exit status 1; warn(): message, continue;
 *   - alloc2float(n1, n2): one contiguous block, row pointers p[i2];
 *   - SU traces: 240-byte header (segy.h) followed by ns native floats;
 *   - ints8r: returns the input samples when the output axis lands on input
 *     samples (the only case the modelling programs meet: the source trace is
 *     written at the modelling dt with f1 = 0), yinl/yinr outside the input.
 *     Off-grid resampling uses an 8-point Hann-windowed sinc of this file's
 *     own design; SU's least-squares sinc table is not reproduced, so
 *     off-grid source resampling is "parity unpinned" and warns.
 */
#include <stdarg.h>

#include "cwp.h"
#include "par.h"
#include "su.h"

int xargc = 0;
char **xargv = NULL;

void initargs(int argc, char **argv)
{
  xargc = argc;
  xargv = argv;
}

void requestdoc(int flag)
{
  (void)flag;
  if (xargc <= 1) {
    for (char **p = sdoc; *p != NULL; ++p) fprintf(stderr, "%s\n", *p);
    exit(EXIT_FAILURE);
  }
}

static const char *progname(void) { return (xargv && xargv[0]) ? xargv[0] : "oracle"; }

/* value of the last `name=value` argument, or NULL */
static char *lookup(const char *name)
{
  size_t n = strlen(name);
  char *found = NULL;
  for (int i = 1; i < xargc; ++i) {
    const char *a = xargv[i];
    if (strncmp(a, name, n) == 0 && a[n] == '=') found = (char *)(a + n + 1);
  }
  return found;
}

int getparint(char *name, int *p)
{
  char *v = lookup(name);
  if (!v) return 0;
  *p = (int)strtol(v, NULL, 10);
  return 1;
}

int getparfloat(char *name, float *p)
{
  char *v = lookup(name);
  if (!v) return 0;
  *p = (float)strtod(v, NULL);
  return 1;
}

int getpardouble(char *name, double *p)
{
  char *v = lookup(name);
  if (!v) return 0;
  *p = strtod(v, NULL);
  return 1;
}

int getparstring(char *name, char **p)
{
  char *v = lookup(name);
  if (!v) return 0;
  *p = v;
  return 1;
}

void err(char *fmt, ...)
{
  va_list ap;
  fflush(stdout);
  fprintf(stderr, "%s: ", progname());
  va_start(ap, fmt);
  vfprintf(stderr, fmt, ap);
  va_end(ap);
  fprintf(stderr, "\n");
  exit(EXIT_FAILURE);
}

void warn(char *fmt, ...)
{
  va_list ap;
  if (getenv("SUSHIM_QUIET")) return;
  fprintf(stderr, "%s: ", progname());
  va_start(ap, fmt);
  vfprintf(stderr, fmt, ap);
  va_end(ap);
  fprintf(stderr, "\n");
}

FILE *efopen(const char *file, const char *mode)
{
  FILE *fp = fopen(file, mode);
  if (!fp) err("efopen: cannot open %s", (char *)file);
  return fp;
}

size_t efread(void *ptr, size_t size, size_t nitems, FILE *stream)
{
  size_t got = fread(ptr, size, nitems, stream);
  if (got != nitems && ferror(stream)) err("efread: read error");
  return got;
}

size_t efwrite(void *ptr, size_t size, size_t nitems, FILE *stream)
{
  size_t put = fwrite(ptr, size, nitems, stream);
  if (put != nitems) err("efwrite: write error");
  return put;
}

int efclose(FILE *stream)
{
  if (stream == NULL) return 0;
  if (fclose(stream)) err("efclose: close error");
  return 0;
}

/* ---------------- allocators ---------------- */
void *alloc1(size_t n1, size_t size)
{
  void *p = malloc(n1 * size ? n1 * size : 1);
  if (!p) err("alloc1: out of memory");
  return p;
}
void free1(void *p) { free(p); }
float *alloc1float(size_t n1) { return (float *)alloc1(n1, sizeof(float)); }
int *alloc1int(size_t n1) { return (int *)alloc1(n1, sizeof(int)); }
double *alloc1double(size_t n1) { return (double *)alloc1(n1, sizeof(double)); }
void free1float(float *p) { free(p); }
void free1int(int *p) { free(p); }
void free1double(double *p) { free(p); }

float **alloc2float(size_t n1, size_t n2)
{
  float **rows = (float **)alloc1(n2 ? n2 : 1, sizeof(float *));
  float *blk = (float *)alloc1(n1 * n2, sizeof(float));
  for (size_t i = 0; i < n2; ++i) rows[i] = blk + i * n1;
  if (n2 == 0) rows[0] = blk;
  return rows;
}
int **alloc2int(size_t n1, size_t n2)
{
  int **rows = (int **)alloc1(n2 ? n2 : 1, sizeof(int *));
  int *blk = (int *)alloc1(n1 * n2, sizeof(int));
  for (size_t i = 0; i < n2; ++i) rows[i] = blk + i * n1;
  if (n2 == 0) rows[0] = blk;
  return rows;
}
void free2float(float **p)
{
  if (!p) return;
  free(p[0]);
  free(p);
}
void free2int(int **p)
{
  if (!p) return;
  free(p[0]);
  free(p);
}
float ***alloc3float(size_t n1, size_t n2, size_t n3)
{
  float ***planes = (float ***)alloc1(n3 ? n3 : 1, sizeof(float **));
  float **rows = (float **)alloc1(n2 * n3 ? n2 * n3 : 1, sizeof(float *));
  float *blk = (float *)alloc1(n1 * n2 * n3, sizeof(float));
  for (size_t i3 = 0; i3 < n3; ++i3) {
    planes[i3] = rows + i3 * n2;
    for (size_t i2 = 0; i2 < n2; ++i2) planes[i3][i2] = blk + (i3 * n2 + i2) * n1;
  }
  return planes;
}
void free3float(float ***p)
{
  if (!p) return;
  free(p[0][0]);
  free(p[0]);
  free(p);
}

/* ---------------- SU traces ---------------- */
static int read_trace(FILE *fp, segy *tp)
{
  size_t got = fread(tp, 1, HDRBYTES, fp);
  if (got == 0) return 0;
  if (got != HDRBYTES) err("fgettr: truncated trace header");
  size_t ns = tp->ns;
  if (ns > SU_NFLTS) err("fgettr: ns=%d exceeds SU_NFLTS", (int)ns);
  if (fread(tp->data, sizeof(float), ns, fp) != ns) err("fgettr: truncated trace data");
  return (int)(HDRBYTES + ns * sizeof(float));
}

int fgettr(FILE *fp, segy *tp) { return read_trace(fp, tp); }
int fvgettr(FILE *fp, segy *tp) { return read_trace(fp, tp); }

void fputtr(FILE *fp, segy *tp)
{
  size_t ns = tp->ns;
  if (fwrite(tp, 1, HDRBYTES, fp) != HDRBYTES) err("fputtr: write error");
  if (fwrite(tp->data, sizeof(float), ns, fp) != ns) err("fputtr: write error");
}

/* ---------------- ints8r ---------------- */
static float sample_or_edge(int i, int nxin, const float *yin, float yinl, float yinr)
{
  if (i < 0) return yinl;
  if (i >= nxin) return yinr;
  return yin[i];
}

void ints8r(int nxin, float dxin, float fxin, float yin[], float yinl, float yinr, int nxout, float xout[],
            float yout[])
{
  static int warned = 0;
  for (int io = 0; io < nxout; ++io) {
    double p = ((double)xout[io] - (double)fxin) / (double)dxin;
    double n = floor(p + 0.5);
    if (fabs(p - n) <= 1.0e-4) {
      yout[io] = sample_or_edge((int)n, nxin, yin, yinl, yinr);
      continue;
    }
    if (!warned) {
      warned = 1;
      warn("ints8r: off-grid resampling (windowed sinc; not SU's table)");
    }
    int i0 = (int)floor(p);
    double frac = p - i0, acc = 0.0;
    for (int k = -3; k <= 4; ++k) {
      double x = k - frac;
      double s = fabs(x) < 1e-12 ? 1.0 : sin(PI * x) / (PI * x);
      double w = 0.5 * (1.0 + cos(PI * x / 4.5));
      acc += s * w * sample_or_edge(i0 + k, nxin, yin, yinl, yinr);
    }
    yout[io] = (float)acc;
  }
}
