/* sumksrc2d: writes the SU source file read by the modelling programs
 * (drop-in for src/main/wavelet/sumksrc2d.c of the reference): one trace on
 * stdout, sdepth/sx scaled by scalel = scalco = -1000 (cells x 1000), dt in
 * microseconds, ns = nt, ntr = 1. Wavelets follow src/lib/wavelet/wavelet.c:
 *   wtype 1 Ricker, 2 first derivative of a Gaussian, 3 first derivative of a
 *   Ricker, 4 Gaussian; all shifted by `delay` (default 1.5/fpeak), zero for
 *   t > delay after the shift, first sample zero; or a raw wavelet file. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../hostio.h"

/* the wavelet formulas of src/lib/wavelet/wavelet.c, in float as there */
static void wavelet(int wtype, float *w, float A, float fpeak, float delay, float dt, int nt)
{
  const float pi = 3.141592654f;
  for (int it = 0; it < nt; ++it) {
    const float t = it * dt - delay;
    if (t > delay) {
      w[it] = 0.0f;
      continue;
    }
    const float a = powf(pi * fpeak * t, 2.0f);
    switch (wtype) {
    case 1: w[it] = A * (1.0f - 2.0f * a) * expf(-1.0f * a); break;
    case 2: w[it] = A * t * expf(-a); break;
    case 3: w[it] = A * (2.0f * powf(pi * fpeak, 2.0f) * t) * (2.0f * a - 3.0f) * expf(-1.0f * a); break;
    default: w[it] = 0.5f / powf(pi * fpeak, 2.0f) * expf(-a); break;
    }
  }
  if (nt > 0) w[0] = 0.0f;
}

int main(int argc, char **argv)
{
  hio_initargs(argc, argv);
  if (argc == 1) {
    fputs(" SUMKSRC2D - write source file\n sumksrc2d sdepth= sx= dt= nt= [wtype=1 A=1 fpeak=10 delay=1.5/fpeak "
          "wfile=] > stdout\n",
          stderr);
    return 1;
  }
  int nt, wtype, sdepth, sx;
  float dt, A, fpeak, delay;
  char *wfile = NULL;
  hio_getstring("wfile", &wfile);
  if (!hio_getint("nt", &nt)) hio_err("<error>: must specify number of samples in time dimension!");
  if (!hio_getint("wtype", &wtype)) wtype = 1;
  if (!hio_getint("sdepth", &sdepth)) hio_err("<error>: must specify source position in 2nd dimension!");
  if (!hio_getint("sx", &sx)) hio_err("<error>: must specify source position in 1st dimension!");
  if (!hio_getfloat("dt", &dt)) hio_err("<error>: must specify sampleing interval in time dimension!");
  if (!hio_getfloat("A", &A)) A = 1.0f;
  if (!hio_getfloat("fpeak", &fpeak)) fpeak = 10.0f;
  if (!hio_getfloat("delay", &delay)) delay = 1.5f / fpeak;
  if (nt < 0 || nt > 65535) hio_err("<error>: nt=%d does not fit an SU trace", nt);
  float *w = (float *)calloc(nt > 0 ? nt : 1, sizeof(float));
  if (wfile) {
    FILE *fp = fopen(wfile, "rb");
    if (!fp) hio_err("<error>: failed to open wavelet file (%s)!", wfile);
    if (fread(w, sizeof(float), nt, fp) != (size_t)nt) hio_warn("<warning>: short wavelet file %s", wfile);
    fclose(fp);
  } else {
    wavelet(wtype, w, A, fpeak, delay, dt, nt);
  }
  unsigned char h[HIO_SU_HDR];
  memset(h, 0, sizeof h);
  hio_put_i32(h, HIO_TRACL, 1);
  hio_put_i16(h, HIO_TRID, 1);
  hio_put_i16(h, HIO_SCALEL, -1000);
  hio_put_i16(h, HIO_SCALCO, -1000);
  hio_put_i32(h, HIO_SDEPTH, hio_scalar_write((float)sdepth, -1000));
  hio_put_i32(h, HIO_SX, hio_scalar_write((float)sx, -1000));
  hio_put_u16(h, HIO_NS, nt);
  hio_put_u16(h, HIO_DT, (unsigned short)(dt * 1000000));
  hio_put_f32(h, HIO_F1, 0.0f);
  hio_put_f32(h, HIO_D1, dt);
  hio_put_i32(h, HIO_NTR, 1);
  hio_write_trace(stdout, h, w, nt);
  free(w);
  return 0;
}
