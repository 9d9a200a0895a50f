/* sumkrcev2d: writes the SU receiver-position file read by the modelling
 * programs (drop-in for src/main/wavelet/sumkrcev2d.c of the reference):
 * trace 1 holds gx, trace 2 gz (= gdel), in cells, one sample per receiver.
 * Receivers lie every dtr cells at offsets offsetmin..offsetmax from sx inside
 * [0, nx): mode 0 both sides (sx itself once when offsetmin = 0), 1 left
 * side, 2 right side. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../hostio.h"

int main(int argc, char **argv)
{
  hio_initargs(argc, argv);
  if (argc == 1) {
    fputs(" SUMKRCEV2D - write receiver file\n sumkrcev2d sx= offsetmax= nx= [gdel=0 offsetmin=0 dtr=1 mode=0] > "
          "stdout\n",
          stderr);
    return 1;
  }
  int sx, gdel, offsetmin, dtr, offsetmax, nx, mode;
  if (!hio_getint("sx", &sx)) hio_err("<error>: didn't specify source position in 2nd dimension (unit: cell)!");
  if (!hio_getint("gdel", &gdel)) gdel = 0;
  if (!hio_getint("offsetmin", &offsetmin)) offsetmin = 0;
  if (!hio_getint("dtr", &dtr)) dtr = 1;
  if (!hio_getint("offsetmax", &offsetmax)) hio_err("<error>: didn't specify maximum offset(unit: cell).");
  if (!hio_getint("nx", &nx)) hio_err("<error>: didn't specify number of samples in 2nd dimension (unit: cell).");
  if (!hio_getint("mode", &mode)) mode = 0;
  if (dtr < 1) hio_err("<error>: dtr must be positive");
  /* left side: gx = sx - offsetmin, sx - offsetmin - dtr, ... while gx >= 0
   * and sx - gx <= offsetmax; right side mirrored inside [0, nx) */
  int nl = 0, nr = 0, gl = 0, gr = 0;
  if (mode == 0 || mode == 1)
    for (int g = sx - offsetmin; g >= 0 && sx - g <= offsetmax; g -= dtr) {
      ++nl;
      gl = g;
    }
  if (mode == 0 || mode == 2)
    for (int g = sx + offsetmin; g < nx && g - sx <= offsetmax; g += dtr) {
      ++nr;
      gr = g;
    }
  int ntr = nl + nr;
  if (mode == 0 && offsetmin == 0) { /* sx counted on both sides */
    --ntr;
    --nl;
  }
  if (ntr < 0) ntr = 0;
  if (ntr > 32767) hio_err("<error>: the number of traces is too much.");
  float *gx = (float *)calloc(ntr > 0 ? ntr : 1, sizeof(float));
  float *gz = (float *)calloc(ntr > 0 ? ntr : 1, sizeof(float));
  for (int i = 0; i < nl; ++i) gx[i] = (float)(gl + i * dtr);       /* ascending from the leftmost */
  for (int i = 0; i < nr; ++i) gx[ntr - 1 - i] = (float)(gr - i * dtr); /* descending from the rightmost */
  for (int i = 0; i < ntr; ++i) gz[i] = (float)gdel;
  unsigned char h[HIO_SU_HDR];
  memset(h, 0, sizeof h);
  hio_put_i32(h, HIO_TRACL, 1);
  hio_put_i16(h, HIO_TRID, 1);
  hio_put_i16(h, HIO_SCALEL, -1000);
  hio_put_i16(h, HIO_SCALCO, -1000);
  hio_put_i32(h, HIO_GDEL, hio_scalar_write((float)gdel, -1000));
  hio_put_i32(h, HIO_SX, hio_scalar_write((float)sx, -1000));
  hio_put_u16(h, HIO_NS, ntr);
  hio_put_i32(h, HIO_NTR, 2);
  /* the reference stores dtr * 10^7 into the 16-bit dt field; keep the same bits */
  hio_put_u16(h, HIO_DT, (unsigned short)(dtr * 10000000));
  hio_put_f32(h, HIO_F1, 0.0f);
  hio_put_f32(h, HIO_D1, (float)dtr);
  hio_write_trace(stdout, h, gx, ntr);
  hio_write_trace(stdout, h, gz, ntr);
  free(gx);
  free(gz);
  return 0;
}
