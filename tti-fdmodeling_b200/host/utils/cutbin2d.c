/* cutbin2d: crops a raw FP32 2D array (drop-in for src/main/wavelet/cutbin2d.c
 * of the reference): stdin holds n2 records of n1 floats; stdout receives
 * records fx2 .. fx2+nx2-1, samples fx1 .. fx1+nx1-1 of each. */
#include <stdio.h>
#include <stdlib.h>

#include "../hostio.h"

int main(int argc, char **argv)
{
  hio_initargs(argc, argv);
  if (argc == 1) {
    fputs(" CUTBIN2D - cut a binary file\n cutbin2d <stdin n1= n2= fx1= fx2= nx1= nx2= >stdout\n", stderr);
    return 1;
  }
  int n1, n2, fx1, fx2, nx1, nx2;
  if (!hio_getint("n1", &n1)) hio_err("<error>: must specify number of samples in 1st (fast) dimension!");
  if (!hio_getint("n2", &n2)) hio_err("<error>: must specify number of samples in 2nd (slow) dimension!");
  if (!hio_getint("fx1", &fx1)) fx1 = 0;
  if (!hio_getint("fx2", &fx2)) fx2 = 0;
  if (!hio_getint("nx1", &nx1)) nx1 = n1;
  if (!hio_getint("nx2", &nx2)) nx2 = n2;
  if (fx1 < 0 || fx2 < 0 || nx1 < 0 || nx2 < 0 || fx1 + nx1 > n1 || fx2 + nx2 > n2)
    hio_err("<error>: the cut window lies outside the %d x %d input", n1, n2);
  float *in = (float *)malloc(sizeof(float) * (size_t)(n1 > 0 ? n1 : 1));
  for (int i2 = 0; i2 < fx2 + nx2; ++i2) {
    if (fread(in, sizeof(float), n1, stdin) != (size_t)n1) hio_err("<error>: short input at record %d", i2);
    if (i2 >= fx2 && fwrite(in + fx1, sizeof(float), nx1, stdout) != (size_t)nx1) hio_err("<error>: write error");
  }
  free(in);
  return 0;
}
