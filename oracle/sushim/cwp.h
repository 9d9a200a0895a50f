/* Minimal stand-in for the Seismic Unix / CWP "cwp.h" interface.
 *
 * TEST INFRASTRUCTURE ONLY. This header exists so that the reference's own
 * C sources compile unmodified into oracle/_ref/ (the oracle). It is written
 * from the publicly documented CWP/SU API (names and signatures); no SU source
 * is present in this environment and none was copied. Only the subset the
 * reference's hot-path files call is provided.
 */
#ifndef ORACLE_SUSHIM_CWP_H
#define ORACLE_SUSHIM_CWP_H

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef PI
#define PI (3.141592653589793)
#endif
#ifndef MAX
#define MAX(x, y) ((x) > (y) ? (x) : (y))
#endif
#ifndef MIN
#define MIN(x, y) ((x) < (y) ? (x) : (y))
#endif
#ifndef ABS
#define ABS(x) ((x) < 0 ? -(x) : (x))
#endif
#ifndef SGN
#define SGN(x) ((x) < 0 ? -1.0 : 1.0)
#endif
#ifndef NINT
#define NINT(x) ((int)((x) > 0.0 ? (x) + 0.5 : (x)-0.5))
#endif
#ifndef FSIZE
#define FSIZE ((int)sizeof(float))
#endif
#ifndef ISIZE
#define ISIZE ((int)sizeof(int))
#endif
#ifndef DSIZE
#define DSIZE ((int)sizeof(double))
#endif

/* CWP programs end with `return (CWP_Exit());` */
#define CWP_Exit() (EXIT_SUCCESS)

/* contiguous allocators: an n2 x n1 array is one block, p[i2] = block + i2*n1 */
void *alloc1(size_t n1, size_t size);
void free1(void *p);
float *alloc1float(size_t n1);
int *alloc1int(size_t n1);
double *alloc1double(size_t n1);
void free1float(float *p);
void free1int(int *p);
void free1double(double *p);
float **alloc2float(size_t n1, size_t n2);
int **alloc2int(size_t n1, size_t n2);
void free2float(float **p);
void free2int(int **p);
float ***alloc3float(size_t n1, size_t n2, size_t n3);
void free3float(float ***p);

/* 8-point sinc interpolation of a uniformly sampled function */
void ints8r(int nxin, float dxin, float fxin, float yin[], float yinl, float yinr, int nxout, float xout[],
            float yout[]);

#endif
