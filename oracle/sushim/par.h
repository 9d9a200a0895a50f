/* Minimal stand-in for the Seismic Unix "par.h" interface (getpar, err/warn,
 * checked file I/O). TEST INFRASTRUCTURE ONLY: lets the reference's own C
 * sources compile into oracle/_ref/. Written from SU's documented API. */
#ifndef ORACLE_SUSHIM_PAR_H
#define ORACLE_SUSHIM_PAR_H

#include "cwp.h"

extern int xargc;
extern char **xargv;
extern char *sdoc[];

void initargs(int argc, char **argv);
void requestdoc(int flag);
int getparint(char *name, int *p);
int getparfloat(char *name, float *p);
int getpardouble(char *name, double *p);
int getparstring(char *name, char **p);

void err(char *fmt, ...);
void warn(char *fmt, ...);

FILE *efopen(const char *file, const char *mode);
size_t efread(void *ptr, size_t size, size_t nitems, FILE *stream);
size_t efwrite(void *ptr, size_t size, size_t nitems, FILE *stream);
int efclose(FILE *stream);

#endif
