/* Minimal stand-in for SU's "su.h" trace I/O. TEST INFRASTRUCTURE ONLY. */
#ifndef ORACLE_SUSHIM_SU_H
#define ORACLE_SUSHIM_SU_H

#include "par.h"
#include "segy.h"

int fgettr(FILE *fp, segy *tp);
int fvgettr(FILE *fp, segy *tp);
void fputtr(FILE *fp, segy *tp);
#define gettr(tp) fgettr(stdin, (tp))
#define vgettr(tp) fvgettr(stdin, (tp))
#define puttr(tp) fputtr(stdout, (tp))

#endif
