/* Stand-in for SU's "header.h". TEST INFRASTRUCTURE ONLY. */
#ifndef ORACLE_SUSHIM_HEADER_H
#define ORACLE_SUSHIM_HEADER_H
#include "segy.h"
#endif
