/* Minimal stand-in for MATLAB's mex.h.
 *
 * Test infrastructure only: it lets the reference's C MEX sources
 * (tom_rotatec.c, tom_peakinc.c, tom_calc_weight_functioninc.c) compile as
 * plain shared libraries so the oracle can call their compute routines
 * (rot3d, find_max, weight3d) through ctypes.  The MEX gateway
 * (mexFunction) is compiled but never called; every mx* function here aborts.
 */
#ifndef ORACLE_STUB_MEX_H
#define ORACLE_STUB_MEX_H
#include <stdio.h>
#include <stdlib.h>
#include "matrix.h"

static void mexErrMsgTxt(const char *m) { fprintf(stderr, "%s\n", m); abort(); }
#endif
