/* Private helpers shared by jk_oracle.c and jk_oracle_z.c. TEST INFRASTRUCTURE ONLY. */
#ifndef JK_ORACLE_IMPL_H
#define JK_ORACLE_IMPL_H

#include "jk_oracle.h"
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdbool.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* src/shared/params.F90:31-41 */
#define JO_TH1FIX 0.75
#define JO_EH 1024
#define JO_ET (-1021)
#define JO_MINF 4.9406564584124654e-324 /* Z'0000000000000001' */

static inline double jo_twof(void) { return sqrt(DBL_MAX); }

/* column-major 2x2: [0]=(1,1) [1]=(2,1) [2]=(1,2) [3]=(2,2) */
#define M11 0
#define M21 1
#define M12 2
#define M22 3

/* Fortran SIGN(1,x) .EQ. -1 with signed zeros */
static inline bool jo_neg(double x) { return signbit(x) != 0; }

static inline int jo_imin(int a, int b) { return a < b ? a : b; }

static inline jo_z jo_zc(double re, double im) { jo_z z; z.re = re; z.im = im; return z; }

#endif
