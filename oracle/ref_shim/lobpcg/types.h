/*
 * lobpcg/types.h -- scalar types of the external "LOBPCG" library that
 * pstuermer/BDG_LOBPCG includes (src/bdg_internal.h:5, include/bdg/bdg.h:4).
 * That library is not vendored; this oracle-build header supplies the two
 * names the reference uses.  TEST INFRASTRUCTURE ONLY.
 */
#ifndef LOBPCG_TYPES_H
#define LOBPCG_TYPES_H
#include <complex.h>
typedef double f64;
typedef double _Complex c64;
#endif
