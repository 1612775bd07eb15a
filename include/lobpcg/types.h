/*
 * Scalar types used by the BdG C API.
 *
 * The reference library takes f64 / c64 from its external eigensolver's
 * header "lobpcg/types.h" (included at include/bdg/bdg.h:4 of
 * pstuermer/BDG_LOBPCG).  This header provides the same two names so code
 * written against the reference API compiles unchanged.
 */
#ifndef LOBPCG_TYPES_H
#define LOBPCG_TYPES_H

typedef double f64;

#ifndef __cplusplus
#include <complex.h>
typedef double _Complex c64;
#endif

#endif /* LOBPCG_TYPES_H */
