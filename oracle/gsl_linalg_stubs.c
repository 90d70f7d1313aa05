/*
 * TEST INFRASTRUCTURE ONLY (linked into oracle/_ref/libjurassic_ref_ret.so,
 * never into the product).
 *
 * The reference's retrievalmodel.c is compiled from its own source so that
 * the oracle can call its kernel() (the finite-difference Jacobian).  The
 * same object also holds optimal_estimation() and the error analysis,
 * which call GSL's BLAS and Cholesky routines; those are outside the
 * bundled-GSL subset this build compiles.  The definitions below satisfy
 * the linker for those unused entry points and abort if anything calls
 * them.  kernel(), x2atm(), obs2y() and y2obs() do not.
 */
#include <stdio.h>
#include <stdlib.h>

#define ORACLE_UNUSED(name)                                                  \
  int name(void) {                                                           \
    fprintf(stderr, "oracle: %s is not part of the oracle build\n", #name);  \
    abort();                                                                 \
  }

ORACLE_UNUSED(gsl_blas_ddot)
ORACLE_UNUSED(gsl_blas_dgemm)
ORACLE_UNUSED(gsl_blas_dgemv)
ORACLE_UNUSED(gsl_linalg_cholesky_decomp)
ORACLE_UNUSED(gsl_linalg_cholesky_invert)
ORACLE_UNUSED(gsl_linalg_cholesky_solve)
