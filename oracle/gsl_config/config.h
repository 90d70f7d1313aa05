/* Minimal configuration for compiling the handful of GSL 1.15 source files
 * the reference forward model links against (sys/expm1.c, sys/log1p.c,
 * sys/infnan.c, sort/sort.c, statistics/minmax.c, complex/math.c, err/*.c).
 * Written for glibc on x86-64, where every C99 math declaration exists and
 * IEEE comparisons/denormals behave normally.  Test infrastructure only. */
#ifndef ORACLE_GSL_CONFIG_H
#define ORACLE_GSL_CONFIG_H

#define HAVE_IEEE_COMPARISONS 1
#define HAVE_IEEE_DENORMALS 1
#define HAVE_DECL_ISFINITE 1
#define HAVE_DECL_FINITE 1
#define HAVE_DECL_ISNAN 1
#define HAVE_DECL_ISINF 1
#define HAVE_DECL_EXPM1 1
#define HAVE_DECL_LOG1P 1
#define HAVE_DECL_HYPOT 1
#define HAVE_DECL_ACOSH 1
#define HAVE_DECL_ASINH 1
#define HAVE_DECL_ATANH 1
#define HAVE_DECL_LDEXP 1
#define HAVE_DECL_FREXP 1
#define HAVE_DECL_FEENABLEEXCEPT 1
#define HAVE_INLINE 1
#define HAVE_C99_INLINE 1
#define RETURN_IF_NULL(x) if (!x) { return ; }

#endif
