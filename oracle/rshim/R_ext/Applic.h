/*
 * Oracle-only stand-in for R's <R_ext/Applic.h>: the two QUADPACK drivers
 * libprofit calls (src/libprofit/src/profit/utils.cpp:228-242), with R's
 * calling convention (vectorised integrand, Fortran-style pointer args).
 * Definitions in rshim.c restate QUADPACK (Piessens et al., 1983).
 */
#ifndef PF_ORACLE_APPLIC_SHIM_H
#define PF_ORACLE_APPLIC_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef void integr_fn(double *x, int n, void *ex);

void Rdqags(integr_fn f, void *ex, double *a, double *b,
            double *epsabs, double *epsrel,
            double *result, double *abserr, int *neval, int *ier,
            int *limit, int *lenw, int *last, int *iwork, double *work);

void Rdqagi(integr_fn f, void *ex, double *bound, int *inf,
            double *epsabs, double *epsrel,
            double *result, double *abserr, int *neval, int *ier,
            int *limit, int *lenw, int *last, int *iwork, double *work);

#ifdef __cplusplus
}
#endif

#endif
