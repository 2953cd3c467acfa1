/*
 * Oracle-only stand-in for R's <Rmath.h>, declaring the four special
 * functions libprofit calls through utils.cpp (src/libprofit/src/profit/
 * utils.cpp:193-207): Rf_qgamma, Rf_pgamma, Rf_gammafn and Rf_beta.
 *
 * This is test infrastructure.  The definitions live in rshim.c and follow
 * published methods, not R's sources (R is not vendored by the reference).
 */
#ifndef PF_ORACLE_RMATH_SHIM_H
#define PF_ORACLE_RMATH_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

double Rf_qgamma(double p, double shape, double scale, int lower_tail, int log_p);
double Rf_pgamma(double x, double shape, double scale, int lower_tail, int log_p);
double Rf_gammafn(double x);
double Rf_beta(double a, double b);

#ifdef __cplusplus
}
#endif

#endif
