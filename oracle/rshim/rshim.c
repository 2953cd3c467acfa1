/*
 * ORACLE (test infrastructure only).  Stand-ins for the R math routines that
 * libprofit 1.9.3 calls (src/libprofit/src/profit/utils.cpp:193-258):
 *
 *   Rf_qgamma(p, shape, 1, 1, 0)   lower-tail gamma quantile
 *   Rf_pgamma(x, shape, 1, 1, 0)   regularised lower incomplete gamma P(a, x)
 *   Rf_gammafn(x)                  Gamma(x)
 *   Rf_beta(a, b)                  Beta(a, b)
 *   Rdqags / Rdqagi                QUADPACK adaptive integrators
 *
 * R itself is not part of the reference tree (DESCRIPTION: "Depends R (>= 3.0)",
 * no pinned version), so these are written from published methods:
 *   - P(a, x): power series for x < a + 1, Lentz continued fraction for Q
 *     otherwise (Numerical-analysis textbook forms, e.g. Press et al. 6.2);
 *     prefactor x^a e^-x / Gamma(a) evaluated in log space with lgamma().
 *   - quantile: safeguarded Newton/Halley on P(a, x) - p with bisection
 *     fallback, started at the Wilson-Hilferty / small-x approximations.
 *   - QUADPACK dqagse/dqagie/dqk21/dqk15i/dqpsrt/dqelg from R. Piessens,
 *     E. de Doncker-Kapenga, C. Ueberhuber, D. Kahaner, "QUADPACK: a
 *     subroutine package for automatic integration", Springer 1983.
 *     Gauss-Kronrod nodes/weights are the published tables.
 *
 * Only tests, the smoke check and the CPU-baseline leg of the benchmark load
 * the library built from this file.
 */
#define _GNU_SOURCE
#include <float.h>
#include <math.h>
#include <stdlib.h>

#include "Rmath.h"
#include "R_ext/Applic.h"

/* ------------------------------------------------------------------------- */
/* Gamma, Beta                                                               */
/* ------------------------------------------------------------------------- */

double Rf_gammafn(double x)
{
	return tgamma(x);
}

double Rf_beta(double a, double b)
{
	/* Same guard structure as the usual Beta implementations: direct product of
	 * Gamma values while a + b stays below the Gamma overflow point, log form
	 * beyond it. */
	const double xmax = 171.61447887182298;
	if (isnan(a) || isnan(b)) return a + b;
	if (a < 0 || b < 0) return NAN;
	if (a == 0 || b == 0) return INFINITY;
	if (isinf(a) || isinf(b)) return 0;
	if (a + b < xmax) {
		return (1.0 / tgamma(a + b)) * (tgamma(a) * tgamma(b));
	}
	return exp(lgamma(a) + lgamma(b) - lgamma(a + b));
}

/* ------------------------------------------------------------------------- */
/* Regularised incomplete gamma                                              */
/* ------------------------------------------------------------------------- */

/* log(x^a e^-x / Gamma(a)) */
static double log_gamma_prefactor(double a, double x)
{
	return a * log(x) - x - lgamma(a);
}

/* P(a, x) by the power series  x^a e^-x / Gamma(a+1) * sum x^n / ((a+1)...(a+n)) */
static double p_series(double a, double x)
{
	double term = 1.0 / a;
	double sum = term;
	for (int n = 1; n < 10000; n++) {
		term *= x / (a + n);
		sum += term;
		if (fabs(term) < fabs(sum) * 1e-17) break;
	}
	return sum * exp(log_gamma_prefactor(a, x));
}

/* Q(a, x) by the modified Lentz continued fraction */
static double q_contfrac(double a, double x)
{
	const double tiny = 1e-300;
	double b = x + 1.0 - a;
	double c = 1.0 / tiny;
	double d = 1.0 / b;
	double h = d;
	for (int i = 1; i < 10000; i++) {
		double an = -i * (i - a);
		b += 2.0;
		d = an * d + b;
		if (fabs(d) < tiny) d = tiny;
		c = b + an / c;
		if (fabs(c) < tiny) c = tiny;
		d = 1.0 / d;
		double del = d * c;
		h *= del;
		if (fabs(del - 1.0) < 1e-17) break;
	}
	return exp(log_gamma_prefactor(a, x)) * h;
}

static double p_lower(double a, double x)
{
	if (x <= 0) return 0.0;
	if (isinf(x)) return 1.0;
	if (x < a + 1.0) return p_series(a, x);
	return 1.0 - q_contfrac(a, x);
}

static double q_upper(double a, double x)
{
	if (x <= 0) return 1.0;
	if (isinf(x)) return 0.0;
	if (x < a + 1.0) return 1.0 - p_series(a, x);
	return q_contfrac(a, x);
}

double Rf_pgamma(double x, double shape, double scale, int lower_tail, int log_p)
{
	if (isnan(x) || isnan(shape) || isnan(scale)) return x + shape + scale;
	if (shape < 0 || scale <= 0) return NAN;
	x /= scale;
	double v;
	if (shape == 0) {
		v = (x <= 0) ? (lower_tail ? 0.0 : 1.0) : (lower_tail ? 1.0 : 0.0);
	}
	else {
		v = lower_tail ? p_lower(shape, x) : q_upper(shape, x);
	}
	return log_p ? log(v) : v;
}

/* dP(a, x)/dx = x^(a-1) e^-x / Gamma(a) */
static double p_density(double a, double x)
{
	if (x <= 0) return 0.0;
	return exp((a - 1.0) * log(x) - x - lgamma(a));
}

double Rf_qgamma(double p, double shape, double scale, int lower_tail, int log_p)
{
	if (isnan(p) || isnan(shape) || isnan(scale)) return p + shape + scale;
	if (log_p) p = exp(p);
	if (!lower_tail) p = 1.0 - p;
	if (p < 0 || p > 1 || shape < 0 || scale <= 0) return NAN;
	if (shape == 0) return 0.0;
	if (p == 0) return 0.0;
	if (p == 1) return INFINITY;

	const double a = shape;

	/* Starting point. */
	double x;
	{
		/* Wilson-Hilferty needs a normal quantile; a few Newton steps on the
		 * normal CDF via erfc give it to full precision. */
		double z = 0.0;
		for (int it = 0; it < 60; it++) {
			double cdf = 0.5 * erfc(-z / sqrt(2.0));
			double pdf = exp(-0.5 * z * z) / sqrt(2.0 * M_PI);
			double step = (cdf - p) / pdf;
			if (step > 5) step = 5;
			if (step < -5) step = -5;
			z -= step;
			if (fabs(step) < 1e-14) break;
		}
		double c = 1.0 / (9.0 * a);
		double t = 1.0 - c + z * sqrt(c);
		x = a * t * t * t;
		double small = exp((log(p) + lgamma(a + 1.0)) / a);
		if (!(x > 0) || x < small) x = small;
	}

	/* Bracket [lo, hi] with P(lo) < p < P(hi). */
	double lo = 0.0, hi = INFINITY;
	for (int it = 0; it < 400; it++) {
		double P = p_lower(a, x);
		double f = P - p;
		if (f == 0) return x * scale;
		if (f < 0) lo = x; else hi = x;
		double d = p_density(a, x);
		double xn;
		if (d > 0 && isfinite(d)) {
			double newton = f / d;
			/* Halley correction: P'' / P' = (a - 1)/x - 1 */
			double corr = 1.0 - 0.5 * newton * ((a - 1.0) / x - 1.0);
			double step = newton;
			if (corr > 0.5 && corr < 2.0) step = newton / corr;
			xn = x - step;
		}
		else {
			xn = NAN;
		}
		if (!(xn > lo && xn < hi)) {
			xn = isinf(hi) ? (2.0 * x + 1.0) : 0.5 * (lo + hi);
		}
		if (fabs(xn - x) <= 4 * DBL_EPSILON * fabs(xn)) {
			x = xn;
			break;
		}
		x = xn;
	}
	return x * scale;
}

/* ------------------------------------------------------------------------- */
/* QUADPACK restatement                                                      */
/* ------------------------------------------------------------------------- */

typedef struct {
	integr_fn *f;
	void *ex;
} qp_fun;

/* 21-point Gauss-Kronrod abscissae and weights (published tables). */
static const double qk21_xgk[11] = {
	0.995657163025808080735527280689003, 0.973906528517171720077964012084452,
	0.930157491355708226001207180059508, 0.865063366688984510732096688423493,
	0.780817726586416897063717578345042, 0.679409568299024406234327365114874,
	0.562757134668604683339000099272694, 0.433395394129247190799265943165784,
	0.294392862701460198131126603103866, 0.148874338981631210884826001129720,
	0.000000000000000000000000000000000};
static const double qk21_wgk[11] = {
	0.011694638867371874278064396062192, 0.032558162307964727478818972459390,
	0.054755896574351996031381300244580, 0.075039674810919952767043140916190,
	0.093125454583697605535065465083366, 0.109387158802297641899210590325805,
	0.123491976262065851077600525452925, 0.134709217311473325928054001771707,
	0.142775938577060080797094273138717, 0.147739104901338491374841515972068,
	0.149445554002916905664936468389821};
static const double qk21_wg[5] = {
	0.066671344308688137593568809893332, 0.149451349150580593145776339657697,
	0.219086362515982043995534934228163, 0.269266719309996355091226921569469,
	0.295524224714752870173892994651338};

/* 15-point Gauss-Kronrod for the (0,1] transformed semi-infinite range. */
static const double qk15i_xgk[8] = {
	0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
	0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
	0.586087235467691130294144845693013, 0.405845151377397166906606412076961,
	0.207784955007898467600689403773245, 0.000000000000000000000000000000000};
static const double qk15i_wgk[8] = {
	0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
	0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
	0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
	0.204432940075298892414161999234649, 0.209482141084727828012999174891714};
static const double qk15i_wg[8] = {
	0.000000000000000000000000000000000, 0.129484966168869693270611432679082,
	0.000000000000000000000000000000000, 0.279705391489276667901467771423780,
	0.000000000000000000000000000000000, 0.381830050505118944950369775488975,
	0.000000000000000000000000000000000, 0.417959183673469387755102040816327};

static double qp_eval(const qp_fun *F, double x)
{
	double v = x;
	F->f(&v, 1, F->ex);
	return v;
}

static void qk21(const qp_fun *F, double a, double b, double *result,
                 double *abserr, double *resabs, double *resasc)
{
	const double epmach = DBL_EPSILON, uflow = DBL_MIN;
	double fv1[10], fv2[10];
	double centr = 0.5 * (a + b);
	double hlgth = 0.5 * (b - a);
	double dhlgth = fabs(hlgth);
	double resg = 0.0;
	double fc = qp_eval(F, centr);
	double resk = qk21_wgk[10] * fc;
	*resabs = fabs(resk);
	for (int j = 0; j < 5; j++) {
		int jtw = 2 * j + 1;
		double absc = hlgth * qk21_xgk[jtw];
		double f1 = qp_eval(F, centr - absc);
		double f2 = qp_eval(F, centr + absc);
		fv1[jtw] = f1;
		fv2[jtw] = f2;
		double fsum = f1 + f2;
		resg += qk21_wg[j] * fsum;
		resk += qk21_wgk[jtw] * fsum;
		*resabs += qk21_wgk[jtw] * (fabs(f1) + fabs(f2));
	}
	for (int j = 0; j < 5; j++) {
		int jtwm1 = 2 * j;
		double absc = hlgth * qk21_xgk[jtwm1];
		double f1 = qp_eval(F, centr - absc);
		double f2 = qp_eval(F, centr + absc);
		fv1[jtwm1] = f1;
		fv2[jtwm1] = f2;
		double fsum = f1 + f2;
		resk += qk21_wgk[jtwm1] * fsum;
		*resabs += qk21_wgk[jtwm1] * (fabs(f1) + fabs(f2));
	}
	double reskh = resk * 0.5;
	*resasc = qk21_wgk[10] * fabs(fc - reskh);
	for (int j = 0; j < 10; j++) {
		*resasc += qk21_wgk[j] * (fabs(fv1[j] - reskh) + fabs(fv2[j] - reskh));
	}
	*result = resk * hlgth;
	*resabs *= dhlgth;
	*resasc *= dhlgth;
	*abserr = fabs((resk - resg) * hlgth);
	if (*resasc != 0.0 && *abserr != 0.0) {
		double r = pow(200.0 * *abserr / *resasc, 1.5);
		*abserr = *resasc * (r < 1.0 ? r : 1.0);
	}
	if (*resabs > uflow / (50.0 * epmach)) {
		double m = epmach * 50.0 * *resabs;
		if (m > *abserr) *abserr = m;
	}
}

/* Integrand on [bound, inf) mapped onto (0, 1] by x = bound + (1 - t)/t. */
static void qk15i(const qp_fun *F, double boun, int inf, double a, double b,
                  double *result, double *abserr, double *resabs, double *resasc)
{
	const double epmach = DBL_EPSILON, uflow = DBL_MIN;
	double fv1[7], fv2[7];
	double dinf = (double)(inf < 1 ? inf : 1);
	double centr = 0.5 * (a + b);
	double hlgth = 0.5 * (b - a);
	double tabsc1 = boun + dinf * (1.0 - centr) / centr;
	double fval1 = qp_eval(F, tabsc1);
	if (inf == 2) fval1 += qp_eval(F, -tabsc1);
	double fc = (fval1 / centr) / centr;
	double resg = qk15i_wg[7] * fc;
	double resk = qk15i_wgk[7] * fc;
	*resabs = fabs(resk);
	for (int j = 0; j < 7; j++) {
		double absc = hlgth * qk15i_xgk[j];
		double absc1 = centr - absc;
		double absc2 = centr + absc;
		double t1 = boun + dinf * (1.0 - absc1) / absc1;
		double t2 = boun + dinf * (1.0 - absc2) / absc2;
		double f1 = qp_eval(F, t1);
		double f2 = qp_eval(F, t2);
		if (inf == 2) {
			f1 += qp_eval(F, -t1);
			f2 += qp_eval(F, -t2);
		}
		f1 = (f1 / absc1) / absc1;
		f2 = (f2 / absc2) / absc2;
		fv1[j] = f1;
		fv2[j] = f2;
		double fsum = f1 + f2;
		resg += qk15i_wg[j] * fsum;
		resk += qk15i_wgk[j] * fsum;
		*resabs += qk15i_wgk[j] * (fabs(f1) + fabs(f2));
	}
	double reskh = resk * 0.5;
	*resasc = qk15i_wgk[7] * fabs(fc - reskh);
	for (int j = 0; j < 7; j++) {
		*resasc += qk15i_wgk[j] * (fabs(fv1[j] - reskh) + fabs(fv2[j] - reskh));
	}
	*result = resk * hlgth;
	*resasc *= hlgth;
	*resabs *= hlgth;
	*abserr = fabs((resk - resg) * hlgth);
	if (*resasc != 0.0 && *abserr != 0.0) {
		double r = pow(200.0 * *abserr / *resasc, 1.5);
		*abserr = *resasc * (r < 1.0 ? r : 1.0);
	}
	if (*resabs > uflow / (50.0 * epmach)) {
		double m = epmach * 50.0 * *resabs;
		if (m > *abserr) *abserr = m;
	}
}

/* Maintains the descending ordering of error estimates (1-based arrays). */
static void qpsrt(int limit, int last, int *maxerr, double *ermax,
                  const double *elist, int *iord, int *nrmax)
{
	int i, j, k, isucc, jbnd, jupbn, ibeg, ido;
	double errmax, errmin;

	if (last <= 2) {
		iord[1] = 1;
		iord[2] = 2;
		goto done;
	}
	errmax = elist[*maxerr];
	if (*nrmax != 1) {
		ido = *nrmax - 1;
		for (i = 1; i <= ido; i++) {
			isucc = iord[*nrmax - 1];
			if (errmax <= elist[isucc]) break;
			iord[*nrmax] = isucc;
			(*nrmax)--;
		}
	}
	jupbn = last;
	if (last > limit / 2 + 2) jupbn = limit + 3 - last;
	errmin = elist[last];
	jbnd = jupbn - 1;
	ibeg = *nrmax + 1;
	if (ibeg <= jbnd) {
		for (i = ibeg; i <= jbnd; i++) {
			isucc = iord[i];
			if (errmax >= elist[isucc]) goto insert_min;
			iord[i - 1] = isucc;
		}
	}
	iord[jbnd] = *maxerr;
	iord[jupbn] = last;
	goto done;

insert_min:
	iord[i - 1] = *maxerr;
	k = jbnd;
	for (j = i; j <= jbnd; j++) {
		isucc = iord[k];
		if (errmin < elist[isucc]) {
			iord[k + 1] = last;
			goto done;
		}
		iord[k + 1] = isucc;
		k--;
	}
	iord[i] = last;

done:
	*maxerr = iord[*nrmax];
	*ermax = elist[*maxerr];
}

/* Wynn's epsilon algorithm (1-based epstab[1..52], res3la[1..3]). */
static void qelg(int *n, double *epstab, double *result, double *abserr,
                 double *res3la, int *nres)
{
	const double epmach = DBL_EPSILON, oflow = DBL_MAX;
	int i, ib, ie, ib2, indx, k1, k2, k3, num, newelm;
	const int limexp = 50;
	double e0, e1, e2, e3, e1abs, res, delta1, delta2, delta3;
	double err1, err2, err3, tol1, tol2, tol3, ss, epsinf, error;

	(*nres)++;
	*abserr = oflow;
	*result = epstab[*n];
	if (*n < 3) goto finish;
	epstab[*n + 2] = epstab[*n];
	newelm = (*n - 1) / 2;
	epstab[*n] = oflow;
	num = *n;
	k1 = *n;
	for (i = 1; i <= newelm; i++) {
		k2 = k1 - 1;
		k3 = k1 - 2;
		res = epstab[k1 + 2];
		e0 = epstab[k3];
		e1 = epstab[k2];
		e2 = res;
		e1abs = fabs(e1);
		delta2 = e2 - e1;
		err2 = fabs(delta2);
		tol2 = fmax(fabs(e2), e1abs) * epmach;
		delta3 = e1 - e0;
		err3 = fabs(delta3);
		tol3 = fmax(e1abs, fabs(e0)) * epmach;
		if (err2 <= tol2 && err3 <= tol3) {
			*result = res;
			*abserr = err2 + err3;
			goto finish;
		}
		e3 = epstab[k1];
		epstab[k1] = e1;
		delta1 = e1 - e3;
		err1 = fabs(delta1);
		tol1 = fmax(e1abs, fabs(e3)) * epmach;
		if (err1 <= tol1 || err2 <= tol2 || err3 <= tol3) {
			*n = i + i - 1;
			break;
		}
		ss = 1.0 / delta1 + 1.0 / delta2 - 1.0 / delta3;
		epsinf = fabs(ss * e1);
		if (!(epsinf > 1e-4)) {
			*n = i + i - 1;
			break;
		}
		res = e1 + 1.0 / ss;
		epstab[k1] = res;
		k1 -= 2;
		error = err2 + fabs(res - e2) + err3;
		if (error > *abserr) continue;
		*abserr = error;
		*result = res;
	}

	if (*n == limexp) *n = (limexp / 2) * 2 - 1;
	ib = (num % 2 == 0) ? 2 : 1;
	ie = newelm + 1;
	for (i = 1; i <= ie; i++) {
		ib2 = ib + 2;
		epstab[ib] = epstab[ib2];
		ib = ib2;
	}
	if (num != *n) {
		indx = num - *n + 1;
		for (i = 1; i <= *n; i++) {
			epstab[i] = epstab[indx];
			indx++;
		}
	}
	if (*nres < 4) {
		res3la[*nres] = *result;
		*abserr = oflow;
	}
	else {
		*abserr = fabs(*result - res3la[3]) + fabs(*result - res3la[2]) +
		          fabs(*result - res3la[1]);
		res3la[1] = res3la[2];
		res3la[2] = res3la[3];
		res3la[3] = *result;
	}

finish:
	*abserr = fmax(*abserr, 5.0 * epmach * fabs(*result));
}

typedef void (*qp_rule)(const qp_fun *F, double boun, int inf, double a,
                        double b, double *result, double *abserr,
                        double *resabs, double *resasc);

static void rule21(const qp_fun *F, double boun, int inf, double a, double b,
                   double *result, double *abserr, double *resabs, double *resasc)
{
	(void)boun;
	(void)inf;
	qk21(F, a, b, result, abserr, resabs, resasc);
}

/*
 * Shared body of dqagse (finite range, 21-point rule, small = 0.375 |b - a|)
 * and dqagie (semi-infinite range mapped to (0, 1], 15-point rule,
 * small = 0.375).  Arrays are 1-based with room for `limit` intervals.
 */
static void qag_extrap(const qp_fun *F, qp_rule rule, double boun, int inf,
                       double a, double b, double small0,
                       double epsabs, double epsrel, int limit,
                       double *result, double *abserr, int *neval, int *ier,
                       int *last_out)
{
	const double epmach = DBL_EPSILON, uflow = DBL_MIN, oflow = DBL_MAX;
	double *alist = (double *)calloc(limit + 1, sizeof(double));
	double *blist = (double *)calloc(limit + 1, sizeof(double));
	double *rlist = (double *)calloc(limit + 1, sizeof(double));
	double *elist = (double *)calloc(limit + 1, sizeof(double));
	int *iord = (int *)calloc(limit + 1, sizeof(int));
	double rlist2[53], res3la[4];
	double area, area1, area2, area12, a1, a2, b1, b2, defabs, defab1, defab2;
	double dres, erlarg = 0, erlast, errbnd, errmax, error1, error2, erro12;
	double errsum, ertest = 0, resabs, reseps, abseps, correc = 0, small = 0;
	int id, ierro, iroff1, iroff2, iroff3, jupbnd, k, ksgn, ktmin, last;
	int maxerr, nres, nrmax, numrl2;
	int extrap, noext;

	*ier = 0;
	*neval = 0;
	last = 0;
	*result = 0.0;
	*abserr = 0.0;
	alist[1] = a;
	blist[1] = b;
	rlist[1] = 0.0;
	elist[1] = 0.0;
	iord[1] = 0;

	if (epsabs <= 0.0 && epsrel < fmax(50.0 * epmach, 0.5e-28)) {
		*ier = 6;
		goto cleanup;
	}

	ierro = 0;
	rule(F, boun, inf, a, b, result, abserr, &defabs, &resabs);
	dres = fabs(*result);
	errbnd = fmax(epsabs, epsrel * dres);
	last = 1;
	rlist[1] = *result;
	elist[1] = *abserr;
	iord[1] = 1;
	if (*abserr <= 100.0 * epmach * defabs && *abserr > errbnd) *ier = 2;
	if (limit == 1) *ier = 1;
	if (*ier != 0 || (*abserr <= errbnd && *abserr != resabs) || *abserr == 0.0)
		goto finish_neval;

	rlist2[1] = *result;
	errmax = *abserr;
	maxerr = 1;
	area = *result;
	errsum = *abserr;
	*abserr = oflow;
	nrmax = 1;
	nres = 0;
	numrl2 = 2;
	ktmin = 0;
	extrap = 0;
	noext = 0;
	iroff1 = iroff2 = iroff3 = 0;
	ksgn = -1;
	if (dres >= (1.0 - 50.0 * epmach) * defabs) ksgn = 1;

	for (last = 2; last <= limit; last++) {
		a1 = alist[maxerr];
		b1 = 0.5 * (alist[maxerr] + blist[maxerr]);
		a2 = b1;
		b2 = blist[maxerr];
		erlast = errmax;
		rule(F, boun, inf, a1, b1, &area1, &error1, &resabs, &defab1);
		rule(F, boun, inf, a2, b2, &area2, &error2, &resabs, &defab2);

		area12 = area1 + area2;
		erro12 = error1 + error2;
		errsum = errsum + erro12 - errmax;
		area = area + area12 - rlist[maxerr];
		if (!(defab1 == error1 || defab2 == error2)) {
			if (fabs(rlist[maxerr] - area12) <= 1e-5 * fabs(area12) &&
			    erro12 >= 0.99 * errmax) {
				if (extrap) iroff2++;
				else iroff1++;
			}
			if (last > 10 && erro12 > errmax) iroff3++;
		}
		rlist[maxerr] = area1;
		rlist[last] = area2;
		errbnd = fmax(epsabs, epsrel * fabs(area));

		if (iroff1 + iroff2 >= 10 || iroff3 >= 20) *ier = 2;
		if (iroff2 >= 5) ierro = 3;
		if (last == limit) *ier = 1;
		if (fmax(fabs(a1), fabs(b2)) <= (1.0 + 100.0 * epmach) * (fabs(a2) + 1000.0 * uflow))
			*ier = 4;

		if (error2 > error1) {
			alist[maxerr] = a2;
			alist[last] = a1;
			blist[last] = b1;
			rlist[maxerr] = area2;
			rlist[last] = area1;
			elist[maxerr] = error2;
			elist[last] = error1;
		}
		else {
			alist[last] = a2;
			blist[maxerr] = b1;
			blist[last] = b2;
			elist[maxerr] = error1;
			elist[last] = error2;
		}

		qpsrt(limit, last, &maxerr, &errmax, elist, iord, &nrmax);

		if (errsum <= errbnd) goto sum_result;
		if (*ier != 0) goto final_result;
		if (last == 2) {
			small = small0;
			erlarg = errsum;
			ertest = errbnd;
			rlist2[2] = area;
			continue;
		}
		if (noext) continue;

		erlarg -= erlast;
		if (fabs(b1 - a1) > small) erlarg += erro12;
		if (!extrap) {
			if (fabs(blist[maxerr] - alist[maxerr]) > small) continue;
			extrap = 1;
			nrmax = 2;
		}
		if (ierro != 3 && erlarg > ertest) {
			int jump = 0;
			id = nrmax;
			jupbnd = last;
			if (last > 2 + limit / 2) jupbnd = limit + 3 - last;
			for (k = id; k <= jupbnd; k++) {
				maxerr = iord[nrmax];
				errmax = elist[maxerr];
				if (fabs(blist[maxerr] - alist[maxerr]) > small) {
					jump = 1;
					break;
				}
				nrmax++;
			}
			if (jump) continue;
		}

		numrl2++;
		rlist2[numrl2] = area;
		qelg(&numrl2, rlist2, &reseps, &abseps, res3la, &nres);
		ktmin++;
		if (ktmin > 5 && *abserr < 1e-3 * errsum) *ier = 5;
		if (abseps < *abserr) {
			ktmin = 0;
			*abserr = abseps;
			*result = reseps;
			correc = erlarg;
			ertest = fmax(epsabs, epsrel * fabs(reseps));
			if (*abserr <= ertest) goto final_result;
		}
		if (numrl2 == 1) noext = 1;
		if (*ier == 5) goto final_result;
		maxerr = iord[1];
		errmax = elist[maxerr];
		nrmax = 1;
		extrap = 0;
		small *= 0.5;
		erlarg = errsum;
	}
	if (last > limit) last = limit;

final_result:
	if (*abserr == oflow) goto sum_result;
	if (*ier + ierro != 0) {
		if (ierro == 3) *abserr += correc;
		if (*ier == 0) *ier = 3;
		if (*result == 0.0 || area == 0.0) {
			if (*abserr > errsum) goto sum_result;
			if (area == 0.0) goto decrement;
		}
		else if (*abserr / fabs(*result) > errsum / fabs(area)) {
			goto sum_result;
		}
	}
	if (!(ksgn == -1 && fmax(fabs(*result), fabs(area)) <= defabs * 0.01)) {
		if (0.01 > *result / area || *result / area > 100.0 || errsum > fabs(area))
			*ier = 6;
	}
	goto decrement;

sum_result:
	*result = 0.0;
	for (k = 1; k <= last; k++) *result += rlist[k];
	*abserr = errsum;

decrement:
	if (*ier > 2) (*ier)--;

finish_neval:
	if (rule == rule21) *neval = 42 * last - 21;
	else *neval = 30 * last - 15;
	if (inf == 2 && rule != rule21) *neval *= 2;

cleanup:
	*last_out = last;
	free(alist);
	free(blist);
	free(rlist);
	free(elist);
	free(iord);
}

void Rdqags(integr_fn f, void *ex, double *a, double *b,
            double *epsabs, double *epsrel,
            double *result, double *abserr, int *neval, int *ier,
            int *limit, int *lenw, int *last, int *iwork, double *work)
{
	(void)lenw;
	(void)iwork;
	(void)work;
	qp_fun F = {f, ex};
	qag_extrap(&F, rule21, 0.0, 0, *a, *b, fabs(*b - *a) * 0.375, *epsabs,
	           *epsrel, *limit, result, abserr, neval, ier, last);
}

void Rdqagi(integr_fn f, void *ex, double *bound, int *inf,
            double *epsabs, double *epsrel,
            double *result, double *abserr, int *neval, int *ier,
            int *limit, int *lenw, int *last, int *iwork, double *work)
{
	(void)lenw;
	(void)iwork;
	(void)work;
	qp_fun F = {f, ex};
	double boun = *bound;
	if (*inf == 2) boun = 0.0;
	qag_extrap(&F, qk15i, boun, *inf, 0.0, 1.0, 0.375, *epsabs, *epsrel,
	           *limit, result, abserr, neval, ier, last);
}
