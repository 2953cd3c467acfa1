// FP64 special functions for the per-profile scalar prologue, usable on the
// host and on the device.
//
// libprofit calls R's qgamma/pgamma/gammafn/beta and QUADPACK dqags/dqagi
// through utils.cpp:193-258 (epsabs = epsrel = 1e-4, limit = 100).  These are
// independent implementations of the same mathematics:
//  - Gamma(x): the C library / CUDA tgamma.
//  - Beta(a, b): Gamma(a) Gamma(b) / Gamma(a+b) below the Gamma overflow point,
//    log-Gamma form above it.
//  - P(a, x): Taylor series for x < a + 1, else 1 - Q with Q from the
//    Legendre continued fraction (modified Lentz).
//  - qgamma(p, a): median-type start, then Halley steps on P(a, x) - p inside a
//    shrinking bracket.
//  - digamma(x): recurrence to x >= 10 then the asymptotic Bernoulli series.
//  - QUADPACK dqagse / dqagie (Piessens, de Doncker-Kapenga, Ueberhuber,
//    Kahaner 1983): 21-point Gauss-Kronrod on finite ranges, 15-point on
//    (0, 1] for [a, inf) after x = a + (1 - t)/t, bisection of the interval
//    with the largest error and Wynn's epsilon extrapolation.  Nodes and
//    weights are the published Kronrod tables.  The same decisions are taken
//    as in the reference's integrator so lumtot agrees to rounding.
#pragma once

#include <cfloat>
#include <cmath>

#ifdef __CUDACC__
#define PF_HD __host__ __device__
#else
#define PF_HD
#endif

namespace pf {

PF_HD inline double pf_fmax(double a, double b) { return a > b ? a : b; }
PF_HD inline double pf_fmin(double a, double b) { return a < b ? a : b; }

PF_HD inline double gamma_fn(double x) { return tgamma(x); }

PF_HD inline double beta_fn(double a, double b)
{
	if (isnan(a) || isnan(b)) return a + b;
	if (a < 0 || b < 0) return NAN;
	if (a == 0 || b == 0) return INFINITY;
	if (isinf(a) || isinf(b)) return 0;
	if (a + b < 171.61447887182298) {
		return (1.0 / tgamma(a + b)) * (tgamma(a) * tgamma(b));
	}
	return exp(lgamma(a) + lgamma(b) - lgamma(a + b));
}

// log of x^a e^-x / Gamma(a)
PF_HD inline double gamma_log_kernel(double a, double x) { return a * log(x) - x - lgamma(a); }

PF_HD inline double gamma_p_series(double a, double x)
{
	double term = 1.0 / a, sum = term;
	for (int n = 1; n < 5000; n++) {
		term *= x / (a + n);
		sum += term;
		if (fabs(term) <= fabs(sum) * 1e-17) break;
	}
	return sum * exp(gamma_log_kernel(a, x));
}

PF_HD inline double gamma_q_cf(double a, double x)
{
	const double tiny = 1e-300;
	double b = x + 1.0 - a, c = 1.0 / tiny, d = 1.0 / b, h = d;
	for (int i = 1; i < 5000; i++) {
		double an = -i * (i - a);
		b += 2.0;
		d = an * d + b;
		if (fabs(d) < tiny) d = tiny;
		c = b + an / c;
		if (fabs(c) < tiny) c = tiny;
		d = 1.0 / d;
		double del = d * c;
		h *= del;
		if (fabs(del - 1.0) <= 1e-17) break;
	}
	return exp(gamma_log_kernel(a, x)) * h;
}

// Regularised lower incomplete gamma P(a, x), a > 0.
PF_HD inline double pgamma(double x, double a)
{
	if (!(x > 0)) return 0.0;
	if (isinf(x)) return 1.0;
	if (x < a + 1.0) return gamma_p_series(a, x);
	return 1.0 - gamma_q_cf(a, x);
}

// Inverse of P(a, .) at p in (0, 1).
PF_HD inline double qgamma(double p, double a)
{
	if (isnan(p) || isnan(a) || a <= 0 || p < 0 || p > 1) return NAN;
	if (p == 0) return 0.0;
	if (p == 1) return INFINITY;
	// Start: Wilson-Hilferty with a rational normal-quantile approximation
	// refined below by the gamma iteration itself; for small p the
	// leading term of the series, x ~ (p Gamma(a+1))^(1/a).
	double t = sqrt(-2.0 * log(p < 0.5 ? p : 1.0 - p));
	double z = t - (2.515517 + 0.802853 * t + 0.010328 * t * t) /
	               (1.0 + 1.432788 * t + 0.189269 * t * t + 0.001308 * t * t * t);
	if (p < 0.5) z = -z;
	double c = 1.0 / (9.0 * a);
	double w = 1.0 - c + z * sqrt(c);
	double x = a * w * w * w;
	double xs = exp((log(p) + lgamma(a + 1.0)) / a);
	if (!(x > 0) || x < xs) x = xs;

	double lo = 0.0, hi = INFINITY;
	double lga = lgamma(a);
	for (int it = 0; it < 300; it++) {
		double f = pgamma(x, a) - p;
		if (f == 0) return x;
		if (f < 0) lo = x;
		else hi = x;
		double dens = exp((a - 1.0) * log(x) - x - lga);
		double xn = NAN;
		if (dens > 0 && isfinite(dens)) {
			double u = f / dens;
			double corr = 1.0 - 0.5 * u * ((a - 1.0) / x - 1.0);
			xn = (corr > 0.5 && corr < 2.0) ? x - u / corr : x - u;
		}
		if (!(xn > lo && xn < hi)) xn = isinf(hi) ? 2.0 * x + 1.0 : 0.5 * (lo + hi);
		if (fabs(xn - x) <= 4.0 * DBL_EPSILON * fabs(xn)) return xn;
		x = xn;
	}
	return x;
}

// digamma(x) for x > 0; NaN for x <= 0 or NaN (the recurrence below would
// never reach 10 from -inf, and no caller needs the negative axis).
PF_HD inline double digamma(double x)
{
	if (!(x > 0.0)) return NAN;
	double r = 0;
	while (x < 10.0) {
		r -= 1.0 / x;
		x += 1.0;
	}
	double f = 1.0 / (x * x);
	// B2k / (2k) for k = 1..6
	double t = f * (-1.0 / 12 + f * (1.0 / 120 + f * (-1.0 / 252 + f * (1.0 / 240 + f * (-1.0 / 132 + f * (691.0 / 32760))))));
	return r + log(x) - 0.5 / x + t;
}

// ------------------------------------------------------------------------
// QUADPACK restatement
// ------------------------------------------------------------------------

struct GK21 {
	PF_HD static double xgk(int i)
	{
		const double v[11] = {
			0.995657163025808080735527280689003, 0.973906528517171720077964012084452,
			0.930157491355708226001207180059508, 0.865063366688984510732096688423493,
			0.780817726586416897063717578345042, 0.679409568299024406234327365114874,
			0.562757134668604683339000099272694, 0.433395394129247190799265943165784,
			0.294392862701460198131126603103866, 0.148874338981631210884826001129720, 0.0};
		return v[i];
	}
	PF_HD static double wgk(int i)
	{
		const double v[11] = {
			0.011694638867371874278064396062192, 0.032558162307964727478818972459390,
			0.054755896574351996031381300244580, 0.075039674810919952767043140916190,
			0.093125454583697605535065465083366, 0.109387158802297641899210590325805,
			0.123491976262065851077600525452925, 0.134709217311473325928054001771707,
			0.142775938577060080797094273138717, 0.147739104901338491374841515972068,
			0.149445554002916905664936468389821};
		return v[i];
	}
	PF_HD static double wg(int i)
	{
		const double v[5] = {0.066671344308688137593568809893332, 0.149451349150580593145776339657697,
		                     0.219086362515982043995534934228163, 0.269266719309996355091226921569469,
		                     0.295524224714752870173892994651338};
		return v[i];
	}
};

struct GK15 {
	PF_HD static double xgk(int i)
	{
		const double v[8] = {0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
		                     0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
		                     0.586087235467691130294144845693013, 0.405845151377397166906606412076961,
		                     0.207784955007898467600689403773245, 0.0};
		return v[i];
	}
	PF_HD static double wgk(int i)
	{
		const double v[8] = {0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
		                     0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
		                     0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
		                     0.204432940075298892414161999234649, 0.209482141084727828012999174891714};
		return v[i];
	}
	PF_HD static double wg(int i)
	{
		const double v[8] = {0.0, 0.129484966168869693270611432679082, 0.0, 0.279705391489276667901467771423780,
		                     0.0, 0.381830050505118944950369775488975, 0.0, 0.417959183673469387755102040816327};
		return v[i];
	}
};

struct QuadRule {
	double result, abserr, resabs, resasc;
};

PF_HD inline void gk_error(QuadRule &q, double resk, double resg, double hlgth)
{
	const double epmach = DBL_EPSILON, uflow = DBL_MIN;
	q.abserr = fabs((resk - resg) * hlgth);
	if (q.resasc != 0.0 && q.abserr != 0.0) {
		double r = pow(200.0 * q.abserr / q.resasc, 1.5);
		q.abserr = q.resasc * (r < 1.0 ? r : 1.0);
	}
	if (q.resabs > uflow / (50.0 * epmach)) q.abserr = pf_fmax(epmach * 50.0 * q.resabs, q.abserr);
}

// 21-point Kronrod rule with embedded 10-point Gauss rule on [a, b].
template <class F>
PF_HD QuadRule gk21(const F &f, double a, double b)
{
	QuadRule q;
	double fv1[10], fv2[10];
	double centr = 0.5 * (a + b), hlgth = 0.5 * (b - a), dhlgth = fabs(hlgth);
	double resg = 0.0, fc = f(centr);
	double resk = GK21::wgk(10) * fc;
	q.resabs = fabs(resk);
	for (int j = 0; j < 5; j++) {
		int k = 2 * j + 1;
		double absc = hlgth * GK21::xgk(k);
		double f1 = f(centr - absc), f2 = f(centr + absc);
		fv1[k] = f1;
		fv2[k] = f2;
		resg += GK21::wg(j) * (f1 + f2);
		resk += GK21::wgk(k) * (f1 + f2);
		q.resabs += GK21::wgk(k) * (fabs(f1) + fabs(f2));
	}
	for (int j = 0; j < 5; j++) {
		int k = 2 * j;
		double absc = hlgth * GK21::xgk(k);
		double f1 = f(centr - absc), f2 = f(centr + absc);
		fv1[k] = f1;
		fv2[k] = f2;
		resk += GK21::wgk(k) * (f1 + f2);
		q.resabs += GK21::wgk(k) * (fabs(f1) + fabs(f2));
	}
	double reskh = resk * 0.5;
	q.resasc = GK21::wgk(10) * fabs(fc - reskh);
	for (int j = 0; j < 10; j++) q.resasc += GK21::wgk(j) * (fabs(fv1[j] - reskh) + fabs(fv2[j] - reskh));
	q.result = resk * hlgth;
	q.resabs *= dhlgth;
	q.resasc *= dhlgth;
	gk_error(q, resk, resg, hlgth);
	return q;
}

// 15-point Kronrod rule on the transformed sub-range [a, b] of (0, 1] for
// the integral of f over [boun, inf).
template <class F>
PF_HD QuadRule gk15_semi_infinite(const F &f, double boun, double a, double b)
{
	QuadRule q;
	double fv1[7], fv2[7];
	double centr = 0.5 * (a + b), hlgth = 0.5 * (b - a);
	double fc = (f(boun + (1.0 - centr) / centr) / centr) / centr;
	double resg = GK15::wg(7) * fc, resk = GK15::wgk(7) * fc;
	q.resabs = fabs(resk);
	for (int j = 0; j < 7; j++) {
		double absc = hlgth * GK15::xgk(j);
		double a1 = centr - absc, a2 = centr + absc;
		double f1 = f(boun + (1.0 - a1) / a1), f2 = f(boun + (1.0 - a2) / a2);
		f1 = (f1 / a1) / a1;
		f2 = (f2 / a2) / a2;
		fv1[j] = f1;
		fv2[j] = f2;
		resg += GK15::wg(j) * (f1 + f2);
		resk += GK15::wgk(j) * (f1 + f2);
		q.resabs += GK15::wgk(j) * (fabs(f1) + fabs(f2));
	}
	double reskh = resk * 0.5;
	q.resasc = GK15::wgk(7) * fabs(fc - reskh);
	for (int j = 0; j < 7; j++) q.resasc += GK15::wgk(j) * (fabs(fv1[j] - reskh) + fabs(fv2[j] - reskh));
	q.result = resk * hlgth;
	q.resasc *= hlgth;
	q.resabs *= hlgth;
	gk_error(q, resk, resg, hlgth);
	return q;
}

// Adaptive integrator state, 1-based arrays as in the published algorithm.
struct QagWork {
	static const int LIMIT = 100;
	double alist[LIMIT + 1], blist[LIMIT + 1], rlist[LIMIT + 1], elist[LIMIT + 1];
	int iord[LIMIT + 1];
	double epstab[53], res3la[4];
};

PF_HD inline void qag_sort(int limit, int last, int &maxerr, double &ermax, const double *elist, int *iord, int &nrmax)
{
	if (last <= 2) {
		iord[1] = 1;
		iord[2] = 2;
		maxerr = iord[nrmax];
		ermax = elist[maxerr];
		return;
	}
	double errmax = elist[maxerr];
	if (nrmax != 1) {
		int ido = nrmax - 1;
		for (int i = 1; i <= ido; i++) {
			int isucc = iord[nrmax - 1];
			if (errmax <= elist[isucc]) break;
			iord[nrmax] = isucc;
			nrmax--;
		}
	}
	int jupbn = last;
	if (last > limit / 2 + 2) jupbn = limit + 3 - last;
	double errmin = elist[last];
	int jbnd = jupbn - 1, ibeg = nrmax + 1;
	int i = ibeg;
	bool found = false;
	for (; i <= jbnd; i++) {
		int isucc = iord[i];
		if (errmax >= elist[isucc]) {
			found = true;
			break;
		}
		iord[i - 1] = isucc;
	}
	if (!found) {
		iord[jbnd] = maxerr;
		iord[jupbn] = last;
	}
	else {
		iord[i - 1] = maxerr;
		int k = jbnd;
		bool placed = false;
		for (int j = i; j <= jbnd; j++) {
			int isucc = iord[k];
			if (errmin < elist[isucc]) {
				iord[k + 1] = last;
				placed = true;
				break;
			}
			iord[k + 1] = isucc;
			k--;
		}
		if (!placed) iord[i] = last;
	}
	maxerr = iord[nrmax];
	ermax = elist[maxerr];
}

// Wynn epsilon table step (1-based epstab, res3la).
PF_HD inline void qag_extrapolate(int &n, double *epstab, double &result, double &abserr, double *res3la, int &nres)
{
	const double epmach = DBL_EPSILON, oflow = DBL_MAX;
	const int limexp = 50;
	nres++;
	abserr = oflow;
	result = epstab[n];
	if (n < 3) {
		abserr = pf_fmax(abserr, 5.0 * epmach * fabs(result));
		return;
	}
	epstab[n + 2] = epstab[n];
	int newelm = (n - 1) / 2;
	epstab[n] = oflow;
	int num = n, k1 = n;
	for (int i = 1; i <= newelm; i++) {
		int k2 = k1 - 1, k3 = k1 - 2;
		double res = epstab[k1 + 2];
		double e0 = epstab[k3], e1 = epstab[k2], e2 = res;
		double e1abs = fabs(e1);
		double delta2 = e2 - e1, err2 = fabs(delta2);
		double tol2 = pf_fmax(fabs(e2), e1abs) * epmach;
		double delta3 = e1 - e0, err3 = fabs(delta3);
		double tol3 = pf_fmax(e1abs, fabs(e0)) * epmach;
		if (err2 <= tol2 && err3 <= tol3) {
			result = res;
			abserr = err2 + err3;
			abserr = pf_fmax(abserr, 5.0 * epmach * fabs(result));
			return;
		}
		double e3 = epstab[k1];
		epstab[k1] = e1;
		double delta1 = e1 - e3, err1 = fabs(delta1);
		double tol1 = pf_fmax(e1abs, fabs(e3)) * epmach;
		if (err1 <= tol1 || err2 <= tol2 || err3 <= tol3) {
			n = i + i - 1;
			break;
		}
		double ss = 1.0 / delta1 + 1.0 / delta2 - 1.0 / delta3;
		double epsinf = fabs(ss * e1);
		if (!(epsinf > 1e-4)) {
			n = i + i - 1;
			break;
		}
		res = e1 + 1.0 / ss;
		epstab[k1] = res;
		k1 -= 2;
		double error = err2 + fabs(res - e2) + err3;
		if (error > abserr) continue;
		abserr = error;
		result = res;
	}
	if (n == limexp) n = (limexp / 2) * 2 - 1;
	int ib = (num % 2 == 0) ? 2 : 1;
	int ie = newelm + 1;
	for (int i = 1; i <= ie; i++) {
		epstab[ib] = epstab[ib + 2];
		ib += 2;
	}
	if (num != n) {
		int indx = num - n + 1;
		for (int i = 1; i <= n; i++) epstab[i] = epstab[indx++];
	}
	if (nres < 4) {
		res3la[nres] = result;
		abserr = oflow;
	}
	else {
		abserr = fabs(result - res3la[3]) + fabs(result - res3la[2]) + fabs(result - res3la[1]);
		res3la[1] = res3la[2];
		res3la[2] = res3la[3];
		res3la[3] = result;
	}
	abserr = pf_fmax(abserr, 5.0 * epmach * fabs(result));
}

// Adaptive bisection with extrapolation.  `rule(a, b)` returns a QuadRule
// (result, abserr, resabs = integral of |f|, resasc) on [a, b].
template <class Rule>
PF_HD double qag_adaptive(const Rule &rule, double a, double b, double small0, QagWork &w)
{
	const double epmach = DBL_EPSILON, uflow = DBL_MIN, oflow = DBL_MAX;
	const double epsabs = 1e-4, epsrel = 1e-4;
	const int limit = QagWork::LIMIT;
	double *alist = w.alist, *blist = w.blist, *rlist = w.rlist, *elist = w.elist;
	int *iord = w.iord;
	int ier = 0, ierro = 0, last;
	alist[1] = a;
	blist[1] = b;
	QuadRule q0 = rule(a, b);
	double result = q0.result, abserr = q0.abserr, defabs = q0.resabs, resabs0 = q0.resasc;
	double dres = fabs(result);
	double errbnd = pf_fmax(epsabs, epsrel * dres);
	last = 1;
	rlist[1] = result;
	elist[1] = abserr;
	iord[1] = 1;
	if (abserr <= 100.0 * epmach * defabs && abserr > errbnd) ier = 2;
	if (ier != 0 || (abserr <= errbnd && abserr != resabs0) || abserr == 0.0) return result;

	w.epstab[1] = result;
	double errmax = abserr, area = result, errsum = abserr;
	int maxerr = 1, nrmax = 1, nres = 0, numrl2 = 2, ktmin = 0;
	bool extrap = false, noext = false;
	int iroff1 = 0, iroff2 = 0, iroff3 = 0;
	int ksgn = (dres >= (1.0 - 50.0 * epmach) * defabs) ? 1 : -1;
	double small = 0, erlarg = 0, ertest = 0, correc = 0, erlast, area12, erro12;
	abserr = oflow;
	bool summed = false;

	for (last = 2; last <= limit; last++) {
		double a1 = alist[maxerr], b1 = 0.5 * (alist[maxerr] + blist[maxerr]);
		double a2 = b1, b2 = blist[maxerr];
		erlast = errmax;
		QuadRule q1 = rule(a1, b1), q2 = rule(a2, b2);
		area12 = q1.result + q2.result;
		erro12 = q1.abserr + q2.abserr;
		errsum = errsum + erro12 - errmax;
		area = area + area12 - rlist[maxerr];
		if (!(q1.resasc == q1.abserr || q2.resasc == q2.abserr)) {
			if (fabs(rlist[maxerr] - area12) <= 1e-5 * fabs(area12) && erro12 >= 0.99 * errmax) {
				if (extrap) iroff2++;
				else iroff1++;
			}
			if (last > 10 && erro12 > errmax) iroff3++;
		}
		rlist[maxerr] = q1.result;
		rlist[last] = q2.result;
		errbnd = pf_fmax(epsabs, epsrel * fabs(area));
		if (iroff1 + iroff2 >= 10 || iroff3 >= 20) ier = 2;
		if (iroff2 >= 5) ierro = 3;
		if (last == limit) ier = 1;
		if (pf_fmax(fabs(a1), fabs(b2)) <= (1.0 + 100.0 * epmach) * (fabs(a2) + 1000.0 * uflow)) ier = 4;
		if (q2.abserr > q1.abserr) {
			alist[maxerr] = a2;
			alist[last] = a1;
			blist[last] = b1;
			rlist[maxerr] = q2.result;
			rlist[last] = q1.result;
			elist[maxerr] = q2.abserr;
			elist[last] = q1.abserr;
		}
		else {
			alist[last] = a2;
			blist[maxerr] = b1;
			blist[last] = b2;
			elist[maxerr] = q1.abserr;
			elist[last] = q2.abserr;
		}
		qag_sort(limit, last, maxerr, errmax, elist, iord, nrmax);
		if (errsum <= errbnd) {
			summed = true;
			break;
		}
		if (ier != 0) break;
		if (last == 2) {
			small = small0;
			erlarg = errsum;
			ertest = errbnd;
			w.epstab[2] = area;
			continue;
		}
		if (noext) continue;
		erlarg -= erlast;
		if (fabs(b1 - a1) > small) erlarg += erro12;
		if (!extrap) {
			if (fabs(blist[maxerr] - alist[maxerr]) > small) continue;
			extrap = true;
			nrmax = 2;
		}
		if (ierro != 3 && erlarg > ertest) {
			bool jump = false;
			int jupbnd = last;
			if (last > 2 + limit / 2) jupbnd = limit + 3 - last;
			for (int k = nrmax; k <= jupbnd; k++) {
				maxerr = iord[nrmax];
				errmax = elist[maxerr];
				if (fabs(blist[maxerr] - alist[maxerr]) > small) {
					jump = true;
					break;
				}
				nrmax++;
			}
			if (jump) continue;
		}
		numrl2++;
		w.epstab[numrl2] = area;
		double reseps, abseps;
		qag_extrapolate(numrl2, w.epstab, reseps, abseps, w.res3la, nres);
		ktmin++;
		if (ktmin > 5 && abserr < 1e-3 * errsum) ier = 5;
		if (abseps < abserr) {
			ktmin = 0;
			abserr = abseps;
			result = reseps;
			correc = erlarg;
			ertest = pf_fmax(epsabs, epsrel * fabs(reseps));
			if (abserr <= ertest) break;
		}
		if (numrl2 == 1) noext = true;
		if (ier == 5) break;
		maxerr = iord[1];
		errmax = elist[maxerr];
		nrmax = 1;
		extrap = false;
		small *= 0.5;
		erlarg = errsum;
	}
	if (last > limit) last = limit;

	if (!summed) {
		// final result selection of the published algorithm
		if (abserr == oflow) {
			summed = true;
		}
		else if (ier + ierro != 0) {
			if (ierro == 3) abserr += correc;
			if (result == 0.0 || area == 0.0) {
				if (abserr > errsum) summed = true;
				else if (area == 0.0) return result;
			}
			else if (abserr / fabs(result) > errsum / fabs(area)) {
				summed = true;
			}
		}
	}
	if (summed) {
		result = 0.0;
		for (int k = 1; k <= last; k++) result += rlist[k];
	}
	(void)ksgn;
	return result;
}

template <class F>
struct Rule21 {
	const F &f;
	PF_HD QuadRule operator()(double a, double b) const { return gk21(f, a, b); }
};

template <class F>
struct Rule15Inf {
	const F &f;
	double boun;
	PF_HD QuadRule operator()(double a, double b) const { return gk15_semi_infinite(f, boun, a, b); }
};

// integral of f over [a, b]  (libprofit integrate_qags)
template <class F>
PF_HD double integrate_qags(const F &f, double a, double b)
{
	QagWork w;
	Rule21<F> rule{f};
	return qag_adaptive(rule, a, b, fabs(b - a) * 0.375, w);
}

// integral of f over [a, inf)  (libprofit integrate_qagi)
template <class F>
PF_HD double integrate_qagi(const F &f, double a)
{
	QagWork w;
	Rule15Inf<F> rule{f, a};
	return qag_adaptive(rule, 0.0, 1.0, 0.375, w);
}

}  // namespace pf
