/*
 * ORACLE (test infrastructure only).  Plain-C restatement of the model-image
 * hot path of libprofit 1.9.3 (src/libprofit/src/profit/) and of ProFit's
 * "norm" likelihood (R/profitLikeModel.R:263-276).  It is the checker for the
 * CUDA library, never part of it.  Each function names the reference lines
 * it restates; arithmetic order follows the reference wherever the result
 * depends on it, so on the same libm this file reproduces the compiled
 * reference bit for bit (tests pin that), and it adds what the reference
 * cannot report: a per-pixel log of subsampling decisions.
 *
 * Differences from the reference, on purpose:
 *  - derived per-profile values (adjusted acc, resolution, rscale_switch,
 *    rscale_max) live in separate fields and are recomputed from the user's
 *    parameters on every evaluation.  libprofit overwrites the user's fields
 *    in RadialProfile::initial_calculations (radial.cpp:164-183), so a second
 *    evaluate() of the same profit::Model compounds acc; ProFit never sees
 *    that because R_profit_make_model builds a fresh Model per call
 *    (r_profit.cpp:575).  This file behaves like the fresh-Model case.
 *  - the brute-force convolution computes only the outputs that survive the
 *    crop (model.cpp:307-324); libprofit computes the whole padded image.
 *  - the FFT convolver is restated as the exact linear convolution it
 *    computes (convolve.cpp:283-312 with the no-wrap padding of
 *    convolve.cpp:245-261): same kernel placement and crop offset, summed
 *    directly in FP64.  FFTW is not available to build the reference's.
 *  - masks (calcregion) are not supported yet.
 */
#define _GNU_SOURCE
#include "profit_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "Rmath.h"
#include "R_ext/Applic.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

static __thread char g_err[512];

static int fail(const char *fmt, const char *arg)
{
	snprintf(g_err, sizeof(g_err), fmt, arg ? arg : "");
	return -1;
}

const char *pfo_last_error(void) { return g_err; }

/* ------------------------------------------------------------------------- */
/* Special functions as libprofit calls them (utils.cpp:193-207)             */
/* ------------------------------------------------------------------------- */

static double u_qgamma(double p, double shape) { return Rf_qgamma(p, shape, 1, 1, 0); }
static double u_pgamma(double q, double shape) { return Rf_pgamma(q, shape, 1, 1, 0); }
static double u_gammafn(double x) { return Rf_gammafn(x); }
static double u_beta(double a, double b) { return Rf_beta(a, b); }

typedef double (*radial_fn)(double r, const void *ctx);
struct integr_ctx {
	radial_fn f;
	const void *ctx;
};

static void integr_tramp(double *x, int n, void *ex)
{
	struct integr_ctx *c = (struct integr_ctx *)ex;
	for (int i = 0; i < n; i++) x[i] = c->f(x[i], c->ctx);
}

/* utils.cpp:209-258 (R branch): epsabs = epsrel = 1e-4, limit 100 */
static double integrate_qag(radial_fn f, const void *ctx, double a, double b, int to_inf)
{
	int neval, ier, last, limit = 100, lenw = 4 * limit;
	int iwork[100];
	double work[400];
	double result, abserr, epsabs = 1e-4, epsrel = 1e-4;
	struct integr_ctx c = {f, ctx};
	if (to_inf) {
		int inf = 1;
		Rdqagi(integr_tramp, &c, &a, &inf, &epsabs, &epsrel, &result, &abserr, &neval,
		       &ier, &limit, &lenw, &last, iwork, work);
	}
	else {
		Rdqags(integr_tramp, &c, &a, &b, &epsabs, &epsrel, &result, &abserr, &neval,
		       &ier, &limit, &lenw, &last, iwork, work);
	}
	return result;
}

/* utils.cpp:101-103 with the default tolerance of utils.h:46 */
static int almost_equals(double x, double y) { return fabs(x - y) < 1e-10; }

/* ------------------------------------------------------------------------- */
/* Profiles                                                                  */
/* ------------------------------------------------------------------------- */

enum kind { K_SERSIC, K_MOFFAT, K_FERRER, K_CORESERSIC, K_KING, K_BROKENEXP, K_SKY, K_PSF, K_NULL };

/* Sersic r_factor specialisations of sersic.cpp:78-189 */
enum rf_spec { RF_GENERAL, RF_POINTFIVE, RF_ONE, RF_TWO, RF_THREE, RF_FOUR, RF_EIGHT, RF_SIXTEEN };

#define MAX_LEVELS 16

typedef struct {
	int kind;
	char name[16];
	int convolve;
	/* radial user parameters, defaults of radial.cpp:724-752 */
	double xcen, ycen, mag, ang, axrat, box;
	int rough, adjust, force_cpu;
	double acc, rscale_switch, rscale_max;
	unsigned resolution, max_recursions;
	/* profile-specific user parameters */
	double re, nser;
	int rescale_flux;
	double fwhm, con;
	double rout, a, b;
	double rb, rc, rt, h1, h2;
	double bg;
	/* derived at evaluation time */
	double d_acc, d_rscale_switch, d_rscale_max;
	unsigned d_resolution;
	double rscale, ie, bn, rescale_factor, cos_ang, sin_ang, cos_q, sin_q;
	double cx, cy, magzero, lumtot, flux_scale;
	int boxy, spec;
	double sky_bg;
	/* instrumentation */
	int *decisions;
	size_t n_decisions;
	long level_counts[MAX_LEVELS];
	long n_evals; /* evaluate_at calls of the last evaluation */
} profile_t;

struct pfo_model {
	unsigned width, height;
	double magzero, scale_x, scale_y, psf_scale_x, psf_scale_y;
	unsigned finesampling;
	int return_finesampled;
	int conv_kind; /* 0 brute, 1 fft, 2 null */
	double *psf;
	unsigned psf_w, psf_h;
	int threads;
	profile_t *profiles;
	int n_profiles;
	double img_scale_x, img_scale_y;
};

static void radial_defaults(profile_t *p)
{
	p->xcen = 0;
	p->ycen = 0;
	p->mag = 15;
	p->ang = 0;
	p->axrat = 1;
	p->box = 0;
	p->rough = 0;
	p->acc = 0.1;
	p->rscale_switch = 1;
	p->resolution = 9;
	p->max_recursions = 2;
	p->adjust = 1;
	p->rscale_max = 0;
	p->force_cpu = 0;
}

/* Parameter registry: which names each profile accepts (register_parameter calls). */
typedef struct {
	const char *name;
	char type; /* 'd', 'u', 'b' */
	size_t off;
} param_desc;

#define PD(n, t) {#n, t, offsetof(profile_t, n)}
static const param_desc radial_params[] = {
	PD(xcen, 'd'), PD(ycen, 'd'), PD(mag, 'd'), PD(ang, 'd'), PD(axrat, 'd'), PD(box, 'd'),
	PD(rough, 'b'), PD(adjust, 'b'), PD(force_cpu, 'b'), PD(acc, 'd'),
	PD(rscale_switch, 'd'), PD(rscale_max, 'd'), PD(max_recursions, 'u'),
	PD(resolution, 'u'), PD(convolve, 'b'), {NULL, 0, 0}};
static const param_desc sersic_params[] = {PD(re, 'd'), PD(nser, 'd'), PD(rescale_flux, 'b'), {NULL, 0, 0}};
static const param_desc moffat_params[] = {PD(fwhm, 'd'), PD(con, 'd'), {NULL, 0, 0}};
static const param_desc ferrer_params[] = {PD(rout, 'd'), PD(a, 'd'), PD(b, 'd'), {NULL, 0, 0}};
static const param_desc coresersic_params[] = {PD(re, 'd'), PD(rb, 'd'), PD(nser, 'd'), PD(a, 'd'), PD(b, 'd'), {NULL, 0, 0}};
static const param_desc king_params[] = {PD(rc, 'd'), PD(rt, 'd'), PD(a, 'd'), {NULL, 0, 0}};
static const param_desc brokenexp_params[] = {PD(h1, 'd'), PD(h2, 'd'), PD(rb, 'd'), PD(a, 'd'), {NULL, 0, 0}};
static const param_desc sky_params[] = {PD(bg, 'd'), PD(convolve, 'b'), {NULL, 0, 0}};
static const param_desc psf_params[] = {PD(xcen, 'd'), PD(ycen, 'd'), PD(mag, 'd'), PD(convolve, 'b'), {NULL, 0, 0}};
static const param_desc null_params[] = {PD(convolve, 'b'), {NULL, 0, 0}};

static const param_desc *find_param(const profile_t *p, const char *name)
{
	const param_desc *lists[2] = {NULL, NULL};
	switch (p->kind) {
	case K_SERSIC: lists[0] = radial_params; lists[1] = sersic_params; break;
	case K_MOFFAT: lists[0] = radial_params; lists[1] = moffat_params; break;
	case K_FERRER: lists[0] = radial_params; lists[1] = ferrer_params; break;
	case K_CORESERSIC: lists[0] = radial_params; lists[1] = coresersic_params; break;
	case K_KING: lists[0] = radial_params; lists[1] = king_params; break;
	case K_BROKENEXP: lists[0] = radial_params; lists[1] = brokenexp_params; break;
	case K_SKY: lists[0] = sky_params; break;
	case K_PSF: lists[0] = psf_params; break;
	default: lists[0] = null_params; break;
	}
	for (int l = 0; l < 2; l++) {
		if (!lists[l]) continue;
		for (const param_desc *d = lists[l]; d->name; d++) {
			if (strcmp(d->name, name) == 0) return d;
		}
	}
	return NULL;
}

static int is_radial(const profile_t *p) { return p->kind <= K_BROKENEXP; }

static double boxy_r(const profile_t *p, double x, double y)
{
	/* radial.h:93-102 */
	if (p->box == 0) return sqrt(x * x + y * y);
	double box_plus_2 = p->box + 2.;
	return pow(pow(fabs(x), box_plus_2) + pow(fabs(y), box_plus_2), 1. / box_plus_2);
}

static double sersic_eval(const profile_t *p, double x, double y)
{
	/* sersic.cpp:142-205 */
	double B = p->box + 2;
	double base, invexp, rf;
	if (p->boxy) {
		base = pow(fabs(x / p->re), B) + pow(fabs(y / p->re), B);
		invexp = p->nser * B;
		switch (p->spec) {
		case RF_POINTFIVE: rf = base * base; break;
		case RF_ONE: rf = base; break;
		case RF_TWO: rf = sqrt(base); break;
		case RF_THREE: rf = cbrt(base); break;
		case RF_FOUR: rf = sqrt(sqrt(base)); break;
		case RF_EIGHT: rf = sqrt(sqrt(sqrt(base))); break;
		case RF_SIXTEEN: rf = sqrt(sqrt(sqrt(sqrt(base)))); break;
		default: rf = pow(base, 1 / invexp); break;
		}
	}
	else {
		base = (x * x + y * y) / (p->re * p->re);
		invexp = p->nser;
		switch (p->spec) {
		case RF_POINTFIVE: rf = base; break;
		case RF_ONE: rf = sqrt(base); break;
		case RF_TWO: rf = sqrt(sqrt(base)); break;
		case RF_THREE: rf = cbrt(sqrt(base)); break;
		case RF_FOUR: rf = sqrt(sqrt(sqrt(base))); break;
		case RF_EIGHT: rf = sqrt(sqrt(sqrt(sqrt(base)))); break;
		case RF_SIXTEEN: rf = sqrt(sqrt(sqrt(sqrt(sqrt(base))))); break;
		default: rf = pow(sqrt(base), 1 / invexp); break;
		}
	}
	return exp(-p->bn * (rf - 1));
}

static double moffat_eval(const profile_t *p, double x, double y)
{
	/* moffat.cpp:52-58 */
	double r = boxy_r(p, x, y);
	double r_factor = r / p->rscale;
	return pow(1 + r_factor * r_factor, -p->con);
}

static double ferrer_eval(const profile_t *p, double x, double y)
{
	/* ferrer.cpp:50-60 */
	double r = boxy_r(p, x, y);
	double r_factor = r / p->rscale;
	if (r_factor < 1) return pow(1 - pow(r_factor, 2 - p->b), p->a);
	return 0;
}

static double coresersic_radial(double r, const profile_t *p)
{
	/* coresersic.cpp:51-59 */
	return pow(1 + pow(r / p->rb, -p->a), p->b / p->a) *
	       exp(-p->bn * pow((pow(r, p->a) + pow(p->rb, p->a)) / pow(p->re, p->a), 1 / (p->nser * p->a)));
}

static double king_radial(double r, const profile_t *p)
{
	/* king.cpp:51-59 */
	if (r < p->rt) {
		return pow(1 / pow(1 + pow(r / p->rc, 2), 1 / p->a) - 1 / pow(1 + pow(p->rt / p->rc, 2), 1 / p->a), p->a);
	}
	return 0;
}

static double brokenexp_radial(double r, const profile_t *p)
{
	/* brokenexponential.cpp:38-77 */
	double base = r - p->rb;
	double expo = 1 / p->h1 - 1 / p->h2;
	if (p->a * base < 40) base = log(1 + exp(p->a * base)) / p->a;
	return exp(-r / p->h1 + expo * base);
}

static double evaluate_at(const profile_t *p, double x, double y)
{
	switch (p->kind) {
	case K_SERSIC: return sersic_eval(p, x, y);
	case K_MOFFAT: return moffat_eval(p, x, y);
	case K_FERRER: return ferrer_eval(p, x, y);
	case K_CORESERSIC: return coresersic_radial(boxy_r(p, x, y), p);
	case K_KING: return king_radial(boxy_r(p, x, y), p);
	case K_BROKENEXP: return brokenexp_radial(boxy_r(p, x, y), p);
	default: return 0;
	}
}

static double integrand_coresersic(double r, const void *c) { return r * coresersic_radial(r, (const profile_t *)c); }
static double integrand_king(double r, const void *c) { return r * king_radial(r, (const profile_t *)c); }
static double integrand_brokenexp(double r, const void *c) { return r * brokenexp_radial(r, (const profile_t *)c); }

static double sersic_fluxfrac(const profile_t *p, double fraction)
{
	/* sersic.cpp:257-260 */
	double ratio = u_qgamma(fraction, 2 * p->nser) / p->bn;
	return p->re * pow(ratio, p->nser);
}

static double moffat_fluxfrac(const profile_t *p, double fraction)
{
	/* moffat.cpp:73-75 */
	return p->rscale * sqrt(pow(1 - fraction, 1 / (1 - p->con)) - 1);
}

static double get_rscale(const profile_t *p)
{
	switch (p->kind) {
	case K_SERSIC: return p->re;                                            /* sersic.cpp:327-329 */
	case K_MOFFAT: return p->fwhm / (2 * sqrt(pow(2, (1 / p->con)) - 1));  /* moffat.cpp:81-83 */
	case K_FERRER: return p->rout;                                          /* ferrer.cpp:111-113 */
	case K_CORESERSIC: return p->re;                                        /* coresersic.cpp:127-129 */
	case K_KING: return p->rt;                                              /* king.cpp:107-109 */
	case K_BROKENEXP: return p->h1 * 4;                                     /* brokenexponential.cpp:137-139 */
	default: return 0;
	}
}

static double get_lumtot(profile_t *p)
{
	switch (p->kind) {
	case K_SERSIC: {
		/* sersic.cpp:283-289 */
		double g_factor = u_gammafn(2 * p->nser);
		return pow(p->re, 2) * 2 * M_PI * p->nser * g_factor * exp(p->bn) / pow(p->bn, 2 * p->nser);
	}
	case K_MOFFAT:
		/* moffat.cpp:77-79 */
		return pow(p->rscale, 2) * M_PI / (p->con - 1);
	case K_FERRER: {
		/* ferrer.cpp:78-101 */
		double g_factor = p->a * u_beta(p->a, 1 + 2 / (2 - p->b));
		return pow(p->rout, 2) * M_PI * g_factor;
	}
	case K_CORESERSIC:
		/* coresersic.cpp:92-104 */
		return 2 * M_PI * integrate_qag(integrand_coresersic, p, 0, 0, 1);
	case K_KING:
		/* king.cpp:87-97 */
		return 2 * M_PI * integrate_qag(integrand_king, p, 0, p->rt, 0);
	case K_BROKENEXP:
		/* brokenexponential.cpp:115-127 */
		return 2 * M_PI * integrate_qag(integrand_brokenexp, p, 0, 0, 1);
	default:
		return 0;
	}
}

static double adjust_rscale_switch(const profile_t *p)
{
	switch (p->kind) {
	case K_SERSIC: {
		/* sersic.cpp:262-273 */
		double rs = ceil(sersic_fluxfrac(p, 1. - p->nser * p->nser / 2e3));
		rs = fmax(fmin(rs, 20.), 2.);
		return rs / p->re;
	}
	case K_MOFFAT: {
		/* moffat.cpp:89-92 */
		double rs = fmax(moffat_fluxfrac(p, 0.9999), 1.823 * p->fwhm);
		return fmax(fmin(rs, 20.), 2.) / p->rscale;
	}
	case K_FERRER: return 0.5;     /* ferrer.cpp:103-105 */
	case K_CORESERSIC: return 1;   /* coresersic.cpp:119-121 */
	case K_KING: return 0.5;       /* king.cpp:99-101 */
	case K_BROKENEXP: return 1;    /* brokenexponential.cpp:129-131 */
	default: return 1;
	}
}

static double adjust_rscale_max(const profile_t *p)
{
	switch (p->kind) {
	case K_SERSIC: return ceil(fmax(sersic_fluxfrac(p, 0.9999), 2.) / p->re);        /* sersic.cpp:275-277 */
	case K_MOFFAT: return ceil(fmax(moffat_fluxfrac(p, 0.9999), 2.) / p->rscale);    /* moffat.cpp:94-96 */
	case K_FERRER: return 1;          /* ferrer.cpp:107-109 */
	case K_CORESERSIC: return 100;    /* coresersic.cpp:123-125 */
	case K_KING: return 1.5;          /* king.cpp:103-105 */
	case K_BROKENEXP: return 100;     /* brokenexponential.cpp:133-135 */
	default: return 0;
	}
}

static double adjust_acc(const profile_t *p, double acc)
{
	switch (p->kind) {
	case K_SERSIC:
		/* sersic.cpp:279-282 */
		acc /= sqrt(p->nser);
		return fmax(0.1, acc) / p->axrat;
	case K_MOFFAT:
		/* moffat.cpp:98-100 */
		return 0.1 / p->axrat;
	default:
		/* radial.cpp:224-227 */
		return acc;
	}
}

static int validate(const pfo_model *m, const profile_t *p)
{
	if (p->kind == K_PSF) {
		if (!m->psf) return fail("No psf present in the model, cannot produce a psf profile%s", NULL);
		return 0;
	}
	if (!is_radial(p)) return 0;
	/* radial.cpp:204-214 */
	if (p->axrat <= 0) return fail("axrat <= 0, must have axrat > 0%s", NULL);
	if (p->axrat > 1) return fail("axrat > 1, must have axrat <= 1%s", NULL);
	if (p->box <= -2) return fail("box <= -2, must have box > -2%s", NULL);
	switch (p->kind) {
	case K_SERSIC:
		if (p->re <= 0) return fail("re <= 0, must have re > 0%s", NULL);
		if (p->nser <= 0) return fail("nser <= 0, must have nser > 0%s", NULL);
		break;
	case K_MOFFAT:
		if (p->fwhm <= 0) return fail("fwhm <= 0, must have fwhm > 0%s", NULL);
		if (p->con < 0) return fail("con < 0, must have con >= 0%s", NULL);
		break;
	case K_FERRER:
		if (p->rout <= 0) return fail("rout <= 0, must have rout >= 0%s", NULL);
		if (p->a < 0) return fail("a < 0, must have a >= 0%s", NULL);
		if (p->b > 2) return fail("b > 2, must have b <= 2%s", NULL);
		break;
	case K_CORESERSIC:
		if (p->re <= 0) return fail("re <= 0, must have re > 0%s", NULL);
		if (p->rb <= 0) return fail("rb <= 0, must have rb > 0%s", NULL);
		if (p->nser <= 0) return fail("nser <= 0, must have nser > 0%s", NULL);
		if (p->a <= 0) return fail("a <= 0, must have a > 0%s", NULL);
		if (p->b > 1.999) return fail("b > 1.999, must have b < 1.999%s", NULL);
		break;
	case K_KING:
		if (p->rc <= 0) return fail("rc <= 0, must have rc > 0%s", NULL);
		if (p->rt <= 0) return fail("rt <= 0, must have rt > 0%s", NULL);
		if (p->a < 0) return fail("a < 0, must have a >=0%s", NULL);
		break;
	case K_BROKENEXP:
		if (p->h1 <= 0) return fail("h1 <= 0, must have h1 > 0%s", NULL);
		if (p->h2 <= 0) return fail("h2 <= 0, must have h2 > 0%s", NULL);
		if (p->rb <= 0) return fail("rb <= 0, must have rb > 0%s", NULL);
		break;
	}
	return 0;
}

/* sersic.cpp:225-252: specialisation chosen from nser (and box) */
static void choose_sersic_spec(profile_t *p)
{
	double inv_exponent = p->nser;
	p->boxy = p->box != 0;
	if (p->boxy) inv_exponent *= (p->box + 2);
	if (almost_equals(inv_exponent, 0.5)) p->spec = RF_POINTFIVE;
	else if (almost_equals(inv_exponent, 1)) p->spec = RF_ONE;
	else if (almost_equals(inv_exponent, 2)) p->spec = RF_TWO;
	else if (almost_equals(inv_exponent, 3)) p->spec = RF_THREE;
	else if (almost_equals(inv_exponent, 4)) p->spec = RF_FOUR;
	else if (almost_equals(inv_exponent, 8)) p->spec = RF_EIGHT;
	else if (almost_equals(inv_exponent, 16)) p->spec = RF_SIXTEEN;
	else p->spec = RF_GENERAL;
}

/* radial.cpp:136-199 plus sersic.cpp:291-313 and coresersic.cpp:106-117 */
static void initial_calculations(profile_t *p, double magzero)
{
	p->magzero = magzero;
	if (p->kind == K_SERSIC || p->kind == K_CORESERSIC) {
		p->bn = u_qgamma(0.5, 2 * p->nser);
	}
	p->d_acc = p->acc;
	p->d_rscale_switch = p->rscale_switch;
	p->d_resolution = p->resolution;
	p->d_rscale_max = p->rscale_max;

	p->rscale = get_rscale(p);
	double b2 = p->box + 2;
	double r_box = M_PI * b2 / (2 * u_beta(1 / b2, 1 / b2));
	double lumtot = get_lumtot(p) * p->axrat / r_box;
	p->lumtot = lumtot;
	p->ie = pow(10, -0.4 * (p->mag - magzero)) / lumtot;

	if (p->adjust) {
		p->d_rscale_switch = adjust_rscale_switch(p);
		unsigned res = (unsigned)ceil(160 / (p->d_rscale_switch * p->rscale));
		res += res % 2;
		if (res > 16U) res = 16U;
		if (res < 4U) res = 4U;
		p->d_resolution = res;
		if (p->d_rscale_max == 0) p->d_rscale_max = adjust_rscale_max(p);
		p->d_acc = adjust_acc(p, p->d_acc);
	}

	double angrad = fmod(p->ang + 90, 360.) * M_PI / 180.;
	p->cos_ang = cos(angrad);
	p->sin_ang = sin(angrad);
	p->cos_q = p->cos_ang / p->axrat;
	p->sin_q = p->sin_ang / p->axrat;

	p->rescale_factor = 1;
	if (p->kind == K_SERSIC && p->adjust && p->rescale_flux) {
		/* sersic.cpp:304-311 */
		double flux_r = p->bn * pow(p->d_rscale_max / p->re, 1 / p->nser);
		flux_r = u_pgamma(flux_r, 2 * p->nser);
		p->rescale_factor = 1 / flux_r;
	}
}

/* radial.cpp:46-52 */
static inline void to_profile(const profile_t *p, double x, double y, double *xp, double *yp)
{
	x -= p->cx;
	y -= p->cy;
	*xp = x * p->cos_ang + y * p->sin_ang;
	*yp = -x * p->sin_q + y * p->cos_q;
}

/*
 * radial.cpp:54-134: adaptive sub-pixel integration.  Points that fail the
 * accuracy test are deferred to the end of the level, in (i, j) order, and
 * each deferred point is then integrated recursively, depth first.
 */
static double subsample_pixel(profile_t *p, double x0, double x1, double y0, double y1,
                              unsigned recur_level, unsigned max_recursions,
                              unsigned resolution, int *ncalls)
{
	double xbin = (x1 - x0) / resolution;
	double ybin = (y1 - y0) / resolution;
	double half_xbin = xbin / 2.;
	double half_ybin = ybin / 2.;
	double total = 0;
	double xp, yp;
	int recurse = resolution > 1 && recur_level < max_recursions;

	(*ncalls)++;
	if (recur_level < MAX_LEVELS) {
#pragma omp atomic
		p->level_counts[recur_level]++;
	}
	/* res^2 sub-points below, each evaluated twice when testing */
#pragma omp atomic
	p->n_evals += (long)resolution * resolution * (recurse ? 2 : 1);

	double *pts = NULL;
	size_t npts = 0;
	double x = x0;
	if (recurse) {
		pts = (double *)malloc(sizeof(double) * 2 * resolution * resolution);
		for (unsigned i = 0; i < resolution; i++) {
			x += half_xbin;
			double y = y0;
			for (unsigned j = 0; j < resolution; j++) {
				y += half_ybin;
				to_profile(p, x, y, &xp, &yp);
				double subval = evaluate_at(p, xp, yp);
				double delta_y_prof = -xbin * p->sin_q + ybin * p->cos_q;
				double testval = evaluate_at(p, fabs(xp), fabs(yp) + fabs(delta_y_prof));
				if (fabs(testval - subval) > p->d_acc * subval) {
					pts[2 * npts] = x;
					pts[2 * npts + 1] = y;
					npts++;
				}
				else {
					total += subval;
				}
				y += half_ybin;
			}
			x += half_xbin;
		}
	}
	else {
		for (unsigned i = 0; i < resolution; i++) {
			x += half_xbin;
			double y = y0;
			for (unsigned j = 0; j < resolution; j++) {
				y += half_ybin;
				to_profile(p, x, y, &xp, &yp);
				total += evaluate_at(p, xp, yp);
				y += half_ybin;
			}
			x += half_xbin;
		}
	}
	for (size_t k = 0; k < npts; k++) {
		double px = pts[2 * k], py = pts[2 * k + 1];
		total += subsample_pixel(p, px - half_xbin, px + half_xbin, py - half_ybin, py + half_ybin,
		                         recur_level + 1, max_recursions, resolution, ncalls);
	}
	free(pts);
	return total / (resolution * resolution);
}

/* radial.cpp:239-344 (CPU path) plus sersic.cpp:315-347 */
static void radial_evaluate(const pfo_model *m, profile_t *p, double *image, unsigned width,
                            unsigned height, double sx, double sy, double offx, double offy)
{
	if (p->kind == K_SERSIC) choose_sersic_spec(p);
	initial_calculations(p, m->magzero);
	p->cx = p->xcen + offx * sx;
	p->cy = p->ycen + offy * sy;
	memset(p->level_counts, 0, sizeof(p->level_counts));
	p->n_evals = 0;
	free(p->decisions);
	p->n_decisions = (size_t)width * height;
	p->decisions = (int *)calloc(p->n_decisions, sizeof(int));

	double half_xbin = sx / 2.;
	double half_ybin = sy / 2.;
	double flux_scale = sx * sy * p->ie;
	if (p->kind == K_SERSIC && p->rescale_flux) flux_scale *= p->rescale_factor;
	p->flux_scale = flux_scale;

#pragma omp parallel for schedule(dynamic, 4) num_threads(m->threads)
	for (unsigned j = 0; j < height; j++) {
		for (unsigned i = 0; i < width; i++) {
			double xp, yp;
			double y = half_ybin + j * sx;
			double x = half_xbin + i * sy;
			to_profile(p, x, y, &xp, &yp);
			double r_prof = sqrt(xp * xp + yp * yp);
			double pixel_val;
			int ncalls = 0;
			if (p->d_rscale_max > 0 && r_prof > p->d_rscale_max * p->rscale) {
				pixel_val = 0.;
				ncalls = -1;
			}
			else if (p->rough || r_prof > p->d_rscale_switch * p->rscale) {
				pixel_val = evaluate_at(p, xp, yp);
#pragma omp atomic
				p->n_evals++;
			}
			else {
				unsigned res = p->d_resolution, maxrec = p->max_recursions;
				if (p->kind == K_SERSIC) {
					int center = fabs(x - p->cx) < m->img_scale_x && fabs(y - p->cy) < m->img_scale_y;
					if (p->adjust && center && p->nser > 1) {
						res = 8;
						maxrec = 10;
					}
				}
				pixel_val = subsample_pixel(p, x - half_xbin, x + half_xbin, y - half_ybin,
				                            y + half_ybin, 0, maxrec, res, &ncalls);
			}
			p->decisions[i + (size_t)j * width] = ncalls;
			image[i + (size_t)j * width] += flux_scale * pixel_val;
		}
	}
}

/* sky.cpp:42-63 (no mask support) */
static void sky_evaluate(profile_t *p, double *image, size_t n, unsigned fs)
{
	p->sky_bg = p->bg / (fs * fs);
	for (size_t k = 0; k < n; k++) image[k] += p->sky_bg;
}

static unsigned bind_u(double value, unsigned max)
{
	/* psf.cpp:48-56 */
	int intval = (int)floor(value);
	if (intval < 0) return 0;
	unsigned u = (unsigned)intval;
	return u < max ? u : max;
}

/* psf.cpp:58-145, including its x/y offset quirks (lines 79-82, 106) */
static void psf_evaluate(const pfo_model *m, profile_t *p, double *image, unsigned width,
                         unsigned height, double scale_x, double scale_y, double offx, double offy)
{
	double scale = pow(10, -0.4 * (p->mag - m->magzero));
	double psf_scale_x = m->psf_scale_x, psf_scale_y = m->psf_scale_y;
	unsigned psf_width = m->psf_w, psf_height = m->psf_h;

	double origin_x = p->xcen + offx * scale_x - psf_width * psf_scale_x / 2;
	double end_x = p->xcen + offy * scale_y + psf_width * psf_scale_x / 2;
	double origin_y = p->ycen + offx * scale_x - psf_height * psf_scale_y / 2;
	double end_y = p->ycen + offy * scale_y + psf_height * psf_scale_y / 2;

	unsigned x0 = bind_u(origin_x / scale_x, width - 1);
	unsigned y0 = bind_u(origin_y / scale_y, height - 1);
	unsigned x1 = bind_u(end_x / scale_x, width - 1);
	unsigned y1 = bind_u(end_y / scale_y, height - 1);

	for (unsigned pix_y = y0; pix_y <= y1; pix_y++) {
		double y = pix_y * scale_y;
		for (unsigned pix_x = x0; pix_x <= x1; pix_x++) {
			double x = pix_x * scale_x;
			int px0 = (int)bind_u(floor((x - origin_x) / psf_scale_x), psf_width - 1);
			int px1 = (int)bind_u(floor((x - origin_x + scale_x) / psf_scale_x), psf_height - 1);
			int py0 = (int)bind_u(floor((y - origin_y) / psf_scale_y), psf_width - 1);
			int py1 = (int)bind_u(floor((y - origin_y + scale_y) / psf_scale_y), psf_height - 1);
			double val = 0;
			for (int psf_pix_y = py0; psf_pix_y <= py1; psf_pix_y++) {
				double psf_y = psf_pix_y * psf_scale_y + origin_y;
				for (int psf_pix_x = px0; psf_pix_x <= px1; psf_pix_x++) {
					double psf_x = psf_pix_x * psf_scale_x + origin_x;
					double ix = fmin(x + scale_x, psf_x + psf_scale_x) - fmax(x, psf_x);
					double iy = fmin(y + scale_y, psf_y + psf_scale_y) - fmax(y, psf_y);
					val += m->psf[psf_pix_x + psf_pix_y * psf_width] * (ix * iy) / (psf_scale_x * psf_scale_y);
				}
			}
			image[pix_x + (size_t)pix_y * width] += val * scale;
		}
	}
}

/* ------------------------------------------------------------------------- */
/* Convolution                                                               */
/* ------------------------------------------------------------------------- */

/*
 * convolve.cpp:158-231 (AssociativeBruteForceConvolver): out(i, j) is the sum
 * over kernel rows of the dot product of a source row with the reversed
 * kernel row, clipped at the image edges.  Only outputs inside
 * [cx0, cx0 + cw) x [cy0, cy0 + ch) are computed and written into out[ch][cw].
 */
static void brute_convolve_crop(const pfo_model *m, const double *src, unsigned sw, unsigned sh,
                                const double *krn, unsigned kw, unsigned kh, unsigned cx0,
                                unsigned cy0, unsigned cw, unsigned ch, double *out)
{
	const unsigned khw = kw / 2, khh = kh / 2;
	double *ikrn = (double *)malloc(sizeof(double) * kw * kh);
	for (size_t k = 0; k < (size_t)kw * kh; k++) ikrn[k] = krn[(size_t)kw * kh - 1 - k];

#pragma omp parallel for schedule(dynamic, 4) num_threads(m->threads)
	for (unsigned jj = 0; jj < ch; jj++) {
		unsigned j = jj + cy0;
		for (unsigned ii = 0; ii < cw; ii++) {
			unsigned i = ii + cx0;
			unsigned l_min = 0, l_max = kh, k_min = 0, k_max = kw;
			if (j < khh) l_min = khh - j;
			else if ((j + khh) >= sh) l_max = sh + khh - j;
			if (i < khw) k_min = khw - i;
			else if ((i + khw) >= sw) k_max = sw + khw - i;
			double pixel = 0;
			for (unsigned l = l_min; l < l_max; l++) {
				const double *s = src + (size_t)(j + l - khh) * sw + (i + k_min - khw);
				const double *k = ikrn + (size_t)l * kw + k_min;
				double dot = 0;
				for (unsigned c = 0; c < k_max - k_min; c++) dot += s[c] * k[c];
				pixel += dot;
			}
			out[ii + (size_t)jj * cw] = pixel;
		}
	}
	free(ikrn);
}

/*
 * convolve.cpp:245-312 (FFTConvolver) restated as the linear convolution it
 * computes: the source sits at (0, 0) and the kernel at (src - krn)/2 of a
 * 2*max(src, krn) buffer, so the cyclic product never wraps; the result is
 * read back from offset_after_convolution (convolve.cpp:270-281).
 */
static void fft_convolve_crop(const pfo_model *m, const double *src, unsigned sw, unsigned sh,
                              const double *krn, unsigned kw, unsigned kh, unsigned cx0,
                              unsigned cy0, unsigned cw, unsigned ch, double *out)
{
	int kx0 = (int)((sw - kw) / 2), ky0 = (int)((sh - kh) / 2);
	int ox = (int)(sw / 2), oy = (int)(sh / 2);
	if (sw % 2 == 0 || kw % 2 == 0) ox -= 1;
	if (sh % 2 == 0 || kh % 2 == 0) oy -= 1;
	int dx = ox - kx0, dy = oy - ky0;
#pragma omp parallel for schedule(dynamic, 4) num_threads(m->threads)
	for (unsigned jj = 0; jj < ch; jj++) {
		int y = (int)(jj + cy0);
		for (unsigned ii = 0; ii < cw; ii++) {
			int x = (int)(ii + cx0);
			double acc = 0;
			for (int v = 0; v < (int)kh; v++) {
				int sy = y + dy - v;
				if (sy < 0 || sy >= (int)sh) continue;
				for (int u = 0; u < (int)kw; u++) {
					int sxx = x + dx - u;
					if (sxx < 0 || sxx >= (int)sw) continue;
					acc += krn[u + (size_t)v * kw] * src[sxx + (size_t)sy * sw];
				}
			}
			out[ii + (size_t)jj * cw] = acc;
		}
	}
}

/* ------------------------------------------------------------------------- */
/* Model                                                                     */
/* ------------------------------------------------------------------------- */

pfo_model *pfo_model_new(unsigned width, unsigned height)
{
	pfo_model *m = (pfo_model *)calloc(1, sizeof(pfo_model));
	m->width = width;
	m->height = height;
	m->scale_x = m->scale_y = 1;
	m->psf_scale_x = m->psf_scale_y = 1;
	m->finesampling = 1;
	m->return_finesampled = 1;
	m->threads = 1;
	return m;
}

void pfo_model_free(pfo_model *m)
{
	if (!m) return;
	for (int i = 0; i < m->n_profiles; i++) free(m->profiles[i].decisions);
	free(m->profiles);
	free(m->psf);
	free(m);
}

int pfo_add_profile(pfo_model *m, const char *name)
{
	/* model.cpp:103-135 */
	int kind;
	if (strcmp(name, "null") == 0) kind = K_NULL;
	else if (strcmp(name, "sky") == 0) kind = K_SKY;
	else if (strcmp(name, "sersic") == 0) kind = K_SERSIC;
	else if (strcmp(name, "moffat") == 0) kind = K_MOFFAT;
	else if (strcmp(name, "ferrer") == 0 || strcmp(name, "ferrers") == 0) kind = K_FERRER;
	else if (strcmp(name, "coresersic") == 0) kind = K_CORESERSIC;
	else if (strcmp(name, "king") == 0) kind = K_KING;
	else if (strcmp(name, "brokenexp") == 0) kind = K_BROKENEXP;
	else if (strcmp(name, "psf") == 0) kind = K_PSF;
	else return fail("Unknown profile name: %s", name);

	m->profiles = (profile_t *)realloc(m->profiles, sizeof(profile_t) * (m->n_profiles + 1));
	profile_t *p = &m->profiles[m->n_profiles];
	memset(p, 0, sizeof(*p));
	p->kind = kind;
	snprintf(p->name, sizeof(p->name), "%s", name);
	radial_defaults(p);
	switch (kind) {
	case K_SERSIC: p->re = 1; p->nser = 1; p->rescale_flux = 0; break;          /* sersic.cpp:350-359 */
	case K_MOFFAT: p->fwhm = 3; p->con = 2; break;                              /* moffat.cpp:102-108 */
	case K_FERRER: p->rout = 3; p->a = 1; p->b = 1; p->acc = 1; break;          /* ferrer.cpp:115-126 */
	case K_CORESERSIC: p->re = 1; p->rb = 1; p->nser = 4; p->a = 1; p->b = 1; break; /* coresersic.cpp:131-140 */
	case K_KING: p->rc = 1; p->rt = 3; p->a = 2; break;                        /* king.cpp:111-119 */
	case K_BROKENEXP: p->h1 = 1; p->h2 = 1; p->rb = 1; p->a = 1; break;        /* brokenexponential.cpp:141-150 */
	case K_PSF: p->xcen = 0; p->ycen = 0; p->mag = 0; break;                   /* psf.cpp:147-156 */
	default: break;
	}
	return m->n_profiles++;
}

static int set_param(pfo_model *m, int idx, const char *name, char type, double dv, unsigned uv, int bv)
{
	if (idx < 0 || idx >= m->n_profiles) return fail("profile index out of range%s", NULL);
	profile_t *p = &m->profiles[idx];
	const param_desc *d = find_param(p, name);
	if (!d || d->type != type) {
		const char *tn = type == 'd' ? "double" : type == 'u' ? "unsigned int" : "bool";
		snprintf(g_err, sizeof(g_err), "Unknown %s parameter in profile %s: %s", tn, p->name, name);
		return -1;
	}
	char *base = (char *)p + d->off;
	if (type == 'd') *(double *)base = dv;
	else if (type == 'u') *(unsigned *)base = uv;
	else *(int *)base = bv != 0;
	return 0;
}

int pfo_profile_set_double(pfo_model *m, int idx, const char *name, double v) { return set_param(m, idx, name, 'd', v, 0, 0); }
int pfo_profile_set_uint(pfo_model *m, int idx, const char *name, unsigned v) { return set_param(m, idx, name, 'u', 0, v, 0); }
int pfo_profile_set_bool(pfo_model *m, int idx, const char *name, int v) { return set_param(m, idx, name, 'b', 0, 0, v); }

int pfo_set_psf(pfo_model *m, const double *psf, unsigned w, unsigned h)
{
	/* model.h:160-170 with Image::normalize (image.cpp:231-237) */
	free(m->psf);
	m->psf = (double *)malloc(sizeof(double) * w * h);
	double sum = 0;
	for (size_t k = 0; k < (size_t)w * h; k++) sum += psf[k];
	for (size_t k = 0; k < (size_t)w * h; k++) m->psf[k] = sum > 0 ? psf[k] / sum : psf[k];
	m->psf_w = w;
	m->psf_h = h;
	return 0;
}

void pfo_set_magzero(pfo_model *m, double mz) { m->magzero = mz; }
void pfo_set_scale(pfo_model *m, double sx, double sy) { m->scale_x = sx; m->scale_y = sy; }
void pfo_set_psf_scale(pfo_model *m, double sx, double sy) { m->psf_scale_x = sx; m->psf_scale_y = sy; }
void pfo_set_return_finesampled(pfo_model *m, int v) { m->return_finesampled = v != 0; }
void pfo_set_threads(pfo_model *m, int n) { m->threads = n > 0 ? n : 1; }

int pfo_set_finesampling(pfo_model *m, unsigned fs)
{
	if (fs == 0) return fail("finesampling must be > 0%s", NULL);
	m->finesampling = fs;
	return 0;
}

int pfo_set_convolver(pfo_model *m, const char *kind)
{
	if (strcmp(kind, "brute") == 0 || strcmp(kind, "brute-old") == 0) m->conv_kind = 0;
	else if (strcmp(kind, "fft") == 0) m->conv_kind = 1;
	else if (strcmp(kind, "null") == 0) m->conv_kind = 2;
	else return fail("Unknown convolver type: %s", kind);
	return 0;
}

static int convolution_required(const pfo_model *m)
{
	for (int i = 0; i < m->n_profiles; i++)
		if (m->profiles[i].convolve) return 1;
	return 0;
}

int pfo_drawing_dims(pfo_model *m, unsigned *w, unsigned *h)
{
	/* model.cpp:152-219 without masks */
	if (m->width == 0 || m->height == 0) return fail("Model's requested dimensions are 0%s", NULL);
	unsigned pw = 0, ph = 0;
	if (convolution_required(m)) {
		if (!m->psf) return fail("No psf provided but profile(s) requested convolution%s", NULL);
		pw = m->psf_w / 2;
		ph = m->psf_h / 2;
	}
	*w = m->width * m->finesampling + 2 * pw;
	*h = m->height * m->finesampling + 2 * ph;
	return 0;
}

int pfo_evaluate(pfo_model *m, double *out, size_t cap, unsigned *ow, unsigned *oh, int *ox, int *oy)
{
	unsigned dw, dh;
	if (m->scale_x <= 0) return fail("Model's scale_x cannot be negative or zero%s", NULL);
	if (m->scale_y <= 0) return fail("Model's scale_y cannot be negative or zero%s", NULL);
	if (pfo_drawing_dims(m, &dw, &dh)) return -1;
	for (int i = 0; i < m->n_profiles; i++)
		if (validate(m, &m->profiles[i])) return -1;

	int conv = convolution_required(m);
	unsigned padx = conv ? m->psf_w / 2 : 0, pady = conv ? m->psf_h / 2 : 0;
	unsigned fs = m->finesampling;
	double sx = m->scale_x / fs, sy = m->scale_y / fs;
	m->img_scale_x = m->scale_x;
	m->img_scale_y = m->scale_y;
	size_t npix = (size_t)dw * dh;
	double *model_image = (double *)calloc(npix, sizeof(double));
	double *to_convolve = conv ? (double *)calloc(npix, sizeof(double)) : NULL;

	/* model.cpp:340-366 */
	for (int i = 0; i < m->n_profiles; i++) {
		profile_t *p = &m->profiles[i];
		double *target = p->convolve ? to_convolve : model_image;
		if (is_radial(p)) radial_evaluate(m, p, target, dw, dh, sx, sy, padx, pady);
		else if (p->kind == K_SKY) sky_evaluate(p, target, npix, fs);
		else if (p->kind == K_PSF) psf_evaluate(m, p, target, dw, dh, sx, sy, padx, pady);
	}

	/* convolve (model.cpp:369-377) and crop the PSF padding (model.cpp:307-324) */
	unsigned cw = dw - 2 * padx, ch = dh - 2 * pady;
	double *img = (double *)malloc(sizeof(double) * cw * ch);
	if (conv) {
		if (m->conv_kind == 0)
			brute_convolve_crop(m, to_convolve, dw, dh, m->psf, m->psf_w, m->psf_h, padx, pady, cw, ch, img);
		else if (m->conv_kind == 1)
			fft_convolve_crop(m, to_convolve, dw, dh, m->psf, m->psf_w, m->psf_h, padx, pady, cw, ch, img);
		else
			for (unsigned j = 0; j < ch; j++)
				for (unsigned i = 0; i < cw; i++) img[i + (size_t)j * cw] = to_convolve[(i + padx) + (size_t)(j + pady) * dw];
		for (unsigned j = 0; j < ch; j++)
			for (unsigned i = 0; i < cw; i++)
				img[i + (size_t)j * cw] += model_image[(i + padx) + (size_t)(j + pady) * dw];
	}
	else {
		memcpy(img, model_image, sizeof(double) * npix);
	}

	/* downsample (model.cpp:326-329, image.cpp:285-298) */
	unsigned fw = cw, fh = ch;
	int offx = 0, offy = 0;
	if (fs > 1 && !m->return_finesampled) {
		fw = (cw + fs - 1) / fs;
		fh = (ch + fs - 1) / fs;
		double *down = (double *)calloc((size_t)fw * fh, sizeof(double));
		for (unsigned row = 0; row < ch; row++)
			for (unsigned col = 0; col < cw; col++)
				down[col / fs + (size_t)(row / fs) * fw] += img[col + (size_t)row * cw];
		free(img);
		img = down;
	}

	int st = 0;
	if ((size_t)fw * fh > cap) st = fail("output buffer too small%s", NULL);
	else memcpy(out, img, sizeof(double) * fw * fh);
	*ow = fw;
	*oh = fh;
	*ox = offx;
	*oy = offy;
	free(img);
	free(model_image);
	free(to_convolve);
	return st;
}

int pfo_decisions(pfo_model *m, int idx, int *out, size_t cap)
{
	if (idx < 0 || idx >= m->n_profiles) return fail("profile index out of range%s", NULL);
	profile_t *p = &m->profiles[idx];
	if (!p->decisions) return fail("no decisions recorded%s", NULL);
	if (p->n_decisions > cap) return fail("buffer too small%s", NULL);
	memcpy(out, p->decisions, sizeof(int) * p->n_decisions);
	return (int)p->n_decisions;
}

long pfo_evaluations(pfo_model *m, int idx)
{
	if (idx < 0 || idx >= m->n_profiles) return fail("profile index out of range%s", NULL);
	return m->profiles[idx].n_evals;
}

int pfo_level_counts(pfo_model *m, int idx, long *out, int max_levels)
{
	if (idx < 0 || idx >= m->n_profiles) return fail("profile index out of range%s", NULL);
	profile_t *p = &m->profiles[idx];
	int n = 0;
	for (int l = 0; l < max_levels && l < MAX_LEVELS; l++) {
		out[l] = p->level_counts[l];
		if (p->level_counts[l]) n = l + 1;
	}
	return n;
}

int pfo_profile_scalars(pfo_model *m, int idx, double *out, int n)
{
	if (idx < 0 || idx >= m->n_profiles) return fail("profile index out of range%s", NULL);
	profile_t *p = &m->profiles[idx];
	double v[12] = {p->rscale, p->ie, p->bn, p->d_acc, p->d_rscale_switch, p->d_rscale_max,
	                (double)p->d_resolution, p->flux_scale, p->cos_ang, p->sin_ang, p->lumtot,
	                p->rescale_factor};
	for (int k = 0; k < n && k < 12; k++) out[k] = v[k];
	return 12;
}

/* R/profitLikeModel.R:263-276: sum(dnorm(cutsig, log = TRUE)) with
 * dnorm(x, 0, 1, log) = -(log(sqrt(2 pi)) + x^2 / 2), Neumaier summation. */
double pfo_loglike_norm(const double *image, const double *sigma, const double *model,
                        const unsigned char *region, size_t n)
{
	const double ln_sqrt_2pi = 0.918938533204672741780329736406;
	double sum = 0, comp = 0;
	for (size_t k = 0; k < n; k++) {
		if (region && !region[k]) continue;
		double x = (image[k] - model[k]) / sigma[k];
		double term = -(ln_sqrt_2pi + 0.5 * x * x);
		double t = sum + term;
		if (fabs(sum) >= fabs(term)) comp += (sum - t) + term;
		else comp += (term - t) + sum;
		sum = t;
	}
	return sum + comp;
}
