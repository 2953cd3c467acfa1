// Profile parameters, the per-profile scalar prologue and the FP64 profile
// evaluators of the plain form.
//
// The FP64 evaluators keep libprofit's operation order (and Sersic's
// pow-avoiding specialisations) so that, with sm_100a FP64 arithmetic
// compiled without FMA contraction, the subsampling tests
// |f(|x'|,|y'|+|dy'|) - f(x',y')| > acc * f(x',y') take the same branches as
// the reference.  Sources: radial.cpp:46-199, radial.h:93-102,
// sersic.cpp:78-347, moffat.cpp:52-100, ferrer.cpp:50-113,
// coresersic.cpp:51-125, king.cpp:51-109, brokenexponential.cpp:38-139.
#pragma once

#include <cstdint>

#include "specfun.cuh"

namespace pf {

enum ProfileKind : int32_t {
	PK_SERSIC = 0,
	PK_MOFFAT = 1,
	PK_FERRER = 2,
	PK_CORESERSIC = 3,
	PK_KING = 4,
	PK_BROKENEXP = 5,
	PK_SKY = 6,
	PK_PSF = 7,
	PK_NULL = 8
};

PF_HD inline bool is_radial_kind(int k) { return k >= PK_SERSIC && k <= PK_BROKENEXP; }

// Shape parameters with an adjoint, per radial kind, in tangent-slot order:
// sersic (re, nser), moffat (fwhm, con), ferrer (rout, a, b), coresersic
// (re, rb, nser, a, b), king (rc, rt, a), brokenexp (h1, h2, rb, a).
constexpr int MAX_SHAPE = 5;
PF_HD inline int shape_count(int kind)
{
	switch (kind) {
	case PK_SERSIC: return 2;
	case PK_MOFFAT: return 2;
	case PK_FERRER: return 3;
	case PK_CORESERSIC: return 5;
	case PK_KING: return 3;
	case PK_BROKENEXP: return 4;
	default: return 0;
	}
}

// Sersic r_factor forms of sersic.cpp:78-189
enum SersicForm : int32_t { SF_GENERAL = 0, SF_HALF, SF_ONE, SF_TWO, SF_THREE, SF_FOUR, SF_EIGHT, SF_SIXTEEN };

// User-facing parameters of one profile, with libprofit's defaults
// (radial.cpp:724-752 and each profile's constructor).
struct ProfileParams {
	int32_t kind;
	int32_t convolve, rough, adjust, force_cpu, rescale_flux;
	uint32_t resolution, max_recursions;
	double xcen, ycen, mag, ang, axrat, box;
	double acc, rscale_switch, rscale_max;
	double re, nser, fwhm, con, rout, a, b, rb, rc, rt, h1, h2, bg;
};

// Everything a pixel kernel needs for one profile.
struct DevProfile {
	int32_t kind, form, boxy, rough;
	int32_t target;          // 0: image to convolve, 1: unconvolved image
	int32_t centre_override; // Sersic nser > 1 with adjust (sersic.cpp:339-345)
	uint32_t resolution, max_rec;
	double cx, cy;                     // centre in drawing-pixel coordinates
	double cos_ang, sin_ang, cos_q, sin_q;
	double rscale, r_switch, r_max;    // r_switch = rscale_switch*rscale, r_max = rscale_max*rscale (0 = none)
	double acc, flux_scale, bn;
	double re, nser, box, invexp;
	double con, a, b, rb, rc, rt, h1, h2, king_t;
	double img_sx, img_sy;             // image pixel scale (centre-pixel test)
	double bg;                         // sky value per drawing pixel
	double psf_flux, px, py;           // psf point source: 10^(-0.4(mag-magzero)), centre
	// derivatives of log(flux_scale) w.r.t. parameters (FP32+adjoint path):
	// magnitude, axis ratio, box, and the shape parameters in the order of
	// shape_param_name()
	double dlnI_dmag, dlnI_dq, dlnI_dbox, dlnI_dp[MAX_SHAPE];
	double dbn_dn;
	double axrat;
};

struct ModelGeom {
	double magzero;
	double sx, sy;          // profile pixel scale (image scale / finesampling)
	double img_sx, img_sy;  // image pixel scale
	double offx, offy;      // PSF padding in drawing pixels
	unsigned finesampling;
};

PF_HD inline bool almost_eq(double x, double y) { return fabs(x - y) < 1e-10; }

// ---- radial functions (values), reference operation order ---------------

PF_HD inline double boxy_r(const DevProfile &p, double x, double y)
{
	if (p.box == 0) return sqrt(x * x + y * y);
	double bp2 = p.box + 2.;
	return pow(pow(fabs(x), bp2) + pow(fabs(y), bp2), 1. / bp2);
}

PF_HD inline double coresersic_r(double r, double rb, double a, double b, double re, double nser, double bn)
{
	return pow(1 + pow(r / rb, -a), b / a) * exp(-bn * pow((pow(r, a) + pow(rb, a)) / pow(re, a), 1 / (nser * a)));
}

PF_HD inline double king_r(double r, double rc, double rt, double a)
{
	if (r < rt) return pow(1 / pow(1 + pow(r / rc, 2), 1 / a) - 1 / pow(1 + pow(rt / rc, 2), 1 / a), a);
	return 0;
}

PF_HD inline double brokenexp_r(double r, double h1, double h2, double rb, double a)
{
	double base = r - rb;
	double expo = 1 / h1 - 1 / h2;
	if (a * base < 40) base = log(1 + exp(a * base)) / a;
	return exp(-r / h1 + expo * base);
}

PF_HD inline double sersic64(const DevProfile &p, double x, double y)
{
	double base, rf;
	if (p.boxy) {
		double B = p.box + 2;
		base = pow(fabs(x / p.re), B) + pow(fabs(y / p.re), B);
		switch (p.form) {
		case SF_HALF: rf = base * base; break;
		case SF_ONE: rf = base; break;
		case SF_TWO: rf = sqrt(base); break;
		case SF_THREE: rf = cbrt(base); break;
		case SF_FOUR: rf = sqrt(sqrt(base)); break;
		case SF_EIGHT: rf = sqrt(sqrt(sqrt(base))); break;
		case SF_SIXTEEN: rf = sqrt(sqrt(sqrt(sqrt(base)))); break;
		default: rf = pow(base, 1 / p.invexp); break;
		}
	}
	else {
		base = (x * x + y * y) / (p.re * p.re);
		switch (p.form) {
		case SF_HALF: rf = base; break;
		case SF_ONE: rf = sqrt(base); break;
		case SF_TWO: rf = sqrt(sqrt(base)); break;
		case SF_THREE: rf = cbrt(sqrt(base)); break;
		case SF_FOUR: rf = sqrt(sqrt(sqrt(base))); break;
		case SF_EIGHT: rf = sqrt(sqrt(sqrt(sqrt(base)))); break;
		case SF_SIXTEEN: rf = sqrt(sqrt(sqrt(sqrt(sqrt(base))))); break;
		default: rf = pow(sqrt(base), 1 / p.invexp); break;
		}
	}
	return exp(-p.bn * (rf - 1));
}

PF_HD inline double eval64(const DevProfile &p, double x, double y)
{
	switch (p.kind) {
	case PK_SERSIC: return sersic64(p, x, y);
	case PK_MOFFAT: {
		double r = boxy_r(p, x, y);
		double rf = r / p.rscale;
		return pow(1 + rf * rf, -p.con);
	}
	case PK_FERRER: {
		double r = boxy_r(p, x, y);
		double rf = r / p.rscale;
		if (rf < 1) return pow(1 - pow(rf, 2 - p.b), p.a);
		return 0;
	}
	case PK_CORESERSIC: return coresersic_r(boxy_r(p, x, y), p.rb, p.a, p.b, p.re, p.nser, p.bn);
	case PK_KING: return king_r(boxy_r(p, x, y), p.rc, p.rt, p.a);
	case PK_BROKENEXP: return brokenexp_r(boxy_r(p, x, y), p.h1, p.h2, p.rb, p.a);
	default: return 0;
	}
}

// image -> profile coordinates (radial.cpp:46-52)
PF_HD inline void to_profile64(const DevProfile &p, double x, double y, double &xp, double &yp)
{
	x -= p.cx;
	y -= p.cy;
	xp = x * p.cos_ang + y * p.sin_ang;
	yp = -x * p.sin_q + y * p.cos_q;
}

// ---- validation (radial.cpp:204-214 and each profile's validate) --------

// Returns nullptr if valid, else libprofit's message.
inline const char *validate_profile(const ProfileParams &p, bool have_psf)
{
	if (p.kind == PK_PSF) return have_psf ? nullptr : "No psf present in the model, cannot produce a psf profile";
	if (!is_radial_kind(p.kind)) return nullptr;
	if (p.axrat <= 0) return "axrat <= 0, must have axrat > 0";
	if (p.axrat > 1) return "axrat > 1, must have axrat <= 1";
	if (p.box <= -2) return "box <= -2, must have box > -2";
	switch (p.kind) {
	case PK_SERSIC:
		if (p.re <= 0) return "re <= 0, must have re > 0";
		if (p.nser <= 0) return "nser <= 0, must have nser > 0";
		break;
	case PK_MOFFAT:
		if (p.fwhm <= 0) return "fwhm <= 0, must have fwhm > 0";
		if (p.con < 0) return "con < 0, must have con >= 0";
		break;
	case PK_FERRER:
		if (p.rout <= 0) return "rout <= 0, must have rout >= 0";
		if (p.a < 0) return "a < 0, must have a >= 0";
		if (p.b > 2) return "b > 2, must have b <= 2";
		break;
	case PK_CORESERSIC:
		if (p.re <= 0) return "re <= 0, must have re > 0";
		if (p.rb <= 0) return "rb <= 0, must have rb > 0";
		if (p.nser <= 0) return "nser <= 0, must have nser > 0";
		if (p.a <= 0) return "a <= 0, must have a > 0";
		if (p.b > 1.999) return "b > 1.999, must have b < 1.999";
		break;
	case PK_KING:
		if (p.rc <= 0) return "rc <= 0, must have rc > 0";
		if (p.rt <= 0) return "rt <= 0, must have rt > 0";
		if (p.a < 0) return "a < 0, must have a >=0";
		break;
	case PK_BROKENEXP:
		if (p.h1 <= 0) return "h1 <= 0, must have h1 > 0";
		if (p.h2 <= 0) return "h2 <= 0, must have h2 > 0";
		if (p.rb <= 0) return "rb <= 0, must have rb > 0";
		break;
	}
	return nullptr;
}

// Device-side form of validate_profile for batched proposals (a psf profile
// is valid when the model has a PSF; the batch entry point checks that).
PF_HD inline bool params_valid(const ProfileParams &p)
{
	if (!is_radial_kind(p.kind)) return true;
	if (!(p.axrat > 0) || p.axrat > 1 || !(p.box > -2)) return false;
	switch (p.kind) {
	case PK_SERSIC: return p.re > 0 && p.nser > 0;
	case PK_MOFFAT: return p.fwhm > 0 && p.con >= 0;
	case PK_FERRER: return p.rout > 0 && p.a >= 0 && p.b <= 2;
	case PK_CORESERSIC: return p.re > 0 && p.rb > 0 && p.nser > 0 && p.a > 0 && p.b <= 1.999;
	case PK_KING: return p.rc > 0 && p.rt > 0 && p.a >= 0;
	case PK_BROKENEXP: return p.h1 > 0 && p.h2 > 0 && p.rb > 0;
	}
	return true;
}

// ---- per-profile prologue ------------------------------------------------

struct CoreSersicIntegrand {
	double rb, a, b, re, nser, bn;
	PF_HD double operator()(double r) const { return r * coresersic_r(r, rb, a, b, re, nser, bn); }
};
struct KingIntegrand {
	double rc, rt, a;
	PF_HD double operator()(double r) const { return r * king_r(r, rc, rt, a); }
};
struct BrokenExpIntegrand {
	double h1, h2, rb, a;
	PF_HD double operator()(double r) const { return r * brokenexp_r(r, h1, h2, rb, a); }
};

// Fills the derived scalars of `d` from the user parameters `p`
// (RadialProfile::initial_calculations and the profile overrides).  Values
// libprofit writes back into the profile (acc, rscale_switch, resolution,
// rscale_max) are derived here without touching `p`, which is what a fresh
// profit::Model per evaluation (R_profit_make_model) observes.
// Total luminosity of a radial profile before the axis-ratio and box
// factors (the get_lumtot overrides: sersic.cpp:291-313, moffat.cpp,
// ferrer.cpp, coresersic.cpp:106-117, king.cpp, brokenexponential.cpp).
// bn: Sersic / core-Sersic b_n; rscale: the profile's scale radius.
PF_HD inline double profile_lum(const ProfileParams &p, double bn, double rscale)
{
	switch (p.kind) {
	case PK_SERSIC: {
		double g_factor = gamma_fn(2 * p.nser);
		return pow(p.re, 2) * 2 * M_PI * p.nser * g_factor * exp(bn) / pow(bn, 2 * p.nser);
	}
	case PK_MOFFAT: return pow(rscale, 2) * M_PI / (p.con - 1);
	case PK_FERRER: {
		double g_factor = p.a * beta_fn(p.a, 1 + 2 / (2 - p.b));
		return pow(p.rout, 2) * M_PI * g_factor;
	}
	case PK_CORESERSIC: {
		CoreSersicIntegrand f{p.rb, p.a, p.b, p.re, p.nser, bn};
		return 2 * M_PI * integrate_qagi(f, 0.0);
	}
	case PK_KING: {
		KingIntegrand f{p.rc, p.rt, p.a};
		return 2 * M_PI * integrate_qags(f, 0.0, p.rt);
	}
	default: {
		BrokenExpIntegrand f{p.h1, p.h2, p.rb, p.a};
		return 2 * M_PI * integrate_qagi(f, 0.0);
	}
	}
}

// Shape parameter k of a profile kind (the tangent slot order), or null.
PF_HD inline double *shape_param(ProfileParams &p, int k)
{
	switch (p.kind) {
	case PK_SERSIC: return k == 0 ? &p.re : k == 1 ? &p.nser : nullptr;
	case PK_MOFFAT: return k == 0 ? &p.fwhm : k == 1 ? &p.con : nullptr;
	case PK_FERRER: return k == 0 ? &p.rout : k == 1 ? &p.a : k == 2 ? &p.b : nullptr;
	case PK_CORESERSIC:
		return k == 0 ? &p.re : k == 1 ? &p.rb : k == 2 ? &p.nser : k == 3 ? &p.a : k == 4 ? &p.b : nullptr;
	case PK_KING: return k == 0 ? &p.rc : k == 1 ? &p.rt : k == 2 ? &p.a : nullptr;
	case PK_BROKENEXP: return k == 0 ? &p.h1 : k == 1 ? &p.h2 : k == 2 ? &p.rb : k == 3 ? &p.a : nullptr;
	default: return nullptr;
	}
}

// Kinds whose luminosity has no closed-form derivative here: the prologue
// takes central differences of the luminosity (Beta function or QUADPACK) in
// each shape parameter.
PF_HD inline bool lum_by_difference(int kind)
{
	return kind == PK_FERRER || kind == PK_CORESERSIC || kind == PK_KING || kind == PK_BROKENEXP;
}

// Luminosity evaluations of such a profile: slot 0 the profile's own, slots
// 1 + 2k and 2 + 2k the shape parameter k moved by +h and -h.
constexpr int LUM_SLOTS = 1 + 2 * MAX_SHAPE;
PF_HD inline int lum_slots(int kind) { return lum_by_difference(kind) ? 1 + 2 * shape_count(kind) : 0; }

// Luminosity evaluation `slot` of profile p (a lum_by_difference kind); the
// QUADPACK ones are independent, so a batch prologue can run them in
// parallel and hand the values to derive_profile.
PF_HD inline double lum_slot(const ProfileParams &p, int slot)
{
	ProfileParams q = p;
	if (slot > 0) {
		double *v = shape_param(q, (slot - 1) / 2);
		const double v0 = *v, h = 1e-6 * fabs(v0) + 1e-9;
		*v = (slot & 1) ? v0 + h : v0 - h;
	}
	// (the scale radius matters to the Moffat luminosity only)
	return profile_lum(q, q.kind == PK_CORESERSIC ? qgamma(0.5, 2 * q.nser) : 0.0, 0.0);
}

// Scalars of a profile that depend on its shape parameters alone, most of
// the cost of a Sersic profile's prologue: the gamma quantiles (bn =
// qgamma(0.5, 2n) and, for adjusted Sersic profiles, those behind
// rscale_switch, qgamma(1 - n^2/2000, 2n), and rscale_max, qgamma(0.9999,
// 2n)), d bn / d n and d ln L / d n (functions of nser), and the boxiness
// factor r_box and d ln r_box / d B (functions of box).  A host caller keeps
// one per profile and refills only what a changed nser or box invalidates;
// every value comes from the same functions derive_profile uses without it.
struct ShapeMemo {
	double nser = -1, box = NAN;
	double q_half = 0, q_switch = 0, q_max = 0, dbn_dn = 0, dlnL_dn = 0;
	double r_box = 0, dlnI_dbox = 0;
	bool has_half = false, has_switch = false, has_max = false, has_nser_terms = false, has_box = false;
};

// Quantile k of p (0: bn, 1: rscale_switch's, 2: rscale_max's), or 0 where
// derive_profile does not use it.
PF_HD inline double nser_quantile(const ProfileParams &p, int k)
{
	if (p.kind != PK_SERSIC && p.kind != PK_CORESERSIC) return 0;
	if (k == 0) return qgamma(0.5, 2 * p.nser);
	if (p.kind != PK_SERSIC || !p.adjust) return 0;
	if (k == 1) return qgamma(1. - p.nser * p.nser / 2e3, 2 * p.nser);
	return p.rscale_max == 0 ? qgamma(0.9999, 2 * p.nser) : 0.0;
}

// r_box = pi B / (2 Beta(1/B, 1/B)), B = box + 2 (the boxiness factor of
// the luminosity) and d ln r_box / d B.
PF_HD inline double r_box_of(double b2) { return M_PI * b2 / (2 * beta_fn(1 / b2, 1 / b2)); }
PF_HD inline double dln_rbox_dB(double B) { return 1.0 / B + (2.0 / (B * B)) * (digamma(1.0 / B) - digamma(2.0 / B)); }

// b_n solves P(2n, b_n) = 1/2, so d b_n / d n = -2 (dP/da) / (dP/dx) at
// (a, x) = (2n, b_n): dP/dx is the gamma density, dP/da a central difference
// of P at fixed x (two P evaluations instead of two more quantile solves).
PF_HD inline double dbn_dn_of(double nser, double bn)
{
	const double a = 2 * nser, h = 1e-6 * a;
	const double dP_da = (pgamma(bn, a + h) - pgamma(bn, a - h)) / (2 * h);
	const double dP_dx = exp((a - 1) * log(bn) - bn - lgamma(a));
	return -2 * dP_da / dP_dx;
}

// d ln L / d n of a Sersic profile, L = re^2 2 pi n Gamma(2n) e^bn / bn^(2n).
PF_HD inline double sersic_dlnL_dn(double n, double bn, double dbn)
{
	return 1.0 / n + 2.0 * digamma(2 * n) + dbn - 2.0 * log(bn) - 2.0 * n * dbn / bn;
}

// Fills (or keeps, for the same nser and box) what p needs; null for kinds
// with nothing to keep.
inline const ShapeMemo *shape_memo(ShapeMemo &c, const ProfileParams &p)
{
	if (!is_radial_kind(p.kind)) return nullptr;
	if (!(c.nser == p.nser)) {
		const double box = c.box, r_box = c.r_box, dl = c.dlnI_dbox;
		const bool hb = c.has_box;
		c = ShapeMemo();
		c.nser = p.nser;
		c.box = box;
		c.r_box = r_box;
		c.dlnI_dbox = dl;
		c.has_box = hb;
	}
	if (!(c.box == p.box)) {
		c.box = p.box;
		c.r_box = r_box_of(p.box + 2);
		c.dlnI_dbox = dln_rbox_dB(p.box + 2);
		c.has_box = true;
	}
	if (p.kind == PK_SERSIC || p.kind == PK_CORESERSIC) {
		if (!c.has_half) {
			c.q_half = nser_quantile(p, 0);
			c.has_half = true;
		}
		if (!c.has_nser_terms) {
			c.dbn_dn = dbn_dn_of(p.nser, c.q_half);
			c.dlnL_dn = sersic_dlnL_dn(p.nser, c.q_half, c.dbn_dn);
			c.has_nser_terms = true;
		}
	}
	if (p.kind == PK_SERSIC && p.adjust) {
		if (!c.has_switch) {
			c.q_switch = nser_quantile(p, 1);
			c.has_switch = true;
		}
		if (p.rscale_max == 0 && !c.has_max) {
			c.q_max = nser_quantile(p, 2);
			c.has_max = true;
		}
	}
	return &c;
}

// lum_pre (optional, lum_by_difference kinds): the profile's lum_slot values,
// computed beforehand.  nq (optional): shape_memo of p.
PF_HD inline void derive_profile(const ProfileParams &p, const ModelGeom &g, DevProfile &d,
                                 const double *lum_pre = nullptr, const ShapeMemo *nq = nullptr)
{
	d.kind = p.kind;
	d.target = p.convolve ? 0 : 1;
	d.rough = p.rough;
	d.form = SF_GENERAL;
	d.boxy = 0;
	d.img_sx = g.img_sx;
	d.img_sy = g.img_sy;
	d.dlnI_dmag = -0.4 * 2.302585092994045684;
	d.dlnI_dq = d.dlnI_dbox = d.dbn_dn = 0;
	for (int k = 0; k < MAX_SHAPE; k++) d.dlnI_dp[k] = 0;
	d.centre_override = 0;
	d.bn = 0;
	d.axrat = p.axrat;

	if (p.kind == PK_SKY) {
		d.bg = p.bg / (g.finesampling * g.finesampling);
		return;
	}
	if (p.kind == PK_PSF) {
		d.psf_flux = pow(10, -0.4 * (p.mag - g.magzero));
		d.px = p.xcen;
		d.py = p.ycen;
		return;
	}
	if (!is_radial_kind(p.kind)) return;

	d.re = p.re;
	d.nser = p.nser;
	d.box = p.box;
	d.con = p.con;
	d.a = p.a;
	d.b = p.b;
	d.rb = p.rb;
	d.rc = p.rc;
	d.rt = p.rt;
	d.h1 = p.h1;
	d.h2 = p.h2;

	if (p.kind == PK_SERSIC) {
		double inv_exponent = p.nser;
		d.boxy = p.box != 0;
		if (d.boxy) inv_exponent *= (p.box + 2);
		d.invexp = inv_exponent;
		if (almost_eq(inv_exponent, 0.5)) d.form = SF_HALF;
		else if (almost_eq(inv_exponent, 1)) d.form = SF_ONE;
		else if (almost_eq(inv_exponent, 2)) d.form = SF_TWO;
		else if (almost_eq(inv_exponent, 3)) d.form = SF_THREE;
		else if (almost_eq(inv_exponent, 4)) d.form = SF_FOUR;
		else if (almost_eq(inv_exponent, 8)) d.form = SF_EIGHT;
		else if (almost_eq(inv_exponent, 16)) d.form = SF_SIXTEEN;
		else d.form = SF_GENERAL;
		// the specialised forms recompute 1/invexp with the same operands
		d.invexp = d.boxy ? p.nser * (p.box + 2) : p.nser;
	}
	if (p.kind == PK_SERSIC || p.kind == PK_CORESERSIC) d.bn = nq ? nq->q_half : qgamma(0.5, 2 * p.nser);

	// rscale (get_rscale overrides)
	double rscale;
	switch (p.kind) {
	case PK_MOFFAT: rscale = p.fwhm / (2 * sqrt(pow(2, (1 / p.con)) - 1)); break;
	case PK_FERRER: rscale = p.rout; break;
	case PK_KING: rscale = p.rt; break;
	case PK_BROKENEXP: rscale = p.h1 * 4; break;
	default: rscale = p.re; break;
	}
	d.rscale = rscale;

	// lumtot (get_lumtot overrides)
	const double lum = (lum_pre && lum_by_difference(p.kind)) ? lum_pre[0] : profile_lum(p, d.bn, rscale);

	double b2 = p.box + 2;
	double r_box = nq ? nq->r_box : r_box_of(b2);
	double lumtot = lum * p.axrat / r_box;
	double ie = pow(10, -0.4 * (p.mag - g.magzero)) / lumtot;

	double acc = p.acc, rscale_switch = p.rscale_switch, rscale_max = p.rscale_max;
	unsigned resolution = p.resolution;
	if (p.adjust) {
		switch (p.kind) {
		case PK_SERSIC: {
			double fr = p.re * pow((nq ? nq->q_switch : qgamma(1. - p.nser * p.nser / 2e3, 2 * p.nser)) / d.bn, p.nser);
			double rs = ceil(fr);
			rs = pf_fmax(pf_fmin(rs, 20.), 2.);
			rscale_switch = rs / p.re;
			break;
		}
		case PK_MOFFAT: {
			double ff = rscale * sqrt(pow(1 - 0.9999, 1 / (1 - p.con)) - 1);
			double rs = pf_fmax(ff, 1.823 * p.fwhm);
			rscale_switch = pf_fmax(pf_fmin(rs, 20.), 2.) / rscale;
			break;
		}
		case PK_FERRER: rscale_switch = 0.5; break;
		case PK_KING: rscale_switch = 0.5; break;
		default: rscale_switch = 1; break;
		}
		unsigned res = (unsigned)ceil(160 / (rscale_switch * rscale));
		res += res % 2;
		res = res > 16U ? 16U : res;
		res = res < 4U ? 4U : res;
		resolution = res;
		if (rscale_max == 0) {
			switch (p.kind) {
			case PK_SERSIC: {
				double ff = p.re * pow((nq ? nq->q_max : qgamma(0.9999, 2 * p.nser)) / d.bn, p.nser);
				rscale_max = ceil(pf_fmax(ff, 2.) / p.re);
				break;
			}
			case PK_MOFFAT: {
				double ff = rscale * sqrt(pow(1 - 0.9999, 1 / (1 - p.con)) - 1);
				rscale_max = ceil(pf_fmax(ff, 2.) / rscale);
				break;
			}
			case PK_FERRER: rscale_max = 1; break;
			case PK_KING: rscale_max = 1.5; break;
			default: rscale_max = 100; break;
			}
		}
		if (p.kind == PK_SERSIC) {
			acc /= sqrt(p.nser);
			acc = pf_fmax(0.1, acc) / p.axrat;
		}
		else if (p.kind == PK_MOFFAT) {
			acc = 0.1 / p.axrat;
		}
	}
	d.acc = acc;
	d.resolution = resolution;
	d.max_rec = p.max_recursions;
	d.r_switch = rscale_switch * rscale;
	d.r_max = rscale_max > 0 ? rscale_max * rscale : 0;

	double angrad = fmod(p.ang + 90, 360.) * M_PI / 180.;
	d.cos_ang = cos(angrad);
	d.sin_ang = sin(angrad);
	d.cos_q = d.cos_ang / p.axrat;
	d.sin_q = d.sin_ang / p.axrat;

	double rescale_factor = 1;
	if (p.kind == PK_SERSIC && p.adjust && p.rescale_flux) {
		double flux_r = d.bn * pow(rscale_max / p.re, 1 / p.nser);
		flux_r = pgamma(flux_r, 2 * p.nser);
		rescale_factor = 1 / flux_r;
	}
	double flux_scale = g.sx * g.sy * ie;
	if (p.kind == PK_SERSIC && p.rescale_flux) flux_scale *= rescale_factor;
	d.flux_scale = flux_scale;
	d.cx = p.xcen + g.offx * g.sx;
	d.cy = p.ycen + g.offy * g.sy;
	d.centre_override = (p.kind == PK_SERSIC && p.adjust && p.nser > 1) ? 1 : 0;
	d.king_t = (p.kind == PK_KING) ? 1 / pow(1 + pow(p.rt / p.rc, 2), 1 / p.a) : 0;

	// d log(flux_scale) / d parameter, used by the adjoint.
	// flux_scale = sx sy 10^(-0.4(mag - mz)) r_box / (L axrat)
	d.dlnI_dq = -1.0 / p.axrat;
	d.dlnI_dbox = nq ? nq->dlnI_dbox : dln_rbox_dB(b2);
	if (p.kind == PK_SERSIC || p.kind == PK_CORESERSIC) d.dbn_dn = nq ? nq->dbn_dn : dbn_dn_of(p.nser, d.bn);
	if (p.kind == PK_SERSIC) {
		d.dlnI_dp[0] = -2.0 / p.re;  // re
		d.dlnI_dp[1] = -(nq ? nq->dlnL_dn : sersic_dlnL_dn(p.nser, d.bn, d.dbn_dn));  // nser
	}
	else if (p.kind == PK_MOFFAT) {
		// L = rscale^2 pi / (con - 1), rscale = fwhm / (2 sqrt(2^(1/con) - 1))
		double c = p.con;
		double t = pow(2.0, 1.0 / c);
		double drs_dc_over_rs = 0.5 * t * log(2.0) / (c * c * (t - 1.0));
		d.dlnI_dp[0] = -2.0 / p.fwhm;                          // fwhm
		d.dlnI_dp[1] = -(2.0 * drs_dc_over_rs - 1.0 / (c - 1.0));  // con
	}
	else {
		// Ferrer (Beta function), core-Sersic, King and broken exponential
		// (QUADPACK): central differences of the same FP64 luminosity, so the
		// gradient differentiates exactly the normalisation the image uses.
		for (int k = 0; k < shape_count(p.kind); k++) {
			ProfileParams q = p;
			const double v0 = *shape_param(q, k), h = 1e-6 * fabs(v0) + 1e-9;
			const double lp = lum_pre ? lum_pre[1 + 2 * k] : lum_slot(p, 1 + 2 * k);
			const double lm = lum_pre ? lum_pre[2 + 2 * k] : lum_slot(p, 2 + 2 * k);
			d.dlnI_dp[k] = -(log(lp) - log(lm)) / (2 * h);
		}
	}
}

}  // namespace pf
