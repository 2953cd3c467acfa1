// ProFit's fit space around the likelihood, for batches of sampler proposals.
//
// A sampler moves a vector parm of fitted values; ProFit's R layer turns it
// into model parameters (profitRemakeModellist, R/profitRemakeModelList.R:
// 27-166) and adds normal priors (profitMakePriors, R/profitUtility.R:
// 124-176) to the likelihood: LP = LL + priors (R/profitLikeModel.R:225-240,
// 342).  Here the same mapping runs per proposal on the device (one thread
// per proposal, or on the host for the few-proposal path), and the chain rule
// turns the adjoint's d LL / d theta into d LP / d parm.
//
// The mapping is a list of entries in unlist(modellist) order, each one
// model parameter.  For one proposal (R's steps, in its order):
//   1. parmin = unlist(modellist); parmin[fitted] = parm
//   2. fitted entries with tolog: parmin = 10^parmin
//   3. offsets: xcen += offset[1], ycen += offset[2], ang += offset[3],
//      then size parameters (re, fwhm, rb, rout, rc, rt, xcen, ycen) *=
//      offset[4] (steps 3 and 3b apply to every entry, fitted or not)
//   4. tied entries (tofit NA) take the entry before: parmin[i] = parmin[i-1]
//   5. interval limits: theta = max(lo, min(hi, value))
//   6. tied entries again take the entry before (after its clamp)
//   7. parm_out: fitted entries' theta with the offsets taken off
//      (x - offset[1] ... then / offset[4]) and log10 where unlogged
// Steps 4-6 in one pass: an untied entry's theta is its clamped value, a
// tied entry's theta is the theta of the entry before it.
//
// Derivatives: d theta_i / d parm_i = (theta_i ln 10 if tolog, else 1)
//   x (offset[4] for size entries) x (0 where the clamp moved the value),
// and a tied entry's d LP / d theta flows to the entry before it.  Priors:
// dnorm(x, mean, sigma, log) with x = theta (or log10 theta and log10 mean
// with the prior's tolog), d/d theta = -(x - mean) / sigma^2 (/ (theta ln 10)).
#pragma once

#include <cmath>
#include <cstdint>

#include "profiles.cuh"

namespace pf {

enum FitFlag : int32_t { FIT_FIXED = 0, FIT_FREE = 1, FIT_TIED = -1 };
enum FitOffsetBits : int32_t { OFS_X = 1, OFS_Y = 2, OFS_ANG = 4, OFS_SIZE = 8 };

struct FitEntry {
	int32_t fit;          // FIT_FREE, FIT_FIXED or FIT_TIED (R's NA: takes the entry before)
	int32_t tolog;        // a free entry is fitted as log10 of its value
	int32_t fit_index;    // position in parm (free entries), else -1
	int32_t ref_index;    // position among the model's gradient references (free and tied), else -1
	int32_t offset_bits;  // OFS_* shifts that apply to this parameter (by its name)
	int32_t prior;        // 1: normal prior on this entry
	int32_t prior_tolog;  // the prior is on log10 theta
	int32_t limited;      // an interval applies (lo, hi)
	double init;          // model-space value (unlist(modellist))
	double lo, hi;        // interval limits
	double prior_mean, prior_sigma;
};

// offset = (x, y, ang, size); ang 0 and size 1 stand for R's NA.
struct FitOffset {
	double x, y, ang, size;
};

struct FitSpaceView {
	const FitEntry *e;
	int n, nfit, nrefs;
	FitOffset off;
};

constexpr double FIT_LN10 = 2.302585092994045684;
constexpr double FIT_HALF_LN_2PI = 0.918938533204672741780329736406;

// Value of an entry after steps 1-3 (before ties and clamps).
PF_HD inline double fit_pre_value(const FitEntry &e, const FitOffset &off, const double *parm)
{
	double v = e.init;
	if (e.fit == FIT_FREE) {
		v = parm[e.fit_index];
		if (e.tolog) v = pow(10.0, v);
	}
	if (e.offset_bits & OFS_X) v += off.x;
	if (e.offset_bits & OFS_Y) v += off.y;
	if (e.offset_bits & OFS_ANG) v += off.ang;
	if (e.offset_bits & OFS_SIZE) v *= off.size;
	return v;
}

// R's max(lo, min(hi, v, na.rm = TRUE), na.rm = TRUE); fmin/fmax drop a NaN
// operand the same way.
PF_HD inline double fit_clamp(const FitEntry &e, double v) { return e.limited ? fmax(e.lo, fmin(e.hi, v)) : v; }

// Steps 1-7 for one proposal: theta of every free and tied entry into
// values[ref_index], the fitted vector R hands back into parm_out[fit_index]
// (either may be null); returns the log prior.
PF_HD inline double fit_remake(const FitSpaceView &fs, const double *parm, double *values, double *parm_out)
{
	double prev = 0.0, lp = 0.0;
	for (int i = 0; i < fs.n; i++) {
		const FitEntry &e = fs.e[i];
		const double theta = e.fit == FIT_TIED ? prev : fit_clamp(e, fit_pre_value(e, fs.off, parm));
		prev = theta;
		if (values && e.ref_index >= 0) values[e.ref_index] = theta;
		if (parm_out && e.fit == FIT_FREE) {
			double o = theta;
			if (e.offset_bits & OFS_X) o -= fs.off.x;
			if (e.offset_bits & OFS_Y) o -= fs.off.y;
			if (e.offset_bits & OFS_ANG) o -= fs.off.ang;
			if (e.offset_bits & OFS_SIZE) o /= fs.off.size;
			parm_out[e.fit_index] = e.tolog ? log10(o) : o;
		}
		if (e.prior) {
			const double x = e.prior_tolog ? log10(theta) : theta;
			const double mu = e.prior_tolog ? log10(e.prior_mean) : e.prior_mean;
			const double z = (x - mu) / e.prior_sigma;
			lp += -(FIT_HALF_LN_2PI + log(e.prior_sigma)) - 0.5 * z * z;
		}
	}
	return lp;
}

// d LP / d parm from d LL / d theta of the references (grad_ll[ref_index])
// at the values fit_remake wrote; dlp[fit_index] for every free entry.
PF_HD inline void fit_chain(const FitSpaceView &fs, const double *parm, const double *values, const double *grad_ll,
                            double *dlp)
{
	double carry = 0.0;  // d LP / d theta flowing from tied entries to the entry before
	for (int i = fs.n - 1; i >= 0; i--) {
		const FitEntry &e = fs.e[i];
		if (e.fit == FIT_FIXED) {  // does not move with parm: what flows into it is dropped
			carry = 0.0;
			continue;
		}
		const double theta = values[e.ref_index];
		double g = grad_ll[e.ref_index] + carry;
		if (e.prior) {
			const double x = e.prior_tolog ? log10(theta) : theta;
			const double mu = e.prior_tolog ? log10(e.prior_mean) : e.prior_mean;
			double d = -(x - mu) / (e.prior_sigma * e.prior_sigma);
			if (e.prior_tolog) d /= theta * FIT_LN10;
			g += d;
		}
		if (e.fit == FIT_TIED) {
			carry = g;
			continue;
		}
		carry = 0.0;
		const double pre = fit_pre_value(e, fs.off, parm);
		double f = fit_clamp(e, pre) != pre ? 0.0 : 1.0;
		if (e.tolog) f *= pow(10.0, parm[e.fit_index]) * FIT_LN10;
		if (e.offset_bits & OFS_SIZE) f *= fs.off.size;
		dlp[e.fit_index] = g * f;
	}
}

// Per proposal: LP = LL + log prior, d LP / d parm; an invalid proposal
// (LL = -inf) gets LP = -inf and a zero gradient.  out: [batch] LP,
// [batch][nfit] gradient, [batch] LL (parm_out is written by the remake).
PF_HD inline void fit_finish_one(const FitSpaceView &fs, const double *parm, const double *values, double ll,
                                 const double *grad_ll, double *lp, double *dlp, double *ll_out)
{
	*ll_out = ll;
	if (!(ll > -INFINITY)) {
		*lp = -INFINITY;
		for (int j = 0; j < fs.nfit; j++) dlp[j] = 0.0;
		return;
	}
	*lp = ll + fit_remake(fs, parm, nullptr, nullptr);
	fit_chain(fs, parm, values, grad_ll, dlp);
}

}  // namespace pf
