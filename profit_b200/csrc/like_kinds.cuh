// The other likelihoods of ProFit's profitLikeModel (R/profitLikeModel.R:
// 257-332) and their adjoint seeds dLL/dmodel.  With x = (data - model)/sigma
// over the region's n pixels:
//
//   chisq  LL = log dchisq(X2, n),  X2 = sum x^2           (R/profitLikeModel.R:277-280)
//          dLL/dm_i = ((n/2 - 1)/X2 - 1/2) * (-2 x_i / sigma_i)
//   t      LL = sum log dt(x_i, nu),  nu = max(1, 2 v/(v - 1)), v the sample
//          variance of x (R/profitLikeModel.R:281-287); nu depends on the
//          model, so dLL/dm_i = (-1/sigma_i) [ -(nu+1) x_i/(nu + x_i^2)
//          + (dLL/dnu)(dnu/dv) 2 (x_i - mean)/(n - 1) ], dnu/dv = -2/(v-1)^2
//          (0 where nu is clamped at 1, and the normal form where v = 1)
//   pois   LL = -sum (s m_i - s d_i log(s m_i)), s = max(|d|/sigma^2) when that
//          lies outside [0.1, 10], else 1 (R/profitLikeModel.R:321-327)
//          dLL/dm_i = s (d_i/m_i - 1)
//
// The skew-t ("st") form fits its own parameters with LaplacesDemon and the
// sn package and is not provided.
//
// Passes, all over a fixed grid with Neumaier sums (deterministic):
//   1. statistics per image: chisq (X2, n), t (sum x, sum x^2, n),
//      pois (max |d|/sigma^2, n);
//   2. per-pixel terms: t (sum log1p terms, sum dnu terms), pois (LL terms and
//      the seed); chisq writes its seed here;
//   3. t only: the seed, once dLL/dnu is known.
// The closed forms use lgamma; R evaluates dchisq and dt with Loader's
// saddle-point expansions, which agree with them to ~1e-10 absolute even at
// 1e5 pixels.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"
#include "like.cuh"
#include "specfun.cuh"

namespace pf {

constexpr int LIKE_STATS = 4;  // doubles per image of the statistics record

// Student-t form from the pass-1 sums: nu, the mean, the sample variance.
struct TParams {
	double nu, mean, var, n;
	bool normal, clamped;
};

__host__ __device__ inline TParams t_params(const double *st)
{
	TParams p;
	p.n = st[2];
	p.mean = st[0] / p.n;
	p.var = (st[1] - st[0] * p.mean) / (p.n - 1);
	p.normal = false;
	p.clamped = false;
	if (!(p.n > 1) || p.var == 1.0) {
		p.nu = INFINITY;  // R: min(Inf, NA or Inf) -> Inf
		p.normal = true;
	}
	else {
		const double raw = 2 * p.var / (p.var - 1);
		if (raw < 1) {
			p.nu = 1;
			p.clamped = true;
		}
		else {
			p.nu = raw;
		}
	}
	return p;
}

// Pass 1: per-block partial statistics, partials[b][block] = (s0, s1, s2, max);
// s2 is the region's pixel count for every kind.
template <int KIND>
__global__ void k_like_stats(const double *__restrict__ model, const double *__restrict__ data,
                             const double *__restrict__ sigma, const uint8_t *__restrict__ region, int n,
                             int data_batch_stride, double *__restrict__ partials)
{
	pdl_enter();
	const int b = blockIdx.y;
	model += (size_t)b * n;
	data += (size_t)b * data_batch_stride;
	sigma += (size_t)b * data_batch_stride;
	if (region) region += (size_t)b * data_batch_stride;
	Neumaier a0{0, 0}, a1{0, 0}, a2{0, 0};
	double mx = 0;
	for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		if (region && !region[k]) continue;
		const double s = sigma[k], d = data[k];
		if (KIND == LIKE_POIS) {
			mx = fmax(mx, fabs(d) / (fabs(s) * fabs(s)));
			neumaier_add(a2, 1.0);
			continue;
		}
		const double x = (d - model[k]) / s;
		if (KIND == LIKE_CHISQ) {
			neumaier_add(a0, x * x);
		}
		else {
			neumaier_add(a0, x);
			neumaier_add(a1, x * x);
		}
		neumaier_add(a2, 1.0);
	}
	a0 = neumaier_block(a0);
	__syncthreads();
	a1 = neumaier_block(a1);
	__syncthreads();
	a2 = neumaier_block(a2);
	__shared__ double s_mx[32];
	for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
	if ((threadIdx.x & 31) == 0) s_mx[threadIdx.x >> 5] = mx;
	__syncthreads();
	if (threadIdx.x == 0) {
		for (int w = 1; w < (int)(blockDim.x >> 5); w++) mx = fmax(mx, s_mx[w]);
		double *o = partials + ((size_t)b * gridDim.x + blockIdx.x) * 4;
		o[0] = a0.s + a0.c;
		o[1] = a1.s + a1.c;
		o[2] = a2.s + a2.c;
		o[3] = mx;
	}
}

// Merges the pass-1 partials of each image (blockIdx.x) in block order.
__global__ void k_like_stats_final(const double *__restrict__ partials, int nparts, double *__restrict__ stats)
{
	pdl_enter();
	const int b = blockIdx.x;
	if (threadIdx.x != 0) return;
	Neumaier a0{0, 0}, a1{0, 0}, a2{0, 0};
	double mx = 0;
	for (int k = 0; k < nparts; k++) {
		const double *p = partials + ((size_t)b * nparts + k) * 4;
		neumaier_add(a0, p[0]);
		neumaier_add(a1, p[1]);
		neumaier_add(a2, p[2]);
		mx = fmax(mx, p[3]);
	}
	double *st = stats + (size_t)b * LIKE_STATS;
	st[0] = a0.s + a0.c;
	st[1] = a1.s + a1.c;
	st[2] = a2.s + a2.c;
	st[3] = mx;
}

// Pass 2: per-pixel terms (partials[b][block] = (s0, s1)) and, for chisq and
// pois, the adjoint seed.
template <int KIND>
__global__ void k_like_terms(const double *__restrict__ model, const double *__restrict__ data,
                             const double *__restrict__ sigma, const uint8_t *__restrict__ region, int n,
                             int data_batch_stride, const double *__restrict__ stats, double2 *__restrict__ partials,
                             float *__restrict__ wseed)
{
	pdl_enter();
	const int b = blockIdx.y;
	model += (size_t)b * n;
	data += (size_t)b * data_batch_stride;
	sigma += (size_t)b * data_batch_stride;
	if (region) region += (size_t)b * data_batch_stride;
	if (wseed) wseed += (size_t)b * n;
	const double *st = stats + (size_t)b * LIKE_STATS;
	Neumaier a0{0, 0}, a1{0, 0};
	double coef = 0, scale = 1;
	TParams tp{};
	if (KIND == LIKE_CHISQ) coef = (st[2] / 2 - 1) / st[0] - 0.5;  // st[2]: pixel count
	if (KIND == LIKE_POIS) scale = (st[3] < 0.1 || st[3] > 10) ? st[3] : 1.0;
	if (KIND == LIKE_T) tp = t_params(st);
	for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		const bool use = !region || region[k];
		const double m = model[k], d = data[k], s = sigma[k];
		float seed = 0.0f;
		if (use) {
			if (KIND == LIKE_CHISQ) {
				const double x = (d - m) / s;
				seed = (float)(coef * (-2.0 * x / s));
			}
			else if (KIND == LIKE_POIS) {
				const double sm = scale * m;
				neumaier_add(a0, -(sm - scale * d * log(sm)));
				seed = (float)(scale * (d / m - 1.0));
			}
			else {  // t
				const double x = (d - m) / s;
				if (tp.normal) {
					neumaier_add(a0, -(LN_SQRT_2PI + 0.5 * x * x));
				}
				else {
					const double q = x * x / tp.nu;
					const double l1 = log1p(q);
					neumaier_add(a0, -0.5 * (tp.nu + 1) * l1);
					neumaier_add(a1, -0.5 * l1 + 0.5 * (tp.nu + 1) * q / (tp.nu + x * x));
				}
			}
		}
		if (wseed && KIND != LIKE_T) wseed[k] = seed;
	}
	a0 = neumaier_block(a0);
	__syncthreads();
	a1 = neumaier_block(a1);
	if (threadIdx.x == 0) {
		partials[((size_t)b * gridDim.x + blockIdx.x) * 2] = make_double2(a0.s, a0.c);
		partials[((size_t)b * gridDim.x + blockIdx.x) * 2 + 1] = make_double2(a1.s, a1.c);
	}
}

// LL per image from the pass-2 partials; for t also the coefficient
// (dLL/dnu)(dnu/dv) of pass 3 into coef[b].
template <int KIND>
__global__ void k_like_terms_final(const double2 *__restrict__ partials, int nparts, const double *__restrict__ stats,
                                   double *__restrict__ out, double *__restrict__ coef)
{
	pdl_enter();
	const int b = blockIdx.x;
	if (threadIdx.x != 0) return;
	Neumaier a0{0, 0}, a1{0, 0};
	for (int k = 0; k < nparts; k++) {
		const double2 p0 = partials[((size_t)b * nparts + k) * 2], p1 = partials[((size_t)b * nparts + k) * 2 + 1];
		a0 = neumaier_merge(a0, Neumaier{p0.x, p0.y});
		a1 = neumaier_merge(a1, Neumaier{p1.x, p1.y});
	}
	const double *st = stats + (size_t)b * LIKE_STATS;
	const double s0 = a0.s + a0.c, s1 = a1.s + a1.c;
	if (KIND == LIKE_CHISQ) {
		const double X2 = st[0], k = st[2];
		out[b] = (k / 2 - 1) * log(X2) - X2 / 2 - (k / 2) * log(2.0) - lgamma(k / 2);
	}
	else if (KIND == LIKE_POIS) {
		out[b] = s0;
	}
	else {
		const TParams tp = t_params(st);
		if (tp.normal) {
			out[b] = s0;
			if (coef) coef[b] = 0;
		}
		else {
			const double nu = tp.nu, n = tp.n;
			const double c0 = lgamma((nu + 1) / 2) - lgamma(nu / 2) - 0.5 * log(nu * M_PI);
			out[b] = n * c0 + s0;
			// dLL/dnu = n [psi((nu+1)/2)/2 - psi(nu/2)/2 - 1/(2 nu)] + s1
			const double dll_dnu = n * (0.5 * digamma((nu + 1) / 2) - 0.5 * digamma(nu / 2) - 0.5 / nu) + s1;
			const double dnu_dv = tp.clamped ? 0.0 : -2.0 / ((tp.var - 1) * (tp.var - 1));
			if (coef) coef[b] = dll_dnu * dnu_dv;
		}
	}
}

// Pass 3 (t): the seed dLL/dm_i.
__global__ void k_like_t_seed(const double *__restrict__ model, const double *__restrict__ data,
                              const double *__restrict__ sigma, const uint8_t *__restrict__ region, int n,
                              int data_batch_stride, const double *__restrict__ stats, const double *__restrict__ coef,
                              float *__restrict__ wseed)
{
	pdl_enter();
	const int b = blockIdx.y;
	model += (size_t)b * n;
	data += (size_t)b * data_batch_stride;
	sigma += (size_t)b * data_batch_stride;
	if (region) region += (size_t)b * data_batch_stride;
	wseed += (size_t)b * n;
	const TParams tp = t_params(stats + (size_t)b * LIKE_STATS);
	const double c = coef[b];
	for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		float seed = 0.0f;
		if (!region || region[k]) {
			const double s = sigma[k], x = (data[k] - model[k]) / s;
			double dldx;
			if (tp.normal) dldx = -x;
			else dldx = -(tp.nu + 1) * x / (tp.nu + x * x) + c * 2 * (x - tp.mean) / (tp.n - 1);
			seed = (float)(-dldx / s);
		}
		wseed[k] = seed;
	}
}

}  // namespace pf
