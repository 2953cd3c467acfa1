// FP32 rendering with forward tangents, the fast form behind the adjoint.
//
// Same work decomposition as render64.cu (pixel pass + per-level subsample
// warps over the device work queue), but per-pixel arithmetic is FP32 and
// every evaluation also returns the partial derivatives of the profile value
// with respect to profile coordinates and shape parameters.  For each
// radial profile and drawing pixel the pass stores NTAN sums
//   J0 = sum w f,   J1 = sum w df/dx',  J2 = sum w df/dy',
//   J3 = sum w df/dx' y',  J4 = sum w df/dy' x',  J5 = sum w df/dy' y',
//   J6..J8 = sum w df/d(shape parameter 1..3)
// over the pixel's quadrature points (w = sub-cell weights of the chosen
// subsampling).  The gradient of logL with respect to xcen, ycen, mag, ang,
// axrat and the shape parameters is a fixed linear combination of
// sum_pixels g(pixel) J_k(pixel), g being the adjoint of the convolution
// applied to dlogL/dmodel; the combination is done in FP64 on the host.
//
// FP64 is kept where FP32 would lose the answer:
//  - pixel and sub-cell coordinates relative to the profile centre are
//    formed in FP64 before rounding to FP32 (positions on a 2000-pixel
//    image would otherwise carry 1e-4 pixel errors), and sub-cell bounds
//    stay FP64 in the work queue (centre cells reach 8^-10 pixel);
//  - cells from recursion level 3 on (only the Sersic central cusp with
//    max_recursions = 10 gets there) are evaluated in FP64.

#include "common.cuh"
#include "conv.cuh"
#include "conv2.cuh"
#include "launch.h"
#include "like.cuh"

namespace pf {

template <class T>
struct Tan {
	T f, fx, fy, s1, s2, s3;
};

template <class T>
__device__ __forceinline__ T t_exp(T x);
template <>
__device__ __forceinline__ float t_exp<float>(float x) { return expf(x); }
template <>
__device__ __forceinline__ double t_exp<double>(double x) { return exp(x); }
template <class T>
__device__ __forceinline__ T t_log(T x);
template <>
__device__ __forceinline__ float t_log<float>(float x) { return logf(x); }
template <>
__device__ __forceinline__ double t_log<double>(double x) { return log(x); }
template <class T>
__device__ __forceinline__ T t_pow(T x, T y);
template <>
__device__ __forceinline__ float t_pow<float>(float x, float y) { return powf(x, y); }
template <>
__device__ __forceinline__ double t_pow<double>(double x, double y) { return pow(x, y); }
template <class T>
__device__ __forceinline__ T t_sqrt(T x);
template <>
__device__ __forceinline__ float t_sqrt<float>(float x) { return sqrtf(x); }
template <>
__device__ __forceinline__ double t_sqrt<double>(double x) { return sqrt(x); }

// x * log(x) with the limit 0 at x = 0
template <class T>
__device__ __forceinline__ T xlogx(T x)
{
	return x > T(0) ? x * t_log<T>(x) : T(0);
}

// Sersic: f = exp(-bn (base^(1/(n B)) - 1)), base = |x/re|^B + |y/re|^B.
// Shape partials: s1 = df/dre, s2 = df/dnser (including dbn/dnser),
// s3 = df/dbox.
template <class T>
__device__ __forceinline__ Tan<T> sersic_tan(const FProfile &p, T xp, T yp)
{
	Tan<T> t;
	const T re = (T)p.re, B = (T)p.B, n = (T)p.nser, bn = (T)p.bn;
	const T u = fabs(xp) / re, v = fabs(yp) / re;
	T uB, vB, base;
	if (B == T(2)) {
		uB = u * u;
		vB = v * v;
	}
	else {
		uB = t_pow<T>(u, B);
		vB = t_pow<T>(v, B);
	}
	base = uB + vB;
	if (!(base > T(0))) {
		t.f = t_exp<T>(bn);
		t.fx = t.fy = t.s1 = t.s2 = t.s3 = T(0);
		return t;
	}
	const T inv_nB = T(1) / (n * B);
	const T lnb = t_log<T>(base);
	const T rf = t_exp<T>(lnb * inv_nB);
	const T f = t_exp<T>(-bn * (rf - T(1)));
	const T dfdrf = -bn * f;
	const T g = dfdrf * rf * inv_nB / base;  // df/dbase
	// dbase/dx' = B * uB / x'
	t.f = f;
	t.fx = xp != T(0) ? g * B * uB / xp : T(0);
	t.fy = yp != T(0) ? g * B * vB / yp : T(0);
	t.s1 = -dfdrf * rf / (n * re);
	t.s2 = dfdrf * (-rf * lnb * inv_nB / n) - (rf - T(1)) * f * (T)p.dbn_dn;
	const T dbase_dB = (u > T(0) ? uB * t_log<T>(u) : T(0)) + (v > T(0) ? vB * t_log<T>(v) : T(0));
	t.s3 = dfdrf * rf * inv_nB * (dbase_dB / base - lnb / B);
	return t;
}

// Moffat: f = (1 + (r/rscale)^2)^-con, r = boxy radius.  Shape partials:
// s1 = df/dfwhm, s2 = df/dcon, s3 = df/dbox.
template <class T>
__device__ __forceinline__ Tan<T> moffat_tan(const FProfile &p, T xp, T yp)
{
	Tan<T> t;
	const T B = (T)p.B, rs = (T)p.rscale, con = (T)p.con;
	const T ax = fabs(xp), ay = fabs(yp);
	T r, drdx, drdy, drdB;
	if (B == T(2)) {
		r = t_sqrt<T>(xp * xp + yp * yp);
		drdx = r > T(0) ? xp / r : T(0);
		drdy = r > T(0) ? yp / r : T(0);
		const T S = xp * xp + yp * yp;
		drdB = S > T(0) ? r * ((xlogx<T>(ax) * ax + xlogx<T>(ay) * ay) / (B * S) - t_log<T>(S) / (B * B)) : T(0);
	}
	else {
		const T xB = t_pow<T>(ax, B), yB = t_pow<T>(ay, B);
		const T S = xB + yB;
		r = S > T(0) ? t_pow<T>(S, T(1) / B) : T(0);
		drdx = (r > T(0) && xp != T(0)) ? (xB / S) * r / xp : T(0);
		drdy = (r > T(0) && yp != T(0)) ? (yB / S) * r / yp : T(0);
		T lx = ax > T(0) ? xB * t_log<T>(ax) : T(0);
		T ly = ay > T(0) ? yB * t_log<T>(ay) : T(0);
		drdB = S > T(0) ? r * ((lx + ly) / (B * S) - t_log<T>(S) / (B * B)) : T(0);
	}
	const T rf = r / rs;
	const T q = T(1) + rf * rf;
	const T lq = t_log<T>(q);
	const T f = t_exp<T>(-con * lq);
	const T dfdrf = -T(2) * con * rf * f / q;
	t.f = f;
	t.fx = dfdrf * drdx / rs;
	t.fy = dfdrf * drdy / rs;
	t.s1 = dfdrf * (-rf) * (T)p.a;          // a holds 1/fwhm for Moffat
	t.s2 = -lq * f + dfdrf * (-rf) * (T)p.b; // b holds dln(rscale)/dcon
	t.s3 = dfdrf * drdB / rs;
	return t;
}

template <class T>
__device__ __forceinline__ T boxy_r_t(const FProfile &p, T x, T y)
{
	if (p.B == 2.0f) return t_sqrt<T>(x * x + y * y);
	T B = (T)p.B;
	return t_pow<T>(t_pow<T>(fabs(x), B) + t_pow<T>(fabs(y), B), T(1) / B);
}

// Value-only evaluation for the profiles without a hand-written tangent.
template <class T>
__device__ __forceinline__ Tan<T> other_tan(const FProfile &p, T xp, T yp)
{
	Tan<T> t;
	t.fx = t.fy = t.s1 = t.s2 = t.s3 = T(0);
	T r = boxy_r_t<T>(p, xp, yp);
	switch (p.kind) {
	case PK_FERRER: {
		T rf = r / (T)p.rscale;
		t.f = rf < T(1) ? t_pow<T>(T(1) - t_pow<T>(rf, T(2) - (T)p.b), (T)p.a) : T(0);
		break;
	}
	case PK_CORESERSIC: {
		T a = (T)p.a;
		t.f = t_pow<T>(T(1) + t_pow<T>(r / (T)p.rb, -a), (T)p.b / a) *
		      t_exp<T>(-(T)p.bn * t_pow<T>((t_pow<T>(r, a) + t_pow<T>((T)p.rb, a)) / t_pow<T>((T)p.re, a),
		                                   T(1) / ((T)p.nser * a)));
		break;
	}
	case PK_KING: {
		T a = (T)p.a;
		t.f = r < (T)p.rt ? t_pow<T>(T(1) / t_pow<T>(T(1) + (r / (T)p.rc) * (r / (T)p.rc), T(1) / a) - (T)p.king_t, a)
		                  : T(0);
		break;
	}
	case PK_BROKENEXP: {
		T a = (T)p.a, base = r - (T)p.rb;
		T expo = T(1) / (T)p.h1 - T(1) / (T)p.h2;
		if (a * base < T(40)) base = t_log<T>(T(1) + t_exp<T>(a * base)) / a;
		t.f = t_exp<T>(-r / (T)p.h1 + expo * base);
		break;
	}
	default: t.f = T(0);
	}
	return t;
}

template <class T>
__device__ __forceinline__ Tan<T> eval_tan(const FProfile &p, T xp, T yp)
{
	if (p.kind == PK_SERSIC) return sersic_tan<T>(p, xp, yp);
	if (p.kind == PK_MOFFAT) return moffat_tan<T>(p, xp, yp);
	return other_tan<T>(p, xp, yp);
}

template <class T>
__device__ __forceinline__ T eval_val(const FProfile &p, T xp, T yp)
{
	return eval_tan<T>(p, xp, yp).f;
}

// How one drawing pixel is integrated for one radial profile
// (radial.cpp:321-339): not at all (beyond rscale_max), by one evaluation,
// or by subsampling.  The forward pass and the recomputing adjoint must agree
// pixel for pixel, so this is written with round-to-nearest intrinsics,
// which no contraction or reassociation can change between kernels.
enum PixelDecision : int { PD_ZERO = 0, PD_DIRECT = 1, PD_SUBSAMPLE = 2 };

__device__ __forceinline__ int pixel_decision32(const FProfile &p, double x, double y, float &xp, float &yp)
{
	const float dx = __double2float_rn(__dsub_rn(x, p.cx));
	const float dy = __double2float_rn(__dsub_rn(y, p.cy));
	xp = __fadd_rn(__fmul_rn(dx, p.cos_ang), __fmul_rn(dy, p.sin_ang));
	yp = __fadd_rn(__fmul_rn(-dx, p.sin_q), __fmul_rn(dy, p.cos_q));
	const float r = __fsqrt_rn(__fadd_rn(__fmul_rn(xp, xp), __fmul_rn(yp, yp)));
	if (p.r_max > 0.f && r > p.r_max) return PD_ZERO;
	if (p.rough || r > p.r_switch) return PD_DIRECT;
	return PD_SUBSAMPLE;
}

__device__ __forceinline__ void tan_to_j(const Tan<float> &t, float xp, float yp, float w, float *j)
{
	j[0] += w * t.f;
	j[1] += w * t.fx;
	j[2] += w * t.fy;
	j[3] += w * t.fx * yp;
	j[4] += w * t.fy * xp;
	j[5] += w * t.fy * yp;
	j[6] += w * t.s1;
	j[7] += w * t.s2;
	j[8] += w * t.s3;
}

// One thread per drawing pixel and per batch entry (blockIdx.z).  `model_of`
// maps the profile range of each batch entry; profiles are FProfile records.
__global__ void k_pixels32(const FProfile *__restrict__ profiles, const int *__restrict__ prof_begin,
                           unsigned width, unsigned height, double sx, double sy, float *__restrict__ img_conv,
                           float *__restrict__ img_plain, float *__restrict__ jac, QueueSet q)
{
	const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
	const unsigned j = blockIdx.y * blockDim.y + threadIdx.y;
	const int b = blockIdx.z;
	if (i >= width || j >= height) return;
	const size_t npix = (size_t)width * height;
	const uint32_t pix = i + j * width;
	const int p0 = prof_begin[b], p1 = prof_begin[b + 1];
	float acc[2] = {0.f, 0.f};
	const double half_xbin = sx / 2., half_ybin = sy / 2.;
	const double y = half_ybin + j * sx;
	const double x = half_xbin + i * sy;

	for (int pi = p0; pi < p1; pi++) {
		const FProfile &p = profiles[pi];
		if (p.kind == PK_SKY) {
			acc[p.target] += p.flux_scale;  // sky value is kept in flux_scale
			continue;
		}
		if (!is_radial_kind(p.kind)) continue;
		float xp, yp;
		const int decision = pixel_decision32(p, x, y, xp, yp);
		float jl[NTAN];
#pragma unroll
		for (int k = 0; k < NTAN; k++) jl[k] = 0.f;
		if (decision == PD_ZERO) {
			// zero
		}
		else if (decision == PD_DIRECT) {
			Tan<float> t = eval_tan<float>(p, xp, yp);
			acc[p.target] += p.flux_scale * t.f;
			tan_to_j(t, xp, yp, 1.0f, jl);
		}
		else {
			unsigned res = p.resolution, max_rec = p.max_rec;
			if (p.centre_override && fabs(x - p.cx) < p.img_sx && fabs(y - p.cy) < p.img_sy) {
				res = 8;
				max_rec = 10;
			}
			SubItem it;
			const double ddx = x - p.cx, ddy = y - p.cy;
			it.x0 = ddx - half_xbin;
			it.x1 = ddx + half_xbin;
			it.y0 = ddy - half_ybin;
			it.y1 = ddy + half_ybin;
			it.weight = 1.0 / (res * res);
			it.pixel = pix + (uint32_t)(b * npix);
			it.profile = (uint16_t)pi;
			it.res = (uint8_t)res;
			it.max_rec = (uint8_t)max_rec;
			queue_push(q, 0, it);
			note_max_res(q, res);
		}
		if (jac) {
			float *jp = jac + (size_t)pi * NTAN * npix + pix;
#pragma unroll
			for (int k = 0; k < NTAN; k++) jp[(size_t)k * npix] = jl[k];
		}
	}
	img_conv[(size_t)b * npix + pix] = acc[0];
	img_plain[(size_t)b * npix + pix] = acc[1];
}

// Sub-points [base0, base1) of an item (multiples of 32), one per lane and
// chunk.
template <class T>
__device__ __forceinline__ void level_points(const FProfile &p, const SubItem &it, int level, const double *s_xy,
                                             int lane, const QueueSet &q, float *sums, uint32_t *mask_out,
                                             unsigned base0, unsigned base1)
{
	const unsigned res = it.res;
	const double xbin = (it.x1 - it.x0) / res, ybin = (it.y1 - it.y0) / res;
	const double half_xbin = xbin / 2., half_ybin = ybin / 2.;
	const bool recurse = res > 1 && (unsigned)level < it.max_rec;
	const T adyp = fabs((T)(-xbin * (double)p.sin_q + ybin * (double)p.cos_q));
	const T cos_a = (T)p.cos_ang, sin_a = (T)p.sin_ang, cos_q = (T)p.cos_q, sin_q = (T)p.sin_q;
	const unsigned nsub = res * res;
	// sub-points in warp-wide chunks of 32 so each chunk's accept bits can be
	// gathered with one ballot (mask_out: the item's 8 words, or null)
	for (unsigned base = base0; base < base1 && base < nsub; base += 32) {
		const unsigned k = base + lane;
		bool accepted = false;
		if (k < nsub) {
			unsigned ii = k / res, jj = k - ii * res;
			const double x = s_xy[ii], y = s_xy[16 + jj];
			const T dx = (T)x, dy = (T)y;
			const T xp = dx * cos_a + dy * sin_a;
			const T yp = -dx * sin_q + dy * cos_q;
			// the test point is evaluated beside the sub-point (independent
			// chains the scheduler can interleave)
			Tan<T> t = eval_tan<T>(p, xp, yp);
			const T testval = recurse ? eval_val<T>(p, fabs(xp), fabs(yp) + adyp) : T(0);
			accepted = true;
			if (recurse) {
				if (fabs(testval - t.f) > (T)p.acc * t.f) {
					accepted = false;
					SubItem c;
					c.x0 = x - half_xbin;
					c.x1 = x + half_xbin;
					c.y0 = y - half_ybin;
					c.y1 = y + half_ybin;
					c.weight = it.weight / nsub;
					c.pixel = it.pixel;
					c.profile = it.profile;
					c.res = it.res;
					c.max_rec = it.max_rec;
					if ((uint32_t)level + 1 < q.levels) queue_push(q, level + 1, c);
					else atomicOr(q.overflow, 2u);
				}
			}
			if (accepted) {
				Tan<float> tf;
				tf.f = (float)t.f;
				tf.fx = (float)t.fx;
				tf.fy = (float)t.fy;
				tf.s1 = (float)t.s1;
				tf.s2 = (float)t.s2;
				tf.s3 = (float)t.s3;
				tan_to_j(tf, (float)xp, (float)yp, 1.0f, sums);
			}
		}
		const unsigned bits = __ballot_sync(0xffffffffu, accepted);
		if (mask_out && lane == 0) mask_out[base >> 5] = bits;
	}
}

// Adjoint of one item with its frozen decisions: the tangents of the
// sub-points the forward pass accepted (mask bit set), summed.
template <class T>
__device__ __forceinline__ void adjoint_points(const FProfile &p, const SubItem &it, const double *s_xy, int lane,
                                               const uint32_t *mask, float *sums)
{
	const unsigned res = it.res;
	const T cos_a = (T)p.cos_ang, sin_a = (T)p.sin_ang, cos_q = (T)p.cos_q, sin_q = (T)p.sin_q;
	const unsigned nsub = res * res;
	for (unsigned k = lane; k < nsub; k += 32) {
		if (!((mask[k >> 5] >> (k & 31)) & 1u)) continue;
		unsigned ii = k / res, jj = k - ii * res;
		const double x = s_xy[ii], y = s_xy[16 + jj];
		const T dx = (T)x, dy = (T)y;
		const T xp = dx * cos_a + dy * sin_a;
		const T yp = -dx * sin_q + dy * cos_q;
		Tan<T> t = eval_tan<T>(p, xp, yp);
		Tan<float> tf;
		tf.f = (float)t.f;
		tf.fx = (float)t.fx;
		tf.fy = (float)t.fy;
		tf.s1 = (float)t.s1;
		tf.s2 = (float)t.s2;
		tf.s3 = (float)t.s3;
		tan_to_j(tf, (float)xp, (float)yp, 1.0f, sums);
	}
}

// Sub-points [base0, base1) of one SubItem integrated by one warp (s_xy:
// this warp's 32 doubles); FP64 sub-points from level 3 on (the Sersic cusp).
template <bool Deep>
__device__ __forceinline__ void level32_item(const FProfile *__restrict__ profiles, const SubItem &it, int level,
                                             unsigned npix, float *__restrict__ img_conv,
                                             float *__restrict__ img_plain, float *__restrict__ jac,
                                             const QueueSet &q, double *s_xy, int lane, uint32_t *mask_out,
                                             unsigned base0, unsigned base1)
{
	const FProfile &p = profiles[it.profile];
	const unsigned res = it.res;
	const double half_xbin = (it.x1 - it.x0) / res / 2., half_ybin = (it.y1 - it.y0) / res / 2.;
	if (lane < 16) {
		if (lane < (int)res) s_xy[lane] = it.x0 + (2 * lane + 1) * half_xbin;
	}
	else if (lane - 16 < (int)res) {
		s_xy[lane] = it.y0 + (2 * (lane - 16) + 1) * half_ybin;
	}
	__syncwarp();
	float sums[NTAN];
#pragma unroll
	for (int k = 0; k < NTAN; k++) sums[k] = 0.f;
	if constexpr (Deep) level_points<double>(p, it, level, s_xy, lane, q, sums, mask_out, base0, base1);
	else level_points<float>(p, it, level, s_xy, lane, q, sums, mask_out, base0, base1);
#pragma unroll
	for (int k = 0; k < NTAN; k++) sums[k] = warp_sum(sums[k]);
	if (lane == 0) {
		const float wgt = (float)it.weight;
		const uint32_t b = it.pixel / npix, pix = it.pixel - b * npix;
		float *img = p.target == 0 ? img_conv : img_plain;
		atomicAdd(&img[it.pixel], (float)(p.flux_scale64 * it.weight * (double)sums[0]));
		if (jac) {
			float *jp = jac + (size_t)it.profile * NTAN * npix + pix;
#pragma unroll
			for (int k = 0; k < NTAN; k++) atomicAdd(&jp[(size_t)k * npix], wgt * sums[k]);
		}
	}
	__syncwarp();
}

__global__ void __launch_bounds__(256) k_level32(const FProfile *__restrict__ profiles, int level, unsigned npix,
                                                 float *__restrict__ img_conv, float *__restrict__ img_plain,
                                                 float *__restrict__ jac, QueueSet q)
{
	__shared__ double s_xy[8][32];
	const int lane = threadIdx.x & 31;
	const int wib = threadIdx.x >> 5;
	const uint32_t n = min(q.counts[level], q.cap[level]);
	const SubItem *items = q.items + q.off[level];
	const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
	// Fewer items than warps (a single image): one warp per (item, chunk of
	// 32 sub-points), so an item's chunks run side by side; otherwise one warp
	// per item.
	uint32_t cpi = 1;
	if (n < nwarps) {
		uint32_t maxres = q.maxres ? *q.maxres : 16u;
		if (maxres == 0 || maxres > 16) maxres = 16;
		cpi = (maxres * maxres + 31) / 32;
	}
	const uint32_t total = n * cpi;
	for (uint32_t w = blockIdx.x * (blockDim.x >> 5) + wib; w < total; w += nwarps) {
		const uint32_t item = w / cpi, chunk = w - item * cpi;
		const SubItem it = items[item];
		const unsigned base0 = cpi == 1 ? 0u : chunk * 32, base1 = cpi == 1 ? 256u : base0 + 32;
		if (base0 >= (unsigned)it.res * it.res) continue;
		level32_item<false>(profiles, it, level, npix, img_conv, img_plain, jac, q, s_xy[wib], lane,
		                    q.masks ? q.masks + ((size_t)q.off[level] + item) * MASK_WORDS : nullptr, base0,
		                    base1);
	}
}

// Levels first..levels-1 in one CTA.  Only the Sersic central cusp
// (max_recursions = 10) reaches these levels, a few hundred cells per level
// at most, so one block walks them in order; __syncthreads separates the
// levels, which makes every push of level L visible before level L+1 is read.
__global__ void __launch_bounds__(512) k_deep_levels32(const FProfile *__restrict__ profiles, int first, int levels,
                                                        unsigned npix, float *__restrict__ img_conv,
                                                        float *__restrict__ img_plain, float *__restrict__ jac,
                                                        QueueSet q)
{
	__shared__ double s_xy[16][32];
	const int lane = threadIdx.x & 31;
	const int wib = threadIdx.x >> 5;
	const uint32_t nwarps = blockDim.x >> 5;
	for (int level = first; level < levels; level++) {
		__syncthreads();
		const uint32_t n = min(*(volatile uint32_t *)&q.counts[level], q.cap[level]);
		const SubItem *items = q.items + q.off[level];
		for (uint32_t w = wib; w < n; w += nwarps)
			level32_item<true>(profiles, items[w], level, npix, img_conv, img_plain, jac, q, s_xy[wib], lane,
			                   q.masks ? q.masks + ((size_t)q.off[level] + w) * MASK_WORDS : nullptr, 0, 256);
	}
}

// ---------------------------------------------------------------------------
// Recomputing adjoint (no stored tangent planes): used when the planes would
// not fit, e.g. hundreds of profiles on a large field.  The forward pass
// rendered values only and recorded each queued cell's accepted sub-points;
// these kernels recompute the tangents against the known seed g.
// ---------------------------------------------------------------------------

// Directly evaluated pixels, one profile per blockIdx.z, 64 x 32 pixel tiles.
// A tile whose nearest pixel centre is farther than rscale_max (+2 px) from
// the profile centre is skipped: the elliptical radius is never smaller than
// the Euclidean distance, so such pixels were zeroed by the forward pass.
__global__ void __launch_bounds__(256) k_adjoint_pixels32(const FProfile *__restrict__ profiles,
                                                          const int *__restrict__ prof_batch, unsigned width,
                                                          unsigned height, double sx, double sy,
                                                          const float *__restrict__ g_conv,
                                                          const float *__restrict__ g_plain, double *__restrict__ T)
{
	const int pi = blockIdx.z;
	const FProfile &p = profiles[pi];
	if (!is_radial_kind(p.kind)) return;
	const unsigned tx0 = blockIdx.x * 64, ty0 = blockIdx.y * 32;
	const double half_xbin = sx / 2., half_ybin = sy / 2.;
	if (p.r_max > 0.f) {
		const unsigned tx1 = min(tx0 + 63, width - 1), ty1 = min(ty0 + 31, height - 1);
		const double xlo = half_xbin + tx0 * sy, xhi = half_xbin + tx1 * sy;
		const double ylo = half_ybin + ty0 * sx, yhi = half_ybin + ty1 * sx;
		const double nx = fmin(fmax(p.cx, xlo), xhi) - p.cx, ny = fmin(fmax(p.cy, ylo), yhi) - p.cy;
		if (sqrt(nx * nx + ny * ny) > (double)p.r_max + 2.0) return;
	}
	const size_t npix = (size_t)width * height;
	const float *g = (p.target == 0 ? g_conv : g_plain) + (size_t)prof_batch[pi] * npix;
	float acc[NTAN];
#pragma unroll
	for (int k = 0; k < NTAN; k++) acc[k] = 0.f;
	const unsigned i = tx0 + (threadIdx.x & 63);
	for (unsigned r = threadIdx.x >> 6; r < 32; r += 4) {
		const unsigned j = ty0 + r;
		if (i >= width || j >= height) continue;
		const float gv = g[i + (size_t)j * width];
		if (gv == 0.f) continue;
		const double y = half_ybin + j * sx, x = half_xbin + i * sy;
		float xp, yp;
		if (pixel_decision32(p, x, y, xp, yp) != PD_DIRECT) continue;
		Tan<float> t = eval_tan<float>(p, xp, yp);
		tan_to_j(t, xp, yp, gv, acc);
	}
	__shared__ double s_red[NTAN][8];
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
	for (int k = 0; k < NTAN; k++) {
		double v = warp_sum((double)acc[k]);
		if (lane == 0) s_red[k][wid] = v;
	}
	__syncthreads();
	if (threadIdx.x < NTAN) {
		double v = 0;
		for (int w = 0; w < 8; w++) v += s_red[threadIdx.x][w];
		if (v != 0.0) atomicAdd(&T[(size_t)pi * NTAN + threadIdx.x], v);
	}
}

// Every queued cell of every level, one warp per cell: the tangents of the
// accepted sub-points, times the cell weight and g(pixel).
__global__ void __launch_bounds__(256) k_adjoint_items32(const FProfile *__restrict__ profiles, int levels,
                                                         const float *__restrict__ g_conv,
                                                         const float *__restrict__ g_plain, QueueSet q,
                                                         double *__restrict__ T)
{
	__shared__ double s_xy[8][32];
	const int lane = threadIdx.x & 31;
	const int wib = threadIdx.x >> 5;
	const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
	const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + wib;
	for (int level = 0; level < levels; level++) {
		const uint32_t n = min(q.counts[level], q.cap[level]);
		const SubItem *items = q.items + q.off[level];
		for (uint32_t w = gw; w < n; w += nwarps) {
			const SubItem it = items[w];
			const FProfile &p = profiles[it.profile];
			const unsigned res = it.res;
			const double half_xbin = (it.x1 - it.x0) / res / 2., half_ybin = (it.y1 - it.y0) / res / 2.;
			if (lane < 16) {
				if (lane < (int)res) s_xy[wib][lane] = it.x0 + (2 * lane + 1) * half_xbin;
			}
			else if (lane - 16 < (int)res) {
				s_xy[wib][lane] = it.y0 + (2 * (lane - 16) + 1) * half_ybin;
			}
			__syncwarp();
			const uint32_t *mask = q.masks + ((size_t)q.off[level] + w) * MASK_WORDS;
			float sums[NTAN];
#pragma unroll
			for (int k = 0; k < NTAN; k++) sums[k] = 0.f;
			if (level >= 3) adjoint_points<double>(p, it, s_xy[wib], lane, mask, sums);
			else adjoint_points<float>(p, it, s_xy[wib], lane, mask, sums);
#pragma unroll
			for (int k = 0; k < NTAN; k++) sums[k] = warp_sum(sums[k]);
			if (lane == 0) {
				const float gv = (p.target == 0 ? g_conv : g_plain)[it.pixel];
				const double coef = (double)gv * it.weight;
				if (coef != 0.0) {
#pragma unroll
					for (int k = 0; k < NTAN; k++) atomicAdd(&T[(size_t)it.profile * NTAN + k], coef * (double)sums[k]);
				}
			}
			__syncwarp();
		}
	}
}

cudaError_t launch_adjoint_recompute(const FProfile *profiles, const int *prof_batch, int n_profiles, unsigned width,
                                     unsigned height, double sx, double sy, const float *g_conv, const float *g_plain,
                                     int levels, const QueueSet &q, double *T, cudaStream_t s)
{
	dim3 grid((width + 63) / 64, (height + 31) / 32, n_profiles);
	k_adjoint_pixels32<<<grid, 256, 0, s>>>(profiles, prof_batch, width, height, sx, sy, g_conv, g_plain, T);
	k_adjoint_items32<<<148 * 8, 256, 0, s>>>(profiles, levels, g_conv, g_plain, q, T);
	note_launches(2);
	return cudaGetLastError();
}

// sum over pixels of g(pixel) * J_k(pixel) for each radial profile:
// blockIdx.y = profile, blockIdx.x strides over the pixels, four pixels per
// thread and step with every load issued before the products (enough bytes
// in flight to stream the tangent planes at HBM speed).  Each block writes
// its NTAN sums to `partials`; the block that finishes last (an atomic
// ticket per profile, no waiting) adds the partials in block order and
// resets the ticket, so the result does not depend on block scheduling.
__global__ void __launch_bounds__(256) k_jac_reduce(const float *__restrict__ jac, const float *__restrict__ g_conv,
                                                    const float *__restrict__ g_plain,
                                                    const FProfile *__restrict__ profiles,
                                                    const int *__restrict__ prof_batch, unsigned npix,
                                                    double *__restrict__ partials, unsigned *__restrict__ tickets,
                                                    double *__restrict__ out)
{
	constexpr int U = 4;
	const int pi = blockIdx.y;
	const FProfile &p = profiles[pi];
	if (!is_radial_kind(p.kind)) return;
	const int b = prof_batch[pi];
	const float *g = (p.target == 0 ? g_conv : g_plain) + (size_t)b * npix;
	const float *jp = jac + (size_t)pi * NTAN * npix;
	double acc[NTAN];
#pragma unroll
	for (int k = 0; k < NTAN; k++) acc[k] = 0.0;
	const unsigned step = gridDim.x * blockDim.x * U;
	for (unsigned t0 = blockIdx.x * blockDim.x * U + threadIdx.x; t0 < npix; t0 += step) {
		float gv[U], jv[U][NTAN];
#pragma unroll
		for (int u = 0; u < U; u++) {
			const unsigned t = t0 + u * blockDim.x;
			const bool in = t < npix;
			gv[u] = in ? g[t] : 0.f;
#pragma unroll
			for (int k = 0; k < NTAN; k++) jv[u][k] = in ? jp[(size_t)k * npix + t] : 0.f;
		}
#pragma unroll
		for (int u = 0; u < U; u++)
			if (gv[u] != 0.f) {
#pragma unroll
				for (int k = 0; k < NTAN; k++) acc[k] += (double)(gv[u] * jv[u][k]);
			}
	}
	__shared__ double s_red[NTAN][8];
	__shared__ bool s_last;
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
	for (int k = 0; k < NTAN; k++) {
		double v = warp_sum(acc[k]);
		if (lane == 0) s_red[k][wid] = v;
	}
	__syncthreads();
	double *mine = partials + ((size_t)pi * gridDim.x + blockIdx.x) * NTAN;
	if (threadIdx.x < NTAN) {
		double v = 0;
		for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += s_red[threadIdx.x][w];
		mine[threadIdx.x] = v;
		__threadfence();
	}
	__syncthreads();
	if (threadIdx.x == 0) s_last = atomicAdd(&tickets[pi], 1u) == gridDim.x - 1;
	__syncthreads();
	if (!s_last) return;
	__threadfence();
	if (threadIdx.x < NTAN) {
		const double *all = partials + (size_t)pi * gridDim.x * NTAN;
		double v = 0;
		for (unsigned blk = 0; blk < gridDim.x; blk++) v += ((volatile const double *)all)[blk * NTAN + threadIdx.x];
		out[(size_t)pi * NTAN + threadIdx.x] = v;
	}
	if (threadIdx.x == 0) tickets[pi] = 0;
}

// Scatter the residual weights w (cropped grid) into the padded grid of the
// unconvolved image: g_plain(u) = w(u - pad).
__global__ void k_embed_seed(const float *__restrict__ w, unsigned ow, unsigned oh, unsigned padx, unsigned pady,
                             unsigned dw, unsigned dh, float *__restrict__ g_plain)
{
	const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
	const unsigned j = blockIdx.y * blockDim.y + threadIdx.y;
	const int b = blockIdx.z;
	if (i >= dw || j >= dh) return;
	float v = 0.f;
	if (i >= padx && j >= pady && i - padx < ow && j - pady < oh) v = w[(size_t)b * ow * oh + (i - padx) + (j - pady) * ow];
	g_plain[(size_t)b * dw * dh + i + j * dw] = v;
}

__global__ void k_crop32(const float *__restrict__ src, unsigned sw, unsigned ox, unsigned oy,
                         float *__restrict__ out, unsigned ow, unsigned oh, const float *__restrict__ add,
                         unsigned src_stride)
{
	unsigned i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
	const int b = blockIdx.z;
	if (i >= ow || j >= oh) return;
	size_t s = (size_t)b * src_stride + (i + ox) + (size_t)(j + oy) * sw;
	float v = src[s];
	if (add) v += add[s];
	out[(size_t)b * ow * oh + i + (size_t)j * ow] = v;
}

static inline unsigned cdiv(unsigned a, unsigned b) { return (a + b - 1) / b; }

cudaError_t launch_pixels32(const FProfile *profiles, const int *prof_begin, int batch, unsigned width,
                            unsigned height, double sx, double sy, float *img_conv, float *img_plain, float *jac,
                            const QueueSet &q, cudaStream_t s)
{
	dim3 block(32, 8), grid(cdiv(width, 32), cdiv(height, 8), batch);
	k_pixels32<<<grid, block, 0, s>>>(profiles, prof_begin, width, height, sx, sy, img_conv, img_plain, jac, q);
	note_launches(1);
	return cudaGetLastError();
}

cudaError_t launch_levels32(const FProfile *profiles, int n_levels, unsigned npix, float *img_conv, float *img_plain,
                            float *jac, const QueueSet &q, cudaStream_t s)
{
	const int wide = n_levels < 3 ? n_levels : 3;
	for (int l = 0; l < wide; l++) k_level32<<<148 * 8, 256, 0, s>>>(profiles, l, npix, img_conv, img_plain, jac, q);
	note_launches(wide);
	if (n_levels > wide) {
		k_deep_levels32<<<1, 512, 0, s>>>(profiles, wide, n_levels, npix, img_conv, img_plain, jac, q);
		note_launches(1);
	}
	return cudaGetLastError();
}

unsigned jac_reduce_blocks(unsigned npix, int n_profiles)
{
	unsigned bx = cdiv(npix, 256 * 4);
	const unsigned target = cdiv(148u * 8u, (unsigned)n_profiles);  // about 8 blocks per SM in all
	if (bx > target) bx = target;
	return bx < 1 ? 1 : bx;
}

cudaError_t launch_jac_reduce(const float *jac, const float *g_conv, const float *g_plain, const FProfile *profiles,
                              const int *prof_batch, int n_profiles, unsigned npix, double *partials,
                              unsigned *tickets, double *out, cudaStream_t s)
{
	const unsigned bx = jac_reduce_blocks(npix, n_profiles);
	k_jac_reduce<<<dim3(bx, n_profiles), 256, 0, s>>>(jac, g_conv, g_plain, profiles, prof_batch, npix, partials,
	                                                  tickets, out);
	note_launches(1);
	return cudaGetLastError();
}

cudaError_t launch_embed_seed(const float *w, unsigned ow, unsigned oh, unsigned padx, unsigned pady, unsigned dw,
                              unsigned dh, int batch, float *g_plain, cudaStream_t s)
{
	dim3 block(32, 8), grid(cdiv(dw, 32), cdiv(dh, 8), batch);
	k_embed_seed<<<grid, block, 0, s>>>(w, ow, oh, padx, pady, dw, dh, g_plain);
	note_launches(1);
	return cudaGetLastError();
}

// FP32 taps, FP64 column accumulation; FP32 output (adjoint) or FP64 output
// (forward model, so the likelihood sees the full-precision sum).
template <class TOut>
static cudaError_t conv32_any(const float *src, int sw, int sh, int ox, int oy, const float *K, int kw, int kh,
                              TOut *out, int ow, int oh, const float *add, int add_stride, int add_ox, int add_oy,
                              int batch, int batch_src_stride, int batch_out_stride, double *scratch,
                              size_t scratch_bytes, cudaStream_t s)
{
	note_launches(1);
	static const ConvCandidate cands[] = {
	    // packed-FMA kernels: (lanes per row, rows per thread, row groups, column groups, column splits)
	    {Conv3Variant<TOut, 32, 8, 2, 4, 1>::smem, Conv3Variant<TOut, 32, 8, 2, 4, 1>::run},
	    {Conv3Variant<TOut, 32, 8, 4, 1, 1>::smem, Conv3Variant<TOut, 32, 8, 4, 1, 1>::run},
	    {Conv3Variant<TOut, 32, 12, 4, 1, 1>::smem, Conv3Variant<TOut, 32, 12, 4, 1, 1>::run},
	    {Conv3Variant<TOut, 32, 8, 1, 8, 1>::smem, Conv3Variant<TOut, 32, 8, 1, 8, 1>::run},
	    {Conv3Variant<TOut, 16, 8, 2, 1, 1>::smem, Conv3Variant<TOut, 16, 8, 2, 1, 1>::run},
	    {Conv3Variant<TOut, 16, 8, 4, 1, 1>::smem, Conv3Variant<TOut, 16, 8, 4, 1, 1>::run},
	    {Conv3Variant<TOut, 16, 12, 2, 1, 1>::smem, Conv3Variant<TOut, 16, 12, 2, 1, 1>::run},
	    {Conv3Variant<TOut, 16, 8, 1, 4, 1>::smem, Conv3Variant<TOut, 16, 8, 1, 4, 1>::run},
	    {Conv3Variant<TOut, 16, 8, 1, 8, 1>::smem, Conv3Variant<TOut, 16, 8, 1, 8, 1>::run},
	    {Conv3Variant<TOut, 16, 8, 1, 4, 2>::smem, Conv3Variant<TOut, 16, 8, 1, 4, 2>::run},
	    {Conv3Variant<TOut, 16, 8, 1, 4, 4>::smem, Conv3Variant<TOut, 16, 8, 1, 4, 4>::run},
	    {Conv3Variant<TOut, 16, 8, 1, 2, 4>::smem, Conv3Variant<TOut, 16, 8, 1, 2, 4>::run},
	    {Conv3Variant<TOut, 16, 8, 2, 2, 2>::smem, Conv3Variant<TOut, 16, 8, 2, 2, 2>::run},
	    {Conv3Variant<TOut, 32, 8, 1, 4, 2>::smem, Conv3Variant<TOut, 32, 8, 1, 4, 2>::run},
	    // one-column-per-lane kernels
	    {ConvVariant<float, double, TOut, 8, 1, 8>::smem, ConvVariant<float, double, TOut, 8, 1, 8>::run},
	    {ConvVariant<float, double, TOut, 8, 2, 4>::smem, ConvVariant<float, double, TOut, 8, 2, 4>::run},
	};
	ConvArgs a{src, sw, sh, ox, oy, K, kw, kh, out, ow, oh, add, add_stride, add_ox, add_oy, batch,
	           batch_src_stride, batch_out_stride, scratch, scratch_bytes};
	return conv_autotuned(cands, (int)(sizeof(cands) / sizeof(cands[0])), sizeof(TOut) == 8 ? 2 : 1, a, s);
}

size_t conv32_scratch_bytes(int ow, int oh, int batch)
{
	const size_t bytes = (size_t)ow * oh * batch * 4 * sizeof(double);  // up to 4 column splits
	return bytes <= ((size_t)64 << 20) ? bytes : 0;
}

cudaError_t launch_conv32(const float *src, int sw, int sh, int ox, int oy, const float *K, int kw, int kh,
                          float *out, int ow, int oh, const float *add, int add_stride, int add_ox, int add_oy,
                          int batch, int batch_src_stride, int batch_out_stride, double *scratch, size_t scratch_bytes,
                          cudaStream_t s)
{
	return conv32_any<float>(src, sw, sh, ox, oy, K, kw, kh, out, ow, oh, add, add_stride, add_ox, add_oy, batch,
	                         batch_src_stride, batch_out_stride, scratch, scratch_bytes, s);
}

cudaError_t launch_conv32_to64(const float *src, int sw, int sh, int ox, int oy, const float *K, int kw, int kh,
                               double *out, int ow, int oh, const float *add, int add_stride, int add_ox, int add_oy,
                               int batch, int batch_src_stride, int batch_out_stride, double *scratch,
                               size_t scratch_bytes, cudaStream_t s)
{
	return conv32_any<double>(src, sw, sh, ox, oy, K, kw, kh, out, ow, oh, add, add_stride, add_ox, add_oy, batch,
	                          batch_src_stride, batch_out_stride, scratch, scratch_bytes, s);
}

cudaError_t launch_loglike32(const float *model, const double *data, const double *sigma, const uint8_t *region,
                             int n, int batch, int data_batch_stride, double2 *partials, int nparts, double *out,
                             float *wseed, cudaStream_t s)
{
	k_loglike_partial<float><<<dim3(nparts, batch), 256, 0, s>>>(model, data, sigma, region, n, partials, wseed,
	                                                             data_batch_stride);
	k_loglike_final<<<batch, 256, 0, s>>>(partials, nparts, out);
	note_launches(2);
	return cudaGetLastError();
}

cudaError_t launch_crop32(const float *src, unsigned sw, unsigned ox, unsigned oy, float *out, unsigned ow,
                          unsigned oh, const float *add, int batch, unsigned src_stride, cudaStream_t s)
{
	dim3 block(32, 8), grid(cdiv(ow, 32), cdiv(oh, 8), batch);
	k_crop32<<<grid, block, 0, s>>>(src, sw, ox, oy, out, ow, oh, add, src_stride);
	note_launches(1);
	return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Batched proposals: device-side prologue and gradient assembly
// ---------------------------------------------------------------------------

// One thread per (proposal, profile): the model's parameters with this
// proposal's values written in, checked like RadialProfile::validate, then the
// FP64 scalar prologue (b_n, luminosity, Ie, auto-adjusted subsampling).  A
// proposal with an invalid profile is flagged and its profiles become null
// profiles, so nothing is drawn for it.
__global__ void k_batch_prologue(const ProfileParams *__restrict__ tmpl, int nprof, int batch,
                                 const int *__restrict__ ref_profile, const int *__restrict__ ref_offset, int nrefs,
                                 const double *__restrict__ values, ModelGeom g, DevProfile *__restrict__ dev,
                                 FProfile *__restrict__ fprof, int *__restrict__ invalid)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= batch * nprof) return;
	const int b = t / nprof, p = t - b * nprof;
	ProfileParams pp = tmpl[p];
	for (int r = 0; r < nrefs; r++)
		if (ref_profile[r] == p)
			*reinterpret_cast<double *>(reinterpret_cast<char *>(&pp) + ref_offset[r]) = values[(size_t)b * nrefs + r];
	if (!params_valid(pp)) {
		invalid[b] = 1;
		pp.kind = PK_NULL;
	}
	DevProfile d;
	derive_profile(pp, g, d);
	dev[t] = d;
	fprof[t] = to_fprofile(d, pp);
}

// One thread per (proposal, parameter): d logL / d parameter from the tangent
// reductions; invalid proposals get logL = -inf and a zero gradient.
__global__ void k_batch_gradient(const DevProfile *__restrict__ dev, int nprof, int batch,
                                 const int *__restrict__ ref_profile, const int *__restrict__ ref_code, int nrefs,
                                 const double *__restrict__ T, const double *__restrict__ ll, const int *__restrict__ invalid,
                                 double *__restrict__ out_ll, double *__restrict__ out_grad)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t < batch) out_ll[t] = invalid[t] ? -INFINITY : ll[t];
	if (t >= batch * nrefs) return;
	const int b = t / nrefs, r = t - b * nrefs;
	const int pi = b * nprof + ref_profile[r];
	out_grad[t] = invalid[b] ? 0.0 : gradient_from_tangents(ref_code[r], dev[pi].axrat, dev[pi], T + (size_t)pi * NTAN);
}

cudaError_t launch_batch_prologue(const ProfileParams *tmpl, int nprof, int batch, const int *ref_profile,
                                  const int *ref_offset, int nrefs, const double *values, const ModelGeom &g,
                                  DevProfile *dev, FProfile *fprof, int *invalid, cudaStream_t s)
{
	int n = batch * nprof;
	k_batch_prologue<<<(n + 127) / 128, 128, 0, s>>>(tmpl, nprof, batch, ref_profile, ref_offset, nrefs, values, g,
	                                                 dev, fprof, invalid);
	note_launches(1);
	return cudaGetLastError();
}

cudaError_t launch_batch_gradient(const DevProfile *dev, int nprof, int batch, const int *ref_profile,
                                  const int *ref_code, int nrefs, const double *T, const double *ll,
                                  const int *invalid, double *out_ll, double *out_grad, cudaStream_t s)
{
	int n = batch * (nrefs > 1 ? nrefs : 1);
	k_batch_gradient<<<(n + 255) / 256, 256, 0, s>>>(dev, nprof, batch, ref_profile, ref_code, nrefs, T, ll, invalid,
	                                                 out_ll, out_grad);
	note_launches(1);
	return cudaGetLastError();
}

cudaError_t launch_loglike64_batch(const double *model, const double *data, const double *sigma,
                                   const uint8_t *region, int n, int batch, int data_batch_stride, double2 *partials,
                                   int nparts, double *out, float *wseed, cudaStream_t s)
{
	k_loglike_partial<double><<<dim3(nparts, batch), 256, 0, s>>>(model, data, sigma, region, n, partials, wseed,
	                                                              data_batch_stride);
	k_loglike_final<<<batch, 256, 0, s>>>(partials, nparts, out);
	note_launches(2);
	return cudaGetLastError();
}

}  // namespace pf
