// Plain FP64 rendering: libprofit's RadialProfile::evaluate_cpu
// (radial.cpp:291-344) with its adaptive subsample_pixel recursion
// (radial.cpp:54-134), sky (sky.cpp:47-63) and psf point sources
// (psf.cpp:58-145).
//
// Work decomposition (sm_100a, 148 SMs):
//  1. k_pixels64: one thread per drawing pixel, all profiles in order.  A
//     pixel is either zero (beyond rscale_max), evaluated once, or becomes a
//     level-0 SubItem in the device work queue.
//  2. k_level64 (once per recursion level): one warp per SubItem.  Lanes
//     split the res x res sub-points; each lane evaluates subval and the
//     libprofit test value and either keeps subval or pushes a child cell to
//     the next level.  The accepted sum, weighted by flux_scale/res^(2(L+1)),
//     is added to the pixel with one atomic per item.  Levels replace the
//     reference's depth-first recursion; sums are equal up to rounding order.
// Sub-point coordinates repeat the reference's running sums (x += half_xbin
// twice per step) so decisions are taken on bit-identical coordinates.
// This file is compiled with --fmad=false so products and sums round like
// the reference's scalar code.

#include "common.cuh"
#include "conv.cuh"
#include "launch.h"
#include "like.cuh"
#include "like_kinds.cuh"

namespace pf {

// mask (optional, drawing size): radial and sky profiles skip the pixels it
// leaves out (radial.cpp:306, sky.cpp:56-58); psf profiles ignore it.
__global__ void k_pixels64(const DevProfile *__restrict__ profiles, int n_profiles, unsigned width,
                           unsigned height, double sx, double sy, double *__restrict__ img_conv,
                           double *__restrict__ img_plain, const uint8_t *__restrict__ mask, QueueSet q)
{
	unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
	unsigned j = blockIdx.y * blockDim.y + threadIdx.y;
	if (i >= width || j >= height) return;
	const uint32_t pix = i + j * width;
	if (mask && !mask[pix]) {
		img_conv[pix] = 0.0;
		img_plain[pix] = 0.0;
		return;
	}
	double acc[2] = {0.0, 0.0};
	double half_xbin = sx / 2., half_ybin = sy / 2.;
	// radial.cpp:313-314 computes y with scale.x and x with scale.y
	double y = half_ybin + j * sx;
	double x = half_xbin + i * sy;

	for (int p = 0; p < n_profiles; p++) {
		const DevProfile &d = profiles[p];
		if (d.kind == PK_SKY) {
			acc[d.target] += d.bg;
			continue;
		}
		if (!is_radial_kind(d.kind)) continue;
		double xp, yp;
		to_profile64(d, x, y, xp, yp);
		double r = sqrt(xp * xp + yp * yp);
		int32_t decision = 0;
		if (d.r_max > 0 && r > d.r_max) {
			decision = -1;
		}
		else if (d.rough || r > d.r_switch) {
			acc[d.target] += d.flux_scale * eval64(d, xp, yp);
			if (q.evals) atomicAdd(&q.evals[(size_t)p * (1 + MAX_LEVELS)], 1ull);
		}
		else {
			unsigned res = d.resolution, max_rec = d.max_rec;
			if (d.centre_override && fabs(x - d.cx) < d.img_sx && fabs(y - d.cy) < d.img_sy) {
				res = 8;
				max_rec = 10;
			}
			SubItem it;
			it.x0 = x - half_xbin;
			it.x1 = x + half_xbin;
			it.y0 = y - half_ybin;
			it.y1 = y + half_ybin;
			it.weight = d.flux_scale / (res * res);
			it.pixel = pix;
			it.profile = (uint16_t)p;
			it.res = (uint8_t)res;
			it.max_rec = (uint8_t)max_rec;
			queue_push(q, 0, it);
		}
		if (q.decisions) q.decisions[(size_t)p * width * height + pix] = decision;
	}
	img_conv[pix] = acc[0];
	img_plain[pix] = acc[1];
}

// One SubItem of `level` integrated by one warp (s_xy: the warp's 32 doubles).
__device__ __forceinline__ void level64_item(const DevProfile *__restrict__ profiles, const SubItem it, int level,
                                             double *__restrict__ img_conv, double *__restrict__ img_plain,
                                             const QueueSet &q, double *s_xy_w, int lane)
{
		double(*s_xy)[32] = reinterpret_cast<double(*)[32]>(s_xy_w);
		const int wib = 0;
		const DevProfile &d = profiles[it.profile];
		const unsigned res = it.res;
		const double xbin = (it.x1 - it.x0) / res;
		const double ybin = (it.y1 - it.y0) / res;
		const double half_xbin = xbin / 2.;
		const double half_ybin = ybin / 2.;
		// sub-point centres exactly as the reference's running sums
		if (lane < 16) {
			if (lane < (int)res) {
				double x = it.x0;
				for (int k = 0; k < lane; k++) {
					x += half_xbin;
					x += half_xbin;
				}
				x += half_xbin;
				s_xy[wib][lane] = x;
			}
		}
		else {
			int l = lane - 16;
			if (l < (int)res) {
				double y = it.y0;
				for (int k = 0; k < l; k++) {
					y += half_ybin;
					y += half_ybin;
				}
				y += half_ybin;
				s_xy[wib][16 + l] = y;
			}
		}
		__syncwarp();
		const bool recurse = res > 1 && (unsigned)level < it.max_rec;
		const double delta_y_prof = -xbin * d.sin_q + ybin * d.cos_q;
		const double adyp = fabs(delta_y_prof);
		double sum = 0.0;
		const unsigned nsub = res * res;
		for (unsigned k = lane; k < nsub; k += 32) {
			unsigned ii = k / res, jj = k - ii * res;
			double x = s_xy[wib][ii], y = s_xy[wib][16 + jj];
			double xp, yp;
			to_profile64(d, x, y, xp, yp);
			double subval = eval64(d, xp, yp);
			if (recurse) {
				double testval = eval64(d, fabs(xp), fabs(yp) + adyp);
				if (fabs(testval - subval) > d.acc * subval) {
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
					continue;
				}
			}
			sum += subval;
		}
		sum = warp_sum(sum);
		if (lane == 0) {
			double *img = d.target == 0 ? img_conv : img_plain;
			atomicAdd(&img[it.pixel], it.weight * sum);
		}
		__syncwarp();
}

__global__ void __launch_bounds__(256) k_level64(const DevProfile *__restrict__ profiles, int level,
                                                 double *__restrict__ img_conv, double *__restrict__ img_plain,
                                                 QueueSet q)
{
	__shared__ double s_xy[8][32];
	const int lane = threadIdx.x & 31;
	const int wib = threadIdx.x >> 5;
	const uint32_t n = min(q.counts[level], q.cap[level]);
	const SubItem *items = q.items + q.off[level];
	const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
	for (uint32_t w = blockIdx.x * (blockDim.x >> 5) + wib; w < n; w += nwarps)
		level64_item(profiles, items[w], level, img_conv, img_plain, q, s_xy[wib], lane);
}

// Levels first..levels-1 in one CTA (the Sersic central cusp only); see
// k_deep_levels32 in render32.cu.
__global__ void __launch_bounds__(512) k_deep_levels64(const DevProfile *__restrict__ profiles, int first, int levels,
                                                        double *__restrict__ img_conv, double *__restrict__ img_plain,
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
			level64_item(profiles, items[w], level, img_conv, img_plain, q, s_xy[wib], lane);
	}
}

// Per-pixel and per-level decision counters for the debug mode: one thread
// per item, after all levels ran.
__global__ void k_count_decisions(QueueSet q, int level, size_t npix)
{
	const uint32_t n = min(q.counts[level], q.cap[level]);
	const SubItem *items = q.items + q.off[level];
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
		const SubItem &it = items[t];
		atomicAdd(&q.decisions[(size_t)it.profile * npix + it.pixel], 1);
		atomicAdd(&q.level_counts[(size_t)it.profile * MAX_LEVELS + level], 1ull);
		// res^2 sub-points, each evaluated twice (value and test point) when the
		// level may still recurse (radial.cpp:54-134)
		if (q.evals) {
			const unsigned long long res = it.res;
			const bool recurse = res > 1 && (unsigned)level < it.max_rec;
			atomicAdd(&q.evals[(size_t)it.profile * (1 + MAX_LEVELS) + 1 + level], res * res * (recurse ? 2ull : 1ull));
		}
	}
}

// libprofit's psf profile (psf.cpp:58-145): area-weighted resampling of the
// normalised PSF image, one thread per covered target pixel.  The x/y offset
// quirks of psf.cpp:79-82 and the height bound at psf.cpp:106 are kept.

__global__ void k_psf_stamp64(const DevProfile *__restrict__ profiles, int p, const double *__restrict__ psf, unsigned psf_w,
                              unsigned psf_h, double psf_sx, double psf_sy, double scale_x, double scale_y,
                              double offx, double offy, unsigned width, unsigned height,
                              double *__restrict__ img_conv, double *__restrict__ img_plain)
{
	const DevProfile &d = profiles[p];
	double origin_x = d.px + offx * scale_x - psf_w * psf_sx / 2;
	double end_x = d.px + offy * scale_y + psf_w * psf_sx / 2;
	double origin_y = d.py + offx * scale_x - psf_h * psf_sy / 2;
	double end_y = d.py + offy * scale_y + psf_h * psf_sy / 2;
	unsigned x0 = bind_u(origin_x / scale_x, width - 1);
	unsigned y0 = bind_u(origin_y / scale_y, height - 1);
	unsigned x1 = bind_u(end_x / scale_x, width - 1);
	unsigned y1 = bind_u(end_y / scale_y, height - 1);
	if (x1 < x0 || y1 < y0) return;
	unsigned nx = x1 - x0 + 1, ny = y1 - y0 + 1;
	double *img = d.target == 0 ? img_conv : img_plain;
	for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < nx * ny; t += gridDim.x * blockDim.x) {
		unsigned pix_x = x0 + t % nx, pix_y = y0 + t / nx;
		double y = pix_y * scale_y;
		double x = pix_x * scale_x;
		int px0 = (int)bind_u(floor((x - origin_x) / psf_sx), psf_w - 1);
		int px1 = (int)bind_u(floor((x - origin_x + scale_x) / psf_sx), psf_h - 1);
		int py0 = (int)bind_u(floor((y - origin_y) / psf_sy), psf_w - 1);
		int py1 = (int)bind_u(floor((y - origin_y + scale_y) / psf_sy), psf_h - 1);
		// psf.cpp:104-107 bounds x1 by the height and y0 by the width; for
		// non-square PSFs that can index outside the PSF, which libprofit reads
		// anyway.  Here those indices are clamped to the PSF instead.
		px1 = min(px1, (int)psf_w - 1);
		py0 = min(py0, (int)psf_h - 1);
		double val = 0;
		for (int yy = py0; yy <= py1; yy++) {
			double psf_y = yy * psf_sy + origin_y;
			for (int xx = px0; xx <= px1; xx++) {
				double psf_x = xx * psf_sx + origin_x;
				double ix = fmin(x + scale_x, psf_x + psf_sx) - fmax(x, psf_x);
				double iy = fmin(y + scale_y, psf_y + psf_sy) - fmax(y, psf_y);
				val += psf[xx + yy * psf_w] * (ix * iy) / (psf_sx * psf_sy);
			}
		}
		img[pix_x + (size_t)pix_y * width] += val * d.psf_flux;
	}
}

// Crop of the padded image plus the unconvolved image when no convolution
// is needed (model.cpp:307-324), and the SUM downsampling of
// image.cpp:285-298 for finesampled models.
__global__ void k_crop64(const double *__restrict__ src, unsigned sw, unsigned ox, unsigned oy,
                         double *__restrict__ out, unsigned ow, unsigned oh, const double *__restrict__ add)
{
	unsigned i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
	if (i >= ow || j >= oh) return;
	size_t s = (i + ox) + (size_t)(j + oy) * sw;
	double v = src[s];
	if (add) v += add[s];
	out[i + (size_t)j * ow] = v;
}

__global__ void k_downsample64(const double *__restrict__ src, unsigned sw, unsigned sh, unsigned fs,
                               double *__restrict__ out, unsigned ow, unsigned oh)
{
	unsigned i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
	if (i >= ow || j >= oh) return;
	double v = 0;
	for (unsigned row = j * fs; row < min((j + 1) * fs, sh); row++)
		for (unsigned col = i * fs; col < min((i + 1) * fs, sw); col++) v += src[col + (size_t)row * sw];
	out[i + (size_t)j * ow] = v;
}

static inline unsigned cdiv(unsigned a, unsigned b) { return (a + b - 1) / b; }

cudaError_t launch_pixels64(const DevProfile *profiles, int n_profiles, unsigned width, unsigned height, double sx,
                            double sy, double *img_conv, double *img_plain, const uint8_t *mask, const QueueSet &q,
                            cudaStream_t s)
{
	dim3 block(32, 8), grid(cdiv(width, 32), cdiv(height, 8));
	k_pixels64<<<grid, block, 0, s>>>(profiles, n_profiles, width, height, sx, sy, img_conv, img_plain, mask, q);
	note_launches(1);
	return cudaGetLastError();
}

// Masked convolution (convolve.cpp:185, model.cpp:372-376): an output pixel
// the drawing mask leaves out gets no convolved flux, only the unconvolved
// image, out(i, j) = plain(i + ox, j + oy) there.
__global__ void k_mask_select64(double *__restrict__ out, unsigned ow, unsigned oh, const double *__restrict__ plain,
                                const uint8_t *__restrict__ mask, unsigned dw, unsigned ox, unsigned oy)
{
	const unsigned i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
	if (i >= ow || j >= oh) return;
	const size_t d = (i + ox) + (size_t)(j + oy) * dw;
	if (!mask[d]) out[i + (size_t)j * ow] = plain[d];
}

// image &= mask (image.cpp:369-381).
__global__ void k_mask_and64(double *__restrict__ out, const uint8_t *__restrict__ mask, size_t n)
{
	for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
		if (!mask[t]) out[t] = 0.0;
}

cudaError_t launch_mask_select64(double *out, unsigned ow, unsigned oh, const double *plain, const uint8_t *mask,
                                 unsigned dw, unsigned ox, unsigned oy, cudaStream_t s)
{
	dim3 block(32, 8), grid(cdiv(ow, 32), cdiv(oh, 8));
	k_mask_select64<<<grid, block, 0, s>>>(out, ow, oh, plain, mask, dw, ox, oy);
	note_launches(1);
	return cudaGetLastError();
}

cudaError_t launch_mask_and64(double *out, const uint8_t *mask, size_t n, cudaStream_t s)
{
	k_mask_and64<<<148 * 4, 256, 0, s>>>(out, mask, n);
	note_launches(1);
	return cudaGetLastError();
}

cudaError_t launch_levels64(const DevProfile *profiles, int n_levels, double *img_conv, double *img_plain,
                            const QueueSet &q, cudaStream_t s)
{
	const int wide = n_levels < 3 ? n_levels : 3;
	for (int l = 0; l < wide; l++) k_level64<<<148 * 8, 256, 0, s>>>(profiles, l, img_conv, img_plain, q);
	note_launches(wide);
	if (n_levels > wide) {
		k_deep_levels64<<<1, 512, 0, s>>>(profiles, wide, n_levels, img_conv, img_plain, q);
		note_launches(1);
	}
	return cudaGetLastError();
}

cudaError_t launch_count_decisions(const QueueSet &q, int n_levels, size_t npix, cudaStream_t s)
{
	for (int l = 0; l < n_levels; l++) k_count_decisions<<<148 * 4, 256, 0, s>>>(q, l, npix);
	note_launches(n_levels);
	return cudaGetLastError();
}

cudaError_t launch_psf_stamp64(const DevProfile *profiles, int p, const double *psf, unsigned psf_w, unsigned psf_h,
                               double psf_sx, double psf_sy, double scale_x, double scale_y, double offx, double offy,
                               unsigned width, unsigned height, double *img_conv, double *img_plain, cudaStream_t s)
{
	k_psf_stamp64<<<64, 256, 0, s>>>(profiles, p, psf, psf_w, psf_h, psf_sx, psf_sy, scale_x, scale_y, offx, offy,
	                                  width, height, img_conv, img_plain);
	note_launches(1);
	return cudaGetLastError();
}

cudaError_t launch_conv64(const double *src, int sw, int sh, int ox, int oy, const double *K, int kw, int kh,
                          double *out, int ow, int oh, const double *add, int add_stride, int add_ox, int add_oy,
                          cudaStream_t s)
{
	note_launches(1);
	static const ConvCandidate cands[] = {
	    {ConvVariant<double, double, double, 8, 4, 2>::smem, ConvVariant<double, double, double, 8, 4, 2>::run},
	    {ConvVariant<double, double, double, 8, 1, 8>::smem, ConvVariant<double, double, double, 8, 1, 8>::run},
	    {ConvVariant<double, double, double, 4, 2, 8>::smem, ConvVariant<double, double, double, 4, 2, 8>::run},
	    {ConvVariant<double, double, double, 8, 2, 4>::smem, ConvVariant<double, double, double, 8, 2, 4>::run},
	    {ConvVariant<double, double, double, 4, 4, 2>::smem, ConvVariant<double, double, double, 4, 4, 2>::run},
	};
	ConvArgs a{src, sw, sh, ox, oy, K, kw, kh, out, ow, oh, add, add_stride, add_ox, add_oy, 1, 0, 0};
	return conv_autotuned(cands, (int)(sizeof(cands) / sizeof(cands[0])), 3, a, s);
}

cudaError_t launch_loglike64(const double *model, const double *data, const double *sigma, const uint8_t *region,
                             int n, double2 *partials, int nparts, double *out, cudaStream_t s)
{
	k_loglike_partial<double><<<dim3(nparts, 1), 256, 0, s>>>(model, data, sigma, region, n, partials, nullptr, 0);
	k_loglike_final<<<1, 256, 0, s>>>(partials, nparts, out);
	note_launches(2);
	return cudaGetLastError();
}

cudaError_t launch_crop64(const double *src, unsigned sw, unsigned ox, unsigned oy, double *out, unsigned ow,
                          unsigned oh, const double *add, cudaStream_t s)
{
	dim3 block(32, 8), grid(cdiv(ow, 32), cdiv(oh, 8));
	k_crop64<<<grid, block, 0, s>>>(src, sw, ox, oy, out, ow, oh, add);
	note_launches(1);
	return cudaGetLastError();
}

cudaError_t launch_downsample64(const double *src, unsigned sw, unsigned sh, unsigned fs, double *out, unsigned ow,
                                unsigned oh, cudaStream_t s)
{
	dim3 block(32, 8), grid(cdiv(ow, 32), cdiv(oh, 8));
	k_downsample64<<<grid, block, 0, s>>>(src, sw, sh, fs, out, ow, oh);
	note_launches(1);
	return cudaGetLastError();
}

__global__ void k_widen(const float *__restrict__ src, double *__restrict__ dst, size_t n)
{
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
		dst[i] = (double)src[i];
}

cudaError_t launch_widen(const float *src, double *dst, size_t n, cudaStream_t s)
{
	k_widen<<<148 * 4, 256, 0, s>>>(src, dst, n);
	note_launches(1);
	return cudaGetLastError();
}

cudaError_t launch_like64(int kind, const double *model, const double *data, const double *sigma,
                          const uint8_t *region, int n, int batch, int data_batch_stride, double2 *partials,
                          int nparts, double *stats, double *out, float *wseed, cudaStream_t s, unsigned *tickets)
{
	// launched with programmatic serialisation: these kernels run inside the
	// FP32 pipeline's graph right after the convolution
	const dim3 grid(nparts, batch), b256(256), b32(32), gb(batch);
	cudaError_t e = cudaSuccess;
	auto go = [&](cudaError_t r) {
		if (e == cudaSuccess) e = r;
	};
	if (kind == LIKE_NORM && tickets) {
		go(launch_pdl(k_loglike_fused<double>, grid, b256, 0, s, model, data, sigma, region, n, partials, wseed,
		              data_batch_stride, tickets, out));
		note_launches(1);
		return e;
	}
	if (kind == LIKE_NORM) {
		go(launch_pdl(k_loglike_partial<double>, grid, b256, 0, s, model, data, sigma, region, n, partials, wseed,
		              data_batch_stride));
		go(launch_pdl(k_loglike_final, gb, b256, 0, s, (const double2 *)partials, nparts, out));
		note_launches(2);
		return e;
	}
	double *p1 = reinterpret_cast<double *>(partials);
	double *coef = stats + (size_t)batch * LIKE_STATS;
	switch (kind) {
	case LIKE_CHISQ:
		go(launch_pdl(k_like_stats<LIKE_CHISQ>, grid, b256, 0, s, model, data, sigma, region, n, data_batch_stride,
		              p1));
		go(launch_pdl(k_like_stats_final, gb, b32, 0, s, (const double *)p1, nparts, stats));
		go(launch_pdl(k_like_terms<LIKE_CHISQ>, grid, b256, 0, s, model, data, sigma, region, n, data_batch_stride,
		              (const double *)stats, partials, wseed));
		go(launch_pdl(k_like_terms_final<LIKE_CHISQ>, gb, b32, 0, s, (const double2 *)partials, nparts,
		              (const double *)stats, out, coef));
		note_launches(4);
		break;
	case LIKE_T:
		go(launch_pdl(k_like_stats<LIKE_T>, grid, b256, 0, s, model, data, sigma, region, n, data_batch_stride, p1));
		go(launch_pdl(k_like_stats_final, gb, b32, 0, s, (const double *)p1, nparts, stats));
		go(launch_pdl(k_like_terms<LIKE_T>, grid, b256, 0, s, model, data, sigma, region, n, data_batch_stride,
		              (const double *)stats, partials, (float *)nullptr));
		go(launch_pdl(k_like_terms_final<LIKE_T>, gb, b32, 0, s, (const double2 *)partials, nparts,
		              (const double *)stats, out, coef));
		note_launches(4);
		if (wseed) {
			go(launch_pdl(k_like_t_seed, grid, b256, 0, s, model, data, sigma, region, n, data_batch_stride,
			              (const double *)stats, (const double *)coef, wseed));
			note_launches(1);
		}
		break;
	case LIKE_POIS:
		go(launch_pdl(k_like_stats<LIKE_POIS>, grid, b256, 0, s, model, data, sigma, region, n, data_batch_stride,
		              p1));
		go(launch_pdl(k_like_stats_final, gb, b32, 0, s, (const double *)p1, nparts, stats));
		go(launch_pdl(k_like_terms<LIKE_POIS>, grid, b256, 0, s, model, data, sigma, region, n, data_batch_stride,
		              (const double *)stats, partials, wseed));
		go(launch_pdl(k_like_terms_final<LIKE_POIS>, gb, b32, 0, s, (const double2 *)partials, nparts,
		              (const double *)stats, out, coef));
		note_launches(4);
		break;
	default: return cudaErrorInvalidValue;
	}
	return e;
}

cudaError_t launch_loglike64_seed(const double *model, const double *data, const double *sigma,
                                  const uint8_t *region, int n, double2 *partials, int nparts, double *out,
                                  float *wseed, cudaStream_t s)
{
	k_loglike_partial<double><<<dim3(nparts, 1), 256, 0, s>>>(model, data, sigma, region, n, partials, wseed, 0);
	k_loglike_final<<<1, 256, 0, s>>>(partials, nparts, out);
	note_launches(2);
	return cudaGetLastError();
}

}  // namespace pf
