// Shared device-side types of the render / convolution / likelihood kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "profiles.cuh"

namespace pf {

// Programmatic dependent launch.  The kernels of the FP32 pipeline are
// launched with programmatic stream serialisation (launch_pdl): the next
// kernel of the stream may be scheduled onto free SM slots while this one
// runs, and it waits in griddepcontrol.wait until this grid has finished and
// its writes are visible, which hides the launch gap between dependent
// kernels.  Every kernel launched that way calls pdl_enter() before its first
// access to memory that an earlier kernel of the stream writes or reads; for
// an ordinary launch both instructions are no-ops.
__device__ __forceinline__ void pdl_enter()
{
	asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
	asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args... args)
{
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = grid;
	cfg.blockDim = block;
	cfg.dynamicSmemBytes = smem;
	cfg.stream = s;
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	attr[0].val.programmaticStreamSerializationAllowed = 1;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
	return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Tangent slots per radial profile: f, df/dx', df/dy', df/dx' y', df/dy' x',
// df/dy' y', then the shape-parameter partials (per kind, shape_count of
// them) and df/dbox.  Models whose profiles need fewer slots store fewer
// planes (tangent_stride).
constexpr int NTAN = 12;

// profitLikeModel's like.func (R/profitUtility.R:99-121, without "st").
enum LikeKind : int { LIKE_NORM = 0, LIKE_CHISQ = 1, LIKE_T = 2, LIKE_POIS = 3 };
constexpr int LIKE_SCRATCH_PER_IMAGE = 5;  // doubles of launch_like64's stats scratch per image

// Partial sums per image of the likelihood reduction (its grid) for `batch`
// images of n pixels: enough blocks in all to fill the GPU, at least about
// two pixels per thread (a batch of thousands of small images would
// otherwise spend its time reducing near-empty blocks), at most
// LIKE_MAX_PARTS.  The merge order of the partials, hence the last bit of
// logL, follows from this count.
constexpr int LIKE_MAX_PARTS = 296;  // 2 per SM
inline int like_parts(int n, int batch)
{
	const int b = batch > 1 ? batch : 1;
	const int fill = (148 * 16 + b - 1) / b;
	const int work = (n + 511) / 512;
	int p = fill < work ? fill : work;
	p = p < LIKE_MAX_PARTS ? p : LIKE_MAX_PARTS;
	return p > 1 ? p : 1;
}
constexpr int NTAN_GEOM = 6;

// Tangent slots a profile of this kind fills (geometry, shape, box).
PF_HD inline int tangent_count(int kind) { return NTAN_GEOM + shape_count(kind) + 1; }

// One cell waiting to be integrated by adaptive subsampling
// (one pending call of RadialProfile::subsample_pixel, radial.cpp:54).
// FP64 path: bounds in drawing-pixel coordinates.  FP32 path: bounds
// relative to the profile centre.
struct SubItem {
	double x0, x1, y0, y1;
	double weight;      // flux_scale / (res^2)^(level+1)
	uint32_t pixel;     // drawing-pixel index (x + y*width)
	uint16_t profile;
	uint8_t res, max_rec;
};

// Device work queue: one segment per recursion level inside one buffer.
// counts[L] keeps counting past cap[L]; the host reads it back to size a
// retry, so an overflow is reported (never written out of bounds).
constexpr int MAX_LEVELS = 16;
// Control words after counts[MAX_LEVELS], overflow and maxres: per wide level
// (0..2) a histogram of the items' radial kinds and the scatter cursors.
constexpr int KIND_CTR = MAX_LEVELS + 2;
constexpr int N_RADIAL_KINDS = 6;
// Accepted sub-points of an item (res^2 <= 256 bits), recorded by the
// forward pass when the adjoint recomputes instead of storing tangents.
constexpr int MASK_WORDS = 8;
struct QueueSet {
	SubItem *items;
	uint32_t *masks;       // optional [items][MASK_WORDS], parallel to items
	uint32_t *counts;      // [MAX_LEVELS]
	uint32_t *overflow;    // set to 1 when an item had to be dropped
	int32_t *decisions;    // optional [n_profiles][npix] subsample_pixel calls per pixel
	unsigned long long *level_counts;  // optional [n_profiles][MAX_LEVELS]
	// optional [n_profiles][1 + MAX_LEVELS]: profile evaluations (evaluate_at
	// calls in libprofit's terms), the direct ones first, then per level
	unsigned long long *evals = nullptr;
	uint32_t *maxres = nullptr;  // optional: largest resolution of the level-0 items pushed
	// optional: per level, the items' indices grouped by profile kind (filled
	// by launch_levels32 before each wide level when set; same offsets as items)
	uint32_t *perm = nullptr;
	uint32_t levels;
	uint32_t off[MAX_LEVELS];
	uint32_t cap[MAX_LEVELS];
};

// Compact FP32 copy of a radial profile's scalars for the FP32 kernels.
struct FProfile {
	int32_t kind, target, rough, centre_override;
	uint32_t resolution, max_rec;
	float cos_ang, sin_ang, cos_q, sin_q;
	float r_switch, r_max, acc;
	float re, nser, bn, B, inv_nB, dbn_dn;
	float rscale, con, a, b, rb, rc, rt, h1, h2, king_t;
	float flux_scale;
	// Per-profile constants of the FP32 profile functions, formed in FP64 and
	// rounded once (an FP32 reciprocal of an FP32 parameter would round twice,
	// and that error is the same at every pixel): inv_B = 1/B and
	// box_e = (2 - B)/(2 B) for the boxy radius, and by kind
	//   sersic:     1/re, 1/nser
	//   moffat:     1/rscale;  ferrer: 1/rout
	//   king:       1/a, 1/rc, 1/(1 + (rt/rc)^2), ln(1 + (rt/rc)^2)
	//   brokenexp:  1/h1, 1/h2, 1/a
	//   coresersic: 1/a, 1/nser, ln rb, ln re, rb^a, re^-a, 1/(nser a)
	float inv_B, box_e;
	float k[7];
	double cx, cy, img_sx, img_sy, flux_scale64;
};

PF_HD inline FProfile to_fprofile(const DevProfile &d, const ProfileParams &p)
{
	FProfile f = {};
	f.kind = d.kind;
	f.target = d.target;
	f.rough = d.rough;
	f.centre_override = d.centre_override;
	f.resolution = d.resolution;
	f.max_rec = d.max_rec;
	f.cos_ang = (float)d.cos_ang;
	f.sin_ang = (float)d.sin_ang;
	f.cos_q = (float)d.cos_q;
	f.sin_q = (float)d.sin_q;
	f.r_switch = (float)d.r_switch;
	f.r_max = (float)d.r_max;
	f.acc = (float)d.acc;
	f.re = (float)d.re;
	f.nser = (float)d.nser;
	f.bn = (float)d.bn;
	f.B = (float)(p.box + 2);
	f.inv_nB = (float)(1.0 / (p.nser * (p.box + 2)));
	f.dbn_dn = (float)d.dbn_dn;
	f.rscale = (float)d.rscale;
	f.con = (float)d.con;
	f.a = (float)d.a;
	f.b = (float)d.b;
	f.rb = (float)d.rb;
	f.rc = (float)d.rc;
	f.rt = (float)d.rt;
	f.h1 = (float)d.h1;
	f.h2 = (float)d.h2;
	f.king_t = (float)d.king_t;
	f.flux_scale = (float)d.flux_scale;
	f.flux_scale64 = d.flux_scale;
	f.cx = d.cx;
	f.cy = d.cy;
	f.img_sx = d.img_sx;
	f.img_sy = d.img_sy;
	if (d.kind == PK_SKY) f.flux_scale = (float)d.bg;
	if (d.kind == PK_MOFFAT) {
		// Moffat keeps 1/fwhm and d ln(rscale)/d con in the a, b slots
		double c = p.con, t = pow(2.0, 1.0 / c);
		f.a = (float)(1.0 / p.fwhm);
		f.b = (float)(0.5 * t * log(2.0) / (c * c * (t - 1.0)));
	}
	const double B = p.box + 2;
	f.inv_B = (float)(1.0 / B);
	f.box_e = (float)((2.0 - B) / (2.0 * B));
	switch (d.kind) {
	case PK_SERSIC:
		f.k[0] = (float)(1.0 / d.re);
		f.k[1] = (float)(1.0 / d.nser);
		break;
	case PK_MOFFAT:
	case PK_FERRER: f.k[0] = (float)(1.0 / d.rscale); break;
	case PK_KING: {
		const double Y = 1.0 + (d.rt / d.rc) * (d.rt / d.rc);
		f.k[0] = (float)(1.0 / d.a);
		f.k[1] = (float)(1.0 / d.rc);
		f.k[2] = (float)(1.0 / Y);
		f.k[3] = (float)log(Y);
		break;
	}
	case PK_BROKENEXP:
		f.k[0] = (float)(1.0 / d.h1);
		f.k[1] = (float)(1.0 / d.h2);
		f.k[2] = (float)(1.0 / d.a);
		break;
	case PK_CORESERSIC:
		f.k[0] = (float)(1.0 / d.a);
		f.k[1] = (float)(1.0 / d.nser);
		f.k[2] = (float)log(d.rb);
		f.k[3] = (float)log(d.re);
		f.k[4] = (float)pow(d.rb, d.a);
		f.k[5] = (float)pow(d.re, -d.a);
		f.k[6] = (float)(1.0 / (d.nser * d.a));
		break;
	default: break;
	}
	return f;
}

// Parameters with a hand-written adjoint, and how their derivative is
// assembled from the tangent reductions T[0..8] of the render pass:
//   x' = dx c + dy s,  y' = (-dx s + dy c)/q,  theta = (ang + 90) pi/180,
//   d x'/d xcen = -c, d y'/d xcen = s/q, d x'/d ycen = -s, d y'/d ycen = -c/q,
//   d x'/d theta = q y', d y'/d theta = -x'/q, d y'/d q = -y'/q,
// and flux_scale F carries d ln F / d(mag, q, box, shape) from the prologue.
// G_SHAPE + k: shape parameter k of the profile's kind (shape_count order).
enum GradCode : int32_t { G_XCEN = 0, G_YCEN, G_MAG, G_ANG, G_AXRAT, G_BOX, G_SHAPE };

PF_HD inline double gradient_from_tangents(int code, double axrat, const DevProfile &d, const double *T)
{
	if (d.kind == PK_PSF) {
		// psf point source: T = sums of g times its stamp and the stamp's
		// derivatives in xcen and ycen (k_psf_adjoint32), flux 10^(-0.4(mag-mz))
		switch (code) {
		case G_XCEN: return d.psf_flux * T[1];
		case G_YCEN: return d.psf_flux * T[2];
		case G_MAG: return d.psf_flux * d.dlnI_dmag * T[0];
		default: return 0.0;
		}
	}
	const double F = d.flux_scale, q = axrat, c = d.cos_ang, s = d.sin_ang;
	switch (code) {
	case G_XCEN: return F * (-c * T[1] + (s / q) * T[2]);
	case G_YCEN: return F * (-s * T[1] - (c / q) * T[2]);
	case G_MAG: return F * d.dlnI_dmag * T[0];
	case G_ANG: return F * (M_PI / 180.0) * (q * T[3] - T[4] / q);
	case G_AXRAT: return F * (-T[5] / q + d.dlnI_dq * T[0]);
	case G_BOX: return F * (T[NTAN_GEOM + shape_count(d.kind)] + d.dlnI_dbox * T[0]);
	default: {
		const int k = code - G_SHAPE;
		return F * (T[NTAN_GEOM + k] + d.dlnI_dp[k] * T[0]);
	}
	}
}

// floor(value) bounded to [0, max] (libprofit's bind for the psf profile's
// pixel ranges, psf.cpp:40-50).
__device__ __forceinline__ unsigned bind_u(double value, unsigned max)
{
	int intval = (int)floor(value);
	if (intval < 0) return 0;
	unsigned u = (unsigned)intval;
	return u < max ? u : max;
}

__device__ __forceinline__ uint32_t warp_push(uint32_t *counter)
{
	uint32_t mask = __activemask();
	int lane = threadIdx.x & 31;
	int leader = __ffs(mask) - 1;
	uint32_t rank = __popc(mask & ((1u << lane) - 1u));
	uint32_t base = 0;
	if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
	base = __shfl_sync(mask, base, leader);
	return base + rank;
}

// Raises *q.maxres to `res` (one atomic per warp of pushing threads).
__device__ __forceinline__ void note_max_res(const QueueSet &q, uint32_t res)
{
	if (!q.maxres) return;
	const uint32_t mask = __activemask();
	const uint32_t m = __reduce_max_sync(mask, res);
	if ((int)(threadIdx.x & 31) == __ffs(mask) - 1) atomicMax(q.maxres, m);
}

__device__ __forceinline__ void queue_push(const QueueSet &q, uint32_t level, const SubItem &it)
{
	uint32_t idx = warp_push(&q.counts[level]);
	if (idx < q.cap[level]) {
		q.items[(size_t)q.off[level] + idx] = it;
	}
	else {
		atomicOr(q.overflow, 1u);
	}
}

template <class T>
__device__ __forceinline__ T warp_sum(T v)
{
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

// Sums of N <= 16 values over the warp with 16 shuffles instead of 5 per
// value: at each halving step a lane keeps one half of its values and adds
// the partner's copy of that half.  Returns, in lanes 2m and 2m + 1, the
// warp's sum of value m (zero for m >= N).
template <int N, class T>
__device__ __forceinline__ T warp_sums_spread(const T (&v)[N], int lane)
{
	static_assert(N <= 16, "up to 16 values");
	T a[16];
#pragma unroll
	for (int i = 0; i < 16; i++) a[i] = i < N ? v[i] : T(0);
#pragma unroll
	for (int h = 8; h >= 1; h >>= 1) {
		const bool upper = lane & (2 * h);  // this lane keeps values h .. 2h-1 of the current block
#pragma unroll
		for (int i = 0; i < h; i++) {
			const T keep = upper ? a[i + h] : a[i];
			const T give = upper ? a[i] : a[i + h];
			a[i] = keep + __shfl_xor_sync(0xffffffffu, give, 2 * h);
		}
	}
	return a[0] + __shfl_xor_sync(0xffffffffu, a[0], 1);
}

}  // namespace pf
