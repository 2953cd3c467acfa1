// Shared device-side types of the render / convolution / likelihood kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "profiles.cuh"

namespace pf {

// Number of per-pixel tangent sums kept for each radial profile by the FP32
// path: f, df/dx', df/dy', df/dx'*y', df/dy'*x', df/dy'*y', and the three
// shape partials (Sersic: re, nser, box; Moffat: fwhm, con, box).
constexpr int NTAN = 9;

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
struct QueueSet {
	SubItem *items;
	uint32_t *counts;      // [MAX_LEVELS]
	uint32_t *overflow;    // set to 1 when an item had to be dropped
	int32_t *decisions;    // optional [n_profiles][npix] subsample_pixel calls per pixel
	unsigned long long *level_counts;  // optional [n_profiles][MAX_LEVELS]
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
	double cx, cy, img_sx, img_sy, flux_scale64;
};

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

}  // namespace pf
