// ProFit's "norm" log-likelihood (R/profitLikeModel.R:263-276):
//   cutsig = (image - model) / sigma,  LL = sum(dnorm(cutsig, log = TRUE))
// with dnorm(x, 0, 1, log) = -(log(sqrt(2 pi)) + x^2/2).
//
// The sum runs in FP64 with Neumaier compensation per thread, a shuffle
// reduction of (sum, compensation) pairs per warp and block, one partial per
// block, and a one-block final pass: deterministic for a fixed grid.  The
// same pass can write the adjoint seed dLL/dmodel = (image - model)/sigma^2.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace pf {

struct Neumaier {
	double s, c;
};

__device__ __forceinline__ void neumaier_add(Neumaier &a, double x)
{
	double t = a.s + x;
	if (fabs(a.s) >= fabs(x)) a.c += (a.s - t) + x;
	else a.c += (x - t) + a.s;
	a.s = t;
}

__device__ __forceinline__ Neumaier neumaier_merge(Neumaier a, Neumaier b)
{
	Neumaier r;
	r.c = a.c + b.c;
	r.s = a.s;
	neumaier_add(r, b.s);
	return r;
}

__device__ __forceinline__ Neumaier neumaier_warp(Neumaier v)
{
	for (int o = 16; o > 0; o >>= 1) {
		Neumaier other;
		other.s = __shfl_xor_sync(0xffffffffu, v.s, o);
		other.c = __shfl_xor_sync(0xffffffffu, v.c, o);
		v = neumaier_merge(v, other);
	}
	return v;
}

__device__ __forceinline__ Neumaier neumaier_block(Neumaier v)
{
	__shared__ double s_s[32], s_c[32];
	int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	v = neumaier_warp(v);
	if (lane == 0) {
		s_s[wid] = v.s;
		s_c[wid] = v.c;
	}
	__syncthreads();
	int nw = (blockDim.x + 31) >> 5;
	if (wid == 0) {
		Neumaier u{0.0, 0.0};
		if (lane < nw) {
			u.s = s_s[lane];
			u.c = s_c[lane];
		}
		v = neumaier_warp(u);
	}
	return v;
}

constexpr double LN_SQRT_2PI = 0.918938533204672741780329736406;

// The terms of image b handled by this block (grid-stride over its n
// pixels), Neumaier-summed per thread and merged over the block (the total
// is valid in thread 0); writes the adjoint seed when wseed is set.
template <class T>
__device__ __forceinline__ Neumaier loglike_block_terms(const T *__restrict__ model, const double *__restrict__ data,
                                                        const double *__restrict__ sigma,
                                                        const uint8_t *__restrict__ region, int n,
                                                        float *__restrict__ wseed, int data_batch_stride, int b)
{
	model += (size_t)b * n;
	data += (size_t)b * data_batch_stride;
	sigma += (size_t)b * data_batch_stride;
	if (region) region += (size_t)b * data_batch_stride;
	if (wseed) wseed += (size_t)b * n;
	Neumaier acc{0.0, 0.0};
	for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		bool use = !region || region[k];
		double m = (double)model[k];
		double s = sigma[k];
		double diff = data[k] - m;
		if (use) {
			double x = diff / s;
			neumaier_add(acc, -(LN_SQRT_2PI + 0.5 * x * x));
		}
		if (wseed) wseed[k] = use ? (float)(diff / (s * s)) : 0.0f;
	}
	return neumaier_block(acc);
}

// logL of one image from its nparts partials: thread t merges partials t,
// t + blockDim, ... in order, then the block merges in a fixed order, so
// the value does not depend on which blocks produced the partials first.
// The partials are read from L2 (they may have been written by other SMs in
// this same kernel).
__device__ __forceinline__ void loglike_merge_partials(const double2 *partials, int nparts, double *out)
{
	Neumaier acc{0.0, 0.0};
	for (int k = threadIdx.x; k < nparts; k += blockDim.x) {
		double2 p = __ldcg(partials + k);
		acc = neumaier_merge(acc, Neumaier{p.x, p.y});
	}
	acc = neumaier_block(acc);
	if (threadIdx.x == 0) *out = acc.s + acc.c;
}

// n pixels per image, `batch` images laid out back to back; one partial
// (s, c) per block in partials[batch][gridDim.x].
template <class T>
__global__ void k_loglike_partial(const T *__restrict__ model, const double *__restrict__ data,
                                  const double *__restrict__ sigma, const uint8_t *__restrict__ region, int n,
                                  double2 *__restrict__ partials, float *__restrict__ wseed,
                                  int data_batch_stride)
{
	pdl_enter();
	const int b = blockIdx.y;
	const Neumaier acc = loglike_block_terms<T>(model, data, sigma, region, n, wseed, data_batch_stride, b);
	if (threadIdx.x == 0) partials[(size_t)b * gridDim.x + blockIdx.x] = make_double2(acc.s, acc.c);
}

static __global__ void k_loglike_final(const double2 *__restrict__ partials, int nparts, double *__restrict__ out)
{
	pdl_enter();
	const int b = blockIdx.x;
	loglike_merge_partials(partials + (size_t)b * nparts, nparts, out + b);
}

// k_loglike_partial and k_loglike_final in one launch: the block that
// finishes image b last (a ticket per image, counted with atomics after each
// block's partial is visible) merges its partials exactly as the final
// kernel does and resets the ticket.  tickets[batch] start at zero.
template <class T>
__global__ void k_loglike_fused(const T *__restrict__ model, const double *__restrict__ data,
                                const double *__restrict__ sigma, const uint8_t *__restrict__ region, int n,
                                double2 *__restrict__ partials, float *__restrict__ wseed, int data_batch_stride,
                                unsigned *__restrict__ tickets, double *__restrict__ out)
{
	pdl_enter();
	const int b = blockIdx.y;
	const Neumaier acc = loglike_block_terms<T>(model, data, sigma, region, n, wseed, data_batch_stride, b);
	__shared__ bool s_last;
	if (threadIdx.x == 0) {
		partials[(size_t)b * gridDim.x + blockIdx.x] = make_double2(acc.s, acc.c);
		__threadfence();
		s_last = atomicAdd(&tickets[b], 1u) == gridDim.x - 1;
	}
	__syncthreads();  // also orders this block's reuse of neumaier_block's shared arrays
	if (!s_last) return;
	__threadfence();
	loglike_merge_partials(partials + (size_t)b * gridDim.x, gridDim.x, out + b);
	if (threadIdx.x == 0) tickets[b] = 0;
}

}  // namespace pf
