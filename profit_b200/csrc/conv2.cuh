// FP32 brute-force convolution on the packed FP32 FMA of sm_100
// (fma.rn.f32x2 through __ffma2_rn): the same correlation as k_conv_tile,
//
//   out(i, j) = sum_{k < kw, l < kh} src(i + ox + k, j + oy + l) * K(k, l),
//
// summed the same way (the taps of one kernel column in FP32 in increasing l,
// the column sums in FP64, partial results merged in a fixed order), with
// half the FMA instructions: a lane owns output columns i and i + HL and
// updates both with one packed FMA.
//
// Work decomposition.  A CTA owns a (2 HL) x TY output tile and a range of
// kernel columns (KSPLIT ranges per tile, blockIdx.z = image * KSPLIT +
// range).  Inside the CTA, warps are TYT row groups x KS column groups; a
// warp holds 32/HL row groups of HL lanes, each thread RY rows of its two
// columns.  With KSPLIT > 1 each CTA writes its FP64 partial tile to a
// scratch buffer and k_conv_split_sum adds the ranges in order (plus the
// `add` image): small images then spread over all SMs without atomics, and
// the result does not depend on scheduling.
//
// Shared memory.  The source tile is stored pre-paired and transposed: entry
// (j, row) = (src col j, src col j + HL) at j * thp + row, thp = th rounded
// up to odd.  A lane's window slides down contiguous entries, so every tap
// address is a base register plus an immediate; consecutive lanes are thp
// entries apart (odd), which keeps 8-byte loads free of bank conflicts.
// Kernel taps are stored duplicated, (K, K), two taps per 16-byte load.
//
// Inner loop: per tap one 8-byte load, half a 16-byte load and RY packed
// FMAs.  The window is a ring of WR = RY + 2 registers indexed at compile
// time (the loop over kernel rows is unrolled by WR), so sliding it moves
// nothing, and each row is loaded two taps before its first use, which
// keeps the shared-memory latency off the FMA chain.  The last two rows of
// the tile (one past the halo) are loaded by that prefetch but never used.
#pragma once

#include <algorithm>

#include <cuda_runtime.h>

#include "conv.cuh"
#include "launch.h"

namespace pf {

// 4-byte asynchronous global->shared copy; with `valid` false nothing is read
// and the destination is zero-filled (the halo outside the image).
__device__ __forceinline__ void cp_async4_zfill(float *dst, const float *src, bool valid)
{
	unsigned d = (unsigned)__cvta_generic_to_shared(dst);
	int n = valid ? 4 : 0;
	asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
	asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

__host__ __device__ constexpr int conv3_ncols(int kw, int ksplit) { return (kw + ksplit - 1) / ksplit; }

template <int HL, int RY, int TYT, int KS, int KSPLIT>
struct Conv3Shape {
	static constexpr int NG = 32 / HL;         // row groups per warp
	static constexpr int TX = 2 * HL;          // output columns per tile
	static constexpr int TY = TYT * NG * RY;   // output rows per tile
	static constexpr int NTHR = 32 * TYT * KS;
	__host__ __device__ static int khp(int kh) { return (kh + 1) & ~1; }
	// rows TY + kh - 1 of the tile plus one the prefetch reads, rounded to odd
	__host__ __device__ static int thp(int kh) { return (TY + kh + 1) | 1; }
	__host__ __device__ static int twj(int kw) { return HL + conv3_ncols(kw, KSPLIT) - 1; }
	__host__ __device__ static size_t tile_bytes(int kw, int kh)
	{
		return 8 * ((size_t)conv3_ncols(kw, KSPLIT) * khp(kh) + (size_t)twj(kw) * thp(kh));
	}
	static size_t smem(int kw, int kh)
	{
		size_t red = 16 * (size_t)(KS - 1) * RY * TYT * 32;  // reuses the tile after the column loop
		size_t t = tile_bytes(kw, kh);
		return t > red ? t : red;
	}
};

// One tap at ring position Q: prefetch the row two taps ahead, then RY
// packed FMAs on the rows Q .. Q + RY - 1.
template <int RY, int Q>
__device__ __forceinline__ void conv3_tap(float2 (&win)[RY + 2], float2 (&acc)[RY], const float2 *col, float2 c)
{
	constexpr int WR = RY + 2;
	win[(Q + RY + 1) % WR] = col[Q + RY + 1];
#pragma unroll
	for (int r = 0; r < RY; r++) acc[r] = __ffma2_rn(win[(Q + r) % WR], c, acc[r]);
}

// WR taps starting at kernel row l (col and kc already advanced to l).
template <int RY, int Q>
__device__ __forceinline__ void conv3_steps(float2 (&win)[RY + 2], float2 (&acc)[RY], const float2 *col,
                                            const float4 *kc)
{
	if constexpr (Q < RY + 2) {
		float4 c2 = kc[Q >> 1];
		conv3_tap<RY, Q>(win, acc, col, make_float2(c2.x, c2.y));
		conv3_tap<RY, Q + 1>(win, acc, col, make_float2(c2.z, c2.w));
		conv3_steps<RY, Q + 2>(win, acc, col, kc);
	}
}

// The last rem < WR taps of a column, same ring positions.
template <int RY, int Q>
__device__ __forceinline__ void conv3_tail(float2 (&win)[RY + 2], float2 (&acc)[RY], const float2 *col,
                                           const float4 *kc, int rem)
{
	if constexpr (Q < RY + 2) {
		if (Q < rem) {
			float4 c2 = kc[Q >> 1];
			conv3_tap<RY, Q>(win, acc, col, make_float2(c2.x, c2.y));
			if (Q + 1 < rem) conv3_tap<RY, Q + 1>(win, acc, col, make_float2(c2.z, c2.w));
			conv3_tail<RY, Q + 2>(win, acc, col, kc, rem);
		}
	}
}

// All KHC taps of a kernel column with the window ring at compile-time
// positions (tap L uses ring slots (L + r) % (RY + 2)): no loop and no tail.
template <int RY, int L, int KHC>
__device__ __forceinline__ void conv3_column(float2 (&win)[RY + 2], float2 (&acc)[RY], const float2 *col,
                                             const float4 *kc)
{
	if constexpr (L < KHC) {
		const float4 c2 = kc[L >> 1];
		conv3_tap<RY, L>(win, acc, col, make_float2(c2.x, c2.y));
		if constexpr (L + 1 < KHC) conv3_tap<RY, L + 1>(win, acc, col, make_float2(c2.z, c2.w));
		conv3_column<RY, L + 2, KHC>(win, acc, col, kc);
	}
}

// TOut: output type (FP32 adjoint image or FP64 model image).  `part` is the
// FP64 scratch [batch][KSPLIT][oh][ow] used when KSPLIT > 1.  KHC > 0: the
// kernel height fixed at compile time (launches with another height are not
// applicable), the taps of a column fully unrolled.
template <class TOut, int HL, int RY, int TYT, int KS, int KSPLIT, int KHC = 0>
__global__ void __launch_bounds__(32 * TYT * KS)
    k_conv3_tile(const float *__restrict__ src, int sw, int sh, int ox, int oy, const float *__restrict__ K, int kw,
                 int kh_arg, TOut *__restrict__ out, int ow, int oh, const float *__restrict__ add, int add_stride,
                 int add_ox, int add_oy, int batch_src_stride, int batch_out_stride, int batch_k_stride,
                 double *__restrict__ part)
{
	using S = Conv3Shape<HL, RY, TYT, KS, KSPLIT>;
	const int kh = KHC > 0 ? KHC : kh_arg;
	static_assert(RY % 2 == 0, "taps are consumed in pairs");
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int khp = S::khp(kh), thp = S::thp(kh);
	const int th = S::TY + kh - 1;

	const int b = blockIdx.z / KSPLIT, split = blockIdx.z - b * KSPLIT;
	const int ncol = conv3_ncols(kw, KSPLIT);
	const int k_lo = split * ncol;
	const int nk = max(0, min(kw, k_lo + ncol) - k_lo);  // kernel columns of this CTA
	const int twj = HL + nk - 1;
	float2 *s_k = reinterpret_cast<float2 *>(smem_raw);  // [ncol][khp], (K, K)
	float2 *s_src = s_k + (size_t)ncol * khp;            // [twj][thp], transposed pairs

	src += (size_t)b * batch_src_stride;
	K += (size_t)b * batch_k_stride;
	const int i0 = blockIdx.x * S::TX;
	const int j0 = blockIdx.y * S::TY;
	constexpr int NWARPS = TYT * KS;
	const int wid = threadIdx.y + TYT * threadIdx.z;

	// fill, every copy in flight at once: kernel columns (lane per tap), then
	// source rows (lane per entry, coalesced global reads)
	for (int k = wid; k < nk; k += NWARPS)
		for (int l = threadIdx.x; l < khp; l += 32) {
			const bool v = l < kh;
			const float *g = v ? K + (k_lo + k) + (size_t)l * kw : K;
			float *d = reinterpret_cast<float *>(s_k + (size_t)k * khp + l);
			cp_async4_zfill(d, g, v);
			cp_async4_zfill(d + 1, g, v);
		}
	// the kernel taps are static; the source is the previous kernel's output
	pdl_enter();
	for (int ty = wid; ty < th; ty += NWARPS) {
		const int sy = j0 + oy + ty;
		const bool rv = sy >= 0 && sy < sh;
		const float *row = rv ? src + (size_t)sy * sw : src;
		for (int tx = threadIdx.x; tx < twj; tx += 32) {
			const int sx = i0 + ox + k_lo + tx;
			const bool va = rv && sx >= 0 && sx < sw;
			const bool vc = rv && sx + HL >= 0 && sx + HL < sw;
			float *d = reinterpret_cast<float *>(s_src + (size_t)tx * thp + ty);
			cp_async4_zfill(d, va ? row + sx : src, va);
			cp_async4_zfill(d + 1, vc ? row + sx + HL : src, vc);
		}
	}
	cp_async_wait_all();
	__syncthreads();

	const int hl = threadIdx.x % HL;
	const int r0 = (threadIdx.y * S::NG + threadIdx.x / HL) * RY;
	double2 tot[RY];
#pragma unroll
	for (int r = 0; r < RY; r++) tot[r] = make_double2(0.0, 0.0);

	for (int k = threadIdx.z; k < nk; k += KS) {
		const float2 *col = s_src + (size_t)(hl + k) * thp + r0;
		const float4 *kc = reinterpret_cast<const float4 *>(s_k + (size_t)k * khp);
		constexpr int WR = RY + 2;
		float2 acc[RY], win[WR];
#pragma unroll
		for (int r = 0; r < RY; r++) acc[r] = make_float2(0.0f, 0.0f);
#pragma unroll
		for (int r = 0; r < RY + 1; r++) win[r] = col[r];
		if constexpr (KHC > 0) {
			conv3_column<RY, 0, KHC>(win, acc, col, kc);
		}
		else {
			int l = 0;
			for (; l + WR <= kh; l += WR) conv3_steps<RY, 0>(win, acc, col + l, kc + (l >> 1));
			conv3_tail<RY, 0>(win, acc, col + l, kc + (l >> 1), kh - l);
		}
#pragma unroll
		for (int r = 0; r < RY; r++) {
			tot[r].x += (double)acc[r].x;
			tot[r].y += (double)acc[r].y;
		}
	}

	if (KS > 1) {
		// column groups 1..KS-1 hand their sums to group 0 (fixed order)
		__syncthreads();
		double2 *s_red = reinterpret_cast<double2 *>(smem_raw);
		const int t = threadIdx.y * 32 + threadIdx.x;
		if (threadIdx.z > 0) {
#pragma unroll
			for (int r = 0; r < RY; r++) s_red[((threadIdx.z - 1) * RY + r) * (TYT * 32) + t] = tot[r];
		}
		__syncthreads();
		if (threadIdx.z > 0) return;
#pragma unroll
		for (int g = 1; g < KS; g++)
#pragma unroll
			for (int r = 0; r < RY; r++) {
				double2 v = s_red[((g - 1) * RY + r) * (TYT * 32) + t];
				tot[r].x += v.x;
				tot[r].y += v.y;
			}
	}

	const int ia = i0 + hl, ib = ia + HL;
	if (KSPLIT > 1) {
		double *p = part + (size_t)blockIdx.z * oh * ow;
#pragma unroll
		for (int r = 0; r < RY; r++) {
			int j = j0 + r0 + r;
			if (j >= oh) break;
			if (ia < ow) p[ia + (size_t)j * ow] = tot[r].x;
			if (ib < ow) p[ib + (size_t)j * ow] = tot[r].y;
		}
		return;
	}
	out += (size_t)b * batch_out_stride;
	if (add) add += (size_t)b * batch_src_stride;
#pragma unroll
	for (int r = 0; r < RY; r++) {
		int j = j0 + r0 + r;
		if (j >= oh) break;
		double va = tot[r].x, vb = tot[r].y;
		if (add) {
			const float *arow = add + (size_t)(j + add_oy) * add_stride + add_ox;
			if (ia < ow) va += (double)arow[ia];
			if (ib < ow) vb += (double)arow[ib];
		}
		if (ia < ow) out[ia + (size_t)j * ow] = (TOut)va;
		if (ib < ow) out[ib + (size_t)j * ow] = (TOut)vb;
	}
}

// Adds the KSPLIT partial images of each output in order, then the `add`
// image, and converts to TOut.
template <class TOut>
__global__ void k_conv_split_sum(const double *__restrict__ part, int ksplit, TOut *__restrict__ out, int ow, int oh,
                                 int batch, const float *__restrict__ add, int add_stride, int add_ox, int add_oy,
                                 int batch_src_stride, int batch_out_stride)
{
	pdl_enter();
	const size_t n = (size_t)ow * oh;
	for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n * batch; t += (size_t)gridDim.x * blockDim.x) {
		const size_t b = t / n, p = t - b * n;
		const int j = (int)(p / ow), i = (int)(p - (size_t)j * ow);
		const double *q = part + b * ksplit * n + p;
		double v = q[0];
		for (int s = 1; s < ksplit; s++) v += q[s * n];
		if (add) v += (double)add[b * batch_src_stride + (size_t)(j + add_oy) * add_stride + i + add_ox];
		out[b * batch_out_stride + p] = (TOut)v;
	}
}

template <class TOut, int HL, int RY, int TYT, int KS, int KSPLIT, int KHC = 0>
struct Conv3Variant {
	using S = Conv3Shape<HL, RY, TYT, KS, KSPLIT>;
	// a fixed-height variant does not apply to other kernel heights
	static size_t smem(int kw, int kh) { return (KHC > 0 && kh != KHC) ? ~(size_t)0 >> 1 : S::smem(kw, kh); }
	static cudaError_t run(const ConvArgs &a, cudaStream_t s)
	{
		if (KHC > 0 && a.kh != KHC) return cudaErrorInvalidValue;
		if (KSPLIT > 1 && (!a.scratch || a.scratch_bytes < (size_t)a.batch * KSPLIT * a.ow * a.oh * sizeof(double)))
			return cudaErrorInvalidValue;  // not applicable without scratch
		if (KSPLIT > a.kw) return cudaErrorInvalidValue;
		size_t smem = S::smem(a.kw, a.kh);
		if (smem > 227 * 1024) return cudaErrorInvalidValue;
		static bool configured = false;
		if (!configured) {
			cudaError_t e = cudaFuncSetAttribute(k_conv3_tile<TOut, HL, RY, TYT, KS, KSPLIT, KHC>,
			                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
			if (e != cudaSuccess) return e;
			configured = true;
		}
		dim3 block(32, TYT, KS);
		dim3 grid((a.ow + S::TX - 1) / S::TX, (a.oh + S::TY - 1) / S::TY, a.batch * KSPLIT);
		cudaError_t e = launch_pdl(
		    k_conv3_tile<TOut, HL, RY, TYT, KS, KSPLIT, KHC>, grid, block, smem, s, static_cast<const float *>(a.src), a.sw,
		    a.sh, a.ox, a.oy, static_cast<const float *>(a.K), a.kw, a.kh, static_cast<TOut *>(a.out), a.ow, a.oh,
		    static_cast<const float *>(a.add), a.add_stride, a.add_ox, a.add_oy, a.batch_src_stride,
		    a.batch_out_stride, a.batch_k_stride, static_cast<double *>(a.scratch));
		if (e != cudaSuccess) return e;
		if (KSPLIT > 1) {
			size_t n = (size_t)a.ow * a.oh * a.batch;
			int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 8);
			e = launch_pdl(k_conv_split_sum<TOut>, dim3(blocks), dim3(256), 0, s,
			               static_cast<const double *>(a.scratch), KSPLIT, static_cast<TOut *>(a.out), a.ow, a.oh,
			               a.batch, static_cast<const float *>(a.add), a.add_stride, a.add_ox, a.add_oy,
			               a.batch_src_stride, a.batch_out_stride);
			note_launches(1);
			if (e != cudaSuccess) return e;
		}
		return cudaGetLastError();
	}
};

}  // namespace pf
