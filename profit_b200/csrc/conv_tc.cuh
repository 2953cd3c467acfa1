// Brute-force PSF convolution on the 5th-generation tensor cores (tcgen05):
// the same correlation as k_conv3_tile,
//
//   out(i, j) = sum_{k < kw, l < kh} src(i + ox + k, j + oy + l) * K(k, l),
//
// written, for each kernel row l, as a product of a source tile and a banded
// (Toeplitz) matrix of that kernel row:
//
//   D_l[j, i] = sum_c A_l[j, c] * B_l[i, c],
//   A_l[j, c] = src(i0 + ox + c, j0 + oy + l + j),  B_l[i, c] = K(c - i, l) (0 <= c - i < kw, else 0),
//
// with M = 128 output rows (tensor-memory lanes), N = NT output columns and
// K = c over NT + kw - 1 source columns (rounded up to 8).  A_l for every l
// is the same shared-memory tile read from row l on: in the canonical K-major
// layout without swizzle (8-row core matrices of 16-byte rows stored one
// after the other, SBO = 128) rows are 16 bytes apart throughout, so the
// descriptor of A_l is the tile's descriptor advanced by 16 l bytes.
//
// Precision.  Operands are TF32; each FP32 value x is split into
// hi = tf32(x) and lo = tf32(x - hi), and every kernel row accumulates
// A_hi B_hi + A_hi B_lo + A_lo B_hi in FP32 in tensor memory (the dropped
// A_lo B_lo term is 2^-22 relative).  The per-row sums are added in FP64 in
// registers, in increasing l, so one FP32 accumulation never spans more than
// one kernel row (the same bound as k_conv3_tile's per-column FP32 sums).
//
// Pipeline per CTA (128 threads; kernel rows [l0, l0 + nl) of one output
// tile): the A tile (hi and lo) is built once; for each kernel row every
// thread helps build B_l (hi and lo) into one of two buffers, one elected
// thread issues the 3 (K/8) MMAs into one of two accumulators and commits
// them to that accumulator's mbarrier, and while they run the threads drain
// the previous row's accumulator (tcgen05.ld, warp w reads lanes 32w..32w+31)
// into FP64.  Every wait on an mbarrier is bounded; a wait that runs out
// records g_conv_tc_error, waits (bounded) for the MMAs in flight, frees
// the tensor memory and leaves the output unwritten.
#pragma once

#include <algorithm>
#include <cstdint>

#include <cuda_runtime.h>

#include "conv.cuh"
#include "conv2.cuh"
#include "launch.h"

namespace pf {

// Nonzero after a tensor-core convolution launch gave up on a wait (never
// expected; readable with cudaMemcpyFromSymbol when debugging).
__device__ unsigned g_conv_tc_error = 0;

namespace tc {

constexpr int TM = 128;          // output rows per tile (tensor-memory lanes)
constexpr int NTHREADS = 128;
constexpr uint32_t WAIT_TRIES = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint32_t to_tf32(float x)
{
	uint32_t r;
	asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
	return r;
}

// x = hi + lo + O(2^-22 |x|), hi and lo TF32 values
__device__ __forceinline__ void split_tf32(float x, uint32_t &hi, uint32_t &lo)
{
	hi = to_tf32(x);
	lo = to_tf32(x - __uint_as_float(hi));
}

// Shared-memory matrix descriptor, K-major canonical layout without swizzle:
// byte offset of (row r, k) = (r % 8) 16 + (r / 8) sbo + (k % 4) 4 + (k / 4) lbo.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
	uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
	d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
	d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
	d |= (uint64_t)1 << 46;  // descriptor version of sm_100; base offset 0, no swizzle
	return d;
}

// Instruction descriptor: D FP32, A and B TF32, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N)
{
	return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "setp.ne.b32 p, %4, 0;\n\t"
	    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
	    "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
	             : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// Waits for the completion of the phase of parity `parity`; false when the
// bounded number of tries ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity)
{
	for (uint32_t t = 0; t < WAIT_TRIES; t++) {
		uint32_t done;
		asm volatile(
		    "{\n\t.reg .pred P1;\n\t"
		    "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
		    "selp.b32 %0, 1, 0, P1;\n\t}\n"
		    : "=r"(done)
		    : "r"(mbar), "r"(parity)
		    : "memory");
		if (done) return true;
	}
	return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor cores' reads
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 lanes (this warp's quarter) x 32 consecutive columns of FP32 from
// tensor memory, waited for before the registers are returned.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
	uint32_t r[32];
	asm volatile(
	    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
	    "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
	    "tcgen05.wait::ld.sync.aligned;\n"
	    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
	      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
	      "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
	      "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
	    : "r"(taddr)
	    : "memory");
#pragma unroll
	for (int k = 0; k < 32; k++) v[k] = __uint_as_float(r[k]);
}

// Shared-memory plan of one CTA, the same on host and device.
struct TcPlan {
	int nl;        // kernel rows per CTA
	int kp;        // K extent: NT + kw - 1 rounded up to 8
	int rows;      // A tile rows: TM + nl - 1 rounded up to 8
	uint32_t lbo_a, lbo_b;                 // bytes between 4-column groups
	uint32_t a_hi, a_lo, b[2][2], ks, bar, tptr, total;  // byte offsets

	__host__ __device__ TcPlan(int NT, int KSPLIT, int kw, int kh)
	{
		nl = (kh + KSPLIT - 1) / KSPLIT;
		kp = (NT + kw - 1 + 7) & ~7;
		rows = (TM + nl - 1 + 7) & ~7;
		lbo_a = (uint32_t)rows * 16;
		lbo_b = (uint32_t)NT * 16;
		const uint32_t a_bytes = lbo_a * (uint32_t)(kp / 4), b_bytes = lbo_b * (uint32_t)(kp / 4);
		a_hi = 0;
		a_lo = a_hi + a_bytes;
		uint32_t o = a_lo + a_bytes;
		for (int u = 0; u < 2; u++)
			for (int h = 0; h < 2; h++) {
				b[u][h] = o;
				o += b_bytes;
			}
		ks = o;
		o += (uint32_t)(nl * kw) * 4;
		bar = (o + 15) & ~15u;
		tptr = bar + 16;
		total = tptr + 16;
	}
};

}  // namespace tc

template <class TOut, int NT, int KSPLIT>
__global__ void __launch_bounds__(tc::NTHREADS, 1)
    k_conv_tc(const float *__restrict__ src, int sw, int sh, int ox, int oy, const float *__restrict__ K, int kw,
              int kh, TOut *__restrict__ out, int ow, int oh, const float *__restrict__ add, int add_stride,
              int add_ox, int add_oy, int batch_src_stride, int batch_out_stride, int batch_k_stride,
              double *__restrict__ part)
{
	using namespace tc;
	static_assert(NT == 32, "one 32x32b.x32 tensor-memory load per accumulator row");
	extern __shared__ __align__(128) unsigned char smem[];
	const TcPlan P(NT, KSPLIT, kw, kh);
	// (no static shared memory: the dynamic size may then take the whole 227 KB)
	volatile int &s_fail = *reinterpret_cast<volatile int *>(smem + P.tptr + 8);
	const int tid = threadIdx.x, warp = tid >> 5;
	const int b = blockIdx.z / KSPLIT, split = blockIdx.z - b * KSPLIT;
	const int l0 = split * P.nl;
	const int nl = max(0, min(kh, l0 + P.nl) - l0);
	const int i0 = blockIdx.x * NT, j0 = blockIdx.y * TM;
	src += (size_t)b * batch_src_stride;
	K += (size_t)b * batch_k_stride;
	float *ks = reinterpret_cast<float *>(smem + P.ks);
	const uint32_t sbase = smem_u32(smem);
	const uint32_t bar0 = sbase + P.bar, bar1 = bar0 + 8;
	uint32_t *tptr = reinterpret_cast<uint32_t *>(smem + P.tptr);

	if (tid == 0) {
		s_fail = 0;
		mbar_init(bar0, 1);
		mbar_init(bar1, 1);
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if (warp == 0) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + P.tptr),
		             "r"(2 * NT)
		             : "memory");
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
	}
	// this CTA's kernel rows
	for (int t = tid; t < nl * kw; t += NTHREADS) ks[t] = K[(size_t)l0 * kw + t];
	// A tile, hi and lo: row r = source row j0 + oy + l0 + r, 4-column group g;
	// threads run over rows, so consecutive threads store consecutive 16 bytes
	const int ng = P.kp / 4;
	for (int t = tid; t < P.rows * ng; t += NTHREADS) {
		const int r = t % P.rows, g = t / P.rows;
		const int y = j0 + oy + l0 + r;
		const bool rv = r < TM + nl - 1 && y >= 0 && y < sh;
		float v[4];
#pragma unroll
		for (int q = 0; q < 4; q++) {
			const int x = i0 + ox + 4 * g + q;
			v[q] = (rv && x >= 0 && x < sw) ? src[(size_t)y * sw + x] : 0.f;
		}
		uint4 hi, lo;
		split_tf32(v[0], hi.x, lo.x);
		split_tf32(v[1], hi.y, lo.y);
		split_tf32(v[2], hi.z, lo.z);
		split_tf32(v[3], hi.w, lo.w);
		const uint32_t off = (uint32_t)r * 16 + (uint32_t)g * P.lbo_a;
		*reinterpret_cast<uint4 *>(smem + P.a_hi + off) = hi;
		*reinterpret_cast<uint4 *>(smem + P.a_lo + off) = lo;
	}
	fence_before();
	__syncthreads();
	fence_after();
	const uint32_t tmem = *tptr;
	const uint32_t idesc = idesc_tf32(TM, NT);

	double tot[NT];
#pragma unroll
	for (int n = 0; n < NT; n++) tot[n] = 0.0;
	int issued = 0;  // MMA groups committed

	for (int it = 0; it < nl; it++) {
		const int u = it & 1;
		// B for kernel row l0 + it (its buffer's last reader, the MMAs of row
		// it - 2, were waited for in the previous iteration)
		for (int t = tid; t < NT * ng; t += NTHREADS) {
			const int i = t % NT, g = t / NT;
			float v[4];
#pragma unroll
			for (int q = 0; q < 4; q++) {
				const int d = 4 * g + q - i;
				v[q] = (d >= 0 && d < kw) ? ks[it * kw + d] : 0.f;
			}
			uint4 hi, lo;
			split_tf32(v[0], hi.x, lo.x);
			split_tf32(v[1], hi.y, lo.y);
			split_tf32(v[2], hi.z, lo.z);
			split_tf32(v[3], hi.w, lo.w);
			const uint32_t off = (uint32_t)i * 16 + (uint32_t)g * P.lbo_b;
			*reinterpret_cast<uint4 *>(smem + (u ? P.b[1][0] : P.b[0][0]) + off) = hi;
			*reinterpret_cast<uint4 *>(smem + (u ? P.b[1][1] : P.b[0][1]) + off) = lo;
		}
		fence_proxy_async();
		fence_before();
		__syncthreads();
		if (s_fail) break;
		if (tid == 0) {
			fence_after();
			const uint32_t d = tmem + (uint32_t)(u * NT);
			const uint32_t ahi = sbase + P.a_hi + (uint32_t)it * 16, alo = sbase + P.a_lo + (uint32_t)it * 16;
			const uint32_t bhi = sbase + (u ? P.b[1][0] : P.b[0][0]), blo = sbase + (u ? P.b[1][1] : P.b[0][1]);
			for (int s = 0; s < P.kp / 8; s++) {
				const uint32_t ka = 2u * s * P.lbo_a, kb = 2u * s * P.lbo_b;
				const uint64_t dah = sdesc(ahi + ka, P.lbo_a, 128), dal = sdesc(alo + ka, P.lbo_a, 128);
				const uint64_t dbh = sdesc(bhi + kb, P.lbo_b, 128), dbl = sdesc(blo + kb, P.lbo_b, 128);
				mma_tf32(d, dah, dbh, idesc, s > 0 ? 1u : 0u);
				mma_tf32(d, dah, dbl, idesc, 1u);
				mma_tf32(d, dal, dbh, idesc, 1u);
			}
			mma_commit(u ? bar1 : bar0);
		}
		issued = it + 1;
		if (it > 0) {
			// drain the previous row's accumulator while this row's MMAs run
			const int pu = (it - 1) & 1;
			if (!mbar_wait(pu ? bar1 : bar0, (uint32_t)(((it - 1) >> 1) & 1))) s_fail = 1;
			__syncthreads();
			if (s_fail) break;
			fence_after();
			float v[32];
			tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(pu * NT), v);
#pragma unroll
			for (int n = 0; n < NT; n++) tot[n] += (double)v[n];
		}
	}
	if (!s_fail && issued > 0) {
		const int last = issued - 1, pu = last & 1;
		if (!mbar_wait(pu ? bar1 : bar0, (uint32_t)((last >> 1) & 1))) s_fail = 1;
		__syncthreads();
		if (!s_fail) {
			fence_after();
			float v[32];
			tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(pu * NT), v);
#pragma unroll
			for (int n = 0; n < NT; n++) tot[n] += (double)v[n];
		}
	}
	if (s_fail) {
		// give the MMAs in flight a bounded chance to finish before the tensor
		// memory is released; the output stays unwritten
		if (tid == 0) {
			atomicExch(&g_conv_tc_error, 1u);
			for (int k = (issued > 1 ? issued - 2 : 0); k < issued; k++)
				mbar_wait((k & 1) ? bar1 : bar0, (uint32_t)((k >> 1) & 1));
		}
	}
	fence_before();
	__syncthreads();
	if (warp == 0) {
		fence_after();
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * NT) : "memory");
	}
	if (s_fail) return;

	// transpose through shared memory (the A tile is no longer read) so the
	// stores run along output rows
	double *s_out = reinterpret_cast<double *>(smem);
	constexpr int LD = NT + 1;
#pragma unroll
	for (int n = 0; n < NT; n++) s_out[tid * LD + n] = tot[n];
	__syncthreads();
	if (KSPLIT > 1) {
		double *p = part + (size_t)blockIdx.z * oh * ow;
		for (int t = tid; t < TM * NT; t += NTHREADS) {
			const int r = t / NT, n = t - r * NT;
			const int j = j0 + r, i = i0 + n;
			if (j < oh && i < ow) p[(size_t)j * ow + i] = s_out[r * LD + n];
		}
		return;
	}
	out += (size_t)b * batch_out_stride;
	if (add) add += (size_t)b * batch_src_stride;
	for (int t = tid; t < TM * NT; t += NTHREADS) {
		const int r = t / NT, n = t - r * NT;
		const int j = j0 + r, i = i0 + n;
		if (j < oh && i < ow) {
			double v = s_out[r * LD + n];
			if (add) v += (double)add[(size_t)(j + add_oy) * add_stride + i + add_ox];
			out[(size_t)j * ow + i] = (TOut)v;
		}
	}
}

template <class TOut, int NT, int KSPLIT>
struct ConvTcVariant {
	static size_t smem(int kw, int kh)
	{
		const tc::TcPlan P(NT, KSPLIT, kw, kh);
		const size_t out_bytes = (size_t)tc::TM * (NT + 1) * 8;  // the epilogue's transpose reuses the A tiles
		const size_t a_bytes = (size_t)P.b[0][0];
		return out_bytes > a_bytes ? (size_t)P.total + (out_bytes - a_bytes) : (size_t)P.total;
	}
	static cudaError_t run(const ConvArgs &a, cudaStream_t s)
	{
		if (KSPLIT > 1 && (!a.scratch || a.scratch_bytes < (size_t)a.batch * KSPLIT * a.ow * a.oh * sizeof(double)))
			return cudaErrorInvalidValue;
		if (KSPLIT > a.kh || a.batch * KSPLIT > 65535) return cudaErrorInvalidValue;
		const size_t bytes = smem(a.kw, a.kh);
		if (bytes > 227 * 1024) return cudaErrorInvalidValue;
		static bool configured = false;
		if (!configured) {
			cudaError_t e = cudaFuncSetAttribute(k_conv_tc<TOut, NT, KSPLIT>,
			                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
			if (e != cudaSuccess) return e;
			configured = true;
		}
		dim3 grid((a.ow + NT - 1) / NT, (a.oh + tc::TM - 1) / tc::TM, a.batch * KSPLIT);
		k_conv_tc<TOut, NT, KSPLIT><<<grid, tc::NTHREADS, bytes, s>>>(
		    static_cast<const float *>(a.src), a.sw, a.sh, a.ox, a.oy, static_cast<const float *>(a.K), a.kw, a.kh,
		    static_cast<TOut *>(a.out), a.ow, a.oh, static_cast<const float *>(a.add), a.add_stride, a.add_ox,
		    a.add_oy, a.batch_src_stride, a.batch_out_stride, a.batch_k_stride, static_cast<double *>(a.scratch));
		if (KSPLIT > 1) {
			size_t n = (size_t)a.ow * a.oh * a.batch;
			int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 8);
			k_conv_split_sum<TOut><<<blocks, 256, 0, s>>>(static_cast<const double *>(a.scratch), KSPLIT,
			                                              static_cast<TOut *>(a.out), a.ow, a.oh, a.batch,
			                                              static_cast<const float *>(a.add), a.add_stride, a.add_ox,
			                                              a.add_oy, a.batch_src_stride, a.batch_out_stride);
			note_launches(1);
		}
		return cudaGetLastError();
	}
};

}  // namespace pf
