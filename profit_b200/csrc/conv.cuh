// Brute-force PSF convolution as a shared-memory-tiled direct correlation:
//
//   out(i, j) = sum_{k < kw, l < kh} src(i + ox + k, j + oy + l) * K(k, l)
//
// with src read as zero outside [0, sw) x [0, sh).  Two uses:
//  - forward (AssociativeBruteForceConvolver, convolve.cpp:158-231, followed
//    by the crop of model.cpp:307-324): src = padded image, ox = oy = 0,
//    K = the reversed PSF, out = the cropped model.  Only the outputs that
//    survive the crop are computed; with padding psf/2 none of them touches
//    the image edge, so the edge clipping of convolve.cpp:199-210 never
//    applies to them.
//  - adjoint: src = residual weights w on the cropped grid, ox = 1 - kw,
//    oy = 1 - kh, K = the PSF itself: out(u) = sum_k w(u - k) ikrn(k) over
//    the padded grid, the transpose of the forward map.
//
// Work decomposition: a CTA owns a 32 x (TYT*RY) output tile; its source
// tile with the (kw-1, kh-1) halo and the whole kernel sit in shared memory.
// The kernel columns k are split over KS warp groups (threadIdx.z), so even a
// single 400x400 image keeps ~16 warps per SM busy.  Each thread holds RY
// vertically adjacent outputs and slides an RY-row window down the tile: per
// tap one shared load of the source, a quarter of a vector load of the
// kernel (stored transposed so four rows are contiguous) and RY FMAs.
//
// Precision: the taps of one kernel column are summed in T (FP32 on the fast
// path); the column sums are accumulated in Acc (FP64), and the KS partial
// results are added in a fixed order.  A 51x51 PSF then has 51-term FP32
// sums instead of one 2601-term sum, which brings the FP32 convolution error
// from ~1e-6 to a few 1e-8 of the value (the FP32 rounding of the inputs).
// An optional `add` image (the unconvolved profiles) is added in the
// epilogue, which fuses model.cpp:377.
#pragma once

#include <cuda_runtime.h>

namespace pf {

template <class T, class Acc>
__host__ __device__ inline size_t conv_red_offset(int kw, int kh, int TY)
{
	size_t khp = (size_t)((kh + 3) & ~3);
	size_t bytes = sizeof(T) * ((size_t)kw * khp + (size_t)(32 + kw - 1) * (TY + kh - 1));
	return (bytes + 15) & ~(size_t)15;
}

template <class T, class Acc, class TOut, int RY, int TYT, int KS>
__global__ void __launch_bounds__(32 * TYT * KS)
    k_conv_tile(const T *__restrict__ src, int sw, int sh, int ox, int oy, const T *__restrict__ K, int kw, int kh,
                TOut *__restrict__ out, int ow, int oh, const T *__restrict__ add, int add_stride, int add_ox,
                int add_oy, int batch_src_stride, int batch_out_stride, int batch_k_stride)
{
	extern __shared__ __align__(16) unsigned char smem_raw[];
	constexpr int TX = 32;
	constexpr int TY = TYT * RY;
	const int tw = TX + kw - 1;
	const int th = TY + kh - 1;
	const int khp = (kh + 3) & ~3;  // transposed kernel rows padded to 4
	T *s_k = reinterpret_cast<T *>(smem_raw);             // [kw][khp], K(k, l) at k*khp + l
	T *s_src = s_k + (size_t)kw * khp;                     // [th][tw]
	Acc *s_red = reinterpret_cast<Acc *>(smem_raw + conv_red_offset<T, Acc>(kw, kh, TY));

	const int b = blockIdx.z;
	src += (size_t)b * batch_src_stride;
	out += (size_t)b * batch_out_stride;
	K += (size_t)b * batch_k_stride;
	if (add) add += (size_t)b * batch_src_stride;

	const int i0 = blockIdx.x * TX;
	const int j0 = blockIdx.y * TY;
	const int nthr = TX * TYT * KS;
	const int tid = threadIdx.x + TX * (threadIdx.y + TYT * threadIdx.z);

	for (int t = tid; t < kw * khp; t += nthr) {
		int k = t / khp, l = t - k * khp;
		s_k[t] = l < kh ? K[k + l * kw] : T(0);
	}
	for (int t = tid; t < tw * th; t += nthr) {
		int ty = t / tw, tx = t - ty * tw;
		int sx = i0 + ox + tx, sy = j0 + oy + ty;
		T v = T(0);
		if (sx >= 0 && sx < sw && sy >= 0 && sy < sh) v = src[sx + (size_t)sy * sw];
		s_src[t] = v;
	}
	__syncthreads();

	const int tx = threadIdx.x;
	const int r0 = threadIdx.y * RY;
	Acc tot[RY];
#pragma unroll
	for (int r = 0; r < RY; r++) tot[r] = Acc(0);

	for (int k = threadIdx.z; k < kw; k += KS) {
		const T *col = s_src + tx + k;
		const T *kcol = s_k + k * khp;
		T acc[RY];
		T win[RY];
#pragma unroll
		for (int r = 0; r < RY; r++) acc[r] = T(0);
#pragma unroll
		for (int r = 0; r < RY - 1; r++) win[r] = col[(r0 + r) * tw];
		int l = 0;
		for (; l + 4 <= kh; l += 4) {
			T c4[4];
			if constexpr (sizeof(T) == 4) {
				float4 v = *reinterpret_cast<const float4 *>(kcol + l);
				c4[0] = v.x;
				c4[1] = v.y;
				c4[2] = v.z;
				c4[3] = v.w;
			}
			else {
				double2 v0 = *reinterpret_cast<const double2 *>(kcol + l);
				double2 v1 = *reinterpret_cast<const double2 *>(kcol + l + 2);
				c4[0] = v0.x;
				c4[1] = v0.y;
				c4[2] = v1.x;
				c4[3] = v1.y;
			}
#pragma unroll
			for (int q = 0; q < 4; q++) {
				win[RY - 1] = col[(r0 + l + q + RY - 1) * tw];
#pragma unroll
				for (int r = 0; r < RY; r++) acc[r] += win[r] * c4[q];
#pragma unroll
				for (int r = 0; r < RY - 1; r++) win[r] = win[r + 1];
			}
		}
		for (; l < kh; l++) {
			win[RY - 1] = col[(r0 + l + RY - 1) * tw];
			const T c = kcol[l];
#pragma unroll
			for (int r = 0; r < RY; r++) acc[r] += win[r] * c;
#pragma unroll
			for (int r = 0; r < RY - 1; r++) win[r] = win[r + 1];
		}
#pragma unroll
		for (int r = 0; r < RY; r++) tot[r] += (Acc)acc[r];
	}

	if (KS > 1) {
		// groups 1..KS-1 hand their partial sums to group 0 (fixed order)
		if (threadIdx.z > 0) {
#pragma unroll
			for (int r = 0; r < RY; r++) s_red[((threadIdx.z - 1) * TY + r0 + r) * TX + tx] = tot[r];
		}
		__syncthreads();
		if (threadIdx.z > 0) return;
#pragma unroll
		for (int g = 1; g < KS; g++)
#pragma unroll
			for (int r = 0; r < RY; r++) tot[r] += s_red[((g - 1) * TY + r0 + r) * TX + tx];
	}

	const int i = i0 + tx;
	if (i >= ow) return;
#pragma unroll
	for (int r = 0; r < RY; r++) {
		int j = j0 + r0 + r;
		if (j < oh) {
			Acc v = tot[r];
			if (add) v += (Acc)add[(i + add_ox) + (size_t)(j + add_oy) * add_stride];
			out[i + (size_t)j * ow] = (TOut)v;
		}
	}
}

template <class T, class Acc, int RY, int TYT, int KS>
inline size_t conv_smem_bytes(int kw, int kh)
{
	constexpr int TY = TYT * RY;
	return conv_red_offset<T, Acc>(kw, kh, TY) + sizeof(Acc) * (size_t)(KS - 1) * TY * 32;
}

template <class T, class Acc, class TOut, int RY, int TYT, int KS>
inline cudaError_t launch_conv(const T *src, int sw, int sh, int ox, int oy, const T *K, int kw, int kh, TOut *out,
                               int ow, int oh, const T *add, int add_stride, int add_ox, int add_oy, int batch,
                               int batch_src_stride, int batch_out_stride, int batch_k_stride, cudaStream_t stream)
{
	size_t smem = conv_smem_bytes<T, Acc, RY, TYT, KS>(kw, kh);
	static bool configured = false;
	if (!configured) {
		cudaError_t e = cudaFuncSetAttribute(k_conv_tile<T, Acc, TOut, RY, TYT, KS>,
		                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
		if (e != cudaSuccess) return e;
		configured = true;
	}
	if (smem > 227 * 1024) return cudaErrorInvalidValue;
	dim3 block(32, TYT, KS);
	dim3 grid((ow + 31) / 32, (oh + TYT * RY - 1) / (TYT * RY), batch);
	k_conv_tile<T, Acc, TOut, RY, TYT, KS><<<grid, block, smem, stream>>>(
	    src, sw, sh, ox, oy, K, kw, kh, out, ow, oh, add, add_stride, add_ox, add_oy, batch_src_stride,
	    batch_out_stride, batch_k_stride);
	return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Autotuned dispatch.  The best tile (RY x TYT rows, KS column groups) depends
// on the output size, the PSF size and the batch: a single 400x400 image needs
// small tiles and many column groups to spread over 148 SMs, a batch of
// thousands prefers large tiles with little halo.  The first call for a given
// (type, sizes) key times every candidate that fits in shared memory with
// CUDA events and caches the fastest; later calls (and CUDA-graph captures)
// use the cached choice.
// ---------------------------------------------------------------------------

struct ConvArgs {
	const void *src;
	int sw, sh, ox, oy;
	const void *K;
	int kw, kh;
	void *out;
	int ow, oh;
	const void *add;
	int add_stride, add_ox, add_oy, batch, batch_src_stride, batch_out_stride;
	void *scratch = nullptr;  // FP64 partial images for kernels that split the kernel columns over CTAs
	size_t scratch_bytes = 0;
	int batch_k_stride = 0;   // kernel elements between batch entries (0: one kernel for all)
};

template <class T, class Acc, class TOut, int RY, int TYT, int KS>
struct ConvVariant {
	static size_t smem(int kw, int kh) { return conv_smem_bytes<T, Acc, RY, TYT, KS>(kw, kh); }
	static cudaError_t run(const ConvArgs &a, cudaStream_t s)
	{
		return launch_conv<T, Acc, TOut, RY, TYT, KS>(
		    static_cast<const T *>(a.src), a.sw, a.sh, a.ox, a.oy, static_cast<const T *>(a.K), a.kw, a.kh,
		    static_cast<TOut *>(a.out), a.ow, a.oh, static_cast<const T *>(a.add), a.add_stride, a.add_ox, a.add_oy,
		    a.batch, a.batch_src_stride, a.batch_out_stride, a.batch_k_stride, s);
	}
};

struct ConvCandidate {
	size_t (*smem)(int, int);
	cudaError_t (*run)(const ConvArgs &, cudaStream_t);
	bool tuned = true;  // false: only run when forced (PF_CONV_FORCE), never picked by the autotuner
};

cudaError_t conv_autotuned(const ConvCandidate *cands, int n_cands, int type_tag, const ConvArgs &a,
                           cudaStream_t s);

}  // namespace pf
