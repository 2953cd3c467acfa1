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
// A CTA owns a 32 x (TYT*RY) output tile.  The source tile with its
// (kw-1, kh-1) halo and the whole kernel sit in shared memory; each thread
// keeps RY vertically adjacent outputs in registers and slides an RY-row
// window down the tile, so every tap costs one shared load, one broadcast
// kernel load and RY FMAs.  An optional `add` image (the unconvolved
// profiles) is added in the epilogue, which fuses model.cpp:377.
#pragma once

#include <cuda_runtime.h>

namespace pf {

template <class T, int RY, int TYT>
__global__ void __launch_bounds__(32 * TYT) k_conv_tile(const T *__restrict__ src, int sw, int sh, int ox, int oy,
                                                        const T *__restrict__ K, int kw, int kh,
                                                        T *__restrict__ out, int ow, int oh,
                                                        const T *__restrict__ add, int add_stride, int add_ox,
                                                        int add_oy, int batch_src_stride, int batch_out_stride)
{
	extern __shared__ unsigned char smem_raw[];
	T *s_src = reinterpret_cast<T *>(smem_raw);
	constexpr int TX = 32;
	constexpr int TY = TYT * RY;
	const int tw = TX + kw - 1;
	const int th = TY + kh - 1;
	T *s_k = s_src + (size_t)tw * th;

	const int b = blockIdx.z;
	src += (size_t)b * batch_src_stride;
	out += (size_t)b * batch_out_stride;
	if (add) add += (size_t)b * batch_src_stride;

	const int i0 = blockIdx.x * TX;
	const int j0 = blockIdx.y * TY;
	const int nthr = TX * TYT;
	const int tid = threadIdx.x + threadIdx.y * TX;

	for (int t = tid; t < kw * kh; t += nthr) s_k[t] = K[t];
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
	T acc[RY];
#pragma unroll
	for (int r = 0; r < RY; r++) acc[r] = T(0);

	for (int k = 0; k < kw; k++) {
		const T *col = s_src + tx + k;
		T win[RY];
#pragma unroll
		for (int r = 0; r < RY - 1; r++) win[r] = col[(r0 + r) * tw];
		const T *krow = s_k + k;
		for (int l = 0; l < kh; l++) {
			win[RY - 1] = col[(r0 + l + RY - 1) * tw];
			const T c = krow[l * kw];
#pragma unroll
			for (int r = 0; r < RY; r++) acc[r] += win[r] * c;
#pragma unroll
			for (int r = 0; r < RY - 1; r++) win[r] = win[r + 1];
		}
	}

	const int i = i0 + tx;
	if (i >= ow) return;
#pragma unroll
	for (int r = 0; r < RY; r++) {
		int j = j0 + r0 + r;
		if (j < oh) {
			T v = acc[r];
			if (add) v += add[(i + add_ox) + (size_t)(j + add_oy) * add_stride];
			out[i + (size_t)j * ow] = v;
		}
	}
}

template <class T, int RY, int TYT>
inline size_t conv_smem_bytes(int kw, int kh)
{
	return sizeof(T) * ((size_t)(32 + kw - 1) * (TYT * RY + kh - 1) + (size_t)kw * kh);
}

template <class T, int RY, int TYT>
inline cudaError_t launch_conv(const T *src, int sw, int sh, int ox, int oy, const T *K, int kw, int kh, T *out,
                               int ow, int oh, const T *add, int add_stride, int add_ox, int add_oy, int batch,
                               int batch_src_stride, int batch_out_stride, cudaStream_t stream)
{
	size_t smem = conv_smem_bytes<T, RY, TYT>(kw, kh);
	static bool configured = false;
	if (!configured) {
		cudaError_t e = cudaFuncSetAttribute(k_conv_tile<T, RY, TYT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
		                                     227 * 1024);
		if (e != cudaSuccess) return e;
		configured = true;
	}
	if (smem > 227 * 1024) return cudaErrorInvalidValue;
	dim3 block(32, TYT);
	dim3 grid((ow + 31) / 32, (oh + TYT * RY - 1) / (TYT * RY), batch);
	k_conv_tile<T, RY, TYT><<<grid, block, smem, stream>>>(src, sw, sh, ox, oy, K, kw, kh, out, ow, oh, add,
	                                                       add_stride, add_ox, add_oy, batch_src_stride,
	                                                       batch_out_stride);
	return cudaGetLastError();
}

}  // namespace pf
