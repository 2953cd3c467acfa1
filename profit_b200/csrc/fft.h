// Host interface of the FFT convolver kernels (fft.cu).
#pragma once

#include <cstddef>
#include <type_traits>

#include <cuda_runtime.h>

namespace pf {

constexpr int FFT_MAX_STAGES = 16;
// one row (two ping-pong buffers of complex doubles) must fit in shared memory
constexpr int FFT_MAX_LEN = 6912;
constexpr size_t FFT_SMEM_BYTES = 227 * 1024;

// Stockham stages of a length-n transform: stage s has radix R = radix[s],
// ns[s] = product of the earlier radices, nb[s] = n / R butterflies and
// twiddle stride tstep[s] = n / (ns R); j / ns = umulhi(j, ns_magic) for
// j < 2^16 (ns_magic = ceil(2^32 / ns), unused when ns = 1).  A stage's
// radix is 2, 3, 4 or 5, or the product of two of them (6, 8, 9, 10, 12, 15,
// 16), whose butterfly one thread computes in registers: two Stockham stages
// for one round trip through shared memory.
struct FftPlan {
	int n;
	int nstages;
	int radix[FFT_MAX_STAGES];
	int ns[FFT_MAX_STAGES];
	int nb[FFT_MAX_STAGES];
	int tstep[FFT_MAX_STAGES];
	unsigned ns_magic[FFT_MAX_STAGES];
};

// Fills the stage tables of plan from plan.n and plan.radix.
void fft_plan_stages(FftPlan &plan);

// The stages of a length-n transform (n 2-3-5 smooth): the prime factors
// paired into radices of at most 16; false if n has another factor.
bool fft_factor(int n, FftPlan &plan);

// Smallest even size >= need whose prime factors are 2, 3 and 5.
int fft_good_size(int need);

// 2-D linear convolution through an M x N FFT grid (M, N even, 2-3-5 smooth,
// >= source + kernel - 1 in each direction so nothing wraps).  T is the
// arithmetic of the transforms; spectra are [M][N/2+1] complex of T.
template <class T>
struct FftConv {
	using Cplx = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
	int M = 0, N = 0, ld = 0;
	FftPlan plan_m{}, plan_n{};
	const Cplx *tw_m = nullptr, *tw_n = nullptr;
	bool have_kernel = false;

	cudaError_t setup(int M, int N);
	size_t spectrum_elems() const { return (size_t)M * ld; }

	// Spectrum of the kernel placed at (0, 0).
	cudaError_t set_kernel(const T *psf_dev, int kw, int kh, Cplx *kspec, cudaStream_t s);
	// Spectra of `batch` kernels of one size (kernel i at psf_dev + i *
	// psf_batch), spectrum i at kspec + i * spectrum_elems().
	cudaError_t set_kernels(const float *psf_dev, int kw, int kh, size_t psf_batch, Cplx *kspec, int batch,
	                        cudaStream_t s);

	// out(x, y) = c(x + dx, y + dy) [+ add(x + add_ox, y + add_oy)] for x < ow,
	// y < oh, where c is the linear convolution of src (placed at (sx0, sy0))
	// with the kernel (adjoint = false) or the correlation with it (adjoint =
	// true, conjugated spectrum).  work holds batch spectra.  Image i of the
	// batch uses the kernel spectrum at kspec + i * kspec_batch.
	template <class TIn, class TOut, class TAdd>
	cudaError_t convolve(const TIn *src, int sw, int sh, int sx0, int sy0, const Cplx *kspec, bool adjoint,
	                     Cplx *work, int dx, int dy, TOut *out, int ow, int oh, const TAdd *add, int add_stride,
	                     int add_ox, int add_oy, int batch, size_t src_batch, size_t out_batch, size_t add_batch,
	                     cudaStream_t s, size_t kspec_batch = 0);

	template <class TIn>
	cudaError_t forward_rows(const TIn *src, int sw, int sh, int sx0, int sy0, Cplx *spec, int batch,
	                         size_t src_batch, cudaStream_t s);
};

}  // namespace pf
