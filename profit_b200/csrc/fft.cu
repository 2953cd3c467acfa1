// The "fft" convolver (FFTConvolver, convolve.cpp:233-312) as hand-written
// FFT kernels.
//
// libprofit pads source and PSF into a 2*max(src, psf) buffer, takes a 1-D
// real FFT of the flattened buffer (fft.cpp:113-158), multiplies, transforms
// back, divides by N and reads the result from offset_after_convolution
// (convolve.cpp:270-281).  Because the padding prevents any wrap-around, that
// is exactly the linear convolution
//     c(X, Y) = sum_{u,v} psf(u, v) src(X - u, Y - v)
// read at (x + dx, y + dy), dx = offset_x - (src_w - psf_w)/2.  Here the same
// linear convolution is computed with 2-D FFTs of an M x N grid chosen as
// the smallest sizes >= src + psf - 1 whose prime factors are 2, 3 and 5.
//
// Kernels (one CTA per row pair or column group, everything in shared memory):
//  - row pass: two real rows packed as one complex row, one length-N FFT,
//    split into the two half spectra (Hermitian symmetry), [M][N/2+1] layout;
//  - column pass: CB columns per CTA, length-M FFT, pointwise product with
//    the PSF spectrum (or its conjugate for the adjoint), inverse length-M
//    FFT, all fused;
//  - inverse row pass: two half spectra rebuilt to one complex row, inverse
//    FFT, real and imaginary parts are the two output rows, scaled by 1/(MN)
//    and written only where the crop needs them (plus the unconvolved image).
// The 1-D FFT is a self-sorting Stockham iteration (Govindaraju et al., "High
// performance discrete Fourier transforms on graphics processors", SC 2008),
// radices 2, 3, 4, 5, twiddles from a table built once per length.
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "fft.h"

namespace pf {

template <class T>
struct Cx;
template <>
struct Cx<float> {
	using type = float2;
};
template <>
struct Cx<double> {
	using type = double2;
};

template <class C>
__device__ __forceinline__ C cmul(C a, C b)
{
	C r;
	r.x = a.x * b.x - a.y * b.y;
	r.y = a.x * b.y + a.y * b.x;
	return r;
}

template <class C>
__device__ __forceinline__ C cadd(C a, C b)
{
	C r;
	r.x = a.x + b.x;
	r.y = a.y + b.y;
	return r;
}

template <class C>
__device__ __forceinline__ C csub(C a, C b)
{
	C r;
	r.x = a.x - b.x;
	r.y = a.y - b.y;
	return r;
}

// multiply by -i (sign = +1) or +i (sign = -1)
template <class C, class T>
__device__ __forceinline__ C mul_mi(C a, T sign)
{
	C r;
	r.x = sign * a.y;
	r.y = -sign * a.x;
	return r;
}

// In-place DFT of size R on v (forward: sign = +1 gives exp(-2 pi i nk/R)).
template <class T, class C>
__device__ __forceinline__ void small_dft(C *v, int R, T sign)
{
	if (R == 2) {
		C a = v[0], b = v[1];
		v[0] = cadd(a, b);
		v[1] = csub(a, b);
	}
	else if (R == 4) {
		C s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
		C s13 = cadd(v[1], v[3]), d13 = csub(v[1], v[3]);
		v[0] = cadd(s02, s13);
		v[2] = csub(s02, s13);
		C t = mul_mi<C, T>(d13, sign);  // -i d13 forward
		v[1] = cadd(d02, t);
		v[3] = csub(d02, t);
	}
	else if (R == 3) {
		const T h = T(0.86602540378443864676372317075294);  // sin(2 pi/3)
		C s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
		C x0 = v[0];
		C m;
		m.x = x0.x - T(0.5) * s.x;
		m.y = x0.y - T(0.5) * s.y;
		C t = mul_mi<C, T>(d, sign);
		t.x *= h;
		t.y *= h;
		v[0] = cadd(x0, s);
		v[1] = cadd(m, t);
		v[2] = csub(m, t);
	}
	else {  // R == 5
		const T c1 = T(0.30901699437494742410229341718282);   // cos(2 pi/5)
		const T c2 = T(-0.80901699437494742410229341718282);  // cos(4 pi/5)
		const T s1 = T(0.95105651629515357211643933337938);   // sin(2 pi/5)
		const T s2 = T(0.58778525229247312916870595463907);   // sin(4 pi/5)
		C x0 = v[0];
		C a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
		C a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
		C t1, t2, u1, u2;
		t1.x = x0.x + c1 * a1.x + c2 * a2.x;
		t1.y = x0.y + c1 * a1.y + c2 * a2.y;
		t2.x = x0.x + c2 * a1.x + c1 * a2.x;
		t2.y = x0.y + c2 * a1.y + c1 * a2.y;
		u1.x = s1 * b1.x + s2 * b2.x;
		u1.y = s1 * b1.y + s2 * b2.y;
		u2.x = s2 * b1.x - s1 * b2.x;
		u2.y = s2 * b1.y - s1 * b2.y;
		C iu1 = mul_mi<C, T>(u1, sign), iu2 = mul_mi<C, T>(u2, sign);
		v[0] = cadd(x0, cadd(a1, a2));
		v[1] = cadd(t1, iu1);
		v[4] = csub(t1, iu1);
		v[2] = cadd(t2, iu2);
		v[3] = csub(t2, iu2);
	}
}

// Stockham FFT of `cols` interleaved vectors of length n held in shared
// memory: element t of vector c at buf[t * cols + c].  Returns the buffer
// holding the result (a or b).  tw[t] = exp(-2 pi i t / n).
template <class T, class C>
__device__ C *fft_block(C *a, C *b, int n, int cols, const FftPlan &plan, const C *__restrict__ tw, bool inverse)
{
	const T sign = inverse ? T(-1) : T(1);
	int Ns = 1;
	C *in = a, *out = b;
	for (int s = 0; s < plan.nstages; s++) {
		const int R = plan.radix[s];
		const int nb = n / R;
		const int tstep = n / (Ns * R);
		for (int t = threadIdx.x; t < nb * cols; t += blockDim.x) {
			const int j = t / cols, c = t - j * cols;
			const int k = j % Ns;
			C v[5];
#pragma unroll
			for (int r = 0; r < 5; r++)
				if (r < R) v[r] = in[(j + r * nb) * cols + c];
#pragma unroll
			for (int r = 1; r < 5; r++) {
				if (r < R) {
					C w = tw[r * k * tstep];
					if (inverse) w.y = -w.y;
					v[r] = cmul(v[r], w);
				}
			}
			small_dft<T, C>(v, R, sign);
			const int idx = (j / Ns) * Ns * R + k;
#pragma unroll
			for (int r = 0; r < 5; r++)
				if (r < R) out[(idx + r * Ns) * cols + c] = v[r];
		}
		__syncthreads();
		C *tmp = in;
		in = out;
		out = tmp;
		Ns *= R;
	}
	return in;
}

// Row pass, forward.  Rows y0 = 2*blockIdx.x and y0 + 1 of the source (placed
// at (sx0, sy0) of the M x N grid, zero elsewhere) -> half spectra.
template <class T, class TIn>
__global__ void k_fft_rows_fwd(const TIn *__restrict__ src, int sw, int sh, int sx0, int sy0, int N, FftPlan plan,
                               const typename Cx<T>::type *__restrict__ tw, typename Cx<T>::type *__restrict__ spec,
                               int spec_ld, size_t src_batch, size_t spec_batch)
{
	using C = typename Cx<T>::type;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *a = reinterpret_cast<C *>(smem_raw);
	C *b = a + N;
	src += blockIdx.y * src_batch;
	spec += blockIdx.y * spec_batch;
	const int y0 = 2 * blockIdx.x;
	const int ra = y0 - sy0, rb = y0 + 1 - sy0;
	const bool has_a = ra >= 0 && ra < sh, has_b = rb >= 0 && rb < sh;
	for (int x = threadIdx.x; x < N; x += blockDim.x) {
		int sx = x - sx0;
		C z;
		z.x = (has_a && sx >= 0 && sx < sw) ? (T)src[(size_t)ra * sw + sx] : T(0);
		z.y = (has_b && sx >= 0 && sx < sw) ? (T)src[(size_t)rb * sw + sx] : T(0);
		a[x] = z;
	}
	__syncthreads();
	C *Z = (has_a || has_b) ? fft_block<T, C>(a, b, N, 1, plan, tw, false) : a;
	C *ra_out = spec + (size_t)y0 * spec_ld, *rb_out = ra_out + spec_ld;
	for (int k = threadIdx.x; k <= N / 2; k += blockDim.x) {
		C zk = Z[k], zm = Z[(N - k) % N];
		C A, B;
		// A = (Z[k] + conj(Z[N-k]))/2, B = (Z[k] - conj(Z[N-k]))/(2i)
		A.x = T(0.5) * (zk.x + zm.x);
		A.y = T(0.5) * (zk.y - zm.y);
		B.x = T(0.5) * (zk.y + zm.y);
		B.y = T(-0.5) * (zk.x - zm.x);
		ra_out[k] = A;
		rb_out[k] = B;
	}
}

// Column pass: CB columns of the half spectrum per CTA.  mode 0: forward FFT
// only (PSF spectrum); mode 1: forward, times K, inverse; mode 2: forward,
// times conj(K), inverse.
template <class T, int CB>
__global__ void k_fft_cols(typename Cx<T>::type *__restrict__ spec, int spec_ld, int ncols, int M, FftPlan plan,
                           const typename Cx<T>::type *__restrict__ tw, const typename Cx<T>::type *__restrict__ K,
                           int mode, size_t spec_batch)
{
	using C = typename Cx<T>::type;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *a = reinterpret_cast<C *>(smem_raw);
	C *b = a + (size_t)M * CB;
	spec += blockIdx.y * spec_batch;
	const int c0 = blockIdx.x * CB;
	for (int t = threadIdx.x; t < M * CB; t += blockDim.x) {
		int row = t / CB, c = t - row * CB;
		C v;
		v.x = T(0);
		v.y = T(0);
		if (c0 + c < ncols) v = spec[(size_t)row * spec_ld + c0 + c];
		a[t] = v;
	}
	__syncthreads();
	C *S = fft_block<T, C>(a, b, M, CB, plan, tw, false);
	if (mode == 0) {
		for (int t = threadIdx.x; t < M * CB; t += blockDim.x) {
			int row = t / CB, c = t - row * CB;
			if (c0 + c < ncols) spec[(size_t)row * spec_ld + c0 + c] = S[t];
		}
		return;
	}
	for (int t = threadIdx.x; t < M * CB; t += blockDim.x) {
		int row = t / CB, c = t - row * CB;
		if (c0 + c < ncols) {
			C k = K[(size_t)row * spec_ld + c0 + c];
			if (mode == 2) k.y = -k.y;
			S[t] = cmul(S[t], k);
		}
	}
	__syncthreads();
	C *other = (S == a) ? b : a;
	C *R = fft_block<T, C>(S, other, M, CB, plan, tw, true);
	for (int t = threadIdx.x; t < M * CB; t += blockDim.x) {
		int row = t / CB, c = t - row * CB;
		if (c0 + c < ncols) spec[(size_t)row * spec_ld + c0 + c] = R[t];
	}
}

// Inverse row pass: rows y0, y0+1 of the result; out(x, y) = c(x + dx, y + dy)
// / (M N) (+ add) for the output window [0, ow) x [0, oh).
template <class T, class TOut, class TAdd>
__global__ void k_fft_rows_inv(const typename Cx<T>::type *__restrict__ spec, int spec_ld, int N, int M, FftPlan plan,
                               const typename Cx<T>::type *__restrict__ tw, int dx, int dy, TOut *__restrict__ out,
                               int ow, int oh, const TAdd *__restrict__ add, int add_stride, int add_ox, int add_oy,
                               size_t spec_batch, size_t out_batch, size_t add_batch)
{
	using C = typename Cx<T>::type;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *a = reinterpret_cast<C *>(smem_raw);
	C *b = a + N;
	spec += blockIdx.y * spec_batch;
	out += blockIdx.y * out_batch;
	if (add) add += blockIdx.y * add_batch;
	const int y0 = 2 * blockIdx.x;
	const int oa = y0 - dy, ob = y0 + 1 - dy;  // output rows fed by this pair
	const bool want_a = oa >= 0 && oa < oh, want_b = ob >= 0 && ob < oh;
	if (!want_a && !want_b) return;
	const C *ra = spec + (size_t)y0 * spec_ld, *rb = ra + spec_ld;
	for (int k = threadIdx.x; k < N; k += blockDim.x) {
		C A, B;
		if (k <= N / 2) {
			A = ra[k];
			B = rb[k];
		}
		else {
			A = ra[N - k];
			B = rb[N - k];
			A.y = -A.y;
			B.y = -B.y;
		}
		C z;  // A + i B
		z.x = A.x - B.y;
		z.y = A.y + B.x;
		a[k] = z;
	}
	__syncthreads();
	C *Z = fft_block<T, C>(a, b, N, 1, plan, tw, true);
	const T scale = T(1) / ((T)M * (T)N);
	for (int x = threadIdx.x; x < ow; x += blockDim.x) {
		int X = x + dx;
		T va = (X >= 0 && X < N) ? Z[X].x * scale : T(0);
		T vb = (X >= 0 && X < N) ? Z[X].y * scale : T(0);
		if (want_a) {
			T v = va;
			if (add) v += (T)add[(size_t)(oa + add_oy) * add_stride + x + add_ox];
			out[(size_t)oa * ow + x] = (TOut)v;
		}
		if (want_b) {
			T v = vb;
			if (add) v += (T)add[(size_t)(ob + add_oy) * add_stride + x + add_ox];
			out[(size_t)ob * ow + x] = (TOut)v;
		}
	}
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

static bool factor_235(int n, FftPlan &plan)
{
	plan.n = n;
	plan.nstages = 0;
	int m = n;
	while (m % 4 == 0 && plan.nstages < FFT_MAX_STAGES) {
		plan.radix[plan.nstages++] = 4;
		m /= 4;
	}
	const int rs[3] = {2, 3, 5};
	for (int r : rs)
		while (m % r == 0 && plan.nstages < FFT_MAX_STAGES) {
			plan.radix[plan.nstages++] = r;
			m /= r;
		}
	return m == 1;
}

int fft_good_size(int need)
{
	for (int n = (need + 1) & ~1;; n += 2) {
		FftPlan p;
		if (factor_235(n, p)) return n;
	}
}

template <class T>
static const typename Cx<T>::type *twiddles(int n)
{
	using C = typename Cx<T>::type;
	static std::mutex mu;
	static std::map<int, C *> cache;
	std::lock_guard<std::mutex> g(mu);
	auto it = cache.find(n);
	if (it != cache.end()) return it->second;
	std::vector<C> h(n);
	for (int t = 0; t < n; t++) {
		long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)t / (long double)n;
		h[t].x = (T)cosl(ang);
		h[t].y = (T)sinl(ang);
	}
	C *d = nullptr;
	if (cudaMalloc(&d, sizeof(C) * n) != cudaSuccess) return nullptr;
	cudaMemcpy(d, h.data(), sizeof(C) * n, cudaMemcpyHostToDevice);
	cache[n] = d;
	return d;
}

template <class T>
static int cols_per_block(int M)
{
	// two ping-pong buffers of M x CB complex values within 200 KB
	size_t per = 2 * sizeof(typename Cx<T>::type) * (size_t)M;
	int cb = (int)((200 * 1024) / per);
	if (cb >= 8) return 8;
	if (cb >= 4) return 4;
	if (cb >= 2) return 2;
	return 1;
}

template <class T, int CB>
static cudaError_t launch_cols(typename Cx<T>::type *spec, int spec_ld, int ncols, int M, const FftPlan &pm,
                               const typename Cx<T>::type *tw, const typename Cx<T>::type *K, int mode, int batch,
                               size_t spec_batch, cudaStream_t s)
{
	size_t smem = 2 * sizeof(typename Cx<T>::type) * (size_t)M * CB;
	cudaFuncSetAttribute(k_fft_cols<T, CB>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
	dim3 grid((ncols + CB - 1) / CB, batch);
	k_fft_cols<T, CB><<<grid, 256, smem, s>>>(spec, spec_ld, ncols, M, pm, tw, K, mode, spec_batch);
	return cudaGetLastError();
}

template <class T>
static cudaError_t cols_any(typename Cx<T>::type *spec, int spec_ld, int ncols, int M, const FftPlan &pm,
                            const typename Cx<T>::type *tw, const typename Cx<T>::type *K, int mode, int batch,
                            size_t spec_batch, cudaStream_t s)
{
	switch (cols_per_block<T>(M)) {
	case 8: return launch_cols<T, 8>(spec, spec_ld, ncols, M, pm, tw, K, mode, batch, spec_batch, s);
	case 4: return launch_cols<T, 4>(spec, spec_ld, ncols, M, pm, tw, K, mode, batch, spec_batch, s);
	case 2: return launch_cols<T, 2>(spec, spec_ld, ncols, M, pm, tw, K, mode, batch, spec_batch, s);
	default: return launch_cols<T, 1>(spec, spec_ld, ncols, M, pm, tw, K, mode, batch, spec_batch, s);
	}
}

template <class T>
cudaError_t FftConv<T>::setup(int M_, int N_)
{
	if (M_ == M && N_ == N && tw_m && tw_n) return cudaSuccess;
	M = M_;
	N = N_;
	if (!factor_235(M, plan_m) || !factor_235(N, plan_n) || (M & 1) || (N & 1)) return cudaErrorInvalidValue;
	if (N > FFT_MAX_LEN || M > FFT_MAX_LEN) return cudaErrorInvalidValue;
	tw_m = twiddles<T>(M);
	tw_n = twiddles<T>(N);
	if (!tw_m || !tw_n) return cudaErrorMemoryAllocation;
	ld = N / 2 + 1;
	for (int f : {0, 1})
		cudaFuncSetAttribute(f ? (const void *)k_fft_rows_fwd<T, float> : (const void *)k_fft_rows_fwd<T, double>,
		                     cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
	cudaFuncSetAttribute(k_fft_rows_inv<T, double, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
	cudaFuncSetAttribute(k_fft_rows_inv<T, double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
	cudaFuncSetAttribute(k_fft_rows_inv<T, float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
	have_kernel = false;
	return cudaGetLastError();
}

template <class T>
template <class TIn>
cudaError_t FftConv<T>::forward_rows(const TIn *src, int sw, int sh, int sx0, int sy0, Cplx *spec, int batch,
                                     size_t src_batch, cudaStream_t s)
{
	size_t smem = 2 * sizeof(Cplx) * (size_t)N;
	dim3 grid(M / 2, batch);
	k_fft_rows_fwd<T, TIn><<<grid, 256, smem, s>>>(src, sw, sh, sx0, sy0, N, plan_n, tw_n, spec, ld, src_batch,
	                                               (size_t)M * ld);
	return cudaGetLastError();
}

template <class T>
cudaError_t FftConv<T>::set_kernel(const T *psf_dev, int kw, int kh, Cplx *kspec, cudaStream_t s)
{
	cudaError_t e = forward_rows<T>(psf_dev, kw, kh, 0, 0, kspec, 1, 0, s);
	if (e != cudaSuccess) return e;
	e = cols_any<T>(kspec, ld, ld, M, plan_m, tw_m, nullptr, 0, 1, 0, s);
	have_kernel = e == cudaSuccess;
	return e;
}

template <class T>
template <class TIn, class TOut, class TAdd>
cudaError_t FftConv<T>::convolve(const TIn *src, int sw, int sh, int sx0, int sy0, const Cplx *kspec, bool adjoint,
                                 Cplx *work, int dx, int dy, TOut *out, int ow, int oh, const TAdd *add,
                                 int add_stride, int add_ox, int add_oy, int batch, size_t src_batch,
                                 size_t out_batch, size_t add_batch, cudaStream_t s)
{
	cudaError_t e = forward_rows<TIn>(src, sw, sh, sx0, sy0, work, batch, src_batch, s);
	if (e != cudaSuccess) return e;
	e = cols_any<T>(work, ld, ld, M, plan_m, tw_m, kspec, adjoint ? 2 : 1, batch, (size_t)M * ld, s);
	if (e != cudaSuccess) return e;
	size_t smem = 2 * sizeof(Cplx) * (size_t)N;
	dim3 grid(M / 2, batch);
	k_fft_rows_inv<T, TOut, TAdd><<<grid, 256, smem, s>>>(work, ld, N, M, plan_n, tw_n, dx, dy, out, ow, oh, add,
	                                                      add_stride, add_ox, add_oy, (size_t)M * ld, out_batch,
	                                                      add_batch);
	return cudaGetLastError();
}

template struct FftConv<double>;
template struct FftConv<float>;
template cudaError_t FftConv<double>::convolve<double, double, double>(const double *, int, int, int, int,
                                                                      const Cplx *, bool, Cplx *, int, int, double *,
                                                                      int, int, const double *, int, int, int, int,
                                                                      size_t, size_t, size_t, cudaStream_t);
template cudaError_t FftConv<double>::convolve<float, double, float>(const float *, int, int, int, int, const Cplx *,
                                                                    bool, Cplx *, int, int, double *, int, int,
                                                                    const float *, int, int, int, int, size_t,
                                                                    size_t, size_t, cudaStream_t);
template cudaError_t FftConv<double>::convolve<float, float, float>(const float *, int, int, int, int, const Cplx *,
                                                                   bool, Cplx *, int, int, float *, int, int,
                                                                   const float *, int, int, int, int, size_t, size_t,
                                                                   size_t, cudaStream_t);
template cudaError_t FftConv<float>::convolve<float, float, float>(const float *, int, int, int, int, const Cplx *,
                                                                  bool, Cplx *, int, int, float *, int, int,
                                                                  const float *, int, int, int, int, size_t, size_t,
                                                                  size_t, cudaStream_t);

}  // namespace pf
