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
// radices 2, 3, 4, 5 and their pairwise products up to 16 (a composite
// radix's butterfly is two Cooley-Tukey steps in one thread's registers, so
// two stages cost one exchange through shared memory), twiddles from a table
// built once per length.
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "common.cuh"
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
template <int R, class T, class C>
__device__ __forceinline__ void small_dft(C *v, T sign)
{
	if constexpr (R == 2) {
		C a = v[0], b = v[1];
		v[0] = cadd(a, b);
		v[1] = csub(a, b);
	}
	else if constexpr (R == 4) {
		C s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
		C s13 = cadd(v[1], v[3]), d13 = csub(v[1], v[3]);
		v[0] = cadd(s02, s13);
		v[2] = csub(s02, s13);
		C t = mul_mi<C, T>(d13, sign);  // -i d13 forward
		v[1] = cadd(d02, t);
		v[3] = csub(d02, t);
	}
	else if constexpr (R == 3) {
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
		static_assert(R == 5, "radix");
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

// Roots of unity exp(-2 pi i m / Q) for the composite radices (Q <= 16,
// m < Q), filled from long double values on first use on each device.
__constant__ double2 c_roots64[17][16];
__constant__ float2 c_roots32[17][16];

template <class C>
__device__ __forceinline__ C root_of(int Q, int m);
template <>
__device__ __forceinline__ double2 root_of<double2>(int Q, int m) { return c_roots64[Q][m]; }
template <>
__device__ __forceinline__ float2 root_of<float2>(int Q, int m) { return c_roots32[Q][m]; }

// DFT of size Q = R1 R2 on v (input index r = R2 r1 + r2) into X (output
// index s = s1 + R1 s2): R2 transforms of size R1, the twiddles
// exp(-+2 pi i r2 s1 / Q), then R1 transforms of size R2.
template <int R1, int R2, class T, class C>
__device__ __forceinline__ void fused_dft(const C (&v)[R1 * R2], C (&X)[R1 * R2], T sign)
{
	constexpr int Q = R1 * R2;
	C y[R2][R1];
#pragma unroll
	for (int r2 = 0; r2 < R2; r2++) {
#pragma unroll
		for (int r1 = 0; r1 < R1; r1++) y[r2][r1] = v[R2 * r1 + r2];
		small_dft<R1, T, C>(y[r2], sign);
	}
#pragma unroll
	for (int r2 = 1; r2 < R2; r2++)
#pragma unroll
		for (int s1 = 1; s1 < R1; s1++) {
			C w = root_of<C>(Q, r2 * s1);
			w.y *= sign;
			y[r2][s1] = cmul(y[r2][s1], w);
		}
#pragma unroll
	for (int s1 = 0; s1 < R1; s1++) {
		C t[R2];
#pragma unroll
		for (int r2 = 0; r2 < R2; r2++) t[r2] = y[r2][s1];
		small_dft<R2, T, C>(t, sign);
#pragma unroll
		for (int s2 = 0; s2 < R2; s2++) X[s1 + R1 * s2] = t[s2];
	}
}

// One Stockham stage of composite radix Q = R1 R2 over COLS interleaved
// vectors, the same data movement as fft_stage with the butterfly computed
// by fused_dft.
template <int R1, int R2, int COLS, class T, class C>
__device__ __forceinline__ void fft_stage_fused(const C *in, C *out, const C *stw, int nb, int ns, unsigned magic,
                                                int tstep, bool inverse)
{
	constexpr int Q = R1 * R2;
	const T sign = inverse ? T(-1) : T(1);
	for (int t = threadIdx.x; t < nb * COLS; t += blockDim.x) {
		const int j = t / COLS, c = t - j * COLS;
		const int q = ns == 1 ? j : (int)__umulhi((unsigned)j, magic);
		const int k = j - q * ns;
		C v[Q];
#pragma unroll
		for (int r = 0; r < Q; r++) v[r] = in[(j + r * nb) * COLS + c];
#pragma unroll
		for (int r = 1; r < Q; r++) {
			C w = stw[r * k * tstep];
			if (inverse) w.y = -w.y;
			v[r] = cmul(v[r], w);
		}
		C X[Q];
		fused_dft<R1, R2, T, C>(v, X, sign);
		const int idx = (j - k) * Q + k;
#pragma unroll
		for (int r = 0; r < Q; r++) out[(idx + r * ns) * COLS + c] = X[r];
	}
}

// One radix-R Stockham stage over COLS interleaved vectors (element t of
// vector c at buf[t * COLS + c]); stw: twiddles exp(-2 pi i t / n) in shared
// memory.  Butterfly j = q ns + k reads in[j + r nb] and writes
// out[q ns R + k + r ns] = out[(j - k) R + k + r ns].
template <int R, int COLS, class T, class C>
__device__ __forceinline__ void fft_stage(const C *in, C *out, const C *stw, int nb, int ns, unsigned magic,
                                          int tstep, bool inverse)
{
	const T sign = inverse ? T(-1) : T(1);
	for (int t = threadIdx.x; t < nb * COLS; t += blockDim.x) {
		const int j = t / COLS, c = t - j * COLS;
		const int q = ns == 1 ? j : (int)__umulhi((unsigned)j, magic);
		const int k = j - q * ns;
		C v[R];
#pragma unroll
		for (int r = 0; r < R; r++) v[r] = in[(j + r * nb) * COLS + c];
#pragma unroll
		for (int r = 1; r < R; r++) {
			C w = stw[r * k * tstep];
			if (inverse) w.y = -w.y;
			v[r] = cmul(v[r], w);
		}
		small_dft<R, T, C>(v, sign);
		const int idx = (j - k) * R + k;
#pragma unroll
		for (int r = 0; r < R; r++) out[(idx + r * ns) * COLS + c] = v[r];
	}
}

// Stockham FFT of COLS interleaved vectors of length plan.n held in shared
// memory (buffers a and b); returns the buffer holding the result.  The
// caller has filled stw and synchronised.
template <int COLS, class T, class C>
__device__ __forceinline__ C *fft_block(C *a, C *b, const FftPlan &plan, const C *stw, bool inverse)
{
	C *in = a, *out = b;
	for (int s = 0; s < plan.nstages; s++) {
		const int nb = plan.nb[s], ns = plan.ns[s], ts = plan.tstep[s];
		const unsigned mg = plan.ns_magic[s];
		switch (plan.radix[s]) {
		case 2: fft_stage<2, COLS, T, C>(in, out, stw, nb, ns, mg, ts, inverse); break;
		case 3: fft_stage<3, COLS, T, C>(in, out, stw, nb, ns, mg, ts, inverse); break;
		case 4: fft_stage<4, COLS, T, C>(in, out, stw, nb, ns, mg, ts, inverse); break;
		case 5: fft_stage<5, COLS, T, C>(in, out, stw, nb, ns, mg, ts, inverse); break;
		case 6: fft_stage_fused<2, 3, COLS, T, C>(in, out, stw, nb, ns, mg, ts, inverse); break;
		case 8: fft_stage_fused<2, 4, COLS, T, C>(in, out, stw, nb, ns, mg, ts, inverse); break;
		case 9: fft_stage_fused<3, 3, COLS, T, C>(in, out, stw, nb, ns, mg, ts, inverse); break;
		case 10: fft_stage_fused<2, 5, COLS, T, C>(in, out, stw, nb, ns, mg, ts, inverse); break;
		case 12: fft_stage_fused<3, 4, COLS, T, C>(in, out, stw, nb, ns, mg, ts, inverse); break;
		case 15: fft_stage_fused<3, 5, COLS, T, C>(in, out, stw, nb, ns, mg, ts, inverse); break;
		default: fft_stage_fused<4, 4, COLS, T, C>(in, out, stw, nb, ns, mg, ts, inverse); break;
		}
		__syncthreads();
		C *tmp = in;
		in = out;
		out = tmp;
	}
	return in;
}

// 16-byte asynchronous global -> shared copy (both addresses 16-byte
// aligned); completed by cp_async_wait() before the barrier that publishes
// the buffer.
__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
	unsigned d = (unsigned)__cvta_generic_to_shared(dst);
	asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_wait()
{
	asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// One complex element global -> shared: asynchronous for 16-byte elements,
// a plain copy otherwise.
template <class C>
__device__ __forceinline__ void cp_async_elem(C *dst, const C *src)
{
	if constexpr (sizeof(C) == 16) cp_async16(dst, src);
	else *dst = *src;
}

// Starts the copy of the twiddle table into shared memory (when it fits
// beside the buffers, TWS), else returns the global table, read through L1.
// Complex values of 8 or 16 bytes: 16-byte copies cover the table (n is
// even).  TWS is a template argument so that the stages' twiddle loads are
// compiled as shared-memory loads.
template <bool TWS, class C>
__device__ __forceinline__ const C *load_twiddles(C *smem, const C *__restrict__ tw, int n)
{
	if constexpr (!TWS) return tw;
	constexpr int PER = 16 / sizeof(C);
	for (int t = threadIdx.x; t * PER < n; t += blockDim.x) cp_async16(smem + t * PER, tw + t * PER);
	return smem;
}

// Row pass, forward.  Rows y0 = 2*blockIdx.x and y0 + 1 of the source (placed
// at (sx0, sy0) of the M x N grid, zero elsewhere) -> half spectra.
// Shared memory: two N-element buffers and the N twiddles.
template <class T, class TIn, bool TWS>
__global__ void k_fft_rows_fwd(const TIn *__restrict__ src, int sw, int sh, int sx0, int sy0, int N, FftPlan plan,
                               const typename Cx<T>::type *__restrict__ tw, typename Cx<T>::type *__restrict__ spec,
                               int spec_ld, size_t src_batch, size_t spec_batch)
{
	pdl_enter();
	using C = typename Cx<T>::type;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *a = reinterpret_cast<C *>(smem_raw);
	C *b = a + N;
	src += blockIdx.y * src_batch;
	spec += blockIdx.y * spec_batch;
	const int y0 = 2 * blockIdx.x;
	const int ra = y0 - sy0, rb = y0 + 1 - sy0;
	const bool has_a = ra >= 0 && ra < sh, has_b = rb >= 0 && rb < sh;
	C *ra_out = spec + (size_t)y0 * spec_ld, *rb_out = ra_out + spec_ld;
	if (!has_a && !has_b) {
		C z;
		z.x = T(0);
		z.y = T(0);
		for (int k = threadIdx.x; k <= N / 2; k += blockDim.x) {
			ra_out[k] = z;
			rb_out[k] = z;
		}
		return;
	}
	const C *stw = load_twiddles<TWS>(b + N, tw, N);
	// U elements per thread in flight before any is stored
	constexpr int U = 4;
	for (int x0 = threadIdx.x; x0 < N; x0 += U * blockDim.x) {
		C z[U];
#pragma unroll
		for (int u = 0; u < U; u++) {
			const int x = x0 + u * blockDim.x, sx = x - sx0;
			const bool in = x < N && sx >= 0 && sx < sw;
			z[u].x = (has_a && in) ? (T)src[(size_t)ra * sw + sx] : T(0);
			z[u].y = (has_b && in) ? (T)src[(size_t)rb * sw + sx] : T(0);
		}
#pragma unroll
		for (int u = 0; u < U; u++)
			if (x0 + u * blockDim.x < N) a[x0 + u * blockDim.x] = z[u];
	}
	cp_async_wait();
	__syncthreads();
	C *Z = fft_block<1, T, C>(a, b, plan, stw, false);
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
// times conj(K), inverse.  Transform blockIdx.y of a batch reads the kernel
// spectrum at K + blockIdx.y * k_batch (0: one kernel for the whole batch).
// Shared memory: two M x CB buffers and M twiddles.
template <class T, int CB, bool TWS>
__global__ void k_fft_cols(typename Cx<T>::type *__restrict__ spec, int spec_ld, int ncols, int M, FftPlan plan,
                           const typename Cx<T>::type *__restrict__ tw, const typename Cx<T>::type *__restrict__ K,
                           int mode, size_t spec_batch, size_t k_batch, bool k_smem)
{
	pdl_enter();
	using C = typename Cx<T>::type;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *a = reinterpret_cast<C *>(smem_raw);
	C *b = a + (size_t)M * CB;
	spec += blockIdx.y * spec_batch;
	if (K) K += blockIdx.y * k_batch;
	const int c0 = blockIdx.x * CB;
	const C *stw = load_twiddles<TWS>(b + (size_t)M * CB, tw, M);
	// the kernel spectrum's columns, fetched with the data (k_smem: after the
	// twiddles in shared memory)
	C *sk = b + (size_t)M * CB + (TWS ? M : 0);
	if (mode != 0 && k_smem)
		for (int t = threadIdx.x; t < M * CB; t += blockDim.x) {
			int row = t / CB, c = t - row * CB;
			if (c0 + c < ncols) cp_async_elem(sk + t, K + (size_t)row * spec_ld + c0 + c);
		}
	for (int t = threadIdx.x; t < M * CB; t += blockDim.x) {
		int row = t / CB, c = t - row * CB;
		if (c0 + c < ncols) {
			cp_async_elem(a + t, spec + (size_t)row * spec_ld + c0 + c);
		}
		else {
			C v;
			v.x = T(0);
			v.y = T(0);
			a[t] = v;
		}
	}
	cp_async_wait();
	__syncthreads();
	C *S = fft_block<CB, T, C>(a, b, plan, stw, false);
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
			C k = k_smem ? sk[t] : K[(size_t)row * spec_ld + c0 + c];
			if (mode == 2) k.y = -k.y;
			S[t] = cmul(S[t], k);
		}
	}
	__syncthreads();
	C *other = (S == a) ? b : a;
	C *R = fft_block<CB, T, C>(S, other, plan, stw, true);
	for (int t = threadIdx.x; t < M * CB; t += blockDim.x) {
		int row = t / CB, c = t - row * CB;
		if (c0 + c < ncols) spec[(size_t)row * spec_ld + c0 + c] = R[t];
	}
}

// Inverse row pass: rows y0, y0+1 of the result; out(x, y) = c(x + dx, y + dy)
// / (M N) (+ add) for the output window [0, ow) x [0, oh).
template <class T, class TOut, class TAdd, bool TWS>
__global__ void k_fft_rows_inv(const typename Cx<T>::type *__restrict__ spec, int spec_ld, int N, int M, FftPlan plan,
                               const typename Cx<T>::type *__restrict__ tw, int dx, int dy, TOut *__restrict__ out,
                               int ow, int oh, const TAdd *__restrict__ add, int add_stride, int add_ox, int add_oy,
                               size_t spec_batch, size_t out_batch, size_t add_batch)
{
	pdl_enter();
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
	// the two half-spectrum rows land in b[0 .. N/2] and b[N/2+1 .. N+1]
	// (b holds N + 2 elements), the twiddles after them
	const int h = N / 2 + 1;
	const C *stw = load_twiddles<TWS>(b + N + 2, tw, N);
	const C *ra = spec + (size_t)y0 * spec_ld, *rb = ra + spec_ld;
	for (int k = threadIdx.x; k < 2 * h; k += blockDim.x) cp_async_elem(b + k, k < h ? ra + k : rb + (k - h));
	cp_async_wait();
	__syncthreads();
	for (int k = threadIdx.x; k < N; k += blockDim.x) {
		C A, B;
		if (k < h) {
			A = b[k];
			B = b[h + k];
		}
		else {
			A = b[N - k];
			B = b[h + N - k];
			A.y = -A.y;
			B.y = -B.y;
		}
		C z;  // A + i B
		z.x = A.x - B.y;
		z.y = A.y + B.x;
		a[k] = z;
	}
	__syncthreads();
	C *Z = fft_block<1, T, C>(a, b, plan, stw, true);
	const T scale = T(1) / ((T)M * (T)N);
	// U outputs per thread, their `add` loads in flight together
	constexpr int U = 4;
	const TAdd *adda = add ? add + (size_t)(oa + add_oy) * add_stride + add_ox : nullptr;
	const TAdd *addb = add ? add + (size_t)(ob + add_oy) * add_stride + add_ox : nullptr;
	for (int x0 = threadIdx.x; x0 < ow; x0 += U * blockDim.x) {
		T pa[U], pb[U];
#pragma unroll
		for (int u = 0; u < U; u++) {
			const int x = x0 + u * blockDim.x;
			pa[u] = (add && want_a && x < ow) ? (T)adda[x] : T(0);
			pb[u] = (add && want_b && x < ow) ? (T)addb[x] : T(0);
		}
#pragma unroll
		for (int u = 0; u < U; u++) {
			const int x = x0 + u * blockDim.x;
			if (x >= ow) break;
			const int X = x + dx;
			const T va = (X >= 0 && X < N) ? Z[X].x * scale : T(0);
			const T vb = (X >= 0 && X < N) ? Z[X].y * scale : T(0);
			if (want_a) out[(size_t)oa * ow + x] = (TOut)(va + pa[u]);
			if (want_b) out[(size_t)ob * ow + x] = (TOut)(vb + pb[u]);
		}
	}
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

void fft_plan_stages(FftPlan &plan)
{
	int ns = 1;
	for (int s = 0; s < plan.nstages; s++) {
		const int R = plan.radix[s];
		plan.ns[s] = ns;
		plan.nb[s] = plan.n / R;
		plan.tstep[s] = plan.n / (ns * R);
		plan.ns_magic[s] = ns > 1 ? (unsigned)((0x100000000ull + ns - 1) / ns) : 0u;
		ns *= R;
	}
}

bool fft_factor(int n, FftPlan &plan)
{
	plan.n = n;
	plan.nstages = 0;
	int c[6] = {0, 0, 0, 0, 0, 0};  // multiplicity of the primes 2, 3, 5
	int m = n;
	for (int p : {2, 3, 5})
		while (m > 1 && m % p == 0) {
			c[p]++;
			m /= p;
		}
	if (m != 1 || n < 2) return false;
	auto push = [&](int r) {
		if (plan.nstages < FFT_MAX_STAGES) plan.radix[plan.nstages++] = r;
	};
	// pairs first (one register butterfly for two stages), then what is left
	while (c[5] && c[3]) { push(15); c[5]--; c[3]--; }
	while (c[5] && c[2]) { push(10); c[5]--; c[2]--; }
	while (c[3] >= 2) { push(9); c[3] -= 2; }
	while (c[3] && c[2] >= 2) { push(12); c[3]--; c[2] -= 2; }
	while (c[3] && c[2]) { push(6); c[3]--; c[2]--; }
	while (c[2] >= 4) { push(16); c[2] -= 4; }
	while (c[2] >= 3) { push(8); c[2] -= 3; }
	while (c[2] >= 2) { push(4); c[2] -= 2; }
	while (c[5]) { push(5); c[5]--; }
	while (c[3]) { push(3); c[3]--; }
	while (c[2]) { push(2); c[2]--; }
	fft_plan_stages(plan);
	int prod = 1;
	for (int s = 0; s < plan.nstages; s++) prod *= plan.radix[s];
	return prod == n;
}

int fft_good_size(int need)
{
	for (int n = (need + 1) & ~1;; n += 2) {
		FftPlan p;
		if (fft_factor(n, p)) return n;
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

static int sm_count()
{
	static int n = 0;
	if (n <= 0) {
		int dev = 0;
		cudaGetDevice(&dev);
		if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
		cudaGetLastError();
	}
	return n;
}

// Threads for `cols` interleaved transforms of length plan.n: one per
// butterfly of the widest stage (n / smallest radix), in whole warps.
static int fft_threads(const FftPlan &plan, int cols)
{
	int rmin = 16;
	for (int s = 0; s < plan.nstages; s++) rmin = plan.radix[s] < rmin ? plan.radix[s] : rmin;
	int t = (plan.n / rmin) * cols;
	t = (t + 31) / 32 * 32;
	return t < 64 ? 64 : (t > 512 ? 512 : t);
}

// Columns per CTA of the column pass: as many as share memory allows (two
// ping-pong buffers of M x CB complex values within 200 KB) while the grid
// still gives every SM two CTAs; a lone small transform leaves the rest of
// the GPU idle, so parallelism wins over sector efficiency.
template <class T>
static int cols_per_block(int M, int ncols, int batch)
{
	const size_t per = 2 * sizeof(typename Cx<T>::type) * (size_t)M;
	int cb = 8;
	while (cb > 1 && (per * cb + per / 2 > 200 * 1024 || (size_t)((ncols + cb - 1) / cb) * batch < 2 * (size_t)sm_count()))
		cb /= 2;
	return cb;
}

template <class T, int CB>
static cudaError_t launch_cols(typename Cx<T>::type *spec, int spec_ld, int ncols, int M, const FftPlan &pm,
                               const typename Cx<T>::type *tw, const typename Cx<T>::type *K, int mode, int batch,
                               size_t spec_batch, size_t k_batch, cudaStream_t s)
{
	const size_t e = sizeof(typename Cx<T>::type);
	size_t smem = e * (size_t)M * 2 * CB;
	const bool tws = smem + e * (size_t)M <= FFT_SMEM_BYTES;
	if (tws) smem += e * (size_t)M;
	// the kernel columns in shared memory only while two CTAs still fit an SM
	const bool ks = mode != 0 && 2 * (smem + e * (size_t)M * CB) <= FFT_SMEM_BYTES;
	if (ks) smem += e * (size_t)M * CB;
	auto kern = tws ? k_fft_cols<T, CB, true> : k_fft_cols<T, CB, false>;
	static bool configured[2] = {false, false};  // per instantiation; setting it twice is harmless
	if (!configured[tws]) configured[tws] = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                                               FFT_SMEM_BYTES) == cudaSuccess;
	dim3 grid((ncols + CB - 1) / CB, batch);
	return launch_pdl(kern, grid, dim3(fft_threads(pm, CB)), smem, s, spec, spec_ld, ncols, M, pm, tw, K, mode,
	                  spec_batch, k_batch, ks);
}

template <class T>
static cudaError_t cols_any(typename Cx<T>::type *spec, int spec_ld, int ncols, int M, const FftPlan &pm,
                            const typename Cx<T>::type *tw, const typename Cx<T>::type *K, int mode, int batch,
                            size_t spec_batch, size_t k_batch, cudaStream_t s)
{
	switch (cols_per_block<T>(M, ncols, batch)) {
	case 8: return launch_cols<T, 8>(spec, spec_ld, ncols, M, pm, tw, K, mode, batch, spec_batch, k_batch, s);
	case 4: return launch_cols<T, 4>(spec, spec_ld, ncols, M, pm, tw, K, mode, batch, spec_batch, k_batch, s);
	case 2: return launch_cols<T, 2>(spec, spec_ld, ncols, M, pm, tw, K, mode, batch, spec_batch, k_batch, s);
	default: return launch_cols<T, 1>(spec, spec_ld, ncols, M, pm, tw, K, mode, batch, spec_batch, k_batch, s);
	}
}

// The composite radices' roots of unity in constant memory, once per device.
static cudaError_t ensure_roots()
{
	static std::mutex mu;
	static bool done[64] = {};
	int dev = 0;
	cudaError_t e = cudaGetDevice(&dev);
	if (e != cudaSuccess) return e;
	std::lock_guard<std::mutex> g(mu);
	if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
	static double2 r64[17][16];
	static float2 r32[17][16];
	for (int Q = 1; Q <= 16; Q++)
		for (int m = 0; m < 16; m++) {
			const long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)(m % Q) / (long double)Q;
			r64[Q][m] = make_double2((double)cosl(ang), (double)sinl(ang));
			r32[Q][m] = make_float2((float)cosl(ang), (float)sinl(ang));
		}
	e = cudaMemcpyToSymbol(c_roots64, r64, sizeof(r64));
	if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_roots32, r32, sizeof(r32));
	if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev] = true;
	return e;
}

template <class T>
cudaError_t FftConv<T>::setup(int M_, int N_)
{
	cudaError_t re = ensure_roots();
	if (re != cudaSuccess) return re;
	if (M_ == M && N_ == N && tw_m && tw_n) return cudaSuccess;
	M = M_;
	N = N_;
	if (!fft_factor(M, plan_m) || !fft_factor(N, plan_n) || (M & 1) || (N & 1)) return cudaErrorInvalidValue;
	if (N > FFT_MAX_LEN || M > FFT_MAX_LEN) return cudaErrorInvalidValue;
	tw_m = twiddles<T>(M);
	tw_n = twiddles<T>(N);
	if (!tw_m || !tw_n) return cudaErrorMemoryAllocation;
	ld = N / 2 + 1;
	have_kernel = false;
	return cudaGetLastError();
}

template <class T>
template <class TIn>
cudaError_t FftConv<T>::forward_rows(const TIn *src, int sw, int sh, int sx0, int sy0, Cplx *spec, int batch,
                                     size_t src_batch, cudaStream_t s)
{
	const bool tws = 3 * sizeof(Cplx) * (size_t)N <= FFT_SMEM_BYTES;
	size_t smem = (tws ? 3 : 2) * sizeof(Cplx) * (size_t)N;
	dim3 grid(M / 2, batch);
	auto kern = tws ? k_fft_rows_fwd<T, TIn, true> : k_fft_rows_fwd<T, TIn, false>;
	static bool configured[2] = {false, false};  // per instantiation; setting it twice is harmless
	if (!configured[tws]) configured[tws] = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                                               FFT_SMEM_BYTES) == cudaSuccess;
	return launch_pdl(kern, grid, dim3(fft_threads(plan_n, 1)), smem, s, src, sw, sh, sx0, sy0, N, plan_n, tw_n, spec,
	                  ld, src_batch, (size_t)M * ld);
}

template <class T>
cudaError_t FftConv<T>::set_kernel(const T *psf_dev, int kw, int kh, Cplx *kspec, cudaStream_t s)
{
	cudaError_t e = forward_rows<T>(psf_dev, kw, kh, 0, 0, kspec, 1, 0, s);
	if (e != cudaSuccess) return e;
	e = cols_any<T>(kspec, ld, ld, M, plan_m, tw_m, nullptr, 0, 1, 0, 0, s);
	have_kernel = e == cudaSuccess;
	return e;
}

template <class T>
cudaError_t FftConv<T>::set_kernels(const float *psf_dev, int kw, int kh, size_t psf_batch, Cplx *kspec, int batch,
                                    cudaStream_t s)
{
	cudaError_t e = forward_rows<float>(psf_dev, kw, kh, 0, 0, kspec, batch, psf_batch, s);
	if (e != cudaSuccess) return e;
	e = cols_any<T>(kspec, ld, ld, M, plan_m, tw_m, nullptr, 0, batch, spectrum_elems(), 0, s);
	have_kernel = e == cudaSuccess;
	return e;
}

template <class T>
template <class TIn, class TOut, class TAdd>
cudaError_t FftConv<T>::convolve(const TIn *src, int sw, int sh, int sx0, int sy0, const Cplx *kspec, bool adjoint,
                                 Cplx *work, int dx, int dy, TOut *out, int ow, int oh, const TAdd *add,
                                 int add_stride, int add_ox, int add_oy, int batch, size_t src_batch,
                                 size_t out_batch, size_t add_batch, cudaStream_t s, size_t kspec_batch)
{
	cudaError_t e = forward_rows<TIn>(src, sw, sh, sx0, sy0, work, batch, src_batch, s);
	if (e != cudaSuccess) return e;
	e = cols_any<T>(work, ld, ld, M, plan_m, tw_m, kspec, adjoint ? 2 : 1, batch, (size_t)M * ld, kspec_batch, s);
	if (e != cudaSuccess) return e;
	const bool tws = sizeof(Cplx) * (3 * (size_t)N + 2) <= FFT_SMEM_BYTES;
	size_t smem = sizeof(Cplx) * ((tws ? 3 : 2) * (size_t)N + 2);
	dim3 grid(M / 2, batch);
	auto kern = tws ? k_fft_rows_inv<T, TOut, TAdd, true> : k_fft_rows_inv<T, TOut, TAdd, false>;
	static bool configured[2] = {false, false};  // per instantiation; setting it twice is harmless
	if (!configured[tws]) configured[tws] = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                                               FFT_SMEM_BYTES) == cudaSuccess;
	return launch_pdl(kern, grid, dim3(fft_threads(plan_n, 1)), smem, s, (const Cplx *)work, ld, N, M, plan_n, tw_n, dx,
	                  dy, out, ow, oh, add, add_stride, add_ox, add_oy, (size_t)M * ld, out_batch, add_batch);
}

template struct FftConv<double>;
template struct FftConv<float>;
template cudaError_t FftConv<double>::convolve<double, double, double>(const double *, int, int, int, int,
                                                                      const Cplx *, bool, Cplx *, int, int, double *,
                                                                      int, int, const double *, int, int, int, int,
                                                                      size_t, size_t, size_t, cudaStream_t, size_t);
template cudaError_t FftConv<double>::convolve<float, double, float>(const float *, int, int, int, int, const Cplx *,
                                                                    bool, Cplx *, int, int, double *, int, int,
                                                                    const float *, int, int, int, int, size_t,
                                                                    size_t, size_t, cudaStream_t, size_t);
template cudaError_t FftConv<double>::convolve<float, float, float>(const float *, int, int, int, int, const Cplx *,
                                                                   bool, Cplx *, int, int, float *, int, int,
                                                                   const float *, int, int, int, int, size_t, size_t,
                                                                   size_t, cudaStream_t, size_t);
template cudaError_t FftConv<float>::convolve<float, float, float>(const float *, int, int, int, int, const Cplx *,
                                                                  bool, Cplx *, int, int, float *, int, int,
                                                                  const float *, int, int, int, int, size_t, size_t,
                                                                  size_t, cudaStream_t, size_t);

}  // namespace pf
