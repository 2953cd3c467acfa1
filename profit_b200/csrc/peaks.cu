// Non-tensor FMA throughput of this GPU (FP32 and FP64), the roofline
// denominators of the convolution and render kernels.  Built into its own
// library (libpf_peaks.so) and used by the benchmark only.
//
// Each thread runs 8 independent FMA chains of `iters` steps; the grid is a
// multiple of the SM count with 1024 threads per SM.  FLOPs = 2 * 8 * iters
// per thread.  The chains are written back so nothing is dead code.
#include <cuda_runtime.h>

namespace {

template <class T>
__global__ void k_fma(T *out, int iters, T a, T b)
{
	T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
	for (int i = 0; i < iters; i++) {
		x0 = x0 * a + b;
		x1 = x1 * a + b;
		x2 = x2 * a + b;
		x3 = x3 * a + b;
		x4 = x4 * a + b;
		x5 = x5 * a + b;
		x6 = x6 * a + b;
		x7 = x7 * a + b;
	}
	out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

// The same with packed FP32 pairs (fma.rn.f32x2 on sm_100): 16 FMAs per
// thread and step from 8 packed instructions.
__global__ void k_fma2(float *out, int iters, float a, float b)
{
	const float2 A = make_float2(a, a), B = make_float2(b, b);
	float t = threadIdx.x;
	float2 x0 = make_float2(t, t + 1), x1 = make_float2(t + 2, t + 3), x2 = make_float2(t + 4, t + 5),
	       x3 = make_float2(t + 6, t + 7), x4 = make_float2(t + 8, t + 9), x5 = make_float2(t + 10, t + 11),
	       x6 = make_float2(t + 12, t + 13), x7 = make_float2(t + 14, t + 15);
	for (int i = 0; i < iters; i++) {
		x0 = __ffma2_rn(x0, A, B);
		x1 = __ffma2_rn(x1, A, B);
		x2 = __ffma2_rn(x2, A, B);
		x3 = __ffma2_rn(x3, A, B);
		x4 = __ffma2_rn(x4, A, B);
		x5 = __ffma2_rn(x5, A, B);
		x6 = __ffma2_rn(x6, A, B);
		x7 = __ffma2_rn(x7, A, B);
	}
	float s = x0.x + x0.y + x1.x + x1.y + x2.x + x2.y + x3.x + x3.y + x4.x + x4.y + x5.x + x5.y + x6.x + x6.y +
	          x7.x + x7.y;
	out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Transcendental (XU / MUFU) throughput: 8 independent chains of the fast
// exponential per thread (one XU operation and one multiply per step); the
// result is XU operations per second.
__global__ void k_xu(float *out, int iters, float a)
{
	float t = threadIdx.x * 1e-6f;
	float x0 = t, x1 = t + 1e-3f, x2 = t + 2e-3f, x3 = t + 3e-3f, x4 = t + 4e-3f, x5 = t + 5e-3f, x6 = t + 6e-3f,
	      x7 = t + 7e-3f;
	for (int i = 0; i < iters; i++) {
		x0 = __expf(x0 * a);
		x1 = __expf(x1 * a);
		x2 = __expf(x2 * a);
		x3 = __expf(x3 * a);
		x4 = __expf(x4 * a);
		x5 = __expf(x5 * a);
		x6 = __expf(x6 * a);
		x7 = __expf(x7 * a);
	}
	out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

double run_xu(int iters, int reps)
{
	int dev = 0, sms = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	const int threads = 256, blocks = sms * 4;
	float *out = nullptr;
	if (cudaMalloc(&out, sizeof(float) * threads * blocks) != cudaSuccess) return -1;
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	k_xu<<<blocks, threads>>>(out, iters, -0.5f);
	float best = 1e30f;
	for (int r = 0; r < reps; r++) {
		cudaEventRecord(e0);
		k_xu<<<blocks, threads>>>(out, iters, -0.5f);
		cudaEventRecord(e1);
		cudaEventSynchronize(e1);
		float ms = 0;
		cudaEventElapsedTime(&ms, e0, e1);
		if (ms < best) best = ms;
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaFree(out);
	if (cudaGetLastError() != cudaSuccess) return -1;
	return 8.0 * iters * threads * (double)blocks / (best * 1e-3) / 1e12;
}

template <class T, bool Packed = false>
double run(int iters, int reps)
{
	int dev = 0, sms = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	const int threads = 256, blocks = sms * 4;
	T *out = nullptr;
	if (cudaMalloc(&out, sizeof(T) * threads * blocks) != cudaSuccess) return -1;
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	auto launch = [&]() {
		if constexpr (Packed)
			k_fma2<<<blocks, threads>>>(out, iters, 0.999999f, 1e-6f);
		else
			k_fma<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-6);
	};
	launch();
	float best = 1e30f;
	for (int r = 0; r < reps; r++) {
		cudaEventRecord(e0);
		launch();
		cudaEventRecord(e1);
		cudaEventSynchronize(e1);
		float ms = 0;
		cudaEventElapsedTime(&ms, e0, e1);
		if (ms < best) best = ms;
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaFree(out);
	if (cudaGetLastError() != cudaSuccess) return -1;
	double flops = 2.0 * (Packed ? 16.0 : 8.0) * iters * threads * (double)blocks;
	return flops / (best * 1e-3) / 1e12;
}

}  // namespace

extern "C" {

// TFLOP/s of dependent-chain FMA streams, best of `reps` launches.
// kind: 0 = FP32 FMA, 1 = FP64 FMA, 2 = packed FP32 pairs (FFMA2),
// 3 = transcendental (XU) operations in Tops/s (fast exponentials).
double pf_peak_fma_tflops(int kind, int iters, int reps)
{
	if (kind == 3) return run_xu(iters, reps);
	if (kind == 1) return run<double>(iters, reps);
	if (kind == 2) return run<float, true>(iters, reps);
	return run<float>(iters, reps);
}
}
