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

template <class T>
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
	k_fma<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-6);
	float best = 1e30f;
	for (int r = 0; r < reps; r++) {
		cudaEventRecord(e0);
		k_fma<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-6);
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
	double flops = 2.0 * 8.0 * iters * threads * (double)blocks;
	return flops / (best * 1e-3) / 1e12;
}

}  // namespace

extern "C" {

// TFLOP/s of dependent-chain FMA streams, best of `reps` launches.
double pf_peak_fma_tflops(int fp64, int iters, int reps)
{
	return fp64 ? run<double>(iters, reps) : run<float>(iters, reps);
}
}
