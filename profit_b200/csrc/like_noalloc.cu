// The "norm" log-likelihood of ProFit's profitLikeModel (R/profitLikeModel.R:
// 263-276) over model images that the caller already holds in device memory,
// computed without allocating anything.
//
// The kernels are the ones pf_model_loglike runs (like.cuh: Neumaier partial
// sums over a fixed grid of 296 blocks per image, then one block per image
// merging the partials), so equal inputs give the same number to the last
// bit.  The difference is where the block partials live:
// pf_model_loglike keeps them in a buffer its model handle allocates, while
// this entry point uses the file-scope device array below, whose address is
// looked up once per device.
//
// Sharing: every call on every stream of a device uses the same array, and
// the array keeps whatever the last call left in it.  Nothing in it has to
// start at zero: each block of the partial pass writes its own slot before
// the final pass of the same call reads it, so leftovers of an earlier call
// are never read.  Two calls whose kernels can overlap on the GPU (calls on
// different streams without an ordering between them) overwrite each other's
// partials and return wrong values; calls on one stream are ordered and safe.
#include <atomic>
#include <climits>
#include <cstdio>
#include <mutex>

#include "launch.h"
#include "like.cuh"
#include "profit_b200.h"

namespace {

constexpr int PARTS = 296;  // block partials per image (the grid of pf_model_loglike)
constexpr int MAX_DEVICES = 64;

// Scratch of the partial pass: PF_LOGLIKE_NOALLOC_MAX_BATCH images x PARTS
// (sum, compensation) pairs = 303,104 bytes on each device.
static __device__ __align__(256) double2 g_partials[PF_LOGLIKE_NOALLOC_MAX_BATCH * PARTS];

std::mutex g_setup_mu;
std::atomic<double2 *> g_partials_addr[MAX_DEVICES];

int cuda_failure(const char *what, cudaError_t e)
{
	char msg[256];
	snprintf(msg, sizeof msg, "%s: %s", what, cudaGetErrorString(e));
	return pf::report_error(PF_E_CUDA, msg);
}

// Device address of g_partials on the calling thread's current device.  The
// first call on a device looks it up with that device current; later calls
// read the cached address.
int partials_address(double2 **out)
{
	int dev = -1;
	cudaError_t e = cudaGetDevice(&dev);
	if (e != cudaSuccess) return cuda_failure("cudaGetDevice", e);
	if (dev < 0 || dev >= MAX_DEVICES) return pf::report_error(PF_E_CUDA, "device index beyond 63");
	double2 *p = g_partials_addr[dev].load(std::memory_order_acquire);
	if (!p) {
		std::lock_guard<std::mutex> g(g_setup_mu);
		p = g_partials_addr[dev].load(std::memory_order_acquire);
		if (!p) {
			e = cudaGetSymbolAddress((void **)&p, g_partials);
			if (e != cudaSuccess) return cuda_failure("cudaGetSymbolAddress(g_partials)", e);
			g_partials_addr[dev].store(p, std::memory_order_release);
		}
	}
	*out = p;
	return PF_OK;
}

}  // namespace

extern "C" int pf_loglike_norm_noalloc(const double *model, const double *data, const double *sigma,
                                       const uint8_t *region, size_t npix, int batch, double *loglike,
                                       void *stream)
{
	if (!model || !data || !sigma || !loglike) return pf::report_error(PF_E_INVALID, "null argument");
	if (batch < 1) return pf::report_error(PF_E_INVALID, "batch must be at least 1");
	if (batch > PF_LOGLIKE_NOALLOC_MAX_BATCH)
		return pf::report_error(PF_E_CAPACITY,
		                        "batch exceeds PF_LOGLIKE_NOALLOC_MAX_BATCH (64 images), the size of the static scratch");
	if (npix > (size_t)INT_MAX) return pf::report_error(PF_E_CAPACITY, "npix exceeds 2^31 - 1 pixels per image");
	double2 *partials = nullptr;
	int st = partials_address(&partials);
	if (st != PF_OK) return st;
	cudaStream_t s = (cudaStream_t)stream;
	pf::k_loglike_partial<double><<<dim3(PARTS, batch), 256, 0, s>>>(model, data, sigma, region, (int)npix,
	                                                                   partials, nullptr, 0);
	pf::k_loglike_final<<<batch, 256, 0, s>>>(partials, PARTS, loglike);
	pf::note_launches(2);
	cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess) return cuda_failure("log-likelihood launch", e);
	return PF_OK;
}
