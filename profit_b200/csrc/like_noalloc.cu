// The "norm" log-likelihood of ProFit's profitLikeModel (R/profitLikeModel.R:
// 263-276) over model images that the caller already holds in device memory,
// computed without allocating anything.
//
// The kernels are the ones pf_model_loglike (PF_FP64) runs: Neumaier partial
// sums over like_parts(npix, 1) blocks per image (common.cuh), then a merge of
// those partials in a fixed order.  pf_model_loglike forms the same partials
// over the same grid and merges them in the same order, so equal images give
// the same logL to the last bit.  The difference is where the block partials
// live: pf_model_loglike keeps them in a buffer its model handle allocates,
// while this entry point uses the file-scope device array below.
//
// Sharing: every call on every stream of a device uses the same array, and
// the array keeps whatever the last call left in it.  Nothing in it has to
// start at zero: each block of the partial pass writes its own slot before
// the final pass of the same call reads it, so leftovers of an earlier call
// are never read.  Two calls whose kernels can overlap on the GPU (calls on
// different streams without an ordering between them) overwrite each other's
// partials and return wrong values; calls on one stream are ordered and safe.
#include <climits>
#include <cstdio>
#include <cuda.h>
#include <mutex>

#include "launch.h"
#include "like.cuh"
#include "profit_b200.h"

namespace {

constexpr int PARTS = pf::LIKE_MAX_PARTS;  // most block partials per image
constexpr int MAX_DEVICES = 64;

// Scratch of the partial pass: PF_LOGLIKE_NOALLOC_MAX_BATCH images x PARTS
// (sum, compensation) pairs = 303,104 bytes on each device.
static __device__ __align__(256) double2 g_partials[PF_LOGLIKE_NOALLOC_MAX_BATCH * PARTS];

// The array's address is a property of the context that loaded this
// library's device code: a cudaDeviceReset, or another context made current
// on the device, gives the array a new address.  The cache therefore keeps,
// per device, the unique id of the context it looked the address up in
// (cuCtxGetId, reached through the runtime's driver entry points so that no
// link against libcuda is needed) and looks it up again when the current
// context's id differs.
struct Slot {
	unsigned long long ctx_id;  // 0 = not looked up yet
	double2 *addr;
};
std::mutex g_setup_mu;
Slot g_slots[MAX_DEVICES];  // guarded by g_setup_mu

using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

int cuda_failure(const char *what, cudaError_t e)
{
	char msg[256];
	snprintf(msg, sizeof msg, "%s: %s", what, cudaGetErrorString(e));
	return pf::report_error(PF_E_CUDA, msg);
}

// Unique id of the calling thread's current context (0 if none is current).
int current_context_id(unsigned long long *id)
{
	static CtxGetCurrentFn get_current = nullptr;
	static CtxGetIdFn get_id = nullptr;
	static std::once_flag once;
	static cudaError_t lookup = cudaSuccess;
	std::call_once(once, [] {
		cudaDriverEntryPointQueryResult q1, q2;
		cudaError_t e1 = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", (void **)&get_current, 12000,
		                                                  cudaEnableDefault, &q1);
		cudaError_t e2 =
		    cudaGetDriverEntryPointByVersion("cuCtxGetId", (void **)&get_id, 12000, cudaEnableDefault, &q2);
		if (e1 != cudaSuccess) lookup = e1;
		else if (e2 != cudaSuccess) lookup = e2;
		else if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !get_current || !get_id)
			lookup = cudaErrorSymbolNotFound;
	});
	if (lookup != cudaSuccess) return cuda_failure("driver entry points cuCtxGetCurrent/cuCtxGetId", lookup);
	CUcontext ctx = nullptr;
	if (get_current(&ctx) != CUDA_SUCCESS) return pf::report_error(PF_E_CUDA, "cuCtxGetCurrent failed");
	*id = 0;
	if (ctx && get_id(ctx, id) != CUDA_SUCCESS) return pf::report_error(PF_E_CUDA, "cuCtxGetId failed");
	return PF_OK;
}

// Device address of g_partials in the calling thread's current context.  The
// first call in a context looks it up (cudaGetSymbolAddress, with the
// device current; it creates the device's primary context if none is
// current yet); later calls in the same context read the cached address.
int partials_address(double2 **out)
{
	int dev = -1;
	cudaError_t e = cudaGetDevice(&dev);
	if (e != cudaSuccess) return cuda_failure("cudaGetDevice", e);
	if (dev < 0 || dev >= MAX_DEVICES) return pf::report_error(PF_E_CUDA, "device index beyond 63");
	unsigned long long id = 0;
	int st = current_context_id(&id);
	if (st != PF_OK) return st;
	std::lock_guard<std::mutex> g(g_setup_mu);
	if (id != 0 && g_slots[dev].ctx_id == id) {
		*out = g_slots[dev].addr;
		return PF_OK;
	}
	double2 *p = nullptr;
	e = cudaGetSymbolAddress((void **)&p, g_partials);
	if (e != cudaSuccess) return cuda_failure("cudaGetSymbolAddress(g_partials)", e);
	st = current_context_id(&id);  // the lookup above made a context current if none was
	if (st != PF_OK) return st;
	g_slots[dev] = Slot{id, p};
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
	// the grid pf_model_loglike uses for one image of npix pixels (at most
	// PARTS blocks, so each image's partials fit its PARTS slots)
	const int parts = pf::like_parts((int)npix, 1);
	cudaStream_t s = (cudaStream_t)stream;
	pf::k_loglike_partial<double><<<dim3(parts, batch), 256, 0, s>>>(model, data, sigma, region, (int)npix,
	                                                                   partials, nullptr, 0);
	pf::k_loglike_final<<<batch, 256, 0, s>>>(partials, parts, loglike);
	pf::note_launches(2);
	cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess) return cuda_failure("log-likelihood launch", e);
	return PF_OK;
}
