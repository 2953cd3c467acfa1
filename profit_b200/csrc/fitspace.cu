// Device kernels of the fit space (fitspace.cuh): one thread per proposal.
#include "common.cuh"
#include "fitspace.cuh"
#include "launch.h"

namespace pf {

// parm[batch][nfit] -> values[batch][nrefs] (theta of the free and tied
// entries, what the batch prologue sets on the profiles) and
// parm_out[batch][nfit] (the fitted vector ProFit hands back).
__global__ void k_fit_remake(FitSpaceView fs, int batch, const double *__restrict__ parm, double *__restrict__ values,
                             double *__restrict__ parm_out)
{
	pdl_enter();
	const int b = blockIdx.x * blockDim.x + threadIdx.x;
	if (b >= batch) return;
	fit_remake(fs, parm + (size_t)b * fs.nfit, values + (size_t)b * fs.nrefs, parm_out + (size_t)b * fs.nfit);
}

// LP, d LP / d parm and LL per proposal from the adjoint's LL and
// d LL / d theta: out = [batch] LP, [batch][nfit] gradient, [batch] LL.
__global__ void k_fit_finish(FitSpaceView fs, int batch, const double *__restrict__ parm,
                             const double *__restrict__ values, const double *__restrict__ ll,
                             const double *__restrict__ grad_ll, double *__restrict__ out)
{
	pdl_enter();
	const int b = blockIdx.x * blockDim.x + threadIdx.x;
	if (b >= batch) return;
	fit_finish_one(fs, parm + (size_t)b * fs.nfit, values + (size_t)b * fs.nrefs, ll[b],
	               grad_ll + (size_t)b * fs.nrefs, out + b, out + batch + (size_t)b * fs.nfit,
	               out + batch + (size_t)batch * fs.nfit + b);
}

cudaError_t launch_fit_remake(const FitSpaceView &fs, int batch, const double *parm, double *values, double *parm_out,
                              cudaStream_t s)
{
	note_launches(1);
	return launch_pdl(k_fit_remake, dim3((batch + 127) / 128), dim3(128), 0, s, fs, batch, parm, values, parm_out);
}

cudaError_t launch_fit_finish(const FitSpaceView &fs, int batch, const double *parm, const double *values,
                              const double *ll, const double *grad_ll, double *out, cudaStream_t s)
{
	note_launches(1);
	return launch_pdl(k_fit_finish, dim3((batch + 127) / 128), dim3(128), 0, s, fs, batch, parm, values, ll, grad_ll,
	                  out);
}

}  // namespace pf
