// Host-side launch wrappers of the kernels (one translation unit each, so the
// FP64 parity kernels can be compiled without FMA contraction).
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

#include "common.cuh"

namespace pf {

// Adds n to the process-wide count of kernels launched by this library.
void note_launches(int n);

// Stores `msg` as the calling thread's pf_last_error() text; returns `code`.
int report_error(int code, const char *msg);

// render64.cu
// mask: optional drawing-size calculation mask (radial and sky profiles skip its zeros)
cudaError_t launch_pixels64(const DevProfile *profiles, int n_profiles, unsigned width, unsigned height, double sx,
                            double sy, double *img_conv, double *img_plain, const uint8_t *mask, const QueueSet &q,
                            cudaStream_t s);
// out(i, j) = plain(i + ox, j + oy) where the drawing mask is 0 (masked convolution)
cudaError_t launch_mask_select64(double *out, unsigned ow, unsigned oh, const double *plain, const uint8_t *mask,
                                 unsigned dw, unsigned ox, unsigned oy, cudaStream_t s);
// out &= mask
cudaError_t launch_mask_and64(double *out, const uint8_t *mask, size_t n, cudaStream_t s);
cudaError_t launch_levels64(const DevProfile *profiles, int n_levels, double *img_conv, double *img_plain,
                            const QueueSet &q, cudaStream_t s);
cudaError_t launch_count_decisions(const QueueSet &q, int n_levels, size_t npix, cudaStream_t s);
cudaError_t launch_psf_stamp64(const DevProfile *profiles, int p, const double *psf, unsigned psf_w, unsigned psf_h,
                               double psf_sx, double psf_sy, double scale_x, double scale_y, double offx, double offy,
                               unsigned width, unsigned height, double *img_conv, double *img_plain, cudaStream_t s);
cudaError_t launch_conv64(const double *src, int sw, int sh, int ox, int oy, const double *K, int kw, int kh,
                          double *out, int ow, int oh, const double *add, int add_stride, int add_ox, int add_oy,
                          cudaStream_t s);
cudaError_t launch_loglike64(const double *model, const double *data, const double *sigma, const uint8_t *region,
                             int n, double2 *partials, int nparts, double *out, cudaStream_t s);
cudaError_t launch_crop64(const double *src, unsigned sw, unsigned ox, unsigned oy, double *out, unsigned ow,
                          unsigned oh, const double *add, cudaStream_t s);
cudaError_t launch_downsample64(const double *src, unsigned sw, unsigned sh, unsigned fs, double *out, unsigned ow,
                                unsigned oh, cudaStream_t s);

// render32.cu
// Tangent planes of the stored-tangent adjoint, nt per profile
// (tangent_stride of the model): FP32, or FP64 where a subsampled pixel's
// cells must be added without FP32 cancellation (tiny, bright profiles).
struct JacPlanes {
	void *p = nullptr;
	bool fp64 = false;
	JacPlanes() = default;
	JacPlanes(float *f) : p(f), fp64(false) {}
	JacPlanes(double *d) : p(d), fp64(true) {}
	JacPlanes(std::nullptr_t) {}
};
// jac: tangent planes (null: values only);
// all_kinds: the model has radial profiles other than Sersic and Moffat.
// mask: optional drawing-size calculation mask shared by the batch entries
// extent: optional, per batch entry the part of the drawing (x < extent.x,
// y < extent.y) that its outputs read; beyond it the images are zero and no
// tangent planes are written (a catalogue galaxy in a larger shared canvas)
cudaError_t launch_pixels32(const FProfile *profiles, const int *prof_begin, int batch, unsigned width,
                            unsigned height, double sx, double sy, float *img_conv, float *img_plain, JacPlanes jac,
                            int nt, bool all_kinds, const QueueSet &q, cudaStream_t s, const uint8_t *mask = nullptr,
                            const int2 *extent = nullptr);
// psf point-source profiles in the FP32 pipeline: the stamp (forward) and the
// sums of the adjoint image against the stamp and its centre derivatives.
cudaError_t launch_psf_stamp32(const DevProfile *dev, const int *prof_begin, int batch, const double *psf,
                               unsigned psf_w, unsigned psf_h, double psf_sx, double psf_sy, double scale_x,
                               double scale_y, double offx, double offy, unsigned width, unsigned height,
                               float *img_conv, float *img_plain, cudaStream_t s);
cudaError_t launch_psf_adjoint32(const DevProfile *dev, const int *prof_begin, int batch, int nprof_max,
                                 const double *psf, unsigned psf_w, unsigned psf_h, double psf_sx, double psf_sy,
                                 double scale_x, double scale_y, double offx, double offy, unsigned width,
                                 unsigned height, const float *g_conv, const float *g_plain, double *T, cudaStream_t s);
// Masked convolution select, finesampling sum-down and output mask of the
// FP32 pipeline (sel, mask_out optional), and their adjoint seeds.
cudaError_t launch_model_finish32(const double *fine, unsigned cw, unsigned ch, const float *plain, const uint8_t *sel,
                                  unsigned dw, unsigned dh, unsigned padx, unsigned pady, unsigned fs,
                                  const uint8_t *mask_out, double *out, unsigned ow, unsigned oh, int batch,
                                  cudaStream_t s);
cudaError_t launch_seed_finish32(const float *w, unsigned ow, unsigned oh, const uint8_t *mask_out, const uint8_t *sel,
                                 unsigned fs, unsigned cw, unsigned ch, unsigned padx, unsigned pady, unsigned dw,
                                 unsigned dh, int batch, float *seed_conv, float *g_plain, cudaStream_t s);
// Levels >= 3 (reached only by Sersic centre cusps) run in one CTA when the
// launch holds at most this many cusps, else one grid-wide launch per level.
constexpr int DEEP_ONE_CTA_MAX_CUSPS = 8;
// cusps: Sersic profiles with adjust across the launch's batch entries (those
// that may recurse past level 2).
cudaError_t launch_levels32(const FProfile *profiles, int n_levels, unsigned npix, float *img_conv, float *img_plain,
                            JacPlanes jac, int nt, bool all_kinds, int cusps, const QueueSet &q, cudaStream_t s);
// partials: n_profiles * jac_reduce_blocks(width, height, n_profiles) * NTAN doubles;
// tickets: n_profiles zero-initialised counters (left at zero again), one
// more when grad is given.  grad (optional): the arguments of
// launch_batch_gradient; the reduction then also runs that step (in the block
// that completes the last profile) and the separate launch is not needed.
// Only valid when nothing else writes T after the reduction (no psf profile).
struct GradStepArgs {
	const DevProfile *dev;
	int nprof, batch, nrefs;
	const int *ref_profile, *ref_code;
	const double *ll;
	const int *invalid;
	double *out_ll, *out_grad;
	// optional (folded form): after the step, ctrl_in[0 .. ctrl_words) is
	// copied to ctrl_out (e.g. the queue counters into a mapped host buffer)
	const uint32_t *ctrl_in = nullptr;
	uint32_t *ctrl_out = nullptr;
	int ctrl_words = 0;
	// optional: after everything above is written, *seq_in is stored to
	// *seq_out (a word of mapped host memory the caller polls)
	const unsigned *seq_in = nullptr;
	unsigned *seq_out = nullptr;
};
unsigned jac_reduce_blocks(unsigned width, unsigned height, int n_profiles);
// width, height, sx, sy, extent: the drawing grid and extents as given to
// launch_pixels32, whose tiles skipped by a profile, and pixels beyond its
// batch entry's extent, hold no tangent planes of that profile.
cudaError_t launch_jac_reduce(JacPlanes jac, const float *g_conv, const float *g_plain, const FProfile *profiles,
                              const int *prof_batch, int n_profiles, unsigned width, unsigned height, double sx,
                              double sy, int nt, double *partials, unsigned *tickets, double *out, cudaStream_t s,
                              const GradStepArgs *grad = nullptr, const int2 *extent = nullptr);
// Copies `bytes` (a multiple of 16, both addresses 16-byte aligned) from
// pinned host memory mapped into the device's address space to dst, and
// zeroes ctrl[0 .. ctrl_words); one launch in place of a copy and a memset.
cudaError_t launch_stage_in(void *dst, const void *host_src, size_t bytes, uint32_t *ctrl, int ctrl_words,
                            cudaStream_t s);
cudaError_t launch_embed_seed(const float *w, unsigned ow, unsigned oh, unsigned padx, unsigned pady, unsigned dw,
                              unsigned dh, int batch, float *g_plain, cudaStream_t s);
cudaError_t launch_conv32_to64(const float *src, int sw, int sh, int ox, int oy, const float *K, int kw, int kh,
                               double *out, int ow, int oh, const float *add, int add_stride, int add_ox, int add_oy,
                               int batch, int batch_src_stride, int batch_out_stride, double *scratch,
                               size_t scratch_bytes, int batch_k_stride, cudaStream_t s);
// batch_k_stride: elements between the kernels of consecutive batch entries
// (0: one kernel for the whole batch)
cudaError_t launch_conv32(const float *src, int sw, int sh, int ox, int oy, const float *K, int kw, int kh,
                          float *out, int ow, int oh, const float *add, int add_stride, int add_ox, int add_oy,
                          int batch, int batch_src_stride, int batch_out_stride, double *scratch, size_t scratch_bytes,
                          int batch_k_stride, cudaStream_t s);
// FP64 scratch (bytes) that lets the FP32 convolution split kernel columns
// over CTAs for `batch` outputs of ow x oh; 0 when the batch is large enough
// to fill the GPU without it.
size_t conv32_scratch_bytes(int ow, int oh, int batch);
cudaError_t launch_loglike32(const float *model, const double *data, const double *sigma, const uint8_t *region,
                             int n, int batch, int data_batch_stride, double2 *partials, int nparts, double *out,
                             float *wseed, cudaStream_t s);
cudaError_t launch_crop32(const float *src, unsigned sw, unsigned ox, unsigned oy, float *out, unsigned ow,
                          unsigned oh, const float *add, int batch, unsigned src_stride, cudaStream_t s);

}  // namespace pf

namespace pf {
// render64.cu: FP32 -> FP64 copy and the FP64 likelihood that also writes the
// adjoint seed (mixed-precision path).
cudaError_t launch_widen(const float *src, double *dst, size_t n, cudaStream_t s);
cudaError_t launch_loglike64_seed(const double *model, const double *data, const double *sigma,
                                  const uint8_t *region, int n, double2 *partials, int nparts, double *out,
                                  float *wseed, cudaStream_t s);
}  // namespace pf

namespace pf {
// render32.cu: batched proposals
cudaError_t launch_batch_prologue(const ProfileParams *tmpl, int nprof, int batch, const int *ref_profile,
                                  const int *ref_offset, int nrefs, const double *values, const ModelGeom &g,
                                  DevProfile *dev, FProfile *fprof, int *invalid, cudaStream_t s);
cudaError_t launch_batch_gradient(const DevProfile *dev, int nprof, int batch, const int *ref_profile,
                                  const int *ref_code, int nrefs, const double *T, const double *ll,
                                  const int *invalid, double *out_ll, double *out_grad, cudaStream_t s);
cudaError_t launch_loglike64_batch(const double *model, const double *data, const double *sigma,
                                   const uint8_t *region, int n, int batch, int data_batch_stride, double2 *partials,
                                   int nparts, double *out, float *wseed, cudaStream_t s,
                                   unsigned *tickets = nullptr);
}  // namespace pf

namespace pf {
// render32.cu: recomputing adjoint of the render (no stored tangent planes).
// Models with at least ADJOINT_LIST_MIN_PROFILES profiles per batch entry
// take the per-tile profile lists (k_adjoint_pixels32_listed), others one
// block per tile and profile.
constexpr int ADJOINT_LIST_MIN_PROFILES = 8;
cudaError_t launch_adjoint_recompute(const FProfile *profiles, const int *prof_batch, const int *prof_begin,
                                     int batch, int n_profiles, unsigned width, unsigned height, double sx, double sy,
                                     const float *g_conv, const float *g_plain, int levels, bool all_kinds,
                                     const QueueSet &q, double *T, cudaStream_t s, const uint8_t *mask = nullptr);
}  // namespace pf

namespace pf {
// render32.cu: catalogue batches (each entry with its own profiles)
// pad: per profile, the drawing offset (PSF padding) of its bucket
// lum (optional, n * LUM_SLOTS doubles of scratch): the QUADPACK
// luminosities run first, one thread per evaluation (k_cat_lum)
cudaError_t launch_cat_prologue(const ProfileParams *params, const int2 *pad, int n, const ModelGeom &g,
                                double *lum, DevProfile *dev, FProfile *fprof, cudaStream_t s);
cudaError_t launch_cat_gradient(const DevProfile *dev, int n, const double *T, const int *grad_off, double *grad,
                                cudaStream_t s);

// A block of rows of one galaxy's data and sigma, packed in a staging
// buffer (data rows, then sigma rows), to be placed in its canvas slot.
struct CatPiece {
	unsigned long long dst;  // canvas element of the block's first pixel
	unsigned long long src;  // staging element of its first data value
	int w, rows, W;          // block width and rows; canvas row stride
	int pad_;
};
// Writes every piece's data, sigma and region (= 1) into the canvases.
cudaError_t launch_cat_scatter(const CatPiece *pieces, int n_pieces, int max_pixels, const double *stage,
                               double *data, double *sigma, uint8_t *region, cudaStream_t s);
}  // namespace pf

namespace pf {
// render64.cu: the likelihood of kind `kind` (LikeKind: norm, chisq, t, pois)
// for `batch` model images against data with the given batch stride (0:
// one data image); writes logL per image and, with wseed, the adjoint seed.
// partials: batch * nparts * 2 double2; stats: batch * LIKE_SCRATCH_PER_IMAGE doubles.
// tickets (optional, batch zero-initialised words the kernel leaves at zero):
// the norm likelihood then runs as one launch whose last block per image
// merges the partials.
cudaError_t launch_like64(int kind, const double *model, const double *data, const double *sigma,
                          const uint8_t *region, int n, int batch, int data_batch_stride, double2 *partials,
                          int nparts, double *stats, double *out, float *wseed, cudaStream_t s,
                          unsigned *tickets = nullptr);
}  // namespace pf

#include "fitspace.cuh"

namespace pf {
// fitspace.cu: ProFit's fit space for batches, one thread per proposal.
// parm[batch][nfit] -> values[batch][nrefs] and parm_out[batch][nfit]
cudaError_t launch_fit_remake(const FitSpaceView &fs, int batch, const double *parm, double *values, double *parm_out,
                              cudaStream_t s);
// out = [batch] LP, [batch][nfit] d LP / d parm, [batch] LL
cudaError_t launch_fit_finish(const FitSpaceView &fs, int batch, const double *parm, const double *values,
                              const double *ll, const double *grad_ll, double *out, cudaStream_t s);
}  // namespace pf
