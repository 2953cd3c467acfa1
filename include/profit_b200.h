/*
 * profit_b200: B200-native (sm_100a) model images and likelihoods for the
 * ProFit / libprofit galaxy-profile path, behind a plain C ABI.
 *
 * The entry points mirror libprofit 1.9.3's C++ Model/Profile/Convolver API
 * (src/libprofit/src/profit/model.h, profile.h, convolve.h) and the R glue
 * R_profit_make_model (src/r_profit.cpp:549-680) so that ProFit's
 * profitMakeModel (R/profitMakeModel.R:283) and profitLikeModel
 * (R/profitLikeModel.R:225-379) can call this library instead of libprofit.
 *
 * Conventions
 *  - Every function returns PF_OK (0) or a negative PF_E* status; the message
 *    of the last failure on the calling thread is pf_last_error().  No C++
 *    exception crosses this boundary.
 *  - Images are row-major doubles with x fastest: pixel (x, y) of a W x H
 *    image is at [x + y*W].  This is libprofit's Image layout
 *    (image.h:262-267) and R's column-major matrix with nrow = W
 *    (r_profit.cpp:26-27).
 *  - Host pointers are caller-owned and only read/written during the call.
 *  - A pf_model owns one CUDA stream and its device buffers.  It is not
 *    re-entrant: use one handle per host thread.
 *  - The library needs a CUDA device of compute capability 10.0 (B200).
 *    There is no CPU fallback: without one, pf_model_create fails with
 *    PF_E_CUDA.
 */
#ifndef PROFIT_B200_H
#define PROFIT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  libprofit throws profit::invalid_parameter /
 * unknown_parameter (exceptions.h:41-100); those map to PF_E_INVALID and
 * PF_E_UNKNOWN_PARAM here. */
#define PF_OK 0
#define PF_E_INVALID -1          /* invalid parameter value or model setup */
#define PF_E_UNKNOWN_PARAM -2    /* profile has no parameter of that name/type */
#define PF_E_CUDA -3             /* CUDA runtime error (message has details) */
#define PF_E_CAPACITY -4         /* a device work queue could not grow enough */
#define PF_E_BUFFER -5           /* caller's output buffer too small */
#define PF_E_STATE -6            /* call out of order (e.g. likelihood without data) */

/* Arithmetic of the pixel path.
 *  PF_FP64: the plain form.  Same subsampling decisions as libprofit, pixel
 *           for pixel; images within 1e-12 relative of the reference.
 *  PF_FP32: per-pixel rendering and convolution in FP32; FP64 for the
 *           per-profile scalars (Sersic b_n, normalisation), sub-pixel
 *           coordinates, and the likelihood sum.  Required for gradients. */
#define PF_FP64 0
#define PF_FP32 1
/*  PF_FP32_CONV64: as PF_FP32, but the forward convolution and the model
 *           image the likelihood sees are summed in FP64 (the adjoint stays
 *           FP32).  For bright sources, where the residual data - model is a
 *           small difference of large numbers. */
#define PF_FP32_CONV64 2

typedef struct pf_model pf_model;

/* Last error message of the calling thread ("" if none). */
const char *pf_last_error(void);

/* Library version string, e.g. "profit_b200 0.1 (libprofit 1.9.3 API)". */
const char *pf_version(void);

/* ---- Model life cycle -------------------------------------------------
 * Replaces profit::Model::Model(width, height) (model.h:88-100). */
int pf_model_create(unsigned width, unsigned height, pf_model **out);
int pf_model_destroy(pf_model *m);

/* ---- Profiles ---------------------------------------------------------
 * pf_model_add_profile replaces Model::add_profile (model.cpp:103-135):
 * names "sersic", "moffat", "ferrer"/"ferrers", "coresersic", "king",
 * "brokenexp", "sky", "psf", "null".  *index receives the profile's index.
 * Parameters keep libprofit's names and types (profile.h:150-177):
 *   double: xcen ycen mag ang axrat box acc rscale_switch rscale_max
 *           re nser fwhm con rout a b rb rc rt h1 h2 bg
 *   uint:   resolution max_recursions
 *   bool:   convolve rough adjust force_cpu rescale_flux
 * Setting a name the profile lacks, or with the wrong type, returns
 * PF_E_UNKNOWN_PARAM like Profile::parameter (profile.cpp:81-93). */
int pf_model_add_profile(pf_model *m, const char *name, int *index);
int pf_profile_set_double(pf_model *m, int index, const char *name, double value);
int pf_profile_set_uint(pf_model *m, int index, const char *name, unsigned value);
int pf_profile_set_bool(pf_model *m, int index, const char *name, int value);
/* "name = value", like Profile::parameter(const std::string&) (profile.cpp:136-158). */
int pf_profile_set(pf_model *m, int index, const char *spec);
int pf_profile_get_double(pf_model *m, int index, const char *name, double *value);
int pf_model_profile_count(pf_model *m, int *count);
/* Removes all profiles (R rebuilds the Model on every call; handles can be reused). */
int pf_model_clear_profiles(pf_model *m);

/* ---- Model settings (model.h:142-343) --------------------------------- */
/* PSF is copied and normalised to unit sum, like Model::set_psf (model.h:160-170). */
int pf_model_set_psf(pf_model *m, const double *psf, unsigned width, unsigned height);
int pf_model_set_magzero(pf_model *m, double magzero);
int pf_model_set_image_pixel_scale(pf_model *m, double scale_x, double scale_y);
int pf_model_set_psf_pixel_scale(pf_model *m, double scale_x, double scale_y);
int pf_model_set_finesampling(pf_model *m, unsigned finesampling);
int pf_model_set_return_finesampled(pf_model *m, int value);
/* Calculation mask, like Model::set_mask / set_adjust_mask (model.h:196-214):
 * width x height bytes, nonzero = compute the pixel; NULL clears it.  With
 * adjust_mask (the default) the mask has the model's dimensions and is
 * upsampled, padded and dilated by psf/2 for the drawing, the PSF padding is
 * left out when the mask keeps psf/2 pixels clear of the edges, and the
 * result is zeroed outside the mask (model.cpp:152-183, 230-246, 330-334).
 * Without it the mask must have the drawing dimensions.  Both forms (FP64
 * plain, FP32 with the adjoint gradient). */
int pf_model_set_mask(pf_model *m, const uint8_t *mask, unsigned width, unsigned height);
int pf_model_set_adjust_mask(pf_model *m, int value);
/* Model::set_dimensions (model.h:142-147); a width or height of 0 makes the
 * next evaluation fail with "Model's requested dimensions are 0". */
int pf_model_set_dimensions(pf_model *m, unsigned width, unsigned height);
/* Model::set_dry_run (model.h:293-296): evaluations check their inputs and
 * return a zeroed image of the drawing dimensions (model.cpp:279-286). */
int pf_model_set_dry_run(pf_model *m, int value);
/* Model::set_omp_threads (model.h:333-336): accepted for compatibility; the
 * work runs on the GPU, so the value has no effect. */
int pf_model_set_omp_threads(pf_model *m, unsigned threads);
/* Model::set_crop (model.h:281-283; evaluate, model.cpp:307-322).  With the
 * brute-force ("brute", "brute-old") and null convolvers crop = false returns
 * the same image as crop = true, as libprofit does (those convolvers add no
 * padding of their own).  With the "fft" convolver crop = false, whose result
 * is the convolver's whole 2 max(image, psf) buffer, fails with PF_E_INVALID
 * at evaluation. */
int pf_model_set_crop(pf_model *m, int value);
/* "brute" (default, like Model::ensure_convolver, model.cpp:144-150),
 * "brute-old", "fft" or "null" (create_convolver, convolve.cpp:526-594). */
int pf_model_set_convolver(pf_model *m, const char *type);
/* The convolver choice of profitSetupData with benchmarking
 * (profitDataBenchmark, R/profitSetupData.R:95-110: profitBenchmark, then
 * profitBenchmarkResultBest, R/profitBenchmark.R:16-38): times "brute" and
 * "fft" over nbench evaluations of the model as set up (FP32: logL and its
 * adjoint gradient; FP64: logL; the image when no data are set), keeps the
 * faster one as the model's convolver and writes its name to best (NUL
 * terminated, best_cap bytes).  ms_brute / ms_fft (optional) receive the mean
 * device times in ms (-1 where a convolver does not apply). */
int pf_model_benchmark_convolvers(pf_model *m, int nbench, char *best, size_t best_cap, double *ms_brute,
                                  double *ms_fft);
int pf_model_set_precision(pf_model *m, int precision);

/* Dimensions the profiles are drawn on before convolution and crop
 * (Model::get_drawing_dimensions, model.cpp:152-219). */
int pf_model_drawing_dims(pf_model *m, unsigned *width, unsigned *height);

/* ---- Evaluation ---------------------------------------------------------
 * Replaces Model::evaluate(Image&, Point&) (model.cpp:271-338).  `image`
 * receives the cropped (and, with finesampling and !return_finesampled,
 * downsampled) model of out_w x out_h pixels; `capacity` is its length in
 * doubles.  offset_x/y receive the offset Model::evaluate reports.  Any of
 * the out pointers may be NULL. */
int pf_model_evaluate(pf_model *m, double *image, size_t capacity,
                      unsigned *out_w, unsigned *out_h, int *offset_x, int *offset_y);

/* ---- Likelihood (R/profitLikeModel.R:244-276, like.func = "norm") ------
 * Data image and sigma map of the model's output size; region (optional,
 * 1 = use pixel, like Data$region_which) may be NULL.  Copied to the device
 * once, as profitSetupData prepares Data once per fit. */
int pf_model_set_data(pf_model *m, const double *image, const double *sigma,
                      const uint8_t *region, unsigned width, unsigned height);

/* logL of profitLikeModel for the model's likelihood function
 * (pf_model_set_likelihood; "norm" by default: the sum over the region of
 * log dnorm((image - model)/sigma)). */
int pf_model_loglike(pf_model *m, double *loglike);

/* The likelihood function, profitLikeModel's like.func with the aliases of
 * profitParseLikefunc (R/profitUtility.R:99-121): "norm" (default), "chisq",
 * "t" (dof from the residual variance, R/profitLikeModel.R:281-287), "pois"
 * (R/profitLikeModel.R:321-327).  It applies to pf_model_loglike, the FD
 * gradient, pf_model_loglike_grad and its batch form.  "st" (skew-t, whose
 * parameters profitLikeModel fits with LaplacesDemon) fails with
 * PF_E_INVALID, as does an unknown name. */
int pf_model_set_likelihood(pf_model *m, const char *name);

/* Parameters the gradient is taken with respect to.  Each entry names a
 * profile index and one of its double parameters ("xcen", "ycen", "mag",
 * "ang", "axrat", "box", "re", "nser", "fwhm", "con", ...). */
typedef struct {
	int profile;
	const char *name;
} pf_param_ref;

/* Sets values[i] on every double parameter params[i] in one call, the way a
 * sampler moves to its next proposal (profitRemakeModellist writes the new
 * parameter vector into the model list, R/profitRemakeModelList.R:27-166). */
int pf_model_set_parameters(pf_model *m, const pf_param_ref *params, int n_params,
                            const double *values);

/* logL and d(logL)/d(parameter) for every entry of `params`, by the
 * hand-written adjoint (precision PF_FP32).  The reference has no gradient;
 * this is new.  Subsampling decisions are held fixed, as the derivative of
 * the chosen quadrature. */
int pf_model_loglike_grad(pf_model *m, const pf_param_ref *params, int n_params,
                          double *loglike, double *grad);

/* Batched proposals (new): logL[b] and grad[b][i] = d logL / d params[i] for
 * `batch` proposals, proposal b being this model with params[i] set to
 * values[b * n_params + i].  All proposals share the model's structure, PSF
 * and data (a sampler's population or a batch of MCMC candidates).  The
 * FP64 scalar prologue runs on the device; proposals are processed in chunks
 * that fit a memory budget, each chunk's pipeline replayed from a CUDA graph.
 * A proposal that fails libprofit's parameter validation gets
 * logL = -INFINITY and a zero gradient instead of failing the call.  `grad`
 * may be NULL. */
int pf_model_loglike_grad_batch(pf_model *m, const pf_param_ref *params, int n_params, int batch,
                                const double *values, double *loglike, double *grad);

/* ---- Fit space: LP and d LP / d parm for batches of sampler proposals ----
 * ProFit's samplers move a vector parm of fitted values, which
 * profitRemakeModellist (R/profitRemakeModelList.R:27-166) turns into model
 * parameters, and profitLikeModel returns LP = LL + priors
 * (R/profitLikeModel.R:225-240, 342) with profitMakePriors' normal priors
 * (R/profitUtility.R:124-176).  pf_model_set_fit_space installs that mapping
 * on the model; pf_model_lp_grad_batch then evaluates LP and its gradient with
 * respect to parm for a batch of fitted vectors (new: the reference has no
 * gradient), the mapping and the chain rule running on the device, one thread
 * per proposal (on the host for a few proposals).
 *
 * The n entries are model parameters in unlist(modellist) order:
 *   params[i]   the profile and double parameter the entry sets
 *   init[i]     its value in the model list (model space, not logged)
 *   tofit[i]    1 fitted, 0 fixed at init, -1 takes the value of entry i-1
 *               (R's NA in tofit; not allowed for entry 0)
 *   tolog[i]    (NULL: none) a fitted entry is sampled as log10 of its value
 *   lower/upper (NULL, or NaN entries: no limit) interval limits; an entry
 *               the interval moves gets a zero gradient
 *   offset      (NULL: none) R's offset: xcen += offset[0], ycen +=
 *               offset[1], ang += offset[2] (NaN: none), then re, fwhm, rb,
 *               rout, rc, rt, xcen and ycen *= offset[3] (NaN: none)
 *   prior_sigma (NULL: no priors) sigma of a normal prior per entry, > 0;
 *               +inf is a flat prior (profitMakePriors' allowflat)
 *   prior_mean  (NULL: init) its mean (model space)
 *   prior_tolog (NULL: tolog) the prior is on log10 of the value
 *   prior_on    (NULL: every entry, profitMakePriors without tofit) which
 *               entries carry a prior (pass tofit == 1 for its tofit form)
 * Fixed entries' values (offsets and limits applied) are set on the profiles.
 * Free and tied entries must have an adjoint (pf_model_loglike_grad). */
int pf_model_set_fit_space(pf_model *m, int n, const pf_param_ref *params, const double *init, const int *tofit,
                           const int *tolog, const double *lower, const double *upper, const double *offset,
                           const double *prior_sigma, const double *prior_mean, const int *prior_tolog,
                           const int *prior_on);
/* Number of fitted entries (the length of parm) and of all entries. */
int pf_model_fit_size(pf_model *m, int *n_fit, int *n_entries);
/* For `batch` fitted vectors parm[b * n_fit + j]: lp[b] = LL + log prior,
 * grad[b * n_fit + j] = d LP / d parm_j, parm_out[b * n_fit + j] the vector
 * profitRemakeModellist hands back (limits applied, logged again), loglike[b]
 * = LL.  grad, parm_out and loglike may be NULL.  A proposal whose model
 * parameters fail validation gets lp = loglike = -INFINITY and a zero
 * gradient. */
int pf_model_lp_grad_batch(pf_model *m, int batch, const double *parm, double *lp, double *grad, double *parm_out,
                           double *loglike);

/* How the adjoint of the render is formed.  PF_ADJOINT_STORE keeps, per
 * radial profile, nine FP32 tangent planes of the drawing size from the
 * forward pass (fastest for a few profiles); PF_ADJOINT_RECOMPUTE records
 * only the subsampling decisions and recomputes the tangents against the
 * adjoint seed (no planes: for hundreds of profiles on large fields);
 * PF_ADJOINT_AUTO (default) stores while the planes stay under 256 MB per
 * proposal. */
#define PF_ADJOINT_AUTO 0
#define PF_ADJOINT_STORE 1
#define PF_ADJOINT_RECOMPUTE 2
int pf_model_set_adjoint_mode(pf_model *m, int mode);

/* Same quantities by central finite differences of the plain form (FP64),
 * 2*n_params + 1 evaluations with relative step `rel_step` (absolute step
 * rel_step*max(|p|, 1)); the baseline that pf_model_loglike_grad replaces. */
int pf_model_loglike_grad_fd(pf_model *m, const pf_param_ref *params, int n_params,
                             double rel_step, double *loglike, double *grad);

/* ---- Catalogue batches --------------------------------------------------
 * No counterpart in libprofit: ProFit fits one galaxy at a time, one
 * profitMakeModel / profitLikeModel call per galaxy (R/profitLikeModel.R:
 * 225-379).  A catalogue holds many galaxies, each with its own image size,
 * data, sigma map, PSF and 1+ radial profiles, and evaluates logL and the
 * gradient of every galaxy in one call on the FP32 adjoint path.  Galaxies of
 * a similar size and the same PSF size are batched together on the device.
 *
 * pf_catalogue_add_galaxy: data and sigma are width x height row-major
 * doubles, the PSF psf_w x psf_h (normalised on copy); all pixels count.
 * pf_catalogue_add_profile: a radial profile (sersic, moffat, ferrer,
 * coresersic, king, brokenexp) with n_params "name"/value pairs over
 * libprofit's defaults; convolve defaults to true here.
 * pf_catalogue_loglike_grad: loglike[galaxy]; grad holds, galaxy after
 * galaxy and profile after profile, d logL / d(xcen, ycen, mag, ang, axrat,
 * box, then the kind's shape parameters: sersic re, nser; moffat fwhm, con;
 * ferrer rout, a, b; coresersic re, rb, nser, a, b; king rc, rt, a;
 * brokenexp h1, h2, rb, a).  pf_catalogue_gradient_offset gives a galaxy's
 * slice, pf_catalogue_size the totals. */
typedef struct pf_catalogue pf_catalogue;
int pf_catalogue_create(pf_catalogue **out);
int pf_catalogue_destroy(pf_catalogue *c);
int pf_catalogue_set_magzero(pf_catalogue *c, double magzero);
/* How the batched galaxies are convolved with their PSFs: "auto" (default;
 * each batch times the brute-force kernels against FP64 FFTs of the same
 * geometry, once, at the first evaluation after galaxies are added, and keeps
 * the faster), "brute" or "fft" (batches whose FFT grid would exceed 6912
 * points a side stay brute force).  The FFT form gives the brute-force sums
 * to FP64 transform roundoff.  A batch that convolves through FFTs keeps each
 * of its galaxies' PSF spectra on the device (16 bytes per point of half the
 * FFT grid, about 8 bytes per drawing pixel); batches beyond 16 GB of spectra
 * in all stay brute force.  pf_catalogue_convolvers: how many of the batches
 * convolve through FFTs, of how many (after an evaluation).  No counterpart in
 * libprofit, whose FFTConvolver serves one image (convolve.cpp:245-312). */
int pf_catalogue_set_convolver(pf_catalogue *c, const char *name);
int pf_catalogue_convolvers(const pf_catalogue *c, int *fft_chunks, int *chunks);
int pf_catalogue_add_galaxy(pf_catalogue *c, unsigned width, unsigned height, const double *data,
                            const double *sigma, const double *psf, unsigned psf_w, unsigned psf_h, int *index);
int pf_catalogue_add_profile(pf_catalogue *c, int galaxy, const char *kind, int n_params,
                             const char *const *names, const double *values);
int pf_catalogue_size(pf_catalogue *c, int *n_galaxies, int *n_grad);
int pf_catalogue_gradient_offset(pf_catalogue *c, int galaxy, int *offset, int *count);
int pf_catalogue_loglike_grad(pf_catalogue *c, double *loglike, double *grad);
/* The parameters of every profile in the layout of the gradient (galaxy after
 * galaxy, profile after profile: xcen, ycen, mag, ang, axrat, box, then the
 * kind's shape parameters).  set_values checks every profile first and
 * changes none on error; the next pf_catalogue_loglike_grad uploads the new
 * values and keeps the galaxies' images, batching and recorded launches (a
 * sampler's step over the catalogue). */
int pf_catalogue_set_values(pf_catalogue *c, const double *values);
int pf_catalogue_get_values(pf_catalogue *c, double *values);
/* Device time (ms, CUDA events) of the last pf_catalogue_loglike_grad. */
int pf_catalogue_last_time(pf_catalogue *c, float *ms);

/* ---- Likelihood of device-resident images, allocating nothing ----------
 * No counterpart in libprofit or ProFit: it is the "norm" log-likelihood of
 * profitLikeModel (R/profitLikeModel.R:263-276), the sum pf_model_loglike
 * forms, over images that the caller already keeps on the device.
 *
 * It exists for callers that cannot allocate device memory between
 * evaluations.  A sampler that has reserved nearly all of the GPU's memory
 * for its own pool of proposals would see a cudaMalloc fail; and cudaMalloc
 * and cudaFree can synchronise the whole device, stalling every other stream
 * the caller keeps busy.  So this call allocates nothing, on the device or on
 * the host: its scratch (the per-block partial sums) is a fixed array inside
 * this library, PF_LOGLIKE_NOALLOC_MAX_BATCH x 296 x 16 bytes (296 KiB) per
 * device.
 *
 *   model    device, batch images of npix doubles each, back to back
 *   data     device, npix doubles (the same image for every model)
 *   sigma    device, npix doubles
 *   region   device, npix bytes, nonzero = pixel used; NULL = all pixels
 *   loglike  device, batch doubles, written by the call
 *   stream   a cudaStream_t (NULL = the legacy default stream)
 *
 * The call only queues two kernels on `stream` on the calling thread's
 * current device and returns; read `loglike` after the stream has finished.
 * It forms pf_model_loglike's (PF_FP64) compensated sum over the same grid
 * of blocks for every image size (like_parts(npix, 1): at most 296 blocks,
 * fewer for images under 151,552 pixels) and merges the partials in the same
 * order, so equal images give equal results to the last bit.
 * batch above PF_LOGLIKE_NOALLOC_MAX_BATCH, or npix above
 * 2^31 - 1, fails with PF_E_CAPACITY before anything is queued.
 *
 * The first call in each CUDA context (per device: the primary context, and
 * again after a cudaDeviceReset or with another context current) looks up
 * the scratch array's address with that device current (cudaGetSymbolAddress,
 * which may load this library's device code); make that first call before any
 * stream capture begins.
 * All calls on a device share the one array, which keeps the last call's
 * contents (no call relies on it starting at zero).  Calls whose kernels can
 * run at the same time on the GPU, i.e. on different streams with nothing
 * ordering them, corrupt each other's sums: issue them on one stream, or
 * order the streams with events. */
#define PF_LOGLIKE_NOALLOC_MAX_BATCH 64
int pf_loglike_norm_noalloc(const double *model, const double *data, const double *sigma,
                            const uint8_t *region, size_t npix, int batch, double *loglike,
                            void *stream);

/* ---- Instrumentation ---------------------------------------------------
 * With debug on, evaluations record for each radial profile the number of
 * subsample_pixel calls per drawing pixel (-1 = beyond rscale_max, 0 =
 * evaluated directly) and per recursion level, like libprofit's PROFIT_DEBUG
 * counters (radial.cpp:70-78). */
int pf_model_set_debug(pf_model *m, int value);
int pf_model_decisions(pf_model *m, int profile, int32_t *out, size_t capacity);
int pf_model_level_counts(pf_model *m, int profile, int64_t *out, int max_levels, int *n_levels);
/* Profile evaluations (evaluate_at calls, radial.cpp:54-134,291-344) of the
 * last debug evaluation for one profile: out[0] the pixels evaluated
 * directly, out[1 + L] the sub-point evaluations at recursion level L (two
 * per sub-point where the level may recurse, else one); *total their sum.
 * No counter of its own in libprofit: it is the work count of the render. */
int pf_model_evaluation_counts(pf_model *m, int profile, int64_t *out, int max_levels, int64_t *total);

/* Number of CUDA kernels this library has launched in this process. */
unsigned long long pf_kernel_launches(void);

/* Device time (ms, CUDA events) of the last evaluation's phases:
 * [0] total, [1] render, [2] convolution, [3] likelihood/adjoint.  The FP32
 * likelihood+gradient pipeline replayed from its recorded graph times only
 * the total (events on the stream around the launch); [1]-[3] are NaN
 * there unless phase timing is on. */
int pf_model_last_timings(pf_model *m, float *ms, int n);
/* Phase timing on (nonzero): recorded FP32 pipelines carry the render /
 * convolution / likelihood events as graph nodes, which costs each replay a
 * few microseconds of device time.  Off by default. */
int pf_model_set_phase_timing(pf_model *m, int on);

#ifdef __cplusplus
}
#endif

#endif /* PROFIT_B200_H */
