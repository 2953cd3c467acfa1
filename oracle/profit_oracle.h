/*
 * ORACLE (test infrastructure only): plain-C restatement of libprofit 1.9.3's
 * model-image path and ProFit's "norm" likelihood.  See profit_oracle.c.
 */
#ifndef PF_ORACLE_H
#define PF_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pfo_model pfo_model;

pfo_model *pfo_model_new(unsigned width, unsigned height);
void pfo_model_free(pfo_model *m);
const char *pfo_last_error(void);

int pfo_add_profile(pfo_model *m, const char *name);
int pfo_profile_set_double(pfo_model *m, int idx, const char *name, double v);
int pfo_profile_set_uint(pfo_model *m, int idx, const char *name, unsigned v);
int pfo_profile_set_bool(pfo_model *m, int idx, const char *name, int v);

int pfo_set_psf(pfo_model *m, const double *psf, unsigned w, unsigned h);
void pfo_set_magzero(pfo_model *m, double mz);
void pfo_set_scale(pfo_model *m, double sx, double sy);
void pfo_set_psf_scale(pfo_model *m, double sx, double sy);
int pfo_set_finesampling(pfo_model *m, unsigned fs);
void pfo_set_return_finesampled(pfo_model *m, int v);
int pfo_set_convolver(pfo_model *m, const char *kind);
void pfo_set_threads(pfo_model *m, int n);

int pfo_drawing_dims(pfo_model *m, unsigned *w, unsigned *h);
int pfo_evaluate(pfo_model *m, double *out, size_t cap, unsigned *w, unsigned *h,
                 int *ox, int *oy);

/* Per-pixel decision log of radial profile idx over the drawing dims of the
 * last evaluation: -1 beyond rscale_max (0 written), 0 evaluated directly,
 * k>0 = number of subsample_pixel calls made for that pixel. */
int pfo_decisions(pfo_model *m, int idx, int *out, size_t cap);
/* Per-level subsample_pixel counts of profile idx (last evaluation). */
int pfo_level_counts(pfo_model *m, int idx, long *out, int max_levels);
/* evaluate_at calls of the last evaluation of profile idx (direct + sub-points) */
long pfo_evaluations(pfo_model *m, int idx);
/* Derived per-profile scalars of the last evaluation (rscale, ie, bn, acc,
 * rscale_switch, rscale_max, resolution, flux_scale, ...). */
int pfo_profile_scalars(pfo_model *m, int idx, double *out, int n);

/* sum over pixels of log dnorm((image - model)/sigma), Neumaier compensated */
double pfo_loglike_norm(const double *image, const double *sigma, const double *model,
                        const unsigned char *region, size_t n);

#ifdef __cplusplus
}
#endif

#endif
