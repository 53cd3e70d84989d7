/*
 * Build shim (test infrastructure): the part of GSL's 1-D interpolation API
 * that the reference's Interp1D (src/utils/interp_1d.cc:65-87) calls, with
 * the linear method only.  Semantics restated from GSL's documented
 * behaviour: an argument outside [xa[0], xa[n-1]] is a domain error (non-zero
 * return), otherwise the cell is the last i <= n-2 with xa[i] <= x and the
 * value is the straight line through its two end points.  Implemented in
 * oracle/ref_shim/gsl_shim.cc.
 */
#ifndef Y3_REF_SHIM_GSL_INTERP_H
#define Y3_REF_SHIM_GSL_INTERP_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gsl_interp_type_s {
  const char* name;
  unsigned int min_size;
} gsl_interp_type;

typedef struct gsl_interp_accel_s gsl_interp_accel;

typedef struct gsl_interp_s {
  const gsl_interp_type* type;
  double xmin, xmax;
  size_t size;
} gsl_interp;

extern const gsl_interp_type* gsl_interp_linear;

gsl_interp* gsl_interp_alloc(const gsl_interp_type* T, size_t size);
int gsl_interp_init(gsl_interp* interp, const double xa[], const double ya[],
                    size_t size);
int gsl_interp_eval_e(const gsl_interp* interp, const double xa[],
                      const double ya[], double x, gsl_interp_accel* acc,
                      double* y);
void gsl_interp_free(gsl_interp* interp);
size_t gsl_interp_bsearch(const double xa[], double x, size_t index_lo,
                          size_t index_hi);

#ifdef __cplusplus
}
#endif

#endif
