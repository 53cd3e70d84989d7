/*
 * Build shim (test infrastructure): the part of GSL's 2-D interpolation API
 * that the reference's Interp2D (src/utils/interp_2d.cc:115-135) calls, with
 * the bilinear method only.  z values are stored with x fastest
 * (za[j * xsize + i] belongs to (xa[i], ya[j])), as GSL documents.  An
 * argument outside the grid is a domain error; otherwise the cell is found
 * per axis as in gsl_interp_bsearch and the value is the tensor-product
 * linear blend of the cell's four corners.  Implemented in
 * oracle/ref_shim/gsl_shim.cc.
 */
#ifndef Y3_REF_SHIM_GSL_INTERP2D_H
#define Y3_REF_SHIM_GSL_INTERP2D_H

#include "gsl/gsl_interp.h"

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gsl_interp2d_type_s {
  const char* name;
  unsigned int min_size;
} gsl_interp2d_type;

typedef struct gsl_interp2d_s {
  const gsl_interp2d_type* type;
  double xmin, xmax, ymin, ymax;
  size_t xsize, ysize;
} gsl_interp2d;

extern const gsl_interp2d_type* gsl_interp2d_bilinear;

gsl_interp2d* gsl_interp2d_alloc(const gsl_interp2d_type* T, size_t xsize,
                                 size_t ysize);
int gsl_interp2d_init(gsl_interp2d* interp, const double xa[],
                      const double ya[], const double za[], size_t xsize,
                      size_t ysize);
int gsl_interp2d_eval_e(const gsl_interp2d* interp, const double xa[],
                        const double ya[], const double za[], double x,
                        double y, gsl_interp_accel* xa_acc,
                        gsl_interp_accel* ya_acc, double* z);
void gsl_interp2d_free(gsl_interp2d* interp);

#ifdef __cplusplus
}
#endif

#endif
