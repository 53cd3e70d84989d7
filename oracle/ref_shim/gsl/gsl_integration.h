/* Build shim (test infrastructure): GSL's adaptive 1-D quadrature interface
 * (gsl_integration_qag / qagp) as declared, for the reference's adaptive
 * projection-shear classes that are compiled but never run here.  The
 * implementations in gsl_shim.cc report failure without integrating. */
#ifndef Y3_REF_SHIM_GSL_INTEGRATION_H
#define Y3_REF_SHIM_GSL_INTEGRATION_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double (*function)(double x, void* params);
  void* params;
} gsl_function;

typedef struct gsl_integration_workspace_s {
  size_t limit;
} gsl_integration_workspace;

enum { GSL_INTEG_GAUSS15 = 1, GSL_INTEG_GAUSS21 = 2, GSL_INTEG_GAUSS31 = 3,
       GSL_INTEG_GAUSS41 = 4, GSL_INTEG_GAUSS51 = 5, GSL_INTEG_GAUSS61 = 6 };

gsl_integration_workspace* gsl_integration_workspace_alloc(size_t n);
void gsl_integration_workspace_free(gsl_integration_workspace* w);
int gsl_integration_qag(const gsl_function* f, double a, double b,
                        double epsabs, double epsrel, size_t limit, int key,
                        gsl_integration_workspace* workspace, double* result,
                        double* abserr);
int gsl_integration_qagp(const gsl_function* f, double* pts, size_t npts,
                         double epsabs, double epsrel, size_t limit,
                         gsl_integration_workspace* workspace, double* result,
                         double* abserr);

#ifdef __cplusplus
}
#endif
#endif
