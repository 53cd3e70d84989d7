// Build shim (test infrastructure): linear and bilinear interpolation with
// GSL's documented interface and domain rules, so that the reference's
// src/utils/interp_1d.cc and src/utils/interp_2d.cc link without GSL.
// Written from the definition of the methods, not from GSL's sources.
#include "gsl/gsl_interp.h"
#include "gsl/gsl_interp2d.h"

#include <cstdlib>

namespace {
  gsl_interp_type const linear_type{"linear", 2};
  gsl_interp2d_type const bilinear_type{"bilinear", 2};
  constexpr int kOk = 0;
  constexpr int kDomain = 1;    // GSL_EDOM
  constexpr int kInvalid = 4;   // GSL_EINVAL
}

extern "C" {

const gsl_interp_type* gsl_interp_linear = &linear_type;
const gsl_interp2d_type* gsl_interp2d_bilinear = &bilinear_type;

size_t
gsl_interp_bsearch(const double xa[], double x, size_t lo, size_t hi)
{
  // Largest i in [lo, hi) with xa[i] <= x, for xa[lo] <= x <= xa[hi].
  while (hi > lo + 1) {
    size_t const mid = (lo + hi) / 2;
    if (xa[mid] > x)
      hi = mid;
    else
      lo = mid;
  }
  return lo;
}

gsl_interp*
gsl_interp_alloc(const gsl_interp_type* T, size_t size)
{
  if (size < T->min_size) return nullptr;
  auto* p = static_cast<gsl_interp*>(std::calloc(1, sizeof(gsl_interp)));
  if (p) {
    p->type = T;
    p->size = size;
  }
  return p;
}

int
gsl_interp_init(gsl_interp* interp, const double xa[], const double*,
                size_t size)
{
  for (size_t i = 1; i < size; ++i)
    if (!(xa[i - 1] < xa[i])) return kInvalid;
  interp->xmin = xa[0];
  interp->xmax = xa[size - 1];
  return kOk;
}

int
gsl_interp_eval_e(const gsl_interp* interp, const double xa[],
                  const double ya[], double x, gsl_interp_accel*, double* y)
{
  if (x < interp->xmin || x > interp->xmax) {
    *y = 0.0;
    return kDomain;
  }
  size_t const i = gsl_interp_bsearch(xa, x, 0, interp->size - 1);
  double const dx = xa[i + 1] - xa[i];
  if (!(dx > 0.0)) {
    *y = 0.0;
    return kInvalid;
  }
  *y = ya[i] + (x - xa[i]) / dx * (ya[i + 1] - ya[i]);
  return kOk;
}

void
gsl_interp_free(gsl_interp* interp)
{
  std::free(interp);
}

gsl_interp2d*
gsl_interp2d_alloc(const gsl_interp2d_type* T, size_t xsize, size_t ysize)
{
  if (xsize < T->min_size || ysize < T->min_size) return nullptr;
  auto* p = static_cast<gsl_interp2d*>(std::calloc(1, sizeof(gsl_interp2d)));
  if (p) {
    p->type = T;
    p->xsize = xsize;
    p->ysize = ysize;
  }
  return p;
}

int
gsl_interp2d_init(gsl_interp2d* interp, const double xa[], const double ya[],
                  const double*, size_t xsize, size_t ysize)
{
  for (size_t i = 1; i < xsize; ++i)
    if (!(xa[i - 1] < xa[i])) return kInvalid;
  for (size_t j = 1; j < ysize; ++j)
    if (!(ya[j - 1] < ya[j])) return kInvalid;
  interp->xmin = xa[0];
  interp->xmax = xa[xsize - 1];
  interp->ymin = ya[0];
  interp->ymax = ya[ysize - 1];
  return kOk;
}

int
gsl_interp2d_eval_e(const gsl_interp2d* interp, const double xa[],
                    const double ya[], const double za[], double x, double y,
                    gsl_interp_accel*, gsl_interp_accel*, double* z)
{
  if (x < interp->xmin || x > interp->xmax || y < interp->ymin ||
      y > interp->ymax) {
    *z = 0.0;
    return kDomain;
  }
  size_t const nx = interp->xsize;
  size_t const i = gsl_interp_bsearch(xa, x, 0, nx - 1);
  size_t const j = gsl_interp_bsearch(ya, y, 0, interp->ysize - 1);
  double const t = (x - xa[i]) / (xa[i + 1] - xa[i]);
  double const u = (y - ya[j]) / (ya[j + 1] - ya[j]);
  double const z00 = za[j * nx + i];
  double const z10 = za[j * nx + i + 1];
  double const z01 = za[(j + 1) * nx + i];
  double const z11 = za[(j + 1) * nx + i + 1];
  *z = (1.0 - t) * (1.0 - u) * z00 + t * (1.0 - u) * z10 +
       (1.0 - t) * u * z01 + t * u * z11;
  return kOk;
}

void
gsl_interp2d_free(gsl_interp2d* interp)
{
  std::free(interp);
}

} // extern "C"

// Adaptive quadrature is declared for the reference's adaptive modules only;
// nothing on the fixed-grid path calls it.  These report failure.
#include "gsl/gsl_integration.h"

#include <new>

extern "C" {

gsl_integration_workspace*
gsl_integration_workspace_alloc(size_t n)
{
  auto* w = new (std::nothrow) gsl_integration_workspace;
  if (w) w->limit = n;
  return w;
}

void
gsl_integration_workspace_free(gsl_integration_workspace* w)
{
  delete w;
}

int
gsl_integration_qag(const gsl_function*, double, double, double, double, size_t, int,
                    gsl_integration_workspace*, double* result, double* abserr)
{
  *result = 0.0;
  *abserr = 0.0;
  return 5;  // GSL_EFAILED
}

int
gsl_integration_qagp(const gsl_function*, double*, size_t, double, double, size_t,
                     gsl_integration_workspace*, double* result, double* abserr)
{
  *result = 0.0;
  *abserr = 0.0;
  return 5;  // GSL_EFAILED
}

}  // extern "C"
