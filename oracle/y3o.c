/*
 * y3o.c -- FP64 CPU oracle for the cluster-observable hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see y3o.h).  A plain restatement of the
 * reference algorithm; every function cites the reference file:line that
 * defines it.  Nothing here is tuned: clarity over speed.
 */
#include "y3o.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

static const double SQRT2 = 1.41421356237309504880;
static const double SQRT2PI = 2.50662827463100050242;
static const double RHOC = 2.77533742639e+11; /* nfw_dsigma_mis.hh:26 */

/* ------------------------------------------------------------------------ */
/* Gauss-Legendre nodes on [a,b] by Newton iteration on P_N.
 * Restates p_op_detail::gl_nodes, src/models/p_operator_cuhre_t.hh:66-95. */
void
y3o_gl_nodes(double a, double b, int n, double* xs, double* ws)
{
  const double eps = 1e-14;
  const double mid = 0.5 * (a + b);
  const double hlen = 0.5 * (b - a);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = cos(M_PI * ((double)i + 0.75) / ((double)n + 0.5));
    double z1, pp;
    do {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 0; j < n; ++j) {
        double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j + 1.0) * z * p2 - j * p3) / (j + 1.0);
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
    } while (fabs(z - z1) > eps);
    xs[i] = mid - hlen * z;
    xs[n - 1 - i] = mid + hlen * z;
    double w = 2.0 * hlen / ((1.0 - z * z) * pp * pp);
    ws[i] = w;
    ws[n - 1 - i] = w;
  }
}

/* ------------------------------------------------------------------------ */
/* GSL-equivalent interpolation.  The reference wraps GSL's
 * gsl_interp_linear (src/utils/interp_1d.cc:65-87) and gsl_interp2d_bilinear
 * (src/utils/interp_2d.cc:115-135): a binary search for the cell
 * (x_lo <= x < x_hi, the last cell taking x == x_max), then linear /
 * bilinear weights; a query outside [min,max] is a domain error, and
 * clamp() first clamps each coordinate to the axis range
 * (interp_1d.hh:51-54, interp_2d.hh:82-86). */
static int
bsearch_cell(const double* xs, int n, double x)
{
  int ilo = 0, ihi = n - 1;
  while (ihi > ilo + 1) {
    int i = (ihi + ilo) / 2;
    if (xs[i] > x)
      ihi = i;
    else
      ilo = i;
  }
  return ilo;
}

int
y3o_interp1d(const double* xs, const double* ys, int n, double x, double* out)
{
  if (!(x >= xs[0] && x <= xs[n - 1])) {
    *out = NAN;
    return 1;
  }
  int i = bsearch_cell(xs, n, x);
  double dx = xs[i + 1] - xs[i];
  *out = (dx > 0.0) ? ys[i] + (x - xs[i]) / dx * (ys[i + 1] - ys[i]) : 0.0;
  return 0;
}

double
y3o_interp1d_clamp(const double* xs, const double* ys, int n, double x)
{
  double xx = x < xs[0] ? xs[0] : (x > xs[n - 1] ? xs[n - 1] : x);
  double out;
  y3o_interp1d(xs, ys, n, xx, &out);
  return out;
}

/* zs is row-major with y slow: zs[j * nx + i] (GSL's IDX2D convention). */
double
y3o_interp2d(const double* xs, int nx, const double* ys, int ny,
             const double* zs, double x, double y)
{
  int xi = bsearch_cell(xs, nx, x);
  int yi = bsearch_cell(ys, ny, y);
  double xmin = xs[xi], xmax = xs[xi + 1];
  double ymin = ys[yi], ymax = ys[yi + 1];
  double zmm = zs[yi * nx + xi];
  double zMm = zs[yi * nx + xi + 1];
  double zmM = zs[(yi + 1) * nx + xi];
  double zMM = zs[(yi + 1) * nx + xi + 1];
  double t = (x - xmin) / (xmax - xmin);
  double u = (y - ymin) / (ymax - ymin);
  return (1.0 - t) * (1.0 - u) * zmm + t * (1.0 - u) * zMm +
         (1.0 - t) * u * zmM + t * u * zMM;
}

double
y3o_interp2d_clamp(const double* xs, int nx, const double* ys, int ny,
                   const double* zs, double x, double y)
{
  double xx = x < xs[0] ? xs[0] : (x > xs[nx - 1] ? xs[nx - 1] : x);
  double yy = y < ys[0] ? ys[0] : (y > ys[ny - 1] ? ys[ny - 1] : y);
  return y3o_interp2d(xs, nx, ys, ny, zs, xx, yy);
}

/* ------------------------------------------------------------------------ */
/* E(z) for LCDM: src/models/ez.hh:16-27 and ez_sq.hh:10-17. */
double
y3o_ez(double om, double ol, double ok, double z)
{
  double zp1 = 1.0 + z;
  return sqrt(om * zp1 * zp1 * zp1 + ok * zp1 * zp1 + ol);
}

/* dV/dOmega/dz = 2997.92 (1+z)^2 (d_a h)^2 / E(z)  [(Mpc/h)^3], with d_a
 * from an unclamped linear interpolation of distances/{z,d_a} [Mpc]:
 * src/models/dv_do_dz_t.hh:23-31. */
int
y3o_dv_do_dz(const double* dz, const double* da, int nd, double om, double ol,
             double ok, double h, double z, double* out)
{
  double d;
  if (y3o_interp1d(dz, da, nd, z, &d)) return 1;
  *out = 2997.92 * (1.0 + z) * (1.0 + z) * d * h * d * h / y3o_ez(om, ol, ok, z);
  return 0;
}

/* Horner evaluation, highest power first: src/utils/polynomial.hh:16-31. */
static double
poly6(const double* c, double x)
{
  double out = 0.0;
  for (int i = 0; i < 6; ++i) out = c[i] + x * out;
  return out;
}

/* Effective survey area [rad^2]: src/models/omega_z_des.hh:15-33. */
double
y3o_omega_z_des(double zt)
{
  static const double f1[6] = {0.0, 0.0, 0.0, -0.00262353, 0.01940118,
                               0.45133063};
  static const double f2[6] = {1.33647377e+4, 1.35291046e+3, -1.26204891e+2,
                               -2.83454918e+1, -2.26465905, 3.84958753e-1};
  static const double f3[6] = {0, 0, -1.88101967, 4.8071839, -4.11424324,
                               1.18196785};
  if (zt < 0.504) return poly6(f1, zt);
  if (zt < 0.7) return poly6(f2, zt - 0.6);
  return poly6(f3, zt);
}

/* HMF_t::operator(): clamped bilinear n(lnM, z) times the (s, q) nuisance
 * factor, src/models/hmf_t.hh:44-50.  lnm_axis is already
 * ln(m_h (Omega_M - Omega_nu)) (hmf_t.hh:15-25). */
double
y3o_hmf(const double* lnm_axis, int nm, const double* z_axis, int nz,
        const double* dndlnmh, double s, double q, double lnM, double z)
{
  return y3o_interp2d_clamp(lnm_axis, nm, z_axis, nz, dndlnmh, lnM, z) *
         (s * (lnM * 0.4342944819 - 13.8124426028) + q);
}

/* ------------------------------------------------------------------------ */
/* Standard normal CDF, src/models/richness_kernel_t.hh:30-32. */
double
y3o_phi(double x)
{
  return 0.5 * (1.0 + erf(x / SQRT2));
}

/* erfcx(t) = exp(t^2) erfc(t) below 25, asymptotic series above:
 * src/models/richness_kernel_t.hh:37-47. */
double
y3o_erfcx(double t)
{
  if (t < 25.0) return exp(t * t) * erfc(t);
  double inv = 1.0 / t, inv2 = inv * inv;
  return inv / sqrt(M_PI) *
         (1.0 - 0.5 * inv2 * (1.0 - 1.5 * inv2 * (1.0 - 2.5 * inv2)));
}

/* tail(x) = exp(A) Phi(z - tau sigma) in the erfcx form used by
 * sel_function.py:173-187 (_cdf_lob) and richness_kernel_t.hh:56-73. */
double
y3o_emg_tail(double x, double mu, double sigma, double tau)
{
  double z = (x - mu) / sigma;
  double u = (tau * sigma - z) * (1.0 / SQRT2);
  double tail = 0.5 * y3o_erfcx(fabs(u)) * exp(-0.5 * z * z);
  if (u < 0.0) {
    double A = -tau * (x - mu) + 0.5 * (tau * sigma) * (tau * sigma);
    if (A < -700.0) A = -700.0;
    if (A > 700.0) A = 700.0;
    tail = exp(A) - tail;
  }
  return tail;
}

/* Costanzi EMG-mixture CDF, clipped to [0,1]: sel_function.py:153-192. */
double
y3o_cdf_lob(double x, double mu, double sigma, double tau, double fprj)
{
  double z = (x - mu) / sigma;
  double out = y3o_phi(z) - fprj * y3o_emg_tail(x, mu, sigma, tau);
  return out < 0.0 ? 0.0 : (out > 1.0 ? 1.0 : out);
}

/* The density whose CDF is y3o_cdf_lob (before clipping):
 * (1 - f) N(x; mu, sigma) + f tau tail(x), i.e. d/dx of
 * Phi(z) - f tail (sel_function.py:157-161). */
double
y3o_pdf_lob(double x, double mu, double sigma, double tau, double fprj)
{
  double z = (x - mu) / sigma;
  double g = exp(-0.5 * z * z) / (SQRT2PI * sigma);
  return (1.0 - fprj) * g + fprj * tau * y3o_emg_tail(x, mu, sigma, tau);
}

/* K_j(z) = Phi((zmax - z)/s) - Phi((zmin - z)/s): sel_function.py:260-262,
 * richness_kernel_t.hh:120-125. */
double
y3o_kj(double z, double zmin, double zmax, double sigz)
{
  return y3o_phi((zmax - z) / sigz) - y3o_phi((zmin - z) / sigz);
}

/* Linear spline in z with constant extrapolation (scipy
 * InterpolatedUnivariateSpline k=1, ext=3): y3_buzzard/prj_params.py:122-130. */
static double
spline_k1_ext3(const double* zs, const double* v, int n, double z)
{
  return y3o_interp1d_clamp(zs, v, n, z);
}

/* The four EMG parameters at (ltr, z): sel_function.py:99-150.
 * plob_coef holds 8 rows of n_plob values in the order
 * a_tau, b_tau, a_mu, b_mu, a_sig, b_sig, a_fprj, b_fprj (prj_params.py:58-61). */
void
y3o_plob_params(int n_plob, const double* plob_z, const double* plob_coef,
                double ltr, double z, double* mu, double* sigma, double* tau,
                double* fprj)
{
  double c[8];
  for (int k = 0; k < 8; ++k)
    c[k] = spline_k1_ext3(plob_z, plob_coef + k * n_plob, n_plob, z);
  double a_tau = c[0], b_tau = c[1], a_mu = c[2], b_mu = c[3];
  double a_sig = c[4], b_sig = c[5], a_fprj = c[6], b_fprj = c[7];
  *mu = a_mu + b_mu * ltr;
  *sigma = b_sig * pow(ltr, a_sig);
  *tau = b_tau / pow(ltr, a_tau);
  double f = b_fprj / pow(1.0 + exp(-ltr), a_fprj);
  *fprj = f < 1.0 ? f : 1.0;
}

/* ------------------------------------------------------------------------ */
/* HOD shifted-Poisson P(ltr | M, z): sel_function.py:276-343 (mirrors
 * src/models/mor_hod_t.hh:92-116).  hod = {log10_Mmin, log10_M1, alpha,
 * epsilon, sigma_lambda, z_pivot}. */
static double
mu_sat(double M, double z, const double* hod)
{
  double Mmin = pow(10.0, hod[0]), M1 = pow(10.0, hod[1]);
  double dM1 = M1 - Mmin;
  if (dM1 <= 0.0) return 0.0;
  double dM = M - Mmin > 0.0 ? M - Mmin : 0.0;
  double base = dM > 0.0 ? dM / dM1 : 0.0;
  if (!(base > 0.0)) return 0.0;
  return pow(base, hod[2]) * pow((1.0 + z) / (1.0 + hod[5]), hod[3]);
}

double
y3o_p_hod(double ltr, double lnM, double z, const double* hod)
{
  double M = exp(lnM);
  double ms = mu_sat(M, z, hod);
  double lcentral = (M >= pow(10.0, hod[0])) ? 1.0 : 0.0;
  double delta = (hod[4] * ms) * (hod[4] * ms);
  double nu = ms + delta;
  double density;
  if (ms <= 1e-8) {
    double t = (ltr - lcentral) / 1.0e-3;
    density = exp(-0.5 * t * t) / (SQRT2PI * 1.0e-3);
  } else {
    double x = ltr - lcentral + delta;
    if (x > 0.0) {
      double log_nu = log(nu > 1e-300 ? nu : 1e-300);
      density = exp(-nu + (x - 1.0) * log_nu - lgamma(x));
    } else {
      density = 0.0;
    }
  }
  if (ltr < 0.0 || ltr < lcentral) density = 0.0;
  return density;
}

/* Lognormal MOR of the synthetic configs: ln lam ~ N(A + B ln(M/Mpiv) +
 * C ln(1+z), sigma), truncated to [lam_lo, lam_hi] and renormalised by an
 * erf difference (FP64).  Returned as a density in lam. */
static double
phi_diff(double a, double b) /* Phi(b) - Phi(a), b >= a, cancellation-free */
{
  if (a >= 0.0) return 0.5 * (erfc(a / SQRT2) - erfc(b / SQRT2));
  if (b <= 0.0) return 0.5 * (erfc(-b / SQRT2) - erfc(-a / SQRT2));
  return 1.0 - 0.5 * erfc(-a / SQRT2) - 0.5 * erfc(b / SQRT2);
}

/* ln(Phi(b) - Phi(a)) where the difference itself underflows (mu about 38
 * sigma or more outside [lam_lo, lam_hi]; the direct quotient is then 0/0):
 * with Q(x) = erfc(x / sqrt 2) / 2 = erfcx(x / sqrt 2) exp(-x^2 / 2) / 2,
 * ln(Q(a) - Q(b)) = ln Q(a) + log1p(-Q(b) / Q(a)) for 0 < a < b, and the
 * mirror image for a < b < 0. */
static double
ln_phi_diff(double a, double b)
{
  if (a > 0.0) {
    double ra = y3o_erfcx(a / SQRT2), rb = y3o_erfcx(b / SQRT2);
    return log(0.5 * ra) - 0.5 * a * a + log1p(-(rb / ra) * exp(-0.5 * (b - a) * (b + a)));
  }
  if (b < 0.0) {
    double ra = y3o_erfcx(-a / SQRT2), rb = y3o_erfcx(-b / SQRT2);
    return log(0.5 * rb) - 0.5 * b * b + log1p(-(ra / rb) * exp(-0.5 * (a - b) * (a + b)));
  }
  return log(phi_diff(a, b));
}

static double
lognormal_mu(const double* mor, double lnM, double z)
{
  return mor[0] + mor[1] * (lnM - log(mor[4])) + mor[2] * log1p(z);
}

/* ------------------------------------------------------------------------ */
/* S_stack producer, sel_function.py:516-615 (execute), with the per-cell
 * lambda_t bracket of _compute_lam_nodes_and_P_HOD (516-547, L = 6) and the
 * closed-form K_i by CDF differencing at the unique edges (195-226, 592-600).
 *
 * mor_kind HOD: mor = {log10_Mmin, log10_M1, alpha, epsilon, sigma_lambda,
 * z_pivot} exactly as the reference.  mor_kind LOGNORMAL: mor = {A, B, C,
 * sigma, Mpiv, lam_lo, lam_hi}; the bracket is [exp(mu - 6 sigma),
 * exp(mu + 6 sigma)] intersected with [lam_lo, lam_hi] -- the swap-in for
 * the synthetic configs, used identically by the fixture generator. */
int
y3o_sel_function(int n_bins, const double* lam_min, const double* lam_max,
                 const double* zob_min, const double* zob_max,
                 const double* sigma_z, double zt_low, double zt_high,
                 double lnm_low, double lnm_high, int n_lnm, int n_z, int n_q,
                 int mor_kind, const double* mor, int n_plob,
                 const double* plob_z, const double* plob_coef,
                 double* lnm_out, double* z_out, double* S_out)
{
  const double L = 6.0;
  /* unique sorted edges (np.unique(concat(lam_min, lam_max))) */
  double* edges = (double*)malloc(sizeof(double) * 2 * n_bins);
  int ne = 0;
  for (int k = 0; k < 2 * n_bins; ++k) {
    double v = k < n_bins ? lam_min[k] : lam_max[k - n_bins];
    int dup = 0;
    for (int e = 0; e < ne; ++e)
      if (edges[e] == v) dup = 1;
    if (!dup) edges[ne++] = v;
  }
  for (int a = 0; a < ne; ++a) /* insertion sort */
    for (int b = a + 1; b < ne; ++b)
      if (edges[b] < edges[a]) {
        double t = edges[a];
        edges[a] = edges[b];
        edges[b] = t;
      }
  int* lo_i = (int*)malloc(sizeof(int) * n_bins);
  int* hi_i = (int*)malloc(sizeof(int) * n_bins);
  for (int k = 0; k < n_bins; ++k) {
    for (int e = 0; e < ne; ++e) {
      if (edges[e] == lam_min[k]) lo_i[k] = e;
      if (edges[e] == lam_max[k]) hi_i[k] = e;
    }
  }
  /* linear shared grids (np.linspace) */
  for (int m = 0; m < n_lnm; ++m)
    lnm_out[m] = n_lnm > 1 ? lnm_low + (lnm_high - lnm_low) * m / (n_lnm - 1)
                           : lnm_low;
  for (int j = 0; j < n_z; ++j)
    z_out[j] = n_z > 1 ? zt_low + (zt_high - zt_low) * j / (n_z - 1) : zt_low;

  double* gt = (double*)malloc(sizeof(double) * n_q);
  double* gw = (double*)malloc(sizeof(double) * n_q);
  y3o_gl_nodes(-1.0, 1.0, n_q, gt, gw);
  double* cdf = (double*)malloc(sizeof(double) * ne);
  double* Spair = (double*)malloc(sizeof(double) * n_bins);

  for (int m = 0; m < n_lnm; ++m) {
    double lnM = lnm_out[m];
    double M = exp(lnM);
    for (int j = 0; j < n_z; ++j) {
      double z = z_out[j];
      double a, b, mu_ln = 0.0, D = 1.0;
      if (mor_kind == Y3O_MOR_HOD) {
        double ms = mu_sat(M, z, mor);
        double lcentral = (M >= pow(10.0, mor[0])) ? 1.0 : 0.0;
        double mu_eff = lcentral + ms;
        double v = ms + (mor[4] * ms) * (mor[4] * ms);
        double sig_eff = sqrt(v > 0.0 ? v : 0.0);
        a = mu_eff - L * sig_eff;
        if (a < 0.0) a = 0.0;
        b = mu_eff + L * sig_eff;
      } else {
        mu_ln = lognormal_mu(mor, lnM, z);
        a = exp(mu_ln - L * mor[3]);
        b = exp(mu_ln + L * mor[3]);
        if (a < mor[5]) a = mor[5];
        if (b > mor[6]) b = mor[6];
        D = phi_diff((log(mor[5]) - mu_ln) / mor[3],
                     (log(mor[6]) - mu_ln) / mor[3]);
      }
      int degenerate = !(b > a);
      double half = 0.5 * (b - a), mid = 0.5 * (a + b);
      for (int k = 0; k < n_bins; ++k) Spair[k] = 0.0;
      for (int t = 0; t < n_q; ++t) {
        double ltr = mid + half * gt[t];
        double W = half * gw[t];
        double P;
        if (mor_kind == Y3O_MOR_HOD) {
          P = y3o_p_hod(ltr, lnM, z, mor);
        } else {
          double d = (log(ltr) - mu_ln) / mor[3];
          P = exp(-0.5 * d * d) / (SQRT2PI * mor[3] * ltr * D);
        }
        double mu, sg, tau, fp;
        y3o_plob_params(n_plob, plob_z, plob_coef, ltr, z, &mu, &sg, &tau, &fp);
        for (int e = 0; e < ne; ++e) cdf[e] = y3o_cdf_lob(edges[e], mu, sg, tau, fp);
        for (int k = 0; k < n_bins; ++k)
          Spair[k] += W * (cdf[hi_i[k]] - cdf[lo_i[k]]) * P;
      }
      for (int k = 0; k < n_bins; ++k) {
        double Si = degenerate ? 0.0 : Spair[k];
        double Kj = y3o_kj(z, zob_min[k], zob_max[k], sigma_z[k]);
        S_out[((size_t)k * n_z + j) * n_lnm + m] = Si * Kj;
      }
    }
  }
  free(edges);
  free(lo_i);
  free(hi_i);
  free(gt);
  free(gw);
  free(cdf);
  free(Spair);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* SelGLCore::build_weights, src/models/n_operator_sel_gl_t.hh:91-143, with
 * SelFunction_t (sel_function_t.hh:29-82: a bin's (n_z, n_lnm) plane,
 * bilinear, zero outside the tabulated box), HMF_t, DV_DO_DZ_t and
 * OMEGA_Z_DES.  If n_sci > 0 the z-factor includes the clamped
 * Sigma_crit^-1 (lensing_weights.hh:54-59), as Shear1hMisSelGL does.
 * Returns 1 if d_a is queried outside its table (the reference throws). */
int
y3o_selgl_weights(int n_lnm, int n_z, double zt_lo, double zt_hi,
                  double lnm_lo, double lnm_hi, const y3o_cosmo* c, int n_hm,
                  const double* hmf_m_h, int n_hz, const double* hmf_z,
                  const double* dndlnmh, int nd, const double* dist_z,
                  const double* dist_da, int n_sci, const double* sci_z,
                  const double* sci_val, int n_bins, int n_sel_lnm,
                  const double* sel_lnm, int n_sel_z, const double* sel_z,
                  const double* S_stack, double* W_out, double* norm_out,
                  double* lnm_eff_out, double* mu2_out)
{
  double* xm = (double*)malloc(sizeof(double) * n_lnm);
  double* wm = (double*)malloc(sizeof(double) * n_lnm);
  double* xz = (double*)malloc(sizeof(double) * n_z);
  double* wz = (double*)malloc(sizeof(double) * n_z);
  double* zfac = (double*)malloc(sizeof(double) * n_z);
  double* hax = (double*)malloc(sizeof(double) * n_hm);
  y3o_gl_nodes(lnm_lo, lnm_hi, n_lnm, xm, wm);
  y3o_gl_nodes(zt_lo, zt_hi, n_z, xz, wz);
  for (int i = 0; i < n_hm; ++i) hax[i] = log(hmf_m_h[i] * (c->om - c->onu));
  int rc = 0;
  for (int q = 0; q < n_z; ++q) {
    double dv;
    if (y3o_dv_do_dz(dist_z, dist_da, nd, c->om, c->ol, c->ok, c->h0, xz[q], &dv)) {
      rc = 1;
      dv = NAN;
    }
    double sci = n_sci > 0 ? y3o_interp1d_clamp(sci_z, sci_val, n_sci, xz[q]) : 1.0;
    zfac[q] = wz[q] * dv * y3o_omega_z_des(xz[q]) * sci;
  }
  double slo = sel_lnm[0], shi = sel_lnm[0], zlo = sel_z[0], zhi = sel_z[0];
  for (int i = 0; i < n_sel_lnm; ++i) {
    if (sel_lnm[i] < slo) slo = sel_lnm[i];
    if (sel_lnm[i] > shi) shi = sel_lnm[i];
  }
  for (int i = 0; i < n_sel_z; ++i) {
    if (sel_z[i] < zlo) zlo = sel_z[i];
    if (sel_z[i] > zhi) zhi = sel_z[i];
  }
  for (int b = 0; b < n_bins; ++b) {
    const double* plane = S_stack + (size_t)b * n_sel_z * n_sel_lnm;
    double* Wb = W_out + (size_t)b * n_lnm;
    for (int k = 0; k < n_lnm; ++k) {
      double lnM = xm[k];
      double acc = 0.0;
      for (int q = 0; q < n_z; ++q) {
        double z = xz[q];
        double h = y3o_hmf(hax, n_hm, hmf_z, n_hz, dndlnmh, c->hmf_s, c->hmf_q, lnM, z);
        double s = (lnM < slo || lnM > shi || z < zlo || z > zhi)
                     ? 0.0
                     : y3o_interp2d_clamp(sel_lnm, n_sel_lnm, sel_z, n_sel_z, plane, lnM, z);
        acc += zfac[q] * h * s;
      }
      Wb[k] = acc;
    }
    double n0 = 0.0, n1 = 0.0;
    for (int k = 0; k < n_lnm; ++k) {
      n0 += wm[k] * Wb[k];
      n1 += wm[k] * Wb[k] * xm[k];
    }
    norm_out[b] = n0;
    double eff = (n0 != 0.0) ? n1 / n0 : 0.5 * (lnm_lo + lnm_hi);
    if (lnm_eff_out) lnm_eff_out[b] = eff;
    double m2 = 0.0;
    for (int k = 0; k < n_lnm; ++k) {
      double d = xm[k] - eff;
      m2 += wm[k] * Wb[k] * d * d;
    }
    if (mu2_out) mu2_out[b] = (n0 != 0.0) ? m2 / n0 : 0.0;
  }
  free(xm);
  free(wm);
  free(xz);
  free(wz);
  free(zfac);
  free(hax);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* Projected NFW profile in units of 2 r_s delta_c rho (Wright & Brainerd
 * 2000; the reference's closed form is src/models/nfw_sigma_t.hh:34-43 and
 * its miscentred tables are normalised the same way, nfw_dsigma_mis.hh:95-114).
 *   Sigma(x)     = (g(x) - 1) / (1 - x^2),
 *   Sigma_bar(x) = 2 (g(x) + ln(x/2)) / x^2,
 *   g(x) = artanh(y)/y, y = sqrt(1 - x^2) (x < 1);  arctan(y)/y,
 *          y = sqrt(x^2 - 1) (x > 1);  = sum_n w^n/(2n+1), w = 1 - x^2.
 * Near x = 1 the power series in w is used; for small x Sigma_bar is
 * rewritten so that no O(1) terms cancel. */
static double
nfw_g(double x)
{
  double w = 1.0 - x * x;
  if (fabs(w) < 0.1) {
    double s = 0.0, p = 1.0;
    for (int n = 0; n < 40; ++n) {
      s += p / (2 * n + 1);
      p *= w;
    }
    return s;
  }
  if (x < 1.0) {
    double y = sqrt(w);
    return atanh(y) / y;
  }
  double y = sqrt(-w);
  return atan(y) / y;
}

double
y3o_nfw_sigma_unit(double x)
{
  double w = 1.0 - x * x;
  if (fabs(w) < 0.1) { /* (g - 1)/w = sum_n w^n/(2n+3) */
    double s = 0.0, p = 1.0;
    for (int n = 0; n < 40; ++n) {
      s += p / (2 * n + 3);
      p *= w;
    }
    return s;
  }
  return (nfw_g(x) - 1.0) / w;
}

static double
nfw_sigma_bar_unit(double x)
{
  if (x < 0.5) {
    /* g - L with L = ln(2/x): arccosh(1/x) = L + ln((1+y)/2),
     * ln((1+y)/2) = log1p(-x^2 / (2 (1+y))), so
     * Sigma_bar = (2/y) [L/(1+y) + log1p(-x^2/(2(1+y)))/x^2]. */
    double y = sqrt(1.0 - x * x);
    double L = log(2.0 / x);
    double x2 = x * x;
    return (2.0 / y) * (L / (1.0 + y) + log1p(-x2 / (2.0 * (1.0 + y))) / x2);
  }
  return 2.0 * (nfw_g(x) + log(0.5 * x)) / (x * x);
}

double
y3o_nfw_dsigma_unit(double x)
{
  return nfw_sigma_bar_unit(x) - y3o_nfw_sigma_unit(x);
}

/* r_s = r_200 / c with r_200 = cbrt(3 M / (800 pi rho)); nfw_dsigma_mis.hh:88-93. */
double
y3o_nfw_rs(double lnM, double c, double rho)
{
  return cbrt(3.0 * exp(lnM) / (800.0 * M_PI * rho)) / c;
}

/* 2 r_s delta_c rho * 1e-12  [h Msun / pc^2]; nfw_dsigma_mis.hh:98-113. */
double
y3o_nfw_norm(double lnM, double c, double rho)
{
  double delta_c = (200.0 * c * c * c / 3.0) / (log(1.0 + c) - c / (1.0 + c));
  return 2.0 * y3o_nfw_rs(lnM, c, rho) * delta_c * rho * 1e-12;
}

/* Gamma miscentring kernel P(x) = x/tau^2 exp(-x/tau): roffset_t.hh:18-23. */
double
y3o_roffset(double x, double tau)
{
  return x / tau / tau * exp(-x / tau);
}

/* Miscentred profiles in x = R/r_s units for the gamma kernel with scale
 * xmis (lensing_weights.hh:130-153; cluster_toolkit's kernel='gamma'):
 *   Sigma_mis(x)  = int_0^inf ds s e^-s (1/pi) int_0^pi dth Sigma(d),
 *   DSigma_mis(x) = int_0^inf ds s e^-s (1/pi) int_0^pi dth DSigma(d) cos 2phi,
 * with offset r = xmis s, d^2 = x^2 + r^2 - 2 x r cos th and
 * cos 2phi = 2 (x - r cos th)^2 / d^2 - 1.  The second line is the
 * tangential-shear form of Sigma_bar(<x) - Sigma(x) of the offset profile
 * (the mean tangential shear on a circle equals the mean enclosed minus
 * the mean boundary surface density for any mass distribution), so no
 * inner radial integral is needed.  Gauss-Legendre in th on [0, pi]; in s
 * the integrand has a kink where the offset ring crosses the aperture
 * (s_k = x / xmis), so the s nodes are two Gauss-Legendre panels
 * [0, s_k] and [s_k, s_max] of n_s/2 and n_s - n_s/2 nodes (one panel on
 * [0, s_max] when s_k >= s_max). */
void
y3o_mis_s_nodes(double x, double xmis, int n_s, double s_max, double* sn,
                double* wsn)
{
  double sk = x / xmis;
  if (sk < s_max && n_s >= 2) {
    int n1 = n_s / 2;
    y3o_gl_nodes(0.0, sk, n1, sn, wsn);
    y3o_gl_nodes(sk, s_max, n_s - n1, sn + n1, wsn + n1);
  } else {
    y3o_gl_nodes(0.0, s_max, n_s, sn, wsn);
  }
}

static double
mis_integral(double x, double xmis, int n_theta, int n_s, double s_max,
             int want_delta)
{
  double* th = (double*)malloc(sizeof(double) * n_theta);
  double* wth = (double*)malloc(sizeof(double) * n_theta);
  double* sn = (double*)malloc(sizeof(double) * n_s);
  double* wsn = (double*)malloc(sizeof(double) * n_s);
  y3o_gl_nodes(0.0, M_PI, n_theta, th, wth);
  y3o_mis_s_nodes(x, xmis, n_s, s_max, sn, wsn);
  double acc = 0.0;
  for (int n = 0; n < n_s; ++n) {
    double r = xmis * sn[n];
    double inner = 0.0;
    for (int t = 0; t < n_theta; ++t) {
      double ct = cos(th[t]);
      double d2 = x * x + r * r - 2.0 * x * r * ct;
      double d = sqrt(d2);
      double v;
      if (want_delta) {
        double a = x - r * ct;
        v = y3o_nfw_dsigma_unit(d) * (2.0 * a * a / d2 - 1.0);
      } else {
        v = y3o_nfw_sigma_unit(d);
      }
      inner += wth[t] * v;
    }
    acc += wsn[n] * sn[n] * exp(-sn[n]) * inner / M_PI;
  }
  free(th);
  free(wth);
  free(sn);
  free(wsn);
  return acc;
}

double
y3o_dsigma_mis_unit(double x, double xmis, int n_theta, int n_s, double s_max)
{
  return mis_integral(x, xmis, n_theta, n_s, s_max, 1);
}

double
y3o_sigma_mis_unit(double x, double xmis, int n_theta, int n_s, double s_max)
{
  return mis_integral(x, xmis, n_theta, n_s, s_max, 0);
}

/* ------------------------------------------------------------------------ */
/* Shear1hMisSelGL::evaluate ("exact" method), n_operator_sel_gl_t.hh:293-349:
 *   out[b, R] = sum_k w_k W_b[k] phi(b, R, lnM_k),
 *   phi = (1 - f) dSigma_nfw.clamp(R, lnM) + f NFW_DSIGMA_MIS(R, r_mis_b, lnM),
 * r_mis_b = tau R_lambda(lob_centers[b % n_lob]) (269-291,
 * lensing_weights.hh:167-198), NFW_DSIGMA_MIS with concentration conc.  The
 * module constructs that class with rho_c = RHOC and then calls
 * set_rho_mult(Omega_M) (n_operator_sel_gl_t.hh:248,264), so r_s comes from
 * rho_c alone while the amplitude 2 r_s delta_c rho_c rho_mult carries Omega_M
 * (nfw_dsigma_mis.hh:95-114).  The miscentred profile comes from
 * y3o_dsigma_mis_unit (the reference reads the same quantity from a table
 * that is not in the snapshot).
 * dsig_tab is the haloModel/dSigma_nfw ndarray, extents (n_ml, n_rs). */
int
y3o_shear1h_mis(int n_lnm, const double* lnm_x, const double* lnm_w,
                int n_bins, const double* W_gamma, int n_R, const double* R,
                double f_mis, double tau_mis, int n_lob,
                const double* lob_centers, double omega_m, double conc,
                int n_rs, const double* r_sigma, int n_ml,
                const double* lnM_tab, const double* dsig_tab, int n_theta,
                int n_s, double s_max, double* out)
{
  for (int b = 0; b < n_bins; ++b) {
    double rmis = tau_mis * pow(lob_centers[b % n_lob] / 100.0, 0.2);
    for (int r = 0; r < n_R; ++r) {
      double acc = 0.0;
      for (int k = 0; k < n_lnm; ++k) {
        double lnM = lnm_x[k];
        double rs = y3o_nfw_rs(lnM, conc, RHOC);
        double cen = y3o_interp2d_clamp(r_sigma, n_rs, lnM_tab, n_ml, dsig_tab, R[r], lnM);
        double mis = y3o_nfw_norm(lnM, conc, RHOC) * omega_m *
                     y3o_dsigma_mis_unit(R[r] / rs, rmis / rs, n_theta, n_s, s_max);
        double phi = (1.0 - f_mis) * cen + f_mis * mis;
        acc += lnm_w[k] * W_gamma[(size_t)b * n_lnm + k] * phi;
      }
      out[(size_t)b * n_R + r] = acc;
    }
  }
  return 0;
}

/* NFW_DSIGMA_MIS::operator() as the reference evaluates it
 * (nfw_dsigma_mis.hh:95-114): the unit miscentred profile is read from the
 * table log_tab[j * n_lx + i] on the axes (logx[i], logxmis[j]) (the files
 * nfw_off_center/table_1000_1e-03_5e+03_{gamma_logx, gamma_logxmis,
 * log_deltasigma_gamma}.txt, x fastest) by clamped bilinear interpolation
 * at (ln x, ln x_mis), x = r / r_s with r_s from rho_c, then scaled by
 * 2 r_s delta_c rho_c rho_mult * 1e-12. */
double
y3o_dsigma_mis_tab(double r, double rmis, double lnM, double conc, double rhoc,
                   double rho_mult, int n_lx, const double* logx, int n_lxm,
                   const double* logxmis, const double* log_tab)
{
  double rs = y3o_nfw_rs(lnM, conc, rhoc);
  double v = y3o_interp2d_clamp(logx, n_lx, logxmis, n_lxm, log_tab, log(r / rs),
                                log(rmis / rs));
  return y3o_nfw_norm(lnM, conc, rhoc) * rho_mult * exp(v);
}

/* Shear1hMisSelGL::evaluate with the tabulated miscentred profile, both
 * methods (n_operator_sel_gl_t.hh:293-319):
 *   exact (method 0): sum_k w_k W_b[k] phi(b, R, lnM_k);
 *   idea2 (method 1): norm_b [phi(y0) + mu2_b/2 (phi(y0+h) - 2 phi(y0)
 *                     + phi(y0-h)) / h^2] at y0 = lnm_eff_b. */
int
y3o_shear1h_mis_tab(int n_lnm, const double* lnm_x, const double* lnm_w,
                    int n_bins, const double* W_gamma, const double* norm,
                    const double* lnm_eff, const double* mu2, int method,
                    double stencil_h, int n_R, const double* R, double f_mis,
                    double tau_mis, int n_lob, const double* lob_centers,
                    double omega_m, double conc, int n_rs, const double* r_sigma,
                    int n_ml, const double* lnM_tab, const double* dsig_tab,
                    int n_lx, const double* logx, int n_lxm,
                    const double* logxmis, const double* log_tab, double* out)
{
#define Y3O_PHI(LNM)                                                            \
  ((1.0 - f_mis) * y3o_interp2d_clamp(r_sigma, n_rs, lnM_tab, n_ml, dsig_tab,  \
                                      R[r], (LNM)) +                            \
   f_mis * y3o_dsigma_mis_tab(R[r], rmis, (LNM), conc, RHOC, omega_m, n_lx,     \
                              logx, n_lxm, logxmis, log_tab))
  for (int b = 0; b < n_bins; ++b) {
    double rmis = tau_mis * pow(lob_centers[b % n_lob] / 100.0, 0.2);
    for (int r = 0; r < n_R; ++r) {
      double v;
      if (method == 0) {
        v = 0.0;
        for (int k = 0; k < n_lnm; ++k)
          v += lnm_w[k] * W_gamma[(size_t)b * n_lnm + k] * Y3O_PHI(lnm_x[k]);
      } else {
        double h = stencil_h, y0 = lnm_eff[b];
        double c = Y3O_PHI(y0), p = Y3O_PHI(y0 + h), m = Y3O_PHI(y0 - h);
        double d2 = (p - 2.0 * c + m) / (h * h);
        v = norm[b] * (c + 0.5 * mu2[b] * d2);
      }
      out[(size_t)b * n_R + r] = v;
    }
  }
#undef Y3O_PHI
  return 0;
}

/* ------------------------------------------------------------------------ */
/* <Sigma_crit^-1>(z_l) = h0 * trapz_zs max(0, p(zs + dz) 4 pi G/c^2
 * D_l D_ls / D_s), D_ls = D_s - (1+z_l)/(1+z_s) D_l, D from a linear
 * interpolation of distances/d_a [Mpc]:
 * src/modules/average_sigma_crit_inv/average_sigma_crit_inv.py:40-58. */
int
y3o_sigma_crit_inv(int n_zl, const double* zl, int n_zs, const double* zs,
                   const double* pz, double delta_z, double h0, int nd,
                   const double* dist_z, const double* dist_da, double* out)
{
  const double G = 4.51710305e-48, cl = 9.71561189e-15;
  const double k = 4.0 * M_PI * G / cl / cl;
  double* f = (double*)malloc(sizeof(double) * n_zs);
  int rc = 0;
  for (int j = 0; j < n_zl; ++j) {
    double dl;
    if (y3o_interp1d(dist_z, dist_da, nd, zl[j], &dl)) rc = 1;
    for (int i = 0; i < n_zs; ++i) {
      double ds, p;
      if (y3o_interp1d(dist_z, dist_da, nd, zs[i], &ds)) rc = 1;
      if (y3o_interp1d(zs, pz, n_zs, zs[i] + delta_z, &p)) rc = 1;
      double dls = ds - (1.0 + zl[j]) / (1.0 + zs[i]) * dl;
      double v = ds > 0.0 ? p * k * dl * dls / ds : 0.0;
      f[i] = v > 0.0 ? v : 0.0;
    }
    double acc = 0.0;
    for (int i = 0; i + 1 < n_zs; ++i)
      acc += 0.5 * (f[i] + f[i + 1]) * (zs[i + 1] - zs[i]);
    out[j] = acc * h0;
  }
  free(f);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* Direct nested Gauss-Legendre quadrature of
 *   N_ij = int dz_t dV/dz Omega(z) int dlnM n(M,z) int dlam_t P(lam_t|M,z)
 *          int_{bin i} dlam_o P(lam_o|lam_t,z) int_{bin j} dz_o P(z_o|z_t)
 * on fixed nodes (lnM, z_t, ln lam_t, lam_o per richness bin, z_o per z
 * bin), contracted in the order lam_o -> lam_t -> (z_t, lnM) of
 * SelGLCore (n_operator_sel_gl_t.hh:91-143):
 *   K_i(t,q)  = sum_o a_o P(lam_o | lam_t, z_q)          (pdf of sel_function.py:153-192)
 *   K_j(q)    = sum_zo b N(z_o; z_q, sz0 (1+z_q) + sz_bin[j])
 *               (sz_bin[j] alone is sel_function.py's constant sigma_z of
 *               the z bin, _K_j at sel_function.py:260-262)
 *   S_i(k,q)  = sum_t u_t K_i(t,q) phi((l_t - mu_kq)/s) / (s D_kq)
 *   W_ij(k)   = sum_q v_q dV(z_q) Omega(z_q) [Sci(z_q)] K_j(q) n(M_k,z_q) S_i(k,q)
 *   N_ij      = sum_k w_k W_ij(k),   N_ij(R) = sum_k w_k W^gamma_ij(k) Phi_i(R,k)
 * Bins are richness-fast (b = i + n_lam_bins * j).  W_out (optional) gets
 * the counts weights [b][k]. */
int
y3o_direct_eval(const y3o_direct_grid* g, int n_plob, const double* plob_z,
                const double* plob_coef, const y3o_lognormal* mor,
                const y3o_cosmo* c, int n_hm, const double* hmf_m_h, int n_hz,
                const double* hmf_z, const double* dndlnmh, int nd,
                const double* dist_z, const double* dist_da,
                const y3o_shear_opts* shear, double* counts_out, double* W_out,
                double* shear_out)
{
  int nI = g->n_lam_bins, nJ = g->n_z_bins, nB = nI * nJ;
  int nm = g->n_m, nz = g->n_z, nt = g->n_t;
  double *xm = malloc(sizeof(double) * nm), *wm = malloc(sizeof(double) * nm);
  double *xz = malloc(sizeof(double) * nz), *wz = malloc(sizeof(double) * nz);
  double *xl = malloc(sizeof(double) * nt), *wl = malloc(sizeof(double) * nt);
  y3o_gl_nodes(g->lnm_lo, g->lnm_hi, nm, xm, wm);
  y3o_gl_nodes(g->zt_lo, g->zt_hi, nz, xz, wz);
  double ll_lo = log(g->lam_t_lo), ll_hi = log(g->lam_t_hi);
  y3o_gl_nodes(ll_lo, ll_hi, nt, xl, wl);
  double* lo_x = malloc(sizeof(double) * g->n_o * nI);
  double* lo_w = malloc(sizeof(double) * g->n_o * nI);
  for (int i = 0; i < nI; ++i)
    y3o_gl_nodes(g->lam_edges[i], g->lam_edges[i + 1], g->n_o, lo_x + i * g->n_o,
                 lo_w + i * g->n_o);
  double* zo_x = malloc(sizeof(double) * g->n_zo * nJ);
  double* zo_w = malloc(sizeof(double) * g->n_zo * nJ);
  for (int j = 0; j < nJ; ++j)
    y3o_gl_nodes(g->zob_edges[j], g->zob_edges[j + 1], g->n_zo, zo_x + j * g->n_zo,
                 zo_w + j * g->n_zo);

  /* K_i(t, q) */
  double* Ki = malloc(sizeof(double) * nI * nt * nz);
  for (int q = 0; q < nz; ++q)
    for (int t = 0; t < nt; ++t) {
      double lam = exp(xl[t]);
      double mu, sg, tau, fp;
      y3o_plob_params(n_plob, plob_z, plob_coef, lam, xz[q], &mu, &sg, &tau, &fp);
      for (int i = 0; i < nI; ++i) {
        double acc = 0.0;
        for (int o = 0; o < g->n_o; ++o)
          acc += lo_w[i * g->n_o + o] * y3o_pdf_lob(lo_x[i * g->n_o + o], mu, sg, tau, fp);
        Ki[((size_t)i * nz + q) * nt + t] = acc;
      }
    }
  /* K_j(q) */
  double* Kj = malloc(sizeof(double) * nJ * nz);
  for (int q = 0; q < nz; ++q) {
    for (int j = 0; j < nJ; ++j) {
      double sz = g->sz0 * (1.0 + xz[q]) + (g->sz_bin ? g->sz_bin[j] : 0.0);
      double acc = 0.0;
      for (int o = 0; o < g->n_zo; ++o) {
        double d = (zo_x[j * g->n_zo + o] - xz[q]) / sz;
        acc += zo_w[j * g->n_zo + o] * exp(-0.5 * d * d) / (SQRT2PI * sz);
      }
      Kj[j * nz + q] = acc;
    }
  }
  /* z factors */
  double* cz = malloc(sizeof(double) * nz);
  double* sci = malloc(sizeof(double) * nz);
  int rc = 0;
  for (int q = 0; q < nz; ++q) {
    double dv;
    if (y3o_dv_do_dz(dist_z, dist_da, nd, c->om, c->ol, c->ok, c->h0, xz[q], &dv)) rc = 1;
    cz[q] = wz[q] * dv * y3o_omega_z_des(xz[q]);
    sci[q] = (shear && shear->n_sci > 0)
               ? y3o_interp1d_clamp(shear->sci_z, shear->sci_val, shear->n_sci, xz[q])
               : 1.0;
  }
  double* hax = malloc(sizeof(double) * n_hm);
  for (int i = 0; i < n_hm; ++i) hax[i] = log(hmf_m_h[i] * (c->om - c->onu));

  double* W = calloc((size_t)nB * nm, sizeof(double));
  double* Wg = calloc((size_t)nB * nm, sizeof(double));
  double* S = malloc(sizeof(double) * nI);
  const double sig = mor->sigma;
  for (int k = 0; k < nm; ++k) {
    for (int q = 0; q < nz; ++q) {
      double mu = mor->A + mor->B * (xm[k] - log(mor->Mpiv)) + mor->C * log1p(xz[q]);
      double D = phi_diff((ll_lo - mu) / sig, (ll_hi - mu) / sig);
      /* below 1e-280 the quotient is taken in logs (its limit, not 0/0) */
      double lnD = D > 1e-280 ? 0.0 : ln_phi_diff((ll_lo - mu) / sig, (ll_hi - mu) / sig);
      double n = y3o_hmf(hax, n_hm, hmf_z, n_hz, dndlnmh, c->hmf_s, c->hmf_q, xm[k], xz[q]);
      for (int i = 0; i < nI; ++i) S[i] = 0.0;
      for (int t = 0; t < nt; ++t) {
        double d = (xl[t] - mu) / sig;
        double p = D > 1e-280 ? exp(-0.5 * d * d) / (SQRT2PI * sig * D)
                              : exp(-0.5 * d * d - lnD) / (SQRT2PI * sig);
        for (int i = 0; i < nI; ++i)
          S[i] += wl[t] * Ki[((size_t)i * nz + q) * nt + t] * p;
      }
      for (int j = 0; j < nJ; ++j)
        for (int i = 0; i < nI; ++i) {
          double v = cz[q] * Kj[j * nz + q] * n * S[i];
          W[(size_t)(i + nI * j) * nm + k] += v;
          Wg[(size_t)(i + nI * j) * nm + k] += v * sci[q];
        }
    }
  }
  for (int b = 0; b < nB; ++b) {
    double acc = 0.0;
    for (int k = 0; k < nm; ++k) acc += wm[k] * W[(size_t)b * nm + k];
    counts_out[b] = acc;
  }
  if (W_out) memcpy(W_out, W, sizeof(double) * nB * nm);

  if (shear && shear_out) {
    double rho = RHOC * c->om;
    for (int b = 0; b < nB; ++b) {
      int i = b % nI;
      double rmis = shear->tau_mis * pow(shear->lob_centers[i] / 100.0, 0.2);
      for (int r = 0; r < shear->n_R; ++r) {
        double acc = 0.0;
        for (int k = 0; k < nm; ++k) {
          double M = exp(xm[k]);
          double cc = shear->c0 * pow(M / shear->c_pivot, shear->c_slope);
          double rs = y3o_nfw_rs(xm[k], cc, rho);
          double nrm = y3o_nfw_norm(xm[k], cc, rho);
          double x = shear->R[r] / rs;
          double cen = y3o_nfw_dsigma_unit(x);
          double mis = y3o_dsigma_mis_unit(x, rmis / rs, shear->n_theta, shear->n_s,
                                           shear->s_max);
          double phi = nrm * ((1.0 - shear->f_mis) * cen + shear->f_mis * mis);
          acc += wm[k] * Wg[(size_t)b * nm + k] * phi;
        }
        shear_out[(size_t)b * shear->n_R + r] = acc;
      }
    }
  }
  free(xm); free(wm); free(xz); free(wz); free(xl); free(wl);
  free(lo_x); free(lo_w); free(zo_x); free(zo_w);
  free(Ki); free(Kj); free(cz); free(sci); free(hax);
  free(W); free(Wg); free(S);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* Gaussian log-likelihood of y3_buzzard/likelihood_cp.py:132-200:
 *   shear theory[b, r] = (NC_b > 0 ? S1h[b, r] / NC_b : 0) + prj[b, r]
 *   (NC repeated over the n_R radii of each bin, bin slow and R fast),
 *   delta = data - theory, or ln data - ln max(theory, 1e-300) in log space
 *   (data already logged and invcov already the delta-method one, as setup()
 *   stores them: likelihood_cp.py:79-92,113-118),
 *   logL = -0.5 (delta_NC^T C^-1 delta_NC + delta_Sh^T C^-1 delta_Sh),
 *   a diagonal invcov (dense = 0) as sum delta^2 ic, a dense one as a
 *   matrix product (likelihood_cp.py:66-72).  prj may be NULL (zero). */
static double
y3o_chi2(int n, const double* delta, const double* ic, int dense)
{
  double acc = 0.0;
  if (!dense) {
    for (int i = 0; i < n; ++i) acc += delta[i] * delta[i] * ic[i];
    return acc;
  }
  for (int i = 0; i < n; ++i) {
    double row = 0.0;
    for (int j = 0; j < n; ++j) row += ic[(size_t)i * n + j] * delta[j];
    acc += delta[i] * row;
  }
  return acc;
}

double
y3o_loglike(int n_bins, int n_R, const double* nc, const double* s1h,
            const double* prj, int log_space, const double* data_nc,
            const double* ic_nc, int nc_dense, const double* data_sh,
            const double* ic_sh, int sh_dense)
{
  int nsh = n_bins * n_R;
  double* d = calloc((size_t)(n_bins > nsh ? n_bins : nsh) + 1, sizeof(double));
  for (int b = 0; b < n_bins; ++b)
    d[b] = log_space ? data_nc[b] - log(nc[b] > 1e-300 ? nc[b] : 1e-300)
                     : data_nc[b] - nc[b];
  double chi2 = y3o_chi2(n_bins, d, ic_nc, nc_dense);
  for (int b = 0; b < n_bins; ++b)
    for (int r = 0; r < n_R; ++r) {
      int u = b * n_R + r;
      double th = (nc[b] <= 0.0 ? 0.0 : s1h[u] / nc[b]) + (prj ? prj[u] : 0.0);
      d[u] = log_space ? data_sh[u] - log(th > 1e-300 ? th : 1e-300) : data_sh[u] - th;
    }
  chi2 += y3o_chi2(nsh, d, ic_sh, sh_dense);
  free(d);
  return -0.5 * chi2;
}

/* Miscentred Delta Sigma for an offset fixed at x_mis (the "single" kernel
 * of NFW_DSIGMA_MIS, nfw_dsigma_mis.hh:53-55): the mean tangential shear on
 * the circle of radius x around the offset centre,
 *   (1/pi) int_0^pi dth DSigma(d) cos 2phi,  d^2 = x^2 + x_mis^2 - 2 x x_mis cos th,
 * in units of 2 r_s delta_c rho; n_theta GL nodes on [0, pi]. */
double
y3o_dsigma_single_unit(double x, double xmis, int n_theta)
{
  double* th = (double*)malloc(sizeof(double) * n_theta);
  double* wth = (double*)malloc(sizeof(double) * n_theta);
  y3o_gl_nodes(0.0, M_PI, n_theta, th, wth);
  double acc = 0.0;
  for (int t = 0; t < n_theta; ++t) {
    double ct = cos(th[t]);
    double d2 = x * x + xmis * xmis - 2.0 * x * xmis * ct;
    double a = x - xmis * ct;
    acc += wth[t] * y3o_nfw_dsigma_unit(sqrt(d2)) * (2.0 * a * a / d2 - 1.0);
  }
  free(th);
  free(wth);
  return acc / M_PI;
}
