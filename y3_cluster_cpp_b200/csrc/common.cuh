// common.cuh -- shared device helpers for the y3b CUDA library (sm_100a).
//
// Device restatements of the reference's numerics: GSL-equivalent
// linear/bilinear interpolation with the reference's clamp semantics
// (src/utils/interp_1d.cc:65-87, interp_2d.cc:115-135, interp_2d.hh:82-86),
// the richness/photo-z kernels (src/models/richness_kernel_t.hh:30-125,
// src/modules/sel_function/sel_function.py:77-262), the cosmology helpers
// (ez.hh, dv_do_dz_t.hh, omega_z_des.hh, hmf_t.hh) and the projected NFW
// profile (Wright & Brainerd form, src/models/nfw_sigma_t.hh:34-43;
// normalisation nfw_dsigma_mis.hh:95-114).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/y3b.h"

namespace y3b {

constexpr double kSqrt2 = 1.41421356237309504880;
constexpr double kSqrt2Pi = 2.50662827463100050242;
constexpr double kPi = 3.14159265358979323846;
constexpr double kRhoCrit = 2.77533742639e+11;  // h^2 Msun / Mpc^3
constexpr double kLog10e = 0.4342944819;        // hmf_t.hh:48 literal
constexpr double kHmfPivot = 13.8124426028;     // hmf_t.hh:48 literal

// Device-side error codes, reported through a status word that the host
// reads after the launch (never a trap).
enum DevErr : int {
  kDevOk = 0,
  kDevDomain = 1,   // a query outside an unclamped table (d_a, n(z))
  kDevTimeout = 2,  // a bounded wait ran out
  kDevShape = 3,    // launch shape / size mismatch detected on device
  kDevNonFinite = 4,  // a table entry is NaN or infinite
  kDevRange = 5,      // mixed form: a factor's exponent is outside the safe FP32 range
};

__device__ __forceinline__ void
set_err(int* status, int code)
{
  if (status) atomicCAS(status, 0, code);
}

// ---------------------------------------------------------------------------
// Interpolation.  bsearch_cell returns ilo with xs[ilo] <= x < xs[ilo+1]
// (x == xs[n-1] maps to the last cell), as GSL's gsl_interp_bsearch.
template <typename T>
__device__ __forceinline__ int
bsearch_cell(const T* xs, int n, T x)
{
  int ilo = 0, ihi = n - 1;
  while (ihi > ilo + 1) {
    int i = (ihi + ilo) >> 1;
    if (xs[i] > x)
      ihi = i;
    else
      ilo = i;
  }
  return ilo;
}

// Unclamped linear interpolation; returns false outside [xs[0], xs[n-1]]
// (the reference throws std::domain_error there, interp_1d.cc:76-77).
__device__ __forceinline__ bool
interp1d(const double* xs, const double* ys, int n, double x, double* out)
{
  if (!(x >= xs[0] && x <= xs[n - 1])) return false;
  int i = bsearch_cell(xs, n, x);
  double dx = xs[i + 1] - xs[i];
  *out = (dx > 0.0) ? ys[i] + (x - xs[i]) / dx * (ys[i + 1] - ys[i]) : 0.0;
  return true;
}

__device__ __forceinline__ double
interp1d_clamp(const double* xs, const double* ys, int n, double x)
{
  double xx = fmin(fmax(x, xs[0]), xs[n - 1]);
  double out;
  interp1d(xs, ys, n, xx, &out);
  return out;
}

// Clamped bilinear interpolation; zs[j * nx + i] (y slow).
__device__ __forceinline__ double
interp2d_clamp(const double* xs, int nx, const double* ys, int ny,
               const double* zs, double x, double y)
{
  double xx = fmin(fmax(x, xs[0]), xs[nx - 1]);
  double yy = fmin(fmax(y, ys[0]), ys[ny - 1]);
  int xi = bsearch_cell(xs, nx, xx);
  int yi = bsearch_cell(ys, ny, yy);
  double t = (xx - xs[xi]) / (xs[xi + 1] - xs[xi]);
  double u = (yy - ys[yi]) / (ys[yi + 1] - ys[yi]);
  const double* r0 = zs + (size_t)yi * nx + xi;
  const double* r1 = r0 + nx;
  return (1.0 - t) * (1.0 - u) * r0[0] + t * (1.0 - u) * r0[1] +
         (1.0 - t) * u * r1[0] + t * u * r1[1];
}

// 2^x on the MUFU unit (PTX ex2.approx.ftz.f32; ~2 ulp, subnormals flush
// to zero -- used only where such values are negligible).
__device__ __forceinline__ float
fast_exp2(float x)
{
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Split 8 FP32 values (4 pairs) into bf16 hi + bf16 lo and store one 16-byte
// core-matrix row of each.  hi rounds to nearest (cvt.rn.bf16x2.f32, one
// instruction per pair); lo = v - hi is exact in FP32 and keeps its top 16
// bits, so |v - hi - lo| <= 2^-16 |v|; the products hi*hi + hi*lo + lo*hi
// then carry a relative error of a few 2^-17.
__device__ __forceinline__ void
store_split8(uint8_t* hi, uint8_t* lo, const float2* v)
{
  uint32_t h[4], l[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    uint32_t hh;  // .y in the upper half, .x in the lower (memory order x, y)
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(hh) : "f"(v[k].y), "f"(v[k].x));
    const float2 hf = make_float2(__uint_as_float(hh << 16), __uint_as_float(hh & 0xFFFF0000u));
    const float2 r = __ffma2_rn(hf, make_float2(-1.f, -1.f), v[k]);
    h[k] = hh;
    l[k] = __byte_perm(__float_as_uint(r.x), __float_as_uint(r.y), 0x7632);
  }
  *reinterpret_cast<uint4*>(hi) = make_uint4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<uint4*>(lo) = make_uint4(l[0], l[1], l[2], l[3]);
}

// ---------------------------------------------------------------------------
// Cosmology.
__device__ __forceinline__ double
ez(double om, double ol, double ok, double z)
{
  double zp1 = 1.0 + z;
  return sqrt(om * zp1 * zp1 * zp1 + ok * zp1 * zp1 + ol);
}

// dV/dOmega/dz [(Mpc/h)^3] (dv_do_dz_t.hh:82-90); false if z is outside the
// d_a table.
__device__ __forceinline__ bool
dv_do_dz(const double* dz, const double* da, int nd, double om, double ol,
         double ok, double h, double z, double* out)
{
  double d;
  if (!interp1d(dz, da, nd, z, &d)) return false;
  *out = 2997.92 * (1.0 + z) * (1.0 + z) * d * h * d * h / ez(om, ol, ok, z);
  return true;
}

__device__ __forceinline__ double
poly6(const double* c, double x)
{
  double out = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) out = c[i] + x * out;
  return out;
}

// Effective survey area [rad^2], omega_z_des.hh:15-33 (Horner, highest power
// first as polynomial.hh:16-31).
__device__ __forceinline__ double
omega_z_des(double zt)
{
  const double f1[6] = {0.0, 0.0, 0.0, -0.00262353, 0.01940118, 0.45133063};
  const double f2[6] = {1.33647377e+4, 1.35291046e+3, -1.26204891e+2,
                        -2.83454918e+1, -2.26465905, 3.84958753e-1};
  const double f3[6] = {0, 0, -1.88101967, 4.8071839, -4.11424324, 1.18196785};
  if (zt < 0.504) return poly6(f1, zt);
  if (zt < 0.7) return poly6(f2, zt - 0.6);
  return poly6(f3, zt);
}

// ---------------------------------------------------------------------------
// Richness and photo-z kernels.
__device__ __forceinline__ double
phi_cdf(double x)
{
  return 0.5 * (1.0 + erf(x / kSqrt2));
}

// Phi(b) - Phi(a) for b >= a without cancellation.
__device__ __forceinline__ double
phi_diff(double a, double b)
{
  if (a >= 0.0) return 0.5 * (erfc(a / kSqrt2) - erfc(b / kSqrt2));
  if (b <= 0.0) return 0.5 * (erfc(-b / kSqrt2) - erfc(-a / kSqrt2));
  return 1.0 - 0.5 * erfc(-a / kSqrt2) - 0.5 * erfc(b / kSqrt2);
}

// exp(A) Phi(z - tau sigma), the EMG tail in the scaled-erfc form of
// sel_function.py:173-187.  erfcx is CUDA's scaled complementary error
// function.
__device__ __forceinline__ double
emg_tail(double x, double mu, double sigma, double tau)
{
  double z = (x - mu) / sigma;
  double u = (tau * sigma - z) * (1.0 / kSqrt2);
  double tail = 0.5 * erfcx(fabs(u)) * exp(-0.5 * z * z);
  if (u < 0.0) {
    double A = -tau * (x - mu) + 0.5 * (tau * sigma) * (tau * sigma);
    A = fmin(fmax(A, -700.0), 700.0);
    tail = exp(A) - tail;
  }
  return tail;
}

__device__ __forceinline__ double
cdf_lob(double x, double mu, double sigma, double tau, double fprj)
{
  double z = (x - mu) / sigma;
  double out = phi_cdf(z) - fprj * emg_tail(x, mu, sigma, tau);
  return fmin(fmax(out, 0.0), 1.0);
}

// (1 - f) N(x; mu, sigma) + f tau tail(x): the density of cdf_lob.
__device__ __forceinline__ double
pdf_lob(double x, double mu, double sigma, double tau, double fprj)
{
  double z = (x - mu) / sigma;
  double g = exp(-0.5 * z * z) / (kSqrt2Pi * sigma);
  return (1.0 - fprj) * g + fprj * tau * emg_tail(x, mu, sigma, tau);
}

// The eight EMG coefficients are linear splines in z with constant
// extrapolation (prj_params.py:122-130); coef is [8][n].
__device__ __forceinline__ void
plob_params(int n, const double* zs, const double* coef, double ltr, double z,
            double* mu, double* sigma, double* tau, double* fprj)
{
  double c[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) c[k] = interp1d_clamp(zs, coef + k * n, n, z);
  *mu = c[2] + c[3] * ltr;
  *sigma = c[5] * pow(ltr, c[4]);
  *tau = c[1] / pow(ltr, c[0]);
  *fprj = fmin(1.0, c[7] / pow(1.0 + exp(-ltr), c[6]));
}

// ---------------------------------------------------------------------------
// Projected NFW in units of 2 r_s delta_c rho.  g(x) = artanh(y)/y with
// y = sqrt(1 - x^2) (x < 1), arctan(y)/y with y = sqrt(x^2 - 1) (x > 1),
// equal to sum_n w^n / (2n + 1), w = 1 - x^2, which is used near x = 1.
//   Sigma     = (g - 1) / w
//   Sigma_bar = 2 (g + ln(x/2)) / x^2
// For x < 1/2 Sigma_bar is evaluated as
//   (2/y) [ln(2/x)/(1+y) + log1p(-x^2/(2(1+y)))/x^2]
// so no O(1) terms cancel.
template <typename T>
struct NfwUnit;

template <>
struct NfwUnit<double> {
  static __device__ __forceinline__ double g(double x)
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
  static __device__ __forceinline__ double sigma(double x)
  {
    double w = 1.0 - x * x;
    if (fabs(w) < 0.1) {
      double s = 0.0, p = 1.0;
      for (int n = 0; n < 40; ++n) {
        s += p / (2 * n + 3);
        p *= w;
      }
      return s;
    }
    return (g(x) - 1.0) / w;
  }
  static __device__ __forceinline__ double sigma_bar(double x)
  {
    if (x < 0.5) {
      double y = sqrt(1.0 - x * x);
      double x2 = x * x;
      return (2.0 / y) *
             (log(2.0 / x) / (1.0 + y) + log1p(-x2 / (2.0 * (1.0 + y))) / x2);
    }
    return 2.0 * (g(x) + log(0.5 * x)) / (x * x);
  }
  // sigma_bar(x) - sigma(x) with g(x) evaluated once where both need it
  // (x >= 0.5 away from x = 1): the same values as the two calls.
  static __device__ __forceinline__ double dsigma(double x)
  {
    const double w = 1.0 - x * x;
    if (x < 0.5 || fabs(w) < 0.1) return sigma_bar(x) - sigma(x);
    const double gx = g(x);
    return 2.0 * (gx + log(0.5 * x)) / (x * x) - (gx - 1.0) / w;
  }
};

template <>
struct NfwUnit<float> {
  // FP32 variant: same branches; the series near x = 1 is truncated at the
  // terms that matter in single precision (|w| < 0.05, 8 terms).
  static __device__ __forceinline__ float g(float x)
  {
    float w = 1.0f - x * x;
    if (fabsf(w) < 0.05f) {
      float s = 1.0f / 15.0f;
#pragma unroll
      for (int n = 6; n >= 0; --n) s = 1.0f / (2 * n + 1) + w * s;
      return s;
    }
    if (x < 1.0f) {
      float y = sqrtf(w);
      return atanhf(y) / y;
    }
    float y = sqrtf(-w);
    return atanf(y) / y;
  }
  static __device__ __forceinline__ float sigma(float x)
  {
    float w = 1.0f - x * x;
    if (fabsf(w) < 0.05f) {
      float s = 1.0f / 17.0f;
#pragma unroll
      for (int n = 6; n >= 0; --n) s = 1.0f / (2 * n + 3) + w * s;
      return s;
    }
    return (g(x) - 1.0f) / w;
  }
  static __device__ __forceinline__ float sigma_bar(float x)
  {
    if (x < 0.5f) {
      float y = sqrtf(1.0f - x * x);
      float x2 = x * x;
      return (2.0f / y) * (logf(2.0f / x) / (1.0f + y) +
                           log1pf(-x2 / (2.0f * (1.0f + y))) / x2);
    }
    return 2.0f * (g(x) + logf(0.5f * x)) / (x * x);
  }
  static __device__ __forceinline__ float dsigma(float x)
  {
    const float w = 1.0f - x * x;
    if (x < 0.5f || fabsf(w) < 0.05f) return sigma_bar(x) - sigma(x);
    const float gx = g(x);
    return 2.0f * (gx + logf(0.5f * x)) / (x * x) - (gx - 1.0f) / w;
  }
};

// Single-offset miscentred DeltaSigma (the "single" kernel of
// NFW_DSIGMA_MIS, nfw_dsigma_mis.hh:53-55) in units of 2 r_s delta_c rho:
// the mean tangential shear on the circle of radius x around the offset
// centre, (1/pi) int_0^pi dth DSigma(d) (2 a^2 / d^2 - 1) with
// d^2 = x^2 + x_mis^2 - 2 x x_mis cos th, a = x - x_mis cos th.  Returns the
// sum over the GL nodes t0, t0 + dt, ... of [0, pi] (without the 1/pi), so
// a warp can split the nodes.  The _cos form takes cos(theta) of the nodes.
__device__ __forceinline__ double
dsigma_single_partial_cos(const double* cth, const double* wth, int n, double x, double xm,
                          int t0, int dt)
{
  double acc = 0.0;
  for (int t = t0; t < n; t += dt) {
    const double ct = cth[t];
    const double d2 = x * x + xm * xm - 2.0 * x * xm * ct, a = x - xm * ct;
    acc += wth[t] * NfwUnit<double>::dsigma(sqrt(d2)) * (2.0 * a * a / d2 - 1.0);
  }
  return acc;
}

__device__ __forceinline__ double
dsigma_single_partial(const double* th, const double* wth, int n, double x, double xm, int t0,
                      int dt)
{
  double acc = 0.0;
  for (int t = t0; t < n; t += dt) {
    const double ct = cos(th[t]);
    const double d2 = x * x + xm * xm - 2.0 * x * xm * ct, a = x - xm * ct;
    acc += wth[t] * NfwUnit<double>::dsigma(sqrt(d2)) * (2.0 * a * a / d2 - 1.0);
  }
  return acc;
}

__device__ __forceinline__ double
nfw_rs(double lnM, double c, double rho)
{
  return cbrt(3.0 * exp(lnM) / (800.0 * kPi * rho)) / c;
}

__device__ __forceinline__ double
nfw_norm(double lnM, double c, double rho)  // 2 r_s delta_c rho 1e-12
{
  double delta_c = (200.0 * c * c * c / 3.0) / (log(1.0 + c) - c / (1.0 + c));
  return 2.0 * nfw_rs(lnM, c, rho) * delta_c * rho * 1e-12;
}

// ---------------------------------------------------------------------------
// Gauss-Legendre nodes on [a,b] by Newton iteration on P_N, one thread per
// node pair (p_operator_cuhre_t.hh:66-95).  Writes n nodes at x[0..n).
__device__ __forceinline__ void
gl_node_pair(double a, double b, int n, int i, double* xs, double* ws)
{
  const double mid = 0.5 * (a + b), hlen = 0.5 * (b - a);
  double z = cos(kPi * ((double)i + 0.75) / ((double)n + 0.5));
  double z1, pp;
  int guard = 0;
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
  } while (fabs(z - z1) > 1e-14 && ++guard < 100);
  xs[i] = mid - hlen * z;
  xs[n - 1 - i] = mid + hlen * z;
  double w = 2.0 * hlen / ((1.0 - z * z) * pp * pp);
  ws[i] = w;
  ws[n - 1 - i] = w;
}

// Deterministic block-wide sum (fixed tree; blockDim.x a power of two <= 1024).
template <int MAXT>
__device__ __forceinline__ double
block_sum(double v, double* sh)
{
  int t = threadIdx.x;
  sh[t] = v;
  __syncthreads();
  for (int s = blockDim.x >> 1; s > 0; s >>= 1) {
    if (t < s) sh[t] += sh[t + s];
    __syncthreads();
  }
  double r = sh[0];
  __syncthreads();
  return r;
}

}  // namespace y3b
