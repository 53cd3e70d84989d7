// mis_quad.cuh -- quadrature of the miscentred NFW profiles.
//
//   Sigma_mis(x)  = int_0^inf ds s e^-s (1/pi) int_0^pi dth Sigma(d)
//   DSigma_mis(x) = int_0^inf ds s e^-s (1/pi) int_0^pi dth DSigma(d) cos 2phi
// for the gamma offset kernel P(R') = R'/R_mis^2 exp(-R'/R_mis)
// (src/models/roffset_t.hh:18-23, the "gamma" kernel of
// src/models/nfw_dsigma_mis.hh), with r = x_mis s, d^2 = x^2 + r^2 -
// 2 x r cos th and cos 2phi = 2 (x - r cos th)^2 / d^2 - 1.  The DSigma line
// is the tangential-shear form of Sigma_bar(<x) - Sigma(x) of the offset
// profile (the mean tangential shear on a circle equals the mean enclosed
// minus the mean boundary surface density for any mass distribution), so no
// inner radial integral is needed.  Nodes: Gauss-Legendre in th on [0, pi];
// in s two Gauss-Legendre panels split at the kink s_k = x / x_mis where the
// offset ring crosses the aperture.
#pragma once

#include "common.cuh"
#include "host_common.h"

namespace y3b {

int gl_nodes_device(double a, double b, int n, double* xs, double* ws, cudaStream_t s);

// Miscentred profile quadrature nodes in s: two GL panels split at the
// ring-crossing kink s_k = x / x_mis (R / R_mis, mass independent).
struct MisQuad {
  int n_theta, n_s, n1;          // n1 = nodes in the first s panel
  double s_max;
  const double* th;              // GL nodes on [0, pi] [n_theta]
  const double* wth;
  const double* t1;              // GL nodes on [-1,1] [n1]
  const double* w1;
  const double* t2;              // [n_s - n1]
  const double* w2;
  const double* t0;              // single-panel GL on [-1,1] [n_s]
  const double* w0;
};

// sum over the warp's share of (s, theta) nodes of the miscentred
// integrand; x, r in units of r_s.  want_delta selects DeltaSigma
// (tangential-shear form) or Sigma.
template <typename T>
__device__ __forceinline__ T
mis_partial(const MisQuad& q, T x, T xmis, bool want_delta, int lane)
{
  const double sk = (double)x / (double)xmis;
  const bool split = sk < q.s_max && q.n_s >= 2;
  T acc = 0;
  for (int n = 0; n < q.n_s; ++n) {
    double s, ws;
    if (split) {
      if (n < q.n1) {
        s = 0.5 * sk * (1.0 + q.t1[n]);
        ws = 0.5 * sk * q.w1[n];
      } else {
        s = 0.5 * (sk + q.s_max) + 0.5 * (q.s_max - sk) * q.t2[n - q.n1];
        ws = 0.5 * (q.s_max - sk) * q.w2[n - q.n1];
      }
    } else {
      s = 0.5 * q.s_max * (1.0 + q.t0[n]);
      ws = 0.5 * q.s_max * q.w0[n];
    }
    const T r = xmis * (T)s;
    T inner = 0;
    for (int t = lane; t < q.n_theta; t += 32) {
      T ct = (T)cos(q.th[t]);
      T d2 = x * x + r * r - (T)2 * x * r * ct;
      T d = sqrt(d2);
      T v;
      if (want_delta) {
        T a = x - r * ct;
        v = NfwUnit<T>::dsigma(d) * ((T)2 * a * a / d2 - (T)1);
      } else {
        v = NfwUnit<T>::sigma(d);
      }
      inner += (T)q.wth[t] * v;
    }
    acc += (T)(ws * s * exp(-s) / kPi) * inner;
  }
  return acc;
}

template <typename T>
__device__ __forceinline__ T
warp_sum(T v)
{
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Device GL tables for the miscentring quadrature, cached per (n_theta, n_s).
struct MisQuadCache {
  int n_theta = -1, n_s = -1;
  double s_max = 0.0;
  DevBuf<double> th, wth, t1, w1, t2, w2, t0, w0;
  int ensure(int nt, int ns, double smax, cudaStream_t s)
  {
    if (nt == n_theta && ns == n_s && smax == s_max) return Y3B_OK;
    if (nt < 1 || ns < 2 || !(smax > 0.0)) {
      set_error("miscentring quadrature: need n_theta >= 1, n_s >= 2, s_max > 0");
      return Y3B_ERR_INVALID;
    }
    int n1 = ns / 2;
    Y3B_TRY(th.alloc(nt));
    Y3B_TRY(wth.alloc(nt));
    Y3B_TRY(t1.alloc(n1));
    Y3B_TRY(w1.alloc(n1));
    Y3B_TRY(t2.alloc(ns - n1));
    Y3B_TRY(w2.alloc(ns - n1));
    Y3B_TRY(t0.alloc(ns));
    Y3B_TRY(w0.alloc(ns));
    Y3B_TRY(gl_nodes_device(0.0, kPi, nt, th.get(), wth.get(), s));
    Y3B_TRY(gl_nodes_device(-1.0, 1.0, n1, t1.get(), w1.get(), s));
    Y3B_TRY(gl_nodes_device(-1.0, 1.0, ns - n1, t2.get(), w2.get(), s));
    Y3B_TRY(gl_nodes_device(-1.0, 1.0, ns, t0.get(), w0.get(), s));
    n_theta = nt;
    n_s = ns;
    s_max = smax;
    return Y3B_OK;
  }
  MisQuad view() const
  {
    MisQuad q;
    q.n_theta = n_theta;
    q.n_s = n_s;
    q.n1 = n_s / 2;
    q.s_max = s_max;
    q.th = th.get();
    q.wth = wth.get();
    q.t1 = t1.get();
    q.w1 = w1.get();
    q.t2 = t2.get();
    q.w2 = w2.get();
    q.t0 = t0.get();
    q.w0 = w0.get();
    return q;
  }
};

}  // namespace y3b
