// engine.cu -- batched evaluation of the cluster-observable integrals on
// fixed nested Gauss-Legendre nodes (the fast_mass form of
// src/models/n_operator_sel_gl_t.hh with the lambda_t / lambda_o / z_o
// integrals of src/modules/sel_function/sel_function.py done on nodes):
//
//   K_i(t,q) = sum_o a_o P(lam_o | lam_t, z_q)           per grid, FP64
//   K_j(q)   = sum_zo b N(z_o; z_q, sz0 (1 + z_q))       per grid, FP64
//   S_i(k,q) = sum_t u_t K_i(t,q) phi((l_t - mu_kq)/s) / (s D_kq)
//   W_ij(k)  = sum_q v_q dV(z_q) Omega(z_q) [Sci(z_q)] K_j(q) n(M_k, z_q) S_i(k,q)
//   N_ij     = sum_k w_k W_ij(k);   N_ij(R) = sum_k w_k W^g_ij(k) Phi_i(R, k)
//
// Two precisions share the per-point prep (FP64 tables, z factors, MOR
// normalisation D_kq by an erf difference):
//   * FP64 "plain" form: one exp per (k, q, t) in FP64 (direct_main_kernel).
//   * mixed form: the lambda_t sum as a split-BF16 tcgen05 GEMM
//     (mixed_gemm.cu) with FP32 integrands and FP64 final sums.
// Reductions are fixed-order trees; reruns are bit-identical.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "common.cuh"
#include "engine_internal.h"
#include "host_common.h"
#include "likelihood.cuh"
#include "mis_quad.cuh"

namespace y3b {

// ---------------------------------------------------------------------------
// Per-grid precompute.
__global__ void
ki_kernel(int nI, int n_z, int n_t, int n_o, const double* xz, const double* xl,
          const double* lo_x, const double* lo_w, int n_plob, const double* plob_z,
          const double* plob_coef, double* Ki)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nI * n_z * n_t) return;
  const int t = idx % n_t, q = (idx / n_t) % n_z, i = idx / (n_t * n_z);
  const double lam = exp(xl[t]);
  double mu, sg, tau, fp;
  plob_params(n_plob, plob_z, plob_coef, lam, xz[q], &mu, &sg, &tau, &fp);
  double acc = 0.0;
  for (int o = 0; o < n_o; ++o)
    acc += lo_w[i * n_o + o] * pdf_lob(lo_x[i * n_o + o], mu, sg, tau, fp);
  Ki[idx] = acc;
}

__global__ void
uk_kernel(int nI, int n_z, int n_t, int n_t_pad, const double* wl, const double* Ki, float* UK)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nI * n_z * n_t_pad) return;
  const int t = idx % n_t_pad, iq = idx / n_t_pad;
  UK[idx] = t < n_t ? (float)(wl[t] * Ki[(size_t)iq * n_t + t]) : 0.f;
}

struct SzBins {
  double v[8];
};

__global__ void
kj_kernel(int nJ, int n_z, int n_zo, double sz0, SzBins szb, const double* xz,
          const double* zo_x, const double* zo_w, double* Kj, double* omz)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nJ * n_z) return;
  const int q = idx % n_z, j = idx / n_z;
  const double z = xz[q], sz = sz0 * (1.0 + z) + szb.v[j];
  double acc = 0.0;
  for (int o = 0; o < n_zo; ++o) {
    double d = (zo_x[j * n_zo + o] - z) / sz;
    acc += zo_w[j * n_zo + o] * exp(-0.5 * d * d) / (kSqrt2Pi * sz);
  }
  Kj[idx] = acc;
  if (j == 0) omz[q] = omega_z_des(z);
}

// ---------------------------------------------------------------------------
// Per-point prep.  One CTA per point.  The point's packed tables are staged
// into shared memory with one bulk (TMA) copy completing on an mbarrier.
__device__ __forceinline__ uint32_t
smem_addr(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Bulk async copy global -> shared completing on mbarrier `bar` (16-byte
// aligned addresses, a size that is a multiple of 16).
__device__ __forceinline__ void
bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
  asm volatile(
    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
      smem_addr(dst)),
    "l"(src), "r"(bytes), "r"(smem_addr(bar))
    : "memory");
}

struct PrepArgs {
  const GridDev* grids;
  const PointDev* pts;
  const double* tables;
  const int* slot;  // table block of point p: tables + slot[p] * stride (null: p)
  TableLayout lay;
  int mixed;
  double* s64;
  float* s32;
  int* status;
  int grid_mask;
  uint8_t* fbuf;    // mixed form: F(t, k) blocks, f_stride bytes per point
  size_t f_stride;
  int* win_tile;    // mixed form: [n][win_stride] lam_t stage window per local tile
  int win_stride;
};

// MOR normalisation D = Phi(b) - Phi(a) in FP64, a = (l_lo - mu)/s,
// b = (l_hi - mu)/s.  The lam_t domain is many sigma wide, so at most one
// tail is open: D = 1 exactly when both are below half an FP64 ulp
// (a < -8.5, b > 8.5); with one tail closed D = Phi(b) or Phi(-a), a single
// erfc on the side that does not cancel.  Kept out of line: the rare path.
__device__ __noinline__ double
mor_norm_slow(double a, double b)
{
  constexpr double kInvSqrt2 = 0.70710678118654752440;
  if (a < -8.5)  // low tail closed: D = Phi(b)
    return b < 0.0 ? 0.5 * erfc(-b * kInvSqrt2) : 1.0 - 0.5 * erfc(b * kInvSqrt2);
  if (b > 8.5)  // high tail closed: D = Phi(-a)
    return a > 0.0 ? 0.5 * erfc(a * kInvSqrt2) : 1.0 - 0.5 * erfc(-a * kInvSqrt2);
  return phi_diff(a, b);
}

__device__ __forceinline__ double
mor_norm(double a, double b)
{
  if (a < -8.5 && b > 8.5) return 1.0;
  return mor_norm_slow(a, b);
}

// v 2^e for an integer-valued e: two power-of-two factors, each a normal
// FP32 value, so the product is exact wherever it is a normal or subnormal
// FP32 number (e is clamped to [-252, 254], far past both ends of the range).
__device__ __forceinline__ float
mul_pow2(float v, double e)
{
  const int ei = (int)fmin(fmax(e, -252.0), 254.0);
  const int e1 = ei >> 1, e2 = ei - e1;
  return (v * __int_as_float((e1 + 127) << 23)) * __int_as_float((e2 + 127) << 23);
}

// ln D for the same D, finite where D itself underflows FP64 (mu more than
// ~38 sigma outside the lam_t domain).  With Q(x) = erfc(x / sqrt 2) / 2 =
// erfcx(x / sqrt 2) exp(-x^2 / 2) / 2: for 0 < a < b, D = Q(a) - Q(b) and
// ln D = ln Q(a) + log1p(-Q(b) / Q(a)); for a < b < 0, D = Q(-b) - Q(-a)
// likewise; otherwise mu lies inside the domain and D is not small.
__device__ __noinline__ double
ln_mor_norm(double a, double b)
{
  constexpr double kInvSqrt2 = 0.70710678118654752440;
  if (a > 0.0) {
    const double ra = erfcx(a * kInvSqrt2), rb = erfcx(b * kInvSqrt2);
    return log(0.5 * ra) - 0.5 * a * a + log1p(-(rb / ra) * exp(-0.5 * (b - a) * (b + a)));
  }
  if (b < 0.0) {
    const double ra = erfcx(-a * kInvSqrt2), rb = erfcx(-b * kInvSqrt2);
    return log(0.5 * rb) - 0.5 * b * b + log1p(-(ra / rb) * exp(-0.5 * (a - b) * (a + b)));
  }
  return log(mor_norm(a, b));
}

// ln D in FP32, the same cases as ln_mor_norm; with both tails open (mu
// inside the domain) D = 1 - Q(-a) - Q(b) and ln D = log1p(-Q(-a) - Q(b)),
// accurate to FP32 rounding near saturation.
__device__ __forceinline__ float
ln_mor_norm_f(float a, float b)
{
  constexpr float kInvSqrt2f = 0.70710678f;
  if (a > 0.f) {
    const float ra = erfcxf(a * kInvSqrt2f), rb = erfcxf(b * kInvSqrt2f);
    return logf(0.5f * ra) - 0.5f * a * a + log1pf(-(rb / ra) * expf(-0.5f * (b - a) * (b + a)));
  }
  if (b < 0.f) {
    const float ra = erfcxf(-a * kInvSqrt2f), rb = erfcxf(-b * kInvSqrt2f);
    return logf(0.5f * rb) - 0.5f * b * b + log1pf(-(ra / rb) * expf(-0.5f * (a - b) * (a + b)));
  }
  return log1pf(-0.5f * erfcf(-a * kInvSqrt2f) - 0.5f * erfcf(b * kInvSqrt2f));
}

// The mixed form reads log2 D(mu) from a per-point FP64 table: log2 D and
// its derivative at kDTab equally spaced mu over the point's range of
// alpha_k + beta_q, cubic Hermite interpolation (log D is smooth, so the
// relative error of D stays ~1e-9 from the domain's interior to deep tails).
constexpr int kDTab = 1024;
// Threads of the prep kernel's CTA (one point): 128, eight CTAs per SM (the
// kernel is latency-bound on short FP64 and shared-memory chains, so more
// points in flight beat more threads per point).
constexpr int kPrepThreads = 128;
constexpr int kYfHdr = 8;        // floats of yf_kernel's FP32 header
constexpr int kYfRowFields = 8;  // fields of yf_kernel's per-row block

constexpr int kEvalChunks = 8;  // chunks of a large host-buffer evaluation

// Per-point prep, one CTA per point.  The point's packed tables (without the
// HMF grid, which is read from global memory) are staged into shared memory
// with bulk (TMA) copies completing on an mbarrier; then, per point:
//   both forms: cz_q = v_q dV(z_q) Omega(z_q), czs_q = cz_q Sci(z_q),
//         alpha_k, beta_q (s64);
//   FP64 form: P0 = n(M_k,z_q) / (sqrt(2 pi) s D_kq);
//   mixed form: a_k, b_q, delta_t, c1, c2, C_j(q), C^g_j(q) for the
//         contraction, the lam_t windows, and yf_kernel's inputs (row
//         blocks, z rows, the log2 D table).
// Shared memory: table block | the grid's lnM and z_t nodes, z_t weights,
// Omega(z_t) and K_j(z_t) (staged with it) | per-k and per-q vectors |
// FP32 delta_t.
__host__ __device__ inline size_t
prep_smem_bytes(const TableLayout& L, int n_m, int n_z, int n_t_pad, int nJ)
{
  // table block without dn/dlnM, grid nodes, weights, K_j; later the log2 D table
  const size_t b0 = (L.off[2] + L.stride - L.off[3]) + ((n_m + 1) & ~1) + (size_t)(3 + nJ) * n_z;
  size_t b = (b0 > 2 * (size_t)kDTab ? b0 : 2 * (size_t)kDTab) * 8;
  b += (size_t)n_m * (8 + 8 + 8 + 4);                      // alpha, t, kf, xi
  b += (size_t)n_z * (8 + 8 + 4);                          // beta, u, yi
  b += 16 + (size_t)n_t_pad * 4;                           // FP32 delta_t (mixed form)
  return b + 64;
}

// Largest |log2| of a factor of the mixed form's Gaussian (G and H) that the
// prep kernel admits; FP32 and BF16 hold 2^-126 .. 2^127.
constexpr double kMaxExp2 = 100.0;

__global__ void __launch_bounds__(kPrepThreads, 8)
prep_kernel(PrepArgs a)
{
  extern __shared__ __align__(16) double psh[];
  const int p = blockIdx.x;
  const PointDev pt = a.pts[p];
  if (!grid_in_mask(a.grid_mask, pt.grid)) {
    if (threadIdx.x == 0) set_err(a.status, kDevShape);  // no such grid
    return;
  }
  const GridDev* __restrict__ Gp = a.grids + pt.grid;
  const int n_m = Gp->n_m, n_z = Gp->n_z, n_m_pad = Gp->n_m_pad, tid = threadIdx.x;
  const TableLayout& L = a.lay;
  const int n_hm = L.n_hm, n_hz = L.n_hz;
  // The small tables (HMF axes, distances, Sigma_crit) are staged in shared
  // memory; the n_hz x n_hm HMF grid stays in global memory (the FP64 form
  // reads it there, yf_kernel stages the mixed form's FP32 copy).
  const size_t head = L.off[2], tail = L.stride - L.off[3];
  double* tab = psh;                                                  // [head + tail]
  const int nJ = Gp->nJ, n_m2 = (n_m + 1) & ~1;
  double* g_xm = tab + head + tail;  // [n_m2]  the grid's arrays, staged with the tables
  double* g_xz = g_xm + n_m2;        // [n_z]
  double* g_wz = g_xz + n_z;         // [n_z]
  double* g_omz = g_wz + n_z;        // [n_z]
  double* g_Kj = g_omz + n_z;        // [nJ n_z]
  // Once the per-lnM and per-z factors are formed, the log2 D table is built
  // over the region of the staged tables and grid arrays.
  double* dtS = psh;  // [2 kDTab]
  double* k_alpha = psh + max((size_t)(g_Kj + (size_t)nJ * n_z - psh), (size_t)2 * kDTab);
  double* k_t = k_alpha + n_m;
  double* k_f = k_t + n_m;
  double* q_beta = k_f + n_m;
  double* q_u = q_beta + n_z;
  int* k_x = reinterpret_cast<int*>(q_u + n_z);
  int* q_y = k_x + n_m;
  __shared__ __align__(8) uint64_t bar;
  __shared__ int timed_out;
  int bad = 0;  // a non-finite table entry seen by this thread
  __shared__ double red[6];
  __shared__ int swin[16];  // lam_t stage window per lnM tile (n_m <= 1024)

  const double* src = a.tables + (size_t)(a.slot ? a.slot[p] : p) * L.stride;
  const uint32_t bytes =
    (uint32_t)((head + tail + n_m2 + (size_t)(3 + nJ) * n_z) * sizeof(double));
  if (tid == 0) {
    timed_out = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&bar)),
                 "r"(bytes)
                 : "memory");
    asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
        "r"(smem_addr(tab)),
      "l"(src), "r"((uint32_t)(head * sizeof(double))), "r"(smem_addr(&bar))
      : "memory");
    if (tail)
      asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
        "[%3];" ::"r"(smem_addr(tab + head)),
        "l"(src + L.off[3]), "r"((uint32_t)(tail * sizeof(double))), "r"(smem_addr(&bar))
        : "memory");
    bulk_copy_g2s(g_xm, Gp->xm, (uint32_t)(n_m2 * 8), &bar);
    bulk_copy_g2s(g_xz, Gp->xz, (uint32_t)(n_z * 8), &bar);
    bulk_copy_g2s(g_wz, Gp->wz, (uint32_t)(n_z * 8), &bar);
    bulk_copy_g2s(g_omz, Gp->omz, (uint32_t)(n_z * 8), &bar);
    bulk_copy_g2s(g_Kj, Gp->Kj, (uint32_t)((size_t)nJ * n_z * 8), &bar);
    // The mixed form's HMF grid is read next by yf_kernel (both of the
    // point's lnM tiles): start bringing it into L2 now.
    if (a.mixed) {
      const size_t n_dn = (size_t)n_hz * n_hm;
      const uint32_t hb = (uint32_t)(L.hmf_f32 ? ((n_dn + 1) / 2 + 1) / 2 * 16 : (n_dn * 8 + 15) & ~size_t(15));
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src + L.off[2]), "r"(hb)
                   : "memory");
    }
  }
  {
    long long t0 = clock64();
    uint32_t ok = 0;
    while (!ok) {
      asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_addr(&bar))
        : "memory");
      if (!ok && clock64() - t0 > 2000000000LL) {
        timed_out = 1;
        break;
      }
    }
  }
  __syncthreads();
  if (timed_out) {  // uniform exit; the copy only targets this CTA's shared memory
    if (tid == 0) set_err(a.status, kDevTimeout);
    return;
  }
  // Every table entry must be finite: the staged sections (not their
  // alignment padding) and, for the FP64 form, the HMF grid in global memory
  // (yf_kernel checks the mixed form's copy of it).
  {
    const int len[7] = {n_hm, n_hz, 0, L.n_dist, L.n_dist, L.n_sci, L.n_sci};
    for (int sct = 0; sct < 7; ++sct) {
      const double* base = sct < 2 ? tab + L.off[sct] : tab + head + (L.off[sct] - L.off[3]);
      for (int i = tid; i < len[sct]; i += blockDim.x) bad |= !isfinite(base[i]);
    }
    if (!a.mixed) {
      const double* __restrict__ dng = src + L.off[2];
      for (int i = tid; i < n_hz * n_hm; i += blockDim.x) bad |= !isfinite(__ldg(dng + i));
    }
    if (__syncthreads_or(bad)) {
      if (tid == 0) set_err(a.status, kDevNonFinite);
      return;
    }
  }
  double* mh = tab + L.off[0];
  const double* hz = tab + L.off[1];
  const double* __restrict__ dn = src + L.off[2];  // global
  const double* dz = tab + head;
  const double* da = tab + head + (L.off[4] - L.off[3]);
  const double* sz = tab + head + (L.off[5] - L.off[3]);
  const double* sv = tab + head + (L.off[6] - L.off[3]);
  // HMF mass axis ln(m_h (Omega_M - Omega_nu)) (hmf_t.hh:15-25), in place.
  for (int i = tid; i < n_hm; i += blockDim.x) mh[i] = log(mh[i] * (pt.om - pt.onu));
  __syncthreads();
  double* s64 = a.s64 + (size_t)p * Gp->s64_stride;
  float* s32 = a.s32 + (size_t)p * Gp->s32_stride;
  const double lnMpiv = log(pt.Mpiv);
  const double* xm = g_xm;
  const double* xz = g_xz;
  for (int k = tid; k < n_m; k += blockDim.x) {
    const double x = xm[k];
    const double alpha = pt.B * (x - lnMpiv);
    k_alpha[k] = alpha;
    s64[Gp->o_alpha + k] = alpha;
    const double xx = fmin(fmax(x, mh[0]), mh[n_hm - 1]);
    const int xi = bsearch_cell(mh, n_hm, xx);
    k_x[k] = xi;
    k_t[k] = (xx - mh[xi]) / (mh[xi + 1] - mh[xi]);
    k_f[k] = pt.hmf_s * (x * kLog10e - kHmfPivot) + pt.hmf_q;
  }
  const size_t o_cz = Gp->o_cz, o_czs = Gp->o_czs, o_beta = Gp->o_beta;
  const double* Kj = g_Kj;
  for (int q = tid; q < n_z; q += blockDim.x) {
    const double z = xz[q];
    const double beta = pt.A + pt.C * log1p(z);
    q_beta[q] = beta;
    s64[o_beta + q] = beta;
    const double zz = fmin(fmax(z, hz[0]), hz[n_hz - 1]);
    const int yi = bsearch_cell(hz, n_hz, zz);
    q_y[q] = yi;
    q_u[q] = (zz - hz[yi]) / (hz[yi + 1] - hz[yi]);
    double dv;
    if (!dv_do_dz(dz, da, L.n_dist, pt.om, pt.ol, pt.ok, pt.h0, z, &dv)) {
      set_err(a.status, kDevDomain);
      dv = 0.0;
    }
    const double cz = g_wz[q] * dv * g_omz[q];
    const double czs = cz * (L.n_sci > 1 ? interp1d_clamp(sz, sv, L.n_sci, z) : 1.0);
    s64[o_cz + q] = cz;
    s64[o_czs + q] = czs;
    if (a.mixed) {
      for (int j = 0; j < nJ; ++j) {
        s32[Gp->f_CN + j * n_z + q] = (float)(cz * Kj[j * n_z + q]);
        s32[Gp->f_CG + j * n_z + q] = (float)(czs * Kj[j * n_z + q]);
      }
    }
  }
  __syncthreads();
  {  // centres of the alpha and beta ranges: block min/max
    double amin = 1e300, amax = -1e300, bmin = 1e300, bmax = -1e300;
    for (int k = tid; k < n_m; k += blockDim.x) {
      amin = fmin(amin, k_alpha[k]);
      amax = fmax(amax, k_alpha[k]);
    }
    for (int q = tid; q < n_z; q += blockDim.x) {
      bmin = fmin(bmin, q_beta[q]);
      bmax = fmax(bmax, q_beta[q]);
    }
    for (int off = 16; off > 0; off >>= 1) {
      amin = fmin(amin, __shfl_xor_sync(0xffffffffu, amin, off));
      amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, off));
      bmin = fmin(bmin, __shfl_xor_sync(0xffffffffu, bmin, off));
      bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, off));
    }
    __shared__ double wred[4][32];
    const int w = tid >> 5, nw = blockDim.x >> 5;
    if ((tid & 31) == 0) {
      wred[0][w] = amin;
      wred[1][w] = amax;
      wred[2][w] = bmin;
      wred[3][w] = bmax;
    }
    __syncthreads();
    if (tid == 0) {
      for (int i = 1; i < nw; ++i) {
        amin = fmin(amin, wred[0][i]);
        amax = fmax(amax, wred[1][i]);
        bmin = fmin(bmin, wred[2][i]);
        bmax = fmax(bmax, wred[3][i]);
      }
      red[0] = 0.5 * (amin + amax);
      red[1] = 0.5 * (bmin + bmax);
      red[2] = amin + bmin;  // range of mu = alpha_k + beta_q
      red[3] = amax + bmax;
      red[4] = bmin;
      red[5] = bmax;
      s64[Gp->o_scal] = red[0];
      s64[Gp->o_scal + 1] = red[1];
    }
  }
  __syncthreads();
  const double A0 = red[0], B0 = red[1];
  const double sig = pt.sigma, inv_s = 1.0 / sig;
  const double norm0 = 1.0 / (kSqrt2Pi * sig);
  const double ll_lo = Gp->ll_lo, ll_hi = Gp->ll_hi;
  if (!a.mixed) {
    double* __restrict__ P0 = s64 + Gp->o_P0;
    const double xl0 = Gp->xl[0], xl1 = Gp->xl[Gp->n_t - 1];
    for (int idx = tid; idx < n_z * n_m; idx += blockDim.x) {
      const int q = idx / n_m, k = idx - q * n_m;
      const double t = k_t[k], u = q_u[q];
      const double* r0 = dn + (size_t)q_y[q] * n_hm + k_x[k];
      const double* r1 = r0 + n_hm;
      const double n = ((1.0 - t) * (1.0 - u) * r0[0] + t * (1.0 - u) * r0[1] +
                        (1.0 - t) * u * r1[0] + t * u * r1[1]) *
                       k_f[k];
      const double mu = k_alpha[k] + q_beta[q];
      const double aa = (ll_lo - mu) * inv_s, bb = (ll_hi - mu) * inv_s;
      // A mu outside the lam_t nodes' span [xl_0, xl_last] carries the
      // factor exp(-v^2 / 2 s^2) of its distance v to the span here, and the
      // lam_t sum takes exp(-((l - mu)^2 - v^2) / 2 s^2): both stay finite
      // however far outside mu lies (D alone underflows near 38 sigma).
      const double c = fmin(fmax(mu, xl0), xl1);
      if (c == mu) {
        P0[idx] = n * norm0 / mor_norm(aa, bb);
      } else {
        const double v = (c - mu) * inv_s;
        P0[idx] = n * norm0 * exp(-0.5 * v * v - ln_mor_norm(aa, bb));
      }
    }
    return;
  }
  // Mixed form: the contraction's factor vectors and, for yf_kernel, the
  // per-tile row blocks, the z rows, the log2 D table and the windows.
  const double L0 = A0 + B0;
  const int n_t = Gp->n_t, n_t_pad = Gp->n_t_pad, n_mt = n_m_pad / kGemmRows;
  for (int k = tid; k < n_m_pad; k += blockDim.x)
    s32[Gp->f_a + k] = k < n_m ? (float)(k_alpha[k] - A0) : 0.f;
  for (int q = tid; q < n_z; q += blockDim.x) s32[Gp->f_b + q] = (float)(q_beta[q] - B0);
  for (int t = tid; t < n_t_pad; t += blockDim.x)
    s32[Gp->f_delta + t] = t < n_t ? (float)(Gp->xl[t] - L0) : 0.f;
  constexpr double kLog2e = 1.4426950408889634;
  const double c1d = kLog2e * 0.5 / (sig * sig), c2d = kLog2e / (sig * sig);
  const float sc1 = sqrtf((float)c1d);
  // Y is FP32: where mu is more than 5.6 sigma inside the lam_t domain,
  // 1 - D < 2^-26 and (float)D is exactly 1, the saturated scale.  The FP32
  // test keeps a 1e-3 margin; everything else reads the table of log2 D.
  const float mu_sat_lo = (float)(ll_lo + 5.6 * sig - L0) + 1e-3f;
  const float mu_sat_hi = (float)(ll_hi - 5.6 * sig - L0) - 1e-3f;
  // log2 D(mu) and h dlog2D/dmu on kDTab equally spaced mu over the point's
  // range of alpha_k + beta_q, evaluated and stored in FP64 and, rounded, in
  // FP32 for yf_kernel's cubic Hermite (FP32 where |log2 D| <= 16, FP64
  // deeper in a tail).  ln D comes from ln_mor_norm (finite however
  // far mu lies outside the domain) and dlnD/dmu = (phi(a) - phi(b)) / (s D),
  // taken in logs.  Only nodes next to a mu that fails the FP32 saturation
  // test are read (the test's margin is 1e-3 plus FP32 rounding, and the
  // nodes used lie within hmu of mu): the interior nodes hold 0 without an
  // erfc.
  const double mu0 = red[2];
  const double hmu = red[3] > red[2] ? (red[3] - red[2]) / (kDTab - 1) : 1.0;
  const double inv_hmu = 1.0 / hmu;
  {
    float* dt32 = s32 + Gp->f_dt32;
    double* dt64 = s64 + Gp->o_dt64;
    const int j_sat0 =
      (int)fmin(fmax(ceil((ll_lo + 5.6 * sig + 0.01 - mu0) * inv_hmu) + 2.0, 0.0), (double)kDTab);
    const int j_sat1 =
      (int)fmin(fmax(floor((ll_hi - 5.6 * sig - 0.01 - mu0) * inv_hmu) - 2.0, 0.0), (double)kDTab);
    const int n_lo = min(j_sat0 + 1, kDTab), n_hi = kDTab - max(j_sat1, n_lo);
    for (int j = n_lo + tid; j < kDTab - n_hi; j += blockDim.x) {
      dtS[j] = 0.0;
      dtS[kDTab + j] = 0.0;
    }
    // Nodes evaluated in FP32 (transcendentals an order of magnitude faster
    // than FP64 here); where log2 D < -12 (the FP32 value's absolute error
    // would pass 1e-6) the node is evaluated again in FP64 for both tables.
    // The FP64 table is read only by cells with log2 D < -16, whose Hermite
    // nodes lie in that range.
    for (int r = tid; r < n_lo + n_hi; r += blockDim.x) {
      const int j = r < n_lo ? r : kDTab - n_hi + (r - n_lo);
      const double mu = mu0 + j * hmu;
      const double aa = (ll_lo - mu) * inv_s, bb = (ll_hi - mu) * inv_s;
      const float lnDf = ln_mor_norm_f((float)aa, (float)bb);
      double l2, dl2;
      if (lnDf * (float)kLog2e >= -12.f) {
        const float af = (float)aa, bf = (float)bb;
        l2 = (double)(lnDf * (float)kLog2e);
        dl2 = (double)((float)(hmu * inv_s * kLog2e / kSqrt2Pi) *
                       (expf(-0.5f * af * af - lnDf) - expf(-0.5f * bf * bf - lnDf)));
      } else {
        const double lnD = ln_mor_norm(aa, bb);
        l2 = kLog2e * lnD;
        dl2 = hmu * inv_s * kLog2e * (exp(-0.5 * aa * aa - lnD) - exp(-0.5 * bb * bb - lnD)) /
              kSqrt2Pi;
      }
      dtS[j] = l2;
      dtS[kDTab + j] = dl2;
    }
    __syncthreads();
    // The FP64 table, and yf_kernel's FP32 one: per interval [j, j + 1] the
    // cubic Hermite in t = (mu - mu_j) / h as coefficients
    // c0 + c1 t + c2 t^2 + c3 t^3 (one 16-byte load and three FMAs per
    // cell), formed in FP64.
    for (int j = tid; j < kDTab; j += blockDim.x) {
      const int j1 = min(j + 1, kDTab - 1);
      const double T0 = dtS[j], T1 = dtS[j1], D0 = dtS[kDTab + j], D1 = dtS[kDTab + j1];
      dt64[j] = T0;
      dt64[kDTab + j] = D0;
      *reinterpret_cast<float4*>(dt32 + 4 * j) =
        make_float4((float)T0, (float)D0, (float)(3.0 * (T1 - T0) - 2.0 * D0 - D1),
                    (float)(2.0 * (T0 - T1) + D0 + D1));
    }
  }
  if (tid == 0) {
    s32[Gp->f_scal] = (float)c1d;      // c1: F = exp2(-(d - a)^2 c1)
    s32[Gp->f_scal + 1] = (float)c2d;  // c2: G = exp2(d b c2)
    float* fh = s32 + Gp->f_hdr;
    fh[0] = (float)c2d;
    fh[1] = mu_sat_lo;
    fh[2] = mu_sat_hi;
    fh[3] = sc1;
    fh[4] = (float)(mu0 - L0);
    fh[5] = (float)inv_hmu;
    fh[6] = 0.f;
    fh[7] = 0.f;
    double* th = s64 + Gp->o_thdr;
    th[0] = A0;
    th[1] = B0;
    th[2] = mu0;
    th[3] = inv_hmu;
    th[4] = c2d;
    th[5] = ll_lo;
    th[6] = ll_hi;
    th[7] = inv_s;
  }
  {  // z rows: HMF z cell, its weight, b_q = beta_q - B0
    const int nzp = Gp->nzp;
    int* qy = reinterpret_cast<int*>(s32 + Gp->f_q);
    float* qu = s32 + Gp->f_q + nzp;
    float* qb = qu + nzp;
    for (int q = tid; q < nzp; q += blockDim.x) {
      qy[q] = q < n_z ? q_y[q] : 0;
      qu[q] = q < n_z ? (float)q_u[q] : 0.f;
      qb[q] = q < n_z ? (float)(q_beta[q] - B0) : 0.f;
    }
  }
  float* dt_f = reinterpret_cast<float*>(
    (reinterpret_cast<uintptr_t>(q_y + n_z) + 15) & ~uintptr_t(15));  // [n_t_pad]
  for (int t = tid; t < n_t_pad; t += blockDim.x) dt_f[t] = t < n_t ? (float)(Gp->xl[t] - L0) : 0.f;
  __shared__ float tile_af[16];  // per lnM tile: min and max of its rows' FP32 a_k
  __shared__ int tile_sc[8];     // per lnM tile: some row carries a scale
  for (int mt = tid; mt < 8; mt += blockDim.x) tile_sc[mt] = 0;
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
  // lam_t window of the contraction per lnM tile, one warp per tile.  Each
  // (k, q) cell's density exp(-(l - mu)^2 / 2 s^2) / D is renormalised to the
  // lam_t domain [ll_lo, ll_hi], where it peaks at c = clamp(mu, ll_lo,
  // ll_hi); it is below 4e-6 of that peak outside mu -+ R(mu),
  // R = sqrt((c - mu)^2 + (5 s)^2).  For mu inside the domain that is
  // mu -+ 5 s (Gaussian mass 3e-7 per side); for mu below ll_lo (above
  // ll_hi) the window reaches from the domain edge to where the renormalised
  // density has fallen by the same factor, so cells whose in-range mass D is
  // small keep all of it.  mu -+ R(mu) increase with mu, so the tile's window
  // runs from the lower end for its smallest mu to the upper end for its
  // largest; stages outside add less than the rounding of the split-BF16
  // products.  The stage count is rounded up to pairs.
  {
    constexpr double kWin = 5.0;
    const int nk = n_t_pad / 16;
    for (int mt = warp; mt < n_mt; mt += nw) {
      double amn = 1e300, amx = -1e300;
      for (int k = mt * kGemmRows + lane; k < min(n_m, (mt + 1) * kGemmRows); k += 32) {
        amn = fmin(amn, k_alpha[k]);
        amx = fmax(amx, k_alpha[k]);
      }
      for (int off = 16; off > 0; off >>= 1) {
        amn = fmin(amn, __shfl_xor_sync(0xffffffffu, amn, off));
        amx = fmax(amx, __shfl_xor_sync(0xffffffffu, amx, off));
      }
      if (lane == 0) {
        int lo = 0, hi = nk;
        if (amx >= amn) {
          const double mu_lo = amn + red[4], mu_hi = amx + red[5];
          const double e_lo = fmin(fmax(mu_lo, ll_lo), ll_hi) - mu_lo;
          const double e_hi = fmin(fmax(mu_hi, ll_lo), ll_hi) - mu_hi;
          const double w2 = (kWin * sig) * (kWin * sig);
          const float dlo = (float)(mu_lo - sqrt(e_lo * e_lo + w2) - L0);
          const float dhi = (float)(mu_hi + sqrt(e_hi * e_hi + w2) - L0);
          int a = 0, b = n_t;  // first t with delta_t >= dlo (nodes ascend)
          while (a < b) {
            const int m = (a + b) >> 1;
            if (dt_f[m] < dlo) a = m + 1; else b = m;
          }
          const int t_lo = a;
          a = t_lo;
          b = n_t;  // first t with delta_t > dhi
          while (a < b) {
            const int m = (a + b) >> 1;
            if (dt_f[m] <= dhi) a = m + 1; else b = m;
          }
          const int t_hi = a;
          // Stages [t_lo / 16, ceil(t_hi / 16)), the count rounded up to
          // pairs (at least one pair; nk is even) and kept inside [0, nk).
          const int s_lo = t_lo / 16, s_hi = (t_hi + 15) / 16;
          const int cnt = max(2, (s_hi - s_lo + 1) & ~1);
          lo = min(s_lo, nk - cnt);
          hi = lo + cnt;
        }
        swin[2 * mt] = lo;
        swin[2 * mt + 1] = hi;
        // The tile's range of a_k = alpha_k - A0 as FP32: rounding is
        // monotone, so these are the min and max of its rows' FP32 a_k.
        tile_af[2 * mt] = (float)(amn - A0);
        tile_af[2 * mt + 1] = (float)(amx - A0);
      }
    }
  }
  __syncthreads();
  // Row scale.  F(t, k) = 2^-((delta_t - a_k)^2 c1) underflows FP32 on every
  // issued node when a_k lies far outside the issued nodes' span [e_lo, e_hi]
  // of its tile (mu many sigma outside the lam_t domain), while its
  // Y(k, q) = n H / D overflows: the product, the renormalised density at
  // the domain edge, is moderate.  With c_k = clamp(a_k, e_lo, e_hi) and
  // v_k = c_k - a_k the row carries F'(t, k) = F 2^(v_k^2 c1) =
  // 2^-((delta_t - c_k)(delta_t - c_k + 2 v_k) c1) <= 1 and
  // Y'(k, q) = Y 2^-(v_k^2 c1), formed from ln D in FP64.  Rows inside the
  // span keep v_k = 0 and the unscaled factors bit for bit.  Row block of
  // yf_kernel, per tile [field][128]: t, cell, kf / (sqrt(2 pi) s), a,
  // F centre c sqrt(c1), 2 v sqrt(c1), v^2 c1, valid.
  for (int r = tid; r < n_m_pad; r += blockDim.x) {
    const int mt = r / kGemmRows, k = r;
    const int t_first = swin[2 * mt] * 16, t_last = min(swin[2 * mt + 1] * 16, n_t) - 1;
    float am = 1e18f, vs2 = 0.f;
    double vv = 0.0;
    if (k < n_m) {
      const double ak = k_alpha[k] - A0;
      const double c_lo = t_last >= t_first ? (double)dt_f[t_first] : -1e300;
      const double c_hi = t_last >= t_first ? (double)dt_f[t_last] : 1e300;
      if (ak < c_lo || ak > c_hi) {
        const float cf = ak < c_lo ? dt_f[t_first] : dt_f[t_last];
        const double v = (double)cf - ak;
        am = cf * sc1;
        vs2 = (float)(2.0 * v) * sc1;
        vv = v * v * c1d;
      } else {
        am = (float)ak * sc1;
      }
    }
    float* rw = s32 + Gp->f_rows + (size_t)mt * kYfRowFields * kGemmRows + (r & (kGemmRows - 1));
    const bool ok = k < n_m;
    rw[0 * kGemmRows] = ok ? (float)k_t[k] : 0.f;
    rw[1 * kGemmRows] = __int_as_float(ok ? k_x[k] : 0);
    rw[2 * kGemmRows] = ok ? (float)(k_f[k] * norm0) : 0.f;
    rw[3 * kGemmRows] = ok ? (float)(k_alpha[k] - A0) : 0.f;
    rw[4 * kGemmRows] = am;
    rw[5 * kGemmRows] = vs2;
    rw[6 * kGemmRows] = (float)vv;
    rw[7 * kGemmRows] = __int_as_float(ok ? 1 : 0);
    s64[Gp->o_vv + r] = vv;
    if (vv != 0.0) tile_sc[mt] = 1;
  }
  __syncthreads();
  // Per tile: the stages each contraction tile (lnM tile, richness-bin group)
  // issues, yf_kernel's info and the exponent-range guard.  A contraction
  // tile issues the MOR window intersected with the stages where its bins'
  // kernels K_i(t, q) reach 1e-12 of their maximum (outside, every term is
  // below that fraction of the bin's kernel): the count rounded up to pairs
  // inside [0, nk); where the two do not meet (the tile's MOR density lies
  // where none of its bins' kernels does, so its terms are negligible) one
  // pair at the window's start, which keeps its accumulator defined.
  // yf_kernel writes F over the hull of the lnM tile's issued ranges.
  // G = 2^(delta b c2) over the issued stages and H = 2^(-(a b + b^2/2) c2)
  // must stay well inside FP32 / BF16 (2^-126 .. 2^127).  |a| <=
  // (max alpha - min alpha) / 2 and |b| <= (max beta - min beta) / 2 after
  // centring, so the bound below holds for every factor; a point beyond it
  // reports kDevRange (its FP64 form is unaffected).
  for (int mt = tid; mt < n_mt; mt += blockDim.x) {
    const int nk = n_t_pad / 16, lo = swin[2 * mt], hi = swin[2 * mt + 1];
    int h_lo = nk, h_hi = 0;
    for (int bg = 0; bg < Gp->n_bg; ++bg) {
      const int i0 = bg * Gp->nIc, i1 = min(Gp->nI, i0 + Gp->nIc);
      int klo = n_t, khi = -1;
      for (int i = i0; i < i1; ++i) {
        klo = min(klo, Gp->kt_lo[i]);
        khi = max(khi, Gp->kt_hi[i]);
      }
      int s0 = max(lo, klo / 16), s1 = min(hi, khi / 16 + 1);
      if (s1 <= s0) {
        s0 = lo;
        s1 = lo + 2;
      }
      if ((s1 - s0) & 1) {
        if (s1 < nk) ++s1; else --s0;
      }
      h_lo = min(h_lo, s0);
      h_hi = max(h_hi, s1);
      a.win_tile[(size_t)p * a.win_stride + mt * Gp->n_bg + bg] = s0 | (s1 << 16);
    }
    float* ti = s32 + Gp->f_tinfo + 4 * mt;
    ti[0] = tile_af[2 * mt];
    ti[1] = tile_af[2 * mt + 1];
    ti[2] = __int_as_float(tile_sc[mt]);
    ti[3] = __int_as_float(h_lo | (h_hi << 16));
    double dmax = 0.0;
    const int t0 = h_lo * 16, t1 = min(h_hi * 16, n_t) - 1;
    if (t1 >= t0) dmax = fmax(fabs((double)dt_f[t0]), fabs((double)dt_f[t1]));
    const double bmax = 0.5 * (red[5] - red[4]);
    const double amax = 0.5 * ((red[3] - red[2]) - (red[5] - red[4]));
    const double e = c2d * bmax * fmax(dmax, amax + 0.5 * bmax);
    if (!(e <= kMaxExp2)) set_err(a.status, kDevRange);
  }
}

// Shared memory of yf_kernel: HMF grid in FP32 | row block | row scale |
// tile info | headers | z rows | log2 D table | delta_t.
__host__ __device__ inline size_t
yf_h32_bytes(const TableLayout& L)
{
  const size_t n_dn = (size_t)L.n_hz * L.n_hm;
  return L.hmf_f32 ? ((n_dn + 1) / 2 + 1) / 2 * 16 : (n_dn * 4 + 15) & ~size_t(15);
}

__host__ __device__ inline size_t
yf_smem_bytes(const TableLayout& L, int nzp_max, int n_t_pad_max)
{
  return yf_h32_bytes(L) + (size_t)kYfRowFields * kGemmRows * 4 + kGemmRows * 8 + 16 +
         kYfHdr * 4 + 8 * 8 + 3 * (size_t)nzp_max * 4 + 4 * (size_t)kDTab * 4 +
         (size_t)n_t_pad_max * 4;
}

// Mixed form, one CTA per (point, 128-row lnM tile): Y(k, q) of the tile's
// rows and its F(t, k) stage blocks, from the inputs the prep kernel wrote,
// staged into shared memory by bulk copies on one mbarrier (the HMF grid
// too when the packed tables hold it in FP32; an FP64 grid is converted
// while the copies fly).
__global__ void __launch_bounds__(256, 3)
yf_kernel(PrepArgs a)
{
  extern __shared__ __align__(16) uint8_t ysh[];
  const int p = blockIdx.x, mt0 = blockIdx.y, tid = threadIdx.x;
  const PointDev pt = a.pts[p];
  if (!grid_in_mask(a.grid_mask, pt.grid)) return;  // the prep kernel reported it
  const GridDev* __restrict__ Gp = a.grids + pt.grid;
  const int n_m = Gp->n_m, n_z = Gp->n_z, n_t_pad = Gp->n_t_pad, nzp = Gp->nzp;
  if (mt0 >= Gp->n_m_pad / kGemmRows) return;
  const TableLayout& L = a.lay;
  const int n_hm = L.n_hm, n_hz = L.n_hz;
  float* s32 = a.s32 + (size_t)p * Gp->s32_stride;
  const double* s64 = a.s64 + (size_t)p * Gp->s64_stride;
  const double* src = a.tables + (size_t)(a.slot ? a.slot[p] : p) * L.stride;
  size_t o = 0;
  float* h32 = reinterpret_cast<float*>(ysh);  // [n_hz n_hm]
  o += yf_h32_bytes(L);
  float* rows = reinterpret_cast<float*>(ysh + o);  // [kYfRowFields][128]
  o += kYfRowFields * kGemmRows * 4;
  double* row_vv = reinterpret_cast<double*>(ysh + o);  // [128]
  o += kGemmRows * 8;
  const int* tinfo = reinterpret_cast<const int*>(ysh + o);  // [4]
  o += 16;
  const float* fh = reinterpret_cast<const float*>(ysh + o);  // [kYfHdr]
  o += kYfHdr * 4;
  const double* th = reinterpret_cast<const double*>(ysh + o);  // [8]
  o += 8 * 8;
  const int* qy = reinterpret_cast<const int*>(ysh + o);  // [3][nzp]
  const float* qu = reinterpret_cast<const float*>(qy + nzp);
  const float* qb = qu + nzp;
  o += 3 * (size_t)nzp * 4;
  const float* dt32 = reinterpret_cast<const float*>(ysh + o);  // [kDTab][4] cubic coefficients
  o += 4 * (size_t)kDTab * 4;
  const float* dt_f = reinterpret_cast<const float*>(ysh + o);  // [n_t_pad]
  // Two groups of copies: what the F blocks need (row block, headers,
  // z rows, delta_t) on `bar`, the HMF grid and the log2 D table on `bar2`,
  // which land while the F blocks are written.
  __shared__ __align__(8) uint64_t bar, bar2;
  __shared__ int timed_out;
  int bad = 0;
  const size_t n_dn = (size_t)n_hz * n_hm;
  const uint32_t h_bytes = L.hmf_f32 ? (uint32_t)yf_h32_bytes(L) : 0u;
  const uint32_t bytes = kYfRowFields * kGemmRows * 4 + kGemmRows * 8 + 16 + kYfHdr * 4 + 64 +
                         12u * nzp + 4u * n_t_pad;
  const uint32_t bytes2 = h_bytes + 16u * kDTab;
  if (tid == 0) {
    timed_out = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar2)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&bar)),
                 "r"(bytes)
                 : "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&bar2)),
                 "r"(bytes2)
                 : "memory");
    if (h_bytes) bulk_copy_g2s(h32, src + L.off[2], h_bytes, &bar2);
    bulk_copy_g2s(rows, s32 + Gp->f_rows + (size_t)mt0 * kYfRowFields * kGemmRows,
                  kYfRowFields * kGemmRows * 4, &bar);
    bulk_copy_g2s(row_vv, s64 + Gp->o_vv + (size_t)mt0 * kGemmRows, kGemmRows * 8, &bar);
    bulk_copy_g2s((void*)tinfo, s32 + Gp->f_tinfo + 4 * mt0, 16, &bar);
    bulk_copy_g2s((void*)fh, s32 + Gp->f_hdr, kYfHdr * 4, &bar);
    bulk_copy_g2s((void*)th, s64 + Gp->o_thdr, 64, &bar);
    bulk_copy_g2s((void*)qy, s32 + Gp->f_q, 12u * nzp, &bar);
    bulk_copy_g2s((void*)dt32, s32 + Gp->f_dt32, 16u * kDTab, &bar2);
    bulk_copy_g2s((void*)dt_f, s32 + Gp->f_delta, 4u * n_t_pad, &bar);
  }
  // Bounded waits (every thread polls the phase); a CTA that gives up on the
  // first group still waits, bounded, for the second before it leaves.
  auto wait_bar = [&](uint64_t* b) {
    long long t0 = clock64();
    uint32_t ok = 0;
    while (!ok) {
      asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_addr(b))
        : "memory");
      if (!ok && clock64() - t0 > 2000000000LL) {
        timed_out = 1;
        break;
      }
    }
  };
  wait_bar(&bar);
  __syncthreads();
  if (timed_out) {  // uniform exit; the copies only target this CTA's shared memory
    wait_bar(&bar2);
    if (tid == 0) set_err(a.status, kDevTimeout);
    return;
  }
  const float sc1 = fh[3];
  // F'(t, k) for the contraction (the row scale above), split into bf16
  // hi + lo and written in its shared-memory stage layout: block
  // (lnM tile, stage) of kFStageBytes, hi planes then lo planes, each plane
  // 8 lam_t nodes x 128 rows of 16 bytes.  Rows past n_m are zero.  The
  // exponent is >= 0 on every real node; the padded nodes past n_t (whose G
  // is zero) take its magnitude, so F' <= 1 stays finite there too.  Only
  // the stages inside the tile's window are ever read.
  const int win = tinfo[3], w_lo = win & 0xFFFF, w_hi = win >> 16;
  const float* row_am = rows + 4 * kGemmRows;
  const float* row_vs2 = rows + 5 * kGemmRows;
  const float2 sc2 = make_float2(sc1, sc1);
  uint8_t* fb = a.fbuf + (size_t)p * a.f_stride;
  const int nk = n_t_pad / 16;
  for (int it = w_lo * 2 * kGemmRows + tid; it < w_hi * 2 * kGemmRows; it += blockDim.x) {
    const int r = it % kGemmRows, t8 = it / kGemmRows;
    const float am = row_am[r], vs = row_vs2[r];
    const float2 nam2 = make_float2(-am, -am), vs2 = make_float2(vs, vs);
    const float4 d0 = *reinterpret_cast<const float4*>(dt_f + t8 * 8);
    const float4 d1 = *reinterpret_cast<const float4*>(dt_f + t8 * 8 + 4);
    const float2 dd[4] = {make_float2(d0.x, d0.y), make_float2(d0.z, d0.w),
                          make_float2(d1.x, d1.y), make_float2(d1.z, d1.w)};
    float2 v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const float2 x = __ffma2_rn(dd[u], sc2, nam2);
      const float2 e = __fmul2_rn(x, __fadd2_rn(x, vs2));
      v[u] = make_float2(fast_exp2(-fabsf(e.x)), fast_exp2(-fabsf(e.y)));
    }
    uint8_t* st = fb + ((size_t)mt0 * nk + (t8 >> 1)) * kFStageBytes + (t8 & 1) * 2048 + r * 16;
    store_split8(st, st + kFStageBytes / 2, v);
  }
  if (!L.hmf_f32) {  // FP64 grid: convert while the copies are in flight
    const double* __restrict__ dng = src + L.off[2];
    const int nn = (int)n_dn;
    for (int i0 = tid; i0 < nn; i0 += 4 * blockDim.x) {
      double v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = i0 + u * blockDim.x;
        v[u] = i < nn ? __ldg(dng + i) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = i0 + u * blockDim.x;
        if (i < nn) h32[i] = (float)v[u];
        bad |= !isfinite(v[u]) || !isfinite((float)v[u]);
      }
    }
  }
  wait_bar(&bar2);
  __syncthreads();
  if (timed_out) {
    if (tid == 0) set_err(a.status, kDevTimeout);
    return;
  }
  if (L.hmf_f32)
    for (int i = tid; i < (int)n_dn; i += blockDim.x) bad |= !isfinite(h32[i]);
  if (__syncthreads_or(bad)) {
    if (tid == 0) set_err(a.status, kDevNonFinite);
    return;
  }
  const int warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
  const float c2 = fh[0], mu_sat_lo = fh[1], mu_sat_hi = fh[2];
  const float mu0c = fh[4], inv_hmu_f = fh[5];
  // Y(k, q) = n(M_k, z_q) kf_k H(k, q) 2^-(v_k^2 c1) / (sqrt(2 pi) s D_kq).
  // Warp w takes a contiguous run of z rows and lane the tile rows
  // lane + 32 j (j < 4).  Each lane keeps, in registers, the two HMF z rows
  // around the current z_q interpolated in mass and scaled by
  // kf_k / (sqrt(2 pi) s), and advances them with q (the z nodes ascend).  A
  // z row whose tile cells all have mu more than 5.6 sigma inside the domain
  // (D = 1 in FP32) is FP32 only.  Otherwise an unsaturated cell takes
  // log2 D from the table by a cubic Hermite in FP32 where D >= 2^-16 (its
  // relative error there ~1e-6); deeper in a tail, and in rows that carry a
  // scale, by the Hermite of the FP64 table (read through L1), and forms
  // 2^(log2 H - v^2 c1 - log2 D) in FP64, applied as an exact power of two
  // times 2^(fraction) in FP32.
  {
    const float* rt_s = rows;
    const int* rx_s = reinterpret_cast<const int*>(rows + kGemmRows);
    const float* rn_s = rows + 2 * kGemmRows;
    const float* ra_s = rows + 3 * kGemmRows;
    const float* rvf_s = rows + 6 * kGemmRows;
    // Runs of whole pairs of z rows (n_z is a multiple of 16): Y is stored
    // [lnM tile][z / 2][128 rows][2], one float2 per lane and row.
    const int qs = ((n_z / 2 + nw - 1) / nw) * 2, qa = warp * qs, qb_end = min(n_z, qa + qs);
    float rn[4], rk[4], R0[4], R1[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      rn[j] = rn_s[lane + 32 * j];
      rk[j] = ra_s[lane + 32 * j];
      R0[j] = R1[j] = 0.f;
    }
    const float tmin = __int_as_float(tinfo[0]), tmax = __int_as_float(tinfo[1]);
    const bool scaled = tinfo[2] != 0;
    float* __restrict__ yblk = s32 + Gp->f_Yt + (size_t)mt0 * n_z * kGemmRows;
    int ycur = -2;
    for (int q0 = qa; q0 < qb_end; q0 += 2) {
    float yv[4][2];
#pragma unroll
    for (int dq = 0; dq < 2; ++dq) {
      const int q = q0 + dq;
      const int yq = qy[q];
      if (yq != ycur) {  // warp-uniform
        const float* h1 = h32 + (size_t)(yq + 1) * n_hm;
        if (yq == ycur + 1) {
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int x = rx_s[lane + 32 * j];
            R0[j] = R1[j];
            R1[j] = fmaf(rt_s[lane + 32 * j], h1[x + 1] - h1[x], h1[x]) * rn[j];
          }
        } else {
          const float* h0 = h1 - n_hm;
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int x = rx_s[lane + 32 * j];
            const float t = rt_s[lane + 32 * j];
            R0[j] = fmaf(t, h0[x + 1] - h0[x], h0[x]) * rn[j];
            R1[j] = fmaf(t, h1[x + 1] - h1[x], h1[x]) * rn[j];
          }
        }
        ycur = yq;
      }
      const float u = qu[q], bb = qb[q];
      const float hx = -bb * c2, hy = -0.5f * bb * bb * c2;  // H = 2^(a hx + hy)
      const float sat_lo = mu_sat_lo - bb, sat_hi = mu_sat_hi - bb;
      float y[4], nv[4], e[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        nv[j] = fmaf(u, R1[j] - R0[j], R0[j]);
        e[j] = scaled ? fmaf(rk[j], hx, hy) - rvf_s[lane + 32 * j] : fmaf(rk[j], hx, hy);
        y[j] = nv[j] * fast_exp2(e[j]);
      }
      if (!(tmin > sat_lo && tmax < sat_hi)) {  // some cell of this z row is unsaturated
        // The lane's four cells side by side and without branches (their
        // chains interleave): the FP32 Hermite of log2 D for each, kept
        // where the cell is unsaturated.  Deep-tail cells and rows that
        // carry a scale follow in the rare FP64 pass below.
        unsigned deep = 0u;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int r = lane + 32 * j;
          const bool sl = mt0 * kGemmRows + r < n_m && !(rk[j] > sat_lo && rk[j] < sat_hi);
          const float uu = (rk[j] + bb - mu0c) * inv_hmu_f;
          const int jj = min(max((int)floorf(uu), 0), kDTab - 2);
          const float t = uu - (float)jj;
          const float4 cf = *reinterpret_cast<const float4*>(dt32 + 4 * jj);
          const float l2d = fmaf(fmaf(fmaf(cf.w, t, cf.z), t, cf.y), t, cf.x);
          const float ys = nv[j] * fast_exp2(e[j] - l2d);
          const bool shallow = l2d >= -16.f && (!scaled || rvf_s[r] == 0.f);
          y[j] = sl && shallow ? ys : y[j];
          deep |= (sl && !shallow) ? 1u << j : 0u;
        }
        if (deep) {
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            if (!(deep & (1u << j))) continue;
            const int r = lane + 32 * j;
            const int k = mt0 * kGemmRows + r;
            const double alpha = __ldg(s64 + Gp->o_alpha + k), beta = __ldg(s64 + Gp->o_beta + q);
            const double mu = alpha + beta;
            const double ud = (mu - th[2]) * th[3];
            const int jd = min(max((int)floor(ud), 0), kDTab - 2);
            const double td = ud - jd, td2 = td * td, td3 = td2 * td;
            const double* d64 = s64 + Gp->o_dt64;
            const double l2 = (2.0 * td3 - 3.0 * td2 + 1.0) * __ldg(d64 + jd) +
                              (td3 - 2.0 * td2 + td) * __ldg(d64 + kDTab + jd) +
                              (3.0 * td2 - 2.0 * td3) * __ldg(d64 + jd + 1) +
                              (td3 - td2) * __ldg(d64 + kDTab + jd + 1);
            const double ad = alpha - th[0], bd = beta - th[1];
            const double ex = -(ad * bd + 0.5 * bd * bd) * th[4] - row_vv[r] - l2;
            const double ei = rint(ex);
            const float yf = mul_pow2(nv[j] * fast_exp2((float)(ex - ei)), ei);
            if (!(fabsf(yf) <= 3.402823466e38f)) {  // not representable: report, never a NaN
              set_err(a.status, kDevRange);
              y[j] = 0.f;
            } else {
              y[j] = yf;
            }
          }
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) yv[j][dq] = y[j];
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
      *reinterpret_cast<float2*>(yblk + ((size_t)(q0 >> 1) * kGemmRows + lane + 32 * j) * 2) =
        make_float2(yv[j][0], yv[j][1]);
    }
  }
}

// ---------------------------------------------------------------------------
// FP64 plain form.  CTA = (z node q, point); thread k sums over lam_t with one
// FP64 exp per node: V_i(q, k) = P0_kq sum_t u_t K_i(t, q) exp(-(l_t - mu)^2/2s^2)
// (with the edge factor exp(-v^2 / 2 s^2) moved into P0 for mu outside the
// nodes' span).
__global__ void __launch_bounds__(256)
direct_main_kernel(const GridDev* grids, const PointDev* pts, double* s64all, int grid_mask)
{
  extern __shared__ double dsh[];
  const int p = blockIdx.y, q = blockIdx.x;
  const PointDev pt = pts[p];
  if (!grid_in_mask(grid_mask, pt.grid)) return;
  const GridDev& G = grids[pt.grid];
  if (q >= G.n_z) return;
  const int n_t = G.n_t, nI = G.nI;
  double* wk = dsh;                 // [nI][n_t] = u_t K_i(t, q)
  double* xl = dsh + nI * n_t;      // [n_t]
  for (int u = threadIdx.x; u < nI * n_t; u += blockDim.x) {
    const int i = u / n_t, t = u % n_t;
    wk[u] = G.wl[t] * G.Ki[((size_t)i * G.n_z + q) * n_t + t];
  }
  for (int t = threadIdx.x; t < n_t; t += blockDim.x) xl[t] = G.xl[t];
  __syncthreads();
  double* s64 = s64all + (size_t)p * G.s64_stride;
  const double beta = s64[G.o_beta + q];
  const double inv2s2 = 0.5 / (pt.sigma * pt.sigma);
  for (int k = threadIdx.x; k < G.n_m; k += blockDim.x) {
    const double mu = s64[G.o_alpha + k] + beta;
    // (l - mu)^2 - v^2 = w (w + 2 v), w = l - c, v = c - mu, c = mu clamped
    // to the nodes' span (v = 0 and w = l - mu inside it).
    const double c = fmin(fmax(mu, xl[0]), xl[n_t - 1]), v2 = 2.0 * (c - mu);
    double S[kMaxLamBins];
    for (int i = 0; i < nI; ++i) S[i] = 0.0;
    for (int t = 0; t < n_t; ++t) {
      const double w = xl[t] - c;
      const double e = exp(-w * (w + v2) * inv2s2);
      for (int i = 0; i < nI; ++i) S[i] += wk[i * n_t + t] * e;
    }
    const double P0 = s64[G.o_P0 + (size_t)q * G.n_m + k];
    for (int i = 0; i < nI; ++i) s64[G.o_V + ((size_t)i * G.n_z + q) * G.n_m + k] = P0 * S[i];
  }
}

// W_ij(k) = sum_q cz_q K_j(q) V_i(q, k) (and the Sigma_crit-weighted W^g),
// fixed order over q.  CTA per point.
__global__ void __launch_bounds__(256)
direct_wreduce_kernel(const GridDev* grids, const PointDev* pts, const double* s64all,
                      double* W, double* Wg, int w_stride, int grid_mask)
{
  const int p = blockIdx.x;
  const PointDev pt = pts[p];
  if (!grid_in_mask(grid_mask, pt.grid)) return;
  const GridDev& G = grids[pt.grid];
  const double* s64 = s64all + (size_t)p * G.s64_stride;
  for (int k = threadIdx.x; k < G.n_m; k += blockDim.x) {
    for (int i = 0; i < G.nI; ++i) {
      double acc[kMaxZBins], accg[kMaxZBins];
      for (int j = 0; j < G.nJ; ++j) acc[j] = accg[j] = 0.0;
      for (int q = 0; q < G.n_z; ++q) {
        const double v = s64[G.o_V + ((size_t)i * G.n_z + q) * G.n_m + k];
        const double c = s64[G.o_cz + q], cs = s64[G.o_czs + q];
        for (int j = 0; j < G.nJ; ++j) {
          const double kj = G.Kj[j * G.n_z + q];
          acc[j] += c * kj * v;
          accg[j] += cs * kj * v;
        }
      }
      for (int j = 0; j < G.nJ; ++j) {
        const size_t o = ((size_t)p * G.nB + i + G.nI * j) * w_stride + k;
        W[o] = acc[j];
        Wg[o] = accg[j];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Stacked miscentred profile Phi_i(R, k) = norm_k [(1 - f) DSigma(R / r_s)
// + f DSigma_mis(R / r_s, tau R_lambda(lam_i) / r_s)], c(M) = c0 (M/Mp)^s,
// rho = Omega_m rho_crit.  One warp per (point, i, R, k).
template <typename T>
__global__ void __launch_bounds__(128)
shear_phi_kernel(const GridDev* grids, const PointDev* pts, int n_points, int w_stride,
                 ShearDev sh, MisQuad quad, double* Phi, int nI_max, int grid_mask)
{
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const long long per_point = (long long)nI_max * sh.n_R * w_stride;
  if (w >= per_point * n_points) return;
  const int p = (int)(w / per_point);
  long long r = w % per_point;
  const int k = (int)(r % w_stride);
  r /= w_stride;
  const int iR = (int)(r % sh.n_R);
  const int i = (int)(r / sh.n_R);
  const PointDev pt = pts[p];
  if (!grid_in_mask(grid_mask, pt.grid)) return;
  const GridDev& G = grids[pt.grid];
  if (i >= G.nI || k >= G.n_m) return;
  const double lnM = G.xm[k];
  const double c = sh.c0 * pow(exp(lnM) / sh.c_pivot, sh.c_slope);
  const double rho = kRhoCrit * pt.om;
  const double rs = nfw_rs(lnM, c, rho);
  const double rmis = sh.tau_mis * pow(sh.lob[i] / 100.0, 0.2);
  const double R = sh.R[iR];
  T mis = mis_partial<T>(quad, (T)(R / rs), (T)(rmis / rs), true, lane);
  mis = warp_sum(mis);
  if (lane == 0) {
    const double cen = (double)NfwUnit<T>::dsigma((T)(R / rs));
    Phi[(((size_t)p * nI_max + i) * sh.n_R + iR) * w_stride + k] =
      nfw_norm(lnM, c, rho) * ((1.0 - sh.f_mis) * cen + sh.f_mis * (double)mis);
  }
}

// Miscentred profile table for the mixed form.  For a richness bin i and a
// radius R the ratio x_mis / x = r_mis,i / R does not depend on the point or
// the mass, so DeltaSigma_mis(x, x_mis) is a smooth function of u = ln x
// alone: tabulated once per engine in FP64 at kMisNx nodes per (i, R) pair
// (the same direct quadrature as the FP64 form), read with 4-point Lagrange
// interpolation in u (relative error ~1e-8 at this spacing).  One more row
// after the (i, R) pairs holds the centred DeltaSigma_NFW(x) on the same
// nodes, so the mixed form reads both profiles with the same weights.
constexpr int kMisNx = 2048;

__global__ void __launch_bounds__(128)
mis_table_kernel(ShearDev sh, MisQuad quad, int n_pairs, double u0, double du, double* tab)
{
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= (long long)(n_pairs + 1) * kMisNx) return;
  const int pair = (int)(w / kMisNx), j = (int)(w % kMisNx);
  if (pair == n_pairs) {  // the centred profile (warp-uniform branch)
    if (lane == 0) tab[w] = NfwUnit<double>::dsigma(exp(u0 + j * du));
    return;
  }
  const int i = pair / sh.n_R, iR = pair % sh.n_R;
  const double ratio = sh.tau_mis * pow(sh.lob[i] / 100.0, 0.2) / sh.R[iR];
  const double x = exp(u0 + j * du);
  const double v = warp_sum(mis_partial<double>(quad, x, ratio * x, true, lane));
  if (lane == 0) tab[w] = v;
}

// Phi_i(R, k) of the mixed form from the table, one thread per (point, k):
// c(M), r_s and the normalisation once; per R the table position
// u = ln R - ln r_s and its 4-point Lagrange weights, then the centred
// profile and the miscentred one of each bin i from their rows.  A point
// whose x = R / r_s falls outside the table reports a domain error (the
// table covers Omega_m from 0.01 to 1 over the engine's masses and radii).
__global__ void __launch_bounds__(128)
shear_tab_kernel(const GridDev* grids, const PointDev* pts, int n_points, int w_stride,
                 ShearDev sh, const double* tab, double u0, double inv_du, double* Phi,
                 int nI_max, int grid_mask, int* status)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n_points * w_stride) return;
  const int p = (int)(t / w_stride), k = (int)(t % w_stride);
  const PointDev pt = pts[p];
  if (!grid_in_mask(grid_mask, pt.grid)) return;
  const GridDev& G = grids[pt.grid];
  if (k >= G.n_m) return;
  const double lnM = G.xm[k];
  const double c = sh.c0 * pow(exp(lnM) / sh.c_pivot, sh.c_slope);
  const double rho = kRhoCrit * pt.om;
  const double rs = nfw_rs(lnM, c, rho);
  const double norm = nfw_norm(lnM, c, rho);
  const double ln_rs = log(rs);
  const double* cen_row = tab + (size_t)nI_max * sh.n_R * kMisNx;
  bool bad = false;
  for (int iR = 0; iR < sh.n_R; ++iR) {
    const double tt = (sh.lnR[iR] - ln_rs - u0) * inv_du;
    int j = (int)floor(tt);
    if (!(tt >= 1.0 && tt <= kMisNx - 2.0)) {
      bad = true;
      j = min(max(j, 1), kMisNx - 3);
    }
    const double f = tt - j;
    const double l0 = -f * (f - 1.0) * (f - 2.0) / 6.0, l1 = (f + 1.0) * (f - 1.0) * (f - 2.0) * 0.5;
    const double l2 = -(f + 1.0) * f * (f - 2.0) * 0.5, l3 = (f + 1.0) * f * (f - 1.0) / 6.0;
    const double* yc = cen_row + j;
    const double cen =
      (1.0 - sh.f_mis) * (l0 * __ldg(yc - 1) + l1 * __ldg(yc) + l2 * __ldg(yc + 1) + l3 * __ldg(yc + 2));
    for (int i = 0; i < G.nI; ++i) {
      const double* y = tab + ((size_t)i * sh.n_R + iR) * kMisNx + j;
      const double mis = l0 * __ldg(y - 1) + l1 * __ldg(y) + l2 * __ldg(y + 1) + l3 * __ldg(y + 2);
      Phi[(((size_t)p * nI_max + i) * sh.n_R + iR) * w_stride + k] =
        norm * (cen + sh.f_mis * mis);
    }
  }
  if (bad) set_err(status, kDevDomain);
}

// N_b = sum_k w_k W_b(k); N_b(R) = sum_k w_k W^g_b(k) Phi_i(R, k).  CTA per
// point, warp per output, fixed xor-tree order.
__global__ void __launch_bounds__(256)
finalize_kernel(const GridDev* grids, const PointDev* pts, const double* W, const double* Wg,
                const double* Phi, int w_stride, int nB_max, int nI_max, int n_R,
                double* counts, double* shear, int grid_mask, LikeDev like, double* logL)
{
  __shared__ double s_nc[kMaxLamBins * kMaxZBins];
  __shared__ double s_sh[kMaxLamBins * kMaxZBins * kMaxR];
  __shared__ double s_red[256];
  const int p = blockIdx.x, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const PointDev pt = pts[p];
  if (!grid_in_mask(grid_mask, pt.grid)) return;
  const GridDev& G = grids[pt.grid];
  const int nw = blockDim.x >> 5;
  for (int b = warp; b < G.nB; b += nw) {
    const double* Wb = W + ((size_t)p * G.nB + b) * w_stride;
    double acc = 0.0;
    for (int k = lane; k < G.n_m; k += 32) acc += G.wm[k] * Wb[k];
    acc = warp_sum(acc);
    if (lane == 0) {
      counts[(size_t)p * nB_max + b] = acc;
      s_nc[b] = acc;
    }
  }
  if (shear && Phi) {
    // Four outputs per warp pass, their loads and shuffle trees side by side
    // (each output's own order is unchanged: lane partials over k, then the
    // xor tree).
    const int n_out = G.nB * n_R;
    for (int u0 = warp; u0 < n_out; u0 += 4 * nw) {
      double acc[4];
      const double* Wb[4];
      const double* ph[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int u = min(u0 + c * nw, n_out - 1);
        const int b = u / n_R, iR = u % n_R, i = b % G.nI;
        Wb[c] = Wg + ((size_t)p * G.nB + b) * w_stride;
        ph[c] = Phi + (((size_t)p * nI_max + i) * n_R + iR) * w_stride;
        acc[c] = 0.0;
      }
      for (int k = lane; k < G.n_m; k += 32) {
        const double wk = G.wm[k];
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[c] += wk * Wb[c][k] * ph[c][k];
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[c] = warp_sum(acc[c]);
      if (lane == 0) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int u = u0 + c * nw;
          if (u >= n_out) break;
          const int b = u / n_R, iR = u % n_R;
          shear[((size_t)p * nB_max + b) * n_R + iR] = acc[c];
          s_sh[u] = acc[c];
        }
      }
    }
  }
  // The point's Gaussian likelihood, in the block that produced its counts
  // and shear (likelihood_cp.py:132-200): no second pass over them.
  if (like.on && logL) {
    __syncthreads();
    const double v = gaussian_loglike_block(like, G.nB, like.n_R, s_nc, s_sh, s_red);
    if (threadIdx.x == 0) logL[p] = v;
  }
}

int gl_nodes_device(double a, double b, int n, double* xs, double* ws, cudaStream_t s);

struct GridBufs {
  DevBuf<double> xm, wm, xz, wz, xl, wl, lo_x, lo_w, zo_x, zo_w, Ki, Kj, omz;
  DevBuf<float> UK;
};

}  // namespace y3b

struct y3b_engine {
  y3b_engine_config cfg;
  std::vector<double> plob_z, plob_coef;
  std::vector<y3b_grid> grids_in;
  std::vector<y3b::GridDev> grids;
  std::vector<y3b::GridBufs*> gbufs;
  y3b::DevBuf<y3b::GridDev> d_grids;
  y3b::TableLayout lay;
  y3b::ShearDev shear;
  y3b::MisQuadCache quad;
  y3b::DevBuf<double> mis_tab;          // [nI_max * n_R + 1][kMisNx], mixed form
  double mis_u0 = 0.0, mis_du = 1.0;
  cudaStream_t stream = nullptr;
  y3b::DevBuf<y3b::PointDev> pts;
  y3b::DevBuf<double> tables, s64, W, Wg, Phi, counts, shear_out;
  y3b::DevBuf<float> s32;
  y3b::DevBuf<int> status, order, tile_start;
  y3b::DevBuf<int> stage_ct;  // [2] lam_t stages issued / dense, last contraction
  y3b::DevBuf<int> tile_list;
  y3b::DevBuf<int> win_tile;  // [max_points][tile_cap_pp] stage windows (prep -> contraction)
  y3b::DevBuf<uint8_t> fbuf;  // F(t, k) stage blocks of the mixed form
  y3b::LikeDev like{};        // Gaussian likelihood fused into the final sums (on = 0: none)
  y3b::DevBuf<double> like_buf, logL;
  size_t f_stride = 0;        // bytes per point
  int max_tiles_pp = 0, tile_cap_pp = 0;
  int max_mtiles = 1;  // largest number of 128-row lnM tiles of a grid
  y3b::ContractShape cshape{};
  int cstages = 0, n_ctas = 0;  // contraction ring depth and persistent CTAs
  // Chunked host-buffer evaluation: copy stream, one event and one pinned
  // status word per chunk.
  cudaStream_t xstream = nullptr;
  // The tile planner's stream and the events that fork it from, and join it
  // back to, an evaluation's stream.
  cudaStream_t pstream = nullptr;
  cudaEvent_t plan_fork = nullptr, plan_join = nullptr;
  cudaEvent_t chunk_ev[y3b::kEvalChunks] = {};
  int* chunk_status = nullptr;
  // CUDA graphs of whole evaluations, keyed by their arguments: an
  // evaluation seen before replays its graph (one launch from the host).
  struct GraphKey {
    int prec, n, mask;
    const void *pts, *tables, *slot, *counts, *shear;
    size_t w_off;
    bool operator==(const GraphKey& o) const
    {
      return prec == o.prec && n == o.n && mask == o.mask && pts == o.pts &&
             tables == o.tables && slot == o.slot && counts == o.counts && shear == o.shear &&
             w_off == o.w_off;
    }
  };
  struct GraphEntry {
    GraphKey key;
    cudaGraphExec_t exec;
    unsigned long long kernels;  // kernel launches the graph holds
    unsigned long long used;
  };
  int graph_mode = 1;                 // 0: off, 1: capture a repeated evaluation
  std::vector<GraphEntry> graphs;     // at most kMaxGraphs
  std::vector<GraphKey> seen;         // recent evaluations without a graph
  unsigned long long graph_clock = 0;
  size_t s64_stride = 0, s32_stride = 0;
  int w_stride = 0, nB_max = 0, nI_max = 0, nz_max = 0, nt_max = 0;
  size_t prep_smem = 0, yf_smem = 0, direct_smem = 0;
  size_t device_bytes = 0;
  int last_n = 0;
  std::vector<std::array<double, 2>> zt_node_range;  // per grid: min, max z_t node
  // stage timing (y3b_engine_profile)
  bool prof = false;
  int prof_evals = 0;
  double prof_ms[4] = {0, 0, 0, 0};
  struct Pending {
    int stage;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pending;
  ~y3b_engine()
  {
    for (auto& p : pending) {
      cudaEventDestroy(p.a);
      cudaEventDestroy(p.b);
    }
    for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
    for (auto* g : gbufs) delete g;
    for (auto ev : chunk_ev)
      if (ev) cudaEventDestroy(ev);
    if (chunk_status) cudaFreeHost(chunk_status);
    if (xstream) cudaStreamDestroy(xstream);
    if (pstream) cudaStreamDestroy(pstream);
    if (plan_fork) cudaEventDestroy(plan_fork);
    if (plan_join) cudaEventDestroy(plan_join);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace y3b {

static size_t
pad2(size_t n)
{
  return (n + 1) & ~size_t(1);
}

// Richness bins per contraction tile (nIc n_z <= 256 accumulator columns)
// and what follows from it.
static void
set_bins_per_tile(GridDev& g, int nIc)
{
  g.nIc = nIc;
  g.n_bg = (g.nI + g.nIc - 1) / g.nIc;
  g.ncp_c = (g.nIc * g.n_z + 15) / 16 * 16;
  g.tiles_pp = (g.n_m_pad / kGemmRows) * g.n_bg;
}

// Most expensive tiles (lam_t steps x accumulator columns) first, ties by index.
static void
rank_grids(y3b_engine* e)
{
  const int n_grids = (int)e->grids.size();
  std::vector<int> idx(n_grids);
  for (int g = 0; g < n_grids; ++g) idx[g] = g;
  auto cost = [&](int g) { return (long long)e->grids[g].n_t_pad * e->grids[g].ncp_c; };
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return cost(a) > cost(b); });
  for (int r = 0; r < n_grids; ++r) e->grids[idx[r]].cost_rank = r;
  e->max_tiles_pp = 0;
  for (const auto& g : e->grids) e->max_tiles_pp = std::max(e->max_tiles_pp, g.tiles_pp);
  e->max_mtiles = 1;
  for (const auto& g : e->grids) e->max_mtiles = std::max(e->max_mtiles, g.n_m_pad / kGemmRows);
}

static int
build_grid(y3b_engine* e, int gi)
{
  const y3b_grid& in = e->grids_in[gi];
  GridDev g{};
  GridBufs* b = e->gbufs[gi];
  cudaStream_t s = e->stream;
  g.n_m = in.n_m;
  g.n_z = in.n_z;
  g.n_t = in.n_t;
  g.n_o = in.n_o;
  g.n_zo = in.n_zo;
  g.nI = in.n_lam_bins;
  g.nJ = in.n_z_bins;
  g.nB = g.nI * g.nJ;
  g.n_m_pad = (g.n_m + kGemmRows - 1) / kGemmRows * kGemmRows;
  g.n_t_pad = (g.n_t + kKChunk - 1) / kKChunk * kKChunk;
  g.n_cols = g.nI * g.n_z;
  g.n_cols_pad = (g.n_cols + 15) / 16 * 16;
  set_bins_per_tile(g, std::max(1, std::min(g.nI, 256 / g.n_z)));
  g.lnm_lo = in.lnm_lo;
  g.lnm_hi = in.lnm_hi;
  g.zt_lo = in.zt_lo;
  g.zt_hi = in.zt_hi;
  g.ll_lo = std::log(in.lam_t_lo);
  g.ll_hi = std::log(in.lam_t_hi);
  g.sz0 = in.sz0;
  for (int j = 0; j < 8; ++j) g.sz_bin[j] = j < in.n_z_bins ? in.sz_bin[j] : 0.0;
  Y3B_TRY(b->xm.alloc(pad2(g.n_m)));  // even, for the prep kernel's bulk copy
  Y3B_TRY(b->wm.alloc(g.n_m));
  Y3B_TRY(b->xz.alloc(g.n_z));
  Y3B_TRY(b->wz.alloc(g.n_z));
  Y3B_TRY(b->xl.alloc(g.n_t));
  Y3B_TRY(b->wl.alloc(g.n_t));
  Y3B_TRY(b->lo_x.alloc((size_t)g.n_o * g.nI));
  Y3B_TRY(b->lo_w.alloc((size_t)g.n_o * g.nI));
  Y3B_TRY(b->zo_x.alloc((size_t)g.n_zo * g.nJ));
  Y3B_TRY(b->zo_w.alloc((size_t)g.n_zo * g.nJ));
  Y3B_TRY(b->Ki.alloc((size_t)g.nI * g.n_z * g.n_t));
  Y3B_TRY(b->UK.alloc((size_t)g.nI * g.n_z * g.n_t_pad));
  Y3B_TRY(b->Kj.alloc((size_t)g.nJ * g.n_z));
  Y3B_TRY(b->omz.alloc(g.n_z));
  Y3B_TRY(gl_nodes_device(in.lnm_lo, in.lnm_hi, g.n_m, b->xm.get(), b->wm.get(), s));
  Y3B_TRY(gl_nodes_device(in.zt_lo, in.zt_hi, g.n_z, b->xz.get(), b->wz.get(), s));
  {
    std::vector<double> xz(g.n_z);
    Y3B_CUDA(cudaMemcpyAsync(xz.data(), b->xz.get(), g.n_z * sizeof(double),
                             cudaMemcpyDeviceToHost, s));
    Y3B_CUDA(cudaStreamSynchronize(s));
    e->zt_node_range[gi][0] = *std::min_element(xz.begin(), xz.end());
    e->zt_node_range[gi][1] = *std::max_element(xz.begin(), xz.end());
  }
  Y3B_TRY(gl_nodes_device(g.ll_lo, g.ll_hi, g.n_t, b->xl.get(), b->wl.get(), s));
  for (int i = 0; i < g.nI; ++i)
    Y3B_TRY(gl_nodes_device(in.lam_edges[i], in.lam_edges[i + 1], g.n_o, b->lo_x.get() + i * g.n_o,
                            b->lo_w.get() + i * g.n_o, s));
  for (int j = 0; j < g.nJ; ++j)
    Y3B_TRY(gl_nodes_device(in.zob_edges[j], in.zob_edges[j + 1], g.n_zo,
                            b->zo_x.get() + j * g.n_zo, b->zo_w.get() + j * g.n_zo, s));
  DevBuf<double> pz, pc;
  Y3B_TRY(pz.upload(e->plob_z.data(), e->plob_z.size(), s));
  Y3B_TRY(pc.upload(e->plob_coef.data(), e->plob_coef.size(), s));
  int nki = g.nI * g.n_z * g.n_t;
  ki_kernel<<<(nki + 127) / 128, 128, 0, s>>>(g.nI, g.n_z, g.n_t, g.n_o, b->xz.get(), b->xl.get(),
                                             b->lo_x.get(), b->lo_w.get(), (int)e->plob_z.size(),
                                             pz.get(), pc.get(), b->Ki.get());
  count_launch();
  Y3B_CUDA(cudaGetLastError());
  int nuk = g.nI * g.n_z * g.n_t_pad;
  uk_kernel<<<(nuk + 255) / 256, 256, 0, s>>>(g.nI, g.n_z, g.n_t, g.n_t_pad, b->wl.get(),
                                             b->Ki.get(), b->UK.get());
  count_launch();
  Y3B_CUDA(cudaGetLastError());
  int nkj = g.nJ * g.n_z;
  SzBins szb;
  for (int j = 0; j < 8; ++j) szb.v[j] = g.sz_bin[j];
  kj_kernel<<<(nkj + 127) / 128, 128, 0, s>>>(g.nJ, g.n_z, g.n_zo, g.sz0, szb, b->xz.get(),
                                             b->zo_x.get(), b->zo_w.get(), b->Kj.get(),
                                             b->omz.get());
  count_launch();
  Y3B_CUDA(cudaGetLastError());
  Y3B_CUDA(cudaStreamSynchronize(s));  // pz/pc are freed on return
  {
    // Support of each bin's kernel in lam_t: outside it K_i(t, q) is below
    // 1e-12 of its maximum over t (for every q), so the contraction skips
    // those stages for the bin's tiles.
    std::vector<double> hk((size_t)nki);
    Y3B_CUDA(cudaMemcpy(hk.data(), b->Ki.get(), hk.size() * sizeof(double),
                        cudaMemcpyDeviceToHost));
    for (int i = 0; i < kMaxLamBins; ++i) {
      g.kt_lo[i] = 0;
      g.kt_hi[i] = g.n_t - 1;
    }
    for (int i = 0; i < g.nI; ++i) {
      int lo = g.n_t, hi = -1;
      for (int q = 0; q < g.n_z; ++q) {
        const double* k = hk.data() + ((size_t)i * g.n_z + q) * g.n_t;
        double mx = 0.0;
        for (int t = 0; t < g.n_t; ++t) mx = std::max(mx, k[t]);
        if (!(mx > 0.0)) continue;
        for (int t = 0; t < g.n_t; ++t)
          if (k[t] > 1e-12 * mx) {
            lo = std::min(lo, t);
            hi = std::max(hi, t);
          }
      }
      if (hi >= lo) {
        g.kt_lo[i] = lo;
        g.kt_hi[i] = hi;
      }
    }
  }
  g.uk_zindep = 1;
  {
    const int np = (int)e->plob_z.size();
    for (int r = 0; r < 8 && g.uk_zindep; ++r)
      for (int i = 1; i < np; ++i)
        if (e->plob_coef[(size_t)r * np + i] != e->plob_coef[(size_t)r * np]) {
          g.uk_zindep = 0;
          break;
        }
  }
  g.xm = b->xm.get();
  g.wm = b->wm.get();
  g.xz = b->xz.get();
  g.wz = b->wz.get();
  g.xl = b->xl.get();
  g.wl = b->wl.get();
  g.Ki = b->Ki.get();
  g.UK = b->UK.get();
  g.Kj = b->Kj.get();
  g.omz = b->omz.get();
  // Scratch layouts.
  size_t o = 0;
  g.o_scal = o;
  o += 4;
  g.o_kx = o;
  o += pad2(g.n_m);
  g.o_kt = o;
  o += pad2(g.n_m);
  g.o_kf = o;
  o += pad2(g.n_m);
  g.o_qy = o;
  o += pad2(g.n_z);
  g.o_qu = o;
  o += pad2(g.n_z);
  g.o_cz = o;
  o += pad2(g.n_z);
  g.o_czs = o;
  o += pad2(g.n_z);
  g.o_alpha = o;
  o += pad2(g.n_m);
  g.o_beta = o;
  o += pad2(g.n_z);
  g.o_P0 = o;
  o += pad2((size_t)g.n_z * g.n_m);
  g.o_V = o;
  o += pad2((size_t)g.nI * g.n_z * g.n_m);
  g.o_thdr = o;
  o += 8;
  g.o_vv = o;
  o += pad2(g.n_m_pad);
  g.o_dt64 = o;
  o += 2 * (size_t)kDTab;
  g.s64_stride = o;
  // FP32 scratch: every section a multiple of 4 floats (16 bytes), so that
  // the bulk copies of yf_kernel and the contraction start aligned.
  g.nzp = (g.n_z + 3) & ~3;
  size_t f = 0;
  g.f_a = f;
  f += g.n_m_pad;
  g.f_b = f;
  f += g.nzp;
  g.f_delta = f;
  f += g.n_t_pad;
  g.f_scal = f;
  f += 4;
  g.f_hdr = f;
  f += kYfHdr;
  g.f_tinfo = f;
  f += 4 * (size_t)(g.n_m_pad / kGemmRows);
  g.f_q = f;
  f += 3 * (size_t)g.nzp;
  g.f_dt32 = f;
  f += 4 * (size_t)kDTab;
  g.f_rows = f;
  f += (size_t)kYfRowFields * g.n_m_pad;
  g.f_Yt = f;
  f += (size_t)g.n_z * g.n_m_pad;
  g.f_CN = f;
  f += (size_t)g.nJ * g.n_z;
  g.f_CG = f;
  f += (size_t)g.nJ * g.n_z;
  g.s32_stride = (f + 3) & ~size_t(3);
  e->grids[gi] = g;
  return Y3B_OK;
}

static int
validate_grid(const y3b_grid& g)
{
  if (g.n_m < 2 || g.n_z < 2 || g.n_t < 2 || g.n_o < 1 || g.n_zo < 1 || g.n_lam_bins < 1 ||
      g.n_z_bins < 1 || g.n_lam_bins > kMaxLamBins || g.n_z_bins > kMaxZBins) {
    set_error("y3b_engine_create: grid needs n >= 2 nodes per axis and 1..8 bins per axis");
    return Y3B_ERR_INVALID;
  }
  if (g.n_m > 1024 || g.n_z % 16 != 0 || g.n_z > 256 || g.n_t > 4096) {
    set_error("y3b_engine_create: unsupported grid (n_m <= 1024, n_z a multiple of 16 and "
              "<= 256, n_t <= 4096)");
    return Y3B_ERR_UNSUPPORTED;
  }
  if (!(g.lnm_hi > g.lnm_lo) || !(g.zt_hi > g.zt_lo) || !(g.lam_t_lo > 0.0) ||
      !(g.lam_t_hi > g.lam_t_lo) || !(g.sz0 >= 0.0)) {
    set_error("y3b_engine_create: grid bounds must be ordered and positive");
    return Y3B_ERR_INVALID;
  }
  for (int j = 0; j < g.n_z_bins && j < 8; ++j)
    if (!(g.sz_bin[j] >= 0.0) || !(g.sz0 + g.sz_bin[j] > 0.0)) {
      set_error("y3b_engine_create: sigma_z must be positive in every z_obs bin");
      return Y3B_ERR_INVALID;
    }
  for (int i = 0; i < g.n_lam_bins; ++i)
    if (!(g.lam_edges[i + 1] > g.lam_edges[i])) {
      set_error("y3b_engine_create: lam_edges must increase");
      return Y3B_ERR_INVALID;
    }
  for (int j = 0; j < g.n_z_bins; ++j)
    if (!(g.zob_edges[j + 1] > g.zob_edges[j])) {
      set_error("y3b_engine_create: zob_edges must increase");
      return Y3B_ERR_INVALID;
    }
  return Y3B_OK;
}

}  // namespace y3b

using namespace y3b;

extern "C" void
y3b_engine_destroy(y3b_engine* e)
{
  delete e;
}

extern "C" int
y3b_engine_create(const y3b_grid* grids, int n_grids, const y3b_engine_config* cfg,
                  y3b_engine** out)
{
  clear_error();
  if (!grids || !cfg || !out || n_grids < 1 || n_grids > 31) {
    set_error("y3b_engine_create: need 1..31 grids, a config and an output handle");
    return Y3B_ERR_INVALID;
  }
  *out = nullptr;
  for (int g = 0; g < n_grids; ++g) {
    Y3B_TRY(validate_grid(grids[g]));
    if (grids[g].n_lam_bins != grids[0].n_lam_bins || grids[g].n_z_bins != grids[0].n_z_bins) {
      set_error("y3b_engine_create: all grids must share the bin layout");
      return Y3B_ERR_INVALID;
    }
  }
  if (cfg->n_hm < 2 || cfg->n_hz < 2 || cfg->n_dist < 2 || cfg->max_points < 1 ||
      cfg->max_points > 65535 ||
      cfg->plob.n < 1 || !cfg->plob.z || !cfg->plob.coef ||
      (cfg->with_shear && (cfg->n_sci < 2 || cfg->shear.n_R < 1 || cfg->shear.n_R > kMaxR))) {
    set_error("y3b_engine_create: invalid table shapes, capacity (1..65535), P(lam_o|lam_t) table or "
              "shear options (n_sci >= 2 and 1 <= n_R <= 32 with shear)");
    return Y3B_ERR_INVALID;
  }
  Y3B_TRY(require_device());
  y3b_engine* e = new (std::nothrow) y3b_engine();
  if (!e) {
    set_error("y3b_engine_create: out of host memory");
    return Y3B_ERR_NOMEM;
  }
  auto fail = [&](int rc) {
    delete e;
    return rc;
  };
  e->cfg = *cfg;
  e->plob_z.assign(cfg->plob.z, cfg->plob.z + cfg->plob.n);
  e->plob_coef.assign(cfg->plob.coef, cfg->plob.coef + 8 * (size_t)cfg->plob.n);
  e->cfg.plob.z = e->plob_z.data();
  e->cfg.plob.coef = e->plob_coef.data();
  e->grids_in.assign(grids, grids + n_grids);
  e->grids.resize(n_grids);
  e->zt_node_range.resize(n_grids);
  for (int g = 0; g < n_grids; ++g) e->gbufs.push_back(new (std::nothrow) GridBufs());
  int rc = cuda_status(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking),
                       "cudaStreamCreate");
  if (rc) return fail(rc);
  for (int g = 0; g < n_grids; ++g) {
    rc = build_grid(e, g);
    if (rc) return fail(rc);
  }
  // Table layout: each section 16-byte aligned.
  TableLayout& L = e->lay;
  L.n_hm = cfg->n_hm;
  L.n_hz = cfg->n_hz;
  L.n_dist = cfg->n_dist;
  L.n_sci = cfg->n_sci;
  L.hmf_f32 = cfg->hmf_fp32 != 0;
  const size_t n_dn = (size_t)cfg->n_hz * cfg->n_hm;
  size_t sizes[7] = {(size_t)cfg->n_hm,   (size_t)cfg->n_hz,   L.hmf_f32 ? (n_dn + 1) / 2 : n_dn,
                     (size_t)cfg->n_dist, (size_t)cfg->n_dist, (size_t)cfg->n_sci,
                     (size_t)cfg->n_sci};
  size_t o = 0;
  for (int i = 0; i < 7; ++i) {
    L.off[i] = o;
    o += pad2(sizes[i]);
  }
  L.stride = o;
  for (const auto& g : e->grids) {
    e->s64_stride = std::max(e->s64_stride, g.s64_stride);
    e->s32_stride = std::max(e->s32_stride, g.s32_stride);
    e->w_stride = std::max(e->w_stride, g.n_m);
    e->nB_max = std::max(e->nB_max, g.nB);
    e->nI_max = std::max(e->nI_max, g.nI);
    e->nz_max = std::max(e->nz_max, g.n_z);
    e->nt_max = std::max(e->nt_max, g.n_t);
  }
  // Every grid uses the engine-wide strides (offsets are within a block).
  for (auto& g : e->grids) {
    g.s64_stride = e->s64_stride;
    g.s32_stride = e->s32_stride;
  }
  int ntp_max = 0;
  for (const auto& g : e->grids) ntp_max = std::max(ntp_max, g.n_t_pad);
  e->prep_smem = prep_smem_bytes(L, e->w_stride, e->nz_max, ntp_max, e->grids[0].nJ);
  e->yf_smem = yf_smem_bytes(L, (e->nz_max + 3) & ~3, ntp_max);
  e->direct_smem = ((size_t)e->nI_max * e->nt_max + e->nt_max) * 8;
  if (e->prep_smem > 200 * 1024 || e->yf_smem > 200 * 1024 || e->direct_smem > 200 * 1024) {
    set_error("y3b_engine_create: per-point tables too large for shared-memory staging");
    return fail(Y3B_ERR_UNSUPPORTED);
  }
  {
    ContractShape& c = e->cshape;
    c.nJ = e->grids[0].nJ;
    c.nz_max = e->nz_max;
    c.ntp_max = 0;
    c.uk_max = 0;
    for (const auto& g : e->grids) {
      c.ntp_max = std::max(c.ntp_max, g.n_t_pad);
      if (g.uk_zindep) c.uk_max = std::max(c.uk_max, g.nIc * g.n_t_pad);
    }
    if (c.uk_max > 4096) c.uk_max = 0;  // larger per-tile slices are read from global memory
  }
  if (contract_stages(e->cshape) == 0) {
    set_error("y3b_engine_create: the contraction needs more shared memory than one CTA has");
    return fail(Y3B_ERR_UNSUPPORTED);
  }
  e->cstages = contract_stages(e->cshape);
  {
    int dev = 0;
    cudaGetDevice(&dev);
    if ((rc = cuda_status(cudaDeviceGetAttribute(&e->n_ctas, cudaDevAttrMultiProcessorCount, dev),
                          "cudaDeviceGetAttribute")))
      return fail(rc);
  }
  if ((rc = contract_prepare(e->cshape))) return fail(rc);
  rc = cuda_status(cudaStreamCreateWithFlags(&e->xstream, cudaStreamNonBlocking), "cudaStreamCreate");
  if (!rc)
    rc = cuda_status(cudaStreamCreateWithFlags(&e->pstream, cudaStreamNonBlocking),
                     "cudaStreamCreate");
  if (!rc)
    rc = cuda_status(cudaEventCreateWithFlags(&e->plan_fork, cudaEventDisableTiming),
                     "cudaEventCreate");
  if (!rc)
    rc = cuda_status(cudaEventCreateWithFlags(&e->plan_join, cudaEventDisableTiming),
                     "cudaEventCreate");
  for (int c = 0; c < kEvalChunks && !rc; ++c)
    rc = cuda_status(cudaEventCreateWithFlags(&e->chunk_ev[c], cudaEventDisableTiming),
                     "cudaEventCreate");
  if (!rc)
    rc = cuda_status(cudaHostAlloc((void**)&e->chunk_status, kEvalChunks * sizeof(int),
                                   cudaHostAllocDefault),
                     "cudaHostAlloc");
  if (rc) return fail(rc);
  // Contraction schedule: grids with the most expensive tiles first.  The
  // tile list holds the most tiles any tuning can give (one bin per tile).
  rank_grids(e);
  e->tile_cap_pp = 0;
  for (const auto& g : e->grids)
    e->tile_cap_pp = std::max(e->tile_cap_pp, (g.n_m_pad / kGemmRows) * g.nI);
  // Shear options.
  ShearDev& sh = e->shear;
  std::memset(&sh, 0, sizeof(sh));
  if (cfg->with_shear) {
    sh.n_R = cfg->shear.n_R;
    for (int r = 0; r < sh.n_R; ++r) {
      sh.R[r] = cfg->shear.R[r];
      sh.lnR[r] = std::log(sh.R[r]);
    }
    sh.f_mis = cfg->shear.f_mis;
    sh.tau_mis = cfg->shear.tau_mis;
    for (int i = 0; i < kMaxLamBins; ++i) sh.lob[i] = cfg->shear.lob_centers[i];
    sh.c0 = cfg->shear.c0;
    sh.c_slope = cfg->shear.c_slope;
    sh.c_pivot = cfg->shear.c_pivot;
    rc = e->quad.ensure(cfg->shear.n_theta, cfg->shear.n_s, cfg->shear.s_max, e->stream);
    if (rc) return fail(rc);
    // Table range of x = R / r_s over the grids' masses, the radii and
    // Omega_m in [0.01, 1], widened by 1.5 on both sides.
    double x_lo = 1e300, x_hi = 0.0, r_lo = 1e300, r_hi = 0.0;
    for (int r = 0; r < sh.n_R; ++r) {
      r_lo = std::min(r_lo, sh.R[r]);
      r_hi = std::max(r_hi, sh.R[r]);
    }
    for (const auto& g : e->grids)
      for (double lnM : {g.lnm_lo, g.lnm_hi})
        for (double om : {0.01, 1.0}) {
          const double M = std::exp(lnM), c = sh.c0 * std::pow(M / sh.c_pivot, sh.c_slope);
          const double rs = std::cbrt(3.0 * M / (800.0 * kPi * kRhoCrit * om)) / c;
          x_lo = std::min(x_lo, r_lo / rs);
          x_hi = std::max(x_hi, r_hi / rs);
        }
    e->mis_u0 = std::log(x_lo / 1.5);
    e->mis_du = (std::log(x_hi * 1.5) - e->mis_u0) / (kMisNx - 1);
    const int n_pairs = e->nI_max * sh.n_R;
    if ((rc = e->mis_tab.alloc((size_t)(n_pairs + 1) * kMisNx))) return fail(rc);
    const long long threads = (long long)(n_pairs + 1) * kMisNx * 32;
    mis_table_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, e->stream>>>(
      sh, e->quad.view(), n_pairs, e->mis_u0, e->mis_du, e->mis_tab.get());
    count_launch();
    if ((rc = cuda_status(cudaGetLastError(), "mis_table_kernel"))) return fail(rc);
  }
  // Device memory against the HBM budget.
  const size_t N = cfg->max_points;
  size_t bytes = N * sizeof(PointDev) + N * L.stride * 8 + N * e->s64_stride * 8 +
                 N * e->s32_stride * 4 + 2 * N * e->nB_max * (size_t)e->w_stride * 8 +
                 N * e->nB_max * 8 + (2 * N + 1) * sizeof(int) +
                 2 * N * (size_t)e->tile_cap_pp * sizeof(int);
  for (const auto& g : e->grids)
    e->f_stride = std::max(e->f_stride, (size_t)(g.n_m_pad / kGemmRows) * (g.n_t_pad / 16) *
                                          kFStageBytes);
  bytes += N * e->f_stride;
  if (cfg->with_shear)
    bytes += N * (size_t)e->nI_max * sh.n_R * e->w_stride * 8 + N * e->nB_max * sh.n_R * 8;
  const size_t budget = cfg->hbm_budget ? cfg->hbm_budget : (size_t)150 << 30;
  if (bytes > budget) {
    set_error("y3b_engine_create: %zu bytes for %d points exceed the HBM budget of %zu bytes",
              bytes, cfg->max_points, budget);
    return fail(Y3B_ERR_BUDGET);
  }
  e->device_bytes = bytes;
  if ((rc = e->pts.alloc(N)) || (rc = e->tables.alloc(N * L.stride)) ||
      (rc = e->s64.alloc(N * e->s64_stride)) || (rc = e->s32.alloc(N * e->s32_stride)) ||
      (rc = e->W.alloc(N * e->nB_max * (size_t)e->w_stride)) ||
      (rc = e->Wg.alloc(N * e->nB_max * (size_t)e->w_stride)) ||
      (rc = e->counts.alloc(N * e->nB_max)) || (rc = e->status.alloc(1)) ||
      (rc = e->stage_ct.alloc(2)) ||
      (rc = e->order.alloc(N)) || (rc = e->tile_start.alloc(N + 1)) ||
      (rc = e->tile_list.alloc(N * (size_t)e->tile_cap_pp)) ||
      (rc = e->win_tile.alloc(N * (size_t)e->tile_cap_pp)) ||
      (rc = e->fbuf.alloc(N * e->f_stride)))
    return fail(rc);
  if (cfg->with_shear) {
    if ((rc = e->Phi.alloc(N * (size_t)e->nI_max * sh.n_R * e->w_stride)) ||
        (rc = e->shear_out.alloc(N * e->nB_max * (size_t)sh.n_R)))
      return fail(rc);
  }
  // Zero the weight buffers once: rows a grid does not fill stay zero.
  rc = cuda_status(cudaMemsetAsync(e->W.get(), 0, e->W.size() * 8, e->stream), "memset");
  if (!rc) rc = cuda_status(cudaMemsetAsync(e->Wg.get(), 0, e->Wg.size() * 8, e->stream), "memset");
  if (!rc) rc = e->d_grids.upload(e->grids.data(), e->grids.size(), e->stream);
  if (!rc) rc = cuda_status(cudaStreamSynchronize(e->stream), "sync");
  if (rc) return fail(rc);
  Y3B_CUDA(cudaFuncSetAttribute(prep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)e->prep_smem));
  Y3B_CUDA(cudaFuncSetAttribute(yf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)e->yf_smem));
  // Several 256-thread CTAs per SM (three for yf_kernel, the register limit,
  // at ~37 KB each at 256 lnM x 128 z nodes): ask for the largest carveout.
  Y3B_CUDA(cudaFuncSetAttribute(prep_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared));
  Y3B_CUDA(cudaFuncSetAttribute(yf_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared));
  Y3B_CUDA(cudaFuncSetAttribute(direct_main_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)e->direct_smem));
  *out = e;
  return Y3B_OK;
}

extern "C" size_t
y3b_engine_table_stride(const y3b_engine* e)
{
  return e ? e->lay.stride : 0;
}

extern "C" int
y3b_engine_table_offsets(const y3b_engine* e, size_t* off7)
{
  if (!e || !off7) return Y3B_ERR_INVALID;
  for (int i = 0; i < 7; ++i) off7[i] = e->lay.off[i];
  return Y3B_OK;
}

extern "C" int
y3b_engine_n_bins(const y3b_engine* e)
{
  return e ? e->nB_max : 0;
}

extern "C" size_t
y3b_engine_device_bytes(const y3b_engine* e)
{
  return e ? e->device_bytes : 0;
}

namespace y3b {

// Enqueue one evaluation on `s`.  grid_mask selects the grids present.
// Records an event pair around one stage when profiling is on.
struct StageTimer {
  y3b_engine* e;
  cudaStream_t s;
  int stage;
  cudaEvent_t a = nullptr;
  StageTimer(y3b_engine* e_, cudaStream_t s_, int st) : e(e_), s(s_), stage(st)
  {
    if (e->prof && cudaEventCreate(&a) == cudaSuccess) cudaEventRecord(a, s);
  }
  ~StageTimer()
  {
    if (!a) return;
    cudaEvent_t b;
    if (cudaEventCreate(&b) == cudaSuccess) {
      cudaEventRecord(b, s);
      e->pending.push_back({stage, a, b});
    } else {
      cudaEventDestroy(a);
    }
  }
};

// w_off: index of the call's first point in the engine's W / W^g / Phi
// buffers (a chunked evaluation keeps every chunk's weights).
static int
enqueue(y3b_engine* e, int prec, int n, const PointDev* d_pts, const double* d_tables,
        const int* d_slot, double* d_counts, double* d_shear, cudaStream_t s, int grid_mask,
        size_t w_off = 0)
{
  double* W = e->W.get() + w_off * e->nB_max * e->w_stride;
  double* Wg = e->Wg.get() + w_off * e->nB_max * e->w_stride;
  double* Phi = e->Phi.get() ? e->Phi.get() + w_off * e->nI_max * e->shear.n_R * e->w_stride
                             : nullptr;
  if (prec == Y3B_FP64 && e->lay.hmf_f32) {
    set_error("an engine with FP32 dndlnmh tables (hmf_fp32) evaluates the mixed form only");
    return Y3B_ERR_INVALID;
  }
  Y3B_CUDA(cudaMemsetAsync(e->status.get(), 0, sizeof(int), s));
  // The stage counters cover one evaluation call: zeroed by its first chunk.
  if (w_off == 0 && prec == Y3B_MIXED)
    Y3B_CUDA(cudaMemsetAsync(e->stage_ct.get(), 0, 2 * sizeof(int), s));
  if (e->prof) ++e->prof_evals;
  PrepArgs pa{e->d_grids.get(), d_pts, d_tables, d_slot, e->lay, prec == Y3B_MIXED,
              e->s64.get(), e->s32.get(), e->status.get(), grid_mask, e->fbuf.get(), e->f_stride,
              e->win_tile.get(), e->tile_cap_pp};
  ContractLaunch L{e->d_grids.get(), (int)e->grids.size(), grid_mask, d_pts, n,
                   e->order.get(), e->tile_start.get(), e->tile_list.get(), e->win_tile.get(),
                   e->tile_cap_pp, (long long)n * e->max_tiles_pp, e->cshape, e->cstages,
                   e->n_ctas, e->fbuf.get(), e->f_stride, e->s32.get(), W, Wg, e->w_stride,
                   e->status.get(), e->stage_ct.get(), e->pstream, s,
                   e->cfg.with_shear && d_shear != nullptr};
  // Mixed form: the tile planner runs on its own stream beside the prep
  // kernel (it reads only the points and grids) and joins before the
  // contraction.  The fork comes after everything already on `s`, so a
  // previous evaluation's contraction has finished with the tile list.
  const bool mixed = prec == Y3B_MIXED;
  if (mixed) {
    Y3B_TRY(contract_check(L));
    Y3B_CUDA(cudaEventRecord(e->plan_fork, s));
    Y3B_CUDA(cudaStreamWaitEvent(e->pstream, e->plan_fork, 0));
    const int prc = launch_plan(L);
    Y3B_CUDA(cudaEventRecord(e->plan_join, e->pstream));
    if (prc) {  // join before returning, so that a capture in progress stays whole
      cudaStreamWaitEvent(s, e->plan_join, 0);
      return prc;
    }
  }
  {
    StageTimer t(e, s, 0);
    prep_kernel<<<n, kPrepThreads, e->prep_smem, s>>>(pa);
    count_launch();
    cudaError_t perr = cudaGetLastError();
    if (mixed && perr == cudaSuccess) {
      yf_kernel<<<dim3(n, e->max_mtiles), 256, e->yf_smem, s>>>(pa);
      count_launch();
      perr = cudaGetLastError();
    }
    if (mixed) Y3B_CUDA(cudaStreamWaitEvent(s, e->plan_join, 0));
    Y3B_CUDA(perr);
  }
  StageTimer* tc = new StageTimer(e, s, 1);
  if (prec == Y3B_FP64) {
    dim3 g1(e->nz_max, n);
    direct_main_kernel<<<g1, 256, e->direct_smem, s>>>(e->d_grids.get(), d_pts, e->s64.get(),
                                                       grid_mask);
    count_launch();
    Y3B_CUDA(cudaGetLastError());
    direct_wreduce_kernel<<<n, 256, 0, s>>>(e->d_grids.get(), d_pts, e->s64.get(), W, Wg,
                                            e->w_stride, grid_mask);
    count_launch();
    Y3B_CUDA(cudaGetLastError());
  } else {
    const int rc = launch_contract(L);
    if (rc) {
      delete tc;
      return rc;
    }
  }
  delete tc;
  const bool shear = e->cfg.with_shear && d_shear;
  if (shear) {
    StageTimer t(e, s, 2);
    long long warps = (long long)n * e->nI_max * e->shear.n_R * e->w_stride;
    long long blocks = (warps * 32 + 127) / 128;
    if (prec == Y3B_FP64)
      shear_phi_kernel<double><<<(unsigned)blocks, 128, 0, s>>>(
        e->d_grids.get(), d_pts, n, e->w_stride, e->shear, e->quad.view(), Phi,
        e->nI_max, grid_mask);
    else
      shear_tab_kernel<<<(unsigned)(((long long)n * e->w_stride + 127) / 128), 128, 0, s>>>(
        e->d_grids.get(), d_pts, n, e->w_stride, e->shear, e->mis_tab.get(), e->mis_u0,
        1.0 / e->mis_du, Phi, e->nI_max, grid_mask, e->status.get());
    count_launch();
    Y3B_CUDA(cudaGetLastError());
  }
  {
    StageTimer t(e, s, 3);
    // The likelihood needs the shear when its data vector has one.
    const bool like = e->like.on && (e->like.n_R == 0 || shear);
    finalize_kernel<<<n, 256, 0, s>>>(e->d_grids.get(), d_pts, W, Wg,
                                      shear ? Phi : nullptr, e->w_stride, e->nB_max,
                                      e->nI_max, e->shear.n_R, d_counts,
                                      shear ? d_shear : nullptr, grid_mask, e->like,
                                      like ? e->logL.get() + w_off : nullptr);
    count_launch();
    Y3B_CUDA(cudaGetLastError());
  }
  e->last_n = n;
  return Y3B_OK;
}

constexpr size_t kMaxGraphs = 16;
constexpr size_t kSeenKeys = 32;

// Runs one evaluation on `s`.  With graphs on (and stage timing off), an
// evaluation whose arguments were seen before is captured once into a CUDA
// graph and replayed from then on: one host launch for the whole sequence
// (status reset, prep, planner, contraction, profiles, final sums).  The
// graph holds the device pointers of the call, so the buffers must be the
// same ones (same addresses) when it is replayed, as they are for a repeated
// call.
static int
run(y3b_engine* e, int prec, int n, const PointDev* d_pts, const double* d_tables,
    const int* d_slot, double* d_counts, double* d_shear, cudaStream_t s, int grid_mask,
    size_t w_off = 0)
{
  if (e->graph_mode == 0 || e->prof)
    return enqueue(e, prec, n, d_pts, d_tables, d_slot, d_counts, d_shear, s, grid_mask, w_off);
  const y3b_engine::GraphKey key{prec,   n,        grid_mask, d_pts, d_tables,
                                 d_slot, d_counts, d_shear,   w_off};
  ++e->graph_clock;
  for (auto& g : e->graphs)
    if (g.key == key) {
      g.used = e->graph_clock;
      Y3B_CUDA(cudaGraphLaunch(g.exec, s));
      count_launch((unsigned)g.kernels);
      e->last_n = n;
      return Y3B_OK;
    }
  bool repeated = false;
  for (const auto& k : e->seen) repeated |= k == key;
  if (!repeated) {
    if (e->seen.size() >= kSeenKeys) e->seen.erase(e->seen.begin());
    e->seen.push_back(key);
    return enqueue(e, prec, n, d_pts, d_tables, d_slot, d_counts, d_shear, s, grid_mask, w_off);
  }
  // Capture.  The kernels counted while capturing are the ones the first
  // replay below runs.
  const unsigned long long before = g_launches.load();
  Y3B_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  const int rc =
    enqueue(e, prec, n, d_pts, d_tables, d_slot, d_counts, d_shear, s, grid_mask, w_off);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(s, &graph);
  if (rc != Y3B_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  Y3B_CUDA(ce);
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  Y3B_CUDA(ie);
  if (e->graphs.size() >= kMaxGraphs) {  // evict the least recently used
    size_t lru = 0;
    for (size_t i = 1; i < e->graphs.size(); ++i)
      if (e->graphs[i].used < e->graphs[lru].used) lru = i;
    cudaGraphExecDestroy(e->graphs[lru].exec);
    e->graphs.erase(e->graphs.begin() + lru);
  }
  e->graphs.push_back({key, exec, g_launches.load() - before, e->graph_clock});
  Y3B_CUDA(cudaGraphLaunch(exec, s));
  e->last_n = n;
  return Y3B_OK;
}

}  // namespace y3b

extern "C" int
y3b_engine_eval_device(y3b_engine* e, int precision, int n, const y3b_point* pts_dev,
                       const double* tables_dev, double* counts_dev, double* shear_dev,
                       void* stream)
{
  clear_error();
  if (!e || n < 1 || n > e->cfg.max_points || !pts_dev || !tables_dev || !counts_dev ||
      (precision != Y3B_FP64 && precision != Y3B_MIXED)) {
    set_error("y3b_engine_eval_device: invalid arguments (1 <= n <= max_points)");
    return Y3B_ERR_INVALID;
  }
  if (((uintptr_t)tables_dev & 15u) != 0) {
    set_error("y3b_engine_eval_device: tables must be 16-byte aligned");
    return Y3B_ERR_INVALID;
  }
  static_assert(sizeof(y3b_point) == sizeof(PointDev), "y3b_point layout");
  cudaStream_t s = stream ? (cudaStream_t)stream : e->stream;
  int mask = (1 << (int)e->grids.size()) - 1;
  return run(e, precision, n, reinterpret_cast<const PointDev*>(pts_dev), tables_dev,
                 nullptr, counts_dev, shear_dev, s, mask);
}

extern "C" int
y3b_engine_eval_pooled(y3b_engine* e, int precision, int n, const y3b_point* pts_dev,
                       const double* pool_dev, const int* slot_dev, double* counts_dev,
                       double* shear_dev, void* stream)
{
  clear_error();
  if (!e || n < 1 || n > e->cfg.max_points || !pts_dev || !pool_dev || !slot_dev ||
      !counts_dev || (precision != Y3B_FP64 && precision != Y3B_MIXED)) {
    set_error("y3b_engine_eval_pooled: invalid arguments (1 <= n <= max_points)");
    return Y3B_ERR_INVALID;
  }
  if (((uintptr_t)pool_dev & 15u) != 0) {
    set_error("y3b_engine_eval_pooled: the table pool must be 16-byte aligned");
    return Y3B_ERR_INVALID;
  }
  cudaStream_t s = stream ? (cudaStream_t)stream : e->stream;
  int mask = (1 << (int)e->grids.size()) - 1;
  return run(e, precision, n, reinterpret_cast<const PointDev*>(pts_dev), pool_dev,
                 slot_dev, counts_dev, shear_dev, s, mask);
}

int
y3b::engine_check_points(const y3b_engine* e, int n, const y3b_point* pts, int* mask)
{
  *mask = 0;
  for (int i = 0; i < n; ++i) {
    const y3b_point& p = pts[i];
    if (p.grid < 0 || p.grid >= (int)e->grids.size()) {
      set_error("point %d has grid %d outside [0, %d)", i, p.grid, (int)e->grids.size());
      return Y3B_ERR_INVALID;
    }
    if (!(p.sigma > 0.0) || !(p.Mpiv > 0.0) || !(p.cosmo.om - p.cosmo.onu > 0.0) ||
        !(p.cosmo.h0 > 0.0)) {
      set_error("point %d has non-positive sigma, Mpiv, h0 or omega_M - omega_nu", i);
      return Y3B_ERR_INVALID;
    }
    *mask |= 1 << p.grid;
  }
  return Y3B_OK;
}

int
y3b::engine_check_tables(const y3b_engine* e, int n, const y3b_point* pts, const double* tables)
{
  const size_t st = e->lay.stride;
  const int nd = e->lay.n_dist;
  for (int i = 0; i < n; ++i) {
    const double* dz = tables + (size_t)i * st + e->lay.off[3];
    const auto& zr = e->zt_node_range[pts[i].grid];
    if (!(dz[0] <= zr[0] && zr[1] <= dz[nd - 1])) {
      set_error("point %d: distances/z [%g, %g] does not cover the z_t nodes [%g, %g] of its "
                "grid", i, dz[0], dz[nd - 1], zr[0], zr[1]);
      return Y3B_ERR_DOMAIN;
    }
  }
  return Y3B_OK;
}

void
y3b::engine_info(const y3b_engine* e, EngineInfo* out)
{
  out->n_grids = (int)e->grids.size();
  out->n_bins = e->nB_max;
  out->n_R = e->cfg.with_shear ? e->shear.n_R : 0;
  out->with_shear = e->cfg.with_shear;
  out->max_points = e->cfg.max_points;
  out->stride = e->lay.stride;
  out->device_bytes = e->device_bytes;
}

int
y3b::engine_status_to_host(y3b_engine* e, int* host, cudaStream_t s)
{
  Y3B_CUDA(cudaMemcpyAsync(host, e->status.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  return Y3B_OK;
}

extern "C" int
y3b_engine_set_graphs(y3b_engine* e, int mode)
{
  clear_error();
  if (!e || (mode != 0 && mode != 1)) {
    set_error("y3b_engine_set_graphs: mode must be 0 (off) or 1 (on)");
    return Y3B_ERR_INVALID;
  }
  e->graph_mode = mode;
  if (mode == 0) {
    Y3B_CUDA(cudaStreamSynchronize(e->stream));
    for (auto& g : e->graphs) cudaGraphExecDestroy(g.exec);
    e->graphs.clear();
    e->seen.clear();
  }
  return Y3B_OK;
}

extern "C" int
y3b_engine_sync(y3b_engine* e, void* stream)
{
  clear_error();
  if (!e) return Y3B_ERR_INVALID;
  cudaStream_t s = stream ? (cudaStream_t)stream : e->stream;
  return read_device_status(e->status.get(), s);
}

extern "C" int
y3b_engine_eval(y3b_engine* e, int precision, int n, const y3b_point* pts,
                const double* tables, double* counts, double* shear)
{
  clear_error();
  if (!e || n < 1 || n > e->cfg.max_points || !pts || !tables || !counts ||
      (precision != Y3B_FP64 && precision != Y3B_MIXED)) {
    set_error("y3b_engine_eval: invalid arguments (1 <= n <= max_points)");
    return Y3B_ERR_INVALID;
  }
  int mask = 0;
  Y3B_TRY(y3b::engine_check_points(e, n, pts, &mask));
  // Chunked: chunk c's points and tables are copied on the copy stream while
  // chunk c-1 is evaluated on the compute stream (with pinned host buffers
  // the copies overlap the kernels).  Chunks run one after the other on the
  // compute stream, so they share the per-point scratch; their weights and
  // outputs land at their own offsets.
  cudaStream_t s = e->stream, xs = e->xstream;
  // About 256 points a chunk: the copies are the long pole, and only the
  // last chunk's kernels run after them.
  // Chunks of about 12.5 MB of host tables (at least 256 points, at most
  // eight): the copy of the next chunk then outlasts the evaluation of the
  // current one, whose fixed cost grows relative to its work as chunks
  // shrink.  On one B200 over PCIe, 2048 points with FP32-HMF tables
  // (25.5 KB per point) ran at 1.28 / 1.49 / 1.58 / 1.66 M points/s in
  // 8 / 2 / 3 / 4 chunks, with FP64 tables (45.5 KB) best in eight.
  const size_t st = e->lay.stride;
  const double host_bytes = (double)n * (double)(st * sizeof(double) + sizeof(y3b_point));
  int chunks = (int)std::min<double>(y3b::kEvalChunks, std::max(1.0, std::floor(host_bytes / 12.5e6)));
  chunks = std::max(1, std::min(chunks, n / 256));
  const int csz = (n + chunks - 1) / chunks;
  const int nB = e->nB_max, nR = e->shear.n_R;
  const bool want_shear = e->cfg.with_shear && shear;
  int used = 0;
  auto upload = [&]() -> int {
    for (int c = 0; c < chunks; ++c) {
      const int off = c * csz, m = std::min(csz, n - off);
      if (m <= 0) break;
      Y3B_CUDA(cudaMemcpyAsync(e->pts.get() + off, pts + off, m * sizeof(y3b_point),
                               cudaMemcpyHostToDevice, xs));
      Y3B_CUDA(cudaMemcpyAsync(e->tables.get() + off * st, tables + off * st,
                               m * st * sizeof(double), cudaMemcpyHostToDevice, xs));
      Y3B_CUDA(cudaEventRecord(e->chunk_ev[c], xs));
      used = c + 1;
    }
    return Y3B_OK;
  };
  if (const int rc = upload()) {
    cudaStreamSynchronize(xs);
    return rc;
  }
  auto evaluate = [&]() -> int {
    for (int c = 0; c < used; ++c) {
      const int off = c * csz, m = std::min(csz, n - off);
      Y3B_CUDA(cudaStreamWaitEvent(s, e->chunk_ev[c], 0));
      Y3B_TRY(run(e, precision, m, e->pts.get() + off, e->tables.get() + off * st, nullptr,
                  e->counts.get() + (size_t)off * nB,
                  want_shear ? e->shear_out.get() + (size_t)off * nB * nR : nullptr, s, mask,
                  (size_t)off));
      Y3B_TRY(y3b::engine_status_to_host(e, e->chunk_status + c, s));
      Y3B_CUDA(cudaMemcpyAsync(counts + (size_t)off * nB, e->counts.get() + (size_t)off * nB,
                               (size_t)m * nB * sizeof(double), cudaMemcpyDeviceToHost, s));
      if (want_shear)
        Y3B_CUDA(cudaMemcpyAsync(shear + (size_t)off * nB * nR,
                                 e->shear_out.get() + (size_t)off * nB * nR,
                                 (size_t)m * nB * nR * sizeof(double), cudaMemcpyDeviceToHost,
                                 s));
    }
    return Y3B_OK;
  };
  if (const int rc = evaluate()) {
    // Nothing queued may touch the caller's buffers after we return.
    cudaStreamSynchronize(xs);
    cudaStreamSynchronize(s);
    return rc;
  }
  Y3B_CUDA(cudaStreamSynchronize(s));
  e->last_n = n;
  for (int c = 0; c < used; ++c) {
    const int h = e->chunk_status[c];
    if (h != y3b::kDevOk) return y3b::device_status_rc(h);
  }
  return Y3B_OK;
}

extern "C" int
y3b_engine_weights(y3b_engine* e, int n, double* W)
{
  clear_error();
  if (!e || !W || n < 1 || n > e->last_n) {
    set_error("y3b_engine_weights: n must be within the last evaluation");
    return Y3B_ERR_INVALID;
  }
  Y3B_CUDA(cudaStreamSynchronize(e->stream));
  Y3B_CUDA(cudaMemcpy(W, e->W.get(), (size_t)n * e->nB_max * e->w_stride * sizeof(double),
                      cudaMemcpyDeviceToHost));
  return Y3B_OK;
}

extern "C" int
y3b_engine_stage_count(const y3b_engine* e, long long* executed, long long* dense)
{
  clear_error();
  if (!e || !executed || !dense) return Y3B_ERR_INVALID;
  int h[2] = {0, 0};
  if (e->stage_ct.get())
    Y3B_CUDA(cudaMemcpy(h, e->stage_ct.get(), sizeof(h), cudaMemcpyDeviceToHost));
  *executed = h[0];
  *dense = h[1];
  return Y3B_OK;
}

extern "C" int
y3b_engine_profile(y3b_engine* e, int enable)
{
  clear_error();
  if (!e) return Y3B_ERR_INVALID;
  if (enable) {
    for (auto& p : e->pending) {
      cudaEventDestroy(p.a);
      cudaEventDestroy(p.b);
    }
    e->pending.clear();
    for (double& v : e->prof_ms) v = 0.0;
    e->prof_evals = 0;
  }
  e->prof = enable != 0;
  return Y3B_OK;
}

extern "C" int
y3b_engine_profile_read(y3b_engine* e, double* ms, int* n_evals)
{
  clear_error();
  if (!e || !ms) return Y3B_ERR_INVALID;
  for (auto& p : e->pending) {
    Y3B_CUDA(cudaEventSynchronize(p.b));
    float t = 0.f;
    Y3B_CUDA(cudaEventElapsedTime(&t, p.a, p.b));
    e->prof_ms[p.stage] += t;
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  e->pending.clear();
  for (int i = 0; i < 4; ++i) ms[i] = e->prof_ms[i];
  if (n_evals) *n_evals = e->prof_evals;
  return Y3B_OK;
}

// ---------------------------------------------------------------------------
// Autotuner: ring depth of the contraction and richness bins per tile of each
// grid, chosen by timing the contraction stage on the caller's batch.

namespace y3b {

// Mean contraction milliseconds of `reps` evaluations with the current
// settings (one untimed evaluation first).
static int
time_contraction(y3b_engine* e, int n, const PointDev* d_pts, const double* d_tables,
                 double* d_counts, cudaStream_t s, int reps, double* ms)
{
  Y3B_TRY(enqueue(e, Y3B_MIXED, n, d_pts, d_tables, nullptr, d_counts, nullptr, s,
                  (1 << (int)e->grids.size()) - 1));
  Y3B_TRY(y3b_engine_profile(e, 1));
  for (int r = 0; r < reps; ++r)
    Y3B_TRY(enqueue(e, Y3B_MIXED, n, d_pts, d_tables, nullptr, d_counts, nullptr, s,
                    (1 << (int)e->grids.size()) - 1));
  double st[4];
  int ne = 0;
  const int rc = y3b_engine_profile_read(e, st, &ne);
  y3b_engine_profile(e, 0);
  Y3B_TRY(rc);
  Y3B_TRY(read_device_status(e->status.get(), s));
  *ms = st[1] / std::max(ne, 1);
  return Y3B_OK;
}

static int
upload_grids(y3b_engine* e)
{
  rank_grids(e);
  Y3B_TRY(e->d_grids.upload(e->grids.data(), e->grids.size(), e->stream));
  Y3B_CUDA(cudaStreamSynchronize(e->stream));
  return Y3B_OK;
}

}  // namespace y3b

extern "C" int
y3b_engine_autotune(y3b_engine* e, int n, const y3b_point* pts_dev, const double* tables_dev,
                    double* counts_dev, double* best_ms)
{
  using namespace y3b;
  clear_error();
  if (!e || n < 1 || n > e->cfg.max_points || !pts_dev || !tables_dev || !counts_dev ||
      ((uintptr_t)tables_dev & 15u) != 0) {
    set_error("y3b_engine_autotune: invalid arguments (1 <= n <= max_points, 16-byte aligned "
              "tables)");
    return Y3B_ERR_INVALID;
  }
  // Tuning changes kernel arguments that captured graphs hold: drop them.
  const int mode = e->graph_mode;
  Y3B_TRY(y3b_engine_set_graphs(e, 0));
  const PointDev* pts = reinterpret_cast<const PointDev*>(pts_dev);
  cudaStream_t s = e->stream;
  constexpr int kReps = 3;
  double best = 0.0;
  int rc = time_contraction(e, n, pts, tables_dev, counts_dev, s, kReps, &best);
  // 1. ring depth
  const int st_max = contract_stages(e->cshape);
  int best_st = e->cstages;
  for (int st : {2, 3, 4, 6, 8}) {
    if (rc || st > st_max || st == best_st) continue;
    const int keep = e->cstages;
    e->cstages = st;
    double ms = 0.0;
    rc = time_contraction(e, n, pts, tables_dev, counts_dev, s, kReps, &ms);
    if (!rc && ms < best) {
      best = ms;
      best_st = st;
    } else {
      e->cstages = keep;
    }
  }
  e->cstages = best_st;
  // 2. bins per tile, grid by grid
  for (size_t g = 0; g < e->grids.size() && !rc; ++g) {
    GridDev& gd = e->grids[g];
    const int nic_max = std::max(1, std::min(gd.nI, 256 / gd.n_z));
    int best_nic = gd.nIc;
    for (int nic : {1, 2, 4, 8}) {
      if (rc || nic > nic_max || nic == best_nic) continue;
      set_bins_per_tile(gd, nic);
      if ((rc = upload_grids(e))) break;
      double ms = 0.0;
      rc = time_contraction(e, n, pts, tables_dev, counts_dev, s, kReps, &ms);
      if (!rc && ms < best) {
        best = ms;
        best_nic = nic;
      }
    }
    set_bins_per_tile(gd, best_nic);
    const int urc = upload_grids(e);
    if (!rc) rc = urc;
  }
  const int grc = y3b_engine_set_graphs(e, mode);
  if (rc) return rc;
  Y3B_TRY(grc);
  if (best_ms) *best_ms = best;
  return Y3B_OK;
}

extern "C" int
y3b_engine_tuning(const y3b_engine* e, int* stages, int* bins_per_tile, int cap)
{
  y3b::clear_error();
  if (!e || !stages || !bins_per_tile || cap < (int)e->grids.size()) {
    y3b::set_error("y3b_engine_tuning: need room for one entry per grid");
    return Y3B_ERR_INVALID;
  }
  *stages = e->cstages;
  for (size_t g = 0; g < e->grids.size(); ++g) bins_per_tile[g] = e->grids[g].nIc;
  return Y3B_OK;
}

// ===========================================================================
// Gaussian likelihood (y3_buzzard/likelihood_cp.py:94-200).
namespace y3b {

// Host side of likelihood_cp.setup(): checks the sizes and, in log space,
// stores ln(data) and the delta-method inverse covariance invcov * d d^T
// (likelihood_cp.py:79-92, 113-118).  The device copy is one buffer.
static int
like_upload(const y3b_likelihood* L, DevBuf<double>& buf, LikeDev* out, cudaStream_t s)
{
  const int nB = L->n_bins, nR = L->n_R, nsh = nB * nR;
  if (nB < 1 || nB > kMaxLamBins * kMaxZBins || nR < 0 || nR > kMaxR || !L->data_nc ||
      !L->invcov_nc || (nsh && (!L->data_sh || !L->invcov_sh))) {
    set_error("likelihood: need 1 <= n_bins <= %d, 0 <= n_R <= %d and the data and inverse "
              "covariance of each observable", kMaxLamBins * kMaxZBins, kMaxR);
    return Y3B_ERR_INVALID;
  }
  const size_t icn = L->nc_dense ? (size_t)nB * nB : nB;
  const size_t ics = L->sh_dense ? (size_t)nsh * nsh : nsh;
  std::vector<double> h;
  h.reserve(nB + icn + nsh + ics + (L->shear_prj ? nsh : 0));
  auto put = [&](const double* d, const double* ic, int n, int dense) -> int {
    for (int i = 0; i < n; ++i) {
      if (!std::isfinite(d[i]) || (L->log_space && !(d[i] > 0.0))) {
        set_error("likelihood: %s data entry %d (log space requires data > 0)",
                  std::isfinite(d[i]) ? "non-positive" : "non-finite", i);
        return Y3B_ERR_INVALID;
      }
      h.push_back(L->log_space ? std::log(d[i]) : d[i]);
    }
    const size_t m = dense ? (size_t)n * n : n;
    for (size_t u = 0; u < m; ++u) {
      const size_t i = dense ? u / n : u, j = dense ? u % n : u;
      h.push_back(L->log_space ? ic[u] * d[i] * d[j] : ic[u]);
    }
    return Y3B_OK;
  };
  Y3B_TRY(put(L->data_nc, L->invcov_nc, nB, L->nc_dense != 0));
  if (nsh) Y3B_TRY(put(L->data_sh, L->invcov_sh, nsh, L->sh_dense != 0));
  if (nsh && L->shear_prj) h.insert(h.end(), L->shear_prj, L->shear_prj + nsh);
  Y3B_TRY(buf.upload(h.data(), h.size(), s));
  Y3B_CUDA(cudaStreamSynchronize(s));
  const double* d = buf.get();
  LikeDev& o = *out;
  o.on = 1;
  o.log_space = L->log_space != 0;
  o.n_R = nR;
  o.nc_dense = L->nc_dense != 0;
  o.sh_dense = L->sh_dense != 0;
  o.data_nc = d;
  o.ic_nc = d + nB;
  o.data_sh = nsh ? o.ic_nc + icn : nullptr;
  o.ic_sh = nsh ? o.data_sh + nsh : nullptr;
  o.prj = nsh && L->shear_prj ? o.ic_sh + ics : nullptr;
  return Y3B_OK;
}

// One data vector (the CosmoSIS likelihood module's case).
__global__ void __launch_bounds__(256)
loglike_kernel(LikeDev L, int nB, const double* nc, const double* sh, double* out)
{
  __shared__ double s_nc[kMaxLamBins * kMaxZBins];
  __shared__ double s_sh[kMaxLamBins * kMaxZBins * kMaxR];
  __shared__ double s_red[256];
  for (int b = threadIdx.x; b < nB; b += blockDim.x) s_nc[b] = nc[b];
  for (int u = threadIdx.x; u < nB * L.n_R; u += blockDim.x) s_sh[u] = sh[u];
  __syncthreads();
  const double v = gaussian_loglike_block(L, nB, L.n_R, s_nc, s_sh, s_red);
  if (threadIdx.x == 0) *out = v;
}

}  // namespace y3b

extern "C" int
y3b_engine_set_likelihood(y3b_engine* e, const y3b_likelihood* L)
{
  using namespace y3b;
  clear_error();
  if (!e) return Y3B_ERR_INVALID;
  // Captured graphs hold the previous settings: drop them (they are
  // re-captured on repeat).
  const int mode = e->graph_mode;
  Y3B_TRY(y3b_engine_set_graphs(e, 0));
  e->graph_mode = mode;
  e->like = LikeDev{};
  if (!L) return Y3B_OK;
  for (const auto& g : e->grids)
    if (g.nB != L->n_bins) {
      set_error("y3b_engine_set_likelihood: n_bins %d differs from a grid's %d bins", L->n_bins,
                g.nB);
      return Y3B_ERR_INVALID;
    }
  if (L->n_R && (!e->cfg.with_shear || L->n_R != e->shear.n_R)) {
    set_error("y3b_engine_set_likelihood: a shear data vector needs an engine with shear and "
              "the same %d radii", e->shear.n_R);
    return Y3B_ERR_INVALID;
  }
  LikeDev ld{};
  Y3B_TRY(like_upload(L, e->like_buf, &ld, e->stream));
  Y3B_TRY(e->logL.alloc(e->cfg.max_points));
  e->like = ld;
  return Y3B_OK;
}

extern "C" int
y3b_engine_loglike(y3b_engine* e, int n, double* logL, void* stream)
{
  using namespace y3b;
  clear_error();
  if (!e || !logL || n < 1 || n > e->cfg.max_points || !e->like.on) {
    set_error("y3b_engine_loglike: no likelihood set, or n outside 1..max_points");
    return Y3B_ERR_INVALID;
  }
  cudaStream_t s = stream ? (cudaStream_t)stream : e->stream;
  Y3B_CUDA(cudaMemcpyAsync(logL, e->logL.get(), n * sizeof(double), cudaMemcpyDeviceToHost, s));
  Y3B_CUDA(cudaStreamSynchronize(s));
  return Y3B_OK;
}

extern "C" int
y3b_engine_eval_loglike(y3b_engine* e, int precision, int n, const y3b_point* pts,
                        const double* tables, double* logL)
{
  using namespace y3b;
  clear_error();
  if (!e || !logL || !e->like.on) {
    set_error("y3b_engine_eval_loglike: no likelihood set (y3b_engine_set_likelihood)");
    return Y3B_ERR_INVALID;
  }
  std::vector<double> counts((size_t)std::max(n, 0) * e->nB_max);
  std::vector<double> shear(e->like.n_R ? (size_t)std::max(n, 0) * e->nB_max * e->shear.n_R : 0);
  Y3B_TRY(y3b_engine_eval(e, precision, n, pts, tables, counts.data(),
                          e->like.n_R ? shear.data() : nullptr));
  return y3b_engine_loglike(e, n, logL, nullptr);
}

extern "C" int
y3b_gaussian_loglike(const y3b_likelihood* L, const double* counts, const double* shear_1h,
                     double* logL)
{
  using namespace y3b;
  clear_error();
  if (!L || !counts || !logL || (L->n_R && !shear_1h)) {
    set_error("y3b_gaussian_loglike: null argument");
    return Y3B_ERR_INVALID;
  }
  Y3B_TRY(require_device());
  DevBuf<double> buf, in, out;
  LikeDev ld{};
  Y3B_TRY(like_upload(L, buf, &ld, 0));
  const int nB = L->n_bins, nsh = nB * L->n_R;
  std::vector<double> h(counts, counts + nB);
  if (nsh) h.insert(h.end(), shear_1h, shear_1h + nsh);
  Y3B_TRY(in.upload(h.data(), h.size(), 0));
  Y3B_TRY(out.alloc(1));
  loglike_kernel<<<1, 256>>>(ld, nB, in.get(), nsh ? in.get() + nB : nullptr, out.get());
  count_launch();
  Y3B_CUDA(cudaGetLastError());
  Y3B_CUDA(cudaMemcpy(logL, out.get(), sizeof(double), cudaMemcpyDeviceToHost));
  return Y3B_OK;
}
