// ref_modules.cu -- reference-compatible FP64 kernels behind the CosmoSIS
// module boundary:
//   * y3b_sel_function   sel_function.py:555-615 (S_stack producer)
//   * y3b_selgl_*        SelGLCore / NumCountsSelGL / Shear1hMisSelGL,
//                        src/models/n_operator_sel_gl_t.hh:75-361
//   * y3b_sigma_crit_inv average_sigma_crit_inv.py:40-58
//   * y3b_nfw_mis        NFW_DSIGMA_MIS / NFW_SIGMA_MIS operator()
// All arithmetic is FP64 so the module outputs track the reference chain to
// <= 1e-8 relative.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "host_common.h"
#include "mis_quad.cuh"

namespace y3b {

// ---------------------------------------------------------------------------
// GL nodes on [a,b]: one thread per node pair.
__global__ void
gl_nodes_kernel(double a, double b, int n, double* xs, double* ws)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < (n + 1) / 2) gl_node_pair(a, b, n, i, xs, ws);
}

int
gl_nodes_device(double a, double b, int n, double* xs, double* ws, cudaStream_t s)
{
  int pairs = (n + 1) / 2;
  gl_nodes_kernel<<<(pairs + 127) / 128, 128, 0, s>>>(a, b, n, xs, ws);
  count_launch();
  return cuda_status(cudaGetLastError(), "gl_nodes_kernel");
}

// ---------------------------------------------------------------------------
// sel_function: one warp per (lnM, z) cell; lanes stride over the N_q GL
// lambda_t nodes of the cell's bracket (sel_function.py:516-547), evaluate the
// MOR density, the EMG CDF at the unique edges (195-226) and accumulate
// W_k (CDF[hi] - CDF[lo]) P per distinct edge pair; a fixed xor-tree warp
// reduction makes the sum order independent of scheduling.
constexpr int kMaxEdges = 32;
constexpr int kMaxPairs = 32;

struct SelFuncArgs {
  int n_lnm, n_z, n_q, n_bins, n_edges, n_pairs;
  double lnm_low, lnm_high, zt_low, zt_high;
  int mor_kind;
  double mor[8];
  int n_plob;
  const double* plob_z;
  const double* plob_coef;
  const double* edges;       // [n_edges]
  const int* pair_lo;        // [n_pairs] edge index
  const int* pair_hi;
  const int* bin_pair;       // [n_bins] -> pair
  const double* zob_min;     // [n_bins]
  const double* zob_max;
  const double* sigma_z;
  const double* gl_t;        // [n_q] on [-1,1]
  const double* gl_w;
  double* lnm_out;
  double* z_out;
  double* S_out;             // [n_bins][n_z][n_lnm]
};

__device__ __forceinline__ double
hod_mu_sat(double M, double z, const double* hod)
{
  double Mmin = pow(10.0, hod[0]), M1 = pow(10.0, hod[1]);
  double dM1 = M1 - Mmin;
  if (dM1 <= 0.0) return 0.0;
  double dM = fmax(M - Mmin, 0.0);
  double base = dM > 0.0 ? dM / dM1 : 0.0;
  if (!(base > 0.0)) return 0.0;
  return pow(base, hod[2]) * pow((1.0 + z) / (1.0 + hod[5]), hod[3]);
}

// P_HOD(ltr | M, z): sel_function.py:295-343.
__device__ __forceinline__ double
hod_density(double ltr, double M, double ms, double lcentral, const double* hod)
{
  double delta = (hod[4] * ms) * (hod[4] * ms);
  double nu = ms + delta;
  double density;
  if (ms <= 1e-8) {
    double t = (ltr - lcentral) / 1.0e-3;
    density = exp(-0.5 * t * t) / (kSqrt2Pi * 1.0e-3);
  } else {
    double x = ltr - lcentral + delta;
    density = x > 0.0 ? exp(-nu + (x - 1.0) * log(fmax(nu, 1e-300)) - lgamma(x)) : 0.0;
  }
  if (ltr < 0.0 || ltr < lcentral) density = 0.0;
  return density;
}

__global__ void __launch_bounds__(128)
sel_function_kernel(SelFuncArgs a)
{
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int n_cells = a.n_lnm * a.n_z;
  if (warp >= n_cells) return;
  const int m = warp / a.n_z;  // lnM index
  const int j = warp % a.n_z;  // z index
  const double lnM = a.n_lnm > 1 ? a.lnm_low + (a.lnm_high - a.lnm_low) * m / (a.n_lnm - 1)
                                 : a.lnm_low;
  const double z = a.n_z > 1 ? a.zt_low + (a.zt_high - a.zt_low) * j / (a.n_z - 1) : a.zt_low;
  const double M = exp(lnM);
  if (lane == 0) {
    if (j == 0) a.lnm_out[m] = lnM;
    if (m == 0) a.z_out[j] = z;
  }
  // Bracket (per cell).
  double lo, hi, mu_ln = 0.0, D = 1.0, ms = 0.0, lcentral = 0.0;
  if (a.mor_kind == Y3B_MOR_HOD) {
    ms = hod_mu_sat(M, z, a.mor);
    lcentral = (M >= pow(10.0, a.mor[0])) ? 1.0 : 0.0;
    double mu_eff = lcentral + ms;
    double sig_eff = sqrt(fmax(ms + (a.mor[4] * ms) * (a.mor[4] * ms), 0.0));
    lo = fmax(0.0, mu_eff - 6.0 * sig_eff);
    hi = mu_eff + 6.0 * sig_eff;
  } else {
    mu_ln = a.mor[0] + a.mor[1] * (lnM - log(a.mor[4])) + a.mor[2] * log1p(z);
    lo = fmax(a.mor[5], exp(mu_ln - 6.0 * a.mor[3]));
    hi = fmin(a.mor[6], exp(mu_ln + 6.0 * a.mor[3]));
    D = phi_diff((log(a.mor[5]) - mu_ln) / a.mor[3], (log(a.mor[6]) - mu_ln) / a.mor[3]);
  }
  const bool degenerate = !(hi > lo);
  const double half = 0.5 * (hi - lo), mid = 0.5 * (hi + lo);

  double acc[kMaxPairs];
  for (int p = 0; p < a.n_pairs; ++p) acc[p] = 0.0;
  for (int t = lane; t < a.n_q; t += 32) {
    double ltr = mid + half * a.gl_t[t];
    double W = half * a.gl_w[t];
    double P;
    if (a.mor_kind == Y3B_MOR_HOD) {
      P = hod_density(ltr, M, ms, lcentral, a.mor);
    } else {
      double d = (log(ltr) - mu_ln) / a.mor[3];
      P = exp(-0.5 * d * d) / (kSqrt2Pi * a.mor[3] * ltr * D);
    }
    double mu, sg, tau, fp;
    plob_params(a.n_plob, a.plob_z, a.plob_coef, ltr, z, &mu, &sg, &tau, &fp);
    double cdf[kMaxEdges];
    for (int e = 0; e < a.n_edges; ++e) cdf[e] = cdf_lob(a.edges[e], mu, sg, tau, fp);
    for (int p = 0; p < a.n_pairs; ++p)
      acc[p] += W * (cdf[a.pair_hi[p]] - cdf[a.pair_lo[p]]) * P;
  }
  for (int p = 0; p < a.n_pairs; ++p) {
    double v = acc[p];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    acc[p] = v;
  }
  if (lane == 0) {
    for (int k = 0; k < a.n_bins; ++k) {
      double Si = degenerate ? 0.0 : acc[a.bin_pair[k]];
      double Kj = phi_cdf((a.zob_max[k] - z) / a.sigma_z[k]) -
                  phi_cdf((a.zob_min[k] - z) / a.sigma_z[k]);
      a.S_out[((size_t)k * a.n_z + j) * a.n_lnm + m] = Si * Kj;
    }
  }
}

}  // namespace y3b

using namespace y3b;

extern "C" int
y3b_sel_function(const y3b_selfunc_config* cfg, const y3b_mor* mor,
                 const y3b_plob* plob, double* lnm_out, double* z_out, double* S_out)
{
  clear_error();
  if (!cfg || !mor || !plob || !lnm_out || !z_out || !S_out) {
    set_error("y3b_sel_function: null argument");
    return Y3B_ERR_INVALID;
  }
  if (cfg->n_bins <= 0 || cfg->n_lnm <= 0 || cfg->n_z <= 0 || cfg->n_q <= 0 ||
      plob->n < 1 || (mor->kind != Y3B_MOR_HOD && mor->kind != Y3B_MOR_LOGNORMAL)) {
    set_error("y3b_sel_function: invalid sizes or MOR kind");
    return Y3B_ERR_INVALID;
  }
  Y3B_TRY(require_device());
  const int nb = cfg->n_bins;
  // Unique sorted edges and per-bin edge pairs (np.unique + searchsorted,
  // sel_function.py:550-552, 592-599).
  std::vector<double> edges;
  for (int k = 0; k < nb; ++k) {
    edges.push_back(cfg->lam_min[k]);
    edges.push_back(cfg->lam_max[k]);
  }
  std::sort(edges.begin(), edges.end());
  edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
  if ((int)edges.size() > kMaxEdges) {
    set_error("y3b_sel_function: more than %d unique richness edges", kMaxEdges);
    return Y3B_ERR_UNSUPPORTED;
  }
  std::vector<int> plo, phi_, bin_pair(nb);
  for (int k = 0; k < nb; ++k) {
    int lo = int(std::lower_bound(edges.begin(), edges.end(), cfg->lam_min[k]) - edges.begin());
    int hi = int(std::lower_bound(edges.begin(), edges.end(), cfg->lam_max[k]) - edges.begin());
    int p = 0;
    for (; p < (int)plo.size(); ++p)
      if (plo[p] == lo && phi_[p] == hi) break;
    if (p == (int)plo.size()) {
      plo.push_back(lo);
      phi_.push_back(hi);
    }
    bin_pair[k] = p;
  }
  if ((int)plo.size() > kMaxPairs) {
    set_error("y3b_sel_function: more than %d distinct richness bins", kMaxPairs);
    return Y3B_ERR_UNSUPPORTED;
  }
  cudaStream_t s = 0;
  DevBuf<double> d_edges, d_zmin, d_zmax, d_sz, d_pz, d_pc, d_glt, d_glw, d_lnm, d_z, d_S;
  DevBuf<int> d_plo, d_phi, d_bp;
  Y3B_TRY(d_edges.upload(edges.data(), edges.size(), s));
  Y3B_TRY(d_zmin.upload(cfg->zob_min, nb, s));
  Y3B_TRY(d_zmax.upload(cfg->zob_max, nb, s));
  Y3B_TRY(d_sz.upload(cfg->sigma_z, nb, s));
  Y3B_TRY(d_pz.upload(plob->z, plob->n, s));
  Y3B_TRY(d_pc.upload(plob->coef, 8 * (size_t)plob->n, s));
  Y3B_TRY(d_plo.upload(plo.data(), plo.size(), s));
  Y3B_TRY(d_phi.upload(phi_.data(), phi_.size(), s));
  Y3B_TRY(d_bp.upload(bin_pair.data(), nb, s));
  Y3B_TRY(d_glt.alloc(cfg->n_q));
  Y3B_TRY(d_glw.alloc(cfg->n_q));
  Y3B_TRY(d_lnm.alloc(cfg->n_lnm));
  Y3B_TRY(d_z.alloc(cfg->n_z));
  size_t nS = (size_t)nb * cfg->n_z * cfg->n_lnm;
  Y3B_TRY(d_S.alloc(nS));
  Y3B_TRY(gl_nodes_device(-1.0, 1.0, cfg->n_q, d_glt.get(), d_glw.get(), s));

  SelFuncArgs a;
  a.n_lnm = cfg->n_lnm;
  a.n_z = cfg->n_z;
  a.n_q = cfg->n_q;
  a.n_bins = nb;
  a.n_edges = (int)edges.size();
  a.n_pairs = (int)plo.size();
  a.lnm_low = cfg->lnm_low;
  a.lnm_high = cfg->lnm_high;
  a.zt_low = cfg->zt_low;
  a.zt_high = cfg->zt_high;
  a.mor_kind = mor->kind;
  for (int i = 0; i < 8; ++i) a.mor[i] = mor->p[i];
  a.n_plob = plob->n;
  a.plob_z = d_pz.get();
  a.plob_coef = d_pc.get();
  a.edges = d_edges.get();
  a.pair_lo = d_plo.get();
  a.pair_hi = d_phi.get();
  a.bin_pair = d_bp.get();
  a.zob_min = d_zmin.get();
  a.zob_max = d_zmax.get();
  a.sigma_z = d_sz.get();
  a.gl_t = d_glt.get();
  a.gl_w = d_glw.get();
  a.lnm_out = d_lnm.get();
  a.z_out = d_z.get();
  a.S_out = d_S.get();
  long long warps = (long long)cfg->n_lnm * cfg->n_z;
  int blocks = (int)((warps * 32 + 127) / 128);
  sel_function_kernel<<<blocks, 128, 0, s>>>(a);
  count_launch();
  Y3B_CUDA(cudaGetLastError());
  Y3B_CUDA(cudaMemcpyAsync(lnm_out, d_lnm.get(), cfg->n_lnm * sizeof(double), cudaMemcpyDeviceToHost, s));
  Y3B_CUDA(cudaMemcpyAsync(z_out, d_z.get(), cfg->n_z * sizeof(double), cudaMemcpyDeviceToHost, s));
  Y3B_CUDA(cudaMemcpyAsync(S_out, d_S.get(), nS * sizeof(double), cudaMemcpyDeviceToHost, s));
  Y3B_CUDA(cudaStreamSynchronize(s));
  return Y3B_OK;
}

// ===========================================================================
// SelGLCore
namespace y3b {

struct SelGLTablesDev {
  int n_hm, n_hz, n_dist, n_sci;
  const double* hax;       // ln(m_h (om - onu)) [n_hm]
  const double* hz;        // [n_hz]
  const double* dn;        // [n_hz][n_hm]
  const double* dz;
  const double* da;
  const double* sz;
  const double* sv;
};

__global__ void
hmf_axis_kernel(const double* m_h, int n, double om_minus_onu, double* out)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = log(m_h[i] * om_minus_onu);
}

// One CTA per bin b; thread k evaluates W_b[k] = sum_q zfac[q] hmf(k,q)
// sel_b(k,q) (n_operator_sel_gl_t.hh:115-124); the block then forms the
// plain lnM moments n0, n1, m2 with fixed-order tree sums (129-141).
__global__ void __launch_bounds__(256)
selgl_build_kernel(int n_lnm, int n_z, const double* lnm_x, const double* lnm_w,
                   const double* z_x, const double* z_w, double lnm_lo, double lnm_hi,
                   y3b_cosmo c, SelGLTablesDev t, int include_sci, int n_sel_lnm,
                   const double* sel_lnm, int n_sel_z, const double* sel_z,
                   const double* S_stack, double* W, double* norm, double* lnm_eff,
                   double* mu2, int* status)
{
  extern __shared__ double sh[];
  double* zfac = sh;             // [n_z]
  double* red = sh + n_z;        // [blockDim.x]
  const int b = blockIdx.x;
  for (int q = threadIdx.x; q < n_z; q += blockDim.x) {
    double z = z_x[q], dv;
    if (!dv_do_dz(t.dz, t.da, t.n_dist, c.om, c.ol, c.ok, c.h0, z, &dv)) {
      set_err(status, kDevDomain);
      dv = 0.0;
    }
    double sci = (include_sci && t.n_sci > 0) ? interp1d_clamp(t.sz, t.sv, t.n_sci, z) : 1.0;
    zfac[q] = z_w[q] * dv * omega_z_des(z) * sci;
  }
  __syncthreads();
  // Table box of the selection function (sel_function_t.hh:228-242).
  const double slo = sel_lnm[0], shi = sel_lnm[n_sel_lnm - 1];
  const double zlo = sel_z[0], zhi = sel_z[n_sel_z - 1];
  const double* plane = S_stack + (size_t)b * n_sel_z * n_sel_lnm;
  double n0 = 0.0, n1 = 0.0;
  for (int k = threadIdx.x; k < n_lnm; k += blockDim.x) {
    double lnM = lnm_x[k];
    double acc = 0.0;
    for (int q = 0; q < n_z; ++q) {
      double z = z_x[q];
      double h = interp2d_clamp(t.hax, t.n_hm, t.hz, t.n_hz, t.dn, lnM, z) *
                 (c.hmf_s * (lnM * kLog10e - kHmfPivot) + c.hmf_q);
      double s = (lnM < slo || lnM > shi || z < zlo || z > zhi)
                   ? 0.0
                   : interp2d_clamp(sel_lnm, n_sel_lnm, sel_z, n_sel_z, plane, lnM, z);
      acc += zfac[q] * h * s;
    }
    W[(size_t)b * n_lnm + k] = acc;
    n0 += lnm_w[k] * acc;
    n1 += lnm_w[k] * acc * lnM;
  }
  n0 = block_sum<1024>(n0, red);
  n1 = block_sum<1024>(n1, red);
  double eff = (n0 != 0.0) ? n1 / n0 : 0.5 * (lnm_lo + lnm_hi);
  double m2 = 0.0;
  for (int k = threadIdx.x; k < n_lnm; k += blockDim.x) {
    double d = lnm_x[k] - eff;
    m2 += lnm_w[k] * W[(size_t)b * n_lnm + k] * d * d;
  }
  m2 = block_sum<1024>(m2, red);
  if (threadIdx.x == 0) {
    norm[b] = n0;
    lnm_eff[b] = eff;
    mu2[b] = (n0 != 0.0) ? m2 / n0 : 0.0;
  }
}

// The miscentred-profile table NFW_DSIGMA_MIS reads: log of the unit profile
// on ln x (fastest) and ln x_mis axes (nfw_dsigma_mis.hh:62-72,95-114).
struct MisTable {
  int n_lx, n_lxm;
  const double* logx;
  const double* logxmis;
  const double* log_tab;  // [n_lxm][n_lx]
};

// phi(b, R, lnM) = (1 - f) dSigma_nfw.clamp(R, lnM) + f NFW_DSIGMA_MIS(R,
// r_mis_b, lnM) for a list of (rmis, R, lnM) triples; one warp per triple
// (n_operator_sel_gl_t.hh:343-349).  The module builds NFW_DSIGMA_MIS with
// rho_c and sets rho_mult = Omega_M (n_operator_sel_gl_t.hh:248,264), so r_s
// comes from rho_c and the amplitude 2 r_s delta_c rho_c rho_mult carries
// Omega_M.  The profile is the reference's table (clamped bilinear at
// (ln x, ln x_mis)) when one is loaded, otherwise the direct quadrature that
// generates such a table.
__global__ void __launch_bounds__(128)
phi_list_kernel(int n, const double* rmis, const double* R, const double* lnM,
                double f_mis, double conc, double rhoc, double rho_mult, int n_r,
                const double* r_sigma, int n_ml, const double* lnM_tab, const double* dsig,
                MisQuad q, MisTable tab, double* out)
{
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= n) return;
  const double rs = nfw_rs(lnM[w], conc, rhoc);
  double mis;
  if (tab.log_tab) {
    mis = exp(interp2d_clamp(tab.logx, tab.n_lx, tab.logxmis, tab.n_lxm, tab.log_tab,
                             log(R[w] / rs), log(rmis[w] / rs)));
  } else {
    mis = mis_partial<double>(q, R[w] / rs, rmis[w] / rs, true, lane);
    mis = warp_sum(mis);
  }
  if (lane == 0) {
    double cen = interp2d_clamp(r_sigma, n_r, lnM_tab, n_ml, dsig, R[w], lnM[w]);
    out[w] = (1.0 - f_mis) * cen + f_mis * (nfw_norm(lnM[w], conc, rhoc) * rho_mult) * mis;
  }
}

// NFW_DSIGMA_MIS / NFW_SIGMA_MIS at arbitrary points, one warp per point.
__global__ void __launch_bounds__(128)
nfw_mis_kernel(int which, int n, const double* r, const double* rmis, const double* lnM,
               double conc, double rho, MisQuad q, double* out)
{
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= n) return;
  const double rs = nfw_rs(lnM[w], conc, rho);
  double v = which == 2
               ? dsigma_single_partial(q.th, q.wth, q.n_theta, r[w] / rs, rmis[w] / rs, lane, 32) /
                   kPi
               : mis_partial<double>(q, r[w] / rs, rmis[w] / rs, which == 0, lane);
  v = warp_sum(v);
  if (lane == 0) out[w] = nfw_norm(lnM[w], conc, rho) * v;
}

// sum_k w_k W_b[k] phi[k] for each query (exact method); one warp per query.
__global__ void
shear_contract_kernel(int n, int n_lnm, const int* bin, const double* lnm_w,
                      const double* W, const double* phi, double* out)
{
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= n) return;
  const double* Wb = W + (size_t)bin[w] * n_lnm;
  const double* ph = phi + (size_t)w * n_lnm;
  double acc = 0.0;
  for (int k = lane; k < n_lnm; k += 32) acc += lnm_w[k] * Wb[k] * ph[k];
  acc = warp_sum(acc);
  if (lane == 0) out[w] = acc;
}

}  // namespace y3b

struct y3b_selgl {
  y3b_selgl_config cfg;
  cudaStream_t stream = nullptr;
  y3b::DevBuf<double> lnm_x, lnm_w, z_x, z_w;
  y3b::DevBuf<double> W, norm, eff, mu2;
  y3b::DevBuf<double> hax, hz, dn, dz, da, sz, sv, sel_lnm, sel_z, S;
  y3b::DevBuf<int> status;
  y3b::MisQuadCache quad;
  y3b::DevBuf<double> tab_lx, tab_lxm, tab_v;  // miscentred-profile table (optional)
  int tab_nlx = 0, tab_nlxm = 0;
  std::vector<double> h_norm, h_eff, h_mu2, h_lnm_x, h_lnm_w;
  int n_bins = 0;
  bool built = false;
  double omega_m = 0.0;
};

extern "C" int
y3b_selgl_create(const y3b_selgl_config* cfg, y3b_selgl** out)
{
  clear_error();
  if (!cfg || !out) {
    set_error("y3b_selgl_create: null argument");
    return Y3B_ERR_INVALID;
  }
  *out = nullptr;
  if (cfg->n_lnm < 1 || cfg->n_z < 1 || cfg->n_lnm > 4096 || cfg->n_z > 4096 ||
      !(cfg->lnm_high > cfg->lnm_low) || !(cfg->zt_high > cfg->zt_low)) {
    set_error("y3b_selgl_create: invalid grid (n_lnm, n_z in [1, 4096], ordered bounds)");
    return Y3B_ERR_INVALID;
  }
  Y3B_TRY(require_device());
  y3b_selgl* h = new (std::nothrow) y3b_selgl();
  if (!h) {
    set_error("y3b_selgl_create: out of host memory");
    return Y3B_ERR_NOMEM;
  }
  h->cfg = *cfg;
  int rc = y3b::cuda_status(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking),
                            "cudaStreamCreate");
  if (rc == Y3B_OK) rc = h->lnm_x.alloc(cfg->n_lnm);
  if (rc == Y3B_OK) rc = h->lnm_w.alloc(cfg->n_lnm);
  if (rc == Y3B_OK) rc = h->z_x.alloc(cfg->n_z);
  if (rc == Y3B_OK) rc = h->z_w.alloc(cfg->n_z);
  if (rc == Y3B_OK) rc = h->status.alloc(1);
  if (rc == Y3B_OK)
    rc = y3b::gl_nodes_device(cfg->lnm_low, cfg->lnm_high, cfg->n_lnm, h->lnm_x.get(),
                              h->lnm_w.get(), h->stream);
  if (rc == Y3B_OK)
    rc = y3b::gl_nodes_device(cfg->zt_low, cfg->zt_high, cfg->n_z, h->z_x.get(), h->z_w.get(),
                              h->stream);
  if (rc == Y3B_OK) {
    h->h_lnm_x.resize(cfg->n_lnm);
    h->h_lnm_w.resize(cfg->n_lnm);
    rc = y3b::cuda_status(cudaMemcpyAsync(h->h_lnm_x.data(), h->lnm_x.get(),
                                          cfg->n_lnm * sizeof(double), cudaMemcpyDeviceToHost,
                                          h->stream),
                          "copy lnm_x");
  }
  if (rc == Y3B_OK)
    rc = y3b::cuda_status(cudaMemcpyAsync(h->h_lnm_w.data(), h->lnm_w.get(),
                                          cfg->n_lnm * sizeof(double), cudaMemcpyDeviceToHost,
                                          h->stream),
                          "copy lnm_w");
  if (rc == Y3B_OK) rc = y3b::cuda_status(cudaStreamSynchronize(h->stream), "sync");
  if (rc != Y3B_OK) {
    y3b_selgl_destroy(h);
    return rc;
  }
  *out = h;
  return Y3B_OK;
}

extern "C" void
y3b_selgl_destroy(y3b_selgl* h)
{
  if (!h) return;
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

extern "C" int
y3b_selgl_n_bins(const y3b_selgl* h)
{
  return h ? h->n_bins : 0;
}

extern "C" int
y3b_selgl_build(y3b_selgl* h, const y3b_cosmo* c, const y3b_tables* t,
                const y3b_selection* sel, int include_sci)
{
  using namespace y3b;
  clear_error();
  if (!h || !c || !t || !sel || !sel->S_stack || !sel->lnm || !sel->z) {
    set_error("y3b_selgl_build: null argument");
    return Y3B_ERR_INVALID;
  }
  if (t->n_hm < 2 || t->n_hz < 2 || t->n_dist < 2 || sel->n_bins < 1 || sel->n_lnm < 2 ||
      sel->n_z < 2 || (include_sci && t->n_sci < 2)) {
    set_error("y3b_selgl_build: tables need >= 2 nodes per axis and >= 1 bin");
    return Y3B_ERR_INVALID;
  }
  if (!(c->om - c->onu > 0.0)) {
    set_error("y3b_selgl_build: omega_M - omega_nu must be positive");
    return Y3B_ERR_INVALID;
  }
  cudaStream_t s = h->stream;
  const int nb = sel->n_bins;
  Y3B_TRY(h->W.alloc((size_t)nb * h->cfg.n_lnm));
  Y3B_TRY(h->norm.alloc(nb));
  Y3B_TRY(h->eff.alloc(nb));
  Y3B_TRY(h->mu2.alloc(nb));
  Y3B_TRY(h->hz.upload(t->hmf_z, t->n_hz, s));
  Y3B_TRY(h->dn.upload(t->dndlnmh, (size_t)t->n_hz * t->n_hm, s));
  Y3B_TRY(h->dz.upload(t->dist_z, t->n_dist, s));
  Y3B_TRY(h->da.upload(t->dist_da, t->n_dist, s));
  if (include_sci) {
    Y3B_TRY(h->sz.upload(t->sci_z, t->n_sci, s));
    Y3B_TRY(h->sv.upload(t->sci_val, t->n_sci, s));
  }
  Y3B_TRY(h->sel_lnm.upload(sel->lnm, sel->n_lnm, s));
  Y3B_TRY(h->sel_z.upload(sel->z, sel->n_z, s));
  Y3B_TRY(h->S.upload(sel->S_stack, (size_t)nb * sel->n_z * sel->n_lnm, s));
  // HMF mass axis ln(m_h (Omega_M - Omega_nu)) (hmf_t.hh:15-25).
  DevBuf<double> mh;
  Y3B_TRY(mh.upload(t->hmf_m_h, t->n_hm, s));
  Y3B_TRY(h->hax.alloc(t->n_hm));
  hmf_axis_kernel<<<(t->n_hm + 127) / 128, 128, 0, s>>>(mh.get(), t->n_hm, c->om - c->onu,
                                                        h->hax.get());
  count_launch();
  Y3B_CUDA(cudaGetLastError());
  Y3B_CUDA(cudaMemsetAsync(h->status.get(), 0, sizeof(int), s));
  SelGLTablesDev td{t->n_hm, t->n_hz, t->n_dist, include_sci ? t->n_sci : 0,
                    h->hax.get(), h->hz.get(), h->dn.get(), h->dz.get(), h->da.get(),
                    include_sci ? h->sz.get() : nullptr, include_sci ? h->sv.get() : nullptr};
  int threads = 32;
  while (threads < h->cfg.n_lnm && threads < 256) threads <<= 1;
  size_t shm = (h->cfg.n_z + threads) * sizeof(double);
  selgl_build_kernel<<<nb, threads, shm, s>>>(
    h->cfg.n_lnm, h->cfg.n_z, h->lnm_x.get(), h->lnm_w.get(), h->z_x.get(), h->z_w.get(),
    h->cfg.lnm_low, h->cfg.lnm_high, *c, td, include_sci, sel->n_lnm, h->sel_lnm.get(),
    sel->n_z, h->sel_z.get(), h->S.get(), h->W.get(), h->norm.get(), h->eff.get(), h->mu2.get(),
    h->status.get());
  count_launch();
  Y3B_CUDA(cudaGetLastError());
  h->h_norm.resize(nb);
  h->h_eff.resize(nb);
  h->h_mu2.resize(nb);
  Y3B_CUDA(cudaMemcpyAsync(h->h_norm.data(), h->norm.get(), nb * sizeof(double),
                           cudaMemcpyDeviceToHost, s));
  Y3B_CUDA(cudaMemcpyAsync(h->h_eff.data(), h->eff.get(), nb * sizeof(double),
                           cudaMemcpyDeviceToHost, s));
  Y3B_CUDA(cudaMemcpyAsync(h->h_mu2.data(), h->mu2.get(), nb * sizeof(double),
                           cudaMemcpyDeviceToHost, s));
  int st = read_device_status(h->status.get(), s);
  h->n_bins = nb;
  h->omega_m = c->om;
  h->built = (st == Y3B_OK);
  if (st == Y3B_ERR_DOMAIN)
    set_error("y3b_selgl_build: a GL z node lies outside distances/z (argument out of range in Interp1D)");
  return st;
}

extern "C" int
y3b_selgl_counts(y3b_selgl* h, int n, const int* bin_index, double* vals)
{
  y3b::clear_error();
  if (!h || (n > 0 && (!bin_index || !vals))) {
    y3b::set_error("y3b_selgl_counts: null argument");
    return Y3B_ERR_INVALID;
  }
  if (!h->built) {
    y3b::set_error("y3b_selgl_counts: no sample built");
    return Y3B_ERR_INVALID;
  }
  for (int i = 0; i < n; ++i) {
    int b = bin_index[i];
    if (b < 0 || b >= h->n_bins) {
      y3b::set_error("NumCountsSelGL: bin_index outside sel_function/S_stack range");
      return Y3B_ERR_INVALID;
    }
    vals[i] = h->h_norm[b];
  }
  return Y3B_OK;
}

extern "C" int
y3b_selgl_weights(y3b_selgl* h, double* W, double* norm, double* lnm_eff, double* mu2,
                  double* lnm_x, double* lnm_w)
{
  y3b::clear_error();
  if (!h || !h->built) {
    y3b::set_error("y3b_selgl_weights: no sample built");
    return Y3B_ERR_INVALID;
  }
  const int nb = h->n_bins, nl = h->cfg.n_lnm;
  if (W)
    Y3B_CUDA(cudaMemcpy(W, h->W.get(), (size_t)nb * nl * sizeof(double), cudaMemcpyDeviceToHost));
  if (norm) std::memcpy(norm, h->h_norm.data(), nb * sizeof(double));
  if (lnm_eff) std::memcpy(lnm_eff, h->h_eff.data(), nb * sizeof(double));
  if (mu2) std::memcpy(mu2, h->h_mu2.data(), nb * sizeof(double));
  if (lnm_x) std::memcpy(lnm_x, h->h_lnm_x.data(), nl * sizeof(double));
  if (lnm_w) std::memcpy(lnm_w, h->h_lnm_w.data(), nl * sizeof(double));
  return Y3B_OK;
}

// NFW_DSIGMA_MIS's profile table (nfw_dsigma_mis.hh:62-72): kept on the
// device for the handle's shear evaluations; n_lx = 0 drops it.
extern "C" int
y3b_selgl_set_mis_table(y3b_selgl* h, int n_lx, const double* logx, int n_lxm,
                        const double* logxmis, const double* log_tab)
{
  using namespace y3b;
  clear_error();
  if (!h) {
    set_error("y3b_selgl_set_mis_table: null handle");
    return Y3B_ERR_INVALID;
  }
  if (n_lx == 0) {
    h->tab_nlx = h->tab_nlxm = 0;
    return Y3B_OK;
  }
  if (n_lx < 2 || n_lxm < 2 || !logx || !logxmis || !log_tab) {
    set_error("y3b_selgl_set_mis_table: need at least 2 x 2 nodes and three arrays");
    return Y3B_ERR_INVALID;
  }
  for (int i = 1; i < n_lx; ++i)
    if (!(logx[i] > logx[i - 1])) {
      set_error("y3b_selgl_set_mis_table: ln x axis not increasing");
      return Y3B_ERR_INVALID;
    }
  for (int j = 1; j < n_lxm; ++j)
    if (!(logxmis[j] > logxmis[j - 1])) {
      set_error("y3b_selgl_set_mis_table: ln x_mis axis not increasing");
      return Y3B_ERR_INVALID;
    }
  const size_t nv = (size_t)n_lx * n_lxm;
  for (size_t i = 0; i < nv; ++i)
    if (!std::isfinite(log_tab[i])) {
      set_error("y3b_selgl_set_mis_table: non-finite table entry");
      return Y3B_ERR_DOMAIN;
    }
  h->tab_nlx = h->tab_nlxm = 0;
  Y3B_TRY(h->tab_lx.upload(logx, n_lx, h->stream));
  Y3B_TRY(h->tab_lxm.upload(logxmis, n_lxm, h->stream));
  Y3B_TRY(h->tab_v.upload(log_tab, nv, h->stream));
  Y3B_CUDA(cudaStreamSynchronize(h->stream));
  h->tab_nlx = n_lx;
  h->tab_nlxm = n_lxm;
  return Y3B_OK;
}

// Shear1hMisSelGL::evaluate (n_operator_sel_gl_t.hh:293-319): exact =
// sum_k w_k W_b[k] phi(b, R, lnM_k); idea2 = norm_b [phi + mu2/2 d2phi] at
// lnm_eff with a 3-point stencil.
extern "C" int
y3b_selgl_shear(y3b_selgl* h, const y3b_shear_table* st, int n, const int* bin_index,
                const double* r, double* vals)
{
  using namespace y3b;
  clear_error();
  if (!h || !st || (n > 0 && (!bin_index || !r || !vals))) {
    set_error("y3b_selgl_shear: null argument");
    return Y3B_ERR_INVALID;
  }
  if (!h->built) {
    set_error("y3b_selgl_shear: no sample built");
    return Y3B_ERR_INVALID;
  }
  if (st->n_lob < 1 || st->n_r < 2 || st->n_lnm < 2 || !st->r_sigma || !st->lnM || !st->dsigma) {
    set_error("Shear1hMisSelGL: lob_centers is empty or haloModel table missing");
    return Y3B_ERR_INVALID;
  }
  for (int i = 0; i < n; ++i)
    if (bin_index[i] < 0 || bin_index[i] >= h->n_bins) {
      set_error("Shear1hMisSelGL: bin_index outside sel_function/S_stack range");
      return Y3B_ERR_INVALID;
    }
  if (n == 0) return Y3B_OK;
  cudaStream_t s = h->stream;
  if (!h->tab_nlx) Y3B_TRY(h->quad.ensure(st->n_theta, st->n_s, st->s_max, s));
  MisTable tab{h->tab_nlx, h->tab_nlxm, h->tab_lx.get(), h->tab_lxm.get(),
               h->tab_nlx ? h->tab_v.get() : nullptr};
  const int nl = h->cfg.n_lnm;
  // Triples (rmis, R, lnM) of phi evaluations.
  std::vector<double> trm, tR, tM;
  if (!st->use_idea2) {
    trm.reserve((size_t)n * nl);
    for (int i = 0; i < n; ++i) {
      double rmis = st->tau_mis * std::pow(st->lob_centers[bin_index[i] % st->n_lob] / 100.0, 0.2);
      for (int k = 0; k < nl; ++k) {
        trm.push_back(rmis);
        tR.push_back(r[i]);
        tM.push_back(h->h_lnm_x[k]);
      }
    }
  } else {
    for (int i = 0; i < n; ++i) {
      int b = bin_index[i];
      double rmis = st->tau_mis * std::pow(st->lob_centers[b % st->n_lob] / 100.0, 0.2);
      double y0 = h->h_eff[b];
      for (double dy : {0.0, st->stencil_h, -st->stencil_h}) {
        trm.push_back(rmis);
        tR.push_back(r[i]);
        tM.push_back(y0 + dy);
      }
    }
  }
  const int nt = (int)trm.size();
  DevBuf<double> d_rm, d_R, d_M, d_phi, d_rs, d_lt, d_ds, d_out;
  DevBuf<int> d_bin;
  Y3B_TRY(d_rm.upload(trm.data(), nt, s));
  Y3B_TRY(d_R.upload(tR.data(), nt, s));
  Y3B_TRY(d_M.upload(tM.data(), nt, s));
  Y3B_TRY(d_phi.alloc(nt));
  Y3B_TRY(d_rs.upload(st->r_sigma, st->n_r, s));
  Y3B_TRY(d_lt.upload(st->lnM, st->n_lnm, s));
  Y3B_TRY(d_ds.upload(st->dsigma, (size_t)st->n_r * st->n_lnm, s));
  phi_list_kernel<<<(nt * 32 + 127) / 128, 128, 0, s>>>(
    nt, d_rm.get(), d_R.get(), d_M.get(), st->f_mis, st->conc, kRhoCrit, h->omega_m, st->n_r,
    d_rs.get(), st->n_lnm, d_lt.get(), d_ds.get(), h->tab_nlx ? MisQuad{} : h->quad.view(), tab,
    d_phi.get());
  count_launch();
  Y3B_CUDA(cudaGetLastError());
  if (!st->use_idea2) {
    Y3B_TRY(d_bin.upload(bin_index, n, s));
    Y3B_TRY(d_out.alloc(n));
    shear_contract_kernel<<<(n * 32 + 127) / 128, 128, 0, s>>>(
      n, nl, d_bin.get(), h->lnm_w.get(), h->W.get(), d_phi.get(), d_out.get());
    count_launch();
    Y3B_CUDA(cudaGetLastError());
    Y3B_CUDA(cudaMemcpyAsync(vals, d_out.get(), n * sizeof(double), cudaMemcpyDeviceToHost, s));
    Y3B_CUDA(cudaStreamSynchronize(s));
  } else {
    std::vector<double> phi(nt);
    Y3B_CUDA(cudaMemcpyAsync(phi.data(), d_phi.get(), nt * sizeof(double),
                             cudaMemcpyDeviceToHost, s));
    Y3B_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < n; ++i) {
      int b = bin_index[i];
      double c0 = phi[3 * i], p = phi[3 * i + 1], m = phi[3 * i + 2];
      double hh = st->stencil_h;
      double d2 = (p - 2.0 * c0 + m) / (hh * hh);
      vals[i] = h->h_norm[b] * (c0 + 0.5 * h->h_mu2[b] * d2);
    }
  }
  return Y3B_OK;
}

// ===========================================================================
namespace y3b {

// <Sigma_crit^-1>(z_l): one CTA per lens redshift, threads over sources,
// trapezoid by a fixed-order tree (average_sigma_crit_inv.py:53-58).
__global__ void __launch_bounds__(256)
sigma_crit_inv_kernel(const double* zl, int n_zs, const double* zs, const double* pz,
                      double delta_z, double h0, int nd, const double* dz, const double* da,
                      double* out, int* status)
{
  __shared__ double red[256];
  const double G = 4.51710305e-48, cl = 9.71561189e-15;
  const double kk = 4.0 * kPi * G / cl / cl;
  const int j = blockIdx.x;
  double dl;
  if (!interp1d(dz, da, nd, zl[j], &dl)) {
    set_err(status, kDevDomain);
    dl = 0.0;
  }
  auto f = [&](int i) -> double {
    double ds, p;
    if (!interp1d(dz, da, nd, zs[i], &ds) || !interp1d(zs, pz, n_zs, zs[i] + delta_z, &p)) {
      set_err(status, kDevDomain);
      return 0.0;
    }
    double dls = ds - (1.0 + zl[j]) / (1.0 + zs[i]) * dl;
    double v = ds > 0.0 ? p * kk * dl * dls / ds : 0.0;
    return v > 0.0 ? v : 0.0;
  };
  double acc = 0.0;
  for (int i = threadIdx.x; i + 1 < n_zs; i += blockDim.x)
    acc += 0.5 * (f(i) + f(i + 1)) * (zs[i + 1] - zs[i]);
  acc = block_sum<256>(acc, red);
  if (threadIdx.x == 0) out[j] = acc * h0;
}

}  // namespace y3b

extern "C" int
y3b_sigma_crit_inv(int n_zl, const double* zl, int n_zs, const double* zs, const double* pz,
                   double delta_z, double h0, int n_dist, const double* dist_z,
                   const double* dist_da, double* out)
{
  using namespace y3b;
  clear_error();
  if (n_zl < 1 || n_zs < 2 || n_dist < 2 || !zl || !zs || !pz || !dist_z || !dist_da || !out) {
    set_error("y3b_sigma_crit_inv: invalid arguments");
    return Y3B_ERR_INVALID;
  }
  Y3B_TRY(require_device());
  cudaStream_t s = 0;
  DevBuf<double> a, b, c, d, e, o;
  DevBuf<int> st;
  Y3B_TRY(a.upload(zl, n_zl, s));
  Y3B_TRY(b.upload(zs, n_zs, s));
  Y3B_TRY(c.upload(pz, n_zs, s));
  Y3B_TRY(d.upload(dist_z, n_dist, s));
  Y3B_TRY(e.upload(dist_da, n_dist, s));
  Y3B_TRY(o.alloc(n_zl));
  Y3B_TRY(st.alloc(1));
  Y3B_CUDA(cudaMemsetAsync(st.get(), 0, sizeof(int), s));
  sigma_crit_inv_kernel<<<n_zl, 256, 0, s>>>(a.get(), n_zs, b.get(), c.get(), delta_z, h0,
                                             n_dist, d.get(), e.get(), o.get(), st.get());
  count_launch();
  Y3B_CUDA(cudaGetLastError());
  Y3B_CUDA(cudaMemcpyAsync(out, o.get(), n_zl * sizeof(double), cudaMemcpyDeviceToHost, s));
  int rc = read_device_status(st.get(), s);
  if (rc == Y3B_ERR_DOMAIN) set_error("y3b_sigma_crit_inv: redshift outside distances or n(z) table");
  return rc;
}

extern "C" int
y3b_nfw_mis(int which, int n, const double* r, const double* rmis, const double* lnM,
            double conc, double rho, int n_theta, int n_s, double s_max, double* out)
{
  using namespace y3b;
  clear_error();
  if (n < 0 || (n > 0 && (!r || !rmis || !lnM || !out)) || which < 0 || which > 2 ||
      !(conc > 0.0) || !(rho > 0.0)) {
    set_error("y3b_nfw_mis: invalid arguments");
    return Y3B_ERR_INVALID;
  }
  if (n == 0) return Y3B_OK;
  Y3B_TRY(require_device());
  cudaStream_t s = 0;
  MisQuadCache quad;
  Y3B_TRY(quad.ensure(n_theta, n_s, s_max, s));
  DevBuf<double> a, b, c, o;
  Y3B_TRY(a.upload(r, n, s));
  Y3B_TRY(b.upload(rmis, n, s));
  Y3B_TRY(c.upload(lnM, n, s));
  Y3B_TRY(o.alloc(n));
  nfw_mis_kernel<<<(n * 32 + 127) / 128, 128, 0, s>>>(which, n, a.get(), b.get(), c.get(), conc,
                                                     rho, quad.view(), o.get());
  count_launch();
  Y3B_CUDA(cudaGetLastError());
  Y3B_CUDA(cudaMemcpyAsync(out, o.get(), n * sizeof(double), cudaMemcpyDeviceToHost, s));
  Y3B_CUDA(cudaStreamSynchronize(s));
  return Y3B_OK;
}

// ===========================================================================
// y3b_sel_function_noalloc: the S_stack producer for callers that cannot
// allocate device memory.  Everything the kernel needs besides the caller's
// output buffers (Gauss-Legendre nodes, the unique richness edges and their
// bin pairing, the per-bin photo-z edges and widths, the projection table)
// lives in one file-scope __device__ array of fixed size that every call
// shares.
#include <cuda.h>

#include <mutex>

namespace y3b {

constexpr int kNoAllocMaxQ = 1024;      // N_q
constexpr int kNoAllocMaxBins = 256;    // bins
constexpr int kNoAllocMaxPlob = 256;    // projection-table z nodes
constexpr size_t kNoAllocScratchDoubles =
  2 * kNoAllocMaxQ + kMaxEdges + 3 * kNoAllocMaxBins + 9 * kNoAllocMaxPlob +
  (2 * kMaxPairs + kNoAllocMaxBins);    // last term holds the int tables
static __device__ __align__(256) double g_selfunc_scratch[kNoAllocScratchDoubles];

// Device address of g_selfunc_scratch, looked up once per device context
// (host code may not use the symbol itself: it names a host-side stand-in).
// The address belongs to the context the module image was loaded into: a
// caller that resets the device gets a new context, in which the array lives
// elsewhere, so the cache is keyed by the context's unique id and the lookup
// is repeated for a new one.
static std::mutex g_scratch_mu;
static void* g_scratch_addr[128];
static unsigned long long g_scratch_ctx[128];

// Unique id of the calling thread's current context (0 if it cannot be
// read, in which case the address is looked up on every call).  The driver
// entry points are fetched through the runtime: the library links no
// driver-API import.
static unsigned long long
current_context_id()
{
  using GetCurrentFn = CUresult (*)(CUcontext*);
  using GetIdFn = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrentFn get_current = nullptr;
  static GetIdFn get_id = nullptr;
  static bool resolved = false;
  if (!resolved) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetIdFn>(f);
    resolved = true;
  }
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx ||
      get_id(ctx, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

static int
scratch_address(double** out)
{
  int dev = 0;
  Y3B_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) {
    set_error("y3b_sel_function_noalloc: device index %d out of range", dev);
    return Y3B_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  const unsigned long long ctx = current_context_id();
  if (!g_scratch_addr[dev] || ctx == 0 || ctx != g_scratch_ctx[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_selfunc_scratch);
    if (e != cudaSuccess || !p) {
      set_error("cudaGetSymbolAddress(g_selfunc_scratch): %s", cudaGetErrorString(e));
      return Y3B_ERR_CUDA;
    }
    g_scratch_addr[dev] = p;
    // The lookup made the device's context current if it was not yet.
    g_scratch_ctx[dev] = ctx ? ctx : current_context_id();
  }
  *out = static_cast<double*>(g_scratch_addr[dev]);
  return Y3B_OK;
}

}  // namespace y3b

extern "C" int
y3b_sel_function_noalloc(const y3b_selfunc_config* cfg, const y3b_mor* mor,
                         const y3b_plob* plob, double* lnm_dev, double* z_dev, double* S_dev,
                         void* stream)
{
  using namespace y3b;
  clear_error();
  if (!cfg || !mor || !plob || !lnm_dev || !z_dev || !S_dev || !plob->z || !plob->coef ||
      !cfg->lam_min || !cfg->lam_max || !cfg->zob_min || !cfg->zob_max || !cfg->sigma_z) {
    set_error("y3b_sel_function_noalloc: null argument");
    return Y3B_ERR_INVALID;
  }
  if (cfg->n_bins <= 0 || cfg->n_lnm <= 0 || cfg->n_z <= 0 || cfg->n_q <= 0 || plob->n < 1 ||
      (mor->kind != Y3B_MOR_HOD && mor->kind != Y3B_MOR_LOGNORMAL)) {
    set_error("y3b_sel_function_noalloc: invalid sizes or MOR kind");
    return Y3B_ERR_INVALID;
  }
  if (cfg->n_q > kNoAllocMaxQ || cfg->n_bins > kNoAllocMaxBins || plob->n > kNoAllocMaxPlob) {
    set_error("y3b_sel_function_noalloc: sizes exceed the fixed scratch (N_q <= %d, "
              "n_bins <= %d, projection-table nodes <= %d); use y3b_sel_function",
              kNoAllocMaxQ, kNoAllocMaxBins, kNoAllocMaxPlob);
    return Y3B_ERR_INVALID;
  }
  Y3B_TRY(require_device());
  const int nb = cfg->n_bins;
  std::vector<double> edges;
  for (int k = 0; k < nb; ++k) {
    edges.push_back(cfg->lam_min[k]);
    edges.push_back(cfg->lam_max[k]);
  }
  std::sort(edges.begin(), edges.end());
  edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
  if ((int)edges.size() > kMaxEdges) {
    set_error("y3b_sel_function_noalloc: more than %d unique richness edges", kMaxEdges);
    return Y3B_ERR_UNSUPPORTED;
  }
  std::vector<int> ints;  // pair_lo | pair_hi | bin_pair
  std::vector<int> plo, phi_, bin_pair(nb);
  for (int k = 0; k < nb; ++k) {
    int lo = int(std::lower_bound(edges.begin(), edges.end(), cfg->lam_min[k]) - edges.begin());
    int hi = int(std::lower_bound(edges.begin(), edges.end(), cfg->lam_max[k]) - edges.begin());
    int p = 0;
    for (; p < (int)plo.size(); ++p)
      if (plo[p] == lo && phi_[p] == hi) break;
    if (p == (int)plo.size()) {
      plo.push_back(lo);
      phi_.push_back(hi);
    }
    bin_pair[k] = p;
  }
  if ((int)plo.size() > kMaxPairs) {
    set_error("y3b_sel_function_noalloc: more than %d distinct richness bins", kMaxPairs);
    return Y3B_ERR_UNSUPPORTED;
  }
  double* scratch = nullptr;
  Y3B_TRY(scratch_address(&scratch));
  // Scratch layout (doubles, then ints).
  const int nq = cfg->n_q, np = plob->n;
  double* d_glt = scratch;
  double* d_glw = d_glt + nq;
  double* d_edges = d_glw + nq;
  double* d_zmin = d_edges + edges.size();
  double* d_zmax = d_zmin + nb;
  double* d_sz = d_zmax + nb;
  double* d_pz = d_sz + nb;
  double* d_pc = d_pz + np;
  int* d_ints = reinterpret_cast<int*>(d_pc + 8 * (size_t)np);
  int* d_plo = d_ints;
  int* d_phi = d_plo + plo.size();
  int* d_bp = d_phi + phi_.size();
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  auto put = [&](void* dst, const void* src, size_t bytes) {
    return cuda_status(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s),
                       "y3b_sel_function_noalloc: copy to scratch");
  };
  Y3B_TRY(put(d_edges, edges.data(), edges.size() * sizeof(double)));
  Y3B_TRY(put(d_zmin, cfg->zob_min, nb * sizeof(double)));
  Y3B_TRY(put(d_zmax, cfg->zob_max, nb * sizeof(double)));
  Y3B_TRY(put(d_sz, cfg->sigma_z, nb * sizeof(double)));
  Y3B_TRY(put(d_pz, plob->z, np * sizeof(double)));
  Y3B_TRY(put(d_pc, plob->coef, 8 * (size_t)np * sizeof(double)));
  Y3B_TRY(put(d_plo, plo.data(), plo.size() * sizeof(int)));
  Y3B_TRY(put(d_phi, phi_.data(), phi_.size() * sizeof(int)));
  Y3B_TRY(put(d_bp, bin_pair.data(), nb * sizeof(int)));
  Y3B_TRY(gl_nodes_device(-1.0, 1.0, nq, d_glt, d_glw, s));

  SelFuncArgs a;
  a.n_lnm = cfg->n_lnm;
  a.n_z = cfg->n_z;
  a.n_q = nq;
  a.n_bins = nb;
  a.n_edges = (int)edges.size();
  a.n_pairs = (int)plo.size();
  a.lnm_low = cfg->lnm_low;
  a.lnm_high = cfg->lnm_high;
  a.zt_low = cfg->zt_low;
  a.zt_high = cfg->zt_high;
  a.mor_kind = mor->kind;
  for (int i = 0; i < 8; ++i) a.mor[i] = mor->p[i];
  a.n_plob = np;
  a.plob_z = d_pz;
  a.plob_coef = d_pc;
  a.edges = d_edges;
  a.pair_lo = d_plo;
  a.pair_hi = d_phi;
  a.bin_pair = d_bp;
  a.zob_min = d_zmin;
  a.zob_max = d_zmax;
  a.sigma_z = d_sz;
  a.gl_t = d_glt;
  a.gl_w = d_glw;
  a.lnm_out = lnm_dev;
  a.z_out = z_dev;
  a.S_out = S_dev;
  long long warps = (long long)cfg->n_lnm * cfg->n_z;
  int blocks = (int)((warps * 32 + 127) / 128);
  sel_function_kernel<<<blocks, 128, 0, s>>>(a);
  count_launch();
  return cuda_status(cudaGetLastError(), "sel_function_kernel (noalloc)");
}
