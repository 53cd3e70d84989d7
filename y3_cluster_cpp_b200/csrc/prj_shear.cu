// prj_shear.cu -- the frozen-physics projection-shear observable
// <DeltaSigma_prj>(R | lambda bin, z_obs) of ShearPrjFrozenPhysics
// (src/models/sigma_prj_frozen_t.hh:34-512) on the GPU.
//
// Per sample and per (richness bin, z_obs) slice the reference builds, once:
//   * a log-GL theta grid split at the slice's breakpoints (inner cut, the
//     line-of-sight exclusion angle, theta_R = R / D_A for every radius,
//     theta_lambda, 2 theta_lambda, theta_max; sigma_prj_t.hh:95-180),
//   * a line-of-sight z grid: GL on the exclusion ring around z_obs and
//     log-GL in comoving distance in front of and behind it
//     (sigma_prj_frozen_t.hh:380-455),
// then accumulates, in FP64,
//   wrnd(M)    = sum_z c_z n(M, z) w_M,                   (random channel)
//   Psi(theta) = sum_z c_z a_b(z) xi_NL(dchi(z, theta), z_obs)   over theta > theta_excl(z),
//   a_b(z)     = sum_M w_M r_s(M) n(M, z) b(M, z) / sum_M w_M r_s(M) n(M, z_obs) b(M, z_obs),
//   c_z        = dV/dz Omega(z) w_z (1 - u^2)_{|u| < 1},  u = (z - z_obs) / sigma_z(z),
// and per grid point (slice, R)
//   rnd = sum_theta g_theta sum_M wrnd(M) DSigma_mis(R | theta D_A, M),
//   cl  = sum_theta g_theta b_sel(theta) Psi(theta) sum_M w_M n(M, z_obs) b(M, z_obs) DSigma_mis,
// g_theta = w_theta 2 pi sin theta, b_sel a sigmoid between the
// b_sel_marginalised asymptotes; the shear is the same times
// Sigma_crit^-1(z_obs).  DSigma_mis is NFW_DSIGMA_MIS with the single
// (fixed-offset) kernel: the reference's table when loaded, else its direct
// quadrature.
//
// The grids (a few hundred nodes per slice) are built on the host in FP64 in
// the reference's order; the z-line-of-sight sums, Psi, and the (theta, M)
// dot products run on the device, one thread or block per independent sum,
// each summed in a fixed order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "common.cuh"
#include "host_common.h"
#include "zkernel_table.h"

namespace y3b {
namespace {

constexpr double kPiP = 3.14159265358979323846;
constexpr double kConc = 4.0;  // NFW_DSIGMA_MIS(4, RHOC, SINGLE), sigma_prj_frozen_t.hh:71

// ---- host-side interpolation with the reference's (GSL) semantics --------
int
h_cell(const double* xs, int n, double x)
{
  int lo = 0, hi = n - 1;
  while (hi > lo + 1) {
    int m = (lo + hi) / 2;
    if (xs[m] > x)
      hi = m;
    else
      lo = m;
  }
  return lo;
}

double
h_lin_clamp(const double* xs, const double* ys, int n, double x)
{
  x = std::min(std::max(x, xs[0]), xs[n - 1]);
  int i = h_cell(xs, n, x);
  double dx = xs[i + 1] - xs[i];
  return dx > 0.0 ? ys[i] + (x - xs[i]) / dx * (ys[i + 1] - ys[i]) : 0.0;
}

bool
h_lin(const double* xs, const double* ys, int n, double x, double* out)
{
  if (!(x >= xs[0] && x <= xs[n - 1])) return false;
  *out = h_lin_clamp(xs, ys, n, x);
  return true;
}

double
h_bilin_clamp(const double* xs, int nx, const double* ys, int ny, const double* zs, double x,
              double y)
{
  x = std::min(std::max(x, xs[0]), xs[nx - 1]);
  y = std::min(std::max(y, ys[0]), ys[ny - 1]);
  int i = h_cell(xs, nx, x), j = h_cell(ys, ny, y);
  double t = (x - xs[i]) / (xs[i + 1] - xs[i]);
  double u = (y - ys[j]) / (ys[j + 1] - ys[j]);
  const double* r0 = zs + (size_t)j * nx + i;
  const double* r1 = r0 + nx;
  return (1.0 - t) * (1.0 - u) * r0[0] + t * (1.0 - u) * r0[1] + (1.0 - t) * u * r1[0] +
         t * u * r1[1];
}

// Gauss-Legendre nodes on [a, b] (p_operator_cuhre_t.hh:66-95).
void
h_gl(double a, double b, int n, std::vector<double>& x, std::vector<double>& w)
{
  gl_nodes_host(a, b, n, x, w);
}

double
omega_z_host(double z)  // OMEGA_Z_DES (omega_z_des.hh:15-33)
{
  static const double f1[6] = {0.0, 0.0, 0.0, -0.00262353, 0.01940118, 0.45133063};
  static const double f2[6] = {1.33647377e+4, 1.35291046e+3, -1.26204891e+2,
                               -2.83454918e+1, -2.26465905, 3.84958753e-1};
  static const double f3[6] = {0, 0, -1.88101967, 4.8071839, -4.11424324, 1.18196785};
  const double* c = z < 0.504 ? f1 : (z < 0.7 ? f2 : f3);
  const double x = z < 0.504 ? z : (z < 0.7 ? z - 0.6 : z);
  double out = 0.0;
  for (int i = 0; i < 6; ++i) out = c[i] + x * out;
  return out;
}

// ---- device side ----------------------------------------------------------
struct PrjTables {
  int n_hm, n_hz;
  const double *mh, *hz, *dn;  // ln(m_h (Omega_M - Omega_nu)), z, dn/dlnM [n_hz][n_hm]
  double hmf_s, hmf_q;
  int n_bl, n_bz;
  const double *bl, *bz, *bias;  // haloModel lnM, z, bias [n_bz][n_bl]
  int n_xr, n_xz;
  const double *xr, *xz, *xi;    // xi_nl r, z, xi [n_xz][n_xr]
  int n_lx, n_lxm;
  const double *lx, *lxm, *ltab; // single-kernel table (n_lx = 0: quadrature)
  int n_th;
  const double *th, *wth;        // cos(theta) and weights of the GL nodes on [0, pi]
  double omega_m;
};

__device__ __forceinline__ double
hmf_dev(const PrjTables& T, double lnM, double z)
{
  return interp2d_clamp(T.mh, T.n_hm, T.hz, T.n_hz, T.dn, lnM, z) *
         (T.hmf_s * (lnM * kLog10e - kHmfPivot) + T.hmf_q);
}

// NFW_DSIGMA_MIS(R, R_mis, lnM), single kernel (nfw_dsigma_mis.hh:95-114):
// r_s from rho_c, amplitude 2 r_s delta_c rho_c Omega_M 1e-12 [h Msun/pc^2].
__device__ double
dsigma_single(const PrjTables& T, double R, double Rmis, double lnM)
{
  const double rs = nfw_rs(lnM, kConc, kRhoCrit);
  const double x = R / rs, xm = Rmis / rs;
  double unit;
  if (T.n_lx) {
    unit = exp(interp2d_clamp(T.lx, T.n_lx, T.lxm, T.n_lxm, T.ltab, log(x), log(xm)));
  } else {  // mean tangential shear on the circle x around the offset centre
    unit = dsigma_single_partial_cos(T.th, T.wth, T.n_th, x, xm, 0, 1) / kPiP;
  }
  return nfw_norm(lnM, kConc, kRhoCrit) * T.omega_m * unit;
}

// Per (slice, z node): a_b(z) and the random-channel weights.  One block of
// 128 threads per (slice, z); thread iM takes the mass nodes iM, iM + 128, ...
__global__ void __launch_bounds__(128)
prj_z_kernel(PrjTables T, int n_lnm, const double* lnm_x, const double* lnm_w,
             const int* zslice, const double* zz, const double* zc, const double* anchor,
             const double* denom, double* AB, double* WZ)
{
  __shared__ double red[128];
  const int u = blockIdx.x, sl = zslice[u];
  const double z = zz[u], c = zc[u];
  double num = 0.0;
  for (int iM = threadIdx.x; iM < n_lnm; iM += blockDim.x) {
    const double x = lnm_x[iM];
    const double n = hmf_dev(T, x, z);
    const double b = interp2d_clamp(T.bl, T.n_bl, T.bz, T.n_bz, T.bias, x, z);
    num += anchor[(size_t)sl * n_lnm + iM] * n * b;
    WZ[(size_t)u * n_lnm + iM] = c * n * lnm_w[iM];
  }
  num = block_sum<128>(num, red);
  if (threadIdx.x == 0) AB[u] = c * (num / denom[sl]);
}

// wrnd(slice, M) = sum over the slice's z nodes in order.
__global__ void
prj_wrnd_kernel(int n_slices, int n_lnm, const int* z0, const double* WZ, double* wrnd)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_slices * n_lnm) return;
  const int sl = i / n_lnm, iM = i % n_lnm;
  double acc = 0.0;
  for (int u = z0[sl]; u < z0[sl + 1]; ++u) acc += WZ[(size_t)u * n_lnm + iM];
  wrnd[i] = acc;
}

// Psi(theta) of every slice's theta node, z nodes in order.
__global__ void
prj_psi_kernel(PrjTables T, int n_theta_tot, const int* tslice, const double* theta,
               const int* z0, const double* chi_z, const double* th_excl, const double* AB,
               const double* chi_o, const double* zob, double* psi)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_theta_tot) return;
  const int sl = tslice[i];
  const double th = theta[i], ct = cos(th), co = chi_o[sl], zo = zob[sl];
  double acc = 0.0;
  for (int u = z0[sl]; u < z0[sl + 1]; ++u) {
    if (th <= th_excl[u]) continue;
    const double cz = chi_z[u];
    const double dchi = sqrt(fmax(cz * cz + co * co - 2.0 * cz * co * ct, 0.0));
    acc += AB[u] * interp2d_clamp(T.xr, T.n_xr, T.xz, T.n_xz, T.xi, dchi, zo);
  }
  psi[i] = acc;
}

// The single-kernel profile DSigma_mis(R | theta D_A, M) of every (grid
// point, theta node of its slice, mass node): one thread each, written to
// V[g][(it - t0) n_lnm + iM] (max_pairs per grid point).
__global__ void __launch_bounds__(256)
prj_profile_kernel(PrjTables T, int n_lnm, const double* lnm_x, const int* gp_slice,
                   const double* gp_R, const int* t0, const double* theta, const double* DA,
                   int max_pairs, double* V)
{
  const int g = blockIdx.y, sl = gp_slice[g];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n_pairs = (t0[sl + 1] - t0[sl]) * n_lnm;
  if (k >= n_pairs) return;
  const int it = t0[sl] + k / n_lnm, iM = k % n_lnm;
  V[(size_t)g * max_pairs + k] = dsigma_single(T, gp_R[g], theta[it] * DA[sl], lnm_x[iM]);
}

// One block per grid point: the (theta, M) sums of both channels over the
// profile values of prj_profile_kernel.
__global__ void __launch_bounds__(256)
prj_eval_kernel(int n_lnm, const int* gp_slice, const int* t0, const double* geom,
                const double* bsel, const double* psi, const double* wrnd, const double* wcl,
                const double* sci, int max_pairs, const double* V, double* out)
{
  __shared__ double red[256];
  const int g = blockIdx.x, sl = gp_slice[g];
  const double* Vg = V + (size_t)g * max_pairs;
  double rnd = 0.0, cl = 0.0;
  for (int it = t0[sl] + threadIdx.x; it < t0[sl + 1]; it += blockDim.x) {
    const double* v_it = Vg + (size_t)(it - t0[sl]) * n_lnm;
    double ar = 0.0, ac = 0.0;
    for (int iM = 0; iM < n_lnm; ++iM) {
      const double v = v_it[iM];
      ar += wrnd[(size_t)sl * n_lnm + iM] * v;
      ac += wcl[(size_t)sl * n_lnm + iM] * v;
    }
    rnd += geom[it] * ar;
    cl += geom[it] * bsel[it] * psi[it] * ac;
  }
  rnd = block_sum<256>(rnd, red);
  cl = block_sum<256>(cl, red);
  if (threadIdx.x == 0) {
    const double tot = rnd + cl, s = sci[sl];
    double* o = out + (size_t)g * 9;
    o[0] = tot;
    o[1] = rnd;
    o[2] = cl;
    o[3] = o[6] = tot * s;
    o[4] = o[7] = rnd * s;
    o[5] = o[8] = cl * s;
  }
}

}  // namespace

// Device buffers of one evaluation, kept by the handle and grown on demand.
struct PrjBufs {
  DevBuf<double> d_mh, d_hz, d_dn, d_bl, d_bz, d_bi, d_xr, d_xz, d_xi, d_lx, d_lxm, d_lt, d_th,
    d_wth, d_lnx, d_lnw, d_theta, d_geom, d_bsel, d_zz, d_zc, d_chiz, d_thex, d_anchor, d_denom,
    d_wcl, d_AB, d_WZ, d_wrnd, d_psi, d_chio, d_zob, d_da, d_sci, d_gpR, d_out, d_V;
  DevBuf<int> d_t0, d_z0, d_ts, d_zs, d_gps;
};

}  // namespace y3b

struct y3b_prj {
  y3b_prj_config cfg;
  std::vector<double> lob;                   // richness-bin centres
  std::vector<int> gp_lb;                    // per grid point
  std::vector<double> gp_zob, gp_R;
  std::vector<int> gp_slice;
  std::vector<int> sl_lb;                    // per slice (first-appearance order)
  std::vector<double> sl_zob;
  std::vector<std::vector<double>> sl_Rs;    // distinct radii, first-appearance order
  std::vector<double> lnm_x, lnm_w;
  std::vector<double> tab_lx, tab_lxm, tab_v;
  y3b::PrjBufs bufs;
  cudaStream_t stream = nullptr;
  ~y3b_prj()
  {
    if (stream) cudaStreamDestroy(stream);
  }
};

extern "C" int
y3b_prj_create(const y3b_prj_config* cfg, y3b_prj** out)
{
  using namespace y3b;
  clear_error();
  if (!cfg || !out || cfg->n_gp < 1 || cfg->n_gp > 65535 || !cfg->lambda_bin || !cfg->zo_low ||
      !cfg->zo_high ||
      !cfg->radii || cfg->n_lnm < 1 || cfg->n_per_seg < 1 || cfg->n_zring < 1 ||
      cfg->n_zouter < 1 || !(cfg->zt_high > cfg->zt_low) || !(cfg->lnm_high > cfg->lnm_low)) {
    set_error("y3b_prj_create: invalid configuration (1..65535 grid points, node counts >= 1, "
              "ordered bounds)");
    return Y3B_ERR_INVALID;
  }
  *out = nullptr;
  Y3B_TRY(require_device());
  y3b_prj* h = new (std::nothrow) y3b_prj();
  if (!h) return Y3B_ERR_NOMEM;
  h->cfg = *cfg;
  if (cfg->lob_centers && cfg->n_lob > 0)
    h->lob.assign(cfg->lob_centers, cfg->lob_centers + cfg->n_lob);
  else
    h->lob = {25.0, 37.5, 52.5, 130.0};  // sp_detail::default_lob_centers
  for (int i = 0; i < cfg->n_gp; ++i) {
    const int lb = cfg->lambda_bin[i];
    if (lb < 0 || lb >= (int)h->lob.size()) {
      set_error("y3b_prj_create: lambda_bin %d outside lob_centers", lb);
      delete h;
      return Y3B_ERR_INVALID;
    }
    const double zob = 0.5 * (cfg->zo_low[i] + cfg->zo_high[i]), R = cfg->radii[i];
    int found = -1;  // the slice registry of sigma_prj_frozen_t.hh:81-107
    for (size_t k = 0; k < h->sl_lb.size(); ++k)
      if (h->sl_lb[k] == lb && std::abs(h->sl_zob[k] - zob) < 1e-12) {
        found = (int)k;
        break;
      }
    if (found < 0) {
      h->sl_lb.push_back(lb);
      h->sl_zob.push_back(zob);
      h->sl_Rs.emplace_back();
      found = (int)h->sl_lb.size() - 1;
    }
    auto& Rs = h->sl_Rs[found];
    bool have = false;
    for (double x : Rs) have |= std::abs(x - R) < 1e-12;
    if (!have) Rs.push_back(R);
    h->gp_lb.push_back(lb);
    h->gp_zob.push_back(zob);
    h->gp_R.push_back(R);
    h->gp_slice.push_back(found);
  }
  h_gl(cfg->lnm_low, cfg->lnm_high, cfg->n_lnm, h->lnm_x, h->lnm_w);
  int rc = cuda_status(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking),
                       "cudaStreamCreate");
  if (rc) {
    delete h;
    return rc;
  }
  *out = h;
  return Y3B_OK;
}

extern "C" void
y3b_prj_destroy(y3b_prj* h)
{
  delete h;
}

extern "C" int
y3b_prj_set_mis_table(y3b_prj* h, int n_lx, const double* logx, int n_lxm,
                      const double* logxmis, const double* log_tab)
{
  using namespace y3b;
  clear_error();
  if (!h) return Y3B_ERR_INVALID;
  if (n_lx == 0) {
    h->tab_lx.clear();
    h->tab_lxm.clear();
    h->tab_v.clear();
    return Y3B_OK;
  }
  if (n_lx < 2 || n_lxm < 2 || !logx || !logxmis || !log_tab) {
    set_error("y3b_prj_set_mis_table: need at least 2 x 2 nodes and three arrays");
    return Y3B_ERR_INVALID;
  }
  for (size_t i = 0; i < (size_t)n_lx * n_lxm; ++i)
    if (!std::isfinite(log_tab[i])) {
      set_error("y3b_prj_set_mis_table: non-finite table entry");
      return Y3B_ERR_DOMAIN;
    }
  h->tab_lx.assign(logx, logx + n_lx);
  h->tab_lxm.assign(logxmis, logxmis + n_lxm);
  h->tab_v.assign(log_tab, log_tab + (size_t)n_lx * n_lxm);
  return Y3B_OK;
}

extern "C" int
y3b_prj_eval(y3b_prj* h, const y3b_prj_sample* S, double* out)
{
  using namespace y3b;
  clear_error();
  if (!h || !S || !out || !S->dist_dc || S->t.n_dist < 2 || S->t.n_hm < 2 ||
      S->t.n_hz < 2 || S->n_hl < 2 || S->n_hz < 2 || S->n_xr < 2 || S->n_xz < 2 ||
      S->n_blob < 1 || S->n_bzob < 1 || !S->bsel_lob || !S->bsel_zob || !S->b_small ||
      !S->b_large) {
    set_error("y3b_prj_eval: incomplete sample (tables of at least two nodes each)");
    return Y3B_ERR_INVALID;
  }
  const y3b_prj_config& c = h->cfg;
  const y3b_tables& t = S->t;
  const double h0 = S->cosmo.h0, om = S->cosmo.om;
  const int n_lnm = c.n_lnm, nsl = (int)h->sl_lb.size();
  const double* dz = t.dist_z;
  auto chi = [&](double z) { return h_lin_clamp(dz, S->dist_dc, t.n_dist, z) * h0; };
  // HMF on the host for the slices' z_obs: ln(m_h (Omega_M - Omega_nu)) axis.
  std::vector<double> mh(t.n_hm);
  for (int i = 0; i < t.n_hm; ++i) mh[i] = std::log(t.hmf_m_h[i] * (om - S->cosmo.onu));
  auto hmf = [&](double lnM, double z) {
    return h_bilin_clamp(mh.data(), t.n_hm, t.hmf_z, t.n_hz, t.dndlnmh, lnM, z) *
           (S->cosmo.hmf_s * (lnM * 0.4342944819 - 13.8124426028) + S->cosmo.hmf_q);
  };
  auto hmb = [&](double lnM, double z) {
    return h_bilin_clamp(S->halo_lnM, S->n_hl, S->halo_z, S->n_hz, S->bias, lnM, z);
  };
  auto r_s = [&](double lnM) {  // NFW_DSIGMA_MIS::r_s (nfw_dsigma_mis.hh:82-88)
    return std::cbrt(3.0 * std::exp(lnM) / (800.0 * kPiP * kRhoCrit)) / kConc;
  };
  auto invert_chi = [&](double target) {  // sigma_prj_frozen_t.hh:458-468
    double lo = 0.001, hi = 2.0;
    for (int it = 0; it < 40; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (chi(mid) < target)
        lo = mid;
      else
        hi = mid;
    }
    return 0.5 * (lo + hi);
  };
  // Host-built per-slice grids and factors.
  std::vector<int> t0(1, 0), z0(1, 0), tslice, zslice;
  std::vector<double> theta, geom, bsel, zz, zc, chiz, thex;
  std::vector<double> sl_chi(nsl), sl_da(nsl), sl_sci(nsl), denom(nsl);
  std::vector<double> anchor((size_t)nsl * n_lnm), wcl((size_t)nsl * n_lnm);
  for (int k = 0; k < nsl; ++k) {
    const double lobc = h->lob[h->sl_lb[k]], zob = h->sl_zob[k];
    const double chi_o = chi(zob), D_A_o = chi_o / (1.0 + zob);
    const double Rl = std::pow(lobc / 100.0, 0.2), R_excl = Rl * (1.0 + zob);
    sl_chi[k] = chi_o;
    sl_da[k] = D_A_o;
    sl_sci[k] = t.n_sci > 1 ? h_lin_clamp(t.sci_z, t.sci_val, t.n_sci, zob) : 0.0;
    // theta grid (sp_detail::build_theta_grid, sigma_prj_t.hh:95-180)
    const auto& Rs = h->sl_Rs[k];
    const double th_lam = Rl * (1.0 + zob) / chi_o, th_ex = R_excl / chi_o;
    double trmin = th_lam, trmax = th_lam;
    if (!Rs.empty()) {
      trmin = trmax = Rs[0] / D_A_o;
      for (double R : Rs) {
        trmin = std::min(trmin, R / D_A_o);
        trmax = std::max(trmax, R / D_A_o);
      }
    }
    const double th_max = std::max(c.R_max_cMpch / D_A_o, 3.0 * trmax);
    const double lower = std::max(1.0e-8, 0.1 * std::min({th_ex, trmin, th_lam}));
    std::vector<double> bp{lower, th_ex};
    for (double R : Rs) bp.push_back(R / D_A_o);
    bp.push_back(th_lam);
    bp.push_back(2.0 * th_lam);
    bp.push_back(th_max);
    std::vector<double> bc;
    for (double x : bp)
      if (std::isfinite(x) && x > 0.0 && x <= th_max) bc.push_back(x);
    std::sort(bc.begin(), bc.end());
    if (bc.empty() || bc.front() > lower) bc.insert(bc.begin(), lower);
    if (bc.back() < th_max) bc.push_back(th_max);
    std::vector<double> bd{bc.front()};
    for (size_t i = 1; i < bc.size(); ++i)
      if (bc[i] > bd.back() * (1.0 + 1.0e-6)) bd.push_back(bc[i]);
    // b_sel asymptotes linear in z_obs (sigma_prj_frozen_t.hh:200-217)
    const int nzb = S->n_bzob, nlb = S->n_blob;
    int j = 0;
    while (j + 1 < nzb && S->bsel_zob[j + 1] < zob) ++j;
    const int j0 = j + 1 < nzb ? j : std::max(nzb - 2, 0), j1 = j + 1 < nzb ? j + 1 : nzb - 1;
    const double za = S->bsel_zob[j0], zb = S->bsel_zob[j1];
    const double f = std::clamp(zb > za ? (zob - za) / (zb - za) : 0.0, 0.0, 1.0);
    const int lb = h->sl_lb[k];
    if (lb >= nlb) {
      set_error("y3b_prj_eval: b_sel_marginalised has %d richness bins, bin %d requested", nlb,
                lb);
      return Y3B_ERR_INVALID;
    }
    const double Bs = (1.0 - f) * S->b_small[j0 * nlb + lb] + f * S->b_small[j1 * nlb + lb];
    const double Bl = (1.0 - f) * S->b_large[j0 * nlb + lb] + f * S->b_large[j1 * nlb + lb];
    const double k_sig = 2.5 / th_lam, th0 = 0.5 * th_lam;
    std::vector<double> ux, uw;
    for (size_t s = 0; s + 1 < bd.size(); ++s) {
      h_gl(std::log(bd[s]), std::log(bd[s + 1]), c.n_per_seg, ux, uw);
      for (int q = 0; q < c.n_per_seg; ++q) {
        const double th = std::exp(ux[q]), w = uw[q] * th;
        theta.push_back(th);
        geom.push_back(w * 2.0 * kPiP * std::sin(th));
        bsel.push_back(Bs + (Bl - Bs) * (1.0 / (1.0 + std::exp(-k_sig * (th - th0)))));
        tslice.push_back(k);
      }
    }
    t0.push_back((int)theta.size());
    // n, b at z_obs, the a_b(z) anchor and the cl-channel mass weights
    double den = 0.0;
    for (int iM = 0; iM < n_lnm; ++iM) {
      const double x = h->lnm_x[iM], no = hmf(x, zob), bo = hmb(x, zob);
      const double a = h->lnm_w[iM] * r_s(x);
      anchor[(size_t)k * n_lnm + iM] = a;
      den += a * no * bo;
      wcl[(size_t)k * n_lnm + iM] = h->lnm_w[iM] * no * bo;
    }
    denom[k] = den + 1.0e-300;
    // line-of-sight z grid (sigma_prj_frozen_t.hh:380-455)
    const double dz1 = 1.0e-3;
    const double chi_fg = chi(c.zt_low), chi_bg = chi(c.zt_high);
    const double dchi_dz = (chi(zob + dz1) - chi(zob - dz1)) / (2.0 * dz1);
    const double dz_ex = R_excl / dchi_dz;
    const double zr_lo = std::max(zob - dz_ex, c.zt_low), zr_hi = std::min(zob + dz_ex, c.zt_high);
    std::vector<double> zs, wzs, zr, wr;
    std::vector<double> zf, wf, zb2, wb2;
    if (zr_hi > zr_lo) h_gl(zr_lo, zr_hi, c.n_zring, zr, wr);
    auto outer = [&](double dis_max, double sign, std::vector<double>& zo_, std::vector<double>& wo_) {
      if (!(R_excl < dis_max)) return;
      h_gl(std::log(R_excl), std::log(dis_max), c.n_zouter, ux, uw);
      zo_.resize(c.n_zouter);
      wo_.resize(c.n_zouter);
      for (int i = 0; i < c.n_zouter; ++i) {
        const double dis = std::exp(ux[i]);
        const double zi = invert_chi(chi_o + sign * dis);
        const double ddz = (chi(zi + dz1) - chi(zi - dz1)) / (2.0 * dz1);
        zo_[i] = zi;
        wo_[i] = uw[i] * dis / ddz;
      }
    };
    outer(chi_o - chi_fg, -1.0, zf, wf);
    outer(chi_bg - chi_o, 1.0, zb2, wb2);
    for (size_t i = zf.size(); i--;) {
      zs.push_back(zf[i]);
      wzs.push_back(wf[i]);
    }
    zs.insert(zs.end(), zr.begin(), zr.end());
    wzs.insert(wzs.end(), wr.begin(), wr.end());
    zs.insert(zs.end(), zb2.begin(), zb2.end());
    wzs.insert(wzs.end(), wb2.begin(), wb2.end());
    for (size_t i = 0; i < zs.size(); ++i) {
      const double z = zs[i], chz = chi(z);
      double da;
      if (!h_lin(dz, t.dist_da, t.n_dist, z, &da)) {
        set_error("argument out of range in Interp1D (z = %g outside distances/z)", z);
        return Y3B_ERR_DOMAIN;
      }
      const double ez = std::sqrt(om * (1 + z) * (1 + z) * (1 + z) +
                                  S->cosmo.ok * (1 + z) * (1 + z) + S->cosmo.ol);
      const double dv = 2997.92 * (1.0 + z) * (1.0 + z) * da * h0 * da * h0 / ez;
      const double omz = c.include_omega_z ? omega_z_host(z) : 1.0;
      const double sgz = h_lin_clamp(kZKernelZ, kZKernelSigma, kZKernelNodes, z);
      const double up = (z - zob) / sgz;
      const double wph = std::abs(up) < 1.0 ? 1.0 - up * up : 0.0;
      const double cz = dv * omz * wzs[i] * wph;
      if (cz == 0.0) continue;  // the reference skips these nodes entirely
      zz.push_back(z);
      zc.push_back(cz);
      chiz.push_back(chz);
      // sp_detail::theta_excl_at_z (sigma_prj_t.hh:185-194)
      double ce = (chz * chz + chi_o * chi_o - R_excl * R_excl) / (2.0 * chz * chi_o + 1.0e-30);
      thex.push_back(ce >= 1.0 - 1.0e-12 ? 0.0 : std::acos(std::max(ce, -1.0)));
      zslice.push_back(k);
    }
    z0.push_back((int)zz.size());
  }
  // Device buffers.
  cudaStream_t s = h->stream;
  y3b::PrjBufs& B = h->bufs;  // kept by the handle: no device allocation after the first call
  Y3B_TRY(B.d_mh.upload(mh.data(), mh.size(), s));
  Y3B_TRY(B.d_hz.upload(t.hmf_z, t.n_hz, s));
  Y3B_TRY(B.d_dn.upload(t.dndlnmh, (size_t)t.n_hz * t.n_hm, s));
  Y3B_TRY(B.d_bl.upload(S->halo_lnM, S->n_hl, s));
  Y3B_TRY(B.d_bz.upload(S->halo_z, S->n_hz, s));
  Y3B_TRY(B.d_bi.upload(S->bias, (size_t)S->n_hl * S->n_hz, s));
  Y3B_TRY(B.d_xr.upload(S->xi_r, S->n_xr, s));
  Y3B_TRY(B.d_xz.upload(S->xi_z, S->n_xz, s));
  Y3B_TRY(B.d_xi.upload(S->xi_nl, (size_t)S->n_xr * S->n_xz, s));
  const bool table = !h->tab_lx.empty();
  std::vector<double> thq, wthq;
  if (table) {
    Y3B_TRY(B.d_lx.upload(h->tab_lx.data(), h->tab_lx.size(), s));
    Y3B_TRY(B.d_lxm.upload(h->tab_lxm.data(), h->tab_lxm.size(), s));
    Y3B_TRY(B.d_lt.upload(h->tab_v.data(), h->tab_v.size(), s));
  } else {
    h_gl(0.0, kPiP, 256, thq, wthq);
    for (double& x : thq) x = std::cos(x);  // the quadrature reads cos(theta) of its nodes
    Y3B_TRY(B.d_th.upload(thq.data(), thq.size(), s));
    Y3B_TRY(B.d_wth.upload(wthq.data(), wthq.size(), s));
  }
  Y3B_TRY(B.d_lnx.upload(h->lnm_x.data(), n_lnm, s));
  Y3B_TRY(B.d_lnw.upload(h->lnm_w.data(), n_lnm, s));
  Y3B_TRY(B.d_theta.upload(theta.data(), theta.size(), s));
  Y3B_TRY(B.d_geom.upload(geom.data(), geom.size(), s));
  Y3B_TRY(B.d_bsel.upload(bsel.data(), bsel.size(), s));
  Y3B_TRY(B.d_ts.upload(tslice.data(), tslice.size(), s));
  Y3B_TRY(B.d_t0.upload(t0.data(), t0.size(), s));
  Y3B_TRY(B.d_z0.upload(z0.data(), z0.size(), s));
  const int nz_tot = (int)zz.size(), nth_tot = (int)theta.size(), ngp = c.n_gp;
  if (nz_tot) {
    Y3B_TRY(B.d_zz.upload(zz.data(), nz_tot, s));
    Y3B_TRY(B.d_zc.upload(zc.data(), nz_tot, s));
    Y3B_TRY(B.d_chiz.upload(chiz.data(), nz_tot, s));
    Y3B_TRY(B.d_thex.upload(thex.data(), nz_tot, s));
    Y3B_TRY(B.d_zs.upload(zslice.data(), nz_tot, s));
  }
  Y3B_TRY(B.d_anchor.upload(anchor.data(), anchor.size(), s));
  Y3B_TRY(B.d_denom.upload(denom.data(), nsl, s));
  Y3B_TRY(B.d_wcl.upload(wcl.data(), wcl.size(), s));
  Y3B_TRY(B.d_chio.upload(sl_chi.data(), nsl, s));
  Y3B_TRY(B.d_zob.upload(h->sl_zob.data(), nsl, s));
  Y3B_TRY(B.d_da.upload(sl_da.data(), nsl, s));
  Y3B_TRY(B.d_sci.upload(sl_sci.data(), nsl, s));
  Y3B_TRY(B.d_gps.upload(h->gp_slice.data(), ngp, s));
  Y3B_TRY(B.d_gpR.upload(h->gp_R.data(), ngp, s));
  Y3B_TRY(B.d_AB.alloc(std::max(nz_tot, 1)));
  Y3B_TRY(B.d_WZ.alloc((size_t)std::max(nz_tot, 1) * n_lnm));
  Y3B_TRY(B.d_wrnd.alloc((size_t)nsl * n_lnm));
  Y3B_TRY(B.d_psi.alloc(std::max(nth_tot, 1)));
  Y3B_TRY(B.d_out.alloc((size_t)ngp * 9));
  PrjTables T{t.n_hm, t.n_hz, B.d_mh.get(), B.d_hz.get(), B.d_dn.get(), S->cosmo.hmf_s,
              S->cosmo.hmf_q, S->n_hl, S->n_hz, B.d_bl.get(), B.d_bz.get(), B.d_bi.get(), S->n_xr,
              S->n_xz, B.d_xr.get(), B.d_xz.get(), B.d_xi.get(),
              table ? (int)h->tab_lx.size() : 0, table ? (int)h->tab_lxm.size() : 0,
              B.d_lx.get(), B.d_lxm.get(), B.d_lt.get(), table ? 0 : (int)thq.size(), B.d_th.get(),
              B.d_wth.get(), om};
  if (nz_tot) {
    prj_z_kernel<<<nz_tot, 128, 0, s>>>(T, n_lnm, B.d_lnx.get(), B.d_lnw.get(), B.d_zs.get(),
                                        B.d_zz.get(), B.d_zc.get(), B.d_anchor.get(), B.d_denom.get(),
                                        B.d_AB.get(), B.d_WZ.get());
    count_launch();
    Y3B_CUDA(cudaGetLastError());
  }
  prj_wrnd_kernel<<<(nsl * n_lnm + 127) / 128, 128, 0, s>>>(nsl, n_lnm, B.d_z0.get(), B.d_WZ.get(),
                                                             B.d_wrnd.get());
  count_launch();
  Y3B_CUDA(cudaGetLastError());
  prj_psi_kernel<<<(nth_tot + 127) / 128, 128, 0, s>>>(T, nth_tot, B.d_ts.get(), B.d_theta.get(),
                                                       B.d_z0.get(), B.d_chiz.get(), B.d_thex.get(),
                                                       B.d_AB.get(), B.d_chio.get(), B.d_zob.get(),
                                                       B.d_psi.get());
  count_launch();
  Y3B_CUDA(cudaGetLastError());
  int max_nt = 0;
  for (int k = 0; k < nsl; ++k) max_nt = std::max(max_nt, t0[k + 1] - t0[k]);
  const int max_pairs = std::max(max_nt * n_lnm, 1);
  Y3B_TRY(B.d_V.alloc((size_t)ngp * max_pairs));
  prj_profile_kernel<<<dim3((max_pairs + 255) / 256, ngp), 256, 0, s>>>(
    T, n_lnm, B.d_lnx.get(), B.d_gps.get(), B.d_gpR.get(), B.d_t0.get(), B.d_theta.get(), B.d_da.get(),
    max_pairs, B.d_V.get());
  count_launch();
  Y3B_CUDA(cudaGetLastError());
  prj_eval_kernel<<<ngp, 256, 0, s>>>(n_lnm, B.d_gps.get(), B.d_t0.get(), B.d_geom.get(),
                                      B.d_bsel.get(), B.d_psi.get(), B.d_wrnd.get(), B.d_wcl.get(),
                                      B.d_sci.get(), max_pairs, B.d_V.get(), B.d_out.get());
  count_launch();
  Y3B_CUDA(cudaGetLastError());
  Y3B_CUDA(cudaMemcpyAsync(out, B.d_out.get(), (size_t)ngp * 9 * sizeof(double),
                           cudaMemcpyDeviceToHost, s));
  Y3B_CUDA(cudaStreamSynchronize(s));
  return Y3B_OK;
}
