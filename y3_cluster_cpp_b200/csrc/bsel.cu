// bsel.cu -- the selection-bias operators P1, I1, J of P_operator
// (src/models/p_operator_t.hh:76-718, CosmoSIS module b_sel_marg, outputs
// b_sel_marg_P1 / _I1 / _J) on the GPU, batched over samples.
//
// Per sample the reference tabulates, on a linear reference grid z_r
// (p_operator_t.hh:124-219):
//   chi(z_r) h, dV/dz(z_r), sigma_z(z_r), n(M, z_r), b(M, z_r), and
//   p(lt | M, z_r) = exp(-lam + (lt + mi - 1) ln lam - lgamma(lt + mi)),
//   lam = l_sat + mi, mi = (l_sat sigma_lambda)^2,
//   l_sat = ((M - Mmin) / (M1 - Mmin))^alpha ((1 + z) / (1 + z_pivot))^epsilon,
// on each richness bin's own lambda_true GL nodes (0, lob_centre];
// then per grid point (z_obs bin, richness bin) (p_operator_t.hh:222-477):
//   a line-of-sight grid (GL on the exclusion ring around z_obs, log-GL in
//   comoving distance in front of and behind it), the tables interpolated
//   linearly in z onto it, the mass sums
//     W_P1[lt, z] = c_z lt w_lt sum_M w_M n p,  W_I = the same with n b,
//     c_z = (1 - u^2)_{|u| < 1} dV/dz w_z,  u = (z - z_obs) / sigma_z(z),
//   a theta grid on [min_z theta_excl(z), 2 theta_lob] split at theta_lob,
//   and
//     P1 = sum_th g_th sum_z sum_lt f_A W_P1,
//     I1 = sum_th g_th s(th) sum_z xi sum_lt f_A W_I,
//     J  = sum_th g_th (1 - s(th)) sum_z xi sum_lt f_A W_I,
//   over theta > theta_excl(z), with g_th = w_th 2 pi sin th, s the sigmoid
//   of the richness aperture, f_A the two-disk overlap fraction and xi the
//   nonlinear correlation function at z_obs and the 3-D separation.
//
// Device layout: one packed FP64 block per sample (scalars and tables);
// one kernel per (reference z node, sample) writes the per-sample tables and
// the MOR table of the richness bins in use; one 512-thread CTA per
// (grid point, sample) builds its grids in shared memory and does the sums.
// Every sum runs in the reference's order (mass, lambda_true, z, theta), and
// this file is compiled without FMA contraction, so the results follow the
// reference's FP64 arithmetic up to the last bits of the transcendental
// functions.
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

// Richness-bin centres for the edges [20, 30, 45, 60, 200] (p_op_detail::lob_center).
__host__ __device__ inline double
lob_centre(int b)
{
  return b == 0 ? 25.0 : (b == 1 ? 37.5 : (b == 2 ? 52.5 : 130.0));
}
constexpr int kPointThreads = 512;
constexpr int kSampleThreads = 128;
constexpr int kScal = 16;  // scalars at the head of a sample block

// Shapes, offsets and constant tables shared by the kernels of one call.
struct BselDims {
  int n_lt, n_zring, n_zouter, n_lnm, n_th, n_zr, n_gp, nz_max;
  double zr_lo, inv_dz_ref;
  // per-sample block: scal[16] | ln(m_h (Om - Onu)) | hmf z | dn/dlnM | dist z | d_a |
  // d_c | halo lnM | halo z | bias | xi r | xi z | xi
  int n_hm, n_hz, nd, n_hl, n_bz, n_xr, n_xz;
  long o_mh, o_hz, o_dn, o_dz, o_da, o_dc, o_bl, o_bz, o_bi, o_xr, o_xz, o_xi, blk;
  // per-sample work: chi | dV | sigma_z (n_zr each) | n, b [n_zr][n_lnm] | MOR [4][n_zr][n_lnm][n_lt]
  long w_chi, w_dv, w_sig, w_hmf, w_hmb, w_mor, mor_bin, work;
  unsigned bins_used;
  // constants (device): lnM nodes / weights, lambda_true nodes / weights /
  // R_lambda per bin [4][n_lt], reference z grid, photo-z width table,
  // grid points
  const double *lnm_x, *lnm_w, *lt_x, *lt_w, *rl, *zr, *zk_z, *zk_s;
  const double *gp_zob, *gp_zfg, *gp_zbg;
  const int* gp_bin;
};

__device__ __forceinline__ double
chi_at(const BselDims& D, const double* B, double z)  // chi_.clamp(z) h0
{
  return interp1d_clamp(B + D.o_dz, B + D.o_dc, D.nd, z) * B[4];
}

// Two-disk overlap fraction f_A(theta; theta_lob, theta_lt)
// (p_op_detail::area_overlap, p_operator_cuhre_t.hh:97-125).
__device__ __forceinline__ double
area_overlap(double theta, double theta_lob, double theta_lt)
{
  if (theta > theta_lob + theta_lt) return 0.0;
  if (theta <= fabs(theta_lob - theta_lt)) {
    if (theta_lt <= theta_lob) return 1.0;
    const double r = theta_lob / theta_lt;
    return r * r;
  }
  const double tt = theta, ll = theta_lt, lo = theta_lob;
  double c1 = (tt * tt + ll * ll - lo * lo) / (2.0 * tt * ll);
  double c2 = (tt * tt + lo * lo - ll * ll) / (2.0 * tt * lo);
  c1 = c1 < -1.0 ? -1.0 : (1.0 < c1 ? 1.0 : c1);
  c2 = c2 < -1.0 ? -1.0 : (1.0 < c2 ? 1.0 : c2);
  double sq = (-tt + ll + lo) * (tt + ll - lo) * (tt - ll + lo) * (tt + ll + lo);
  sq = sq < 0.0 ? 0.0 : sq;
  const double A = ll * ll * acos(c1) + lo * lo * acos(c2) - 0.5 * sqrt(sq);
  return A / (kPi * ll * ll);
}

// Per (reference z node, sample): chi, dV/dz, sigma_z, n(M, z), b(M, z) and
// the shifted-Poisson MOR of every richness bin in use
// (P_operator::set_sample, p_operator_t.hh:150-219).  A reference node
// outside distances/z sets the domain status (the reference's Interp1D
// throws there); the host checks this range before the launch.
__global__ void __launch_bounds__(kSampleThreads)
bsel_sample_kernel(BselDims D, const double* __restrict__ blocks, double* __restrict__ work,
                   int* status)
{
  extern __shared__ double ssm[];  // mi, lam, ln lam [n_lnm] each
  const int iz = blockIdx.x, s = blockIdx.y, tid = threadIdx.x;
  const double* B = blocks + (size_t)s * D.blk;
  double* W = work + (size_t)s * D.work;
  const double z = D.zr[iz];
  const int NM = D.n_lnm, NL = D.n_lt;
  if (tid == 0) {
    W[D.w_chi + iz] = chi_at(D, B, z);
    double dv = 0.0;
    if (!dv_do_dz(B + D.o_dz, B + D.o_da, D.nd, B[0], B[2], B[3], B[4], z, &dv))
      set_err(status, kDevDomain);
    W[D.w_dv + iz] = dv;
    W[D.w_sig + iz] = interp1d_clamp(D.zk_z, D.zk_s, kZKernelNodes, z);
  }
  double* mi_s = ssm;
  double* lam_s = mi_s + NM;
  double* llam_s = lam_s + NM;
  const double Mmin = pow(10.0, B[7]), M1 = pow(10.0, B[8]);
  const double alpha = B[9], eps = B[10], sig_l = B[11], zpiv = B[12];
  const double dM1 = M1 - Mmin;
  const double zfac = pow((1.0 + z) / (1.0 + zpiv), eps);
  for (int iM = tid; iM < NM; iM += blockDim.x) {
    const double x = D.lnm_x[iM];
    W[D.w_hmf + (size_t)iz * NM + iM] =
      interp2d_clamp(B + D.o_mh, D.n_hm, B + D.o_hz, D.n_hz, B + D.o_dn, x, z) *
      (B[5] * (x * kLog10e - kHmfPivot) + B[6]);
    W[D.w_hmb + (size_t)iz * NM + iM] =
      interp2d_clamp(B + D.o_bl, D.n_hl, B + D.o_bz, D.n_bz, B + D.o_bi, x, z);
    const double M = exp(x);
    const double dM = fmax(M - Mmin, 0.0);
    const double l_sat = (dM > 0.0 && dM1 > 0.0) ? pow(dM / dM1, alpha) * zfac : 0.0;
    const double mi = (l_sat * sig_l) * (l_sat * sig_l);
    const double lam = fmax(l_sat + mi, 1.0e-300);
    mi_s[iM] = mi;
    lam_s[iM] = lam;
    llam_s[iM] = log(lam);
  }
  __syncthreads();
  const int per_bin = NM * NL;
  for (int bb = 0; bb < 4; ++bb) {
    if (!((D.bins_used >> bb) & 1u)) continue;
    double* dst = W + D.w_mor + (size_t)bb * D.mor_bin + (size_t)iz * per_bin;
    const double* ltx = D.lt_x + bb * NL;
    for (int k = tid; k < per_bin; k += blockDim.x) {
      const int iM = k / NL, il = k - iM * NL;
      const double x = ltx[il] + mi_s[iM];
      dst[k] = exp(-lam_s[iM] + (x - 1.0) * llam_s[iM] - lgamma(x));
    }
  }
}

// Shared-memory doubles of bsel_point_kernel for the shapes in D.
__host__ __device__ inline long
point_smem_doubles(const BselDims& D)
{
  const long NZ = D.nz_max;
  return 9 * NZ + 4L * D.n_zouter + 5L * D.n_th + D.n_xr + 2L * D.n_lt * NZ +
         3L * D.n_th * NZ + kScal + 16 + (NZ + 1) / 2;
}

// Lower bracket of z on the reference grid: i = min(trunc(u), n - 2) with
// u = (z - z_r0) / dz, the reference's size_t conversion
// (p_operator_t.hh:263-270); a u at or below -1 wraps to n - 2 there.
__device__ __forceinline__ int
ref_bracket(const BselDims& D, double z, double* f)
{
  const double u = (z - D.zr_lo) * D.inv_dz_ref;
  const long long t = (long long)u;
  const int i = t < 0 ? D.n_zr - 2 : (int)min(t, (long long)(D.n_zr - 2));
  *f = u - i;
  return i;
}

// One CTA per (grid point, sample): P_operator::evaluate
// (p_operator_t.hh:222-477) with its grids in shared memory.
__global__ void __launch_bounds__(kPointThreads, 2)
bsel_point_kernel(BselDims D, const double* __restrict__ blocks,
                  const double* __restrict__ work, double* __restrict__ out)
{
  extern __shared__ double sm[];
  const int g = blockIdx.x, s = blockIdx.y, tid = threadIdx.x, nt = blockDim.x;
  const double* B = blocks + (size_t)s * D.blk;
  const double* Wk = work + (size_t)s * D.work;
  const int NZ = D.nz_max, NL = D.n_lt, NT = D.n_th, NO = D.n_zouter, NR = D.n_zring;
  const int NM = D.n_lnm;
  double* zs = sm;
  double* wzs = zs + NZ;
  double* chz = wzs + NZ;
  double* dvz = chz + NZ;
  double* sgz = dvz + NZ;
  double* wzv = sgz + NZ;
  double* thx = wzv + NZ;
  double* ic1 = thx + NZ;
  double* fzz = ic1 + NZ;
  double* ufg = fzz + NZ;
  double* wufg = ufg + NO;
  double* ubg = wufg + NO;
  double* wubg = ubg + NO;
  double* ths = wubg + NO;
  double* wths = ths + NT;
  double* sgm = wths + NT;
  double* omt = sgm + NT;
  double* cst = omt + NT;
  double* xir = cst + NT;
  double* WP = xir + D.n_xr;
  double* WI = WP + (size_t)NL * NZ;
  double* pP = WI + (size_t)NL * NZ;
  double* pI = pP + (size_t)NT * NZ;
  double* pJ = pI + (size_t)NT * NZ;
  double* sc = pJ + (size_t)NT * NZ;
  int* izl = reinterpret_cast<int*>(sc + kScal + 16);  // after 8 doubles of counts and 5 chi(z)
  // scalars: 0 zob, 1 chi_o, 2 theta_lob, 3 R_excl, 4 ln R_excl, 5 ln(chi_o - chi_fg),
  // 6 ln(chi_bg - chi_o), 7 ring lo, 8 ring hi, 9 th_lo, 10 th_hi, 11 th_mid,
  // 12 ln r_0, 13 1 / dln r, 14 k_sig, 15 th0_sig; ints after: n_fg, n_ring, n_bg, split, empty
  int* cnt = reinterpret_cast<int*>(sc + kScal);
  const int bin = D.gp_bin[g];
  const double ddz = 1.0e-3;

  if (tid < 5) {  // the five chi(z) this point needs, one lookup per thread
    const double zob = D.gp_zob[g];
    const double zq[5] = {zob, D.gp_zfg[g], D.gp_zbg[g], zob + ddz, zob - ddz};
    sc[kScal + 8 + tid] = chi_at(D, B, zq[tid]);
  }
  __syncthreads();
  if (tid == 0) {
    const double zob = D.gp_zob[g];
    const double Rlob = pow(lob_centre(bin) / 100.0, 0.2);  // p_op_detail::R_lambda
    const double* cq = sc + kScal + 8;
    const double chi_o = cq[0];
    const double theta_lob = Rlob * (1.0 + zob) / chi_o;
    const double R_excl = Rlob * (1.0 + zob);
    // build_z_grid_ (p_operator_t.hh:503-583)
    const double zfg = D.gp_zfg[g], zbg = D.gp_zbg[g];
    const double chi_fg = cq[1], chi_bg = cq[2];
    const double dchi_dz = (cq[3] - cq[4]) / (2.0 * ddz);
    const double dz_excl = R_excl / dchi_dz;
    const double zr_lo = fmax(zob - dz_excl, zfg), zr_hi = fmin(zob + dz_excl, zbg);
    const double dfg = chi_o - chi_fg, dbg = chi_bg - chi_o;
    cnt[0] = R_excl < dfg ? NO : 0;
    cnt[1] = zr_hi > zr_lo ? NR : 0;
    cnt[2] = R_excl < dbg ? NO : 0;
    sc[0] = zob;
    sc[1] = chi_o;
    sc[2] = theta_lob;
    sc[3] = R_excl;
    sc[4] = log(R_excl);
    sc[5] = cnt[0] ? log(dfg) : 0.0;
    sc[6] = cnt[2] ? log(dbg) : 0.0;
    sc[7] = zr_lo;
    sc[8] = zr_hi;
    sc[14] = 2.5 / theta_lob;
    sc[15] = 0.5 * theta_lob;
    const double* xr = B + D.o_xr;
    sc[12] = log(xr[0]);
    sc[13] = 1.0 / log(xr[1] / xr[0]);
  }
  __syncthreads();
  const int n_fg = cnt[0], n_ring = cnt[1], n_bg = cnt[2];
  const int Nz = n_fg + n_ring + n_bg;
  const double zob = sc[0], chi_o = sc[1], theta_lob = sc[2], R_excl = sc[3];
  {  // GL nodes of the two log-distance wings and of the ring
    const int hO = (NO + 1) / 2, hR = (NR + 1) / 2;
    for (int i = tid; i < 2 * hO + hR; i += nt) {
      if (i < hO) {
        if (n_fg) gl_node_pair(sc[4], sc[5], NO, i, ufg, wufg);
      } else if (i < 2 * hO) {
        if (n_bg) gl_node_pair(sc[4], sc[6], NO, i - hO, ubg, wubg);
      } else if (n_ring) {
        gl_node_pair(sc[7], sc[8], NR, i - 2 * hO, zs + n_fg, wzs + n_fg);
      }
    }
  }
  __syncthreads();
  for (int i = tid; i < n_fg + n_bg; i += nt) {  // wing nodes: z(chi_o -+ dis)
    const bool fg = i < n_fg;
    const int k = fg ? i : i - n_fg;
    const double dis = exp(fg ? ufg[k] : ubg[k]);
    const double target = fg ? chi_o - dis : chi_o + dis;
    double lo = 0.001, hi = 2.0;  // invert_chi_ (p_operator_t.hh:621-632)
    for (int it = 0; it < 40; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (chi_at(D, B, mid) < target)
        lo = mid;
      else
        hi = mid;
    }
    const double zi = 0.5 * (lo + hi);
    const double dd = (chi_at(D, B, zi + ddz) - chi_at(D, B, zi - ddz)) / (2.0 * ddz);
    const int o = fg ? n_fg - 1 - k : n_fg + n_ring + k;  // fg reversed, ring, bg
    zs[o] = zi;
    wzs[o] = (fg ? wufg[k] : wubg[k]) * dis / dd;
  }
  __syncthreads();
  // z-node tables, photo-z weight, exclusion angle
  for (int iz = tid; iz < Nz; iz += nt) {
    const double z = zs[iz];
    double f;
    const int i = ref_bracket(D, z, &f);
    izl[iz] = i;
    fzz[iz] = f;
    const double* cr = Wk + D.w_chi;
    const double* dr = Wk + D.w_dv;
    const double* sr = Wk + D.w_sig;
    const double cz = cr[i] + f * (cr[i + 1] - cr[i]);
    chz[iz] = cz;
    dvz[iz] = dr[i] + f * (dr[i + 1] - dr[i]);
    const double sg = sr[i] + f * (sr[i + 1] - sr[i]);
    sgz[iz] = sg;
    const double u = (z - zob) / sg;
    wzv[iz] = fabs(u) < 1.0 ? 1.0 - u * u : 0.0;
    double ce = (cz * cz + chi_o * chi_o - R_excl * R_excl) / (2.0 * cz * chi_o);
    ce = ce < -1.0 ? -1.0 : (1.0 < ce ? 1.0 : ce);
    thx[iz] = ce >= 1.0 - 1e-12 ? 1e-6 : acos(ce);
    ic1[iz] = (1.0 + z) / cz;
  }
  __syncthreads();
  if (tid == 0) {  // theta range and split (p_operator_t.hh:352-395)
    const double th_hi = 2.0 * theta_lob;
    double th_lo = th_hi;
    for (int iz = 0; iz < Nz; ++iz)
      if (thx[iz] < th_lo) th_lo = thx[iz];
    const int N1 = NT / 2, N2 = NT - N1;
    const double th_mid = th_lo > theta_lob ? th_lo : (th_hi < theta_lob ? th_hi : theta_lob);
    cnt[3] = !(N1 == 0 || th_mid <= th_lo || N2 == 0 || th_mid >= th_hi);
    cnt[4] = th_lo >= th_hi;
    sc[9] = th_lo;
    sc[10] = th_hi;
    sc[11] = th_mid;
  }
  __syncthreads();
  double* o = out + ((size_t)s * D.n_gp + g) * 3;
  if (cnt[4]) {  // fully excluded: the integrand is zero
    if (tid < 3) o[tid] = 0.0;
    return;
  }
  {
    const int N1 = NT / 2, N2 = NT - N1;
    if (cnt[3]) {
      for (int i = tid; i < (N1 + 1) / 2 + (N2 + 1) / 2; i += nt) {
        if (i < (N1 + 1) / 2)
          gl_node_pair(sc[9], sc[11], N1, i, ths, wths);
        else
          gl_node_pair(sc[11], sc[10], N2, i - (N1 + 1) / 2, ths + N1, wths + N1);
      }
    } else {
      for (int i = tid; i < (NT + 1) / 2; i += nt) gl_node_pair(sc[9], sc[10], NT, i, ths, wths);
    }
  }
  {  // xi_NL(r, z_obs): linear in z on the evenly spaced z axis
    const double* xz = B + D.o_xz;
    const double u = (zob - xz[0]) * (1.0 / (xz[1] - xz[0]));
    int j = (int)floor(u);
    j = j < 0 ? 0 : (j > D.n_xz - 2 ? D.n_xz - 2 : j);
    const double fz = u - j;
    const double* r0 = B + D.o_xi + (size_t)j * D.n_xr;
    const double* r1 = r0 + D.n_xr;
    for (int ir = tid; ir < D.n_xr; ir += nt) xir[ir] = r0[ir] + fz * (r1[ir] - r0[ir]);
  }
  __syncthreads();
  for (int it = tid; it < NT; it += nt) {  // theta-only caches
    const double th = ths[it];
    const double sn = sin(th);
    cst[it] = cos(th);
    sgm[it] = 1.0 / (1.0 + exp(-sc[14] * (th - sc[15])));
    omt[it] = wths[it] * 2.0 * kPi * sn;
  }
  // Mass sums W_P1[lt, z], W_I[lt, z] (p_operator_t.hh:433-455), z nodes in
  // the photo-z support only; lambda_true fastest for the MOR reads.
  {
    const double* ltx = D.lt_x + bin * NL;
    const double* ltw = D.lt_w + bin * NL;
    const double* hm = Wk + D.w_hmf;
    const double* hb = Wk + D.w_hmb;
    const double* mor = Wk + D.w_mor + (size_t)bin * D.mor_bin;
    for (int k = tid; k < Nz * NL; k += nt) {
      const int iz = k / NL, il = k - iz * NL;
      if (wzv[iz] == 0.0) continue;
      const double pref = wzv[iz] * dvz[iz] * wzs[iz];
      const double lt_wlt = ltx[il] * ltw[il];
      const int i = izl[iz];
      const double f = fzz[iz];
      const double* h0r = hm + (size_t)i * NM;
      const double* h1r = h0r + NM;
      const double* b0r = hb + (size_t)i * NM;
      const double* b1r = b0r + NM;
      const double* m0 = mor + (size_t)i * NM * NL + il;
      const double* m1 = m0 + (size_t)NM * NL;
      double aP = 0.0, aI = 0.0;
      for (int iM = 0; iM < NM; ++iM) {
        const double nM = h0r[iM] + f * (h1r[iM] - h0r[iM]);
        const double bM = b0r[iM] + f * (b1r[iM] - b0r[iM]);
        const double a = m0[(size_t)iM * NL], b = m1[(size_t)iM * NL];
        const double pm = a + f * (b - a);
        const double common = D.lnm_w[iM] * nM * pm;
        aP += common;
        aI += common * bM;
      }
      WP[(size_t)il * NZ + iz] = pref * lt_wlt * aP;
      WI[(size_t)il * NZ + iz] = pref * lt_wlt * aI;
    }
  }
  __syncthreads();
  // (theta, z) partial sums over lambda_true (p_operator_t.hh:457-505)
  {
    const double* rl = D.rl + bin * NL;
    const double r_lo = B[D.o_xr], r_hi = B[D.o_xr + D.n_xr - 1];
    for (int k = tid; k < NT * Nz; k += nt) {
      const int it = k / Nz, iz = k - it * Nz;
      const double theta = ths[it];
      double sP1 = 0.0, sI1 = 0.0, sJ = 0.0;
      if (wzv[iz] != 0.0 && theta > thx[iz]) {
        const double cz = chz[iz];
        const double dchi =
          sqrt(fmax(cz * cz + chi_o * chi_o - 2.0 * cz * chi_o * cst[it], 0.0));
        // xi_lookup_ (p_operator_t.hh:636-647)
        const double r = dchi < r_lo ? r_lo : (r_hi < dchi ? r_hi : dchi);
        const double u = (log(r) - sc[12]) * sc[13];
        int ir = (int)floor(u);
        ir = ir < 0 ? 0 : (ir > D.n_xr - 2 ? D.n_xr - 2 : ir);
        const double fr = u - ir;
        const double xi = xir[ir] + fr * (xir[ir + 1] - xir[ir]);
        const double icz = ic1[iz];
        for (int il = 0; il < NL; ++il) {
          const double theta_lt = rl[il] * icz;
          const double fA = area_overlap(theta, theta_lob, theta_lt);
          const double wb = fA * WP[(size_t)il * NZ + iz];
          const double wi = fA * WI[(size_t)il * NZ + iz];
          sP1 += wb;
          sI1 += wi * xi;
          sJ += wi * xi;
        }
        sI1 = sI1 * sgm[it];
        sJ = sJ * (1.0 - sgm[it]);
      }
      pP[(size_t)it * NZ + iz] = sP1;
      pI[(size_t)it * NZ + iz] = sI1;
      pJ[(size_t)it * NZ + iz] = sJ;
    }
  }
  __syncthreads();
  // z in order per theta node, then theta in order.
  for (int it = tid; it < NT; it += nt) {
    double a = 0.0, b = 0.0, c = 0.0;
    for (int iz = 0; iz < Nz; ++iz) {
      a += pP[(size_t)it * NZ + iz];
      b += pI[(size_t)it * NZ + iz];
      c += pJ[(size_t)it * NZ + iz];
    }
    pP[(size_t)it * NZ] = a;
    pI[(size_t)it * NZ] = b;
    pJ[(size_t)it * NZ] = c;
  }
  __syncthreads();
  if (tid == 0) {
    double P1 = 0.0, I1 = 0.0, J = 0.0;
    for (int it = 0; it < NT; ++it) {
      P1 += omt[it] * pP[(size_t)it * NZ];
      I1 += omt[it] * pI[(size_t)it * NZ];
      J += omt[it] * pJ[(size_t)it * NZ];
    }
    o[0] = P1;
    o[1] = I1;
    o[2] = J;
  }
}

}  // namespace
}  // namespace y3b

struct y3b_bsel {
  y3b_bsel_config cfg;
  std::vector<double> gp_zlo, gp_zhi, gp_zob, gp_zfg, gp_zbg;
  std::vector<int> gp_bin;
  std::vector<double> lnm_x, lnm_w, lt_x, lt_w, rl, zr;  // lt_x, lt_w, rl: [4][n_lt]
  unsigned bins_used = 0;
  int max_samples = 64;
  y3b::DevBuf<double> d_const, d_blocks, d_work, d_out;
  y3b::DevBuf<int> d_int;  // grid-point bins | status word
  double* h_stage = nullptr;  // pinned: sample blocks
  size_t h_stage_cap = 0;
  double* h_out = nullptr;  // pinned: results
  size_t h_out_cap = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};  // around each chunk's kernels
  double last_kernel_ms = 0.0;
  ~y3b_bsel()
  {
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
    if (h_stage) cudaFreeHost(h_stage);
    if (h_out) cudaFreeHost(h_out);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace y3b {
namespace {

double
h_sigma_z(double z)  // Interp1D(z_kernel_z, z_kernel_sigma).clamp(z)
{
  z = std::min(std::max(z, kZKernelZ[0]), kZKernelZ[kZKernelNodes - 1]);
  int lo = 0, hi = kZKernelNodes - 1;
  while (hi > lo + 1) {
    const int m = (lo + hi) / 2;
    if (kZKernelZ[m] > z)
      hi = m;
    else
      lo = m;
  }
  const double dx = kZKernelZ[lo + 1] - kZKernelZ[lo];
  return kZKernelSigma[lo] + (z - kZKernelZ[lo]) / dx * (kZKernelSigma[lo + 1] - kZKernelSigma[lo]);
}

// Photo-z support of a z_obs: z_fg + sigma_z(z_fg) = z_obs and
// z_bg - sigma_z(z_bg) = z_obs by bisection (bisect_photoz_fg_ / _bg_,
// p_operator_t.hh:590-618).
double
bisect_fg(double zob)
{
  double lo = 0.01, hi = zob;
  if (lo + h_sigma_z(lo) - zob > 0.0) return lo;
  for (int it = 0; it < 50; ++it) {
    const double mid = 0.5 * (lo + hi);
    const double f = mid + h_sigma_z(mid) - zob;
    if (f < 0.0)
      lo = mid;
    else
      hi = mid;
  }
  return 0.5 * (lo + hi);
}

double
bisect_bg(double zob)
{
  double lo = zob, hi = 1.5;
  if (hi - h_sigma_z(hi) - zob < 0.0) return hi;
  for (int it = 0; it < 50; ++it) {
    const double mid = 0.5 * (lo + hi);
    const double f = mid - h_sigma_z(mid) - zob;
    if (f < 0.0)
      lo = mid;
    else
      hi = mid;
  }
  return 0.5 * (lo + hi);
}

// Shapes and offsets of one call's sample blocks and work areas.
void
layout(const y3b_bsel* h, const y3b_bsel_sample& s0, BselDims& D)
{
  const y3b_bsel_config& c = h->cfg;
  D.n_lt = c.n_lt;
  D.n_zring = c.n_zring;
  D.n_zouter = c.n_zouter;
  D.n_lnm = c.n_lnm;
  D.n_th = c.n_theta;
  D.n_zr = c.n_zt_ref;
  D.n_gp = c.n_gp;
  D.nz_max = c.n_zring + 2 * c.n_zouter;
  D.zr_lo = c.zt_ref_low;
  D.inv_dz_ref = 1.0 / ((c.zt_ref_high - c.zt_ref_low) / (c.n_zt_ref - 1));
  D.n_hm = s0.t.n_hm;
  D.n_hz = s0.t.n_hz;
  D.nd = s0.t.n_dist;
  D.n_hl = s0.n_hl;
  D.n_bz = s0.n_hz;
  D.n_xr = s0.n_xr;
  D.n_xz = s0.n_xz;
  long o = kScal;
  D.o_mh = o, o += D.n_hm;
  D.o_hz = o, o += D.n_hz;
  D.o_dn = o, o += (long)D.n_hm * D.n_hz;
  D.o_dz = o, o += D.nd;
  D.o_da = o, o += D.nd;
  D.o_dc = o, o += D.nd;
  D.o_bl = o, o += D.n_hl;
  D.o_bz = o, o += D.n_bz;
  D.o_bi = o, o += (long)D.n_hl * D.n_bz;
  D.o_xr = o, o += D.n_xr;
  D.o_xz = o, o += D.n_xz;
  D.o_xi = o, o += (long)D.n_xr * D.n_xz;
  D.blk = (o + 1) & ~1L;
  long w = 0;
  D.w_chi = w, w += D.n_zr;
  D.w_dv = w, w += D.n_zr;
  D.w_sig = w, w += D.n_zr;
  D.w_hmf = w, w += (long)D.n_zr * D.n_lnm;
  D.w_hmb = w, w += (long)D.n_zr * D.n_lnm;
  D.w_mor = (w + 1) & ~1L;
  D.mor_bin = (long)D.n_zr * D.n_lnm * D.n_lt;
  D.work = D.w_mor + 4 * D.mor_bin;
  D.bins_used = h->bins_used;
}

}  // namespace
}  // namespace y3b

extern "C" int
y3b_bsel_create(const y3b_bsel_config* cfg, y3b_bsel** out)
{
  using namespace y3b;
  clear_error();
  if (!cfg || !out || cfg->n_gp < 1 || !cfg->zo_low || !cfg->zo_high || !cfg->lambda_bin ||
      cfg->n_lt < 1 || cfg->n_zring < 1 || cfg->n_zouter < 1 || cfg->n_lnm < 1 ||
      cfg->n_theta < 1 || cfg->n_zt_ref < 2 || !(cfg->zt_ref_high > cfg->zt_ref_low) ||
      !(cfg->lnm_high > cfg->lnm_low) || cfg->max_samples < 0 ||
      cfg->max_samples > 65535) {
    set_error("y3b_bsel_create: invalid configuration (grid points, node counts >= 1, "
              "n_zt_ref >= 2, ordered bounds, max_samples <= 65535)");
    return Y3B_ERR_INVALID;
  }
  *out = nullptr;
  Y3B_TRY(require_device());
  y3b_bsel* h = new (std::nothrow) y3b_bsel();
  if (!h) return Y3B_ERR_NOMEM;
  h->cfg = *cfg;
  if (cfg->max_samples > 0) h->max_samples = cfg->max_samples;
  const int ngp = cfg->n_gp;
  for (int i = 0; i < ngp; ++i) {
    const int b = cfg->lambda_bin[i];
    if (b < 0 || b > 3) {
      set_error("y3b_bsel_create: lambda_bin %d outside the four richness bins", b);
      delete h;
      return Y3B_ERR_INVALID;
    }
    const double zob = 0.5 * (cfg->zo_low[i] + cfg->zo_high[i]);
    h->gp_zlo.push_back(cfg->zo_low[i]);
    h->gp_zhi.push_back(cfg->zo_high[i]);
    h->gp_zob.push_back(zob);
    h->gp_bin.push_back(b);
    h->gp_zfg.push_back(bisect_fg(zob));
    h->gp_zbg.push_back(bisect_bg(zob));
    h->bins_used |= 1u << b;
  }
  h->cfg.zo_low = h->gp_zlo.data();
  h->cfg.zo_high = h->gp_zhi.data();
  h->cfg.lambda_bin = h->gp_bin.data();
  gl_nodes_host(cfg->lnm_low, cfg->lnm_high, cfg->n_lnm, h->lnm_x, h->lnm_w);
  std::vector<double> x, w;
  for (int b = 0; b < 4; ++b) {
    gl_nodes_host(1.0e-6, lob_centre(b), cfg->n_lt, x, w);
    for (int il = 0; il < cfg->n_lt; ++il) {
      h->lt_x.push_back(x[il]);
      h->lt_w.push_back(w[il]);
      h->rl.push_back(std::pow(x[il] / 100.0, 0.2));
    }
  }
  const double dz_ref = (cfg->zt_ref_high - cfg->zt_ref_low) / (cfg->n_zt_ref - 1);
  for (int i = 0; i < cfg->n_zt_ref; ++i) h->zr.push_back(cfg->zt_ref_low + i * dz_ref);
  // Constant tables in one device buffer.
  std::vector<double> cst;
  auto put = [&](const double* p, size_t n) { cst.insert(cst.end(), p, p + n); };
  put(h->lnm_x.data(), h->lnm_x.size());
  put(h->lnm_w.data(), h->lnm_w.size());
  put(h->lt_x.data(), h->lt_x.size());
  put(h->lt_w.data(), h->lt_w.size());
  put(h->rl.data(), h->rl.size());
  put(h->zr.data(), h->zr.size());
  put(kZKernelZ, kZKernelNodes);
  put(kZKernelSigma, kZKernelNodes);
  put(h->gp_zob.data(), ngp);
  put(h->gp_zfg.data(), ngp);
  put(h->gp_zbg.data(), ngp);
  int rc = cuda_status(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking),
                       "cudaStreamCreate");
  std::vector<int> ints(h->gp_bin);
  ints.push_back(0);
  for (int i = 0; i < 2 && !rc; ++i)
    rc = cuda_status(cudaEventCreate(&h->ev[i]), "cudaEventCreate");
  if (!rc) rc = h->d_const.upload(cst.data(), cst.size(), h->stream);
  if (!rc) rc = h->d_int.upload(ints.data(), ints.size(), h->stream);
  if (!rc) rc = cuda_status(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  if (rc) {
    delete h;
    return rc;
  }
  *out = h;
  return Y3B_OK;
}

extern "C" int
y3b_bsel_kernel_ms(const y3b_bsel* h, double* ms)
{
  y3b::clear_error();
  if (!h || !ms) {
    y3b::set_error("y3b_bsel_kernel_ms: invalid arguments");
    return Y3B_ERR_INVALID;
  }
  *ms = h->last_kernel_ms;
  return Y3B_OK;
}

extern "C" void
y3b_bsel_destroy(y3b_bsel* h)
{
  delete h;
}

extern "C" int
y3b_bsel_eval(y3b_bsel* h, int n_samples, const y3b_bsel_sample* S, double* out)
{
  using namespace y3b;
  clear_error();
  if (!h || n_samples < 0 || (n_samples && (!S || !out))) {
    set_error("y3b_bsel_eval: invalid arguments");
    return Y3B_ERR_INVALID;
  }
  if (n_samples == 0) return Y3B_OK;
  const y3b_bsel_config& c = h->cfg;
  const y3b_bsel_sample& s0 = S[0];
  for (int k = 0; k < n_samples; ++k) {
    const y3b_bsel_sample& s = S[k];
    const y3b_tables& t = s.t;
    if (!t.hmf_m_h || !t.hmf_z || !t.dndlnmh || !t.dist_z || !t.dist_da || !s.dist_dc ||
        !s.halo_lnM || !s.halo_z || !s.bias || !s.xi_r || !s.xi_z || !s.xi_nl || t.n_hm < 2 ||
        t.n_hz < 2 || t.n_dist < 2 || s.n_hl < 2 || s.n_hz < 2 || s.n_xr < 2 || s.n_xz < 2) {
      set_error("y3b_bsel_eval: sample %d is incomplete (tables of at least two nodes each)", k);
      return Y3B_ERR_INVALID;
    }
    if (t.n_hm != s0.t.n_hm || t.n_hz != s0.t.n_hz || t.n_dist != s0.t.n_dist ||
        s.n_hl != s0.n_hl || s.n_hz != s0.n_hz || s.n_xr != s0.n_xr || s.n_xz != s0.n_xz) {
      set_error("y3b_bsel_eval: sample %d has table shapes different from sample 0", k);
      return Y3B_ERR_INVALID;
    }
    if (!(c.zt_ref_low >= t.dist_z[0] && c.zt_ref_high <= t.dist_z[t.n_dist - 1])) {
      set_error("argument out of range in Interp1D (sample %d: the reference z grid "
                "[%g, %g] leaves distances/z)", k, c.zt_ref_low, c.zt_ref_high);
      return Y3B_ERR_DOMAIN;
    }
  }
  BselDims D;
  layout(h, s0, D);
  const size_t smem = (size_t)point_smem_doubles(D) * sizeof(double);
  if (smem > 227 * 1024) {
    set_error("y3b_bsel_eval: node counts need %zu bytes of shared memory per grid point "
              "(at most 227 KB)", smem);
    return Y3B_ERR_INVALID;
  }
  Y3B_CUDA(cudaFuncSetAttribute(bsel_point_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem));
  const double* cd = h->d_const.get();
  const int NL = c.n_lt, ngp = c.n_gp;
  D.lnm_x = cd;
  D.lnm_w = D.lnm_x + c.n_lnm;
  D.lt_x = D.lnm_w + c.n_lnm;
  D.lt_w = D.lt_x + 4 * NL;
  D.rl = D.lt_w + 4 * NL;
  D.zr = D.rl + 4 * NL;
  D.zk_z = D.zr + c.n_zt_ref;
  D.zk_s = D.zk_z + kZKernelNodes;
  D.gp_zob = D.zk_s + kZKernelNodes;
  D.gp_zfg = D.gp_zob + ngp;
  D.gp_zbg = D.gp_zfg + ngp;
  D.gp_bin = h->d_int.get();
  int* d_status = h->d_int.get() + ngp;
  const int chunk = std::min(n_samples, h->max_samples);
  // Pinned staging for the sample blocks and the results.
  const size_t stage = (size_t)chunk * D.blk, outn = (size_t)chunk * ngp * 3;
  if (h->h_stage_cap < stage) {
    if (h->h_stage) cudaFreeHost(h->h_stage);
    h->h_stage = nullptr;
    h->h_stage_cap = 0;
    Y3B_CUDA(cudaHostAlloc((void**)&h->h_stage, stage * sizeof(double), cudaHostAllocDefault));
    h->h_stage_cap = stage;
  }
  if (h->h_out_cap < outn) {
    if (h->h_out) cudaFreeHost(h->h_out);
    h->h_out = nullptr;
    h->h_out_cap = 0;
    Y3B_CUDA(cudaHostAlloc((void**)&h->h_out, outn * sizeof(double), cudaHostAllocDefault));
    h->h_out_cap = outn;
  }
  Y3B_TRY(h->d_blocks.alloc(stage));
  Y3B_TRY(h->d_work.alloc((size_t)chunk * D.work));
  Y3B_TRY(h->d_out.alloc(outn));
  cudaStream_t st = h->stream;
  Y3B_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), st));
  h->last_kernel_ms = 0.0;
  for (int k0 = 0; k0 < n_samples; k0 += chunk) {
    const int nk = std::min(chunk, n_samples - k0);
    // The previous chunk's copies out of the staging buffers are done.
    Y3B_CUDA(cudaStreamSynchronize(st));
    for (int k = 0; k < nk; ++k) {
      const y3b_bsel_sample& s = S[k0 + k];
      double* b = h->h_stage + (size_t)k * D.blk;
      const double sc[kScal] = {s.cosmo.om, s.cosmo.onu, s.cosmo.ol, s.cosmo.ok, s.cosmo.h0,
                                s.cosmo.hmf_s, s.cosmo.hmf_q, s.hod[0], s.hod[1], s.hod[2],
                                s.hod[3], s.hod[4], s.hod[5], 0.0, 0.0, 0.0};
      std::memcpy(b, sc, sizeof sc);
      for (int i = 0; i < D.n_hm; ++i)  // HMF_t's log mass axis (hmf_t.hh:16-25)
        b[D.o_mh + i] = std::log(s.t.hmf_m_h[i] * (s.cosmo.om - s.cosmo.onu));
      std::memcpy(b + D.o_hz, s.t.hmf_z, sizeof(double) * D.n_hz);
      std::memcpy(b + D.o_dn, s.t.dndlnmh, sizeof(double) * D.n_hz * D.n_hm);
      std::memcpy(b + D.o_dz, s.t.dist_z, sizeof(double) * D.nd);
      std::memcpy(b + D.o_da, s.t.dist_da, sizeof(double) * D.nd);
      std::memcpy(b + D.o_dc, s.dist_dc, sizeof(double) * D.nd);
      std::memcpy(b + D.o_bl, s.halo_lnM, sizeof(double) * D.n_hl);
      std::memcpy(b + D.o_bz, s.halo_z, sizeof(double) * D.n_bz);
      std::memcpy(b + D.o_bi, s.bias, sizeof(double) * D.n_hl * D.n_bz);
      std::memcpy(b + D.o_xr, s.xi_r, sizeof(double) * D.n_xr);
      std::memcpy(b + D.o_xz, s.xi_z, sizeof(double) * D.n_xz);
      std::memcpy(b + D.o_xi, s.xi_nl, sizeof(double) * D.n_xr * D.n_xz);
    }
    Y3B_CUDA(cudaMemcpyAsync(h->d_blocks.get(), h->h_stage, sizeof(double) * nk * D.blk,
                             cudaMemcpyHostToDevice, st));
    Y3B_CUDA(cudaEventRecord(h->ev[0], st));
    bsel_sample_kernel<<<dim3(D.n_zr, nk), kSampleThreads, 3 * sizeof(double) * c.n_lnm, st>>>(
      D, h->d_blocks.get(), h->d_work.get(), d_status);
    count_launch();
    Y3B_CUDA(cudaGetLastError());
    bsel_point_kernel<<<dim3(ngp, nk), kPointThreads, smem, st>>>(D, h->d_blocks.get(),
                                                                 h->d_work.get(), h->d_out.get());
    count_launch();
    Y3B_CUDA(cudaGetLastError());
    Y3B_CUDA(cudaEventRecord(h->ev[1], st));
    Y3B_CUDA(cudaMemcpyAsync(h->h_out, h->d_out.get(), sizeof(double) * nk * ngp * 3,
                             cudaMemcpyDeviceToHost, st));
    Y3B_CUDA(cudaStreamSynchronize(st));
    float ms = 0.f;
    Y3B_CUDA(cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]));
    h->last_kernel_ms += ms;
    std::memcpy(out + (size_t)k0 * ngp * 3, h->h_out, sizeof(double) * nk * ngp * 3);
  }
  return read_device_status(d_status, st);
}
