// engine_internal.h -- shared layout of the batched engine (host + device).
//
// Per grid (node density) the engine keeps FP64 nodes/weights and the
// walker-independent kernels K_i(lam_t, z_q) = sum_o a_o P(lam_o | lam_t, z_q)
// and K_j(z_q) = sum_zo b N(z_o; z_q, sigma_z).  Per point the prep kernel
// writes FP64 z-factors and either the FP64 mass/MOR factors of the direct
// form or the FP32 factor vectors of the mixed (tensor-core) form.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/y3b.h"

namespace y3b {

constexpr int kMaxLamBins = 8;
constexpr int kMaxZBins = 8;
constexpr int kMaxR = 32;
constexpr int kGemmRows = 128;   // MMA M (lnM rows per CTA)
constexpr int kKChunk = 32;      // lam_t nodes per pipeline stage
constexpr int kMaxCols = 512;    // TMEM columns = n_lam_bins * n_z (padded)

struct GridDev {
  int n_m, n_z, n_t, n_o, n_zo, nI, nJ, nB;
  int n_m_pad;     // rows padded to kGemmRows
  int n_t_pad;     // lam_t nodes padded to kKChunk
  int n_cols;      // nI * n_z
  int n_cols_pad;  // padded to 16
  int uk_zindep;   // P(lam_o | lam_t) has no z dependence: K_i(t, q) = K_i(t)
  int nIc;         // richness bins per tensor-core CTA (nIc * n_z <= 256 columns)
  int n_bg;        // bin groups = ceil(nI / nIc)
  int ncp_c;       // TMEM columns per CTA: nIc * n_z padded to 16
  double lnm_lo, lnm_hi, zt_lo, zt_hi, ll_lo, ll_hi, sz0;
  const double* xm;   // [n_m]  lnM nodes
  const double* wm;
  const double* xz;   // [n_z]  z_t nodes
  const double* wz;
  const double* xl;   // [n_t]  ln lam_t nodes
  const double* wl;
  const double* Ki;   // [nI][n_z][n_t] FP64
  const float* UK;    // [nI][n_z][n_t_pad] = wl_t K_i(t, q) in FP32
  const double* Kj;   // [nJ][n_z]
  const double* omz;  // [n_z] survey area Omega(z_q)
  // per-point scratch layout (offsets in elements of the scratch block)
  size_t s64_stride;  // doubles per point in the FP64 scratch
  size_t o_scal, o_kx, o_kt, o_kf, o_qy, o_qu;  // A0/B0, HMF cells and weights
  size_t o_cz, o_czs, o_alpha, o_beta, o_P0, o_V;
  size_t s32_stride;  // floats per point in the FP32 scratch
  size_t f_a, f_b, f_delta, f_scal, f_Yt, f_CN, f_CG;
};

struct PointDev {  // mirrors y3b_point
  double om, ol, ok, h0, onu, hmf_s, hmf_q;
  double A, B, C, sigma, Mpiv;
  int grid;
  int reserved;
};

struct TableLayout {
  int n_hm, n_hz, n_dist, n_sci;
  size_t stride;   // doubles per point
  size_t off[7];   // m_h, hmf_z, dndlnmh, dist_z, dist_da, sci_z, sci_val
};

struct ShearDev {
  int n_R;
  double R[kMaxR];
  double f_mis, tau_mis;
  double lob[kMaxLamBins];
  double c0, c_slope, c_pivot;
};

struct MixedLaunch {
  const GridDev* grids;     // device array
  const PointDev* pts;      // device array
  int grid_id;              // only points of this grid do work
  int n_points;
  const GridDev* g_host;    // host copy of grids[grid_id] (dims)
  float* s32;               // FP32 scratch base
  double* W;                // [n][nB][w_stride]
  double* Wg;
  int w_stride;             // max n_m over grids
  int* status;
  cudaStream_t stream;
  bool shear;               // also accumulate the Sigma_crit-weighted W^g
};

int launch_mixed_gemm(const MixedLaunch& L);

// Enqueues a copy of the engine's device status word (the result of the
// device-side checks of the evaluations enqueued before it on `s`) to `host`.
int engine_status_to_host(::y3b_engine* e, int* host, cudaStream_t s);

struct EngineInfo {
  int n_grids, n_bins, n_R, with_shear, max_points;
  size_t stride;        // doubles per point's table block
  size_t device_bytes;  // what the engine holds
};
void engine_info(const ::y3b_engine* e, EngineInfo* out);

// Host-side checks of points (grid index, positive sigma, Mpiv, h0 and
// omega_M - omega_nu); sets the error message.  *mask gets the grids used.
int engine_check_points(const ::y3b_engine* e, int n, const y3b_point* pts, int* mask);

// Host-side copy of the device domain check: every z_t node of a point's grid
// must lie inside its distances/z table (host tables).  Y3B_ERR_DOMAIN if not.
int engine_check_tables(const ::y3b_engine* e, int n, const y3b_point* pts, const double* tables);
size_t mixed_gemm_smem_bytes(int ncp, int n_z, int n_t_pad, int nJ, int nIc);

}  // namespace y3b
