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
// F(t, k) operand of one contraction stage (16 lam_t nodes x 128 lnM rows),
// bf16 hi then lo, each as two 2 KB planes of 8 nodes (16-byte rows): the
// layout of the stage in shared memory, so one bulk copy moves it.
constexpr int kFStageBytes = 8192;

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
  int tiles_pp;    // contraction tiles per point: (n_m_pad / kGemmRows) * n_bg
  int cost_rank;   // 0 = the grid with the most expensive tiles (scheduled first)
  // lam_t nodes where richness bin i's kernel K_i(t, q) exceeds 1e-12 of its
  // maximum over t, for some z_t node q: [kt_lo[i], kt_hi[i]]
  int kt_lo[kMaxLamBins], kt_hi[kMaxLamBins];
  double lnm_lo, lnm_hi, zt_lo, zt_hi, ll_lo, ll_hi, sz0;
  double sz_bin[8];   // sigma_z(z, j) = sz0 (1 + z) + sz_bin[j]
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
  size_t o_thdr, o_vv;  // mixed form: FP64 header and row scale v_k^2 c1 of yf_kernel
  size_t o_dt64;        // mixed form: FP64 log2 D table (deep tails)
  size_t s32_stride;  // floats per point in the FP32 scratch
  size_t f_a, f_b, f_delta, f_scal, f_Yt, f_CN, f_CG;
  // mixed form, prep -> yf_kernel: FP32 header, per-tile info, z rows,
  // log2 D table, per-tile row block
  size_t f_hdr, f_tinfo, f_q, f_dt32, f_rows;
  int nzp;  // n_z rounded up to 4
};

struct PointDev {  // mirrors y3b_point
  double om, ol, ok, h0, onu, hmf_s, hmf_q;
  double A, B, C, sigma, Mpiv;
  int grid;
  int reserved;
};

struct TableLayout {
  int n_hm, n_hz, n_dist, n_sci;
  int hmf_f32;     // dndlnmh section in FP32 (mixed form only)
  size_t stride;   // doubles per point
  size_t off[7];   // m_h, hmf_z, dndlnmh, dist_z, dist_da, sci_z, sci_val
};

struct ShearDev {
  int n_R;
  double R[kMaxR];
  double lnR[kMaxR];  // ln R, for the mixed form's table reads
  double f_mis, tau_mis;
  double lob[kMaxLamBins];
  double c0, c_slope, c_pivot;
};

// Shared-memory shape of the contraction, fixed per engine.
struct ContractShape {
  int nJ;       // z_obs bins (shared by all grids)
  int nz_max;   // largest n_z
  int ntp_max;  // largest n_t_pad
  int uk_max;   // floats of staged u_t K_i(t) per tile (0: read from global)
};

struct ContractLaunch {
  const GridDev* grids;     // device array
  int n_grids, grid_mask;   // points of grids outside the mask get no tiles
  const PointDev* pts;      // device array
  int n_points;
  int* order;               // [n_points] device scratch: points by grid cost
  int* tile_start;          // [n_points + 1] device scratch: tile offsets
  int* tile_list;           // [max_tiles] device scratch: (point << 8) | local tile
  const int* win_tile;      // [n][win_stride]: lam_t stage window of each local tile,
  int win_stride;           //   first | end << 16 (written by the prep kernel)
  long long max_tiles;      // upper bound of the launch's tiles (grid size)
  ContractShape shape;
  int stages;               // ring depth, 2..contract_stages(shape)
  int n_ctas;               // persistent CTAs (at most one per SM)
  const uint8_t* fbuf;      // F(t, k) stage blocks written by the prep kernel
  size_t f_stride;          // bytes per point
  float* s32;               // FP32 scratch base
  double* W;                // [n][nB][w_stride]
  double* Wg;
  int w_stride;             // max n_m over grids
  int* status;
  int* stage_count;         // [2] device: lam_t stages issued, stages of the full range
  cudaStream_t plan_stream; // the tile planner runs here, beside the prep kernel
  cudaStream_t stream;
  bool shear;               // also accumulate the Sigma_crit-weighted W^g
};

// The tile planner depends only on the points and their grids, so it runs on
// L.plan_stream while the prep kernel runs; the persistent contraction over
// the points of every grid runs on L.stream once both are done.
int contract_check(const ContractLaunch& L);  // ring depth and CTA count
int launch_plan(const ContractLaunch& L);
int launch_contract(const ContractLaunch& L);
size_t contract_smem_bytes(const ContractShape& c);  // (size_t)-1 if it does not fit
int contract_stages(const ContractShape& c);
// Sets the kernels' shared-memory limit once, outside any stream capture.
int contract_prepare(const ContractShape& c);

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

// A point's grid index is valid and selected.
__host__ __device__ inline bool
grid_in_mask(int mask, int g)
{
  return (unsigned)g < 31u && ((mask >> g) & 1);
}

}  // namespace y3b
