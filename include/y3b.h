/*
 * y3b.h -- C ABI of the B200 engine for the DES-Y3 cluster-observable
 * integrals (number counts N(lambda_obs bin, z_obs bin) and the stacked
 * miscentred-NFW DeltaSigma one-halo profile in the same bins).
 *
 * Plain C: POD structs, raw pointers and sizes, integer status codes.  No
 * function throws; every failure returns a non-zero y3b_status and leaves a
 * message for y3b_last_error().  All compute runs on the current CUDA device
 * (or the one chosen with y3b_device_init); there is no CPU fallback -- on a
 * machine without a usable sm_100 device every compute entry point returns
 * Y3B_ERR_CUDA.
 *
 * Reference interfaces replaced (paths inside estevesjh/y3_cluster_cpp):
 *   y3b_sel_function        src/modules/sel_function/sel_function.py:555-615
 *                           (execute: S_stack producer)
 *   y3b_selgl_*             src/models/n_operator_sel_gl_t.hh:75-361
 *                           (SelGLCore, NumCountsSelGL, Shear1hMisSelGL)
 *   y3b_sigma_crit_inv      src/modules/average_sigma_crit_inv/
 *                           average_sigma_crit_inv.py:32-61
 *   y3b_nfw_mis             src/models/nfw_dsigma_mis.hh:95-114 and
 *                           src/models/nfw_sigma_mis.hh:53-66
 *   y3b_prj_*               src/models/sigma_prj_frozen_t.hh:34-512
 *                           (ShearPrjFrozenPhysics, module
 *                           src/modules/sigma_prj_cpu/ShearPrjFrozenPhysics.cc)
 *   y3b_bsel_*              src/models/p_operator_t.hh:76-718
 *                           (P_operator: the selection-bias operators P1,
 *                           I1, J; module src/modules/b_sel_marg_cpu/
 *                           BSelMargIntegrand.cc)
 *   y3b_engine_*            the fused fast_mass form of the same integrals
 *                           (NumCountsFastMass / Shear1hFastMass, documented
 *                           as identical to the two modules above), with the
 *                           lambda_t / lambda_o / z_o integrals of
 *                           sel_function.py done on fixed quadrature nodes.
 * The CosmoSIS module ABI (setup/execute/cleanup of
 * src/utils/module_macros.hh:76-99) is declared in y3b_cosmosis.h.
 */
#ifndef Y3B_H
#define Y3B_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define Y3B_VERSION 1

typedef enum {
  Y3B_OK = 0,
  Y3B_ERR_INVALID = 1,     /* bad argument or shape */
  Y3B_ERR_DOMAIN = 2,      /* query outside an unclamped table (the reference throws std::domain_error) */
  Y3B_ERR_CUDA = 3,        /* CUDA runtime failure or no usable device */
  Y3B_ERR_NOMEM = 4,       /* device allocation failed */
  Y3B_ERR_TIMEOUT = 5,     /* a bounded device-side wait ran out */
  Y3B_ERR_BUDGET = 6,      /* request exceeds the configured HBM budget */
  Y3B_ERR_UNSUPPORTED = 7, /* shape the kernel does not support */
  Y3B_ERR_RANGE = 8,       /* mixed form: a point's Gaussian factors would leave the FP32
                              exponent range (sigma_int too small for the factorisation);
                              evaluate that point in Y3B_FP64 */
  Y3B_ERR_CANCELLED = 9    /* the request was cancelled (y3b_server_cancel) */
} y3b_status;

/* Message of the last failure on the calling thread ("" if none). */
const char* y3b_last_error(void);
int y3b_version(void);
/* Select the CUDA device for the calling thread; checks it is sm_100. */
int y3b_device_init(int device);
/* Number of kernel launches issued by this library since load (all threads). */
unsigned long long y3b_launch_count(void);

/* ---------------------------------------------------------------------- */
/* Shared POD types                                                        */

typedef struct {
  double om, ol, ok, h0, onu, hmf_s, hmf_q; /* cosmological_parameters/{omega_M,
                                               omega_lambda, omega_k, h0, omega_nu},
                                               cluster_abundance/{hmf_s, hmf_q} */
} y3b_cosmo;

/* Per-sample tables, as the DataBlock holds them (all FP64, host or device
 * memory depending on the call). */
typedef struct {
  int n_hm;  const double* hmf_m_h;   /* mass_function/m_h             */
  int n_hz;  const double* hmf_z;     /* mass_function/z               */
  const double* dndlnmh;              /* mass_function/dndlnmh [n_hz][n_hm] */
  int n_dist; const double* dist_z;   /* distances/z                   */
  const double* dist_da;              /* distances/d_a [Mpc]           */
  int n_sci; const double* sci_z;     /* average_sigma_crit_inv/zlense (0 if unused) */
  const double* sci_val;              /* average_sigma_crit_inv/sci_average */
} y3b_tables;

/* P(lambda_obs | lambda_true, z) coefficient table: 8 rows of n values in
 * the order a_tau, b_tau, a_mu, b_mu, a_sig, b_sig, a_fprj, b_fprj
 * (plob_ltr_params section; y3_buzzard/prj_params.py:58-61). */
typedef struct {
  int n;
  const double* z;
  const double* coef;
} y3b_plob;

typedef enum { Y3B_MOR_HOD = 0, Y3B_MOR_LOGNORMAL = 1 } y3b_mor_kind;

/* HOD: p = {log10_Mmin, log10_M1, alpha, epsilon, sigma_lambda, z_pivot}
 * (cluster_mor section, sel_function.py:493-513).
 * LOGNORMAL: p = {A, B, C, sigma, Mpiv, lam_lo, lam_hi}: ln lambda ~
 * N(A + B ln(M/Mpiv) + C ln(1+z), sigma) truncated to [lam_lo, lam_hi]. */
typedef struct {
  int kind;
  double p[8];
} y3b_mor;

/* ---------------------------------------------------------------------- */
/* sel_function: S_ij(lnM, z) on a shared linear grid (sel_function.py).   */

typedef struct {
  int n_bins;
  const double* lam_min; const double* lam_max;   /* per bin */
  const double* zob_min; const double* zob_max;
  const double* sigma_z;
  double zt_low, zt_high, lnm_low, lnm_high;
  int n_lnm, n_z, n_q;                            /* n_lnm, n_z_shared, N_q */
} y3b_selfunc_config;

/* Host buffers: lnm_out[n_lnm], z_out[n_z], S_out[n_bins][n_z][n_lnm].
 * Replaces sel_function.py:555-615. */
int y3b_sel_function(const y3b_selfunc_config* cfg, const y3b_mor* mor,
                     const y3b_plob* plob, double* lnm_out, double* z_out,
                     double* S_out);

/* The same S_stack producer for callers that cannot allocate device memory
 * (no counterpart in the reference).  Such callers -- a sampler that has
 * reserved all of its device memory up front in its own pool, or a host
 * whose device allocations belong to another runtime's allocator and where
 * a cudaMalloc would synchronise the device mid-run -- pass device buffers
 * lnm_dev[n_lnm], z_dev[n_z], S_dev[n_bins][n_z][n_lnm]; the configuration
 * and the projection table stay in host memory.  Scratch (GL nodes, edge and
 * bin tables, the copied configuration) lives in one fixed file-scope device
 * array of 43 KiB, so the call allocates nothing and rejects N_q > 1024,
 * n_bins > 256 or more than 256 projection-table nodes with Y3B_ERR_INVALID.
 * The array is shared by every call on a device and keeps the last call's
 * contents: calls that overlap on the GPU (other streams or threads) race on
 * it and must be serialised by the caller.  The first call on each device
 * (and the first after that device's context was reset) looks the array's
 * device address up (cudaGetSymbolAddress); make that first call before any
 * stream capture.  Asynchronous on `stream` (a cudaStream_t, NULL = the
 * legacy default stream): the per-bin arrays of cfg and the projection table
 * are copied from the caller's memory on that stream, so when they are in
 * pinned memory they must stay valid until the stream has finished the
 * call's work; synchronise before reading the outputs. */
int y3b_sel_function_noalloc(const y3b_selfunc_config* cfg, const y3b_mor* mor,
                             const y3b_plob* plob, double* lnm_dev, double* z_dev,
                             double* S_dev, void* stream);

/* ---------------------------------------------------------------------- */
/* SelGLCore: fixed-GL z-contracted mass weights and the two evaluators.  */

typedef struct {
  int n_lnm, n_z;                       /* defaults 96, 64 */
  double zt_low, zt_high, lnm_low, lnm_high;
} y3b_selgl_config;

typedef struct {
  int n_bins;
  int n_lnm; const double* lnm;         /* sel_function/lnM */
  int n_z;   const double* z;           /* sel_function/z   */
  const double* S_stack;                /* [n_bins][n_z][n_lnm] */
} y3b_selection;

/* Centred DeltaSigma table haloModel/{r_sigma, lnM, dSigma_nfw[n_lnm][n_r]}
 * and the miscentring settings of Shear1hMisSelGL. */
typedef struct {
  int n_r;   const double* r_sigma;
  int n_lnm; const double* lnM;
  const double* dsigma;
  double f_mis, tau_mis;                /* miscentering/{f_mis, tau_mis}    */
  int n_lob; const double* lob_centers; /* module option lob_centers        */
  double conc;                          /* NFW_DSIGMA_MIS concentration (4) */
  int n_theta, n_s; double s_max;       /* miscentring quadrature (64, 128, 20) */
  int use_idea2; double stencil_h;      /* method = idea2 / stencil_h       */
} y3b_shear_table;

typedef struct y3b_selgl y3b_selgl;

/* setup(): GL nodes for the configured box.  n_z/GL on device. */
int y3b_selgl_create(const y3b_selgl_config* cfg, y3b_selgl** out);
/* set_sample(): build W_b(lnM_k) (include_sci adds Sigma_crit^-1(z)).
 * Returns Y3B_ERR_DOMAIN if a GL z node lies outside distances/z. */
int y3b_selgl_build(y3b_selgl* h, const y3b_cosmo* c, const y3b_tables* t,
                    const y3b_selection* sel, int include_sci);
/* NumCountsSelGL::evaluate over a wall of bin indices -> vals[n]. */
int y3b_selgl_counts(y3b_selgl* h, int n, const int* bin_index, double* vals);
/* Shear1hMisSelGL::evaluate over (bin_index[i], r[i]) pairs -> vals[n].
 * NFW_DSIGMA_MIS follows the module's construction (n_operator_sel_gl_t.hh:
 * 248,264): r_s from rho_c = 2.77533742639e11, amplitude
 * 2 r_s delta_c rho_c Omega_M 1e-12.  Its unit profile comes from the table
 * set with y3b_selgl_set_mis_table, else from the direct quadrature
 * (n_theta, n_s, s_max of the y3b_shear_table). */
int y3b_selgl_shear(y3b_selgl* h, const y3b_shear_table* st, int n,
                    const int* bin_index, const double* r, double* vals);
/* The miscentred-profile table NFW_DSIGMA_MIS reads
 * (src/models/nfw_dsigma_mis.hh:62-72, files nfw_off_center/
 * table_1000_1e-03_5e+03_{gamma_logx, gamma_logxmis,
 * log_deltasigma_gamma}.txt): axes ln x[n_lx], ln x_mis[n_lxm] (increasing)
 * and log_tab[n_lxm][n_lx] (x fastest), read by clamped bilinear
 * interpolation at (ln R/r_s, ln R_mis/r_s).  Host buffers, copied.
 * n_lx = 0 returns the handle to the direct quadrature. */
int y3b_selgl_set_mis_table(y3b_selgl* h, int n_lx, const double* logx,
                            int n_lxm, const double* logxmis,
                            const double* log_tab);
/* Copy out W [n_bins][n_lnm], norm, lnm_eff, mu2 and the GL nodes/weights. */
int y3b_selgl_weights(y3b_selgl* h, double* W, double* norm, double* lnm_eff,
                      double* mu2, double* lnm_x, double* lnm_w);
int y3b_selgl_n_bins(const y3b_selgl* h);
void y3b_selgl_destroy(y3b_selgl* h);

/* ---------------------------------------------------------------------- */
/* Frozen-physics projection shear <DeltaSigma_prj>(R | lambda bin, z_obs) */
/* (ShearPrjFrozenPhysics, src/models/sigma_prj_frozen_t.hh:34-512).       */

/* Module options (the constructor's keys and defaults). */
typedef struct {
  int n_lnm, n_per_seg, n_zring, n_zouter;  /* 24, 10, 20, 20 */
  double zt_low, zt_high, lnm_low, lnm_high;
  double R_max_cMpch;                       /* 30 */
  int include_omega_z;                      /* 1 */
  int n_lob; const double* lob_centers;     /* NULL: {25, 37.5, 52.5, 130} */
  int n_gp;                                 /* grid points (wall of numbers): */
  const int* lambda_bin;                    /*   richness bin                 */
  const double *zo_low, *zo_high;           /*   z_obs bin edges              */
  const double* radii;                      /*   R [Mpc/h]                    */
} y3b_prj_config;

/* One sample: cosmology, the counts' tables (HMF, distances/{z, d_a},
 * optional average_sigma_crit_inv) and distances/d_c [Mpc] on distances/z,
 * haloModel/{lnM, z, bias[n_hz][n_hl]}, xi_nl/{r, z, xi_nl[n_xz][n_xr]},
 * b_sel_marginalised/{lob, zob, b_small, b_large [n_bzob][n_blob]}. */
typedef struct {
  y3b_cosmo cosmo;
  y3b_tables t;
  const double* dist_dc;
  int n_hl, n_hz; const double *halo_lnM, *halo_z, *bias;
  int n_xr, n_xz; const double *xi_r, *xi_z, *xi_nl;
  int n_blob, n_bzob; const double *bsel_lob, *bsel_zob, *b_small, *b_large;
} y3b_prj_sample;

typedef struct y3b_prj y3b_prj;
/* setup(): the grid points and their (richness bin, z_obs) slices. */
int y3b_prj_create(const y3b_prj_config* cfg, y3b_prj** out);
/* The single-kernel miscentring table NFW_DSIGMA_MIS reads
 * (nfw_off_center/table_1000_1e-03_5e+03_{single_logx, single_logxmis,
 * log_deltasigma_single}.txt), as y3b_selgl_set_mis_table; n_lx = 0
 * returns to the direct quadrature of the fixed-offset kernel. */
int y3b_prj_set_mis_table(y3b_prj* h, int n_lx, const double* logx, int n_lxm,
                          const double* logxmis, const double* log_tab);
/* set_sample() + evaluate() of every grid point -> out[n_gp][9]: DeltaSigma
 * total, random, clustered; the tangential shear (times Sigma_crit^-1(z_obs),
 * 0 without that table) total, random, clustered; and the shear_prj alias of
 * the shear triple.  Host buffers; Y3B_ERR_DOMAIN if a line-of-sight z node
 * lies outside distances/z. */
int y3b_prj_eval(y3b_prj* h, const y3b_prj_sample* s, double* out);
void y3b_prj_destroy(y3b_prj* h);

/* ---------------------------------------------------------------------- */
/* Selection-bias operators P1, I1, J on the (zo_low, zo_high, lambda_bin) */
/* wall grid (P_operator, module label b_sel_marg,                          */
/* src/models/p_operator_t.hh:76-718; outputs b_sel_marg_P1 / _I1 / _J).   */

/* Module options (p_operator_t.hh:95-110): node counts (defaults n_lt 60,
 * n_zring 20, n_zouter 30, n_lnm 24, n_theta 10, n_zt_ref 80), the reference
 * z grid [zt_ref_low, zt_ref_high] (0.05, 0.90) and the mass range (required).
 * max_samples bounds one device batch (the MOR table takes
 * 4 n_zt_ref n_lnm n_lt doubles per sample); eval splits larger calls. */
typedef struct {
  int n_lt, n_zring, n_zouter, n_lnm, n_theta, n_zt_ref;
  double zt_ref_low, zt_ref_high, lnm_low, lnm_high;
  int n_gp;                              /* grid points (wall of numbers): */
  const double *zo_low, *zo_high;        /*   z_obs bin edges              */
  const int* lambda_bin;                 /*   richness bin 0..3            */
  int max_samples;
} y3b_bsel_config;

/* One sample: cosmology and HMF / distances/{z, d_a} tables (the sci arrays
 * are not read), distances/d_c [Mpc] on distances/z, haloModel/{lnM, z,
 * bias [n_hz][n_hl]}, xi_nl/{r, z, xi_nl [n_xz][n_xr]} (r log-spaced and z
 * evenly spaced, as the reference's lookup assumes) and the cluster_mor HOD
 * parameters {log10_Mmin, log10_M1, alpha, epsilon, sigma_lambda, z_pivot}
 * (z_pivot 0.45 when the section has none). */
typedef struct {
  y3b_cosmo cosmo;
  y3b_tables t;
  const double* dist_dc;
  int n_hl, n_hz; const double *halo_lnM, *halo_z, *bias;
  int n_xr, n_xz; const double *xi_r, *xi_z, *xi_nl;
  double hod[6];
} y3b_bsel_sample;

typedef struct y3b_bsel y3b_bsel;
/* setup(): GL nodes of lnM and of each richness bin's lambda_true range, the
 * reference z grid, and each grid point's photo-z support (which depends on
 * z_obs only). */
int y3b_bsel_create(const y3b_bsel_config* cfg, y3b_bsel** out);
/* set_sample() + evaluate() of every grid point for n_samples samples (all
 * with the shapes of samples[0]) -> out[n_samples][n_gp][3] = (P1, I1, J).
 * Host buffers; FP64 throughout.  Y3B_ERR_DOMAIN if the reference z grid
 * leaves distances/z (the reference's Interp1D throws there). */
int y3b_bsel_eval(y3b_bsel* h, int n_samples, const y3b_bsel_sample* samples, double* out);
/* Device time of the last y3b_bsel_eval's kernels (CUDA events around each
 * chunk's two kernels, summed; the copies and host packing excluded). */
int y3b_bsel_kernel_ms(const y3b_bsel* h, double* ms);
void y3b_bsel_destroy(y3b_bsel* h);

/* ---------------------------------------------------------------------- */
/* <Sigma_crit^-1>(z_l) (average_sigma_crit_inv.py:40-58), host buffers.   */
int y3b_sigma_crit_inv(int n_zl, const double* zl, int n_zs, const double* zs,
                       const double* pz, double delta_z, double h0,
                       int n_dist, const double* dist_z, const double* dist_da,
                       double* out);

/* Miscentred NFW profiles at n points: out[i] = 2 r_s delta_c rho 1e-12 *
 * <profile>(r[i]/r_s, rmis[i]/r_s), r_s from lnM[i], concentration conc and
 * rho (NFW_DSIGMA_MIS(c, rho) / NFW_SIGMA_MIS(c, rho) operator()).
 * which = 0: DeltaSigma_mis, 1: Sigma_mis (both for offsets drawn from the
 * gamma kernel), 2: DeltaSigma for a single offset rmis (the "single" kernel:
 * mean tangential shear on the circle of radius r around the offset centre,
 * n_theta GL nodes on [0, pi]; n_s and s_max are checked but unused).  Host
 * buffers. */
int y3b_nfw_mis(int which, int n, const double* r, const double* rmis,
                const double* lnM, double conc, double rho, int n_theta,
                int n_s, double s_max, double* out);

/* ---------------------------------------------------------------------- */
/* Engine: many parameter points (walkers) on fixed nested Gauss-Legendre */
/* nodes; FP64 direct form or the mixed form (FP32 integrands, split-BF16  */
/* tensor-core contraction, FP64 final sums).                              */

typedef struct {
  int n_m, n_z, n_t, n_o, n_zo;         /* lnM, z_t, ln lam_t, lam_o/bin, z_o/bin */
  double lnm_lo, lnm_hi, zt_lo, zt_hi;  /* integration box */
  double lam_t_lo, lam_t_hi;            /* lam_t domain of the MOR */
  int n_lam_bins, n_z_bins;             /* <= 8, <= 8 */
  double lam_edges[9];
  double zob_edges[9];
  double sz0;                           /* sigma_z(z_t, j) = sz0 (1 + z_t) + sz_bin[j] */
  double sz_bin[8];                     /* per z_obs bin; sz0 = 0 and sz_bin = the bins'
                                           sigma_z is sel_function.py's photo-z model
                                           (_K_j, sel_function.py:260-262) */
} y3b_grid;

typedef struct {
  int n_R;
  double R[32];                         /* projected radii [Mpc/h] */
  double f_mis, tau_mis;
  double lob_centers[8];                /* per richness bin */
  double c0, c_slope, c_pivot;          /* c(M) = c0 (M / c_pivot)^c_slope */
  int n_theta, n_s;
  double s_max;
} y3b_shear_opts;

typedef struct {
  int n_hm, n_hz, n_dist, n_sci;        /* table shapes shared by all points */
  y3b_plob plob;                        /* P(lam_o | lam_t, z) coefficients */
  int max_points;                       /* capacity of one eval call */
  size_t hbm_budget;                    /* bytes of device memory the engine may hold (0: 150 GB) */
  int with_shear;
  y3b_shear_opts shear;
  int hmf_fp32;                         /* 1: the packed tables carry mass_function/dndlnmh
                                           in FP32 (the mixed form rounds it to FP32 on the
                                           device anyway, so its results do not change);
                                           such an engine evaluates the mixed form only */
} y3b_engine_config;

typedef struct {
  y3b_cosmo cosmo;
  double A, B, C, sigma, Mpiv;          /* lognormal MOR */
  int grid;                             /* index into the engine's grids */
  int reserved;
} y3b_point;

typedef enum { Y3B_FP64 = 0, Y3B_MIXED = 1 } y3b_precision;

/* An engine (like a server) is used by one host thread at a time; engines
 * are independent, one per device or per stream if wanted. */
typedef struct y3b_engine y3b_engine;

int y3b_engine_create(const y3b_grid* grids, int n_grids,
                      const y3b_engine_config* cfg, y3b_engine** out);
void y3b_engine_destroy(y3b_engine* e);
/* Doubles per point in the packed table buffer (each section 16-byte
 * aligned): hmf_m_h[n_hm] | hmf_z[n_hz] | dndlnmh[n_hz*n_hm] | dist_z[n_dist]
 * | dist_da[n_dist] | sci_z[n_sci] | sci_val[n_sci]; with hmf_fp32 the
 * dndlnmh section holds n_hz*n_hm floats (half as many doubles). */
size_t y3b_engine_table_stride(const y3b_engine* e);
/* Offsets (in doubles) of the seven sections inside one point's block. */
int y3b_engine_table_offsets(const y3b_engine* e, size_t* off7);
int y3b_engine_n_bins(const y3b_engine* e);
/* Device bytes the engine holds (tables, scratch, outputs). */
size_t y3b_engine_device_bytes(const y3b_engine* e);

/* Host-buffer evaluation: copies points and tables in, evaluates, copies
 * counts [n][n_bins] (and shear [n][n_bins][n_R] if enabled) out.
 * Synchronous on the engine's stream. */
int y3b_engine_eval(y3b_engine* e, int precision, int n,
                    const y3b_point* pts, const double* tables,
                    double* counts, double* shear);
/* Device-buffer evaluation, asynchronous on `stream` (a cudaStream_t; NULL
 * = the engine's stream).  All pointers are device pointers; counts/shear
 * as above.  Returns after enqueueing; the status of device-side checks is
 * read with y3b_engine_sync. */
int y3b_engine_eval_device(y3b_engine* e, int precision, int n,
                           const y3b_point* pts_dev, const double* tables_dev,
                           double* counts_dev, double* shear_dev, void* stream);
/* As y3b_engine_eval_device, but point i reads its table block from a
 * resident pool: pool_dev + slot_dev[i] * y3b_engine_table_stride(e)
 * doubles (device pointers; the pool 16-byte aligned).  Lets tables stay on
 * the device across evaluations (the request server keeps them there).
 * Points are not checked on the device: their grid must be valid. */
int y3b_engine_eval_pooled(y3b_engine* e, int precision, int n,
                           const y3b_point* pts_dev, const double* pool_dev,
                           const int* slot_dev, double* counts_dev,
                           double* shear_dev, void* stream);
/* CUDA graphs (mode 1, the default): an evaluation whose arguments (precision,
 * n, the device buffers) repeat a recent call is captured once into a CUDA
 * graph and replayed from then on, one host launch for the whole sequence of
 * kernels.  Stage timing (y3b_engine_profile) bypasses the graphs.  mode 0
 * turns them off and frees the captured graphs. */
int y3b_engine_set_graphs(y3b_engine* e, int mode);
/* Autotuner: times the tensor-core contraction on the caller's batch (device
 * buffers as for y3b_engine_eval_device, mixed form) for ring depths 2..8
 * (what shared memory allows) and, grid by grid, 1/2/4/8 richness bins per
 * tile (at most 256 accumulator columns), and keeps the fastest for the
 * engine's life.  Results of different settings differ only by FP32
 * rounding; once tuned, an engine's results are fixed.  best_ms (optional):
 * the contraction time of the chosen setting.  Synchronous. */
int y3b_engine_autotune(y3b_engine* e, int n, const y3b_point* pts_dev,
                        const double* tables_dev, double* counts_dev, double* best_ms);
/* The current setting: ring depth and bins per tile of each grid (cap >= grids). */
int y3b_engine_tuning(const y3b_engine* e, int* stages, int* bins_per_tile, int cap);
/* lam_t stages of the last mixed-form evaluation call (all its chunks): the
 * stages its tiles issued (each tile skips the stages where the
 * domain-renormalised MOR density of all its (lnM, z) pairs is below 4e-6 of
 * its peak) and the stages of the full lam_t range.  Reads device memory:
 * call after that evaluation completed. */
int y3b_engine_stage_count(const y3b_engine* e, long long* executed, long long* dense);
/* Wait for the engine's work on `stream` and report device-side errors. */
int y3b_engine_sync(y3b_engine* e, void* stream);
/* Optional: the mass weights W_b(lnM_k) of the last eval ([n][n_bins][n_m]
 * of each point's grid, padded to the largest n_m), host buffer. */
int y3b_engine_weights(y3b_engine* e, int n, double* W);

/* Gaussian likelihood of the counts + tangential shear data vector, as
 * y3_buzzard/likelihood_cp.py:94-200 computes it from numcountssel/vals,
 * shear1hmissel/vals and shear_prj/vals:
 *   shear theory[b][r] = (N_b > 0 ? S1h[b][r] / N_b : 0) + prj[b][r],
 *   logL = -0.5 (d_NC^T C^-1 d_NC + d_Sh^T C^-1 d_Sh), d = data - theory, or
 *   ln data - ln max(theory, 1e-300) in log space (the inverse covariance then
 *   becomes invcov * data data^T, as the reference's setup() does).
 * Inverse covariances are diagonal ([n]) or dense ([n][n], *_dense = 1); the
 * shear vector is bin slow, R fast; n_R = 0 uses the counts alone. */
typedef struct {
  int log_space;
  int n_bins, n_R;
  const double* data_nc;  const double* invcov_nc; int nc_dense;
  const double* data_sh;  const double* invcov_sh; int sh_dense;
  const double* shear_prj;              /* [n_bins][n_R] projection shear, or NULL */
} y3b_likelihood;
/* Fuses the likelihood into every later evaluation: the block that sums a
 * point's counts and shear also writes its logL (n_bins must match every
 * grid; a shear data vector needs the engine's shear and radii).  Copies the
 * vectors; NULL switches it off.  Drops captured CUDA graphs. */
int y3b_engine_set_likelihood(y3b_engine* e, const y3b_likelihood* L);
/* logL [n] of the last evaluation's points, copied on `stream` (NULL: the
 * engine's stream) and synchronised. */
int y3b_engine_loglike(y3b_engine* e, int n, double* logL, void* stream);
/* Host-buffer evaluation that returns only each point's logL [n]. */
int y3b_engine_eval_loglike(y3b_engine* e, int precision, int n,
                            const y3b_point* pts, const double* tables,
                            double* logL);
/* The same likelihood of one data vector (counts [n_bins], N_i-weighted
 * one-halo shear [n_bins][n_R]) on the device: the CosmoSIS likelihood
 * module's evaluation. */
int y3b_gaussian_loglike(const y3b_likelihood* L, const double* counts,
                         const double* shear_1h, double* logL);

/* Stage timing with CUDA events recorded on the launching stream around each
 * stage of every evaluation: 0 = per-point prep, 1 = lambda_t contraction
 * (tcgen05 GEMM or FP64 direct sum + z reduction), 2 = miscentred profile,
 * 3 = final sums.  enable = 1 starts (and zeroes) the accumulators, 0 stops.
 * y3b_engine_profile_read synchronises the engine's work and writes the
 * accumulated milliseconds ms[4] and the number of evaluations timed. */
int y3b_engine_profile(y3b_engine* e, int enable);
int y3b_engine_profile_read(y3b_engine* e, double* ms, int* n_evals);

/* Self-test of the bounded device wait: launches a kernel that waits on a
 * barrier nobody arrives at for ~`usec` microseconds and must come back
 * with Y3B_ERR_TIMEOUT (the context stays usable). */
int y3b_selftest_wait_timeout(int usec);

/* ---------------------------------------------------------------------- */
/* Request server: continuous batching of likelihood-evaluation requests   */
/* from a running sampler over one engine.  The reference evaluates one     */
/* point per CosmoSIS execute() call and has no counterpart.                */
/*                                                                          */
/* A request is n points with their own table blocks (host memory, packed   */
/* as for y3b_engine_eval).  Its tables are copied once into a device table */
/* pool when the pool has room (admission in arrival order, bounded by the  */
/* HBM budget); every launch evaluates up to max_batch points drawn from    */
/* all admitted requests, oldest first, splitting large requests across     */
/* launches, with up to max_inflight launches queued on the device.  The    */
/* server's worker thread owns the engine: do not evaluate on that engine   */
/* while the server exists.                                                 */

typedef struct {
  int pool_points;     /* table-pool slots, one per resident point (0: what the
                          budget allows, at most 65536) */
  size_t hbm_budget;   /* bytes for engine + launch buffers + pool (0: 150 GiB) */
  int max_batch;       /* points per launch (0: the engine's max_points) */
  int precision;       /* Y3B_MIXED or Y3B_FP64 */
  int with_shear;      /* also return DeltaSigma (engine created with_shear) */
  int max_inflight;    /* launches queued on the device at once, 1..4 (0: 2) */
} y3b_server_config;

typedef struct {
  long long requests_done, points_done, launches;
  int max_launch_points;
  int pool_points, pool_free_points;
  int waiting;         /* submitted, not yet admitted to the pool */
  int unscheduled;     /* admitted, with points not yet in a launch */
  long long requests_cancelled;
  size_t device_bytes;      /* HBM the server holds: engine, launch buffers, table pool */
  size_t pool_bytes_in_use; /* of which table-pool slots now holding a request's tables */
} y3b_server_stats;

typedef struct y3b_server y3b_server;

int y3b_server_create(y3b_engine* e, const y3b_server_config* cfg,
                      y3b_server** out);
/* Queues a request and returns at once with its ticket.  pts, tables,
 * counts ([n][n_bins]) and shear ([n][n_bins][n_R], with_shear only) are
 * host buffers that must stay valid until y3b_server_wait has returned for
 * the ticket; pinned tables upload fastest.  Points and their distance
 * tables are checked here (Y3B_ERR_INVALID / Y3B_ERR_DOMAIN); a request
 * larger than the whole pool gets Y3B_ERR_BUDGET. */
int y3b_server_submit(y3b_server* s, int n, const y3b_point* pts,
                      const double* tables, double* counts, double* shear,
                      long long* ticket);
/* Blocks until the request is complete (timeout_s < 0: no limit) and
 * returns its status; Y3B_ERR_TIMEOUT leaves it running and the ticket
 * valid.  latency_s (optional) = completion - submission.  One waiter per
 * ticket; a ticket is collected by the wait that returns its status. */
int y3b_server_wait(y3b_server* s, long long ticket, double timeout_s,
                    double* latency_s);
int y3b_server_stats_read(y3b_server* s, y3b_server_stats* out);
/* Cancels a request: a request still waiting for admission leaves the queue,
 * an admitted one gets no further points launched.  Points already on the
 * device finish; the request completes once they are back, and
 * y3b_server_wait then returns Y3B_ERR_CANCELLED (results not written).  Its
 * host buffers must stay valid until that wait has returned.  Returns Y3B_OK,
 * or Y3B_ERR_INVALID for an unknown ticket; a request that had already
 * completed keeps its own status. */
int y3b_server_cancel(y3b_server* s, long long ticket);
/* Finishes every submitted request, then frees the server (not the engine). */
void y3b_server_destroy(y3b_server* s);

/* The server's scheduling policy on its own (host only, no device): FIFO
 * admission of requests into contiguous runs of pool slots, launches of up
 * to max_batch points, slots released when a request completes.  For
 * capacity planning and tests of the policy. */
typedef struct y3b_planner y3b_planner;
int y3b_planner_create(int pool_points, int max_batch, y3b_planner** out);
void y3b_planner_destroy(y3b_planner* p);
int y3b_planner_submit(y3b_planner* p, long long id, int n_points);
/* Admits waiting requests in order while they fit: ids[i] gets slot0[i]. */
int y3b_planner_admit(y3b_planner* p, long long* ids, int* slot0, int cap,
                      int* n_out);
/* Next launch: up to cap chunks (request id, first point, count, slot). */
int y3b_planner_next_batch(y3b_planner* p, long long* ids, int* first,
                           int* count, int* slot, int cap, int* n_chunks,
                           int* n_points);
/* count points of request id came back; *finished = 1 when it completed. */
int y3b_planner_complete(y3b_planner* p, long long id, int count,
                         int* finished);
/* Stops scheduling request id: *finished = 1 when none of its points is out
 * (it left the planner, slots free), 0 when launched points must still
 * complete. */
int y3b_planner_cancel(y3b_planner* p, long long id, int* finished);
int y3b_planner_free_points(const y3b_planner* p);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif
