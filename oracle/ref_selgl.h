/*
 * ref_selgl.h -- C interface to the reference's own fixed-GL module classes
 * (SelGLCore, NumCountsSelGL, Shear1hMisSelGL of
 * src/models/n_operator_sel_gl_t.hh:75-361), compiled from the reference's
 * sources against the build shims in oracle/ref_shim/.
 *
 * TEST INFRASTRUCTURE ONLY.  The library (oracle/_ref/libselgl_ref.so) is
 * built by `make -C oracle ref` from the reference checkout and is never
 * committed.  It pins the oracle (oracle/y3o.c) and the CUDA path to the
 * reference's own arithmetic, and serves as the timed reference CPU path.
 * The product library never links or calls it.
 *
 * Arrays follow the DataBlock layouts the reference reads:
 *   mass_function/dndlnmh  [n_hz][n_hm]   (z slow, mass fast)
 *   sel_function/S_stack   [n_bins][n_sel_z][n_sel_lnm]
 *   haloModel/dSigma_nfw   [n_hl][n_rs]   (lnM slow, R fast)
 * Every call returns 0 on success; otherwise it copies the reference's
 * exception text into err and returns non-zero.
 */
#ifndef Y3_REF_SELGL_H
#define Y3_REF_SELGL_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int n_lnm, n_z;          /* <= 0: leave unset (reference defaults 96, 64) */
  double zt_low, zt_high, lnm_low, lnm_high;
} y3r_cfg;

typedef struct {
  double omega_m, omega_nu, omega_lambda, omega_k, h0, hmf_s, hmf_q;
  int n_hm, n_hz;
  const double *m_h, *hmf_z, *dndlnmh;
  int nd;
  const double *dist_z, *dist_da;
  int n_sci;                       /* 0: no average_sigma_crit_inv section */
  const double *sci_z, *sci_val;
  int n_bins, n_sel_z, n_sel_lnm;
  const double *sel_lnm, *sel_z, *S_stack;
  int n_rs, n_hl;                  /* 0: no haloModel section */
  const double *r_sigma, *halo_lnM, *dsigma_nfw;
  int has_f_mis, has_tau_mis;      /* miscentering/{f_mis,tau_mis} present */
  double f_mis, tau_mis;
} y3r_sample;

/* SelGLCore::build_weights -> W [n_bins][n_lnm], norm, lnm_eff, mu2 per bin,
 * and the GL mass nodes/weights (each may be NULL). */
int y3r_selgl_weights(const y3r_cfg* cfg, const y3r_sample* s, int include_sci,
                      double* W, double* norm, double* lnm_eff, double* mu2,
                      double* lnm_x, double* lnm_w, char* err, int errlen);

/* NumCountsSelGL: set_sample, then evaluate every bin -> vals[n_bins]. */
int y3r_numcounts(const y3r_cfg* cfg, const y3r_sample* s, double* vals,
                  char* err, int errlen);

/* Shear1hMisSelGL: set_sample, then evaluate the (bin, R) product, bin slow
 * and R fast -> vals[n_bins * n_R].  method: 0 exact, 1 idea2, -1 unset;
 * stencil_h < 0: unset; lob_centers NULL: unset.  data_root is the directory
 * holding data/nfw_off_center/ (exported as Y3_CLUSTER_CPP_DIR before the
 * module is constructed, as the reference expects). */
int y3r_shear1h(const y3r_cfg* cfg, int method, double stencil_h, int n_lob,
                const double* lob_centers, const char* data_root,
                const y3r_sample* s, int n_R, const double* R, double* vals,
                char* err, int errlen);

/* NFW_DSIGMA_MIS(c = 4, rho = RHOC, gamma kernel) with rho_mult = omega_m, at
 * n points (r, r_mis, lnM) -> out[n]. */
int y3r_nfw_dsigma_mis(const char* data_root, double omega_m, int n,
                       const double* r, const double* rmis, const double* lnM,
                       double* out, char* err, int errlen);

/* Inputs of the frozen-physics projection shear (ShearPrjFrozenPhysics,
 * src/models/sigma_prj_frozen_t.hh:34-512) beyond the y3r_sample tables. */
typedef struct {
  int n_lnm, n_per_seg, n_zring, n_zouter;  /* <= 0: leave unset (24, 10, 20, 20) */
  double zt_low, zt_high, lnm_low, lnm_high;
  double R_max_cMpch;                       /* < 0: unset (30) */
  int include_omega_z;                      /* < 0: unset (1) */
  int n_lob; const double* lob_centers;     /* NULL: unset */
  int n_gp;                                 /* grid points: lambda_bin, zo_low, zo_high, radii */
  const double *lambda_bin, *zo_low, *zo_high, *radii;
} y3r_prj_cfg;

typedef struct {
  int nd; const double* dist_dc;            /* distances/d_c on y3r_sample's distances/z */
  int n_hl, n_hz; const double *halo_lnM, *halo_z, *bias;      /* bias [n_hz][n_hl] */
  int n_xr, n_xz; const double *xi_r, *xi_z, *xi_nl;            /* xi_nl [n_xz][n_xr] */
  int n_blob, n_bzob; const double *bsel_lob, *bsel_zob, *b_small, *b_large;  /* [n_bzob * n_blob] */
} y3r_prj_sample;

/* ShearPrjFrozenPhysics: set_sample, then evaluate every grid point -> out
 * [n_gp][9] (dsigma total, rnd, cl; gt total, rnd, cl; the shear_prj alias of
 * the gt triple).  data_root holds data/nfw_off_center/ with the single-
 * kernel miscentring table files. */
int y3r_shear_prj_frozen(const y3r_prj_cfg* cfg, const char* data_root,
                         const y3r_sample* s, const y3r_prj_sample* ps, double* out,
                         char* err, int errlen);

/* Options of the selection-bias operators (P_operator, module label
 * b_sel_marg, src/models/p_operator_t.hh:76-110). */
typedef struct {
  int n_lt, n_zring, n_zouter, n_lnm, n_theta, n_zt_ref;  /* <= 0: unset (60, 20, 30, 24, 10, 80) */
  double zt_ref_low, zt_ref_high;                         /* < 0: unset (0.05, 0.90) */
  double lnm_low, lnm_high;
  int n_gp;                                               /* wall grid: zo_low, zo_high, lambda_bin */
  const double *zo_low, *zo_high, *lambda_bin;
} y3r_bsel_cfg;

/* cluster_mor HOD parameters (MOR_HOD_t(DataBlock&), mor_hod_t.hh:72-83);
 * has_z_pivot = 0 leaves z_pivot unset (0.45). */
typedef struct {
  double log10_Mmin, log10_M1, alpha, epsilon, sigma_lambda, z_pivot;
  int has_z_pivot;
} y3r_hod;

/* P_operator: set_sample, then evaluate every grid point -> out[n_gp][3]
 * (P1, I1, J).  Reads distances/d_c, haloModel/{lnM, z, bias} and
 * xi_nl/{r, z, xi_nl} from ps (its b_sel_marginalised arrays are unused). */
int y3r_bsel_marg(const y3r_bsel_cfg* cfg, const y3r_sample* s, const y3r_prj_sample* ps,
                  const y3r_hod* hod, double* out, char* err, int errlen);

#ifdef __cplusplus
}
#endif
#endif
