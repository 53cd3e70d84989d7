/*
 * y3o.h -- FP64 CPU oracle for the cluster-observable hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (estevesjh/y3_cluster_cpp), written to check the CUDA path.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it;
 * the product library never links or calls it.
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the reference project root).  Pins: tests/golden/ holds vectors produced by
 * the reference's own Python code (sel_function.py) and the reference's own
 * KAT files (dv/dz, gamma R_mis kernel, photo-z erf difference, NFW
 * miscentring values from cluster_toolkit); tests/test_oracle_golden.py checks
 * this oracle against all of them.
 */
#ifndef Y3O_H
#define Y3O_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- quadrature / interpolation (a1, a7 semantics) -------------------- */
void   y3o_gl_nodes(double a, double b, int n, double* x, double* w);
int    y3o_interp1d(const double* xs, const double* ys, int n, double x,
                    double* out);
double y3o_interp1d_clamp(const double* xs, const double* ys, int n, double x);
double y3o_interp2d(const double* xs, int nx, const double* ys, int ny,
                    const double* zs, double x, double y);
double y3o_interp2d_clamp(const double* xs, int nx, const double* ys, int ny,
                          const double* zs, double x, double y);

/* ---- cosmology (a2-a4) ------------------------------------------------- */
double y3o_ez(double om, double ol, double ok, double z);
int    y3o_dv_do_dz(const double* dz, const double* da, int nd, double om,
                    double ol, double ok, double h, double z, double* out);
double y3o_omega_z_des(double z);
double y3o_hmf(const double* lnm_axis, int nm, const double* z_axis, int nz,
               const double* dndlnmh, double s, double q, double lnM,
               double z);

/* ---- richness / photo-z kernels (a9, a10) ------------------------------ */
double y3o_phi(double x);
double y3o_erfcx(double t);
double y3o_emg_tail(double x, double mu, double sigma, double tau);
double y3o_cdf_lob(double x, double mu, double sigma, double tau, double fprj);
double y3o_pdf_lob(double x, double mu, double sigma, double tau, double fprj);
double y3o_kj(double z, double zmin, double zmax, double sigz);
void   y3o_plob_params(int n_plob, const double* plob_z,
                       const double* plob_coef, double ltr, double z,
                       double* mu, double* sigma, double* tau, double* fprj);

/* ---- MOR (a11) ---------------------------------------------------------- */
enum { Y3O_MOR_HOD = 0, Y3O_MOR_LOGNORMAL = 1 };
double y3o_p_hod(double ltr, double lnM, double z, const double* hod);

/* ---- sel_function S_stack producer (a8) -------------------------------- */
int y3o_sel_function(int n_bins, const double* lam_min, const double* lam_max,
                     const double* zob_min, const double* zob_max,
                     const double* sigma_z, double zt_low, double zt_high,
                     double lnm_low, double lnm_high, int n_lnm, int n_z,
                     int n_q, int mor_kind, const double* mor,
                     int n_plob, const double* plob_z, const double* plob_coef,
                     double* lnm_out, double* z_out, double* S_out);

/* ---- SelGLCore / NumCountsSel (a5, a6) ---------------------------------- */
typedef struct {
  double om, ol, ok, h0, onu, hmf_s, hmf_q;
} y3o_cosmo;

int y3o_selgl_weights(int n_lnm, int n_z, double zt_lo, double zt_hi,
                      double lnm_lo, double lnm_hi, const y3o_cosmo* c,
                      int n_hm, const double* hmf_m_h, int n_hz,
                      const double* hmf_z, const double* dndlnmh, int nd,
                      const double* dist_z, const double* dist_da, int n_sci,
                      const double* sci_z, const double* sci_val, int n_bins,
                      int n_sel_lnm, const double* sel_lnm, int n_sel_z,
                      const double* sel_z, const double* S_stack,
                      double* W_out, double* norm_out, double* lnm_eff_out,
                      double* mu2_out);

/* ---- NFW + miscentring (a14, a16) ---------------------------------------- */
double y3o_nfw_sigma_unit(double x);
double y3o_nfw_dsigma_unit(double x);
double y3o_nfw_norm(double lnM, double c, double rho);
double y3o_nfw_rs(double lnM, double c, double rho);
double y3o_dsigma_mis_unit(double x, double xmis, int n_theta, int n_s,
                           double s_max);
double y3o_sigma_mis_unit(double x, double xmis, int n_theta, int n_s,
                          double s_max);
double y3o_roffset(double x, double tau);
double y3o_dsigma_single_unit(double x, double xmis, int n_theta);
void   y3o_mis_s_nodes(double x, double xmis, int n_s, double s_max,
                       double* sn, double* wsn);

/* ---- Shear1hMisSel (a12, a15) -------------------------------------------- */
int y3o_shear1h_mis(int n_lnm, const double* lnm_x, const double* lnm_w,
                    int n_bins, const double* W_gamma, int n_R,
                    const double* R, double f_mis, double tau_mis,
                    int n_lob, const double* lob_centers, double omega_m,
                    double conc, int n_rs, const double* r_sigma, int n_ml,
                    const double* lnM_tab, const double* dsig_tab,
                    int n_theta, int n_s, double s_max, double* out);
/* The same with the miscentred profile read from the reference's table
 * (log unit profile on ln x fastest, ln x_mis slow), exact (0) or idea2 (1). */
double y3o_dsigma_mis_tab(double r, double rmis, double lnM, double conc,
                          double rhoc, double rho_mult, int n_lx,
                          const double* logx, int n_lxm, const double* logxmis,
                          const double* log_tab);
int y3o_shear1h_mis_tab(int n_lnm, const double* lnm_x, const double* lnm_w,
                        int n_bins, const double* W_gamma, const double* norm,
                        const double* lnm_eff, const double* mu2, int method,
                        double stencil_h, int n_R, const double* R,
                        double f_mis, double tau_mis, int n_lob,
                        const double* lob_centers, double omega_m, double conc,
                        int n_rs, const double* r_sigma, int n_ml,
                        const double* lnM_tab, const double* dsig_tab,
                        int n_lx, const double* logx, int n_lxm,
                        const double* logxmis, const double* log_tab,
                        double* out);

/* ---- average Sigma_crit^-1 (a13) ----------------------------------------- */
int y3o_sigma_crit_inv(int n_zl, const double* zl, int n_zs, const double* zs,
                       const double* pz, double delta_z, double h0, int nd,
                       const double* dist_z, const double* dist_da,
                       double* out);

/* ---- Gaussian likelihood (y3_buzzard/likelihood_cp.py:132-200) ------------ */
double y3o_loglike(int n_bins, int n_R, const double* nc, const double* s1h,
                   const double* prj, int log_space, const double* data_nc,
                   const double* ic_nc, int nc_dense, const double* data_sh,
                   const double* ic_sh, int sh_dense);

/* ---- direct nested Gauss-Legendre quadrature (the configs' form) ---------- */
typedef struct {
  int n_m, n_z, n_t, n_o, n_zo;          /* nodes: lnM, z_t, ln lam_t, lam_o/bin, z_o/bin */
  double lnm_lo, lnm_hi, zt_lo, zt_hi;   /* integration box */
  double lam_t_lo, lam_t_hi;             /* lam_t domain (MOR normalisation) */
  int n_lam_bins, n_z_bins;
  const double* lam_edges;               /* n_lam_bins + 1 */
  const double* zob_edges;               /* n_z_bins + 1 */
  double sz0;                            /* sigma_z = sz0 (1 + z_t) + sz_bin[j] */
  const double* sz_bin;                  /* n_z_bins constants, or NULL */
} y3o_direct_grid;

typedef struct {
  double A, B, C, sigma, Mpiv;           /* lognormal MOR */
} y3o_lognormal;

typedef struct {
  int n_R;
  const double* R;                       /* projected radii [Mpc/h] */
  double f_mis, tau_mis;
  const double* lob_centers;             /* n_lam_bins */
  double c0, c_slope, c_pivot;           /* c(M) = c0 (M / c_pivot)^c_slope */
  int n_theta, n_s;
  double s_max;
  int n_sci;
  const double* sci_z;
  const double* sci_val;
} y3o_shear_opts;

int y3o_direct_eval(const y3o_direct_grid* g, int n_plob, const double* plob_z,
                    const double* plob_coef, const y3o_lognormal* mor,
                    const y3o_cosmo* c, int n_hm, const double* hmf_m_h,
                    int n_hz, const double* hmf_z, const double* dndlnmh,
                    int nd, const double* dist_z, const double* dist_da,
                    const y3o_shear_opts* shear, double* counts_out,
                    double* W_out, double* shear_out);

#ifdef __cplusplus
}
#endif
#endif
