// ref_selgl.cc -- TEST INFRASTRUCTURE: drives the reference's own fixed-GL
// classes (src/models/n_operator_sel_gl_t.hh:75-361) from flat arrays.
//
// The reference headers are compiled unmodified, from the reference checkout,
// against the build shims in oracle/ref_shim/ (DataBlock subset, fmt, cubacpp
// type names, GSL linear/bilinear).  This file only fills a DataBlock with the
// sections and keys those classes read (n_operator_sel_gl_t.hh:77-89,
// 245-267; hmf_t.hh:37-45; dv_do_dz_t.hh:17-23; ez.hh:16-20;
// sel_function_t.hh:22-80; lensing_weights.hh:54-59,182-198) and calls
// set_sample / evaluate the way the CosmoSIS scalar-evaluator module does
// (CosmoSISScalarEvaluatorModule.hh:101-136): every grid point in order, bin
// slow, R fast.  y3r_bsel_marg drives P_operator (src/models/p_operator_t.hh)
// the same way over its (zo_low, zo_high, lambda_bin) wall grid.
#include "ref_selgl.h"

#include "models/n_operator_sel_gl_t.hh"
#include "models/sigma_prj_frozen_t.hh"
#include "models/p_operator_t.hh"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

namespace {

  using doubles = std::vector<double>;

  doubles
  vec(const double* p, int n)
  {
    return doubles(p, p + n);
  }

  void
  put_config(cosmosis::DataBlock& b, char const* label, const y3r_cfg* c)
  {
    if (c->n_lnm > 0) b.put_val(label, "n_lnm", c->n_lnm);
    if (c->n_z > 0) b.put_val(label, "n_z", c->n_z);
    b.put_val(label, "zt_low", c->zt_low);
    b.put_val(label, "zt_high", c->zt_high);
    b.put_val(label, "lnm_low", c->lnm_low);
    b.put_val(label, "lnm_high", c->lnm_high);
  }

  void
  put_sample(cosmosis::DataBlock& b, const y3r_sample* s)
  {
    char const* cp = "cosmological_parameters";
    b.put_val(cp, "omega_m", s->omega_m);
    b.put_val(cp, "omega_nu", s->omega_nu);
    b.put_val(cp, "omega_lambda", s->omega_lambda);
    b.put_val(cp, "omega_k", s->omega_k);
    b.put_val(cp, "h0", s->h0);
    b.put_val("cluster_abundance", "hmf_s", s->hmf_s);
    b.put_val("cluster_abundance", "hmf_q", s->hmf_q);
    b.put_val("mass_function", "m_h", vec(s->m_h, s->n_hm));
    b.put_val("mass_function", "z", vec(s->hmf_z, s->n_hz));
    b.put_val("mass_function", "dndlnmh",
              cosmosis::ndarray<double>(
                vec(s->dndlnmh, s->n_hm * s->n_hz),
                {static_cast<std::size_t>(s->n_hz),
                 static_cast<std::size_t>(s->n_hm)}));
    b.put_val("distances", "z", vec(s->dist_z, s->nd));
    b.put_val("distances", "d_a", vec(s->dist_da, s->nd));
    if (s->n_sci > 0) {
      b.put_val("average_sigma_crit_inv", "zlense", vec(s->sci_z, s->n_sci));
      b.put_val("average_sigma_crit_inv", "sci_average",
                vec(s->sci_val, s->n_sci));
    }
    b.put_val("sel_function", "lnM", vec(s->sel_lnm, s->n_sel_lnm));
    b.put_val("sel_function", "z", vec(s->sel_z, s->n_sel_z));
    b.put_val("sel_function", "S_stack",
              cosmosis::ndarray<double>(
                vec(s->S_stack, s->n_bins * s->n_sel_z * s->n_sel_lnm),
                {static_cast<std::size_t>(s->n_bins),
                 static_cast<std::size_t>(s->n_sel_z),
                 static_cast<std::size_t>(s->n_sel_lnm)}));
    if (s->n_rs > 0) {
      b.put_val("haloModel", "r_sigma", vec(s->r_sigma, s->n_rs));
      b.put_val("haloModel", "lnM", vec(s->halo_lnM, s->n_hl));
      b.put_val("haloModel", "dSigma_nfw",
                cosmosis::ndarray<double>(
                  vec(s->dsigma_nfw, s->n_rs * s->n_hl),
                  {static_cast<std::size_t>(s->n_hl),
                   static_cast<std::size_t>(s->n_rs)}));
    }
    if (s->has_f_mis) b.put_val("miscentering", "f_mis", s->f_mis);
    if (s->has_tau_mis) b.put_val("miscentering", "tau_mis", s->tau_mis);
  }

  int
  fail(char* err, int errlen, char const* what)
  {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", what);
    return 1;
  }

  void
  set_data_root(char const* root)
  {
    if (root) setenv("Y3_CLUSTER_CPP_DIR", root, 1);
  }

} // namespace

extern "C" {

int
y3r_selgl_weights(const y3r_cfg* cfg, const y3r_sample* s, int include_sci,
                  double* W, double* norm, double* lnm_eff, double* mu2,
                  double* lnm_x, double* lnm_w, char* err, int errlen)
{
  try {
    cosmosis::DataBlock c, b;
    put_config(c, "NumCountsSel", cfg);
    put_sample(b, s);
    y3_cluster::nosel_gl_detail::SelGLCore core(c, "NumCountsSel");
    core.build_weights(b, include_sci != 0);
    std::size_t const nb = core.n_bins();
    std::size_t const nm = core.lnm_x().size();
    for (std::size_t i = 0; i != nb; ++i) {
      if (W)
        for (std::size_t k = 0; k != nm; ++k) W[i * nm + k] = core.weights(i)[k];
      if (norm) norm[i] = core.norm(i);
      if (lnm_eff) lnm_eff[i] = core.lnm_eff(i);
      if (mu2) mu2[i] = core.mu2(i);
    }
    for (std::size_t k = 0; k != nm; ++k) {
      if (lnm_x) lnm_x[k] = core.lnm_x()[k];
      if (lnm_w) lnm_w[k] = core.lnm_w()[k];
    }
    return 0;
  }
  catch (std::exception const& e) {
    return fail(err, errlen, e.what());
  }
}

int
y3r_numcounts(const y3r_cfg* cfg, const y3r_sample* s, double* vals,
              char* err, int errlen)
{
  try {
    cosmosis::DataBlock c, b;
    put_config(c, y3_cluster::NumCountsSelGL::module_label(), cfg);
    put_sample(b, s);
    y3_cluster::NumCountsSelGL m(c);
    m.set_sample(b);
    for (int i = 0; i != s->n_bins; ++i) {
      y3_cluster::NumCountsSelGL::grid_point_t pt{static_cast<double>(i)};
      vals[i] = m.evaluate(pt)[0];
    }
    return 0;
  }
  catch (std::exception const& e) {
    return fail(err, errlen, e.what());
  }
}

int
y3r_shear1h(const y3r_cfg* cfg, int method, double stencil_h, int n_lob,
            const double* lob_centers, const char* data_root,
            const y3r_sample* s, int n_R, const double* R, double* vals,
            char* err, int errlen)
{
  try {
    set_data_root(data_root);
    char const* label = y3_cluster::Shear1hMisSelGL::module_label();
    cosmosis::DataBlock c, b;
    put_config(c, label, cfg);
    if (method >= 0)
      c.put_val(label, "method", std::string(method ? "idea2" : "exact"));
    if (stencil_h >= 0) c.put_val(label, "stencil_h", stencil_h);
    if (lob_centers) c.put_val(label, "lob_centers", vec(lob_centers, n_lob));
    put_sample(b, s);
    y3_cluster::Shear1hMisSelGL m(c);
    m.set_sample(b);
    for (int i = 0; i != s->n_bins; ++i)
      for (int r = 0; r != n_R; ++r) {
        y3_cluster::Shear1hMisSelGL::grid_point_t pt{static_cast<double>(i),
                                                     R[r]};
        vals[i * n_R + r] = m.evaluate(pt)[0];
      }
    return 0;
  }
  catch (std::exception const& e) {
    return fail(err, errlen, e.what());
  }
}

int
y3r_nfw_dsigma_mis(const char* data_root, double omega_m, int n,
                   const double* r, const double* rmis, const double* lnM,
                   double* out, char* err, int errlen)
{
  try {
    set_data_root(data_root);
    y3_cluster::NFW_DSIGMA_MIS f(4.0, 2.77533742639e+11, y3_cluster::GAMMA);
    f.set_rho_mult(omega_m);
    for (int i = 0; i != n; ++i) out[i] = f(r[i], rmis[i], lnM[i]);
    return 0;
  }
  catch (std::exception const& e) {
    return fail(err, errlen, e.what());
  }
}

int
y3r_shear_prj_frozen(const y3r_prj_cfg* c, const char* data_root, const y3r_sample* s,
                     const y3r_prj_sample* ps, double* out, char* err, int errlen)
{
  try {
    set_data_root(data_root);
    char const* label = y3_cluster::ShearPrjFrozenPhysics::module_label();
    cosmosis::DataBlock cfg, b;
    if (c->n_lnm > 0) cfg.put_val(label, "n_lnm", c->n_lnm);
    if (c->n_per_seg > 0) cfg.put_val(label, "n_per_seg", c->n_per_seg);
    if (c->n_zring > 0) cfg.put_val(label, "n_zring", c->n_zring);
    if (c->n_zouter > 0) cfg.put_val(label, "n_zouter", c->n_zouter);
    cfg.put_val(label, "zt_low", c->zt_low);
    cfg.put_val(label, "zt_high", c->zt_high);
    cfg.put_val(label, "lnm_low", c->lnm_low);
    cfg.put_val(label, "lnm_high", c->lnm_high);
    if (c->R_max_cMpch >= 0) cfg.put_val(label, "R_max_cMpch", c->R_max_cMpch);
    if (c->include_omega_z >= 0) cfg.put_val(label, "include_omega_z", c->include_omega_z);
    if (c->lob_centers) cfg.put_val(label, "lob_centers", vec(c->lob_centers, c->n_lob));
    cfg.put_val(label, "lambda_bin", vec(c->lambda_bin, c->n_gp));
    cfg.put_val(label, "zo_low", vec(c->zo_low, c->n_gp));
    cfg.put_val(label, "zo_high", vec(c->zo_high, c->n_gp));
    cfg.put_val(label, "radii", vec(c->radii, c->n_gp));
    put_sample(b, s);
    b.put_val("distances", "d_c", vec(ps->dist_dc, ps->nd));
    b.put_val("haloModel", "lnM", vec(ps->halo_lnM, ps->n_hl));
    b.put_val("haloModel", "z", vec(ps->halo_z, ps->n_hz));
    b.put_val("haloModel", "bias",
              cosmosis::ndarray<double>(vec(ps->bias, ps->n_hl * ps->n_hz),
                                        {static_cast<std::size_t>(ps->n_hz),
                                         static_cast<std::size_t>(ps->n_hl)}));
    b.put_val("xi_nl", "r", vec(ps->xi_r, ps->n_xr));
    b.put_val("xi_nl", "z", vec(ps->xi_z, ps->n_xz));
    b.put_val("xi_nl", "xi_nl",
              cosmosis::ndarray<double>(vec(ps->xi_nl, ps->n_xr * ps->n_xz),
                                        {static_cast<std::size_t>(ps->n_xz),
                                         static_cast<std::size_t>(ps->n_xr)}));
    b.put_val("b_sel_marginalised", "lob", vec(ps->bsel_lob, ps->n_blob));
    b.put_val("b_sel_marginalised", "zob", vec(ps->bsel_zob, ps->n_bzob));
    int const nbs = ps->n_blob * ps->n_bzob;
    std::vector<std::size_t> ext{static_cast<std::size_t>(ps->n_bzob),
                                 static_cast<std::size_t>(ps->n_blob)};
    b.put_val("b_sel_marginalised", "b_small",
              cosmosis::ndarray<double>(vec(ps->b_small, nbs), ext));
    b.put_val("b_sel_marginalised", "b_large",
              cosmosis::ndarray<double>(vec(ps->b_large, nbs), ext));
    y3_cluster::ShearPrjFrozenPhysics m(cfg);
    m.set_sample(b);
    for (int i = 0; i != c->n_gp; ++i) {
      y3_cluster::ShearPrjFrozenPhysics::grid_point_t pt{c->lambda_bin[i], c->zo_low[i],
                                                         c->zo_high[i], c->radii[i]};
      auto const v = m.evaluate(pt);
      for (int k = 0; k != 9; ++k) out[(size_t)i * 9 + k] = v[k];
    }
    return 0;
  }
  catch (std::exception const& e) {
    return fail(err, errlen, e.what());
  }
}

int
y3r_bsel_marg(const y3r_bsel_cfg* c, const y3r_sample* s, const y3r_prj_sample* ps,
              const y3r_hod* hod, double* out, char* err, int errlen)
{
  try {
    char const* label = y3_cluster::P_operator::module_label();
    cosmosis::DataBlock cfg, b;
    if (c->n_lt > 0) cfg.put_val(label, "n_lt", c->n_lt);
    if (c->n_zring > 0) cfg.put_val(label, "n_zring", c->n_zring);
    if (c->n_zouter > 0) cfg.put_val(label, "n_zouter", c->n_zouter);
    if (c->n_lnm > 0) cfg.put_val(label, "n_lnm", c->n_lnm);
    if (c->n_theta > 0) cfg.put_val(label, "n_theta", c->n_theta);
    if (c->n_zt_ref > 0) cfg.put_val(label, "n_zt_ref", c->n_zt_ref);
    if (c->zt_ref_low >= 0) cfg.put_val(label, "zt_ref_low", c->zt_ref_low);
    if (c->zt_ref_high >= 0) cfg.put_val(label, "zt_ref_high", c->zt_ref_high);
    cfg.put_val(label, "lnm_low", c->lnm_low);
    cfg.put_val(label, "lnm_high", c->lnm_high);
    put_sample(b, s);
    b.put_val("distances", "d_c", vec(ps->dist_dc, ps->nd));
    b.put_val("haloModel", "lnM", vec(ps->halo_lnM, ps->n_hl));
    b.put_val("haloModel", "z", vec(ps->halo_z, ps->n_hz));
    b.put_val("haloModel", "bias",
              cosmosis::ndarray<double>(vec(ps->bias, ps->n_hl * ps->n_hz),
                                        {static_cast<std::size_t>(ps->n_hz),
                                         static_cast<std::size_t>(ps->n_hl)}));
    b.put_val("xi_nl", "r", vec(ps->xi_r, ps->n_xr));
    b.put_val("xi_nl", "z", vec(ps->xi_z, ps->n_xz));
    b.put_val("xi_nl", "xi_nl",
              cosmosis::ndarray<double>(vec(ps->xi_nl, ps->n_xr * ps->n_xz),
                                        {static_cast<std::size_t>(ps->n_xz),
                                         static_cast<std::size_t>(ps->n_xr)}));
    b.put_val("cluster_mor", "log10_Mmin", hod->log10_Mmin);
    b.put_val("cluster_mor", "log10_M1", hod->log10_M1);
    b.put_val("cluster_mor", "alpha", hod->alpha);
    b.put_val("cluster_mor", "epsilon", hod->epsilon);
    b.put_val("cluster_mor", "sigma_lambda", hod->sigma_lambda);
    if (hod->has_z_pivot) b.put_val("cluster_mor", "z_pivot", hod->z_pivot);
    y3_cluster::P_operator m(cfg);
    m.set_sample(b);
    for (int i = 0; i != c->n_gp; ++i) {
      y3_cluster::P_operator::grid_point_t pt{c->zo_low[i], c->zo_high[i], c->lambda_bin[i]};
      auto const v = m.evaluate(pt);
      for (int k = 0; k != 3; ++k) out[(size_t)i * 3 + k] = v[k];
    }
    return 0;
  }
  catch (std::exception const& e) {
    return fail(err, errlen, e.what());
  }
}

} // extern "C"
