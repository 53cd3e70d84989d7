// bsel_module.cpp -- CosmoSIS module BSelMargIntegrand.so wrapping the y3b
// selection-bias operators (P_operator, src/models/p_operator_t.hh:76-718;
// module src/modules/b_sel_marg_cpu/BSelMargIntegrand.cc).  Section label
// b_sel_marg: the grid is the wall of numbers zo_low, zo_high, lambda_bin;
// the options n_lt (60), n_zring (20), n_zouter (30), n_lnm (24), n_theta
// (10), n_zt_ref (80), zt_ref_low (0.05), zt_ref_high (0.90), lnm_low,
// lnm_high.  Per sample it reads cosmological_parameters, cluster_abundance
// hmf_s / hmf_q, mass_function, distances/{z, d_a, d_c}, haloModel/{lnM, z,
// bias}, xi_nl/{r, z, xi_nl} and the cluster_mor HOD parameters (log10_M1
// or log10_ratio, optional z_pivot), and writes one value per grid point to
// b_sel_marg_P1/vals, b_sel_marg_I1/vals and b_sel_marg_J/vals.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "y3b.h"
#include "y3b_cosmosis.h"

namespace {

const char* const kLabel = "b_sel_marg";

struct Failure {
  std::string msg;
};

void
report(const std::string& m)
{
  std::fprintf(stderr, "[%s] %s\n", kLabel, m.c_str());
}

const char*
opt_section(c_datablock* b, const char* key)
{
  if (c_datablock_has_value(b, kLabel, key)) return kLabel;
  if (c_datablock_has_value(b, "module_options", key)) return "module_options";
  return nullptr;
}

double
need_d(c_datablock* b, const char* sec, const char* key)
{
  double v;
  if (!sec || c_datablock_get_double(b, sec, key, &v) != DBS_SUCCESS)
    throw Failure{std::string("missing ") + (sec ? sec : kLabel) + "/" + key};
  return v;
}

double
opt_d(c_datablock* b, const char* key, double dflt)
{
  const char* s = opt_section(b, key);
  double v;
  return (s && c_datablock_get_double(b, s, key, &v) == DBS_SUCCESS) ? v : dflt;
}

int
opt_i(c_datablock* b, const char* key, int dflt)
{
  const char* s = opt_section(b, key);
  int v;
  return (s && c_datablock_get_int(b, s, key, &v) == DBS_SUCCESS) ? v : dflt;
}

std::vector<double>
get_vec(c_datablock* b, const char* sec, const char* key)
{
  double* p = nullptr;
  int n = 0;
  if (sec && c_datablock_get_double_array_1d(b, sec, key, &p, &n) == DBS_SUCCESS) {
    std::vector<double> out(p, p + n);
    std::free(p);
    return out;
  }
  int* ip = nullptr;
  if (sec && c_datablock_get_int_array_1d(b, sec, key, &ip, &n) == DBS_SUCCESS) {
    std::vector<double> out(ip, ip + n);
    std::free(ip);
    return out;
  }
  throw Failure{std::string("missing array ") + (sec ? sec : kLabel) + "/" + key};
}

std::vector<double>
get_nd(c_datablock* b, const char* sec, const char* key, std::vector<int>& ext)
{
  int nd = 0;
  if (c_datablock_get_array_ndim(b, sec, key, &nd) != DBS_SUCCESS || nd != 2)
    throw Failure{std::string(sec) + "/" + key + " must be a 2-D array"};
  ext.assign(2, 0);
  if (c_datablock_get_double_array_shape(b, sec, key, 2, ext.data()) != DBS_SUCCESS)
    throw Failure{std::string("cannot read shape of ") + sec + "/" + key};
  std::vector<double> out((size_t)ext[0] * ext[1]);
  if (c_datablock_get_double_array(b, sec, key, out.data(), 2, ext.data()) != DBS_SUCCESS)
    throw Failure{std::string("cannot read ") + sec + "/" + key};
  return out;
}

struct Module {
  y3b_bsel* h = nullptr;
  int n_gp = 0;
  ~Module() { y3b_bsel_destroy(h); }
};

}  // namespace

extern "C" void*
setup(c_datablock* o)
{
  Module* m = nullptr;
  try {
    y3b_bsel_config c{};
    c.n_lt = opt_i(o, "n_lt", 60);
    c.n_zring = opt_i(o, "n_zring", 20);
    c.n_zouter = opt_i(o, "n_zouter", 30);
    c.n_lnm = opt_i(o, "n_lnm", 24);
    c.n_theta = opt_i(o, "n_theta", 10);
    c.n_zt_ref = opt_i(o, "n_zt_ref", 80);
    c.zt_ref_low = opt_d(o, "zt_ref_low", 0.05);
    c.zt_ref_high = opt_d(o, "zt_ref_high", 0.90);
    c.lnm_low = need_d(o, opt_section(o, "lnm_low"), "lnm_low");
    c.lnm_high = need_d(o, opt_section(o, "lnm_high"), "lnm_high");
    std::vector<double> zl = get_vec(o, opt_section(o, "zo_low"), "zo_low");
    std::vector<double> zh = get_vec(o, opt_section(o, "zo_high"), "zo_high");
    std::vector<double> lb = get_vec(o, opt_section(o, "lambda_bin"), "lambda_bin");
    if (zh.size() != zl.size() || lb.size() != zl.size())
      throw Failure{"zo_low, zo_high and lambda_bin must have one length"};
    std::vector<int> lbi(lb.size());
    for (size_t i = 0; i < lb.size(); ++i) lbi[i] = (int)lb[i];
    c.n_gp = (int)zl.size();
    c.zo_low = zl.data();
    c.zo_high = zh.data();
    c.lambda_bin = lbi.data();
    c.max_samples = 1;
    m = new Module();
    m->n_gp = c.n_gp;
    if (y3b_bsel_create(&c, &m->h) != Y3B_OK) throw Failure{y3b_last_error()};
    return m;
  } catch (const Failure& f) {
    report("setup failed: " + f.msg);
  } catch (...) {
    report("setup failed: unknown error");
  }
  delete m;
  return nullptr;
}

extern "C" DATABLOCK_STATUS
execute(c_datablock* b, void* module)
{
  Module* m = static_cast<Module*>(module);
  if (!m) {
    report("execute called without a module (setup failed)");
    return 1;
  }
  try {
    const char* cp = "cosmological_parameters";
    const char* cm = "cluster_mor";
    y3b_bsel_sample s{};
    s.cosmo.om = need_d(b, cp, "omega_m");
    s.cosmo.ol = need_d(b, cp, "omega_lambda");
    s.cosmo.ok = need_d(b, cp, "omega_k");
    s.cosmo.h0 = need_d(b, cp, "h0");
    s.cosmo.onu = need_d(b, cp, "omega_nu");
    s.cosmo.hmf_s = need_d(b, "cluster_abundance", "hmf_s");
    s.cosmo.hmf_q = need_d(b, "cluster_abundance", "hmf_q");
    // MOR_HOD_t(DataBlock&) (mor_hod_t.hh:72-83, 186-195): log10_ratio wins
    // over log10_M1; z_pivot defaults to 0.45.
    s.hod[0] = need_d(b, cm, "log10_Mmin");
    s.hod[1] = c_datablock_has_value(b, cm, "log10_ratio")
                 ? s.hod[0] + need_d(b, cm, "log10_ratio")
                 : need_d(b, cm, "log10_M1");
    s.hod[2] = need_d(b, cm, "alpha");
    s.hod[3] = need_d(b, cm, "epsilon");
    s.hod[4] = need_d(b, cm, "sigma_lambda");
    s.hod[5] = c_datablock_has_value(b, cm, "z_pivot") ? need_d(b, cm, "z_pivot") : 0.45;
    std::vector<int> e1, e2, e3;
    std::vector<double> mh = get_vec(b, "mass_function", "m_h");
    std::vector<double> hz = get_vec(b, "mass_function", "z");
    std::vector<double> dn = get_nd(b, "mass_function", "dndlnmh", e1);
    std::vector<double> dz = get_vec(b, "distances", "z");
    std::vector<double> da = get_vec(b, "distances", "d_a");
    std::vector<double> dc = get_vec(b, "distances", "d_c");
    if (e1[0] != (int)hz.size() || e1[1] != (int)mh.size())
      throw Failure{"Interp2D -- ndarray wrong dimensions (mass_function/dndlnmh)"};
    if (da.size() != dz.size() || dc.size() != dz.size())
      throw Failure{"distances/z, d_a and d_c differ in length"};
    std::vector<double> hl = get_vec(b, "haloModel", "lnM");
    std::vector<double> hzz = get_vec(b, "haloModel", "z");
    std::vector<double> bias = get_nd(b, "haloModel", "bias", e2);
    if (e2[0] != (int)hzz.size() || e2[1] != (int)hl.size())
      throw Failure{"Interp2D -- ndarray wrong dimensions (haloModel/bias)"};
    std::vector<double> xr = get_vec(b, "xi_nl", "r");
    std::vector<double> xz = get_vec(b, "xi_nl", "z");
    std::vector<double> xi = get_nd(b, "xi_nl", "xi_nl", e3);
    if (e3[0] != (int)xz.size() || e3[1] != (int)xr.size())
      throw Failure{"Interp2D -- ndarray wrong dimensions (xi_nl/xi_nl)"};
    s.t = y3b_tables{(int)mh.size(), mh.data(), (int)hz.size(), hz.data(), dn.data(),
                     (int)dz.size(), dz.data(), da.data(), 0, nullptr, nullptr};
    s.dist_dc = dc.data();
    s.n_hl = (int)hl.size();
    s.n_hz = (int)hzz.size();
    s.halo_lnM = hl.data();
    s.halo_z = hzz.data();
    s.bias = bias.data();
    s.n_xr = (int)xr.size();
    s.n_xz = (int)xz.size();
    s.xi_r = xr.data();
    s.xi_z = xz.data();
    s.xi_nl = xi.data();
    std::vector<double> out((size_t)m->n_gp * 3);
    if (y3b_bsel_eval(m->h, 1, &s, out.data()) != Y3B_OK) throw Failure{y3b_last_error()};
    // P_operator::output_sections (p_operator_t.hh:480-486), key "vals"
    static const char* const sec[3] = {"b_sel_marg_P1", "b_sel_marg_I1", "b_sel_marg_J"};
    std::vector<double> col(m->n_gp);
    for (int k = 0; k < 3; ++k) {
      for (int i = 0; i < m->n_gp; ++i) col[i] = out[(size_t)i * 3 + k];
      if (c_datablock_put_double_array_1d(b, sec[k], "vals", col.data(), m->n_gp) !=
          DBS_SUCCESS)
        throw Failure{std::string("cannot write ") + sec[k] + "/vals"};
    }
    return DBS_SUCCESS;
  } catch (const Failure& f) {
    report("execute failed: " + f.msg);
  } catch (...) {
    report("execute failed: unknown error");
  }
  return 1;
}

extern "C" int
cleanup(void* module)
{
  delete static_cast<Module*>(module);
  return 0;
}
