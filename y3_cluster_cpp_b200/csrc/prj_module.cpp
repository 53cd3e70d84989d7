// prj_module.cpp -- CosmoSIS module ShearPrjFrozenPhysics.so wrapping the
// y3b projection-shear observable (ShearPrjFrozenPhysics,
// src/models/sigma_prj_frozen_t.hh:34-512; module
// src/modules/sigma_prj_cpu/ShearPrjFrozenPhysics.cc).  Section label
// shear_prj_frozen_physics: the grid is the wall of numbers lambda_bin,
// zo_low, zo_high, radii; the options n_lnm (24), n_per_seg (10), n_zring
// (20), n_zouter (20), zt_low, zt_high, lnm_low, lnm_high, R_max_cMpch (30),
// include_omega_z (1), lob_centers.  Outputs, one value per grid point:
// dsigma_prj_frozen_physics/{vals, rnd, cl}, shear_prj_frozen_physics/{vals,
// rnd, cl} and the shear_prj/{vals, rnd, cl} alias
// (sigma_prj_frozen_t.hh:354-370).  The single-kernel miscentring table is
// read from $Y3_CLUSTER_CPP_DIR/data/nfw_off_center/ when present
// (mis_profile = table|quadrature, default: the table when the files exist).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "y3b.h"
#include "y3b_cosmosis.h"

namespace {

const char* const kLabel = "shear_prj_frozen_physics";

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

bool
read_numbers(const std::string& path, std::vector<double>& out)
{
  std::ifstream f(path);
  if (!f) return false;
  out.clear();
  std::string line;
  while (std::getline(f, line)) {
    if (line.rfind('#', 0) == 0) continue;
    std::istringstream ls(line);
    double v;
    while (ls >> v) out.push_back(v);
  }
  return true;
}

struct Module {
  y3b_prj* h = nullptr;
  int n_gp = 0;
  ~Module() { y3b_prj_destroy(h); }
};

}  // namespace

extern "C" void*
setup(c_datablock* o)
{
  Module* m = nullptr;
  try {
    y3b_prj_config c{};
    c.n_lnm = opt_i(o, "n_lnm", 24);
    c.n_per_seg = opt_i(o, "n_per_seg", 10);
    c.n_zring = opt_i(o, "n_zring", 20);
    c.n_zouter = opt_i(o, "n_zouter", 20);
    c.zt_low = need_d(o, opt_section(o, "zt_low"), "zt_low");
    c.zt_high = need_d(o, opt_section(o, "zt_high"), "zt_high");
    c.lnm_low = need_d(o, opt_section(o, "lnm_low"), "lnm_low");
    c.lnm_high = need_d(o, opt_section(o, "lnm_high"), "lnm_high");
    c.R_max_cMpch = opt_d(o, "R_max_cMpch", 30.0);
    c.include_omega_z = opt_i(o, "include_omega_z", 1);
    std::vector<double> lob;
    if (const char* ls = opt_section(o, "lob_centers")) lob = get_vec(o, ls, "lob_centers");
    if (!lob.empty()) {
      c.n_lob = (int)lob.size();
      c.lob_centers = lob.data();
    }
    std::vector<double> lb = get_vec(o, opt_section(o, "lambda_bin"), "lambda_bin");
    std::vector<double> zl = get_vec(o, opt_section(o, "zo_low"), "zo_low");
    std::vector<double> zh = get_vec(o, opt_section(o, "zo_high"), "zo_high");
    std::vector<double> rr = get_vec(o, opt_section(o, "radii"), "radii");
    if (zl.size() != lb.size() || zh.size() != lb.size() || rr.size() != lb.size())
      throw Failure{"lambda_bin, zo_low, zo_high and radii must have one length"};
    std::vector<int> lbi(lb.size());
    for (size_t i = 0; i < lb.size(); ++i) lbi[i] = (int)lb[i];
    c.n_gp = (int)lb.size();
    c.lambda_bin = lbi.data();
    c.zo_low = zl.data();
    c.zo_high = zh.data();
    c.radii = rr.data();
    m = new Module();
    m->n_gp = c.n_gp;
    if (y3b_prj_create(&c, &m->h) != Y3B_OK) throw Failure{y3b_last_error()};
    std::string mode = "auto";
    if (const char* ps = opt_section(o, "mis_profile")) {
      char* str = nullptr;
      if (c_datablock_get_string(o, ps, "mis_profile", &str) == DBS_SUCCESS && str) {
        mode = str;
        std::free(str);
      }
    }
    if (mode != "auto" && mode != "table" && mode != "quadrature")
      throw Failure{"mis_profile must be 'table' or 'quadrature', got '" + mode + "'"};
    if (mode != "quadrature") {
      const char* root = std::getenv("Y3_CLUSTER_CPP_DIR");
      const std::string stem =
        std::string(root ? root : "") + "/data/nfw_off_center/table_1000_1e-03_5e+03_";
      std::vector<double> lx, lxm, tab;
      const bool ok = root && read_numbers(stem + "single_logx.txt", lx) &&
                      read_numbers(stem + "single_logxmis.txt", lxm) &&
                      read_numbers(stem + "log_deltasigma_single.txt", tab);
      if (ok) {
        if (tab.size() != lx.size() * lxm.size())
          throw Failure{"Interp2D -- wrong number of z values passed (" + stem +
                        "log_deltasigma_single.txt)"};
        if (y3b_prj_set_mis_table(m->h, (int)lx.size(), lx.data(), (int)lxm.size(),
                                  lxm.data(), tab.data()) != Y3B_OK)
          throw Failure{y3b_last_error()};
      } else if (mode == "table") {
        throw Failure{"Failed to open file: " + stem + "*single*.txt"};
      }
    }
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
    y3b_prj_sample s{};
    s.cosmo.om = need_d(b, cp, "omega_m");
    s.cosmo.ol = need_d(b, cp, "omega_lambda");
    s.cosmo.ok = need_d(b, cp, "omega_k");
    s.cosmo.h0 = need_d(b, cp, "h0");
    s.cosmo.onu = need_d(b, cp, "omega_nu");
    s.cosmo.hmf_s = need_d(b, "cluster_abundance", "hmf_s");
    s.cosmo.hmf_q = need_d(b, "cluster_abundance", "hmf_q");
    std::vector<int> e1, e2, e3, e4, e5;
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
    std::vector<double> sz, sv;
    if (c_datablock_has_value(b, "average_sigma_crit_inv", "zlense")) {
      sz = get_vec(b, "average_sigma_crit_inv", "zlense");
      sv = get_vec(b, "average_sigma_crit_inv", "sci_average");
    }
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
    std::vector<double> blob = get_vec(b, "b_sel_marginalised", "lob");
    std::vector<double> bzob = get_vec(b, "b_sel_marginalised", "zob");
    std::vector<double> bs = get_nd(b, "b_sel_marginalised", "b_small", e4);
    std::vector<double> bl = get_nd(b, "b_sel_marginalised", "b_large", e5);
    if ((size_t)e4[0] * e4[1] != blob.size() * bzob.size() ||
        (size_t)e5[0] * e5[1] != blob.size() * bzob.size())
      throw Failure{"b_sel_marginalised/b_small, b_large must be n_zob x n_lob"};
    s.t = y3b_tables{(int)mh.size(), mh.data(), (int)hz.size(), hz.data(), dn.data(),
                     (int)dz.size(), dz.data(), da.data(), (int)sz.size(),
                     sz.empty() ? nullptr : sz.data(), sv.empty() ? nullptr : sv.data()};
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
    s.n_blob = (int)blob.size();
    s.n_bzob = (int)bzob.size();
    s.bsel_lob = blob.data();
    s.bsel_zob = bzob.data();
    s.b_small = bs.data();
    s.b_large = bl.data();
    std::vector<double> out((size_t)m->n_gp * 9);
    if (y3b_prj_eval(m->h, &s, out.data()) != Y3B_OK) throw Failure{y3b_last_error()};
    static const char* const sec[9] = {
      "dsigma_prj_frozen_physics", "dsigma_prj_frozen_physics", "dsigma_prj_frozen_physics",
      "shear_prj_frozen_physics",  "shear_prj_frozen_physics",  "shear_prj_frozen_physics",
      "shear_prj",                 "shear_prj",                 "shear_prj"};
    static const char* const name[9] = {"vals", "rnd", "cl", "vals", "rnd", "cl",
                                        "vals", "rnd", "cl"};
    std::vector<double> col(m->n_gp);
    for (int k = 0; k < 9; ++k) {
      for (int i = 0; i < m->n_gp; ++i) col[i] = out[(size_t)i * 9 + k];
      if (c_datablock_put_double_array_1d(b, sec[k], name[k], col.data(), m->n_gp) !=
          DBS_SUCCESS)
        throw Failure{std::string("cannot write ") + sec[k] + "/" + name[k]};
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
