// cosmosis_module.cpp -- CosmoSIS module wrapping the y3b engine.  Built once
// per module label:
//   Y3B_MODULE_SHEAR = 0: NumCountsSel / NumCountsFastMass
//                         (NumCountsSelGL, n_operator_sel_gl_t.hh:178-224)
//   Y3B_MODULE_SHEAR = 1: Shear1hMisSel / Shear1hFastMass
//                         (Shear1hMisSelGL, n_operator_sel_gl_t.hh:239-361)
// Y3B_MODULE_LABEL is the ini section read in setup (module_label()) and
// Y3B_MODULE_OUTPUT the hard-coded output section (output_sections()).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "y3b.h"
#include "y3b_cosmosis.h"

#ifndef Y3B_MODULE_SHEAR
#error "define Y3B_MODULE_SHEAR"
#endif

namespace {

const char* const kLabel = Y3B_MODULE_LABEL;
const char* const kOutput = Y3B_MODULE_OUTPUT;
const char* const kOptionSection = "module_options";

struct Failure {
  std::string msg;
};

void
report(const std::string& m)
{
  std::fprintf(stderr, "[%s] %s\n", kLabel, m.c_str());
}

// Option lookup: the module's own section first (the reference reads
// cfg.view(label, key)), then CosmoSIS's alias section for module options.
const char*
opt_section(c_datablock* b, const char* key)
{
  if (c_datablock_has_value(b, kLabel, key)) return kLabel;
  if (c_datablock_has_value(b, kOptionSection, key)) return kOptionSection;
  return nullptr;
}

bool
get_d(c_datablock* b, const char* sec, const char* key, double* v)
{
  return c_datablock_get_double(b, sec, key, v) == DBS_SUCCESS;
}

[[maybe_unused]] double
need_d(c_datablock* b, const char* sec, const char* key)
{
  double v;
  if (!sec || !get_d(b, sec, key, &v))
    throw Failure{std::string("missing ") + (sec ? sec : kLabel) + "/" + key};
  return v;
}

[[maybe_unused]] double
opt_d(c_datablock* b, const char* key, double dflt)
{
  const char* s = opt_section(b, key);
  double v;
  return (s && get_d(b, s, key, &v)) ? v : dflt;
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
  if (!sec || c_datablock_get_double_array_1d(b, sec, key, &p, &n) != DBS_SUCCESS)
    throw Failure{std::string("missing array ") + (sec ? sec : kLabel) + "/" + key};
  std::vector<double> out(p, p + n);
  std::free(p);
  return out;
}

std::vector<int>
get_ivec(c_datablock* b, const char* sec, const char* key)
{
  int* p = nullptr;
  int n = 0;
  if (sec && c_datablock_get_int_array_1d(b, sec, key, &p, &n) == DBS_SUCCESS) {
    std::vector<int> out(p, p + n);
    std::free(p);
    return out;
  }
  std::vector<double> d = get_vec(b, sec, key);  // ints written as doubles
  std::vector<int> out;
  for (double x : d) out.push_back((int)std::lround(x));
  return out;
}

std::vector<double>
get_nd(c_datablock* b, const char* sec, const char* key, int ndim_expected,
       std::vector<int>& ext)
{
  int nd = 0;
  if (c_datablock_get_array_ndim(b, sec, key, &nd) != DBS_SUCCESS || nd != ndim_expected)
    throw Failure{std::string(sec) + "/" + key + " must be a " + std::to_string(ndim_expected) +
                  "-D array"};
  ext.assign(nd, 0);
  if (c_datablock_get_double_array_shape(b, sec, key, nd, ext.data()) != DBS_SUCCESS)
    throw Failure{std::string("cannot read shape of ") + sec + "/" + key};
  size_t n = 1;
  for (int e : ext) n *= (size_t)e;
  std::vector<double> out(n);
  if (c_datablock_get_double_array(b, sec, key, out.data(), nd, ext.data()) != DBS_SUCCESS)
    throw Failure{std::string("cannot read ") + sec + "/" + key};
  return out;
}

// Numbers of a whitespace-separated text file, skipping lines that start
// with '#', as the reference's read_vector does (src/utils/read_vector.hh).
[[maybe_unused]] bool
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
  y3b_selgl* core = nullptr;
  std::vector<int> bins;
  std::vector<double> r_perp;  // shear only
  std::vector<double> lob_centers;
  bool idea2 = false;
  double stencil_h = 0.15;
  ~Module() { y3b_selgl_destroy(core); }
};

// Sample tables held while one execute() runs.
struct Sample {
  y3b_cosmo c{};
  std::vector<double> mh, hz, dn, dz, da, sz, sv, sl, szz, S;
  std::vector<int> dn_ext, S_ext;
};

void
read_sample(c_datablock* b, Sample& s, bool with_sci)
{
  const char* cp = "cosmological_parameters";
  s.c.om = need_d(b, cp, "omega_m");
  s.c.ol = need_d(b, cp, "omega_lambda");
  s.c.ok = need_d(b, cp, "omega_k");
  s.c.h0 = need_d(b, cp, "h0");
  s.c.onu = need_d(b, cp, "omega_nu");
  s.c.hmf_s = need_d(b, "cluster_abundance", "hmf_s");
  s.c.hmf_q = need_d(b, "cluster_abundance", "hmf_q");
  s.mh = get_vec(b, "mass_function", "m_h");
  s.hz = get_vec(b, "mass_function", "z");
  s.dn = get_nd(b, "mass_function", "dndlnmh", 2, s.dn_ext);
  if (s.dn_ext[0] != (int)s.hz.size() || s.dn_ext[1] != (int)s.mh.size())
    throw Failure{"Interp2D -- ndarray wrong dimensions (mass_function/dndlnmh)"};
  s.dz = get_vec(b, "distances", "z");
  s.da = get_vec(b, "distances", "d_a");
  if (s.dz.size() != s.da.size()) throw Failure{"distances/z and d_a differ in length"};
  if (with_sci) {
    s.sz = get_vec(b, "average_sigma_crit_inv", "zlense");
    s.sv = get_vec(b, "average_sigma_crit_inv", "sci_average");
    if (s.sz.size() != s.sv.size()) throw Failure{"average_sigma_crit_inv arrays differ in length"};
  }
  s.sl = get_vec(b, "sel_function", "lnM");
  s.szz = get_vec(b, "sel_function", "z");
  s.S = get_nd(b, "sel_function", "S_stack", 3, s.S_ext);
  if (s.S_ext[1] != (int)s.szz.size() || s.S_ext[2] != (int)s.sl.size())
    throw Failure{"sel_function: S_stack extents mismatch"};
}

int
build(Module* m, Sample& s, bool with_sci)
{
  y3b_tables t{(int)s.mh.size(), s.mh.data(), (int)s.hz.size(), s.hz.data(), s.dn.data(),
               (int)s.dz.size(), s.dz.data(), s.da.data(),
               with_sci ? (int)s.sz.size() : 0, with_sci ? s.sz.data() : nullptr,
               with_sci ? s.sv.data() : nullptr};
  y3b_selection sel{s.S_ext[0], (int)s.sl.size(), s.sl.data(), (int)s.szz.size(), s.szz.data(),
                    s.S.data()};
  return y3b_selgl_build(m->core, &s.c, &t, &sel, with_sci ? 1 : 0);
}

}  // namespace

extern "C" void*
setup(c_datablock* options)
{
  Module* m = nullptr;
  try {
    y3b_selgl_config cfg;
    cfg.n_lnm = opt_i(options, "n_lnm", 96);
    cfg.n_z = opt_i(options, "n_z", 64);
    cfg.zt_low = need_d(options, opt_section(options, "zt_low"), "zt_low");
    cfg.zt_high = need_d(options, opt_section(options, "zt_high"), "zt_high");
    cfg.lnm_low = need_d(options, opt_section(options, "lnm_low"), "lnm_low");
    cfg.lnm_high = need_d(options, opt_section(options, "lnm_high"), "lnm_high");
    m = new Module();
    m->bins = get_ivec(options, opt_section(options, "bin_index"), "bin_index");
#if Y3B_MODULE_SHEAR
    m->r_perp = get_vec(options, opt_section(options, "r_perp"), "r_perp");
    const char* ls = opt_section(options, "lob_centers");
    m->lob_centers = ls ? get_vec(options, ls, "lob_centers")
                        : std::vector<double>{25.0, 37.5, 52.5, 130.0};
    if (m->lob_centers.empty()) throw Failure{"Shear1hMisSelGL: lob_centers is empty"};
    m->stencil_h = opt_d(options, "stencil_h", 0.15);
    const char* ms = opt_section(options, "method");
    if (ms) {
      char* str = nullptr;
      if (c_datablock_get_string(options, ms, "method", &str) == DBS_SUCCESS && str) {
        std::string v(str);
        std::free(str);
        if (v == "exact")
          m->idea2 = false;
        else if (v == "idea2")
          m->idea2 = true;
        else
          throw Failure{"Shear1hMisSelGL: method must be 'exact' or 'idea2', got '" + v + "'"};
      }
    }
#endif
    int rc = y3b_selgl_create(&cfg, &m->core);
    if (rc != Y3B_OK) throw Failure{std::string("y3b_selgl_create: ") + y3b_last_error()};
#if Y3B_MODULE_SHEAR
    // NFW_DSIGMA_MIS reads its gamma-kernel profile table from
    // $Y3_CLUSTER_CPP_DIR/data/nfw_off_center/ when the module is constructed
    // (nfw_dsigma_mis.hh:33-55,62-72).  mis_profile = table requires those
    // files, quadrature computes the profile directly, and the default uses
    // the table when the files are present.
    std::string mode = "auto";
    if (const char* ps = opt_section(options, "mis_profile")) {
      char* str = nullptr;
      if (c_datablock_get_string(options, ps, "mis_profile", &str) == DBS_SUCCESS && str) {
        mode = str;
        std::free(str);
      }
    }
    if (mode != "auto" && mode != "table" && mode != "quadrature")
      throw Failure{"mis_profile must be 'table' or 'quadrature', got '" + mode + "'"};
    if (mode != "quadrature") {
      const char* root = std::getenv("Y3_CLUSTER_CPP_DIR");
      std::string stem = std::string(root ? root : "") +
                         "/data/nfw_off_center/table_1000_1e-03_5e+03_";
      std::vector<double> lx, lxm, tab;
      bool ok = root && read_numbers(stem + "gamma_logx.txt", lx) &&
                read_numbers(stem + "gamma_logxmis.txt", lxm) &&
                read_numbers(stem + "log_deltasigma_gamma.txt", tab);
      if (ok) {
        if (tab.size() != lx.size() * lxm.size())
          throw Failure{"Interp2D -- wrong number of z values passed (" + stem +
                        "log_deltasigma_gamma.txt)"};
        rc = y3b_selgl_set_mis_table(m->core, (int)lx.size(), lx.data(), (int)lxm.size(),
                                     lxm.data(), tab.data());
        if (rc != Y3B_OK) throw Failure{y3b_last_error()};
      } else if (mode == "table") {
        throw Failure{"Failed to open file: " + stem + "*_gamma*.txt"};
      }
    }
#endif
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
execute(c_datablock* block, void* module)
{
  Module* m = static_cast<Module*>(module);
  if (!m) {
    report("execute called without a module (setup failed)");
    return 1;
  }
  try {
    Sample s;
#if !Y3B_MODULE_SHEAR
    read_sample(block, s, false);
    int rc = build(m, s, false);
    if (rc != Y3B_OK) throw Failure{y3b_last_error()};
    std::vector<double> vals(m->bins.size());
    rc = y3b_selgl_counts(m->core, (int)m->bins.size(), m->bins.data(), vals.data());
    if (rc != Y3B_OK) throw Failure{y3b_last_error()};
#else
    read_sample(block, s, true);
    int rc = build(m, s, true);
    if (rc != Y3B_OK) throw Failure{y3b_last_error()};
    std::vector<int> ext;
    std::vector<double> rs = get_vec(block, "haloModel", "r_sigma");
    std::vector<double> lm = get_vec(block, "haloModel", "lnM");
    std::vector<double> ds = get_nd(block, "haloModel", "dSigma_nfw", 2, ext);
    if (ext[0] != (int)lm.size() || ext[1] != (int)rs.size())
      throw Failure{"Interp2D -- ndarray wrong dimensions (haloModel/dSigma_nfw)"};
    double f_mis = 0.22, tau_mis = 0.17;  // lensing_weights.hh:168-169
    get_d(block, "miscentering", "f_mis", &f_mis);
    get_d(block, "miscentering", "tau_mis", &tau_mis);
    y3b_shear_table st{(int)rs.size(), rs.data(), (int)lm.size(), lm.data(), ds.data(),
                       f_mis, tau_mis, (int)m->lob_centers.size(), m->lob_centers.data(),
                       4.0, 64, 128, 20.0, m->idea2 ? 1 : 0, m->stencil_h};
    // Cartesian product bin_index x r_perp, bin slow and R fast.
    std::vector<int> pb;
    std::vector<double> pr;
    for (int b : m->bins)
      for (double r : m->r_perp) {
        pb.push_back(b);
        pr.push_back(r);
      }
    std::vector<double> vals(pb.size());
    rc = y3b_selgl_shear(m->core, &st, (int)pb.size(), pb.data(), pr.data(), vals.data());
    if (rc != Y3B_OK) throw Failure{y3b_last_error()};
#endif
    if (c_datablock_put_double_array_1d(block, kOutput, "vals", vals.data(), (int)vals.size()) !=
        DBS_SUCCESS)
      throw Failure{std::string("cannot write ") + kOutput + "/vals"};
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
