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

#include "prj_table.h"
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

// engine = fused: the whole number-count integral on the engine's nested
// Gauss-Legendre nodes, one parameter point per execute.
struct Fused {
  y3b_grid grid{};
  int precision = Y3B_MIXED;
  bool write_s = false;
  y3b_selfunc_config scfg{};                 // S_stack grid (write_s_stack)
  std::vector<double> lam_min, lam_max, zob_min, zob_max, sigma_z;
  y3b_engine* e = nullptr;
  int n_hm = -1, n_hz = -1, n_dist = -1;
  std::vector<double> plob_z, plob_coef;
  std::vector<double> packed;
  ~Fused() { y3b_engine_destroy(e); }
};

struct Module {
  y3b_selgl* core = nullptr;
  Fused* fused = nullptr;
  std::vector<int> bins;
  std::vector<double> r_perp;  // shear only
  std::vector<double> lob_centers;
  bool idea2 = false;
  double stencil_h = 0.15;
  ~Module()
  {
    y3b_selgl_destroy(core);
    delete fused;
  }
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

std::string
opt_string(c_datablock* b, const char* key, const char* dflt)
{
  const char* s = opt_section(b, key);
  char* str = nullptr;
  if (s && c_datablock_get_string(b, s, key, &str) == DBS_SUCCESS && str) {
    std::string v(str);
    std::free(str);
    return v;
  }
  return dflt;
}

[[maybe_unused]] bool
opt_bool(c_datablock* b, const char* key, bool dflt)
{
  const char* s = opt_section(b, key);
  if (!s) return dflt;
  int v;
  if (c_datablock_get_int(b, s, key, &v) == DBS_SUCCESS) return v != 0;
  std::string t = opt_string(b, key, "");
  if (t == "T" || t == "t" || t == "true" || t == "True" || t == "1") return true;
  if (t == "F" || t == "f" || t == "false" || t == "False" || t == "0") return false;
  throw Failure{std::string("option ") + key + " must be a boolean"};
}

// sel_function's per-bin option, from the module's section or the
// sel_function section of the same ini.
[[maybe_unused]] std::vector<double>
bin_option(c_datablock* b, const char* key)
{
  const char* s = opt_section(b, key);
  if (!s && c_datablock_has_value(b, "sel_function", key)) s = "sel_function";
  return get_vec(b, s, key);
}

// Distinct intervals in order, from a per-bin edge list with a period.
[[maybe_unused]] void
product_edges(const std::vector<double>& lo, const std::vector<double>& hi, int stride,
              int count, std::vector<double>& edges, const char* what)
{
  edges.clear();
  for (int k = 0; k < count; ++k) {
    double a = lo[(size_t)k * stride], c = hi[(size_t)k * stride];
    if (!(c > a)) throw Failure{std::string(what) + " bins must have max > min"};
    if (k == 0)
      edges.push_back(a);
    else if (a != edges.back())
      throw Failure{std::string("engine = fused needs contiguous ") + what + " bins"};
    edges.push_back(c);
  }
}

#if !Y3B_MODULE_SHEAR
// setup() of the fused form: the sel_function bins become the engine grid's
// richness-fast product of contiguous lambda_obs and z_obs bins.
void
setup_fused(c_datablock* options, Module* m)
{
  Fused* f = m->fused = new Fused();
  f->lam_min = bin_option(options, "lam_min");
  f->lam_max = bin_option(options, "lam_max");
  f->zob_min = bin_option(options, "zob_min");
  f->zob_max = bin_option(options, "zob_max");
  f->sigma_z = bin_option(options, "sigma_z");
  const size_t nb = f->lam_min.size();
  if (nb == 0 || f->lam_max.size() != nb || f->zob_min.size() != nb ||
      f->zob_max.size() != nb || f->sigma_z.size() != nb)
    throw Failure{"sel_function bin arrays must be non-empty and of one length"};
  int nI = 1;
  while ((size_t)nI < nb && f->zob_min[nI] == f->zob_min[0] && f->zob_max[nI] == f->zob_max[0])
    ++nI;
  if (nb % nI != 0) throw Failure{"engine = fused needs a richness-fast product of bins"};
  const int nJ = (int)(nb / nI);
  if (nI > 8 || nJ > 8) throw Failure{"engine = fused supports at most 8 x 8 bins"};
  for (int j = 0; j < nJ; ++j)
    for (int i = 0; i < nI; ++i) {
      size_t b = (size_t)j * nI + i;
      if (f->lam_min[b] != f->lam_min[i] || f->lam_max[b] != f->lam_max[i] ||
          f->zob_min[b] != f->zob_min[(size_t)j * nI] ||
          f->zob_max[b] != f->zob_max[(size_t)j * nI] ||
          f->sigma_z[b] != f->sigma_z[(size_t)j * nI])
        throw Failure{"engine = fused needs a richness-fast product of bins with one sigma_z "
                      "per z_obs bin"};
    }
  std::vector<double> le, ze;
  product_edges(f->lam_min, f->lam_max, 1, nI, le, "lambda_obs");
  product_edges(f->zob_min, f->zob_max, nI, nJ, ze, "z_obs");
  y3b_grid& g = f->grid;
  g.n_m = opt_i(options, "n_lnm", 64);
  g.n_z = opt_i(options, "n_z", 32);
  g.n_t = opt_i(options, "n_lt", 64);
  g.n_o = opt_i(options, "n_lo", 64);
  g.n_zo = opt_i(options, "n_zo", 16);
  g.lnm_lo = need_d(options, opt_section(options, "lnm_low"), "lnm_low");
  g.lnm_hi = need_d(options, opt_section(options, "lnm_high"), "lnm_high");
  g.zt_lo = need_d(options, opt_section(options, "zt_low"), "zt_low");
  g.zt_hi = need_d(options, opt_section(options, "zt_high"), "zt_high");
  g.lam_t_lo = opt_d(options, "lam_t_min", 1.0);
  g.lam_t_hi = opt_d(options, "lam_t_max", 1000.0);
  g.n_lam_bins = nI;
  g.n_z_bins = nJ;
  for (int i = 0; i <= nI; ++i) g.lam_edges[i] = le[i];
  for (int j = 0; j <= nJ; ++j) g.zob_edges[j] = ze[j];
  g.sz0 = opt_d(options, "sz0", 0.0);
  for (int j = 0; j < nJ; ++j) g.sz_bin[j] = f->sigma_z[(size_t)j * nI];
  const std::string prec = opt_string(options, "precision", "mixed");
  if (prec == "mixed")
    f->precision = Y3B_MIXED;
  else if (prec == "fp64")
    f->precision = Y3B_FP64;
  else
    throw Failure{"precision must be 'mixed' or 'fp64', got '" + prec + "'"};
  for (int b : m->bins)
    if (b < 0 || b >= (int)nb)
      throw Failure{"NumCountsSelGL: bin_index outside sel_function/S_stack range"};
  f->write_s = opt_bool(options, "write_s_stack", false);
  if (f->write_s) {
    y3b_selfunc_config& s = f->scfg;
    auto sel_i = [&](const char* k, int d) {
      int v;
      return c_datablock_get_int(options, "sel_function", k, &v) == DBS_SUCCESS ? v : d;
    };
    s.n_bins = (int)nb;
    s.zt_low = g.zt_lo;
    s.zt_high = g.zt_hi;
    s.lnm_low = g.lnm_lo;
    s.lnm_high = g.lnm_hi;
    s.n_lnm = sel_i("n_lnm", 40);  // sel_function.py:437-446 defaults
    s.n_z = sel_i("n_z_shared", sel_i("n_z", 20));
    s.n_q = sel_i("N_q", 32);
  }
}

// execute() of the fused form for one parameter point.
void
execute_fused(c_datablock* block, Module* m, std::vector<double>& vals)
{
  Fused* f = m->fused;
  const char* cp = "cosmological_parameters";
  y3b_point pt{};
  pt.cosmo.om = need_d(block, cp, "omega_m");
  pt.cosmo.ol = need_d(block, cp, "omega_lambda");
  pt.cosmo.ok = need_d(block, cp, "omega_k");
  pt.cosmo.h0 = need_d(block, cp, "h0");
  pt.cosmo.onu = need_d(block, cp, "omega_nu");
  pt.cosmo.hmf_s = need_d(block, "cluster_abundance", "hmf_s");
  pt.cosmo.hmf_q = need_d(block, "cluster_abundance", "hmf_q");
  pt.A = need_d(block, "cluster_mor", "A");
  pt.B = need_d(block, "cluster_mor", "B");
  pt.C = need_d(block, "cluster_mor", "C");
  pt.sigma = need_d(block, "cluster_mor", "sigma_intr");
  pt.Mpiv = 3e14;
  get_d(block, "cluster_mor", "M_pivot", &pt.Mpiv);
  pt.grid = 0;
  std::vector<double> mh = get_vec(block, "mass_function", "m_h");
  std::vector<double> hz = get_vec(block, "mass_function", "z");
  std::vector<int> ext;
  std::vector<double> dn = get_nd(block, "mass_function", "dndlnmh", 2, ext);
  if (ext[0] != (int)hz.size() || ext[1] != (int)mh.size())
    throw Failure{"Interp2D -- ndarray wrong dimensions (mass_function/dndlnmh)"};
  std::vector<double> dz = get_vec(block, "distances", "z");
  std::vector<double> da = get_vec(block, "distances", "d_a");
  if (dz.size() != da.size()) throw Failure{"distances/z and d_a differ in length"};
  // P(lambda_obs | lambda_true, z): the sample's plob_ltr_params, else the
  // frozen default table (sel_function.py:477-490).
  std::vector<double> pz, pc;
  if (c_datablock_has_value(block, "plob_ltr_params", "z")) {
    pz = get_vec(block, "plob_ltr_params", "z");
    for (const char* k : y3b::kPrjNames) {
      std::vector<double> row = get_vec(block, "plob_ltr_params", k);
      if (row.size() != pz.size()) throw Failure{"plob_ltr_params arrays differ in length"};
      pc.insert(pc.end(), row.begin(), row.end());
    }
  } else {
    pz.assign(y3b::kPrjZ, y3b::kPrjZ + y3b::kPrjNodes);
    for (const auto& row : y3b::kPrjCoef) pc.insert(pc.end(), row, row + y3b::kPrjNodes);
  }
  if (!f->e || f->n_hm != (int)mh.size() || f->n_hz != (int)hz.size() ||
      f->n_dist != (int)dz.size() || pz != f->plob_z || pc != f->plob_coef) {
    y3b_engine_destroy(f->e);
    f->e = nullptr;
    y3b_engine_config ec{};
    ec.n_hm = (int)mh.size();
    ec.n_hz = (int)hz.size();
    ec.n_dist = (int)dz.size();
    ec.plob = y3b_plob{(int)pz.size(), pz.data(), pc.data()};
    ec.max_points = 1;
    int rc = y3b_engine_create(&f->grid, 1, &ec, &f->e);
    if (rc != Y3B_OK) throw Failure{std::string("y3b_engine_create: ") + y3b_last_error()};
    f->n_hm = ec.n_hm;
    f->n_hz = ec.n_hz;
    f->n_dist = ec.n_dist;
    f->plob_z = pz;
    f->plob_coef = pc;
    f->packed.assign(y3b_engine_table_stride(f->e), 0.0);
  }
  size_t off[7];
  y3b_engine_table_offsets(f->e, off);
  std::copy(mh.begin(), mh.end(), f->packed.begin() + off[0]);
  std::copy(hz.begin(), hz.end(), f->packed.begin() + off[1]);
  std::copy(dn.begin(), dn.end(), f->packed.begin() + off[2]);
  std::copy(dz.begin(), dz.end(), f->packed.begin() + off[3]);
  std::copy(da.begin(), da.end(), f->packed.begin() + off[4]);
  std::vector<double> counts(y3b_engine_n_bins(f->e));
  int rc = y3b_engine_eval(f->e, f->precision, 1, &pt, f->packed.data(), counts.data(), nullptr);
  // A MOR scatter too narrow for the mixed form's factorised Gaussian: this
  // point goes through the FP64 form of the same quadrature instead.
  if (rc == Y3B_ERR_RANGE)
    rc = y3b_engine_eval(f->e, Y3B_FP64, 1, &pt, f->packed.data(), counts.data(), nullptr);
  if (rc != Y3B_OK) throw Failure{std::string("y3b_engine_eval: ") + y3b_last_error()};
  vals.resize(m->bins.size());
  for (size_t k = 0; k < m->bins.size(); ++k) vals[k] = counts[m->bins[k]];
  if (f->write_s) {
    const y3b_selfunc_config& s0 = f->scfg;
    y3b_selfunc_config s = s0;
    s.lam_min = f->lam_min.data();
    s.lam_max = f->lam_max.data();
    s.zob_min = f->zob_min.data();
    s.zob_max = f->zob_max.data();
    s.sigma_z = f->sigma_z.data();
    y3b_mor mor{Y3B_MOR_LOGNORMAL,
                {pt.A, pt.B, pt.C, pt.sigma, pt.Mpiv, f->grid.lam_t_lo, f->grid.lam_t_hi, 0.0}};
    y3b_plob pl{(int)pz.size(), pz.data(), pc.data()};
    std::vector<double> lnm(s.n_lnm), z(s.n_z), S((size_t)s.n_bins * s.n_z * s.n_lnm);
    rc = y3b_sel_function(&s, &mor, &pl, lnm.data(), z.data(), S.data());
    if (rc != Y3B_OK) throw Failure{std::string("y3b_sel_function: ") + y3b_last_error()};
    const int e3[3] = {s.n_bins, s.n_z, s.n_lnm};
    if (c_datablock_put_double_array_1d(block, "sel_function", "lnM", lnm.data(), s.n_lnm) !=
            DBS_SUCCESS ||
        c_datablock_put_double_array_1d(block, "sel_function", "z", z.data(), s.n_z) !=
            DBS_SUCCESS ||
        c_datablock_put_double_array(block, "sel_function", "S_stack", S.data(), 3, e3) !=
            DBS_SUCCESS)
      throw Failure{"cannot write sel_function/{lnM, z, S_stack}"};
  }
}
#endif

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
    const std::string eng = opt_string(options, "engine", "selgl");
    if (eng != "selgl" && eng != "fused")
      throw Failure{"engine must be 'selgl' or 'fused', got '" + eng + "'"};
    if (eng == "fused") {
#if Y3B_MODULE_SHEAR
      throw Failure{"engine = fused is available for the number-count modules"};
#else
      setup_fused(options, m);
      return m;
#endif
    }
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
    std::vector<double> vals;
    if (m->fused) {
      execute_fused(block, m, vals);
      if (c_datablock_put_double_array_1d(block, kOutput, "vals", vals.data(),
                                          (int)vals.size()) != DBS_SUCCESS)
        throw Failure{std::string("cannot write ") + kOutput + "/vals"};
      return DBS_SUCCESS;
    }
    read_sample(block, s, false);
    int rc = build(m, s, false);
    if (rc != Y3B_OK) throw Failure{y3b_last_error()};
    vals.resize(m->bins.size());
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
