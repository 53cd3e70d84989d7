"""The CosmoSIS module objects driven through setup / execute / cleanup on a
standalone DataBlock, against the library and the oracle."""
import os

import numpy as np
import pytest

import oracle as O
from y3_cluster_cpp_b200 import engine as E
from y3_cluster_cpp_b200 import sel_function as SF
from y3_cluster_cpp_b200 import synthetic
from y3_cluster_cpp_b200.cosmosis import DataBlock, Module

pytestmark = pytest.mark.gpu

BINS = dict(lam_min=[20.0, 30.0, 45.0, 60.0] * 3, lam_max=[30.0, 45.0, 60.0, 200.0] * 3,
            zob_min=[0.20] * 4 + [0.35] * 4 + [0.50] * 4,
            zob_max=[0.35] * 4 + [0.50] * 4 + [0.65] * 4, sigma_z=[0.03] * 12)


class Options:
    """The CosmoSIS python options API used by sel_function.setup."""

    def __init__(self, d):
        self.d = d

    def get_double_array_1d(self, s, k):
        v = self.d[k]
        if np.ndim(v) == 0:
            raise TypeError(k)
        return np.asarray(v, float)

    def get_int_array_1d(self, s, k):
        return np.asarray(self.d[k], int)

    def get_double(self, s, k):
        return float(self.d[k])

    def get_int(self, s, k):
        v = self.d[k]
        if not isinstance(v, int):
            raise TypeError(k)
        return v

    def get_string(self, s, k):
        return str(self.d[k])


def _sample_block(p, mor="hod"):
    b = DataBlock()
    b["cosmological_parameters", "omega_M"] = p.om
    b["cosmological_parameters", "omega_lambda"] = 1 - p.om
    b["cosmological_parameters", "omega_k"] = 0.0
    b["cosmological_parameters", "h0"] = p.h0
    b["cosmological_parameters", "omega_nu"] = 0.0
    b["cluster_abundance", "hmf_s"] = 0.0
    b["cluster_abundance", "hmf_q"] = 1.0
    t = p.tables
    b["mass_function", "m_h"] = t["hmf_m_h"]
    b["mass_function", "z"] = t["hmf_z"]
    b["mass_function", "dndlnmh"] = t["dndlnmh"]
    b["distances", "z"] = t["dist_z"]
    b["distances", "d_a"] = t["dist_da"]
    b["average_sigma_crit_inv", "zlense"] = t["sci_z"]
    b["average_sigma_crit_inv", "sci_average"] = t["sci_val"]
    for k, v in dict(log10_Mmin=11.4, log10_M1=12.7, alpha=0.86, epsilon=0.0,
                     sigma_lambda=0.18).items():
        b["cluster_mor", k] = v
    return b


def test_pipeline_sel_function_then_numcounts(gpu):
    """sel_function (python module) -> NumCountsSel.so on one DataBlock, as
    the des_y3.ini pipeline runs them; compared with the oracle chain."""
    p = synthetic.fiducial()
    opts = dict(BINS, zt_low=0.05, zt_high=0.8, lnm_low=29.9336, lnm_high=36.8414,
                n_lnm=96, n_z_shared=32, N_q=24)
    cfg = SF.setup(Options(opts))
    block = _sample_block(p)
    assert SF.execute(block, cfg) == 0
    S = block["sel_function", "S_stack"]
    assert S.shape == (12, 32, 96)

    m = Module("NumCountsSel")
    o = DataBlock()
    o["NumCountsSel", "bin_index"] = np.arange(12)
    o["NumCountsSel", "zt_low"] = 0.1
    o["NumCountsSel", "zt_high"] = 0.8
    o["NumCountsSel", "lnm_low"] = 29.9336
    o["NumCountsSel", "lnm_high"] = 35.69
    o["NumCountsSel", "n_lnm"] = 64
    o["NumCountsSel", "n_z"] = 32
    assert m.setup(o)
    assert m.execute(block) == 0
    vals = block["numcountssel", "vals"]
    sel = (block["sel_function", "lnM"], block["sel_function", "z"], S)
    _, norm, _, _ = O.selgl_weights(64, 32, 0.1, 0.8, 29.9336, 35.69, O.cosmo(p.om, p.h0),
                                    p.tables, sel)
    np.testing.assert_allclose(vals, norm, rtol=1e-8)
    assert m.cleanup() == 0


def test_shear_module_and_fast_mass_aliases(gpu):
    p = synthetic.fiducial()
    pz, pc = synthetic.plob_baseline()
    cfg = dict(BINS, zt_low=0.05, zt_high=0.8, lnm_low=29.9336, lnm_high=36.8414,
               n_lnm=64, n_z=32, n_q=16)
    mor = [11.4, 12.7, 0.86, 0.0, 0.18, 0.45]
    lnm, z, S = E.sel_function(cfg, O.MOR_HOD, mor, pz, pc)
    block = _sample_block(p)
    block["sel_function", "lnM"] = lnm
    block["sel_function", "z"] = z
    block["sel_function", "S_stack"] = S
    R = np.logspace(-2, 1.7, 40)
    lnM = np.linspace(29.9, 36.9, 30)
    block["haloModel", "r_sigma"] = R
    block["haloModel", "lnM"] = lnM
    block["haloModel", "dSigma_nfw"] = np.outer(np.exp(0.1 * (lnM - 32)), 1.0 / (R + 0.1))
    out = {}
    for name, sec in (("Shear1hMisSel", "shear1hmissel"), ("Shear1hFastMass", "shear1h_fast_mass")):
        m = Module(name)
        o = DataBlock()
        o[name, "bin_index"] = np.arange(12)
        o[name, "r_perp"] = np.array([0.2, 1.0, 5.0])
        for k, v in dict(zt_low=0.1, zt_high=0.8, lnm_low=29.9336, lnm_high=36.73).items():
            o[name, k] = v
        o[name, "n_lnm"] = 32
        o[name, "n_z"] = 32
        assert m.setup(o)
        assert m.execute(block) == 0
        out[name] = block[sec, "vals"]
        assert out[name].shape == (36,)
        m.cleanup()
    np.testing.assert_array_equal(out["Shear1hMisSel"], out["Shear1hFastMass"])
    h = E.SelGL(32, 32, 0.1, 0.8, 29.9336, 36.73)
    h.build(E.cosmo(p.om, p.h0), p.tables, (lnm, z, S), include_sci=True)
    halo = dict(r_sigma=R, lnM=lnM, dSigma_nfw=block["haloModel", "dSigma_nfw"])
    direct = h.shear(np.repeat(np.arange(12), 3), np.tile([0.2, 1.0, 5.0], 12), halo)
    np.testing.assert_allclose(out["Shear1hMisSel"], direct, rtol=1e-12)


def test_module_errors_return_nonzero_status(gpu):
    m = Module("NumCountsSel")
    o = DataBlock()
    o["NumCountsSel", "bin_index"] = np.arange(12)
    assert not m.setup(o)            # missing zt_low etc. -> NULL, not an exception
    for k, v in dict(zt_low=0.1, zt_high=0.8, lnm_low=29.9, lnm_high=35.7).items():
        o["NumCountsSel", k] = v
    assert m.setup(o)
    empty = DataBlock()
    assert m.execute(empty) != 0     # missing sample sections -> non-zero status
    m.cleanup()


# ---- parity with the reference's own C++ modules (golden vectors written by
# the compiled reference, tests/golden/make_golden.py) ------------------------

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _golden():
    return np.load(os.path.join(GOLD, "selgl_ref.npz"))


def _golden_block(g, mor):
    t = {k[2:]: g[k] for k in g.files if k.startswith("t_")}
    s = np.load(os.path.join(GOLD, f"sel_function_{mor}.npz"))
    b = DataBlock()
    om = float(g["omega_m"])
    b["cosmological_parameters", "omega_M"] = om
    b["cosmological_parameters", "omega_lambda"] = 1 - om
    b["cosmological_parameters", "omega_k"] = 0.0
    b["cosmological_parameters", "h0"] = float(g["h0"])
    b["cosmological_parameters", "omega_nu"] = 0.0
    b["cluster_abundance", "hmf_s"] = 0.0
    b["cluster_abundance", "hmf_q"] = 1.0
    b["mass_function", "m_h"] = t["hmf_m_h"]
    b["mass_function", "z"] = t["hmf_z"]
    b["mass_function", "dndlnmh"] = t["dndlnmh"]
    b["distances", "z"] = t["dist_z"]
    b["distances", "d_a"] = t["dist_da"]
    b["average_sigma_crit_inv", "zlense"] = t["sci_z"]
    b["average_sigma_crit_inv", "sci_average"] = t["sci_val"]
    b["sel_function", "lnM"] = s["lnM"]
    b["sel_function", "z"] = s["z"]
    b["sel_function", "S_stack"] = s["S_stack"]
    b["haloModel", "r_sigma"] = g["halo_r_sigma"]
    b["haloModel", "lnM"] = g["halo_lnM"]
    b["haloModel", "dSigma_nfw"] = g["halo_dSigma_nfw"]
    return b


def _module_options(g, label, name):
    o = DataBlock()
    for k in ("zt_low", "zt_high", "lnm_low", "lnm_high"):
        o[label, k] = float(g[f"cfg_{name}_{k}"])
    for k in ("n_lnm", "n_z"):
        if f"cfg_{name}_{k}" in g.files:
            o[label, k] = int(g[f"cfg_{name}_{k}"])
    o[label, "bin_index"] = np.arange(12)
    return o


@pytest.mark.parametrize("name", ["a", "b"])
@pytest.mark.parametrize("mor", ["hod", "lognormal"])
def test_numcounts_module_matches_compiled_reference(gpu, name, mor):
    """NumCountsSel.so (setup/execute on a DataBlock) against numcountssel/vals
    of the reference's NumCountsSelGL on the same inputs: <= 1e-8 relative."""
    g = _golden()
    block = _golden_block(g, mor)
    m = Module("NumCountsSel")
    assert m.setup(_module_options(g, "NumCountsSel", name))
    assert m.execute(block) == 0
    vals = block["numcountssel", "vals"]
    m.cleanup()
    np.testing.assert_allclose(vals, g[f"counts_{name}_{mor}"], rtol=1e-8, atol=0)


def test_selgl_weights_with_sigma_crit_match_compiled_reference(gpu):
    g = _golden()
    t = {k[2:]: g[k] for k in g.files if k.startswith("t_")}
    s = np.load(os.path.join(GOLD, "sel_function_lognormal.npz"))
    h = E.SelGL(int(g["cfg_a_n_lnm"]), int(g["cfg_a_n_z"]), float(g["cfg_a_zt_low"]),
                float(g["cfg_a_zt_high"]), float(g["cfg_a_lnm_low"]), float(g["cfg_a_lnm_high"]))
    h.build(E.cosmo(float(g["omega_m"]), float(g["h0"])), t, (s["lnM"], s["z"], s["S_stack"]),
            include_sci=True)
    w = h.weights()
    h.close()
    np.testing.assert_allclose(w["W"], g["wsci_W"], rtol=1e-8,
                               atol=1e-12 * np.max(g["wsci_W"]))
    np.testing.assert_allclose(w["norm"], g["wsci_norm"], rtol=1e-8, atol=0)
    np.testing.assert_allclose(w["lnm_eff"], g["wsci_eff"], rtol=1e-10, atol=0)
    np.testing.assert_allclose(w["mu2"], g["wsci_mu2"], rtol=1e-8, atol=0)


@pytest.mark.parametrize("case", [("shear_exact_cfg2", "a", "lognormal", "exact", 0.2),
                                  ("shear_idea2_default", "b", "hod", "idea2", None),
                                  ("shear_exact_default_b", "b", "hod", None, None)])
def test_shear_module_table_matches_compiled_reference(gpu, tmp_path, monkeypatch, case):
    """Shear1hMisSel.so reading the miscentring table from
    $Y3_CLUSTER_CPP_DIR/data/nfw_off_center/ (as NFW_DSIGMA_MIS does) against
    shear1hmissel/vals of the reference's Shear1hMisSelGL: <= 1e-8."""
    key, name, mor, method, f_mis = case
    g = _golden()
    d = tmp_path / "data" / "nfw_off_center"
    d.mkdir(parents=True)
    stem = str(d / "table_1000_1e-03_5e+03_")
    np.savetxt(stem + "gamma_logx.txt", g["mis_logx"], fmt="%.17g")
    np.savetxt(stem + "gamma_logxmis.txt", g["mis_logxmis"], fmt="%.17g")
    np.savetxt(stem + "log_deltasigma_gamma.txt", np.ravel(g["mis_log_tab"]), fmt="%.17g")
    monkeypatch.setenv("Y3_CLUSTER_CPP_DIR", str(tmp_path))
    block = _golden_block(g, mor)
    if f_mis is not None:
        block["miscentering", "f_mis"] = f_mis
        block["miscentering", "tau_mis"] = 0.17
    o = _module_options(g, "Shear1hMisSel", name)
    o["Shear1hMisSel", "r_perp"] = g["R"]
    o["Shear1hMisSel", "mis_profile"] = "table"
    if method:
        o["Shear1hMisSel", "method"] = method
    m = Module("Shear1hMisSel")
    assert m.setup(o)
    assert m.execute(block) == 0
    vals = block["shear1hmissel", "vals"]
    m.cleanup()
    ref = g[key]
    np.testing.assert_allclose(vals, ref, rtol=1e-8, atol=1e-12 * np.max(np.abs(ref)))


def test_shear_module_table_mode_requires_files(gpu, tmp_path, monkeypatch):
    monkeypatch.setenv("Y3_CLUSTER_CPP_DIR", str(tmp_path))
    g = _golden()
    o = _module_options(g, "Shear1hMisSel", "a")
    o["Shear1hMisSel", "r_perp"] = g["R"]
    o["Shear1hMisSel", "mis_profile"] = "table"
    assert not Module("Shear1hMisSel").setup(o)   # missing files -> NULL, no throw


def test_sigma_crit_inv_matches_reference_python(gpu):
    s = np.load(os.path.join(GOLD, "sigma_crit_inv.npz"))
    out = E.sigma_crit_inv(s["zl"], s["zs"], s["pz"], float(s["delta_z"]), float(s["h0"]),
                           s["dist_z"], s["dist_da"])
    np.testing.assert_allclose(out, s["sci"], rtol=1e-10, atol=1e-10 * np.max(s["sci"]))


# ---- engine = fused: the whole integral behind the module ABI --------------

def _fused_options(label, g, precision, sigma_z, sz0, bins=None, **extra):
    o = DataBlock()
    o[label, "engine"] = "fused"
    o[label, "precision"] = precision
    o[label, "bin_index"] = np.arange(12) if bins is None else np.asarray(bins)
    le, ze = g["lam_edges"], g["zob_edges"]
    o[label, "lam_min"] = np.tile(le[:-1], 3)
    o[label, "lam_max"] = np.tile(le[1:], 3)
    o[label, "zob_min"] = np.repeat(ze[:-1], 4)
    o[label, "zob_max"] = np.repeat(ze[1:], 4)
    o[label, "sigma_z"] = np.repeat(sigma_z, 4)
    o[label, "sz0"] = sz0
    for k, v in dict(zt_low=g["zt_lo"], zt_high=g["zt_hi"], lnm_low=g["lnm_lo"],
                     lnm_high=g["lnm_hi"]).items():
        o[label, k] = float(v)
    o[label, "n_lnm"], o[label, "n_z"], o[label, "n_lt"] = g["n_m"], g["n_z"], g["n_t"]
    o[label, "n_lo"], o[label, "n_zo"] = g["n_o"], g["n_zo"]
    for k, v in extra.items():
        o[label, k] = v
    return o


def _fused_sample(p, pz, pc):
    b = _sample_block(p)
    for k, v in dict(A=p.A, B=p.B, C=p.C, sigma_intr=p.sigma, M_pivot=p.Mpiv).items():
        b["cluster_mor", k] = v
    b["plob_ltr_params", "z"] = pz
    from y3_cluster_cpp_b200 import prj_params
    for k, row in zip(prj_params.COEFF_NAMES, pc):
        b["plob_ltr_params", k] = row
    return b


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("mixed", 1e-4)])
@pytest.mark.parametrize("photoz", ["baseline", "reference"])
def test_fused_numcounts_module_matches_oracle(gpu, precision, tol, photoz):
    """NumCountsFastMass.so with engine = fused, driven through setup /
    execute / cleanup on a DataBlock, against the FP64 direct quadrature
    (oracle) on the same nodes: the configs' photo-z sigma = 0.01 (1 + z) and
    sel_function's constant per-bin sigma_z."""
    g = synthetic.grid(1)
    if photoz == "baseline":
        sz, sz0 = np.zeros(3), 0.01
    else:
        sz, sz0 = np.full(3, 0.03), 0.0
    g["sz0"], g["sz_bin"] = sz0, sz
    p = synthetic.fiducial()
    pz, pc = synthetic.plob_baseline()
    ref, _, _ = O.direct_eval(g, pz, pc, p.mor, O.cosmo(p.om, p.h0), p.tables)
    bins = [3, 0, 11, 5]
    m = Module("NumCountsFastMass")
    assert m.setup(_fused_options("NumCountsFastMass", g, precision, sz, sz0, bins=bins))
    block = _fused_sample(p, pz, pc)
    for _ in range(2):                       # second call reuses the engine
        assert m.execute(block) == 0
        vals = block["numcounts_fast_mass", "vals"]
        np.testing.assert_allclose(vals, ref[bins], rtol=tol, atol=0)
    m.cleanup()


def test_fused_module_writes_s_stack_and_defaults(gpu):
    """write_s_stack = T also publishes sel_function/{lnM, z, S_stack} (the
    lognormal MOR, as y3b_sel_function); without plob_ltr_params the frozen
    projection table is used, as sel_function.py does."""
    g = synthetic.grid(1)
    p = synthetic.fiducial()
    from y3_cluster_cpp_b200 import prj_params
    pz, pc = prj_params.default_table()
    m = Module("NumCountsFastMass")
    assert m.setup(_fused_options("NumCountsFastMass", g, "fp64", np.full(3, 0.03), 0.0,
                                  write_s_stack=1))
    block = _sample_block(p)
    for k, v in dict(A=p.A, B=p.B, C=p.C, sigma_intr=p.sigma).items():
        block["cluster_mor", k] = v
    assert m.execute(block) == 0
    S = block["sel_function", "S_stack"]
    assert S.shape == (12, 20, 40)
    g2 = dict(g, sz0=0.0, sz_bin=np.full(3, 0.03))
    ref, _, _ = O.direct_eval(g2, pz, pc, p.mor, O.cosmo(p.om, p.h0), p.tables)
    np.testing.assert_allclose(block["numcounts_fast_mass", "vals"], ref, rtol=1e-8)
    cfg = dict(lam_min=np.tile(g["lam_edges"][:-1], 3), lam_max=np.tile(g["lam_edges"][1:], 3),
               zob_min=np.repeat(g["zob_edges"][:-1], 4),
               zob_max=np.repeat(g["zob_edges"][1:], 4), sigma_z=np.full(12, 0.03),
               zt_low=g["zt_lo"], zt_high=g["zt_hi"], lnm_low=g["lnm_lo"],
               lnm_high=g["lnm_hi"], n_lnm=40, n_z=20, n_q=32)
    _, _, S2 = E.sel_function(cfg, O.MOR_LOGNORMAL,
                              [p.A, p.B, p.C, p.sigma, p.Mpiv, 1.0, 1000.0], pz, pc)
    np.testing.assert_array_equal(S, S2)
    m.cleanup()


def test_fused_module_narrow_scatter_falls_back_to_fp64(gpu):
    """sigma_int = 0.05 at the 4x grid leaves the mixed form's exponent range;
    the fused module evaluates such a point in FP64 and still returns it."""
    g = synthetic.grid(4)
    g["sz0"], g["sz_bin"] = 0.01, np.zeros(3)
    p = synthetic.fiducial()
    p.sigma = 0.05
    pz, pc = synthetic.plob_baseline()
    ref, _, _ = O.direct_eval(g, pz, pc, p.mor, O.cosmo(p.om, p.h0), p.tables)
    m = Module("NumCountsFastMass")
    assert m.setup(_fused_options("NumCountsFastMass", g, "mixed", np.zeros(3), 0.01))
    block = _fused_sample(p, pz, pc)
    assert m.execute(block) == 0
    np.testing.assert_allclose(block["numcounts_fast_mass", "vals"], ref, rtol=1e-8)
    m.cleanup()


# ---- Gaussian likelihood (y3_buzzard/likelihood_cp.py) ------------------------

class _Opt(dict):
    def __getitem__(self, key):
        return dict.__getitem__(self, key[1])

    def get_bool(self, section, key, default=False):
        return bool(self.get(key, default))


@pytest.mark.parametrize("form", ["diag", "dense"])
@pytest.mark.parametrize("space", ["lin", "log"])
def test_likelihood_module_matches_reference(gpu, tmp_path, form, space):
    """The likelihood module (setup/execute on a block, evaluated on the GPU)
    against likelihoods/likelihoods_like of the reference's likelihood_cp.py
    on the golden mock data vector and theory blocks."""
    from y3_cluster_cpp_b200 import likelihood_cp as LK
    g = np.load(os.path.join(GOLD, "likelihood_ref.npz"))
    fname = str(tmp_path / "mock.npz")
    np.savez(fname, data_NC=g["data_nc"], invcov_NC=g[f"{form}_nc"], data_Shear=g["data_sh"],
             invcov_Shear=g[f"{form}_sh"])
    cfg = LK.setup(_Opt(filename=fname, log_space=space == "log"))
    ref = g[f"logL_{form}_{space}"]
    for t in range(len(ref)):
        block = {("numcountssel", "vals"): g["thr_nc"][t],
                 ("shear1hmissel", "vals"): g["thr_s1h"][t].ravel(),
                 ("shear_prj", "vals"): g["thr_prj"][t].ravel()}
        assert LK.execute(block, cfg) == 0
        assert block["likelihoods", "likelihoods_like"] == pytest.approx(ref[t], rel=1e-10,
                                                                          abs=1e-8)
