"""Pins the oracle's SelGLCore / Shear1hMisSelGL / Sigma_crit^-1
restatements to the reference's own code: golden vectors written by the
reference's C++ module classes (compiled from the reference's sources against
the shims of oracle/ref_shim/) and by the reference's
average_sigma_crit_inv.py (tests/golden/make_golden.py), and, where the
compiled reference library is present, the library itself on more inputs."""
import os

import numpy as np
import pytest

import oracle as O
from oracle import ref as R

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def g():
    return np.load(os.path.join(GOLD, "selgl_ref.npz"))


def tables(g):
    return {k[2:]: g[k] for k in g.files if k.startswith("t_")}


def cfg(g, name):
    c = dict(zt_low=float(g[f"cfg_{name}_zt_low"]), zt_high=float(g[f"cfg_{name}_zt_high"]),
             lnm_low=float(g[f"cfg_{name}_lnm_low"]), lnm_high=float(g[f"cfg_{name}_lnm_high"]),
             n_lnm=96, n_z=64)
    for k in ("n_lnm", "n_z"):
        if f"cfg_{name}_{k}" in g.files:
            c[k] = int(g[f"cfg_{name}_{k}"])
    return c


def sel(mor):
    s = np.load(os.path.join(GOLD, f"sel_function_{mor}.npz"))
    return s["lnM"], s["z"], s["S_stack"]


def oracle_weights(g, name, mor, with_sci):
    c = cfg(g, name)
    t = tables(g)
    sci = (t["sci_z"], t["sci_val"]) if with_sci else None
    cz = O.cosmo(float(g["omega_m"]), float(g["h0"]))
    return O.selgl_weights(c["n_lnm"], c["n_z"], c["zt_low"], c["zt_high"], c["lnm_low"],
                           c["lnm_high"], cz, t, sel(mor), sci)


@pytest.mark.parametrize("name", ["a", "b"])
@pytest.mark.parametrize("mor", ["hod", "lognormal"])
def test_numcounts_oracle_matches_compiled_reference(g, name, mor):
    _, norm, _, _ = oracle_weights(g, name, mor, False)
    ref = g[f"counts_{name}_{mor}"]
    assert np.all(ref > 0)
    np.testing.assert_allclose(norm, ref, rtol=1e-12, atol=0)


def test_selgl_weights_with_sigma_crit_match_compiled_reference(g):
    W, norm, eff, mu2 = oracle_weights(g, "a", "lognormal", True)
    np.testing.assert_allclose(W, g["wsci_W"], rtol=1e-12, atol=1e-12 * np.max(g["wsci_W"]))
    np.testing.assert_allclose(norm, g["wsci_norm"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(eff, g["wsci_eff"], rtol=1e-13, atol=0)
    np.testing.assert_allclose(mu2, g["wsci_mu2"], rtol=1e-10, atol=0)


def _shear_oracle(g, name, mor, method, f_mis, tau_mis):
    c = cfg(g, name)
    W, norm, eff, mu2 = oracle_weights(g, name, mor, True)
    lx, lw = O.gl_nodes(c["lnm_low"], c["lnm_high"], c["n_lnm"])
    mis = (g["mis_logx"], g["mis_logxmis"], g["mis_log_tab"])
    return O.shear1h_mis_tab(lx, lw, W, norm, eff, mu2, method, 0.15, g["R"], f_mis, tau_mis,
                             [25.0, 37.5, 52.5, 130.0], float(g["omega_m"]), 4.0,
                             g["halo_r_sigma"], g["halo_lnM"], g["halo_dSigma_nfw"], mis)


@pytest.mark.parametrize("case", [("shear_exact_cfg2", "a", "lognormal", 0, 0.2, 0.17),
                                  ("shear_idea2_default", "b", "hod", 1, 0.22, 0.17),
                                  ("shear_exact_default_b", "b", "hod", 0, 0.22, 0.17)])
def test_shear1h_oracle_matches_compiled_reference(g, case):
    key, name, mor, method, f, tau = case
    out = _shear_oracle(g, name, mor, method, f, tau).ravel()
    ref = g[key]
    assert np.all(np.isfinite(ref)) and np.max(np.abs(ref)) > 0
    np.testing.assert_allclose(out, ref, rtol=1e-12, atol=1e-12 * np.max(np.abs(ref)))


def test_sigma_crit_inv_matches_reference_python():
    s = np.load(os.path.join(GOLD, "sigma_crit_inv.npz"))
    out = O.sigma_crit_inv(s["zl"], s["zs"], s["pz"], float(s["delta_z"]), float(s["h0"]),
                           s["dist_z"], s["dist_da"])
    np.testing.assert_allclose(out, s["sci"], rtol=1e-10, atol=1e-10 * np.max(s["sci"]))


@pytest.mark.skipif(not R.available(), reason="compiled reference (make -C oracle ref) absent")
def test_oracle_matches_compiled_reference_on_walkers(g):
    """The live reference library on walkers of the batched prior (their own
    cosmologies and tables): counts and weights with Sigma_crit^-1."""
    from y3_cluster_cpp_b200 import synthetic
    for p in synthetic.walkers(6, seed=3, densities=(1,)):
        cosmo = dict(omega_m=p.om, omega_nu=0.0, omega_lambda=1 - p.om, omega_k=0.0,
                     h0=p.h0, hmf_s=0.0, hmf_q=1.0)
        t = p.tables
        for mor in ("hod", "lognormal"):
            c = cfg(g, "a")
            ref = R.numcounts(c, cosmo, t, sel(mor))
            _, norm, _, _ = O.selgl_weights(c["n_lnm"], c["n_z"], c["zt_low"], c["zt_high"],
                                            c["lnm_low"], c["lnm_high"], O.cosmo(p.om, p.h0),
                                            t, sel(mor))
            np.testing.assert_allclose(norm, ref, rtol=1e-12, atol=0)


def test_direct_quadrature_converges_to_reference_chain():
    """O2 (the direct nested-GL quadrature every engine test compares with)
    against the reference chain (sel_function.py tabulation of S_stack, then
    SelGLCore's interpolation and z/lnM contraction; both restatements are
    pinned above and in test_oracle_golden.py to the reference's own code) on
    the same integral: the lognormal MOR of the configs, the constant-in-z
    projection coefficients and sel_function's photo-z model (constant
    sigma_z = 0.03 per bin).  The chain's only approximation is the bilinear
    interpolation of its S table, so the gap must shrink as O(h^2) when the
    table is refined, to a few 1e-5 at 768 x 256 x 64 cells."""
    from y3_cluster_cpp_b200 import synthetic
    g = synthetic.grid(4)
    g["sz0"], g["sz_bin"] = 0.0, np.full(3, 0.03)
    p = synthetic.fiducial()
    pz, pc = synthetic.plob_baseline()
    c = O.cosmo(p.om, p.h0)
    counts, _, _ = O.direct_eval(g, pz, pc, p.mor, c, p.tables)
    mor = [p.A, p.B, p.C, p.sigma, p.Mpiv, g["lam_t_lo"], g["lam_t_hi"]]
    gaps = []
    for n_lnm, n_z, n_q in ((192, 64, 32), (768, 256, 64)):
        cfgs = dict(lam_min=np.tile(g["lam_edges"][:-1], 3),
                    lam_max=np.tile(g["lam_edges"][1:], 3),
                    zob_min=np.repeat(g["zob_edges"][:-1], 4),
                    zob_max=np.repeat(g["zob_edges"][1:], 4), sigma_z=np.full(12, 0.03),
                    zt_low=g["zt_lo"], zt_high=g["zt_hi"], lnm_low=g["lnm_lo"],
                    lnm_high=g["lnm_hi"], n_lnm=n_lnm, n_z=n_z, n_q=n_q)
        sel = O.sel_function(cfgs, O.MOR_LOGNORMAL, mor, pz, pc)
        _, norm, _, _ = O.selgl_weights(g["n_m"], g["n_z"], g["zt_lo"], g["zt_hi"],
                                        g["lnm_lo"], g["lnm_hi"], c, p.tables, sel)
        gaps.append(np.max(np.abs(norm / counts - 1)))
    assert gaps[1] < 3e-5, gaps
    assert gaps[1] < gaps[0] / 8, gaps


@pytest.mark.parametrize("form", ["diag", "dense"])
@pytest.mark.parametrize("space", ["lin", "log"])
def test_loglike_matches_reference_likelihood(form, space):
    """y3o_loglike against likelihoods/likelihoods_like of the reference's
    y3_buzzard/likelihood_cp.py (setup + execute) on the golden mock data
    vector: counts + (1-halo shear / counts + projection shear)."""
    g = np.load(os.path.join(GOLD, "likelihood_ref.npz"))
    log_space = space == "log"
    dn, ds = g["data_nc"], g["data_sh"]
    icn, ics = g[f"{form}_nc"], g[f"{form}_sh"]
    if log_space:   # what setup() stores (likelihood_cp.py:79-92, 113-118)
        icn = icn * (np.outer(dn, dn) if icn.ndim == 2 else dn * dn)
        ics = ics * (np.outer(ds, ds) if ics.ndim == 2 else ds * ds)
        dn, ds = np.log(dn), np.log(ds)
    ref = g[f"logL_{form}_{space}"]
    for t in range(len(ref)):
        v = O.loglike(g["thr_nc"][t], g["thr_s1h"][t], g["thr_prj"][t], log_space,
                      dn, icn, ds, ics)
        assert v == pytest.approx(ref[t], rel=1e-12, abs=1e-9)


def test_bsel_golden_reproduced_by_compiled_reference():
    """The selection-bias fixture (P_operator of p_operator_t.hh) comes back
    bit for bit from the compiled reference library, where it is present."""
    if not R.available():
        pytest.skip("compiled reference library not present")
    b = np.load(os.path.join(GOLD, "bsel_ref.npz"))

    def sub(pre):
        return {k[len(pre):]: (float(b[k]) if b[k].ndim == 0 else b[k]) for k in b.files
                if k.startswith(pre)}

    om, h0 = float(b["omega_m"]), float(b["h0"])
    cosmo = dict(omega_m=om, omega_nu=0.0, omega_lambda=1.0 - om, omega_k=0.0, h0=h0,
                 hmf_s=0.0, hmf_q=1.0)
    t, prj = sub("t_"), sub("prj_")
    out = R.bsel_marg(sub("cfg_"), cosmo, t, prj, sub("hod_"), sub("gp_"))
    np.testing.assert_array_equal(out, b["vals"])
    cfg2 = {k: (int(v) if k.startswith("n_") else v) for k, v in sub("cfg2_").items()}
    out2 = R.bsel_marg(cfg2, cosmo, t, prj, sub("hod2_"), sub("gp2_"))
    np.testing.assert_array_equal(out2, b["vals2"][1])
