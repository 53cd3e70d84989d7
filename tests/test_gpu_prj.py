"""The frozen-physics projection shear (ShearPrjFrozenPhysics) on the GPU
against the reference's own compiled class: the golden vectors of
tests/golden/prj_ref.npz (written by tests/golden/make_golden.py) and, where
the compiled reference library is present, the library itself on further
walkers.  FP64 throughout; tolerance 1e-8 relative (observed ~1e-13)."""
import os

import numpy as np
import pytest

from y3_cluster_cpp_b200 import engine as E
from y3_cluster_cpp_b200 import synthetic

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-8


def _golden():
    return np.load(os.path.join(GOLD, "prj_ref.npz"))


def _inputs(g):
    t = {k[2:]: g[k] for k in g.files if k.startswith("t_")}
    prj = {k[4:]: g[k] for k in g.files if k.startswith("prj_")}
    grid = {k[3:]: g[k] for k in g.files if k.startswith("gp_")}
    grid["lambda_bin"] = grid["lambda_bin"].astype(int)
    cfg = {k[4:]: float(g[k]) for k in g.files if k.startswith("cfg_")}
    return t, prj, grid, cfg


def _check(out, ref):
    scale = np.max(np.abs(ref), axis=0)
    np.testing.assert_allclose(out, ref, rtol=TOL, atol=TOL * 1e-3 * np.max(scale))


@pytest.mark.parametrize("variant", ["default", "no_omega"])
def test_prj_matches_compiled_reference_golden(gpu, variant):
    g = _golden()
    t, prj, grid, cfg = _inputs(g)
    kw = dict(cfg)
    if variant == "no_omega":
        kw.update(include_omega_z=False, n_lnm=16, n_per_seg=8)
    h = E.PrjShear(grid, **kw)
    h.set_mis_table(g["single_logx"], g["single_logxmis"], g["single_log_tab"])
    out = h.eval(E.cosmo(float(g["omega_m"]), float(g["h0"])), t, prj)
    ref = g["vals" if variant == "default" else "vals_no_omega"]
    assert np.all(np.isfinite(out)) and np.max(np.abs(ref[:, 0])) > 0
    _check(out, ref)
    # a second sample on the same handle
    out2 = h.eval(E.cosmo(float(g["omega_m"]), float(g["h0"])), t, prj)
    np.testing.assert_array_equal(out, out2)
    h.close()


def test_single_offset_profile_matches_oracle(gpu):
    """The single-kernel miscentred profile that the projection shear
    integrates when no table is given (y3b_nfw_mis, which = 2: the same device
    function) against the oracle's FP64 restatement, across x < x_mis (where
    it is negative), x ~ x_mis and x > x_mis."""
    import oracle as O
    L = O.lib()
    rng = np.random.default_rng(5)
    n = 400
    lnM = rng.uniform(30.0, 35.0, n)
    conc, rho = 4.0, 2.77533742639e11 * 0.3
    rs = np.array([L.y3o_nfw_rs(m, conc, rho) for m in lnM])
    x = np.exp(rng.uniform(np.log(1e-3), np.log(50.0), n))
    xm = np.exp(rng.uniform(np.log(1e-2), np.log(20.0), n))
    xm[:40] = x[:40] * (1 + rng.uniform(-1e-3, 1e-3, 40))   # near the ring through the centre
    got = E.nfw_mis("dsigma_single", x * rs, xm * rs, lnM, conc, rho, n_theta=256)
    want = np.array([L.y3o_nfw_norm(m, conc, rho) * L.y3o_dsigma_single_unit(a, b, 256)
                     for m, a, b in zip(lnM, x, xm)])
    assert np.any(want < 0) and np.any(want > 0)
    # The device's closed-form NFW Delta Sigma and the oracle's differ at the
    # 1e-9 level near x = 1 (series branch); the quadrature is the same.
    np.testing.assert_allclose(got, want, rtol=1e-7, atol=1e-12 * np.abs(want).max())


def test_prj_quadrature_runs_the_signed_profile(gpu):
    """Without a table the projection shear integrates the single-kernel
    profile directly, negative values included (x < x_mis).  The reference
    reads the profile as a log table, which carries only its positive part,
    so the two forms differ by the table's clipping.  The output is linear in
    the profile: out(log pos) - out(log neg) + out(empty) with tables of the
    two signed parts approaches the quadrature's output; a log table cannot
    interpolate across the sign change (the cells that straddle it read
    ~0 from both tables, and their totals differ by about 30 %), so the
    agreement is checked in shape: correlation above 0.95 over the first
    three outputs.
    The profile itself is pinned to the oracle by the test above."""
    g = _golden()
    t, prj, grid, cfg = _inputs(g)
    cos = E.cosmo(float(g["omega_m"]), float(g["h0"]))
    lx = np.linspace(-7.0, 8.6, 600)
    lxm = np.linspace(-4.7, 6.3, 240)
    import oracle as O
    X, XM = np.meshgrid(np.exp(lx), np.exp(lxm))
    lnM0, conc, rho = 32.0, 4.0, 1e11
    rs, norm = O.lib().y3o_nfw_rs(lnM0, conc, rho), O.lib().y3o_nfw_norm(lnM0, conc, rho)
    unit = E.nfw_mis("dsigma_single", X.ravel() * rs, XM.ravel() * rs, lnM0, conc, rho,
                     n_theta=256).reshape(X.shape) / norm
    outs = {}
    for name, tab in (("pos", np.maximum(unit, 0.0)), ("neg", np.maximum(-unit, 0.0)),
                      ("zero", np.zeros_like(unit))):
        h = E.PrjShear(grid, **cfg)
        h.set_mis_table(lx, lxm, np.log(np.maximum(tab, 1e-300)))
        outs[name] = h.eval(cos, t, prj)
        h.close()
    h = E.PrjShear(grid, **cfg)
    quad = h.eval(cos, t, prj)
    again = h.eval(cos, t, prj)
    h.close()
    np.testing.assert_array_equal(quad, again)
    assert np.all(np.isfinite(quad))
    want = outs["pos"] - outs["neg"] + outs["zero"]
    qa, wa = quad[:, :3].ravel(), want[:, :3].ravel()
    assert np.corrcoef(qa, wa)[0, 1] > 0.95


def test_prj_matches_live_reference_on_walkers(gpu, tmp_path):
    from oracle import ref as R
    if not R.available():
        pytest.skip("compiled reference (make -C oracle ref) absent")
    g = _golden()
    _, _, grid, cfg = _inputs(g)
    d = tmp_path / "data" / "nfw_off_center"
    d.mkdir(parents=True)
    stem = str(d / "table_1000_1e-03_5e+03_")
    np.savetxt(stem + "single_logx.txt", g["single_logx"], fmt="%.17g")
    np.savetxt(stem + "single_logxmis.txt", g["single_logxmis"], fmt="%.17g")
    np.savetxt(stem + "log_deltasigma_single.txt", np.ravel(g["single_log_tab"]), fmt="%.17g")
    h = E.PrjShear(grid, **cfg)
    h.set_mis_table(g["single_logx"], g["single_logxmis"], g["single_log_tab"])
    for p in synthetic.walkers(3, seed=4, densities=(1,)):
        prj = synthetic.prj_tables(p, n_r=120)
        cosmo = dict(omega_m=p.om, omega_nu=0.0, omega_lambda=1 - p.om, omega_k=0.0, h0=p.h0,
                     hmf_s=0.0, hmf_q=1.0)
        ref = R.shear_prj_frozen(cfg, cosmo, p.tables, prj, grid, str(tmp_path))
        _check(h.eval(E.cosmo(p.om, p.h0), p.tables, prj), ref)
    h.close()


def test_prj_module_setup_execute_matches_golden(gpu, tmp_path, monkeypatch):
    """ShearPrjFrozenPhysics.so through setup / execute / cleanup on a
    DataBlock, reading the single-kernel table from $Y3_CLUSTER_CPP_DIR as the
    reference does: all nine output arrays against the compiled reference."""
    from y3_cluster_cpp_b200.cosmosis import DataBlock, Module
    g = _golden()
    t, prj, grid, cfg = _inputs(g)
    d = tmp_path / "data" / "nfw_off_center"
    d.mkdir(parents=True)
    stem = str(d / "table_1000_1e-03_5e+03_")
    np.savetxt(stem + "single_logx.txt", g["single_logx"], fmt="%.17g")
    np.savetxt(stem + "single_logxmis.txt", g["single_logxmis"], fmt="%.17g")
    np.savetxt(stem + "log_deltasigma_single.txt", np.ravel(g["single_log_tab"]), fmt="%.17g")
    monkeypatch.setenv("Y3_CLUSTER_CPP_DIR", str(tmp_path))
    lab = "shear_prj_frozen_physics"
    o = DataBlock()
    for k, v in cfg.items():
        o[lab, k] = v
    o[lab, "lambda_bin"] = grid["lambda_bin"].astype(np.int32)
    for k in ("zo_low", "zo_high", "radii"):
        o[lab, k] = grid[k]
    o[lab, "mis_profile"] = "table"
    b = DataBlock()
    om, h0 = float(g["omega_m"]), float(g["h0"])
    for k, v in dict(omega_M=om, omega_lambda=1 - om, omega_k=0.0, h0=h0, omega_nu=0.0).items():
        b["cosmological_parameters", k] = v
    b["cluster_abundance", "hmf_s"] = 0.0
    b["cluster_abundance", "hmf_q"] = 1.0
    b["mass_function", "m_h"], b["mass_function", "z"] = t["hmf_m_h"], t["hmf_z"]
    b["mass_function", "dndlnmh"] = t["dndlnmh"]
    b["distances", "z"], b["distances", "d_a"] = t["dist_z"], t["dist_da"]
    b["distances", "d_c"] = prj["dist_dc"]
    b["average_sigma_crit_inv", "zlense"] = t["sci_z"]
    b["average_sigma_crit_inv", "sci_average"] = t["sci_val"]
    b["haloModel", "lnM"], b["haloModel", "z"] = prj["halo_lnM"], prj["halo_z"]
    b["haloModel", "bias"] = prj["bias"]
    b["xi_nl", "r"], b["xi_nl", "z"], b["xi_nl", "xi_nl"] = prj["xi_r"], prj["xi_z"], prj["xi_nl"]
    b["b_sel_marginalised", "lob"] = prj["bsel_lob"]
    b["b_sel_marginalised", "zob"] = prj["bsel_zob"]
    nz, nl = len(prj["bsel_zob"]), len(prj["bsel_lob"])
    b["b_sel_marginalised", "b_small"] = prj["b_small"].reshape(nz, nl)
    b["b_sel_marginalised", "b_large"] = prj["b_large"].reshape(nz, nl)
    m = Module("ShearPrjFrozenPhysics")
    assert m.setup(o)
    assert m.execute(b) == 0
    ref = g["vals"]
    cols = [("dsigma_prj_frozen_physics", "vals"), ("dsigma_prj_frozen_physics", "rnd"),
            ("dsigma_prj_frozen_physics", "cl"), ("shear_prj_frozen_physics", "vals"),
            ("shear_prj_frozen_physics", "rnd"), ("shear_prj_frozen_physics", "cl"),
            ("shear_prj", "vals"), ("shear_prj", "rnd"), ("shear_prj", "cl")]
    out = np.stack([b[s, n] for s, n in cols], axis=1)
    _check(out, ref)
    assert m.cleanup() == 0


def test_prj_line_of_sight_outside_distances_is_a_domain_error(gpu):
    """A line-of-sight z node beyond distances/z (the reference's Interp1D on
    d_a throws there) returns Y3B_ERR_DOMAIN before any launch, and the same
    handle then evaluates a complete sample."""
    g = _golden()
    t, prj, grid, cfg = _inputs(g)
    cos = E.cosmo(float(g["omega_m"]), float(g["h0"]))
    keep = t["dist_z"] <= 0.45
    t_cut = dict(t, dist_z=t["dist_z"][keep], dist_da=t["dist_da"][keep])
    prj_cut = dict(prj, dist_dc=prj["dist_dc"][keep])
    h = E.PrjShear(grid, **cfg)
    h.set_mis_table(g["single_logx"], g["single_logxmis"], g["single_log_tab"])
    with pytest.raises(E.A.Y3BError) as e:
        h.eval(cos, t_cut, prj_cut)
    assert e.value.status == E.A.ERR_DOMAIN
    _check(h.eval(cos, t, prj), g["vals"])
    h.close()
