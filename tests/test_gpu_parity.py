"""GPU parity: the CUDA path through the C ABI against the FP64 CPU oracle
(and the reference's golden vectors).  Tolerances:
  * FP64 paths (sel_function, SelGL, engine FP64): <= 1e-8 relative (the
    north-star bar); observed ~1e-13.
  * mixed engine (FP32 integrands, split-BF16 tcgen05 contraction, FP64
    final sums): <= 1e-4 relative."""
import os

import numpy as np
import pytest

import oracle as O
from y3_cluster_cpp_b200 import engine as E
from y3_cluster_cpp_b200 import prj_params, synthetic

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL64 = 1e-8
TOLMIX = 1e-4


def _cfg(g):
    cfg = {k: g[k] for k in ("lam_min", "lam_max", "zob_min", "zob_max", "sigma_z")}
    cfg.update(zt_low=float(g["zt_low"]), zt_high=float(g["zt_high"]),
               lnm_low=float(g["lnm_low"]), lnm_high=float(g["lnm_high"]),
               n_lnm=int(g["n_lnm"]), n_z=int(g["n_z_shared"]), n_q=int(g["N_q"]))
    return cfg


@pytest.mark.parametrize("kind", ["hod", "lognormal"])
def test_sel_function_gpu_matches_golden_and_oracle(gpu, kind):
    g = np.load(os.path.join(GOLD, f"sel_function_{kind}.npz"))
    if kind == "hod":
        mk = O.MOR_HOD
        mor = [float(g["hod_" + k]) for k in ("log10_Mmin", "log10_M1", "alpha", "epsilon",
                                              "sigma_lambda")] + [0.45]
        pz, pc = prj_params.default_table()
    else:
        mk = O.MOR_LOGNORMAL
        mor = [float(g["ln_" + k]) for k in ("A", "B", "C", "sigma", "Mpiv", "lam_lo", "lam_hi")]
        pz, pc = prj_params.baseline_constant_table()
    lnm, z, S = E.sel_function(_cfg(g), mk, mor, pz, pc)
    _, _, So = O.sel_function(_cfg(g), mk, mor, pz, pc)
    scale = np.max(g["S_stack"])
    assert np.max(np.abs(S - g["S_stack"])) <= 1e-10 * scale
    assert np.max(np.abs(S - So)) <= 1e-12 * scale
    np.testing.assert_allclose(lnm, g["lnM"], atol=1e-12)


def test_sel_function_full_size_reference_grid(gpu):
    """The des_y3.ini production grid (12 bins, 192 lnM x 64 z x 32 lam_t)."""
    g = np.load(os.path.join(GOLD, "sel_function_hod.npz"))
    cfg = _cfg(g)
    cfg.update(n_lnm=192, n_z=64, n_q=32, lnm_high=36.8414)
    mor = [11.4, 12.7, 0.86, 0.0, 0.18, 0.45]
    pz, pc = prj_params.default_table()
    _, _, S = E.sel_function(cfg, O.MOR_HOD, mor, pz, pc)
    _, _, So = O.sel_function(cfg, O.MOR_HOD, mor, pz, pc)
    assert np.max(np.abs(S - So)) <= 1e-12 * np.max(So)


def _selgl_case(n_lnm=96, n_z=64):
    p = synthetic.fiducial()
    g = synthetic.grid(1)
    pz, pc = synthetic.plob_baseline()
    cfg = dict(lam_min=np.tile(g["lam_edges"][:-1], 3), lam_max=np.tile(g["lam_edges"][1:], 3),
               zob_min=np.repeat(g["zob_edges"][:-1], 4),
               zob_max=np.repeat(g["zob_edges"][1:], 4), sigma_z=np.full(12, 0.0145),
               zt_low=0.1, zt_high=0.8, lnm_low=g["lnm_lo"], lnm_high=g["lnm_hi"],
               n_lnm=96, n_z=48, n_q=32)
    mor = [p.A, p.B, p.C, p.sigma, p.Mpiv, 1.0, 1000.0]
    sel = O.sel_function(cfg, O.MOR_LOGNORMAL, mor, pz, pc)
    box = (n_lnm, n_z, 0.1, 0.8, g["lnm_lo"], g["lnm_hi"])
    return p, sel, box


def test_numcounts_selgl_matches_oracle(gpu):
    p, sel, box = _selgl_case()
    c = O.cosmo(p.om, p.h0)
    W, norm, eff, mu2 = O.selgl_weights(*box, c, p.tables, sel)
    h = E.SelGL(*box)
    h.build(E.cosmo(p.om, p.h0), p.tables, sel)
    vals = h.counts(np.arange(12))
    np.testing.assert_allclose(vals, norm, rtol=TOL64)
    w = h.weights()
    np.testing.assert_allclose(w["W"], W, rtol=TOL64, atol=1e-12 * np.max(np.abs(W)))
    np.testing.assert_allclose(w["lnm_eff"], eff, rtol=1e-12)
    np.testing.assert_allclose(w["mu2"], mu2, rtol=1e-8)
    with pytest.raises(E.A.Y3BError):
        h.counts([12])  # bin_index outside S_stack range
    h.close()


def _halo_table(om):
    R = np.logspace(-2, 1.7, 40)
    lnM = np.linspace(np.log(1e13), np.log(10 ** 15.5), 30)
    rho = 2.77533742639e11 * om
    ds = np.empty((len(lnM), len(R)))
    for i, m in enumerate(lnM):
        c = 5.0 * (np.exp(m) / 1e14) ** -0.1
        rs = O.lib().y3o_nfw_rs(m, c, rho)
        nrm = O.lib().y3o_nfw_norm(m, c, rho)
        ds[i] = [nrm * O.lib().y3o_nfw_dsigma_unit(r / rs) for r in R]
    return dict(r_sigma=R, lnM=lnM, dSigma_nfw=ds)


@pytest.mark.parametrize("idea2", [False, True])
def test_shear1h_mis_selgl_matches_oracle(gpu, idea2):
    p, sel, box = _selgl_case(n_lnm=48, n_z=32)
    c = O.cosmo(p.om, p.h0)
    W, norm, eff, mu2 = O.selgl_weights(*box, c, p.tables, sel,
                                        sci=(p.tables["sci_z"], p.tables["sci_val"]))
    halo = _halo_table(p.om)
    R = np.array([0.1, 0.4, 1.5, 6.0])
    h = E.SelGL(*box)
    h.build(E.cosmo(p.om, p.h0), p.tables, sel, include_sci=True)
    bins = np.repeat(np.arange(12), len(R))
    rr = np.tile(R, 12)
    got = h.shear(bins, rr, halo, n_theta=16, n_s=32, idea2=idea2)
    x, w = O.gl_nodes(box[4], box[5], box[0])
    if not idea2:
        ref = O.shear1h_mis(x, w, W, R, 0.22, 0.17, [25, 37.5, 52.5, 130], p.om, 4.0,
                            halo["r_sigma"], halo["lnM"], halo["dSigma_nfw"], 16, 32, 20.0)
        np.testing.assert_allclose(got, ref.ravel(), rtol=TOL64)
    else:
        # idea2: norm [phi(eff) + mu2/2 phi''] with a 3-point stencil
        wts = h.weights()
        one = np.ones(1)
        for b in range(12):
            for r_i, r in enumerate(R):
                vals = []
                for dy in (0.0, 0.15, -0.15):
                    vals.append(O.shear1h_mis(np.array([wts["lnm_eff"][b] + dy]), one,
                                              np.ones((12, 1)), [r], 0.22, 0.17,
                                              [25, 37.5, 52.5, 130], p.om, 4.0,
                                              halo["r_sigma"], halo["lnM"], halo["dSigma_nfw"],
                                              16, 32, 20.0)[b, 0])
                d2 = (vals[1] - 2 * vals[0] + vals[2]) / 0.15 ** 2
                ref = wts["norm"][b] * (vals[0] + 0.5 * wts["mu2"][b] * d2)
                assert got[b * len(R) + r_i] == pytest.approx(ref, rel=1e-8)
    h.close()


def test_sigma_crit_inv_matches_oracle(gpu):
    p = synthetic.fiducial()
    zs, pz = synthetic.source_nz()
    zl = np.linspace(0.05, 0.85, 64)
    got = E.sigma_crit_inv(zl, zs, pz, 0.0, p.h0, p.tables["dist_z"], p.tables["dist_da"])
    ref = O.sigma_crit_inv(zl, zs, pz, 0.0, p.h0, p.tables["dist_z"], p.tables["dist_da"])
    np.testing.assert_allclose(got, ref, rtol=1e-12)
    np.testing.assert_allclose(got, p.tables["sci_val"], rtol=1e-10)


def test_nfw_mis_matches_oracle_and_kats(gpu):
    import json
    kats = json.load(open(os.path.join(GOLD, "kats.json")))
    for which, fn in (("dsigma", O.dsigma_mis_unit), ("sigma", O.sigma_mis_unit)):
        d = kats[which + "_mis"]
        rho = 2.77533742639e11 * 0.3
        n = min(len(d["answers"]), len(d["r"]) * len(d["rmis"]))
        r = np.repeat(d["r"], len(d["rmis"]))[:n]
        rm = np.tile(d["rmis"], len(d["r"]))[:n]
        answers = np.array(d["answers"][:n])
        got = E.nfw_mis(which, r, rm, d["lnM"][0], 4.0, rho)
        rs = O.lib().y3o_nfw_rs(d["lnM"][0], 4.0, rho)
        nrm = O.lib().y3o_nfw_norm(d["lnM"][0], 4.0, rho)
        ref = np.array([nrm * fn(a / rs, b / rs, 64, 128, 20.0) for a, b in zip(r, rm)])
        np.testing.assert_allclose(got, ref, rtol=1e-10)
        tol = np.where((rm >= 2.0) & (r >= 5.0) & (which == "sigma"), 1.5e-3, d["epsrel"])
        assert np.all(np.abs(got / answers - 1) <= tol)


# ---------------------------------------------------------------------------
# Engine (direct nested quadrature, FP64 and mixed)

def _engine(grids, n_max=8, shear=None):
    p = synthetic.fiducial()
    t = p.tables
    pz, pc = synthetic.plob_baseline()
    return E.Engine(grids, len(t["hmf_m_h"]), len(t["hmf_z"]), len(t["dist_z"]), (pz, pc),
                    max_points=n_max, n_sci=len(t["sci_z"]), shear=shear)


@pytest.mark.parametrize("density", [1, 2, 4])
def test_engine_counts_match_oracle(gpu, density):
    g = synthetic.grid(density)
    eng = _engine([g])
    p = synthetic.fiducial()
    pz, pc = synthetic.plob_baseline()
    ref, Wref, _ = O.direct_eval(g, pz, pc, p.mor, O.cosmo(p.om, p.h0), p.tables)
    r64 = eng.eval([p], E.FP64, grid_of=lambda _: 0, weights=True)
    rmx = eng.eval([p], E.MIXED, grid_of=lambda _: 0, weights=True)
    np.testing.assert_allclose(r64["counts"][0], ref, rtol=TOL64)
    np.testing.assert_allclose(rmx["counts"][0], ref, rtol=TOLMIX)
    np.testing.assert_allclose(r64["W"][0], Wref, rtol=TOL64, atol=TOL64 * np.max(Wref))
    np.testing.assert_allclose(rmx["W"][0], Wref, rtol=0, atol=TOLMIX * np.max(Wref))
    eng.close()


def test_engine_stage_window_skips_only_negligible_stages(gpu):
    """The contraction issues only the lam_t stages inside mu +- 5 sigma of
    each lnM tile: a narrow MOR scatter issues fewer stages, and both stay
    within tolerance of the oracle's full-range quadrature."""
    g = synthetic.grid(4)  # two 128-row lnM tiles, each spanning part of the lam_t range
    eng = _engine([g])
    pz, pc = synthetic.plob_baseline()
    issued = {}
    for sigma in (0.12, 0.35):
        p = synthetic.fiducial()
        p.sigma = sigma
        ref, _, _ = O.direct_eval(g, pz, pc, p.mor, O.cosmo(p.om, p.h0), p.tables)
        rmx = eng.eval([p], E.MIXED, grid_of=lambda _: 0)["counts"][0]
        ex, dn = eng.stage_count()
        assert 0 < ex <= dn
        issued[sigma] = ex
        np.testing.assert_allclose(rmx, ref, rtol=TOLMIX)
    assert issued[0.12] < issued[0.35] and issued[0.12] < dn
    eng.close()


def test_engine_batched_walkers_mixed_densities(gpu):
    """Uneven grids in one call; each point equals its own evaluation alone
    (bitwise) and the oracle (tolerance)."""
    grids = [synthetic.grid(d) for d in (1, 2, 4)]
    pts = synthetic.walkers(6, seed=1)
    gi = {1: 0, 2: 1, 4: 2}
    eng = _engine(grids, n_max=8)
    pz, pc = synthetic.plob_baseline()
    for prec, tol in ((E.FP64, TOL64), (E.MIXED, TOLMIX)):
        batch = eng.eval(pts, prec, grid_of=lambda p: gi[p.density])["counts"]
        for i, p in enumerate(pts):
            alone = eng.eval([p], prec, grid_of=lambda q: gi[q.density])["counts"][0]
            assert np.array_equal(alone, batch[i])
            ref, _, _ = O.direct_eval(grids[gi[p.density]], pz, pc, p.mor, O.cosmo(p.om, p.h0),
                                      p.tables)
            np.testing.assert_allclose(batch[i], ref, rtol=tol)
    eng.close()


def test_engine_reruns_bit_identical(gpu):
    eng = _engine([synthetic.grid(4)], n_max=4)
    pts = synthetic.walkers(4, seed=3, densities=(4,))
    for prec in (E.FP64, E.MIXED):
        a = eng.eval(pts, prec, grid_of=lambda _: 0)["counts"]
        b = eng.eval(pts, prec, grid_of=lambda _: 0)["counts"]
        assert np.array_equal(a, b)
    eng.close()


def test_engine_shear_matches_oracle(gpu):
    g = synthetic.grid(1, n_m=32)
    sh = synthetic.shear_opts(n_theta=16, n_s=32, n_R=5)
    eng = _engine([g], n_max=2, shear=sh)
    p = synthetic.fiducial()
    pz, pc = synthetic.plob_baseline()
    so = dict(sh, sci_z=p.tables["sci_z"], sci_val=p.tables["sci_val"])
    ref, _, rsh = O.direct_eval(g, pz, pc, p.mor, O.cosmo(p.om, p.h0), p.tables, shear=so)
    r64 = eng.eval([p], E.FP64, grid_of=lambda _: 0)
    rmx = eng.eval([p], E.MIXED, grid_of=lambda _: 0)
    np.testing.assert_allclose(r64["shear"][0], rsh, rtol=TOL64)
    np.testing.assert_allclose(rmx["shear"][0], rsh, rtol=TOLMIX)
    np.testing.assert_allclose(r64["counts"][0], ref, rtol=TOL64)
    eng.close()


def test_engine_domain_error_and_recovery(gpu):
    g = synthetic.grid(1)
    eng = _engine([g], n_max=2)
    p = synthetic.fiducial()
    bad = synthetic.Point(**{k: getattr(p, k) for k in ("om", "sigma8", "h0", "A", "B", "C",
                                                         "sigma", "Mpiv", "density")})
    bad.tables = dict(p.tables)
    bad.tables["dist_z"] = p.tables["dist_z"] * 0.3   # table ends at z = 0.6 < zt_hi
    with pytest.raises(E.A.Y3BError) as e:
        eng.eval([bad], E.FP64, grid_of=lambda _: 0)
    assert e.value.status == 2
    ok = eng.eval([p], E.MIXED, grid_of=lambda _: 0)["counts"]
    assert np.all(np.isfinite(ok)) and np.all(ok > 0)
    eng.close()


def test_bounded_wait_reports_timeout(gpu):
    assert E.selftest_wait_timeout(2000) == 5  # Y3B_ERR_TIMEOUT
    # the context stays usable
    assert np.all(np.isfinite(E.nfw_mis("dsigma", [0.5], [0.1], [32.0], 4.0, 8e10)))


def test_engine_rejects_bad_arguments(gpu):
    eng = _engine([synthetic.grid(1)], n_max=2)
    p = synthetic.fiducial()
    with pytest.raises(E.A.Y3BError) as e:
        eng.eval([p, p, p], E.FP64, grid_of=lambda _: 0)    # above max_points
    assert e.value.status == 1
    with pytest.raises(E.A.Y3BError):
        eng.eval([p], E.FP64, grid_of=lambda _: 3)          # no such grid
    eng.close()
    with pytest.raises(E.A.Y3BError) as e:
        E.Engine([synthetic.grid(1, n_z=40)], 100, 50, 200, synthetic.plob_baseline())
    assert e.value.status == 7


def test_engine_graph_replay_matches_direct_launches(gpu):
    """Repeated device evaluations are captured once into a CUDA graph and
    replayed; the replayed results equal those of plain launches bitwise and
    the launch accounting counts the graph's kernels on every replay."""
    import ctypes as C
    import torch
    g = synthetic.grid(1)
    eng = _engine([g], n_max=8)
    pts = synthetic.walkers(6, seed=31, densities=(1,))
    parr = eng.points_array(pts, grid_of=lambda _: 0)
    ph = torch.empty(C.sizeof(parr), dtype=torch.uint8)
    C.memmove(ph.data_ptr(), C.addressof(parr), C.sizeof(parr))
    pd = ph.cuda()
    tab = torch.tensor(eng.pack(pts)).cuda()
    out = torch.empty((6, eng.n_bins), dtype=torch.float64, device="cuda")
    res, launches = [], []
    for mode in (0, 1):
        eng.set_graphs(bool(mode))
        for _ in range(4):                     # 1st plain, 2nd captured, 3rd/4th replayed
            l0 = E.launch_count()
            eng.eval_device(E.MIXED, 6, pd.data_ptr(), tab.data_ptr(), out.data_ptr())
            eng.sync()
            launches.append(E.launch_count() - l0)
            res.append(out.cpu().numpy().copy())
    for r in res[1:]:
        np.testing.assert_array_equal(r, res[0])
    assert len(set(launches)) == 1 and launches[0] >= 3
    eng.close()


def test_engine_autotune_keeps_results_within_tolerance(gpu):
    """The autotuner picks a ring depth and bins per tile from its candidate
    set; the tuned engine still meets the 1e-4 bar against FP64 and gives a
    point the same counts alone and in a mixed-density batch."""
    import ctypes as C
    import torch
    grids = [synthetic.grid(1), synthetic.grid(2)]
    eng = _engine(grids, n_max=16)
    pts = synthetic.walkers(12, seed=41, densities=(1, 2))
    gof = {1: 0, 2: 1}
    parr = eng.points_array(pts, grid_of=lambda p: gof[p.density])
    ph = torch.empty(C.sizeof(parr), dtype=torch.uint8)
    C.memmove(ph.data_ptr(), C.addressof(parr), C.sizeof(parr))
    pd = ph.cuda()
    tab = torch.tensor(eng.pack(pts)).cuda()
    out = torch.empty((12, eng.n_bins), dtype=torch.float64, device="cuda")
    t = eng.autotune(12, pd.data_ptr(), tab.data_ptr(), out.data_ptr())
    assert 2 <= t["stages"] <= 8 and t["contraction_ms"] > 0
    assert all(b in (1, 2, 4, 8) for b in t["bins_per_tile"])
    r64 = eng.eval(pts, E.FP64, grid_of=lambda p: gof[p.density])["counts"]
    rmx = eng.eval(pts, E.MIXED, grid_of=lambda p: gof[p.density])["counts"]
    assert np.max(np.abs(rmx / r64 - 1)) <= TOLMIX
    alone = eng.eval(pts[5:6], E.MIXED, grid_of=lambda p: gof[p.density])["counts"]
    np.testing.assert_array_equal(alone[0], rmx[5])
    eng.close()


@pytest.mark.parametrize("n", [1100, 2100])  # four and seven chunks (FP64 tables)
def test_engine_chunked_host_eval_matches_one_launch(gpu, n):
    """A large host-buffer evaluation is split into chunks whose copies
    overlap the previous chunk's kernels; counts and the mass weights equal
    those of a single device launch over the same batch."""
    import ctypes as C
    import torch
    g = synthetic.grid(1)
    eng = _engine([g], n_max=n)
    uniq = synthetic.walkers(20, seed=51, densities=(1,))
    pts = [uniq[i % 20] for i in range(n)]
    tab = eng.pack(pts)
    r = eng.eval(pts, E.MIXED, tables=tab, grid_of=lambda _: 0, weights=True)
    parr = eng.points_array(pts, grid_of=lambda _: 0)
    ph = torch.empty(C.sizeof(parr), dtype=torch.uint8)
    C.memmove(ph.data_ptr(), C.addressof(parr), C.sizeof(parr))
    pd, td = ph.cuda(), torch.tensor(tab).cuda()
    out = torch.empty((n, eng.n_bins), dtype=torch.float64, device="cuda")
    eng.eval_device(E.MIXED, n, pd.data_ptr(), td.data_ptr(), out.data_ptr())
    eng.sync()
    np.testing.assert_array_equal(r["counts"], out.cpu().numpy())
    W = np.empty_like(r["W"])
    E.check(E.lib().y3b_engine_weights(eng.handle, n, E.A.ptr(W)))
    np.testing.assert_array_equal(W, r["W"])
    eng.close()


@pytest.mark.parametrize("lam_t", [(15.0, 1000.0), (44.7, 1000.0), (1.0, 150.0)])
def test_engine_window_with_mass_piled_at_a_domain_edge(gpu, lam_t):
    """lam_t domains that cut into the MOR: with lam_t_lo = 44.7 the first lnM
    tile's largest mu sits about 4 sigma below ln lam_t_lo (its cells keep
    only a Gaussian tail, renormalised by a small in-range mass D), with 15
    the low-mass cells sit far below it, and with lam_t_hi = 150 the
    high-mass cells sit above ln lam_t_hi.  The contraction's stage window
    must follow that renormalised density to the domain edge."""
    g = synthetic.grid(4, lam_t_lo=lam_t[0], lam_t_hi=lam_t[1])
    eng = _engine([g])
    p = synthetic.fiducial()
    pz, pc = synthetic.plob_baseline()
    ref, _, _ = O.direct_eval(g, pz, pc, p.mor, O.cosmo(p.om, p.h0), p.tables)
    r64 = eng.eval([p], E.FP64, grid_of=lambda _: 0)["counts"][0]
    rmx = eng.eval([p], E.MIXED, grid_of=lambda _: 0)["counts"][0]
    np.testing.assert_allclose(r64, ref, rtol=TOL64)
    np.testing.assert_allclose(rmx, ref, rtol=TOLMIX)
    eng.close()


@pytest.mark.parametrize("sigma", [0.09, 0.07])
def test_engine_mor_far_outside_the_lam_t_domain(gpu, sigma):
    """With lam_t_lo = 44.7 and sigma_int = 0.09 (0.07) the lowest-mass cells'
    mu sits about 40 (50) sigma below ln lam_t_lo: the MOR's in-range mass D
    underflows FP64 and the Gaussian at every lam_t node underflows too, while
    their quotient (the density piled at the domain edge) is moderate.  Both
    forms carry that quotient without an inf or a NaN: FP64 within 1e-9 of the
    oracle, the mixed form within 1e-4 or a clean Y3B_ERR_RANGE."""
    g = synthetic.grid(4, lam_t_lo=44.7, lam_t_hi=1000.0)
    eng = _engine([g])
    p = synthetic.fiducial()
    p.sigma = sigma
    pz, pc = synthetic.plob_baseline()
    ref, _, _ = O.direct_eval(g, pz, pc, p.mor, O.cosmo(p.om, p.h0), p.tables)
    assert np.all(np.isfinite(ref)) and np.all(ref > 0)
    r64 = eng.eval([p], E.FP64, grid_of=lambda _: 0)["counts"][0]
    np.testing.assert_allclose(r64, ref, rtol=TOL64)
    try:
        rmx = eng.eval([p], E.MIXED, grid_of=lambda _: 0)["counts"][0]
    except E.A.Y3BError as e:
        assert e.status == E.A.ERR_RANGE
    else:
        assert np.all(np.isfinite(rmx))
        np.testing.assert_allclose(rmx, ref, rtol=TOLMIX)
    eng.close()


@pytest.mark.parametrize("case", [dict(sigma=0.05), dict(sigma=0.1), dict(C=2.0),
                                  dict(sigma=0.05, C=2.0)])
def test_mixed_form_exponent_range_guard(gpu, case):
    """Outside the prior (sigma_int = 0.05, C = 2) the factorised Gaussian's
    exponents grow as (alpha range)(beta range)/sigma^2.  The mixed form either
    stays within 1e-4 of the FP64 oracle or reports Y3B_ERR_RANGE for the
    point; it never returns a NaN or a silently wrong count, and the engine
    stays usable."""
    g = synthetic.grid(4)
    eng = _engine([g])
    p = synthetic.fiducial()
    for k, v in case.items():
        setattr(p, k, v)
    pz, pc = synthetic.plob_baseline()
    ref, _, _ = O.direct_eval(g, pz, pc, p.mor, O.cosmo(p.om, p.h0), p.tables)
    r64 = eng.eval([p], E.FP64, grid_of=lambda _: 0)["counts"][0]
    np.testing.assert_allclose(r64, ref, rtol=TOL64)
    try:
        rmx = eng.eval([p], E.MIXED, grid_of=lambda _: 0)["counts"][0]
    except E.A.Y3BError as e:
        assert e.status == E.A.ERR_RANGE
        assert case.get("sigma", 0.2) <= 0.05        # only the narrowest scatter trips it
    else:
        assert np.all(np.isfinite(rmx))
        np.testing.assert_allclose(rmx, ref, rtol=TOLMIX)
    ok = eng.eval([synthetic.fiducial()], E.MIXED, grid_of=lambda _: 0)["counts"]
    assert np.all(np.isfinite(ok)) and np.all(ok > 0)
    eng.close()


@pytest.mark.parametrize("where", ["dndlnmh", "dist_da", "hmf_m_h"])
@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_engine_rejects_non_finite_tables(gpu, where, bad):
    """A NaN or Inf table entry (host-side injection) gives Y3B_ERR_DOMAIN in
    both precisions instead of flowing into the counts."""
    g = synthetic.grid(1)
    eng = _engine([g], n_max=2)
    p = synthetic.fiducial()
    q = synthetic.Point(**{k: getattr(p, k) for k in ("om", "sigma8", "h0", "A", "B", "C",
                                                       "sigma", "Mpiv", "density")})
    q.tables = {k: np.array(v, copy=True) for k, v in p.tables.items()}
    q.tables[where].flat[3] = bad
    for prec in (E.FP64, E.MIXED):
        with pytest.raises(E.A.Y3BError) as e:
            eng.eval([p, q], prec, grid_of=lambda _: 0)
        assert e.value.status == E.A.ERR_DOMAIN
    ok = eng.eval([p], E.MIXED, grid_of=lambda _: 0)["counts"]
    assert np.all(np.isfinite(ok)) and np.all(ok > 0)
    eng.close()


def _oracle_walker(args):
    """FP64 direct quadrature of one walker (run in a spawned worker)."""
    seed, n, i, shear = args
    import oracle as Ow
    from y3_cluster_cpp_b200 import synthetic as S
    p = S.walkers(n, seed=seed, densities=(1, 2, 4))[i]
    g = S.grid(p.density)
    pz, pc = S.plob_baseline()
    so = None
    if shear is not None:
        so = dict(shear, sci_z=p.tables["sci_z"], sci_val=p.tables["sci_val"])
    c, _, sh = Ow.direct_eval(g, pz, pc, p.mor, Ow.cosmo(p.om, p.h0), p.tables, shear=so)
    return c, sh


def test_batched_config_sample_counts_and_delta_sigma_match_oracle(gpu):
    """A 12-walker sample of the batched config at its full sizes: 1x / 2x / 4x
    grids in thirds, counts and the stacked miscentred DeltaSigma (15 log radii
    0.1-30 Mpc/h, 64 theta x 128 R_mis) for every walker in one evaluation,
    against the oracle walker by walker (FP64 <= 1e-8, mixed <= 1e-4).  The
    first four walkers are the 1x grid of the DeltaSigma config."""
    import concurrent.futures as cf
    import multiprocessing as mp
    sh = synthetic.shear_opts(n_theta=64, n_s=128, n_R=15)
    n, seed = 12, 5
    pts = synthetic.walkers(n, seed=seed, densities=(1, 2, 4))
    assert [p.density for p in pts] == [1] * 4 + [2] * 4 + [4] * 4
    workers = max(1, min(n, os.cpu_count() or 1))
    with cf.ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
        refs = list(ex.map(_oracle_walker, [(seed, n, i, sh) for i in range(n)]))
    grids = [synthetic.grid(d) for d in (1, 2, 4)]
    gi = {1: 0, 2: 1, 4: 2}
    eng = _engine(grids, n_max=n, shear=sh)
    for prec, tol in ((E.FP64, TOL64), (E.MIXED, TOLMIX)):
        r = eng.eval(pts, prec, grid_of=lambda p: gi[p.density])
        for i, (c_ref, s_ref) in enumerate(refs):
            np.testing.assert_allclose(r["counts"][i], c_ref, rtol=tol)
            np.testing.assert_allclose(r["shear"][i], s_ref, rtol=tol)
    eng.close()


@pytest.mark.parametrize("dense", [False, True])
@pytest.mark.parametrize("log_space", [False, True])
def test_engine_fused_likelihood(gpu, dense, log_space):
    """The likelihood fused into the engine's final sums: each point's logL
    equals the oracle's likelihood (restated from likelihood_cp.py, pinned to
    it) of that point's own counts and shear, in both precisions, for the
    device-buffer path and the host-buffer loglike-only call."""
    g = synthetic.grid(1, n_m=32)
    sh = synthetic.shear_opts(n_theta=16, n_s=32, n_R=5)
    eng = _engine([g], n_max=6, shear=sh)
    pts = synthetic.walkers(6, seed=9, densities=(1,))
    rng = np.random.default_rng(3)
    fid = eng.eval([synthetic.fiducial()], E.FP64, grid_of=lambda _: 0)
    d_nc = fid["counts"][0] * rng.uniform(0.9, 1.1, 12)
    d_sh = (fid["shear"][0] / fid["counts"][0][:, None]).ravel() * rng.uniform(0.9, 1.1, 60)
    prj = 0.05 * d_sh * rng.uniform(-1, 1, 60)
    if dense:
        A = rng.normal(size=(12, 12))
        ic_nc = np.linalg.inv(A @ A.T + np.diag(d_nc))
        Bm = rng.normal(size=(60, 60))
        ic_sh = np.linalg.inv(1e-3 * np.diag(d_sh ** 2) @ (np.eye(60) + 0.01 * Bm @ Bm.T))
    else:
        ic_nc, ic_sh = 1.0 / d_nc, 1.0 / (0.1 * d_sh) ** 2
    spec = E.LikelihoodSpec(d_nc, ic_nc, d_sh, ic_sh, shear_prj=prj, log_space=log_space)
    eng.set_likelihood(spec)
    dn, ds, icn, ics = d_nc, d_sh, ic_nc, ic_sh
    if log_space:
        icn = icn * (np.outer(dn, dn) if dense else dn * dn)
        ics = ics * (np.outer(ds, ds) if dense else ds * ds)
        dn, ds = np.log(dn), np.log(ds)
    for prec in (E.FP64, E.MIXED):
        r = eng.eval(pts, prec, grid_of=lambda _: 0)
        ll = eng.loglike(len(pts))
        for i in range(len(pts)):
            ref = O.loglike(r["counts"][i], r["shear"][i], prj, log_space, dn, icn, ds, ics)
            assert ll[i] == pytest.approx(ref, rel=1e-11, abs=1e-9)
        parr = eng.points_array(pts, grid_of=lambda _: 0)
        tab = np.ascontiguousarray(eng.pack(pts))
        out = np.empty(len(pts))
        E.check(E.lib().y3b_engine_eval_loglike(eng.handle, prec, len(pts), parr,
                                                E.A.ptr(tab), E.A.ptr(out)))
        np.testing.assert_array_equal(out, ll)
    eng.set_likelihood(None)
    eng.close()


def test_engine_fp32_hmf_tables_give_identical_mixed_results(gpu):
    """An engine whose packed tables carry the HMF grid in FP32 (half the
    bytes per point on the host-to-device path) returns bitwise the mixed-form
    results of the FP64-table engine, which rounds the grid to FP32 on the
    device; its FP64 form is refused."""
    grids = [synthetic.grid(d) for d in (1, 2, 4)]
    pts = synthetic.walkers(6, seed=12)
    gi = {1: 0, 2: 1, 4: 2}
    t = pts[0].tables
    pz, pc = synthetic.plob_baseline()
    e64 = E.Engine(grids, len(t["hmf_m_h"]), len(t["hmf_z"]), len(t["dist_z"]), (pz, pc),
                   max_points=8, n_sci=len(t["sci_z"]))
    e32 = E.Engine(grids, len(t["hmf_m_h"]), len(t["hmf_z"]), len(t["dist_z"]), (pz, pc),
                   max_points=8, n_sci=len(t["sci_z"]), hmf_fp32=True)
    assert e32.stride < e64.stride
    a = e64.eval(pts, E.MIXED, grid_of=lambda p: gi[p.density])["counts"]
    b = e32.eval(pts, E.MIXED, grid_of=lambda p: gi[p.density])["counts"]
    np.testing.assert_array_equal(a, b)
    with pytest.raises(E.A.Y3BError) as ex:
        e32.eval(pts, E.FP64, grid_of=lambda p: gi[p.density])
    assert ex.value.status == 1
    e64.close()
    e32.close()
