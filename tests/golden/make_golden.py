"""Generate the golden fixtures that pin the oracle to the reference.

Run where a checkout of the reference exists (read-only is fine); the outputs
are committed, so neither the tests nor the GPU runs need the reference at
run time:

    python tests/golden/make_golden.py <reference-checkout>

What it writes (tests/golden/*.npz / *.json):

* sel_function_hod.npz -- S_stack from the reference's own
  src/modules/sel_function/sel_function.py (setup/execute, HOD MOR, default
  projection table from y3_buzzard/prj_params.py) on a reduced grid with the
  DES-Y3 bin layout of cosmosis-models/des_y3.ini:114-133.
* sel_function_lognormal.npz -- the same reference execute() with its MOR
  stage (_compute_lam_nodes_and_P_HOD) swapped for the lognormal MOR of the
  synthetic configs and the constant-in-z projection coefficients published
  through the plob_ltr_params section; everything downstream of the MOR
  (plob params, CDF differencing, K_j, packing) is the reference's code.
* kats.json -- the reference's own known-answer tables read as text:
  data/test_dv_do_dz.txt + z_da_test.txt + d_a_test.txt
  (test/dv_do_dz_t.test.cc), data/test_Rmis.txt (test/roffset_t.test.cc),
  data/test_int_zo_zt_des.txt (test/int_zo_zt_des_t.test.cc), the
  cluster_toolkit answers of test/nfw_dsigma_mis.test.cu:32-48 and
  test/nfw_sigma_mis.test.cu:32-46, and the interpolation KATs of
  test/interp_1d.test.cc / test/interp_2d.test.cc.
* sigma_crit_inv.npz -- <Sigma_crit^-1>(z_l) from the reference's own
  src/modules/average_sigma_crit_inv/average_sigma_crit_inv.py execute()
  (imported with CosmoSIS and astropy stubs; its setup() reads a FITS n(z)
  that is not in the snapshot, so the config tuple is built here with the
  synthetic source n(z): Gaussian, mean 0.9, sigma 0.3, 200 nodes).
* likelihood_ref.npz -- likelihoods/likelihoods_like from the reference's
  y3_buzzard/likelihood_cp.py setup/execute on a seeded mock data vector
  (12 counts, 12 x 10 shear; diagonal and dense inverse covariances; linear
  and log space) for four seeded theory blocks.
* prj_ref.npz -- the nine outputs of the reference's ShearPrjFrozenPhysics
  (src/models/sigma_prj_frozen_t.hh, compiled by `make -C oracle ref`) for
  12 slices x 10 radii on the fiducial synthetic tables (counts' tables plus
  comoving distance, halo bias, xi_NL and the selection-bias asymptotes of
  synthetic.prj_tables), with a stand-in single-kernel miscentring table.
* bsel_ref.npz -- P1, I1, J from the reference's compiled P_operator
  (src/models/p_operator_t.hh, module b_sel_marg) on the same fiducial
  tables with seeded HOD parameters: default node counts on 12 (z_obs bin,
  richness bin) points, reduced, odd node counts on 16 points for two
  samples (the second with its own z_pivot, sigma_lambda and M1), and one
  and two nodes per axis on four edge bins.
* selgl_ref.npz -- numcountssel/vals, SelGLCore weights and
  shear1hmissel/vals (exact and idea2) from the reference's own C++
  (src/models/n_operator_sel_gl_t.hh:75-361), compiled from its sources by
  `make -C oracle ref` against the shims of oracle/ref_shim/, on the
  S_stack fixtures above and the seeded synthetic tables of the configs
  (Tinker-like HMF 100 x 50, flat LCDM distances, Sigma_crit^-1 64 nodes).
  The miscentring table the shear module reads
  (data/nfw_off_center/table_1000_1e-03_5e+03_log_deltasigma_gamma.txt) is
  missing from the snapshot; the fixture carries a stand-in on every 8th ln x
  and every 5th ln x_mis node of the shipped axis files, filled by the
  oracle's direct quadrature of the gamma-kernel profile, and the reference
  reads it through its own file loader.
"""
from __future__ import annotations

import json
import os
import re
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _install_cosmosis_stub():
    mod = types.ModuleType("cosmosis")
    db = types.ModuleType("cosmosis.datablock")
    db.option_section = "module_options"
    names = types.SimpleNamespace(cosmological_parameters="cosmological_parameters")
    db.names = names
    mod.datablock = db
    sys.modules["cosmosis"] = mod
    sys.modules["cosmosis.datablock"] = db


class Options:
    """The subset of the CosmoSIS options API that sel_function.setup uses."""

    def __init__(self, d):
        self.d = d

    def _get(self, key):
        if key not in self.d:
            raise KeyError(key)
        return self.d[key]

    def get_double_array_1d(self, sec, key):
        v = self._get(key)
        if np.ndim(v) == 0:
            raise TypeError(key)
        return np.asarray(v, dtype=float)

    def get_int_array_1d(self, sec, key):
        return np.asarray(self._get(key), dtype=int)

    def get_double(self, sec, key):
        v = self._get(key)
        if np.ndim(v) != 0:
            raise TypeError(key)
        return float(v)

    def get_int(self, sec, key):
        v = self._get(key)
        if not isinstance(v, (int, np.integer)):
            raise TypeError(key)
        return int(v)


class Block(dict):
    """dict keyed by (section, name), like the CosmoSIS DataBlock python API."""


BINS = dict(
    lam_min=[20.0, 30.0, 45.0, 60.0] * 3,
    lam_max=[30.0, 45.0, 60.0, 200.0] * 3,
    zob_min=[0.20] * 4 + [0.35] * 4 + [0.50] * 4,
    zob_max=[0.35] * 4 + [0.50] * 4 + [0.65] * 4,
    sigma_z=[0.03] * 12,
)
ENVELOPE = dict(zt_low=0.05, zt_high=0.80, lnm_low=29.9336, lnm_high=36.8414)
GRID = dict(n_lnm=24, n_z_shared=12, N_q=16)
HOD = dict(log10_Mmin=11.4, log10_M1=12.7, alpha=0.86, epsilon=0.0, sigma_lambda=0.18)
LOGNORMAL = dict(A=3.2, B=0.9, C=0.5, sigma=0.2, Mpiv=3e14, lam_lo=1.0, lam_hi=1000.0)


def lognormal_stage(mor_ln):
    """Swap-in for sel_function._compute_lam_nodes_and_P_HOD: per-cell GL
    bracket exp(mu -+ 6 sigma) clipped to [lam_lo, lam_hi] and the truncated
    lognormal density in lambda, renormalised by an erf difference."""
    from scipy.special import erfc

    def phi_diff(a, b):
        return np.where(a >= 0, 0.5 * (erfc(a / np.sqrt(2)) - erfc(b / np.sqrt(2))),
                        np.where(b <= 0, 0.5 * (erfc(-b / np.sqrt(2)) - erfc(-a / np.sqrt(2))),
                                 1 - 0.5 * erfc(-a / np.sqrt(2)) - 0.5 * erfc(b / np.sqrt(2))))

    def stage(lnM, z, mor, gl_t, gl_w, L=6.0):
        m = mor_ln
        mu = (m["A"] + m["B"] * (lnM[:, None] - np.log(m["Mpiv"]))
              + m["C"] * np.log1p(z[None, :]))
        a = np.maximum(m["lam_lo"], np.exp(mu - L * m["sigma"]))
        b = np.minimum(m["lam_hi"], np.exp(mu + L * m["sigma"]))
        degenerate = b <= a
        half, mid = 0.5 * (b - a), 0.5 * (a + b)
        lam_k = mid[..., None] + half[..., None] * gl_t[None, None, :]
        W_k = half[..., None] * gl_w[None, None, :]
        D = phi_diff((np.log(m["lam_lo"]) - mu) / m["sigma"],
                     (np.log(m["lam_hi"]) - mu) / m["sigma"])
        d = (np.log(lam_k) - mu[..., None]) / m["sigma"]
        P = np.exp(-0.5 * d * d) / (np.sqrt(2 * np.pi) * m["sigma"] * lam_k * D[..., None])
        return lam_k, W_k, P, degenerate

    return stage


def run_sel_function(ref, lognormal):
    sys.path.insert(0, os.path.join(ref, "src", "modules", "sel_function"))
    sys.path.insert(0, ref)
    import sel_function as sf
    from y3_buzzard import prj_params as pp

    opts = dict(BINS)
    opts.update(ENVELOPE)
    opts["n_lnm"] = GRID["n_lnm"]
    opts["n_z_shared"] = GRID["n_z_shared"]
    opts["N_q"] = GRID["N_q"]
    cfg = sf.setup(Options(opts))
    block = Block()
    for k, v in HOD.items():
        block["cluster_mor", k] = v
    saved = sf._compute_lam_nodes_and_P_HOD
    try:
        if lognormal:
            sf._compute_lam_nodes_and_P_HOD = lognormal_stage(LOGNORMAL)
            i = int(np.argmin(np.abs(pp.PrjParams.default().z - 0.45)))
            base = pp.PrjParams.default()
            block["plob_ltr_params", "z"] = np.array([0.0, 2.0])
            const = dict(a_tau=base.a_tau[i], b_tau=base.b_tau[i], a_mu=0.0, b_mu=1.0,
                         a_sig=1.0, b_sig=0.1, a_fprj=0.0, b_fprj=0.1)
            for k, v in const.items():
                block["plob_ltr_params", k] = np.array([v, v])
        sf.execute(block, cfg)
    finally:
        sf._compute_lam_nodes_and_P_HOD = saved
    return (np.asarray(block["sel_function", "lnM"]), np.asarray(block["sel_function", "z"]),
            np.asarray(block["sel_function", "S_stack"]))


def _floats(text):
    return [float(x) for x in re.findall(r"[-+]?\d*\.\d+(?:[eE][-+]?\d+)?|[-+]?\d+(?:[eE][-+]?\d+)?", text)]


def _array_literal(src, name):
    m = re.search(r"std::vector<double>\s+" + name + r"\s*\{(.*?)\};", src, re.S)
    body = re.sub(r"//[^\n]*", "", m.group(1))
    return _floats(body)


def kats(ref):
    out = {}
    d = os.path.join(ref, "data")
    tab = np.loadtxt(os.path.join(d, "test_dv_do_dz.txt"))
    out["dv_do_dz"] = dict(z=tab[:, 0].tolist(), dv=tab[:, 1].tolist(),
                           dist_z=np.loadtxt(os.path.join(d, "z_da_test.txt")).tolist(),
                           dist_da=np.loadtxt(os.path.join(d, "d_a_test.txt")).tolist(),
                           om=0.3, ol=0.7, ok=0.0, h=0.7, epsrel=1e-3,
                           source="test/dv_do_dz_t.test.cc:15-53")
    tab = np.loadtxt(os.path.join(d, "test_Rmis.txt"), comments="#")
    out["roffset"] = dict(r=tab[:, 0].tolist(), p=tab[:, 1].tolist(), tau=0.15,
                          epsrel=1e-6, source="test/roffset_t.test.cc:10-55")
    tab = np.loadtxt(os.path.join(d, "test_int_zo_zt_des.txt"), comments="#")
    out["int_zo_zt"] = dict(zmin=tab[:, 0].tolist(), zmax=tab[:, 1].tolist(),
                            zt=tab[:, 2].tolist(), sigma=tab[:, 3].tolist(),
                            integral=tab[:, 4].tolist(), epsrel=1e-6, epsabs=1e-12,
                            source="test/int_zo_zt_des_t.test.cc:13-60")
    for name, fn, tol in (("dsigma_mis", "nfw_dsigma_mis.test.cu", 5e-3),
                          ("sigma_mis", "nfw_sigma_mis.test.cu", 1e-3)):
        src = open(os.path.join(ref, "test", fn)).read()
        out[name] = dict(r=_array_literal(src, "r"), rmis=_array_literal(src, "rmis"),
                         lnM=_array_literal(src, "lnMs"), answers=_array_literal(src, "answers"),
                         conc=4.0, omega_m=0.3, epsrel=tol, epsabs=1e-12,
                         source=f"test/{fn}:18-77")
    out["interp2d"] = dict(
        xs=[1.0, 2.0, 3.0], ys=[4.0, 5.0], f="3*x*y + 2*x + 4*y",
        cases=[[2.5, 4.5, 56.75]],
        clamp=[[0, 4.5, 1, 4.5], [4, 4.5, 3, 4.5], [2, 3, 2, 4], [2, 5.5, 2, 5],
               [0, 0, 1, 4], [4, 3, 3, 4], [0, 6, 1, 5], [4, 6, 3, 5]],
        source="test/interp_2d.test.cc:27-60")
    out["interp2d_linear"] = dict(xs=[1.0, 2.0, 3.0], ys=[1.0, 2.0, 3.0, 4.0],
                                  f="2*x + 3*y - 5", cases=[[2.5, 1.5, 4.5]],
                                  source="test/interp_2d.test.cc:92-114")
    out["interp1d"] = dict(xs=[1.0, 2.0, 3.0], f="x*x", cases=[[1.41421, 2.24263, 1e-4]],
                           throws=[[-5.0, 5.0, -10.0], [-5.0, 5.0, 10.0]],
                           source="test/interp_1d.test.cc:23-44")
    return out


def sigma_crit_inv_reference(ref):
    """Runs average_sigma_crit_inv.execute() of the reference on synthetic
    distances and n(z)."""
    fits = types.ModuleType("astropy.io.fits")
    io = types.ModuleType("astropy.io")
    io.fits = fits
    astropy = types.ModuleType("astropy")
    astropy.io = io
    sys.modules.update({"astropy": astropy, "astropy.io": io, "astropy.io.fits": fits})
    sys.path.insert(0, os.path.join(ref, "src", "modules", "average_sigma_crit_inv"))
    import average_sigma_crit_inv as sci_mod
    from y3_cluster_cpp_b200 import synthetic

    p = synthetic.fiducial()
    zs, pz = synthetic.source_nz()
    zl = np.linspace(0.05, 0.85, 64)
    block = Block()
    block["cosmological_parameters", "h0"] = p.h0
    block["photoz", "delta_z"] = 0.0
    block["distances", "z"] = p.tables["dist_z"]
    block["distances", "d_a"] = p.tables["dist_da"]
    sci_mod.execute(block, (zs, pz, zl, False))
    return dict(zs=zs, pz=pz, zl=zl, h0=p.h0, delta_z=0.0, dist_z=p.tables["dist_z"],
                dist_da=p.tables["dist_da"],
                sci=np.asarray(block["average_sigma_crit_inv", "sci_average"]))


def _write_mis_table(root, logx, logxmis, log_tab):
    d = os.path.join(root, "data", "nfw_off_center")
    os.makedirs(d, exist_ok=True)
    stem = os.path.join(d, "table_1000_1e-03_5e+03_")
    np.savetxt(stem + "gamma_logx.txt", logx, fmt="%.17g")
    np.savetxt(stem + "gamma_logxmis.txt", logxmis, fmt="%.17g")
    np.savetxt(stem + "log_deltasigma_gamma.txt", np.ravel(log_tab), fmt="%.17g")


def selgl_reference(ref):
    """Runs the reference's compiled SelGLCore / NumCountsSelGL /
    Shear1hMisSelGL on fixture inputs."""
    import subprocess

    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", "REF=" + ref],
                   check=True)
    import oracle as O
    from oracle import ref as R
    from y3_cluster_cpp_b200 import synthetic

    p = synthetic.fiducial()
    t = p.tables
    cosmo = dict(omega_m=p.om, omega_nu=0.0, omega_lambda=1.0 - p.om, omega_k=0.0, h0=p.h0,
                 hmf_s=0.0, hmf_q=1.0)
    out = dict(omega_m=p.om, h0=p.h0, **{"t_" + k: np.asarray(v) for k, v in t.items()})
    cfgs = dict(a=dict(n_lnm=64, n_z=32, zt_low=0.1, zt_high=0.8, lnm_low=29.9336,
                       lnm_high=35.69),
                b=dict(zt_low=0.2, zt_high=0.65, lnm_low=30.0, lnm_high=36.5))
    for name, c in cfgs.items():
        for k, v in c.items():
            out[f"cfg_{name}_{k}"] = v
    sels = {}
    for mor in ("hod", "lognormal"):
        g = np.load(os.path.join(HERE, f"sel_function_{mor}.npz"))
        sels[mor] = (g["lnM"], g["z"], g["S_stack"])
    for cname in ("a", "b"):
        for mor in ("hod", "lognormal"):
            out[f"counts_{cname}_{mor}"] = R.numcounts(cfgs[cname], cosmo, t, sels[mor])
    sci = (t["sci_z"], t["sci_val"])
    W, norm, eff, mu2, lx, lw = R.selgl_weights(cfgs["a"], cosmo, t, sels["lognormal"], sci)
    out.update(wsci_W=W, wsci_norm=norm, wsci_eff=eff, wsci_mu2=mu2, lnm_x=lx, lnm_w=lw)
    # Miscentring table stand-in on a subset of the shipped axes.
    axes = os.path.join(ref, "data", "nfw_off_center", "table_1000_1e-03_5e+03_gamma_")
    lx_full = np.loadtxt(axes + "logx.txt")
    lxm_full = np.loadtxt(axes + "logxmis.txt")
    logx = lx_full[np.r_[0:len(lx_full):8, len(lx_full) - 1]]
    logxmis = lxm_full[np.r_[0:len(lxm_full):5, len(lxm_full) - 1]]
    # Where x << x_mis the profile is below 1e-11 and the quadrature loses it
    # to cancellation (values of either sign); those corners, far from any
    # (R, R_mis, M) the fixtures query, are floored at 1e-30 before the log.
    tab = np.array([[np.log(max(O.dsigma_mis_unit(np.exp(a), np.exp(b)), 1e-30))
                     for a in logx] for b in logxmis])
    out.update(mis_logx=logx, mis_logxmis=logxmis, mis_log_tab=tab)
    # Centred DeltaSigma table haloModel/{r_sigma, lnM, dSigma_nfw}: the
    # analytic NFW (c = 4, rho = RHOC Omega_m) on 40 radii x 30 masses.
    r_sigma = np.logspace(-2, 1.7, 40)
    halo_lnM = np.linspace(29.9, 36.9, 30)
    rho = 2.77533742639e11 * p.om
    ds = np.array([[O.lib().y3o_nfw_norm(m, 4.0, rho) *
                    O.lib().y3o_nfw_dsigma_unit(r / O.lib().y3o_nfw_rs(m, 4.0, rho))
                    for r in r_sigma] for m in halo_lnM])
    halo = dict(r_sigma=r_sigma, lnM=halo_lnM, dSigma_nfw=ds)
    out.update(halo_r_sigma=r_sigma, halo_lnM=halo_lnM, halo_dSigma_nfw=ds)
    R15 = np.logspace(np.log10(0.1), np.log10(30.0), 15)
    out["R"] = R15
    with tempfile.TemporaryDirectory() as d:
        _write_mis_table(d, logx, logxmis, tab)
        out["shear_exact_cfg2"] = R.shear1h(cfgs["a"], cosmo, t, sels["lognormal"], sci, halo,
                                            R15, d, method=0,
                                            mis=dict(f_mis=0.2, tau_mis=0.17))
        out["shear_idea2_default"] = R.shear1h(cfgs["b"], cosmo, t, sels["hod"], sci, halo,
                                               R15, d, method=1)
        out["shear_exact_default_b"] = R.shear1h(cfgs["b"], cosmo, t, sels["hod"], sci, halo,
                                                 R15, d)
    return out


def likelihood_reference(ref):
    """Runs the reference's y3_buzzard/likelihood_cp.py setup/execute on a
    synthetic mock data vector (12 counts, 12 x 10 shear) with diagonal and
    dense inverse covariances, in linear and log space, for a set of seeded
    theory blocks (counts, 1-halo shear, projection shear)."""
    sys.path.insert(0, os.path.join(ref, "y3_buzzard"))
    import likelihood_cp as L

    rng = np.random.default_rng(7)
    nb, nr = 12, 10
    data_nc = rng.uniform(50.0, 500.0, nb)
    data_sh = rng.uniform(0.005, 0.05, nb * nr)
    A = rng.normal(size=(nb, nb))
    dense_nc = np.linalg.inv(A @ A.T + nb * np.diag(data_nc))
    B = rng.normal(size=(nb * nr, nb * nr))
    dense_sh = np.linalg.inv(1e-6 * (B @ B.T) + np.diag((0.1 * data_sh) ** 2))
    diag_nc = 1.0 / (0.1 * data_nc) ** 2
    diag_sh = 1.0 / (0.1 * data_sh) ** 2
    thr_nc = data_nc[None, :] * rng.uniform(0.8, 1.2, (4, nb))
    thr_nc[3, 5] = -1.0                      # a non-positive count: shear theory 0 there
    thr_s1h = (data_sh.reshape(nb, nr) * data_nc[:, None])[None] * rng.uniform(0.7, 1.1, (4, nb, nr))
    thr_prj = 0.1 * data_sh.reshape(nb, nr)[None] * rng.uniform(-1.0, 1.0, (4, nb, nr))
    out = dict(data_nc=data_nc, data_sh=data_sh, dense_nc=dense_nc, dense_sh=dense_sh,
               diag_nc=diag_nc, diag_sh=diag_sh, thr_nc=thr_nc, thr_s1h=thr_s1h,
               thr_prj=thr_prj)
    with tempfile.TemporaryDirectory() as d:
        for form in ("diag", "dense"):
            fname = os.path.join(d, f"mock_{form}.npz")
            ic_nc = diag_nc if form == "diag" else dense_nc
            ic_sh = diag_sh if form == "diag" else dense_sh
            np.savez(fname, data_NC=data_nc, invcov_NC=ic_nc, data_Shear=data_sh,
                     invcov_Shear=ic_sh)
            for log_space in (False, True):
                cfg = L.setup(_OptionsIndex(filename=fname, log_space=log_space,
                                            verbose=False))
                vals = []
                for t in range(4):
                    block = Block()
                    block["numcountssel", "vals"] = thr_nc[t]
                    block["shear1hmissel", "vals"] = thr_s1h[t].ravel()
                    block["shear_prj", "vals"] = thr_prj[t].ravel()
                    L.execute(block, cfg)
                    vals.append(block["likelihoods", "likelihoods_like"])
                out[f"logL_{form}_{'log' if log_space else 'lin'}"] = np.array(vals)
    return out


def prj_reference(ref):
    """Runs the reference's compiled ShearPrjFrozenPhysics on the fiducial
    synthetic tables: 12 (richness, z_obs) slices x 10 radii 0.2-5 Mpc/h,
    default options.  The single-kernel miscentring table it reads is missing
    from the snapshot; the fixture carries a stand-in on every 8th ln x and
    every 5th ln x_mis node of the shipped single-kernel axis files, filled
    by the oracle's ring average of the NFW profile (256 GL nodes)."""
    import oracle as O
    from oracle import ref as R
    from y3_cluster_cpp_b200 import synthetic

    p = synthetic.fiducial()
    prj = synthetic.prj_tables(p, n_r=120)
    cosmo = dict(omega_m=p.om, omega_nu=0.0, omega_lambda=1.0 - p.om, omega_k=0.0, h0=p.h0,
                 hmf_s=0.0, hmf_q=1.0)
    axes = os.path.join(ref, "data", "nfw_off_center", "table_1000_1e-03_5e+03_single_")
    lx_full = np.loadtxt(axes + "logx.txt")
    lxm_full = np.loadtxt(axes + "logxmis.txt")
    logx = lx_full[np.r_[0:len(lx_full):8, len(lx_full) - 1]]
    logxmis = lxm_full[np.r_[0:len(lxm_full):5, len(lxm_full) - 1]]
    tab = np.array([[np.log(max(O.lib().y3o_dsigma_single_unit(np.exp(a), np.exp(b), 256), 1e-30))
                     for a in logx] for b in logxmis])
    R10 = np.logspace(np.log10(0.2), np.log10(5.0), 10)
    grid = dict(lambda_bin=np.repeat(np.tile(np.arange(4), 3), 10).astype(float),
                zo_low=np.repeat(np.repeat([0.2, 0.35, 0.5], 4), 10),
                zo_high=np.repeat(np.repeat([0.35, 0.5, 0.65], 4), 10),
                radii=np.tile(R10, 12))
    cfg = dict(zt_low=0.1, zt_high=0.8, lnm_low=np.log(1e13), lnm_high=np.log(10 ** 15.5))
    out = dict(omega_m=p.om, h0=p.h0, **{"t_" + k: np.asarray(v) for k, v in p.tables.items()},
               **{"prj_" + k: np.asarray(v) for k, v in prj.items()},
               **{"gp_" + k: v for k, v in grid.items()},
               **{"cfg_" + k: v for k, v in cfg.items()},
               single_logx=logx, single_logxmis=logxmis, single_log_tab=tab)
    with tempfile.TemporaryDirectory() as d:
        dd = os.path.join(d, "data", "nfw_off_center")
        os.makedirs(dd)
        stem = os.path.join(dd, "table_1000_1e-03_5e+03_")
        np.savetxt(stem + "single_logx.txt", logx, fmt="%.17g")
        np.savetxt(stem + "single_logxmis.txt", logxmis, fmt="%.17g")
        np.savetxt(stem + "log_deltasigma_single.txt", np.ravel(tab), fmt="%.17g")
        out["vals"] = R.shear_prj_frozen(cfg, cosmo, p.tables, prj, grid, d)
        out["vals_no_omega"] = R.shear_prj_frozen(dict(cfg, include_omega_z=0, n_lnm=16,
                                                       n_per_seg=8), cosmo, p.tables, prj,
                                                  grid, d)
    return out


BSEL_HOD = dict(log10_Mmin=11.7, log10_M1=12.9, alpha=0.85, epsilon=0.2, sigma_lambda=0.2)


def bsel_reference(ref):
    """Runs the reference's compiled P_operator (src/models/p_operator_t.hh,
    module b_sel_marg) on the fiducial synthetic tables and HOD parameters:
    default node counts on 12 (z_obs bin, richness bin) points, and reduced,
    odd node counts (theta split 3 + 4) on 16 points that add a low-z_obs bin
    and a second sample with its own z_pivot and sigma_lambda."""
    from oracle import ref as R
    from y3_cluster_cpp_b200 import synthetic

    p = synthetic.fiducial()
    prj = synthetic.prj_tables(p, n_r=120)
    cosmo = dict(omega_m=p.om, omega_nu=0.0, omega_lambda=1.0 - p.om, omega_k=0.0, h0=p.h0,
                 hmf_s=0.0, hmf_q=1.0)
    grid = dict(zo_low=np.repeat([0.2, 0.35, 0.5], 4), zo_high=np.repeat([0.35, 0.5, 0.65], 4),
                lambda_bin=np.tile(np.arange(4), 3).astype(float))
    grid2 = dict(zo_low=np.repeat([0.1, 0.2, 0.35, 0.5], 4),
                 zo_high=np.repeat([0.2, 0.35, 0.5, 0.65], 4),
                 lambda_bin=np.tile(np.arange(4), 4).astype(float))
    cfg = dict(lnm_low=np.log(1e13), lnm_high=np.log(10 ** 15.5))
    cfg2 = dict(cfg, n_lt=24, n_zring=9, n_zouter=15, n_lnm=16, n_theta=7, n_zt_ref=40)
    hod2 = dict(BSEL_HOD, z_pivot=0.3, sigma_lambda=0.3, log10_M1=13.1)
    # Degenerate node counts (one node per axis; two) on edge bins: a narrow
    # low-z_obs bin and one whose line of sight leaves the reference z grid.
    grid3 = dict(zo_low=np.array([0.1, 0.5, 0.8, 0.2]), zo_high=np.array([0.12, 0.65, 0.86, 0.35]),
                 lambda_bin=np.array([0.0, 3.0, 1.0, 2.0]))
    cfg3 = dict(cfg, n_lt=1, n_zring=1, n_zouter=1, n_lnm=1, n_theta=1, n_zt_ref=2)
    cfg4 = dict(cfg, n_lt=3, n_zring=2, n_zouter=2, n_lnm=2, n_theta=2, n_zt_ref=5)
    return dict(omega_m=p.om, h0=p.h0, **{"t_" + k: np.asarray(v) for k, v in p.tables.items()},
                **{"prj_" + k: np.asarray(v) for k, v in prj.items()},
                **{"gp_" + k: v for k, v in grid.items()},
                **{"gp2_" + k: v for k, v in grid2.items()},
                **{"cfg_" + k: v for k, v in cfg.items()},
                **{"cfg2_" + k: v for k, v in cfg2.items()},
                **{"hod_" + k: v for k, v in BSEL_HOD.items()},
                **{"hod2_" + k: v for k, v in hod2.items()},
                **{"gp3_" + k: v for k, v in grid3.items()},
                **{"cfg3_" + k: v for k, v in cfg3.items()},
                **{"cfg4_" + k: v for k, v in cfg4.items()},
                vals3=R.bsel_marg(cfg3, cosmo, p.tables, prj, BSEL_HOD, grid3),
                vals4=R.bsel_marg(cfg4, cosmo, p.tables, prj, BSEL_HOD, grid3),
                vals=R.bsel_marg(cfg, cosmo, p.tables, prj, BSEL_HOD, grid),
                vals2=np.stack([R.bsel_marg(cfg2, cosmo, p.tables, prj, h, grid2)
                                for h in (BSEL_HOD, hod2)]))


class _OptionsIndex(dict):
    """options[section, key] and options.get_bool(section, key, default)."""

    def __getitem__(self, key):
        return dict.__getitem__(self, key[1])

    def get_bool(self, section, key, default=False):
        return bool(self.get(key, default))


def main(ref=None, *only):
    """Writes every fixture, or with names after the checkout path (e.g.
    `bsel_ref`) only those."""
    if ref is None:
        raise SystemExit("usage: make_golden.py <reference-checkout> [fixture ...]")
    if only:
        for name in only:
            fn = {"bsel_ref": bsel_reference, "prj_ref": prj_reference,
                  "selgl_ref": selgl_reference, "likelihood_ref": likelihood_reference,
                  "sigma_crit_inv": sigma_crit_inv_reference}[name]
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **fn(ref))
        print("wrote", ", ".join(only), "to", HERE)
        return
    _install_cosmosis_stub()
    with tempfile.TemporaryDirectory():
        lnm, z, S = run_sel_function(ref, lognormal=False)
        np.savez(os.path.join(HERE, "sel_function_hod.npz"), lnM=lnm, z=z, S_stack=S,
                 **{k: np.asarray(v) for k, v in BINS.items()},
                 **{k: np.asarray(v) for k, v in ENVELOPE.items()},
                 **{k: np.asarray(v) for k, v in GRID.items()},
                 **{"hod_" + k: np.asarray(v) for k, v in HOD.items()})
        lnm, z, S = run_sel_function(ref, lognormal=True)
        np.savez(os.path.join(HERE, "sel_function_lognormal.npz"), lnM=lnm, z=z, S_stack=S,
                 **{k: np.asarray(v) for k, v in BINS.items()},
                 **{k: np.asarray(v) for k, v in ENVELOPE.items()},
                 **{k: np.asarray(v) for k, v in GRID.items()},
                 **{"ln_" + k: np.asarray(v) for k, v in LOGNORMAL.items()})
    with open(os.path.join(HERE, "kats.json"), "w") as f:
        json.dump(kats(ref), f, indent=1)
    np.savez_compressed(os.path.join(HERE, "sigma_crit_inv.npz"), **sigma_crit_inv_reference(ref))
    np.savez_compressed(os.path.join(HERE, "selgl_ref.npz"), **selgl_reference(ref))
    np.savez_compressed(os.path.join(HERE, "likelihood_ref.npz"), **likelihood_reference(ref))
    np.savez_compressed(os.path.join(HERE, "prj_ref.npz"), **prj_reference(ref))
    np.savez_compressed(os.path.join(HERE, "bsel_ref.npz"), **bsel_reference(ref))
    print("wrote golden fixtures to", HERE)


if __name__ == "__main__":
    main(*sys.argv[1:])
