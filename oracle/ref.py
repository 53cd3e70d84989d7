"""ctypes bindings for ``oracle/_ref/libselgl_ref.so`` -- TEST INFRASTRUCTURE.

That library is the reference's own ``SelGLCore`` / ``NumCountsSelGL`` /
``Shear1hMisSelGL`` (src/models/n_operator_sel_gl_t.hh:75-361) compiled from
the reference's sources against the shims in ``oracle/ref_shim/`` by
``make -C oracle ref`` (see ``oracle/Makefile``).  It is built only where the
reference checkout exists, is never committed, and travels to GPU hosts with
the rest of the built artefacts.  Only tests, golden-vector generation and the
reference arm of ``bench.py`` may use it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libselgl_ref.so")
_lib = None

D = C.c_double
I = C.c_int
PD = C.POINTER(C.c_double)


class Cfg(C.Structure):
    _fields_ = [("n_lnm", I), ("n_z", I), ("zt_low", D), ("zt_high", D),
                ("lnm_low", D), ("lnm_high", D)]


class Sample(C.Structure):
    _fields_ = [("omega_m", D), ("omega_nu", D), ("omega_lambda", D), ("omega_k", D),
                ("h0", D), ("hmf_s", D), ("hmf_q", D),
                ("n_hm", I), ("n_hz", I), ("m_h", PD), ("hmf_z", PD), ("dndlnmh", PD),
                ("nd", I), ("dist_z", PD), ("dist_da", PD),
                ("n_sci", I), ("sci_z", PD), ("sci_val", PD),
                ("n_bins", I), ("n_sel_z", I), ("n_sel_lnm", I),
                ("sel_lnm", PD), ("sel_z", PD), ("S_stack", PD),
                ("n_rs", I), ("n_hl", I), ("r_sigma", PD), ("halo_lnM", PD),
                ("dsigma_nfw", PD),
                ("has_f_mis", I), ("has_tau_mis", I), ("f_mis", D), ("tau_mis", D)]


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("reference library not built: run `make -C oracle ref` "
                               "where the reference checkout exists")
        L = C.CDLL(LIB_PATH)
        L.y3r_selgl_weights.argtypes = [C.POINTER(Cfg), C.POINTER(Sample), I,
                                        PD, PD, PD, PD, PD, PD, C.c_char_p, I]
        L.y3r_numcounts.argtypes = [C.POINTER(Cfg), C.POINTER(Sample), PD, C.c_char_p, I]
        L.y3r_shear1h.argtypes = [C.POINTER(Cfg), I, D, I, PD, C.c_char_p,
                                  C.POINTER(Sample), I, PD, PD, C.c_char_p, I]
        L.y3r_nfw_dsigma_mis.argtypes = [C.c_char_p, D, I, PD, PD, PD, PD, C.c_char_p, I]
        _lib = L
    return _lib


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _p(a):
    return None if a is None else a.ctypes.data_as(PD)


class _Inputs:
    """Keeps the arrays a Sample points into alive."""

    def __init__(self, cosmo, tables, sel, sci=None, halo=None, mis=None):
        self.keep = []

        def arr(a):
            a = _f64(a)
            self.keep.append(a)
            return a

        t = tables
        mh, hz, dn = arr(t["hmf_m_h"]), arr(t["hmf_z"]), arr(t["dndlnmh"])
        dz, da = arr(t["dist_z"]), arr(t["dist_da"])
        sl, sz, S = arr(sel[0]), arr(sel[1]), arr(sel[2])
        s = Sample()
        for k in ("omega_m", "omega_nu", "omega_lambda", "omega_k", "h0", "hmf_s", "hmf_q"):
            setattr(s, k, float(cosmo[k]))
        s.n_hm, s.n_hz, s.m_h, s.hmf_z, s.dndlnmh = len(mh), len(hz), _p(mh), _p(hz), _p(dn)
        s.nd, s.dist_z, s.dist_da = len(dz), _p(dz), _p(da)
        if sci is not None:
            scz, scv = arr(sci[0]), arr(sci[1])
            s.n_sci, s.sci_z, s.sci_val = len(scz), _p(scz), _p(scv)
        s.n_bins, s.n_sel_z, s.n_sel_lnm = S.shape[0], S.shape[1], S.shape[2]
        s.sel_lnm, s.sel_z, s.S_stack = _p(sl), _p(sz), _p(S)
        if halo is not None:
            rs, hl, ds = arr(halo["r_sigma"]), arr(halo["lnM"]), arr(halo["dSigma_nfw"])
            s.n_rs, s.n_hl, s.r_sigma, s.halo_lnM, s.dsigma_nfw = (
                len(rs), len(hl), _p(rs), _p(hl), _p(ds))
        if mis is not None:
            if "f_mis" in mis:
                s.has_f_mis, s.f_mis = 1, float(mis["f_mis"])
            if "tau_mis" in mis:
                s.has_tau_mis, s.tau_mis = 1, float(mis["tau_mis"])
        self.sample = s


def _cfg(cfg):
    return Cfg(int(cfg.get("n_lnm", 0)), int(cfg.get("n_z", 0)), float(cfg["zt_low"]),
               float(cfg["zt_high"]), float(cfg["lnm_low"]), float(cfg["lnm_high"]))


def _check(rc, err):
    if rc:
        raise RuntimeError("reference: " + err.value.decode(errors="replace"))


def selgl_weights(cfg, cosmo, tables, sel, sci=None):
    """SelGLCore::build_weights; returns W [bins, n_lnm], norm, lnm_eff, mu2,
    lnm_x, lnm_w.  include_sci follows whether sci is given."""
    c = _cfg(cfg)
    inp = _Inputs(cosmo, tables, sel, sci)
    nb = inp.sample.n_bins
    nm = c.n_lnm if c.n_lnm > 0 else 96
    W = np.empty((nb, nm))
    norm, eff, mu2 = np.empty(nb), np.empty(nb), np.empty(nb)
    lx, lw = np.empty(nm), np.empty(nm)
    err = C.create_string_buffer(512)
    rc = lib().y3r_selgl_weights(C.byref(c), C.byref(inp.sample), int(sci is not None),
                                 _p(W), _p(norm), _p(eff), _p(mu2), _p(lx), _p(lw), err, 512)
    _check(rc, err)
    return W, norm, eff, mu2, lx, lw


def numcounts(cfg, cosmo, tables, sel):
    """NumCountsSelGL: numcountssel/vals for every bin."""
    c = _cfg(cfg)
    inp = _Inputs(cosmo, tables, sel)
    out = np.empty(inp.sample.n_bins)
    err = C.create_string_buffer(512)
    _check(lib().y3r_numcounts(C.byref(c), C.byref(inp.sample), _p(out), err, 512), err)
    return out


def shear1h(cfg, cosmo, tables, sel, sci, halo, R, data_root, method=-1, stencil_h=-1.0,
            lob_centers=None, mis=None):
    """Shear1hMisSelGL: shear1hmissel/vals, bin slow and R fast.  data_root
    holds data/nfw_off_center/ with the gamma-kernel table files."""
    c = _cfg(cfg)
    inp = _Inputs(cosmo, tables, sel, sci, halo, mis)
    R = _f64(R)
    lob = None if lob_centers is None else _f64(lob_centers)
    out = np.empty(inp.sample.n_bins * len(R))
    err = C.create_string_buffer(512)
    rc = lib().y3r_shear1h(C.byref(c), int(method), float(stencil_h),
                           0 if lob is None else len(lob), _p(lob),
                           str(data_root).encode(), C.byref(inp.sample), len(R), _p(R),
                           _p(out), err, 512)
    _check(rc, err)
    return out


def nfw_dsigma_mis(data_root, omega_m, r, rmis, lnM):
    r, rmis, lnM = _f64(r), _f64(rmis), _f64(lnM)
    out = np.empty(len(r))
    err = C.create_string_buffer(512)
    rc = lib().y3r_nfw_dsigma_mis(str(data_root).encode(), omega_m, len(r), _p(r), _p(rmis),
                                  _p(lnM), _p(out), err, 512)
    _check(rc, err)
    return out


class PrjCfg(C.Structure):
    _fields_ = [("n_lnm", I), ("n_per_seg", I), ("n_zring", I), ("n_zouter", I),
                ("zt_low", D), ("zt_high", D), ("lnm_low", D), ("lnm_high", D),
                ("R_max_cMpch", D), ("include_omega_z", I), ("n_lob", I), ("lob_centers", PD),
                ("n_gp", I), ("lambda_bin", PD), ("zo_low", PD), ("zo_high", PD),
                ("radii", PD)]


class PrjSample(C.Structure):
    _fields_ = [("nd", I), ("dist_dc", PD), ("n_hl", I), ("n_hz", I), ("halo_lnM", PD),
                ("halo_z", PD), ("bias", PD), ("n_xr", I), ("n_xz", I), ("xi_r", PD),
                ("xi_z", PD), ("xi_nl", PD), ("n_blob", I), ("n_bzob", I), ("bsel_lob", PD),
                ("bsel_zob", PD), ("b_small", PD), ("b_large", PD)]


def shear_prj_frozen(cfg, cosmo, tables, prj, grid, data_root):
    """ShearPrjFrozenPhysics (sigma_prj_frozen_t.hh): cfg dict (zt_low,
    zt_high, lnm_low, lnm_high and optional n_lnm, n_per_seg, n_zring,
    n_zouter, R_max_cMpch, include_omega_z, lob_centers); grid dict of the
    grid-point arrays lambda_bin, zo_low, zo_high, radii; prj the tables of
    synthetic.prj_tables.  Returns [n_gp, 9]."""
    L = lib()
    if not hasattr(L, "_prj_declared"):
        L.y3r_shear_prj_frozen.argtypes = [C.POINTER(PrjCfg), C.c_char_p, C.POINTER(Sample),
                                           C.POINTER(PrjSample), PD, C.c_char_p, I]
        L._prj_declared = True
    keep = []

    def arr(a):
        a = _f64(a)
        keep.append(a)
        return a

    c = PrjCfg()
    for k, d in (("n_lnm", 0), ("n_per_seg", 0), ("n_zring", 0), ("n_zouter", 0)):
        setattr(c, k, int(cfg.get(k, d)))
    for k in ("zt_low", "zt_high", "lnm_low", "lnm_high"):
        setattr(c, k, float(cfg[k]))
    c.R_max_cMpch = float(cfg.get("R_max_cMpch", -1.0))
    c.include_omega_z = int(cfg.get("include_omega_z", -1))
    if cfg.get("lob_centers") is not None:
        lc = arr(cfg["lob_centers"])
        c.n_lob, c.lob_centers = len(lc), _p(lc)
    gp = {k: arr(grid[k]) for k in ("lambda_bin", "zo_low", "zo_high", "radii")}
    c.n_gp = len(gp["radii"])
    for k, v in gp.items():
        setattr(c, k, _p(v))
    inp = _Inputs(cosmo, tables, (np.array([0.0, 1.0]), np.array([0.0, 1.0]),
                                  np.zeros((1, 2, 2))),
                  sci=(tables["sci_z"], tables["sci_val"]) if "sci_z" in tables else None)
    ps = PrjSample()
    dc = arr(prj["dist_dc"])
    ps.nd, ps.dist_dc = len(dc), _p(dc)
    hl, hz, bi = arr(prj["halo_lnM"]), arr(prj["halo_z"]), arr(prj["bias"])
    ps.n_hl, ps.n_hz, ps.halo_lnM, ps.halo_z, ps.bias = len(hl), len(hz), _p(hl), _p(hz), _p(bi)
    xr, xz, xn = arr(prj["xi_r"]), arr(prj["xi_z"]), arr(prj["xi_nl"])
    ps.n_xr, ps.n_xz, ps.xi_r, ps.xi_z, ps.xi_nl = len(xr), len(xz), _p(xr), _p(xz), _p(xn)
    bl, bz = arr(prj["bsel_lob"]), arr(prj["bsel_zob"])
    bs, bg = arr(prj["b_small"]), arr(prj["b_large"])
    ps.n_blob, ps.n_bzob = len(bl), len(bz)
    ps.bsel_lob, ps.bsel_zob, ps.b_small, ps.b_large = _p(bl), _p(bz), _p(bs), _p(bg)
    out = np.empty((c.n_gp, 9))
    err = C.create_string_buffer(512)
    rc = L.y3r_shear_prj_frozen(C.byref(c), str(data_root).encode(), C.byref(inp.sample),
                                C.byref(ps), _p(out), err, 512)
    _check(rc, err)
    return out


class BselCfg(C.Structure):
    _fields_ = [("n_lt", I), ("n_zring", I), ("n_zouter", I), ("n_lnm", I), ("n_theta", I),
                ("n_zt_ref", I), ("zt_ref_low", D), ("zt_ref_high", D), ("lnm_low", D),
                ("lnm_high", D), ("n_gp", I), ("zo_low", PD), ("zo_high", PD),
                ("lambda_bin", PD)]


class Hod(C.Structure):
    _fields_ = [("log10_Mmin", D), ("log10_M1", D), ("alpha", D), ("epsilon", D),
                ("sigma_lambda", D), ("z_pivot", D), ("has_z_pivot", I)]


def bsel_marg(cfg, cosmo, tables, prj, hod, grid):
    """P_operator (p_operator_t.hh), module label b_sel_marg: cfg dict
    (lnm_low, lnm_high and optional n_lt, n_zring, n_zouter, n_lnm, n_theta,
    n_zt_ref, zt_ref_low, zt_ref_high); hod dict (log10_Mmin, log10_M1, alpha,
    epsilon, sigma_lambda, optional z_pivot); grid dict of the wall-grid
    arrays zo_low, zo_high, lambda_bin; prj the tables of synthetic.prj_tables
    (distances/d_c, haloModel bias, xi_nl).  Returns [n_gp, 3] = (P1, I1, J)."""
    L = lib()
    if not hasattr(L, "_bsel_declared"):
        L.y3r_bsel_marg.argtypes = [C.POINTER(BselCfg), C.POINTER(Sample), C.POINTER(PrjSample),
                                    C.POINTER(Hod), PD, C.c_char_p, I]
        L._bsel_declared = True
    keep = []

    def arr(a):
        a = _f64(a)
        keep.append(a)
        return a

    c = BselCfg()
    for k in ("n_lt", "n_zring", "n_zouter", "n_lnm", "n_theta", "n_zt_ref"):
        setattr(c, k, int(cfg.get(k, 0)))
    c.zt_ref_low = float(cfg.get("zt_ref_low", -1.0))
    c.zt_ref_high = float(cfg.get("zt_ref_high", -1.0))
    c.lnm_low, c.lnm_high = float(cfg["lnm_low"]), float(cfg["lnm_high"])
    gp = {k: arr(grid[k]) for k in ("zo_low", "zo_high", "lambda_bin")}
    c.n_gp = len(gp["zo_low"])
    for k, v in gp.items():
        setattr(c, k, _p(v))
    inp = _Inputs(cosmo, tables, (np.array([0.0, 1.0]), np.array([0.0, 1.0]),
                                  np.zeros((1, 2, 2))))
    ps = PrjSample()
    dc = arr(prj["dist_dc"])
    ps.nd, ps.dist_dc = len(dc), _p(dc)
    hl, hz, bi = arr(prj["halo_lnM"]), arr(prj["halo_z"]), arr(prj["bias"])
    ps.n_hl, ps.n_hz, ps.halo_lnM, ps.halo_z, ps.bias = len(hl), len(hz), _p(hl), _p(hz), _p(bi)
    xr, xz, xn = arr(prj["xi_r"]), arr(prj["xi_z"]), arr(prj["xi_nl"])
    ps.n_xr, ps.n_xz, ps.xi_r, ps.xi_z, ps.xi_nl = len(xr), len(xz), _p(xr), _p(xz), _p(xn)
    h = Hod(float(hod["log10_Mmin"]), float(hod["log10_M1"]), float(hod["alpha"]),
            float(hod["epsilon"]), float(hod["sigma_lambda"]), float(hod.get("z_pivot", 0.0)),
            int("z_pivot" in hod))
    out = np.empty((c.n_gp, 3))
    err = C.create_string_buffer(512)
    rc = L.y3r_bsel_marg(C.byref(c), C.byref(inp.sample), C.byref(ps), C.byref(h), _p(out),
                         err, 512)
    _check(rc, err)
    return out
