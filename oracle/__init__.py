"""FP64 CPU oracle for the cluster-observable hot path -- TEST INFRASTRUCTURE.

Thin ctypes bindings over ``oracle/_build/liby3o.so`` (built from
``oracle/y3o.c`` by ``oracle/Makefile``).  The C file restates the reference
algorithm (estevesjh/y3_cluster_cpp) with a file:line citation per function.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker or the timed CPU
baseline; the product library ``y3_cluster_cpp_b200`` never touches it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liby3o.so")
_lib = None

D = C.c_double
I = C.c_int
PD = C.POINTER(C.c_double)

MOR_HOD = 0
MOR_LOGNORMAL = 1


def build() -> str:
    """Compile the oracle shared library (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


class Cosmo(C.Structure):
    _fields_ = [(n, D) for n in ("om", "ol", "ok", "h0", "onu", "hmf_s", "hmf_q")]


class DirectGrid(C.Structure):
    _fields_ = [("n_m", I), ("n_z", I), ("n_t", I), ("n_o", I), ("n_zo", I),
                ("lnm_lo", D), ("lnm_hi", D), ("zt_lo", D), ("zt_hi", D),
                ("lam_t_lo", D), ("lam_t_hi", D),
                ("n_lam_bins", I), ("n_z_bins", I),
                ("lam_edges", PD), ("zob_edges", PD), ("sz0", D), ("sz_bin", PD)]


class Lognormal(C.Structure):
    _fields_ = [(n, D) for n in ("A", "B", "C", "sigma", "Mpiv")]


class ShearOpts(C.Structure):
    _fields_ = [("n_R", I), ("R", PD), ("f_mis", D), ("tau_mis", D),
                ("lob_centers", PD), ("c0", D), ("c_slope", D), ("c_pivot", D),
                ("n_theta", I), ("n_s", I), ("s_max", D),
                ("n_sci", I), ("sci_z", PD), ("sci_val", PD)]


def _declare(L):
    L.y3o_gl_nodes.argtypes = [D, D, I, PD, PD]
    L.y3o_interp1d.argtypes = [PD, PD, I, D, PD]
    L.y3o_interp1d_clamp.argtypes = [PD, PD, I, D]
    L.y3o_interp1d_clamp.restype = D
    L.y3o_interp2d.argtypes = [PD, I, PD, I, PD, D, D]
    L.y3o_interp2d.restype = D
    L.y3o_interp2d_clamp.argtypes = [PD, I, PD, I, PD, D, D]
    L.y3o_interp2d_clamp.restype = D
    L.y3o_ez.argtypes = [D, D, D, D]
    L.y3o_ez.restype = D
    L.y3o_dv_do_dz.argtypes = [PD, PD, I, D, D, D, D, D, PD]
    L.y3o_omega_z_des.argtypes = [D]
    L.y3o_omega_z_des.restype = D
    for name in ("y3o_phi", "y3o_erfcx"):
        getattr(L, name).argtypes = [D]
        getattr(L, name).restype = D
    L.y3o_emg_tail.argtypes = [D, D, D, D]
    L.y3o_emg_tail.restype = D
    for name in ("y3o_cdf_lob", "y3o_pdf_lob"):
        getattr(L, name).argtypes = [D, D, D, D, D]
        getattr(L, name).restype = D
    L.y3o_kj.argtypes = [D, D, D, D]
    L.y3o_kj.restype = D
    L.y3o_p_hod.argtypes = [D, D, D, PD]
    L.y3o_p_hod.restype = D
    L.y3o_sel_function.argtypes = [I, PD, PD, PD, PD, PD, D, D, D, D, I, I, I,
                                   I, PD, I, PD, PD, PD, PD, PD]
    L.y3o_selgl_weights.argtypes = [I, I, D, D, D, D, C.POINTER(Cosmo),
                                    I, PD, I, PD, PD, I, PD, PD, I, PD, PD,
                                    I, I, PD, I, PD, PD, PD, PD, PD, PD]
    for name in ("y3o_nfw_sigma_unit", "y3o_nfw_dsigma_unit"):
        getattr(L, name).argtypes = [D]
        getattr(L, name).restype = D
    for name in ("y3o_nfw_norm", "y3o_nfw_rs"):
        getattr(L, name).argtypes = [D, D, D]
        getattr(L, name).restype = D
    for name in ("y3o_dsigma_mis_unit", "y3o_sigma_mis_unit"):
        getattr(L, name).argtypes = [D, D, I, I, D]
        getattr(L, name).restype = D
    L.y3o_dsigma_single_unit.argtypes = [D, D, I]
    L.y3o_dsigma_single_unit.restype = D
    L.y3o_roffset.argtypes = [D, D]
    L.y3o_roffset.restype = D
    L.y3o_shear1h_mis.argtypes = [I, PD, PD, I, PD, I, PD, D, D, I, PD, D, D,
                                  I, PD, I, PD, PD, I, I, D, PD]
    L.y3o_sigma_crit_inv.argtypes = [I, PD, I, PD, PD, D, D, I, PD, PD, PD]
    L.y3o_dsigma_mis_tab.argtypes = [D, D, D, D, D, D, I, PD, I, PD, PD]
    L.y3o_dsigma_mis_tab.restype = D
    L.y3o_shear1h_mis_tab.argtypes = [I, PD, PD, I, PD, PD, PD, PD, I, D, I, PD, D, D,
                                      I, PD, D, D, I, PD, I, PD, PD, I, PD, I, PD, PD, PD]
    L.y3o_loglike.argtypes = [I, I, PD, PD, PD, I, PD, PD, I, PD, PD, I]
    L.y3o_loglike.restype = D
    L.y3o_direct_eval.argtypes = [C.POINTER(DirectGrid), I, PD, PD,
                                  C.POINTER(Lognormal), C.POINTER(Cosmo),
                                  I, PD, I, PD, PD, I, PD, PD,
                                  C.POINTER(ShearOpts), PD, PD, PD]


def _p(a):
    """Pointer to a C-contiguous float64 array (None -> NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(PD)


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


# ---- scalar helpers --------------------------------------------------------

def gl_nodes(a, b, n):
    x = np.empty(n)
    w = np.empty(n)
    lib().y3o_gl_nodes(a, b, n, _p(x), _p(w))
    return x, w


def interp1d(xs, ys, x):
    xs, ys = _f64(xs), _f64(ys)
    out = D()
    rc = lib().y3o_interp1d(_p(xs), _p(ys), len(xs), x, C.byref(out))
    if rc:
        raise ValueError("argument out of range in interp1d")
    return out.value


def interp2d_clamp(xs, ys, zs, x, y):
    xs, ys, zs = _f64(xs), _f64(ys), _f64(zs)
    return lib().y3o_interp2d_clamp(_p(xs), len(xs), _p(ys), len(ys), _p(zs), x, y)


def dv_do_dz(dist_z, dist_da, om, ol, ok, h, z):
    dz, da = _f64(dist_z), _f64(dist_da)
    out = D()
    if lib().y3o_dv_do_dz(_p(dz), _p(da), len(dz), om, ol, ok, h, z, C.byref(out)):
        raise ValueError("z outside distances table")
    return out.value


def scalar(name, *args):
    return getattr(lib(), name)(*args)


def p_hod(ltr, lnM, z, hod):
    h = _f64(hod)
    return lib().y3o_p_hod(ltr, lnM, z, _p(h))


# ---- sel_function ----------------------------------------------------------

def sel_function(cfg, mor_kind, mor, plob_z, plob_coef):
    """S_stack producer.  cfg keys: lam_min, lam_max, zob_min, zob_max,
    sigma_z (per bin), zt_low, zt_high, lnm_low, lnm_high, n_lnm, n_z, n_q."""
    arr = {k: _f64(cfg[k]) for k in ("lam_min", "lam_max", "zob_min", "zob_max", "sigma_z")}
    nb = len(arr["lam_min"])
    n_lnm, n_z, n_q = int(cfg["n_lnm"]), int(cfg["n_z"]), int(cfg["n_q"])
    lnm = np.empty(n_lnm)
    z = np.empty(n_z)
    S = np.empty((nb, n_z, n_lnm))
    mor, pz, pc = _f64(mor), _f64(plob_z), _f64(plob_coef)
    lib().y3o_sel_function(nb, _p(arr["lam_min"]), _p(arr["lam_max"]),
                           _p(arr["zob_min"]), _p(arr["zob_max"]), _p(arr["sigma_z"]),
                           cfg["zt_low"], cfg["zt_high"], cfg["lnm_low"], cfg["lnm_high"],
                           n_lnm, n_z, n_q, mor_kind, _p(mor), len(pz), _p(pz), _p(pc),
                           _p(lnm), _p(z), _p(S))
    return lnm, z, S


def cosmo(om, h0, ol=None, ok=0.0, onu=0.0, hmf_s=0.0, hmf_q=1.0):
    return Cosmo(om, 1.0 - om - ok if ol is None else ol, ok, h0, onu, hmf_s, hmf_q)


def selgl_weights(n_lnm, n_z, zt_lo, zt_hi, lnm_lo, lnm_hi, cz, tables, sel,
                  sci=None):
    """SelGLCore::build_weights.  tables: dict with hmf_m_h, hmf_z, dndlnmh
    (n_hz, n_hm), dist_z, dist_da.  sel: (lnM, z, S_stack).  sci: optional
    (z_l, value).  Returns W [bins, n_lnm], norm, lnm_eff, mu2."""
    mh, hz, dn = _f64(tables["hmf_m_h"]), _f64(tables["hmf_z"]), _f64(tables["dndlnmh"])
    dz, da = _f64(tables["dist_z"]), _f64(tables["dist_da"])
    sl, sz, S = _f64(sel[0]), _f64(sel[1]), _f64(sel[2])
    nb = S.shape[0]
    W = np.empty((nb, n_lnm))
    norm, eff, mu2 = np.empty(nb), np.empty(nb), np.empty(nb)
    if sci is None:
        scz = scv = None
        nsc = 0
    else:
        scz, scv = _f64(sci[0]), _f64(sci[1])
        nsc = len(scz)
    rc = lib().y3o_selgl_weights(n_lnm, n_z, zt_lo, zt_hi, lnm_lo, lnm_hi, C.byref(cz),
                                 len(mh), _p(mh), len(hz), _p(hz), _p(dn),
                                 len(dz), _p(dz), _p(da), nsc, _p(scz), _p(scv),
                                 nb, len(sl), _p(sl), len(sz), _p(sz), _p(S),
                                 _p(W), _p(norm), _p(eff), _p(mu2))
    if rc:
        raise ValueError("z outside distances table")
    return W, norm, eff, mu2


def shear1h_mis(lnm_x, lnm_w, W_gamma, R, f_mis, tau_mis, lob_centers, omega_m,
                conc, r_sigma, lnM_tab, dsig_tab, n_theta=64, n_s=128, s_max=20.0):
    lx, lw, Wg, Rr = _f64(lnm_x), _f64(lnm_w), _f64(W_gamma), _f64(R)
    lob, rs, lt, ds = _f64(lob_centers), _f64(r_sigma), _f64(lnM_tab), _f64(dsig_tab)
    nb = Wg.shape[0]
    out = np.empty((nb, len(Rr)))
    lib().y3o_shear1h_mis(len(lx), _p(lx), _p(lw), nb, _p(Wg), len(Rr), _p(Rr),
                          f_mis, tau_mis, len(lob), _p(lob), omega_m, conc,
                          len(rs), _p(rs), len(lt), _p(lt), _p(ds),
                          n_theta, n_s, s_max, _p(out))
    return out


def shear1h_mis_tab(lnm_x, lnm_w, W_gamma, norm, lnm_eff, mu2, method, stencil_h, R,
                    f_mis, tau_mis, lob_centers, omega_m, conc, r_sigma, lnM_tab, dsig_tab,
                    mis_table):
    """Shear1hMisSelGL::evaluate with the miscentred profile read from the
    reference's NFW_DSIGMA_MIS table; mis_table = (logx, logxmis, log_tab)
    with log_tab [n_lxm, n_lx].  method 0 exact, 1 idea2."""
    lx, lw, Wg, Rr = _f64(lnm_x), _f64(lnm_w), _f64(W_gamma), _f64(R)
    nrm, eff, m2 = _f64(norm), _f64(lnm_eff), _f64(mu2)
    lob, rs, lt, ds = _f64(lob_centers), _f64(r_sigma), _f64(lnM_tab), _f64(dsig_tab)
    tx, txm, tv = (_f64(a) for a in mis_table)
    nb = Wg.shape[0]
    out = np.empty((nb, len(Rr)))
    lib().y3o_shear1h_mis_tab(len(lx), _p(lx), _p(lw), nb, _p(Wg), _p(nrm), _p(eff), _p(m2),
                              int(method), float(stencil_h), len(Rr), _p(Rr), f_mis, tau_mis,
                              len(lob), _p(lob), omega_m, conc, len(rs), _p(rs), len(lt),
                              _p(lt), _p(ds), len(tx), _p(tx), len(txm), _p(txm), _p(tv),
                              _p(out))
    return out


def sigma_crit_inv(zl, zs, pz, delta_z, h0, dist_z, dist_da):
    zl, zs, pz, dz, da = map(_f64, (zl, zs, pz, dist_z, dist_da))
    out = np.empty(len(zl))
    if lib().y3o_sigma_crit_inv(len(zl), _p(zl), len(zs), _p(zs), _p(pz), delta_z, h0,
                                len(dz), _p(dz), _p(da), _p(out)):
        raise ValueError("redshift outside distances / n(z) table")
    return out


def dsigma_mis_unit(x, xmis, n_theta=64, n_s=128, s_max=20.0):
    return lib().y3o_dsigma_mis_unit(x, xmis, n_theta, n_s, s_max)


def sigma_mis_unit(x, xmis, n_theta=64, n_s=128, s_max=20.0):
    return lib().y3o_sigma_mis_unit(x, xmis, n_theta, n_s, s_max)


# ---- direct nested quadrature ------------------------------------------------

def direct_eval(grid, plob_z, plob_coef, mor, cz, tables, shear=None):
    """Direct FP64 nested-GL evaluation of one parameter point.

    grid: dict (n_m, n_z, n_t, n_o, n_zo, lnm_lo, lnm_hi, zt_lo, zt_hi,
    lam_t_lo, lam_t_hi, lam_edges, zob_edges, sz0, optional sz_bin); mor: dict (A, B, C,
    sigma, Mpiv); shear: optional dict (R, f_mis, tau_mis, lob_centers, c0,
    c_slope, c_pivot, n_theta, n_s, s_max, sci_z, sci_val).
    Returns counts [n_bins], W [n_bins, n_m], shear [n_bins, n_R] or None."""
    le, ze = _f64(grid["lam_edges"]), _f64(grid["zob_edges"])
    szb = None if grid.get("sz_bin") is None else _f64(grid["sz_bin"])
    g = DirectGrid(grid["n_m"], grid["n_z"], grid["n_t"], grid["n_o"], grid["n_zo"],
                   grid["lnm_lo"], grid["lnm_hi"], grid["zt_lo"], grid["zt_hi"],
                   grid["lam_t_lo"], grid["lam_t_hi"], len(le) - 1, len(ze) - 1,
                   _p(le), _p(ze), grid["sz0"], _p(szb))
    m = Lognormal(mor["A"], mor["B"], mor["C"], mor["sigma"], mor["Mpiv"])
    pz, pc = _f64(plob_z), _f64(plob_coef)
    mh, hz, dn = _f64(tables["hmf_m_h"]), _f64(tables["hmf_z"]), _f64(tables["dndlnmh"])
    dz, da = _f64(tables["dist_z"]), _f64(tables["dist_da"])
    nb = (len(le) - 1) * (len(ze) - 1)
    counts = np.empty(nb)
    W = np.empty((nb, grid["n_m"]))
    sh_ptr = None
    sh_out = None
    keep = []
    if shear is not None:
        R = _f64(shear["R"])
        lob = _f64(shear["lob_centers"])
        scz, scv = _f64(shear["sci_z"]), _f64(shear["sci_val"])
        keep += [R, lob, scz, scv]
        so = ShearOpts(len(R), _p(R), shear["f_mis"], shear["tau_mis"], _p(lob),
                       shear["c0"], shear["c_slope"], shear["c_pivot"],
                       shear["n_theta"], shear["n_s"], shear["s_max"],
                       len(scz), _p(scz), _p(scv))
        sh_ptr = C.byref(so)
        sh_out = np.empty((nb, len(R)))
    rc = lib().y3o_direct_eval(C.byref(g), len(pz), _p(pz), _p(pc), C.byref(m),
                               C.byref(cz), len(mh), _p(mh), len(hz), _p(hz), _p(dn),
                               len(dz), _p(dz), _p(da), sh_ptr, _p(counts), _p(W),
                               _p(sh_out))
    if rc:
        raise ValueError("z outside distances table")
    return counts, W, sh_out


# ---- Gaussian likelihood ------------------------------------------------------

def loglike(nc, s1h, prj, log_space, data_nc, ic_nc, data_sh, ic_sh):
    """likelihood_cp.execute's logL from the module outputs; data and invcov
    as setup() stores them (logged / delta-method in log space).  s1h and
    prj are [n_bins, n_R] (prj may be None)."""
    nc, s1h = _f64(nc), _f64(s1h)
    nb = nc.size
    nr = s1h.size // nb
    dn, icn, ds, ics = _f64(data_nc), _f64(ic_nc), _f64(data_sh), _f64(ic_sh)
    pj = None if prj is None else _f64(prj)
    return lib().y3o_loglike(nb, nr, _p(nc), _p(s1h), _p(pj), int(bool(log_space)), _p(dn),
                             _p(icn), int(icn.ndim == 2), _p(ds), _p(ics), int(ics.ndim == 2))
