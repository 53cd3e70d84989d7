"""Python host API over the y3b C ABI.

* :func:`sel_function` -- S_ij(lnM, z) producer (sel_function.py execute).
* :class:`SelGL` -- SelGLCore / NumCountsSelGL / Shear1hMisSelGL.
* :func:`sigma_crit_inv`, :func:`nfw_mis` -- the lensing helpers.
* :class:`Engine` -- many parameter points on fixed nested quadrature nodes,
  FP64 direct form or the mixed tensor-core form.

Every call runs on the GPU through ``lib/liby3b.so``; a failure raises
:class:`Y3BError` with the library's message.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A
from ._capi import check, f64, lib, ptr

FP64 = A.FP64
MIXED = A.MIXED


def _mor(kind, params):
    m = A.Mor()
    m.kind = kind
    for i, v in enumerate(params):
        m.p[i] = float(v)
    return m


def _plob(z, coef, keep):
    z, coef = f64(z), f64(coef)
    keep += [z, coef]
    return A.Plob(len(z), ptr(z), ptr(coef))


def sel_function(cfg, mor_kind, mor, plob_z, plob_coef):
    """S_stack producer: returns (lnM [n_lnm], z [n_z], S [n_bins, n_z, n_lnm]).

    cfg: lam_min, lam_max, zob_min, zob_max, sigma_z (per bin), zt_low,
    zt_high, lnm_low, lnm_high, n_lnm, n_z (n_z_shared), n_q (N_q)."""
    keep = []
    arrs = {k: f64(cfg[k]) for k in ("lam_min", "lam_max", "zob_min", "zob_max", "sigma_z")}
    nb = len(arrs["lam_min"])
    for k, v in arrs.items():
        if len(v) != nb:
            raise ValueError(f"sel_function: axis '{k}' size {len(v)} != {nb}")
    c = A.SelFuncConfig(nb, ptr(arrs["lam_min"]), ptr(arrs["lam_max"]), ptr(arrs["zob_min"]),
                        ptr(arrs["zob_max"]), ptr(arrs["sigma_z"]), cfg["zt_low"],
                        cfg["zt_high"], cfg["lnm_low"], cfg["lnm_high"], int(cfg["n_lnm"]),
                        int(cfg["n_z"]), int(cfg["n_q"]))
    lnm = np.empty(int(cfg["n_lnm"]))
    z = np.empty(int(cfg["n_z"]))
    S = np.empty((nb, int(cfg["n_z"]), int(cfg["n_lnm"])))
    m = _mor(mor_kind, mor)
    pl = _plob(plob_z, plob_coef, keep)
    check(lib().y3b_sel_function(C.byref(c), C.byref(m), C.byref(pl), ptr(lnm), ptr(z), ptr(S)))
    return lnm, z, S


def cosmo(om, h0, ol=None, ok=0.0, onu=0.0, hmf_s=0.0, hmf_q=1.0):
    return A.Cosmo(om, 1.0 - om - ok if ol is None else ol, ok, h0, onu, hmf_s, hmf_q)


class SelGL:
    """SelGLCore + the two fixed-GL evaluators (n_operator_sel_gl_t.hh)."""

    def __init__(self, n_lnm=96, n_z=64, zt_low=0.05, zt_high=0.8, lnm_low=29.9336,
                 lnm_high=36.73):
        cfg = A.SelGLConfig(n_lnm, n_z, zt_low, zt_high, lnm_low, lnm_high)
        h = C.c_void_p()
        check(lib().y3b_selgl_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self.n_lnm = n_lnm

    def close(self):
        if self._h:
            lib().y3b_selgl_destroy(self._h)
            self._h = None

    __del__ = close

    def build(self, cz, tables, sel, include_sci=False):
        keep = [f64(tables[k]) for k in ("hmf_m_h", "hmf_z", "dndlnmh", "dist_z", "dist_da")]
        sci = None
        if include_sci:
            sci = [f64(tables["sci_z"]), f64(tables["sci_val"])]
        t = A.Tables(len(keep[0]), ptr(keep[0]), len(keep[1]), ptr(keep[1]), ptr(keep[2]),
                     len(keep[3]), ptr(keep[3]), ptr(keep[4]),
                     len(sci[0]) if sci else 0, ptr(sci[0]) if sci else None,
                     ptr(sci[1]) if sci else None)
        sl, sz, S = f64(sel[0]), f64(sel[1]), f64(sel[2])
        s = A.Selection(S.shape[0], len(sl), ptr(sl), len(sz), ptr(sz), ptr(S))
        check(lib().y3b_selgl_build(self._h, C.byref(cz), C.byref(t), C.byref(s),
                                    1 if include_sci else 0))
        self.n_bins = S.shape[0]
        return self

    def counts(self, bins):
        b = np.ascontiguousarray(np.asarray(bins, dtype=np.int32))
        out = np.empty(len(b))
        check(lib().y3b_selgl_counts(self._h, len(b), ptr(b), ptr(out)))
        return out

    def weights(self):
        nb = self.n_bins
        W = np.empty((nb, self.n_lnm))
        norm, eff, mu2 = np.empty(nb), np.empty(nb), np.empty(nb)
        x, w = np.empty(self.n_lnm), np.empty(self.n_lnm)
        check(lib().y3b_selgl_weights(self._h, ptr(W), ptr(norm), ptr(eff), ptr(mu2), ptr(x),
                                      ptr(w)))
        return dict(W=W, norm=norm, lnm_eff=eff, mu2=mu2, lnm_x=x, lnm_w=w)

    def set_mis_table(self, logx=None, logxmis=None, log_tab=None):
        """Miscentred-profile table (NFW_DSIGMA_MIS's file contents): ln x,
        ln x_mis axes and log_tab [n_lxm, n_lx]; None returns to the direct
        quadrature."""
        if logx is None:
            check(lib().y3b_selgl_set_mis_table(self._h, 0, None, 0, None, None))
            return self
        lx, lxm, tv = f64(logx), f64(logxmis), f64(log_tab)
        check(lib().y3b_selgl_set_mis_table(self._h, len(lx), ptr(lx), len(lxm), ptr(lxm),
                                            ptr(tv)))
        return self

    def shear(self, bins, r, halo, f_mis=0.22, tau_mis=0.17,
              lob_centers=(25.0, 37.5, 52.5, 130.0), conc=4.0, n_theta=64, n_s=128,
              s_max=20.0, idea2=False, stencil_h=0.15):
        b = np.ascontiguousarray(np.asarray(bins, dtype=np.int32))
        rr = f64(r)
        rs, lm, ds = f64(halo["r_sigma"]), f64(halo["lnM"]), f64(halo["dSigma_nfw"])
        lob = f64(lob_centers)
        st = A.ShearTable(len(rs), ptr(rs), len(lm), ptr(lm), ptr(ds), f_mis, tau_mis, len(lob),
                          ptr(lob), conc, n_theta, n_s, s_max, 1 if idea2 else 0, stencil_h)
        out = np.empty(len(b))
        check(lib().y3b_selgl_shear(self._h, C.byref(st), len(b), ptr(b), ptr(rr), ptr(out)))
        return out


class LikelihoodSpec:
    """Host arrays of a y3b_likelihood kept alive with the struct: data and
    inverse covariance (1-D: diagonal, 2-D: dense) of the counts and, when
    data_sh is given, of the shear (bin slow, R fast); shear_prj optional."""

    def __init__(self, data_nc, invcov_nc, data_sh=None, invcov_sh=None, shear_prj=None,
                 log_space=False):
        self.keep = [f64(data_nc), f64(invcov_nc)]
        nb = self.keep[0].size
        L = A.Likelihood()
        L.log_space = int(bool(log_space))
        L.n_bins = nb
        L.data_nc, L.invcov_nc = ptr(self.keep[0]), ptr(self.keep[1])
        L.nc_dense = int(self.keep[1].ndim == 2)
        if data_sh is not None:
            ds, ics = f64(data_sh).ravel(), f64(invcov_sh)
            self.keep += [ds, ics]
            L.n_R = ds.size // nb
            L.data_sh, L.invcov_sh = ptr(ds), ptr(ics)
            L.sh_dense = int(ics.ndim == 2)
            if shear_prj is not None:
                pj = f64(shear_prj).ravel()
                self.keep.append(pj)
                L.shear_prj = ptr(pj)
        self.struct = L


def gaussian_loglike(spec, counts, shear_1h=None):
    """The likelihood of one data vector on the device (y3b_gaussian_loglike)."""
    c = f64(counts)
    s = None if shear_1h is None else f64(shear_1h).ravel()
    out = C.c_double()
    check(lib().y3b_gaussian_loglike(C.byref(spec.struct), ptr(c), ptr(s), C.byref(out)))
    return out.value


class PrjShear:
    """Frozen-physics projection shear (ShearPrjFrozenPhysics): the grid
    points (lambda_bin, zo_low, zo_high, radii) are fixed at construction,
    eval() takes one sample's tables and returns [n_gp, 9]."""

    def __init__(self, grid, zt_low=0.1, zt_high=0.8, lnm_low=np.log(1e13),
                 lnm_high=np.log(10 ** 15.5), n_lnm=24, n_per_seg=10, n_zring=20, n_zouter=20,
                 R_max_cMpch=30.0, include_omega_z=True, lob_centers=None):
        self._keep = [np.ascontiguousarray(np.asarray(grid["lambda_bin"], dtype=np.int32))]
        self._keep += [f64(grid[k]) for k in ("zo_low", "zo_high", "radii")]
        c = A.PrjConfig()
        c.n_lnm, c.n_per_seg, c.n_zring, c.n_zouter = n_lnm, n_per_seg, n_zring, n_zouter
        c.zt_low, c.zt_high, c.lnm_low, c.lnm_high = zt_low, zt_high, lnm_low, lnm_high
        c.R_max_cMpch, c.include_omega_z = R_max_cMpch, int(bool(include_omega_z))
        if lob_centers is not None:
            lc = f64(lob_centers)
            self._keep.append(lc)
            c.n_lob, c.lob_centers = len(lc), ptr(lc)
        c.n_gp = len(self._keep[0])
        c.lambda_bin = ptr(self._keep[0])
        c.zo_low, c.zo_high, c.radii = (ptr(a) for a in self._keep[1:4])
        h = C.c_void_p()
        check(lib().y3b_prj_create(C.byref(c), C.byref(h)))
        self._h = h
        self.n_gp = c.n_gp

    def close(self):
        if getattr(self, "_h", None):
            lib().y3b_prj_destroy(self._h)
            self._h = None

    __del__ = close

    def set_mis_table(self, logx=None, logxmis=None, log_tab=None):
        if logx is None:
            check(lib().y3b_prj_set_mis_table(self._h, 0, None, 0, None, None))
            return self
        lx, lxm, tv = f64(logx), f64(logxmis), f64(log_tab)
        check(lib().y3b_prj_set_mis_table(self._h, len(lx), ptr(lx), len(lxm), ptr(lxm),
                                          ptr(tv)))
        return self

    def eval(self, cz, tables, prj):
        keep = [f64(tables[k]) for k in ("hmf_m_h", "hmf_z", "dndlnmh", "dist_z", "dist_da")]
        sci = [f64(tables["sci_z"]), f64(tables["sci_val"])] if "sci_z" in tables else None
        t = A.Tables(len(keep[0]), ptr(keep[0]), len(keep[1]), ptr(keep[1]), ptr(keep[2]),
                     len(keep[3]), ptr(keep[3]), ptr(keep[4]),
                     len(sci[0]) if sci else 0, ptr(sci[0]) if sci else None,
                     ptr(sci[1]) if sci else None)
        s = A.PrjSample()
        s.cosmo, s.t = cz, t
        arrs = {k: f64(prj[k]) for k in ("dist_dc", "halo_lnM", "halo_z", "bias", "xi_r", "xi_z",
                                         "xi_nl", "bsel_lob", "bsel_zob", "b_small", "b_large")}
        s.dist_dc = ptr(arrs["dist_dc"])
        s.n_hl, s.n_hz = len(arrs["halo_lnM"]), len(arrs["halo_z"])
        s.halo_lnM, s.halo_z, s.bias = ptr(arrs["halo_lnM"]), ptr(arrs["halo_z"]), ptr(arrs["bias"])
        s.n_xr, s.n_xz = len(arrs["xi_r"]), len(arrs["xi_z"])
        s.xi_r, s.xi_z, s.xi_nl = ptr(arrs["xi_r"]), ptr(arrs["xi_z"]), ptr(arrs["xi_nl"])
        s.n_blob, s.n_bzob = len(arrs["bsel_lob"]), len(arrs["bsel_zob"])
        s.bsel_lob, s.bsel_zob = ptr(arrs["bsel_lob"]), ptr(arrs["bsel_zob"])
        s.b_small, s.b_large = ptr(arrs["b_small"]), ptr(arrs["b_large"])
        out = np.empty((self.n_gp, 9))
        check(lib().y3b_prj_eval(self._h, C.byref(s), ptr(out)))
        return out


class BselMarg:
    """Selection-bias operators P1, I1, J of P_operator (module b_sel_marg):
    the wall grid (zo_low, zo_high, lambda_bin) and node counts are fixed at
    construction; eval() takes a list of samples, each (cosmo, tables, prj,
    hod) with tables as synthetic.make_tables, prj as synthetic.prj_tables
    (distances/d_c, haloModel bias, xi_nl) and hod the cluster_mor
    parameters (log10_Mmin, log10_M1, alpha, epsilon, sigma_lambda, optional
    z_pivot), and returns [n_samples, n_gp, 3]."""

    HOD_KEYS = ("log10_Mmin", "log10_M1", "alpha", "epsilon", "sigma_lambda")

    def __init__(self, grid, lnm_low, lnm_high, n_lt=60, n_zring=20, n_zouter=30, n_lnm=24,
                 n_theta=10, n_zt_ref=80, zt_ref_low=0.05, zt_ref_high=0.90, max_samples=64):
        self._keep = [f64(grid["zo_low"]), f64(grid["zo_high"]),
                      np.ascontiguousarray(np.asarray(grid["lambda_bin"], dtype=np.int32))]
        c = A.BselConfig()
        c.n_lt, c.n_zring, c.n_zouter, c.n_lnm = n_lt, n_zring, n_zouter, n_lnm
        c.n_theta, c.n_zt_ref = n_theta, n_zt_ref
        c.zt_ref_low, c.zt_ref_high, c.lnm_low, c.lnm_high = (zt_ref_low, zt_ref_high, lnm_low,
                                                              lnm_high)
        c.n_gp = len(self._keep[0])
        c.zo_low, c.zo_high, c.lambda_bin = (ptr(a) for a in self._keep)
        c.max_samples = max_samples
        h = C.c_void_p()
        check(lib().y3b_bsel_create(C.byref(c), C.byref(h)))
        self._h = h
        self.n_gp = c.n_gp

    def close(self):
        if getattr(self, "_h", None):
            lib().y3b_bsel_destroy(self._h)
            self._h = None

    __del__ = close

    def eval(self, samples):
        n = len(samples)
        arr = (A.BselSample * max(n, 1))()
        keep = []
        for k, (cz, tables, prj, hod) in enumerate(samples):
            t = [f64(tables[x]) for x in ("hmf_m_h", "hmf_z", "dndlnmh", "dist_z", "dist_da")]
            p = {x: f64(prj[x]) for x in ("dist_dc", "halo_lnM", "halo_z", "bias", "xi_r",
                                          "xi_z", "xi_nl")}
            keep += t + list(p.values())
            s = arr[k]
            s.cosmo = cz
            s.t = A.Tables(len(t[0]), ptr(t[0]), len(t[1]), ptr(t[1]), ptr(t[2]), len(t[3]),
                           ptr(t[3]), ptr(t[4]), 0, None, None)
            s.dist_dc = ptr(p["dist_dc"])
            s.n_hl, s.n_hz = len(p["halo_lnM"]), len(p["halo_z"])
            s.halo_lnM, s.halo_z, s.bias = ptr(p["halo_lnM"]), ptr(p["halo_z"]), ptr(p["bias"])
            s.n_xr, s.n_xz = len(p["xi_r"]), len(p["xi_z"])
            s.xi_r, s.xi_z, s.xi_nl = ptr(p["xi_r"]), ptr(p["xi_z"]), ptr(p["xi_nl"])
            for i, key in enumerate(self.HOD_KEYS):
                s.hod[i] = float(hod[key])
            s.hod[5] = float(hod.get("z_pivot", 0.45))
        out = np.empty((n, self.n_gp, 3))
        check(lib().y3b_bsel_eval(self._h, n, arr, ptr(out)))
        return out

    def kernel_ms(self):
        """Device time of the last eval's kernels (copies and packing excluded)."""
        ms = C.c_double()
        check(lib().y3b_bsel_kernel_ms(self._h, C.byref(ms)))
        return ms.value


def sigma_crit_inv(zl, zs, pz, delta_z, h0, dist_z, dist_da):
    zl, zs, pz, dz, da = map(f64, (zl, zs, pz, dist_z, dist_da))
    out = np.empty(len(zl))
    check(lib().y3b_sigma_crit_inv(len(zl), ptr(zl), len(zs), ptr(zs), ptr(pz), delta_z, h0,
                                   len(dz), ptr(dz), ptr(da), ptr(out)))
    return out


def nfw_mis(which, r, rmis, lnM, conc, rho, n_theta=64, n_s=128, s_max=20.0):
    """which='dsigma' (NFW_DSIGMA_MIS, gamma kernel), 'sigma' (NFW_SIGMA_MIS)
    or 'dsigma_single' (NFW_DSIGMA_MIS for the single offset rmis)."""
    kinds = {"dsigma": 0, "sigma": 1, "dsigma_single": 2}
    if which not in kinds:
        raise ValueError(f"nfw_mis: which must be one of {sorted(kinds)}")
    r, rmis, lnM = np.broadcast_arrays(f64(r), f64(rmis), f64(lnM))
    r, rmis, lnM = f64(r), f64(rmis), f64(lnM)
    out = np.empty(r.shape)
    check(lib().y3b_nfw_mis(kinds[which], r.size, ptr(r), ptr(rmis), ptr(lnM),
                            conc, rho, n_theta, n_s, s_max, ptr(out)))
    return out


def make_grid(g):
    """C grid struct from a dict (see synthetic.grid)."""
    G = A.Grid()
    for k in ("n_m", "n_z", "n_t", "n_o", "n_zo"):
        setattr(G, k, int(g[k]))
    for k in ("lnm_lo", "lnm_hi", "zt_lo", "zt_hi", "lam_t_lo", "lam_t_hi", "sz0"):
        setattr(G, k, float(g[k]))
    le, ze = list(g["lam_edges"]), list(g["zob_edges"])
    G.n_lam_bins, G.n_z_bins = len(le) - 1, len(ze) - 1
    for i, v in enumerate(le):
        G.lam_edges[i] = v
    for i, v in enumerate(ze):
        G.zob_edges[i] = v
    for j, v in enumerate(g.get("sz_bin") if g.get("sz_bin") is not None else []):
        G.sz_bin[j] = float(v)
    return G


class Engine:
    """Batched evaluation of N_ij (and the stacked miscentred DeltaSigma).

    grids: list of grid dicts (synthetic.grid); table shapes are fixed per
    engine; points carry their own tables (packed with :meth:`pack`)."""

    SECTIONS = ("hmf_m_h", "hmf_z", "dndlnmh", "dist_z", "dist_da", "sci_z", "sci_val")

    def __init__(self, grids, n_hm, n_hz, n_dist, plob, max_points=256, n_sci=0,
                 shear=None, hbm_budget=0, hmf_fp32=False):
        self._keep = []
        self.hmf_fp32 = bool(hmf_fp32)
        self.grids = list(grids)
        G = (A.Grid * len(grids))(*[make_grid(g) for g in grids])
        cfg = A.EngineConfig()
        cfg.n_hm, cfg.n_hz, cfg.n_dist, cfg.n_sci = n_hm, n_hz, n_dist, n_sci
        cfg.plob = _plob(plob[0], plob[1], self._keep)
        cfg.max_points = max_points
        cfg.hbm_budget = hbm_budget
        cfg.with_shear = 1 if shear is not None else 0
        cfg.hmf_fp32 = int(self.hmf_fp32)
        if shear is not None:
            so = cfg.shear
            so.n_R = len(shear["R"])
            for i, v in enumerate(shear["R"]):
                so.R[i] = v
            so.f_mis, so.tau_mis = shear["f_mis"], shear["tau_mis"]
            for i, v in enumerate(shear["lob_centers"]):
                so.lob_centers[i] = v
            so.c0, so.c_slope, so.c_pivot = shear["c0"], shear["c_slope"], shear["c_pivot"]
            so.n_theta, so.n_s, so.s_max = shear["n_theta"], shear["n_s"], shear["s_max"]
        self.n_R = len(shear["R"]) if shear is not None else 0
        h = C.c_void_p()
        check(lib().y3b_engine_create(G, len(grids), C.byref(cfg), C.byref(h)))
        self._h = h
        self.max_points = max_points
        self.stride = lib().y3b_engine_table_stride(h)
        off = (C.c_size_t * 7)()
        check(lib().y3b_engine_table_offsets(h, off))
        self.offsets = list(off)
        self.n_bins = lib().y3b_engine_n_bins(h)
        self.shapes = (n_hm, n_hz, n_dist, n_sci)

    def close(self):
        if getattr(self, "_h", None):
            lib().y3b_engine_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def handle(self):
        return self._h

    def device_bytes(self):
        return lib().y3b_engine_device_bytes(self._h)

    def pack(self, points, out=None):
        """Packed per-point table buffer [n, stride] (float64)."""
        n = len(points)
        buf = np.zeros((n, self.stride)) if out is None else out
        n_hm, n_hz, n_dist, n_sci = self.shapes
        sizes = (n_hm, n_hz, n_hz * n_hm, n_dist, n_dist, n_sci, n_sci)
        for i, p in enumerate(points):
            t = p.tables
            for sec, o, s in zip(self.SECTIONS, self.offsets, sizes):
                if s == 0:
                    continue
                v = np.asarray(t[sec], dtype=np.float64).ravel()
                if v.size != s:
                    raise ValueError(f"point {i}: {sec} has {v.size} values, engine expects {s}")
                if sec == "dndlnmh" and self.hmf_fp32:  # n floats in the section's doubles
                    buf[i, o:o + (s + 1) // 2].view(np.float32)[:s] = v.astype(np.float32)
                else:
                    buf[i, o:o + s] = v
        return buf

    @staticmethod
    def point_struct(p, grid_index):
        c = cosmo(p.om, p.h0)
        return A.Point(c, p.A, p.B, p.C, p.sigma, p.Mpiv, grid_index, 0)

    def points_array(self, points, grid_of=None):
        arr = (A.Point * len(points))()
        for i, p in enumerate(points):
            g = grid_of(p) if grid_of else p.grid_index
            arr[i] = self.point_struct(p, g)
        return arr

    def eval(self, points, precision=MIXED, tables=None, grid_of=None, weights=False):
        """Host-buffer evaluation.  Returns counts [n, n_bins] (and shear
        [n, n_bins, n_R] when the engine has shear)."""
        n = len(points)
        pts = self.points_array(points, grid_of)
        tab = self.pack(points) if tables is None else tables
        counts = np.empty((n, self.n_bins))
        sh = np.empty((n, self.n_bins, self.n_R)) if self.n_R else None
        check(lib().y3b_engine_eval(self._h, precision, n, pts, ptr(tab), ptr(counts), ptr(sh)))
        out = {"counts": counts}
        if sh is not None:
            out["shear"] = sh
        if weights:
            w_stride = max(g["n_m"] for g in self.grids)
            W = np.empty((n, self.n_bins, w_stride))
            check(lib().y3b_engine_weights(self._h, n, ptr(W)))
            out["W"] = W
        return out

    def eval_device(self, precision, n, pts_dev, tables_dev, counts_dev, shear_dev=0, stream=0):
        """Device-pointer evaluation (integers: device addresses / cudaStream_t)."""
        check(lib().y3b_engine_eval_device(self._h, precision, n, C.c_void_p(pts_dev),
                                           C.c_void_p(tables_dev), C.c_void_p(counts_dev),
                                           C.c_void_p(shear_dev or None),
                                           C.c_void_p(stream or None)))

    def autotune(self, n, pts_dev, tables_dev, counts_dev):
        """Tune the contraction (ring depth, bins per tile) on a device batch;
        returns {"stages", "bins_per_tile", "contraction_ms"}."""
        ms = C.c_double()
        check(lib().y3b_engine_autotune(self._h, n, C.c_void_p(pts_dev), C.c_void_p(tables_dev),
                                        C.c_void_p(counts_dev), C.byref(ms)))
        out = self.tuning()
        out["contraction_ms"] = ms.value
        return out

    def tuning(self):
        st = C.c_int()
        nic = (C.c_int * len(self.grids))()
        check(lib().y3b_engine_tuning(self._h, C.byref(st), nic, len(self.grids)))
        return {"stages": st.value, "bins_per_tile": list(nic)}

    def stage_count(self):
        """(issued, dense) lam_t stages of the last mixed-form contraction;
        call after that evaluation completed."""
        ex, dn = C.c_longlong(), C.c_longlong()
        check(lib().y3b_engine_stage_count(self._h, C.byref(ex), C.byref(dn)))
        return ex.value, dn.value

    def set_likelihood(self, spec):
        """Fuse a Gaussian likelihood (LikelihoodSpec, None: off) into every
        later evaluation."""
        self._like = spec
        check(lib().y3b_engine_set_likelihood(self._h, None if spec is None
                                              else C.byref(spec.struct)))

    def loglike(self, n):
        out = np.empty(n)
        check(lib().y3b_engine_loglike(self._h, n, ptr(out), None))
        return out

    def set_graphs(self, on=True):
        """CUDA-graph replay of repeated evaluations (on by default)."""
        check(lib().y3b_engine_set_graphs(self._h, 1 if on else 0))

    def profile(self, enable=True):
        check(lib().y3b_engine_profile(self._h, 1 if enable else 0))

    def profile_read(self):
        """Accumulated stage milliseconds (prep, contraction, shear, final) and
        the number of evaluations timed."""
        ms = np.zeros(4)
        n = C.c_int()
        check(lib().y3b_engine_profile_read(self._h, ptr(ms), C.byref(n)))
        return dict(prep=ms[0], contraction=ms[1], shear=ms[2], final=ms[3], evals=n.value)

    def sync(self, stream=0):
        check(lib().y3b_engine_sync(self._h, C.c_void_p(stream or None)))


def launch_count():
    return lib().y3b_launch_count()


def selftest_wait_timeout(usec=2000):
    """Runs the bounded-wait self-test; returns the library status (5 = TIMEOUT)."""
    return lib().y3b_selftest_wait_timeout(int(usec))
