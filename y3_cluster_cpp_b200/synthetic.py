"""Seeded synthetic inputs for the cluster-observable integrals.

The reference evaluates its modules on tables that CAMB / halo-model
producers write into the CosmoSIS DataBlock (mass_function/*, distances/*,
average_sigma_crit_inv/*).  None of those producers is part of the hot path,
so the benchmark and the tests run on seeded synthetic tables of the same
shapes:

* HMF: dn/dlnM on 100 log-spaced masses 1e13..10^15.5 Msun/h x 50 redshifts
  0.1..0.8, Tinker-like f(sigma) = A(z) (sigma/b(z))^-a(z) exp(-c/sigma^2)
  with a power-law sigma(M, z) = sigma8 (M / 2e14)^-0.2 D(z).  Published as
  mass_function/m_h = M / (Omega_m - Omega_nu), so the reference's HMF_t mass
  shift (hmf_t.hh:15-25) maps it back to ln M.
* distances: flat LCDM comoving distance by FP64 cumulative integration,
  d_a = chi / (1 + z) [Mpc] on 200 nodes 0..2.
* Sigma_crit^-1: 64 lens redshifts x 200 source redshifts with a Gaussian
  n(z_s) (0.9, 0.3), averaged with the formula of
  average_sigma_crit_inv.py:40-58.
* walkers: Omega_m ~ U[0.2, 0.4], sigma8 ~ U[0.7, 0.9], A, B, sigma_int each
  uniform within +-20% of (3.2, 0.9, 0.2).

All generation is numpy FP64 on the host: it stands in for upstream modules,
it is not part of the measured path.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import prj_params

RHO_CRIT = 2.77533742639e11       # h^2 Msun / Mpc^3 (nfw_dsigma_mis.hh:26)
C_OVER_H0 = 2997.92458            # Mpc/h
LAM_EDGES = np.array([20.0, 30.0, 45.0, 60.0, 200.0])
ZOB_EDGES = np.array([0.20, 0.35, 0.50, 0.65])
LOB_CENTERS = np.array([25.0, 37.5, 52.5, 130.0])

# Node counts per density: (lnM, z_t, ln lam_t, lam_o per bin, z_o per bin).
DENSITIES = {
    1: (64, 32, 64, 64, 16),
    2: (128, 64, 128, 128, 32),
    4: (256, 128, 256, 256, 64),
}


def grid(density=1, **over):
    """Quadrature grid of the synthetic configs at 1x/2x/4x node density."""
    n_m, n_z, n_t, n_o, n_zo = DENSITIES[density]
    g = dict(n_m=n_m, n_z=n_z, n_t=n_t, n_o=n_o, n_zo=n_zo,
             lnm_lo=np.log(1e13), lnm_hi=np.log(10 ** 15.5),
             zt_lo=0.1, zt_hi=0.8, lam_t_lo=1.0, lam_t_hi=1000.0,
             lam_edges=LAM_EDGES.copy(), zob_edges=ZOB_EDGES.copy(), sz0=0.01)
    g.update(over)
    return g


def shear_opts(n_theta=64, n_s=128, n_R=15):
    """Stacked miscentred DeltaSigma options of the synthetic ΔΣ config."""
    return dict(R=np.logspace(np.log10(0.1), np.log10(30.0), n_R), f_mis=0.2,
                tau_mis=0.17, lob_centers=LOB_CENTERS.copy(), c0=5.0,
                c_slope=-0.1, c_pivot=1e14, n_theta=n_theta, n_s=n_s, s_max=20.0)


@dataclass
class Point:
    """One sampler parameter point (walker)."""
    om: float = 0.3
    sigma8: float = 0.8
    h0: float = 0.7
    A: float = 3.2
    B: float = 0.9
    C: float = 0.5
    sigma: float = 0.2
    Mpiv: float = 3e14
    density: int = 1
    tables: dict = field(default_factory=dict)

    @property
    def mor(self):
        return dict(A=self.A, B=self.B, C=self.C, sigma=self.sigma, Mpiv=self.Mpiv)


def growth(z, om):
    """Linear growth D(z)/D(0) (Carroll, Press & Turner 1992 fit) x 1/(1+z)."""
    z = np.asarray(z, dtype=np.float64)

    def g(zz):
        a3 = (1 + zz) ** 3
        e2 = om * a3 + (1 - om)
        omz = om * a3 / e2
        olz = (1 - om) / e2
        return 2.5 * omz / (omz ** (4 / 7) - olz + (1 + omz / 2) * (1 + olz / 70))

    return g(z) / g(0.0) / (1 + z)


def hmf_table(om, sigma8, n_m=100, n_z=50, m_lo=1e13, m_hi=10 ** 15.5,
              z_lo=0.1, z_hi=0.8, onu=0.0):
    """(m_h [n_m], z [n_z], dndlnmh [n_z, n_m]) with m_h = M / (om - onu)."""
    M = np.logspace(np.log10(m_lo), np.log10(m_hi), n_m)
    z = np.linspace(z_lo, z_hi, n_z)
    rho_m = om * RHO_CRIT
    sig = sigma8 * (M[None, :] / 2e14) ** -0.2 * growth(z, om)[:, None]
    zp = 1 + z[:, None]
    alpha = 10 ** (-(0.75 / np.log10(200 / 75.0)) ** 1.2)
    A = 0.186 * zp ** -0.14
    a = 1.47 * zp ** -0.06
    b = 2.57 * zp ** -alpha
    f = A * (sig / b) ** -a * np.exp(-1.19 / sig ** 2)
    dn = f * rho_m / M[None, :] * 0.2
    return M / (om - onu), z, np.ascontiguousarray(dn)


def distances(om, h0, n=200, z_max=2.0):
    """(z [n], d_a [n] in Mpc) for flat LCDM by cumulative Simpson integration."""
    z = np.linspace(0.0, z_max, n)
    sub = 16
    zz = np.linspace(0.0, z_max, (n - 1) * sub + 1)
    inv_e = 1.0 / np.sqrt(om * (1 + zz) ** 3 + (1 - om))
    h = zz[1] - zz[0]
    # cumulative Simpson over pairs of sub-intervals
    chi_fine = np.zeros_like(zz)
    chi_fine[2::2] = np.cumsum(h / 3 * (inv_e[:-2:2] + 4 * inv_e[1:-1:2] + inv_e[2::2]))
    chi_fine[1::2] = chi_fine[0:-1:2] + h / 2 * (inv_e[0:-1:2] + inv_e[1::2])
    chi = chi_fine[::sub] * C_OVER_H0 / h0
    return z, chi / (1 + z)


def source_nz(n=200, z_lo=0.01, z_hi=2.0, mean=0.9, sig=0.3):
    zs = np.linspace(z_lo, z_hi, n)
    p = np.exp(-0.5 * ((zs - mean) / sig) ** 2)
    p /= np.trapezoid(p, zs)
    return zs, p


def sigma_crit_inv(h0, dist_z, dist_da, n_l=64, z_l_lo=0.05, z_l_hi=0.85, nz=None):
    """<Sigma_crit^-1>(z_l) table, average_sigma_crit_inv.py:40-58 (numpy)."""
    zs, pz = nz if nz is not None else source_nz()
    zl = np.linspace(z_l_lo, z_l_hi, n_l)
    G, c = 4.51710305e-48, 9.71561189e-15
    dl = np.interp(zl, dist_z, dist_da)
    ds = np.interp(zs, dist_z, dist_da)
    out = np.empty(n_l)
    for j in range(n_l):
        dls = ds - (1 + zl[j]) / (1 + zs) * dl[j]
        f = np.maximum(0.0, pz * 4 * np.pi * G / c / c * dl[j] * dls / ds)
        out[j] = np.trapezoid(f, zs) * h0
    return zl, out


def make_tables(p: Point, with_sci=True):
    mh, hz, dn = hmf_table(p.om, p.sigma8)
    dz, da = distances(p.om, p.h0)
    t = dict(hmf_m_h=mh, hmf_z=hz, dndlnmh=dn, dist_z=dz, dist_da=da)
    if with_sci:
        zl, sci = sigma_crit_inv(p.h0, dz, da)
        t["sci_z"], t["sci_val"] = zl, sci
    return t


def prj_tables(p: Point, n_m=60, n_z=40, n_r=200):
    """Tables the projection-shear observable reads besides the counts'
    ones (seeded synthetic, smooth): comoving distance distances/d_c [Mpc],
    the linear halo bias haloModel/{lnM, z, bias [n_z, n_m]} (peak-background
    split of the synthetic sigma(M, z)), the nonlinear correlation function
    xi_nl/{r [Mpc/h], z, xi_nl [n_z, n_r]} (power law (r / 5)^-1.8 D(z)^2 with
    an exponential cut at 200 Mpc/h) and the selection-bias asymptotes
    b_sel_marginalised/{lob, zob, b_small, b_large [n_zob x n_lob]}."""
    dz, da = p.tables["dist_z"], p.tables["dist_da"]
    lnM = np.linspace(np.log(1e12), np.log(10 ** 16), n_m)
    z = np.linspace(0.0, 1.2, n_z)
    dc = 1.686
    sig = p.sigma8 * (np.exp(lnM)[None, :] / 2e14) ** -0.2 * growth(z, p.om)[:, None]
    nu = dc / sig
    bias = 1.0 + (nu * nu - 1.0) / dc
    r = np.logspace(-2, np.log10(5000.0), n_r)
    xi = (r[None, :] / 5.0) ** -1.8 * np.exp(-r[None, :] / 200.0) * growth(z, p.om)[:, None] ** 2
    lob = np.array([25.0, 37.5, 52.5, 130.0])
    zob = np.array([0.275, 0.425, 0.575])
    b_small = 1.0 + 0.1 * np.arange(4)[None, :] + 0.2 * zob[:, None]
    b_large = 2.0 + 0.3 * np.arange(4)[None, :] + 0.5 * zob[:, None]
    return dict(dist_dc=da * (1 + dz), halo_lnM=lnM, halo_z=z, bias=bias, xi_r=r, xi_z=z,
                xi_nl=xi, bsel_lob=lob, bsel_zob=zob, b_small=b_small.ravel(),
                b_large=b_large.ravel())


def fiducial(density=1, with_sci=True) -> Point:
    p = Point(density=density)
    p.tables = make_tables(p, with_sci)
    return p


def walkers(n, seed=1, densities=(1, 2, 4), with_sci=True):
    """n walkers from the batched-config prior; densities cycle in equal thirds."""
    rng = np.random.default_rng(seed)
    pts = []
    for i in range(n):
        p = Point(om=rng.uniform(0.2, 0.4), sigma8=rng.uniform(0.7, 0.9),
                  A=3.2 * rng.uniform(0.8, 1.2), B=0.9 * rng.uniform(0.8, 1.2),
                  sigma=0.2 * rng.uniform(0.8, 1.2),
                  density=densities[(i * len(densities)) // max(n, 1)])
        p.tables = make_tables(p, with_sci)
        pts.append(p)
    return pts


def plob_baseline():
    return prj_params.baseline_constant_table()
