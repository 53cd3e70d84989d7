"""CosmoSIS module: the Gaussian likelihood of the cluster counts and
tangential shear -- drop-in for y3_buzzard/likelihood_cp.py.

Same ini options (``filename`` of an .npz with data_NC, invcov_NC,
data_Shear, invcov_Shear; ``log_space``; ``verbose``), same inputs
(numcountssel/vals, shear1hmissel/vals, shear_prj/vals) and the same output
(likelihoods/likelihoods_like).  The shear theory is the N_i-weighted
one-halo shear divided by the counts of its bin plus the projection shear
(bin slow, R fast); diagonal (1-D) or dense (2-D) inverse covariances; in log
space the residuals are taken between logarithms and the inverse covariance
is propagated by the delta method about the fixed data (as the reference's
setup() does).  The evaluation runs on the GPU (y3b_gaussian_loglike); the
engine can instead fuse the same likelihood into its final sums
(Engine.set_likelihood).
"""
from __future__ import annotations

import numpy as np

from . import engine

try:  # pragma: no cover - only inside CosmoSIS
    from cosmosis.datablock import option_section
except Exception:  # noqa: BLE001
    option_section = "module_options"


def _get_bool(options, key, default):
    try:
        return bool(options.get_bool(option_section, key, default=default))
    except Exception:  # noqa: BLE001
        return default


def setup(options):
    fname = options[option_section, "filename"]
    vec = np.load(fname, allow_pickle=False)
    d_nc = np.asarray(vec["data_NC"], dtype=float).ravel()
    d_sh = np.asarray(vec["data_Shear"], dtype=float).ravel()
    ic_nc = np.asarray(vec["invcov_NC"], dtype=float)
    ic_sh = np.asarray(vec["invcov_Shear"], dtype=float)
    for name, d, ic in (("NC", d_nc, ic_nc), ("Shear", d_sh, ic_sh)):
        if ic.ndim == 1 and ic.size != d.size or ic.ndim == 2 and ic.shape != (d.size, d.size):
            raise ValueError(f"likelihood_cp: invcov_{name} does not match data_{name} "
                             f"({ic.shape} vs {d.size})")
    if d_sh.size % d_nc.size:
        raise ValueError("likelihood_cp: data_Shear is not n_bins x n_R")
    log_space = _get_bool(options, "log_space", False)
    if log_space and (np.any(d_nc <= 0.0) or np.any(d_sh <= 0.0)):
        raise ValueError("likelihood_cp: log_space requires data > 0")
    return {"filename": fname, "spec_args": (d_nc, ic_nc, d_sh, ic_sh, log_space),
            "verbose": _get_bool(options, "verbose", False), "n_bins": d_nc.size,
            "n_sh": d_sh.size}


def execute(block, config):
    nb, nsh = config["n_bins"], config["n_sh"]
    nc = np.asarray(block["numcountssel", "vals"], dtype=float).ravel()
    s1h = np.asarray(block["shear1hmissel", "vals"], dtype=float).ravel()
    prj = np.asarray(block["shear_prj", "vals"], dtype=float).ravel()
    for name, v, n in (("numcountssel/vals", nc, nb), ("shear1hmissel/vals", s1h, nsh),
                       ("shear_prj/vals", prj, nsh)):
        if v.size != n:
            raise ValueError(f"likelihood_cp: {name} size {v.size} != {n}")
    d_nc, ic_nc, d_sh, ic_sh, log_space = config["spec_args"]
    spec = engine.LikelihoodSpec(d_nc, ic_nc, d_sh, ic_sh, shear_prj=prj, log_space=log_space)
    logL = engine.gaussian_loglike(spec, nc, s1h)
    if config["verbose"]:
        print(f"[likelihood_cp] logL={logL:.4e}")
    block["likelihoods", "likelihoods_like"] = float(logL)
    return 0


def cleanup(config):
    return 0
