"""CosmoSIS module: S_ij(lnM, z) on the GPU -- drop-in for
src/modules/sel_function/sel_function.py.

Same ini options (lam_min, lam_max, zob_min, zob_max, sigma_z per bin;
zt_low, zt_high, lnm_low, lnm_high; n_lnm, n_z, n_z_shared, N_q), same
inputs (cluster_mor/*, optional plob_ltr_params/*) and the same output
section (sel_function/{lnM, z, S_stack} with S_stack of shape
(n_bins, n_z, n_lnm)).  The whole tensor -- per-cell lambda_t brackets, the
MOR density, the EMG CDF differences at the unique richness edges and the
photo-z kernel -- is evaluated by ``y3b_sel_function`` in FP64 on the GPU.

One extra option, ``mor`` (``hod`` by default, as the reference), selects
the lognormal mass-richness relation of the synthetic benchmark configs,
read from cluster_mor/{A, B, C, sigma_intr, M_pivot, lam_t_min, lam_t_max}.
"""
from __future__ import annotations

import numpy as np

from . import engine, prj_params
from ._capi import MOR_HOD, MOR_LOGNORMAL

try:  # pragma: no cover - only inside CosmoSIS
    from cosmosis.datablock import option_section
except Exception:  # noqa: BLE001
    option_section = "module_options"

Z_PIVOT_DEFAULT = 0.45


def _read_array(options, section, name):
    try:
        return np.asarray(options.get_double_array_1d(section, name), dtype=float)
    except Exception:  # noqa: BLE001
        return np.asarray(options.get_int_array_1d(section, name), dtype=float)


def _read_scalar_or_first(options, section, name, default):
    try:
        return float(np.asarray(options.get_double_array_1d(section, name), dtype=float).ravel()[0])
    except Exception:  # noqa: BLE001
        try:
            return float(options.get_double(section, name))
        except Exception:  # noqa: BLE001
            return float(default)


def _read_int(options, section, name, default):
    try:
        return int(options.get_int(section, name))
    except Exception:  # noqa: BLE001
        return int(default)


def setup(options):
    """Mirror of sel_function.setup (sel_function.py:417-472)."""
    sec = option_section
    cfg = {k: _read_array(options, sec, k)
           for k in ("lam_min", "lam_max", "zob_min", "zob_max", "sigma_z")}
    cfg["zt_low"] = _read_scalar_or_first(options, sec, "zt_low", 0.05)
    cfg["zt_high"] = _read_scalar_or_first(options, sec, "zt_high", 0.80)
    cfg["lnm_low"] = _read_scalar_or_first(options, sec, "lnm_low", np.log(1.0e13))
    cfg["lnm_high"] = _read_scalar_or_first(options, sec, "lnm_high", np.log(9.0e15))
    cfg["n_lnm"] = _read_int(options, sec, "n_lnm", 40)
    n_z = _read_int(options, sec, "n_z", 20)
    cfg["n_z"] = _read_int(options, sec, "n_z_shared", n_z)
    cfg["n_q"] = _read_int(options, sec, "N_q", 32)
    try:
        cfg["mor"] = str(options.get_string(sec, "mor")).strip().lower()
    except Exception:  # noqa: BLE001
        cfg["mor"] = "hod"
    if cfg["mor"] not in ("hod", "lognormal"):
        raise ValueError(f"sel_function: mor must be 'hod' or 'lognormal', got {cfg['mor']!r}")
    n = cfg["lam_min"].size
    for key in ("lam_max", "zob_min", "zob_max", "sigma_z"):
        if cfg[key].size != n:
            raise ValueError(f"sel_function: axis '{key}' size {cfg[key].size} != {n}")
    cfg["n_bins"] = n
    return cfg


def _get(block, sec, key, default=None):
    try:
        return block[sec, key]
    except Exception:  # noqa: BLE001
        if default is None:
            raise
        return default


def _plob(block):
    try:
        z = np.asarray(block["plob_ltr_params", "z"], dtype=float)
        coef = np.array([np.asarray(block["plob_ltr_params", k], dtype=float)
                         for k in prj_params.COEFF_NAMES])
        return z, coef
    except Exception:  # noqa: BLE001
        return prj_params.default_table()


def _mor(block, kind):
    if kind == "hod":
        log10_Mmin = float(block["cluster_mor", "log10_Mmin"])
        try:
            log10_M1 = log10_Mmin + float(block["cluster_mor", "log10_ratio"])
        except Exception:  # noqa: BLE001
            log10_M1 = float(block["cluster_mor", "log10_M1"])
        z_pivot = float(_get(block, "cluster_mor", "z_pivot", Z_PIVOT_DEFAULT))
        return MOR_HOD, [log10_Mmin, log10_M1, float(block["cluster_mor", "alpha"]),
                         float(block["cluster_mor", "epsilon"]),
                         float(block["cluster_mor", "sigma_lambda"]), z_pivot]
    return MOR_LOGNORMAL, [float(block["cluster_mor", "A"]), float(block["cluster_mor", "B"]),
                           float(block["cluster_mor", "C"]),
                           float(block["cluster_mor", "sigma_intr"]),
                           float(_get(block, "cluster_mor", "M_pivot", 3e14)),
                           float(_get(block, "cluster_mor", "lam_t_min", 1.0)),
                           float(_get(block, "cluster_mor", "lam_t_max", 1000.0))]


def execute(block, config):
    """Mirror of sel_function.execute (sel_function.py:555-615)."""
    kind, params = _mor(block, config["mor"])
    pz, pc = _plob(block)
    lnm, z, S = engine.sel_function(config, kind, params, pz, pc)
    block["sel_function", "lnM"] = lnm
    block["sel_function", "z"] = z
    block["sel_function", "S_stack"] = np.ascontiguousarray(S)
    return 0


def cleanup(config):
    return 0
