"""ctypes bindings of the y3b C ABI (include/y3b.h).

The shared library lives in-tree at ``y3_cluster_cpp_b200/lib/liby3b.so``
(built by ``y3_cluster_cpp_b200/csrc/Makefile``).  Loading fails loudly when
it is missing: there is no Python or CPU fallback for any compute call.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "lib")
LIB_PATH = os.path.join(LIB_DIR, "liby3b.so")

D = C.c_double
I = C.c_int
PD = C.POINTER(C.c_double)
PI = C.POINTER(C.c_int)
VP = C.c_void_p

Y3B_OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID", 2: "DOMAIN", 3: "CUDA", 4: "NOMEM", 5: "TIMEOUT",
                6: "BUDGET", 7: "UNSUPPORTED", 8: "RANGE", 9: "CANCELLED"}
ERR_INVALID, ERR_DOMAIN, ERR_RANGE, ERR_CANCELLED = 1, 2, 8, 9
FP64 = 0
MIXED = 1
MOR_HOD = 0
MOR_LOGNORMAL = 1


class Y3BError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"y3b status {status} ({STATUS_NAMES.get(status, '?')}): {msg}")
        self.status = status


class Cosmo(C.Structure):
    _fields_ = [(n, D) for n in ("om", "ol", "ok", "h0", "onu", "hmf_s", "hmf_q")]


class Tables(C.Structure):
    _fields_ = [("n_hm", I), ("hmf_m_h", PD), ("n_hz", I), ("hmf_z", PD), ("dndlnmh", PD),
                ("n_dist", I), ("dist_z", PD), ("dist_da", PD),
                ("n_sci", I), ("sci_z", PD), ("sci_val", PD)]


class Plob(C.Structure):
    _fields_ = [("n", I), ("z", PD), ("coef", PD)]


class Mor(C.Structure):
    _fields_ = [("kind", I), ("p", D * 8)]


class SelFuncConfig(C.Structure):
    _fields_ = [("n_bins", I), ("lam_min", PD), ("lam_max", PD), ("zob_min", PD),
                ("zob_max", PD), ("sigma_z", PD), ("zt_low", D), ("zt_high", D),
                ("lnm_low", D), ("lnm_high", D), ("n_lnm", I), ("n_z", I), ("n_q", I)]


class SelGLConfig(C.Structure):
    _fields_ = [("n_lnm", I), ("n_z", I), ("zt_low", D), ("zt_high", D), ("lnm_low", D),
                ("lnm_high", D)]


class Selection(C.Structure):
    _fields_ = [("n_bins", I), ("n_lnm", I), ("lnm", PD), ("n_z", I), ("z", PD),
                ("S_stack", PD)]


class ShearTable(C.Structure):
    _fields_ = [("n_r", I), ("r_sigma", PD), ("n_lnm", I), ("lnM", PD), ("dsigma", PD),
                ("f_mis", D), ("tau_mis", D), ("n_lob", I), ("lob_centers", PD),
                ("conc", D), ("n_theta", I), ("n_s", I), ("s_max", D),
                ("use_idea2", I), ("stencil_h", D)]


class Grid(C.Structure):
    _fields_ = [("n_m", I), ("n_z", I), ("n_t", I), ("n_o", I), ("n_zo", I),
                ("lnm_lo", D), ("lnm_hi", D), ("zt_lo", D), ("zt_hi", D),
                ("lam_t_lo", D), ("lam_t_hi", D), ("n_lam_bins", I), ("n_z_bins", I),
                ("lam_edges", D * 9), ("zob_edges", D * 9), ("sz0", D), ("sz_bin", D * 8)]


class ShearOpts(C.Structure):
    _fields_ = [("n_R", I), ("R", D * 32), ("f_mis", D), ("tau_mis", D),
                ("lob_centers", D * 8), ("c0", D), ("c_slope", D), ("c_pivot", D),
                ("n_theta", I), ("n_s", I), ("s_max", D)]


class EngineConfig(C.Structure):
    _fields_ = [("n_hm", I), ("n_hz", I), ("n_dist", I), ("n_sci", I), ("plob", Plob),
                ("max_points", I), ("hbm_budget", C.c_size_t), ("with_shear", I),
                ("shear", ShearOpts), ("hmf_fp32", I)]


class Point(C.Structure):
    _fields_ = [("cosmo", Cosmo), ("A", D), ("B", D), ("C", D), ("sigma", D), ("Mpiv", D),
                ("grid", I), ("reserved", I)]


class ServerConfig(C.Structure):
    _fields_ = [("pool_points", I), ("hbm_budget", C.c_size_t), ("max_batch", I),
                ("precision", I), ("with_shear", I), ("max_inflight", I)]


class Likelihood(C.Structure):
    _fields_ = [("log_space", I), ("n_bins", I), ("n_R", I),
                ("data_nc", PD), ("invcov_nc", PD), ("nc_dense", I),
                ("data_sh", PD), ("invcov_sh", PD), ("sh_dense", I),
                ("shear_prj", PD)]


class PrjConfig(C.Structure):
    _fields_ = [("n_lnm", I), ("n_per_seg", I), ("n_zring", I), ("n_zouter", I),
                ("zt_low", D), ("zt_high", D), ("lnm_low", D), ("lnm_high", D),
                ("R_max_cMpch", D), ("include_omega_z", I), ("n_lob", I), ("lob_centers", PD),
                ("n_gp", I), ("lambda_bin", PI), ("zo_low", PD), ("zo_high", PD),
                ("radii", PD)]


class PrjSample(C.Structure):
    _fields_ = [("cosmo", Cosmo), ("t", Tables), ("dist_dc", PD),
                ("n_hl", I), ("n_hz", I), ("halo_lnM", PD), ("halo_z", PD), ("bias", PD),
                ("n_xr", I), ("n_xz", I), ("xi_r", PD), ("xi_z", PD), ("xi_nl", PD),
                ("n_blob", I), ("n_bzob", I), ("bsel_lob", PD), ("bsel_zob", PD),
                ("b_small", PD), ("b_large", PD)]


class BselConfig(C.Structure):
    _fields_ = [("n_lt", I), ("n_zring", I), ("n_zouter", I), ("n_lnm", I), ("n_theta", I),
                ("n_zt_ref", I), ("zt_ref_low", D), ("zt_ref_high", D), ("lnm_low", D),
                ("lnm_high", D), ("n_gp", I), ("zo_low", PD), ("zo_high", PD),
                ("lambda_bin", PI), ("max_samples", I)]


class BselSample(C.Structure):
    _fields_ = [("cosmo", Cosmo), ("t", Tables), ("dist_dc", PD),
                ("n_hl", I), ("n_hz", I), ("halo_lnM", PD), ("halo_z", PD), ("bias", PD),
                ("n_xr", I), ("n_xz", I), ("xi_r", PD), ("xi_z", PD), ("xi_nl", PD),
                ("hod", D * 6)]


class ServerStats(C.Structure):
    _fields_ = [("requests_done", C.c_longlong), ("points_done", C.c_longlong),
                ("launches", C.c_longlong), ("max_launch_points", I), ("pool_points", I),
                ("pool_free_points", I), ("waiting", I), ("unscheduled", I),
                ("requests_cancelled", C.c_longlong), ("device_bytes", C.c_size_t),
                ("pool_bytes_in_use", C.c_size_t)]


_lib = None


def lib():
    """Load liby3b.so (raises if the CUDA library was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"y3b CUDA library not found at {LIB_PATH}; build it with "
                "`make -C y3_cluster_cpp_b200/csrc` (or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def _declare(L):
    L.y3b_last_error.restype = C.c_char_p
    L.y3b_version.restype = I
    L.y3b_device_init.argtypes = [I]
    L.y3b_launch_count.restype = C.c_ulonglong
    L.y3b_sel_function.argtypes = [C.POINTER(SelFuncConfig), C.POINTER(Mor), C.POINTER(Plob),
                                   PD, PD, PD]
    L.y3b_selgl_create.argtypes = [C.POINTER(SelGLConfig), C.POINTER(VP)]
    L.y3b_selgl_build.argtypes = [VP, C.POINTER(Cosmo), C.POINTER(Tables),
                                  C.POINTER(Selection), I]
    L.y3b_selgl_counts.argtypes = [VP, I, PI, PD]
    L.y3b_selgl_shear.argtypes = [VP, C.POINTER(ShearTable), I, PI, PD, PD]
    L.y3b_selgl_set_mis_table.argtypes = [VP, I, PD, I, PD, PD]
    L.y3b_selgl_weights.argtypes = [VP, PD, PD, PD, PD, PD, PD]
    L.y3b_selgl_n_bins.argtypes = [VP]
    L.y3b_selgl_destroy.argtypes = [VP]
    L.y3b_selgl_destroy.restype = None
    L.y3b_sigma_crit_inv.argtypes = [I, PD, I, PD, PD, D, D, I, PD, PD, PD]
    L.y3b_nfw_mis.argtypes = [I, I, PD, PD, PD, D, D, I, I, D, PD]
    L.y3b_engine_create.argtypes = [C.POINTER(Grid), I, C.POINTER(EngineConfig), C.POINTER(VP)]
    L.y3b_engine_destroy.argtypes = [VP]
    L.y3b_engine_destroy.restype = None
    L.y3b_engine_table_stride.argtypes = [VP]
    L.y3b_engine_table_stride.restype = C.c_size_t
    L.y3b_engine_table_offsets.argtypes = [VP, C.POINTER(C.c_size_t)]
    L.y3b_engine_n_bins.argtypes = [VP]
    L.y3b_engine_device_bytes.argtypes = [VP]
    L.y3b_engine_device_bytes.restype = C.c_size_t
    L.y3b_engine_eval.argtypes = [VP, I, I, C.POINTER(Point), PD, PD, PD]
    L.y3b_engine_eval_device.argtypes = [VP, I, I, VP, VP, VP, VP, VP]
    L.y3b_engine_sync.argtypes = [VP, VP]
    L.y3b_engine_weights.argtypes = [VP, I, PD]
    L.y3b_selftest_wait_timeout.argtypes = [I]
    L.y3b_sel_function_noalloc.argtypes = [C.POINTER(SelFuncConfig), C.POINTER(Mor),
                                           C.POINTER(Plob), VP, VP, VP, VP]
    L.y3b_engine_eval_pooled.argtypes = [VP, I, I, VP, VP, VP, VP, VP, VP]
    L.y3b_engine_set_graphs.argtypes = [VP, I]
    L.y3b_engine_autotune.argtypes = [VP, I, VP, VP, VP, PD]
    L.y3b_engine_tuning.argtypes = [VP, PI, PI, I]
    L.y3b_engine_stage_count.argtypes = [VP, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
    L.y3b_server_create.argtypes = [VP, C.POINTER(ServerConfig), C.POINTER(VP)]
    L.y3b_server_submit.argtypes = [VP, I, VP, VP, VP, VP, C.POINTER(C.c_longlong)]
    L.y3b_server_wait.argtypes = [VP, C.c_longlong, D, PD]
    L.y3b_server_stats_read.argtypes = [VP, C.POINTER(ServerStats)]
    L.y3b_server_cancel.argtypes = [VP, C.c_longlong]
    L.y3b_server_destroy.argtypes = [VP]
    L.y3b_server_destroy.restype = None
    PLL = C.POINTER(C.c_longlong)
    L.y3b_planner_create.argtypes = [I, I, C.POINTER(VP)]
    L.y3b_planner_destroy.argtypes = [VP]
    L.y3b_planner_destroy.restype = None
    L.y3b_planner_submit.argtypes = [VP, C.c_longlong, I]
    L.y3b_planner_admit.argtypes = [VP, PLL, PI, I, PI]
    L.y3b_planner_next_batch.argtypes = [VP, PLL, PI, PI, PI, I, PI, PI]
    L.y3b_planner_complete.argtypes = [VP, C.c_longlong, I, PI]
    L.y3b_planner_cancel.argtypes = [VP, C.c_longlong, PI]
    L.y3b_planner_free_points.argtypes = [VP]
    L.y3b_engine_set_likelihood.argtypes = [VP, C.POINTER(Likelihood)]
    L.y3b_engine_loglike.argtypes = [VP, I, PD, VP]
    L.y3b_engine_eval_loglike.argtypes = [VP, I, I, C.POINTER(Point), PD, PD]
    L.y3b_gaussian_loglike.argtypes = [C.POINTER(Likelihood), PD, PD, PD]
    L.y3b_prj_create.argtypes = [C.POINTER(PrjConfig), C.POINTER(VP)]
    L.y3b_prj_set_mis_table.argtypes = [VP, I, PD, I, PD, PD]
    L.y3b_prj_eval.argtypes = [VP, C.POINTER(PrjSample), PD]
    L.y3b_prj_destroy.argtypes = [VP]
    L.y3b_prj_destroy.restype = None
    L.y3b_bsel_create.argtypes = [C.POINTER(BselConfig), C.POINTER(VP)]
    L.y3b_bsel_eval.argtypes = [VP, I, C.POINTER(BselSample), PD]
    L.y3b_bsel_kernel_ms.argtypes = [VP, PD]
    L.y3b_bsel_destroy.argtypes = [VP]
    L.y3b_bsel_destroy.restype = None
    L.y3b_engine_profile.argtypes = [VP, I]
    L.y3b_engine_profile_read.argtypes = [VP, PD, PI]


def check(rc):
    if rc != Y3B_OK:
        raise Y3BError(rc, lib().y3b_last_error().decode())
    return rc


def f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def ptr(a):
    if a is None:
        return None
    if a.dtype == np.int32:
        return a.ctypes.data_as(PI)
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(PD)


EXPORTED = [
    "y3b_last_error", "y3b_version", "y3b_device_init", "y3b_launch_count",
    "y3b_sel_function", "y3b_selgl_create", "y3b_selgl_build", "y3b_selgl_counts",
    "y3b_selgl_shear", "y3b_selgl_set_mis_table", "y3b_selgl_weights", "y3b_selgl_n_bins", "y3b_selgl_destroy",
    "y3b_sigma_crit_inv", "y3b_nfw_mis", "y3b_engine_create", "y3b_engine_destroy",
    "y3b_engine_table_stride", "y3b_engine_table_offsets", "y3b_engine_n_bins",
    "y3b_engine_device_bytes", "y3b_engine_eval", "y3b_engine_eval_device",
    "y3b_engine_sync", "y3b_engine_weights", "y3b_selftest_wait_timeout",
    "y3b_engine_profile", "y3b_engine_profile_read", "y3b_sel_function_noalloc",
    "y3b_engine_eval_pooled", "y3b_engine_set_graphs", "y3b_engine_autotune",
    "y3b_engine_tuning", "y3b_engine_stage_count", "y3b_server_create", "y3b_server_submit", "y3b_server_wait",
    "y3b_server_stats_read", "y3b_server_cancel", "y3b_server_destroy", "y3b_planner_create",
    "y3b_planner_destroy", "y3b_planner_submit", "y3b_planner_admit",
    "y3b_planner_next_batch", "y3b_planner_complete", "y3b_planner_cancel",
    "y3b_planner_free_points", "y3b_engine_set_likelihood", "y3b_engine_loglike",
    "y3b_engine_eval_loglike", "y3b_gaussian_loglike", "y3b_prj_create",
    "y3b_prj_set_mis_table", "y3b_prj_eval", "y3b_prj_destroy",
    "y3b_bsel_create", "y3b_bsel_eval", "y3b_bsel_kernel_ms", "y3b_bsel_destroy",
]
