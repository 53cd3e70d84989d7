"""y3b_sel_function_noalloc: the selection-function producer for callers that
cannot allocate device memory (a sampler that reserved all of its device
memory up front in its own pool, or a host whose device allocations belong to
another runtime's allocator).  The entry point keeps its scratch in a fixed
file-scope device array and writes into device buffers the caller provides.

Checked through the C ABI against the allocating entry point
(y3b_sel_function) on two calls in a row, with the tolerance the other
selection-function tests use (1e-12 of the table maximum).  This file is
collected last so a failure here never hides the other tests.
"""
import ctypes as C
import os

import numpy as np
import pytest

from y3_cluster_cpp_b200 import _capi as A
from y3_cluster_cpp_b200 import engine as E
from y3_cluster_cpp_b200 import prj_params

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _case(kind):
    g = np.load(os.path.join(GOLD, f"sel_function_{kind}.npz"))
    cfg = {k: np.ascontiguousarray(g[k], dtype=np.float64)
           for k in ("lam_min", "lam_max", "zob_min", "zob_max", "sigma_z")}
    cfg.update(zt_low=float(g["zt_low"]), zt_high=float(g["zt_high"]),
               lnm_low=float(g["lnm_low"]), lnm_high=float(g["lnm_high"]),
               n_lnm=int(g["n_lnm"]), n_z=int(g["n_z_shared"]), n_q=int(g["N_q"]))
    if kind == "hod":
        mor = (A.MOR_HOD, [float(g["hod_" + k]) for k in
                           ("log10_Mmin", "log10_M1", "alpha", "epsilon", "sigma_lambda")] + [0.45])
        plob = prj_params.default_table()
    else:
        mor = (A.MOR_LOGNORMAL, [float(g["ln_" + k]) for k in
                                 ("A", "B", "C", "sigma", "Mpiv", "lam_lo", "lam_hi")])
        plob = prj_params.baseline_constant_table()
    return cfg, mor, plob


def _structs(cfg, mor, plob, keep):
    c = A.SelFuncConfig(len(cfg["lam_min"]), A.ptr(cfg["lam_min"]), A.ptr(cfg["lam_max"]),
                        A.ptr(cfg["zob_min"]), A.ptr(cfg["zob_max"]), A.ptr(cfg["sigma_z"]),
                        cfg["zt_low"], cfg["zt_high"], cfg["lnm_low"], cfg["lnm_high"],
                        cfg["n_lnm"], cfg["n_z"], cfg["n_q"])
    m = A.Mor()
    m.kind = mor[0]
    for i, v in enumerate(mor[1]):
        m.p[i] = v
    pz, pc = A.f64(plob[0]), A.f64(plob[1])
    keep += [pz, pc]
    return c, m, A.Plob(len(pz), A.ptr(pz), A.ptr(pc))


@pytest.mark.parametrize("kind", ["hod", "lognormal"])
def test_noalloc_matches_allocating_entry_point_twice(kind):
    import torch
    E.check(A.lib().y3b_device_init(0))
    cfg, mor, plob = _case(kind)
    lnm_ref, z_ref, S_ref = E.sel_function(cfg, mor[0], mor[1], plob[0], plob[1])
    keep = []
    c, m, pl = _structs(cfg, mor, plob, keep)
    nb, nz, nl = len(cfg["lam_min"]), cfg["n_z"], cfg["n_lnm"]
    # Device buffers owned by the caller (torch's allocator here).
    lnm_d = torch.empty(nl, dtype=torch.float64, device="cuda")
    z_d = torch.empty(nz, dtype=torch.float64, device="cuda")
    S_d = torch.empty((nb, nz, nl), dtype=torch.float64, device="cuda")
    scale = np.max(np.abs(S_ref))
    for _ in range(2):
        S_d.fill_(np.nan)
        torch.cuda.synchronize()
        rc = A.lib().y3b_sel_function_noalloc(C.byref(c), C.byref(m), C.byref(pl),
                                              C.c_void_p(lnm_d.data_ptr()),
                                              C.c_void_p(z_d.data_ptr()),
                                              C.c_void_p(S_d.data_ptr()), None)
        E.check(rc)
        torch.cuda.synchronize()
        S = S_d.cpu().numpy()
        assert np.all(np.isfinite(S))
        assert np.max(np.abs(S - S_ref)) <= 1e-12 * scale
        np.testing.assert_allclose(lnm_d.cpu().numpy(), lnm_ref, rtol=0, atol=1e-12)
        np.testing.assert_allclose(z_d.cpu().numpy(), z_ref, rtol=0, atol=1e-14)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    E.check(A.lib().y3b_device_init(0))
    cfg, mor, plob = _case("hod")
    cfg["n_q"] = 2048
    keep = []
    c, m, pl = _structs(cfg, mor, plob, keep)
    buf = torch.empty(16, dtype=torch.float64, device="cuda")
    rc = A.lib().y3b_sel_function_noalloc(C.byref(c), C.byref(m), C.byref(pl),
                                          C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()),
                                          C.c_void_p(buf.data_ptr()), None)
    assert rc == 1
    assert b"scratch" in A.lib().y3b_last_error()
