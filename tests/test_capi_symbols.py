"""The C-ABI libraries load on a CPU-only host and export every function that
include/*.h declares (no compute call is made here)."""
import ctypes as C
import os
import re

import pytest

from y3_cluster_cpp_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_functions(header):
    src = open(os.path.join(INCLUDE, header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    names = re.findall(r"\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", src)
    return sorted(set(n for n in names if n not in ("sizeof",)))


def test_engine_library_exports_header():
    lib = _capi.lib()
    names = declared_functions("y3b.h")
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(_capi.EXPORTED) <= set(names)
    assert lib.y3b_version() == 1


@pytest.mark.parametrize("module", ["NumCountsSel", "Shear1hMisSel", "NumCountsFastMass",
                                    "Shear1hFastMass"])
def test_cosmosis_modules_export_entry_points(module):
    from y3_cluster_cpp_b200 import cosmosis
    cosmosis.shim()
    m = C.CDLL(os.path.join(_capi.LIB_DIR, module + ".so"))
    for n in ("setup", "execute", "cleanup"):
        assert hasattr(m, n)


def test_datablock_shim_exports_accessors():
    from y3_cluster_cpp_b200 import cosmosis
    S = cosmosis.shim()
    for n in declared_functions("y3b_cosmosis.h"):
        if n.startswith("c_datablock"):
            assert hasattr(S, n), n


def test_datablock_roundtrip_without_gpu():
    import numpy as np
    from y3_cluster_cpp_b200.cosmosis import DataBlock
    b = DataBlock()
    b["Sec", "X"] = 2.5
    b["sec", "arr"] = np.arange(6.0).reshape(2, 3)
    assert b["sec", "x"] == 2.5
    np.testing.assert_array_equal(b["SEC", "ARR"], np.arange(6.0).reshape(2, 3))
    assert ("sec", "arr") in b and ("sec", "nope") not in b


def test_compute_without_gpu_fails_loudly():
    """On a host without an sm_100 device every compute entry point returns
    Y3B_ERR_CUDA -- never a CPU answer."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from y3_cluster_cpp_b200 import engine
    with pytest.raises(_capi.Y3BError) as e:
        engine.nfw_mis("dsigma", [0.5], [0.1], [32.0], 4.0, 8e10)
    assert e.value.status == 3


def test_fused_module_setup_validates_bins_on_cpu():
    """engine = fused checks the sel_function bin layout at setup (no device
    work): a richness-fast product of contiguous bins with one sigma_z per
    z_obs bin, known precision."""
    import numpy as np
    from y3_cluster_cpp_b200.cosmosis import DataBlock, Module

    def opts(**over):
        o = DataBlock()
        lab = "NumCountsFastMass"
        d = dict(engine="fused", bin_index=np.arange(12),
                 lam_min=[20.0, 30.0, 45.0, 60.0] * 3, lam_max=[30.0, 45.0, 60.0, 200.0] * 3,
                 zob_min=[0.2] * 4 + [0.35] * 4 + [0.5] * 4,
                 zob_max=[0.35] * 4 + [0.5] * 4 + [0.65] * 4, sigma_z=[0.03] * 12,
                 zt_low=0.1, zt_high=0.8, lnm_low=29.9, lnm_high=35.7)
        d.update(over)
        for k, v in d.items():
            o[lab, k] = np.asarray(v, float) if isinstance(v, list) else v
        return o

    m = Module("NumCountsFastMass")
    assert m.setup(opts())
    m.cleanup()
    assert not Module("NumCountsFastMass").setup(opts(precision="fp16"))
    assert not Module("NumCountsFastMass").setup(opts(engine="other"))
    bad = [20.0, 30.0, 45.0, 61.0] * 3                       # gap between bins
    assert not Module("NumCountsFastMass").setup(opts(lam_min=bad))
    assert not Module("NumCountsFastMass").setup(opts(sigma_z=[0.03] * 11 + [0.05]))
    assert not Module("NumCountsFastMass").setup(opts(bin_index=np.arange(13)))
    assert not Module("Shear1hFastMass").setup(opts())       # counts only


def test_prj_module_rejects_incomplete_options_on_cpu():
    """ShearPrjFrozenPhysics.so setup checks its options before any device
    work: missing box or mismatched grid arrays give NULL, never a throw."""
    import numpy as np
    from y3_cluster_cpp_b200.cosmosis import DataBlock, Module
    lab = "shear_prj_frozen_physics"
    o = DataBlock()
    o[lab, "lambda_bin"] = np.arange(3, dtype=np.int32)
    o[lab, "zo_low"] = np.full(3, 0.2)
    o[lab, "zo_high"] = np.full(3, 0.35)
    o[lab, "radii"] = np.array([0.5, 1.0])           # one short
    for k, v in dict(zt_low=0.1, zt_high=0.8, lnm_low=29.9, lnm_high=35.7).items():
        o[lab, k] = v
    assert not Module("ShearPrjFrozenPhysics").setup(o)
    o2 = DataBlock()
    o2[lab, "radii"] = np.array([0.5])
    assert not Module("ShearPrjFrozenPhysics").setup(o2)   # no box, no grid


def test_bsel_module_rejects_incomplete_options_on_cpu():
    """BSelMargIntegrand.so setup checks its options before any device work:
    a missing mass range or mismatched grid arrays give NULL, never a throw."""
    import numpy as np
    from y3_cluster_cpp_b200.cosmosis import DataBlock, Module
    lab = "b_sel_marg"
    o = DataBlock()
    o[lab, "zo_low"] = np.full(3, 0.2)
    o[lab, "zo_high"] = np.full(2, 0.35)             # one short
    o[lab, "lambda_bin"] = np.arange(3, dtype=np.int32)
    o[lab, "lnm_low"], o[lab, "lnm_high"] = 29.9, 35.7
    assert not Module("BSelMargIntegrand").setup(o)
    o2 = DataBlock()
    o2[lab, "zo_low"], o2[lab, "zo_high"] = np.full(3, 0.2), np.full(3, 0.35)
    o2[lab, "lambda_bin"] = np.arange(3, dtype=np.int32)
    assert not Module("BSelMargIntegrand").setup(o2)  # no mass range
