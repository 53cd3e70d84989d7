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
