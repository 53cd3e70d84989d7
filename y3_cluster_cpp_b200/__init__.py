"""B200 engine for the DES-Y3 cluster-observable integrals.

A drop-in for the fast_mass hot path of estevesjh/y3_cluster_cpp: the
selection-function tabulation (sel_function.py), SelGLCore with the
NumCountsSel / Shear1hMisSel evaluators behind the CosmoSIS module ABI, and a
batched engine that evaluates the number counts N(lambda_obs bin, z_obs bin)
and the stacked miscentred-NFW DeltaSigma on fixed nested quadrature nodes in
FP64 or in a mixed form whose lambda_t contraction runs on the sm_100a tensor
cores.  Compute lives in ``lib/liby3b.so`` (C ABI: ``include/y3b.h``); this
package is the Python host side.
"""
from ._capi import LIB_PATH, Y3BError, lib  # noqa: F401

__all__ = ["LIB_PATH", "Y3BError", "lib"]
