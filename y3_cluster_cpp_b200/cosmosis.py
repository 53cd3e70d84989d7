"""Drive the CosmoSIS module shared objects without CosmoSIS.

``DataBlock`` is the standalone C DataBlock of ``lib/libdatablock_shim.so``
(loaded RTLD_GLOBAL so the module .so files resolve their c_datablock_*
accessors against it, exactly as they would against libcosmosis).
``Module`` dlopen()s one of ``lib/{NumCountsSel,Shear1hMisSel,
NumCountsFastMass,Shear1hFastMass}.so`` and calls setup / execute / cleanup
the way the CosmoSIS runtime does (src/utils/module_macros.hh:76-99).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._capi import LIB_DIR, lib

_shim = None


def shim():
    global _shim
    if _shim is None:
        lib()  # the engine library first (modules link against it)
        path = os.path.join(LIB_DIR, "libdatablock_shim.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} not built")
        S = C.CDLL(path, mode=C.RTLD_GLOBAL)
        S.y3b_datablock_new.restype = C.c_void_p
        S.y3b_datablock_free.argtypes = [C.c_void_p]
        S.c_datablock_has_value.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p]
        S.c_datablock_has_value.restype = C.c_bool
        S.c_datablock_put_int.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_int]
        S.c_datablock_put_double.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_double]
        S.c_datablock_put_string.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p]
        S.c_datablock_put_int_array_1d.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p,
                                                   C.POINTER(C.c_int), C.c_int]
        S.c_datablock_put_double_array.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p,
                                                   C.POINTER(C.c_double), C.c_int,
                                                   C.POINTER(C.c_int)]
        S.c_datablock_get_array_ndim.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p,
                                                 C.POINTER(C.c_int)]
        S.c_datablock_get_double_array_shape.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p,
                                                         C.c_int, C.POINTER(C.c_int)]
        S.c_datablock_get_double_array.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p,
                                                   C.POINTER(C.c_double), C.c_int,
                                                   C.POINTER(C.c_int)]
        S.c_datablock_get_double.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p,
                                             C.POINTER(C.c_double)]
        _shim = S
    return _shim


def _b(s):
    return s.encode()


class DataBlock:
    """Minimal CosmoSIS-like block: ``block[section, key] = value`` / read back."""

    def __init__(self):
        self._p = C.c_void_p(shim().y3b_datablock_new())

    def close(self):
        if self._p:
            shim().y3b_datablock_free(self._p)
            self._p = None

    __del__ = close

    @property
    def ptr(self):
        return self._p

    def __setitem__(self, key, value):
        sec, name = map(_b, key)
        S = shim()
        if isinstance(value, str):
            S.c_datablock_put_string(self._p, sec, name, _b(value))
        elif isinstance(value, (bool, int, np.integer)):
            S.c_datablock_put_int(self._p, sec, name, int(value))
        elif isinstance(value, (float, np.floating)):
            S.c_datablock_put_double(self._p, sec, name, float(value))
        else:
            arr = np.asarray(value)
            if arr.dtype.kind in "iu" and arr.ndim == 1:
                a = np.ascontiguousarray(arr, dtype=np.int32)
                S.c_datablock_put_int_array_1d(self._p, sec, name,
                                               a.ctypes.data_as(C.POINTER(C.c_int)), a.size)
            else:
                a = np.ascontiguousarray(arr, dtype=np.float64)
                ext = (C.c_int * a.ndim)(*a.shape)
                S.c_datablock_put_double_array(self._p, sec, name,
                                               a.ctypes.data_as(C.POINTER(C.c_double)),
                                               a.ndim, ext)

    def __contains__(self, key):
        return bool(shim().c_datablock_has_value(self._p, *map(_b, key)))

    def __getitem__(self, key):
        sec, name = map(_b, key)
        S = shim()
        nd = C.c_int()
        if S.c_datablock_get_array_ndim(self._p, sec, name, C.byref(nd)) == 0:
            ext = (C.c_int * nd.value)()
            S.c_datablock_get_double_array_shape(self._p, sec, name, nd.value, ext)
            out = np.empty(tuple(ext))
            rc = S.c_datablock_get_double_array(self._p, sec, name,
                                                out.ctypes.data_as(C.POINTER(C.c_double)),
                                                nd.value, ext)
            if rc != 0:
                raise KeyError(key)
            return out
        v = C.c_double()
        if S.c_datablock_get_double(self._p, sec, name, C.byref(v)) == 0:
            return v.value
        raise KeyError(key)


class Module:
    """One CosmoSIS module .so driven through setup / execute / cleanup."""

    def __init__(self, name):
        shim()
        path = os.path.join(LIB_DIR, name + ".so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} not built")
        self.lib = C.CDLL(path)
        self.lib.setup.argtypes = [C.c_void_p]
        self.lib.setup.restype = C.c_void_p
        self.lib.execute.argtypes = [C.c_void_p, C.c_void_p]
        self.lib.execute.restype = C.c_int
        self.lib.cleanup.argtypes = [C.c_void_p]
        self.lib.cleanup.restype = C.c_int
        self.handle = None

    def setup(self, options: DataBlock):
        self.handle = self.lib.setup(options.ptr)
        return self.handle

    def execute(self, block: DataBlock) -> int:
        return self.lib.execute(block.ptr, self.handle)

    def cleanup(self) -> int:
        rc = self.lib.cleanup(self.handle)
        self.handle = None
        return rc
