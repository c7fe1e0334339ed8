"""ctypes binding of the reference's own routines translated to C
(``oracle/_ref/libpxr_ref.so``, built by ``make -C oracle ref`` from the
PICSAR Fortran sources with ``oracle/ftrans.py``).

TEST INFRASTRUCTURE ONLY: used by ``tests/test_oracle_vs_reference.py`` to
pin the oracle to the reference's code.  Every Fortran dummy is passed by
reference, so every argument here is a pointer: arrays as data pointers,
scalars boxed in ctypes values of the dummy's kind.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libpxr_ref.so")
# PICSAR src/ tree to translate; when unset, the oracle Makefile's default
REF_SRC = os.environ.get("PXR_REF_SRC")
_lib = None


def available() -> bool:
    """True when the translated reference is built, or can be built here."""
    try:
        lib()
        return True
    except OSError:
        return False


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            cmd = ["make", "-C", _HERE, "-s", "ref-if-present"]
            if REF_SRC:
                cmd.append(f"REF_SRC={REF_SRC}")
            subprocess.run(cmd, check=True)
        if not os.path.exists(LIB_PATH):
            raise OSError("translated reference not built and its sources absent "
                          "(set PXR_REF_SRC to PICSAR's src/ tree)")
        _lib = C.CDLL(LIB_PATH)
    return _lib


def i64(v):
    return C.byref(C.c_int64(int(v)))


def i32(v):
    return C.byref(C.c_int32(int(v)))


def f64(v):
    return C.byref(C.c_double(float(v)))


def arr(a, dtype=np.float64):
    if a.dtype != dtype:
        raise TypeError(f"expected {dtype}, got {a.dtype}")
    if a.ndim >= 2 and not a.flags.f_contiguous:
        raise ValueError("grids must be Fortran-ordered")
    if a.ndim < 2 and not a.flags.c_contiguous:
        raise ValueError("arrays must be contiguous")
    return a.ctypes.data_as(C.c_void_p)


def ivec(*v):
    """An INTEGER(idp) array argument such as nguard(3) or xlo(3)."""
    a = np.array(v, dtype=np.int64)
    return a, a.ctypes.data_as(C.c_void_p)


def set_module(clight=1.0, dt=0.0, particle_pusher=0, mu0=1.0, eps0=1.0):
    L = lib()
    L.pxrref_set_module.argtypes = [C.c_double, C.c_double, C.c_int64, C.c_double, C.c_double]
    L.pxrref_set_module(clight, dt, particle_pusher, mu0, eps0)


def call(name, *args):
    getattr(lib(), "pxrref_" + name)(*args)
