"""Loader of libpicsar_b200.so (the sm_100a kernels) through its C ABI.

There is no fallback: if the shared library is missing, cannot be loaded, or
no CUDA device is present, every entry point raises.  The library is built
in-tree by ``picsar_b200/csrc/Makefile`` (see ``__graft_entry__.build``).
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpicsar_b200.so")

i64, f64, P, I32 = C.c_int64, C.c_double, C.c_void_p, C.c_int

ERRORS = {
    1: "invalid argument (null pointer or inconsistent size)",
    2: "unsupported option (shape order / algorithm)",
    3: "CUDA launch error",
    4: "scratch buffer too small",
    5: "grid too small for its guard cells",
    6: "size above the entry point's fixed maximum",
}


class PicsarB200Error(RuntimeError):
    pass


# argument signatures: i = int64, d = double, p = pointer, s = stream (pointer)
_SIGS = {
    "pxrb_field_gathering_plus_particle_pusher": "i i" + " p" * 13 + " d" * 7 + " i" * 6
    + " p" * 6 + " d d i i d i d s",
    "pxrb_geteb3d_energy_conserving": "i" + " p" * 9 + " d" * 6 + " i" * 9 + " p" * 6
    + " i i i i i s",
    "pxrb_boris_push_u_3d": "i" + " p" * 10 + " d d d d s",
    "pxrb_ebcancelpush3d": "i" + " p" * 10 + " d d d i d s",
    "pxrb_set_gamma": "i p p p p d s",
    "pxrb_pushxyz": "i" + " p" * 7 + " d s",
    "pxrb_depose_jxjyjz": "p p p i" + " p" * 8 + " d" * 8 + " i" * 10 + " p s",
    "pxrb_depose_rho": "i p i p p p p" + " d" * 7 + " i" * 6 + " s",
    "pxrb_push_em3d_evec": " p" * 6 + " p p p" * 9 + " d d d d s",
    "pxrb_push_em3d_bvec": " p" * 6 + " p p p" * 6 + " d d d s",
    "pxrb_field_bc_periodic": "p p p" + " i" * 6 + " s",
    "pxrb_summation_bcs_periodic": "p p p" + " i" * 6 + " s",
    "pxrb_particle_bcs_periodic": "i p p p" + " d" * 6 + " s",
    "pxrb_particle_bin_sorting": "i" + " p" * 8 + " d" * 9 + " p i s",
    "pxrb_particle_bin_sorting_scratch": "=i i",
    "pxrb_push_em3d_evec_norder": "p" * 1 + " p" * 8 + " d p p p" + " i" * 13 + " s",
    "pxrb_push_em3d_bvec_norder": "p" + " p" * 5 + " p p p" + " i" * 13 + " s",
    "pxrb_fd_weights": "p i i",
    "pxrb_particle_bcs_scratch": "=i i",
    "pxrb_geteb2dxz_energy_conserving": "i" + " p" * 9 + " d" * 6 + " i" * 9 + " p" * 6
    + " i i i i i s",
    "pxrb_depose_jxjyjz_2d": "p p p i" + " p" * 8 + " d" * 6 + " i" * 7 + " s",
    "pxrb_push_em2d_evec": " p" * 6 + " p p p" * 9 + " d d d d s",
    "pxrb_push_em2d_bvec": " p" * 6 + " p p p" * 6 + " d d d s",
    "pxrb_pushxz": "i p p p p p d s",
    "pxrb_particle_bcs": "i" + " p" * 9 + " d" * 9 + " p p p p i p s",
}
for _o in (1, 2, 3):
    _SIGS[f"pxrb_field_gathering_plus_particle_pusher_{_o}_{_o}_{_o}"] = (
        "i" + " p" * 13 + " d" * 7 + " i" * 6 + " p" * 6 + " d d i i d i d s")

_CT = {"i": i64, "d": f64, "p": P, "s": P, "I": I32, "f": C.c_float}

_lib = None


def register(sigs: dict):
    """Add signatures (used by the other modules of the package)."""
    _SIGS.update(sigs)
    if _lib is not None:
        _declare(_lib, sigs)


def _declare(L, sigs):
    """A signature "a b c" returns int (status); "=i a b c" returns int64."""
    for name, sig in sigs.items():
        fn = getattr(L, name)
        parts = sig.split()
        restype = I32
        if parts and parts[0] == "=i":
            restype, parts = i64, parts[1:]
        fn.argtypes = [_CT[c] for c in parts]
        fn.restype = restype


def lib():
    """The loaded library (raises if it is absent: there is no CPU path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PicsarB200Error(
                f"{LIB_PATH} is missing: build it with `make -C picsar_b200/csrc` "
                "(there is no CPU fallback)")
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib, _SIGS)
    return _lib


def query(name: str, *args) -> int:
    """Call an entry point that returns a value (not a status)."""
    return int(getattr(lib(), name)(*args))


def call(name: str, *args):
    rc = getattr(lib(), name)(*args)
    if rc != 0:
        raise PicsarB200Error(f"{name} failed with status {rc}: {ERRORS.get(rc, 'unknown')}")
    return rc


def exported_symbols():
    return sorted(_SIGS)
