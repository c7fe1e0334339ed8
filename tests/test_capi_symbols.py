"""The C-ABI library loads on a CPU-only host and exports every entry point
that include/picsar_b200.h declares (no compute calls without a GPU)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(?:int|int32_t|int64_t)\s+(pxrb_\w+)\s*\(", src))
        for o in re.findall(r"PXRB_FGP_DECL\((\d)\)\s*$", src, flags=re.M):
            names.add(f"pxrb_field_gathering_plus_particle_pusher_{o}_{o}_{o}")
    names.discard("pxrb_field_gathering_plus_particle_pusher_")
    return {n for n in names if not n.endswith("##")}


def test_library_exports_all_declared_symbols():
    from picsar_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    declared = _declared()
    assert len(declared) >= 15
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_header():
    from picsar_b200 import _lib
    import picsar_b200.ensemble  # noqa: F401  (these modules register their signatures)
    import picsar_b200.peaks  # noqa: F401
    import picsar_b200.picsar  # noqa: F401
    import picsar_b200.psatd  # noqa: F401
    import picsar_b200.tiled  # noqa: F401
    declared = _declared()
    missing = sorted(declared - set(_lib.exported_symbols()))
    assert not missing, missing


def test_probe_flop_count_host():
    """pxrb_fma_probe_flops is a host function: the FLOPs of a probe launch
    (8 FMA chains per thread, an FMA counting two, packed f32x2 twice)."""
    from picsar_b200 import _lib
    import picsar_b200.peaks  # noqa: F401
    assert _lib.query("pxrb_fma_probe_flops", 0, 2, 64, 10) == 2 * 64 * 10 * 8 * 2
    assert _lib.query("pxrb_fma_probe_flops", 1, 2, 64, 10) == 2 * 64 * 10 * 8 * 2 * 2
    assert _lib.query("pxrb_fma_probe_flops", 2, 3, 32, 7) == 3 * 32 * 7 * 8 * 2
    assert _lib.query("pxrb_fma_probe_flops", 3, 1, 32, 1) == -1
    assert _lib.query("pxrb_fma_probe_flops", 0, 0, 32, 1) == -1


def test_max_threads_host():
    """The particle kernel's largest CTA per accumulator mode (host function)."""
    from picsar_b200 import _lib
    import picsar_b200.tiled  # noqa: F401
    assert _lib.query("pxrb_tiled_max_threads", 1) == 256
    assert _lib.query("pxrb_tiled_max_threads", 4) == 256
    assert _lib.query("pxrb_tiled_max_threads", 3) == 512
