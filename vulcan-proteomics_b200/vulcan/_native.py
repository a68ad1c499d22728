"""Loader of the in-tree native libraries (``vulcan/lib/``, built from ``csrc/`` by ``make -C csrc``).

There is no fallback: a missing or stale library raises, so a search never silently runs anything but the
sm_100a kernels.
"""
from __future__ import annotations

import ctypes as C
import os

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
GPU_SO = os.path.join(LIB_DIR, "libvulcan_b200.so")
CORE_SO = os.path.join(LIB_DIR, "libvulcan_core.so")

_core = None


CSRC = os.path.join(os.path.dirname(LIB_DIR), "..", "csrc")


def _source_digest(which: str) -> str | None:
    """Hash of the library's sources, when they are present next to the package (None otherwise)."""
    stamp_py = os.path.join(CSRC, "stamp.py")
    if not os.path.exists(stamp_py):
        return None
    import importlib.util
    spec = importlib.util.spec_from_file_location("_vk_stamp", stamp_py)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.digest(which)


def _load(path: str, what: str):
    if not os.path.exists(path):
        raise RuntimeError(f"{what} not built: {path} is missing (run `make -C vulcan-proteomics_b200/csrc`)")
    which = "gpu" if path == GPU_SO else "core"
    want = _source_digest(which)
    stamp = path[:-3] + ".sha256"
    if want is not None:
        got = open(stamp).read().strip() if os.path.exists(stamp) else None
        if got != want:
            raise RuntimeError(f"{what} is stale: {path} was not built from the current sources "
                               f"(run `make -C vulcan-proteomics_b200/csrc`)")
    return C.CDLL(path)


def core_lib():
    """libvulcan_core.so: host index-build core."""
    global _core
    if _core is None:
        L = _load(CORE_SO, "native index core")
        L.vc_expand_pairs.restype = C.c_int64
        L.vc_expand_pairs.argtypes = [C.c_int64] + [C.c_void_p] * 9 + [C.c_double, C.c_int, C.c_void_p, C.c_void_p,
                                                                          C.c_double, C.c_double, C.c_uint64,
                                                                          C.c_int] + \
            [C.c_void_p] * 9
        L.vc_xxh64.restype = C.c_uint64
        L.vc_xxh64.argtypes = [C.c_char_p, C.c_int64, C.c_uint64]
        _core = L
    return _core
