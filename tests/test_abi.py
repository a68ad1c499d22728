"""The C ABI: the built library loads without a GPU, exports every function include/vulcan_b200.h declares, and
the ctypes binding of vulcan/gpu/_lib.py matches the header argument for argument."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
HEADER = os.path.join(ROOT, "include", "vulcan_b200.h")
REFERENCE_NAMES = ("vk_set_params", "vk_set_nterm", "vk_set_tol_da", "vk_frag_count", "vk_frag_emit", "vk_k1",
                   "vk_k1_brute", "vk_k2", "vk_k2_shift")


def _decls():
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    return re.findall(r"\b(int|int64_t)\s+(vk_\w+)\s*\(([^)]*)\)\s*;", src)


def _ctype(arg):
    arg = arg.strip()
    if arg == "void":
        return None
    if "*" in arg:
        return C.c_void_p
    t = arg.rsplit(" ", 1)[0]
    return {"int": C.c_int, "int64_t": C.c_int64, "float": C.c_float, "double": C.c_double}[t]


def test_library_exports_every_declared_function():
    from vulcan import _native
    L = _native._load(_native.GPU_SO, "CUDA kernel library")
    names = [n for _, n, _ in _decls()]
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    for n in REFERENCE_NAMES:
        assert n in names


def test_ctypes_binding_matches_header():
    txt = open(os.path.join(ROOT, "vulcan-proteomics_b200", "vulcan", "gpu", "_lib.py")).read()
    ns = {}
    exec("import ctypes as C\nP = C.c_void_p\nI32, I64, F32, F64, U32 = C.c_int, C.c_int64, C.c_float, C.c_double, "
         "C.c_uint32\n" + txt[txt.index("_SIGS = {"):txt.index("_lib = None")], ns)
    sigs = {**ns["_SIGS"], **ns["_SIGS_B200"]}
    for ret, name, args in _decls():
        want = [t for t in (_ctype(a) for a in args.split(",") if a.strip()) if t is not None]
        if name in sigs:
            assert [w.__name__ for w in want] == [g.__name__ for g in sigs[name]], name
            assert ret == "int", name
    for n in REFERENCE_NAMES:
        assert n in sigs


def test_reference_signatures_unchanged():
    """Part 1 keeps the reference's ctypes signature lists (vulcan/gpu/_lib.py:22-35 of the reference)."""
    from vulcan.gpu import _lib as K
    P, I32, I64, F32, F64 = C.c_void_p, C.c_int, C.c_int64, C.c_float, C.c_double
    assert K._SIGS["vk_k1"] == [I32, P, P, P, P, P, P, P, P, P, P, I32, I32, I32, I32, F32, F32, F32, F64, I32, I64,
                                P, P, P, P, P, P, P]
    assert K._SIGS["vk_k2"] == [I32, P, P, P, P, P, P, P, P, P, P, P, P, F32, F32, P, P, P, P, P, P, P, P, I32, P]
    assert K._SIGS["vk_frag_emit"] == [I64, P, P, P, P, P, I32, F32, F32, F64, I32, I64, P, P, P]


def test_stale_library_is_refused(tmp_path, monkeypatch):
    """A library not built from the current sources is refused, never silently used."""
    from vulcan import _native
    fake = tmp_path / "libvulcan_b200.so"
    fake.write_bytes(open(_native.GPU_SO, "rb").read())
    (tmp_path / "libvulcan_b200.sha256").write_text("0" * 64)
    monkeypatch.setattr(_native, "GPU_SO", str(fake))
    with pytest.raises(RuntimeError, match="stale"):
        _native._load(str(fake), "CUDA kernel library")


def test_missing_library_fails_loudly(tmp_path):
    from vulcan import _native
    with pytest.raises(RuntimeError, match="not built"):
        _native._load(str(tmp_path / "nope.so"), "CUDA kernel library")


def test_window_peak_mode_arguments_are_checked_before_any_device_call():
    """vk_k0w_count / vk_k0w_fill refuse a window width that is not positive and finite, and a fragment range past
    999 windows (where the reference's group ids spectrum * 1000 + window would merge spectra), before they touch
    the device: callable here without a GPU."""
    from vulcan import _native
    L = _native._load(_native.GPU_SO, "CUDA kernel library")
    P, I32, F32 = C.c_void_p, C.c_int, C.c_float
    L.vk_k0w_count.argtypes = [I32, P, P, P, F32, F32, F32, I32, P, P, P, P, P]
    L.vk_k0w_fill.argtypes = [I32, P, P, P, F32, F32, F32, I32, I32, P, P, P, P, P, I32, P, P, P, P]
    vk_e_arg = int(re.search(r"#define VK_E_ARG\s+\((-?\d+)\)", open(HEADER).read()).group(1))
    for th, fmin, fmax in ((0.0, 150.0, 2000.0), (-5.0, 150.0, 2000.0), (float("nan"), 150.0, 2000.0),
                           (float("inf"), 150.0, 2000.0), (1.0, 150.0, 2000.0), (2.0, 150.0, 2000.0),
                           (100.0, -150.0, 2000.0)):
        assert L.vk_k0w_count(1, None, None, None, fmin, fmax, th, 15, None, None, None, None, None) == vk_e_arg
        assert L.vk_k0w_fill(1, None, None, None, fmin, fmax, th, 15, 1, None, None, None, None, None, 0, None, None,
                             None, None) == vk_e_arg


def test_scan_launch_shape_is_a_host_rule():
    """vk_scan_kernels (host only, callable without a GPU): 0 kernels for an empty input, 1 up to one block of 4,096
    values, 2 up to 2,048 blocks (each block adds up the block sums before it), 3 beyond."""
    from vulcan import _native
    L = _native._load(_native.GPU_SO, "CUDA kernel library")
    L.vk_scan_kernels.argtypes = [C.c_int64]
    L.vk_scan_kernels.restype = C.c_int
    for n, k in ((0, 0), (1, 1), (4096, 1), (4097, 2), (2048 * 4096, 2), (2048 * 4096 + 1, 3), (1 << 40, 3)):
        assert L.vk_scan_kernels(n) == k, n


def test_header_compiles_as_c_and_links(tmp_path):
    """A C binding (cgo, JNI, N-API) includes the header as C99 and links the library: a program that takes the
    address of every declared entry point compiles, links and loads (it calls none of them)."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    from vulcan import _native
    names = [n for _, n, _ in _decls()]
    src = tmp_path / "bind.c"
    src.write_text('#include "vulcan_b200.h"\n#include <stdio.h>\nint main(void) {\n  const void* fns[] = {'
                   + ", ".join(f"(const void*)&{n}" for n in names)
                   + '};\n  printf("%d\\n", (int)(sizeof fns / sizeof fns[0]));\n  return 0;\n}\n')
    lib = _native.GPU_SO
    r = subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                        "-o", str(tmp_path / "bind"), lib, f"-Wl,-rpath,{os.path.dirname(lib)}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(tmp_path / "bind")], capture_output=True, text=True, timeout=60)   # no device calls
    assert run.returncode == 0 and int(run.stdout) == len(names)
