"""ctypes binding of ``vulcan/lib/libvulcan_b200.so`` (built from ``csrc/`` for sm_100a).

Mirrors the reference's ``vulcan/gpu/_lib.py`` (``lib()``, ``ptr()``, ``stream()``, ``check()``; the reference
signatures of ``_SIGS`` are kept name for name) and adds the B200 entry points of ``include/vulcan_b200.h``.
There is no fallback: if the library is missing, ``lib()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import torch

from .._native import GPU_SO, _load

P = C.c_void_p
I32, I64, F32, F64, U32 = C.c_int, C.c_int64, C.c_float, C.c_double, C.c_uint32


class FragParams(C.Structure):
    """vk_frag_params"""
    _fields_ = [("mono", C.c_float * 26), ("stat", C.c_float * 26), ("var", C.c_float * 26),
                ("nterm", C.c_float), ("tol_da", C.c_int)]


class TIndex(C.Structure):
    """vk_tindex"""
    _fields_ = [("n_rows", C.c_int64), ("n_tiles", C.c_int64), ("n_postings", C.c_int64),
                ("tile_shift", C.c_int32), ("row_bits", C.c_int32), ("mass_bits", C.c_int32),
                ("cbin_bits", C.c_int32), ("fmin_bits", C.c_uint32), ("fmax_bits", C.c_uint32),
                ("min_ion_index", C.c_int32), ("max_tile_postings", C.c_int32),
                ("tile_off", P), ("cbin_off", P), ("postings", P), ("bitmap", P)]


class PsmPackIn(C.Structure):
    """vk_psm_pack_in"""
    _fields_ = [("psm_cand", P), ("psm_rank", P), ("dnext", P), ("dbest", P), ("c_hyp", P), ("c_row", P),
                ("c_cnt", P), ("h_z", P), ("h_iso", P), ("h_pm", P), ("n_hyp", C.c_int64), ("spec_scored", P),
                ("spec_matched", P), ("tic", P), ("hs", P), ("sb", P), ("sy", P), ("ppm", P), ("mb", P), ("my", P),
                ("lb", P), ("ly", P), ("mass32", P), ("length", P), ("pf_id", P), ("missed", P), ("n_var", P),
                ("n_rows", C.c_int64)]


class FusedIn(C.Structure):
    """vk_fused_in"""
    _fields_ = [("n_spec", C.c_int), ("n_work", C.c_int), ("spec_ids", P), ("pk_off", P), ("pk_mass", P),
                ("pk_int", P), ("spec_hyp_off", P), ("h_lo", P), ("h_hi", P), ("h_maxfz", P), ("partner", P),
                ("seq_off", P), ("len", P), ("mask", P), ("mass32", P), ("res", P), ("tol_lo", C.c_float),
                ("tol_hi", C.c_float), ("thr", C.c_int), ("topk", C.c_int), ("pair_closure", C.c_int),
                ("min_matched", C.c_int), ("report", C.c_int)]


_K2_FIELDS = [("hs", P), ("sb", P), ("sy", P), ("ppm", P), ("mb", P), ("my", P), ("lb", P), ("ly", P)]


class PsmOut(C.Structure):
    """vk_psm_out"""
    _fields_ = [("row", P), ("hyp", P), ("k1", P), ("rank", P), ("dnext", P), ("dbest", P)] + _K2_FIELDS


class CandOut(C.Structure):
    """vk_cand_out"""
    _fields_ = [("cap", C.c_int), ("n_cand", P), ("c_hyp", P), ("c_row", P), ("c_cnt", P)] + _K2_FIELDS


# reference-compatible signatures (vulcan/gpu/_lib.py:22-35 of the reference)
_SIGS = {
    "vk_set_params": [P, P, P],
    "vk_frag_count": [I64, P, P, P, P, P, I32, F32, F32, P, P],
    "vk_frag_emit": [I64, P, P, P, P, P, I32, F32, F32, F64, I32, I64, P, P, P],
    "vk_k1": [I32, P, P, P, P, P, P, P, P, P, P, I32, I32, I32, I32, F32, F32, F32, F64, I32, I64, P, P, P, P,
              P, P, P],
    "vk_k1_brute": [I64, P, P, P, P, P, P, P, P, P, P, P, I32, F32, F32, F32, F32, F64, P, P],
    "vk_k2": [I32, P, P, P, P, P, P, P, P, P, P, P, P, F32, F32, P, P, P, P, P, P, P, P, I32, P],
    "vk_set_nterm": [F32],
    "vk_k2_shift": [I32, P, P, P, P, P, P, P, P, P, P, P, P, F32, F32, P, P, P, P, P, P, P, P, P, I32, P],
    "vk_set_tol_da": [I32],
}
# B200 entry points
_SIGS_B200 = {
    "vk_tindex_layout": [I64, I32, F32, F32, I32, I32, P],
    "vk_tindex_count": [P, P, P, P, P, P, P, P, P],
    "vk_tindex_emit": [P, P, P, P, P, P, P, P, P, P],
    "vk_scan_i64": [P, I64, P, P, P],
    "vk_scan_i64_noalloc": [P, I64, P, P],
    "vk_k0_count": [I32, P, P, P, F32, F32, I32, P, P, P, P, P],
    "vk_k0_fill": [I32, P, P, P, F32, F32, I32, I32, P, P, P, P, P, I32, P, P, P, P],
    "vk_k0_fill_easy": [I32, P, P, P, F32, F32, I32, I32, P, P, P, P, P, I32, P, P, P, P],
    "vk_k0_fill_hard": [I32, P, P, P, F32, F32, I32, I32, P, P, P, P, P, I32, P, P, P, P],
    "vk_k0w_count": [I32, P, P, P, F32, F32, F32, I32, P, P, P, P, P],
    "vk_k0w_fill": [I32, P, P, P, F32, F32, F32, I32, I32, P, P, P, P, P, I32, P, P, P, P],
    "vk_hyp_count": [I32, P, P, P, I32, I32, I32, I32, P, P],
    "vk_hyp_fill": [I32, P, P, P, I32, I32, I32, I32, F32, F32, I32, P, I64, P, P, P, P, P, P, P, P, P, P],
    "vk_k1_plan_count": [P, I64, P, P, P, P, P],
    "vk_k1_plan_fill": [P, I64, P, P, P, P, P, I64, P, P],
    "vk_k1_tiles": [P, P, F32, F32, I32, P, P, I64, I64, P, P, P, P, P, I64, P, P, P, P, P, P, P, P, P, I32, I64, P],
    "vk_k1_peak_keys": [P, P, F32, F32, P, P, I32, I64, P, P, P],
    "vk_k1_hits": [P, P, F32, F32, I32, P, P, I64, I64, P, P, P, P, P, I64, P, P, I32, P, P, P, P, P, P, P, P, P, P,
                   P, P, I32, I64, P],
    "vk_select_hits": [I32, P, P, P, P, P, P, P, P, P, P, I32, I32, P, I32, P, P, P, P, P, P, P, P],
    "vk_compact_hits": [I32, I32, P, P, P, P, P, P, P, P, P, P, P, P, P, P],
    "vk_compact_hits_features": [I32, I32, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P],
    "vk_tindex_bitmap": [P, P, P],
    "vk_select_topk": [I32, P, P, P, P, P, I64, P, I32, I32, I32, I32, P, P, P, P, P, P, P, P, P],
    "vk_compact_cands": [I32, I32, P, P, P, P, P, P, P, P, P, P, P, P],
    "vk_k2_spectra": [P, I32, P, P, P, P, P, P, P, P, P, P, P, F32, F32, P, P, P, P, P, P, P, P, P, P],
    "vk_k2_cands": [P, I32, P, P, P, P, P, P, P, P, P, P, P, F32, F32, P, P, P, P, P, P, P, P, P],
    "vk_pack_psms": [P, I64, I32, P, P, P, P],
    "vk_psm_rank": [I32, P, P, P, P, P, I32, I32, P, P, P, P, P, P],
    "vk_psm_rank_sparse": [I32, P, P, P, P, P, I32, I32, P, P, P, P, P, P],
    "vk_search_fused": [P, P, P, I32, I32, I32, P, P, P, P, P, P, P, P, P, P],
    "vk_search_fused_smem": [P, I32, I32, I32, I32, P],
    "vk_search_fused_grid": [P, I32, I32, I32, I32, P],
    "vk_cand_features": [I64, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P],
    "vk_mlp_infer": [I64, P, P, P, P, P, P, P, F32, P, I32, P],
    "vk_mlp_infer_tc": [I64, P, P, P, P, P, P, P, F32, P, I32, P, P],
    "vk_select_pruned": [I32, P, P, P, P, P, P, F32, I32, I32, I32, P, I32, I32, P, P, P, P, P],
    "vk_gemm": [I32, I32, I32, P, I64, I64, P, I32, I64, I64, P, I32, I32, P, I64, I64, P],
    "vk_tc_gemm": [I32, I32, I32, P, I64, I64, P, I32, I64, I64, P, I32, I32, P, I64, I64, P, I64, P, P],
    "vk_colsum": [I32, I32, P, P, P, I64, P, P],
    "vk_relu_mask": [I64, P, P, P],
    "vk_bce": [I32, P, P, P, F32, P, P, P],
    "vk_adam": [I64, P, P, P, P, F32, F32, F32, F32, I32, F32, P, P],
    "vk_to_bf16": [I64, P, P, P],
    "vk_bf16_to_f32": [I64, P, P, P],
}

_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    torch.cuda.init()
    L = _load(GPU_SO, "CUDA kernel library")
    for name, args in {**_SIGS, **_SIGS_B200}.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.vk_scan_tmp_bytes.argtypes = [I64]
    L.vk_scan_tmp_bytes.restype = I64
    L.vk_scan_kernels.argtypes = [I64]
    L.vk_scan_kernels.restype = C.c_int
    L.vk_scan_noalloc_max_n.argtypes = []
    L.vk_scan_noalloc_max_n.restype = I64
    L.vk_mlp_infer_smem.argtypes = []
    L.vk_mlp_infer_smem.restype = I64
    L.vk_tindex_bitmap_bytes.argtypes = [P]
    L.vk_tindex_bitmap_bytes.restype = I64
    L.vk_mlp_infer_tc_smem.argtypes = []
    L.vk_mlp_infer_tc_smem.restype = I64
    L.vk_tc_gemm_ws_floats.argtypes = [I32, I32, I32]
    L.vk_tc_gemm_ws_floats.restype = I64
    L.vk_colsum_ws_floats.argtypes = [I32, I32]
    L.vk_colsum_ws_floats.restype = I64
    _lib = L
    return L


def ptr(t: torch.Tensor | None):
    if t is None:
        return None
    assert t.is_cuda and t.is_contiguous(), "kernels need contiguous CUDA tensors"
    return t.data_ptr()


def stream():
    return torch.cuda.current_stream().cuda_stream


_TRACE = os.environ.get("VK_TRACE") == "1"
# kernels launched by one call of an entry point (counted by `check` into `LAUNCHES`; the default is 1)
_KERNELS_PER_CALL = {"scan": 3, "set_params": 0, "set_nterm": 0, "set_tol_da": 0, "tindex_layout": 0,
                     "fused_grid": 0, "k0_fill": 2, "k0w_fill": 2, "hyp_fill": 2}
LAUNCHES = {"n": 0}


def check(code: int, what: str, kernels: int | None = None):
    """Raise on a nonzero return code; count the call's kernels (``kernels``, else the entry point's usual number)."""
    LAUNCHES["n"] += (_KERNELS_PER_CALL.get(what, 1) if kernels is None else kernels) if code == 0 else 0
    if code != 0:
        raise RuntimeError(f"{what}: CUDA error {code}" if code > 0 else f"{what}: rejected argument ({code})")
    if _TRACE:   # debugging aid: finish every launch and report the stage before the next one
        torch.cuda.synchronize()
        print(f"[vk] {what} ok", file=sys.stderr, flush=True)
