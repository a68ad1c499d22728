"""Kernel goldens: the reference's own CUDA kernels (vulcan/gpu/kernels.cu, compiled unchanged for sm_100a by
`make -C oracle ref` into oracle/_ref/libvulcan_kernels_ref.so) run on the mini fixture.  Needs a GPU.

    python tests/golden/make_golden_ref.py --out tests/golden/golden_ref_kernels.npz

Inputs are the fixture plus the reference-Python goldens (K0 peaks, hypotheses, work items, window candidates of
golden_ref_py.npz), so every kernel sees exactly what the reference's engine would hand it.  The calls follow the
reference's engine (vulcan/gpu/engine.py: GpuIndex index build :82-148, run_k1 :250-281, k1_brute :483-497,
run_k2 :315-351): same entry points, same argument order, same CSR construction.
Outputs per parameter set: frag_count, sorted frag_emit keys, the K1 append set sorted by (hyp, row) with
scored/matched, brute-force counts and K2 outputs (closed and shifted) of every window candidate.
"""
from __future__ import annotations

import argparse
import ctypes as C
import math
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
from tests.golden.make_golden import PARAM_SETS, STATIC, VAR  # noqa: E402

SO = os.path.join(ROOT, "oracle", "_ref", "libvulcan_kernels_ref.so")
SAGE_MONO = np.array([71.03711, 0.0, 103.00919, 115.02694, 129.04259, 147.0684, 57.02146, 137.05891, 113.08406,
                      0.0, 128.09496, 113.08406, 131.0405, 114.04293, 237.14774, 97.05276, 128.05858, 156.1011,
                      87.03203, 101.04768, 150.95363, 99.06841, 186.07932, 0.0, 163.06332, 0.0], np.float32)
Pp = C.c_void_p
I32, I64, F32, F64 = C.c_int, C.c_int64, C.c_float, C.c_double
SIGS = {
    "vk_set_params": [Pp, Pp, Pp], "vk_set_nterm": [F32], "vk_set_tol_da": [I32],
    "vk_frag_count": [I64, Pp, Pp, Pp, Pp, Pp, I32, F32, F32, Pp, Pp],
    "vk_frag_emit": [I64, Pp, Pp, Pp, Pp, Pp, I32, F32, F32, F64, I32, I64, Pp, Pp, Pp],
    "vk_k1": [I32, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, I32, I32, I32, I32, F32, F32, F32, F64, I32, I64, Pp, Pp,
              Pp, Pp, Pp, Pp, Pp],
    "vk_k1_brute": [I64, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, I32, F32, F32, F32, F32, F64, Pp, Pp],
    "vk_k2": [I32, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, F32, F32, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, I32, Pp],
    "vk_k2_shift": [I32, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, F32, F32, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp, Pp,
                    I32, Pp],
}


def load(path=SO):
    L = C.CDLL(path)
    for k, v in SIGS.items():
        getattr(L, k).argtypes = v
        getattr(L, k).restype = C.c_int
    return L


def P(t):
    assert t.is_cuda and t.is_contiguous()
    return t.data_ptr()


def ck(code, what):
    if code != 0:
        raise RuntimeError(f"{what}: {code}")


def run(fx, g, L, name, kw):
    dev = torch.device("cuda")
    st = torch.cuda.current_stream().cuda_stream
    up = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    stat = np.zeros(26, np.float32)
    var = np.zeros(26, np.float32)
    for r, m in STATIC.items():
        stat[ord(r) - 65] = np.float32(m)
    for r, m in VAR.items():
        var[ord(r) - 65] = np.float32(m)
    da = int(kw.get("fragment_unit", "ppm") == "da")
    ck(L.vk_set_params(SAGE_MONO.ctypes.data, stat.ctypes.data, var.ctypes.data), "set_params")
    ck(L.vk_set_nterm(0.0), "set_nterm")
    ck(L.vk_set_tol_da(da), "set_tol_da")
    tol = kw["fragment_ppm"]
    fmin, fmax, min_ion = 150.0, 2000.0, 2
    chunk, tile, bin_ppm = 8192, 1024, 20.0
    seq_off, length = up(fx["idx_seq_off"].astype(np.int64)), up(fx["idx_length"].astype(np.uint8))
    mask, mass32 = up(fx["idx_mask"].view(np.int64)), up(fx["idx_mass32"].astype(np.float32))
    res = up(fx["idx_residues"].astype(np.uint8))
    n = len(fx["idx_pf_id"])
    tab = [P(seq_off), P(length), P(mask), P(mass32), P(res)]
    out = {}
    cnt = torch.empty(n, dtype=torch.int32, device=dev)
    ck(L.vk_frag_count(n, *tab, min_ion, fmin, fmax, P(cnt), st), "frag_count")
    out["frag_count"] = cnt.cpu().numpy()
    inv_logw = 1.0 / math.log1p(bin_ppm * 1e-6)
    n_bins = int(math.floor(math.log(fmax / fmin) * inv_logw)) + 2
    n_chunks = (n + chunk - 1) // chunk
    off = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    torch.cumsum(cnt.to(torch.int64), 0, out=off[1:])
    keys = torch.empty(int(off[-1]), dtype=torch.int64, device=dev)
    ck(L.vk_frag_emit(n, *tab, min_ion, fmin, fmax, inv_logw, chunk, 0, P(off), P(keys), st), "frag_emit")
    keys = torch.sort(keys).values
    out["frag_keys"] = keys.cpu().numpy()
    ent = keys & 0xFFFFFFFF
    entries = torch.where(ent >= 2 ** 31, ent - 2 ** 32, ent).to(torch.int32)
    lin = (keys >> 50) * n_bins + ((keys >> 32) & 0x3FFFF)
    offs = torch.zeros(n_chunks * n_bins + 1, dtype=torch.int64, device=dev)
    torch.cumsum(torch.bincount(lin, minlength=n_chunks * n_bins), 0, out=offs[1:])
    offs = torch.where(offs >= 2 ** 31, offs - 2 ** 32, offs).to(torch.int32)
    # peaks / hypotheses from the reference-Python goldens
    pk_off, pk_mass = up(g[f"{name}/k0_off"].astype(np.int64)), up(g[f"{name}/k0_mass"].astype(np.float32))
    pk_int = up(g[f"{name}/k0_int"].astype(np.float32))
    d_spec = up(g[f"{name}/hyp_spec"].astype(np.int32))
    d_maxfz = up(g[f"{name}/hyp_maxfz"].astype(np.int8))
    n_h = len(g[f"{name}/hyp_spec"])
    wi = {k: up(g[f"{name}/wi_{k}"].astype(np.int32)) for k in ("hyp", "chunk", "lo", "hi")}
    cap = max(1, int((g[f"{name}/hyp_hi"] - g[f"{name}/hyp_lo"]).clip(0).sum()))
    n_out = torch.zeros(1, dtype=torch.int64, device=dev)
    o_h, o_r, o_c = (torch.empty(cap, dtype=torch.int32, device=dev) for _ in range(3))
    scored = torch.zeros(n_h, dtype=torch.int32, device=dev)
    matched = torch.zeros(n_h, dtype=torch.int64, device=dev)
    ck(L.vk_k1(len(g[f"{name}/wi_hyp"]), P(wi["hyp"]), P(wi["chunk"]), P(wi["lo"]), P(wi["hi"]), P(d_spec),
               P(d_maxfz), P(pk_off), P(pk_mass), P(offs), P(entries), n_bins, 0, chunk, tile, tol[0], tol[1], fmin,
               inv_logw, 1, cap, P(n_out), P(o_h), P(o_r), P(o_c), P(scored), P(matched), st), "k1")
    m = int(n_out.item())
    key = (o_h[:m].long() << 32) | o_r[:m].long()
    o = torch.argsort(key)
    out["k1_key"] = key[o].cpu().numpy()
    out["k1_cnt"] = o_c[:m][o].cpu().numpy()
    out["k1_scored"] = scored.cpu().numpy()
    out["k1_matched"] = matched.cpu().numpy()
    h = up(g[f"{name}/win_h"].astype(np.int32))
    r = up(g[f"{name}/win_r"].astype(np.int32))
    bc = torch.empty(len(h), dtype=torch.int32, device=dev)
    ck(L.vk_k1_brute(len(h), P(h), P(r), P(d_spec), P(d_maxfz), P(pk_off), P(pk_mass), *tab, min_ion, fmin, fmax,
                     tol[0], tol[1], inv_logw, P(bc), st), "k1_brute")
    out["brute"] = bc.cpu().numpy()
    # K2 over every window candidate (sorted by spectrum), closed and shifted
    spec = d_spec[h.long()].long()
    us, cn = torch.unique_consecutive(spec, return_counts=True)
    coff = torch.zeros(len(us) + 1, dtype=torch.int64, device=dev)
    torch.cumsum(cn, 0, out=coff[1:])
    sid = us.to(torch.int32).contiguous()
    mfz = d_maxfz[h.long()].contiguous()
    nc = len(h)
    rng = np.random.default_rng(3)
    shift_np = np.where(rng.random(nc) < 0.5, rng.choice([15.9949, 79.96633, -18.010565, 0.984016], nc), 0.0)
    shift = up(shift_np.astype(np.float32))
    for mode in ("closed", "shift"):
        o = {"hs": torch.empty(nc, dtype=torch.float64, device=dev)}
        for k in ("sb", "sy", "ppm"):
            o[k] = torch.empty(nc, dtype=torch.float32, device=dev)
        for k in ("mb", "my", "lb", "ly"):
            o[k] = torch.empty(nc, dtype=torch.int16, device=dev)
        ptrs = [P(o[k]) for k in ("hs", "sb", "sy", "ppm", "mb", "my", "lb", "ly")]
        args = [len(us), P(coff), P(r), P(mfz), P(sid), P(pk_off), P(pk_mass), P(pk_int), *tab, tol[0], tol[1]]
        if mode == "closed":
            ck(L.vk_k2(*args, *ptrs, 128, st), "k2")
        else:
            ck(L.vk_k2_shift(*args, P(shift), *ptrs, 128, st), "k2_shift")
        for k, v in o.items():
            out[f"k2{mode}_{k}"] = v.cpu().numpy()
    out["k2shift_delta"] = shift_np.astype(np.float32)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    fx = dict(np.load(os.path.join(HERE, "mini_fixture.npz")))
    g = dict(np.load(os.path.join(HERE, "golden_ref_py.npz")))
    L = load()
    res = {}
    for name, kw in PARAM_SETS.items():
        for k, v in run(fx, g, L, name, kw).items():
            res[f"{name}/{k}"] = v
    np.savez_compressed(a.out, **res)
    print("wrote", a.out, len(res), "arrays")


if __name__ == "__main__":
    main()
