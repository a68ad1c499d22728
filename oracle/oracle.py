"""CPU oracle of the DDA search hot path -- TEST INFRASTRUCTURE ONLY.

Imported only by tests/, ``__graft_entry__.smoke()`` and ``bench.py`` (its CPU baseline and reference arm), as
the checker or the timed CPU baseline.  The product package never imports it.

Pieces (each cites the reference lines it restates):
  k0_view            vulcan/gpu/engine.py:171-210   peak view (range filter, top max_peaks or top window_k per
                                                    window_th window, mass sort, TIC)
  make_hypotheses    vulcan/gpu/host.py:64-91       precursor hypotheses + row windows (f32 Sage arithmetic)
  window_candidates  vulcan/gpu/engine.py:468-480   exhaustive (hyp, row) set sorted by (spectrum, row)
  k1_windows         vulcan/gpu/kernels.cu:195-232  K1 counts of every window row (C, vk_oracle.c)
  k1_appended        vulcan/gpu/kernels.cu:170-189  threshold append + per-hypothesis scored / matched
  select_topk        vulcan/gpu/engine.py:284-312   per-spectrum top-K + pair closure + unique (spectrum, row)
  k2                 vulcan/gpu/kernels.cu:263-376  exact rescoring (C)
  k2_f64             same matches, FP64 sums        hyperscore oracle (C)
  psm_rank           vulcan/gpu/engine.py:366-392   filter, rank by (hyperscore desc, row asc), delta_next/best
  lnfact             vulcan/gpu/engine.py:354-358
"""
from __future__ import annotations

import ctypes as C
import hashlib
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "libvk_oracle.so")

PROTON = np.float32(1.0072764)
NEUTRON = np.float32(1.00335)
ROW_BITS = 28
SAGE_MONO = np.array([71.03711, 0.0, 103.00919, 115.02694, 129.04259, 147.0684, 57.02146, 137.05891, 113.08406,
                      0.0, 128.09496, 113.08406, 131.0405, 114.04293, 237.14774, 97.05276, 128.05858, 156.1011,
                      87.03203, 101.04768, 150.95363, 99.06841, 186.07932, 0.0, 163.06332, 0.0], np.float32)


class OrParams(C.Structure):
    _fields_ = [("mono", C.c_float * 26), ("stat", C.c_float * 26), ("var", C.c_float * 26),
                ("nterm", C.c_float), ("tol_da", C.c_int)]


def make_params(static_mods: dict, var_mods: dict, fragment_unit: str = "ppm") -> OrParams:
    P = OrParams()
    stat = np.zeros(26, np.float32)
    var = np.zeros(26, np.float32)
    nterm = 0.0
    for r, m in static_mods.items():
        stat[ord(r) - 65] = np.float32(m)
    for r, m in var_mods.items():
        if r == "^":
            nterm = float(m)
            continue
        var[ord(r) - 65] = np.float32(m)
    for i in range(26):
        P.mono[i] = float(SAGE_MONO[i])
        P.stat[i] = float(stat[i])
        P.var[i] = float(var[i])
    P.nterm = nterm
    P.tol_da = int(fragment_unit == "da")
    return P


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            subprocess.run(["make", "-C", HERE, "libvk_oracle.so"], check=True, capture_output=True)
        _lib = C.CDLL(SO)
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def n_threads() -> int:
    return len(os.sched_getaffinity(0))


# ---------------------------------------------------------------------------------------------------- K0
def k0_view(sp, p):
    """engine.py:171-210 on the CPU: keep fragment_min_mz <= mz <= fragment_max_mz (not NaN), mass = mz - PROTON,
    top max_peaks per spectrum by (intensity desc, mass desc, input order), then mass ascending (ties keep
    that order).  TIC = f64 sum of the kept intensities.  valid = kept >= min_peaks.

    Window peak mode (any peak_mode but "global", engine.py:182-183): the groups are spectrum * 1000 +
    floor(mz / window_th) and window_k peaks are kept per group.  The reference evaluates the division on an f32
    CUDA tensor with a Python float divisor, which the device computes as mz * (1.0f / f32(window_th)) in f32; this
    restatement does the same."""
    n = len(sp.offsets) - 1
    mz = np.asarray(sp.mz, np.float32)
    it = np.asarray(sp.intensity, np.float32)
    lens = np.diff(sp.offsets)
    seg = np.repeat(np.arange(n), lens)
    keep = (mz >= np.float32(p.fragment_min_mz)) & (mz <= np.float32(p.fragment_max_mz)) & ~np.isnan(mz)
    mass = (mz - PROTON).astype(np.float32)
    seg, mass, it, mzk = seg[keep], mass[keep], it[keep], mz[keep]
    if p.peak_mode == "global":
        grp, kk = seg, p.max_peaks
    else:
        inv = np.float32(1.0) / np.float32(p.window_th)
        grp = seg * 1000 + np.floor((mzk * inv).astype(np.float32)).astype(np.int64)
        kk = p.window_k
    idx = np.arange(len(seg))
    o = np.lexsort((idx, -mass.astype(np.float64), -it.astype(np.float64), grp))
    g = grp[o]
    first = np.searchsorted(g, g, side="left")
    rank = np.arange(len(g)) - first
    o = o[rank < kk]
    pos = np.empty(len(o), np.int64)
    pos[:] = np.arange(len(o))
    o2 = np.lexsort((pos, mass[o], seg[o]))
    o = o[o2]
    seg, mass, it = seg[o], mass[o], it[o]
    cnt = np.bincount(seg, minlength=n)
    off = np.zeros(n + 1, np.int64)
    np.cumsum(cnt, out=off[1:])
    tic = np.zeros(n, np.float64)
    np.add.at(tic, seg, it.astype(np.float64))
    return {"off": off, "mass": mass, "int": it, "tic": tic.astype(np.float32), "valid": cnt >= p.min_peaks}


def k0_view_c(sp, p, nthreads=None):
    """``k0_view`` for the global peak mode in C, per spectrum on all cores (the same outputs; the tests check
    them against ``k0_view``).  Other peak modes: ``k0_view`` itself."""
    if p.peak_mode != "global":
        return k0_view(sp, p)
    n = len(sp.offsets) - 1
    raw_off = _c(sp.offsets, np.int64)
    mz = _c(sp.mz, np.float32)
    it = _c(sp.intensity, np.float32)
    off = np.empty(n + 1, np.int64)
    mass = np.empty(max(len(mz), 1), np.float32)
    inten = np.empty(max(len(mz), 1), np.float32)
    tic = np.empty(max(n, 1), np.float32)
    valid = np.empty(max(n, 1), np.uint8)
    lib().or_k0_global(C.c_int64(n), _p(raw_off), _p(mz), _p(it), C.c_float(p.fragment_min_mz),
                       C.c_float(p.fragment_max_mz), C.c_int(p.max_peaks), C.c_int(p.min_peaks), _p(off), _p(mass),
                       _p(inten), _p(tic), _p(valid), C.c_int(nthreads or n_threads()))
    k = int(off[-1])
    return {"off": off, "mass": mass[:k].copy(), "int": inten[:k].copy(), "tic": tic[:n].copy(),
            "valid": valid[:n].astype(bool)}


# ---------------------------------------------------------------------------------------------------- hypotheses
def make_hypotheses(sp, valid, idx_mass32, p):
    """host.py:64-91, written with the reference's own concatenate-then-lexsort structure."""
    s_ids, zs, isos = [], [], []
    spec = np.nonzero(np.asarray(valid, bool) & np.isfinite(sp.precursor_mz))[0]
    zi = sp.charge[spec].astype(np.int64)
    known = zi > 0
    zr = np.arange(p.precursor_charge[0], p.precursor_charge[1] + 1)
    for iso in range(p.isotope_errors[0], p.isotope_errors[1] + 1):
        s_ids.append(spec[known])
        zs.append(zi[known])
        isos.append(np.full(known.sum(), iso))
        for z in zr:
            s_ids.append(spec[~known])
            zs.append(np.full((~known).sum(), z))
            isos.append(np.full((~known).sum(), iso))
    s, z, iso = np.concatenate(s_ids), np.concatenate(zs), np.concatenate(isos)
    o = np.lexsort((iso, z, s))
    s, z, iso = s[o], z[o], iso[o]
    mz = (sp.precursor_mz[s].astype(np.float32) - PROTON).astype(np.float32)
    pm = (mz * z.astype(np.float32)).astype(np.float32)
    M = (pm - (iso.astype(np.float32) * NEUTRON).astype(np.float32)).astype(np.float32)
    plo, phi = np.float32(p.precursor_ppm[0]), np.float32(p.precursor_ppm[1])
    lo = (M + (M * plo) / np.float32(1e6)).astype(np.float32)
    hi = (M + (M * phi) / np.float32(1e6)).astype(np.float32)
    rlo = np.searchsorted(idx_mass32, lo, side="left")
    rhi = np.searchsorted(idx_mass32, hi, side="right")
    mfc = p.max_fragment_charge
    maxfz = np.maximum(np.minimum(z, mfc + 1) if mfc else z, 2).astype(np.int8)
    return {"spec": s.astype(np.int32), "z": z.astype(np.int8), "iso": iso.astype(np.int8), "pm": pm, "M": M,
            "lo": rlo.astype(np.int64), "hi": rhi.astype(np.int64), "maxfz": maxfz}


def window_candidates(hyp, spec_subset=None):
    """engine.py:468-480: every (hyp, row) of the windows, sorted by (spectrum, row)."""
    lo, hi = hyp["lo"], hyp["hi"]
    hsel = np.arange(len(lo))
    if spec_subset is not None:
        hsel = hsel[np.isin(hyp["spec"], spec_subset)]
    n = (hi - lo)[hsel]
    hh = np.repeat(hsel, n)
    rr = np.repeat(lo[hsel], n) + (np.arange(n.sum()) - np.repeat(np.cumsum(n) - n, n))
    s = hyp["spec"][hh]
    o = np.lexsort((rr, s))
    return hh[o].astype(np.int64), rr[o].astype(np.int64)


# ---------------------------------------------------------------------------------------------------- K1
def k1_brute(l1, hyp, peaks, h, r, p, P, nthreads=None):
    out = np.empty(len(h), np.int32)
    lib().or_k1_brute(C.c_int64(len(h)), _p(_c(h, np.int32)), _p(_c(r, np.int32)), _p(_c(hyp["spec"], np.int32)),
                      _p(_c(hyp["maxfz"], np.int8)), _p(_c(peaks["off"], np.int64)), _p(_c(peaks["mass"], np.float32)),
                      _p(_c(l1.seq_off, np.int64)), _p(_c(l1.length, np.uint8)), _p(_c(l1.mask, np.uint64)),
                      _p(_c(l1.mass32, np.float32)), _p(_c(l1.residues, np.uint8)), C.c_int(p.min_ion_index),
                      C.c_float(p.fragment_min_mz), C.c_float(p.fragment_max_mz), C.c_float(p.fragment_ppm[0]),
                      C.c_float(p.fragment_ppm[1]), _p(out), C.byref(P), C.c_int(nthreads or n_threads()))
    return out


def k1_windows(l1, hyp, peaks, p, P, nthreads=None, arrays=None, tic=None):
    """Dense K1 counts of every window row; returns (win_off, cnt, scored, matched), plus, when ``tic`` (f32 per
    spectrum) is given, the summed matched intensity of every window row: u32 sum over the matches of
    round_half_even(intensity * f32(2^24 / tic)) (the pruner's intensity feature)."""
    a = arrays or {k: getattr(l1, k) for k in ("seq_off", "length", "mask", "mass32", "residues")}
    lo = _c(hyp["lo"], np.int64)
    hi = _c(hyp["hi"], np.int64)
    n_h = len(lo)
    win_off = np.zeros(n_h + 1, np.int64)
    np.cumsum(hi - lo, out=win_off[1:])
    cnt = np.empty(int(win_off[-1]), np.int32)
    scored = np.zeros(n_h, np.uint32)
    matched = np.zeros(n_h, np.uint64)
    isum = np.zeros(len(cnt), np.uint32) if tic is not None else None
    lib().or_k1_windows(C.c_int64(n_h), _p(_c(hyp["spec"], np.int32)), _p(_c(hyp["maxfz"], np.int8)), _p(lo), _p(hi),
                        _p(win_off), _p(_c(peaks["off"], np.int64)), _p(_c(peaks["mass"], np.float32)),
                        _p(_c(a["seq_off"], np.int64)), _p(_c(a["length"], np.uint8)), _p(_c(a["mask"], np.uint64)),
                        _p(_c(a["mass32"], np.float32)), _p(_c(a["residues"], np.uint8)), C.c_int(p.min_ion_index),
                        C.c_float(p.fragment_min_mz), C.c_float(p.fragment_max_mz), C.c_float(p.fragment_ppm[0]),
                        C.c_float(p.fragment_ppm[1]), _p(cnt), _p(scored), _p(matched),
                        _p(_c(peaks["int"], np.float32)) if tic is not None else None,
                        _p(_c(tic, np.float32)) if tic is not None else None,
                        _p(isum) if tic is not None else None, C.byref(P), C.c_int(nthreads or n_threads()))
    if tic is not None:
        return win_off, cnt, scored, matched, isum
    return win_off, cnt, scored, matched


FRAG_BIN_TH = 0.02   # m/z bin width of the oracle's fragment index (Th)
_FRAG_INDEX = {}


def frag_index(l1, p, P, arrays=None, nthreads=None):
    """The index fragments of every row of ``l1`` (kernels.cu:53-71 arithmetic, ion index > min_ion_index, fmin <= f
    <= fmax) binned by m/z from fmin in FRAG_BIN_TH bins, rows ascending within a bin: (bin_off, mass, row, n_bins).
    Built once per index and fragment setting (the reference's K1 searches such an index, kernels.cu:112-190)."""
    a = arrays or {k: getattr(l1, k) for k in ("seq_off", "length", "mask", "mass32", "residues")}
    m32 = np.asarray(a["mass32"])
    so = np.asarray(a["seq_off"])
    # the index's content (an id can be reused once an index object is freed): length, every 256th mass and the
    # residue total, with the fragment settings
    fp = hashlib.blake2b(np.ascontiguousarray(m32[::max(1, len(m32) // 256)]).tobytes() +
                         np.asarray([len(m32), int(so[-1]) if len(so) else 0], np.int64).tobytes(),
                         digest_size=16).hexdigest()
    key = (fp, p.min_ion_index, float(p.fragment_min_mz), float(p.fragment_max_mz), bytes(P.mono), bytes(P.stat),
           bytes(P.var), float(P.nterm))
    hit = _FRAG_INDEX.get(key)
    if hit is not None:
        return hit
    arr = {k: _c(a[k], dt) for k, dt in (("seq_off", np.int64), ("length", np.uint8), ("mask", np.uint64),
                                         ("mass32", np.float32), ("residues", np.uint8))}
    n = len(arr["mass32"])
    cnt = np.empty(n, np.int32)
    lib().or_frag_count(C.c_int64(n), _p(arr["seq_off"]), _p(arr["length"]), _p(arr["mask"]), _p(arr["mass32"]),
                        _p(arr["residues"]), C.c_int(p.min_ion_index), C.c_float(p.fragment_min_mz),
                        C.c_float(p.fragment_max_mz), _p(cnt), C.byref(P))
    total = int(cnt.sum(dtype=np.int64))
    n_bins = max(1, int(np.ceil((float(np.float32(p.fragment_max_mz)) - float(np.float32(p.fragment_min_mz)))
                               / FRAG_BIN_TH)) + 1)
    bin_off = np.empty(n_bins + 1, np.int64)
    mass = np.empty(max(total, 1), np.float32)
    row = np.empty(max(total, 1), np.int32)
    lib().or_frag_index_build(C.c_int64(n), _p(arr["seq_off"]), _p(arr["length"]), _p(arr["mask"]),
                              _p(arr["mass32"]), _p(arr["residues"]), C.c_int(p.min_ion_index),
                              C.c_float(p.fragment_min_mz), C.c_float(p.fragment_max_mz), C.c_double(FRAG_BIN_TH),
                              C.c_int64(n_bins), _p(bin_off), _p(mass), _p(row), C.byref(P),
                              C.c_int(nthreads or n_threads()))
    _FRAG_INDEX.clear()   # one index at a time (the human index's is about 1.2 GB)
    _FRAG_INDEX[key] = (bin_off, mass, row, n_bins)
    return _FRAG_INDEX[key]


def k1_index(l1, hyp, peaks, p, P, nthreads=None, arrays=None, tic=None):
    """``k1_windows``' outputs (the same counts, statistics and intensity sums) from the fragment index
    (``frag_index``): per peak window the bins it touches, and in each bin the rows of the hypothesis' window."""
    bin_off, mass, row, n_bins = frag_index(l1, p, P, arrays, nthreads)
    lo = _c(hyp["lo"], np.int64)
    hi = _c(hyp["hi"], np.int64)
    n_h = len(lo)
    win_off = np.zeros(n_h + 1, np.int64)
    np.cumsum(hi - lo, out=win_off[1:])
    cnt = np.empty(int(win_off[-1]), np.int32)
    scored = np.zeros(n_h, np.uint32)
    matched = np.zeros(n_h, np.uint64)
    isum = np.zeros(len(cnt), np.uint32) if tic is not None else None
    lib().or_k1_index(C.c_int64(n_h), _p(_c(hyp["spec"], np.int32)), _p(_c(hyp["maxfz"], np.int8)), _p(lo), _p(hi),
                      _p(win_off), _p(_c(peaks["off"], np.int64)), _p(_c(peaks["mass"], np.float32)), _p(bin_off),
                      _p(mass), _p(row), C.c_float(p.fragment_min_mz), C.c_float(p.fragment_max_mz),
                      C.c_double(FRAG_BIN_TH), C.c_int64(n_bins), C.c_float(p.fragment_ppm[0]),
                      C.c_float(p.fragment_ppm[1]), _p(cnt), _p(scored), _p(matched),
                      _p(_c(peaks["int"], np.float32)) if tic is not None else None,
                      _p(_c(tic, np.float32)) if tic is not None else None,
                      _p(isum) if tic is not None else None, C.byref(P), C.c_int(nthreads or n_threads()))
    if tic is not None:
        return win_off, cnt, scored, matched, isum
    return win_off, cnt, scored, matched


def k1_appended(hyp, win_off, cnt, thr):
    """(hyp, row, count) of every window row with count >= thr, sorted by (hyp, row) (kernels.cu:170-180)."""
    lo = hyp["lo"]
    n = np.diff(win_off)
    hh = np.repeat(np.arange(len(lo)), n)
    rr = np.repeat(lo, n) + (np.arange(len(cnt)) - np.repeat(win_off[:-1], n))
    k = cnt >= thr
    return hh[k].astype(np.int64), rr[k].astype(np.int64), cnt[k].astype(np.int64)


# ---------------------------------------------------------------------------------------------------- top-K
def select_topk(o_h, o_r, o_c, hyp_spec, partner, topk, pair_closure=True):
    """engine.py:284-312: per spectrum the topk appended entries by (count desc, row desc), ties by lower
    hypothesis; partner rows added with count -1; unique (spectrum, row) keeps the lowest hypothesis and the
    highest count; result sorted by (spectrum, row)."""
    o_h = np.asarray(o_h, np.int64)
    o_r = np.asarray(o_r, np.int64)
    o_c = np.asarray(o_c, np.int64)
    spec = np.asarray(hyp_spec, np.int64)[o_h]
    o = np.lexsort((o_h, -o_r, -np.minimum(o_c, 32767), spec))
    ss = spec[o]
    first = np.searchsorted(ss, ss, side="left")
    rank = np.arange(len(ss)) - first
    sel = o[rank < topk]
    h, r, c = o_h[sel], o_r[sel], o_c[sel]
    if pair_closure:
        pr = np.asarray(partner, np.int64)[r]
        h = np.concatenate([h, h])
        r = np.concatenate([r, pr])
        c = np.concatenate([c, np.full_like(c, -1)])
    sp = np.asarray(hyp_spec, np.int64)[h]
    key = (sp << ROW_BITS) | r
    uk, inv = np.unique(key, return_inverse=True)
    hh = np.full(len(uk), 2 ** 62, np.int64)
    np.minimum.at(hh, inv, h)
    cc = np.full(len(uk), -1, np.int64)
    np.maximum.at(cc, inv, c)
    return hh, uk & (2 ** ROW_BITS - 1), cc


def topk_windows(hyp, win_off, cnt, thr, partner, topk, pair_closure=True, nthreads=None):
    """``select_topk(*k1_appended(hyp, win_off, cnt, thr), hyp["spec"], partner, topk, pair_closure)`` in C, per
    spectrum on all cores (the same (hyp, row, count) lists; the tests check them against the numpy chain)."""
    spec = np.asarray(hyp["spec"], np.int64)
    n_spec = int(spec.max()) + 1 if len(spec) else 0
    spec_hyp_off = np.searchsorted(spec, np.arange(n_spec + 1), side="left").astype(np.int64)
    cap = max(1, (2 if pair_closure else 1) * int(topk))
    o_h = np.empty(max(n_spec * cap, 1), np.int64)
    o_r = np.empty_like(o_h)
    o_c = np.empty_like(o_h)
    o_n = np.zeros(max(n_spec, 1), np.int32)
    lib().or_topk_windows(C.c_int64(n_spec), _p(spec_hyp_off), _p(_c(hyp["lo"], np.int64)), _p(_c(hyp["hi"], np.int64)),
                          _p(_c(win_off, np.int64)), _p(_c(cnt, np.int32)), C.c_int(int(thr)), C.c_int(int(topk)),
                          C.c_int(int(bool(pair_closure))), _p(_c(partner, np.int64)), C.c_int(cap), _p(o_h), _p(o_r),
                          _p(o_c), _p(o_n), C.c_int(nthreads or n_threads()))
    sel = (np.arange(cap)[None, :] < o_n[:n_spec, None]).ravel()
    return o_h[:n_spec * cap][sel], o_r[:n_spec * cap][sel], o_c[:n_spec * cap][sel]


def _ord_f32(x):
    """Order-preserving u32 image of f32 values (total order, -0 below +0)."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return np.where(u & 0x80000000, (~u) & 0xFFFFFFFF, u | 0x80000000)


def select_pruned(spec_hyp_off, hit_off, hit_hyp, hit_row, hit_cnt, logit, tau, min_keep, max_keep, partner,
                  pair_closure=True, sort_cap=1024):
    """The pruned selection of the learned pruner, per spectrum s over its hits [hit_off[s], hit_off[s+1]) (in
    (row, hypothesis) order): rank by (logit, min(count, 4095), hit position) descending; keep rank < min_keep or
    logit >= tau, at most max_keep (more than sort_cap hits: the first max_keep hits with logit >= tau in hit
    order); then pair closure (partner rows, same hypothesis, count -1) and duplicate rows merged (lowest
    hypothesis, highest count).  Returns per spectrum the (hyp, row, count) lists sorted by row."""
    hit_hyp = np.asarray(hit_hyp, np.int64)
    hit_row = np.asarray(hit_row, np.int64)
    hit_cnt = np.asarray(hit_cnt, np.int64)
    logit = np.asarray(logit, np.float32)
    partner = np.asarray(partner, np.int64)
    out = []
    for s in range(len(hit_off) - 1):
        a, b = int(hit_off[s]), int(hit_off[s + 1])
        n = b - a
        if n > sort_cap:
            ok = np.flatnonzero(logit[a:b] >= tau)[:max_keep]
        else:
            loc = np.arange(n, dtype=np.uint64)
            key = (_ord_f32(logit[a:b]) << np.uint64(32)) | (np.minimum(hit_cnt[a:b], 4095).astype(np.uint64)
                                                              << np.uint64(20)) | loc
            order = np.argsort(key)[::-1][:max_keep]
            rank = np.arange(len(order))
            ok = order[(rank < min_keep) | (logit[a:b][order] >= tau)]
        h, r, c = hit_hyp[a + ok], hit_row[a + ok], hit_cnt[a + ok]
        if pair_closure:
            h = np.concatenate([h, h])
            r = np.concatenate([r, partner[r]])
            c = np.concatenate([c, np.full(len(ok), -1, np.int64)])
        rows = np.unique(r)
        hh = np.array([h[r == x].min() for x in rows], np.int64)
        cc = np.array([c[r == x].max() for x in rows], np.int64)
        out.append((hh, rows, cc))
    return out


# ---------------------------------------------------------------------------------------------------- K2
def _cand_layout(hyp_spec, h):
    spec = np.asarray(hyp_spec, np.int64)[h]
    us, first, cnts = np.unique(spec, return_index=True, return_counts=True)
    if len(spec) and np.any(np.diff(spec) < 0):
        raise ValueError("candidates must be sorted by spectrum")
    off = np.zeros(len(us) + 1, np.int64)
    np.cumsum(cnts, out=off[1:])
    return spec, us.astype(np.int32), off


def k2(l1, hyp, peaks, h, r, p, P, shift=None, nthreads=None):
    spec, us, off = _cand_layout(hyp["spec"], h)
    n = len(r)
    row = _c(r, np.int32)
    mfz = _c(np.asarray(hyp["maxfz"])[h], np.int8)
    out = {"hyperscore": np.empty(n, np.float64)}
    for k in ("summed_b", "summed_y", "ppm"):
        out[k] = np.empty(n, np.float32)
    for k in ("matched_b", "matched_y", "longest_b", "longest_y"):
        out[k] = np.empty(n, np.int16)
    sh = _c(shift, np.float32) if shift is not None else None
    lib().or_k2(C.c_int(len(us)), _p(off), _p(row), _p(mfz), _p(us), _p(_c(peaks["off"], np.int64)),
                _p(_c(peaks["mass"], np.float32)), _p(_c(peaks["int"], np.float32)), _p(_c(l1.seq_off, np.int64)),
                _p(_c(l1.length, np.uint8)), _p(_c(l1.mask, np.uint64)), _p(_c(l1.mass32, np.float32)),
                _p(_c(l1.residues, np.uint8)), C.c_float(p.fragment_ppm[0]), C.c_float(p.fragment_ppm[1]),
                _p(sh), _p(out["hyperscore"]), _p(out["summed_b"]), _p(out["summed_y"]), _p(out["ppm"]),
                _p(out["matched_b"]), _p(out["matched_y"]), _p(out["longest_b"]), _p(out["longest_y"]),
                C.byref(P), C.c_int(nthreads or n_threads()))
    out["spec"] = spec
    return out


def k2_f64(l1, hyp, peaks, h, r, p, P, nthreads=None):
    spec, us, off = _cand_layout(hyp["spec"], h)
    n = len(r)
    hs = np.empty(n, np.float64)
    mb = np.empty(n, np.int16)
    my = np.empty(n, np.int16)
    lib().or_k2_f64(C.c_int(len(us)), _p(off), _p(_c(r, np.int32)), _p(_c(np.asarray(hyp["maxfz"])[h], np.int8)),
                    _p(us), _p(_c(peaks["off"], np.int64)), _p(_c(peaks["mass"], np.float32)),
                    _p(_c(peaks["int"], np.float32)), _p(_c(l1.seq_off, np.int64)), _p(_c(l1.length, np.uint8)),
                    _p(_c(l1.mask, np.uint64)), _p(_c(l1.mass32, np.float32)), _p(_c(l1.residues, np.uint8)),
                    C.c_double(p.fragment_ppm[0]), C.c_double(p.fragment_ppm[1]), _p(hs), _p(mb), _p(my),
                    C.byref(P), C.c_int(nthreads or n_threads()))
    return {"hyperscore": hs, "matched_b": mb, "matched_y": my}


def lnfact(n):
    n = np.asarray(n, np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        v = n * np.log(n) - n + 0.5 * np.log(n) + 0.5 * np.log(2 * np.pi * n)
    return np.where(n == 0, 1.0, v)


# ---------------------------------------------------------------------------------------------------- PSM ranking
def psm_rank(k2out, r, min_matched_peaks, report):
    """engine.py:366-392: candidates with matched_b + matched_y >= min_matched_peaks, ranked per spectrum by
    (hyperscore desc, row asc).  Returns dict with candidate index, spectrum, rank (1-based), delta_next,
    delta_best for ranks <= report."""
    mb = k2out["matched_b"].astype(np.int64)
    my = k2out["matched_y"].astype(np.int64)
    idx = np.flatnonzero(mb + my >= min_matched_peaks)
    spec = k2out["spec"][idx]
    hs = k2out["hyperscore"][idx]
    rr = np.asarray(r)[idx]
    o = np.lexsort((rr, -hs, spec))
    idx, spec, hs = idx[o], spec[o], hs[o]
    first = np.searchsorted(spec, spec, side="left")
    rank = np.arange(len(spec)) - first
    nxt = np.zeros_like(hs)
    if len(hs) > 1:
        same = spec[1:] == spec[:-1]
        nxt[:-1] = np.where(same, hs[1:], 0.0)
    best = hs[first] if len(hs) else hs
    keep = rank < report
    return {"cand": idx[keep], "spec": spec[keep], "rank": rank[keep] + 1, "hyperscore": hs[keep],
            "delta_next": hs[keep] - nxt[keep], "delta_best": best[keep] - hs[keep]}
