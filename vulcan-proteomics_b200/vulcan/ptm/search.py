"""Open and mass-offset search modes on the B200 kernels, with the entry points of the reference's
``vulcan/ptm/search.py`` (``ModeParams``, ``make_mode_hypotheses``, ``k1_topk_modes``, ``search_modes``).

Hypotheses (reference ``ptm/search.py:48-78``): the closed hypotheses of ``make_hypotheses`` first; then, per
offset o (Da, observed - peptide), one hypothesis per (spectrum, charge) at isotope 0 whose rows have Sage f32 mass
in M - o +- the precursor ppm; then, for an open window (lo, hi), one hypothesis per (spectrum, charge) whose rows
have mass in [M - hi, M - lo].  All hypotheses of a spectrum compete in one top-K (K1 count) and one ranking (K2
hyperscore); a (spectrum, row) reached by several hypotheses keeps the lowest hypothesis index (closed, then the
offsets in list order, then open).

K1 runs on the tiled fragment index in hit-list form (``vk_k1_hits``) over all hypotheses of a batch of spectra,
each hypothesis with its own count floor (``p.k1_threshold`` closed and offset, ``k1_threshold_open`` open).  The
hypotheses are grouped by spectrum (their order inside a spectrum kept), so one ``vk_select_hits`` per batch gives
every spectrum's top-K with pair closure.  Batches are cut from the exact window rows of their hypotheses (at most
``append_cap`` hit-list entries, 12 bytes each); a batch whose buffers still overflow (device status bit) is halved
and redone, as the reference's retry on a full append buffer (``ptm/search.py:121-160``).

K2 is ``vk_k2_spectra`` with the per-candidate shift M[h] - mass32[row] (0 for closed hypotheses): shifted and
unshifted b/y ions as the reference's shift mode (``kernels.cu:294-363``).
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import ctypes as C
import numpy as np
import pyarrow as pa
import torch

from vulcan.gpu import _lib as K
from vulcan.gpu import engine as E
from vulcan.gpu.host import NEUTRON, SearchParams, make_hypotheses

MODE_CLOSED, MODE_OFFSET, MODE_OPEN = 0, 1, 2


@dataclass
class ModeParams:
    """Search modes of one run (the reference's fields and defaults)."""
    offsets: tuple = ()                 # mass-offset mode: Da (observed - peptide), each its own hypothesis
    open_da: tuple | None = None        # open mode: (lo, hi) of observed - peptide, e.g. (-150, 500)
    open_tile: int = 4096               # the reference's CSR tile for open windows (the tiled index has its own)
    k1_threshold_open: int = 1
    spectra_per_batch: int = 1000       # open mode: at most this many spectra per K1 batch
    append_cap: int = 600_000_000       # hit-list entries per K1 batch


def _row_window(idx_mass32, lo_mass, hi_mass):
    return (np.searchsorted(idx_mass32, lo_mass, side="left").astype(np.int64),
            np.searchsorted(idx_mass32, hi_mass, side="right").astype(np.int64))


def make_mode_hypotheses(sp, valid, idx_mass32, p: SearchParams, mp: ModeParams) -> dict:
    """Closed, mass-offset and open hypotheses of a run (f32 arithmetic of the reference's windows)."""
    hyp = make_hypotheses(sp, valid, idx_mass32, p)
    n0 = len(hyp["spec"])
    hyp["mode"] = np.zeros(n0, np.uint8)
    hyp["off"] = np.zeros(n0, np.float32)
    base = np.flatnonzero(hyp["iso"] == 0)            # one (spectrum, charge) each
    nb = len(base)
    carried = {k: hyp[k][base] for k in ("spec", "z", "pm", "M", "maxfz")}
    blocks = [hyp]
    offs = np.asarray(mp.offsets, np.float32).reshape(-1)
    if len(offs):
        m = (carried["M"][None, :] - offs[:, None]).astype(np.float32)          # [offsets, base]
        plo, phi = np.float32(p.precursor_ppm[0]), np.float32(p.precursor_ppm[1])
        lo_m = (m + (m * plo) / np.float32(1e6)).astype(np.float32).ravel()
        hi_m = (m + (m * phi) / np.float32(1e6)).astype(np.float32).ravel()
        blk = {k: np.tile(v, len(offs)) for k, v in carried.items()}
        blk["lo"], blk["hi"] = _row_window(idx_mass32, lo_m, hi_m)
        blk["mode"] = np.full(nb * len(offs), MODE_OFFSET, np.uint8)
        blk["off"] = np.repeat(offs, nb)
        blocks.append(blk)
    if mp.open_da is not None:
        blk = dict(carried)
        blk["lo"], blk["hi"] = _row_window(idx_mass32, (carried["M"] - np.float32(mp.open_da[1])).astype(np.float32),
                                           (carried["M"] - np.float32(mp.open_da[0])).astype(np.float32))
        blk["mode"] = np.full(nb, MODE_OPEN, np.uint8)
        blk["off"] = np.full(nb, np.nan, np.float32)
        blocks.append(blk)
    out = {}
    for k in hyp:
        parts = [b[k] if k in b else np.zeros(len(b["spec"]), hyp[k].dtype) for b in blocks]
        out[k] = np.concatenate(parts).astype(hyp[k].dtype)
    return out


def _batches(sizes: np.ndarray, cap: int, max_spec: int) -> list:
    """Consecutive spectrum ranges [a, b) with sum(sizes[a:b]) <= cap (at least one spectrum each) and at most
    max_spec spectra."""
    out, a = [], 0
    n = len(sizes)
    while a < n:
        b, tot = a, 0
        while b < n and b - a < max_spec and (b == a or tot + sizes[b] <= cap):
            tot += int(sizes[b])
            b += 1
        out.append((a, b))
        a = b
    return out


def k1_topk_modes(gi: E.GpuIndex, hyp: dict, peaks: dict, p: SearchParams, mp: ModeParams, st: E.Stats):
    """K1 + per-spectrum top-K + pair closure over every hypothesis of ``hyp``, in batches of spectra.  Returns
    (h, r, c) sorted by (spectrum, row) like ``engine.select_topk``, the per-hypothesis scored / matched counters
    and the device spectrum / fragment-charge arrays of the hypotheses."""
    dev = gi.dev
    n_h = len(hyp["spec"])
    d_spec = torch.from_numpy(np.ascontiguousarray(hyp["spec"], np.int32)).to(dev)
    d_maxfz = torch.from_numpy(np.ascontiguousarray(hyp["maxfz"], np.int8)).to(dev)
    scored = torch.zeros(max(n_h, 1), dtype=torch.int32, device=dev)[:n_h]
    matched = torch.zeros(max(n_h, 1), dtype=torch.int64, device=dev)[:n_h]
    empty = torch.zeros(0, dtype=torch.int64, device=dev)
    if n_h == 0:
        return empty, empty, empty, scored, matched, d_spec, d_maxfz
    lo, hi = np.asarray(hyp["lo"], np.int64), np.asarray(hyp["hi"], np.int64)
    win = np.maximum(hi - lo, 0)
    T = 1 << gi.tix.tile_shift
    items = np.where(win > 0, (hi - 1) // T - lo // T + 1, 0)
    is_open = np.asarray(hyp.get("mode", np.zeros(n_h, np.uint8))) == MODE_OPEN
    thr = np.where(is_open, mp.k1_threshold_open, p.k1_threshold).astype(np.int32)
    order = np.argsort(hyp["spec"], kind="stable")    # grouped by spectrum, closed / offsets / open inside
    us, first = np.unique(np.asarray(hyp["spec"])[order], return_index=True)
    first = np.append(first, n_h)
    spec_rows = np.add.reduceat(win[order], first[:-1]) if len(us) else np.zeros(0, np.int64)
    max_spec = mp.spectra_per_batch if is_open.any() else len(us)
    todo = _batches(spec_rows, mp.append_cap, max(1, max_spec))
    outs = []
    while todo:
        a, b = todo.pop(0)
        hh = order[first[a]:first[b]]
        nb_spec = b - a
        dh = {"spec": torch.from_numpy(np.ascontiguousarray(hyp["spec"][hh], np.int32)).to(dev),
              "maxfz": torch.from_numpy(np.ascontiguousarray(hyp["maxfz"][hh], np.int8)).to(dev),
              "lo": torch.from_numpy(np.ascontiguousarray(lo[hh])).to(dev),
              "hi": torch.from_numpy(np.ascontiguousarray(hi[hh])).to(dev),
              "spec_off": torch.from_numpy((first[a:b + 1] - first[a]).astype(np.int64)).to(dev)}
        caps = (int(items[hh].sum()), int(win[hh].sum()))
        k1h = E._k1_hits(gi, dh, peaks, p, len(hh), 0, isum=False,
                         h_thr=torch.from_numpy(np.ascontiguousarray(thr[hh])).to(dev), caps=caps)
        cand, sums = E._shortlist_hits(gi, p, nb_spec, dh, k1h, p.topk, closure=bool(p.pair_closure))
        status = int(k1h["status"].item())
        if status & 2:   # a bound did not hold: redo the batch in two halves
            if nb_spec == 1:
                raise RuntimeError("K1: the hit lists of a single spectrum overflow")
            st.counts["k1_overflow_retries"] = st.counts.get("k1_overflow_retries", 0) + 1
            mid = a + nb_spec // 2
            todo[:0] = [(a, mid), (mid, b)]
            continue
        E.check_status(k1h["status"], "k1_modes")
        nc = int(cand["cand_off"][nb_spec])
        hh_d = torch.from_numpy(hh.astype(np.int64)).to(dev)
        outs.append((hh_d[cand["c_hyp"][:nc]], cand["c_row"][:nc].clone(), cand["c_cnt"][:nc].clone()))
        scored[hh_d] = sums["hyp_scored"][:len(hh)]
        matched[hh_d] = sums["hyp_matched"][:len(hh)]
        st.counts["k1_window_candidates"] = st.counts.get("k1_window_candidates", 0) + caps[1]
        st.counts["k1_work_items"] = st.counts.get("k1_work_items", 0) + caps[0]
    if not outs:
        return empty, empty, empty, scored, matched, d_spec, d_maxfz
    h = torch.cat([o[0] for o in outs])
    r = torch.cat([o[1] for o in outs])
    c = torch.cat([o[2] for o in outs])
    return h, r, c, scored, matched, d_spec, d_maxfz


def k2_shifted(gi: E.GpuIndex, hyp: dict, h, r, d_spec, d_maxfz, peaks, p: SearchParams, n_spec: int):
    """K2 of candidates (h, r) sorted by (spectrum, row) with shift M[h] - mass32[r] for the open / offset
    hypotheses and 0 for the closed ones (``vk_k2_spectra``, a warp per spectrum).  One output row per candidate."""
    L = K.lib()
    dev = gi.dev
    mode = torch.from_numpy(np.ascontiguousarray(hyp["mode"])).to(dev)[h]
    M = torch.from_numpy(np.ascontiguousarray(hyp["M"], np.float32)).to(dev)[h]
    shift = torch.where(mode == MODE_CLOSED, torch.zeros_like(M), M - gi.mass32[r]).contiguous()
    spec = d_spec[h].long()
    cand_off = torch.zeros(n_spec + 1, dtype=torch.int64, device=dev)
    if len(h):
        torch.cumsum(torch.bincount(spec, minlength=n_spec), 0, out=cand_off[1:])
    row32 = r.to(torch.int32).contiguous()
    mfz = d_maxfz[h].contiguous()
    k2 = E._k2_outputs(max(len(h), 1), dev)
    K.check(L.vk_k2_spectra(C.byref(gi.fp), n_spec, K.ptr(cand_off), K.ptr(row32), K.ptr(mfz), K.ptr(peaks["off"]),
                            K.ptr(peaks["mass"]), K.ptr(peaks["int"]), *gi.table_ptrs(), float(p.fragment_ppm[0]),
                            float(p.fragment_ppm[1]), K.ptr(shift), *E._k2_ptrs(k2), K.stream()), "k2_spectra_shift")
    out = {k: v[:len(h)] for k, v in k2.items()}
    out["spec"] = spec
    out["shift"] = shift
    return out


def search_modes(sp, gi: E.GpuIndex, l1, p: SearchParams, mp: ModeParams, report: int | None = None):
    """Closed + mass-offset + open search of one run (modes per ``mp``).  Returns (PSM table, stats); the table
    adds ``mode`` (u8: 0 closed, 1 mass-offset, 2 open), ``hyp_offset`` (f32, the hypothesis' offset, Da; 0 closed,
    NaN open) and ``mass_shift`` (f32, Da: expmass - isotope_error * NEUTRON - calcmass)."""
    st = E.Stats()
    t0 = time.perf_counter()
    dev = gi.dev
    with torch.cuda.device(dev):
        with E.Timer(st, "k0"):
            peaks = E.k0_preprocess(sp, p, dev, st)
        with E.Timer(st, "hyp"):
            hyp = make_mode_hypotheses(sp, peaks["valid"], gi.mass32_np, p, mp)
        with E.Timer(st, "k1_topk"):
            h, r, c, scored, matched, d_spec, d_maxfz = k1_topk_modes(gi, hyp, peaks, p, mp, st)
        with E.Timer(st, "k2"):
            k2 = k2_shifted(gi, hyp, h, r, d_spec, d_maxfz, peaks, p, len(sp))
        with E.Timer(st, "features"):
            tbl = E.psm_table(sp, gi, l1, hyp, h, r, c, k2, scored, matched, peaks, p, report)
            hh = _psm_hyp_index(tbl, h, r, k2, p, report)
            rows = tbl.column("pf_row").to_numpy()
            iso = tbl.column("isotope_error").to_numpy().astype(np.float32)
            pm = tbl.column("expmass").to_numpy()
            ms = (pm - (iso * NEUTRON).astype(np.float32) - l1.mass32[rows]).astype(np.float32)
            tbl = tbl.append_column("mode", pa.array(hyp["mode"][hh], pa.uint8()))
            tbl = tbl.append_column("hyp_offset", pa.array(hyp["off"][hh], pa.float32()))
            tbl = tbl.append_column("mass_shift", pa.array(ms, pa.float32()))
    st.wall_s["total"] = time.perf_counter() - t0
    st.counts.update(n_spectra=len(sp), n_searched=int(peaks["valid"].sum()), n_hypotheses=len(hyp["spec"]),
                     n_rescored=int(len(r)), n_psms=tbl.num_rows)
    return tbl, st


def _psm_hyp_index(tbl, h, r, k2, p: SearchParams, report):
    """Hypothesis of each reported PSM: the candidates that pass min_matched_peaks ranked per spectrum by
    (hyperscore desc, row asc), the first ``report`` (the table's own order, ``engine.py:366-392``)."""
    report = p.report_psms if report is None else report
    ok = (k2["matched_b"].long() + k2["matched_y"].long()) >= p.min_matched_peaks
    idx = torch.nonzero(ok).squeeze(1)
    key_spec, key_hs, key_row = k2["spec"][idx], k2["hyperscore"][idx], r[idx]
    o = torch.argsort(key_row, stable=True)
    o = o[torch.argsort(-key_hs[o], stable=True)]
    o = o[torch.argsort(key_spec[o], stable=True)]
    idx, key_spec = idx[o], key_spec[o]
    rank = torch.arange(len(idx), device=idx.device) - torch.searchsorted(key_spec, key_spec, side="left")
    sel = idx[rank < report]
    hh = h[sel].cpu().numpy()
    if len(hh) != tbl.num_rows or not np.array_equal(r[sel].cpu().numpy(), tbl.column("pf_row").to_numpy()):
        raise RuntimeError("PSM rows and their hypotheses are out of step")
    return hh
