"""Parity of a device search pass with the oracle on a sample of its spectra -- TEST INFRASTRUCTURE ONLY.

Imported by tests/ and by ``bench.py``'s CPU-baseline leg (the checker of the timed device pass); the product
package never imports it.

``check_plain`` takes the intermediates of one plain device pass (K0 peak view, hypotheses, dense K1 counts with the
per-hypothesis statistics, top-K + pair closure candidate lists, K2 outputs, top-1 PSM slots) and compares the
first ``n`` spectra with the oracle's chain on those spectra (reference order: ``vulcan/gpu/engine.py:435-464``):

  k0        peak offsets, masses, intensities and validity bit-identical (engine.py:171-210)
  hyp       hypotheses and row windows bit-identical (host.py:64-91)
  k1        dense counts of every window row, per-hypothesis scored / matched (kernels.cu:112-190, 195-232),
            from the oracle's fragment index
  topk      candidate (hypothesis, row, count) lists after pair closure (engine.py:284-312)
  k2        f32 sums, ppm and integer outputs bit-identical, f64 hyperscore within 1e-12 of the oracle's
            (device log vs host libm) (kernels.cu:263-376)
  fp64      hyperscore relative error against the FP64-accumulation oracle (largest over all candidates)
  top1      the top-1 PSM (candidate row) of every spectrum (engine.py:366-392)
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


def subset(sp, n):
    """The first n spectra of a run (same arrays, sliced)."""
    from vulcan.gpu.host import Spectra
    n = min(n, len(sp))
    o = np.asarray(sp.offsets[:n + 1], np.int64)
    return Spectra(sp.run, sp.scan[:n], sp.index[:n], sp.rt[:n], sp.precursor_mz[:n], sp.charge[:n],
                   sp.mz[:o[-1]], sp.intensity[:o[-1]], o.copy())


def _np(t):
    return t.detach().cpu().numpy()


def oracle_plain(l1, sp, p, P, arrays=None, f64=True):
    """The oracle's plain search chain on run ``sp``: every intermediate the device pass has.  Its C stages: the K0
    view (``O.k0_view_c``), K1 over the oracle's fragment index (``O.k1_index``, the reference's K1 search on the
    host), the top-K with closure (``O.topk_windows``) and K2; the tests check each against the numpy restatements
    and the window counts of ``O.k1_windows``, which are pinned to the reference's own code."""
    pk = O.k0_view_c(sp, p)
    hyp = O.make_hypotheses(sp, pk["valid"], l1.mass32, p)
    win_off, cnt, sc, mt = O.k1_index(l1, hyp, pk, p, P, arrays=arrays)
    h, r, c = O.topk_windows(hyp, win_off, cnt, p.k1_threshold, l1.partner, p.topk, p.pair_closure)
    k2 = O.k2(l1, hyp, pk, h, r, p, P)
    k2f = O.k2_f64(l1, hyp, pk, h, r, p, P) if f64 else None
    rk = O.psm_rank(k2, r, p.min_matched_peaks, 1)
    return {"pk": pk, "hyp": hyp, "win_off": win_off, "cnt": cnt, "scored": sc, "matched": mt, "h": h, "r": r,
            "c": c, "k2": k2, "k2_f64": k2f, "rank": rk}


def check_plain(l1, sp, p, P, out, n: int, arrays=None, ref=None) -> dict:
    """Compare the first n spectra of the plain device pass ``out`` (``engine._search_device``, report >= 1) with
    the oracle.  Returns {"spectra": n, "k0_equal", "hyp_equal", "k1_equal", "topk_equal", "k2_equal",
    "top1_equal": bool, "hs_max_rel_err": oracle f64-vs-device, "hs_max_rel_err_fp64": FP64 oracle vs device,
    "candidates": checked candidate count, "window_rows": checked window rows}."""
    n = min(n, len(sp))
    sub = subset(sp, n)
    o = ref if ref is not None else oracle_plain(l1, sub, p, P, arrays)
    res = {"spectra": n}
    # K0
    pk = out["peaks"]
    off_d = _np(pk["off"][:n + 1])
    npk = int(off_d[-1])
    res["k0_equal"] = bool(np.array_equal(off_d, o["pk"]["off"])
                           and np.array_equal(_np(pk["mass"][:npk]), o["pk"]["mass"])
                           and np.array_equal(_np(pk["int"][:npk]), o["pk"]["int"])
                           and np.array_equal(_np(pk["valid_d"][:n]).astype(bool), o["pk"]["valid"]))
    # hypotheses
    dh = out["dh"]
    nh = int(_np(dh["spec_off"][n:n + 1])[0])
    hyp = o["hyp"]
    res["hyp_equal"] = bool(nh == len(hyp["spec"]) and all(
        np.array_equal(_np(dh[k][:nh]), np.asarray(hyp[k])) for k in ("spec", "z", "iso", "pm", "M", "lo", "hi",
                                                                      "maxfz")))
    # K1 dense counts and per-hypothesis statistics
    wo = _np(out["win_off"][:nh + 1])
    nw = int(wo[-1])
    res["window_rows"] = nw
    res["k1_equal"] = bool(np.array_equal(wo, o["win_off"]) and np.array_equal(_np(out["cnt"][:nw]), o["cnt"])
                           and np.array_equal(_np(out["hyp_scored"][:nh]).astype(np.int64),
                                              o["scored"].astype(np.int64))
                           and np.array_equal(_np(out["hyp_matched"][:nh]).astype(np.int64),
                                              o["matched"].astype(np.int64)))
    # top-K + closure
    nc = int(_np(out["cand_off"][n:n + 1])[0])
    res["candidates"] = nc
    res["topk_equal"] = bool(nc == len(o["r"]) and np.array_equal(_np(out["c_hyp"][:nc]), o["h"])
                             and np.array_equal(_np(out["c_row"][:nc]), o["r"])
                             and np.array_equal(_np(out["c_cnt"][:nc]), o["c"]))
    # K2
    k2d = {k: _np(v[:nc]) for k, v in out["k2"].items()}
    k2o = o["k2"]
    ok = nc == len(k2o["summed_b"])
    if ok:
        for k in ("summed_b", "summed_y", "matched_b", "matched_y", "longest_b", "longest_y"):
            ok = ok and np.array_equal(k2d[k], k2o[k])
        ok = ok and np.array_equal(k2d["ppm"], k2o["ppm"], equal_nan=True)
    hs_d = k2d["hyperscore"]
    rel = np.abs(hs_d - k2o["hyperscore"]) / np.maximum(np.abs(k2o["hyperscore"]), 1e-300) if ok else np.array([np.inf])
    res["hs_max_rel_err"] = float(rel.max()) if len(rel) else 0.0
    res["k2_equal"] = bool(ok and res["hs_max_rel_err"] <= 1e-12)
    if o["k2_f64"] is not None and ok:
        f = o["k2_f64"]["hyperscore"]
        fin = np.isfinite(f) & np.isfinite(hs_d)
        r64 = np.abs(hs_d[fin] - f[fin]) / np.maximum(np.abs(f[fin]), 1e-300)
        res["hs_max_rel_err_fp64"] = float(r64.max()) if len(r64) else 0.0
        res["fp64_matches_equal"] = bool(np.array_equal(o["k2_f64"]["matched_b"], k2o["matched_b"])
                                         and np.array_equal(o["k2_f64"]["matched_y"], k2o["matched_y"]))
    # top-1 PSM per spectrum
    psm_cand = _np(out["psm"][0])
    report = len(psm_cand) // max(len(sp), 1)
    top = psm_cand[:n * report:report] if report else np.zeros(0, np.int64)
    d_spec = np.flatnonzero(top >= 0)
    d_row = _np(out["c_row"])[top[d_spec]] if len(d_spec) else np.zeros(0, np.int64)
    rk = o["rank"]
    res["top1_equal"] = bool(np.array_equal(d_spec, rk["spec"]) and np.array_equal(d_row, o["r"][rk["cand"]]))
    res["psms"] = int(len(d_spec))
    return res
