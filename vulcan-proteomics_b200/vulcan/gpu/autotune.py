"""Autotuner of the search's launch shapes: fragment-index tile rows and K1 warps per CTA, per peak-count bucket.

The best shapes depend on the index (peptidoform density, fragments per row), the spectra (peak counts, charges)
and the GPU, so they are measured, not guessed: for every candidate layout the index is tiled once, and a full
device pass (plain, or pruned with a pruner) over a sample of the workload is timed with CUDA events (median of
``reps`` after warm-up, L2 flushed before each).  Then, per peak-count bucket (kept peaks 1-64, 65-128, 129-256,
257-512, 513+), K1 alone over that bucket's spectra of the sample is timed for every (tile rows, warps) and the
fastest is kept; the buckets' shapes go into ``SearchParams.k1_shapes`` (each bucket's spectra then run K1 on
their own tiling and warps inside the same pass), and the routed pass is kept if it beats the single layout.
Results are cached in a JSON file keyed by index size, GPU name and tolerances.
"""
from __future__ import annotations

import dataclasses
import hashlib
import json
import os

import numpy as np
import torch

from . import engine as E
from .host import SearchParams, Spectra

TILE_ROWS = (64, 128, 256)
K1_WARPS = (3, 4, 6, 8)
PEAK_BUCKETS = (64, 128, 256, 512, 1 << 30)


def _key(l1, p: SearchParams, dev, pruned: bool) -> str:
    name = torch.cuda.get_device_name(dev)
    d = {"rows": int(len(l1)), "mass0": float(l1.mass32[0]) if len(l1) else 0.0,
         "mass1": float(l1.mass32[-1]) if len(l1) else 0.0, "gpu": name, "prec": list(p.precursor_ppm),
         "frag": list(p.fragment_ppm), "unit": p.fragment_unit, "topk": p.topk, "pruned": pruned}
    return hashlib.sha256(json.dumps(d, sort_keys=True).encode()).hexdigest()[:16]


def _subset(sp: Spectra, sel: np.ndarray) -> Spectra:
    from ..synth import take_spectra
    return take_spectra(sp, sel, sp.run)


def _time_pass(gi, p, sp: Spectra, pruner, reps: int, flush) -> float:
    from . import prune as PR
    run = E.DeviceRun(sp, gi.dev)

    def step():
        if pruner is None:
            return E._search_device(run, gi, p, 1, E.Stats())
        return PR._pruned_device(run, gi, p, pruner, 1, E.Stats())
    for _ in range(2):
        step()
    ts = []
    for _ in range(reps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = step()
        e1.record()
        torch.cuda.synchronize(gi.dev)
        ts.append(e0.elapsed_time(e1))
    E.check_status(out["status"])
    return float(np.median(ts))


def tune(l1, p: SearchParams, static: dict, var: dict, sample: Spectra, pruner=None, device="cuda",
         reps: int = 5, tile_rows=TILE_ROWS, k1_warps=K1_WARPS, cache: str | None = None, log=None):
    """The fastest (tile_rows, k1_warps) for the workload sample; returns (params, report).  With ``cache`` (a JSON
    path) a previous result for the same index, GPU and tolerances is reused."""
    dev = torch.device(device)
    key = _key(l1, p, dev, pruner is not None)
    if cache and os.path.exists(cache):
        with open(cache) as fh:
            known = json.load(fh)
        if key in known:
            r = known[key]
            return (dataclasses.replace(p, tile_rows=r["tile_rows"], k1_warps=r["k1_warps"],
                                        k1_shapes=tuple(tuple(x) for x in r.get("k1_shapes", ()))),
                    dict(r, cached=True))
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device=dev)
    table = []
    best = None
    for tr in tile_rows:
        q0 = dataclasses.replace(p, tile_rows=tr)
        try:
            gi = E.GpuIndex(l1, q0, static, var, device=dev)
        except RuntimeError as e:          # a layout the index cannot use (e.g. tiles over the shared memory)
            table.append({"tile_rows": tr, "error": str(e)})
            continue
        for w in k1_warps:
            q = dataclasses.replace(q0, k1_warps=w)
            try:
                ms = _time_pass(gi, q, sample, pruner, reps, flush)
            except RuntimeError as e:
                table.append({"tile_rows": tr, "k1_warps": w, "error": str(e)})
                continue
            table.append({"tile_rows": tr, "k1_warps": w, "ms": round(ms, 4)})
            if log:
                log(f"tile_rows {tr} k1_warps {w}: {ms:.3f} ms")
            if best is None or ms < best[0]:
                best = (ms, tr, w)
        del gi
        torch.cuda.empty_cache()
    if best is None:
        raise RuntimeError("autotune: no layout ran")
    ms, tr, w = best
    chosen = dataclasses.replace(p, tile_rows=tr, k1_warps=w, k1_shapes=())
    routed, route_report = _tune_buckets(l1, chosen, static, var, sample, pruner, reps, flush, tile_rows, k1_warps,
                                         ms, log)
    if routed is not None:
        chosen = routed
    # per peak-count bucket: the chosen layout's pass time over the spectra of that bucket
    lens = np.diff(np.asarray(sample.offsets, np.int64))
    buckets = []
    gi = E.GpuIndex(l1, chosen, static, var, device=dev)
    lo = 0
    for hi in PEAK_BUCKETS:
        sel = np.flatnonzero((lens > lo) & (lens <= hi))
        if len(sel):
            t = _time_pass(gi, chosen, _subset(sample, sel), pruner, reps, flush)
            buckets.append({"peaks": f"{lo + 1}-{hi if hi < 1 << 30 else 'max'}", "spectra": int(len(sel)),
                            "ms": round(t, 4), "us_per_spectrum": round(1e3 * t / len(sel), 4)})
        lo = hi
    report = {"tile_rows": tr, "k1_warps": w, "ms": round(ms, 4), "sample_spectra": len(sample),
              "candidates": table, "peak_buckets": buckets, "k1_shapes": [list(x) for x in chosen.k1_shapes],
              "per_bucket": route_report, "cached": False}
    if cache:
        known = {}
        if os.path.exists(cache):
            with open(cache) as fh:
                known = json.load(fh)
        known[key] = {k: v for k, v in report.items() if k != "cached"}
        with open(cache, "w") as fh:
            json.dump(known, fh, indent=1)
    return chosen, report


def _time_k1(gi, p, sp: Spectra, pruner, reps: int, flush) -> float:
    """CUDA-event time of K1 alone (planning, window keys, counting; the pruned path's hit-list form with a
    pruner) over a resident run whose K0 and hypotheses are done."""
    run = E.DeviceRun(sp, gi.dev)
    peaks = E._k0_device(run, p, gi.dev)
    dh = E._hyp_device(run, peaks, gi, p)
    thr = max(p.k1_threshold, pruner.min_count) if pruner is not None else p.k1_threshold

    def step():
        if pruner is not None:
            return E._k1_hits(gi, dh, peaks, p, dh["n_max"], thr, isum=True)["status"]
        return E._k1_dense(gi, dh, peaks, p, dh["n_max"])[2]
    for _ in range(2):
        step()
    ts = []
    for _ in range(reps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        status = step()
        e1.record()
        torch.cuda.synchronize(gi.dev)
        ts.append(e0.elapsed_time(e1))
    E.check_status(status)
    return float(np.median(ts))


def _tune_buckets(l1, p: SearchParams, static, var, sample: Spectra, pruner, reps, flush, tile_rows, k1_warps,
                  single_ms: float, log=None):
    """Per peak-count bucket the fastest (tile rows, warps) of K1 over the bucket's spectra; returns (params with
    ``k1_shapes``, report), params None when routing the buckets does not beat the single layout."""
    gi = E.GpuIndex(l1, p, static, var, device=flush.device)
    for tr in tile_rows:
        try:
            gi.tiling(tr)
        except RuntimeError:
            continue
    from ..synth import take_spectra
    lens = np.diff(np.asarray(sample.offsets, np.int64))
    kept = np.minimum(lens, p.max_peaks)           # an upper bound of the kept peaks, the bucket key
    rows, lower = [], 0
    for upper in PEAK_BUCKETS:
        sel = np.flatnonzero((kept > lower) & (kept <= upper))
        if len(sel) >= 64:
            sub = take_spectra(sample, sel, sample.run)
            best = None
            for tr in tile_rows:
                if tr not in gi.tilings:
                    continue
                for w in k1_warps:
                    q = dataclasses.replace(p, k1_shapes=((1 << 30, tr, w),))
                    try:
                        t = _time_k1(gi, q, sub, pruner, reps, flush)
                    except RuntimeError:
                        continue
                    if best is None or t < best[0]:
                        best = (t, tr, w)
            base = _time_k1(gi, p, sub, pruner, reps, flush)
            rows.append({"peaks": f"{lower + 1}-{upper if upper < 1 << 30 else 'max'}", "spectra": int(len(sel)),
                         "tile_rows": best[1], "k1_warps": best[2], "k1_ms": round(best[0], 4),
                         "k1_ms_single_layout": round(base, 4)})
            if log:
                log(f"bucket {rows[-1]['peaks']}: {best[1]} rows x {best[2]} warps {best[0]:.3f} ms "
                    f"(single layout {base:.3f})")
        lower = upper
    shapes = tuple((int(r["peaks"].split("-")[1]) if r["peaks"].split("-")[1] != "max" else 1 << 30,
                    r["tile_rows"], r["k1_warps"]) for r in rows)
    shapes = tuple(x for x in shapes if (x[1], x[2]) != (p.tile_rows, p.k1_warps) or x[0] < (1 << 30))
    report = {"buckets": rows}
    if not shapes or all((x[1], x[2]) == (p.tile_rows, p.k1_warps) for x in shapes):
        report["routed"] = False
        return None, report
    routed = dataclasses.replace(p, k1_shapes=tuple(x for x in shapes if x[0] < (1 << 30)),
                                 tile_rows=shapes[-1][1] if shapes[-1][0] >= (1 << 30) else p.tile_rows,
                                 k1_warps=shapes[-1][2] if shapes[-1][0] >= (1 << 30) else p.k1_warps)
    gi_r = E.GpuIndex(l1, routed, static, var, device=flush.device)
    ms_r = _time_pass(gi_r, routed, sample, pruner, reps, flush)
    report.update(routed_ms=round(ms_r, 4), single_ms=round(single_ms, 4), routed=ms_r < single_ms)
    del gi_r, gi
    torch.cuda.empty_cache()
    return (routed if ms_r < single_ms else None), report
