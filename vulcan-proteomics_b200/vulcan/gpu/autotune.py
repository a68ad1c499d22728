"""Autotuner of the search's launch shapes: fragment-index tile rows and K1 warps per CTA.

The best shapes depend on the index (peptidoform density, fragments per row), the spectra (peak counts, charges)
and the GPU, so they are measured, not guessed: for every candidate layout the index is tiled once, and a full
device pass (plain, or pruned with a pruner) over a sample of the workload is timed with CUDA events (median of
``reps`` after warm-up, L2 flushed before each).  Spectra are grouped into peak-count buckets for the report (the
per-bucket pass time of the chosen layout), so that a workload whose peak counts shift can be re-tuned.  Results
are cached in a JSON file keyed by index size, GPU name and tolerances.
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
            return dataclasses.replace(p, tile_rows=r["tile_rows"], k1_warps=r["k1_warps"]), dict(r, cached=True)
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
    chosen = dataclasses.replace(p, tile_rows=tr, k1_warps=w)
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
              "candidates": table, "peak_buckets": buckets, "cached": False}
    if cache:
        known = {}
        if os.path.exists(cache):
            with open(cache) as fh:
                known = json.load(fh)
        known[key] = {k: v for k, v in report.items() if k != "cached"}
        with open(cache, "w") as fh:
            json.dump(known, fh, indent=1)
    return chosen, report
