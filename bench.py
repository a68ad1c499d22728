#!/usr/bin/env python3
"""Benchmark of the DDA search hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload human|small]

One step = one pass of the search over one MS2 run of the workload (human: 40,000 simulated spectra of uneven
peak counts, 20-600, against the ~5.5M-peptidoform human-scale index, top-k 100).  The headline path (--path
pruned) is the learned-pruned search: K0 peak view, hypotheses, K1 fragment-index counting with intensity sums,
top-k shortlist (count floor), BF16 MLP scores, calibrated selection + pair closure, K2 exact rescoring, PSM
ranking.  Its pruner is trained first on the GPU (untimed) from 200,000 simulated spectra of other runs and
calibrated on one more run to >= 99.95% top-1 recall; the plain exhaustive path (K1 -> top-k -> pair closure ->
K2) is then timed the same way on the same run and the pruned path's top-1 recall and PSMs at 1% q are judged
against it (`vs_plain`).

  value      spectra/s with the run's raw spectra already in HBM (device pass captured once as a CUDA graph and
             replayed, CUDA events on the stream, L2 flushed between steps), summed over ranks (each rank searches
             its own run: weak scaling); eager_ms_per_step is the same pass launched kernel by kernel
  e2e        spectra/s through the public API (engine.Searcher, plain or with the pruner) over the run in pinned host
             memory: H2D of the raw spectra on a copy stream, the graph replay, one D2H of the packed PSM slots and
             the host PSM table, runs queued one ahead (wall clock around all steps)
  roofline   the dominant kernel's algorithmic bytes per launch / its mean CUDA-event duration vs the measured
             HBM copy bandwidth; mlp_roofline: the MLP's FLOPs / duration vs the measured bf16 tensor peak
  cpu_baseline  the CPU oracle (C/OpenMP restatement of the reference kernels) on a bounded sample, all cores

--impl reference times the CPU path of the reference (its C restatement: the reference ships no CPU search of
its own; its CPU comparator is the external Sage binary) on the same workload, a bounded sample per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "vulcan-proteomics_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "spectra/s on 1 B200, learned-pruned vs exhaustive at ≥99.9% top-1 recall"
STATIC = {"C": 57.021464}
VAR = {"M": 15.9949}
CACHE = os.environ.get("VULCAN_BENCH_CACHE", os.path.join(tempfile.gettempdir(), "vulcan_bench_cache"))


def _peaks_json():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _workload_setup(name: str, rank: int):
    from vulcan import synth
    from vulcan.index.build import L1Index, read_labels
    w = synth.WORKLOADS[name]
    t0 = time.perf_counter()
    d = synth.build_index(w, CACHE)
    t_build = time.perf_counter() - t0
    l1 = L1Index(d)
    lab = read_labels(d)
    sp, rows = synth.simulate_run(l1, lab, w, seed=w.spectra_seed + 1000 * rank, run=f"run{rank}")
    return w, l1, lab, sp, t_build


def _params(w, a):
    kw = {"search_method": a.method}
    if a.tile_rows:
        kw["tile_rows"] = a.tile_rows
    elif a.method == "fused":
        kw["tile_rows"] = 64         # the fused kernel stages one tile per warp
    if a.k1_warps:
        kw["k1_warps"] = a.k1_warps
    if a.warps:
        kw["fused_warps"] = a.warps
    return w.search_params(**kw)


def _config(w, p, extra=None):
    cfg = {"workload": f"{w.name}: {w.n_proteins} random proteins (<= {w.missed_cleavages} missed cleavages, "
                       f"length {w.min_len}-{w.max_len}, CAM-C, Met-ox <= {w.max_var}, pseudo-reverse decoys); "
                       f"runs of {w.n_spectra} simulated MS2 spectra, charge {w.charges[0]}-{w.charges[1]}",
           "path": "plain exhaustive search (K1 -> top-k -> pair closure -> K2), no learned pruner",
           "method": ("fused persistent kernel (K1+top-k+K2+ranking per spectrum)" if p.search_method == "fused"
                      else "staged kernels"),
           "precursor_ppm": list(p.precursor_ppm), "fragment_tol": f"+-{p.fragment_ppm[1]} {p.fragment_unit}",
           "topk": p.topk, "max_peaks": p.max_peaks,
           "k1": f"bitmap-filtered per-peak search, {p.k1_warps} warps per tile CTA",
           "l2": "flushed between steps (256 MiB write)"}
    if extra:
        cfg.update(extra)
    return cfg


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples every 200 ms while running."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(device_index)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [ln.split(",") for ln in self.f.read().strip().splitlines() if ln.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_oracle_pass(l1, sp_sub, p, var=None):
    """The oracle's search of a run (K0, hypotheses, K1, top-K + closure, K2, ranking) on the host cores; returns
    every intermediate (``oracle.parity.oracle_plain``), so that the device pass can be checked against it."""
    from oracle import oracle as O
    from oracle import parity
    P = O.make_params(STATIC, VAR if var is None else var, p.fragment_unit)
    return parity.oracle_plain(l1, sp_sub, p, P, arrays=_ARR.get(id(l1)), f64=False)


_ARR = {}


def _oracle_index(l1, p, var=None):
    """The oracle's fragment index of l1 (built once per process, before any timed sample)."""
    from oracle import oracle as O
    P = O.make_params(STATIC, VAR if var is None else var, p.fragment_unit)
    O.frag_index(l1, p, P, arrays=_ARR.get(id(l1)))


def _subset(sp, n):
    from vulcan.gpu.host import Spectra
    n = min(n, len(sp))
    o = sp.offsets[:n + 1]
    return Spectra(sp.run, sp.scan[:n], sp.index[:n], sp.rt[:n], sp.precursor_mz[:n], sp.charge[:n],
                   sp.mz[:o[-1]], sp.intensity[:o[-1]], o.copy())


def cpu_rate(l1, sp, p, budget_s: float, var=None):
    """spectra/s of the CPU oracle on a sample sized to take about budget_s."""
    from oracle import oracle as O
    _ARR[id(l1)] = {k: np.ascontiguousarray(getattr(l1, k)) for k in ("seq_off", "length", "mask", "mass32",
                                                                         "residues")}
    _oracle_index(l1, p, var)   # index-time work, outside the timed samples (as the device index)
    n = 500
    t0 = time.perf_counter()
    cpu_oracle_pass(l1, _subset(sp, n), p, var)
    t = time.perf_counter() - t0
    n2 = int(min(len(sp), max(n, n * budget_s / max(t, 1e-3))))
    t0 = time.perf_counter()
    ref = cpu_oracle_pass(l1, _subset(sp, n2), p, var)
    t2 = time.perf_counter() - t0
    return n2 / t2, n2, t2, O.n_threads(), ref


def parity_check(l1, sp, p, var, out, n, ref):
    """The timed plain device pass ``out`` against the oracle on the first n spectra of the run (the CPU baseline's
    own sample and results): K0, hypotheses, K1 counts and statistics, top-K lists, K2, top-1 PSMs bit for bit, and
    the largest hyperscore error against the FP64 oracle (computed here, untimed)."""
    from oracle import oracle as O
    from oracle import parity
    P = O.make_params(STATIC, VAR if var is None else var, p.fragment_unit)
    ref["k2_f64"] = O.k2_f64(l1, ref["hyp"], ref["pk"], ref["h"], ref["r"], p, P)
    res = parity.check_plain(l1, sp, p, P, out, n, ref=ref)
    res["hs_rtol_fp64"] = 1e-5
    res["all_equal"] = bool(all(res[k] for k in ("k0_equal", "hyp_equal", "k1_equal", "topk_equal", "k2_equal",
                                                 "top1_equal")) and res["hs_max_rel_err_fp64"] <= 1e-5)
    return res


def k1_algorithmic_bytes(gi, dh, peaks, item_off, n_hyp: int, intensities: bool, out_bytes: int):
    """Bytes K1 must move per launch, each piece counted once: every tile with work (postings 4 B each, coarse-bin
    CSR 2 B per bin, presence bitmap 8 B per bin); every hypothesis's spectrum peaks as K1 reads them (one 4-byte
    filter word per kept peak and fragment charge, from vk_k1_peak_keys, plus the 4-byte intensity per kept peak
    with the pruner's sums) and its record (spec 4, maxfz 1, lo/hi 16, peak offsets 16); plus ``out_bytes`` written
    (dense counts / sums per window row, or the hit lists and per-hypothesis totals).  The kernel reads a spectrum's
    filter words once per (tile, hypothesis) item; the re-reads beyond the first are not algorithmic (they mostly hit
    L2), nor are the window keys of the windows that pass the bitmap."""
    nt = gi.tix.n_tiles
    nb = 1 << gi.tix.cbin_bits
    stride = (nb + 1 + 7) & ~7
    busy = (item_off[1:] - item_off[:-1]) > 0
    tile_bytes = ((gi.tile_off[1:nt + 1] - gi.tile_off[:nt]) * 4 + stride * 2 + nb * 8)[busy].sum()
    s = dh["spec"][:n_hyp].long()
    nz = (dh["maxfz"][:n_hyp].long() - 1).clamp(min=0)
    npk = peaks["off"][s + 1] - peaks["off"][s]
    live = dh["hi"][:n_hyp] > dh["lo"][:n_hyp]
    hyp_bytes = ((npk * (4 * nz + (4 if intensities else 0)) + 37) * live).sum()
    return int((tile_bytes + hyp_bytes).item()) + int(out_bytes)


def fused_algorithmic_bytes(gi, dh, peaks, oc, n_spec):
    """Bytes the fused search moves per launch: per (hypothesis, tile) item the staged tile (postings + coarse CSR)
    and the spectrum's peak masses read by the per-peak search (4 B each); per spectrum its peaks staged for K2
    (8 B each, at most 512) and the hypothesis records (33 B each); per candidate the row gather of K2 (seq_off 8,
    length 1, mask 8, mass32 4, residues L) and, for the selected entries, the partner row (8); per spectrum the PSM
    slot written (~100 B)."""
    import torch
    ix = gi.tix
    sh = ix.tile_shift
    cb = (((1 << ix.cbin_bits) + 1 + 7) & ~7) * 2
    nh = int(dh["spec_off"][-1])
    lo, hi = dh["lo"][:nh], dh["hi"][:nh]
    ok = hi > lo
    t0 = lo[ok] >> sh
    t1 = (hi[ok] - 1) >> sh
    tiles = (t1 - t0 + 1)
    tile_b = ((gi.tile_off[t1 + 1] - gi.tile_off[t0]) * 4 + tiles * cb).sum()
    s = dh["spec"][:nh][ok].long()
    npk = peaks["off"][s + 1] - peaks["off"][s]
    peak_item_b = (npk * tiles * 4).sum()
    npk_all = (peaks["off"][1:n_spec + 1] - peaks["off"][:n_spec]).clamp(max=512)
    spec_b = (npk_all * 8).sum() + nh * 33 + n_spec * 100
    cd, cap = oc["cand"], oc["cand_cap"]
    n_cand = cd["n_cand"][:n_spec].clamp(min=0)
    idx = torch.arange(cap, device=n_cand.device)[None, :] < n_cand[:, None]
    rows = cd["c_row"][:n_spec * cap].view(n_spec, cap)[idx]
    cand_b = (21 + gi.length[rows].long()).sum() + n_cand.sum() * 4
    total = int((tile_b + peak_item_b + spec_b + cand_b).item())
    return {"total": total, "tiles": int(tile_b.item()), "peaks_per_item": int(peak_item_b.item()),
            "spectra": int(spec_b.item()), "candidates_gather": int(cand_b.item()), "items": int(tiles.sum().item()),
            "candidates": int(n_cand.sum().item())}


def _pruner_setup(a, w, l1, lab, gi, p, rank):
    """The learned pruner of the headline path: trained here on the GPU (untimed) from simulated runs disjoint
    from the benchmark run (exhaustive rescoring labels), its threshold calibrated on one more run; or loaded."""
    from vulcan import synth
    from vulcan.gpu import prune as PR
    if a.pruner != "train":
        pr = PR.Pruner.load(a.pruner, gi.dev)
        return pr, {"source": os.path.basename(a.pruner), "tau": pr.tau, "min_count": pr.min_count,
                    "shortlist_k": pr.shortlist_k}
    t0 = time.perf_counter()
    n_left, runs, i = a.train_spectra, [], 0
    while n_left > 0:
        n = min(n_left, w.n_spectra)
        runs.append(synth.simulate_run(l1, lab, w, n_spectra=n, seed=70000 + 100 * rank + i, run=f"train{i}")[0])
        n_left -= n
        i += 1
    calib = [synth.simulate_run(l1, lab, w, seed=80000 + rank, run="calib")[0]]
    t_sim = time.perf_counter() - t0
    pr, info = PR.train(gi, p, runs, calib, seed=rank, epochs=a.epochs, batch=8192, target=a.target)
    info.update(source="trained in this run", simulate_s=round(t_sim, 1), min_count=pr.min_count,
                shortlist_k=pr.shortlist_k,
                min_keep=pr.min_keep, max_keep=pr.max_keep, target=a.target,
                losses=[round(x, 5) for x in info["losses"]])
    return pr, info


def _timed_passes(step, flush, steps, world, dist, K):
    """CUDA-event time of `steps` device passes (L2 flushed before each), max over ranks; kernel launches counted."""
    import torch
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    K.LAUNCHES["n"] = 0
    evs = []
    out = None
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = step()
        e1.record()
        evs.append((e0, e1))
    torch.cuda.synchronize()
    launches = K.LAUNCHES["n"]
    if world > 1:
        dist.barrier()
    ms = sum(e0.elapsed_time(e1) for e0, e1 in evs)
    from vulcan.gpu.replicas import max_over_ranks
    return max_over_ranks(ms, flush.device), launches, out


def _h2d_rate(pinned, run, dev, reps: int = 10):
    """The run's input copy alone: the raw peak, offset and precursor arrays from pinned host memory into the
    device run's buffers on a copy stream, CUDA events on that stream; ms per run and GB/s."""
    import torch
    st = torch.cuda.Stream(dev)
    pairs = [(run.mz, pinned.mz), (run.intensity, pinned.intensity), (run.offsets, pinned.offsets),
             (run.precursor_mz, pinned.precursor_mz), (run.charge, pinned.charge)]
    nbytes = sum(a.nbytes for _, a in pairs)
    ms = []
    with torch.cuda.stream(st):
        for i in range(reps + 2):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for dst, a in pairs:
                dst[:len(a)].copy_(torch.from_numpy(a), non_blocking=True)
            e1.record(st)
            e1.synchronize()
            if i >= 2:
                ms.append(e0.elapsed_time(e1))
    t = sum(ms) / len(ms)
    return {"bytes": int(nbytes), "ms": round(t, 4), "gbs": round(nbytes / (t / 1e3) / 1e9, 1)}


def _timed_e2e(call, n_spec, steps, world, dist, dev):
    """Wall-clock spectra/s of `steps` calls through the public API (host buffers in, PSM table out)."""
    import torch
    call()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    st = None
    for _ in range(steps):
        st = call()[1]
    torch.cuda.synchronize()
    from vulcan.gpu.replicas import max_over_ranks
    return n_spec * world * steps / max_over_ranks(time.perf_counter() - t0, dev), st


def run_b200(a):
    import torch
    import torch.distributed as dist
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    from vulcan.gpu import _lib as K
    from vulcan.gpu import engine as E
    from vulcan.gpu import prune as PR
    if world > 1:   # one rank builds the cached index; the others load it after the barrier
        if rank == 0:
            from vulcan import synth
            synth.build_index(a.workload, CACHE)
        dist.barrier()
    w, l1, lab, sp, t_build = _workload_setup(a.workload, rank)
    p = _params(w, a)
    gi = E.GpuIndex(l1, p, STATIC, w.var_mods, device=dev)
    pruned = a.path == "pruned"
    pr, pr_info = _pruner_setup(a, w, l1, lab, gi, p, rank) if pruned else (None, None)
    if pruned and a.save_pruner and rank == 0:
        pr.save(a.save_pruner)
    run = E.DeviceRun(sp, dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device=dev)   # 256 MiB > 126 MB L2
    st = E.Stats()
    # the CPU baseline (rank 0 of a 1-GPU run): the oracle timed on a sample of the run; its results are kept as the
    # checker of the timed plain device pass below
    cpu, cpu_ref, n_cpu = None, None, 0
    if rank == 0 and world == 1:
        rate, n_cpu, t_s, cores, cpu_ref = cpu_rate(l1, sp, p, a.cpu_budget, w.var_mods)
        cpu = {"value": round(rate, 1), "unit": "spectra/s", "cores": cores, "kind": "port",
               "sample": f"first {n_cpu} spectra of the run through the oracle's plain path K0->hypotheses->K1 (its "
                         f"fragment index, built before)->top-k->K2->ranking ({t_s:.1f} s)"}

    def step_plain():
        if p.search_method == "fused":
            return E._search_fused_device(run, gi, p, 1, st)
        return E._search_device(run, gi, p, 1, st)

    def step_pruned():
        return PR._pruned_device(run, gi, p, pr, 1, st)

    def graphed(fn):
        """(replay function, our kernel launches per pass): the pass captured as one CUDA graph."""
        n0 = K.LAUNCHES["n"]
        fn()
        per_pass = K.LAUNCHES["n"] - n0
        gp = E.GraphedPass(fn, dev)
        return gp.replay, per_pass

    def device_timing(fn, graph: bool):
        for _ in range(a.warmup):
            fn()
        step, per_pass = graphed(fn) if graph else (fn, None)
        for _ in range(a.warmup):
            step()
        torch.cuda.synchronize()
        ms, launches, out = _timed_passes(step, flush, a.steps, world, dist, K)
        return ms, (per_pass * a.steps if per_pass is not None else launches), out

    use_graph = p.search_method != "fused"
    clocks = ClockSampler(local)
    ms_max, launches, out = device_timing(step_pruned if pruned else step_plain, use_graph)
    clk = clocks.stop()
    if use_graph:
        E.check_status(out["status"])
    ms_per_step = ms_max / a.steps
    value = len(sp) * world * a.steps / (ms_max / 1e3)
    ms_eager, _, _ = _timed_passes(step_pruned if pruned else step_plain, flush, a.steps, world, dist, K)
    if p.search_method == "fused" and not pruned:
        st_ok = int(out["status"][:len(sp)].max())
        if st_ok:
            raise RuntimeError(f"fused search status {st_ok}: spectra over the window capacity or a copy timeout")
    parity = None
    if cpu_ref is not None and not pruned and use_graph:   # the timed plain pass itself, against the oracle
        parity = parity_check(l1, sp, p, w.var_mods, out, n_cpu, cpu_ref)

    # end to end through the public API: Searcher (graph-captured passes) over runs in pinned host memory, or
    # engine.search for the fused method
    e2e_steps = max(3, min(a.steps, 20))
    pinned = E.pin_spectra(sp)

    def e2e_rate(pruner):
        if not use_graph:
            return _timed_e2e(lambda: E.search(sp, gi, l1, p), len(sp), e2e_steps, world, dist, dev)
        se = E.Searcher(gi, l1, p, pruner=pruner, report=1)
        # warm-up over as many runs as are timed: the pinned result buffers that the timed tables will own are
        # then in the caching host allocator already
        del se.search_many([pinned] * e2e_steps)[:]
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        se.host_s = {k: 0.0 for k in se.host_s}
        t0 = time.perf_counter()
        res = se.search_many([pinned] * e2e_steps)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        e2e_parts.append({"wall_ms_per_run": round(1e3 * wall / e2e_steps, 4),
                          **{f"host_{k}_ms_per_run": round(1e3 * v / e2e_steps, 4) for k, v in se.host_s.items()}})
        from vulcan.gpu.replicas import max_over_ranks
        return len(sp) * world * e2e_steps / max_over_ranks(wall, dev), res[-1][1]
    e2e_parts = []
    e2e, s2 = e2e_rate(pr)
    h2d, d2h = s2.h2d_bytes, s2.d2h_bytes
    h2d_copy = _h2d_rate(pinned, run, dev)
    comparison = None
    if pruned:
        # the plain exhaustive path on the same run, same timing rules, and the pruned path's accuracy against it
        ms_plain, _, out_plain = device_timing(step_plain, True)
        E.check_status(out_plain["status"])
        if cpu_ref is not None:   # the timed plain pass itself, against the oracle
            parity = parity_check(l1, sp, p, w.var_mods, out_plain, n_cpu, cpu_ref)
        del out_plain
        e2e_plain, _ = e2e_rate(None)
        ev = PR.evaluate(sp, gi, l1, lab, p, pr)
        comparison = {"plain_value": round(len(sp) * world * a.steps / (ms_plain / 1e3), 1),
                      "plain_ms_per_step": round(ms_plain / a.steps, 4), "plain_e2e": round(e2e_plain, 1),
                      "speedup_device": round(ms_plain / ms_max, 3), "speedup_e2e": round(e2e / e2e_plain, 3),
                      "top1_recall": round(ev["recall"], 6), "accepted_at_1pct_q_plain": ev["accepted_plain"],
                      "accepted_at_1pct_q_pruned": ev["accepted_pruned"],
                      "delta_accepted": round(ev["delta_accepted"], 6), "shortlist_hits": ev["hits"],
                      "rescored_plain": ev["rescored_plain"], "rescored_pruned": ev["rescored_pruned"]}

    # per-phase device times of both paths (separate passes, phases synchronised)
    phase_ms = {}
    paths = [("staged", lambda q, s: E._search_device(run, gi, q, 1, s, timers=True))]
    if pruned:
        paths.append(("pruned", lambda q, s: PR._pruned_device(run, gi, q, pr, 1, s, timers=True)))
    else:
        paths.append(("fused", lambda q, s: E._search_fused_device(run, gi, E._replace(q, search_method="fused"), 1,
                                                                   s, timers=True)))
    for name, fn in paths:
        st_ph = E.Stats()
        for _ in range(3):
            flush.zero_()
            fn(p, st_ph)
        phase_ms[name] = {k: round(v / 3, 4) for k, v in st_ph.gpu_ms.items()}

    peak_gbs, peak_kind = _peaks_json()
    kern, mlp = _kernel_table(a, p, gi, run, flush, pr, dev)
    dom = max(kern, key=lambda k: kern[k][0])
    k_mean, algo = kern[dom]
    achieved = algo / (k_mean / 1e3) / 1e9
    # DRAM bytes per launch from the committed ncu summary of the same kernel form (profiles/<name>_*.md)
    traffic = _traffic_from_profiles({"k1_tiles_k (hit lists)": "k1_tiles_hits", "k1_tiles_k": "k1_tiles_dense"}.get(
        dom, dom[:-2] if dom.endswith("_k") else dom))
    kernels = {k: {"mean_launch_ms": round(v[0], 4), "algorithmic_bytes": v[1],
                   "algorithmic_gbs": round(v[1] / (v[0] / 1e3) / 1e9, 1)} for k, v in kern.items()}

    if rank == 0:
        extra = {"spectra_per_step_per_gpu": len(sp), "index_rows": len(l1), "index_postings": gi.n_postings,
                 "tile_rows": p.tile_rows, "parallelism": f"replicas x{world} (one run per GPU)",
                 "launch": "one CUDA graph per pass (eager_ms_per_step: the same pass launched kernel by kernel)"
                           if use_graph else "kernel by kernel",
                 "e2e": "Searcher.search_many over the run in pinned host memory, three runs in flight: H2D on a "
                        "copy stream, graph replay on a compute stream, one D2H of the packed PSM slots on a third "
                        "stream, host PSM table" if use_graph else "engine.search"}
        if pruned:
            extra["path"] = ("learned-pruned search: K1 (+ intensity sums) -> shortlist of the top "
                             f"{pr.shortlist_k or p.topk} hits by count with count >= "
                             f"{pr.min_count} -> BF16 MLP 16-256-256-1 -> logit >= calibrated tau or best "
                             f"{pr.min_keep} -> pair closure -> K2 -> ranking")
            extra["pruner"] = pr_info
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": "spectra/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(ms_per_step, 4), "eager_ms_per_step": round(ms_eager / a.steps, 4),
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (MLP: bf16 weights, fp32 accumulate)" if pruned else "f32",
            "data": "synthetic",
            "config": _config(w, p, extra),
            "e2e": {"value": round(e2e, 1), "unit": "spectra/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "h2d_copy_alone": h2d_copy,
                    "per_run": e2e_parts[0] if e2e_parts else None},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1),
                         "peak": peak_gbs, "unit": "GB/s", "frac": round(achieved / peak_gbs, 4),
                         "peak_source": peak_kind, "traffic": traffic, "algorithmic_bytes": algo,
                         "mean_launch_ms": round(k_mean, 4),
                         # the same launch time against the DRAM bytes ncu measured per launch
                         "dram_frac": round(traffic / (k_mean / 1e3) / 1e9 / peak_gbs, 4) if traffic else None},
            "kernels": kernels,
            "cpu_baseline": cpu,
            "clocks": clk,
            "phase_ms": phase_ms,
            "index_build_s": round(t_build, 1),
        }
        if mlp:
            line["mlp_roofline"] = mlp
        if comparison:
            line["vs_plain"] = comparison
        if parity is not None:
            line["parity"] = parity
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def _tensor_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d.get("bf16_tflops", 1590.0)), "measured (burst)"
    return 1590.0, "fallback"


def _kernel_table(a, p, gi, run, flush, pr, dev):
    """Each main kernel of the timed path alone: mean CUDA-event duration over 8 launches after 2 warm-up launches
    (L2 flushed before each) and its algorithmic bytes; for the pruned path also the MLP's tensor roofline."""
    import ctypes as C
    import torch
    from vulcan.gpu import _lib as K
    from vulcan.gpu import engine as E
    from vulcan.gpu import prune as PR
    L = K.lib()
    st = E.Stats()
    pruned = pr is not None
    so = PR._pruned_device(run, gi, p, pr, 1, st) if pruned else E._search_device(run, gi, p, 1, st)
    peaks, dh = so["peaks"], so["dh"]
    n = run.n

    def timed(fn, reps=10):
        ts = []
        for _ in range(reps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return sum(ts[2:]) / len(ts[2:])
    nh = int(dh["spec_off"][-1])
    pl = E._k1_plan(gi, dh, p, dh["n_max"])
    item_off, item_hyp = pl["item_off"], pl["item_hyp"]
    win_off = pl["win_off"]
    n_win = int(win_off[-1])
    kern = {}
    keys, filt, n_kz, kstride = E.peak_keys(gi, peaks, p)
    n_pk = int(peaks["off"][-1])
    ms_keys = timed(lambda: E.peak_keys(gi, peaks, p))
    kern["peak_keys_k"] = (ms_keys, n_pk * (4 + 12 * n_kz))
    # the small stages before K1, each captured as a CUDA graph of its launches and replayed (as in the pass): K0
    # (count, scan of the kept counts, the copy or selection of every spectrum's peaks), the hypotheses (count,
    # scan, fill, row windows), K1's planning (items per tile, scans, fill); bytes: raw peaks read twice and the
    # view written / spectra and hypotheses / items
    n_raw = int(run.offsets[-1])
    ms_k0 = timed(E.GraphedPass(lambda: E._k0_device(run, p, dev), dev).replay)
    kern["k0 stage (graph of its launches)"] = (ms_k0, n_raw * 16 + n_pk * 8 + n * 40)
    ms_hy = timed(E.GraphedPass(lambda: E._hyp_device(run, peaks, gi, p), dev).replay)
    kern["hypotheses stage (graph of its launches)"] = (ms_hy, n * 16 + nh * 40)
    ms_pl = timed(E.GraphedPass(lambda: E._k1_plan(gi, dh, p, dh["n_max"]), dev).replay)
    kern["K1 planning stage (graph of its launches)"] = (ms_pl, nh * 40 + int(item_off[-1]) * 8 +
                                                         gi.tix.n_tiles * 32)
    hits = so["hits"] if pruned else so
    n_hit = int(hits["cand_off"][-1])
    cap = hits["cap"]
    if pruned:
        # K1 in hit-list form (rows with count >= the floor appended per hypothesis), then the shortlist over the
        # hit lists: the kernels of the pruned path
        thr = max(p.k1_threshold, pr.min_count)
        k1h = so["k1_hits"]
        nm = dh["n_max"]
        z = torch.zeros(nm * 3, dtype=torch.int64, device=dev)

        def run_k1():
            z.zero_()
            K.check(L.vk_k1_hits(
                C.byref(gi.tix), C.byref(gi.fp), float(p.fragment_ppm[0]), float(p.fragment_ppm[1]), p.k1_warps,
                K.ptr(item_off), K.ptr(item_hyp), nm, pl["item_cap"], K.ptr(dh["spec"]), K.ptr(dh["maxfz"]),
                K.ptr(dh["lo"]), K.ptr(dh["hi"]), K.ptr(win_off), pl["cnt_cap"], K.ptr(peaks["off"]),
                K.ptr(peaks["mass"]), thr, None, K.ptr(k1h["rc"]), K.ptr(k1h["isum"]), K.ptr(k1h["seg_cnt"]),
                K.ptr(z[2 * nm:].view(torch.int8)[:nm]), K.ptr(z[:nm].view(torch.int32)[:nm]), K.ptr(z[nm:2 * nm]),
                K.ptr(pl["status"]), K.ptr(peaks["int"]), K.ptr(peaks["tic"]), K.ptr(keys), K.ptr(filt), n_kz,
                kstride, K.stream()), "k1_hits")
        ms_k1 = timed(run_k1)
        # the hits K1 keeps: the dense counts of the same windows over the floor
        cnt_d = E._k1_dense(gi, dh, peaks, p, nm)[1]
        n_k1_hits = int((cnt_d[:n_win] >= thr).sum())
        del cnt_d
        kern["k1_tiles_k (hit lists)"] = (ms_k1, k1_algorithmic_bytes(gi, dh, peaks, item_off, nh, True,
                                                                       n_k1_hits * 12 + int(item_off[-1]) * 4 +
                                                                       nh * 13))
        tk = {k: torch.empty(max(n * cap, 1), dtype=torch.int64, device=dev) for k in ("h", "r", "c")}
        ti = torch.empty(max(n * cap, 1), dtype=torch.int32, device=dev)
        tk_n = torch.empty(n, dtype=torch.int64, device=dev)
        ss_ = torch.empty(n, dtype=torch.int64, device=dev)
        sm_ = torch.empty(n, dtype=torch.int64, device=dev)
        ms_tk = timed(lambda: K.check(L.vk_select_hits(
            n, K.ptr(dh["spec_off"]), K.ptr(dh["lo"]), K.ptr(dh["hi"]), K.ptr(win_off), K.ptr(k1h["hyp_shift"]),
            K.ptr(k1h["seg_cnt"]), K.ptr(k1h["rc"]), K.ptr(k1h["isum"]), K.ptr(k1h["hyp_scored"]), K.ptr(k1h["hyp_matched"]), cap, 0,
            None, cap, K.ptr(tk["h"]), K.ptr(tk["r"]),
            K.ptr(tk["c"]), K.ptr(ti), K.ptr(tk_n), K.ptr(ss_), K.ptr(sm_), K.stream()), "select_hits"))
        # hits read (12 B), per-hypothesis windows, totals and tile shift (33 B), per spectrum its hypothesis range
        # and outputs; the shortlist written (28 B per kept hit)
        kern["select_hits_k"] = (ms_tk, n_k1_hits * 12 + int(item_off[-1]) * 4 + nh * 41 + n * 32 + n_hit * 28)
    else:
        cnt = so["cnt"]
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        ms_k1 = timed(lambda: K.check(L.vk_k1_tiles(
            C.byref(gi.tix), C.byref(gi.fp), float(p.fragment_ppm[0]), float(p.fragment_ppm[1]), p.k1_warps,
            K.ptr(item_off), K.ptr(item_hyp), dh["n_max"], pl["item_cap"], K.ptr(dh["spec"]), K.ptr(dh["maxfz"]),
            K.ptr(dh["lo"]), K.ptr(dh["hi"]), K.ptr(win_off), cnt.numel(), K.ptr(peaks["off"]),
            K.ptr(peaks["mass"]), K.ptr(cnt), K.ptr(status), None, None, None, K.ptr(keys), K.ptr(filt), n_kz,
            kstride, K.stream()), "k1_tiles"))
        kern["k1_tiles_k"] = (ms_k1, k1_algorithmic_bytes(gi, dh, peaks, item_off, nh, False, n_win * 4))
        tk = {k: torch.empty(max(n * cap, 1), dtype=torch.int64, device=dev) for k in ("h", "r", "c")}
        tk_n = torch.empty(n, dtype=torch.int64, device=dev)
        hs_ = torch.empty(dh["n_max"], dtype=torch.int32, device=dev)
        hm_ = torch.empty(dh["n_max"], dtype=torch.int64, device=dev)
        ss_ = torch.empty(n, dtype=torch.int64, device=dev)
        sm_ = torch.empty(n, dtype=torch.int64, device=dev)
        ms_tk = timed(lambda: K.check(L.vk_select_topk(
            n, K.ptr(dh["spec_off"]), K.ptr(dh["lo"]), K.ptr(dh["hi"]), K.ptr(win_off), K.ptr(cnt), cnt.numel(),
            K.ptr(gi.partner), p.k1_threshold, p.topk, int(p.pair_closure), cap, K.ptr(tk["h"]), K.ptr(tk["r"]),
            K.ptr(tk["c"]), K.ptr(tk_n), K.ptr(hs_), K.ptr(hm_), K.ptr(ss_), K.ptr(sm_), K.stream()), "select_topk"))
        n_sel = int(((hits["c_cnt"][:n_hit] >= 0)).sum())
        kern["select_topk_k"] = (ms_tk, n_win * 4 + n_sel * 8 + n_hit * 24 + nh * 12 + n * 16)
    mlp = None
    if pruned:
        feat = so["feat"]
        # the shortlist's compaction with the features written on the way (the pass's form), on select_hits' slots
        c_off = E._scan(tk_n[:n])
        cc = {k: torch.empty(max(n * cap, 1), dtype=torch.int64, device=dev) for k in ("h", "r", "c")}
        c32 = torch.empty(max(n * cap, 1), dtype=torch.int32, device=dev)
        cmf = torch.empty(max(n * cap, 1), dtype=torch.int8, device=dev)
        cis = torch.empty(max(n * cap, 1), dtype=torch.int32, device=dev)
        fe = torch.empty(max(n * cap, 1), 16, dtype=torch.bfloat16, device=dev)
        ms_f = timed(lambda: K.check(L.vk_compact_hits_features(
            n, cap, K.ptr(tk_n), K.ptr(c_off), K.ptr(tk["h"]), K.ptr(tk["r"]), K.ptr(tk["c"]), K.ptr(ti),
            K.ptr(dh["maxfz"]), K.ptr(cc["h"]), K.ptr(cc["r"]), K.ptr(cc["c"]), K.ptr(c32), K.ptr(cmf), K.ptr(cis),
            K.ptr(dh["M"]), K.ptr(dh["z"]), K.ptr(gi.mass32), K.ptr(gi.length), K.ptr(gi.missed), K.ptr(pr.mu),
            K.ptr(pr.sd), K.ptr(fe), K.stream()), "compact_hits_features"))
        # per hit: its slot read (28 B), hypothesis / row gathers (12 B), compacted columns (33 B), features (32 B)
        kern["compact_hits_features_k"] = (ms_f, n_hit * 105)
        ms_m = timed(lambda: pr.logits(feat, n_hit))
        flops = 2 * n_hit * (16 * 256 + 256 * 256 + 256)
        mlp_name = "mlp_infer_tc_k" if pr.tensor_cores == "tcgen05" else "mlp_infer_k"
        kern[mlp_name] = (ms_m, n_hit * 36 + 2 * (256 * 16 + 256 * 256) + 4 * 256 * 3)
        tpk, tkind = _tensor_peak()
        ach = flops / (ms_m / 1e3) / 1e12
        mlp = {"bound": "tensor", "kernel": mlp_name, "achieved": round(ach, 1), "peak": tpk,
               "unit": "TFLOP/s", "frac": round(ach / tpk, 4), "peak_source": tkind, "flops_per_launch": flops,
               "hits_per_launch": n_hit, "mean_launch_ms": round(ms_m, 4),
               "instruction": ("tcgen05.mma kind::f16 M128 N256 (bf16, fp32 accumulate in TMEM)"
                               if pr.tensor_cores == "tcgen05" else "mma.sync m16n8k16 bf16 (fp32 accumulate)")}
    n_cand = int(so["cand_off"][-1])
    k2o = E._k2_outputs(max(n_cand, 1), dev)
    k2_args = (C.byref(gi.fp), n, K.ptr(so["cand_off"]), K.ptr(so["c_row32"]), K.ptr(so["c_maxfz"]),
               K.ptr(peaks["off"]), K.ptr(peaks["mass"]), K.ptr(peaks["int"]), *gi.table_ptrs(),
               float(p.fragment_ppm[0]), float(p.fragment_ppm[1]))
    rows = so["c_row"][:n_cand]
    npk = (peaks["off"][1:n + 1] - peaks["off"][:n]).clamp(max=512)
    k2_bytes = int(((21 + gi.length[rows].long() + 5 + 28).sum() + npk.sum() * 8 + n * 16).item())
    # the path's K2 (thread per candidate after the pruner, warp per spectrum otherwise) and the other for reference
    ms_sp = timed(lambda: K.check(L.vk_k2_spectra(*k2_args, None, *E._k2_ptrs(k2o), K.stream()), "k2_spectra"))
    ms_cd = timed(lambda: K.check(L.vk_k2_cands(*k2_args, *E._k2_ptrs(k2o), K.stream()), "k2_cands"))
    if pruned:
        kern["k2_cands_k"] = (ms_cd, k2_bytes)
        kern["k2_spectra_k (not used on this path)"] = (ms_sp, k2_bytes)
    else:
        kern["k2_spectra_k"] = (ms_sp, k2_bytes)
        kern["k2_cands_k (not used on this path)"] = (ms_cd, k2_bytes)
    if p.search_method == "fused" and not pruned:
        kern = {"fused_search_k": (timed(lambda: E._fused_device(gi, p, 1, peaks, dh, run.n)),
                                   fused_algorithmic_bytes(gi, dh, peaks, E._fused_device(gi, p, 1, peaks, dh, run.n,
                                                                                          cand=True), n)["total"])}
    return kern, mlp


BATCH_SETUPS = {   # workload -> (index workload, runs, smallest, largest run, spectra per batch, description)
    "batch64": ("human", 64, 5000, 60000, 262144, "configuration 2: 64 runs, batched, graph-captured"),
    "phospho": ("phospho", 32, 20000, 50000, 65536,
                "configuration 4: phospho S/T/Y <= 3 + Met-ox <= 1 index, 32 runs, batched, graph-captured"),
}


def run_batch(a):
    """Configurations 2 and 4: many runs (sizes log-uniform), drawn from a pool of simulated spectra, searched in
    fixed-shape batches, each batch one replay of a captured CUDA graph; tile rows and K1 warps (per peak-count
    bucket) chosen by the autotuner on a sample; learned-pruned and plain paths, each run's table checked against
    its own search.  With N ranks the same runs are spread over the GPUs (``replicas.shard_runs``, whole runs
    balanced by size): a fixed job, strong scaling.  Rank 0 of a 1-GPU run also times the CPU oracle on a sample of
    the first run and checks the plain device pass against it (parity), and reports the dominant kernel's
    roofline on that run."""
    import torch
    from vulcan import synth
    from vulcan.gpu import autotune as AT
    from vulcan.gpu import engine as E
    from vulcan.gpu import prune as PR
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import torch.distributed as dist
    from vulcan.gpu.replicas import max_over_ranks
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)
    wl, n_runs, lo_run, hi_run, batch_default, desc = BATCH_SETUPS[a.workload]
    batch_spectra = a.batch_spectra or batch_default
    w, l1, lab, _, t_build = _workload_setup(wl, rank)
    var = w.var_mods
    p0 = _params(w, a)
    pool = synth.simulate_run(l1, lab, w, n_spectra=120000, seed=90000, run="pool")[0]
    all_runs = synth.batch_runs(pool, n_runs, lo_run, hi_run, seed=2)
    n_total = sum(len(r) for r in all_runs)
    from vulcan.gpu.replicas import shard_runs
    runs = [all_runs[i] for i in shard_runs(all_runs, rank, world)]       # this rank's share of the job
    gi0 = E.GpuIndex(l1, p0, STATIC, var, device=dev)
    pr, pr_info = _pruner_setup(a, w, l1, lab, gi0, p0, 0)
    del gi0
    torch.cuda.empty_cache()
    cpu, cpu_ref, n_cpu = None, None, 0
    if rank == 0 and world == 1:   # the CPU oracle on a sample of the first run (its results check the device)
        rate, n_cpu, t_s, cores, cpu_ref = cpu_rate(l1, all_runs[0], p0, a.cpu_budget, var)
        cpu = {"value": round(rate, 1), "unit": "spectra/s", "cores": cores, "kind": "port",
               "sample": f"first {n_cpu} spectra of the first run through the oracle's plain path K0->hypotheses->"
                         f"K1->top-k->K2->ranking ({t_s:.1f} s)"}
    sample = synth.take_spectra(pool, np.arange(40000), "sample")
    p, tune_report = AT.tune(l1, p0, STATIC, var, sample, pruner=pr, device=dev)
    gi = E.GpuIndex(l1, p, STATIC, var, device=dev)
    pinned = [E.pin_spectra(r) for r in runs]
    reps = max(2, a.steps // 10)
    res = {}
    clocks = ClockSampler(local)
    for name, prn in (("pruned", pr), ("plain", None)):
        se = E.Searcher(gi, l1, p, pruner=prn, report=1)
        tables = se.search_batch(pinned, batch_spectra=batch_spectra)     # captures the batch shape
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        se.device_ms = 0.0
        t0 = time.perf_counter()
        for _ in range(reps):
            # a step's tables are written out and dropped before the next step: their pinned result buffers go
            # back to the Searcher's pool (a caller keeping every table gets copies once the pool is lent out)
            tables = None
            tables = se.search_batch(pinned, batch_spectra=batch_spectra)
        torch.cuda.synchronize()
        wall = max_over_ranks(time.perf_counter() - t0, dev)
        res[name] = {"tables": [t for t, _ in tables], "device_ms": max_over_ranks(se.device_ms, dev) / reps,
                     "wall_s": wall / reps,
                     "batches": len(E.plan_batches(runs, batch_spectra)), "h2d": sum(s.h2d_bytes for _, s in tables),
                     "d2h": sum(s.d2h_bytes for _, s in tables)}
        del se
        torch.cuda.empty_cache()
    clk = clocks.stop()
    parity = kern = mlp = None
    if cpu_ref is not None:
        run0 = E.DeviceRun(all_runs[0], dev)
        out0 = E._search_device(run0, gi, p, 1, E.Stats())
        E.check_status(out0["status"])
        parity = parity_check(l1, all_runs[0], p, var, out0, n_cpu, cpu_ref)
        del out0
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device=dev)
        kern, mlp = _kernel_table(a, p, gi, run0, flush, pr, dev)
        del run0, flush
    # each run's batched table equals its own search (first two runs)
    for i in range(min(2, len(runs))):
        assert res["plain"]["tables"][i].equals(E.search(runs[i], gi, l1, p)[0]), "batched plain table differs"
        assert res["pruned"]["tables"][i].equals(PR.search_pruned(runs[i], gi, l1, p, pr)[0]), \
            "batched pruned table differs"
    rec = sum(PR.top1_recall(a_, b_) * a_.num_rows for a_, b_ in zip(res["plain"]["tables"], res["pruned"]["tables"]))
    rec /= max(1, sum(t.num_rows for t in res["plain"]["tables"]))
    acc_plain = sum(PR.accepted_psms(t, lab) for t in res["plain"]["tables"])
    acc_pr = sum(PR.accepted_psms(t, lab) for t in res["pruned"]["tables"])
    pr_ms, pl_ms = res["pruned"]["device_ms"], res["plain"]["device_ms"]
    if rank == 0:
        line = {
            "metric": METRIC + f" ({desc})", "value":
                round(n_total / (pr_ms / 1e3), 1), "unit": "spectra/s", "n_gpus": world, "steps": reps,
            "warmup": 1, "ms_per_step": round(pr_ms, 3), "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32 (MLP: bf16 weights, fp32 accumulate)", "data": "synthetic",
            "config": {"workload": f"{n_runs} runs of {lo_run:,}-{hi_run:,} spectra (log-uniform; {n_total} spectra) "
                                   f"drawn from 120,000 simulated spectra, {wl} index ({len(l1)} peptidoforms)"
                                   + (f", {int(100 * w.phospho_frac)}% of spectra from phosphopeptides"
                                      if w.phospho_frac else ""),
                       "topk": p.topk,
                       "batch_spectra": batch_spectra, "batches_rank0": res["pruned"]["batches"],
                       "step": f"all {n_runs} runs once, spread over the GPUs", "tile_rows": p.tile_rows,
                       "k1_warps": p.k1_warps, "k1_shapes": [list(x) for x in p.k1_shapes],
                       "index_resident_gb": round(gi.device_bytes / 1e9, 2),
                       "l2": f"not flushed (batches of up to {batch_spectra:,} spectra, working sets above L2)",
                       "pruner": pr_info},
            "e2e": {"value": round(n_total / res["pruned"]["wall_s"], 1), "unit": "spectra/s",
                    "h2d_bytes_per_step": int(res["pruned"]["h2d"]), "d2h_bytes_per_step": int(res["pruned"]["d2h"])},
            "vs_plain": {"plain_value": round(n_total / (pl_ms / 1e3), 1), "plain_ms_per_step": round(pl_ms, 3),
                         "plain_e2e": round(n_total / res["plain"]["wall_s"], 1),
                         "speedup_device": round(pl_ms / pr_ms, 3),
                         "speedup_e2e": round(res["plain"]["wall_s"] / res["pruned"]["wall_s"], 3),
                         "top1_recall": round(rec, 6), "accepted_at_1pct_q_plain": acc_plain,
                         "accepted_at_1pct_q_pruned": acc_pr,
                         "delta_accepted": round((acc_pr - acc_plain) / max(acc_plain, 1), 6),
                         "tables_checked_against_per_run_search": 2},
            "autotune": tune_report, "clocks": clk, "index_build_s": round(t_build, 1),
            "cpu_baseline": cpu,
        }
        if parity is not None:
            line["parity"] = parity
        if kern:
            peak_gbs, peak_kind = _peaks_json()
            dom = max(kern, key=lambda k: kern[k][0])
            k_mean, algo = kern[dom]
            ach = algo / (k_mean / 1e3) / 1e9
            line["roofline"] = {"bound": "hbm", "kernel": dom, "achieved": round(ach, 1), "peak": peak_gbs,
                                "unit": "GB/s", "frac": round(ach / peak_gbs, 4), "peak_source": peak_kind,
                                "traffic": None, "algorithmic_bytes": algo, "mean_launch_ms": round(k_mean, 4),
                                "on": "the first run, alone (L2 flushed)"}
            line["kernels"] = {k: {"mean_launch_ms": round(v[0], 4), "algorithmic_bytes": v[1]} for k, v in kern.items()}
            if mlp:
                line["mlp_roofline"] = mlp
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def _traffic_from_profiles(kernel: str):
    """DRAM bytes per launch of `kernel` recorded from an ncu capture in profiles/<kernel>_*.md (a line
    'dram_bytes_per_launch: N'), or None."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for f in sorted(os.listdir(d)):
        if f.startswith(kernel) and f.endswith(".md"):
            for ln in open(os.path.join(d, f)):
                if ln.strip().startswith("dram_bytes_per_launch:"):
                    try:
                        return int(float(ln.split(":", 1)[1].strip().split()[0]))
                    except ValueError:
                        return None
    return None


def run_profile(a):
    import torch
    from vulcan.gpu import engine as E
    dev = torch.device("cuda", 0)
    w, l1, _, sp, _ = _workload_setup(a.workload, 0)
    p = _params(w, a)
    gi = E.GpuIndex(l1, p, STATIC, w.var_mods, device=dev)
    run = E.DeviceRun(sp, dev)
    st = E.Stats()
    pr = None
    if a.path == "pruned":   # kernel shapes only: a saved pruner, or an untrained one with a typical count floor
        from vulcan.gpu import prune as PR
        if a.pruner != "train":
            pr = PR.Pruner.load(a.pruner, dev)
        else:   # the count floor and shortlist cap the calibration picks on the human run
            pr = PR.Pruner(dev, tau=0.0, min_count=2)
            pr.shortlist_k = 8
    for _ in range(2):
        if pr is not None:
            PR._pruned_device(run, gi, p, pr, 1, st)
        elif p.search_method == "fused":
            E._search_fused_device(run, gi, p, 1, st)
        else:
            E._search_device(run, gi, p, 1, st)
    torch.cuda.synchronize()
    print(json.dumps({"profile_passes": 2, "path": a.path, "spectra": len(sp), "index_rows": len(l1)}), flush=True)


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    w, l1, _, sp, _ = _workload_setup(BATCH_SETUPS[a.workload][0] if a.workload in BATCH_SETUPS else a.workload, 0)
    p = w.search_params()
    _ARR[id(l1)] = {k: np.ascontiguousarray(getattr(l1, k)) for k in ("seq_off", "length", "mask", "mass32",
                                                                         "residues")}
    _oracle_index(l1, p, w.var_mods)   # index-time work, before any timed sample
    # per-step sample sized so warmup + steps take about a.cpu_total seconds
    t0 = time.perf_counter()
    cpu_oracle_pass(l1, _subset(sp, 300), p, w.var_mods)
    per_spec = (time.perf_counter() - t0) / 300
    n_step = int(max(100, min(len(sp), a.cpu_total / max(1, a.steps + a.warmup) / max(per_spec, 1e-6))))
    for i in range(a.warmup):
        cpu_oracle_pass(l1, _subset(sp, n_step), p, w.var_mods)
    t0 = time.perf_counter()
    for i in range(a.steps):
        cpu_oracle_pass(l1, _subset(sp, n_step), p, w.var_mods)
    t = time.perf_counter() - t0
    value = n_step * a.steps / t
    cores = O.n_threads()
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "spectra/s", "n_gpus": int(os.environ.get("WORLD_SIZE", 1)),
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(t / a.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
        "config": _config(w, p, {"spectra_per_step": n_step}),
        "cpu_baseline": {"value": round(value, 1), "unit": "spectra/s", "cores": cores, "kind": "port",
                         "sample": f"{n_step} spectra per step of the same simulated run (K1 over the oracle's "
                                   f"fragment index, built before the timed steps)"},
        "e2e": {"value": round(value, 1), "unit": "spectra/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _launch_ranks(n: int) -> int:
    """Run this command as n ranks on this node (torch.distributed.run, rendezvous on 127.0.0.1, a free port),
    bounded by a timeout well above the process group's own; returns the launcher's exit status."""
    import socket
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        port = sock.getsockname()[1]
    cmd = ["timeout", "-k", "60", "3600", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={n}", "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--workload", choices=("human", "small", "batch64", "phospho"), default="human",
                    help="batch64: configuration 2 (64 runs, batched graph-captured search, autotuned layout); "
                         "phospho: configuration 4 (phospho var-mod index, 32 runs, batched)")
    ap.add_argument("--batch-spectra", type=int, default=None, help="spectra per batch (batch workloads)")
    ap.add_argument("--cpu-budget", type=float, default=15.0, help="seconds of CPU-baseline work (rank 0, N=1)")
    ap.add_argument("--cpu-total", type=float, default=120.0, help="seconds of the reference arm in total")
    ap.add_argument("--method", choices=("staged", "fused"), default="staged",
                    help="staged: a kernel per stage; fused: one persistent kernel per run after K0 and hypotheses")
    ap.add_argument("--k1-warps", type=int, default=None, help="warps per K1 CTA (one CTA per index tile)")
    ap.add_argument("--warps", type=int, default=None, help="warps per fused-search CTA")
    ap.add_argument("--tile-rows", type=int, default=None, help="rows per fragment-index tile")
    ap.add_argument("--path", choices=("pruned", "plain"), default="pruned",
                    help="pruned: the learned-pruned search (headline; the plain path is timed beside it); plain: "
                         "the exhaustive K1 -> top-k -> K2 path alone")
    ap.add_argument("--pruner", default="train",
                    help="'train': train the pruner on the GPU before timing (untimed); else a saved pruner (.npz)")
    ap.add_argument("--save-pruner", default=None, help="save the trained pruner (.npz) here")
    ap.add_argument("--train-spectra", type=int, default=200000, help="simulated training spectra")
    ap.add_argument("--epochs", type=int, default=3, help="training epochs")
    ap.add_argument("--target", type=float, default=0.9995, help="calibration target of top-1 recall")
    ap.add_argument("--mode", choices=("bench", "profile"), default="bench",
                    help="profile: set up the workload and run two device passes only (for an ncu capture of one "
                         "kernel launch of the second pass, e.g. -k regex:k1_tiles -s 1 -c 1)")
    a = ap.parse_args()
    if a.warmup < 3:
        ap.error("--warmup must be >= 3")
    if a.gpus < 1:
        ap.error("--gpus must be >= 1")
    if a.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: relaunch this command under torch.distributed.run with N ranks (rank 0 prints)
        sys.exit(_launch_ranks(a.gpus))
    if a.impl == "reference":
        run_reference(a)
    elif a.workload in BATCH_SETUPS:
        run_batch(a)
    elif a.mode == "profile":
        run_profile(a)
    else:
        run_b200(a)


if __name__ == "__main__":
    main()
