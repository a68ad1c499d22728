"""GPU closed search on B200: K0 peak view -> hypotheses -> K1 (tiled fragment index) -> top-K + pair closure
-> K2 exact rescoring -> PSM ranking.  Mirror of the reference's ``vulcan/gpu/engine.py``: the same public names
(``SAGE_MONO``, ``Stats``, ``GpuIndex``, ``k0_preprocess``, ``work_items``, ``Timer``, ``run_k1``, ``select_topk``,
``run_k2``, ``lnfact``, ``psm_table``, ``search``, ``window_candidates``, ``k1_brute``, ``search_exhaustive``) with
the same arguments and results.

Where the work runs: every stage of ``search`` is a kernel of ``libvulcan_b200.so`` (``include/vulcan_b200.h``);
torch only allocates device memory and hands pointers across.  Scoring semantics are the reference's (Sage f32
arithmetic; candidate order and tie rules of ``engine.py:284-312`` and ``:366-392``).  Nothing reads labels.
"""
from __future__ import annotations

import collections
import ctypes as C
import math
import resource
import time
import weakref
from dataclasses import dataclass, field

import numpy as np
import pyarrow as pa
import torch

from . import _lib as K
from .host import NEUTRON, PROTON, SearchParams, Spectra, make_hypotheses, max_fragment_z, pre_hypotheses  # noqa: F401

SAGE_MONO = np.array([71.03711, 0.0, 103.00919, 115.02694, 129.04259, 147.0684, 57.02146, 137.05891, 113.08406,
                      0.0, 128.09496, 113.08406, 131.0405, 114.04293, 237.14774, 97.05276, 128.05858, 156.1011,
                      87.03203, 101.04768, 150.95363, 99.06841, 186.07932, 0.0, 163.06332, 0.0], np.float32)

ROW_BITS = 28   # candidate rows < 2^28 (top-K key packing of the reference, engine.py:35)


def cbin_bits(p: SearchParams) -> int:
    """Coarse m/z bins per index tile (log2): p.cbin_bits, or 2^8 per 64 rows (~6 postings per bin)."""
    if p.cbin_bits:
        return int(p.cbin_bits)
    return int(min(12, 8 + max(0, int(math.log2(p.tile_rows)) - 6)))


@dataclass
class Slice:
    """One slice of the reference-layout (chunk, log bin) CSR, for the reference-compatible ``vk_k1``."""
    chunk0: int
    chunk1: int
    offsets: torch.Tensor
    entries: torch.Tensor


@dataclass
class Stats:
    h2d_bytes: int = 0
    d2h_bytes: int = 0
    gpu_ms: dict = field(default_factory=dict)
    wall_s: dict = field(default_factory=dict)
    counts: dict = field(default_factory=dict)


def frag_params(static_mods: dict, var_mods: dict, fragment_unit: str = "ppm") -> K.FragParams:
    fp = K.FragParams()
    stat = np.zeros(26, np.float32)
    var = np.zeros(26, np.float32)
    nterm = 0.0
    for r, m in static_mods.items():
        stat[ord(r) - 65] = np.float32(m)
    for r, m in var_mods.items():
        if r == "^":
            nterm = float(np.float32(m))
            continue
        var[ord(r) - 65] = np.float32(m)
    for i in range(26):
        fp.mono[i] = float(SAGE_MONO[i])
        fp.stat[i] = float(stat[i])
        fp.var[i] = float(var[i])
    fp.nterm = nterm
    if fragment_unit not in ("ppm", "da"):
        raise ValueError("fragment_unit must be 'ppm' or 'da'")
    fp.tol_da = int(fragment_unit == "da")
    return fp


_SIDE: dict = {}


def _side_stream(dev) -> torch.cuda.Stream:
    """A second stream per device for launches that may overlap the pass's own (one per process)."""
    d = torch.device(dev).index or 0
    s = _SIDE.get(d)
    if s is None:
        s = _SIDE[d] = torch.cuda.Stream(device=torch.device("cuda", d))
    return s


class _Forked:
    """Work launched on the side stream after everything queued so far on the current stream (``fn`` launches on
    ``K.stream()`` and allocates nothing); ``get()`` makes the current stream wait for it and returns fn's value.
    Under CUDA-graph capture the two streams become parallel branches of the graph."""

    def __init__(self, dev, fn):
        main = torch.cuda.current_stream(dev)
        self.side = _side_stream(dev)
        self.side.wait_stream(main)
        with torch.cuda.stream(self.side):
            self.value = fn()
        self.joined = False

    def get(self):
        if not self.joined:
            torch.cuda.current_stream(self.side.device).wait_stream(self.side)
            self.joined = True
        return self.value


def _scan(x: torch.Tensor) -> torch.Tensor:
    """Exclusive scan (n+1 entries) of an int64 device vector, on the device."""
    L = K.lib()
    n = x.numel()
    out = torch.empty(n + 1, dtype=torch.int64, device=x.device)
    tmp = torch.empty((L.vk_scan_tmp_bytes(n) + 7) // 8, dtype=torch.int64, device=x.device)
    K.check(L.vk_scan_i64(K.ptr(x), n, K.ptr(out), K.ptr(tmp), K.stream()), "scan", L.vk_scan_kernels(n))
    return out


class GpuIndex:
    """Device-resident peptidoform table + tiled fragment index.

    Tiles of ``params.tile_rows`` mass-sorted rows; per tile the fragments sorted by exact f32 mass in coarse m/z
    bins (CSR), each posting the low key bits and the local row (``include/vulcan_b200.h``).  The
    reference-layout CSR slices (``slices``) used by the reference-compatible ``vk_k1`` are built on first use.
    """

    def __init__(self, l1, params: SearchParams, static_mods: dict, var_mods: dict, device="cuda"):
        t0 = time.perf_counter()
        self.p = params
        self.dev = torch.device(device)
        L = K.lib()
        self.static_mods, self.var_mods = dict(static_mods), dict(var_mods)
        self.fp = frag_params(static_mods, var_mods, params.fragment_unit)
        # process-wide constants of the reference-compatible entry points (as the reference sets them)
        stat = np.array(self.fp.stat[:], np.float32)
        var = np.array(self.fp.var[:], np.float32)
        with torch.cuda.device(self.dev):
            K.check(L.vk_set_params(SAGE_MONO.ctypes.data, stat.ctypes.data, var.ctypes.data), "set_params")
            K.check(L.vk_set_nterm(self.fp.nterm), "set_nterm")
            K.check(L.vk_set_tol_da(self.fp.tol_da), "set_tol_da")
        self.n = len(l1)
        d = self.dev
        self.h2d = 0

        def up(a):
            t = torch.from_numpy(np.array(a, copy=True)).to(d)
            self.h2d += t.numel() * t.element_size()
            return t
        self.mass32_np = l1.mass32
        self.seq_off = up(l1.seq_off.astype(np.int64))
        self.length = up(l1.length.astype(np.uint8))
        self.mask = up(l1.mask.view(np.int64))
        self.mass32 = up(l1.mass32.astype(np.float32))
        self.residues = up(l1.residues.astype(np.uint8))
        self.partner = up(l1.partner.astype(np.int64))
        self.missed = up(np.asarray(l1.missed).astype(np.uint8))
        self.n_var = up(np.asarray(l1.n_var).astype(np.uint8))
        self.pf_id = up(np.asarray(l1.pf_id).astype(np.uint64).view(np.int64))
        if self.n >= 2 ** ROW_BITS:
            raise ValueError("index rows must be < 2^28")
        # reference layout constants (used by the compatible entry points)
        self.inv_logw = 1.0 / math.log1p(params.bin_ppm * 1e-6)
        self.n_bins = int(math.floor(math.log(params.fragment_max_mz / params.fragment_min_mz) * self.inv_logw)) + 2
        self.n_chunks = (self.n + params.chunk_size - 1) // params.chunk_size
        self._slices = None
        self.tilings = {}
        with torch.cuda.device(d):
            self._build_tiles()
            for _, rows, _ in getattr(params, "k1_shapes", ()):   # the other tilings K1's shapes name
                self.tiling(int(rows))
        torch.cuda.synchronize(d)
        self.build_s = time.perf_counter() - t0
        self.device_bytes = sum(t.numel() * t.element_size() for t in
                                [self.seq_off, self.length, self.mask, self.mass32, self.residues, self.partner,
                                 self.missed, self.n_var, self.pf_id]) + \
            sum(sum(x.numel() * x.element_size() for x in tl["tensors"]) for tl in self.tilings.values())

    def table_ptrs(self):
        return (K.ptr(self.seq_off), K.ptr(self.length), K.ptr(self.mask), K.ptr(self.mass32), K.ptr(self.residues))

    def window_bound(self, ppm_lo: float, ppm_hi: float) -> int:
        """Most index rows one precursor window [M(1 + lo/1e6), M(1 + hi/1e6)] can hold, for any M: the largest
        number of rows within a relative mass width of (hi - lo)/1e6 (with a margin for the f32 rounding of the
        window edges).  Sizes the K1 buffers without reading the exact totals back from the device."""
        key = (float(ppm_lo), float(ppm_hi))
        cache = self.__dict__.setdefault("_window_bound", {})
        if key not in cache:
            m = np.asarray(self.mass32_np, np.float64)
            w = max(0.0, (ppm_hi - ppm_lo) * 1e-6) * 1.001 + 1e-6
            if len(m):
                j = np.searchsorted(m, m * (1.0 + w), side="right")
                cache[key] = int((j - np.arange(len(m))).max()) + 2
            else:
                cache[key] = 0
        return cache[key]

    def tiling(self, tile_rows: int) -> dict:
        """The tiled fragment index with ``tile_rows`` rows per tile ({"tix": vk_tindex, "tensors": [...]}), built
        on first use (outside any stream capture).  The search's own tiling is ``p.tile_rows``."""
        if tile_rows not in self.tilings:
            with torch.cuda.device(self.dev):
                self._build_tiles(tile_rows)
        return self.tilings[tile_rows]

    def _build_tiles(self, tile_rows: int | None = None):
        L = K.lib()
        main = tile_rows is None or tile_rows == self.p.tile_rows
        p = self.p if main else _replace(self.p, tile_rows=int(tile_rows), cbin_bits=0)
        ix = K.TIndex()
        K.check(L.vk_tindex_layout(self.n, p.tile_rows, p.fragment_min_mz, p.fragment_max_mz, p.min_ion_index,
                                   cbin_bits(p), C.byref(ix)), "tindex_layout")
        d = self.dev
        nt = ix.n_tiles
        tile_count = torch.empty(max(nt, 1), dtype=torch.int64, device=d)
        K.check(L.vk_tindex_count(C.byref(ix), C.byref(self.fp), *self.table_ptrs(), K.ptr(tile_count), K.stream()),
                "tindex_count")
        tile_off = _scan(tile_count[:nt])
        stats = torch.stack([tile_count[:nt].max() if nt else torch.zeros((), dtype=torch.int64, device=d),
                             tile_off[-1]]).cpu().tolist()
        ix.max_tile_postings = int(stats[0])
        ix.n_postings = int(stats[1])
        stride = ((1 << ix.cbin_bits) + 1 + 7) & ~7
        postings = torch.empty(max(ix.n_postings, 4), dtype=torch.int32, device=d)
        cbin_off = torch.empty(max(nt * stride, 8), dtype=torch.int16, device=d)
        ix.tile_off = K.ptr(tile_off)
        K.check(L.vk_tindex_emit(C.byref(ix), C.byref(self.fp), *self.table_ptrs(), K.ptr(postings),
                                 K.ptr(cbin_off), K.stream()), "tindex_emit")
        ix.cbin_off = K.ptr(cbin_off)
        ix.postings = K.ptr(postings)
        bitmap = torch.empty(max(int(L.vk_tindex_bitmap_bytes(C.byref(ix))) // 4, 4), dtype=torch.int32, device=d)
        K.check(L.vk_tindex_bitmap(C.byref(ix), K.ptr(bitmap), K.stream()), "tindex_bitmap")
        ix.bitmap = K.ptr(bitmap)
        self.tilings[p.tile_rows] = {"tix": ix, "tensors": [tile_off, cbin_off, postings, bitmap]}
        if main:
            self.tile_off, self.cbin_off, self.postings, self.bitmap = tile_off, cbin_off, postings, bitmap
            self.tix = ix
            self.n_postings = ix.n_postings

    # ------------------------------------------------------------------ reference-layout CSR (compatible vk_k1)
    @property
    def slices(self) -> list[Slice]:
        if self._slices is None:
            with torch.cuda.device(self.dev):
                self._slices = self._build_compat_slices()
        return self._slices

    def _build_compat_slices(self):
        """The reference's (chunk, log-ppm bin) CSR (engine.py:101-148), built with the compatible kernels."""
        L = K.lib()
        p, d = self.p, self.dev
        Cs = p.chunk_size
        cnt = torch.empty(self.n, dtype=torch.int32, device=d)
        K.check(L.vk_frag_count(self.n, *self.table_ptrs(), p.min_ion_index, p.fragment_min_mz, p.fragment_max_mz,
                                K.ptr(cnt), K.stream()), "frag_count")
        per_chunk = torch.zeros(self.n_chunks, dtype=torch.int64, device=d)
        per_chunk.index_add_(0, torch.arange(self.n, device=d) // Cs, cnt.to(torch.int64))
        pcs = per_chunk.cpu().numpy()
        bounds, acc, c0 = [], 0, 0
        for c, v in enumerate(pcs):
            if acc + v > p.max_slice_entries and c > c0:
                bounds.append((c0, c))
                c0, acc = c, 0
            acc += int(v)
        bounds.append((c0, self.n_chunks))
        out = []
        for c0, c1 in bounds:
            r0, r1 = c0 * Cs, min(c1 * Cs, self.n)
            off = torch.zeros(r1 - r0 + 1, dtype=torch.int64, device=d)
            torch.cumsum(cnt[r0:r1].to(torch.int64), 0, out=off[1:])
            keys = torch.empty(int(off[-1]), dtype=torch.int64, device=d)
            K.check(L.vk_frag_emit(r1 - r0, K.ptr(self.seq_off[r0:r1]), K.ptr(self.length[r0:r1]),
                                   K.ptr(self.mask[r0:r1]), K.ptr(self.mass32[r0:r1]), K.ptr(self.residues),
                                   p.min_ion_index, p.fragment_min_mz, p.fragment_max_mz, self.inv_logw, Cs, r0,
                                   K.ptr(off), K.ptr(keys), K.stream()), "frag_emit")
            keys = torch.sort(keys).values
            entries = (keys & 0xFFFFFFFF).to(torch.int64)
            entries = torch.where(entries >= 2 ** 31, entries - 2 ** 32, entries).to(torch.int32)
            lin = ((keys >> 50) - c0) * self.n_bins + ((keys >> 32) & 0x3FFFF)
            nb = (c1 - c0) * self.n_bins
            offs = torch.zeros(nb + 1, dtype=torch.int64, device=d)
            torch.cumsum(torch.bincount(lin, minlength=nb), 0, out=offs[1:])
            offs = torch.where(offs >= 2 ** 31, offs - 2 ** 32, offs).to(torch.int32)
            out.append(Slice(c0, c1, offs, entries))
        return out


# ------------------------------------------------------------------------------------------------ spectra
_STORE_COLUMNS = ("ms_level", "scan", "index", "rt_min", "precursor_mz", "precursor_charge", "mz", "intensity")


def load_store(path: str, pinned: bool = False) -> Spectra:
    """The MS2 spectra of one run from its spectral store (reference engine.py:157-168): an Arrow IPC file with one
    row per spectrum (scalar columns and list<float32> ``mz`` / ``intensity``), the run's metadata as JSON under the
    schema's ``vulcan`` key and in a ``.json`` sidecar (reference ``vulcan/io/store.py``).  The file is
    memory-mapped and only the columns the search reads are touched; the MS2 rows' peaks are gathered from the
    Arrow value buffers straight into one flat array each -- in pinned host memory with ``pinned``, so that
    ``Searcher`` copies them to the device without staging.  Unknown charges (null) become 0, a missing precursor
    m/z NaN; the run name is the metadata's ``run_name`` (else the path)."""
    import json
    import os
    reader = pa.ipc.open_file(pa.memory_map(path, "r"))
    meta = {}
    md = reader.schema.metadata or {}
    if b"vulcan" in md:
        meta.update(json.loads(md[b"vulcan"]))
    if os.path.exists(path + ".json"):
        with open(path + ".json") as fh:
            meta.update(json.load(fh))
    batches = [reader.get_batch(i).select(list(_STORE_COLUMNS)) for i in range(reader.num_record_batches)]
    # per batch: the MS2 rows and their peak ranges in the batch's list value buffers
    sel, plans = [], []
    n_spec = n_peaks = 0
    for b in batches:
        ms2 = np.flatnonzero(b.column("ms_level").to_numpy(zero_copy_only=False) == 2)
        mzc, itc = b.column("mz"), b.column("intensity")
        off = mzc.offsets.to_numpy().astype(np.int64)
        if not np.array_equal(off, itc.offsets.to_numpy()):
            raise ValueError(f"{path}: mz and intensity lists differ in length")
        lens = off[1:][ms2] - off[:-1][ms2]
        sel.append(ms2)
        plans.append((off[:-1][ms2], lens, mzc.values, itc.values))
        n_spec += len(ms2)
        n_peaks += int(lens.sum())
    alloc = _pinned_like if pinned else (lambda a: np.empty_like(a))
    mz = alloc(np.empty(n_peaks, np.float32))
    inten = alloc(np.empty(n_peaks, np.float32))
    offsets = alloc(np.empty(n_spec + 1, np.int64))
    offsets[0] = 0
    pos = spec = 0
    for (starts, lens, mzv, itv) in plans:
        tot = int(lens.sum())
        np.cumsum(lens, out=offsets[spec + 1:spec + 1 + len(lens)])
        offsets[spec + 1:spec + 1 + len(lens)] += pos
        if tot:
            src = np.repeat(starts - (offsets[spec:spec + len(lens)] - pos), lens) + np.arange(tot, dtype=np.int64)
            np.take(mzv.to_numpy(zero_copy_only=False), src, out=mz[pos:pos + tot])
            np.take(itv.to_numpy(zero_copy_only=False), src, out=inten[pos:pos + tot])
        pos += tot
        spec += len(lens)

    def col(name, dt=None):
        parts = [b.column(name).to_numpy(zero_copy_only=False)[m] for b, m in zip(batches, sel)]
        v = np.concatenate(parts) if parts else np.zeros(0, dt or np.float64)
        return v if dt is None else np.asarray(v, dt)
    pmz = alloc(np.empty(n_spec, np.float64))
    pmz[:] = col("precursor_mz", np.float64)
    charge = alloc(np.empty(n_spec, np.int8))
    charge[:] = np.nan_to_num(col("precursor_charge", np.float64), nan=0).astype(np.int8)
    return Spectra(meta.get("run_name", path), col("scan", np.uint32), col("index", np.uint32),
                   col("rt_min", np.float64), pmz, charge, mz, inten, offsets)


class DeviceRun:
    """One run's raw spectra on the device (the inputs of K0 and of the hypotheses)."""

    def __init__(self, sp: Spectra, dev, stats: Stats | None = None, pinned: bool = True):
        def up(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            t = torch.from_numpy(a)
            if pinned and dev.type == "cuda":
                t = t.pin_memory()
            g = t.to(dev, non_blocking=True)
            if stats is not None:
                stats.h2d_bytes += g.numel() * g.element_size()
            return g
        self.n = len(sp)
        self.mz = up(sp.mz, np.float32)
        self.intensity = up(sp.intensity, np.float32)
        self.offsets = up(sp.offsets, np.int64)
        self.precursor_mz = up(sp.precursor_mz, np.float64)
        self.charge = up(sp.charge, np.int8)
        lens = np.diff(np.asarray(sp.offsets, np.int64))
        self.max_raw = int(lens.max()) if len(lens) else 0
        self.n_raw = int(np.asarray(sp.offsets)[-1]) if len(sp.offsets) else 0
        self.charge_np = np.asarray(sp.charge)


def _k0_device(run: DeviceRun, p: SearchParams, dev):
    L = K.lib()
    n = run.n
    kept = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    easy = torch.empty(max(n, 1), dtype=torch.uint8, device=dev)
    hard = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    n_hard = torch.empty(1, dtype=torch.int32, device=dev)
    window = p.peak_mode != "global"   # the reference groups by window for any other value (engine.py:182)
    if window:
        K.check(L.vk_k0w_count(n, K.ptr(run.offsets), K.ptr(run.mz), K.ptr(run.intensity), p.fragment_min_mz,
                               p.fragment_max_mz, p.window_th, p.window_k, K.ptr(kept), K.ptr(easy), K.ptr(hard),
                               K.ptr(n_hard), K.stream()), "k0w_count")
    else:
        K.check(L.vk_k0_count(n, K.ptr(run.offsets), K.ptr(run.mz), K.ptr(run.intensity), p.fragment_min_mz,
                              p.fragment_max_mz, p.max_peaks, K.ptr(kept), K.ptr(easy), K.ptr(hard), K.ptr(n_hard),
                              K.stream()), "k0_count")
    off = _scan(kept[:n])
    cap = max(run.n_raw, 1)
    mass = torch.empty(cap, dtype=torch.float32, device=dev)
    inten = torch.empty(cap, dtype=torch.float32, device=dev)
    tic = torch.empty(max(n, 1), dtype=torch.float32, device=dev)
    valid = torch.empty(max(n, 1), dtype=torch.uint8, device=dev)
    if window:
        K.check(L.vk_k0w_fill(n, K.ptr(run.offsets), K.ptr(run.mz), K.ptr(run.intensity), p.fragment_min_mz,
                              p.fragment_max_mz, p.window_th, p.window_k, p.min_peaks, K.ptr(off), K.ptr(mass),
                              K.ptr(inten), K.ptr(tic), K.ptr(valid), run.max_raw, K.ptr(easy), K.ptr(hard),
                              K.ptr(n_hard), K.stream()), "k0w_fill")
    else:
        # the few spectra a CTA selects or sorts (more than max_peaks in range, or out of order) on the side stream,
        # beside the warp-per-spectrum copy of the others: disjoint outputs
        args = (n, K.ptr(run.offsets), K.ptr(run.mz), K.ptr(run.intensity), p.fragment_min_mz, p.fragment_max_mz,
                p.max_peaks, p.min_peaks, K.ptr(off), K.ptr(mass), K.ptr(inten), K.ptr(tic), K.ptr(valid),
                run.max_raw, K.ptr(easy), K.ptr(hard), K.ptr(n_hard))
        hard_fill = _Forked(dev, lambda: K.check(L.vk_k0_fill_hard(*args, K.stream()), "k0_fill_hard"))
        K.check(L.vk_k0_fill_easy(*args, K.stream()), "k0_fill_easy")
        hard_fill.get()
    return {"off": off, "mass": mass, "int": inten, "tic": tic[:n], "valid_d": valid[:n]}


def k0_preprocess(sp: Spectra, p: SearchParams, dev, stats: Stats):
    """K0 on the GPU (reference engine.py:171-210): device peaks + host validity mask."""
    run = DeviceRun(sp, torch.device(dev), stats)
    pk = _k0_device(run, p, torch.device(dev))
    n_kept = int(pk["off"][-1])
    pk["mass"] = pk["mass"][:n_kept]
    pk["int"] = pk["int"][:n_kept]
    pk["valid"] = pk["valid_d"].bool().cpu().numpy()
    return pk


def _hyp_device(run: DeviceRun, peaks, gi: GpuIndex, p: SearchParams):
    """Hypotheses on the device; capacity = the host-known upper bound (charge known or the charge range)."""
    L = K.lib()
    dev = gi.dev
    n = run.n
    z0, z1 = p.precursor_charge
    i0, i1 = p.isotope_errors
    n_iso = i1 - i0 + 1
    n_max = int(np.where(run.charge_np > 0, 1, z1 - z0 + 1).sum()) * n_iso
    # a run in a captured slot carries the slot's hypothesis capacity (>= what any run of that shape needs)
    n_max = max(n_max, int(getattr(run, "n_hyp_cap", 0) or 0))
    cnt = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    K.check(L.vk_hyp_count(n, K.ptr(peaks["valid_d"]), K.ptr(run.precursor_mz), K.ptr(run.charge), z0, z1, i0, i1,
                           K.ptr(cnt), K.stream()), "hyp_count")
    off = _scan(cnt[:n])
    cap = max(n_max, 1)
    # one zeroed allocation for all hypothesis columns (slots past the spectra's hypotheses stay empty windows)
    cols = (("lo", torch.int64), ("hi", torch.int64), ("spec", torch.int32), ("pm", torch.float32),
            ("M", torch.float32), ("z", torch.int8), ("iso", torch.int8), ("maxfz", torch.int8))
    sizes = [(cap * torch.empty(0, dtype=dt).element_size() + 15) & ~15 for _, dt in cols]
    buf = torch.zeros(sum(sizes), dtype=torch.uint8, device=dev)
    h, o = {}, 0
    for (name, dt), sz in zip(cols, sizes):
        h[name] = buf[o:o + sz].view(dt)[:cap]
        o += sz
    mfc = p.max_fragment_charge or 0
    K.check(L.vk_hyp_fill(n, K.ptr(peaks["valid_d"]), K.ptr(run.precursor_mz), K.ptr(run.charge), z0, z1, i0, i1,
                          float(p.precursor_ppm[0]), float(p.precursor_ppm[1]), int(mfc), K.ptr(gi.mass32), gi.n,
                          K.ptr(off), K.ptr(h["spec"]), K.ptr(h["z"]), K.ptr(h["iso"]), K.ptr(h["pm"]), K.ptr(h["M"]),
                          K.ptr(h["lo"]), K.ptr(h["hi"]), K.ptr(h["maxfz"]), K.stream()), "hyp_fill")
    h["spec_off"] = off
    h["n_max"] = n_max
    return h


def work_items(hyp, p: SearchParams):
    """Reference work items (engine.py:213-229) for the compatible ``vk_k1``: tile-aligned pieces of each
    window that never cross a chunk boundary."""
    lo, hi = np.asarray(hyp["lo"]), np.asarray(hyp["hi"])
    T = p.tile
    nz = hi > lo
    h = np.nonzero(nz)[0]
    t0 = lo[h] // T
    t1 = (hi[h] - 1) // T
    nt = (t1 - t0 + 1)
    hh = np.repeat(h, nt)
    tt = np.repeat(t0, nt) + (np.arange(nt.sum()) - np.repeat(np.cumsum(nt) - nt, nt))
    a = np.maximum(lo[hh], tt * T)
    b = np.minimum(hi[hh], (tt + 1) * T)
    chunk = (tt * T) // p.chunk_size
    base = chunk * p.chunk_size
    return {"hyp": hh.astype(np.int32), "chunk": chunk.astype(np.int32), "lo": (a - base).astype(np.int32),
            "hi": (b - base).astype(np.int32), "n_window": int((hi - lo)[nz].sum())}


class Timer:
    """CUDA-event + wall time of a phase, recorded on the current stream."""

    def __init__(self, stats: Stats, name: str):
        self.stats, self.name = stats, name

    def __enter__(self):
        self.e0 = torch.cuda.Event(enable_timing=True)
        self.e1 = torch.cuda.Event(enable_timing=True)
        self.e0.record()
        self.t0 = time.perf_counter()
        return self

    def __exit__(self, *a):
        self.e1.record()
        self.e1.synchronize()
        self.stats.gpu_ms[self.name] = self.stats.gpu_ms.get(self.name, 0.0) + self.e0.elapsed_time(self.e1)
        self.stats.wall_s[self.name] = self.stats.wall_s.get(self.name, 0.0) + time.perf_counter() - self.t0


def _as_dev(hyp, dev):
    out = {}
    for k in ("spec", "z", "iso", "pm", "M", "lo", "hi", "maxfz"):
        v = hyp[k]
        out[k] = v if isinstance(v, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(v)).to(dev)
    return out


def key_charges(p: SearchParams) -> int:
    """Fragment charges whose window keys are precomputed per pass: all of them when max_fragment_charge bounds
    them, else 1 and 2 (K1 computes higher charges itself)."""
    mfc = p.max_fragment_charge or 0
    return mfc if mfc > 0 else 2


def peak_keys(gi: GpuIndex, peaks, p: SearchParams, tix=None, forked: bool = False):
    """Window keys and filter words of every kept peak (vk_k1_peak_keys): (keys, filt, n_kz, kstride), computed once
    per pass for all the (tile, hypothesis) items of K1; the filter words are bitmap positions of the tiling
    ``tix`` (default: the index's own).  ``forked``: launched on the side stream (they need only K0's peaks, so they
    overlap the hypotheses and the K1 planning) and returned as a ``_Forked`` whose ``get()`` joins."""
    n_kz = key_charges(p)
    kstride = int(peaks["mass"].numel())
    keys = torch.empty(max(n_kz * kstride * 2, 2), dtype=torch.int32, device=gi.dev)
    filt = torch.empty(max(n_kz * kstride, 1), dtype=torch.int32, device=gi.dev)
    last = peaks["off"][-1:]

    def launch():
        K.check(K.lib().vk_k1_peak_keys(C.byref(tix or gi.tix), C.byref(gi.fp), float(p.fragment_ppm[0]),
                                        float(p.fragment_ppm[1]), K.ptr(last), K.ptr(peaks["mass"]), n_kz,
                                        kstride, K.ptr(keys), K.ptr(filt), K.stream()), "k1_peak_keys")
        return keys, filt, n_kz, kstride
    return _Forked(gi.dev, launch) if forked else launch()


def early_peak_keys(gi: GpuIndex, peaks, p: SearchParams):
    """The window keys of a pass with one K1 shape, forked right after K0 (None with per-bucket shapes, whose
    tilings each get their own keys when planned)."""
    return peak_keys(gi, peaks, p, forked=True) if len(k1_shape_list(gi, p)) == 1 else None


def k1_shape_list(gi: GpuIndex, p: SearchParams) -> list:
    """K1's launch shapes: [(tiling, k1 warps, lower, upper)] -- the spectra whose kept peaks n satisfy
    lower < n <= upper take that shape (``p.k1_shapes``; one shape for all without it)."""
    out, lower = [], 0
    for upper, rows, warps in sorted(tuple(x) for x in getattr(p, "k1_shapes", ())):
        out.append((gi.tiling(int(rows)), int(warps), lower, int(upper)))
        lower = int(upper)
    out.append((gi.tiling(p.tile_rows), int(p.k1_warps), lower, 1 << 62))
    return out


def _k1_passes(gi: GpuIndex, dh, peaks, p: SearchParams, n_hyp: int, caps: tuple | None = None, keys=None):
    """The K1 launches of a pass: per shape (``k1_shape_list``) its work items -- the hypotheses of the spectra in
    the shape's peak-count bucket, planned on the shape's tiling -- with the window keys of that tiling.  Yields
    (tix, warps, plan, keys, filt, n_kz, kstride); every plan shares one ``win_off`` (the windows of all the
    hypotheses) and one ``status``.  ``keys``: the single shape's keys forked earlier (``early_peak_keys``)."""
    shapes = k1_shape_list(gi, p)
    if len(shapes) == 1:
        tl, warps, _, _ = shapes[0]
        pl = _k1_plan(gi, dh, p, n_hyp, caps, tiling=tl)
        kt = keys.get() if keys is not None else peak_keys(gi, peaks, p, tl["tix"])
        yield (tl["tix"], warps, pl) + kt
        return
    if keys is not None:
        keys.get()
    lo, hi = dh["lo"][:n_hyp], dh["hi"][:n_hyp]
    win_off = _scan((hi - lo).clamp(min=0))
    status = torch.zeros(1, dtype=torch.int32, device=gi.dev)
    npk = (peaks["off"][1:] - peaks["off"][:-1])[dh["spec"][:n_hyp].long()]
    keys_of = {}
    for tl, warps, lower, upper in shapes:
        mine = (npk > lower) & (npk <= upper)
        pl = _k1_plan(gi, dh, p, n_hyp, caps, tiling=tl, hi=torch.where(mine, hi, lo), win_off=win_off,
                      status=status)
        key = id(tl)
        if key not in keys_of:
            keys_of[key] = peak_keys(gi, peaks, p, tl["tix"])
        yield (tl["tix"], warps, pl) + keys_of[key]


def _k1_dense(gi: GpuIndex, dh, peaks, p: SearchParams, n_hyp: int, stats: Stats | None = None,
              isum: bool = False, keys=None):
    """Tiled K1: dense counts of every window row.  Returns (win_off, cnt, status), plus the summed matched
    intensity of every window row (u32, 2^24 = the spectrum's TIC) when ``isum``.  The buffers are sized by the
    index's window bound (``GpuIndex.window_bound``), so nothing is read back from the device: cnt / isum hold
    more entries than the win_off[-1] window rows, and ``status`` gets VK_STATUS_OVERFLOW should a bound not hold.
    With ``p.k1_shapes`` each peak-count bucket's hypotheses run with their own tiling and warps (same counts)."""
    L = K.lib()
    dev = gi.dev
    cnt = isw = pl = None
    for tix, warps, pl, kk, filt, n_kz, kstride in _k1_passes(gi, dh, peaks, p, n_hyp, keys=keys):
        if cnt is None:
            cnt = torch.empty(pl["cnt_cap"], dtype=torch.int32, device=dev)
            isw = torch.empty(pl["cnt_cap"], dtype=torch.int32, device=dev) if isum else None
        K.check(L.vk_k1_tiles(C.byref(tix), C.byref(gi.fp), float(p.fragment_ppm[0]), float(p.fragment_ppm[1]),
                              warps, K.ptr(pl["item_off"]), K.ptr(pl["item_hyp"]), n_hyp, pl["item_cap"],
                              K.ptr(dh["spec"]), K.ptr(dh["maxfz"]), K.ptr(dh["lo"]), K.ptr(dh["hi"]),
                              K.ptr(pl["win_off"]), pl["cnt_cap"], K.ptr(peaks["off"]), K.ptr(peaks["mass"]),
                              K.ptr(cnt), K.ptr(pl["status"]), K.ptr(peaks["int"]) if isum else None,
                              K.ptr(peaks["tic"]) if isum else None, K.ptr(isw) if isum else None, K.ptr(kk),
                              K.ptr(filt), n_kz, kstride, K.stream()), "k1_tiles")
    if isum:
        return pl["win_off"], cnt, pl["status"], isw
    return pl["win_off"], cnt, pl["status"]


def _k1_plan(gi: GpuIndex, dh, p: SearchParams, n_hyp: int, caps: tuple | None = None, tiling: dict | None = None,
             hi=None, win_off=None, status=None) -> dict:
    """The (tile, hypothesis) work items of K1 grouped by tile, and the window offsets, in buffers sized by the
    index's window bound, or by ``caps`` = (items, window rows) (nothing read back).  ``tiling``: plan on that
    tiling of the index (default its own); ``hi``: the window ends to plan items for (default the hypotheses' own;
    an empty window gets no item), with ``win_off`` of the full windows given.  ``status`` (device i32) is zeroed
    here unless given, and collects the pass's overflow / timeout bits."""
    L = K.lib()
    dev = gi.dev
    ix = tiling["tix"] if tiling is not None else gi.tix
    nt = ix.n_tiles
    if caps is None:
        max_win = gi.window_bound(*p.precursor_ppm)
        T = 1 << ix.tile_shift
        item_cap = max(1, n_hyp * ((max_win + T - 1) // T + 1))
        cnt_cap = max(1, n_hyp * max_win)
    else:
        item_cap, cnt_cap = max(1, int(caps[0])), max(1, int(caps[1]))
    h_hi = dh["hi"] if hi is None else hi
    tile_items = torch.empty(max(nt, 1), dtype=torch.int64, device=dev)
    win_len = torch.empty(max(n_hyp, 1), dtype=torch.int64, device=dev)
    K.check(L.vk_k1_plan_count(C.byref(ix), n_hyp, K.ptr(dh["lo"]), K.ptr(h_hi), K.ptr(tile_items),
                               K.ptr(win_len), K.stream()), "k1_plan_count")
    item_off = _scan(tile_items[:nt])
    if win_off is None:
        win_off = _scan(win_len[:n_hyp])
    if status is None:
        status = torch.zeros(1, dtype=torch.int32, device=dev)
    cursor = torch.empty(max(nt, 1), dtype=torch.int64, device=dev)
    item_hyp = torch.empty(item_cap, dtype=torch.int32, device=dev)
    K.check(L.vk_k1_plan_fill(C.byref(ix), n_hyp, K.ptr(dh["lo"]), K.ptr(h_hi), K.ptr(item_off),
                              K.ptr(cursor), K.ptr(item_hyp), item_cap, K.ptr(status), K.stream()), "k1_plan_fill")
    return {"item_off": item_off, "item_hyp": item_hyp, "item_cap": item_cap, "win_off": win_off,
            "cnt_cap": cnt_cap, "status": status}


def _k1_hits(gi: GpuIndex, dh, peaks, p: SearchParams, n_hyp: int, thr: int, isum: bool = True,
             h_thr: torch.Tensor | None = None, caps: tuple | None = None, keys=None):
    """K1 in hit-list form (``vk_k1_hits``): per hypothesis the rows with count >= thr (``h_thr``: a device i32
    threshold per hypothesis instead) -- count << 32 | row, and the summed matched intensity -- in its window's
    region, their number, and the per-hypothesis scored / matched totals.  No dense per-row output.  ``caps``:
    (item capacity, window-row capacity) when the caller knows them (else the index's window bound)."""
    L = K.lib()
    dev = gi.dev
    nh = max(n_hyp, 1)
    # hyp_scored (u32), hyp_matched (u64), hyp_shift (i8): one zeroed allocation
    z = torch.zeros(nh * 3, dtype=torch.int64, device=dev)
    hyp_scored = z[:nh].view(torch.int32)[:nh]
    hyp_matched = z[nh:2 * nh]
    hyp_shift = z[2 * nh:].view(torch.int8)[:nh]
    rc = hisum = pl = None
    for tix, warps, pl, kk, filt, n_kz, kstride in _k1_passes(gi, dh, peaks, p, n_hyp, caps, keys=keys):
        cap = pl["cnt_cap"]
        if rc is None:
            rc = torch.empty(cap, dtype=torch.int64, device=dev)
            seg_cnt = torch.empty(cap, dtype=torch.int32, device=dev)
            hisum = torch.empty(cap, dtype=torch.int32, device=dev) if isum else None
        K.check(L.vk_k1_hits(C.byref(tix), C.byref(gi.fp), float(p.fragment_ppm[0]), float(p.fragment_ppm[1]),
                             warps, K.ptr(pl["item_off"]), K.ptr(pl["item_hyp"]), n_hyp, pl["item_cap"],
                             K.ptr(dh["spec"]), K.ptr(dh["maxfz"]), K.ptr(dh["lo"]), K.ptr(dh["hi"]),
                             K.ptr(pl["win_off"]), cap, K.ptr(peaks["off"]), K.ptr(peaks["mass"]),
                             int(thr) if h_thr is None else 0, K.ptr(h_thr), K.ptr(rc),
                             K.ptr(hisum) if isum else None, K.ptr(seg_cnt), K.ptr(hyp_shift), K.ptr(hyp_scored),
                             K.ptr(hyp_matched),
                             K.ptr(pl["status"]), K.ptr(peaks["int"]) if isum else None,
                             K.ptr(peaks["tic"]) if isum else None, K.ptr(kk), K.ptr(filt), n_kz, kstride,
                             K.stream()), "k1_hits")
    return {"win_off": pl["win_off"], "status": pl["status"], "rc": rc, "isum": hisum, "seg_cnt": seg_cnt,
            "hyp_shift": hyp_shift,
            "hyp_scored": hyp_scored, "hyp_matched": hyp_matched}


def _shortlist_hits(gi: GpuIndex, p: SearchParams, n: int, dh, k1h: dict, topk: int, closure: bool = False,
                    features=None):
    """Top-k of every spectrum by K1 count among its hit lists (``vk_select_hits``), optionally with pair closure,
    compacted to spectrum-ordered candidate lists with their intensity sums (``c_isum``); the same candidates as
    ``_shortlist`` over the dense counts.  ``features`` = (index, mu, sd): the compaction also writes every hit's
    standardised BF16 features (``vk_compact_hits_features``, the rows ``vk_cand_features`` gives) as "feat".
    Returns the candidate dict and the per-hypothesis / per-spectrum K1 sums."""
    L = K.lib()
    dev = gi.dev
    cap = (2 if closure else 1) * topk
    s_hyp = torch.empty(max(n * cap, 1), dtype=torch.int64, device=dev)
    s_row = torch.empty_like(s_hyp)
    s_cnt = torch.empty_like(s_hyp)
    isum = k1h["isum"] is not None
    s_isum = torch.empty(max(n * cap, 1), dtype=torch.int32, device=dev) if isum else None
    n_cand = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    spec_scored = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    spec_matched = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    K.check(L.vk_select_hits(n, K.ptr(dh["spec_off"]), K.ptr(dh["lo"]), K.ptr(dh["hi"]), K.ptr(k1h["win_off"]),
                             K.ptr(k1h["hyp_shift"]), K.ptr(k1h["seg_cnt"]), K.ptr(k1h["rc"]),
                             K.ptr(k1h["isum"]) if isum else None,
                             K.ptr(k1h["hyp_scored"]),
                             K.ptr(k1h["hyp_matched"]), topk, int(closure), K.ptr(gi.partner), cap, K.ptr(s_hyp),
                             K.ptr(s_row), K.ptr(s_cnt),
                             K.ptr(s_isum) if isum else None, K.ptr(n_cand), K.ptr(spec_scored),
                             K.ptr(spec_matched), K.stream()), "select_hits")
    cand_off = _scan(n_cand[:n])
    c_hyp = torch.empty_like(s_hyp)
    c_row = torch.empty_like(s_hyp)
    c_cnt = torch.empty_like(s_hyp)
    c_row32 = torch.empty(max(n * cap, 1), dtype=torch.int32, device=dev)
    c_maxfz = torch.empty(max(n * cap, 1), dtype=torch.int8, device=dev)
    c_isum = torch.empty(max(n * cap, 1), dtype=torch.int32, device=dev) if isum else None
    feat = None
    if features is not None and isum:
        fi, mu, sd = features
        feat = torch.empty(max(n * cap, 1), 16, dtype=torch.bfloat16, device=dev)
        K.check(L.vk_compact_hits_features(n, cap, K.ptr(n_cand), K.ptr(cand_off), K.ptr(s_hyp), K.ptr(s_row),
                                           K.ptr(s_cnt), K.ptr(s_isum), K.ptr(dh["maxfz"]), K.ptr(c_hyp),
                                           K.ptr(c_row), K.ptr(c_cnt), K.ptr(c_row32), K.ptr(c_maxfz), K.ptr(c_isum),
                                           K.ptr(dh["M"]), K.ptr(dh["z"]), K.ptr(fi.mass32), K.ptr(fi.length),
                                           K.ptr(fi.missed), K.ptr(mu), K.ptr(sd), K.ptr(feat), K.stream()),
                "compact_hits_features")
    else:
        K.check(L.vk_compact_hits(n, cap, K.ptr(n_cand), K.ptr(cand_off), K.ptr(s_hyp), K.ptr(s_row), K.ptr(s_cnt),
                                  K.ptr(s_isum) if isum else None, K.ptr(dh["maxfz"]), K.ptr(c_hyp), K.ptr(c_row),
                                  K.ptr(c_cnt), K.ptr(c_row32), K.ptr(c_maxfz), K.ptr(c_isum) if isum else None,
                                  K.stream()), "compact_hits")
    cand = {"cand_off": cand_off, "c_hyp": c_hyp, "c_row": c_row, "c_cnt": c_cnt, "c_row32": c_row32,
            "c_maxfz": c_maxfz, "cap": cap, "n_cand": n_cand, "c_isum": c_isum}
    if feat is not None:
        cand["feat"] = feat
    sums = {"hyp_scored": k1h["hyp_scored"], "hyp_matched": k1h["hyp_matched"], "spec_scored": spec_scored,
            "spec_matched": spec_matched}
    return cand, sums


def check_status(status: torch.Tensor, what: str = "search"):
    """Raise on the device status bits of a pass (one host read)."""
    v = int(status.item())
    if v & 1:
        raise RuntimeError(f"{what}: a bounded device wait timed out (tile copy or tensor-core MMA)")
    if v & 2:
        raise RuntimeError(f"{what}: a device buffer bound was exceeded")
    if v:
        raise RuntimeError(f"{what}: device status {v}")


def run_k1(gi: GpuIndex, hyp, peaks, p: SearchParams, stats: Stats):
    """K1 (reference engine.py:250-281): returns (o_h, o_r, o_c, scored, matched, d_spec, d_maxfz) with the appended
    (hyp, row, count) entries sorted by (hyp, row)."""
    dev = gi.dev
    dh = _as_dev(hyp, dev)
    n_h = len(hyp["spec"])
    win_off, cnt, status = _k1_dense(gi, dh, peaks, p, n_h, stats)
    check_status(status, "k1")
    cnt = cnt[:int(win_off[-1])]
    win_len = (dh["hi"] - dh["lo"]).clamp(min=0)
    hh = torch.repeat_interleave(torch.arange(n_h, device=dev), win_len)
    rr = dh["lo"][hh] + (torch.arange(len(hh), device=dev) - win_off[:-1][hh])
    keep = cnt >= p.k1_threshold
    scored = torch.zeros(n_h, dtype=torch.int32, device=dev).index_add_(0, hh, (cnt > 0).to(torch.int32))
    matched = torch.zeros(n_h, dtype=torch.int64, device=dev).index_add_(0, hh, cnt.to(torch.int64))
    n = int(keep.sum())
    stats.counts["k1_appended"] = stats.counts.get("k1_appended", 0) + n
    return (hh[keep].to(torch.int32), rr[keep].to(torch.int32), cnt[keep], scored, matched, dh["spec"], dh["maxfz"])


def select_topk(o_h, o_r, o_c, d_spec, gi: GpuIndex, p: SearchParams):
    """Top-K per spectrum then pair closure from appended lists (reference engine.py:284-312), tie (count, row)
    broken by the lower hypothesis.  ``search`` runs the same selection in the ``vk_select_topk`` kernel."""
    dev = gi.dev
    spec = d_spec[o_h.long()].long()
    key = (spec << 43) | ((32767 - o_c.long().clamp(max=32767)) << ROW_BITS) | ((2 ** ROW_BITS - 1) - o_r.long())
    o = torch.argsort(o_h.long(), stable=True)
    o = o[torch.argsort(key[o], stable=True)]
    ss = spec[o]
    first = torch.searchsorted(ss, ss, side="left")
    rank = torch.arange(len(ss), device=dev) - first
    sel = o[rank < p.topk]
    h, r, c = o_h[sel].long(), o_r[sel].long(), o_c[sel].long()
    if p.pair_closure:
        pr = gi.partner[r]
        h = torch.cat([h, h])
        r = torch.cat([r, pr])
        c = torch.cat([c, torch.full_like(c, -1)])
    sp = d_spec[h].long()
    k = (sp << ROW_BITS) | r
    uk, inv = torch.unique(k, sorted=True, return_inverse=True)
    hh = torch.full((len(uk),), 2 ** 62, dtype=torch.int64, device=dev).scatter_reduce_(0, inv, h, reduce="amin")
    cc = torch.full((len(uk),), -1, dtype=torch.int64, device=dev).scatter_reduce_(0, inv, c, reduce="amax")
    rr = uk & (2 ** ROW_BITS - 1)
    return hh, rr, cc


def _k2_outputs(n, dev):
    out = {"hyperscore": torch.empty(n, dtype=torch.float64, device=dev)}
    for k in ("summed_b", "summed_y", "ppm"):
        out[k] = torch.empty(n, dtype=torch.float32, device=dev)
    for k in ("matched_b", "matched_y", "longest_b", "longest_y"):
        out[k] = torch.empty(n, dtype=torch.int16, device=dev)
    return out


def _k2_ptrs(out):
    return [K.ptr(out[k]) for k in ("hyperscore", "summed_b", "summed_y", "ppm", "matched_b", "matched_y",
                                    "longest_b", "longest_y")]


def run_k2(gi: GpuIndex, h, r, d_spec, d_maxfz, peaks, p: SearchParams, shift: torch.Tensor | None = None):
    """K2 over candidates sorted by spectrum (reference engine.py:315-351), through the reference-compatible
    ``vk_k2`` / ``vk_k2_shift`` entry points.  Returns a dict of device tensors, one row per candidate."""
    L = K.lib()
    dev = gi.dev
    spec = d_spec[h].long()
    us, cnts = torch.unique_consecutive(spec, return_counts=True)
    off = torch.zeros(len(us) + 1, dtype=torch.int64, device=dev)
    torch.cumsum(cnts, 0, out=off[1:])
    n = len(r)
    row = r.to(torch.int32).contiguous()
    mfz = d_maxfz[h].contiguous()
    out = _k2_outputs(n, dev)
    sid = us.to(torch.int32).contiguous()
    args = [len(us), K.ptr(off), K.ptr(row), K.ptr(mfz), K.ptr(sid), K.ptr(peaks["off"]), K.ptr(peaks["mass"]),
            K.ptr(peaks["int"]), *gi.table_ptrs(), p.fragment_ppm[0], p.fragment_ppm[1]]
    if shift is None:
        K.check(L.vk_k2(*args, *_k2_ptrs(out), p.k2_threads, K.stream()), "k2")
    else:
        sh = shift.to(torch.float32).contiguous()
        K.check(L.vk_k2_shift(*args, K.ptr(sh), *_k2_ptrs(out), p.k2_threads, K.stream()), "k2_shift")
    out["spec"] = spec
    return out


def lnfact(n):
    n = np.asarray(n, np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        v = n * np.log(n) - n + 0.5 * np.log(n) + 0.5 * np.log(2 * np.pi * n)
    return np.where(n == 0, 1.0, v)


def _rank_device(n_spec, cand_off, rows, k2, p: SearchParams, report: int, dev, sparse: bool = False):
    """PSM ranking per spectrum (``vk_psm_rank``; ``vk_psm_rank_sparse``, a thread per spectrum, for the few
    candidates per spectrum the pruner leaves).  Same outputs."""
    L = K.lib()
    slots = max(n_spec * report, 1)
    psm_cand = torch.empty(slots, dtype=torch.int64, device=dev)
    psm_rank = torch.empty(slots, dtype=torch.int32, device=dev)
    dnext = torch.empty(slots, dtype=torch.float64, device=dev)
    dbest = torch.empty(slots, dtype=torch.float64, device=dev)
    n_psm = torch.empty(max(n_spec, 1), dtype=torch.int32, device=dev)
    fn = L.vk_psm_rank_sparse if sparse else L.vk_psm_rank
    K.check(fn(n_spec, K.ptr(cand_off), K.ptr(rows), K.ptr(k2["hyperscore"]), K.ptr(k2["matched_b"]),
               K.ptr(k2["matched_y"]), p.min_matched_peaks, report, K.ptr(psm_cand), K.ptr(psm_rank), K.ptr(dnext),
               K.ptr(dbest), K.ptr(n_psm), K.stream()), "psm_rank")
    return psm_cand[:n_spec * report], psm_rank[:n_spec * report], dnext[:n_spec * report], dbest[:n_spec * report]


def _psm_columns(sp: Spectra, l1, rec: dict, p: SearchParams) -> pa.Table:
    """Host part of the PSM table (reference engine.py:396-432) from the gathered per-PSM records."""
    s = rec["spec"]
    rows = rec["row"]
    mbk, myk = rec["matched_b"].astype(np.int64), rec["matched_y"].astype(np.int64)
    kk = mbk + myk
    sc, mt = rec["spec_scored"], rec["spec_matched"]
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        lam = mt / sc
        pois = lam ** kk * np.exp(-lam) / np.exp(lnfact(kk))
        pois = np.where(np.isinf(pois), 1e-325, pois)
        log_pois = np.log10(pois)
    z = rec["z"].astype(np.int64)
    iso = rec["iso"].astype(np.int64)
    pm = rec["pm"]
    calc = l1.mass32[rows]
    ie = (iso.astype(np.float32) * NEUTRON).astype(np.float32)
    dm = (np.abs(pm - calc - ie) * np.float32(2e6) / (pm - ie + calc)).astype(np.float32)
    plen = l1.length[rows].astype(np.int64)
    sbs = (rec["summed_b"] + rec["summed_y"]).astype(np.float32)
    cols = {
        "run": pa.repeat(pa.scalar(sp.run, pa.string()), len(s)),
        "spec_idx": s.astype(np.int64), "scan": sp.scan[s], "rt": sp.rt[s],
        "rank": rec["rank"].astype(np.int32), "pf_row": rows.astype(np.int64), "pf_id": l1.pf_id[rows],
        "charge": z.astype(np.int8), "isotope_error": iso.astype(np.int8),
        "expmass": pm.astype(np.float32), "calcmass": calc.astype(np.float32), "delta_mass_ppm": dm,
        "hyperscore": rec["hyperscore"], "delta_next": rec["dnext"], "delta_best": rec["dbest"],
        "matched_b": mbk.astype(np.int16), "matched_y": myk.astype(np.int16), "matched_peaks": kk.astype(np.int16),
        "summed_intensity": sbs,
        "matched_intensity_pct": (100.0 * sbs / rec["tic"]).astype(np.float32),
        "average_ppm": rec["ppm"], "longest_b": rec["longest_b"], "longest_y": rec["longest_y"],
        "longest_y_pct": (rec["longest_y"] / plen).astype(np.float32),
        "peptide_len": plen.astype(np.int16), "missed_cleavages": l1.missed[rows], "n_var": l1.n_var[rows],
        "k1_count": rec["k1"].astype(np.int32), "scored_candidates": sc.astype(np.int32), "poisson": log_pois,
    }
    return pa.table(cols)


def _gather_psms(psm_cand, psm_rank, dnext, dbest, c_hyp, c_row, c_cnt, k2, dh, spec_scored, spec_matched, tic,
                 report, stats: Stats | None = None):
    """Device gather of the reported PSMs, one D2H copy per column."""
    ok = psm_cand >= 0
    sel = psm_cand[ok]
    slot = torch.nonzero(ok).squeeze(1)
    s = slot // report
    hh = c_hyp[sel].long()
    cols = {"spec": s, "rank": psm_rank[ok], "dnext": dnext[ok], "dbest": dbest[ok], "row": c_row[sel],
            "hyp": hh, "k1": c_cnt[sel], "z": dh["z"][hh], "iso": dh["iso"][hh], "pm": dh["pm"][hh],
            "spec_scored": spec_scored[s], "spec_matched": spec_matched[s], "tic": tic[s]}
    for k in ("hyperscore", "summed_b", "summed_y", "ppm", "matched_b", "matched_y", "longest_b", "longest_y"):
        cols[k] = k2[k][sel]
    out = {}
    for k, v in cols.items():
        out[k] = v.cpu().numpy()
        if stats is not None:
            stats.d2h_bytes += v.numel() * v.element_size()
    return out


def psm_table(sp: Spectra, gi: GpuIndex, l1, hyp, h, r, k1c, k2, scored, matched, peaks, p: SearchParams,
              report: int | None = None) -> pa.Table:
    """Rank candidates per spectrum by hyperscore (label-blind), Sage-style features, top ``report``
    (reference engine.py:361-432).  h, r, k1c: candidates sorted by (spectrum, row)."""
    report = p.report_psms if report is None else report
    dev = gi.dev
    dh = _as_dev(hyp, dev)
    n_spec = len(sp)
    spec = dh["spec"][h].long()
    cand_off = torch.zeros(n_spec + 1, dtype=torch.int64, device=dev)
    torch.cumsum(torch.bincount(spec, minlength=n_spec), 0, out=cand_off[1:])
    rows = r.long().contiguous()
    psm = _rank_device(n_spec, cand_off, rows, k2, p, report, dev)
    hs_spec = dh["spec"].long()
    sc = torch.zeros(n_spec, dtype=torch.int64, device=dev).index_add_(0, hs_spec, scored.long())
    mt = torch.zeros(n_spec, dtype=torch.int64, device=dev).index_add_(0, hs_spec, matched.long())
    rec = _gather_psms(*psm, h.long(), rows, k1c.long(), k2, dh, sc, mt, peaks["tic"], report)
    return _psm_columns(sp, l1, rec, p)


def _shortlist(gi: GpuIndex, p: SearchParams, n: int, dh, win_off, cnt, topk: int, closure: bool,
               thr: int | None = None):
    """Top-k of every spectrum by K1 count among the rows with count >= thr (default ``p.k1_threshold``;
    ``vk_select_topk``), optionally with pair closure, compacted to spectrum-ordered candidate lists.  Returns the
    candidate dict and the per-hypothesis / per-spectrum K1 sums (which do not depend on thr)."""
    L = K.lib()
    dev = gi.dev
    n_h = dh["n_max"]
    cap = (2 if closure else 1) * topk
    s_hyp = torch.empty(max(n * cap, 1), dtype=torch.int64, device=dev)
    s_row = torch.empty_like(s_hyp)
    s_cnt = torch.empty_like(s_hyp)
    n_cand = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    hyp_scored = torch.empty(max(n_h, 1), dtype=torch.int32, device=dev)
    hyp_matched = torch.empty(max(n_h, 1), dtype=torch.int64, device=dev)
    spec_scored = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    spec_matched = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    K.check(L.vk_select_topk(n, K.ptr(dh["spec_off"]), K.ptr(dh["lo"]), K.ptr(dh["hi"]), K.ptr(win_off),
                             K.ptr(cnt), cnt.numel(), K.ptr(gi.partner), p.k1_threshold if thr is None else thr, topk,
                             int(closure), cap,
                             K.ptr(s_hyp), K.ptr(s_row), K.ptr(s_cnt), K.ptr(n_cand), K.ptr(hyp_scored),
                             K.ptr(hyp_matched), K.ptr(spec_scored), K.ptr(spec_matched), K.stream()),
            "select_topk")
    cand = _compact(n, cap, n_cand, s_hyp, s_row, s_cnt, dh, dev)
    sums = {"hyp_scored": hyp_scored, "hyp_matched": hyp_matched, "spec_scored": spec_scored,
            "spec_matched": spec_matched}
    return cand, sums


def _compact(n: int, cap: int, n_cand, s_hyp, s_row, s_cnt, dh, dev):
    """Per-spectrum candidate slots (``cap`` each) -> contiguous lists in spectrum order (``vk_compact_cands``)."""
    L = K.lib()
    cand_off = _scan(n_cand[:n])
    c_hyp = torch.empty_like(s_hyp)
    c_row = torch.empty_like(s_hyp)
    c_cnt = torch.empty_like(s_hyp)
    c_row32 = torch.empty(max(n * cap, 1), dtype=torch.int32, device=dev)
    c_maxfz = torch.empty(max(n * cap, 1), dtype=torch.int8, device=dev)
    K.check(L.vk_compact_cands(n, cap, K.ptr(n_cand), K.ptr(cand_off), K.ptr(s_hyp), K.ptr(s_row), K.ptr(s_cnt),
                               K.ptr(dh["maxfz"]), K.ptr(c_hyp), K.ptr(c_row), K.ptr(c_cnt), K.ptr(c_row32),
                               K.ptr(c_maxfz), K.stream()), "compact_cands")
    return {"cand_off": cand_off, "c_hyp": c_hyp, "c_row": c_row, "c_cnt": c_cnt, "c_row32": c_row32,
            "c_maxfz": c_maxfz, "cap": cap, "n_cand": n_cand}


def _k2_cands(gi: GpuIndex, p: SearchParams, n: int, cand, peaks, sparse: bool = False):
    """K2 over compacted candidate lists; one output row per candidate.  Dense lists (the exhaustive path's top-k
    per spectrum): ``vk_k2_spectra``, a warp per spectrum over its staged peaks; sparse lists (a few candidates per
    spectrum after the pruner): ``vk_k2_cands``, a thread per candidate.  Same outputs."""
    L = K.lib()
    dev = gi.dev
    k2 = _k2_outputs(max(n * cand["cap"], 1), dev)
    common = (C.byref(gi.fp), n, K.ptr(cand["cand_off"]), K.ptr(cand["c_row32"]), K.ptr(cand["c_maxfz"]),
              K.ptr(peaks["off"]), K.ptr(peaks["mass"]), K.ptr(peaks["int"]), *gi.table_ptrs(),
              float(p.fragment_ppm[0]), float(p.fragment_ppm[1]))
    if sparse:
        K.check(L.vk_k2_cands(*common, *_k2_ptrs(k2), K.stream()), "k2_cands")
    else:
        K.check(L.vk_k2_spectra(*common, None, *_k2_ptrs(k2), K.stream()), "k2_spectra")
    return k2


def _search_device(run: DeviceRun, gi: GpuIndex, p: SearchParams, report: int, st: Stats, timers: bool = False):
    """The whole hot path on the device for one run whose raw spectra are already resident.  Returns the device
    PSM slots and the intermediates."""
    dev = gi.dev
    n = run.n

    def phase(name):
        return Timer(st, name) if timers else _NoTimer()
    with phase("k0"):
        peaks = _k0_device(run, p, dev)
    keys = early_peak_keys(gi, peaks, p)
    with phase("hyp"):
        dh = _hyp_device(run, peaks, gi, p)
    n_h = dh["n_max"]
    with phase("k1"):
        win_off, cnt, status = _k1_dense(gi, dh, peaks, p, n_h, st, keys=keys)
    with phase("topk"):
        cand, sums = _shortlist(gi, p, n, dh, win_off, cnt, p.topk, bool(p.pair_closure))
    with phase("k2"):
        k2 = _k2_cands(gi, p, n, cand, peaks)
    with phase("rank"):
        psm = _rank_device(n, cand["cand_off"], cand["c_row"], k2, p, report, dev)
    return {"peaks": peaks, "dh": dh, "win_off": win_off, "cnt": cnt, "status": status, **cand, "k2": k2,
            "psm": psm, **sums}


_K2_KEYS = (("hs", "hyperscore", torch.float64), ("sb", "summed_b", torch.float32),
            ("sy", "summed_y", torch.float32), ("ppm", "ppm", torch.float32), ("mb", "matched_b", torch.int16),
            ("my", "matched_y", torch.int16), ("lb", "longest_b", torch.int16), ("ly", "longest_y", torch.int16))
_FUSED_GRID = {}


def fused_grid(gi: GpuIndex, p: SearchParams) -> int:
    """Persistent grid of the fused search (resident CTAs per SM x SMs) for this index and parameters."""
    key = (id(gi), p.fused_warps, p.topk, p.pair_closure, p.fused_cnt_cap)
    if key not in _FUSED_GRID:
        g = C.c_int(0)
        with torch.cuda.device(gi.dev):
            K.check(K.lib().vk_search_fused_grid(C.byref(gi.tix), p.fused_warps, p.topk, int(p.pair_closure),
                                                 p.fused_cnt_cap, C.byref(g)), "fused_grid")
        _FUSED_GRID[key] = g.value
    return _FUSED_GRID[key]


def _fused_device(gi: GpuIndex, p: SearchParams, report: int, peaks, dh, n: int, cand: bool = False,
                  spec_ids: torch.Tensor | None = None, warps: int | None = None):
    """The fused persistent search (K1 -> top-K + closure -> K2 -> ranking) over spectra 0..n-1 (or spec_ids)."""
    L = K.lib()
    dev = gi.dev
    slots = max(n * report, 1)
    o = {"status": torch.empty(max(n, 1), dtype=torch.int32, device=dev),
         "n_psm": torch.empty(max(n, 1), dtype=torch.int32, device=dev),
         "spec_scored": torch.zeros(max(n, 1), dtype=torch.int64, device=dev),
         "spec_matched": torch.zeros(max(n, 1), dtype=torch.int64, device=dev),
         "work": torch.empty(1, dtype=torch.int32, device=dev)}
    psm = {"row": torch.full((slots,), -1, dtype=torch.int64, device=dev),
           "hyp": torch.empty(slots, dtype=torch.int64, device=dev),
           "k1": torch.empty(slots, dtype=torch.int64, device=dev),
           "rank": torch.empty(slots, dtype=torch.int32, device=dev),
           "dnext": torch.empty(slots, dtype=torch.float64, device=dev),
           "dbest": torch.empty(slots, dtype=torch.float64, device=dev)}
    for k, _, dt in _K2_KEYS:
        psm[k] = torch.empty(slots, dtype=dt, device=dev)
    po = K.PsmOut(*[K.ptr(psm[f]) for f, _ in K.PsmOut._fields_])
    co = None
    if cand:
        cap = (2 if p.pair_closure else 1) * p.topk
        cs = max(n * cap, 1)
        cd = {"n_cand": torch.full((max(n, 1),), -1, dtype=torch.int64, device=dev),
              "c_hyp": torch.empty(cs, dtype=torch.int64, device=dev),
              "c_row": torch.empty(cs, dtype=torch.int64, device=dev),
              "c_cnt": torch.empty(cs, dtype=torch.int64, device=dev)}
        for k, _, dt in _K2_KEYS:
            cd[k] = torch.empty(cs, dtype=dt, device=dev)
        co = K.CandOut(cap, *[K.ptr(cd[f]) for f, _ in K.CandOut._fields_[1:]])
        o["cand"] = cd
        o["cand_cap"] = cap
    n_h = dh["n_max"]
    o["hyp_scored"] = torch.empty(max(n_h, 1), dtype=torch.int32, device=dev)
    o["hyp_matched"] = torch.empty(max(n_h, 1), dtype=torch.int64, device=dev)
    fin = K.FusedIn(n, n if spec_ids is None else int(spec_ids.numel()), K.ptr(spec_ids), K.ptr(peaks["off"]),
                    K.ptr(peaks["mass"]), K.ptr(peaks["int"]), K.ptr(dh["spec_off"]), K.ptr(dh["lo"]),
                    K.ptr(dh["hi"]), K.ptr(dh["maxfz"]), K.ptr(gi.partner), *gi.table_ptrs(),
                    float(p.fragment_ppm[0]), float(p.fragment_ppm[1]), p.k1_threshold, p.topk, int(p.pair_closure),
                    p.min_matched_peaks, report)
    w = warps or p.fused_warps
    q = p if w == p.fused_warps else _replace(p, fused_warps=w)
    K.check(L.vk_search_fused(C.byref(gi.tix), C.byref(gi.fp), C.byref(fin), w, p.fused_cnt_cap, fused_grid(gi, q),
                              K.ptr(o["work"]), K.ptr(o["status"]), K.ptr(o["n_psm"]), K.ptr(o["spec_scored"]),
                              K.ptr(o["spec_matched"]), C.byref(po), C.byref(co) if co is not None else None,
                              K.ptr(o["hyp_scored"]), K.ptr(o["hyp_matched"]), K.stream()), "search_fused")
    o["psm"] = psm
    return o


def _replace(p: SearchParams, **kw) -> SearchParams:
    import dataclasses
    return dataclasses.replace(p, **kw)


def _search_fused_device(run: DeviceRun, gi: GpuIndex, p: SearchParams, report: int, st: Stats,
                         timers: bool = False, cand: bool = False):
    """K0, hypotheses and the fused search of one run whose raw spectra are already resident."""
    dev = gi.dev

    def phase(name):
        return Timer(st, name) if timers else _NoTimer()
    with phase("k0"):
        peaks = _k0_device(run, p, dev)
    with phase("hyp"):
        dh = _hyp_device(run, peaks, gi, p)
    with phase("fused"):
        o = _fused_device(gi, p, report, peaks, dh, run.n, cand=cand)
    o["peaks"] = peaks
    o["dh"] = dh
    return o


def _gather_fused(o, report, stats: Stats | None = None):
    """Device gather of the fused search's reported PSMs, one D2H copy per column."""
    psm, dh = o["psm"], o["dh"]
    ok = psm["row"] >= 0
    slot = torch.nonzero(ok).squeeze(1)
    s = slot // report
    hh = psm["hyp"][ok]
    cols = {"spec": s, "rank": psm["rank"][ok], "dnext": psm["dnext"][ok], "dbest": psm["dbest"][ok],
            "row": psm["row"][ok], "hyp": hh, "k1": psm["k1"][ok], "z": dh["z"][hh], "iso": dh["iso"][hh],
            "pm": dh["pm"][hh], "spec_scored": o["spec_scored"][s], "spec_matched": o["spec_matched"][s],
            "tic": o["peaks"]["tic"][s]}
    for k, name, _ in _K2_KEYS:
        cols[name] = psm[k][ok]
    out = {}
    for k, v in cols.items():
        out[k] = v.cpu().numpy()
        if stats is not None:
            stats.d2h_bytes += v.numel() * v.element_size()
    return out


class _NoTimer:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def search(sp: Spectra, gi: GpuIndex, l1, p: SearchParams, report: int | None = None, pre_hyp=None,
           timers: bool = False):
    """Full closed search of one run (reference engine.py:435-464).  Returns (PSM table, stats, debug).
    ``pre_hyp`` is accepted for signature compatibility; hypotheses are always computed on the device (they equal
    ``make_hypotheses`` on K0's validity mask)."""
    report = p.report_psms if report is None else report
    st = Stats()
    ru0 = resource.getrusage(resource.RUSAGE_SELF)
    t0 = time.perf_counter()
    with torch.cuda.device(gi.dev):
        run = DeviceRun(sp, gi.dev, st)
        method = p.search_method
        if method == "fused":
            out = _search_fused_device(run, gi, p, report, st, timers)
            stat = int(out["status"][:run.n].max()) if run.n else 0
            if stat & 2:
                raise RuntimeError("search_fused: a tile copy did not complete")
            if stat & 1:   # a spectrum spans more window rows than the fused kernel holds: staged path for the run
                method = "staged"
            else:
                tbl = _read_packed(*_pack_fused(gi, out, report, run.n), sp, st)
        if method == "staged":
            out = _search_device(run, gi, p, report, st, timers)
            check_status(out["status"])
            tbl = _read_packed(*_pack_psms(gi, out, report, run.n), sp, st)
        elif method != "fused":
            raise ValueError(f"unknown search_method {method!r}")
    ru1 = resource.getrusage(resource.RUSAGE_SELF)
    st.wall_s["total"] = time.perf_counter() - t0
    n_rescored = int(out["cand_off"][-1]) if "cand_off" in out else -1
    st.counts.update(n_spectra=len(sp), n_searched=int(out["peaks"]["valid_d"].sum()),
                     n_hypotheses=int(out["dh"]["spec_off"][-1]), n_rescored=n_rescored, n_psms=tbl.num_rows)
    if "win_off" in out:
        st.counts["k1_window_rows"] = int(out["win_off"][-1])
    st.counts["cpu_core_s"] = (ru1.ru_utime - ru0.ru_utime) + (ru1.ru_stime - ru0.ru_stime)
    return tbl, st, out


# ------------------------------------------------------------------------------------------------ graphs
_PSM_TABLE = ("spec_idx", "rank", "pf_row", "pf_id", "charge", "isotope_error", "expmass", "calcmass",
              "delta_mass_ppm", "hyperscore", "delta_next", "delta_best", "matched_b", "matched_y", "matched_peaks",
              "summed_intensity", "matched_intensity_pct", "average_ppm", "longest_b", "longest_y", "longest_y_pct",
              "peptide_len", "missed_cleavages", "n_var", "k1_count", "scored_candidates", "poisson")


def _lnfact_t(n: torch.Tensor) -> torch.Tensor:
    """``lnfact`` on the device (f64; 1.0 at n = 0, as the reference's table code)."""
    x = n.double()
    v = x * torch.log(x) - x + 0.5 * torch.log(x) + 0.5 * torch.log(2 * math.pi * x)
    return torch.where(x == 0, torch.ones_like(v), v)


def _psm_device_cols(gi: GpuIndex, raw: dict) -> dict:
    """The PSM table's columns on the device (reference engine.py:361-432, the features ``_psm_columns`` computes on
    the host), from per-slot raw values: spec, rank, dnext, dbest, row (>= 0), k1, z, iso, pm, spec_scored,
    spec_matched, tic and K2's outputs.  Same operations in the same precisions as the host code: f32 masses and
    percentages, f64 Poisson term (its exp / log / pow may differ from the host's libm in the last bit)."""
    rows = raw["row"]
    mbk, myk = raw["matched_b"].long(), raw["matched_y"].long()
    kk = mbk + myk
    sc, mt = raw["spec_scored"].long(), raw["spec_matched"].long()
    lam = mt.double() / sc.double()
    pois = lam.pow(kk.double()) * torch.exp(-lam) / torch.exp(_lnfact_t(kk))
    pois = torch.where(torch.isinf(pois), torch.full_like(pois, 1e-325), pois)
    log_pois = torch.log10(pois)
    z, iso, pm = raw["z"], raw["iso"], raw["pm"].float()
    calc = gi.mass32[rows]
    # Python scalars enter f32 kernels as f32 operands (NEUTRON and 2e6 are exact f32 values): f32 arithmetic
    ie = iso.float() * float(NEUTRON)
    dm = torch.abs(pm - calc - ie) * 2e6 / (pm - ie + calc)
    plen = gi.length[rows].long()
    sbs = raw["summed_b"] + raw["summed_y"]
    return {
        "spec_idx": raw["spec"].long(), "rank": raw["rank"].int(), "pf_row": rows.long(), "pf_id": gi.pf_id[rows],
        "charge": z.to(torch.int8), "isotope_error": iso.to(torch.int8), "expmass": pm, "calcmass": calc,
        "delta_mass_ppm": dm, "hyperscore": raw["hyperscore"].double(), "delta_next": raw["dnext"].double(),
        "delta_best": raw["dbest"].double(), "matched_b": mbk.to(torch.int16), "matched_y": myk.to(torch.int16),
        "matched_peaks": kk.to(torch.int16), "summed_intensity": sbs, "matched_intensity_pct": 100.0 * sbs / raw["tic"],
        "average_ppm": raw["ppm"], "longest_b": raw["longest_b"], "longest_y": raw["longest_y"],
        "longest_y_pct": (raw["longest_y"].double() / plen.double()).float(), "peptide_len": plen.to(torch.int16),
        "missed_cleavages": gi.missed[rows], "n_var": gi.n_var[rows], "k1_count": raw["k1"].int(),
        "scored_candidates": sc.int(), "poisson": log_pois}


def _pack(cols: dict, valid: torch.Tensor):
    """Device columns (plus the slot mask) in one byte buffer; returns (buffer, layout)."""
    parts, layout, off = [], [], 0
    for name, t in [("valid", valid.to(torch.uint8))] + list(cols.items()):
        t = t.contiguous()
        b = t.view(torch.uint8)
        pad = (-b.numel()) % 8
        parts.append(b)
        if pad:
            parts.append(torch.zeros(pad, dtype=torch.uint8, device=b.device))
        dt = np.dtype("uint64") if name == "pf_id" else np.dtype(str(t.dtype).replace("torch.", ""))
        layout.append((name, dt, off, t.numel()))
        off += b.numel() + pad
    return torch.cat(parts), layout


# columns of the packed PSM slots (vk_pack_psms), in buffer order
_PACK_COLS = (("valid", np.uint8), ("spec_idx", np.int64), ("rank", np.int32), ("pf_row", np.int64),
              ("pf_id", np.uint64), ("charge", np.int8), ("isotope_error", np.int8), ("expmass", np.float32),
              ("calcmass", np.float32), ("delta_mass_ppm", np.float32), ("hyperscore", np.float64),
              ("delta_next", np.float64), ("delta_best", np.float64), ("matched_b", np.int16),
              ("matched_y", np.int16), ("matched_peaks", np.int16), ("summed_intensity", np.float32),
              ("matched_intensity_pct", np.float32), ("average_ppm", np.float32), ("longest_b", np.int16),
              ("longest_y", np.int16), ("longest_y_pct", np.float32), ("peptide_len", np.int16),
              ("missed_cleavages", np.uint8), ("n_var", np.uint8), ("k1_count", np.int32),
              ("scored_candidates", np.int32), ("poisson", np.float64))
_PACK_LAYOUTS = {}


def _pack_layout(slots: int):
    """[(name, numpy dtype, byte offset, count)] of the packed buffer of `slots` PSM slots, its size, and the byte
    offsets as an int64 array for vk_pack_psms (each column padded to 8 bytes)."""
    if slots not in _PACK_LAYOUTS:
        layout, off = [], 0
        for name, dt in _PACK_COLS:
            dt = np.dtype(dt)
            layout.append((name, dt, off, slots))
            off += (slots * dt.itemsize + 7) & ~7
        _PACK_LAYOUTS[slots] = (layout, off, np.array([o for _, _, o, _ in layout], np.int64))
    return _PACK_LAYOUTS[slots]


def _pack_psms(gi: GpuIndex, out: dict, report: int, n: int):
    """Every PSM slot of a staged / pruned pass, its table columns computed on the device by one kernel
    (``vk_pack_psms``) straight into one byte buffer without a host read (empty slots masked): the graph-captured
    pass ends with it and the host reads it in one copy.  Returns (buffer, layout) with layout = [(name, numpy
    dtype, byte offset, count)]; the same buffer as ``_pack_psms_torch``."""
    psm_cand, psm_rank, dnext, dbest = out["psm"]
    slots = n * report
    layout, size, col_off = _pack_layout(slots)
    buf = torch.empty(max(size, 8), dtype=torch.uint8, device=psm_cand.device)
    # filled slots written contiguously in slot order: their rows from a scan of the fill flags
    row_pos = _scan((psm_cand[:slots] >= 0).to(torch.int64))
    dh, k2 = out["dh"], out["k2"]
    pin = K.PsmPackIn(K.ptr(psm_cand), K.ptr(psm_rank), K.ptr(dnext), K.ptr(dbest), K.ptr(out["c_hyp"]),
                      K.ptr(out["c_row"]), K.ptr(out["c_cnt"]), K.ptr(dh["z"]), K.ptr(dh["iso"]), K.ptr(dh["pm"]),
                      dh["z"].numel(), K.ptr(out["spec_scored"]), K.ptr(out["spec_matched"]),
                      K.ptr(out["peaks"]["tic"]), K.ptr(k2["hyperscore"]), K.ptr(k2["summed_b"]),
                      K.ptr(k2["summed_y"]), K.ptr(k2["ppm"]), K.ptr(k2["matched_b"]), K.ptr(k2["matched_y"]),
                      K.ptr(k2["longest_b"]), K.ptr(k2["longest_y"]), K.ptr(gi.mass32), K.ptr(gi.length),
                      K.ptr(gi.pf_id), K.ptr(gi.missed), K.ptr(gi.n_var), gi.n)
    K.check(K.lib().vk_pack_psms(C.byref(pin), slots, report, col_off.ctypes.data, K.ptr(row_pos), K.ptr(buf),
                                 K.stream()), "pack_psms")
    return buf, [("n_rows", np.dtype(np.int64), int(col_off[0]), 1)] + layout[1:]


def _pack_psms_torch(gi: GpuIndex, out: dict, report: int, n: int):
    """The same packed buffer as ``_pack_psms`` built from torch operations (``_psm_device_cols``): the
    formulation the fused search's packing shares, and the check of the kernel."""
    psm_cand, psm_rank, dnext, dbest = out["psm"]
    slots = n * report
    cand = psm_cand[:slots]
    ci = cand.clamp(min=0)
    s = torch.arange(slots, device=cand.device) // max(report, 1)
    dh, k2 = out["dh"], out["k2"]
    # empty slots read candidate 0, which may be unset: clamp every index into its table
    hh = out["c_hyp"][ci].clamp(0, dh["z"].numel() - 1)
    raw = {"spec": s, "rank": psm_rank[:slots], "dnext": dnext[:slots], "dbest": dbest[:slots],
           "row": out["c_row"][ci].clamp(0, max(gi.n - 1, 0)), "k1": out["c_cnt"][ci], "z": dh["z"][hh],
           "iso": dh["iso"][hh],
           "pm": dh["pm"][hh], "spec_scored": out["spec_scored"][s], "spec_matched": out["spec_matched"][s],
           "tic": out["peaks"]["tic"][s]}
    for k in ("hyperscore", "summed_b", "summed_y", "ppm", "matched_b", "matched_y", "longest_b", "longest_y"):
        raw[k] = k2[k][ci]
    return _pack(_psm_device_cols(gi, raw), cand >= 0)


def _pack_fused(gi: GpuIndex, o: dict, report: int, n: int):
    """The fused search's PSM slots, packed like ``_pack_psms``."""
    psm, dh = o["psm"], o["dh"]
    slots = n * report
    ok = psm["row"][:slots] >= 0
    s = torch.arange(slots, device=ok.device) // max(report, 1)
    hh = psm["hyp"][:slots].long().clamp(0, dh["z"].numel() - 1)
    raw = {"spec": s, "rank": psm["rank"][:slots], "dnext": psm["dnext"][:slots], "dbest": psm["dbest"][:slots],
           "row": psm["row"][:slots].long().clamp(0, max(gi.n - 1, 0)), "k1": psm["k1"][:slots], "z": dh["z"][hh], "iso": dh["iso"][hh],
           "pm": dh["pm"][hh], "spec_scored": o["spec_scored"][s], "spec_matched": o["spec_matched"][s],
           "tic": o["peaks"]["tic"][s]}
    for k, name, _ in _K2_KEYS:
        raw[name] = psm[k][:slots]
    return _pack(_psm_device_cols(gi, raw), ok)


def _unpack_psms(host: np.ndarray, layout, copy: bool = True) -> dict:
    """Host records of the filled PSM slots from a packed buffer.  A compacted buffer (layout starting with
    "n_rows": the filled slots first, in slot order) is read as slices: new arrays with ``copy`` (the buffer may be
    reused as soon as this returns), else views of the buffer, which then belongs to the records.  Otherwise the
    "valid" column selects the rows (new arrays)."""
    if layout and layout[0][0] == "n_rows":
        n = int(np.frombuffer(host, dtype=np.int64, count=1, offset=layout[0][2])[0])
        cols = {name: np.frombuffer(host, dtype=dt, count=n, offset=off) for name, dt, off, cnt in layout[1:]}
        return {k: v.copy() for k, v in cols.items()} if copy else cols
    cols = {name: np.frombuffer(host, dtype=dt, count=cnt, offset=off) for name, dt, off, cnt in layout}
    idx = np.flatnonzero(cols.pop("valid"))
    return {k: np.take(v, idx) for k, v in cols.items()}


_RUN_COLUMNS: dict = {}


def _run_column(run: str, n: int) -> pa.Array:
    """The "run" column of n rows: a slice of a cached repeated-string array (the last few run names kept)."""
    col = _RUN_COLUMNS.get(run)
    if col is None or len(col) < n:
        if len(_RUN_COLUMNS) >= 8:
            _RUN_COLUMNS.pop(next(iter(_RUN_COLUMNS)))
        col = _RUN_COLUMNS[run] = pa.repeat(pa.scalar(run, pa.string()), max(n, 1 << 16))
    return col.slice(0, n)


def _table(sp: Spectra, rec: dict) -> pa.Table:
    """The PSM table from device-computed columns: run, scan and retention time added on the host."""
    s = rec["spec_idx"]
    cols = {"run": _run_column(sp.run, len(s)), "spec_idx": s, "scan": sp.scan[s], "rt": sp.rt[s]}
    for k in _PSM_TABLE[1:]:
        cols[k] = rec[k]
    return pa.table(cols)


def _read_packed(buf: torch.Tensor, layout, sp: Spectra, stats: Stats | None = None) -> pa.Table:
    host = buf.cpu().numpy()
    if stats is not None:
        stats.d2h_bytes += host.nbytes
    return _table(sp, _unpack_psms(host, layout))


class GraphedPass:
    """One device pass over the fixed buffers of a resident run, captured once as a CUDA graph and replayed: the
    whole pass (K0 ... ranking and the packed PSM gather) is one launch.  Every buffer size is known on the host
    (bounds), so the pass reads nothing back while it runs.  ``fn()`` runs the pass and returns its outputs."""

    def __init__(self, fn, dev):
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            for _ in range(2):
                fn()
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize(dev)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, capture_error_mode="relaxed"):
            self.out = fn()

    def replay(self):
        self.graph.replay()
        return self.out


def _pinned_like(a: np.ndarray) -> np.ndarray:
    return torch.empty(a.shape, dtype=torch.from_numpy(np.ascontiguousarray(a[:0])).dtype,
                       pin_memory=True).numpy()


def _is_pinned(a: np.ndarray) -> bool:
    try:
        return bool(torch.from_numpy(a).is_pinned())
    except (TypeError, ValueError, RuntimeError):
        return False


class _ResultPool:
    """Pinned result buffers of one size (a run shape's packed PSMs), lent to the tables that view them and
    returned to ``free`` when those tables are dropped; at most ``cap`` exist."""

    def __init__(self, nbytes: int, cap: int):
        self.nbytes, self.cap = nbytes, cap
        self.free, self.n = [], 0

    def take(self):
        """A free buffer, a new one while fewer than ``cap`` exist, else None."""
        if self.free:
            return self.free.pop()
        if self.n < self.cap:
            self.n += 1
            return torch.empty(self.nbytes, dtype=torch.uint8, pin_memory=True)
        return None

    def lent_bytes(self) -> int:
        return (self.n - len(self.free)) * self.nbytes


class _Slot:
    """Device buffers of one run shape (n spectra, cap_raw peaks), the pass captured over them and pinned staging
    for inputs that are not pinned."""

    def __init__(self, searcher: "Searcher", n: int, cap_raw: int, max_raw: int, n_hyp_cap: int):
        se = searcher
        dev = se.gi.dev
        self.n, self.cap_raw = n, cap_raw
        empty = Spectra("slot", np.zeros(n, np.uint32), np.zeros(n, np.uint32), np.zeros(n), np.zeros(n),
                        np.ones(n, np.int8), np.zeros(cap_raw, np.float32), np.zeros(cap_raw, np.float32),
                        np.zeros(n + 1, np.int64))
        self.run = DeviceRun(empty, dev, pinned=False)
        self.run.max_raw = max_raw
        self.run.n_raw = cap_raw
        self.run.n_hyp_cap = n_hyp_cap
        report = se.report

        def fn():
            out = se.device_pass(self.run)
            buf, layout = _pack_psms(se.gi, out, report, self.n)
            out["packed"] = buf
            self.layout = layout
            return out
        self.gp = GraphedPass(fn, dev)
        self.out_bytes = self.gp.out["packed"].numel()
        # the packed PSMs' landing buffer when the shape's result pool has none free: read into copies at once
        self.host_out = torch.empty(self.out_bytes, dtype=torch.uint8, pin_memory=True)
        self.offsets = torch.empty(n + 1, dtype=torch.int64, pin_memory=True)   # offsets staging
        self.stage = {}
        self.h2d_done = torch.cuda.Event()
        self.done = torch.cuda.Event()
        self.busy = False

    def staged(self, key, a: np.ndarray) -> np.ndarray:
        """A pinned copy of a (reusing this slot's staging buffer for key)."""
        st = self.stage.get(key)
        if st is None or len(st) < len(a) or st.dtype != a.dtype:
            st = self.stage[key] = _pinned_like(np.empty(max(len(a), 1), a.dtype))
        np.copyto(st[:len(a)], a)
        return st[:len(a)]


class Searcher:
    """Repeated searches of runs through graph-captured device passes (plain, or pruned with ``pruner``).

    Runs are grouped by shape (spectra, peak capacity, largest peak count, hypothesis bound); each shape gets
    ``depth`` slots of device buffers with a captured pass, used in turn: the host-to-device copies of the next runs
    (on a copy stream) overlap the passes of the earlier ones (on a compute stream), and each pass's packed PSMs go
    back on a third stream, so that the next pass does not wait for them.  ``submit(sp)`` queues a run and returns
    a handle, ``result(handle)`` waits for it and builds its PSM table; ``search(sp)`` does both;
    ``search_many(runs)`` keeps ``depth`` runs in flight while the tables are built.  Inputs already in pinned host memory
    (``pin_spectra``) are copied straight to the device; others are staged through pinned buffers first.  Results
    are identical to ``engine.search`` / ``prune.search_pruned``.

    Each run's packed PSMs come back into a pinned buffer lent from the shape's pool, and the run's table columns
    are views of it (no host copy); the buffer returns to the pool when the table is dropped, so a caller that
    drops (or writes out) its tables reuses the same few buffers.  The pool of a shape holds at most ``hold_bytes``
    of buffers: while all of them are lent to live tables, further runs land in the slot's own pinned buffer and
    their tables get copied columns."""

    def __init__(self, gi: GpuIndex, l1, p: SearchParams, pruner=None, report: int | None = None, depth: int = 3,
                 hold_bytes: int = 1 << 30):
        if depth < 1:
            raise ValueError("depth: at least one run in flight")
        self.gi, self.l1, self.p, self.pruner = gi, l1, p, pruner
        self.report = p.report_psms if report is None else report
        self.depth = depth
        self.hold_bytes = hold_bytes
        self.pools = {}               # packed-buffer size -> _ResultPool
        self.slots = {}
        self.device_ms = 0.0          # summed CUDA-event time of the replayed passes (inputs already copied)
        # host seconds: waiting for results, unpacking them, building tables, submitting runs
        self.host_s = {"wait": 0.0, "unpack": 0.0, "table": 0.0, "submit": 0.0}
        self.copy_stream = torch.cuda.Stream(gi.dev)
        self.compute_stream = torch.cuda.Stream(gi.dev)
        self.d2h_stream = torch.cuda.Stream(gi.dev)
        self._turn = {}

    def device_pass(self, run: DeviceRun):
        if self.pruner is None:
            return _search_device(run, self.gi, self.p, self.report, Stats())
        from . import prune
        return prune._pruned_device(run, self.gi, self.p, self.pruner, self.report, Stats())

    def _n_hyp(self, sp: Spectra) -> int:
        z0, z1 = self.p.precursor_charge
        i0, i1 = self.p.isotope_errors
        return int(np.where(np.asarray(sp.charge) > 0, 1, z1 - z0 + 1).sum()) * (i1 - i0 + 1)

    def _shape(self, parts, n_total: int):
        """(spectra, peak capacity, largest peak count, hypothesis capacity) of consecutive runs padded to n_total
        spectra (padding: empty spectra of known charge)."""
        n_raw = sum(int(np.asarray(sp.offsets)[-1]) for sp in parts)
        mr = max((int(np.diff(np.asarray(sp.offsets, np.int64)).max()) for sp in parts if len(sp)), default=0)
        z0, z1 = self.p.precursor_charge
        i0, i1 = self.p.isotope_errors
        n_max = sum(self._n_hyp(sp) for sp in parts) + (n_total - sum(len(sp) for sp in parts)) * (i1 - i0 + 1)
        cap = 1 << max(10, int(n_raw - 1).bit_length())
        mr2 = 1 << max(5, int(mr - 1).bit_length())
        if getattr(self, "_force", None):
            cap, mr2 = max(cap, self._force[0]), max(mr2, self._force[1])
            n_max = max(n_max, self._force[2])
        return (n_total, cap, mr2, n_max)

    def submit(self, sp: Spectra):
        """Queue one run; returns a handle for ``result``."""
        return self._submit([sp], len(sp))

    def _submit(self, parts, n_total: int):
        key = self._shape(parts, n_total)
        with torch.cuda.device(self.gi.dev):
            if key not in self.slots:
                self.slots[key] = [_Slot(self, *key) for _ in range(self.depth)]
                self._turn[key] = 0
            slot = self.slots[key][self._turn[key]]
            self._turn[key] = (self._turn[key] + 1) % self.depth
            if slot.busy:
                raise RuntimeError("result() of the previous run in this slot was not collected")
            slot.busy = True
            run = slot.run
            # offsets of the concatenated runs (host, into pinned staging), the padding spectra empty
            offs = slot.offsets.numpy()
            base_pk = base_sp = 0
            offs[0] = 0
            for sp in parts:
                o = np.asarray(sp.offsets, np.int64)
                offs[base_sp + 1:base_sp + len(sp) + 1] = o[1:] + base_pk
                base_pk += int(o[-1])
                base_sp += len(sp)
            offs[base_sp + 1:] = base_pk
            # the previous pass over this slot and its read-back must be done before its buffers are reused
            self.copy_stream.wait_event(slot.done)
            h2d = 0
            with torch.cuda.stream(self.copy_stream):
                run.offsets.copy_(slot.offsets, non_blocking=True)
                h2d += slot.offsets.numel() * 8
                bp = bs = 0
                for j, sp in enumerate(parts):
                    nr = int(np.asarray(sp.offsets)[-1])
                    ns = len(sp)
                    for name, dst, a, lo, cnt in (("mz", run.mz, sp.mz, bp, nr), ("int", run.intensity, sp.intensity, bp, nr),
                                                  ("pmz", run.precursor_mz, sp.precursor_mz, bs, ns),
                                                  ("z", run.charge, sp.charge, bs, ns)):
                        if cnt == 0:
                            continue
                        dt = torch.empty(0, dtype=dst.dtype).numpy().dtype
                        a = np.asarray(a)[:cnt]
                        if a.dtype != dt or not a.flags.c_contiguous or not _is_pinned(a):
                            a = slot.staged((name, j), np.ascontiguousarray(a, dtype=dt))
                        dst[lo:lo + cnt].copy_(torch.from_numpy(a), non_blocking=True)
                        h2d += a.nbytes
                    bp += nr
                    bs += ns
                if bs < n_total:
                    run.precursor_mz[bs:n_total].fill_(0.0)
                    run.charge[bs:n_total].fill_(1)
            slot.h2d_done.record(self.copy_stream)
            self.compute_stream.wait_event(slot.h2d_done)
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            with torch.cuda.stream(self.compute_stream):
                ev[0].record(self.compute_stream)
                out = slot.gp.replay()
                ev[1].record(self.compute_stream)
            self.d2h_stream.wait_event(ev[1])
            pool = self.pools.get(slot.out_bytes)
            if pool is None:
                pool = self.pools[slot.out_bytes] = _ResultPool(slot.out_bytes, self.hold_bytes // slot.out_bytes)
            host_out = pool.take()
            lent = host_out is not None
            if not lent:
                host_out = slot.host_out
            with torch.cuda.stream(self.d2h_stream):
                host_out.copy_(out["packed"], non_blocking=True)
                slot.done.record(self.d2h_stream)
            return (parts[0] if len(parts) == 1 else None, slot, h2d, ev, host_out, pool if lent else None)

    def held_bytes(self) -> int:
        """Bytes of pinned result buffers lent to live tables."""
        return sum(pl.lent_bytes() for pl in self.pools.values())

    def _records(self, handle):
        sp, slot, h2d, ev, host_out, pool = handle
        t0 = time.perf_counter()
        slot.done.synchronize()
        t1 = time.perf_counter()
        self.device_ms += ev[0].elapsed_time(ev[1])
        check_status(slot.gp.out["status"])
        nb = host_out.numel()
        host = host_out.numpy()
        rec = _unpack_psms(host, slot.layout, copy=pool is None)
        if pool is not None:   # the records are views of `host`: the buffer goes back to the pool with them
            weakref.finalize(host, pool.free.append, host_out)
        self.host_s["wait"] += t1 - t0
        self.host_s["unpack"] += time.perf_counter() - t1
        slot.busy = False
        st = Stats()
        st.h2d_bytes, st.d2h_bytes = h2d, nb
        return rec, st

    def result(self, handle):
        rec, st = self._records(handle)
        return _table(handle[0], rec), st

    def search(self, sp: Spectra):
        return self.result(self.submit(sp))

    def search_batch(self, runs, batch_spectra: int = 131072):
        """PSM tables of many runs searched in batches: whole runs packed into batches of one fixed shape (padded
        with empty spectra to the largest batch, peak capacity of the largest batch), so that every batch replays
        the same captured pass; each run's arrays are copied straight into the batch's device buffers, and batch
        i+1 is copied while batch i runs.  Each run's table equals its own search.  Returns [(table, stats)], the
        stats (bytes moved) per batch on the batch's first run."""
        groups = plan_batches(runs, batch_spectra)
        n_b = max(sum(len(runs[i]) for i in g) for g in groups) if groups else 0
        raw = max((sum(int(np.asarray(runs[i].offsets)[-1]) for i in g) for g in groups), default=0)
        mr = max((int(np.diff(np.asarray(r.offsets, np.int64)).max()) for r in runs if len(r)), default=0)
        z0, z1 = self.p.precursor_charge
        i0, i1 = self.p.isotope_errors
        n_hyp = max((sum(self._n_hyp(runs[i]) for i in g) + (n_b - sum(len(runs[i]) for i in g)) * (i1 - i0 + 1)
                     for g in groups), default=0)
        self._force = (1 << max(10, int(raw - 1).bit_length()), 1 << max(5, int(mr - 1).bit_length()), n_hyp)
        try:
            tables, inflight, k = [], collections.deque(), 0

            def submit_next():
                nonlocal k
                parts = [runs[i] for i in groups[k]]
                starts = np.concatenate([[0], np.cumsum([len(r) for r in parts])]).tolist()
                inflight.append((self._submit(parts, n_b), parts, starts))
                k += 1
            while k < len(groups) and len(inflight) < self.depth:
                submit_next()
            while inflight:
                h, parts, starts = inflight.popleft()
                rec, st = self._records(h)          # frees the batch's slot ...
                if k < len(groups):
                    submit_next()                   # ... for a later batch, copied while the tables build
                empty = Stats()
                tables += [(t, st if i == 0 else empty) for i, t in enumerate(split_table(rec, parts, starts))]
        finally:
            self._force = None
        return tables

    def search_many(self, runs):
        """PSM tables of many runs, ``depth`` runs in flight: as soon as a run's PSM slots are read back (which
        frees its slot), the next run is submitted into it, so the host-to-device copies stay ahead of the device
        passes while the host builds the tables."""
        runs = list(runs)
        out, inflight, k = [], collections.deque(), 0
        while k < len(runs) and len(inflight) < self.depth:
            inflight.append(self.submit(runs[k]))
            k += 1
        while inflight:
            h = inflight.popleft()
            rec, st = self._records(h)
            t0 = time.perf_counter()
            if k < len(runs):
                inflight.append(self.submit(runs[k]))
                k += 1
            t1 = time.perf_counter()
            out.append((_table(h[0], rec), st))
            self.host_s["submit"] += t1 - t0
            self.host_s["table"] += time.perf_counter() - t1
        return out


    def search_sharded(self, runs, gather: bool = False):
        """Runs spread over the GPUs of the process group (one process per GPU, each with its own ``Searcher`` on
        its index replica): this rank searches its shard (``replicas.shard_runs``, whole runs balanced by size)
        with ``search_many``.  Returns [(run index, table, stats)] of this rank's runs, or every run's on every rank
        with ``gather``.  No collective touches the search itself."""
        from . import replicas
        return replicas.search_runs(list(runs), self.search_many, gather=gather)


def split_table(rec: dict, runs, starts) -> list:
    """Per-run PSM tables from the records of a batch (spectrum indices back to each run's own)."""
    s = rec["spec_idx"]
    out = []
    for r, sp in enumerate(runs):
        lo, hi = np.searchsorted(s, [starts[r], starts[r + 1]])
        sub = {k: v[lo:hi] for k, v in rec.items()}
        sub["spec_idx"] = sub["spec_idx"] - starts[r]
        out.append(_table(sp, sub))
    return out


def plan_batches(runs, batch_spectra: int):
    """Greedy packing of whole runs, in order, into batches of at most batch_spectra spectra (a longer run is a
    batch of its own); returns lists of run indices."""
    batches, cur, size = [], [], 0
    for i, sp in enumerate(runs):
        if cur and size + len(sp) > batch_spectra:
            batches.append(cur)
            cur, size = [], 0
        cur.append(i)
        size += len(sp)
    if cur:
        batches.append(cur)
    return batches


def pin_spectra(sp: Spectra) -> Spectra:
    """The run with its peak and precursor arrays in pinned host memory (copied once), for Searcher.submit."""
    def pin(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        b = _pinned_like(a)
        np.copyto(b, a)
        return b
    return Spectra(sp.run, sp.scan, sp.index, sp.rt, pin(sp.precursor_mz, np.float64), pin(sp.charge, np.int8),
                   pin(sp.mz, np.float32), pin(sp.intensity, np.float32), pin(sp.offsets, np.int64))


# ------------------------------------------------------------------------------------------------ references
def window_candidates(hyp, dev, spec_subset: np.ndarray | None = None):
    """Every (hypothesis, row) in the precursor windows, sorted by (spectrum, row) (reference engine.py:468-480)."""
    lo, hi = np.asarray(hyp["lo"]), np.asarray(hyp["hi"])
    hs = np.asarray(hyp["spec"])
    hsel = np.arange(len(lo))
    if spec_subset is not None:
        hsel = hsel[np.isin(hs, spec_subset)]
    n = (hi - lo)[hsel]
    hh = np.repeat(hsel, n)
    rr = np.repeat(lo[hsel], n) + (np.arange(n.sum()) - np.repeat(np.cumsum(n) - n, n))
    s = hs[hh]
    o = np.lexsort((rr, s))
    return torch.from_numpy(hh[o].astype(np.int64)).to(dev), torch.from_numpy(rr[o].astype(np.int64)).to(dev)


def k1_brute(gi: GpuIndex, hyp, peaks, h: torch.Tensor, r: torch.Tensor, p: SearchParams) -> torch.Tensor:
    """Brute-force preliminary counts for (hyp, row) pairs, no index (reference engine.py:483-497)."""
    L = K.lib()
    dev = gi.dev
    dh = _as_dev(hyp, dev)
    out = torch.empty(len(h), dtype=torch.int32, device=dev)
    hh = h.to(torch.int32).contiguous()
    rr = r.to(torch.int32).contiguous()
    K.check(L.vk_k1_brute(len(h), K.ptr(hh), K.ptr(rr), K.ptr(dh["spec"]), K.ptr(dh["maxfz"]), K.ptr(peaks["off"]),
                          K.ptr(peaks["mass"]), *gi.table_ptrs(), p.min_ion_index, p.fragment_min_mz,
                          p.fragment_max_mz, p.fragment_ppm[0], p.fragment_ppm[1], gi.inv_logw, K.ptr(out),
                          K.stream()), "k1_brute")
    return out


def search_exhaustive(sp: Spectra, gi: GpuIndex, l1, p: SearchParams, report: int | None = None,
                      spec_subset: np.ndarray | None = None, batch: int = 20_000_000):
    """K2 over EVERY candidate of the precursor windows, no K1 shortlist (reference engine.py:500-523)."""
    st = Stats()
    dev = gi.dev
    peaks = k0_preprocess(sp, p, dev, st)
    hyp = make_hypotheses(sp, peaks["valid"], gi.mass32_np, p)
    o_h, o_r, o_c, scored, matched, d_spec, d_maxfz = run_k1(gi, hyp, peaks, p, st)
    h, r = window_candidates(hyp, dev, spec_subset)
    spec = d_spec[h].long()
    parts = []
    i = 0
    n = len(h)
    while i < n:
        j = min(n, i + batch)
        if j < n:
            j = int(torch.searchsorted(spec, spec[j - 1], side="right"))
        parts.append(run_k2(gi, h[i:j], r[i:j], d_spec, d_maxfz, peaks, p))
        i = j
    k2 = {k: torch.cat([q[k] for q in parts]) for k in parts[0]} if parts else None
    c = torch.full((len(h),), -1, dtype=torch.int64, device=dev)
    tbl = psm_table(sp, gi, l1, hyp, h, r, c, k2, scored, matched, peaks, p, report)
    return tbl, st, {"peaks": peaks, "hyp": hyp, "h": h, "r": r, "k2": k2}
