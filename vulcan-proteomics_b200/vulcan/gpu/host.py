"""Torch-free host pieces of the closed search (mirror of the reference's ``vulcan/gpu/host.py``).

``SearchParams``, ``Spectra``, ``make_hypotheses`` and ``pre_hypotheses`` keep the reference's names, fields,
defaults and results.  ``make_hypotheses`` is the host restatement; the search itself computes the same
hypotheses on the device (``vk_hypotheses``) and the tests pin the two against each other and against golden
vectors taken from the reference.
"""
from __future__ import annotations

from dataclasses import asdict, dataclass

import numpy as np

PROTON = np.float32(1.0072764)
NEUTRON = np.float32(1.00335)


@dataclass
class SearchParams:
    """Search knobs (reference ``host.py:14-43``; same names and defaults)."""
    precursor_ppm: tuple = (-10.0, 10.0)
    fragment_ppm: tuple = (-20.0, 20.0)
    fragment_unit: str = "ppm"              # "ppm" or "da" (fragment_ppm then holds Da bounds)
    isotope_errors: tuple = (0, 2)
    precursor_charge: tuple = (2, 4)        # tried when the spectrum carries no charge
    max_peaks: int = 150
    min_peaks: int = 15
    fragment_min_mz: float = 150.0
    fragment_max_mz: float = 2000.0
    min_ion_index: int = 2
    max_fragment_charge: int | None = 1
    min_matched_peaks: int = 4
    topk: int = 500
    k1_threshold: int = 1
    pair_closure: bool = True
    report_psms: int = 1
    peak_mode: str = "global"               # "global" (Sage) | "window" (top window_k per window_th Th window)
    window_th: float = 100.0
    window_k: int = 15
    # reference K1 layout knobs (the compatible entry points use them)
    chunk_size: int = 8192
    bin_ppm: float = 20.0
    tile: int = 1024
    k2_threads: int = 128
    max_slice_entries: int = 2 ** 31 - 1
    # B200 layout knobs: rows per fragment-index tile (power of two, 32..1024; the tile's postings must fit one
    # CTA's shared memory), coarse m/z bins per tile (0 = 2^8 per 64 rows), warps per K1 CTA
    tile_rows: int = 128
    cbin_bits: int = 0
    k1_warps: int = 4
    # K1 shapes per peak-count bucket (chosen by the autotuner): ((most kept peaks, tile_rows, k1_warps), ...) in
    # ascending peak bounds; a spectrum takes the first bucket its kept peaks fit, spectra above the last bound
    # take (tile_rows, k1_warps).  Empty: one shape for every spectrum.  The counts do not depend on the shapes.
    k1_shapes: tuple = ()
    search_method: str = "staged"           # "staged" (a kernel per stage) or "fused" (one persistent kernel)
    fused_warps: int = 4                    # warps of a fused-search CTA (one spectrum at a time)
    fused_cnt_cap: int = 4096               # window rows a spectrum may span in the fused search

    def to_dict(self):
        return asdict(self)


@dataclass
class Spectra:
    """MS2 spectra of one run, host side (reference ``host.py:47-60``)."""
    run: str
    scan: np.ndarray
    index: np.ndarray
    rt: np.ndarray
    precursor_mz: np.ndarray       # f64
    charge: np.ndarray             # i8, 0 = unknown
    mz: np.ndarray                 # f32 flat
    intensity: np.ndarray          # f32 flat
    offsets: np.ndarray            # i64 n+1

    def __len__(self):
        return len(self.scan)


def max_fragment_z(z: np.ndarray, p: SearchParams) -> np.ndarray:
    """Exclusive upper bound of fragment charges searched for precursor charge z (``host.py:88-89``)."""
    mfc = p.max_fragment_charge
    zz = np.minimum(z, mfc + 1) if mfc else z
    return np.maximum(zz, 2).astype(np.int8)


def make_hypotheses(sp: Spectra, valid: np.ndarray, idx_mass32: np.ndarray, p: SearchParams):
    """Precursor hypotheses (spectrum, charge, isotope error) and their index row windows.

    Follows ``host.py:64-91``: hypotheses ordered by (spectrum, charge, isotope); f32 arithmetic
    ``mz = f32(pmz) - PROTON``, ``pm = mz * z``, ``M = pm - iso * NEUTRON``, bounds ``M + (M * ppm) / 1e6``; the
    window is ``[searchsorted(lo, left), searchsorted(hi, right))`` over the mass-sorted index.
    """
    spec = np.flatnonzero(np.asarray(valid, bool) & np.isfinite(sp.precursor_mz))
    zi = sp.charge[spec].astype(np.int64)
    known = zi > 0
    isos = np.arange(p.isotope_errors[0], p.isotope_errors[1] + 1)
    zr = np.arange(p.precursor_charge[0], p.precursor_charge[1] + 1)
    # per spectrum: known charge -> one charge; unknown -> the charge range; each with every isotope error
    n_z = np.where(known, 1, len(zr))
    cnt = n_z * len(isos)
    s = np.repeat(spec, cnt)
    k = np.arange(len(s)) - np.repeat(np.cumsum(cnt) - cnt, cnt)   # position within the spectrum's block
    zpos, ipos = k // len(isos), k % len(isos)
    kn = np.repeat(known, cnt)
    z = np.where(kn, np.repeat(zi, cnt), zr[np.minimum(zpos, len(zr) - 1)] if len(zr) else 0)
    iso = isos[ipos] if len(isos) else np.zeros(0, np.int64)
    mz = (sp.precursor_mz[s].astype(np.float32) - PROTON).astype(np.float32)
    pm = (mz * z.astype(np.float32)).astype(np.float32)
    M = (pm - (iso.astype(np.float32) * NEUTRON).astype(np.float32)).astype(np.float32)
    plo, phi = np.float32(p.precursor_ppm[0]), np.float32(p.precursor_ppm[1])
    lo = (M + (M * plo) / np.float32(1e6)).astype(np.float32)
    hi = (M + (M * phi) / np.float32(1e6)).astype(np.float32)
    rlo = np.searchsorted(idx_mass32, lo, side="left")
    rhi = np.searchsorted(idx_mass32, hi, side="right")
    return {"spec": s.astype(np.int32), "z": z.astype(np.int8), "iso": iso.astype(np.int8), "pm": pm, "M": M,
            "lo": rlo.astype(np.int64), "hi": rhi.astype(np.int64), "maxfz": max_fragment_z(z, p)}


def pre_hypotheses(sp: Spectra, gi, p: SearchParams):
    """Hypotheses computable before K0 (``host.py:94-105``): valid = min(#peaks in range, max_peaks) >= min_peaks."""
    assert p.peak_mode == "global"
    mz = sp.mz
    ok = (mz >= p.fragment_min_mz) & (mz <= p.fragment_max_mz) & ~np.isnan(mz)
    cs = np.zeros(len(ok) + 1, np.int64)
    np.cumsum(ok, out=cs[1:])
    n_in = cs[sp.offsets[1:]] - cs[sp.offsets[:-1]]
    valid = np.minimum(n_in, p.max_peaks) >= p.min_peaks
    return valid, make_hypotheses(sp, valid, gi.mass32_np, p)
