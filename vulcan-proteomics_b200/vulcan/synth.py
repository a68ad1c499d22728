"""Seeded synthetic proteomes and MS2 runs for the search workloads.

No public dataset is read: every workload is a random proteome (log-normal protein lengths, amino acids drawn
from the UniProtKB/Swiss-Prot background composition) digested by :mod:`vulcan.index.build`, and MS2 spectra
simulated from random target peptidoforms of that index (b/y ions at charge 1 present with a fixed
probability, Gaussian ppm m/z error, uniform noise peaks, log-normal intensities).

Workloads (``WORKLOADS``):

  small   2,000 proteins, <= 1 missed cleavage, length 7-30, CAM-C fixed, Met-ox <= 1, pseudo-reverse decoys;
          5,000 spectra, charge 2-3, b/y presence 0.6, 100 noise peaks, 5 ppm error; +-10 ppm precursor,
          +-0.02 Th fragment tolerance, top-k 50.  Runs on the CPU.
  human   20,400 proteins, <= 2 missed cleavages (~1.5M target peptides + as many decoys); 40,000 spectra per run,
          charge 2-4, peak counts log-normal (median 150, clipped to 20-600), b/y presence 0.6; top-k 100.
"""
from __future__ import annotations

import dataclasses
import hashlib
import json
import os
import shutil

import numpy as np

from .gpu.host import NEUTRON, PROTON, SearchParams, Spectra
from .index._core import NTERM_BIT, SAGE_H2O, SAGE_MONO

# UniProtKB/Swiss-Prot amino-acid composition (percent), the usual "background frequencies".
AA_BACKGROUND = {
    "A": 8.25, "R": 5.53, "N": 4.06, "D": 5.45, "C": 1.37, "Q": 3.93, "E": 6.75, "G": 7.07, "H": 2.27,
    "I": 5.96, "L": 9.66, "K": 5.84, "M": 2.42, "F": 3.86, "P": 4.70, "S": 6.56, "T": 5.34, "W": 1.08,
    "Y": 2.92, "V": 6.87,
}


@dataclasses.dataclass
class Workload:
    name: str
    n_proteins: int
    missed_cleavages: int
    min_len: int
    max_len: int
    var_mods: dict
    max_var: int
    n_spectra: int
    charges: tuple
    presence: float
    noise_peaks: int | None          # fixed noise count (small) or None: total peaks log-normal (human)
    peaks_median: float
    peaks_sigma: float
    peaks_clip: tuple
    topk: int
    max_peaks: int
    proteome_seed: int
    spectra_seed: int
    iso_frac: tuple = (0.85, 0.12, 0.03)   # fraction of precursors picked at isotope 0 / +1 / +2
    site_limits: dict | None = None         # site caps per residue group, e.g. {"STY": 3, "M": 1}
    phospho_frac: float | None = None       # fraction of spectra simulated from phosphopeptides (S/T/Y sites)

    def index_params(self) -> dict:
        d = {"enzyme": {"cleave_at": "KR", "restrict": "P", "c_terminal": True,
                        "missed_cleavages": self.missed_cleavages, "min_len": self.min_len,
                        "max_len": self.max_len},
             "static_mods": {"C": 57.021464}, "variable_mods": dict(self.var_mods),
             "max_variable_mods": self.max_var}
        if self.site_limits:
            d["site_limits"] = dict(self.site_limits)
        return d

    def search_params(self, **kw) -> SearchParams:
        d = dict(precursor_ppm=(-10.0, 10.0), fragment_ppm=(-0.02, 0.02), fragment_unit="da",
                 isotope_errors=(0, 2), topk=self.topk, max_peaks=self.max_peaks)
        d.update(kw)
        return SearchParams(**d)


WORKLOADS = {
    "small": Workload("small", 2000, 1, 7, 30, {"M": 15.9949}, 1, 5000, (2, 3), 0.6, 100, 0.0, 0.0, (0, 0),
                      50, 150, 20241, 7),
    "human": Workload("human", 20400, 2, 7, 30, {"M": 15.9949}, 1, 40000, (2, 4), 0.6, None, 150.0, 0.5,
                      (20, 600), 100, 512, 20400, 11),
    # configuration 4: the human proteome with phospho on S/T/Y (at most 3 sites) and Met-ox (at most 1);
    # runs of 20,000-50,000 spectra, 40% from phosphopeptides, top-k 200
    "phospho": Workload("phospho", 20400, 2, 7, 30, {"M": 15.9949, "S": 79.966331, "T": 79.966331,
                                                   "Y": 79.966331}, 4, 40000, (2, 4), 0.6, None, 150.0, 0.5,
                        (20, 600), 200, 512, 20400, 13, site_limits={"STY": 3, "M": 1}, phospho_frac=0.4),
}


def phospho_rows(l1) -> np.ndarray:
    """Whether each row carries a modification on S, T or Y."""
    mask = np.asarray(l1.mask, np.uint64)
    off = np.asarray(l1.seq_off, np.int64)
    ln = np.asarray(l1.length, np.int64)
    res = np.asarray(l1.residues)
    sty = np.zeros(256, bool)
    sty[[ord("S"), ord("T"), ord("Y")]] = True
    out = np.zeros(len(mask), bool)
    for k in range(int(ln.max()) if len(ln) else 0):
        on = ((mask >> np.uint64(k)) & np.uint64(1)).astype(bool) & (ln > k)
        idx = np.flatnonzero(on)
        out[idx] |= sty[res[off[idx] + k]]
    return out


def random_proteome_fasta(n_proteins: int, seed: int, median_len: float = 400.0, sigma: float = 0.6) -> str:
    rng = np.random.default_rng(seed)
    aas = np.array(list(AA_BACKGROUND), dtype="<U1")
    freq = np.array(list(AA_BACKGROUND.values()), np.float64)
    freq /= freq.sum()
    lens = np.maximum(30, np.round(rng.lognormal(np.log(median_len), sigma, n_proteins))).astype(np.int64)
    body = rng.choice(len(aas), int(lens.sum()), p=freq)
    letters = np.frombuffer("".join(aas).encode(), np.uint8)[body]
    off = np.concatenate([[0], np.cumsum(lens)])
    lines = []
    for i in range(n_proteins):
        seq = "M" + letters[off[i] + 1:off[i + 1]].tobytes().decode()
        lines.append(f">sp|SYN{i:06d}|SYN{i:06d}_RANDOM synthetic protein {i}\n{seq}\n")
    return "".join(lines)


def _cache_key(w: Workload) -> str:
    d = {"n": w.n_proteins, "mc": w.missed_cleavages, "len": [w.min_len, w.max_len], "var": w.var_mods,
         "mv": w.max_var, "seed": w.proteome_seed, "v": 2}
    if w.site_limits:
        d["lim"] = w.site_limits
    return hashlib.sha256(json.dumps(d, sort_keys=True).encode()).hexdigest()[:12]


def build_index(w: Workload | str, root: str):
    """Build (or reuse) the workload's L1 index under ``root``; returns its directory."""
    from .index.build import build
    w = WORKLOADS[w] if isinstance(w, str) else w
    d = os.path.join(root, f"{w.name}_{_cache_key(w)}")
    if os.path.exists(os.path.join(d, "meta.json")):
        return d
    # built in a directory of this process and renamed into place, so that processes building the same index at
    # the same time (one per GPU) never see each other's partial files; the first rename wins
    os.makedirs(root, exist_ok=True)
    tmp = f"{d}.tmp{os.getpid()}"
    shutil.rmtree(tmp, ignore_errors=True)
    os.makedirs(tmp)
    fa = os.path.join(tmp, "proteome.fasta")
    with open(fa, "w") as fh:
        fh.write(random_proteome_fasta(w.n_proteins, w.proteome_seed))
    build([fa], tmp, w.index_params())
    try:
        os.rename(tmp, d)
    except OSError:   # another process renamed its copy first
        shutil.rmtree(tmp, ignore_errors=True)
        if not os.path.exists(os.path.join(d, "meta.json")):
            raise
    return d


def fragment_ladders(seq: bytes, mask: int, static: dict, var: dict, nterm: float = 0.0):
    """Neutral b and y fragment masses (f64) of one peptidoform, b_k / y_k for k = 1..L-1."""
    res = np.array([float(SAGE_MONO[c - 65]) for c in seq])
    for k, c in enumerate(seq):
        ch = chr(c)
        if (mask >> k) & 1:
            res[k] += var.get(ch, 0.0)
        else:
            res[k] += static.get(ch, 0.0)
    nt = nterm if mask & NTERM_BIT else 0.0
    cs = np.cumsum(res)
    total = cs[-1] + nt
    b = cs[:-1] + nt
    y = float(SAGE_H2O) + total - b
    return b, y


def simulate_run(l1, labels, w: Workload | str, n_spectra: int | None = None, seed: int | None = None,
                 run: str | None = None):
    """Simulated MS2 run from random target rows of ``l1``.  Returns (Spectra, truth_rows)."""
    w = WORKLOADS[w] if isinstance(w, str) else w
    n = w.n_spectra if n_spectra is None else n_spectra
    rng = np.random.default_rng(w.spectra_seed if seed is None else seed)
    is_dec = np.asarray(labels.column("is_decoy").to_numpy(zero_copy_only=False), bool)
    tgt = np.flatnonzero(~is_dec)
    if w.phospho_frac:
        ph = phospho_rows(l1)[tgt]
        n_ph = int(round(n * w.phospho_frac))
        a, b = tgt[ph], tgt[~ph]
        rows = np.concatenate([rng.choice(a, n_ph, replace=len(a) < n_ph),
                               rng.choice(b, n - n_ph, replace=len(b) < n - n_ph)])
        rows = rows[rng.permutation(n)]
    else:
        rows = rng.choice(tgt, n, replace=len(tgt) < n)
    static = {"C": 57.021464}
    mz_l, it_l = [], []
    off = np.zeros(n + 1, np.int64)
    pmz = np.empty(n)
    ch = rng.integers(w.charges[0], w.charges[1] + 1, n).astype(np.int8)
    iso = rng.choice(3, n, p=np.array(w.iso_frac) / np.sum(w.iso_frac))
    for i, r in enumerate(rows.tolist()):
        seq = l1.residues[l1.seq_off[r]:l1.seq_off[r] + l1.length[r]].tobytes()
        b, y = fragment_ladders(seq, int(l1.mask[r]), static, w.var_mods, nterm=w.var_mods.get("^", 0.0))
        ions = np.concatenate([b, y]) + float(PROTON)
        ions = ions[(ions > 50.0)]
        sig = ions[rng.random(len(ions)) < w.presence]
        if w.noise_peaks is not None:
            n_noise = w.noise_peaks
        else:
            tot = int(np.clip(np.round(rng.lognormal(np.log(w.peaks_median), w.peaks_sigma)), *w.peaks_clip))
            if len(sig) > tot:
                sig = rng.choice(sig, tot, replace=False)
            n_noise = tot - len(sig)
        sig = sig * (1.0 + rng.normal(0.0, 5e-6, len(sig)))
        noise = rng.uniform(150.0, 2000.0, n_noise)
        mz = np.concatenate([sig, noise]).astype(np.float32)
        inten = np.concatenate([rng.lognormal(np.log(3000.0), 0.8, len(sig)),
                                rng.lognormal(np.log(1000.0), 1.0, n_noise)]).astype(np.float32)
        o = np.argsort(mz, kind="stable")
        mz_l.append(mz[o])
        it_l.append(inten[o])
        off[i + 1] = off[i] + len(mz)
        z = float(ch[i])
        mono = float(l1.mass32[r]) + iso[i] * float(NEUTRON)
        pmz[i] = (mono + z * float(PROTON)) / z * (1.0 + rng.normal(0.0, 1e-6))
    sp = Spectra(run or f"synthetic_{w.name}", np.arange(n, dtype=np.uint32), np.arange(n, dtype=np.uint32),
                 np.linspace(0.0, 120.0, n), pmz, ch, np.concatenate(mz_l) if n else np.zeros(0, np.float32),
                 np.concatenate(it_l) if n else np.zeros(0, np.float32), off)
    return sp, rows


def take_spectra(sp: Spectra, sel: np.ndarray, run: str) -> Spectra:
    """The spectra sel (indices, repeats allowed, in that order) of a run, as a new run."""
    sel = np.asarray(sel, np.int64)
    off = np.asarray(sp.offsets, np.int64)
    lens = off[1:][sel] - off[:-1][sel]
    new_off = np.zeros(len(sel) + 1, np.int64)
    np.cumsum(lens, out=new_off[1:])
    idx = np.repeat(off[:-1][sel] - new_off[:-1], lens) + np.arange(int(new_off[-1]))
    return Spectra(run, np.arange(len(sel), dtype=np.uint32), np.arange(len(sel), dtype=np.uint32),
                   np.asarray(sp.rt)[sel], np.asarray(sp.precursor_mz)[sel], np.asarray(sp.charge)[sel],
                   np.asarray(sp.mz)[idx], np.asarray(sp.intensity)[idx], new_off)


def batch_runs(pool: Spectra, n_runs: int = 64, lo: int = 5000, hi: int = 60000, seed: int = 2):
    """Runs for the batched benchmark: sizes log-uniform in [lo, hi], spectra drawn (with replacement, seeded)
    from a pool of simulated spectra."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), n_runs)).astype(np.int64)
    return [take_spectra(pool, rng.integers(0, len(pool), int(n)), f"batch_run{i}") for i, n in enumerate(sizes)]
