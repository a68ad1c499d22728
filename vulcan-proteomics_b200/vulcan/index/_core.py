"""Proteome-index primitives: digestion, peptidoform expansion, Sage f32 masses, hash ids.

The reference does this in a Rust/PyO3 crate (``vulcan/rust/vulcan_core/src/lib.rs``) on top of sage-core
99407db6 (git dependency, not vendored).  This module restates the parts the search path consumes with the same
function names and return dictionaries; the per-peptidoform work runs in the native core
``csrc/vulcan_core.cpp`` (OpenMP):

* ``digest_fasta``   -- ``lib.rs:89-150``: unique I/L-collapsed peptides of standard residues, sorted, with the
  minimum missed-cleavage count and the protein CSR.  The tryptic rule is the one ``build.py:251-254`` states
  (cleave after ``cleave_at`` unless the next residue is in ``restrict``; missed cleavages = skipped internal
  sites).  sage-core's own digester is not available here, so this digestion is the definition of the index for
  the synthetic proteomes (no N-terminal methionine clipping).
* ``expand_pairs``   -- ``lib.rs:283-399``: variable-mod forms of every forward peptide (all subsets of the
  modifiable sites of size <= ``max_var``), carried to the decoy through its permutation, mass-filtered on the
  f64 form mass, ids ``xxh64(canonical, id_seed)`` and Sage f32 masses.
* ``sage_mass32``    -- ``lib.rs:236-254``: ``H2O`` plus residues in sequence order, then plus the f32 sum of the
  per-residue modification deltas (plus the N-terminal delta), all in f32.
* ``canonical``      -- ``lib.rs:215-228``: residues with ``[+d.dddd]`` after each variable-modified residue,
  ``[+d.dddd]-`` in front for a peptide-N-term variable mod.
"""
from __future__ import annotations

import numpy as np
import xxhash

SAGE_COMMIT = "99407db6e3754b31a9b88b7316a0aee67293c93f"

# Sage f32 monoisotopic residue masses, index = ASCII - 'A' (reference vulcan/gpu/engine.py:30-32).
SAGE_MONO = np.array([71.03711, 0.0, 103.00919, 115.02694, 129.04259, 147.0684, 57.02146, 137.05891, 113.08406,
                      0.0, 128.09496, 113.08406, 131.0405, 114.04293, 237.14774, 97.05276, 128.05858, 156.1011,
                      87.03203, 101.04768, 150.95363, 99.06841, 186.07932, 0.0, 163.06332, 0.0], np.float32)
# Sage f32 water mass (reference vulcan/gates/a2_identity.py:35).
SAGE_H2O = np.float32(18.010565)
# Unimod f64 residue masses (reference vulcan/rust/vulcan_core/src/lib.rs:33-61), used for the mass filter.
RESIDUE_F64 = np.array([71.037113805, 0.0, 103.009184505, 115.026943065, 129.042593135, 147.068413945,
                        57.021463721, 137.058911875, 113.084064015, 0.0, 128.094963050, 113.084064015,
                        131.040484645, 114.042927470, 0.0, 97.052763875, 128.058577540, 156.101111050,
                        87.032028435, 101.047678505, 0.0, 99.068413945, 186.079312980, 0.0, 163.063328575, 0.0])
H2O_F64 = 18.010564684
NTERM_BIT = 1 << 63
_STD = np.zeros(256, bool)
_STD[[ord(c) for c in "ACDEFGHIKLMNPQRSTVWY"]] = True


def _is_standard(s: str) -> bool:
    b = np.frombuffer(s.encode(), np.uint8)
    return bool(_STD[b].all())


def parse_fasta(text: str, decoy_tag: str = "rev_"):
    """(accession, sequence) pairs; entries whose accession contains ``decoy_tag`` are skipped."""
    out = []
    for block in text.split(">")[1:]:
        head, _, body = block.partition("\n")
        acc = head.split()[0] if head.split() else ""
        if decoy_tag and decoy_tag in acc:
            continue
        out.append((acc, "".join(body.split())))
    return out


def cleavage_sites(seq: str, cleave_at: str, restrict: str | None, c_terminal: bool = True) -> list[int]:
    n = len(seq)
    rest = restrict or ""
    sites = [0]
    if c_terminal:
        for i in range(n - 1):
            if seq[i] in cleave_at and seq[i + 1] not in rest:
                sites.append(i + 1)
    else:
        for i in range(1, n):
            if seq[i] in cleave_at and seq[i - 1] not in rest:
                sites.append(i)
    sites.append(n)
    return sites


def digest_fasta(fasta_text: str, missed_cleavages: int, min_len: int, max_len: int, cleave_at: str,
                 restrict: str | None, c_terminal: bool) -> dict:
    """Tryptic-style digestion of every protein (vectorised over the whole proteome)."""
    prots = parse_fasta(fasta_text)
    accessions = [a for a, _ in prots]
    seqs = [q for _, q in prots]
    n_prot = len(seqs)
    plen = np.fromiter((len(q) for q in seqs), np.int64, n_prot)
    buf = np.frombuffer("".join(seqs).encode(), np.uint8)
    pstart = np.zeros(n_prot + 1, np.int64)
    np.cumsum(plen, out=pstart[1:])
    pid = np.repeat(np.arange(n_prot), plen)
    cut = np.zeros(256, bool)
    cut[np.frombuffer(cleave_at.encode(), np.uint8)] = True
    rst = np.zeros(256, bool)
    if restrict:
        rst[np.frombuffer(restrict.encode(), np.uint8)] = True
    nb = len(buf)
    if c_terminal:
        # site after position i when buf[i] cleaves, buf[i+1] is not restricted, and i+1 is in the same protein
        ok = cut[buf[:-1]] & ~rst[buf[1:]] & (pid[:-1] == pid[1:]) if nb > 1 else np.zeros(0, bool)
        site_g = np.flatnonzero(ok) + 1
    else:
        ok = cut[buf[1:]] & ~rst[buf[:-1]] & (pid[:-1] == pid[1:]) if nb > 1 else np.zeros(0, bool)
        site_g = np.flatnonzero(ok) + 1
    # sites per protein: start, internal sites, end; ordered by (protein, position)
    s_pos = np.concatenate([pstart[:-1], site_g, pstart[1:]])
    s_pid = np.concatenate([np.arange(n_prot), pid[site_g], np.arange(n_prot)])
    s_end = np.concatenate([np.zeros(n_prot, bool), np.zeros(len(site_g), bool), np.ones(n_prot, bool)])
    o = np.lexsort((s_end, s_pos, s_pid))
    s_pos, s_pid = s_pos[o], s_pid[o]
    starts, ends, miss = [], [], []
    ns = len(s_pos)
    for m in range(missed_cleavages + 1):
        if ns <= 1 + m:
            break
        a = np.arange(ns - 1 - m)
        b = a + 1 + m
        same = s_pid[a] == s_pid[b]
        a, b = a[same], b[same]
        ln = s_pos[b] - s_pos[a]
        keep = (ln >= min_len) & (ln <= max_len)
        starts.append(s_pos[a][keep])
        ends.append(s_pos[b][keep])
        miss.append(np.full(int(keep.sum()), m, np.int64))
    st = np.concatenate(starts) if starts else np.zeros(0, np.int64)
    en = np.concatenate(ends) if ends else np.zeros(0, np.int64)
    mi = np.concatenate(miss) if miss else np.zeros(0, np.int64)
    pp = pid[st] if len(st) else np.zeros(0, np.int64)
    # non-standard residues
    bad = np.concatenate([[0], np.cumsum(~_STD[buf])])
    nonstd = (bad[en] - bad[st]) > 0
    width = int((en - st).max()) if len(st) else 1
    col = np.arange(width)
    lens = en - st

    def fixed(sel, table):
        idx = st[sel][:, None] + col[None, :]
        valid = col[None, :] < lens[sel][:, None]
        mat = np.where(valid, table[np.minimum(idx, nb - 1)], 0).astype(np.uint8)
        return np.ascontiguousarray(mat).view(f"S{width}").ravel()
    n_nonstd = len(np.unique(fixed(nonstd, buf))) if nonstd.any() else 0
    il = buf.copy()
    il[il == ord("I")] = ord("L")
    good = ~nonstd
    keys_b = fixed(good, il)
    uk, inv = np.unique(keys_b, return_inverse=True)
    missed = np.full(len(uk), 255, np.int64)
    np.minimum.at(missed, inv, mi[good])
    pk = np.unique(inv.astype(np.int64) * (n_prot + 1) + pp[good])
    ki, pi = pk // (n_prot + 1), pk % (n_prot + 1)
    prot_off = np.zeros(len(uk) + 1, np.int64)
    np.cumsum(np.bincount(ki, minlength=len(uk)), out=prot_off[1:])
    keys = [k.decode() for k in uk.tolist()]
    return {"keys": keys, "missed": missed.astype(np.uint8), "prot_off": prot_off,
            "prot_idx": pi.astype(np.uint32), "accessions": accessions, "n_nonstandard": int(n_nonstd)}


def _mod_tables(static_mods, var_mods):
    static_res = np.zeros(26)
    var_res = np.zeros(26)
    nterm = 0.0
    for k, v in static_mods:
        if len(k) != 1 or not k.isalpha():
            raise ValueError("only residue static mods are supported")
        static_res[ord(k) - 65] = v
    for k, v in var_mods:
        if k == "^":
            if nterm != 0.0:
                raise ValueError("at most one variable peptide-N-term mod")
            nterm = v
            continue
        if len(k) != 1 or not k.isalpha():
            raise ValueError("only residue and peptide-N-term (^) variable mods are supported")
        i = ord(k) - 65
        if var_res[i] != 0.0 or static_res[i] != 0.0:
            raise ValueError("at most one variable mod per residue, and not on a statically modified residue")
        var_res[i] = v
    return static_res, var_res, nterm


def canonical(seq: str, mask: int, var_res: np.ndarray, nterm: float = 0.0) -> str:
    parts = []
    if mask & NTERM_BIT:
        parts.append(f"[{nterm:+.4f}]-")
    for k, c in enumerate(seq):
        parts.append(c)
        if (mask >> k) & 1:
            parts.append(f"[{var_res[ord(c) - 65]:+.4f}]")
    return "".join(parts)


def peptidoform_id(seq: str, mask: int, var_mods, id_seed: int):
    _, var_res, nterm = _mod_tables([], var_mods)
    s = canonical(seq, mask, var_res, nterm)
    return s, xxhash.xxh64_intdigest(s, id_seed)


def _native():
    from .._native import core_lib
    return core_lib()


def expand_pairs(fwd, dec, perm_flat, perm_off, static_mods, var_mods, max_var, min_mass, max_mass, id_seed,
                 site_limits: dict | None = None, nthreads: int = 0):
    """Paired peptidoforms, one row per (forward form, decoy form) pair (``lib.rs:271-399``), computed by the
    native core (``csrc/vulcan_core.cpp``).  ``site_limits`` optionally caps modification sites under ``max_var``:
    each key is one or more residue letters whose sites are capped together (``{"STY": 3, "M": 1}``: at most three
    phospho sites on S/T/Y in total and one oxidised M)."""
    import ctypes as C
    if len(fwd) != len(dec):
        raise ValueError("fwd and dec differ in length")
    static_res, var_res, nterm = _mod_tables(static_mods, var_mods)
    n = len(fwd)
    lens = np.fromiter((len(s) for s in fwd), np.int64, n)
    if any(len(d) != len(f) for f, d in zip(fwd, dec)):
        raise ValueError("fwd and dec pair lengths differ")
    off = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    fres = np.frombuffer("".join(fwd).encode(), np.uint8)
    dres = np.frombuffer("".join(dec).encode(), np.uint8)
    bad = ~_STD[fres] | ~_STD[dres] if len(fres) else np.zeros(0, bool)
    if bad.any():
        raise ValueError("non-standard residue in a pair")
    perm_flat = np.ascontiguousarray(perm_flat, np.uint8)
    perm_off = np.ascontiguousarray(perm_off, np.int64)
    group = np.arange(26, dtype=np.uint8)
    lim = np.full(26, 255, np.uint8)
    for key, k in (site_limits or {}).items():
        g = ord(key[0]) - 65
        for r in key:
            group[ord(r) - 65] = g
        lim[g] = min(255, int(k))
    mono = np.ascontiguousarray(SAGE_MONO, np.float32)
    resf = np.ascontiguousarray(RESIDUE_F64, np.float64)
    st = np.ascontiguousarray(static_res, np.float64)
    va = np.ascontiguousarray(var_res, np.float64)
    L = _native()
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)
    args = [C.c_int64(n), ptr(fres), ptr(dres), ptr(off), ptr(perm_flat), ptr(perm_off), ptr(mono), ptr(resf),
            ptr(st), ptr(va), C.c_double(nterm), C.c_int(int(max_var)), ptr(group), ptr(lim), C.c_double(min_mass),
            C.c_double(max_mass), C.c_uint64(int(id_seed)), C.c_int(int(nthreads))]
    total = L.vc_expand_pairs(*args, *([None] * 9))
    if total < 0:
        raise ValueError(f"bad pair {-1 - total}")
    out = {"seq": np.empty(total, np.uint32), "mask_f": np.empty(total, np.uint64),
           "mask_d": np.empty(total, np.uint64), "mass": np.empty(total, np.float64),
           "n_var": np.empty(total, np.uint8), "id_f": np.empty(total, np.uint64),
           "id_d": np.empty(total, np.uint64), "mass32_f": np.empty(total, np.float32),
           "mass32_d": np.empty(total, np.float32)}
    got = L.vc_expand_pairs(*args, *[ptr(out[k]) for k in ("seq", "mask_f", "mask_d", "mass", "n_var", "id_f",
                                                             "id_d", "mass32_f", "mass32_d")])
    if got != total:
        raise RuntimeError("vc_expand_pairs: inconsistent form count")
    return out


class _Core:
    """Namespace object standing in for the reference's ``vulcan_core`` extension module."""
    SAGE_COMMIT = SAGE_COMMIT
    RESIDUE_F64 = RESIDUE_F64.tolist()
    H2O_F64 = H2O_F64
    NTERM_BIT = NTERM_BIT
    digest_fasta = staticmethod(digest_fasta)
    expand_pairs = staticmethod(expand_pairs)
    peptidoform_id = staticmethod(peptidoform_id)


core = _Core()
