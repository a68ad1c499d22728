"""L1 proteome index builder (same entry points as the reference's ``vulcan/index/build.py``).

    python -m vulcan.index.build --fasta a.fasta [b.fasta ...] --out DIR

Entry points ``default_params``, ``content_hash``, ``build``, ``L1Index``, ``read_labels``; the files and columns
are the reference's (``build.py:13-21``), because the reference's consumers read them:

  peptidoforms.arrow  pf_id u64, mass32 f32 (Sage f32), seq_off i64, length u8, mask u64, n_var u8, missed u8,
                      partner i64 (row of the target/decoy pair partner; partner[partner[i]] == i)
  residues.npy        u8 residues of all rows in row order (rows point into it with seq_off/length)
  labels.arrow        pf_id, family, entrap_seed, is_decoy, is_entrapment, tdc_pair, entrap_pair, fwd_seq, target_seq
  proteins.arrow      target peptide -> protein CSR
  meta.json           params, counts, timings

Output contract (what the search and the statistics rely on):
  * rows are ordered by (Sage f32 mass, pf_id), so storage order depends on content only, and the rows of a
    precursor window are one contiguous range (``build.py:168``);
  * every expanded form gives two rows, one per side of its target/decoy pair, and ``partner`` links them;
  * the index side (peptidoforms + residues) does not depend on the pair order or on which side is called the
    target: a build with the pair list shuffled and the roles swapped is bit-identical (``build.py:78-82``);
  * the labels follow each row's own sequence.

How it is computed here: the pair list is a table of per-pair attributes (side sequences, permutation, true
forward, family, entrapment seed, target, missed cleavages); the native expansion returns forms (pair index,
per-side mask / mass / id); every row is (form, side), so each output column is one gather of a per-form or
per-pair attribute through the row's (form, side) coordinates, taken directly in the sorted row order.
"""
from __future__ import annotations

import argparse
import dataclasses
import hashlib
import json
import os
import time

import numpy as np
import pyarrow as pa

from . import decoys as D
from ._core import core

INDEX_VERSION = "vulcan-l1-0.1"
FAMILY = {"T": 0, "E": 1, "DT": 2, "DE": 3}


def _write(table: pa.Table, path: str) -> None:
    with pa.OSFile(path + ".partial", "wb") as sink, pa.ipc.new_file(sink, table.schema) as w:
        w.write_table(table)
    os.replace(path + ".partial", path)


def _read(path: str) -> pa.Table:
    with pa.OSFile(path, "rb") as src:
        return pa.ipc.open_file(src).read_all()


def default_params() -> dict:
    """Search-space defaults of the reference (``build.py:52-63``): trypsin KR/P, 2 missed, length 7-50,
    500-5000 Da, carbamidomethyl-C static, Met-oxidation variable (<= 2)."""
    return {
        "enzyme": {"cleave_at": "KR", "restrict": "P", "c_terminal": True, "missed_cleavages": 2,
                   "min_len": 7, "max_len": 50},
        "static_mods": {"C": 57.021464},
        "variable_mods": {"M": 15.9949},
        "max_variable_mods": 2,
        "peptide_min_mass": 500.0, "peptide_max_mass": 5000.0,
        "decoy_seed": D.DECOY_SEED, "entrap_seeds": [], "id_seed": 0,
    }


def content_hash(fasta_paths, params) -> str:
    """Hash of the inputs that define an index: FASTA bytes, parameters, index version, Sage revision."""
    h = hashlib.sha256()
    for path in fasta_paths:
        with open(path, "rb") as fh:
            while True:
                block = fh.read(1 << 22)
                if not block:
                    break
                h.update(block)
    for part in (json.dumps(params, sort_keys=True), INDEX_VERSION, core.SAGE_COMMIT):
        h.update(part.encode())
    return h.hexdigest()[:16]


# ------------------------------------------------------------------------------------------------ string tables
class _Strings:
    """A list of ASCII strings as one byte buffer plus offsets (the form every column below is gathered from)."""

    def __init__(self, strs):
        strs = list(strs)
        self.n = len(strs)
        self.data = np.frombuffer("".join(strs).encode(), np.uint8)
        self.lens = np.fromiter(map(len, strs), np.int64, self.n)
        self.off = np.concatenate([[0], np.cumsum(self.lens)]).astype(np.int64)

    def gather_bytes(self, idx: np.ndarray):
        """(bytes of strings idx concatenated, their offsets)."""
        ln = self.lens[idx]
        off = np.concatenate([[0], np.cumsum(ln)]).astype(np.int64)
        src = np.repeat(self.off[:-1][idx] - off[:-1], ln) + np.arange(off[-1], dtype=np.int64)
        return self.data[src], off

    def arrow(self, idx: np.ndarray) -> pa.Array:
        body, off = self.gather_bytes(idx)
        return pa.Array.from_buffers(pa.large_string(), len(idx), [None, pa.py_buffer(off), pa.py_buffer(body)])


# ------------------------------------------------------------------------------------------------ pair table
@dataclasses.dataclass
class _PairTable:
    """The target/decoy pairs in the order handed to the expansion.

    Side A is expanded as the expansion's "forward" member and side B through the pair's permutation.  ``a_decoy``:
    side A holds the decoys (the role-swapped build)."""
    side_a: list
    side_b: list
    perm_flat: np.ndarray
    perm_off: np.ndarray
    forward: list         # the true forward sequence of each pair
    family: np.ndarray    # u8 family code of the forward sequence ("T" or "E")
    seed: np.ndarray      # i32 entrapment seed (0 for targets)
    target: list          # the target sequence the forward was derived from
    missed: np.ndarray    # u8 missed cleavages of that target in the digest
    a_decoy: bool


def _forward_families(targets: list, p: dict):
    """{forward sequence: (family, seed, target)}: the targets themselves and, per entrapment seed, the paired
    entrapment peptides (``build.py:96-110``); plus the entrapment statistics."""
    fam = {t: ("T", 0, t) for t in targets}
    taken = set(targets)
    stats = {}
    for seed in p["entrap_seeds"]:
        made, n_redraw, n_drop = D.make_entrapment(targets, seed, taken)
        stats[str(seed)] = {"n": len(made), "redrawn": n_redraw, "dropped_unpairable": n_drop}
        fam.update({ent: ("E", seed, t) for t, (ent, _) in made.items()})
    return fam, stats


def _pair_table(families: dict, decoys: dict, missed_of: dict, shuffle_seed, swap: bool) -> _PairTable:
    """Pairs of every forward peptide that has a decoy, in sorted forward order, then permuted by the G0
    ``shuffle_seed``; ``swap`` exchanges the sides (each explicit permutation inverted; the pseudo-reverse is its
    own inverse)."""
    fwd = sorted(f for f in families if f in decoys)
    order = np.arange(len(fwd)) if shuffle_seed is None else np.random.default_rng(shuffle_seed).permutation(len(fwd))
    fwd = [fwd[i] for i in order.tolist()]
    dec = [decoys[f][0] for f in fwd]
    perms = [decoys[f][1] for f in fwd]
    if swap:
        perms = [None if q is None else np.argsort(q).astype(np.uint8) for q in perms]
    sizes = np.fromiter((0 if q is None else len(q) for q in perms), np.int64, len(perms))
    explicit = [q for q in perms if q is not None]
    info = [families[f] for f in fwd]
    return _PairTable(
        side_a=dec if swap else fwd, side_b=fwd if swap else dec,
        perm_flat=np.concatenate(explicit).astype(np.uint8) if explicit else np.zeros(0, np.uint8),
        perm_off=np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64),
        forward=fwd,
        family=np.fromiter((FAMILY[x[0]] for x in info), np.uint8, len(info)),
        seed=np.fromiter((x[1] for x in info), np.int32, len(info)),
        target=[x[2] for x in info],
        missed=np.fromiter((missed_of[x[2]] for x in info), np.uint8, len(info)),
        a_decoy=swap)


def _target_key(seq: str) -> int:
    return int.from_bytes(hashlib.blake2b(seq.encode(), digest_size=8).digest(), "little")


# ------------------------------------------------------------------------------------------------ rows
def _row_coordinates(forms: dict):
    """Rows as (form, side) coordinates in the canonical (mass32, pf_id) order.  Returns (form, side, order)
    where row r of the output is form[r] on side[r] (0 = side A) and order is the permutation of the unsorted
    side-major row list (side A rows of all forms, then side B)."""
    n = len(forms["seq"])
    mass = np.stack([forms["mass32_f"], forms["mass32_d"]]).ravel()
    ids = np.stack([forms["id_f"], forms["id_d"]]).ravel()
    if np.unique(ids).size != ids.size:
        raise RuntimeError("peptidoform id collision")
    order = np.lexsort((ids, mass))
    return order % n, order // n, order


def build(fasta_paths, out_dir: str, params: dict | None = None, workers: int | None = None,
          shuffle_rows_seed: int | None = None, swap_labels: bool = False) -> dict:
    """Build the index (the reference's ``build.py:78-248`` contract).  ``shuffle_rows_seed`` / ``swap_labels``
    permute the pair list and swap the target/decoy sides of every pair; the index side comes out bit-identical
    (G0 invariance), only the labels may differ.  ``workers`` is accepted for signature compatibility."""
    p = default_params()
    p.update(params or {})
    clock = {"t": time.perf_counter()}
    t_start = clock["t"]
    timing = {}

    def lap(name):
        now = time.perf_counter()
        timing[name] = now - clock["t"]
        clock["t"] = now

    e = p["enzyme"]
    text = "".join(open(f).read() for f in fasta_paths)
    dg = core.digest_fasta(text, e["missed_cleavages"], e["min_len"], e["max_len"], e["cleave_at"],
                           e["restrict"], e["c_terminal"])
    targets = list(dg["keys"])
    missed_of = dict(zip(targets, np.asarray(dg["missed"]).tolist()))
    lap("digest_s")

    families, ent_stats = _forward_families(targets, p)
    decoys, n_dec_shuffled = D.make_decoys(sorted(families), p["decoy_seed"])
    lap("families_s")

    pt = _pair_table(families, decoys, missed_of, shuffle_rows_seed, swap_labels)
    forms = core.expand_pairs(pt.side_a, pt.side_b, pt.perm_flat, pt.perm_off, sorted(p["static_mods"].items()),
                              sorted(p["variable_mods"].items()), p["max_variable_mods"], p["peptide_min_mass"],
                              p["peptide_max_mass"], p["id_seed"], site_limits=p.get("site_limits"))
    lap("expand_s")

    # ---- index side: every column gathered through (form, side) in sorted order
    n_forms = len(forms["seq"])
    form, side, order = _row_coordinates(forms)
    pair = forms["seq"].astype(np.int64)[form]
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    partner = rank[np.where(order < n_forms, order + n_forms, order - n_forms)]
    a_str, b_str = _Strings(pt.side_a), _Strings(pt.side_b)
    both = _Strings([])                 # side A sequences then side B sequences, one string table
    both.data = np.concatenate([a_str.data, b_str.data])
    both.lens = np.concatenate([a_str.lens, b_str.lens])
    both.off = np.concatenate([a_str.off[:-1], a_str.off[-1] + b_str.off]).astype(np.int64)
    residues, seq_off = both.gather_bytes(pair + side * len(pt.side_a))
    per_side = lambda f, d: np.where(side == 0, forms[f][form], forms[d][form])
    pf_id = per_side("id_f", "id_d")
    idx_tbl = pa.table({
        "pf_id": pa.array(pf_id, pa.uint64()),
        "mass32": pa.array(per_side("mass32_f", "mass32_d"), pa.float32()),
        "seq_off": pa.array(seq_off[:-1], pa.int64()),
        "length": pa.array(a_str.lens[pair].astype(np.uint8), pa.uint8()),
        "mask": pa.array(per_side("mask_f", "mask_d"), pa.uint64()),
        "n_var": pa.array(forms["n_var"][form], pa.uint8()),
        "missed": pa.array(pt.missed[pair], pa.uint8()),
        "partner": pa.array(partner, pa.int64()),
    })
    lap("arrays_s")

    # ---- labels: a row is a decoy when it sits on the decoy side of its pair
    is_decoy = (side == 0) if pt.a_decoy else (side == 1)
    family = pt.family[pair] + np.where(is_decoy, 2, 0).astype(np.uint8)
    fwd_str = _Strings(pt.forward)
    tgt_str = _Strings(pt.target)
    tgt_key = np.fromiter(map(_target_key, pt.target), np.uint64, len(pt.target))
    lab = pa.table({
        "pf_id": pa.array(pf_id, pa.uint64()),
        "family": pa.array(family.astype(np.uint8)),
        "entrap_seed": pa.array(pt.seed[pair], pa.int32()),
        "is_decoy": pa.array(is_decoy),
        "is_entrapment": pa.array((family % 2) == 1),
        "tdc_pair": pa.array(np.where(is_decoy, pf_id[partner], pf_id), pa.uint64()),
        "entrap_pair": pa.array(tgt_key[pair], pa.uint64()),
        "fwd_seq": fwd_str.arrow(pair),
        "target_seq": tgt_str.arrow(pair),
    })
    prot_off = np.asarray(dg["prot_off"])
    prot = pa.table({
        "peptide": pa.array(targets, pa.string()),
        "prot_off": pa.array(prot_off[:-1], pa.int64()),
        "prot_len": pa.array(np.diff(prot_off), pa.int64()),
    })
    os.makedirs(out_dir, exist_ok=True)
    _write(idx_tbl, os.path.join(out_dir, "peptidoforms.arrow"))
    np.save(os.path.join(out_dir, "residues.npy"), residues)
    _write(lab, os.path.join(out_dir, "labels.arrow"))
    _write(prot, os.path.join(out_dir, "proteins.arrow"))
    np.save(os.path.join(out_dir, "protein_idx.npy"), dg["prot_idx"])
    with open(os.path.join(out_dir, "accessions.txt"), "w") as fh:
        fh.write("\n".join(dg["accessions"]) + "\n")
    timing["total_s"] = time.perf_counter() - t_start
    by_family = np.bincount(family.astype(np.int64), minlength=4)
    meta = {
        "index_version": INDEX_VERSION, "sage_commit": core.SAGE_COMMIT, "params": p,
        "fasta": [os.path.abspath(f) for f in fasta_paths],
        "content_hash": content_hash(fasta_paths, p),
        "n_targets": len(targets), "n_nonstandard_dropped": int(dg["n_nonstandard"]),
        "n_forward_peptides": len(pt.forward), "n_decoy_shuffled": n_dec_shuffled,
        "n_forward_without_decoy": len(families) - len(pt.forward),
        "entrapment": ent_stats,
        "n_peptidoforms": int(order.size),
        "n_peptidoforms_by_family": {k: int(by_family[v]) for k, v in FAMILY.items()},
        "timing_s": timing,
        "g0_test_knobs": {"shuffle_rows_seed": shuffle_rows_seed, "swap_labels": swap_labels},
    }
    with open(os.path.join(out_dir, "meta.json"), "w") as fh:
        json.dump(meta, fh, indent=1)
    return meta


class L1Index:
    """Index side of a built L1 index (label-free), ``build.py:424-450``."""

    def __init__(self, path: str):
        self.path = path
        t = _read(os.path.join(path, "peptidoforms.arrow"))
        for name in ("pf_id", "mass32", "seq_off", "length", "mask", "n_var", "missed", "partner"):
            setattr(self, name, t.column(name).to_numpy())
        self.partners = [self.partner] + [t.column(f"partner_{j}").to_numpy()
                                          for j in range(1, 64) if f"partner_{j}" in t.column_names]
        self.residues = np.load(os.path.join(path, "residues.npy"))
        with open(os.path.join(path, "meta.json")) as fh:
            self.meta = json.load(fh)

    def __len__(self):
        return len(self.pf_id)

    def sequence(self, i: int) -> str:
        o = int(self.seq_off[i])
        return self.residues[o:o + int(self.length[i])].tobytes().decode()


def read_labels(path: str):
    """Labels are read only by the statistics stage, never by the search."""
    return _read(os.path.join(path, "labels.arrow"))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--fasta", nargs="+", required=True)
    ap.add_argument("--out", required=True)
    ap.add_argument("--entrap-seeds", nargs="*", type=int, default=[])
    a = ap.parse_args(argv)
    meta = build(a.fasta, a.out, {"entrap_seeds": a.entrap_seeds})
    print(json.dumps({k: v for k, v in meta.items() if k != "params"}, indent=1))


if __name__ == "__main__":
    main()
