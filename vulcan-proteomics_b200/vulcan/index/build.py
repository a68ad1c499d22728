"""L1 proteome index builder (mirror of the reference's ``vulcan/index/build.py``).

    python -m vulcan.index.build --fasta a.fasta [b.fasta ...] --out DIR

Same entry points (``default_params``, ``build``, ``L1Index``, ``read_labels``), same files, same columns:

  peptidoforms.arrow  pf_id u64, mass32 f32 (Sage f32), seq_off i64, length u8, mask u64, n_var u8, missed u8,
                      partner i64 (row of the target/decoy pair partner; partner[partner[i]] == i)
  residues.npy        u8 residues of all rows in row order (rows point into it with seq_off/length)
  labels.arrow        pf_id, family, entrap_seed, is_decoy, is_entrapment, tdc_pair, entrap_pair, fwd_seq, target_seq
  proteins.arrow      target peptide -> protein CSR
  meta.json           params, counts, timings

Rows are sorted by (Sage f32 mass, pf_id) (``build.py:168``), so the storage order is content-defined and a
row window of a precursor tolerance is one contiguous range.  The search kernels only read the index side.
"""
from __future__ import annotations

import argparse
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
    h = hashlib.sha256()
    for p in fasta_paths:
        with open(p, "rb") as fh:
            for b in iter(lambda: fh.read(1 << 22), b""):
                h.update(b)
    h.update(json.dumps(params, sort_keys=True).encode())
    h.update(INDEX_VERSION.encode())
    return h.hexdigest()[:16]


def _pair_perm(fwd: str, perm) -> np.ndarray:
    """Explicit permutation array of a pair (the pseudo-reverse one when perm is None)."""
    if perm is not None:
        return np.asarray(perm, np.uint8)
    n = len(fwd)
    return np.array([n - 2 - j for j in range(n - 1)] + [n - 1], np.uint8)


def _string_column(strs: list[str], order: np.ndarray) -> pa.Array:
    """Arrow string column of strs[order] built from one byte buffer and an offsets buffer."""
    data = np.frombuffer("".join(strs).encode(), np.uint8)
    ln = np.fromiter((len(q) for q in strs), np.int64, len(strs))
    off = np.zeros(len(strs) + 1, np.int64)
    np.cumsum(ln, out=off[1:])
    ln_s = ln[order]
    off_s = np.zeros(len(order) + 1, np.int64)
    np.cumsum(ln_s, out=off_s[1:])
    gather = np.repeat(off[:-1][order] - off_s[:-1], ln_s) + np.arange(off_s[-1])
    body = data[gather]
    return pa.Array.from_buffers(pa.large_string(), len(order), [None, pa.py_buffer(off_s), pa.py_buffer(body)])


def build(fasta_paths, out_dir: str, params: dict | None = None, workers: int | None = None,
          shuffle_rows_seed: int | None = None, swap_labels: bool = False) -> dict:
    """Build the index (``build.py:78-248``).  ``shuffle_rows_seed`` / ``swap_labels`` permute the pair list and
    swap the forward/decoy roles of every pair; the index side must come out bit-identical (G0 invariance)."""
    p = default_params()
    p.update(params or {})
    t0 = time.perf_counter()
    timing = {}
    text = "".join(open(f).read() for f in fasta_paths)
    e = p["enzyme"]
    dg = core.digest_fasta(text, e["missed_cleavages"], e["min_len"], e["max_len"], e["cleave_at"],
                           e["restrict"], e["c_terminal"])
    targets = list(dg["keys"])
    timing["digest_s"] = time.perf_counter() - t0

    t1 = time.perf_counter()
    taken = set(targets)
    fwd_fam = {t: ("T", 0, t) for t in targets}
    ent_stats = {}
    for s in p["entrap_seeds"]:
        m, nr, nd = D.make_entrapment(targets, s, taken)
        ent_stats[str(s)] = {"n": len(m), "redrawn": nr, "dropped_unpairable": nd}
        for t, (ent, _) in m.items():
            fwd_fam[ent] = ("E", s, t)
    forward = sorted(fwd_fam)
    dec, n_dec_shuffled = D.make_decoys(forward, p["decoy_seed"])
    forward = [f for f in forward if f in dec]
    timing["families_s"] = time.perf_counter() - t1

    t2 = time.perf_counter()
    fw = forward
    dc = [dec[f][0] for f in fw]
    order = np.arange(len(fw))
    if shuffle_rows_seed is not None:
        order = np.random.default_rng(shuffle_rows_seed).permutation(len(fw))
    a_seq = [fw[i] for i in order]
    b_seq = [dc[i] for i in order]
    # explicit permutations only for shuffled decoys; an empty slice is the pseudo-reverse
    perm_lists = [dec[fw[i]][1] for i in order]
    if swap_labels:
        a_seq, b_seq = b_seq, a_seq
        perm_lists = [np.argsort(_pair_perm(b_seq[j], q)).astype(np.uint8) if q is not None else None
                      for j, q in enumerate(perm_lists)]
        # the inverse of the pseudo-reverse permutation is itself, so None stays None
    plens = np.fromiter((0 if q is None else len(q) for q in perm_lists), np.int64, len(perm_lists))
    poff = np.zeros(len(perm_lists) + 1, np.int64)
    np.cumsum(plens, out=poff[1:])
    explicit = [q for q in perm_lists if q is not None]
    pflat = np.concatenate(explicit).astype(np.uint8) if explicit else np.zeros(0, np.uint8)
    smods = sorted(p["static_mods"].items())
    vmods = sorted(p["variable_mods"].items())
    r = core.expand_pairs(a_seq, b_seq, pflat, poff, smods, vmods, p["max_variable_mods"],
                          p["peptide_min_mass"], p["peptide_max_mass"], p["id_seed"],
                          site_limits=p.get("site_limits"))
    timing["expand_s"] = time.perf_counter() - t2

    t3 = time.perf_counter()
    n_pairs = len(r["seq"])
    seq_i = r["seq"].astype(np.int64)
    a_bytes = np.frombuffer("".join(a_seq).encode(), np.uint8)
    b_bytes = np.frombuffer("".join(b_seq).encode(), np.uint8)
    lens = np.fromiter((len(q) for q in a_seq), np.int64, len(a_seq))
    a_off = np.zeros(len(a_seq) + 1, np.int64)
    np.cumsum(lens, out=a_off[1:])
    residues = np.concatenate([a_bytes, b_bytes])
    pf_id = np.concatenate([r["id_f"], r["id_d"]])
    mass32 = np.concatenate([r["mass32_f"], r["mass32_d"]])
    seq_off = np.concatenate([a_off[seq_i], a_off[-1] + a_off[seq_i]])
    length = np.concatenate([lens[seq_i], lens[seq_i]]).astype(np.uint8)
    mask = np.concatenate([r["mask_f"], r["mask_d"]])
    n_var = np.concatenate([r["n_var"], r["n_var"]])
    # missed cleavages: the forward target's digest count, a pair attribute
    fw_arr = np.asarray(fw, dtype=object)
    tgt_of_fw = np.asarray([fwd_fam[f][2] for f in fw], dtype=object) if ent_stats else fw_arr
    tgt_index = {t: i for i, t in enumerate(targets)}
    missed_fw = dg["missed"][np.fromiter((tgt_index[t] for t in tgt_of_fw), np.int64, len(fw))]
    missed_seq = missed_fw[order]
    missed = np.concatenate([missed_seq[seq_i], missed_seq[seq_i]])
    side_b = np.concatenate([np.zeros(n_pairs, bool), np.ones(n_pairs, bool)])
    if len(np.unique(pf_id)) != len(pf_id):
        raise RuntimeError("peptidoform id collision")
    srt = np.lexsort((pf_id, mass32))
    inv = np.empty_like(srt)
    inv[srt] = np.arange(len(srt))
    partner_unsorted = np.concatenate([np.arange(n_pairs) + n_pairs, np.arange(n_pairs)])
    partner = inv[partner_unsorted][srt]
    lens_s = length[srt].astype(np.int64)
    new_off = np.zeros(len(srt) + 1, np.int64)
    np.cumsum(lens_s, out=new_off[1:])
    gather = np.repeat(seq_off[srt] - new_off[:-1], lens_s) + np.arange(new_off[-1])
    residues_s = residues[gather]
    idx_tbl = pa.table({
        "pf_id": pa.array(pf_id[srt], pa.uint64()),
        "mass32": pa.array(mass32[srt], pa.float32()),
        "seq_off": pa.array(new_off[:-1], pa.int64()),
        "length": pa.array(length[srt], pa.uint8()),
        "mask": pa.array(mask[srt], pa.uint64()),
        "n_var": pa.array(n_var[srt], pa.uint8()),
        "missed": pa.array(missed[srt], pa.uint8()),
        "partner": pa.array(partner, pa.int64()),
    })
    timing["arrays_s"] = time.perf_counter() - t3

    fam_fw = np.fromiter((FAMILY[fwd_fam[f][0]] for f in fw), np.uint8, len(fw)) if ent_stats else \
        np.zeros(len(fw), np.uint8)
    seed_fw = np.fromiter((fwd_fam[f][1] for f in fw), np.int32, len(fw)) if ent_stats else np.zeros(len(fw), np.int32)
    fam_fwd, seed_fwd = fam_fw[order], seed_fw[order]
    is_dec = side_b if not swap_labels else ~side_b
    fam_side = np.concatenate([fam_fwd[seq_i], fam_fwd[seq_i]])
    fam = np.where(is_dec, fam_side + 2, fam_side)
    fwd_member_id = np.where(is_dec, pf_id[partner_unsorted], pf_id)
    tgt_pairs = [tgt_of_fw[i] for i in order.tolist()]
    ep = np.fromiter((int.from_bytes(hashlib.blake2b(t.encode(), digest_size=8).digest(), "little")
                      for t in tgt_pairs), np.uint64, len(tgt_pairs))
    ep = np.concatenate([ep[seq_i], ep[seq_i]])
    # string columns straight from byte buffers: the forward (true-label) sequence and its target of every row
    fwd_strs = [x if not swap_labels else y for x, y in zip(a_seq, b_seq)]
    fwd_col = _string_column([fwd_strs[i] for i in seq_i.tolist()] * 2, srt)
    tgt_col = _string_column([tgt_pairs[i] for i in seq_i.tolist()] * 2, srt)
    lab = pa.table({
        "pf_id": pa.array(pf_id[srt], pa.uint64()),
        "family": pa.array(fam[srt].astype(np.uint8)),
        "entrap_seed": pa.array(np.concatenate([seed_fwd[seq_i], seed_fwd[seq_i]])[srt], pa.int32()),
        "is_decoy": pa.array(is_dec[srt]),
        "is_entrapment": pa.array((fam[srt] % 2) == 1),
        "tdc_pair": pa.array(fwd_member_id[srt], pa.uint64()),
        "entrap_pair": pa.array(ep[srt], pa.uint64()),
        "fwd_seq": fwd_col,
        "target_seq": tgt_col,
    })
    prot = pa.table({
        "peptide": pa.array(targets, pa.string()),
        "prot_off": pa.array(dg["prot_off"][:-1], pa.int64()),
        "prot_len": pa.array(np.diff(dg["prot_off"]), pa.int64()),
    })
    os.makedirs(out_dir, exist_ok=True)
    _write(idx_tbl, os.path.join(out_dir, "peptidoforms.arrow"))
    np.save(os.path.join(out_dir, "residues.npy"), residues_s)
    _write(lab, os.path.join(out_dir, "labels.arrow"))
    _write(prot, os.path.join(out_dir, "proteins.arrow"))
    np.save(os.path.join(out_dir, "protein_idx.npy"), dg["prot_idx"])
    with open(os.path.join(out_dir, "accessions.txt"), "w") as fh:
        fh.write("\n".join(dg["accessions"]) + "\n")
    timing["total_s"] = time.perf_counter() - t0
    fams = np.bincount(fam.astype(np.int64), minlength=4)
    meta = {
        "index_version": INDEX_VERSION, "sage_commit": core.SAGE_COMMIT, "params": p,
        "fasta": [os.path.abspath(f) for f in fasta_paths],
        "content_hash": content_hash(fasta_paths, p),
        "n_targets": len(targets), "n_nonstandard_dropped": int(dg["n_nonstandard"]),
        "n_forward_peptides": len(fw), "n_decoy_shuffled": n_dec_shuffled,
        "n_forward_without_decoy": len(fwd_fam) - len(fw),
        "entrapment": ent_stats,
        "n_peptidoforms": int(len(pf_id)),
        "n_peptidoforms_by_family": {k: int(fams[v]) for k, v in FAMILY.items()},
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
        self.pf_id = t.column("pf_id").to_numpy()
        self.mass32 = t.column("mass32").to_numpy()
        self.seq_off = t.column("seq_off").to_numpy()
        self.length = t.column("length").to_numpy()
        self.mask = t.column("mask").to_numpy()
        self.n_var = t.column("n_var").to_numpy()
        self.missed = t.column("missed").to_numpy()
        self.partner = t.column("partner").to_numpy()
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
