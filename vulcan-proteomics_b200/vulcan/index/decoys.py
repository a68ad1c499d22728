"""Peptide-level decoys for the L1 index.

Mirrors ``vulcan/index/decoys.py`` of the reference (same function names, arguments and results):

* decoy = pseudo-reverse with the C-terminal residue kept in place (``decoys.py:28-29``); when that is a
  palindrome, equals a forward peptide, or repeats an earlier decoy, the decoy is the C-term-fixed shuffle drawn
  from ``hash(peptide, seed, attempt)`` (``decoys.py:109-132``).
* the shuffle is a numpy ``Generator`` seeded from an 8-byte blake2b digest of ``"peptide|seed|attempt"``
  and applied to ``arange(n - 1)`` (``decoys.py:32-43``).  The recipe has to be the same draw for the decoys to be
  the same peptides, so the steps are kept; the code is written here from that description.

Everything is processed in sorted order, so the result does not depend on input order.
"""
from __future__ import annotations

import hashlib
import os

import numpy as np

DECOY_SEED = 1001
STD_AA = set("ACDEFGHIKLMNPQRSTVWY")


def pseudo_reverse(pep: str) -> str:
    """Reverse every residue except the last one (the protease C-terminal residue stays put)."""
    head = pep[:-1]
    return head[::-1] + pep[-1:]


def _seeded_generator(*parts) -> np.random.Generator:
    digest = hashlib.blake2b("|".join(str(p) for p in parts).encode(), digest_size=8).digest()
    return np.random.default_rng(int.from_bytes(digest, "little"))


def hash_shuffle_perm(pep: str, seed: int, attempt: int = 0) -> np.ndarray:
    """Permutation ``q`` with ``decoy[j] = pep[q[j]]`` of the C-term-fixed shuffle for (pep, seed, attempt)."""
    n = len(pep)
    head = np.arange(n - 1)
    _seeded_generator(pep, seed, attempt).shuffle(head)
    return np.append(head, n - 1).astype(np.uint8)


def apply_perm(pep: str, perm) -> str:
    return "".join(pep[int(i)] for i in perm)


def hash_shuffle(pep: str, seed: int, attempt: int = 0) -> str:
    return apply_perm(pep, hash_shuffle_perm(pep, seed, attempt))


def _pseudo_reverse_all(peps: list[str]) -> list[str]:
    """pseudo_reverse of every peptide, vectorised over a fixed-width byte matrix."""
    if not peps:
        return []
    lens = np.fromiter((len(q) for q in peps), np.int64, len(peps))
    w = int(lens.max())
    flat = np.frombuffer("".join(peps).encode(), np.uint8)
    off = np.zeros(len(peps) + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    col = np.arange(w)
    # source column of output column j: n-2-j for j < n-1, n-1 for j = n-1
    src = np.where(col[None, :] < lens[:, None] - 1, lens[:, None] - 2 - col[None, :], lens[:, None] - 1)
    valid = col[None, :] < lens[:, None]
    mat = np.where(valid, flat[np.clip(off[:-1, None] + src, 0, len(flat) - 1)], 0).astype(np.uint8)
    return [x.decode() for x in np.ascontiguousarray(mat).view(f"S{w}").ravel().tolist()]


def _make_decoys_sequential(forward: list[str], seed: int, max_tries: int):
    fwd = set(forward)
    used: set[str] = set()
    out: dict[str, tuple[str, np.ndarray | None]] = {}
    n_shuffled = 0
    for pep in sorted(forward):
        dec, perm = pseudo_reverse(pep), None
        attempt = 0
        while dec == pep or dec in fwd or dec in used:
            if attempt >= max_tries:
                dec = None
                break
            perm = hash_shuffle_perm(pep, seed, attempt)
            dec = apply_perm(pep, perm)
            attempt += 1
        if attempt:
            n_shuffled += 1
        if dec is not None:
            out[pep] = (dec, perm)
            used.add(dec)
    return out, n_shuffled


def make_decoys(forward: list[str], seed: int = DECOY_SEED, max_tries: int = 50):
    """Pseudo-reverse decoys of every forward peptide, hash shuffles on collision.

    Returns ``({forward: (decoy, perm or None)}, n_shuffled)``; ``perm`` None means the pseudo-reverse.
    Follows ``vulcan/index/decoys.py:109-132``: peptides in sorted order; a decoy that equals its peptide, any
    forward peptide, or an earlier decoy is replaced by shuffle attempts ``k = 0 .. max_tries-1``; a peptide whose
    every attempt collides gets no decoy.  Pseudo-reverses of distinct peptides are distinct, so only the colliding
    peptides need the sequential rule; if a shuffle lands on a later peptide's pseudo-reverse, the whole list is
    redone sequentially.
    """
    srt = sorted(set(forward))
    rev = _pseudo_reverse_all(srt)
    fwd = set(srt)
    bad = [i for i, (q, d) in enumerate(zip(srt, rev)) if d == q or d in fwd]
    out = {q: (d, None) for q, d in zip(srt, rev)}
    if not bad:
        return out, 0
    rev_pos = {d: i for i, d in enumerate(rev)}
    bad_set = set(bad)
    shuffled: set[str] = set()
    for i in bad:
        pep = srt[i]
        dec, perm, attempt = rev[i], None, 0
        while (dec == pep or dec in fwd or dec in shuffled or
               (dec in rev_pos and rev_pos[dec] < i and rev_pos[dec] not in bad_set)):
            if attempt >= max_tries:
                dec = None
                break
            perm = hash_shuffle_perm(pep, seed, attempt)
            dec = apply_perm(pep, perm)
            attempt += 1
        if dec is None:
            del out[pep]
            continue
        if dec in rev_pos and rev_pos[dec] > i and rev_pos[dec] not in bad_set:
            return _make_decoys_sequential(srt, seed, max_tries)
        out[pep] = (dec, perm)
        shuffled.add(dec)
    return out, len(bad)


def make_entrapment(targets: list[str], seed: int, taken: set[str], workers: int = 1, max_tries: int = 200):
    """Paired shuffled entrapment peptides (``vulcan/index/decoys.py:72-106``).

    An entrapment of target t is the C-term-fixed hash shuffle of t, redrawn while it equals t, a target, an
    earlier entrapment, the pseudo-reverse of a target, its own pseudo-reverse, or when its pseudo-reverse is a
    target or taken.  ``taken`` is updated in place.  Returns ``({target: (entrapment, perm)}, n_redrawn,
    n_dropped)``.  ``workers`` is accepted for signature compatibility; the draw is sequential here.
    """
    targets = sorted(targets)
    tset = set(targets)
    rev_t = {pseudo_reverse(t) for t in targets}
    out: dict[str, tuple[str, np.ndarray]] = {}
    n_redraw = n_drop = 0

    def bad(e: str) -> bool:
        pe = pseudo_reverse(e)
        return e in taken or e in tset or e in rev_t or pe == e or pe in taken or pe in tset

    for t in targets:
        perm = hash_shuffle_perm(t, seed, 0)
        e = apply_perm(t, perm)
        k = 0
        while bad(e) or e == t:
            k += 1
            if k > max_tries:
                e = None
                break
            perm = hash_shuffle_perm(t, seed, k)
            e = apply_perm(t, perm)
        if e is None:
            n_drop += 1
            continue
        n_redraw += k > 0
        out[t] = (e, perm)
        taken.add(e)
    return out, n_redraw, n_drop


def default_workers() -> int:
    return len(os.sched_getaffinity(0))
