"""Target-decoy competition and q-values (reference ``vulcan/stats/tdc.py:45-195``), used to count the PSMs a
search accepts at a q-value threshold.

Conventions as in the reference: higher scores win, NaN scores count as -inf; the FDR at threshold s is
``factor * (D(s) + 1) / max(T(s), 1)`` over everything scoring >= s (tied items share one threshold); q-values
are its reverse running minimum, capped at 1.  Ties inside a competition go to the smallest ``tiebreak`` key.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from ._util import as_codes, make_rng, segment_cumsum, segment_reverse_cummin, segment_starts


def _scores(score) -> np.ndarray:
    s = np.asarray(score, dtype=np.float64)
    return np.where(np.isnan(s), -np.inf, s)


def compete(group, score, seed=None, tiebreak=None) -> np.ndarray:
    """Row index of each group's winner (highest score, then smallest tiebreak), ordered by group key."""
    s = _scores(score)
    if len(s) == 0:
        return np.zeros(0, dtype=np.int64)
    g = as_codes(group)
    tb = make_rng(seed).random(len(s)) if tiebreak is None else np.asarray(tiebreak)
    order = np.lexsort((tb, -s, g))
    return order[segment_starts(g[order])].astype(np.int64)


def psm_competition(spectrum_id, score, seed=None, tiebreak=None) -> np.ndarray:
    return compete(spectrum_id, score, seed=seed, tiebreak=tiebreak)


def tdc_fdr_curve(score, is_decoy, factor: float = 1.0, block=None, plus_one: bool = True):
    """(fdr, targets, decoys) at each item's own score threshold, in input order."""
    s = _scores(score)
    d = np.asarray(is_decoy, dtype=bool)
    n = len(s)
    b = np.zeros(n, dtype=np.int64) if block is None else as_codes(block)
    order = np.lexsort((-s, b))
    ss, ds, bs = s[order], d[order], b[order]
    bstart = segment_starts(bs)
    n_dec = segment_cumsum(ds.astype(np.int64), bstart)
    n_tgt = segment_cumsum((~ds).astype(np.int64), bstart)
    run = bstart.copy()                       # a new threshold where the block or the score changes
    if n > 1:
        run[1:] |= ss[1:] != ss[:-1]
    run_id = np.cumsum(run) - 1
    last = np.append(np.flatnonzero(run)[1:] - 1, n - 1)[run_id]
    D, T = n_dec[last], n_tgt[last]
    fdr = factor * (D + (1.0 if plus_one else 0.0)) / np.maximum(T, 1)
    out = [np.empty(n), np.empty(n, dtype=np.int64), np.empty(n, dtype=np.int64)]
    for o, v in zip(out, (fdr, T, D)):
        o[order] = v
    return tuple(out)


def tdc_qvalues(score, is_decoy, factor: float = 1.0, block=None, plus_one: bool = True) -> np.ndarray:
    s = _scores(score)
    n = len(s)
    if n == 0:
        return np.zeros(0)
    fdr = tdc_fdr_curve(s, is_decoy, factor=factor, block=block, plus_one=plus_one)[0]
    b = np.zeros(n, dtype=np.int64) if block is None else as_codes(block)
    order = np.lexsort((-s, b))
    q = np.empty(n)
    q[order] = segment_reverse_cummin(fdr[order], segment_starts(b[order]), cap=1.0)
    return q


def count_discoveries(q, is_decoy, alpha: float) -> int:
    return int(np.count_nonzero((np.asarray(q) <= alpha) & ~np.asarray(is_decoy, dtype=bool)))


@dataclass
class DoubleCompetitionResult:
    row: np.ndarray
    pair: np.ndarray
    score: np.ndarray
    is_decoy: np.ndarray
    q: np.ndarray
    psm_winners: np.ndarray

    def accepted(self, alpha: float) -> np.ndarray:
        return self.row[(self.q <= alpha) & ~self.is_decoy]


def double_competition(spectrum_id, unit_id, pair_id, score, is_decoy, seed=None, factor: float = 1.0,
                       tiebreak=None) -> DoubleCompetitionResult:
    """Spectrum-level competition, then the best PSM per (unit, side), then each target unit against its paired
    decoy unit (shared ``pair_id``), then q-values over the pair winners."""
    s = _scores(score)
    dec = np.asarray(is_decoy, dtype=bool)
    unit = np.asarray(unit_id)
    pair = np.asarray(pair_id)
    tb = None if tiebreak is None else np.asarray(tiebreak)

    def rng(k):
        return make_rng(seed, k) if seed is not None else None
    w1 = psm_competition(spectrum_id, s, seed=rng(1), tiebreak=tb)
    key = as_codes(unit[w1]) * 2 + dec[w1].astype(np.int64)
    w2 = w1[compete(key, s[w1], seed=rng(2), tiebreak=None if tb is None else tb[w1])]
    w3 = w2[compete(pair[w2], s[w2], seed=rng(3), tiebreak=None if tb is None else tb[w2])]
    q = tdc_qvalues(s[w3], dec[w3], factor=factor)
    return DoubleCompetitionResult(row=w3, pair=pair[w3], score=s[w3], is_decoy=dec[w3], q=q, psm_winners=w1)
