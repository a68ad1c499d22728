"""Golden vectors of the reference's target-decoy statistics (``vulcan/stats/tdc.py``, ``vulcan/stats/_util.py``),
used to pin ``vulcan.stats`` (the restatement that counts PSMs accepted at a q-value threshold).

Run with the reference checkout as the argument:  python tests/golden/make_golden_tdc.py <reference_dir>
Writes tests/golden/golden_tdc.npz: random scored PSM sets with ties (seeded), their q-values, double-competition
winners and q-values, and hash tie-break keys."""
import os
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: make_golden_tdc.py <reference_dir>")
REF = sys.argv[1]
sys.path.insert(0, REF)
from vulcan.stats import _util as RU  # noqa: E402
from vulcan.stats import tdc as R  # noqa: E402

out = {}
rng = np.random.default_rng(20240)
for t in range(8):
    n = int(rng.integers(1, 1500))
    sc = np.round(rng.normal(size=n), 1)
    if t % 3 == 0:
        sc[rng.random(n) < 0.05] = np.nan
    dec = rng.random(n) < 0.4
    spec = rng.integers(0, n // 2 + 1, n)
    unit = rng.integers(0, n // 3 + 1, n).astype(np.uint64)
    pair = unit // 2
    blk = rng.integers(0, 3, n)
    tb = RU.hash_tiebreak(unit, 11)
    r = R.double_competition(spec, unit, pair, sc, dec, seed=11, tiebreak=tb)
    for k, v in {"score": sc, "decoy": dec, "spec": spec, "unit": unit, "block": blk, "tiebreak": tb,
                 "q": R.tdc_qvalues(sc, dec), "q_block": R.tdc_qvalues(sc, dec, block=blk),
                 "dc_row": r.row, "dc_q": r.q, "dc_winners": r.psm_winners,
                 "accepted": np.array([R.count_discoveries(r.q, r.is_decoy, 0.01)])}.items():
        out[f"{t}/{k}"] = v
out["n_sets"] = np.array([8])
np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_tdc.npz"), **out)
print("wrote golden_tdc.npz")
