"""The target-decoy statistics used to count accepted PSMs equal the reference's on its own golden vectors
(tests/golden/golden_tdc.npz, made by tests/golden/make_golden_tdc.py from the reference's vulcan/stats)."""
import os

import numpy as np

from vulcan.stats import _util as U
from vulcan.stats import tdc as T

G = os.path.join(os.path.dirname(__file__), "golden", "golden_tdc.npz")


def test_tdc_matches_reference_goldens():
    g = np.load(G)
    for t in range(int(g["n_sets"][0])):
        k = lambda name: g[f"{t}/{name}"]  # noqa: E731
        sc, dec, spec, unit = k("score"), k("decoy"), k("spec"), k("unit")
        tb = U.hash_tiebreak(unit, 11)
        assert np.array_equal(tb, k("tiebreak"))
        np.testing.assert_array_equal(T.tdc_qvalues(sc, dec), k("q"))
        np.testing.assert_array_equal(T.tdc_qvalues(sc, dec, block=k("block")), k("q_block"))
        r = T.double_competition(spec, unit, unit // 2, sc, dec, seed=11, tiebreak=tb)
        assert np.array_equal(r.row, k("dc_row")) and np.array_equal(r.psm_winners, k("dc_winners"))
        np.testing.assert_array_equal(r.q, k("dc_q"))
        assert T.count_discoveries(r.q, r.is_decoy, 0.01) == int(k("accepted")[0])
