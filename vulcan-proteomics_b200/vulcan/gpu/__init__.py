"""GPU search: K0 peak view, hypotheses, K1 fragment-index counting, top-K, K2 rescoring, PSM table."""
