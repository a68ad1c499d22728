"""B200-native DDA search hot path: index build, K0 peak view, hypotheses, K1 fragment-index counting,
top-K with pair closure, K2 exact rescoring, PSM ranking.  Module names mirror the reference's ``vulcan``."""
