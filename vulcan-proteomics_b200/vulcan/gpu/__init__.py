"""GPU search: K0 peak view, hypotheses, K1 fragment-index counting, top-K, K2 rescoring, PSM table."""

# A drop-in for the reference's package of the same name: its other subpackages and modules (vulcan.rescore,
# vulcan.io, vulcan.ptm, ..., vulcan.gpu.family) stay importable from a reference checkout that comes later on
# sys.path; modules present here take precedence.
__path__ = __import__("pkgutil").extend_path(__path__, __name__)
