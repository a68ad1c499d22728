"""PTM search modes (mass-offset, open) on the B200 kernels; the reference's other PTM modules (CONGA filtering,
localisation) stay importable from a reference checkout later on sys.path."""

__path__ = __import__("pkgutil").extend_path(__path__, __name__)
