"""Test setup: import paths, the `gpu` marker, shared fixtures (mini fixture, reference goldens)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
PKG = os.path.join(ROOT, "vulcan-proteomics_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


class MiniL1:
    """L1Index-like object over the arrays of the mini fixture."""

    def __init__(self, fx):
        for k in fx:
            if k.startswith("idx_"):
                setattr(self, k[4:], fx[k])
        self.partners = [self.partner]

    def __len__(self):
        return len(self.pf_id)

    def sequence(self, i):
        o = int(self.seq_off[i])
        return self.residues[o:o + int(self.length[i])].tobytes().decode()


@pytest.fixture(scope="session")
def mini():
    fx = dict(np.load(os.path.join(GOLDEN, "mini_fixture.npz")))
    from vulcan.gpu.host import Spectra
    sp = Spectra("mini", fx["sp_scan"], fx["sp_index"], fx["sp_rt"], fx["sp_precursor_mz"], fx["sp_charge"],
                 fx["sp_mz"], fx["sp_intensity"], fx["sp_offsets"])
    return MiniL1(fx), sp, fx


@pytest.fixture(scope="session")
def golden_py():
    return dict(np.load(os.path.join(GOLDEN, "golden_ref_py.npz")))


@pytest.fixture(scope="session")
def golden_kernels():
    path = os.path.join(GOLDEN, "golden_ref_kernels.npz")
    if not os.path.exists(path):
        pytest.fail("golden_ref_kernels.npz missing (generate with tests/golden/make_golden_ref.py on a GPU)")
    return dict(np.load(path))


@pytest.fixture(scope="session")
def param_sets():
    from tests.golden.make_golden import PARAM_SETS
    from vulcan.gpu.host import SearchParams
    return {k: SearchParams(**v) for k, v in PARAM_SETS.items()}
