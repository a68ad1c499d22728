"""The package is a drop-in beside the reference's own: with this package first on sys.path and the reference's
after it, ``vulcan.gpu.engine`` / ``vulcan.index.build`` / ``vulcan.stats.tdc`` are this package's, while the
reference's other modules -- the callers of the search path (``vulcan.gpu.family``, ``vulcan.cohort``) and its
neighbours (``vulcan.rescore``, ``vulcan.io``, ``vulcan.ptm.localize``) -- still import, and the callers bind to
this package's engine (``vulcan.ptm.search``, the open / mass-offset modes, is this package's).  Uses the reference installed in baseline/_ref (skipped when it is not installed)."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
PKG = os.path.join(ROOT, "vulcan-proteomics_b200")
REF = os.path.join(ROOT, "baseline", "_ref")

pytestmark = pytest.mark.skipif(not os.path.isfile(os.path.join(REF, "vulcan", "gpu", "engine.py")),
                                reason="the reference is not installed in baseline/_ref")

PROBE = r"""
import os, sys, json
sys.path[:0] = [sys.argv[1], sys.argv[2]]
import vulcan, vulcan.gpu.engine as E, vulcan.index.build as B, vulcan.stats.tdc as T
import vulcan.rescore.post, vulcan.io.store, vulcan.ptm.search as PS, vulcan.ptm.localize as LOC
import vulcan.gpu.family as F, vulcan.cohort
out = {"engine": E.__file__, "build": B.__file__, "tdc": T.__file__, "post": vulcan.rescore.post.__file__,
       "store": vulcan.io.store.__file__, "ptm": PS.__file__, "localize": LOC.__file__, "family": F.__file__,
       "ptm_engine_is_ours": PS.E is E, "family_engine_is_ours": F.E is E, "version": vulcan.__version__}
print(json.dumps(out))
"""


def test_reference_modules_import_beside_the_b200_package():
    import json
    r = subprocess.run([sys.executable, "-c", PROBE, PKG, REF], capture_output=True, text=True, timeout=300,
                       env={**os.environ, "PYTHONPATH": ""}, cwd="/")
    assert r.returncode == 0, r.stderr[-3000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("engine", "build", "tdc", "ptm"):
        assert d[k].startswith(PKG), (k, d[k])
    for k in ("post", "store", "localize", "family"):
        assert d[k].startswith(REF), (k, d[k])
    assert d["ptm_engine_is_ours"] and d["family_engine_is_ours"]
    assert d["version"] == "0.0.1"


def test_mode_hypotheses_equal_the_reference():
    """``vulcan.ptm.search.make_mode_hypotheses`` (closed, mass-offset and open hypotheses and their row windows)
    equals the reference's on the mini fixture's spectra, for offsets and an open window together."""
    import importlib
    import types
    import numpy as np
    from tests.conftest import GOLDEN
    fx = dict(np.load(os.path.join(GOLDEN, "mini_fixture.npz")))
    pkg = types.ModuleType("vulcan_reference")
    pkg.__path__ = [os.path.join(REF, "vulcan")]
    sys.modules["vulcan_reference"] = pkg
    try:
        RH = importlib.import_module("vulcan_reference.gpu.host")
        src = open(os.path.join(REF, "vulcan", "ptm", "search.py")).read()
        # the reference module imports torch-side engine code at its top; only its hypothesis function is needed
        ns = {"np": np, "make_hypotheses": RH.make_hypotheses, "SearchParams": RH.SearchParams,
              "MODE_CLOSED": 0, "MODE_OFFSET": 1, "MODE_OPEN": 2}
        start = src.index("def make_mode_hypotheses")
        end = src.index("\ndef ", start + 10)
        exec(compile("from __future__ import annotations\n" + src[start:end], "reference make_mode_hypotheses",
                     "exec"), ns)
        from vulcan.gpu.host import SearchParams, Spectra
        from vulcan.ptm import search as PS
        sp = Spectra("mini", fx["sp_scan"], fx["sp_index"], fx["sp_rt"], fx["sp_precursor_mz"], fx["sp_charge"],
                     fx["sp_mz"], fx["sp_intensity"], fx["sp_offsets"])
        valid = np.ones(len(sp), bool)
        valid[::5] = False
        mass = fx["idx_mass32"]
        for kw in (dict(offsets=(15.9949, -17.0265, 79.96633), open_da=(-150.0, 500.0)), dict(offsets=()),
                   dict(open_da=(-2.0, 30.0))):
            mine = PS.make_mode_hypotheses(sp, valid, mass, SearchParams(isotope_errors=(-1, 2)), PS.ModeParams(**kw))
            ref_mp = types.SimpleNamespace(offsets=kw.get("offsets", ()), open_da=kw.get("open_da"))
            want = ns["make_mode_hypotheses"](sp, valid, mass, RH.SearchParams(isotope_errors=(-1, 2)), ref_mp)
            assert set(mine) == set(want)
            for k in want:
                assert mine[k].dtype == want[k].dtype, k
                assert np.array_equal(mine[k], want[k], equal_nan=True), (k, kw)
    finally:
        sys.modules.pop("vulcan_reference", None)
