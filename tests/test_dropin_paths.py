"""The package is a drop-in beside the reference's own: with this package first on sys.path and the reference's
after it, ``vulcan.gpu.engine`` / ``vulcan.index.build`` / ``vulcan.stats.tdc`` are this package's, while the
reference's other modules -- the callers of the search path (``vulcan.ptm.search``, ``vulcan.gpu.family``,
``vulcan.cohort``) and its neighbours (``vulcan.rescore``, ``vulcan.io``) -- still import, and the callers bind to
this package's engine.  Uses the reference installed in baseline/_ref (skipped when it is not installed)."""
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
import vulcan.rescore.post, vulcan.io.store, vulcan.ptm.search as PS, vulcan.gpu.family as F, vulcan.cohort
out = {"engine": E.__file__, "build": B.__file__, "tdc": T.__file__, "post": vulcan.rescore.post.__file__,
       "store": vulcan.io.store.__file__, "ptm": PS.__file__, "family": F.__file__,
       "ptm_engine_is_ours": PS.E is E, "family_engine_is_ours": F.E is E, "version": vulcan.__version__}
print(json.dumps(out))
"""


def test_reference_modules_import_beside_the_b200_package():
    import json
    r = subprocess.run([sys.executable, "-c", PROBE, PKG, REF], capture_output=True, text=True, timeout=300,
                       env={**os.environ, "PYTHONPATH": ""}, cwd="/")
    assert r.returncode == 0, r.stderr[-3000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("engine", "build", "tdc"):
        assert d[k].startswith(PKG), (k, d[k])
    for k in ("post", "store", "ptm", "family"):
        assert d[k].startswith(REF), (k, d[k])
    assert d["ptm_engine_is_ours"] and d["family_engine_is_ours"]
    assert d["version"] == "0.0.1"
