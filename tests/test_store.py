"""``engine.load_store`` reads the reference's spectral store (Arrow IPC ``.vspec.arrow``, reference
``vulcan/io/store.py``) into ``Spectra`` exactly as the reference's ``engine.load_store`` does
(``vulcan/gpu/engine.py:157-168``): MS2 rows only, flat peaks with int64 offsets, unknown charge 0, missing precursor
NaN, the run name from the metadata.  The store is written by the reference's own writer (installed in baseline/_ref;
skipped when absent), with MS1 and MS2 rows interleaved over several record batches."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
PKG = os.path.join(ROOT, "vulcan-proteomics_b200")
REF = os.path.join(ROOT, "baseline", "_ref")

pytestmark = pytest.mark.skipif(not os.path.isfile(os.path.join(REF, "vulcan", "io", "store.py")),
                                reason="the reference is not installed in baseline/_ref")

PROBE = r"""
import importlib, os, sys, types
sys.path[:0] = [sys.argv[1], sys.argv[2]]
import numpy as np
from vulcan.io.store import StoreWriter            # the reference's writer (this package has no vulcan.io)
from vulcan.gpu import engine as E                  # this package's reader
path = os.path.join(sys.argv[3], "run.vspec.arrow")
rng = np.random.default_rng(5)
meta = {"store_version": "1", "run_name": "synthetic_store_run", "run_id": 7, "vendor": "none",
        "instrument_model": "none", "source_path": "none", "source_size": 0, "converter": "test",
        "converter_version": "0", "created_utc": "2026-01-01", "n_spectra": None, "n_ms1": None, "n_ms2": None,
        "n_peaks": None, "peak_order": "mz", "acquisition": "dda"}
w = StoreWriter(path, meta)
scan0 = 1
for batch in range(4):
    n = int(rng.integers(5, 40))
    lens = rng.integers(0, 300, n)
    lens[::7] = 0
    off = np.concatenate([[0], np.cumsum(lens)])
    lvl = np.where(rng.random(n) < 0.3, 1, 2).astype(np.uint8)
    pmz = np.where(lvl == 2, rng.uniform(300, 1500, n), np.nan)
    pmz[rng.random(n) < 0.1] = np.nan
    ch = rng.integers(2, 5, n).astype(np.int8)
    w.write({"scan": np.arange(scan0, scan0 + n), "ms_level": lvl, "rt_min": np.linspace(batch, batch + 1, n),
             "precursor_mz": pmz, "precursor_charge": ch, "precursor_charge_mask": rng.random(n) < 0.2,
             "peak_offsets": off, "mz": np.sort(rng.uniform(100, 2000, off[-1])).astype(np.float32),
             "intensity": rng.lognormal(5, 1, off[-1]).astype(np.float32)})
    scan0 += n
w.close()
mine = E.load_store(path)
pkg = types.ModuleType("vulcan_reference")
pkg.__path__ = [os.path.join(sys.argv[2], "vulcan")]
sys.modules["vulcan_reference"] = pkg
ref = importlib.import_module("vulcan_reference.gpu.engine").load_store(path)
assert mine.run == ref.run == "synthetic_store_run", (mine.run, ref.run)
for k in ("scan", "index", "rt", "precursor_mz", "charge", "mz", "intensity", "offsets"):
    a, b = np.asarray(getattr(mine, k)), np.asarray(getattr(ref, k))
    assert a.dtype == b.dtype, (k, a.dtype, b.dtype)
    assert np.array_equal(a, b, equal_nan=True), k
assert len(mine) > 20 and int(mine.offsets[-1]) > 1000 and (mine.charge == 0).any()
print("ok", len(mine), int(mine.offsets[-1]))
"""


def test_load_store_equals_the_reference(tmp_path):
    r = subprocess.run([sys.executable, "-c", PROBE, PKG, REF, str(tmp_path)], capture_output=True, text=True,
                       timeout=300, env={**os.environ, "PYTHONPATH": ""}, cwd="/")
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-3000:])
    assert r.stdout.strip().splitlines()[-1].startswith("ok")
