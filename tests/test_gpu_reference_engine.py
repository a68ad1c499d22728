"""The reference's own engine (``vulcan/gpu/engine.py``, installed unchanged in baseline/_ref) bound to this
library through the stub INTEGRATION.md section 1 gives: the reference's ctypes signatures (``_lib._SIGS``) applied
to ``libvulcan_b200.so``.  Its ``search`` must return the same PSM tables as the same engine bound to the
reference's own kernels (``vulcan/gpu/kernels.cu`` compiled unchanged into oracle/_ref by ``make -C oracle ref``):
the reference-compatible entry points (fragment count / emit of its CSR, its K1 with the threshold append, K2) are
exact replacements.  Runs on the mini fixture (three parameter sets) and on a 2,000-spectrum run of the small
workload."""
import ctypes as C
import importlib
import os
import sys
import tempfile
import types

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
REF = os.path.join(ROOT, "baseline", "_ref")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libvulcan_kernels_ref.so")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (os.path.isfile(os.path.join(REF, "vulcan", "gpu", "engine.py"))
                                      and os.path.isfile(REF_SO)),
                                 reason="needs the reference in baseline/_ref and its kernels in oracle/_ref")]
STATIC = {"C": 57.021464}
VAR = {"M": 15.9949}


@pytest.fixture(scope="module")
def ref_engine():
    """The reference's vulcan.gpu package loaded under another name (it uses relative imports), and a switch that
    binds its ``_lib`` to a shared object with the reference's own signatures."""
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    pkg = types.ModuleType("vulcan_reference")
    pkg.__path__ = [os.path.join(REF, "vulcan")]
    sys.modules["vulcan_reference"] = pkg
    K = importlib.import_module("vulcan_reference.gpu._lib")
    E = importlib.import_module("vulcan_reference.gpu.engine")
    libs = {}

    def bind(path):
        if path not in libs:
            L = C.CDLL(path)
            for name, args in K._SIGS.items():   # the reference's own argument lists, unchanged
                f = getattr(L, name)
                f.argtypes = args
                f.restype = C.c_int
            libs[path] = L
        K._lib = libs[path]
    yield E, bind
    sys.modules.pop("vulcan_reference", None)


def _both(E, bind, l1, sp, p):
    from vulcan._native import GPU_SO
    out = {}
    for name, so in (("reference kernels", REF_SO), ("b200", GPU_SO)):
        bind(so)
        gi = E.GpuIndex(l1, p, STATIC, VAR)
        out[name] = E.search(sp, gi, l1, p, report=3)[0]
    return out["reference kernels"], out["b200"]


@pytest.mark.parametrize("name", ("da", "ppm", "ppm_mfz"))
def test_reference_engine_on_b200_library_equals_its_own_kernels(ref_engine, mini, name):
    E, bind = ref_engine
    from tests.golden.make_golden import PARAM_SETS
    l1, sp, _ = mini
    p = E.SearchParams(**PARAM_SETS[name])
    a, b = _both(E, bind, l1, sp, p)
    assert a.num_rows > 0
    assert a.equals(b), name


def test_reference_engine_small_workload(ref_engine):
    E, bind = ref_engine
    from oracle.parity import subset
    from vulcan import synth
    from vulcan.index.build import L1Index, read_labels
    w = synth.WORKLOADS["small"]
    d = synth.build_index(w, os.environ.get("VULCAN_BENCH_CACHE",
                                            os.path.join(tempfile.gettempdir(), "vulcan_bench_cache")))
    l1 = L1Index(d)
    sp = subset(synth.simulate_run(l1, read_labels(d), w, seed=w.spectra_seed)[0], 2000)
    q = w.search_params()
    p = E.SearchParams(**{k: getattr(q, k) for k in E.SearchParams.__dataclass_fields__})
    a, b = _both(E, bind, l1, sp, p)
    assert a.num_rows > 1000
    assert a.equals(b)
    assert np.array_equal(a.column("pf_row").to_numpy(), b.column("pf_row").to_numpy())
