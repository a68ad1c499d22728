"""Parity of the device search with the oracle at the benchmark configurations, not only on the mini fixture.

* Configuration 0 (``small`` workload: 2,000-protein index, 5,000 spectra, top-k 50): every spectrum.
* Configuration 1 (``human`` workload: ~5.5M-peptidoform index, 40,000-spectrum run, top-k 100): the whole run is
  searched on the device and its first 3,000 spectra are checked (the reference's own correctness run checks K1 on a
  sample of this kind, ``scripts/m2/e2_correctness.py:78-118``).

Checked, bit for bit unless noted: K0 peak view, hypotheses, dense K1 counts with the per-hypothesis scored /
matched statistics, top-K + pair closure candidate lists, K2 f32 / integer outputs, top-1 PSM per spectrum;
hyperscores within 1e-12 of the oracle's and within 1e-5 relative of the FP64-accumulation oracle.  Also the
graph-captured ``Searcher`` against ``engine.search``, and ``search_exhaustive`` (the recall judge, reference
``engine.py:500-523``) against the oracle's window candidates and K2."""
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CACHE = os.environ.get("VULCAN_BENCH_CACHE", os.path.join(tempfile.gettempdir(), "vulcan_bench_cache"))
STATIC = {"C": 57.021464}
FP64_RTOL = 1e-5


def _setup(name, n_spectra=None):
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    from oracle import oracle as O
    from vulcan import synth
    from vulcan.gpu import engine as E
    from vulcan.index.build import L1Index, read_labels
    w = synth.WORKLOADS[name]
    d = synth.build_index(w, CACHE)
    l1 = L1Index(d)
    lab = read_labels(d)
    sp, _ = synth.simulate_run(l1, lab, w, n_spectra=n_spectra, seed=w.spectra_seed, run=f"{name}_parity")
    p = w.search_params()
    gi = E.GpuIndex(l1, p, STATIC, w.var_mods)
    P = O.make_params(STATIC, w.var_mods, p.fragment_unit)
    return w, l1, sp, p, gi, P


@pytest.fixture(scope="module")
def small():
    return _setup("small")


@pytest.fixture(scope="module")
def human():
    return _setup("human")


def _assert_parity(res):
    for k in ("k0_equal", "hyp_equal", "k1_equal", "topk_equal", "k2_equal", "top1_equal", "fp64_matches_equal"):
        assert res[k], f"{k} failed: {res}"
    assert res["hs_max_rel_err_fp64"] <= FP64_RTOL, res


def test_small_every_spectrum_equals_oracle(small):
    from oracle import parity
    from vulcan.gpu import engine as E
    w, l1, sp, p, gi, P = small
    out = E._search_device(E.DeviceRun(sp, gi.dev), gi, p, 1, E.Stats())
    E.check_status(out["status"])
    res = parity.check_plain(l1, sp, p, P, out, len(sp))
    assert res["spectra"] == 5000 and res["candidates"] > 50_000, res
    _assert_parity(res)


def test_human_sample_equals_oracle(human):
    from oracle import parity
    from vulcan.gpu import engine as E
    w, l1, sp, p, gi, P = human
    assert len(sp) == 40_000
    out = E._search_device(E.DeviceRun(sp, gi.dev), gi, p, 1, E.Stats())
    E.check_status(out["status"])
    res = parity.check_plain(l1, sp, p, P, out, 3000)
    assert res["spectra"] == 3000 and res["window_rows"] > 1_000_000, res
    _assert_parity(res)


def test_human_graphed_searcher_equals_search(human):
    from vulcan.gpu import engine as E
    w, l1, sp, p, gi, P = human
    tbl = E.search(sp, gi, l1, p)[0]
    se = E.Searcher(gi, l1, p)
    pinned = E.pin_spectra(sp)
    for t, _ in se.search_many([pinned, pinned]):
        assert t.equals(tbl)


def test_small_search_exhaustive_equals_oracle(small):
    """The exhaustive search (K2 over every window row) against the oracle's window candidates and K2, and its
    top-1 PSMs against the oracle's ranking of them."""
    from oracle import oracle as O
    from vulcan.gpu import engine as E
    from oracle.parity import subset
    w, l1, sp, p, gi, P = small
    s2 = subset(sp, len(sp))
    tbl, st, dbg = E.search_exhaustive(s2, gi, l1, p, report=1)
    pk = O.k0_view(s2, p)
    hyp = O.make_hypotheses(s2, pk["valid"], l1.mass32, p)
    h, r = O.window_candidates(hyp)
    assert np.array_equal(dbg["h"].cpu().numpy(), h)
    assert np.array_equal(dbg["r"].cpu().numpy(), r)
    k2o = O.k2(l1, hyp, pk, h, r, p, P)
    k2d = {k: v.cpu().numpy() for k, v in dbg["k2"].items()}
    for k in ("summed_b", "summed_y", "matched_b", "matched_y", "longest_b", "longest_y"):
        assert np.array_equal(k2d[k], k2o[k]), k
    assert np.array_equal(k2d["ppm"], k2o["ppm"], equal_nan=True)
    np.testing.assert_allclose(k2d["hyperscore"], k2o["hyperscore"], rtol=1e-12)
    f = O.k2_f64(l1, hyp, pk, h, r, p, P)["hyperscore"]
    fin = np.isfinite(f)
    assert np.all(np.abs(k2d["hyperscore"][fin] - f[fin]) <= FP64_RTOL * np.abs(f[fin]))
    rk = O.psm_rank(k2o, r, p.min_matched_peaks, 1)
    assert np.array_equal(tbl.column("spec_idx").to_numpy(), rk["spec"])
    assert np.array_equal(tbl.column("pf_row").to_numpy(), r[rk["cand"]])
    np.testing.assert_allclose(tbl.column("hyperscore").to_numpy(), rk["hyperscore"], rtol=1e-12)
    assert len(h) > 200_000


def test_small_k1_shapes_per_peak_bucket_give_the_same_search(small):
    """K1 shapes routed by peak-count bucket (each bucket's spectra on its own tiling and warps, as the autotuner
    chooses them) give the single-shape pass's counts, statistics, candidates and K2 outputs, and the pruned
    front end's shortlist."""
    import dataclasses
    from vulcan.gpu import engine as E
    from vulcan.gpu import prune as PR
    w, l1, sp, p, gi, P = small
    npk = np.diff(sp.offsets)
    q = dataclasses.replace(p, k1_shapes=((int(np.percentile(npk, 30)), 64, 3), (int(np.percentile(npk, 70)), 256, 8)))
    gq = E.GpuIndex(l1, q, STATIC, w.var_mods)
    assert set(gq.tilings) == {64, 128, 256}
    a = E._search_device(E.DeviceRun(sp, gi.dev), gi, p, 1, E.Stats())
    b = E._search_device(E.DeviceRun(sp, gq.dev), gq, q, 1, E.Stats())
    E.check_status(b["status"])
    nw = int(a["win_off"][-1])
    assert torch_equal(a["win_off"], b["win_off"]) and torch_equal(a["cnt"][:nw], b["cnt"][:nw])
    nc = int(a["cand_off"][-1])
    for k in ("c_hyp", "c_row", "c_cnt"):
        assert torch_equal(a[k][:nc], b[k][:nc]), k
    for k in ("hyperscore", "matched_b", "matched_y", "summed_b", "summed_y"):
        assert torch_equal(a["k2"][k][:nc], b["k2"][k][:nc]), k
    fa = PR._front(E.DeviceRun(sp, gi.dev), gi, p, E.Stats(), False, min_count=2)
    fb = PR._front(E.DeviceRun(sp, gq.dev), gq, q, E.Stats(), False, min_count=2)
    n = len(sp)
    nc = int(fa["hits"]["cand_off"][n])
    assert int(fb["hits"]["cand_off"][n]) == nc
    for k in ("c_hyp", "c_row", "c_cnt", "c_isum"):
        assert torch_equal(fa["hits"][k][:nc], fb["hits"][k][:nc]), k


def torch_equal(x, y):
    import torch
    return bool(torch.equal(x, y))


@pytest.mark.parametrize("min_count", (1, 2))
def test_human_hit_lists_give_the_dense_shortlist(human, min_count):
    """On the whole human run, the pruned path's front end over K1 hit lists (``vk_k1_hits`` + ``vk_select_hits``)
    gives the shortlist, intensity sums and statistics of the dense form (``vk_k1_tiles`` + ``vk_select_topk``).
    With a count floor of 1 most spectra hold more hits than ``vk_select_hits`` keeps in shared memory, so its
    global-memory selection is compared too."""
    from vulcan.gpu import engine as E
    from vulcan.gpu import prune as PR
    w, l1, sp, p, gi, P = human
    st = E.Stats()
    fh = PR._front(E.DeviceRun(sp, gi.dev, st), gi, p, st, False, min_count=min_count)
    fd = PR._front(E.DeviceRun(sp, gi.dev, st), gi, p, st, False, min_count=min_count, dense=True)
    E.check_status(fh["status"])
    E.check_status(fd["status"])
    n = len(sp)
    nc = int(fd["hits"]["cand_off"][n])
    assert int(fh["hits"]["cand_off"][n]) == nc and nc > 100_000
    for k in ("c_hyp", "c_row", "c_cnt"):
        assert torch_equal(fh["hits"][k][:nc], fd["hits"][k][:nc]), k
    dh, hits = fd["dh"], fd["hits"]
    h = hits["c_hyp"][:nc]
    dense_isum = fd["isum"][fd["win_off"][h] + hits["c_row"][:nc] - dh["lo"][h]]
    assert torch_equal(fh["hits"]["c_isum"][:nc], dense_isum)
    for k in ("spec_scored", "spec_matched"):
        assert torch_equal(fh[k][:n], fd[k][:n]), k
    if min_count == 1:   # spectra whose hits outnumber the top-k: the selection ran (over global memory for most)
        per_spec = fh["hits"]["cand_off"][1:n + 1] - fh["hits"]["cand_off"][:n]
        assert int((per_spec == p.topk).sum()) > 1000


@pytest.mark.parametrize("topk", (8, 32))
def test_human_short_hit_lists_give_the_dense_shortlist(human, topk):
    """Short lists (top 8 and 32, no closure: ``vk_select_hits`` keeps them in registers as the hits stream by) give
    the dense form's shortlist of the same size on the whole human run."""
    import dataclasses
    from vulcan.gpu import engine as E
    from vulcan.gpu import prune as PR
    w, l1, sp, p, gi, P = human
    q = dataclasses.replace(p, topk=topk)
    st = E.Stats()
    fh = PR._front(E.DeviceRun(sp, gi.dev, st), gi, q, st, False, min_count=2)
    fd = PR._front(E.DeviceRun(sp, gi.dev, st), gi, q, st, False, min_count=2, dense=True)
    n = len(sp)
    nc = int(fd["hits"]["cand_off"][n])
    assert int(fh["hits"]["cand_off"][n]) == nc and nc > 100_000
    for k in ("c_hyp", "c_row", "c_cnt"):
        assert torch_equal(fh["hits"][k][:nc], fd["hits"][k][:nc]), k
    dh, hits = fd["dh"], fd["hits"]
    h = hits["c_hyp"][:nc]
    assert torch_equal(fh["hits"]["c_isum"][:nc], fd["isum"][fd["win_off"][h] + hits["c_row"][:nc] - dh["lo"][h]])
