"""The CPU oracle against the reference: its own Python code (golden_ref_py.npz, made by
tests/golden/make_golden.py) and its own CUDA kernels (golden_ref_kernels.npz, made by
tests/golden/make_golden_ref.py on a B200).  These pins make the oracle trustworthy before it judges the kernels."""
import os

import numpy as np
import pytest

from oracle import oracle as O

STATIC = {"C": 57.021464}
VAR = {"M": 15.9949}
SETS = ("da", "ppm", "ppm_mfz")


def _peaks(g, name):
    return {k: g[f"{name}/k0_{k}"] for k in ("off", "mass", "int", "tic")}


def _hyp(g, name):
    return {k: g[f"{name}/hyp_{k}"] for k in ("spec", "z", "iso", "pm", "M", "lo", "hi", "maxfz")}


@pytest.mark.parametrize("name", SETS)
def test_k0_view_equals_reference(mini, golden_py, param_sets, name):
    l1, sp, _ = mini
    pk = O.k0_view(sp, param_sets[name])
    g = golden_py
    assert np.array_equal(pk["off"], g[f"{name}/k0_off"])
    assert np.array_equal(pk["mass"], g[f"{name}/k0_mass"])
    assert np.array_equal(pk["int"], g[f"{name}/k0_int"])
    assert np.array_equal(pk["valid"], g[f"{name}/k0_valid"])
    np.testing.assert_allclose(pk["tic"], g[f"{name}/k0_tic"], rtol=1e-7)


@pytest.mark.parametrize("name", SETS)
def test_hypotheses_equal_reference(mini, golden_py, param_sets, name):
    l1, sp, _ = mini
    g = golden_py
    hyp = O.make_hypotheses(sp, g[f"{name}/k0_valid"], l1.mass32, param_sets[name])
    for k in ("spec", "z", "iso", "pm", "M", "lo", "hi", "maxfz"):
        assert np.array_equal(hyp[k], g[f"{name}/hyp_{k}"]), k


@pytest.mark.parametrize("name", SETS)
def test_window_candidates_equal_reference(golden_py, name):
    g = golden_py
    h, r = O.window_candidates(_hyp(g, name))
    assert np.array_equal(h, g[f"{name}/win_h"]) and np.array_equal(r, g[f"{name}/win_r"])


@pytest.mark.parametrize("name", SETS)
def test_select_topk_equals_reference(mini, golden_py, param_sets, name):
    l1, sp, _ = mini
    g = golden_py
    p = param_sets[name]
    hyp = _hyp(g, name)
    P = O.make_params(STATIC, VAR, p.fragment_unit)
    win_off, cnt, sc, mt = O.k1_windows(l1, hyp, _peaks(g, name), p, P)
    oh, orr, oc = O.k1_appended(hyp, win_off, cnt, p.k1_threshold)
    assert len(oh) > p.topk * 10       # enough entries that the per-spectrum cut is exercised
    h, r, c = O.select_topk(oh, orr, oc, hyp["spec"], l1.partner, p.topk)
    assert np.array_equal(h, g[f"{name}/topk_h"])
    assert np.array_equal(r, g[f"{name}/topk_r"])
    assert np.array_equal(c, g[f"{name}/topk_c"])


@pytest.mark.parametrize("name", SETS)
def test_psm_rank_equals_reference(mini, golden_py, param_sets, name):
    """Ranking, delta_next / delta_best and the reported candidates equal the reference's psm_table."""
    l1, sp, _ = mini
    g = golden_py
    p = param_sets[name]
    hyp = _hyp(g, name)
    P = O.make_params(STATIC, VAR, p.fragment_unit)
    h, r = g[f"{name}/topk_h"], g[f"{name}/topk_r"]
    k2 = O.k2(l1, hyp, _peaks(g, name), h, r, p, P)
    rk = O.psm_rank(k2, r, p.min_matched_peaks, 3)
    assert np.array_equal(rk["spec"], g[f"{name}/psm_spec_idx"])
    assert np.array_equal(rk["rank"], g[f"{name}/psm_rank"])
    assert np.array_equal(r[rk["cand"]], g[f"{name}/psm_pf_row"])
    assert np.array_equal(rk["hyperscore"], g[f"{name}/psm_hyperscore"])
    assert np.array_equal(rk["delta_next"], g[f"{name}/psm_delta_next"])
    assert np.array_equal(rk["delta_best"], g[f"{name}/psm_delta_best"])


def test_lnfact_equals_reference(golden_py):
    assert np.array_equal(O.lnfact(golden_py["lnfact_n"]), golden_py["lnfact_v"])


# ---------------------------------------------------------------------------------- against the reference kernels
@pytest.mark.parametrize("name", SETS)
def test_frag_count_and_keys_equal_reference_kernels(mini, golden_kernels, param_sets, name):
    import math
    l1, _, _ = mini
    p = param_sets[name]
    P = O.make_params(STATIC, VAR, p.fragment_unit)
    n = len(l1)
    cnt = np.empty(n, np.int32)
    import ctypes as C
    L = O.lib()
    a = [O._p(O._c(getattr(l1, k), dt)) for k, dt in (("seq_off", np.int64), ("length", np.uint8),
                                                      ("mask", np.uint64), ("mass32", np.float32),
                                                      ("residues", np.uint8))]
    L.or_frag_count(C.c_int64(n), *a, C.c_int(p.min_ion_index), C.c_float(p.fragment_min_mz),
                    C.c_float(p.fragment_max_mz), O._p(cnt), C.byref(P))
    assert np.array_equal(cnt, golden_kernels[f"{name}/frag_count"])
    off = np.zeros(n + 1, np.int64)
    np.cumsum(cnt, out=off[1:])
    keys = np.empty(off[-1], np.int64)
    inv_logw = 1.0 / math.log1p(p.bin_ppm * 1e-6)
    L.or_frag_emit(C.c_int64(n), *a, C.c_int(p.min_ion_index), C.c_float(p.fragment_min_mz),
                   C.c_float(p.fragment_max_mz), C.c_double(inv_logw), C.c_int(p.chunk_size), C.c_int64(0),
                   O._p(off), O._p(keys), C.byref(P))
    # host log() may differ from the device's by an ulp; a key can then move across a quantum boundary
    ref = golden_kernels[f"{name}/frag_keys"]
    assert len(keys) == len(ref)
    assert np.mean(np.sort(keys) == ref) > 0.999


@pytest.mark.parametrize("name", SETS)
def test_k1_brute_equals_reference_kernels(mini, golden_py, golden_kernels, param_sets, name):
    l1, _, _ = mini
    g = golden_py
    p = param_sets[name]
    P = O.make_params(STATIC, VAR, p.fragment_unit)
    cnt = O.k1_brute(l1, _hyp(g, name), _peaks(g, name), g[f"{name}/win_h"], g[f"{name}/win_r"], p, P)
    assert np.array_equal(cnt, golden_kernels[f"{name}/brute"])


@pytest.mark.parametrize("name", SETS)
def test_k1_windows_equal_reference_k1(mini, golden_py, golden_kernels, param_sets, name):
    """The oracle's window counts == the reference's indexed K1 append set, scored and matched (and so equal its
    brute force, as the reference's own test asserts)."""
    l1, _, _ = mini
    g = golden_py
    p = param_sets[name]
    hyp = _hyp(g, name)
    P = O.make_params(STATIC, VAR, p.fragment_unit)
    win_off, cnt, sc, mt = O.k1_windows(l1, hyp, _peaks(g, name), p, P)
    oh, orr, oc = O.k1_appended(hyp, win_off, cnt, p.k1_threshold)
    key = (oh << 32) | orr
    o = np.argsort(key)
    assert np.array_equal(key[o], golden_kernels[f"{name}/k1_key"])
    assert np.array_equal(oc[o], golden_kernels[f"{name}/k1_cnt"])
    assert np.array_equal(sc.astype(np.int64), golden_kernels[f"{name}/k1_scored"].astype(np.int64))
    assert np.array_equal(mt.astype(np.int64), golden_kernels[f"{name}/k1_matched"].astype(np.int64))
    # window counts restricted to the brute-force pairs
    bc = golden_kernels[f"{name}/brute"]
    nz = bc > 0
    bkey = (g[f"{name}/win_h"][nz].astype(np.int64) << 32) | g[f"{name}/win_r"][nz]
    assert np.array_equal(np.sort(bkey), golden_kernels[f"{name}/k1_key"])


@pytest.mark.parametrize("name", SETS)
def test_k1_over_fragment_index_equals_window_counts_and_reference_k1(mini, golden_py, golden_kernels, param_sets,
                                                                       name):
    """The fragment-index K1 (m/z-binned index fragments, rows ascending in a bin -- the reference's K1 search) ==
    the window counts bit for bit (counts, scored, matched and the intensity sums), and so the reference's K1."""
    l1, _, _ = mini
    g = golden_py
    p = param_sets[name]
    hyp = _hyp(g, name)
    pk = _peaks(g, name)
    P = O.make_params(STATIC, VAR, p.fragment_unit)
    a = O.k1_windows(l1, hyp, pk, p, P, tic=pk["tic"])
    b = O.k1_index(l1, hyp, pk, p, P, tic=pk["tic"])
    for x, y in zip(a, b):
        assert np.array_equal(x, y), name
    oh, orr, oc = O.k1_appended(hyp, b[0], b[1], p.k1_threshold)
    key = (oh << 32) | orr
    o = np.argsort(key)
    assert np.array_equal(key[o], golden_kernels[f"{name}/k1_key"])
    assert np.array_equal(oc[o], golden_kernels[f"{name}/k1_cnt"])


@pytest.mark.parametrize("name", SETS)
def test_c_k0_view_and_topk_equal_the_numpy_restatement(mini, golden_py, param_sets, name):
    """The oracle's C K0 view (global peak mode) and C top-K + closure over the window counts == its numpy
    restatements (pinned to the reference's own code) on the mini fixture."""
    l1, sp, _ = mini
    g = golden_py
    p = param_sets[name]
    P = O.make_params(STATIC, VAR, p.fragment_unit)
    a, b = O.k0_view(sp, p), O.k0_view_c(sp, p)
    for k in ("off", "mass", "int", "tic", "valid"):
        assert np.array_equal(a[k], b[k]), (name, k)
    hyp = _hyp(g, name)
    win_off, cnt, _, _ = O.k1_index(l1, hyp, _peaks(g, name), p, P)
    for closure in (True, False):
        for topk in (1, 3, p.topk):
            want = O.select_topk(*O.k1_appended(hyp, win_off, cnt, p.k1_threshold), hyp["spec"], l1.partner, topk,
                                 closure)
            got = O.topk_windows(hyp, win_off, cnt, p.k1_threshold, l1.partner, topk, closure)
            for x, y in zip(want, got):
                assert np.array_equal(x, y), (name, closure, topk)


def test_k1_over_fragment_index_on_a_larger_run():
    """The same equality on 400 spectra of the small synthetic workload (configuration 0's index: 2,000 proteins),
    with precursor windows widened to +-2000 ppm so that windows span many rows of a bin, single-threaded and on all
    cores, and for two fragment settings (the cached index is rebuilt for the second)."""
    import dataclasses
    import tempfile
    from vulcan import synth
    from vulcan.index.build import L1Index, read_labels
    w = synth.WORKLOADS["small"]
    d = synth.build_index(w, os.environ.get("VULCAN_BENCH_CACHE", os.path.join(tempfile.gettempdir(),
                                                                                 "vulcan_bench_cache")))
    l1 = L1Index(d)
    sp, _ = synth.simulate_run(l1, read_labels(d), w, n_spectra=400, seed=5)
    for tol, unit, ppm, mfc in (((-0.02, 0.02), "da", (-10.0, 10.0), 1),
                                ((-20.0, 20.0), "ppm", (-2000.0, 2000.0), None)):
        p = dataclasses.replace(w.search_params(), fragment_ppm=tol, fragment_unit=unit, precursor_ppm=ppm,
                                max_fragment_charge=mfc)
        P = O.make_params(STATIC, w.var_mods, p.fragment_unit)
        pk = O.k0_view(sp, p)
        hyp = O.make_hypotheses(sp, pk["valid"], l1.mass32, p)
        a = O.k1_windows(l1, hyp, pk, p, P, tic=pk["tic"])
        for nt in (1, None):
            b = O.k1_index(l1, hyp, pk, p, P, nthreads=nt, tic=pk["tic"])
            for x, y in zip(a, b):
                assert np.array_equal(x, y), (unit, nt)
        assert int(a[1].max()) >= 3
        # the C K0 view and top-K of the oracle chain on the same run
        pc = O.k0_view_c(sp, p, nthreads=3)
        for k in ("off", "mass", "int", "tic", "valid"):
            assert np.array_equal(pk[k], pc[k]), (unit, k)
        for topk in (5, 50):
            want = O.select_topk(*O.k1_appended(hyp, a[0], a[1], 2), hyp["spec"], l1.partner, topk, True)
            got = O.topk_windows(hyp, a[0], a[1], 2, l1.partner, topk, True)
            for x, y in zip(want, got):
                assert np.array_equal(x, y), (unit, topk)


@pytest.mark.parametrize("name", SETS)
@pytest.mark.parametrize("mode", ("closed", "shift"))
def test_k2_equals_reference_kernels(mini, golden_py, golden_kernels, param_sets, name, mode):
    l1, _, _ = mini
    g = golden_py
    p = param_sets[name]
    P = O.make_params(STATIC, VAR, p.fragment_unit)
    shift = golden_kernels[f"{name}/k2shift_delta"] if mode == "shift" else None
    out = O.k2(l1, _hyp(g, name), _peaks(g, name), g[f"{name}/win_h"], g[f"{name}/win_r"], p, P, shift=shift)
    ref = {k: golden_kernels[f"{name}/k2{mode}_{k}"] for k in ("hs", "sb", "sy", "ppm", "mb", "my", "lb", "ly")}
    for a, b in (("summed_b", "sb"), ("summed_y", "sy"), ("matched_b", "mb"), ("matched_y", "my"),
                 ("longest_b", "lb"), ("longest_y", "ly")):
        assert np.array_equal(out[a], ref[b]), a
    assert np.array_equal(out["ppm"], ref["ppm"], equal_nan=True)
    # host and device log() agree to an ulp or so
    np.testing.assert_allclose(out["hyperscore"], ref["hs"], rtol=1e-13, atol=0)


@pytest.mark.parametrize("name", SETS)
def test_k2_hyperscore_within_fp64_oracle(mini, golden_py, param_sets, name):
    """f32 K2 hyperscores within 1e-5 relative of the all-FP64 oracle wherever both match the same ions."""
    l1, _, _ = mini
    g = golden_py
    p = param_sets[name]
    P = O.make_params(STATIC, VAR, p.fragment_unit)
    h, r = g[f"{name}/win_h"], g[f"{name}/win_r"]
    a = O.k2(l1, _hyp(g, name), _peaks(g, name), h, r, p, P)
    b = O.k2_f64(l1, _hyp(g, name), _peaks(g, name), h, r, p, P)
    same = (a["matched_b"] == b["matched_b"]) & (a["matched_y"] == b["matched_y"])
    assert same.mean() > 0.999
    rel = np.abs(a["hyperscore"][same] - b["hyperscore"][same]) / np.abs(b["hyperscore"][same])
    assert rel.max() <= 1e-5


@pytest.mark.parametrize("name", ("win100", "win64", "win12"))
def test_k0_window_view_equals_reference(name):
    """The window peak mode (engine.py:182-183) against the reference's own K0 on the fixture spectra and the
    window edge cases of golden_window.npz."""
    import os
    from tests.golden.make_golden_window import WINDOW_SETS
    from vulcan.gpu.host import SearchParams, Spectra
    g = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_window.npz")))
    sp = Spectra("window", g["w_scan"], g["w_index"], g["w_rt"], g["w_precursor_mz"], g["w_charge"], g["w_mz"],
                 g["w_intensity"], g["w_offsets"])
    pk = O.k0_view(sp, SearchParams(**WINDOW_SETS[name]))
    assert np.array_equal(pk["off"], g[f"{name}/k0_off"])
    assert np.array_equal(pk["mass"], g[f"{name}/k0_mass"])
    assert np.array_equal(pk["int"], g[f"{name}/k0_int"])
    assert np.array_equal(pk["valid"], g[f"{name}/k0_valid"])
    np.testing.assert_allclose(pk["tic"], g[f"{name}/k0_tic"], rtol=1e-7)
    assert (np.diff(pk["off"]) > 15).any()   # some spectra keep more than a window's worth
