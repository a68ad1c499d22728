"""Whole searches with the reference's other search options (SearchParams, reference vulcan/gpu/host.py:14-43):
no pair closure, a K1 threshold above 1, more matched peaks required and more PSMs reported per spectrum.  The
staged path equals the oracle's chain (K1 counts, candidates, K2, ranking); the fused kernel equals the staged
path."""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STATIC = {"C": 57.021464}
VAR = {"M": 15.9949}

OPTIONS = {
    "no_closure": dict(pair_closure=False),
    "thr3_mm6": dict(k1_threshold=3, min_matched_peaks=6),
    "no_closure_thr2_top3": dict(pair_closure=False, k1_threshold=2, topk=3),
}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    return torch


@pytest.mark.parametrize("report", (1, 3))
@pytest.mark.parametrize("opt", sorted(OPTIONS))
@pytest.mark.parametrize("name", ("da", "ppm_mfz"))
def test_search_options_equal_oracle(mini, param_sets, name, opt, report, torch_cuda):
    from oracle import oracle as O
    from vulcan.gpu import engine as E
    l1, sp, _ = mini
    p = dataclasses.replace(param_sets[name], tile_rows=64, **OPTIONS[opt])
    staged = dataclasses.replace(p, search_method="staged")
    gi = E.GpuIndex(l1, p, STATIC, VAR)
    tbl, _, out = E.search(sp, gi, l1, staged, report=report)
    P = O.make_params(STATIC, VAR, p.fragment_unit)
    pk = O.k0_view(sp, p)
    hyp = O.make_hypotheses(sp, pk["valid"], l1.mass32, p)
    win_off, cnt, _, _ = O.k1_windows(l1, hyp, pk, p, P)
    assert np.array_equal(out["cnt"][:int(out["win_off"][-1])].cpu().numpy(), cnt)
    oh, orr, oc = O.k1_appended(hyp, win_off, cnt, p.k1_threshold)
    h, r, c = O.select_topk(oh, orr, oc, hyp["spec"], l1.partner, p.topk, pair_closure=p.pair_closure)
    nc = int(out["cand_off"][-1])
    assert nc > 0
    assert np.array_equal(out["c_hyp"][:nc].cpu().numpy(), h)
    assert np.array_equal(out["c_row"][:nc].cpu().numpy(), r)
    assert np.array_equal(out["c_cnt"][:nc].cpu().numpy(), c)
    k2 = O.k2(l1, hyp, pk, h, r, p, P)
    np.testing.assert_allclose(out["k2"]["hyperscore"][:nc].cpu().numpy(), k2["hyperscore"], rtol=1e-12)
    rk = O.psm_rank(k2, r, p.min_matched_peaks, report)
    assert tbl.num_rows > 0 and np.array_equal(tbl.column("pf_row").to_numpy(), r[rk["cand"]])
    t_f = E.search(sp, gi, l1, dataclasses.replace(p, search_method="fused"), report=report)[0]
    assert t_f.equals(tbl)


def test_nterm_modified_index_search_equals_oracle(tmp_path, torch_cuda):
    """An index with a variable peptide N-terminal modification ("^", acetyl: mask bit 63, on the b ions and the
    precursor) searched on the device equals the oracle's search: K1 counts, candidates, K2 and the top PSMs."""
    from oracle import oracle as O
    from vulcan import synth
    from vulcan.gpu import engine as E
    from vulcan.index.build import L1Index, read_labels
    w = dataclasses.replace(synth.WORKLOADS["small"], name="nterm_mini", n_proteins=60, n_spectra=300,
                            var_mods={"M": 15.9949, "^": 42.010565}, max_var=2)
    d = synth.build_index(w, str(tmp_path))
    l1, lab = L1Index(d), read_labels(d)
    assert (l1.mask.astype(np.uint64) >> np.uint64(63)).any()
    sp, truth = synth.simulate_run(l1, lab, w)
    p = w.search_params(topk=20)
    static, var = {"C": 57.021464}, w.var_mods
    gi = E.GpuIndex(l1, p, static, var)
    tbl, st, out = E.search(sp, gi, l1, p, report=2)
    P = O.make_params(static, var, p.fragment_unit)
    pk = O.k0_view(sp, p)
    hyp = O.make_hypotheses(sp, pk["valid"], l1.mass32, p)
    win_off, cnt, sc, mt = O.k1_windows(l1, hyp, pk, p, P)
    assert np.array_equal(out["cnt"][:int(out["win_off"][-1])].cpu().numpy(), cnt)
    oh, orr, oc = O.k1_appended(hyp, win_off, cnt, p.k1_threshold)
    h, r, c = O.select_topk(oh, orr, oc, hyp["spec"], l1.partner, p.topk)
    nc = int(out["cand_off"][-1])
    assert np.array_equal(out["c_row"][:nc].cpu().numpy(), r)
    k2 = O.k2(l1, hyp, pk, h, r, p, P)
    np.testing.assert_allclose(out["k2"]["hyperscore"][:nc].cpu().numpy(), k2["hyperscore"], rtol=1e-12)
    rk = O.psm_rank(k2, r, p.min_matched_peaks, 2)
    assert np.array_equal(tbl.column("pf_row").to_numpy(), r[rk["cand"]])
    # the planted N-terminally modified peptidoforms are found at rank 1
    import pyarrow.compute as pc
    top = tbl.filter(pc.equal(tbl.column("rank"), 1))
    rows = dict(zip(top.column("spec_idx").to_pylist(), top.column("pf_row").to_pylist()))
    nt = [i for i, t in enumerate(truth) if int(l1.mask[t]) >> 63]
    assert nt and np.mean([rows.get(i) == truth[i] for i in nt]) > 0.8
