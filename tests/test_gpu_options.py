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
