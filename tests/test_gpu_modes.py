"""Open and mass-offset search modes on the B200 kernels (``vulcan.ptm.search``) against the oracle: the
hypotheses' K1 counts with per-hypothesis count floors, top-K with pair closure over all the hypotheses of each
spectrum, K2 with the per-candidate precursor shift (reference ``kernels.cu:294-363``), the reported PSMs; and the
batch split (several batches, and one batch forced to overflow and be halved) gives the one-batch result."""
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
STATIC = {"C": 57.021464}


@pytest.fixture(scope="module")
def setup():
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    import dataclasses
    from oracle import oracle as O
    from vulcan import synth
    from vulcan.gpu import engine as E
    from vulcan.index.build import L1Index, read_labels
    w = synth.WORKLOADS["small"]
    d = synth.build_index(w, os.environ.get("VULCAN_BENCH_CACHE",
                                            os.path.join(tempfile.gettempdir(), "vulcan_bench_cache")))
    l1 = L1Index(d)
    sp, _ = synth.simulate_run(l1, read_labels(d), w, n_spectra=120, seed=4242)
    p = dataclasses.replace(w.search_params(), topk=20, k1_threshold=2)
    gi = E.GpuIndex(l1, p, STATIC, w.var_mods)
    return l1, sp, p, gi, O.make_params(STATIC, w.var_mods, p.fragment_unit)


def _oracle(l1, sp, p, P, hyp, mp):
    from oracle import oracle as O
    from vulcan.ptm.search import MODE_CLOSED, MODE_OPEN
    pk = O.k0_view(sp, p)
    win_off, cnt, sc, mt = O.k1_windows(l1, hyp, pk, p, P)
    oh, orr, oc = O.k1_appended(hyp, win_off, cnt, 1)
    thr = np.where(hyp["mode"] == MODE_OPEN, mp.k1_threshold_open, p.k1_threshold)
    keep = oc >= thr[oh]
    h, r, c = O.select_topk(oh[keep], orr[keep], oc[keep], hyp["spec"], l1.partner, p.topk, p.pair_closure)
    m = hyp["mode"][h]
    shift = np.where(m == MODE_CLOSED, np.float32(0), (hyp["M"][h] - l1.mass32[r]).astype(np.float32))
    k2 = O.k2(l1, hyp, pk, h, r, p, P, shift=shift.astype(np.float32))
    return {"pk": pk, "h": h, "r": r, "c": c, "scored": sc, "matched": mt, "k2": k2, "shift": shift}


@pytest.mark.parametrize("mp_kw", [dict(offsets=(15.9949, 79.96633)),
                                   dict(offsets=(-17.0265,), open_da=(-5.0, 60.0)),
                                   dict(open_da=(-2.0, 30.0), spectra_per_batch=17)])
def test_modes_equal_oracle(setup, mp_kw):
    from vulcan.gpu import engine as E
    from vulcan.ptm import search as PS
    l1, sp, p, gi, P = setup
    mp = PS.ModeParams(**mp_kw)
    st = E.Stats()
    peaks = E.k0_preprocess(sp, p, gi.dev, st)
    hyp = PS.make_mode_hypotheses(sp, peaks["valid"], gi.mass32_np, p, mp)
    h, r, c, sc, mt, d_spec, d_maxfz = PS.k1_topk_modes(gi, hyp, peaks, p, mp, st)
    o = _oracle(l1, sp, p, P, hyp, mp)
    assert len(o["h"]) > 500
    assert np.array_equal(h.cpu().numpy(), o["h"])
    assert np.array_equal(r.cpu().numpy(), o["r"])
    assert np.array_equal(c.cpu().numpy(), o["c"])
    assert np.array_equal(sc.cpu().numpy().astype(np.int64), o["scored"].astype(np.int64))
    assert np.array_equal(mt.cpu().numpy().astype(np.int64), o["matched"].astype(np.int64))
    k2 = PS.k2_shifted(gi, hyp, h, r, d_spec, d_maxfz, peaks, p, len(sp))
    assert np.array_equal(k2["shift"].cpu().numpy(), o["shift"])
    for k in ("summed_b", "summed_y", "matched_b", "matched_y", "longest_b", "longest_y"):
        assert np.array_equal(k2[k].cpu().numpy(), o["k2"][k]), k
    assert np.array_equal(k2["ppm"].cpu().numpy(), o["k2"]["ppm"], equal_nan=True)
    np.testing.assert_allclose(k2["hyperscore"].cpu().numpy(), o["k2"]["hyperscore"], rtol=1e-12)
    if "open_da" in mp_kw:
        assert (np.abs(o["shift"]) > 1.0).sum() > 100      # shifted candidates were scored
    # the whole search: top-1 PSMs of the oracle's ranking, with the mode of their hypothesis
    tbl = PS.search_modes(sp, gi, l1, p, mp, report=1)[0]
    from oracle import oracle as O
    rk = O.psm_rank(o["k2"], o["r"], p.min_matched_peaks, 1)
    assert np.array_equal(tbl.column("spec_idx").to_numpy(), rk["spec"])
    assert np.array_equal(tbl.column("pf_row").to_numpy(), o["r"][rk["cand"]])
    assert np.array_equal(tbl.column("mode").to_numpy(), hyp["mode"][o["h"][rk["cand"]]])


def test_modes_batches_and_overflow_retry_give_the_one_batch_result(setup, monkeypatch):
    from vulcan.gpu import engine as E
    from vulcan.ptm import search as PS
    l1, sp, p, gi, P = setup
    st = E.Stats()
    peaks = E.k0_preprocess(sp, p, gi.dev, st)
    mp1 = PS.ModeParams(offsets=(15.9949,), open_da=(-5.0, 40.0))
    hyp = PS.make_mode_hypotheses(sp, peaks["valid"], gi.mass32_np, p, mp1)
    one = PS.k1_topk_modes(gi, hyp, peaks, p, mp1, st)
    many = PS.k1_topk_modes(gi, hyp, peaks, p, PS.ModeParams(offsets=(15.9949,), open_da=(-5.0, 40.0),
                                                             spectra_per_batch=7), st)
    for a, b in zip(one[:5], many[:5]):
        assert np.array_equal(a.cpu().numpy(), b.cpu().numpy())
    # a hit-list capacity one short of the first batch's window rows: the device reports the overflow, the batch
    # is halved and redone
    real = E._k1_hits
    calls = {"n": 0}

    def short(gi_, dh, peaks_, p_, n_hyp, thr, isum=True, h_thr=None, caps=None):
        calls["n"] += 1
        if calls["n"] == 1:
            caps = (caps[0], caps[1] - 1)
        return real(gi_, dh, peaks_, p_, n_hyp, thr, isum=isum, h_thr=h_thr, caps=caps)
    monkeypatch.setattr(E, "_k1_hits", short)
    st2 = E.Stats()
    again = PS.k1_topk_modes(gi, hyp, peaks, p, mp1, st2)
    assert st2.counts.get("k1_overflow_retries", 0) >= 1
    for a, b in zip(one[:5], again[:5]):
        assert np.array_equal(a.cpu().numpy(), b.cpu().numpy())
