"""K0 in the window peak mode (reference vulcan/gpu/engine.py:182-183) on the device: equal to the reference's own
outputs (golden_window.npz, made by tests/golden/make_golden_window.py) through all three kernel paths, on window
boundaries where the reference's CUDA division decides, and through whole searches against the oracle."""
import dataclasses
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
WSETS = ("win100", "win64", "win12")
STATIC = {"C": 57.021464}
VAR = {"M": 15.9949}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    return torch


@pytest.fixture(scope="module")
def gw():
    return dict(np.load(os.path.join(GOLDEN, "golden_window.npz")))


def _spectra(g):
    from vulcan.gpu.host import Spectra
    return Spectra("window", g["w_scan"], g["w_index"], g["w_rt"], g["w_precursor_mz"], g["w_charge"], g["w_mz"],
                   g["w_intensity"], g["w_offsets"])


def _params(name):
    from tests.golden.make_golden_window import WINDOW_SETS
    from vulcan.gpu.host import SearchParams
    return SearchParams(**WINDOW_SETS[name])


def _codes(sp, p):
    """The count kernel's per-spectrum path codes and kept counts."""
    import torch
    from vulcan.gpu import _lib as K
    from vulcan.gpu import engine as E
    run = E.DeviceRun(sp, torch.device("cuda"))
    n = run.n
    kept = torch.empty(n, dtype=torch.int64, device="cuda")
    easy = torch.empty(n, dtype=torch.uint8, device="cuda")
    hard = torch.empty(n, dtype=torch.int32, device="cuda")
    n_hard = torch.empty(1, dtype=torch.int32, device="cuda")
    K.check(K.lib().vk_k0w_count(n, K.ptr(run.offsets), K.ptr(run.mz), K.ptr(run.intensity), p.fragment_min_mz,
                                 p.fragment_max_mz, p.window_th, p.window_k, K.ptr(kept), K.ptr(easy),
                                 K.ptr(hard), K.ptr(n_hard), K.stream()), "k0w_count")
    torch.cuda.synchronize()
    return easy.cpu().numpy(), kept.cpu().numpy(), int(n_hard.item())


def _assert_view(pk, ref):
    assert np.array_equal(pk["off"].cpu().numpy(), ref["off"])
    assert np.array_equal(pk["mass"].cpu().numpy(), ref["mass"])
    assert np.array_equal(pk["int"].cpu().numpy(), ref["int"])
    assert np.array_equal(pk["valid"], ref["valid"])
    np.testing.assert_allclose(pk["tic"].cpu().numpy(), ref["tic"], rtol=1e-7)


@pytest.mark.parametrize("name", WSETS)
def test_k0_window_equals_reference(gw, name, torch_cuda):
    """The device view equals the reference's on the fixture spectra and the window edge cases; the copy (1), the
    warp (2) and the CTA (0) paths all run."""
    from vulcan.gpu import engine as E
    sp, p = _spectra(gw), _params(name)
    pk = E.k0_preprocess(sp, p, torch_cuda.device("cuda"), E.Stats())
    _assert_view(pk, {k: gw[f"{name}/k0_{k}"] for k in ("off", "mass", "int", "tic", "valid")})
    codes, kept, n_hard = _codes(sp, p)
    assert np.array_equal(kept, np.diff(gw[f"{name}/k0_off"]))
    assert set(codes.tolist()) == {0, 1, 2}
    assert n_hard == int((codes == 0).sum())


def test_k0_window_boundaries_follow_cuda_division(torch_cuda):
    """Peaks on and next to multiples of window_th = 7, whose f32 reciprocal is inexact: torch's CUDA division (the
    reference's expression) puts each in the window of the f32 reciprocal product -- where the true quotient
    differs -- and the device view, in order and shuffled, equals the oracle's."""
    from oracle import oracle as O
    from vulcan.gpu import engine as E
    from vulcan.gpu.host import SearchParams, Spectra
    f32 = np.float32
    xs = []
    for k in range(22, 286):
        x = f32(k * 7.0)
        xs += [np.nextafter(x, f32(0)), x, np.nextafter(x, f32(np.inf))]
    mz = np.array(xs, f32)
    ref_w = torch_cuda.floor(torch_cuda.from_numpy(mz).cuda() / 7.0).to(torch_cuda.int64).cpu().numpy()
    assert np.array_equal(ref_w, np.floor((mz * (f32(1) / f32(7.0))).astype(f32)).astype(np.int64))
    assert (np.floor(mz / f32(7.0)).astype(np.int64) != ref_w).any()
    rng = np.random.default_rng(5)
    it = rng.lognormal(6, 1, len(mz)).astype(f32)
    o = rng.permutation(len(mz))
    n = 2
    sp = Spectra("edges", np.arange(n, dtype=np.uint32), np.arange(n, dtype=np.uint32), np.zeros(n),
                 np.full(n, 600.0), np.full(n, 2, np.int8), np.concatenate([mz, mz[o]]),
                 np.concatenate([it, it[o]]), np.array([0, len(mz), 2 * len(mz)], np.int64))
    p = SearchParams(peak_mode="window", window_th=7.0, window_k=2, min_peaks=1)
    pk = E.k0_preprocess(sp, p, torch_cuda.device("cuda"), E.Stats())
    _assert_view(pk, O.k0_view(sp, p))
    codes, _, _ = _codes(sp, p)
    assert codes.tolist() == [2, 0]


def test_k0_window_range_outside_group_ids_is_refused(torch_cuda):
    """Windows past 999 (group ids spectrum * 1000 + window would merge neighbouring spectra) are an argument
    error, not a silent difference."""
    from vulcan.gpu import engine as E
    from vulcan.gpu.host import SearchParams, Spectra
    sp = Spectra("one", np.zeros(1, np.uint32), np.zeros(1, np.uint32), np.zeros(1), np.full(1, 600.0),
                 np.full(1, 2, np.int8), np.array([500.0], np.float32), np.array([1.0], np.float32),
                 np.array([0, 1], np.int64))
    with pytest.raises(RuntimeError):
        E.k0_preprocess(sp, SearchParams(peak_mode="window", window_th=1.0), torch_cuda.device("cuda"), E.Stats())


@pytest.mark.parametrize("name", ("da", "ppm_mfz"))
def test_window_mode_search_equals_oracle(mini, param_sets, name, torch_cuda):
    """A whole search with the window peak view equals the oracle's chain: K0, K1 counts, candidates, K2, PSMs."""
    from oracle import oracle as O
    from vulcan.gpu import engine as E
    l1, sp, _ = mini
    p = dataclasses.replace(param_sets[name], peak_mode="window", window_th=100.0, window_k=8, min_peaks=8,
                            search_method="staged")
    gi = E.GpuIndex(l1, p, STATIC, VAR)
    tbl, st, out = E.search(sp, gi, l1, p, report=2)
    P = O.make_params(STATIC, VAR, p.fragment_unit)
    pk = O.k0_view(sp, p)
    hyp = O.make_hypotheses(sp, pk["valid"], l1.mass32, p)
    win_off, cnt, sc, mt = O.k1_windows(l1, hyp, pk, p, P)
    assert np.array_equal(out["cnt"][:int(out["win_off"][-1])].cpu().numpy(), cnt)
    oh, orr, oc = O.k1_appended(hyp, win_off, cnt, p.k1_threshold)
    h, r, c = O.select_topk(oh, orr, oc, hyp["spec"], l1.partner, p.topk)
    nc = int(out["cand_off"][-1])
    assert nc > 0 and np.array_equal(out["c_row"][:nc].cpu().numpy(), r)
    k2 = O.k2(l1, hyp, pk, h, r, p, P)
    np.testing.assert_allclose(out["k2"]["hyperscore"][:nc].cpu().numpy(), k2["hyperscore"], rtol=1e-12)
    rk = O.psm_rank(k2, r, p.min_matched_peaks, 2)
    assert tbl.num_rows > 0 and np.array_equal(tbl.column("pf_row").to_numpy(), r[rk["cand"]])


def _window_params(param_sets, name):
    return dataclasses.replace(param_sets[name], peak_mode="window", window_th=100.0, window_k=8, min_peaks=8)


@pytest.mark.parametrize("name", ("da", "ppm"))
def test_window_mode_through_every_entry_point(mini, param_sets, name, torch_cuda):
    """With the window peak view: the fused search kernel gives the staged search's table, the pruned search
    without pruning is the plain search, and the graph-captured Searcher, plain and with a pruner that prunes,
    returns the per-run searches' tables."""
    import math
    from vulcan.gpu import engine as E
    from vulcan.gpu import prune as PR
    l1, sp, _ = mini
    p = dataclasses.replace(_window_params(param_sets, name), tile_rows=64, search_method="staged")
    gi = E.GpuIndex(l1, p, STATIC, VAR)
    plain = E.search(sp, gi, l1, p, report=2)[0]
    assert E.search(sp, gi, l1, dataclasses.replace(p, search_method="fused"), report=2)[0].equals(plain)
    keep_all = PR.Pruner(gi.dev, seed=3, tau=-math.inf, min_keep=0, max_keep=16)
    assert PR.search_pruned(sp, gi, l1, p, keep_all, report=2)[0].equals(plain)
    for tbl, _ in E.Searcher(gi, l1, p, report=2).search_many([sp, sp]):
        assert tbl.equals(plain)
    pr = PR.Pruner(gi.dev, seed=5)
    pr.tau, pr.min_keep, pr.max_keep, pr.min_count = 0.0, 1, 16, 2
    want = PR.search_pruned(sp, gi, l1, p, pr, report=2)[0]
    for tbl, _ in E.Searcher(gi, l1, p, pruner=pr, report=2).search_many([sp, sp]):
        assert tbl.equals(want)


@pytest.mark.parametrize("mode", ("global150", "global512", "window15", "window4"))
def test_k0_at_run_scale_equals_oracle(mode, torch_cuda):
    """K0 on a run of the bench's size (40,000 spectra, 20-600 peaks log-normal around 150, 6M peaks; three in four
    in m/z order, the rest shuffled, some with duplicated peaks) equals the oracle bit for bit, in both peak modes."""
    from oracle import oracle as O
    from vulcan.gpu import engine as E
    from vulcan.gpu.host import SearchParams, Spectra
    rng = np.random.default_rng(17)
    n = 40000
    lens = np.clip(np.round(rng.lognormal(np.log(150), 0.55, n)), 20, 600).astype(np.int64)
    off = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    mz = rng.uniform(100.0, 2100.0, int(off[-1])).astype(np.float32)
    it = rng.lognormal(7.0, 1.2, int(off[-1])).astype(np.float32)
    for s in range(n):
        a, b = off[s], off[s + 1]
        if s % 4 != 3:
            mz[a:b] = np.sort(mz[a:b])
        if s % 16 == 5 and b - a > 4:       # duplicated peaks: equal keys around the selection threshold
            mz[a + 1:b:2] = mz[a:b - 1:2]
            it[a + 1:b:2] = it[a:b - 1:2]
    sp = Spectra("scale", np.arange(n, dtype=np.uint32), np.arange(n, dtype=np.uint32), np.zeros(n),
                 rng.uniform(400, 1200, n), np.full(n, 2, np.int8), mz, it, off)
    kw = {"global150": dict(max_peaks=150), "global512": dict(max_peaks=512),
          "window15": dict(peak_mode="window", window_k=15), "window4": dict(peak_mode="window", window_k=4)}[mode]
    p = SearchParams(**kw)
    pk = E.k0_preprocess(sp, p, torch_cuda.device("cuda"), E.Stats())
    _assert_view(pk, O.k0_view(sp, p))
