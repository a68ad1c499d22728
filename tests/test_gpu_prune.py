"""The learned candidate pruner on the GPU: its kernels against the CPU oracle (K1 intensity sums, features,
inference, the training forward / backward / Adam step, the pruned selection), the pruned search without pruning
against the plain search, and a trained pruner on the small workload (recall, rescoring work, gain over count-only
pruning)."""
import math

import numpy as np
import pytest

from oracle import mlp_oracle as M
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SETS = ("da", "ppm", "ppm_mfz")
STATIC = {"C": 57.021464}
VAR = {"M": 15.9949}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    return torch


@pytest.fixture(scope="module")
def indexes(mini, param_sets, torch_cuda):
    from vulcan.gpu import engine as E
    l1, _, _ = mini
    return {name: E.GpuIndex(l1, p, STATIC, VAR) for name, p in param_sets.items()}


def _front(sp, gi, p, dense=True):
    """The pruned search's front end; dense: with K1's dense per-row counts and intensity sums (the hit-list form
    keeps only the shortlist's)."""
    from vulcan.gpu import engine as E
    from vulcan.gpu import prune as PR
    st = E.Stats()
    run = E.DeviceRun(sp, gi.dev, st)
    return PR._front(run, gi, p, st, False, dense=dense)


def _np(t):
    return t.cpu().numpy()


@pytest.mark.parametrize("name", SETS)
def test_k1_intensity_sums_equal_oracle(mini, param_sets, indexes, name):
    l1, sp, _ = mini
    p = param_sets[name]
    gi = indexes[name]
    f = _front(sp, gi, p)
    dh = f["dh"]
    hyp = {k: _np(dh[k]) for k in ("spec", "maxfz", "lo", "hi")}
    pk = {"off": _np(f["peaks"]["off"]), "mass": _np(f["peaks"]["mass"]), "int": _np(f["peaks"]["int"])}
    P = O.make_params(STATIC, VAR, p.fragment_unit)
    win_off, cnt, _, _, isum = O.k1_windows(l1, hyp, pk, p, P, tic=_np(f["peaks"]["tic"]))
    assert np.array_equal(_np(f["win_off"]), win_off)
    n_win = int(f["win_off"][-1])
    assert np.array_equal(_np(f["cnt"][:n_win]), cnt)
    assert np.array_equal(_np(f["isum"][:n_win]).view(np.uint32), isum)
    assert isum.max() > 0


@pytest.mark.parametrize("name", SETS)
def test_features_equal_oracle(mini, param_sets, indexes, name, torch_cuda):
    torch = torch_cuda
    from vulcan.gpu import prune as PR
    l1, sp, _ = mini
    p = param_sets[name]
    gi = indexes[name]
    f = _front(sp, gi, p)
    hits = f["hits"]
    n = int(hits["cand_off"][-1])
    assert n > 0
    pr = PR.Pruner(gi.dev, seed=1)
    pr.mu[:6] = torch.tensor([3.0, 0.05, 0.1, 2.5, 14.0, 0.4], device=gi.dev)
    pr.sd[:6] = torch.tensor([2.0, 0.03, 5.7, 0.6, 5.0, 0.6], device=gi.dev)
    feat = pr.features(gi, f["dh"], f["win_off"], f["isum"], hits, n)[:n]
    dh = f["dh"]
    raw = M.raw_features(_np(hits["c_hyp"][:n]), _np(hits["c_row"][:n]), _np(hits["c_cnt"][:n]), _np(f["win_off"]),
                         _np(dh["lo"]), _np(f["isum"]).view(np.uint32), _np(dh["M"]), _np(dh["z"]), l1.mass32,
                         l1.length, l1.missed)
    want = M.standardise(raw, _np(pr.mu), _np(pr.sd))
    got = _np(feat.view(torch.int16)).view(np.uint16)
    assert np.array_equal(got, M.bf16_bits(want))
    # the device-count form reads the count on the device and leaves the rest of the buffer untouched
    n_dev = hits["cand_off"][-1:]
    feat2 = pr.features(gi, f["dh"], f["win_off"], f["isum"], hits, n + 37, n_dev=n_dev)
    assert torch.equal(feat2[:n], feat)
    # the hit-list front end (intensity sums carried with the shortlist) gives the same features
    fh = _front(sp, gi, p, dense=False)
    assert int(fh["hits"]["cand_off"][-1]) == n
    feat3 = pr.features(gi, fh["dh"], fh["win_off"], None, fh["hits"], n)[:n]
    assert torch.equal(feat3, feat)


def _random_pruner(torch, dev, seed):
    from vulcan.gpu import prune as PR
    pr = PR.Pruner(dev, seed=seed)
    g = torch.Generator(device="cpu").manual_seed(seed + 100)
    pr.w["b1"] = (torch.randn(256, generator=g) * 0.1).to(dev)
    pr.w["b2"] = (torch.randn(256, generator=g) * 0.1).to(dev)
    pr.w["W1"] = (torch.randn(256, 16, generator=g) * 0.4).to(dev)
    pr.w["b3"] = torch.tensor([0.25], device=dev)
    pr._sync_bf16()
    return pr


def _weights_np(pr, torch):
    W1b = _np(pr.bf["W1"].float())
    W2b = _np(pr.bf["W2"].float())
    return W1b, _np(pr.w["b1"]), W2b, _np(pr.w["b2"]), _np(pr.w["w3"]), _np(pr.w["b3"])


@pytest.mark.parametrize("kernel", ["tcgen05", "mma.sync"])
@pytest.mark.parametrize("n", [1, 16, 1037, 40000])
def test_mlp_inference_matches_oracle(torch_cuda, n, kernel):
    torch = torch_cuda
    dev = torch.device("cuda")
    pr = _random_pruner(torch, dev, 7)
    pr.tensor_cores = kernel
    g = torch.Generator(device="cpu").manual_seed(n)
    X = torch.zeros(n, 16)
    X[:, :6] = torch.randn(n, 6, generator=g) * 1.5
    Xb = X.to(torch.bfloat16).to(dev)
    z = _np(pr.logits(Xb, n))
    want = M.logits(_np(Xb.float()), *_weights_np(pr, torch))
    # layer-1 activations are rounded to BF16 after a differently ordered f32 sum: rare one-ulp flips
    np.testing.assert_allclose(z, want, rtol=2e-3, atol=2e-3)
    # the training forward computes the same network (fixed order): agrees to the same tolerance
    if n <= 1037:
        zt = _np(pr.forward_train(Xb.float().contiguous(), n).clone())
        np.testing.assert_allclose(zt, want, rtol=2e-3, atol=2e-3)
    # a device count below the buffer size scores only that many rows
    if n > 16:
        out = torch.full((n,), 123.0, device=dev)
        cnt = torch.tensor([n - 9], dtype=torch.int64, device=dev)
        from vulcan.gpu import _lib as K
        args = (K.ptr(Xb), K.ptr(pr.bf["W1"]), K.ptr(pr.w["b1"]), K.ptr(pr.bf["W2"]), K.ptr(pr.w["b2"]),
                K.ptr(pr.w["w3"]), pr._b3, K.ptr(out), 3)
        if kernel == "tcgen05":
            st = torch.zeros(1, dtype=torch.int32, device=dev)
            K.check(K.lib().vk_mlp_infer_tc(n, K.ptr(cnt), *args, K.ptr(st), K.stream()), "mlp_infer_tc")
            assert int(st.item()) == 0
        else:
            K.check(K.lib().vk_mlp_infer(n, K.ptr(cnt), *args, K.stream()), "mlp_infer")
        o = _np(out)
        np.testing.assert_array_equal(o[:n - 9], z[:n - 9])
        assert np.all(o[n - 9:] == 123.0)


@pytest.mark.parametrize("B", [200, 4096])
def test_training_pass_equals_oracle(torch_cuda, B):
    """With the SIMT GEMMs: forward activations and every weight gradient bit-identical to the oracle's f32 pass
    (given the device's loss gradient); the loss gradient and the Adam step within f32 ulps."""
    torch = torch_cuda
    dev = torch.device("cuda")
    pr = _random_pruner(torch, dev, 11)
    pr.train_gemm = "simt"
    g = torch.Generator(device="cpu").manual_seed(B)
    X = torch.zeros(B, 16)
    X[:, :6] = torch.randn(B, 6, generator=g)
    X = X.to(torch.bfloat16).float().to(dev).contiguous()
    y = (torch.rand(B, generator=g) < 0.2).float().to(dev)
    w = (0.5 + torch.rand(B, generator=g)).to(dev)
    z = pr.forward_train(X, B)
    loss, grads = pr.backward(X, y, w, B, 1.0 / B)
    W1b, b1, W2b, b2, w3, b3 = _weights_np(pr, torch)
    Xn = _np(X)
    H1, H2, zo = M.forward_train(Xn, W1b, b1, W2b, b2, w3, b3)
    assert np.array_equal(_np(pr._buf["H1"][:B]), H1)
    assert np.array_equal(_np(pr._buf["H2"][:B]), H2)
    assert np.array_equal(_np(z), zo)
    dz_o, loss_o = M.bce(zo, _np(y), _np(w), 1.0 / B)
    dz = _np(pr._buf["dz"][:B])
    np.testing.assert_allclose(dz, dz_o, rtol=1e-5, atol=1e-9)
    assert abs(float(loss.sum()) - loss_o) <= 1e-5 * abs(loss_o)
    go = M.backward(Xn, H1, H2, dz, W2b, w3)
    for k in ("W1", "b1", "W2", "b2", "w3", "b3"):
        assert np.array_equal(_np(grads[k]).reshape(go[k].shape), go[k]), k
    # one Adam step on every parameter
    before = {k: _np(v).copy() for k, v in pr.w.items()}
    gr = {k: _np(v).copy() for k, v in grads.items()}
    pr.adam_step(1e-3, wd=1e-4)
    for k in before:
        pw, _, _ = M.adam(before[k], gr[k], np.zeros_like(before[k]), np.zeros_like(before[k]), 1e-3, 0.9, 0.999,
                          1e-8, 1, 1e-4)
        np.testing.assert_allclose(_np(pr.w[k]), pw, rtol=1e-6, atol=1e-9)
    np.testing.assert_array_equal(_np(pr.bf["W2"].float()), M.bf16_round(_np(pr.w["W2"])))


def test_compacted_features_equal_the_features_kernel(mini, param_sets, indexes, torch_cuda):
    """The pruned front end's compaction writes every shortlist hit's features (``vk_compact_hits_features``):
    the rows ``vk_cand_features`` computes from the compacted hits, bit for bit."""
    torch = torch_cuda
    from vulcan.gpu import engine as E
    from vulcan.gpu import prune as PR
    l1, sp, _ = mini
    for name in SETS:
        p = param_sets[name]
        gi = indexes[name]
        pr = PR.Pruner(gi.dev, seed=3)
        g = torch.Generator(device="cpu").manual_seed(4)
        pr.mu[:6] = (torch.randn(6, generator=g) * 2).to(gi.dev)
        pr.sd[:6] = (0.5 + torch.rand(6, generator=g)).to(gi.dev)
        st = E.Stats()
        f = PR._front(E.DeviceRun(sp, gi.dev, st), gi, p, st, False, min_count=1, pr=pr)
        hits = f["hits"]
        nc = int(hits["cand_off"][len(sp)])
        assert nc > 100 and "feat" in hits
        want = pr.features(gi, f["dh"], f["win_off"], None, hits, nc)
        assert torch.equal(hits["feat"][:nc], want[:nc]), name


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64)) /
                 max(np.linalg.norm(np.asarray(b, np.float64)), 1e-30))


@pytest.mark.parametrize("B", [200, 4096, 8192])
def test_training_pass_on_tensor_cores_close_to_oracle(torch_cuda, B):
    """With the tcgen05 GEMMs (BF16 operands, FP32 accumulation, K split over the batch for the weight gradients):
    forward activations within BF16 rounding of the oracle's f32 pass, every weight gradient within 1% (relative
    norm) of the oracle's gradients of the same activations, and the f64 gradient of the loss within 2%."""
    torch = torch_cuda
    dev = torch.device("cuda")
    pr = _random_pruner(torch, dev, 11)
    assert pr.train_gemm == "tcgen05"
    g = torch.Generator(device="cpu").manual_seed(B + 1)
    X = torch.zeros(B, 16)
    X[:, :6] = torch.randn(B, 6, generator=g)
    X = X.to(torch.bfloat16).float().to(dev).contiguous()
    y = (torch.rand(B, generator=g) < 0.2).float().to(dev)
    w = (0.5 + torch.rand(B, generator=g)).to(dev)
    z = pr.forward_train(X, B)
    loss, grads = pr.backward(X, y, w, B, 1.0 / float(w.sum()))
    W1b, b1, W2b, b2, w3, b3 = _weights_np(pr, torch)
    Xn = _np(X)
    H1o, H2o, zo = M.forward_train(Xn, W1b, b1, W2b, b2, w3, b3)
    H1, H2 = _np(pr._buf["H1"][:B]), _np(pr._buf["H2"][:B])
    assert _rel(H1, H1o) < 4e-3 and _rel(H2, H2o) < 1e-2 and _rel(_np(z), zo) < 1e-2
    dz = _np(pr._buf["dz"][:B])
    go = M.backward(Xn, H1, H2, dz, W2b, w3)
    for k in ("W1", "b1", "W2", "b2", "w3", "b3"):
        assert _rel(_np(grads[k]).reshape(go[k].shape), go[k]) < 1e-2, k
    params = {"W1": W1b.astype(np.float64), "b1": b1, "W2": W2b.astype(np.float64), "b2": b2, "w3": w3, "b3": b3}
    g64 = M.grad_f64(params, Xn, _np(y), _np(w))
    for k in ("W1", "W2", "w3"):
        assert _rel(_np(grads[k]).reshape(g64[k].shape), g64[k]) < 2e-2, k
    assert int(pr._buf["status"].item()) == 0


@pytest.mark.parametrize("name", SETS)
@pytest.mark.parametrize("keep", [(0.0, 1, 16, 1), (0.5, 2, 32, 1), (-math.inf, 0, 16, 0), (1.5, 0, 128, 1)])
def test_select_pruned_equals_oracle(mini, param_sets, indexes, name, keep, torch_cuda):
    torch = torch_cuda
    from vulcan.gpu import _lib as K
    l1, sp, _ = mini
    p = param_sets[name]
    gi = indexes[name]
    f = _front(sp, gi, p)
    hits = f["hits"]
    n_spec = len(sp)
    n = int(hits["cand_off"][-1])
    tau, min_keep, max_keep, closure = keep
    g = torch.Generator(device="cpu").manual_seed(5)
    logit = torch.round(torch.randn(max(n, 1), generator=g) * 4) / 4      # many exact ties
    logit = logit.to(gi.dev)
    cap = (2 if closure else 1) * max_keep
    out = {k: torch.full((n_spec * cap,), -7, dtype=torch.int64, device=gi.dev) for k in ("h", "r", "c")}
    n_cand = torch.empty(n_spec, dtype=torch.int64, device=gi.dev)
    K.check(K.lib().vk_select_pruned(n_spec, K.ptr(f["dh"]["spec_off"]), K.ptr(hits["cand_off"]),
                                     K.ptr(hits["c_hyp"]), K.ptr(hits["c_row32"]), K.ptr(hits["c_cnt"]),
                                     K.ptr(logit), tau, min_keep, max_keep, closure, K.ptr(gi.partner), cap,
                                     p.topk, K.ptr(out["h"]), K.ptr(out["r"]), K.ptr(out["c"]), K.ptr(n_cand), K.stream()),
            "select_pruned")
    want = O.select_pruned(_np(f["dh"]["spec_off"]), _np(hits["cand_off"]), _np(hits["c_hyp"][:n]),
                           _np(hits["c_row"][:n]), _np(hits["c_cnt"][:n]), _np(logit[:n]), tau, min_keep, max_keep,
                           l1.partner, pair_closure=bool(closure))
    nc = _np(n_cand)
    o = {k: _np(v).reshape(n_spec, cap) for k, v in out.items()}
    for s in range(n_spec):
        h, r, c = want[s]
        assert nc[s] == len(r), s
        assert np.array_equal(o["h"][s, :nc[s]], h) and np.array_equal(o["r"][s, :nc[s]], r)
        assert np.array_equal(o["c"][s, :nc[s]], c), s


@pytest.mark.parametrize("name", SETS)
def test_pruned_search_without_pruning_is_plain(mini, param_sets, indexes, name, torch_cuda):
    from vulcan.gpu import engine as E
    from vulcan.gpu import prune as PR
    l1, sp, _ = mini
    p = param_sets[name]
    gi = indexes[name]
    pr = PR.Pruner(gi.dev, seed=3, tau=-math.inf, min_keep=0, max_keep=16)
    assert p.topk <= pr.max_keep
    t_plain, s_plain, _ = E.search(sp, gi, l1, p, report=3)
    t_pr, s_pr, out = PR.search_pruned(sp, gi, l1, p, pr, report=3)
    assert t_pr.equals(t_plain)
    assert s_pr.counts["n_rescored"] == s_plain.counts["n_rescored"]


@pytest.mark.parametrize("name", SETS)
def test_graphed_pruned_search_equals_search_pruned(mini, param_sets, indexes, name, torch_cuda):
    """The graph-captured Searcher with a pruner returns search_pruned's PSM table (random network, threshold at
    the median logit so that the selection prunes)."""
    from vulcan.gpu import engine as E
    from vulcan.gpu import prune as PR
    l1, sp, _ = mini
    p = param_sets[name]
    gi = indexes[name]
    pr = _random_pruner(torch_cuda, gi.dev, 5)
    pr.tau, pr.min_keep, pr.max_keep, pr.min_count = 0.0, 1, 16, 2
    want, st, out = PR.search_pruned(sp, gi, l1, p, pr, report=2)
    assert st.counts["n_rescored"] < st.counts["n_hits"] * 2
    se = E.Searcher(gi, l1, p, pruner=pr, report=2)
    for tbl, _ in se.search_many([sp, sp, sp]):
        assert tbl.equals(want)


def test_batched_pruned_search_equals_per_run(mini, param_sets, indexes, torch_cuda):
    """The pruned path in padded batches gives every run's own search_pruned table."""
    from vulcan.gpu import engine as E
    from vulcan.gpu import prune as PR
    from vulcan.gpu.host import Spectra
    l1, sp, _ = mini
    p = param_sets["ppm"]
    gi = indexes["ppm"]
    pr = _random_pruner(torch_cuda, gi.dev, 9)
    pr.tau, pr.min_keep, pr.max_keep, pr.min_count = 0.0, 1, 16, 2
    runs = []
    for i, (a, b) in enumerate(((0, 50), (50, 51), (51, 160))):
        o = sp.offsets[a:b + 1]
        runs.append(Spectra(f"r{i}", sp.scan[a:b], sp.index[a:b], sp.rt[a:b], sp.precursor_mz[a:b], sp.charge[a:b],
                            sp.mz[o[0]:o[-1]], sp.intensity[o[0]:o[-1]], o - o[0]))
    se = E.Searcher(gi, l1, p, pruner=pr, report=1)
    for r, (tbl, _) in zip(runs, se.search_batch(runs, batch_spectra=60)):
        assert tbl.equals(PR.search_pruned(r, gi, l1, p, pr, report=1)[0]), r.run
    # with a shortlist cap: the MLP sees the top 3 hits by count of every spectrum, in batches too
    pr.shortlist_k = 3
    se = E.Searcher(gi, l1, p, pruner=pr, report=1)
    for r, (tbl, _) in zip(runs, se.search_batch(runs, batch_spectra=60)):
        assert tbl.equals(PR.search_pruned(r, gi, l1, p, pr, report=1)[0]), r.run
    st = PR.search_pruned(sp, gi, l1, p, pr, report=1)[1]
    assert 0 < st.counts["n_hits"] <= 3 * len(sp)


# ------------------------------------------------------------------------------------------- trained pruner
@pytest.fixture(scope="module")
def small(tmp_path_factory, torch_cuda):
    from vulcan import synth
    from vulcan.gpu import engine as E
    from vulcan.index.build import L1Index, read_labels
    root = str(tmp_path_factory.mktemp("idx"))
    d = synth.build_index("small", root)
    l1, lab = L1Index(d), read_labels(d)
    p = synth.WORKLOADS["small"].search_params()
    gi = E.GpuIndex(l1, p, {"C": 57.021464}, synth.WORKLOADS["small"].var_mods)
    runs = [synth.simulate_run(l1, lab, "small", seed=1000 + i, run=f"r{i}")[0] for i in range(4)]
    return l1, lab, p, gi, runs


def test_trained_pruner_small_workload(small):
    """Train on two runs, calibrate on a third, judge on a held-out run against the plain path; compare with
    the count-only ranking calibrated the same way."""
    from vulcan.gpu import prune as PR
    l1, lab, p, gi, runs = small
    pr, info = PR.train(gi, p, runs[:2], runs[2:3], epochs=3, batch=2048, target=0.9995)
    assert info["losses"][-1] < info["losses"][0]
    assert pr.shortlist_k == 0 or pr.shortlist_k in PR.SHORTLIST_KS
    back = PR.Pruner(gi.dev).load_state_dict(pr.state_dict())
    assert (back.shortlist_k, back.min_count, back.tau) == (pr.shortlist_k, pr.min_count, pr.tau)
    ev = PR.evaluate(runs[3], gi, l1, lab, p, pr)
    assert ev["recall"] >= 0.998, ev
    assert ev["rescored_pruned"] < ev["rescored_plain"], ev
    assert abs(ev["delta_accepted"]) <= 0.005, ev
    cr = PR.count_ranker(gi, p, runs[2:3], target=0.9995)
    ev_c = PR.evaluate(runs[3], gi, l1, lab, p, cr)
    # the gain of the network: fewer candidates rescored than count-only pruning at the same calibration target
    assert ev["rescored_pruned"] < ev_c["rescored_pruned"], (ev, ev_c)
