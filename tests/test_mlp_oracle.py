"""CPU checks of the pruner's oracle: BF16 rounding, the float64 backpropagation against finite differences, the
f32 training pass against the float64 one, the Adam step against torch's, and the pruned selection's rules."""
import numpy as np
import pytest
import torch

from oracle import mlp_oracle as M
from oracle import oracle as O


def test_bf16_round_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(0, 10, 100000), rng.normal(0, 1e-30, 1000), [0.0, -0.0, 1.0, 65504.0, 3e38,
                                                                               -3e38, 1.00390625, 1.01171875]])
    x = x.astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(M.bf16_round(x).view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(M.from_bf16_bits(M.bf16_bits(ref)), ref)


def _small_params(rng, n_in=16, h=8):
    return {"W1": rng.normal(0, 0.5, (h, n_in)), "b1": rng.normal(0, 0.1, h), "W2": rng.normal(0, 0.5, (h, h)),
            "b2": rng.normal(0, 0.1, h), "w3": rng.normal(0, 0.5, h), "b3": rng.normal(0, 0.1, 1)}


def test_f64_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    P = _small_params(rng)
    X = rng.normal(0, 1, (64, 16))
    y = (rng.random(64) < 0.3).astype(np.float64)
    w = rng.uniform(0.5, 2.0, 64)
    g = M.grad_f64(P, X, y, w)
    eps = 1e-6
    for k, v in P.items():
        flat = v.reshape(-1)
        for i in rng.choice(flat.size, min(flat.size, 12), replace=False):
            old = flat[i]
            flat[i] = old + eps
            lp = M.loss_f64(P, X, y, w)
            flat[i] = old - eps
            lm = M.loss_f64(P, X, y, w)
            flat[i] = old
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - g[k].reshape(-1)[i]) <= 1e-6 + 1e-4 * abs(fd), (k, i, fd, g[k].reshape(-1)[i])


def test_f32_training_pass_tracks_f64():
    """The f32 training pass (BF16 weights and layer-1 activations) is the float64 network up to BF16 rounding."""
    rng = np.random.default_rng(2)
    h = M.HIDDEN
    P = {"W1": rng.normal(0, 0.3, (h, 16)), "b1": rng.normal(0, 0.1, h), "W2": rng.normal(0, 0.06, (h, h)),
         "b2": rng.normal(0, 0.1, h), "w3": rng.normal(0, 0.06, h), "b3": rng.normal(0, 0.1, 1)}
    X = M.bf16_round(rng.normal(0, 1, (96, 16)).astype(np.float32))
    W1b = M.bf16_round(P["W1"].astype(np.float32))
    W2b = M.bf16_round(P["W2"].astype(np.float32))
    H1, H2, z = M.forward_train(X, W1b, P["b1"].astype(np.float32), W2b, P["b2"].astype(np.float32),
                                P["w3"].astype(np.float32), P["b3"].astype(np.float32))
    zl = M.logits(X, W1b, P["b1"], W2b, P["b2"], P["w3"], P["b3"])
    np.testing.assert_allclose(z, zl, rtol=1e-3, atol=1e-3)
    y = (rng.random(96) < 0.3).astype(np.float32)
    w = np.ones(96, np.float32)
    dz, loss = M.bce(z, y, w, 1.0 / 96)
    g = M.backward(X, H1, H2, dz, W2b, P["w3"].astype(np.float32))
    Pb = dict(P, W1=W1b.astype(np.float64), W2=W2b.astype(np.float64))
    g64 = M.grad_f64(Pb, X.astype(np.float64), y.astype(np.float64), w.astype(np.float64))
    for k in g:   # relative Frobenius error (ReLU masks may flip for pre-activations near 0 under BF16 rounding)
        assert np.linalg.norm(g[k] - g64[k]) <= 0.05 * np.linalg.norm(g64[k]), k


def test_adam_matches_torch():
    rng = np.random.default_rng(3)
    p0 = rng.normal(0, 1, 1000).astype(np.float32)
    pt = torch.nn.Parameter(torch.from_numpy(p0.copy()))
    opt = torch.optim.Adam([pt], lr=1e-2, betas=(0.9, 0.999), eps=1e-8, weight_decay=1e-4)
    p, m, v = p0.copy(), np.zeros_like(p0), np.zeros_like(p0)
    for step in range(1, 6):
        g = rng.normal(0, 1, 1000).astype(np.float32)
        pt.grad = torch.from_numpy(g.copy())
        opt.step()
        p, m, v = M.adam(p, g, m, v, 1e-2, 0.9, 0.999, 1e-8, step, 1e-4)
    np.testing.assert_allclose(p, pt.detach().numpy(), rtol=2e-6, atol=2e-7)


def test_select_pruned_rules():
    # 2 spectra; hits in (row, hyp) order; partner = row ^ 1
    partner = np.arange(64) ^ 1
    hit_off = np.array([0, 5, 8])
    hyp = np.array([0, 1, 0, 0, 1, 2, 2, 3])
    row = np.array([2, 2, 7, 10, 12, 20, 31, 40])
    cnt = np.array([5, 9, 3, 3, 1, 4, 4, 2])
    logit = np.array([0.5, 0.5, 2.0, -1.0, 3.0, -5.0, -5.0, -6.0], np.float32)
    spec_hyp_off = np.array([0, 2, 4])
    out = O.select_pruned(spec_hyp_off, hit_off, hyp, row, cnt, logit, tau=0.4, min_keep=1, max_keep=16,
                          partner=partner)
    h, r, c = out[0]
    # kept: rows 12 (3.0), 7 (2.0), 2 (0.5, both hyps); closure adds 13, 6, 3
    assert r.tolist() == [2, 3, 6, 7, 12, 13]
    assert h.tolist() == [0, 0, 0, 0, 1, 1]
    assert c.tolist() == [9, -1, -1, 3, 1, -1]
    h, r, c = out[1]
    # nothing reaches tau: min_keep = 1 keeps the best by (logit, count, position): rows 20 and 31 tie on (logit,
    # count); the later position (row 31) wins
    assert r.tolist() == [30, 31] and c.tolist() == [-1, 4]
    out = O.select_pruned(spec_hyp_off, hit_off, hyp, row, cnt, logit, tau=-np.inf, min_keep=0, max_keep=2,
                          partner=partner, pair_closure=False)
    assert out[0][1].tolist() == [7, 12]
