"""CPU oracle of the learned candidate pruner (test infrastructure: only tests, the smoke check and the benchmark's
CPU baseline use it; nothing in the product imports it).

The pruner has no counterpart in the reference (it adds a learned filter in front of the reference's exact
rescoring, ``vulcan/gpu/engine.py:315-351``), so this oracle pins the arithmetic of the CUDA kernels instead:

* ``raw_features`` / ``standardise``: the per-hit features of ``vk_cand_features`` in the same f32 operations and
  the same round-to-nearest-even BF16 conversion (bit-exact);
* ``forward_train`` / ``backward``: the training pass of ``mlp_train.cu`` with its FP32 SIMT GEMMs -- every
  matrix product summed sequentially over k in f32 with separately rounded products (the kernels compile without
  FMA contraction), ReLU, BF16 rounding of the layer-1 activations, the bias and layer-3 gradients as column sums in
  vk_colsum's chunked order -- so given the same loss gradient ``dz`` every weight gradient is bit-identical (the
  tensor-core GEMMs of ``mlp_train_tc.cu`` are checked against it within a tolerance);
* ``bce`` / ``adam``: the loss gradient and the optimiser step (within a few f32 ulps: ``expf`` / ``powf`` of the
  device and of numpy may differ in the last bit);
* ``logits``: the inference network in float64 with the layer-1 activations rounded to BF16, the reference value
  for the tensor-core kernel (which sums in a different order);
* ``grad_f64``: the analytic gradient of the weighted BCE in float64, checked against finite differences.
"""
from __future__ import annotations

import numpy as np

N_IN = 16
HIDDEN = 256
N_FEAT = 6


def bf16_round(x: np.ndarray) -> np.ndarray:
    """f32 -> nearest BF16 value (ties to even), returned as f32 (NaN kept)."""
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(x), x, out)


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """uint16 bit patterns of BF16 values given as f32."""
    return (np.ascontiguousarray(x, np.float32).view(np.uint32) >> 16).astype(np.uint16)


def from_bf16_bits(b: np.ndarray) -> np.ndarray:
    return (np.asarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32)


def raw_features(c_hyp, c_row, c_cnt, win_off, lo, isum, M, z, mass32, length, missed) -> np.ndarray:
    """[n, 6] f32 raw features of the hits (hyp, row, count)."""
    h = np.asarray(c_hyp, np.int64)
    r = np.asarray(c_row, np.int64)
    mr = np.asarray(mass32, np.float32)[r]
    Mh = np.asarray(M, np.float32)[h]
    pos = np.asarray(win_off, np.int64)[h] + (r - np.asarray(lo, np.int64)[h])
    f = np.empty((len(h), N_FEAT), np.float32)
    f[:, 0] = np.asarray(c_cnt).astype(np.float32)
    f[:, 1] = np.asarray(isum, np.uint32)[pos].astype(np.float32) * np.float32(1.0 / 16777216.0)
    f[:, 2] = (Mh - mr) / mr * np.float32(1.0e6)
    f[:, 3] = np.asarray(z, np.int8)[h].astype(np.float32)
    f[:, 4] = np.asarray(length, np.uint8)[r].astype(np.float32)
    f[:, 5] = np.asarray(missed, np.uint8)[r].astype(np.float32)
    return f


def standardise(raw: np.ndarray, mu: np.ndarray, sd: np.ndarray) -> np.ndarray:
    """[n, 16] BF16 values (as f32) of (raw - mu) / sd, zero padded."""
    out = np.zeros((len(raw), N_IN), np.float32)
    mu = np.asarray(mu, np.float32)[:N_FEAT]
    sd = np.asarray(sd, np.float32)[:N_FEAT]
    out[:, :N_FEAT] = bf16_round((np.asarray(raw, np.float32) - mu) / sd)
    return out


def _seq_matmul(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    """C[m, n] = sum_k A[m, k] * B[k, n], summed in f32 sequentially over k with separately rounded products."""
    A = np.asarray(A, np.float32)
    B = np.asarray(B, np.float32)
    C = np.zeros((A.shape[0], B.shape[1]), np.float32)
    for k in range(A.shape[1]):
        C = C + np.outer(A[:, k], B[k, :]).astype(np.float32)
    return C


def forward_train(X, W1b, b1, W2b, b2, w3, b3):
    """(H1, H2, z) of the training forward: H1 = bf16(relu(X W1^T + b1)), H2 = relu(H1 W2^T + b2),
    z = H2 w3 + b3 (f32, sequential sums)."""
    H1 = bf16_round(np.maximum(_seq_matmul(X, np.asarray(W1b, np.float32).T) + np.float32(b1), np.float32(0)))
    H2 = np.maximum(_seq_matmul(H1, np.asarray(W2b, np.float32).T) + np.asarray(b2, np.float32), np.float32(0))
    z = _seq_matmul(H2, np.asarray(w3, np.float32)[:, None])[:, 0] + np.float32(np.asarray(b3).reshape(-1)[0])
    return H1, H2, z.astype(np.float32)


def bce(z, y, w, inv_wsum):
    """(dz, loss) of the weighted BCE with logits (f32)."""
    z = np.asarray(z, np.float32)
    y = np.asarray(y, np.float32)
    w = np.asarray(w, np.float32)
    p = np.float32(1) / (np.float32(1) + np.exp(-z))
    dz = w * (p - y) * np.float32(inv_wsum)
    loss = w * (np.log1p(np.exp(-np.abs(z))) + np.maximum(z, 0) - z * y) * np.float32(inv_wsum)
    return dz.astype(np.float32), float(np.sum(loss, dtype=np.float64))


CS_ROWS = 64   # rows per chunk of the device column sums (csrc/mlp_train.cu, vk_colsum)


def _colsum(D, v=None):
    """Column sums in vk_colsum's order: rows in chunks of CS_ROWS summed sequentially (each term v[i] * D[i] as
    one rounded product when a row weight v is given), the chunk sums added in chunk order."""
    D = np.asarray(D, np.float32)
    tot = np.zeros(D.shape[1], np.float32)
    for c0 in range(0, D.shape[0], CS_ROWS):
        s = np.zeros(D.shape[1], np.float32)
        for i in range(c0, min(D.shape[0], c0 + CS_ROWS)):
            s = s + (D[i] if v is None else (D[i] * np.float32(v[i])).astype(np.float32))
        tot = tot + s
    return tot


def backward(X, H1, H2, dz, W2b, w3):
    """Gradients {W1, b1, W2, b2, w3, b3} from the loss gradient dz, in the kernels' summation order."""
    dz = np.asarray(dz, np.float32)
    g = {"w3": _colsum(H2, dz), "b3": _colsum(dz[:, None])}
    dH2 = (dz[:, None] * np.asarray(w3, np.float32)[None, :]).astype(np.float32)
    dH2 = np.where(H2 > 0, dH2, np.float32(0))
    g["W2"] = _seq_matmul(dH2.T, H1)
    g["b2"] = _colsum(dH2)
    dH1 = _seq_matmul(dH2, np.asarray(W2b, np.float32))
    dH1 = np.where(H1 > 0, dH1, np.float32(0))
    g["W1"] = _seq_matmul(dH1.T, X)
    g["b1"] = _colsum(dH1)
    return g


def adam(p, g, m, v, lr, b1, b2, eps, step, wd):
    """One Adam step in f32 (L2 term wd * p added to the gradient).  Returns (p, m, v)."""
    f = np.float32
    p, g, m, v = (np.asarray(a, np.float32) for a in (p, g, m, v))
    c1 = f(1) - f(np.power(f(b1), f(step)))
    c2 = f(1) - f(np.power(f(b2), f(step)))
    gi = g + f(wd) * p
    mi = f(b1) * m + (f(1) - f(b1)) * gi
    vi = f(b2) * v + (f(1) - f(b2)) * gi * gi
    pi = p - f(lr) * (mi / c1) / (np.sqrt(vi / c2) + f(eps))
    return pi.astype(np.float32), mi.astype(np.float32), vi.astype(np.float32)


def logits(Xb, W1b, b1, W2b, b2, w3, b3) -> np.ndarray:
    """Inference logits in float64 with the layer-1 activations rounded to BF16 (the inference kernel's
    activation format)."""
    X = np.asarray(Xb, np.float64)
    h1 = np.maximum(X @ np.asarray(W1b, np.float64).T + np.asarray(b1, np.float64), 0.0)
    h1 = bf16_round(h1.astype(np.float32)).astype(np.float64)
    h2 = np.maximum(h1 @ np.asarray(W2b, np.float64).T + np.asarray(b2, np.float64), 0.0)
    return h2 @ np.asarray(w3, np.float64) + float(np.asarray(b3).reshape(-1)[0])


def loss_f64(params: dict, X, y, w) -> float:
    """Weighted mean BCE of the float64 network (no BF16 rounding)."""
    X = np.asarray(X, np.float64)
    h1 = np.maximum(X @ params["W1"].T + params["b1"], 0.0)
    h2 = np.maximum(h1 @ params["W2"].T + params["b2"], 0.0)
    z = h2 @ params["w3"] + params["b3"][0]
    lz = np.log1p(np.exp(-np.abs(z))) + np.maximum(z, 0) - z * y
    return float(np.sum(w * lz) / np.sum(w))


def grad_f64(params: dict, X, y, w) -> dict:
    """Analytic gradient of ``loss_f64`` (float64 backpropagation)."""
    X = np.asarray(X, np.float64)
    a1 = X @ params["W1"].T + params["b1"]
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ params["W2"].T + params["b2"]
    h2 = np.maximum(a2, 0.0)
    z = h2 @ params["w3"] + params["b3"][0]
    dz = w * (1.0 / (1.0 + np.exp(-z)) - y) / np.sum(w)
    g = {"w3": h2.T @ dz, "b3": np.array([dz.sum()])}
    d2 = np.outer(dz, params["w3"]) * (a2 > 0)
    g["W2"] = d2.T @ h1
    g["b2"] = d2.sum(0)
    d1 = (d2 @ params["W2"]) * (a1 > 0)
    g["W1"] = d1.T @ X
    g["b1"] = d1.sum(0)
    return g
