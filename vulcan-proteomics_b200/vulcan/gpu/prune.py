"""Learned candidate pruner: a BF16 MLP that predicts which index hits survive exact rescoring.

The plain path rescores (K2) every candidate of its shortlist: the top-k index hits of a spectrum by K1 count plus
their target/decoy partners.  The pruned path computes the same shortlist without pair closure, scores each hit with
the MLP, keeps the hits whose logit reaches a calibrated threshold ``tau`` (and the ``min_keep`` best of every
spectrum), then applies pair closure and rescores only those.  Pruned candidates are therefore a subset of the
plain path's; the plain path stays the fallback (``search_pruned`` without a trained pruner) and the judge of the
pruned path's recall (``evaluate``).  Nothing here reads target/decoy labels during a search: the features are
label-free and pair closure runs after the pruning, so targets and decoys are treated alike.

Features per hit (``vk_cand_features``): K1 shared-peak count, summed matched intensity (fraction of the spectrum's
TIC, K1's fixed-point sums), precursor error in ppm, precursor charge, peptide length, missed cleavages.
Network: 16 -> 256 (ReLU) -> 256 (ReLU) -> 1, BF16 weights and layer-1 activations, FP32 accumulation; inference
on the tcgen05 tensor cores (``vk_mlp_infer_tc``; ``vk_mlp_infer`` is the mma.sync variant).  Training on the GPU
by the project's own kernels: the forward and backward GEMMs of the 256-wide layers on the tcgen05 tensor cores
(``vk_tc_gemm``: BF16 operands, FP32 accumulation, K split over the batch for the weight gradients), the rest --
the 1-wide layer, weighted BCE, ReLU masks, bias sums, Adam -- by the kernels of ``mlp_train.cu``;
``train_gemm="simt"`` runs every GEMM on its FP32 SIMT kernel instead, in a fixed summation order (the pass the
oracle reproduces bit for bit).  Training target: the hit, itself or through its pair-closure partner, lands in the
top 5 of the exhaustive rescoring of its spectrum (K2 over every row of the precursor windows).
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np
import torch

from . import _lib as K
from . import engine as E
from .host import SearchParams, Spectra

N_IN = 16
HIDDEN = 256
FEATURES = ("k1_count", "summed_intensity", "precursor_ppm", "charge", "peptide_len", "missed_cleavages")
N_FEAT = len(FEATURES)
LABEL_TOP = 5
_PARAMS = ("W1", "b1", "W2", "b2", "w3", "b3")


def _n_sm(dev) -> int:
    return torch.cuda.get_device_properties(dev).multi_processor_count


class Pruner:
    """MLP weights (FP32 masters on the device, BF16 copies for the kernels), feature standardisation and the
    selection parameters (``tau``, ``min_keep``, ``max_keep``)."""

    def __init__(self, device="cuda", seed: int = 0, tau: float = -math.inf, min_keep: int = 1,
                 max_keep: int = 128, min_count: int = 1, tensor_cores: str = "tcgen05",
                 train_gemm: str = "tcgen05"):
        self.dev = torch.device(device)
        g = torch.Generator().manual_seed(seed)
        W1 = torch.zeros(HIDDEN, N_IN)
        W1[:, :N_FEAT] = torch.randn(HIDDEN, N_FEAT, generator=g) * math.sqrt(2.0 / N_FEAT)
        w = {"W1": W1, "b1": torch.zeros(HIDDEN),
             "W2": torch.randn(HIDDEN, HIDDEN, generator=g) * math.sqrt(2.0 / HIDDEN), "b2": torch.zeros(HIDDEN),
             "w3": torch.randn(HIDDEN, generator=g) * math.sqrt(1.0 / HIDDEN), "b3": torch.zeros(1)}
        self.w = {k: v.to(self.dev).contiguous() for k, v in w.items()}
        self.mu = torch.zeros(N_IN, device=self.dev)
        self.sd = torch.ones(N_IN, device=self.dev)
        self.tau, self.min_keep, self.max_keep = float(tau), int(min_keep), int(max_keep)
        self.min_count = int(min_count)     # shortlist only hits with K1 count >= min_count (calibrated)
        self.shortlist_k = 0                # shortlist the top shortlist_k hits by K1 count (calibrated; 0: top-k)
        if tensor_cores not in ("tcgen05", "mma.sync"):
            raise ValueError("tensor_cores must be 'tcgen05' or 'mma.sync'")
        self.tensor_cores = tensor_cores    # inference kernel: vk_mlp_infer_tc or vk_mlp_infer
        if train_gemm not in ("tcgen05", "simt"):
            raise ValueError("train_gemm must be 'tcgen05' or 'simt'")
        self.train_gemm = train_gemm        # training GEMMs: vk_tc_gemm or the FP32 SIMT vk_gemm
        self.step = 0
        self._adam = None
        self._sync_bf16()

    # ------------------------------------------------------------------ weights
    def _sync_bf16(self):
        L = K.lib()
        self.bf = {}
        for k in ("W1", "W2"):
            t = torch.empty(self.w[k].shape, dtype=torch.bfloat16, device=self.dev)
            K.check(L.vk_to_bf16(t.numel(), K.ptr(self.w[k]), K.ptr(t), K.stream()), "to_bf16")
            self.bf[k] = t
        self._b3 = float(self.w["b3"].item())

    def state_dict(self) -> dict:
        d = {k: v.detach().cpu().numpy() for k, v in self.w.items()}
        d.update(mu=self.mu.cpu().numpy(), sd=self.sd.cpu().numpy(),
                 sel=np.array([self.tau, self.min_keep, self.max_keep, self.min_count, self.shortlist_k],
                              np.float64))
        return d

    def load_state_dict(self, d: dict):
        for k in _PARAMS:
            self.w[k] = torch.from_numpy(np.asarray(d[k], np.float32)).to(self.dev).contiguous()
        self.mu = torch.from_numpy(np.asarray(d["mu"], np.float32)).to(self.dev)
        self.sd = torch.from_numpy(np.asarray(d["sd"], np.float32)).to(self.dev)
        sel = [float(x) for x in d["sel"]] + [1.0, 0.0]
        self.tau = sel[0]
        self.min_keep, self.max_keep, self.min_count = int(sel[1]), int(sel[2]), int(sel[3])
        self.shortlist_k = int(sel[4]) if len(d["sel"]) > 4 else 0
        self._adam = None
        self._sync_bf16()
        return self

    def save(self, path: str):
        np.savez(path, **self.state_dict())

    @classmethod
    def load(cls, path: str, device="cuda") -> "Pruner":
        return cls(device).load_state_dict(dict(np.load(path)))

    # ------------------------------------------------------------------ features and inference
    def features(self, gi: E.GpuIndex, dh, win_off, isum, cand, n_hits: int, n_dev=None, raw: bool = False):
        """Standardised BF16 features [n_hits, 16] of the compacted hits ``cand`` (raw values when ``raw``).  The
        intensity sums come from ``cand["c_isum"]`` (hit-list shortlist) when present, else from the dense K1 sums
        ``isum`` at ``win_off``."""
        mu = torch.zeros(N_IN, device=self.dev) if raw else self.mu
        sd = torch.ones(N_IN, device=self.dev) if raw else self.sd
        feat = torch.empty(max(n_hits, 1), N_IN, dtype=torch.bfloat16, device=self.dev)
        if cand.get("c_isum") is not None:
            win_off, isum = None, cand["c_isum"]
        K.check(K.lib().vk_cand_features(n_hits, K.ptr(n_dev) if n_dev is not None else None,
                                         K.ptr(cand["c_hyp"]), K.ptr(cand["c_row"]), K.ptr(cand["c_cnt"]),
                                         K.ptr(win_off), K.ptr(dh["lo"]), K.ptr(isum), K.ptr(dh["M"]),
                                         K.ptr(dh["z"]), K.ptr(gi.mass32), K.ptr(gi.length), K.ptr(gi.missed),
                                         K.ptr(mu), K.ptr(sd), K.ptr(feat), K.stream()), "cand_features")
        return feat

    def score(self, feat: torch.Tensor, hits, n: int, n_dev=None, status=None) -> torch.Tensor:
        """Selection score of every hit: the MLP logit."""
        return self.logits(feat, n, n_dev, status)

    def logits(self, feat: torch.Tensor, n: int, n_dev=None, status=None) -> torch.Tensor:
        """MLP logits of n feature rows.  With the tcgen05 kernel a wait timeout is ORed into ``status`` (device
        i32) when given, else checked here (one host sync)."""
        out = torch.empty(max(n, 1), dtype=torch.float32, device=self.dev)
        grid = max(1, min(_n_sm(self.dev), (n + 127) // 128))
        nd = K.ptr(n_dev) if n_dev is not None else None
        args = (K.ptr(feat), K.ptr(self.bf["W1"]), K.ptr(self.w["b1"]), K.ptr(self.bf["W2"]), K.ptr(self.w["b2"]),
                K.ptr(self.w["w3"]), self._b3, K.ptr(out), grid)
        if self.tensor_cores == "tcgen05":
            st = status if status is not None else torch.zeros(1, dtype=torch.int32, device=self.dev)
            K.check(K.lib().vk_mlp_infer_tc(n, nd, *args, K.ptr(st), K.stream()), "mlp_infer_tc")
            if status is None and n > 0 and int(st.item()):
                raise RuntimeError("mlp_infer_tc: a tensor-core MMA did not complete")
        else:
            K.check(K.lib().vk_mlp_infer(n, nd, *args, K.stream()), "mlp_infer")
        return out[:n]

    # ------------------------------------------------------------------ training (GPU kernels)
    def _buffers(self, B: int):
        if getattr(self, "_buf_B", 0) != B:
            f = lambda *s: torch.empty(*s, dtype=torch.float32, device=self.dev)  # noqa: E731
            self._buf = {"H1": f(B, HIDDEN), "H2": f(B, HIDDEN), "z": f(B), "dz": f(B), "dH2": f(B, HIDDEN),
                         "dH1": f(B, HIDDEN), "loss": f((B + 255) // 256)}
            L = K.lib()
            ws = max(L.vk_tc_gemm_ws_floats(m, n, k) for m, n, k in ((B, HIDDEN, N_IN), (B, HIDDEN, HIDDEN),
                                                                   (HIDDEN, HIDDEN, B), (HIDDEN, N_IN, B)))
            self._buf["ws"] = f(max(ws, 1))
            self._buf["ws_cs"] = f(max(L.vk_colsum_ws_floats(B, HIDDEN), 1))
            self._buf["status"] = torch.zeros(1, dtype=torch.int32, device=self.dev)
            self._grad = {k: torch.zeros_like(v) for k, v in self.w.items()}
            self._buf_B = B
        if self._adam is None:
            self._adam = {k: (torch.zeros_like(v), torch.zeros_like(v)) for k, v in self.w.items()}
        return self._buf, self._grad

    def _gemm(self, M, N, Kd, A, sam, sak, Bm, b_bf16, sbk, sbn, bias, relu, rnd, Cm, scm, scn, what):
        """C[M, N] = A[M, K] B[K, N] (+ bias) (ReLU) (BF16 rounding), A FP32 and B BF16 / FP32 given by strides:
        on the tensor cores (``vk_tc_gemm``) when N is a multiple of 16 and ``train_gemm`` is "tcgen05", else on
        the FP32 SIMT kernel (``vk_gemm``)."""
        L = K.lib()
        if self.train_gemm == "tcgen05" and N % 16 == 0:
            bf = self._buf
            K.check(L.vk_tc_gemm(M, N, Kd, K.ptr(A), sam, sak, K.ptr(Bm), b_bf16, sbk, sbn, K.ptr(bias), relu, rnd,
                                 K.ptr(Cm), scm, scn, K.ptr(bf["ws"]), bf["ws"].numel(), K.ptr(bf["status"]),
                                 K.stream()), what)
        else:
            K.check(L.vk_gemm(M, N, Kd, K.ptr(A), sam, sak, K.ptr(Bm), b_bf16, sbk, sbn, K.ptr(bias), relu, rnd,
                              K.ptr(Cm), scm, scn, K.stream()), what)

    def _colsum(self, n, o, D, v, out, what):
        """out[j] = sum_i D[i, j] (v[i] D[i, j] with a row weight v), in ``vk_colsum``'s fixed chunked order."""
        ws = self._buf["ws_cs"]
        K.check(K.lib().vk_colsum(n, o, K.ptr(D), K.ptr(v), K.ptr(ws), ws.numel(), K.ptr(out), K.stream()), what)

    def forward_train(self, X: torch.Tensor, B: int):
        """Training forward of B rows of FP32 features X [B, 16] (BF16 values): H1 (ReLU, rounded to BF16), H2
        (ReLU), logits z -- the arithmetic of the inference kernel (in a fixed summation order with
        ``train_gemm="simt"``)."""
        L = K.lib()
        bf, g = self._buffers(B)
        w, st = self.w, K.stream()
        self._gemm(B, HIDDEN, N_IN, X, N_IN, 1, self.bf["W1"], 1, 1, N_IN, w["b1"], 1, 1, bf["H1"], HIDDEN, 1,
                   "gemm_l1")
        self._gemm(B, HIDDEN, HIDDEN, bf["H1"], HIDDEN, 1, self.bf["W2"], 1, 1, HIDDEN, w["b2"], 1, 0, bf["H2"],
                   HIDDEN, 1, "gemm_l2")
        K.check(L.vk_gemm(B, 1, HIDDEN, K.ptr(bf["H2"]), HIDDEN, 1, K.ptr(w["w3"]), 0, 1, 0, K.ptr(w["b3"]), 0, 0,
                          K.ptr(bf["z"]), 1, 0, st), "gemm_l3")
        return bf["z"][:B]

    def backward(self, X: torch.Tensor, y: torch.Tensor, wt: torch.Tensor, B: int, inv_wsum: float):
        """Weighted BCE loss of the last forward and the gradients of every parameter (into ``self._grad``)."""
        L = K.lib()
        bf, g = self._buffers(B)
        w, st = self.w, K.stream()
        K.check(L.vk_bce(B, K.ptr(bf["z"]), K.ptr(y), K.ptr(wt), inv_wsum, K.ptr(bf["dz"]), K.ptr(bf["loss"]), st),
                "bce")
        # layer 3: gw3[j] = sum_b H2[b, j] dz[b]; gb3 = sum_b dz[b] (chunked column sums); dH2[b, j] = dz[b] w3[j]
        # (H2 > 0)
        self._colsum(B, HIDDEN, bf["H2"], bf["dz"], g["w3"], "colsum_w3")
        self._colsum(B, 1, bf["dz"], None, g["b3"], "colsum_b3")
        K.check(L.vk_gemm(B, HIDDEN, 1, K.ptr(bf["dz"]), 1, 0, K.ptr(w["w3"]), 0, 0, 1, None, 0, 0,
                          K.ptr(bf["dH2"]), HIDDEN, 1, st), "gemm_dh2")
        K.check(L.vk_relu_mask(B * HIDDEN, K.ptr(bf["H2"]), K.ptr(bf["dH2"]), st), "relu_mask2")
        # layer 2: gW2[o, i] = sum_b dH2[b, o] H1[b, i]; gb2; dH1[b, i] = sum_o dH2[b, o] W2[o, i] (H1 > 0)
        self._gemm(HIDDEN, HIDDEN, B, bf["dH2"], 1, HIDDEN, bf["H1"], 0, HIDDEN, 1, None, 0, 0, g["W2"], HIDDEN, 1,
                   "gemm_gw2")
        self._colsum(B, HIDDEN, bf["dH2"], None, g["b2"], "colsum_b2")
        self._gemm(B, HIDDEN, HIDDEN, bf["dH2"], HIDDEN, 1, self.bf["W2"], 1, HIDDEN, 1, None, 0, 0, bf["dH1"],
                   HIDDEN, 1, "gemm_dh1")
        K.check(L.vk_relu_mask(B * HIDDEN, K.ptr(bf["H1"]), K.ptr(bf["dH1"]), st), "relu_mask1")
        # layer 1: gW1[o, i] = sum_b dH1[b, o] X[b, i]; gb1
        self._gemm(HIDDEN, N_IN, B, bf["dH1"], 1, HIDDEN, X, 0, N_IN, 1, None, 0, 0, g["W1"], N_IN, 1, "gemm_gw1")
        self._colsum(B, HIDDEN, bf["dH1"], None, g["b1"], "colsum_b1")
        return bf["loss"][:(B + 255) // 256], g

    def adam_step(self, lr: float, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8, wd: float = 0.0):
        L = K.lib()
        self.step += 1
        for k in _PARAMS:
            m, v = self._adam[k]
            K.check(L.vk_adam(self.w[k].numel(), K.ptr(self.w[k]), K.ptr(self._grad[k]), K.ptr(m), K.ptr(v), lr,
                              b1, b2, eps, self.step, wd, K.ptr(self.bf[k]) if k in self.bf else None, K.stream()),
                    "adam")

    def set_standardisation(self, raw_feat: torch.Tensor):
        x = raw_feat[:, :N_FEAT].float()
        self.mu = torch.zeros(N_IN, device=self.dev)
        self.sd = torch.ones(N_IN, device=self.dev)
        self.mu[:N_FEAT] = x.mean(0)
        self.sd[:N_FEAT] = x.std(0).clamp(min=1e-3)

    def fit(self, feat: torch.Tensor, y: torch.Tensor, weight: torch.Tensor | None = None, epochs: int = 4,
            batch: int = 4096, lr: float = 2e-3, wd: float = 0.0, seed: int = 0, log=None) -> list[float]:
        """Train on standardised BF16 features ``feat`` [n, 16] with 0/1 targets ``y``.  Returns the mean loss
        of every epoch.  Mini-batches in a seeded order; the last partial batch is dropped."""
        L = K.lib()
        n = len(y)
        X = torch.empty(n, N_IN, dtype=torch.float32, device=self.dev)
        K.check(L.vk_bf16_to_f32(n * N_IN, K.ptr(feat), K.ptr(X), K.stream()), "bf16_to_f32")
        y = y.to(self.dev, torch.float32).contiguous()
        wt = (torch.ones(n, device=self.dev) if weight is None else weight.to(self.dev, torch.float32)).contiguous()
        g = torch.Generator(device=self.dev).manual_seed(seed)
        B = min(batch, n)
        losses = []
        n_batch = n // B
        for ep in range(epochs):
            t0 = time.perf_counter()
            perm = torch.randperm(n, generator=g, device=self.dev)
            tot = torch.zeros((), device=self.dev)
            # cosine learning-rate decay over all steps
            for i in range(n_batch):
                idx = perm[i * B:(i + 1) * B]
                Xb, yb, wb = X[idx].contiguous(), y[idx].contiguous(), wt[idx].contiguous()
                self.forward_train(Xb, B)
                loss, _ = self.backward(Xb, yb, wb, B, 1.0 / B)
                frac = (ep * n_batch + i) / max(1, epochs * n_batch)
                self.adam_step(lr * 0.5 * (1.0 + math.cos(math.pi * frac)), wd=wd)
                tot += loss.sum()
            losses.append(float(tot) / max(n_batch, 1))
            E.check_status(self._buf["status"], "training GEMM")
            if log:
                log(f"epoch {ep}: loss {losses[-1]:.5f} ({time.perf_counter() - t0:.1f} s)")
        self._b3 = float(self.w["b3"].item())
        return losses


class CountRanker(Pruner):
    """The method without the network: hits ranked by K1 count alone, with the same calibrated threshold and
    selection (the baseline the learned pruner is compared against)."""

    def score(self, feat, hits, n: int, n_dev=None, status=None) -> torch.Tensor:
        return hits["c_cnt"][:n].to(torch.float32)


# ---------------------------------------------------------------------------------------------- search
def _front(run: E.DeviceRun, gi: E.GpuIndex, p: SearchParams, st: E.Stats, timers: bool, min_count: int = 1,
           dense: bool = False, pr: "Pruner | None" = None):
    """K0, hypotheses, K1 with intensity sums, and the top-k shortlist (hits with count >= min_count) without pair
    closure.  K1 writes hit lists (``vk_k1_hits``: only the rows with count >= the floor) and the shortlist reads
    them; ``dense``: K1's dense per-row counts and sums and the shortlist over those instead (same shortlist; the
    dense arrays are returned as "cnt" / "isum").  With a pruner ``pr`` (hit lists) the shortlist holds the top
    ``pr.shortlist_k`` hits by count (when set) and its compaction also writes their standardised features, as
    ``hits["feat"]``."""
    dev = gi.dev
    n = run.n
    thr = max(p.k1_threshold, min_count)

    def phase(name):
        return E.Timer(st, name) if timers else E._NoTimer()
    with phase("k0"):
        peaks = E._k0_device(run, p, dev)
    keys = E.early_peak_keys(gi, peaks, p)
    with phase("hyp"):
        dh = E._hyp_device(run, peaks, gi, p)
    if dense:
        with phase("k1"):
            win_off, cnt, status, isum = E._k1_dense(gi, dh, peaks, p, dh["n_max"], st, isum=True, keys=keys)
        with phase("topk"):
            hits, sums = E._shortlist(gi, p, n, dh, win_off, cnt, p.topk, False, thr)
        return {"peaks": peaks, "dh": dh, "win_off": win_off, "cnt": cnt, "status": status, "isum": isum,
                "hits": hits, **sums}
    with phase("k1"):
        k1h = E._k1_hits(gi, dh, peaks, p, dh["n_max"], thr, isum=True, keys=keys)
    k = p.topk if pr is None or pr.shortlist_k <= 0 else min(p.topk, pr.shortlist_k)
    with phase("topk"):
        hits, sums = E._shortlist_hits(gi, p, n, dh, k1h, k, features=(gi, pr.mu, pr.sd) if pr is not None else None)
    return {"peaks": peaks, "dh": dh, "win_off": k1h["win_off"], "status": k1h["status"], "k1_hits": k1h,
            "hits": hits, **sums}


def _pruned_device(run: E.DeviceRun, gi: E.GpuIndex, p: SearchParams, pr: Pruner, report: int, st: E.Stats,
                   timers: bool = False):
    """The pruned search of one resident run: front end, MLP over the shortlist, pruned selection with pair
    closure, K2, ranking."""
    L = K.lib()
    dev = gi.dev
    n = run.n
    f = _front(run, gi, p, st, timers, pr.min_count, pr=pr)
    hits = f["hits"]
    n_bound = n * hits["cap"]
    n_dev = hits["cand_off"][n:]

    def phase(name):
        return E.Timer(st, name) if timers else E._NoTimer()
    with phase("prune"):
        feat = hits["feat"] if "feat" in hits else pr.features(gi, f["dh"], f["win_off"], f.get("isum"), hits,
                                                                 n_bound, n_dev=n_dev)
        logit = pr.score(feat, hits, n_bound, n_dev=n_dev, status=f["status"])
        cap = (2 if p.pair_closure else 1) * pr.max_keep
        s_hyp = torch.empty(max(n * cap, 1), dtype=torch.int64, device=dev)
        s_row = torch.empty_like(s_hyp)
        s_cnt = torch.empty_like(s_hyp)
        n_cand = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
        K.check(L.vk_select_pruned(n, K.ptr(f["dh"]["spec_off"]), K.ptr(hits["cand_off"]), K.ptr(hits["c_hyp"]),
                                   K.ptr(hits["c_row32"]), K.ptr(hits["c_cnt"]), K.ptr(logit), pr.tau, pr.min_keep,
                                   pr.max_keep, int(p.pair_closure), K.ptr(gi.partner), cap, p.topk, K.ptr(s_hyp),
                                   K.ptr(s_row), K.ptr(s_cnt), K.ptr(n_cand), K.stream()), "select_pruned")
        cand = E._compact(n, cap, n_cand, s_hyp, s_row, s_cnt, f["dh"], dev)
    with phase("k2"):
        k2 = E._k2_cands(gi, p, n, cand, f["peaks"], sparse=True)
    with phase("rank"):
        psm = E._rank_device(n, cand["cand_off"], cand["c_row"], k2, p, report, dev, sparse=True)
    return {**f, **cand, "logit": logit, "feat": feat, "k2": k2, "psm": psm}


def search_pruned(sp: Spectra, gi: E.GpuIndex, l1, p: SearchParams, pruner: Pruner | None,
                  report: int | None = None, timers: bool = False):
    """Pruned closed search of one run; same outputs as ``engine.search`` (PSM table, stats, debug).  Without a
    pruner (or with tau = -inf and max_keep >= topk) it is the plain path."""
    if pruner is None:
        return E.search(sp, gi, l1, p, report=report, timers=timers)
    import resource
    report = p.report_psms if report is None else report
    if pruner.max_keep < 16 or pruner.max_keep & (pruner.max_keep - 1):
        raise ValueError("max_keep must be a power of two >= 16")
    st = E.Stats()
    ru0 = resource.getrusage(resource.RUSAGE_SELF)
    t0 = time.perf_counter()
    with torch.cuda.device(gi.dev):
        run = E.DeviceRun(sp, gi.dev, st)
        out = _pruned_device(run, gi, p, pruner, report, st, timers)
        E.check_status(out["status"])
        tbl = E._read_packed(*E._pack_psms(gi, out, report, run.n), sp, st)
    ru1 = resource.getrusage(resource.RUSAGE_SELF)
    st.wall_s["total"] = time.perf_counter() - t0
    st.counts.update(n_spectra=len(sp), n_searched=int(out["peaks"]["valid_d"].sum()),
                     n_hypotheses=int(out["dh"]["spec_off"][-1]), n_hits=int(out["hits"]["cand_off"][-1]),
                     n_rescored=int(out["cand_off"][-1]), n_psms=tbl.num_rows)
    st.counts["cpu_core_s"] = (ru1.ru_utime - ru0.ru_utime) + (ru1.ru_stime - ru0.ru_stime)
    return tbl, st, out


# ---------------------------------------------------------------------------------------------- training data
def exhaustive_top(gi: E.GpuIndex, p: SearchParams, peaks, dh, win_off, n: int, top: int = LABEL_TOP):
    """Exact rescoring of every window row of every hypothesis (K2 over the whole precursor windows, no K1
    shortlist) and the ``top`` best rows of each spectrum by the label-blind PSM ranking: [n, top], -1 = none."""
    dev = gi.dev
    n_h = dh["n_max"]
    win_len = (dh["hi"][:n_h] - dh["lo"][:n_h]).clamp(min=0)
    n_win = int(win_off[-1])
    hh = torch.repeat_interleave(torch.arange(n_h, device=dev), win_len)
    rows = dh["lo"][hh] + (torch.arange(n_win, device=dev) - win_off[:-1][hh])
    cand = {"cand_off": win_off[dh["spec_off"].long()].contiguous(), "c_row32": rows.to(torch.int32).contiguous(),
            "c_maxfz": dh["maxfz"][hh].contiguous(), "cap": 0}
    k2 = E._k2_outputs(max(n_win, 1), dev)
    K.check(K.lib().vk_k2_spectra(C.byref(gi.fp), n, K.ptr(cand["cand_off"]), K.ptr(cand["c_row32"]),
                                  K.ptr(cand["c_maxfz"]), K.ptr(peaks["off"]), K.ptr(peaks["mass"]),
                                  K.ptr(peaks["int"]), *gi.table_ptrs(), float(p.fragment_ppm[0]),
                                  float(p.fragment_ppm[1]), None, *E._k2_ptrs(k2), K.stream()), "k2_spectra")
    psm_cand = E._rank_device(n, cand["cand_off"], rows.contiguous(), k2, p, top, dev)[0]
    out = torch.where(psm_cand >= 0, rows[psm_cand.clamp(min=0)], torch.full_like(psm_cand, -1))
    return out.view(n, top)


def hit_labels(gi: E.GpuIndex, hits, top_rows: torch.Tensor, n: int) -> torch.Tensor:
    """1 where the hit's row or its partner is among its spectrum's ``top_rows``."""
    n_hits = int(hits["cand_off"][-1])
    dev = gi.dev
    cnt = hits["cand_off"][1:] - hits["cand_off"][:-1]
    spec = torch.repeat_interleave(torch.arange(n, device=dev), cnt)
    r = hits["c_row"][:n_hits]
    t = top_rows[spec]                                       # [n_hits, top]
    hit = (t == r[:, None]) | (t == gi.partner[r][:, None])
    return (hit & (t >= 0)).any(1)


def collect(sp: Spectra, gi: E.GpuIndex, p: SearchParams, pr: Pruner, raw: bool = False, labels: bool = True):
    """Training / calibration data of one run: the shortlist hits (spectrum, row, count), their standardised
    features (with the pruner's current standardisation; also the raw ones when ``raw``), their labels from the
    exhaustive rescoring (when ``labels``) and the plain path's top-1 row of every spectrum."""
    st = E.Stats()
    with torch.cuda.device(gi.dev):
        run = E.DeviceRun(sp, gi.dev, st)
        f = _front(run, gi, p, st, False)
        n = run.n
        hits = f["hits"]
        n_hits = int(hits["cand_off"][-1])
        d = {"n": n, "hits": {k: (v[:n_hits].clone() if k.startswith("c_") else v) for k, v in hits.items()}}
        d["feat"] = pr.features(gi, f["dh"], f["win_off"], f.get("isum"), hits, n_hits)[:n_hits]
        if raw:
            d["raw"] = pr.features(gi, f["dh"], f["win_off"], f.get("isum"), hits, n_hits, raw=True)[:n_hits]
        if labels:
            top = exhaustive_top(gi, p, f["peaks"], f["dh"], f["win_off"], n)
            d["y"] = hit_labels(gi, hits, top, n)
        plain = E._search_device(run, gi, p, 1, st)
        pc = plain["psm"][0]
        d["top1"] = torch.where(pc >= 0, plain["c_row"][pc.clamp(min=0)], torch.full_like(pc, -1))
        d["spec"] = torch.repeat_interleave(torch.arange(n, device=gi.dev), hits["cand_off"][1:] -
                                            hits["cand_off"][:-1])
        d["row"] = d["hits"]["c_row"]
        d["cnt"] = d["hits"]["c_cnt"]
        d["n_rescored_plain"] = int(plain["cand_off"][-1])
        return d


SHORTLIST_KS = (8, 10, 12, 16, 20, 24, 32, 48, 64)


def _count_rank(d) -> torch.Tensor:
    """Rank of every shortlist hit inside its spectrum in the shortlist's own order: count descending, then row
    descending, then hypothesis ascending (``vk_select_hits``' keys)."""
    spec, cnt, row, hyp = d["spec"], d["cnt"], d["row"], d["hits"]["c_hyp"]
    idx = torch.arange(len(spec), device=spec.device)
    o = torch.argsort(hyp, stable=True)
    o = o[torch.argsort(row[o], descending=True, stable=True)]
    o = o[torch.argsort(cnt[o], descending=True, stable=True)]
    o = o[torch.argsort(spec[o], stable=True)]
    ss = spec[o]
    first = torch.searchsorted(ss, ss, side="left")
    rank = torch.empty_like(idx)
    rank[o] = idx - first
    return rank


def calibrate(pr: Pruner, gi: E.GpuIndex, data: list[dict], target: float = 0.9995, count_share: float = 0.25,
              max_count: int = 16, cap_share: float = 0.25) -> float:
    """Selection parameters from calibration runs (``collect`` data): the spectra with a plain-path top-1 PSM
    must keep a hit that brings that row (the row itself or its pair-closure partner) for at least ``target`` of
    them.  First ``min_count``: the largest shortlist count floor that loses at most ``count_share`` of the
    allowed misses; then ``shortlist_k``: the smallest cap on the shortlist (its top hits by count) that loses at
    most ``cap_share`` more; then ``tau``: the largest threshold that loses no more than the rest, given
    ``min_keep`` and ``max_keep``.  Sets them on the pruner and returns tau."""
    dev = gi.dev
    per = []
    n_top = 0
    for d in data:
        z = pr.score(d["feat"], d["hits"], len(d["row"]))
        t = d["top1"][d["spec"]]
        good = ((d["row"] == t) | (gi.partner[d["row"]] == t)) & (t >= 0)
        bc = torch.full((d["n"],), -1, dtype=torch.int64, device=dev).scatter_reduce(
            0, d["spec"][good], d["cnt"][good], reduce="amax")
        has = d["top1"] >= 0
        n_top += int(has.sum())
        per.append((d, z, good, bc, has))
    allowed = int(math.floor((1.0 - target) * n_top))
    c0 = 1
    for c in range(max_count, 1, -1):
        lost = sum(int((has & (bc < c)).sum()) for _, _, _, bc, has in per)
        if lost <= int(math.floor(count_share * allowed)):
            c0 = c
            break
    lost_c0 = sum(int((has & (bc < c0)).sum()) for _, _, _, bc, has in per)
    # the best count rank of a hit bringing the top-1 row (count >= c0): a cap k loses the spectra where it is >= k
    crank, br = [], []
    for d, z, good, bc, has in per:
        cr = _count_rank(d)
        g = good & (d["cnt"] >= c0)
        crank.append(cr)
        br.append(torch.full((d["n"],), 1 << 30, dtype=torch.int64, device=dev).scatter_reduce(
            0, d["spec"][g], cr[g], reduce="amin"))
    k_cap = 0
    for k in SHORTLIST_KS:
        lost = sum(int((has & (bc >= c0) & (b >= k)).sum()) for (_, _, _, bc, has), b in zip(per, br))
        if lost <= int(math.floor(cap_share * allowed)):
            k_cap = k
            break
    lost_k = lost_c0 + (sum(int((has & (bc >= c0) & (b >= k_cap)).sum()) for (_, _, _, bc, has), b in zip(per, br))
                        if k_cap else 0)
    need = []
    for (d, z, good, bc, has), cr, b in zip(per, crank, br):
        f = (d["cnt"] >= c0) & ((cr < k_cap) if k_cap else True)
        zf, sf, gf = z[f], d["spec"][f], good[f]
        rank = _rank_in_spectrum(zf, d["cnt"][f], sf, d["n"])
        ok = gf & (rank < pr.max_keep)
        best = torch.full((d["n"],), -math.inf, device=dev).scatter_reduce(0, sf[ok], zf[ok], reduce="amax")
        brank = torch.full((d["n"],), 1 << 30, dtype=torch.int64, device=dev).scatter_reduce(
            0, sf[ok], rank[ok], reduce="amin")
        alive = has & (bc >= c0) & ((b < k_cap) if k_cap else True)
        need.append(best[alive & (brank >= pr.min_keep)])
    v = torch.sort(torch.cat(need)).values
    rest = allowed - lost_k
    pr.min_count = c0
    pr.shortlist_k = k_cap
    pr.tau = float(v[rest]) if rest < len(v) else math.inf
    return pr.tau


def _rank_in_spectrum(z, cnt, spec, n):
    """Rank of every hit inside its spectrum by (logit, count, hit order) descending, the selection's order."""
    idx = torch.arange(len(z), device=z.device)
    o = torch.argsort(idx, descending=True)
    o = o[torch.argsort(cnt[o], descending=True, stable=True)]
    o = o[torch.argsort(z[o], descending=True, stable=True)]
    o = o[torch.argsort(spec[o], stable=True)]
    ss = spec[o]
    first = torch.searchsorted(ss, ss, side="left")
    rank = torch.empty_like(idx)
    rank[o] = idx - first
    return rank


# ---------------------------------------------------------------------------------------------- judging
def accepted_psms(tbl, labels, alpha: float = 0.01, seed: int = 11) -> int:
    """Target PSMs accepted at q <= alpha by the paired double competition of the top-1 PSMs (reference
    ``vulcan/rescore/post.py:57-64``: unit = pf_id, pair = tdc_pair, tie-break = hash(pf_id, 11))."""
    from ..stats._util import hash_tiebreak
    from ..stats.tdc import double_competition
    t = tbl.filter(tbl.column("rank").to_numpy() == 1) if tbl.num_rows else tbl
    rows = t.column("pf_row").to_numpy()
    pf = t.column("pf_id").to_numpy()
    dec = np.asarray(labels.column("is_decoy").to_numpy(zero_copy_only=False), bool)[rows]
    pair = labels.column("tdc_pair").to_numpy()[rows]
    r = double_competition(t.column("spec_idx").to_numpy(), pf, pair, t.column("hyperscore").to_numpy(), dec,
                           seed=seed, tiebreak=hash_tiebreak(pf, seed))
    return int(np.count_nonzero((r.q <= alpha) & ~r.is_decoy))


def top1_recall(tbl_plain, tbl_pruned) -> float:
    """Fraction of the plain path's top-1 PSMs (spectrum, row) that the pruned path reports as top-1."""
    def top1(t):
        r = t.column("rank").to_numpy() == 1
        return dict(zip(t.column("spec_idx").to_numpy()[r].tolist(), t.column("pf_row").to_numpy()[r].tolist()))
    a, b = top1(tbl_plain), top1(tbl_pruned)
    if not a:
        return 1.0
    return sum(1 for s, r in a.items() if b.get(s) == r) / len(a)


def evaluate(sp: Spectra, gi: E.GpuIndex, l1, labels, p: SearchParams, pr: Pruner) -> dict:
    """Pruned vs plain on one run: top-1 recall, candidates rescored, PSMs accepted at 1% q."""
    t_plain, s_plain, _ = E.search(sp, gi, l1, p)
    t_pr, s_pr, _ = search_pruned(sp, gi, l1, p, pr)
    a_plain, a_pr = accepted_psms(t_plain, labels), accepted_psms(t_pr, labels)
    return {"recall": top1_recall(t_plain, t_pr), "rescored_plain": s_plain.counts["n_rescored"],
            "rescored_pruned": s_pr.counts["n_rescored"], "hits": s_pr.counts["n_hits"],
            "accepted_plain": a_plain, "accepted_pruned": a_pr,
            "delta_accepted": (a_pr - a_plain) / max(a_plain, 1)}


def train(gi: E.GpuIndex, p: SearchParams, train_runs: list[Spectra], calib_runs: list[Spectra],
          seed: int = 0, epochs: int = 4, batch: int = 4096, lr: float = 2e-3, target: float = 0.9995,
          min_keep: int = 1, max_keep: int = 128, log=None) -> tuple[Pruner, dict]:
    """Train a pruner on the GPU from the exhaustive rescoring of ``train_runs`` and calibrate its threshold on
    ``calib_runs``.  The feature standardisation comes from the first training run.  Returns (pruner, info)."""
    pr = Pruner(gi.dev, seed=seed, min_keep=min_keep, max_keep=max_keep)
    t0 = time.perf_counter()
    d0 = collect(train_runs[0], gi, p, pr, raw=True, labels=False)
    pr.set_standardisation(d0["raw"])
    del d0
    data = [collect(sp, gi, p, pr) for sp in train_runs]
    X = torch.cat([d["feat"] for d in data])
    y = torch.cat([d["y"] for d in data])
    del data
    t_collect = time.perf_counter() - t0
    t1 = time.perf_counter()
    losses = pr.fit(X, y, epochs=epochs, batch=batch, lr=lr, seed=seed, log=log)
    torch.cuda.synchronize(gi.dev)
    t_fit = time.perf_counter() - t1
    cal = [collect(sp, gi, p, pr, labels=False) for sp in calib_runs]
    tau = calibrate(pr, gi, cal, target)
    info = {"train_hits": int(len(y)), "positives": int(y.sum()), "losses": losses, "tau": tau,
            "collect_s": round(t_collect, 2), "fit_s": round(t_fit, 2), "epochs": epochs, "batch": batch,
            "train_spectra": int(sum(len(s) for s in train_runs)),
            "calib_spectra": int(sum(len(s) for s in calib_runs))}
    return pr, info


def count_ranker(gi: E.GpuIndex, p: SearchParams, calib_runs: list[Spectra], target: float = 0.9995,
                 min_keep: int = 1, max_keep: int = 128) -> CountRanker:
    """The count-only baseline, calibrated like the learned pruner."""
    cr = CountRanker(gi.dev, min_keep=min_keep, max_keep=max_keep)
    cal = [collect(sp, gi, p, cr, labels=False) for sp in calib_runs]
    calibrate(cr, gi, cal, target)
    return cr
