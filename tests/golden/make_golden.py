"""Generate the golden fixtures of the test suite (run in a checkout that has the reference next to it).

    python tests/golden/make_golden.py --reference /path/to/vulcan-proteomics

Writes
  mini_fixture.npz    a small index (rows of the L1 table) and MS2 runs (Spectra fields), with edge cases: an
                      empty spectrum, a NaN precursor, too few peaks, more peaks than max_peaks, out-of-range and
                      NaN peaks, duplicate peaks, unknown charges, and peaks placed so that an index fragment lies
                      exactly on a tolerance bound (Da and ppm).
  golden_ref_py.npz   outputs of the reference's own Python code on that fixture, for each parameter set:
                      vulcan/gpu/engine.py k0_preprocess (CPU tensors), host.make_hypotheses, work_items,
                      window_candidates, select_topk, psm_table; vulcan/index/decoys.py; engine.lnfact.
                      select_topk / psm_table consume K1 / K2 values of the CPU oracle, which the kernel goldens
                      (make_golden_ref.py, the reference's CUDA kernels) pin separately.

The fixture's index is built by this repository's index builder; the inputs are stored, so the goldens do not
depend on the builder staying unchanged.
"""
from __future__ import annotations

import argparse
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, os.path.join(ROOT, "vulcan-proteomics_b200"))
sys.path.insert(0, ROOT)

STATIC = {"C": 57.021464}
VAR = {"M": 15.9949}
PARAM_SETS = {
    # name: SearchParams overrides (reference field names)
    "da": dict(precursor_ppm=(-10.0, 10.0), fragment_ppm=(-0.02, 0.02), fragment_unit="da", topk=8, max_peaks=150,
               min_peaks=15),
    "ppm": dict(precursor_ppm=(-10.0, 10.0), fragment_ppm=(-20.0, 20.0), fragment_unit="ppm", topk=5,
                max_peaks=100, min_peaks=10),
    "ppm_mfz": dict(precursor_ppm=(-20.0, 20.0), fragment_ppm=(-20.0, 20.0), fragment_unit="ppm", topk=6,
                    max_peaks=150, min_peaks=10, max_fragment_charge=None, isotope_errors=(-1, 2)),
}


def _f32(x):
    return np.float32(x)


def _edge_peak(frag: np.float32, tol: np.float32, da: bool, lower: bool):
    """A peak mass m (f32) whose tolerance window has `frag` exactly on its lower (or upper) bound, and an m/z
    that maps back to m exactly (m = f32(mz - PROTON)); None if none is found nearby."""
    proton = _f32(1.0072764)

    def bound(m):
        if da:
            return _f32(m + tol)
        return _f32(m + _f32(_f32(m * tol) / _f32(1e6)))
    guess = _f32(frag - tol) if da else _f32(frag / _f32(1.0 + float(tol) * 1e-6))
    m = guess
    for _ in range(4000):
        if bound(m) == frag:
            break
        m = np.nextafter(m, _f32(np.inf) if bound(m) < frag else _f32(-np.inf), dtype=np.float32)
    else:
        return None
    if bound(m) != frag:
        return None
    mz = _f32(m + proton)
    for _ in range(64):
        if _f32(mz - proton) == m:
            return mz
        mz = np.nextafter(mz, _f32(np.inf) if _f32(mz - proton) < m else _f32(-np.inf), dtype=np.float32)
    return None


def build_fixture(tmp: str, seed: int = 5):
    from vulcan import synth
    from vulcan.index.build import L1Index, read_labels
    w = synth.Workload("mini", 150, 1, 7, 30, dict(VAR), 1, 160, (2, 4), 0.7, 60, 0.0, 0.0, (0, 0), 8, 150,
                       4242, seed)
    d = synth.build_index(w, tmp)
    l1 = L1Index(d)
    sp, rows = synth.simulate_run(l1, read_labels(d), w, n_spectra=160, seed=seed)
    rng = np.random.default_rng(seed)
    mz = [sp.mz[sp.offsets[i]:sp.offsets[i + 1]].copy() for i in range(len(sp))]
    it = [sp.intensity[sp.offsets[i]:sp.offsets[i + 1]].copy() for i in range(len(sp))]
    pmz = sp.precursor_mz.copy()
    ch = sp.charge.copy()
    ch[rng.random(len(ch)) < 0.2] = 0                      # unknown charges
    mz[3] = mz[3][:0]; it[3] = it[3][:0]                   # empty spectrum
    pmz[5] = np.nan                                        # NaN precursor
    mz[7] = mz[7][:8]; it[7] = it[7][:8]                   # fewer than min_peaks
    extra = rng.uniform(150, 2000, 320).astype(np.float32)  # more peaks than max_peaks
    mz[9] = np.sort(np.concatenate([mz[9], extra])); it[9] = rng.lognormal(7, 1, len(mz[9])).astype(np.float32)
    mz[11] = np.concatenate([mz[11], np.array([50.0, 2500.0, np.nan, 149.9, 2000.0, 150.0], np.float32)])
    it[11] = np.concatenate([it[11], np.array([5e4, 5e4, 5e4, 10, 10, 10], np.float32)])
    mz[13] = np.concatenate([mz[13], mz[13][:5], mz[13][5:8]])                # duplicate m/z
    it[13] = np.concatenate([it[13], it[13][:5], it[13][5:8] * 2])
    mz[15] = np.concatenate([mz[15], np.full(4, mz[15][10], np.float32)])      # identical peaks
    it[15] = np.concatenate([it[15], np.full(4, it[15][10], np.float32)])
    # exact tolerance-edge peaks: an index fragment of the true row on the lower / upper bound
    from oracle import oracle as O
    P = O.make_params(STATIC, VAR, "da")
    edge_specs = list(range(20, 40))
    for k, i in enumerate(edge_specs):
        r = int(rows[i])
        seq = l1.residues[l1.seq_off[r]:l1.seq_off[r] + l1.length[r]]
        frs = []
        b, y = _f32(0.0), _f32(l1.mass32[r])
        for j, c in enumerate(seq[:-1]):
            rm = _f32(_f32(P.mono[c - 65]) + _f32(P.var[c - 65] if (int(l1.mask[r]) >> j) & 1 else P.stat[c - 65]))
            b = _f32(b + rm)
            y = _f32(y - rm)
            frs += [b, y]
        frs = [f for f in frs if 200 < f < 1900]
        if not frs:
            continue
        add = []
        for f in frs[:3]:
            for da, tol in ((True, _f32(-0.02)), (True, _f32(0.02)), (False, _f32(-20.0)), (False, _f32(20.0))):
                e = _edge_peak(f, tol, da, tol < 0)
                if e is not None:
                    add.append(e)
        if add:
            mz[i] = np.concatenate([mz[i], np.array(add, np.float32)])
            it[i] = np.concatenate([it[i], rng.lognormal(8, 0.5, len(add)).astype(np.float32)])
    off = np.zeros(len(mz) + 1, np.int64)
    off[1:] = np.cumsum([len(x) for x in mz])
    fx = {"idx_" + k: getattr(l1, k) for k in ("pf_id", "mass32", "seq_off", "length", "mask", "n_var", "missed",
                                                 "partner", "residues")}
    fx.update(sp_scan=sp.scan, sp_index=sp.index, sp_rt=sp.rt, sp_precursor_mz=pmz, sp_charge=ch.astype(np.int8),
              sp_mz=np.concatenate(mz).astype(np.float32), sp_intensity=np.concatenate(it).astype(np.float32),
              sp_offsets=off, truth_rows=np.asarray(rows, np.int64))
    return fx


class _L1:
    def __init__(self, fx):
        for k in fx:
            if k.startswith("idx_"):
                setattr(self, k[4:], fx[k])

    def __len__(self):
        return len(self.pf_id)


def reference_python_goldens(fx, ref_root: str):
    # this repository's package is also named `vulcan`: drop it before importing the reference's
    for k in [k for k in sys.modules if k == "vulcan" or k.startswith("vulcan.")]:
        del sys.modules[k]
    sys.path[:] = [q for q in sys.path if "vulcan-proteomics_b200" not in q]
    sys.path.insert(0, ref_root)
    import torch
    from vulcan.gpu import engine as RE      # the reference (ref_root is first on sys.path)
    from vulcan.gpu import host as RH
    from vulcan.index import decoys as RD
    assert os.path.abspath(RE.__file__).startswith(os.path.abspath(ref_root)), RE.__file__
    from oracle import oracle as O
    l1 = _L1(fx)
    out = {}
    sp = RH.Spectra("mini", fx["sp_scan"], fx["sp_index"], fx["sp_rt"], fx["sp_precursor_mz"], fx["sp_charge"],
                    fx["sp_mz"], fx["sp_intensity"], fx["sp_offsets"])
    cpu = torch.device("cpu")
    for name, kw in PARAM_SETS.items():
        p = RH.SearchParams(**kw)
        st = RE.Stats()
        pk = RE.k0_preprocess(sp, p, cpu, st)
        for k in ("off", "mass", "int", "tic"):
            out[f"{name}/k0_{k}"] = pk[k].numpy()
        out[f"{name}/k0_valid"] = pk["valid"]
        hyp = RH.make_hypotheses(sp, pk["valid"], l1.mass32, p)
        for k, v in hyp.items():
            out[f"{name}/hyp_{k}"] = v
        wi = RE.work_items(hyp, p)
        for k in ("hyp", "chunk", "lo", "hi"):
            out[f"{name}/wi_{k}"] = wi[k]
        h, r = RE.window_candidates(hyp, cpu)
        out[f"{name}/win_h"], out[f"{name}/win_r"] = h.numpy(), r.numpy()
        # K1 values of the oracle feed the reference's top-K / PSM table
        P = O.make_params(STATIC, VAR, p.fragment_unit)
        peaks = {k: pk[k].numpy() for k in ("off", "mass", "int")}
        win_off, cnt, sc, mt = O.k1_windows(l1, hyp, peaks, p, P)
        oh, orr, oc = O.k1_appended(hyp, win_off, cnt, p.k1_threshold)
        gi = types.SimpleNamespace(partner=torch.from_numpy(l1.partner.astype(np.int64)), dev=cpu)
        d_spec = torch.from_numpy(hyp["spec"])
        th, tr, tc = RE.select_topk(torch.from_numpy(oh.astype(np.int32)), torch.from_numpy(orr.astype(np.int32)),
                                    torch.from_numpy(oc.astype(np.int32)), d_spec, gi, p)
        out[f"{name}/topk_h"], out[f"{name}/topk_r"], out[f"{name}/topk_c"] = th.numpy(), tr.numpy(), tc.numpy()
        k2 = O.k2(l1, hyp, peaks, th.numpy(), tr.numpy(), p, P)
        k2t = {k: torch.from_numpy(v) for k, v in k2.items()}
        tbl = RE.psm_table(sp, gi, l1, hyp, th, tr, tc, k2t, torch.from_numpy(sc.astype(np.int32)),
                           torch.from_numpy(mt.astype(np.int64)), {"tic": pk["tic"]}, p, report=3)
        for c in tbl.column_names:
            if c == "run":
                continue
            out[f"{name}/psm_{c}"] = tbl.column(c).to_numpy()
    peps = ["PEPTIDEK", "LLLLLLLK", "AGCDEFGHLKR", "MSLVHLPHALMR", "VSLMWRGRNFR", "AAAAAAAR", "QWERTYLPASDFK",
            "KEDITPEPK", "EDITPEPK", "GGGGGGK", "ADAK"]
    out["decoy_pseudo_reverse"] = np.array([RD.pseudo_reverse(q) for q in peps])
    out["decoy_peps"] = np.array(peps)
    perms = [RD.hash_shuffle_perm(q, s, a) for q in peps for s in (1001, 2001) for a in range(3)]
    out["decoy_perms"] = np.array([",".join(map(str, x)) for x in perms])
    dec, n_sh = RD.make_decoys(peps)
    out["decoy_make_keys"] = np.array(sorted(dec))
    out["decoy_make_vals"] = np.array([dec[k][0] for k in sorted(dec)])
    out["decoy_make_nshuffled"] = np.array([n_sh])
    ent, nr, nd = RD.make_entrapment(sorted(peps), 2001, set(peps))
    out["entrap_keys"] = np.array(sorted(ent))
    out["entrap_vals"] = np.array([ent[k][0] for k in sorted(ent)])
    out["lnfact_n"] = np.arange(0, 120)
    out["lnfact_v"] = RE.lnfact(np.arange(0, 120))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True)
    a = ap.parse_args()
    with tempfile.TemporaryDirectory() as tmp:
        fx = build_fixture(tmp)
    np.savez_compressed(os.path.join(HERE, "mini_fixture.npz"), **fx)
    fx = dict(np.load(os.path.join(HERE, "mini_fixture.npz")))
    g = reference_python_goldens(fx, os.path.abspath(a.reference))
    np.savez_compressed(os.path.join(HERE, "golden_ref_py.npz"), **g)
    print("fixture rows", len(fx["idx_pf_id"]), "spectra", len(fx["sp_offsets"]) - 1, "golden keys", len(g))


if __name__ == "__main__":
    main()
