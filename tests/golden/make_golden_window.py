"""Generate golden_window.npz: the reference's own K0 peak view in the window peak mode (run in a checkout that has
the reference next to it).

    python tests/golden/make_golden_window.py --reference /path/to/vulcan-proteomics

Inputs: the spectra of mini_fixture.npz followed by seeded spectra aimed at the window mode -- in-order spectra
with over-full windows, a window of more than 128 peaks, shuffled input, a NaN m/z, every peak twice, peaks on and
next to window boundaries, peaks on and outside the fragment range, an empty spectrum, equal intensities, and
equal m/z with intensities in the wrong order.  Outputs: vulcan/gpu/engine.py k0_preprocess (CPU tensors) for
each parameter set of WINDOW_SETS.  The reference runs the division m/z / window_th on the CPU here; the script
checks that it agrees with the device's evaluation (m/z times the f32 reciprocal) on every peak of the inputs, so
the goldens hold for both.  (With window_th 7 the two differ just below multiples of 7; a GPU test pins that case
against the CUDA division itself.)
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))

WINDOW_SETS = {
    # name: SearchParams overrides (reference field names)
    "win100": dict(peak_mode="window", window_th=100.0, window_k=15, min_peaks=10),
    "win64": dict(peak_mode="window", window_th=64.0, window_k=6, min_peaks=5, fragment_min_mz=128.0),
    "win12": dict(peak_mode="window", window_th=12.5, window_k=3, min_peaks=5),   # 1/12.5 is inexact in f32
}


def _window_spectra(rng):
    """(mz, intensity) arrays of the seeded edge-case spectra."""
    f32 = np.float32
    out = []

    def add(mz, it):
        out.append((np.asarray(mz, f32), np.asarray(it, f32)))

    def lognormal(n):
        return rng.lognormal(7, 1.2, n).astype(f32)

    m = np.sort(rng.uniform(150, 2000, 400).astype(f32))
    add(m, lognormal(400))                                   # in order, windows over window_k
    dense = np.sort(np.concatenate([rng.uniform(500, 599.9, 300), rng.uniform(150, 2000, 60)]).astype(f32))
    add(dense, lognormal(len(dense)))                        # in order, one window of ~300 peaks
    o = rng.permutation(400)
    add(m[o], lognormal(400)[o])                             # shuffled
    mn = m.copy()
    mn[200] = np.nan
    add(mn, lognormal(400))                                  # a NaN m/z
    add(np.repeat(m[::2], 2), np.repeat(lognormal(200), 2))  # every peak twice
    edges = []
    for th in (100.0, 64.0):   # widths whose reciprocal product and division agree on every f32 (7.0 does not)
        for k in range(1, int(2000 // th) + 1):
            x = f32(k * th)
            edges += [np.nextafter(x, f32(0)), x, np.nextafter(x, f32(np.inf))]
    e = np.sort(np.array(edges, f32))
    add(e, lognormal(len(e)))                                # on and next to window boundaries
    add([100.0, 127.9, 128.0, 149.99, 150.0, 1999.99, 2000.0, 2000.01, 2500.0],
        lognormal(9))                                        # on and outside the fragment ranges
    add([], [])                                              # empty
    add(np.sort(rng.uniform(150, 2000, 200).astype(f32)), np.full(200, 1000.0, f32))   # equal intensities
    q = np.sort(rng.uniform(150, 2000, 100).astype(f32))
    add(np.repeat(q, 3), np.tile(np.array([1.0, 5.0, 3.0], f32), 100) * lognormal(300))  # equal m/z, mixed order
    big = np.sort(rng.uniform(150, 2000, 3000).astype(f32))
    add(big, lognormal(3000))                                # more than 2048 raw peaks
    return out


def build_inputs(fx, seed=2024):
    rng = np.random.default_rng(seed)
    extra = _window_spectra(rng)
    mz = [fx["sp_mz"]] + [m for m, _ in extra]
    it = [fx["sp_intensity"]] + [i for _, i in extra]
    lens = np.concatenate([np.diff(fx["sp_offsets"]), [len(m) for m, _ in extra]]).astype(np.int64)
    off = np.zeros(len(lens) + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    n0, n1 = len(fx["sp_offsets"]) - 1, len(extra)
    return {
        "w_mz": np.concatenate(mz).astype(np.float32),
        "w_intensity": np.concatenate(it).astype(np.float32),
        "w_offsets": off,
        "w_scan": np.arange(n0 + n1, dtype=np.uint32),
        "w_index": np.arange(n0 + n1, dtype=np.uint32),
        "w_rt": np.zeros(n0 + n1),
        "w_precursor_mz": np.concatenate([fx["sp_precursor_mz"], rng.uniform(400, 1200, n1)]),
        "w_charge": np.concatenate([fx["sp_charge"], np.full(n1, 2)]).astype(np.int8),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True)
    a = ap.parse_args()
    ref_root = os.path.abspath(a.reference)
    sys.path.insert(0, ref_root)
    import torch
    from vulcan.gpu import engine as RE      # the reference (ref_root is first on sys.path)
    from vulcan.gpu import host as RH
    assert os.path.abspath(RE.__file__).startswith(ref_root), RE.__file__
    fx = dict(np.load(os.path.join(HERE, "mini_fixture.npz")))
    g = build_inputs(fx)
    sp = RH.Spectra("window", g["w_scan"], g["w_index"], g["w_rt"], g["w_precursor_mz"], g["w_charge"], g["w_mz"],
                    g["w_intensity"], g["w_offsets"])
    mz = g["w_mz"][~np.isnan(g["w_mz"])]
    for name, kw in WINDOW_SETS.items():
        th = kw["window_th"]
        cpu_div = np.floor(mz / np.float32(th)).astype(np.int64)
        dev_mul = np.floor((mz * (np.float32(1.0) / np.float32(th))).astype(np.float32)).astype(np.int64)
        assert np.array_equal(cpu_div, dev_mul), f"{name}: division and reciprocal product disagree on an input"
        p = RH.SearchParams(**kw)
        pk = RE.k0_preprocess(sp, p, torch.device("cpu"), RE.Stats())
        for k in ("off", "mass", "int", "tic"):
            g[f"{name}/k0_{k}"] = pk[k].numpy()
        g[f"{name}/k0_valid"] = pk["valid"]
    np.savez_compressed(os.path.join(HERE, "golden_window.npz"), **g)
    print("spectra", len(g["w_offsets"]) - 1, "peaks", len(g["w_mz"]), "keys", len(g))


if __name__ == "__main__":
    main()
