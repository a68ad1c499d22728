"""The native peptidoform expansion (csrc/vulcan_core.cpp, the reference's lib.rs:271-399 contract) equals the
plain-Python oracle (oracle/index_oracle.py) form by form: masks of both sides of every pair, f64 mass, xxh64 ids and
Sage f32 masses, with and without site limits (per residue and per residue group, e.g. phospho on S/T/Y)."""
import numpy as np
import pytest

from oracle import index_oracle as IO
from vulcan.index import _core

AA = "ACDEFGHIKLMNPQRSTVWY"


def _pairs(rng, n):
    fwd, dec, perms, flat, off = [], [], [], [], [0]
    for i in range(n):
        L = int(rng.integers(7, 16))
        f = "".join(rng.choice(list(AA), L - 1)) + rng.choice(["K", "R"])
        if i % 3 == 0:       # shuffled decoy: a permutation that keeps the C-terminal residue
            perm = list(rng.permutation(L - 1)) + [L - 1]
            perms.append(perm)
            flat += perm
        else:                # pseudo-reverse (empty slice in the native layout)
            perm = [L - 2 - j for j in range(L - 1)] + [L - 1]
            perms.append(None)
        d = "".join(f[perm[j]] for j in range(L))
        fwd.append(f)
        dec.append(d)
        off.append(len(flat))
    return fwd, dec, perms, np.array(flat, np.uint8), np.array(off, np.int64)


@pytest.mark.parametrize("nterm", [False, True])
@pytest.mark.parametrize("max_var,limits", [(2, None), (3, {"M": 1}), (4, {"STY": 3, "M": 1}), (3, {"S": 1, "TY": 1})])
def test_native_expansion_equals_oracle(max_var, limits, nterm):
    """nterm: a variable peptide N-terminal modification ("^", acetyl) as well, mask bit 63."""
    rng = np.random.default_rng(max_var * 7 + (len(limits) if limits else 0))
    fwd, dec, perms, flat, off = _pairs(rng, 60)
    static = {"C": 57.021464}
    var = {"M": 15.9949, "S": 79.966331, "T": 79.966331, "Y": 79.966331}
    if nterm:
        var["^"] = 42.010565
    got = _core.expand_pairs(fwd, dec, flat, off, list(static.items()), list(var.items()), max_var, 500.0, 5000.0, 11,
                             site_limits=limits,
                             nthreads=2)
    want = IO.expand_pairs(fwd, dec, perms, static, var, max_var, 500.0, 5000.0, 11, site_limits=limits)
    have = {(int(i), int(mf), int(md), round(float(m), 9), int(a), int(b), float(x), float(y))
            for i, mf, md, m, a, b, x, y in zip(got["seq"], got["mask_f"], got["mask_d"], got["mass"], got["id_f"],
                                                 got["id_d"], got["mass32_f"], got["mass32_d"])}
    assert len(have) == len(got["seq"]) and have == want
    if nterm:
        assert any(int(m) >> 63 for m in got["mask_f"])
    if limits and "STY" in limits:     # the group cap binds: some peptide has 4+ S/T/Y sites
        assert any(sum(c in "STY" for c in f) > 3 for f in fwd)
        sty = [sum(((int(m) >> k) & 1) and fwd[int(i)][k] in "STY" for k in range(len(fwd[int(i)])))
               for i, m in zip(got["seq"], got["mask_f"])]
        assert max(sty) == 3
