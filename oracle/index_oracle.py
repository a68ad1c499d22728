"""CPU oracle of the index side -- TEST INFRASTRUCTURE ONLY (imported by tests/ only).

Plain-Python restatement, for small inputs, of the reference's peptidoform expansion
(vulcan/rust/vulcan_core/src/lib.rs): mod-site enumeration of size <= max_var (:271-399), decoy mask through the
pair permutation (:349-354), canonical string (:215-228), xxh64 id (:230-234, via the `xxhash` package), Sage f32
mass with sequence-order f32 sums (:236-254) and the f64 mass filter (:256-269).  The native expansion
(vulcan-proteomics_b200/csrc/vulcan_core.cpp) is checked against it.
"""
from __future__ import annotations

import itertools

import numpy as np
import xxhash

SAGE_MONO = np.array([71.03711, 0.0, 103.00919, 115.02694, 129.04259, 147.0684, 57.02146, 137.05891, 113.08406,
                      0.0, 128.09496, 113.08406, 131.0405, 114.04293, 237.14774, 97.05276, 128.05858, 156.1011,
                      87.03203, 101.04768, 150.95363, 99.06841, 186.07932, 0.0, 163.06332, 0.0], np.float32)
RESIDUE_F64 = [71.037113805, 0.0, 103.009184505, 115.026943065, 129.042593135, 147.068413945, 57.021463721,
               137.058911875, 113.084064015, 0.0, 128.094963050, 113.084064015, 131.040484645, 114.042927470, 0.0,
               97.052763875, 128.058577540, 156.101111050, 87.032028435, 101.047678505, 0.0, 99.068413945,
               186.079312980, 0.0, 163.063328575, 0.0]
H2O32 = np.float32(18.010565)
H2O64 = 18.010564684
NTERM_BIT = 1 << 63


def canonical(seq, mask, var, nterm):
    s = f"[{nterm:+.4f}]-" if mask & NTERM_BIT else ""
    for k, c in enumerate(seq):
        s += c
        if (mask >> k) & 1:
            s += f"[{var.get(c, 0.0):+.4f}]"
    return s


def mass32(seq, mask, static, var, nterm):
    m = H2O32
    for c in seq:
        m = np.float32(m + SAGE_MONO[ord(c) - 65])
    ms = np.float32(0.0)
    for k, c in enumerate(seq):
        d = np.float32(var.get(c, 0.0)) if (mask >> k) & 1 else np.float32(static.get(c, 0.0))
        ms = np.float32(ms + d)
    if mask & NTERM_BIT:
        ms = np.float32(ms + np.float32(nterm))
    return np.float32(m + ms)


def mass64(seq, mask, static, var, nterm):
    m = H2O64
    for k, c in enumerate(seq):
        m += RESIDUE_F64[ord(c) - 65] + static.get(c, 0.0)
        if (mask >> k) & 1:
            m += var.get(c, 0.0)
    if mask & NTERM_BIT:
        m += nterm
    return m


def expand_pairs(fwd, dec, perms, static, var, max_var, min_mass, max_mass, id_seed, site_limits=None):
    """Rows (i, mask_f, mask_d, mass, id_f, id_d, mass32_f, mass32_d) as a set of tuples; perms[i] None means the
    pseudo-reverse permutation."""
    nterm = var.get("^", 0.0)
    resvar = {k: v for k, v in var.items() if k != "^"}
    out = set()
    for i, (f, d) in enumerate(zip(fwd, dec)):
        n = len(f)
        perm = perms[i] if perms[i] is not None else [n - 2 - j for j in range(n - 1)] + [n - 1]
        sites = [k for k, c in enumerate(f) if c in resvar] + ([63] if nterm else [])
        for r in range(0, min(max_var, len(sites)) + 1):
            for comb in itertools.combinations(sites, r):
                if site_limits:
                    per = {}
                    for k in comb:
                        if k != 63:
                            per[f[k]] = per.get(f[k], 0) + 1
                    # a key of one or more residues caps the sites of those residues together
                    if any(sum(per.get(c, 0) for c in key) > lim for key, lim in site_limits.items()):
                        continue
                m = 0
                for k in comb:
                    m |= 1 << k
                ms = mass64(f, m, static, resvar, nterm)
                if not (min_mass <= ms <= max_mass):
                    continue
                md = m & NTERM_BIT
                for j in range(n):
                    pj = int(perm[j])   # a Python int: m may carry bit 63 (N-terminal), beyond a numpy int64
                    if (m >> pj) & 1 and pj != 63:
                        md |= 1 << j
                idf = xxhash.xxh64_intdigest(canonical(f, m, resvar, nterm), id_seed)
                idd = xxhash.xxh64_intdigest(canonical(d, md, resvar, nterm), id_seed)
                out.add((i, m, md, round(ms, 9), idf, idd, float(mass32(f, m, static, resvar, nterm)),
                         float(mass32(d, md, static, resvar, nterm))))
    return out
