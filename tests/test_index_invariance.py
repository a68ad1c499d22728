"""Label-blind index (the reference's G0 invariance test, tests/gpu/test_k1_k2_small.py:72-84): a build whose pair
list is shuffled and whose target/decoy roles are swapped (build(..., shuffle_rows_seed, swap_labels), reference
vulcan/index/build.py:78-82) gives the same index side bit for bit (the labels are the only output allowed to
differ), so the search cannot tell targets from decoys; on the GPU both indexes give the same PSM table."""
import dataclasses
import os

import numpy as np
import pytest

COLS = ("pf_id", "mass32", "seq_off", "length", "mask", "n_var", "missed", "partner", "residues")


@pytest.fixture(scope="module")
def built(tmp_path_factory):
    from vulcan import synth
    from vulcan.index.build import build
    d = tmp_path_factory.mktemp("g0")
    w = dataclasses.replace(synth.WORKLOADS["small"], name="g0", n_proteins=60)
    fa = os.path.join(d, "proteome.fasta")
    with open(fa, "w") as fh:
        fh.write(synth.random_proteome_fasta(w.n_proteins, w.proteome_seed))
    build([fa], str(d / "a"), w.index_params())
    build([fa], str(d / "b"), w.index_params(), shuffle_rows_seed=3, swap_labels=True)
    return str(d / "a"), str(d / "b"), w


def test_role_swap_and_permutation_leave_the_index_unchanged(built):
    from vulcan.index.build import L1Index, read_labels
    a, b = L1Index(built[0]), L1Index(built[1])
    assert len(a) > 1000
    for k in COLS:
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    la = np.asarray(read_labels(built[0]).column("is_decoy").to_numpy(zero_copy_only=False), bool)
    lb = np.asarray(read_labels(built[1]).column("is_decoy").to_numpy(zero_copy_only=False), bool)
    assert la.sum() == len(la) // 2
    # the labels may differ by the reference's rule; here the swapped build marks the same rows as decoys (a row's
    # label follows its sequence, not the side of the pair it was expanded from)
    assert np.array_equal(la, lb)


@pytest.mark.gpu
def test_role_swap_and_permutation_leave_the_search_unchanged(built):
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    from vulcan import synth
    from vulcan.gpu import engine as E
    from vulcan.index.build import L1Index, read_labels
    a, b = L1Index(built[0]), L1Index(built[1])
    w = built[2]
    sp = synth.simulate_run(a, read_labels(built[0]), w, n_spectra=300)[0]
    p = w.search_params()
    out = []
    for l1 in (a, b):
        gi = E.GpuIndex(l1, p, {"C": 57.021464}, w.var_mods)
        out.append(E.search(sp, gi, l1, p, report=5)[0])
    assert out[0].num_rows > 0 and out[0].equals(out[1])
