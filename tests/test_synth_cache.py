"""The synthetic-workload index cache: processes that build the same index at the same time (one per GPU in a
multi-GPU benchmark) each end with the complete index, never with another process's partial files."""
import multiprocessing as mp
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(root, q):
    sys.path.insert(0, os.path.join(ROOT, "vulcan-proteomics_b200"))
    from vulcan import synth
    from vulcan.index.build import L1Index
    d = synth.build_index("small", root)
    q.put((d, len(L1Index(d))))


def test_concurrent_builds_of_one_index(tmp_path):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_build, args=(str(tmp_path), q)) for _ in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=600) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (d0, n0), (d1, n1) = out
    assert d0 == d1 and n0 == n1 > 0
    assert os.path.exists(os.path.join(d0, "meta.json"))
    assert [f for f in os.listdir(tmp_path) if ".tmp" in f] == []   # the losing copy is removed
