"""Host-side logic of the engine on the CPU (no device calls): the packed PSM buffer -- its layout, the masked and
the compacted forms and their unpacking --, the table assembly, the greedy batch planning, the per-run split of a
batch's records, and the Searcher's argument check."""
import numpy as np
import pyarrow as pa
import pytest
import torch

from vulcan.gpu import engine as E
from vulcan.gpu.host import Spectra


def _columns(n, rng):
    """Random values of every packed column but the mask, as CPU tensors of the packed dtypes."""
    cols = {}
    for name, dt in E._PACK_COLS[1:]:
        dt = np.dtype(dt)
        if dt.kind == "f":
            a = rng.normal(0, 100, n).astype(dt)
        elif dt == np.uint64:
            a = rng.integers(0, 2 ** 63, n, dtype=np.int64).view(np.uint64) | np.uint64(1 << 63)
        else:
            info = np.iinfo(dt)
            a = rng.integers(max(info.min, -1000), min(info.max, 1000), n).astype(dt)
        cols[name] = a
    return cols


def test_pack_layout_is_aligned_and_cached():
    for slots in (0, 1, 7, 40000):
        layout, size, col_off = E._pack_layout(slots)
        assert [name for name, *_ in layout] == [name for name, _ in E._PACK_COLS]
        offs = [off for _, _, off, _ in layout]
        assert all(o % 8 == 0 for o in offs) and offs == sorted(offs) and list(col_off) == offs
        last = layout[-1]
        assert size >= last[2] + last[1].itemsize * slots and size % 8 == 0
        assert E._pack_layout(slots)[0] is layout


def test_masked_pack_unpacks_to_the_filled_slots():
    rng = np.random.default_rng(3)
    n = 1001
    cols = _columns(n, rng)
    ok = rng.random(n) < 0.6
    t = {k: torch.from_numpy(v.view(np.int64) if v.dtype == np.uint64 else v) for k, v in cols.items()}
    buf, layout = E._pack(t, torch.from_numpy(ok))
    rec = E._unpack_psms(buf.numpy(), layout)
    for k, v in cols.items():
        assert np.array_equal(rec[k].view(v.dtype), v[ok]), k


def test_compacted_pack_unpacks_by_row_count():
    """The kernel's form: filled slots first in slot order, their count (int64) where the mask column starts."""
    rng = np.random.default_rng(4)
    slots, n_rows = 500, 321
    layout, size, _ = E._pack_layout(slots)
    host = np.zeros(size, np.uint8)
    cols = _columns(slots, rng)
    for name, dt, off, cnt in layout[1:]:
        host[off:off + cnt * dt.itemsize] = cols[name].view(np.uint8)
    host[layout[0][2]:layout[0][2] + 8] = np.array([n_rows], np.int64).view(np.uint8)
    lay = [("n_rows", np.dtype(np.int64), layout[0][2], 1)] + layout[1:]
    rec = E._unpack_psms(host, lay)
    for k, v in cols.items():
        assert np.array_equal(rec[k], v[:n_rows]), k
    host[:] = 0      # the records own their memory: the pinned buffer may be reused at once
    assert np.array_equal(rec["hyperscore"], cols["hyperscore"][:n_rows])
    host[layout[0][2]:layout[0][2] + 8] = np.array([n_rows], np.int64).view(np.uint8)
    views = E._unpack_psms(host, lay, copy=False)   # views: the buffer belongs to the records
    assert all(v.base is not None and len(v) == n_rows for v in views.values())
    host[layout[1][2]:layout[1][2] + 8] = 7
    assert views[layout[1][0]].view(np.uint8)[0] == 7


def test_run_column_is_a_cached_slice():
    a = E._run_column("runA", 10)
    b = E._run_column("runA", 70_000)
    assert a.to_pylist() == ["runA"] * 10 and len(b) == 70_000 and b[69_999].as_py() == "runA"
    assert E._run_column("runB", 3).to_pylist() == ["runB"] * 3


def _run(name, n, n_peaks=3):
    off = np.arange(n + 1, dtype=np.int64) * n_peaks
    return Spectra(name, np.arange(100, 100 + n, dtype=np.uint32), np.arange(n, dtype=np.uint32),
                   np.linspace(0, 1, n), np.full(n, 500.0), np.full(n, 2, np.int8),
                   np.zeros(n * n_peaks, np.float32), np.zeros(n * n_peaks, np.float32), off)


def test_table_adds_run_scan_and_retention_time():
    rng = np.random.default_rng(5)
    sp = _run("runA", 50)
    cols = _columns(8, rng)
    cols["spec_idx"] = np.array([0, 3, 3, 7, 10, 20, 33, 49], np.int64)
    tbl = E._table(sp, cols)
    assert tbl.column_names == ["run", "spec_idx", "scan", "rt"] + list(E._PSM_TABLE[1:])
    assert tbl.column("run").to_pylist() == ["runA"] * 8
    assert np.array_equal(tbl.column("scan").to_numpy(), sp.scan[cols["spec_idx"]])
    assert np.array_equal(tbl.column("rt").to_numpy(), sp.rt[cols["spec_idx"]])
    assert isinstance(tbl, pa.Table) and tbl.num_rows == 8


def test_plan_batches_packs_whole_runs_in_order():
    runs = [_run(f"r{i}", n) for i, n in enumerate((30, 20, 70, 10, 10, 5, 200, 1))]
    groups = E.plan_batches(runs, 64)
    assert [i for g in groups for i in g] == list(range(len(runs)))      # every run once, in order
    for g in groups:
        size = sum(len(runs[i]) for i in g)
        assert size <= 64 or len(g) == 1                                   # a longer run is a batch of its own
    assert groups == [[0, 1], [2], [3, 4, 5], [6], [7]]
    assert E.plan_batches([], 64) == []


def test_split_table_gives_each_run_its_own_rows():
    rng = np.random.default_rng(6)
    runs = [_run("a", 4), _run("b", 0), _run("c", 6)]
    starts = [0, 4, 4, 10]
    spec = np.array([0, 0, 2, 3, 4, 5, 5, 9], np.int64)
    rec = _columns(len(spec), rng)
    rec["spec_idx"] = spec
    tabs = E.split_table(rec, runs, starts)
    assert [t.num_rows for t in tabs] == [4, 0, 4]
    assert tabs[0].column("spec_idx").to_pylist() == [0, 0, 2, 3]
    assert tabs[2].column("spec_idx").to_pylist() == [0, 1, 1, 5]
    assert tabs[2].column("run").to_pylist() == ["c"] * 4
    assert np.array_equal(tabs[2].column("hyperscore").to_numpy(), rec["hyperscore"][4:])


def test_searcher_refuses_an_empty_pipeline():
    with pytest.raises(ValueError):
        E.Searcher(None, None, None, depth=0)


def test_shortlist_count_rank_follows_the_selection_keys():
    """The calibration's count rank of a shortlist hit: its place in its spectrum by count descending, then row
    descending, then hypothesis ascending -- the order of vk_select_hits' selection keys."""
    from vulcan.gpu import prune as PR
    spec = torch.tensor([0, 0, 0, 0, 1, 1, 1])
    cnt = torch.tensor([3, 5, 3, 3, 2, 2, 9])
    row = torch.tensor([10, 4, 12, 12, 7, 8, 1])
    hyp = torch.tensor([0, 0, 2, 1, 3, 3, 4])
    d = {"spec": spec, "cnt": cnt, "row": row, "hits": {"c_hyp": hyp}}
    assert PR._count_rank(d).tolist() == [3, 0, 2, 1, 2, 1, 0]
