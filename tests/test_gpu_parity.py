"""Parity of the sm_100a kernels with the oracle and with the reference's own kernels, on the mini fixture
(three parameter sets: Da tolerance, ppm tolerance, ppm with fragment charges up to z-1 and isotope errors -1..2).

Integer, index and f32 outputs must be bit-identical; hyperscores (f64 log on the device vs the host libm) within
1e-12 relative of the oracle and bit-identical to the reference's kernels (same device log)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SETS = ("da", "ppm", "ppm_mfz")
STATIC = {"C": 57.021464}
VAR = {"M": 15.9949}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    return torch


@pytest.fixture(scope="module")
def indexes(mini, param_sets, torch_cuda):
    from vulcan.gpu import engine as E
    l1, _, _ = mini
    return {name: E.GpuIndex(l1, p, STATIC, VAR) for name, p in param_sets.items()}


def _hyp(g, name):
    return {k: g[f"{name}/hyp_{k}"] for k in ("spec", "z", "iso", "pm", "M", "lo", "hi", "maxfz")}


@pytest.mark.parametrize("name", SETS)
def test_k0_device_equals_reference(mini, golden_py, param_sets, indexes, name):
    from vulcan.gpu import engine as E
    _, sp, _ = mini
    st = E.Stats()
    pk = E.k0_preprocess(sp, param_sets[name], indexes[name].dev, st)
    g = golden_py
    assert np.array_equal(pk["off"].cpu().numpy(), g[f"{name}/k0_off"])
    assert np.array_equal(pk["mass"].cpu().numpy(), g[f"{name}/k0_mass"])
    assert np.array_equal(pk["int"].cpu().numpy(), g[f"{name}/k0_int"])
    assert np.array_equal(pk["valid"], g[f"{name}/k0_valid"])
    np.testing.assert_allclose(pk["tic"].cpu().numpy(), g[f"{name}/k0_tic"], rtol=1e-7)


@pytest.mark.parametrize("name", SETS)
def test_search_stages_equal_reference(mini, golden_py, golden_kernels, param_sets, indexes, name, torch_cuda):
    """Device hypotheses, dense K1 counts, top-K + closure and K2 of engine.search equal the references."""
    from oracle import oracle as O
    from vulcan.gpu import engine as E
    import dataclasses
    l1, sp, _ = mini
    p = dataclasses.replace(param_sets[name], search_method="staged")
    g = golden_py
    tbl, st, out = E.search(sp, indexes[name], l1, p, report=3)
    dh = out["dh"]
    nh = int(dh["spec_off"][-1])
    for k in ("spec", "z", "iso", "pm", "M", "lo", "hi", "maxfz"):
        assert np.array_equal(dh[k][:nh].cpu().numpy(), g[f"{name}/hyp_{k}"]), k
    # dense K1 counts == oracle window counts; nonzero set == the reference kernels' K1 append set
    hyp = _hyp(g, name)
    P = O.make_params(STATIC, VAR, p.fragment_unit)
    peaks = {k: g[f"{name}/k0_{k}"] for k in ("off", "mass", "int")}
    win_off, cnt, sc, mt = O.k1_windows(l1, hyp, peaks, p, P)
    assert np.array_equal(out["cnt"][:int(out["win_off"][-1])].cpu().numpy(), cnt)
    assert np.array_equal(out["hyp_scored"][:nh].cpu().numpy().astype(np.int64), golden_kernels[f"{name}/k1_scored"])
    assert np.array_equal(out["hyp_matched"][:nh].cpu().numpy().astype(np.int64),
                          golden_kernels[f"{name}/k1_matched"])
    # top-K + pair closure == the reference's select_topk
    nc = int(out["cand_off"][-1])
    assert np.array_equal(out["c_hyp"][:nc].cpu().numpy(), g[f"{name}/topk_h"])
    assert np.array_equal(out["c_row"][:nc].cpu().numpy(), g[f"{name}/topk_r"])
    assert np.array_equal(out["c_cnt"][:nc].cpu().numpy(), g[f"{name}/topk_c"])
    # K2 == oracle (bit-exact f32 / integer outputs)
    k2o = O.k2(l1, hyp, peaks, g[f"{name}/topk_h"], g[f"{name}/topk_r"], p, P)
    for k in ("summed_b", "summed_y", "matched_b", "matched_y", "longest_b", "longest_y"):
        assert np.array_equal(out["k2"][k][:nc].cpu().numpy(), k2o[k]), k
    assert np.array_equal(out["k2"]["ppm"][:nc].cpu().numpy(), k2o["ppm"], equal_nan=True)
    np.testing.assert_allclose(out["k2"]["hyperscore"][:nc].cpu().numpy(), k2o["hyperscore"], rtol=1e-12)
    # the PSM table == the reference's psm_table
    cols = ("spec_idx", "rank", "pf_row", "pf_id", "charge", "isotope_error", "expmass", "calcmass",
            "delta_mass_ppm", "matched_b", "matched_y", "matched_peaks", "summed_intensity", "longest_b",
            "longest_y", "longest_y_pct", "peptide_len", "missed_cleavages", "n_var", "k1_count",
            "scored_candidates", "average_ppm")
    for c in cols:
        assert np.array_equal(tbl.column(c).to_numpy(), g[f"{name}/psm_{c}"], equal_nan=True), c
    for c in ("hyperscore", "delta_next", "delta_best", "poisson"):
        np.testing.assert_allclose(tbl.column(c).to_numpy(), g[f"{name}/psm_{c}"], rtol=1e-9, atol=1e-12)
    # the TIC is an f64 sum rounded to f32 whose summation order differs from the reference's
    np.testing.assert_allclose(tbl.column("matched_intensity_pct").to_numpy(), g[f"{name}/psm_matched_intensity_pct"],
                               rtol=1e-6)


@pytest.mark.parametrize("name", SETS)
def test_compat_entry_points_equal_reference_kernels(mini, golden_py, golden_kernels, param_sets, indexes, name,
                                                     torch_cuda):
    """The reference-named entry points (vk_frag_count/emit, vk_k1 over the reference CSR, vk_k1_brute,
    vk_k2, vk_k2_shift) reproduce the reference's kernels exactly."""
    torch = torch_cuda
    from vulcan.gpu import _lib as K
    from vulcan.gpu import engine as E
    l1, sp, _ = mini
    p = param_sets[name]
    gi = indexes[name]
    g = golden_py
    L = K.lib()
    # the process-wide constants of the compatible entry points follow the last index built; set this one's
    stat = np.array(gi.fp.stat[:], np.float32)
    var = np.array(gi.fp.var[:], np.float32)
    K.check(L.vk_set_params(E.SAGE_MONO.ctypes.data, stat.ctypes.data, var.ctypes.data), "set_params")
    K.check(L.vk_set_tol_da(gi.fp.tol_da), "set_tol_da")
    n = gi.n
    cnt = torch.empty(n, dtype=torch.int32, device=gi.dev)
    K.check(L.vk_frag_count(n, *gi.table_ptrs(), p.min_ion_index, p.fragment_min_mz, p.fragment_max_mz, K.ptr(cnt),
                            K.stream()), "frag_count")
    assert np.array_equal(cnt.cpu().numpy(), golden_kernels[f"{name}/frag_count"])
    gi._slices = None
    sl = gi.slices
    assert len(sl) == 1
    dev = gi.dev
    up = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(dev)
    pk_off, pk_mass = up(g[f"{name}/k0_off"], np.int64), up(g[f"{name}/k0_mass"], np.float32)
    pk_int = up(g[f"{name}/k0_int"], np.float32)
    d_spec, d_maxfz = up(g[f"{name}/hyp_spec"], np.int32), up(g[f"{name}/hyp_maxfz"], np.int8)
    wi = {k: up(g[f"{name}/wi_{k}"], np.int32) for k in ("hyp", "chunk", "lo", "hi")}
    cap = max(1, int((g[f"{name}/hyp_hi"] - g[f"{name}/hyp_lo"]).clip(0).sum()))
    n_out = torch.zeros(1, dtype=torch.int64, device=dev)
    o_h, o_r, o_c = (torch.empty(cap, dtype=torch.int32, device=dev) for _ in range(3))
    n_h = len(g[f"{name}/hyp_spec"])
    scored = torch.zeros(n_h, dtype=torch.int32, device=dev)
    matched = torch.zeros(n_h, dtype=torch.int64, device=dev)
    K.check(L.vk_k1(len(g[f"{name}/wi_hyp"]), K.ptr(wi["hyp"]), K.ptr(wi["chunk"]), K.ptr(wi["lo"]), K.ptr(wi["hi"]),
                    K.ptr(d_spec), K.ptr(d_maxfz), K.ptr(pk_off), K.ptr(pk_mass), K.ptr(sl[0].offsets),
                    K.ptr(sl[0].entries), gi.n_bins, 0, p.chunk_size, p.tile, p.fragment_ppm[0], p.fragment_ppm[1],
                    p.fragment_min_mz, gi.inv_logw, 1, cap, K.ptr(n_out), K.ptr(o_h), K.ptr(o_r), K.ptr(o_c),
                    K.ptr(scored), K.ptr(matched), K.stream()), "k1")
    m = int(n_out.item())
    key = (o_h[:m].long() << 32) | o_r[:m].long()
    o = torch.argsort(key)
    assert np.array_equal(key[o].cpu().numpy(), golden_kernels[f"{name}/k1_key"])
    assert np.array_equal(o_c[:m][o].cpu().numpy(), golden_kernels[f"{name}/k1_cnt"])
    assert np.array_equal(scored.cpu().numpy(), golden_kernels[f"{name}/k1_scored"])
    assert np.array_equal(matched.cpu().numpy(), golden_kernels[f"{name}/k1_matched"])
    h, r = up(g[f"{name}/win_h"], np.int64), up(g[f"{name}/win_r"], np.int64)
    bc = E.k1_brute(gi, _hyp(g, name), {"off": pk_off, "mass": pk_mass}, h, r, p)
    assert np.array_equal(bc.cpu().numpy(), golden_kernels[f"{name}/brute"])
    peaks = {"off": pk_off, "mass": pk_mass, "int": pk_int}
    for mode in ("closed", "shift"):
        shift = up(golden_kernels[f"{name}/k2shift_delta"], np.float32) if mode == "shift" else None
        k2 = E.run_k2(gi, h, r, d_spec, d_maxfz, peaks, p, shift=shift)
        for a, b in (("summed_b", "sb"), ("summed_y", "sy"), ("matched_b", "mb"), ("matched_y", "my"),
                     ("longest_b", "lb"), ("longest_y", "ly"), ("hyperscore", "hs")):
            assert np.array_equal(k2[a].cpu().numpy(), golden_kernels[f"{name}/k2{mode}_{b}"]), (mode, a)
        assert np.array_equal(k2["ppm"].cpu().numpy(), golden_kernels[f"{name}/k2{mode}_ppm"], equal_nan=True)


@pytest.mark.parametrize("name", SETS)
def test_k2_spectra_shift_equals_reference(mini, golden_py, golden_kernels, param_sets, indexes, name, torch_cuda):
    """The B200 K2 entry point (constants by value) in shifted mode == the reference's vk_k2_shift."""
    torch = torch_cuda
    from vulcan.gpu import _lib as K
    from vulcan.gpu import engine as E
    gi = indexes[name]
    p = param_sets[name]
    g = golden_py
    dev = gi.dev
    up = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(dev)
    h = g[f"{name}/win_h"]
    spec = g[f"{name}/hyp_spec"][h].astype(np.int64)
    n_spec = len(g[f"{name}/k0_off"]) - 1
    cand_off = np.zeros(n_spec + 1, np.int64)
    np.cumsum(np.bincount(spec, minlength=n_spec), out=cand_off[1:])
    out = E._k2_outputs(len(h), dev)
    # every device array stays referenced until the asynchronous launch has finished
    d_off, d_row = up(cand_off, np.int64), up(g[f"{name}/win_r"], np.int32)
    d_mfz, d_pko = up(g[f"{name}/hyp_maxfz"][h], np.int8), up(g[f"{name}/k0_off"], np.int64)
    d_pkm, d_pki = up(g[f"{name}/k0_mass"], np.float32), up(g[f"{name}/k0_int"], np.float32)
    d_shift = up(golden_kernels[f"{name}/k2shift_delta"], np.float32)
    K.check(K.lib().vk_k2_spectra(C.byref(gi.fp), n_spec, K.ptr(d_off), K.ptr(d_row), K.ptr(d_mfz), K.ptr(d_pko),
                                  K.ptr(d_pkm), K.ptr(d_pki), *gi.table_ptrs(), p.fragment_ppm[0], p.fragment_ppm[1],
                                  K.ptr(d_shift), *E._k2_ptrs(out), K.stream()), "k2_spectra")
    torch.cuda.synchronize()
    for a, b in (("summed_b", "sb"), ("summed_y", "sy"), ("matched_b", "mb"), ("matched_y", "my"),
                 ("longest_b", "lb"), ("longest_y", "ly"), ("hyperscore", "hs")):
        assert np.array_equal(out[a].cpu().numpy(), golden_kernels[f"{name}/k2shift_{b}"]), a


def test_topk_radix_selection_path(mini, param_sets, torch_cuda):
    """topk far below the appended count forces the radix-select path; result == oracle select_topk."""
    from oracle import oracle as O
    from vulcan.gpu import engine as E
    import dataclasses
    l1, sp, _ = mini
    for k in (1, 2, 3):
        p = dataclasses.replace(param_sets["ppm"], topk=k, search_method="staged")
        gi = E.GpuIndex(l1, p, STATIC, VAR)
        tbl, st, out = E.search(sp, gi, l1, p)
        pk = O.k0_view(sp, p)
        hyp = O.make_hypotheses(sp, pk["valid"], l1.mass32, p)
        P = O.make_params(STATIC, VAR, p.fragment_unit)
        win_off, cnt, sc, mt = O.k1_windows(l1, hyp, pk, p, P)
        oh, orr, oc = O.k1_appended(hyp, win_off, cnt, p.k1_threshold)
        H, R, Cc = O.select_topk(oh, orr, oc, hyp["spec"], l1.partner, p.topk)
        nc = int(out["cand_off"][-1])
        assert np.array_equal(out["c_hyp"][:nc].cpu().numpy(), H)
        assert np.array_equal(out["c_row"][:nc].cpu().numpy(), R)
        assert np.array_equal(out["c_cnt"][:nc].cpu().numpy(), Cc)


@pytest.mark.parametrize("name", SETS)
def test_k2_candidate_parallel_equals_warp_per_spectrum(mini, param_sets, indexes, name, torch_cuda):
    """vk_k2_cands (a thread per candidate, its CTA's peak masses staged) == vk_k2_spectra (a warp per spectrum,
    staged peaks, bucket table) bit for bit on the exhaustive path's candidate lists."""
    import dataclasses
    from vulcan.gpu import engine as E
    l1, sp, _ = mini
    p = dataclasses.replace(param_sets[name], search_method="staged")
    gi = indexes[name]
    st = E.Stats()
    out = E._search_device(E.DeviceRun(sp, gi.dev, st), gi, p, 3, st)
    E.check_status(out["status"])
    cand = {k: out[k] for k in ("cand_off", "c_row32", "c_maxfz", "cap")}
    k2 = E._k2_cands(gi, p, len(sp.charge), cand, out["peaks"], sparse=True)
    nc = int(out["cand_off"][-1])
    assert nc > 0
    for key in out["k2"]:
        a, b = out["k2"][key][:nc], k2[key][:nc]
        assert torch_cuda.equal(a, b) or (a.is_floating_point() and torch_cuda.equal(a.isnan(), b.isnan()) and
                                          torch_cuda.equal(a[~a.isnan()], b[~b.isnan()])), (name, key)


@pytest.mark.parametrize("unit", ("da", "ppm"))
def test_k2_sparse_long_rows_and_high_charges_equal_warp_per_spectrum(unit, torch_cuda):
    """vk_k2_cands == vk_k2_spectra bit for bit on synthetic rows of 2-60 residues with fragment charges up to 5,
    N-terminal and per-position variable modifications, peaks planted on the candidates' own b/y ladders, repeated
    masses and equal intensities, spectra above the 512-peak limit (whose CTAs read their peaks in global memory),
    empty spectra and spectra without candidates."""
    from vulcan.gpu import _lib as K
    from vulcan.gpu import engine as E
    torch = torch_cuda
    f32 = np.float32
    rng = np.random.default_rng(11)
    aa = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWY", np.uint8)
    fp = E.frag_params({"C": 57.021464}, {"M": 15.994915, "^": 42.010565}, unit)
    mono, stat, var = (np.array(list(getattr(fp, k)), f32) for k in ("mono", "stat", "var"))
    n_rows = 400
    lens = rng.integers(2, 61, n_rows).astype(np.uint8)
    seq_off = np.concatenate([[0], np.cumsum(lens.astype(np.int64))])
    res = rng.choice(aa, int(seq_off[-1])).astype(np.uint8)
    mask = rng.integers(0, 2 ** 62, n_rows, dtype=np.int64).astype(np.uint64) & np.uint64(0x0000_0F0F_0F0F_0F0F)
    mask[rng.random(n_rows) < 0.3] |= np.uint64(1 << 63)
    mass32 = rng.uniform(300.0, 6000.0, n_rows).astype(f32)

    def ladder(r, maxfz):
        """m/z of the row's b and y ions at fragment charges 1..maxfz-1, in the kernels' f32 arithmetic"""
        mk = int(mask[r])
        nt = f32(fp.nterm) if mk >> 63 else f32(0.0)
        b, y, out = nt, f32(mass32[r] - nt), []
        for k in range(int(lens[r]) - 1):
            i = int(res[seq_off[r] + k]) - 65
            rm = f32(mono[i] + (var[i] if (mk >> k) & 1 else stat[i]))
            b, y = f32(b + rm), f32(y - rm)
            out += [f32(v / f32(z)) for v in (b, y) for z in range(1, maxfz)]
        return np.array(out, f32)

    n_spec = 300
    offs, masses, ints, cand_off, c_row, c_maxfz = [0], [], [], [0], [], []
    for s in range(n_spec):
        nc = int(rng.choice([0, 1, 3, 4, 5, 9, 17]))
        rows = rng.integers(0, n_rows, nc)
        mfz = rng.integers(2, 7, nc)
        npk = int(rng.choice([0, 5, 60, 150, 700]))
        m = [rng.uniform(100.0, 3000.0, npk).astype(f32)]
        for r, z in zip(rows[:2], mfz[:2]):
            if npk:
                lad = ladder(int(r), int(z))
                lad = lad[rng.random(len(lad)) < 0.6]
                tol = 0.015 if unit == "da" else lad * 1.5e-5
                m.append((lad + rng.uniform(-1, 1, len(lad)) * tol).astype(f32))
        m = np.concatenate(m)
        rep = m[0::7][:len(m[1::7])]
        m[1::7][:len(rep)] = rep                                  # repeated masses
        m = np.sort(m)
        it = rng.lognormal(3.0, 1.0, len(m)).astype(f32)
        eq = it[3::9][:len(it[2::9])]
        it[2::9][:len(eq)] = eq                                   # equal intensities
        masses.append(m)
        ints.append(it)
        offs.append(offs[-1] + len(m))
        c_row.append(rows)
        c_maxfz.append(mfz)
        cand_off.append(cand_off[-1] + nc)
    dev = torch.device("cuda:0")
    t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)   # noqa: E731
    pk_off, pk_mass, pk_int = t(offs, torch.int64), t(np.concatenate(masses), torch.float32), \
        t(np.concatenate(ints), torch.float32)
    c_off = t(cand_off, torch.int64)
    rows = t(np.concatenate(c_row), torch.int32)
    mfz = t(np.concatenate(c_maxfz), torch.int8)
    tab = (t(seq_off, torch.int64), t(lens, torch.uint8), t(mask.view(np.int64), torch.int64),
           t(mass32, torch.float32), t(res, torch.uint8))
    tol = (-0.02, 0.02) if unit == "da" else (-20.0, 20.0)
    nc = int(cand_off[-1])
    L = K.lib()
    outs = []
    for fn in ("vk_k2_cands", "vk_k2_spectra"):
        o = E._k2_outputs(nc, dev)
        args = [C.byref(fp), n_spec, K.ptr(c_off), K.ptr(rows), K.ptr(mfz), K.ptr(pk_off), K.ptr(pk_mass),
                K.ptr(pk_int), *[K.ptr(x) for x in tab], tol[0], tol[1]]
        if fn == "vk_k2_spectra":
            args.append(None)
        K.check(getattr(L, fn)(*args, *E._k2_ptrs(o), K.stream()), fn)
        outs.append(o)
    torch.cuda.synchronize()
    assert int((outs[1]["matched_b"] > 5).sum()) > 50 and int((outs[1]["longest_y"] > 3).sum()) > 20
    for key in outs[0]:
        a, b = outs[0][key], outs[1][key]
        assert torch.equal(a.isnan(), b.isnan()) and torch.equal(a[~a.isnan()], b[~b.isnan()]), (unit, key)


@pytest.mark.parametrize("name", SETS)
def test_psm_rank_sparse_equals_warp_ranking(mini, param_sets, indexes, name, torch_cuda):
    """vk_psm_rank_sparse (a thread per spectrum) ranks exactly like vk_psm_rank (a warp per spectrum): the same
    slots, ranks and deltas, with 1 and 3 PSMs per spectrum."""
    import dataclasses
    from vulcan.gpu import engine as E
    l1, sp, _ = mini
    p = dataclasses.replace(param_sets[name], search_method="staged")
    gi = indexes[name]
    st = E.Stats()
    out = E._search_device(E.DeviceRun(sp, gi.dev, st), gi, p, 1, st)
    n = len(sp.charge)
    for report in (1, 3):
        a = E._rank_device(n, out["cand_off"], out["c_row"], out["k2"], p, report, gi.dev)
        b = E._rank_device(n, out["cand_off"], out["c_row"], out["k2"], p, report, gi.dev, sparse=True)
        filled = a[0] >= 0
        assert int(filled.sum()) > 0
        assert torch_cuda.equal(a[0], b[0]), (name, report)
        for x, y in zip(a[1:], b[1:]):   # rank and deltas of the filled slots (empty slots leave them unwritten)
            assert torch_cuda.equal(x[filled], y[filled]), (name, report)


@pytest.mark.parametrize("name", SETS)
def test_psm_pack_kernel_equals_torch_columns(mini, param_sets, indexes, name, torch_cuda):
    """vk_pack_psms (one kernel, filled slots compacted in slot order) writes the same PSM rows as the torch
    formulation of the table columns (all slots, a valid mask), bit for bit, with 1 and 3 PSMs per spectrum."""
    import dataclasses
    from vulcan.gpu import engine as E
    l1, sp, _ = mini
    p = dataclasses.replace(param_sets[name], search_method="staged")
    gi = indexes[name]
    n = len(sp.charge)
    for report in (1, 3):
        st = E.Stats()
        out = E._search_device(E.DeviceRun(sp, gi.dev, st), gi, p, report, st)
        a_buf, a_lay = E._pack_psms(gi, out, report, n)
        b_buf, b_lay = E._pack_psms_torch(gi, out, report, n)
        assert a_lay[0][0] == "n_rows" and a_lay[1:] == b_lay[1:]   # compacted rows, the same columns
        a = E._unpack_psms(a_buf.cpu().numpy(), a_lay)
        b = E._unpack_psms(b_buf.cpu().numpy(), b_lay)
        assert len(a["spec_idx"]) > 0
        for k in b:
            assert np.array_equal(a[k], b[k], equal_nan=a[k].dtype.kind == "f"), (name, report, k)


@pytest.mark.parametrize("topk", (3, 60))
def test_topk_over_shared_memory_capacity(mini, param_sets, torch_cuda, topk):
    """Precursor windows of +-2% make some spectra append more entries than a warp keeps in shared memory (512
    keys): their threshold comes from the radix select over the dense counts in global memory.  Candidates ==
    oracle select_topk, with and without pair closure."""
    from oracle import oracle as O
    from vulcan.gpu import engine as E
    import dataclasses
    l1, sp, _ = mini
    for closure in (True, False):
        p = dataclasses.replace(param_sets["ppm"], topk=topk, precursor_ppm=(-20000.0, 20000.0),
                                pair_closure=closure, search_method="staged")
        gi = E.GpuIndex(l1, p, STATIC, VAR)
        tbl, st, out = E.search(sp, gi, l1, p)
        pk = O.k0_view(sp, p)
        hyp = O.make_hypotheses(sp, pk["valid"], l1.mass32, p)
        P = O.make_params(STATIC, VAR, p.fragment_unit)
        win_off, cnt, sc, mt = O.k1_windows(l1, hyp, pk, p, P)
        oh, orr, oc = O.k1_appended(hyp, win_off, cnt, p.k1_threshold)
        n_app = np.bincount(np.asarray(hyp["spec"])[oh], minlength=len(sp.charge))
        assert n_app.max() > 512 and (n_app > topk).any()
        H, R, Cc = O.select_topk(oh, orr, oc, hyp["spec"], l1.partner, p.topk, closure)
        nc = int(out["cand_off"][-1])
        assert np.array_equal(out["c_hyp"][:nc].cpu().numpy(), H)
        assert np.array_equal(out["c_row"][:nc].cpu().numpy(), R)
        assert np.array_equal(out["c_cnt"][:nc].cpu().numpy(), Cc)


def test_search_finds_planted_truth(mini, param_sets, indexes):
    from vulcan.gpu import engine as E
    l1, sp, fx = mini
    tbl, _, _ = E.search(sp, indexes["da"], l1, param_sets["da"])
    top = dict(zip(tbl.column("spec_idx").to_pylist(), tbl.column("pf_row").to_pylist()))
    rows = fx["truth_rows"]
    hit = np.mean([top.get(i) == r for i, r in enumerate(rows)])
    assert hit > 0.9


def test_search_is_deterministic(mini, param_sets, indexes):
    from vulcan.gpu import engine as E
    l1, sp, _ = mini
    a = E.search(sp, indexes["ppm"], l1, param_sets["ppm"], report=5)[0]
    b = E.search(sp, indexes["ppm"], l1, param_sets["ppm"], report=5)[0]
    assert a.equals(b)


@pytest.mark.parametrize("layout", [(32, 12, 1), (64, 8, 4), (128, 2, 3), (256, 0, 8), (128, 1, 2),
                                    (512, 11, 16)])
def test_k1_counts_for_every_tile_layout(mini, param_sets, torch_cuda, layout):
    """Dense K1 counts and intensity sums do not depend on the tile size, the coarse bins per tile or the warps
    per CTA: the oracle's for every parameter set.  Many fine bins make tolerance windows straddle bin edges; a
    single bin per half of the key range makes the binary searches long."""
    import dataclasses
    from oracle import oracle as O
    from vulcan.gpu import engine as E
    from vulcan.gpu import prune as PR
    l1, sp, _ = mini
    tile_rows, cbin, warps = layout
    for name, p in param_sets.items():
        q = dataclasses.replace(p, tile_rows=tile_rows, cbin_bits=cbin, k1_warps=warps, search_method="staged")
        gi = E.GpuIndex(l1, q, STATIC, VAR)
        st = E.Stats()
        f = PR._front(E.DeviceRun(sp, gi.dev, st), gi, q, st, False, dense=True)
        hyp = {k: f["dh"][k].cpu().numpy() for k in ("spec", "maxfz", "lo", "hi")}
        pk = {k: f["peaks"][k].cpu().numpy() for k in ("off", "mass", "int")}
        P = O.make_params(STATIC, VAR, q.fragment_unit)
        win_off, cnt, _, _, isum = O.k1_windows(l1, hyp, pk, q, P, tic=f["peaks"]["tic"].cpu().numpy())
        n_win = int(f["win_off"][-1])
        assert np.array_equal(f["cnt"][:n_win].cpu().numpy(), cnt), name
        assert np.array_equal(f["isum"][:n_win].cpu().numpy().view(np.uint32), isum), name
        # the plain search's counts (no intensity sums) are the same
        out = E.search(sp, gi, l1, q)[2]
        assert np.array_equal(out["cnt"][:n_win].cpu().numpy(), cnt), name
        # the hit-list form gives the shortlist of the dense form, with the same intensity sums and statistics
        for thr in (1, 2):
            fh = PR._front(E.DeviceRun(sp, gi.dev, st), gi, q, st, False, min_count=thr)
            fd = PR._front(E.DeviceRun(sp, gi.dev, st), gi, q, st, False, min_count=thr, dense=True)
            _assert_same_shortlist(fh, fd, sp, (name, layout, thr))


def _assert_same_shortlist(fh, fd, sp, what):
    n = len(sp)
    nc = int(fd["hits"]["cand_off"][n])
    assert int(fh["hits"]["cand_off"][n]) == nc, what
    for k in ("c_hyp", "c_row", "c_cnt"):
        assert np.array_equal(fh["hits"][k][:nc].cpu().numpy(), fd["hits"][k][:nc].cpu().numpy()), (what, k)
    dh, hits = fd["dh"], fd["hits"]
    h = hits["c_hyp"][:nc]
    dense_isum = fd["isum"][fd["win_off"][h] + hits["c_row"][:nc] - dh["lo"][h]]
    assert np.array_equal(fh["hits"]["c_isum"][:nc].cpu().numpy(), dense_isum.cpu().numpy()), what
    nh = int(dh["spec_off"][n])
    for k in ("hyp_scored", "hyp_matched"):
        assert np.array_equal(fh[k][:nh].cpu().numpy().astype(np.int64),
                              fd[k][:nh].cpu().numpy().astype(np.int64)), (what, k)
    for k in ("spec_scored", "spec_matched"):
        assert np.array_equal(fh[k][:n].cpu().numpy(), fd[k][:n].cpu().numpy()), (what, k)


@pytest.mark.parametrize("name", SETS)
def test_k1_window_keys_precomputed_or_inline(mini, param_sets, indexes, name, torch_cuda, monkeypatch):
    """vk_k1_peak_keys equals an f32 numpy restatement of the tolerance window (Sage bounds, clamped to the
    fragment range), and K1's counts and intensity sums are the same whether every fragment charge's keys are
    precomputed, some, or none (computed inside the kernel)."""
    from vulcan.gpu import engine as E
    l1, sp, _ = mini
    p, gi = param_sets[name], indexes[name]
    run = E.DeviceRun(sp, gi.dev)
    peaks = E._k0_device(run, p, gi.dev)
    dh = E._hyp_device(run, peaks, gi, p)
    n_h = dh["n_max"]
    keys, filt, n_kz, kstride = E.peak_keys(gi, peaks, p)
    n_pk = int(peaks["off"][-1])
    m = peaks["mass"][:n_pk].cpu().numpy().astype(np.float32)
    kk = keys.cpu().numpy().view(np.uint32).reshape(-1, 2)
    fb, xb = np.uint32(gi.tix.fmin_bits), np.uint32(gi.tix.fmax_bits)
    fmin, fmax = fb.view(np.float32), xb.view(np.float32)
    lo_t, hi_t = np.float32(p.fragment_ppm[0]), np.float32(p.fragment_ppm[1])
    for z in range(1, n_kz + 1):
        mz = m * np.float32(z)
        if p.fragment_unit == "da":
            a, bd = mz + lo_t, mz + hi_t
        else:
            a = mz + (mz * lo_t) / np.float32(1e6)
            bd = mz + (mz * hi_t) / np.float32(1e6)
        ok = (bd >= fmin) & (a <= fmax)
        ka = np.where(a <= fmin, np.uint32(0), a.view(np.uint32) - fb)
        kb = np.where(bd >= fmax, xb - fb, bd.view(np.uint32) - fb)
        ka[~ok], kb[~ok] = 1, 0
        got = kk[(z - 1) * kstride:(z - 1) * kstride + n_pk]
        assert np.array_equal(got[:, 0], ka) and np.array_equal(got[:, 1], kb), (name, z)
        # filter words: bitmap positions of ka and kb (span capped at 4095), 0xffffffff for a missed window
        ix = gi.tix
        low = ix.mass_bits - ix.cbin_bits
        blog = _bitmap_log(gi)
        bits = min(blog, low)
        pos = lambda k: ((k >> low) << blog) | ((k & ((1 << low) - 1)) >> (low - bits))
        ga, gb = pos(ka.astype(np.int64)), pos(kb.astype(np.int64))
        want = (ga | (np.minimum(gb - ga, 4095) << 20)).astype(np.uint32)
        want[~ok] = 0xffffffff
        fw = filt.cpu().numpy().view(np.uint32)[(z - 1) * kstride:(z - 1) * kstride + n_pk]
        assert np.array_equal(fw, want), (name, z)
    ref = E._k1_dense(gi, dh, peaks, p, n_h, isum=True)
    n_win = int(ref[0][-1])
    assert n_win > 0
    for nk in (0, 1, 3):
        monkeypatch.setattr(E, "key_charges", lambda q, nk=nk: nk)
        win_off, cnt, status, isum = E._k1_dense(gi, dh, peaks, p, n_h, isum=True)
        assert int(status.item()) == 0
        assert torch_cuda.equal(cnt[:n_win], ref[1][:n_win]), (name, nk)
        assert torch_cuda.equal(isum[:n_win], ref[3][:n_win]), (name, nk)


def _bitmap_log(gi):
    """log2 of the presence-bitmap bits per coarse bin of the library build."""
    import ctypes as C
    from vulcan.gpu import _lib as K
    total = int(K.lib().vk_tindex_bitmap_bytes(C.byref(gi.tix)))
    per_bin = total * 8 // (gi.tix.n_tiles << gi.tix.cbin_bits)
    assert per_bin in (64, 128)
    return per_bin.bit_length() - 1


@pytest.mark.parametrize("layout", [(64, 8), (128, 9), (128, 1), (512, 11)])
def test_tile_bitmaps_equal_numpy(mini, param_sets, torch_cuda, layout):
    """vk_tindex_bitmap: bit (bin * 2^B + posting >> (32 - bits)) of each tile is set exactly for the postings of the
    tile (B = the build's bits-per-bin log, bits = min(B, low key bits)), recomputed here from the postings and the
    coarse-bin CSR."""
    import dataclasses
    from vulcan.gpu import engine as E
    l1, _, _ = mini
    tile_rows, cbin = layout
    p = dataclasses.replace(param_sets["ppm"], tile_rows=tile_rows, cbin_bits=cbin)
    gi = E.GpuIndex(l1, p, STATIC, VAR)
    ix = gi.tix
    nb = 1 << ix.cbin_bits
    stride = (nb + 1 + 7) & ~7
    blog = _bitmap_log(gi)
    words = (1 << blog) // 32
    bits = min(blog, ix.mass_bits - ix.cbin_bits)
    post = gi.postings.cpu().numpy().view(np.uint32)
    toff = gi.tile_off.cpu().numpy()
    cb = gi.cbin_off.cpu().numpy().view(np.uint16).astype(np.int64)
    bm = gi.bitmap.cpu().numpy().view(np.uint32)
    for t in range(ix.n_tiles):
        c = cb[t * stride:t * stride + nb + 1]
        pt = post[toff[t]:toff[t] + c[-1]].astype(np.int64)
        pos = (np.repeat(np.arange(nb), np.diff(c)) << blog) + (pt >> (32 - bits))
        want = np.zeros(nb * words, np.uint32)
        np.bitwise_or.at(want, pos >> 5, (np.uint32(1) << (pos & 31).astype(np.uint32)))
        assert np.array_equal(bm[t * nb * words:(t + 1) * nb * words], want), t


def test_k1_buffer_bounds_hold_and_overflow_is_reported(mini, param_sets, torch_cuda):
    """K1 buffers sized by the index's window bound never overflow on real windows; buffers made too small on
    purpose are not overrun: the kernels skip what does not fit and report VK_STATUS_OVERFLOW."""
    import ctypes as C
    from vulcan.gpu import _lib as K
    from vulcan.gpu import engine as E
    torch = torch_cuda
    l1, sp, _ = mini
    p = param_sets["da"]
    gi = E.GpuIndex(l1, p, STATIC, VAR)
    run = E.DeviceRun(sp, gi.dev)
    peaks = E._k0_device(run, p, gi.dev)
    dh = E._hyp_device(run, peaks, gi, p)
    n_h = dh["n_max"]
    win = (dh["hi"][:n_h] - dh["lo"][:n_h]).clamp(min=0)
    assert int(win.max()) <= gi.window_bound(*p.precursor_ppm)
    win_off, cnt, status = E._k1_dense(gi, dh, peaks, p, n_h)
    assert int(status.item()) == 0
    n_win = int(win_off[-1])
    L = K.lib()
    ix = gi.tix
    nt = ix.n_tiles
    tile_items = torch.empty(nt, dtype=torch.int64, device=gi.dev)
    wl = torch.empty(n_h, dtype=torch.int64, device=gi.dev)
    K.check(L.vk_k1_plan_count(C.byref(ix), n_h, K.ptr(dh["lo"]), K.ptr(dh["hi"]), K.ptr(tile_items), K.ptr(wl),
                               K.stream()), "k1_plan_count")
    item_off = E._scan(tile_items)
    n_items = int(item_off[-1])
    item_cap, cnt_cap = n_items // 2, n_win // 2
    st = torch.zeros(1, dtype=torch.int32, device=gi.dev)
    cursor = torch.empty(nt, dtype=torch.int64, device=gi.dev)
    item_hyp = torch.full((item_cap,), -1, dtype=torch.int32, device=gi.dev)
    K.check(L.vk_k1_plan_fill(C.byref(ix), n_h, K.ptr(dh["lo"]), K.ptr(dh["hi"]), K.ptr(item_off), K.ptr(cursor),
                              K.ptr(item_hyp), item_cap, K.ptr(st), K.stream()), "k1_plan_fill")
    small = torch.full((cnt_cap + 64,), -5, dtype=torch.int32, device=gi.dev)   # 64 guard entries past the cap
    K.check(L.vk_k1_tiles(C.byref(ix), C.byref(gi.fp), float(p.fragment_ppm[0]), float(p.fragment_ppm[1]),
                          p.k1_warps, K.ptr(item_off), K.ptr(item_hyp), n_h, item_cap, K.ptr(dh["spec"]),
                          K.ptr(dh["maxfz"]), K.ptr(dh["lo"]), K.ptr(dh["hi"]), K.ptr(win_off), cnt_cap,
                          K.ptr(peaks["off"]), K.ptr(peaks["mass"]), K.ptr(small), K.ptr(st), None, None, None,
                          None, None, 0, 0, K.stream()), "k1_tiles")
    assert int(st.item()) & 2
    assert bool((small[cnt_cap:] == -5).all())           # nothing written past the cap
    # rows of the windows that fit hold their exact count, or the fill value where the tile's item was skipped
    head = small[:cnt_cap]
    assert bool(((head == cnt[:cnt_cap]) | (head == -5)).all())
    assert bool((head == cnt[:cnt_cap]).any())


def test_tiles_too_large_for_shared_memory_are_refused(mini, param_sets, torch_cuda):
    """1024-row tiles of the mini index hold more postings than the build sorts in shared memory: refused."""
    import dataclasses
    from vulcan.gpu import engine as E
    l1, _, _ = mini
    q = dataclasses.replace(param_sets["da"], tile_rows=1024)
    with pytest.raises(RuntimeError, match="tindex_emit"):
        E.GpuIndex(l1, q, STATIC, VAR)


@pytest.mark.parametrize("name", ("da", "ppm"))
def test_k0_easy_and_hard_spectra(mini, param_sets, name, torch_cuda):
    """Sorted spectra take the stream-copy path, sorted ones with more in-range peaks than max_peaks the selection
    paths (a warp up to 512 raw peaks, a CTA above; threshold ties included: every peak twice), shuffled ones and
    ones with a NaN m/z the sorting path: every spectrum equals the oracle's peak view."""
    from oracle import oracle as O
    from vulcan.gpu import engine as E
    from vulcan.gpu.host import Spectra
    _, sp, _ = mini
    p = param_sets[name]
    rng = np.random.default_rng(21)
    mz, it, off = [], [], [0]
    for s in range(len(sp)):
        a, b = sp.offsets[s], sp.offsets[s + 1]
        m, i = sp.mz[a:b].copy(), sp.intensity[a:b].copy()
        kind = s % 4
        if kind == 1 and len(m):          # shuffled
            o = rng.permutation(len(m))
            m, i = m[o], i[o]
        elif kind == 2 and len(m):        # a NaN m/z in place
            m[len(m) // 2] = np.nan
        elif kind == 3 and len(m) > 2:    # every peak twice (ties in mass and intensity), still sorted
            m, i = np.repeat(m, 2), np.repeat(i, 2)
        if s in (0, 4):                   # sorted, 400 and 900 raw peaks: both selection paths
            n_raw = 400 if s == 0 else 900
            m = np.sort(rng.uniform(150, 1900, n_raw)).astype(np.float32)
            i = rng.lognormal(7, 1, n_raw).astype(np.float32)
        mz.append(m)
        it.append(i)
        off.append(off[-1] + len(m))
    sp2 = Spectra("mixed", sp.scan, sp.index, sp.rt, sp.precursor_mz, sp.charge, np.concatenate(mz).astype(np.float32),
                  np.concatenate(it).astype(np.float32), np.array(off, np.int64))
    in_order_over = [len(m) for m in mz if len(m) and np.all(np.diff(m) >= 0) and
                     int(((m >= p.fragment_min_mz) & (m <= p.fragment_max_mz)).sum()) > p.max_peaks]
    assert any(n <= 512 for n in in_order_over)   # the warp selection path is reached
    assert any(n > 512 for n in in_order_over)    # the CTA selection path is reached
    pk = E.k0_preprocess(sp2, p, torch_cuda.device("cuda"), E.Stats())
    ref = O.k0_view(sp2, p)
    assert np.array_equal(pk["off"].cpu().numpy(), ref["off"])
    assert np.array_equal(pk["mass"].cpu().numpy(), ref["mass"])
    assert np.array_equal(pk["int"].cpu().numpy(), ref["int"])
    assert np.array_equal(pk["valid"], ref["valid"])
    np.testing.assert_allclose(pk["tic"].cpu().numpy(), ref["tic"], rtol=1e-7)


def test_k0_cta_path_for_large_spectra(mini, param_sets, torch_cuda):
    """Runs with a spectrum of more than 2048 raw peaks use the CTA sort kernel; it equals the oracle too."""
    from oracle import oracle as O
    from vulcan.gpu import engine as E
    from vulcan.gpu.host import Spectra
    l1, sp, _ = mini
    rng = np.random.default_rng(9)
    big = np.sort(rng.uniform(100, 2100, 3000)).astype(np.float32)
    mz = np.concatenate([sp.mz, big])
    it = np.concatenate([sp.intensity, rng.lognormal(7, 1, 3000).astype(np.float32)])
    off = np.concatenate([sp.offsets, [len(mz)]])
    n = len(sp) + 1
    sp2 = Spectra("big", np.arange(n, dtype=np.uint32), np.arange(n, dtype=np.uint32), np.zeros(n),
                  np.concatenate([sp.precursor_mz, [800.0]]), np.concatenate([sp.charge, [2]]).astype(np.int8), mz, it,
                  off.astype(np.int64))
    for name in ("da", "ppm"):
        p = param_sets[name]
        pk = E.k0_preprocess(sp2, p, "cuda", E.Stats())
        ref = O.k0_view(sp2, p)
        assert np.array_equal(pk["off"].cpu().numpy(), ref["off"])
        assert np.array_equal(pk["mass"].cpu().numpy(), ref["mass"])
        assert np.array_equal(pk["int"].cpu().numpy(), ref["int"])
        assert np.array_equal(pk["valid"], ref["valid"])


@pytest.mark.parametrize("name", SETS)
@pytest.mark.parametrize("topk", (None, 2))
def test_fused_search_equals_staged_and_reference(mini, golden_py, param_sets, indexes, name, topk, torch_cuda):
    """The fused persistent kernel gives the staged path's candidates (with K2 outputs) and PSM table, and the
    reference's select_topk / psm_table on the golden fixture."""
    import dataclasses
    from vulcan.gpu import engine as E
    l1, sp, _ = mini
    # the fused kernel stages one index tile per warp: 64-row tiles
    p = dataclasses.replace(param_sets[name], tile_rows=64)
    if topk is not None:
        p = dataclasses.replace(p, topk=topk)
    gi = E.GpuIndex(l1, p, STATIC, VAR)
    staged = dataclasses.replace(p, search_method="staged")
    t_s, _, o_s = E.search(sp, gi, l1, staged, report=3)
    t_f, _, o_f = E.search(sp, gi, l1, p, report=3)
    assert t_f.equals(t_s)
    # candidate-level outputs of the fused kernel
    st = E.Stats()
    run = E.DeviceRun(sp, gi.dev, st)
    of = E._search_fused_device(run, gi, p, 3, st, cand=True)
    cd, cap = of["cand"], of["cand_cap"]
    n_cand = cd["n_cand"].cpu().numpy()
    assert (n_cand >= 0).all()
    sel = np.concatenate([np.arange(s * cap, s * cap + n_cand[s]) for s in range(len(n_cand))]).astype(np.int64)
    nc = int(o_s["cand_off"][-1])
    assert len(sel) == nc
    for a, b in (("c_hyp", "c_hyp"), ("c_row", "c_row"), ("c_cnt", "c_cnt")):
        assert np.array_equal(cd[a].cpu().numpy()[sel], o_s[b][:nc].cpu().numpy()), a
    for k, name2, _ in E._K2_KEYS:
        x, y = cd[k].cpu().numpy()[sel], o_s["k2"][name2][:nc].cpu().numpy()
        assert np.array_equal(x, y, equal_nan=True), k
    assert np.array_equal(of["hyp_scored"][:len(golden_py[f"{name}/hyp_spec"])].cpu().numpy(),
                          o_s["hyp_scored"][:len(golden_py[f"{name}/hyp_spec"])].cpu().numpy())
    if topk is None:
        g = golden_py
        assert np.array_equal(cd["c_hyp"].cpu().numpy()[sel], g[f"{name}/topk_h"])
        assert np.array_equal(cd["c_row"].cpu().numpy()[sel], g[f"{name}/topk_r"])
        assert np.array_equal(t_f.column("pf_row").to_numpy(), g[f"{name}/psm_pf_row"])


@pytest.mark.parametrize("name", SETS)
def test_graphed_searcher_equals_search(mini, param_sets, indexes, name, torch_cuda):
    """The graph-captured Searcher returns engine.search's PSM table, for pinned and pageable inputs, for runs of
    the same shape replayed through the same captured pass and for a run of another shape."""
    import dataclasses
    from vulcan.gpu import engine as E
    from vulcan.gpu.host import Spectra
    l1, sp, _ = mini
    p = dataclasses.replace(param_sets[name], search_method="staged")
    gi = indexes[name]
    want = E.search(sp, gi, l1, p, report=2)[0]
    se = E.Searcher(gi, l1, p, report=2)
    # a second run of the same shape: the peaks of every spectrum reversed in intensity order
    inv = sp.intensity[::-1].copy()
    sp2 = Spectra("other", sp.scan, sp.index, sp.rt, sp.precursor_mz, sp.charge, sp.mz, inv, sp.offsets)
    want2 = E.search(sp2, gi, l1, p, report=2)[0]
    res = se.search_many([sp, E.pin_spectra(sp2), sp, sp2])
    assert res[0][0].equals(want) and res[2][0].equals(want)
    assert res[1][0].equals(want2) and res[3][0].equals(want2)
    # another shape: the first 100 spectra
    n = 100
    o = sp.offsets[:n + 1]
    sp3 = Spectra("head", sp.scan[:n], sp.index[:n], sp.rt[:n], sp.precursor_mz[:n], sp.charge[:n], sp.mz[:o[-1]],
                  sp.intensity[:o[-1]], o.copy())
    assert se.search(sp3)[0].equals(E.search(sp3, gi, l1, p, report=2)[0])
    assert len(se.slots) == 2


@pytest.mark.parametrize("name", SETS)
def test_psm_table_features_on_device_equal_host(mini, param_sets, indexes, name, torch_cuda):
    """The PSM table columns computed on the device (packed gather) equal the host computation of the same
    features from the gathered records: bit for bit, except the f64 Poisson term (device exp / log / pow)."""
    import dataclasses
    from vulcan.gpu import engine as E
    l1, sp, _ = mini
    p = dataclasses.replace(param_sets[name], search_method="staged")
    gi = indexes[name]
    st = E.Stats()
    run = E.DeviceRun(sp, gi.dev, st)
    out = E._search_device(run, gi, p, 3, st)
    dev_tbl = E._read_packed(*E._pack_psms(gi, out, 3, run.n), sp)
    rec = E._gather_psms(*out["psm"], out["c_hyp"], out["c_row"], out["c_cnt"], out["k2"], out["dh"],
                         out["spec_scored"], out["spec_matched"], out["peaks"]["tic"], 3)
    host_tbl = E._psm_columns(sp, l1, rec, p)
    assert dev_tbl.num_rows == host_tbl.num_rows > 0
    assert dev_tbl.column_names == host_tbl.column_names
    for c in dev_tbl.column_names:
        a, b = dev_tbl.column(c).to_numpy(), host_tbl.column(c).to_numpy()
        if c == "poisson":
            np.testing.assert_allclose(a, b, rtol=1e-12)
        else:
            assert np.array_equal(a, b, equal_nan=a.dtype.kind == "f"), c


def _slice_run(sp, a, b, name):
    from vulcan.gpu.host import Spectra
    o = sp.offsets[a:b + 1]
    return Spectra(name, sp.scan[a:b], sp.index[a:b], sp.rt[a:b], sp.precursor_mz[a:b], sp.charge[a:b],
                   sp.mz[o[0]:o[-1]], sp.intensity[o[0]:o[-1]], o - o[0])


@pytest.mark.parametrize("name", SETS)
def test_batched_search_equals_per_run_search(mini, param_sets, indexes, name, torch_cuda):
    """Runs of different sizes packed into fixed-shape padded batches (one captured pass replayed per batch):
    every run's table equals its own engine.search."""
    import dataclasses
    from vulcan.gpu import engine as E
    l1, sp, _ = mini
    p = dataclasses.replace(param_sets[name], search_method="staged")
    gi = indexes[name]
    cuts = [0, 7, 60, 61, 100, 160]
    runs = [_slice_run(sp, a, b, f"run{i}") for i, (a, b) in enumerate(zip(cuts[:-1], cuts[1:]))]
    runs.append(_slice_run(sp, 0, 0, "empty"))
    runs.append(sp)
    se = E.Searcher(gi, l1, p, report=2)
    got = se.search_batch(runs, batch_spectra=64)
    assert len(got) == len(runs)
    for r, (tbl, _) in zip(runs, got):
        want = E.search(r, gi, l1, p, report=2)[0]
        assert tbl.equals(want), r.run
    assert len(se.slots) == 1     # every batch replayed the same captured pass


@pytest.mark.parametrize("depth", (1, 2, 3))
def test_searcher_pipeline_depth(mini, param_sets, indexes, depth, torch_cuda):
    """With 1, 2 or 3 runs in flight (slots per shape), search_many and search_batch return every run's own
    table; a submit into a slot whose result was not collected is refused."""
    import dataclasses
    from vulcan.gpu import engine as E
    from vulcan.gpu.host import Spectra
    l1, sp, _ = mini
    p = dataclasses.replace(param_sets["ppm"], search_method="staged")
    gi = indexes["ppm"]
    inv = sp.intensity[::-1].copy()
    sp2 = Spectra("other", sp.scan, sp.index, sp.rt, sp.precursor_mz, sp.charge, sp.mz, inv, sp.offsets)
    runs = [sp, sp2, E.pin_spectra(sp), sp2, sp]
    want = [E.search(r, gi, l1, p, report=2)[0] for r in runs]
    se = E.Searcher(gi, l1, p, report=2, depth=depth)
    for (tbl, _), w in zip(se.search_many(runs), want):
        assert tbl.equals(w)
    assert len(se.slots[next(iter(se.slots))]) == depth
    parts = [_slice_run(sp, a, b, f"r{i}") for i, (a, b) in enumerate(((0, 50), (50, 90), (90, 160)))]
    for (tbl, _), r in zip(se.search_batch(parts, batch_spectra=60), parts):
        assert tbl.equals(E.search(r, gi, l1, p, report=2)[0])
    handles = [se.submit(sp) for _ in range(depth)]
    with pytest.raises(RuntimeError):
        se.submit(sp)
    for h in handles:
        se.result(h)


def test_searcher_tables_own_their_result_buffers(mini, param_sets, indexes, torch_cuda):
    """Tables kept across many more runs than slots stay intact (each views its own pinned result buffer from the
    Searcher's pool); the buffers return to the pool when the tables are dropped and are reused; with no pool
    (``hold_bytes`` 0) or the pool exhausted the tables get copied columns."""
    import dataclasses
    import gc
    from vulcan.gpu import engine as E
    l1, sp, _ = mini
    p = dataclasses.replace(param_sets["ppm"], search_method="staged")
    gi = indexes["ppm"]
    want = E.search(sp, gi, l1, p, report=2)[0]
    se = E.Searcher(gi, l1, p, report=2, depth=2)
    got = se.search_many([sp] * 7)
    assert se.held_bytes() > 0
    for tbl, _ in got:
        assert tbl.equals(want)
    n_buf = sum(pl.n for pl in se.pools.values())
    del got, tbl
    gc.collect()
    assert se.held_bytes() == 0
    for tbl, _ in se.search_many([sp] * 7):   # the returned buffers are reused: no new ones
        assert tbl.equals(want)
    assert sum(pl.n for pl in se.pools.values()) == n_buf
    se0 = E.Searcher(gi, l1, p, report=2, depth=2, hold_bytes=0)
    for tbl, _ in se0.search_many([sp] * 4):
        assert tbl.equals(want)
    assert se0.held_bytes() == 0
    pool = next(iter(se.pools.values()))
    se2 = E.Searcher(gi, l1, p, report=2, depth=2, hold_bytes=2 * pool.nbytes)   # two buffers, then copies
    kept = se2.search_many([sp] * 5)
    assert all(t.equals(want) for t, _ in kept) and se2.held_bytes() == 2 * pool.nbytes


def test_autotuner_picks_a_measured_layout(mini, param_sets, tmp_path, torch_cuda):
    """The autotuner times every candidate layout on the sample, returns the fastest, reports peak-count buckets,
    and reuses its cached choice."""
    from vulcan.gpu import autotune as AT
    from vulcan.gpu import engine as E
    l1, sp, _ = mini
    p = param_sets["da"]
    cache = str(tmp_path / "tune.json")
    q, rep = AT.tune(l1, p, STATIC, VAR, sp, reps=2, tile_rows=(64, 128), k1_warps=(4, 8), cache=cache)
    ok = [c for c in rep["candidates"] if "ms" in c]
    assert len(ok) == 4 and not rep["cached"]
    best = min(ok, key=lambda c: c["ms"])
    assert (q.tile_rows, q.k1_warps) == (best["tile_rows"], best["k1_warps"])
    assert sum(b["spectra"] for b in rep["peak_buckets"]) == sum(np.diff(sp.offsets) > 0)
    q2, rep2 = AT.tune(l1, p, STATIC, VAR, sp, cache=cache)
    assert rep2["cached"] and (q2.tile_rows, q2.k1_warps) == (q.tile_rows, q.k1_warps)
    # the chosen layout searches like any other
    gi = E.GpuIndex(l1, q, STATIC, VAR)
    assert E.search(sp, gi, l1, q)[0].num_rows > 0


def test_phospho_index_search_equals_oracle(tmp_path, torch_cuda):
    """A small phospho index (S/T/Y at most 3 sites together, Met-ox at most 1; three variable residues) searched
    on the device equals the oracle's search: K1 counts, candidates, K2 and the top PSMs."""
    import dataclasses
    from oracle import oracle as O
    from vulcan import synth
    from vulcan.gpu import engine as E
    from vulcan.index.build import L1Index, read_labels
    w = dataclasses.replace(synth.WORKLOADS["phospho"], name="phospho_mini", n_proteins=60, n_spectra=300)
    d = synth.build_index(w, str(tmp_path))
    l1, lab = L1Index(d), read_labels(d)
    sp = synth.simulate_run(l1, lab, w)[0]
    p = w.search_params(topk=20)
    static, var = {"C": 57.021464}, w.var_mods
    gi = E.GpuIndex(l1, p, static, var)
    tbl, st, out = E.search(sp, gi, l1, p, report=2)
    P = O.make_params(static, var, p.fragment_unit)
    pk = O.k0_view(sp, p)
    hyp = O.make_hypotheses(sp, pk["valid"], l1.mass32, p)
    win_off, cnt, sc, mt = O.k1_windows(l1, hyp, pk, p, P)
    assert np.array_equal(out["cnt"][:int(out["win_off"][-1])].cpu().numpy(), cnt)
    oh, orr, oc = O.k1_appended(hyp, win_off, cnt, p.k1_threshold)
    h, r, c = O.select_topk(oh, orr, oc, hyp["spec"], l1.partner, p.topk)
    nc = int(out["cand_off"][-1])
    assert np.array_equal(out["c_row"][:nc].cpu().numpy(), r)
    k2 = O.k2(l1, hyp, pk, h, r, p, P)
    np.testing.assert_allclose(out["k2"]["hyperscore"][:nc].cpu().numpy(), k2["hyperscore"], rtol=1e-12)
    rk = O.psm_rank(k2, r, p.min_matched_peaks, 2)
    assert np.array_equal(tbl.column("pf_row").to_numpy(), r[rk["cand"]])
    assert tbl.num_rows > 0 and sum(synth.phospho_rows(l1)[tbl.column("pf_row").to_numpy()]) > 0


@pytest.mark.parametrize("topk", (3, 8, 32))
def test_short_hit_lists_with_overlapping_windows(mini, param_sets, torch_cuda, topk):
    """Precursor windows of +-1500 ppm make a spectrum's isotope hypotheses overlap, so rows are reached by several
    hypotheses: the short-list selection over hit lists merges them as the dense top-K does (lowest hypothesis, its
    intensity sum, highest count)."""
    import dataclasses
    from vulcan.gpu import engine as E
    from vulcan.gpu import prune as PR
    l1, sp, _ = mini
    for name in ("da", "ppm"):
        q = dataclasses.replace(param_sets[name], precursor_ppm=(-1500.0, 1500.0), topk=topk,
                                search_method="staged")
        gi = E.GpuIndex(l1, q, STATIC, VAR)
        st = E.Stats()
        fh = PR._front(E.DeviceRun(sp, gi.dev, st), gi, q, st, False, min_count=1)
        fd = PR._front(E.DeviceRun(sp, gi.dev, st), gi, q, st, False, min_count=1, dense=True)
        dh = fd["dh"]
        lo, hi, so = dh["lo"].cpu().numpy(), dh["hi"].cpu().numpy(), dh["spec_off"].cpu().numpy()
        overlap = any(max(lo[a], lo[b]) < min(hi[a], hi[b]) for s in range(len(sp))
                      for a in range(so[s], so[s + 1]) for b in range(a + 1, so[s + 1]))
        assert overlap, name
        _assert_same_shortlist(fh, fd, sp, (name, topk))


def test_scan_equals_cumsum_on_every_launch_shape(torch_cuda):
    """vk_scan_i64 == torch.cumsum (exclusive) at the sizes where its launch shape changes: one block of 4,096
    values (one kernel), up to 2,048 blocks (block sums + an apply kernel that adds the sums before its block),
    beyond (a third kernel scans the block sums); also in place (in == out + 1)."""
    from vulcan.gpu import _lib as K
    from vulcan.gpu import engine as E
    torch = torch_cuda
    L = K.lib()
    g = torch.Generator(device="cuda").manual_seed(5)
    for n in (1, 7, 4096, 4097, 3 * 4096 + 5, 2048 * 4096, 2048 * 4096 + 1, 3_000_001):
        x = torch.randint(-1000, 1 << 20, (n,), device="cuda", dtype=torch.int64, generator=g)
        want = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
        want[1:] = torch.cumsum(x, 0)
        assert torch.equal(E._scan(x), want), n
        kern = L.vk_scan_kernels(n)
        assert kern == (1 if n <= 4096 else (2 if n <= 2048 * 4096 else 3)), (n, kern)
        buf = torch.empty(n + 1, dtype=torch.int64, device="cuda")
        buf[1:] = x
        tmp = torch.empty((L.vk_scan_tmp_bytes(n) + 7) // 8, dtype=torch.int64, device="cuda")
        K.check(L.vk_scan_i64(K.ptr(buf[1:]), n, K.ptr(buf), K.ptr(tmp), K.stream()), "scan")
        assert torch.equal(buf, want), ("in place", n)
