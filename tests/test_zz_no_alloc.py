"""vk_scan_i64_noalloc, the exclusive scan that allocates nothing, against vk_scan_i64 (the same scan with a
caller-provided scratch buffer), through the C ABI.

It serves callers that cannot allocate device memory on this path (a cgo / JNI / plain C binding that holds only
its inputs and outputs, or a stage thread that must not call cudaMalloc / cudaFree because they synchronise the
device): the block partial sums live in a fixed device array inside the library.  The file is named to be
collected last; it passes alone in a fresh process (the first call on the device does the set-up) and after the
other tests.  Integer scan: results must be identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scan_with_scratch(K, x):
    import torch
    L = K.lib()
    n = x.numel()
    out = torch.empty(n + 1, dtype=torch.int64, device=x.device)
    tmp = torch.empty((L.vk_scan_tmp_bytes(n) + 7) // 8, dtype=torch.int64, device=x.device)
    K.check(L.vk_scan_i64(K.ptr(x), n, K.ptr(out), K.ptr(tmp), K.stream()), "scan")
    return out


def _scan_noalloc(K, x):
    import torch
    out = torch.full((x.numel() + 1,), -7, dtype=torch.int64, device=x.device)
    rc = K.lib().vk_scan_i64_noalloc(K.ptr(x), x.numel(), K.ptr(out), K.stream())
    assert rc == 0, rc
    return out


def test_noalloc_scan_matches_scan_with_scratch_on_two_calls_in_a_row():
    import torch
    from vulcan.gpu import _lib as K
    assert torch.cuda.is_available(), "needs a CUDA device"
    L = K.lib()
    max_n = L.vk_scan_noalloc_max_n()
    assert max_n == 8192 * 4096
    g = torch.Generator(device="cpu").manual_seed(11)
    # two calls in a row with different sizes and values: the second must not see the first's partial sums
    for n in (3_000_001, 1_234_567, 4096, 1):
        x = torch.randint(-1000, 100_000, (n,), generator=g, dtype=torch.int64).cuda()
        a = _scan_noalloc(K, x)
        b = _scan_with_scratch(K, x)
        torch.cuda.synchronize()
        assert torch.equal(a, b), n
        assert int(a[0]) == 0 and int(a[-1]) == int(x.sum())
    # the largest accepted size, then one element more is rejected without launching anything
    x = torch.ones(max_n, dtype=torch.int64, device="cuda")
    a = _scan_noalloc(K, x)
    torch.cuda.synchronize()
    assert int(a[-1]) == max_n and torch.equal(a, _scan_with_scratch(K, x))
    del x, a
    y = torch.ones(max_n + 1, dtype=torch.int64, device="cuda")
    out = torch.zeros(2, dtype=torch.int64, device="cuda")
    assert L.vk_scan_i64_noalloc(K.ptr(y), max_n + 1, K.ptr(out), K.stream()) == -3
    # empty input: out[0] = 0
    e = torch.empty(0, dtype=torch.int64, device="cuda")
    z = torch.full((1,), 5, dtype=torch.int64, device="cuda")
    assert L.vk_scan_i64_noalloc(K.ptr(e) if e.numel() else 0, 0, K.ptr(z), K.stream()) == 0
    torch.cuda.synchronize()
    assert int(z[0]) == 0
    assert np.array_equal(_scan_noalloc(K, torch.arange(5, device="cuda")).cpu().numpy(), [0, 0, 1, 3, 6, 10])
