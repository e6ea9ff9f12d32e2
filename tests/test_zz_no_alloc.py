"""The allocation-free scan (dfx_scan_exclusive_i32_static) through the C ABI, against the scan that takes caller
scratch (dfx_scan_exclusive_i32): identical results on two calls in a row (integer sums, so exactly equal), and a
clear error beyond its size limit.

It is for callers that cannot allocate device memory (their memory belongs to a host application's pool or budget):
they pass inputs and outputs only. This file is collected last, so a run that stops at its first failure has run
every other test before it; it needs no other test to have run first."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _scan_with_scratch(lib, x, n, stream):
    out = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    nb = lib.dfx_scan_scratch_bytes(n)
    scratch = torch.empty(nb, dtype=torch.uint8, device="cuda")
    st = lib.dfx_scan_exclusive_i32(x.data_ptr(), out.data_ptr(), n, scratch.data_ptr(), nb, stream)
    assert st == 0
    return out


def test_static_scan_matches_scratch_scan_twice():
    from diffractom_b200 import _lib
    torch.cuda.set_device(0)
    lib = _lib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(11)
    for n in (3_000_001, 77_777):                    # two calls in a row, the second smaller than the first
        host = rng.integers(0, 50, n).astype(np.int32)
        x = torch.as_tensor(host, device="cuda")
        ref = _scan_with_scratch(lib, x, n, stream)
        out = torch.full((n + 1,), -1, dtype=torch.int32, device="cuda")
        st = lib.dfx_scan_exclusive_i32_static(x.data_ptr(), out.data_ptr(), n, stream)
        assert st == 0, lib.dfx_last_error()
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
        expect = np.zeros(n + 1, np.int64)
        np.cumsum(host, out=expect[1:])
        assert np.array_equal(out.cpu().numpy().astype(np.int64), expect)


def test_static_scan_empty_and_largest_sizes():
    """n = 0 (only the tile-sum passes run: out[0] = 0) and n = DFX_SCAN_STATIC_MAX_N, which fills every tile slot
    of the built-in array plus the total's slot."""
    from diffractom_b200 import _lib
    torch.cuda.set_device(0)
    lib = _lib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    one = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.full((1,), -7, dtype=torch.int32, device="cuda")
    assert lib.dfx_scan_exclusive_i32_static(one.data_ptr(), out.data_ptr(), 0, stream) == 0, lib.dfx_last_error()
    torch.cuda.synchronize()
    assert int(out.item()) == 0
    n = 65536 * 2048                                  # DFX_SCAN_STATIC_MAX_N: 512 MiB of int32 input
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    x = torch.randint(0, 8, (n,), dtype=torch.int32, device="cuda", generator=g)
    ref = _scan_with_scratch(lib, x, n, stream)
    out = torch.full((n + 1,), -1, dtype=torch.int32, device="cuda")
    assert lib.dfx_scan_exclusive_i32_static(x.data_ptr(), out.data_ptr(), n, stream) == 0, lib.dfx_last_error()
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
    assert int(out[-1].item()) == int(x.sum(dtype=torch.int64).item())
    del x, out, ref
    torch.cuda.empty_cache()


def test_static_scan_rejects_sizes_beyond_its_limit():
    from diffractom_b200 import _lib
    lib = _lib.lib()
    limit = 65536 * 2048
    x = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = lib.dfx_scan_exclusive_i32_static(x.data_ptr(), x.data_ptr(), limit + 1, None)
    assert st == _lib.DFX_EINVAL
    assert b"beyond" in lib.dfx_last_error()
