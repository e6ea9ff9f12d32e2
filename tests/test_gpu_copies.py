"""The pipelined pinned copies between pageable NumPy arrays and device tensors (streaming.HostCopier) used by the
solvers' NumPy paths: exact round trips at sizes around the chunk size, other dtypes, non-current streams and
concurrent callers."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("n", [1, 1000, (64 << 20) // 4, (64 << 20) // 4 + 3, 5 * ((64 << 20) // 4) + 17])
def test_round_trip_is_exact(n):
    from diffractom_b200.streaming import host_copier
    rng = np.random.default_rng(n)
    a = rng.standard_normal(n).astype(np.float32)
    d = torch.empty(n, dtype=torch.float32, device="cuda")
    s = torch.cuda.Stream()
    host_copier().to_device(a, d, s)
    s.synchronize()
    assert torch.equal(d.cpu(), torch.from_numpy(a))
    with torch.cuda.stream(s):
        d.mul_(2)
    out = np.empty_like(a)
    host_copier().to_host(d, out, s)
    assert np.array_equal(out, 2 * a)


def test_other_dtypes_and_concurrent_callers():
    from diffractom_b200.streaming import host_copier
    errs = []

    def work(seed):
        try:
            rng = np.random.default_rng(seed)
            a = rng.integers(-2 ** 31, 2 ** 31 - 1, 3 * (1 << 22) + seed, dtype=np.int64).astype(np.int32)
            d = torch.empty(a.size, dtype=torch.int32, device="cuda")
            host_copier().to_device(a, d)
            torch.cuda.current_stream().synchronize()
            out = np.empty_like(a)
            host_copier().to_host(d, out)
            assert np.array_equal(out, a)
        except BaseException as e:          # noqa: BLE001 - reported below
            errs.append(e)

    th = [threading.Thread(target=work, args=(i,)) for i in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    if errs:
        raise errs[0]
