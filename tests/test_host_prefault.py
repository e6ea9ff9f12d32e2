"""HostCopier.prefault (mapping the pages of a run's host outputs while the device iterates): keep=True leaves the
contents as they were, keep=False writes zeros at the touched bytes only, at sizes around the chunk size. CPU only:
the copier is built without its pinned chunks, which the page touching does not use."""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

pytest.importorskip("torch")


def _copier():
    from diffractom_b200.streaming import HostCopier
    hc = HostCopier.__new__(HostCopier)
    hc.pool = ThreadPoolExecutor(4)
    return hc


@pytest.mark.parametrize("n", [1, 1023, 1024, (64 << 20) // 4 + 5, 3 * ((64 << 20) // 4) - 7])
def test_prefault_keeps_or_zeroes(n):
    hc = _copier()
    rng = np.random.default_rng(n)
    a = rng.standard_normal(n).astype(np.float32)
    want = a.copy()
    for f in hc.prefault(a, True):
        f.result()
    assert np.array_equal(a, want)
    b = np.full(n, 7.0, np.float32)
    for f in hc.prefault(b, False):
        f.result()
    v = b.view(np.uint8)
    touched = np.zeros(v.size, bool)
    for o in range(0, v.size, 64 << 20):
        touched[o:o + (64 << 20):4096] = True
    assert np.all(v[touched] == 0)
    assert np.array_equal(v[~touched], np.full(n, 7.0, np.float32).view(np.uint8)[~touched])
    hc.pool.shutdown()


def test_prefault_rejects_read_only_arrays_at_once():
    hc = _copier()
    a = np.zeros(1000, np.float32)
    a.setflags(write=False)
    with pytest.raises(ValueError, match="read-only"):
        hc.prefault(a, True)
    hc.pool.shutdown()


def test_read_only_x0_is_copied_for_the_solvers():
    """A solver writes its result into a NumPy x0; a read-only one is replaced by a writeable copy at set-up, so
    nothing fails after the iterations have run."""
    from diffractom_b200.arrays import as_host
    a = np.arange(12, dtype=np.float32).reshape(3, 4)
    assert as_host(a, (3, 4), "x0", writeable=True) is a
    a.setflags(write=False)
    assert as_host(a, (3, 4), "x0") is a
    c = as_host(a, (3, 4), "x0", writeable=True)
    assert c is not a and c.flags.writeable and np.array_equal(c, a)
