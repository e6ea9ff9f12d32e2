"""The parallel random start of estimate_L_power_streamed: column ix of the (K, Ny, Nx) start is the transposed
(Ny, K) standard-normal draw of default_rng([seed, ix]) (streaming.py:363-372); CPU only."""
import numpy as np


def test_parallel_random_start_columns():
    from diffractom_b200.operator import parallel_random_start
    K, Ny, Nx = 5, 4, 7
    x3 = parallel_random_start(K, Ny, Nx, 3, threads=3)
    for ix in (0, 4, 6):
        want = np.random.default_rng([3, ix]).standard_normal((Ny, K)).astype(np.float32).T
        assert np.array_equal(x3[:, :, ix], want)
    assert not np.array_equal(parallel_random_start(K, Ny, Nx, 4), x3)
