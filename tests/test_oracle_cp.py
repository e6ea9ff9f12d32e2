"""The oracle's float64 primal-dual solver (chambolle_pock_poisson_tv, the reference optimum of the tree-TV GPU test)
pinned on small problems against SciPy's L-BFGS-B on the same objective: without TV exactly, with TV through a
smoothed norm sqrt(g^2 + eps^2) that differs from |g| by at most eps per term. CPU only."""
import numpy as np
import pytest

scipy = pytest.importorskip("scipy")


def _problem(seed=0, m=40, n=10, gain=0.5):
    rng = np.random.default_rng(seed)
    A = rng.random((m, n)) * (rng.random((m, n)) < 0.6)
    x_true = rng.random(n) * 2
    b = rng.poisson(A @ x_true / gain) * gain
    rows = []
    for j in range(n - 1):                       # one difference per term, paired with a zero row (2 rows a term)
        r = np.zeros(n)
        r[j], r[j + 1] = -1.0, 1.0
        rows += [r, np.zeros(n)]
    return A, np.array(rows), b.astype(np.float64), gain


def _lbfgs(A, D, b, gain, tv, eps=1e-3, smooth=1e-7):
    from scipy.optimize import minimize
    r = eps * gain

    def f(x):
        mu = A @ x + r
        g = (D @ x).reshape(-1, 2)
        nrm = np.sqrt((g ** 2).sum(axis=1) + smooth ** 2)
        val = np.sum((mu - b + np.where(b > 0, b * np.log(np.where(b > 0, b, 1.0) / mu), 0.0)) / gain) + tv * nrm.sum()
        grad = A.T @ ((1.0 - b / mu) / gain) + tv * D.T @ (g / nrm[:, None]).ravel()
        return val, grad
    res = minimize(f, np.full(A.shape[1], 0.5), jac=True, method="L-BFGS-B", bounds=[(0, None)] * A.shape[1],
                   options=dict(maxiter=20000, ftol=1e-15, gtol=1e-12))
    return res.x


@pytest.mark.parametrize("tv", [0.0, 0.3, 2.0])
def test_primal_dual_reaches_the_lbfgs_optimum(tv):
    from oracle.oracle import chambolle_pock_poisson_tv, poisson_tv_objective
    A, D, b, gain = _problem()
    free = np.ones(A.shape[1], bool)
    x_cp = chambolle_pock_poisson_tv(A, D, b, gain, tv, free, n_iter=40000)
    x_lb = _lbfgs(A, D, b, gain, tv)
    f_cp = poisson_tv_objective(A, D, x_cp, b, gain, tv)
    f_lb = poisson_tv_objective(A, D, x_lb, b, gain, tv)
    n_terms = D.shape[0] // 2
    assert f_cp <= f_lb + 1e-7 * abs(f_lb) + tv * n_terms * 1e-7, (f_cp, f_lb)
    assert f_lb <= f_cp * (1 + 1e-6), (f_cp, f_lb)
    assert np.all(x_cp >= 0)


def test_coefficients_that_are_not_free_stay_zero():
    from oracle.oracle import chambolle_pock_poisson_tv
    A, D, b, gain = _problem(seed=1)
    free = np.ones(A.shape[1], bool)
    free[[2, 7]] = False
    x = chambolle_pock_poisson_tv(A, D, b, gain, 0.3, free, n_iter=2000)
    assert np.all(x[~free] == 0) and np.all(x >= 0)
