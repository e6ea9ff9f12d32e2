"""window_parallax on the GPU (the checks of the reference's tests/test_window_parallax.py): with windows that hold
everything the operator is the plain one bit for bit; otherwise every rotation angle equals a plain operator whose
reflection weights are that angle's window fractions, computed here in float64 (2e-5 of the largest); the local
operator's default positions are its support's centroids; PFGradient carries the fractions."""
import json

import numpy as np
import pytest
from scipy.special import erf

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _op(d, rings=None, pf_mode="sparse", **kw):
    from diffractom_b200 import SinglePhaseForwardOperator
    from diffractom_b200.grid import MatrixGrid
    from diffractom_b200.material import Material
    mat = Material.from_lattice_parameters(**d["material"])
    rings = [(ix, w) for ix, w in json.loads(str(d["rings"]))] if rings is None else rings
    return SinglePhaseForwardOperator(d["cfg"], mat, MatrixGrid(d["rot"], d["sigma64"]), 1e-4, normalized=True,
                                      quadrature=d["quadrature"], radon_kernel=d["kernel"], pf_mode=pf_mode,
                                      rings=rings, reflection_two_theta=True, **kw)


def _point(op, col, row):
    c = np.zeros(op.coeff_shape, np.float32)
    c[0, row, col] = 1.0
    c[3, row, col] = 0.5
    return c


@pytest.mark.parametrize("pf_mode", ["sparse", "generated"])
def test_wide_windows_are_the_plain_operator(golden, pf_mode):
    d = golden("refl_windows")
    P = len(json.loads(str(d["rings"])))
    plain = _op(d, pf_mode=pf_mode)
    wp = _op(d, pf_mode=pf_mode, window_parallax=dict(windows=[[0.0, np.pi]] * P, sigma=1e-3, distance=1e12))
    c = _point(plain, 5, 7)
    assert np.array_equal(plain.direct(c), wp.direct(c))


@pytest.mark.parametrize("pf_mode,lorentz", [("sparse", 0.0), ("generated", 0.0), ("sparse", 0.5)])
def test_every_angle_is_a_plain_operator_with_its_window_fractions(golden, pf_mode, lorentz):
    from diffractom_b200.geometry import image_direction
    d = golden("refl_windows")
    windows = [(ix, w) for ix, w in json.loads(str(d["rings"]))]
    plain = _op(d)
    mat = plain.material
    m = np.asarray(mat.reflections["multiplicity"], np.float64)
    h = np.asarray(mat.h_vecs, np.float64)
    lam = 12.398 / float(d["cfg"]["energy"])
    tth_f = 2 * np.arcsin(np.linalg.norm(h, axis=1) / (4 * np.pi) * lam)
    win = np.array([[tth_f[ix].min() - np.radians(0.15), tth_f[ix].max() + np.radians(0.05)] for ix, _ in windows])
    sig, D, gam = np.radians(0.1), 40.0, np.radians(0.07)
    col, row = 3, 9
    K = plain.K
    pos = np.tile([[col, row]], (K, 1)).astype(np.float64)
    ones = [(ix, [1.0] * len(ix)) for ix, _ in windows]
    wp = _op(d, rings=ones, pf_mode=pf_mode, window_parallax=dict(windows=win, sigma=sig, distance=D, positions=pos,
                                                                  covariances=np.zeros((K, 3)), lorentz=lorentz,
                                                                  gamma=gam))
    c = _point(plain, col, row)
    got = wp.direct(c).reshape(plain.N_Omega, plain.My, plain.N_eta, plain.N_peaks)
    px = plain.image_width / max(plain.Nx, plain.Ny)
    rel = (np.array([col, row]) - [(plain.Nx - 1) / 2, (plain.Ny - 1) / 2]) * px
    b = image_direction(np.asarray(d["cfg"]["p_direction_0"], np.float64)[:2], np.asarray(plain.angles))
    worst = 0.0
    for r in range(plain.N_Omega):
        x = rel @ b[r]
        rings_r, corr = [], []
        for p, (ix, _) in enumerate(windows):
            t = tth_f[ix]
            sh = t - (x / D) * np.sin(t) * np.cos(t)
            fr = 0.5 * (erf((win[p, 1] - sh) / (np.sqrt(2) * sig)) - erf((win[p, 0] - sh) / (np.sqrt(2) * sig)))
            fr = (1 - lorentz) * fr + lorentz * (np.arctan((win[p, 1] - sh) / gam)
                                                 - np.arctan((win[p, 0] - sh) / gam)) / np.pi
            fr = np.maximum(fr, 1e-12)
            rings_r.append((list(ix), fr.tolist()))
            corr.append((m[ix] * fr).sum() / m[ix].sum())
        ref = _op(d, rings=rings_r).direct(c).reshape(got.shape)[r] * np.asarray(corr)[None, None, :]
        worst = max(worst, np.abs(got[r] - ref).max() / max(np.abs(ref).max(), 1e-12))
    assert worst < 2e-5, worst


def test_local_default_positions_and_gradient(golden):
    from diffractom_b200.differentiable import PFGradient
    from diffractom_b200.grid import MatrixGrid
    from diffractom_b200.local import LocalSinglePhaseForwardOperator, LocalSupport, spatial_moments
    from diffractom_b200.material import Material
    d = golden("refl_windows")
    windows = [(ix, w) for ix, w in json.loads(str(d["rings"]))]
    K = len(d["rot"])
    rng = np.random.default_rng(3)
    k = np.repeat(np.arange(K), 6)
    iy, ix = rng.integers(2, 10, len(k)), rng.integers(2, 12, len(k))
    key = np.unique(np.stack([k, iy, ix], 1), axis=0)
    sup = LocalSupport(key[:, 0], key[:, 1], key[:, 2], K, (d["cfg"]["Ny"], d["cfg"]["Nx"]))
    win = [[0.0, np.pi]] * len(windows)
    kw = dict(normalized=True, rings=windows, reflection_two_theta=True, pf_mode="sparse", restrict_to_fov=False)
    mat = Material.from_lattice_parameters(**d["material"])
    grid = MatrixGrid(d["rot"], d["sigma64"])
    op_d = LocalSinglePhaseForwardOperator(d["cfg"], mat, grid, 1e-4, sup, window_parallax=dict(
        windows=win, sigma=0.01, distance=30.0), **kw)
    pos, cov = spatial_moments(sup.k, sup.iy, sup.ix, None, K)
    op_e = LocalSinglePhaseForwardOperator(d["cfg"], mat, grid, 1e-4, sup, window_parallax=dict(
        windows=win, sigma=0.01, distance=30.0, positions=pos, covariances=cov), **kw)
    x = rng.random(op_d.n_coef).astype(np.float32)
    assert np.array_equal(op_d.direct(x), op_e.direct(x))
    # the gradient with wide windows is the plain one bit for bit; cutting windows change it
    plain = _op(d)
    wide = _op(d, window_parallax=dict(windows=[[0.0, np.pi]] * len(windows), sigma=1e-3, distance=1e12))
    c, r = d["c"], d["r"]
    g0, g1 = PFGradient(plain)(c, r, groups=("rot", "sigma")), PFGradient(wide)(c, r, groups=("rot", "sigma"))
    assert np.array_equal(g0["rot"], g1["rot"]) and np.array_equal(g0["sigma"], g1["sigma"])
