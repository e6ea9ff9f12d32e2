"""PF- and projector-parameter gradients on the GPU (PFGradient, ProjGradient) against the reference model's values
in the golden fixtures (1e-4 of the largest, as the reference's tests/test_differentiable.py:66-108), the Gauss-Newton
blocks against the float64 oracle, the parameter updates (set_pf_parameters, set_proj_parameters, set_geometry)
against the reference model's forward at the moved parameters (2e-5 of the largest), and the local basis's gradients
against the global operator's."""
import numpy as np
import pytest

from conftest import case_inputs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

GROUPS = ("rot", "sigma", "eta_offset", "axis_tilt", "two_theta")


def _op(d, **kw):
    from diffractom_b200 import SinglePhaseForwardOperator
    cfg, mat, grid = case_inputs(d)
    kw.setdefault("max_gb", 1e-5)
    kw.setdefault("pf_mode", "sparse")
    return SinglePhaseForwardOperator(cfg, mat, grid, normalized=True, quadrature=d["quadrature"],
                                      radon_kernel=d["kernel"], **kw)


def _close(a, b, rel):
    a, b = np.atleast_1d(np.asarray(a, np.float64)), np.atleast_1d(np.asarray(b, np.float64))
    return np.abs(a - b).max() <= rel * np.abs(b).max()


@pytest.mark.parametrize("name,pf_mode", [("diff_auto_trapezoid", "sparse"), ("diff_auto_trapezoid", "generated"),
                                          ("diff_midpoint_hat", "sparse"), ("ti8_small", "generated"),
                                          ("al5_small", "sparse")])
def test_pf_gradients_equal_reference(golden, name, pf_mode):
    """Against the reference model's float64 values: 1e-4 of the largest on the reference's own test geometry (the
    diff cases); 3e-4 on the others, where the operator's float32 probed directions and poles alone move the
    float64 gradient of the eta offset or the widths by up to 1.6e-4 (narrower kernels, more rings). Against the
    oracle on that float32 geometry (the operator's PF): 1e-4 of the largest everywhere."""
    from diffractom_b200.differentiable import PFGradient
    from oracle.gradients import GradientModel
    d = golden(name)
    op = _op(d, pf_mode=pf_mode)
    pg = PFGradient(op)
    g = pg(d["c"], d["r"], groups=GROUPS)
    tol = 1e-4 if name.startswith("diff") else 3e-4
    ref32 = GradientModel(d, f32_geometry=True).pf_grads(d["c"], d["r"])
    for key in GROUPS:
        assert _close(g[key], d["g_" + key], tol), key
        assert _close(g[key], ref32[key], 1e-4), key
    g2 = pg(torch.as_tensor(d["c"], device="cuda"), torch.as_tensor(d["r"], device="cuda"), groups=("rot", "sigma"))
    assert np.array_equal(g2["rot"], g["rot"]) and np.array_equal(g2["sigma"], g["sigma"])   # reproducible


def test_hessian_blocks_equal_oracle(golden):
    from diffractom_b200.differentiable import PFGradient
    from oracle.gradients import GradientModel
    d = golden("diff_auto_trapezoid")
    op = _op(d)
    curv = (np.random.default_rng(4).random(op.data_shape) + 0.5).astype(np.float32)
    g = PFGradient(op, hessian=True)(d["c"], d["r"], groups=GROUPS, curv=curv)
    ref = GradientModel(d).pf_grads(d["c"], d["r"], curv=curv)
    assert _close(g["hess"], ref["hess"], 1e-4)
    for key in GROUPS:                           # the extra accumulators leave the gradients as they were
        assert _close(g[key], d["g_" + key], 1e-4), key


@pytest.mark.parametrize("name", ["diff_auto_trapezoid", "diff_midpoint_hat", "ti8_small"])
def test_projector_gradients_equal_reference(golden, name):
    from diffractom_b200.differentiable import ProjGradient
    d = golden(name)
    op = _op(d)
    g = ProjGradient(op)(d["c"], d["r"])
    assert _close(g["shift"], d["g_shift"], 1e-4)
    assert abs(g["cor"] - float(d["g_cor"])) <= 1e-4 * abs(float(d["g_cor"]))


@pytest.mark.parametrize("name,pf_mode", [("diff_auto_trapezoid", "sparse"), ("ti8_small", "generated")])
def test_set_pf_parameters_moves_to_reference(golden, name, pf_mode):
    from diffractom_b200.differentiable import PFGradient, rotate_orientations, set_pf_parameters
    d = golden(name)
    op = _op(d, pf_mode=pf_mode)
    pg = PFGradient(op)
    pg(d["c"], d["r"])
    set_pf_parameters(op, rotations=rotate_orientations(op.grid_rot_cpu, d["moved_rot"]), sigma=d["moved_sigma"],
                      two_theta=d["moved_two_theta"], eta_offset=0.01, axis_tilt=np.array([0.01, -0.02]))
    want = d["fwd_pf_moved"]
    assert np.abs(op.direct(d["c"]) - want).max() < 2e-5 * np.abs(want).max()
    g = pg(d["c"], d["r"])                       # the gradient object follows the rebuilt operator
    assert np.all(np.isfinite(g["rot"])) and g["rot"].shape == (op.K, 3)
    op.set_omega_subsets(4)                      # subsets are made again on the new PF matrix
    full = op.direct(d["c"])
    part = torch.zeros(op.data_shape, device="cuda")
    op.direct_cl(torch.as_tensor(d["c"], device="cuda"), part, subset=1)
    rows = op.omega_subsets[1]
    assert np.array_equal(part.cpu().numpy()[rows], full[rows])


def test_set_proj_parameters_moves_to_reference(golden):
    from diffractom_b200.differentiable import set_proj_parameters
    d = golden("diff_auto_trapezoid")
    op = _op(d)
    set_proj_parameters(op, cor=float(d["moved_cor"]), shift=d["moved_shift"])
    want = d["fwd_proj_moved"]
    got = op.direct(d["c"])
    assert np.abs(got - want).max() < 2e-5 * np.abs(want).max()
    rng = np.random.default_rng(6)                # the adjoint follows the new geometry
    x = rng.random(op.coeff_shape).astype(np.float32)
    y = rng.random(op.data_shape).astype(np.float32)
    lhs = float(np.sum(op.direct(x).astype(np.float64) * y))
    rhs = float(np.sum(x.astype(np.float64) * op.adjoint(y)))
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


def test_set_geometry_is_absolute(golden):
    from diffractom_b200.differentiable import rotate_orientations, set_geometry, set_pf_parameters
    d = golden("diff_auto_trapezoid")
    op = _op(d, pf_mode="generated")
    tt = np.asarray(op.two_theta_peaks, np.float64)
    set_geometry(op, eta_offset=-0.02, axis_tilt=[0.03, 0.0], two_theta=tt - 0.004, cor=0.0,
                 shift=np.zeros(op.N_Omega))
    set_geometry(op, eta_offset=0.01, axis_tilt=[0.01, -0.02], two_theta=d["moved_two_theta"],
                 cor=float(d["cfg"]["cor_offset"]), shift=np.zeros(op.N_Omega))
    set_pf_parameters(op, rotations=rotate_orientations(op.grid_rot_cpu, d["moved_rot"]), sigma=d["moved_sigma"])
    want = d["fwd_pf_moved"]
    assert np.abs(op.direct(d["c"]) - want).max() < 2e-5 * np.abs(want).max()


def test_local_basis_gradients_equal_global(golden):
    """PFGradient (with the Gauss-Newton blocks) and ProjGradient on the local operator equal the global operator's on
    the zero-extended coefficients (the local operator's orientations are the global ones at orientation_index),
    also after set_pf_parameters."""
    from diffractom_b200.differentiable import PFGradient, ProjGradient, rotate_orientations, set_pf_parameters
    from diffractom_b200.local import LocalSinglePhaseForwardOperator, LocalSupport
    d = golden("diff_auto_trapezoid")
    cfg, mat, grid = case_inputs(d)
    gop = _op(d)
    rng = np.random.default_rng(3)
    mask = np.zeros((gop.K, gop.Ny, gop.Nx), bool)
    for k in range(gop.K):
        for _ in range(1 + k % 2):
            cy, cx = rng.integers(2, gop.Ny - 2), rng.integers(2, gop.Nx - 2)
            mask[k, max(cy - 2, 0):cy + 2, max(cx - 2, 0):cx + 3] = True
    lop = LocalSinglePhaseForwardOperator(cfg, mat, grid, 1e-5, LocalSupport.from_mask(mask), normalized=True,
                                          quadrature=d["quadrature"], radon_kernel=d["kernel"])
    x = (rng.random(lop.n_coef) * lop.coefficient_mask()).astype(np.float32)
    xd = lop.to_dense(x)
    r = rng.normal(size=lop.data_shape).astype(np.float32)
    oi = lop.orientation_index
    for step in range(2):
        gl = PFGradient(lop, hessian=True)(x, r, groups=("rot", "sigma"))
        gg = PFGradient(gop, hessian=True)(xd, r, groups=("rot", "sigma"))
        for key in ("rot", "sigma", "hess"):
            assert _close(gl[key], gg[key][oi], 1e-4), (step, key)
        inc = 0.003 * rng.normal(size=(lop.K, 3))
        set_pf_parameters(lop, rotations=rotate_orientations(lop.grid_rot_cpu, inc))
        rg = np.asarray(gop.grid_rot_cpu, np.float64).copy()
        rg[oi] = rotate_orientations(rg[oi], inc)
        set_pf_parameters(gop, rotations=rg)
        d1, d2 = lop.direct(x), gop.direct(xd)
        assert np.abs(d1 - d2).max() < 1e-5 * np.abs(d2).max()
    pl, pgl = ProjGradient(lop)(x, r), ProjGradient(gop)(xd, r)
    assert _close(pl["shift"], pgl["shift"], 1e-5)
