"""The parameter-gradient oracle (oracle/gradients.py) against the reference's own float64 values in the golden
fixtures (ReferenceModel.vjp, probed_derivatives), and the package's host half of PFGradient (the probed
directions' derivatives, the tilt basis) against the same fixtures; CPU only."""
import numpy as np
import pytest

from conftest import case_geometry

CASES = ["diff_auto_trapezoid", "diff_midpoint_hat", "adj_0_90", "adj_180_0", "ti8_small", "al5_small"]


def _close(a, b, rel):
    a, b = np.atleast_1d(np.asarray(a, np.float64)), np.atleast_1d(np.asarray(b, np.float64))
    return np.abs(a - b).max() <= rel * max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("name", ["diff_auto_trapezoid", "ti8_small"])
def test_oracle_probed_derivatives_pinned(golden, name):
    from oracle.gradients import probed_derivatives
    d = golden(name)
    R, C = int(d["cfg"]["N_Omega"]), int(d["cfg"]["N_eta"])
    om, eta = d["angles_sub"].reshape(R, -1), d["eta_sub"].reshape(C, -1)
    dv = probed_derivatives(d["cfg"], om, eta, d["two_theta"])
    for key, fk in (("eta_offset", "dv_eta"), ("tilt0", "dv_tilt0"), ("tilt1", "dv_tilt1"), ("two_theta", "dv_tth")):
        assert dv[key].shape == d[fk].shape
        assert _close(dv[key], d[fk], 1e-6), key


@pytest.mark.parametrize("name", CASES)
def test_oracle_parameter_gradients_pinned(golden, name):
    """The float64 restatement reproduces the reference model's PF-parameter and detector-shift gradients."""
    from oracle.gradients import GradientModel
    d = golden(name)
    m = GradientModel(d)
    g = m.pf_grads(d["c"], d["r"])
    for key in ("rot", "sigma", "eta_offset", "axis_tilt", "two_theta"):
        assert _close(g[key], d["g_" + key], 1e-9), key
    sh = m.shift_grads(d["c"], d["r"], d["pf"])
    assert _close(sh["shift"], d["g_shift"], 1e-9)
    assert abs(sh["cor"] - float(d["g_cor"])) <= 1e-9 * abs(float(d["g_cor"]))


def test_oracle_hessian_blocks_are_gauss_newton():
    """The oracle's Gauss-Newton blocks: symmetric positive semi-definite, and the width-width entry of orientation k
    equals sum over the data of (d data / d sigma_k)^2 (curv = 1), the Jacobian column taken by central differences
    of the PF matrix in sigma_k."""
    from conftest import load_case
    from oracle.gradients import GradientModel
    d = load_case("diff_midpoint_hat")
    m = GradientModel(d)
    H = m.pf_grads(d["c"], d["r"])["hess"]
    assert np.allclose(H, H.transpose(0, 2, 1))
    assert np.all(np.linalg.eigvalsh(H) >= -1e-9 * np.abs(H).max())
    _, _, S = m.projections(d["c"])
    for k in (0, 5):
        h = 1e-6 * m.sigma[k]
        sp, sm = m.sigma.copy(), m.sigma.copy()
        sp[k] += h
        sm[k] -= h
        dpf = ((m.pf(sp) - m.pf(sm)) / (2 * h))[:, k].reshape(m.R, -1)       # (R, C P)
        J = dpf[:, None, :] * S[:, :, k][:, :, None]                         # (R, My, C P)
        assert abs(H[k, 3, 3] - np.sum(J * J)) <= 1e-5 * np.sum(J * J)


@pytest.mark.parametrize("name", ["diff_auto_trapezoid", "ti8_small"])
def test_package_probed_derivatives(golden, name):
    """diffractom_b200.differentiable.probed_derivatives (host, float64) of the package's own geometry equals the
    reference's to float32 rounding of the fixture."""
    from diffractom_b200.differentiable import perp_basis, probed_derivatives
    from oracle.gradients import perp_basis as perp_oracle
    d = golden(name)
    geom = case_geometry(d)
    dv = probed_derivatives(geom)
    for key, fk in (("eta_offset", "dv_eta"), (("axis_tilt", 0), "dv_tilt0"), (("axis_tilt", 1), "dv_tilt1"),
                    ("two_theta", "dv_tth")):
        assert _close(dv[key], d[fk], 2e-6), key
    for k in ([0, 0, 1], [1, 0, 0], [0.3, -0.2, 0.9]):
        for a, b in zip(perp_basis(k), perp_oracle(k)):
            assert np.array_equal(a, b)
