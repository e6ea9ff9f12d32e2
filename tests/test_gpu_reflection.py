"""reflection_two_theta on the GPU: the operator against the reference model's float64 forward and transpose for
windows of reflections at different Bragg angles (the reference's tests/test_reflection_two_theta.py geometry), a
window equals the share-weighted sum of its reflections each taken as a one-reflection channel, the stored and the
generated PF give the same bits, the adjoint identity, and a change of two_theta moves the axes with their channel."""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _op(d, rings=None, refl=True, pf_mode="sparse"):
    from diffractom_b200 import SinglePhaseForwardOperator
    from diffractom_b200.grid import MatrixGrid
    from diffractom_b200.material import Material
    mat = Material.from_lattice_parameters(**d["material"])
    rings = [(ix, w) for ix, w in json.loads(str(d["rings"]))] if rings is None else rings
    return SinglePhaseForwardOperator(d["cfg"], mat, MatrixGrid(d["rot"], d["sigma64"]), 1e-4, normalized=True,
                                      quadrature=d["quadrature"], radon_kernel=d["kernel"], pf_mode=pf_mode,
                                      rings=rings, reflection_two_theta=refl)


def test_forward_and_adjoint_equal_reference(golden):
    d = golden("refl_windows")
    op = _op(d)
    fwd = op.direct(d["c"])
    assert np.abs(fwd - d["fwd"]).max() < 3e-5 * np.abs(d["fwd"]).max()
    adj = op.adjoint(d["r"])
    assert np.abs(adj - d["adj"]).max() < 3e-5 * np.abs(d["adj"]).max()


def test_window_is_the_sum_of_its_reflections(golden):
    d = golden("refl_windows")
    windows = [(ix, w) for ix, w in json.loads(str(d["rings"]))]
    op = _op(d)
    c = d["c"]
    dd = op.direct(c).reshape(op.N_Omega, op.My, op.N_eta, op.N_peaks)
    used = [f for ix, _ in windows for f in ix]
    one = _op(d, rings=[([f], [1.0]) for f in used], refl=False)
    d1 = one.direct(c).reshape(op.N_Omega, op.My, op.N_eta, len(used))
    m = np.asarray(op.material.reflections["multiplicity"], np.float64)
    pos = 0
    for p, (ix, w) in enumerate(windows):
        share = m[ix] * np.asarray(w)
        share = share / share.sum()
        want = sum(s * d1[..., pos + i] for i, s in enumerate(share))
        pos += len(ix)
        assert np.abs(dd[..., p] - want).max() <= 3e-5 * np.abs(want).max(), p
    mean = _op(d, refl=False).direct(c).reshape(dd.shape)      # the channel's mean angle is another model
    assert np.abs(mean[..., 0] - dd[..., 0]).max() > 0.02 * np.abs(dd[..., 0]).max()


def test_modes_agree_adjoint_and_two_theta_update(golden):
    from diffractom_b200.differentiable import set_pf_parameters
    d = golden("refl_windows")
    sp, gen = _op(d, pf_mode="sparse"), _op(d, pf_mode="generated")
    c = d["c"]
    a, b = sp.direct(c), gen.direct(c)
    assert np.array_equal(a, b)
    y = np.random.default_rng(3).normal(size=sp.data_shape).astype(np.float32)
    lhs = float(np.sum(a.astype(np.float64) * y))
    rhs = float(np.sum(sp.adjoint(y).astype(np.float64) * c))
    assert abs(lhs - rhs) <= 2e-5 * abs(lhs)
    # moving a channel's two_theta moves all of its axes by the same amount (the others stay)
    tt = np.asarray(sp.two_theta_peaks, np.float64)
    before = np.asarray(sp.axis_two_theta_cpu, np.float64).copy()
    set_pf_parameters(sp, two_theta=tt + np.array([0.002, 0.0, 0.0]))
    moved = np.asarray(sp.axis_two_theta_cpu, np.float64) - before
    s0, s1 = sp.axis_start_cpu[0], sp.axis_start_cpu[1]
    assert np.allclose(moved[s0:s1], 0.002, atol=2e-9) and np.allclose(moved[s1:], 0.0, atol=2e-9)
    assert not np.array_equal(sp.direct(c), a)


def test_pf_gradients_equal_reference(golden):
    """PFGradient with reflection_two_theta against the reference model's float64 gradients, also with the
    Gauss-Newton blocks: 3e-4 of the largest. The operator's probed directions u, w are float32: rounding them alone
    moves the model's float64 width gradient of this case (3 deg kernels) by 1.0e-4 of the largest."""
    from diffractom_b200.differentiable import PF_GROUPS, PFGradient
    d = golden("refl_windows")
    op = _op(d)
    for hess in (False, True):
        g = PFGradient(op, hessian=hess)(d["c"], d["r"], groups=PF_GROUPS)
        for key in PF_GROUPS:
            a, b = np.atleast_1d(g[key]), np.atleast_1d(d["g_" + key])
            assert np.abs(a - b).max() <= 3e-4 * np.abs(b).max(), (hess, key)
