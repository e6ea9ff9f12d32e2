"""The Fourier-slice projector on the GPU (dfx_fr_forward / dfx_fr_backward: pad, cuFFT, slices, lines; lines,
cuFFT, spread, cuFFT, crop) against the exact Fourier-slice projection of the oracle, on channel-fastest batches with
padding channels and several channel slices; a subset's projector gives its angles' rows; forward and backward are
transposes; the operator with projector="fft" against the oracle's operator; precision "bf16" with it (the BF16
contraction of the float32 transforms' output) against the float32 operator, with T streamed."""
import numpy as np
import pytest

from oracle import fourier as orc

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _projector(Nx, Ny, Ns, R, shift, width):
    from diffractom_b200.fourier import FourierHost, FourierProjector
    ang = np.linspace(0, np.pi, R, endpoint=False) + 0.021
    h = FourierHost(ang, Nx, Ny, Ns, width, float(Ns), shift, np.pi / R)
    M, scale, _ = orc.fourier_slice_matrix(ang, Nx, Ny, Ns, width, float(Ns), shift)
    return FourierProjector(h, torch.device("cuda")), M, scale


@pytest.mark.parametrize("Nx, Ny, Ns, R, kb, kstride, channels", [
    (22, 18, 30, 11, 5, 16, 64), (37, 41, 58, 23, 70, 80, 32), (16, 16, 17, 7, 1, 16, 1)])
def test_fourier_projector_matches_exact_projection(Nx, Ny, Ns, R, kb, kstride, channels):
    fp, M, scale = _projector(Nx, Ny, Ns, R, 0.35, float(Nx))
    rng = np.random.default_rng(kb)
    npix = Nx * Ny
    img = np.zeros((npix, kstride), np.float32)
    img[:, :kb] = rng.random((npix, kb))
    s = torch.cuda.current_stream().cuda_stream
    nb = fp.scratch_bytes(channels)
    scr = torch.empty(nb, dtype=torch.uint8, device="cuda")
    img_d = torch.as_tensor(img, device="cuda")
    sino = torch.full((R, Ns, kstride), 7.0, device="cuda")
    fp.forward(img_d.data_ptr(), sino.data_ptr(), kstride, kb, channels, scr.data_ptr(), nb, s)
    ref = orc.forward(M, scale, img[:, :kb])
    out = sino.cpu().numpy()
    assert np.abs(out[..., :kb] - ref).max() <= 1e-4 * np.abs(ref).max()
    assert not out[..., kb:].any()
    y = np.zeros((R, Ns, kstride), np.float32)
    y[..., :kb] = rng.standard_normal((R, Ns, kb))
    back = torch.full((npix, kstride), 3.0, device="cuda")
    fp.backward(torch.as_tensor(y, device="cuda").data_ptr(), back.data_ptr(), kstride, kb, channels, scr.data_ptr(),
                nb, s)
    refb = orc.backward(M, np.pi / R, y[..., :kb])
    outb = back.cpu().numpy()
    assert np.abs(outb[:, :kb] - refb).max() <= 1e-4 * np.abs(refb).max()
    assert not outb[:, kb:].any()
    # transposes: <A x, y> = <x, A^T y> / (scale w) with one angle weight
    lhs = float((out[..., :kb].astype(np.float64) * y[..., :kb]).sum())
    rhs = float((img[:, :kb].astype(np.float64) * outb[:, :kb]).sum()) * scale / (np.pi / R)
    assert abs(lhs - rhs) <= 1e-4 * abs(lhs)


def test_subset_projector_gives_its_rows_and_scratch_is_checked():
    fp, M, scale = _projector(30, 26, 40, 17, -0.2, 30.0)
    idx = np.arange(3, 17, 4)
    sub = fp.subset(idx)
    rng = np.random.default_rng(5)
    kstride, kb = 32, 29
    img = torch.as_tensor(rng.random((30 * 26, kstride)).astype(np.float32), device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    nb = fp.scratch_bytes(32)
    scr = torch.empty(nb, dtype=torch.uint8, device="cuda")
    full = torch.empty((17, 40, kstride), device="cuda")
    part = torch.empty((len(idx), 40, kstride), device="cuda")
    fp.forward(img.data_ptr(), full.data_ptr(), kstride, kb, 32, scr.data_ptr(), nb, s)
    nbs = sub.scratch_bytes(32)
    scr2 = torch.empty(nbs, dtype=torch.uint8, device="cuda")
    sub.forward(img.data_ptr(), part.data_ptr(), kstride, kb, 32, scr2.data_ptr(), nbs, s)
    assert torch.equal(part, full[torch.as_tensor(idx, device="cuda")])
    with pytest.raises(ValueError):
        fp.forward(img.data_ptr(), full.data_ptr(), kstride, kb, 32, scr.data_ptr(), 4096, s)


def _fft_operator_and_reference(golden, name):
    """The operator with projector "fft" and the oracle's composition of the same PF matrix with the exact
    Fourier-slice projection (forward: PF (scale M x); adjoint: backward projection of (R/pi) PF^T y)."""
    from conftest import case_inputs
    from diffractom_b200 import SinglePhaseForwardOperator
    from oracle.oracle import OracleOperator
    d = golden(name)
    cfg, mat, grid = case_inputs(d)
    op = SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"],
                                    projector="fft")
    assert op.projector == "fft" and op.radon_kernel == "hat" and len(op.batches) > 1
    orc = OracleOperator.from_operator(op)
    pf = orc.pf_dense(0, op.K).astype(np.float64).reshape(op.N_Omega, op.K, -1)         # (R, K, CP)
    M, scale, L = orc_f.fourier_slice_matrix(op.angles, op.Nx, op.Ny, op.My, op.image_width, op.My,
                                             op.detector_shifts())
    assert L == op._fft.L

    def fwd(x):                                                  # x (K, Ny, Nx)
        sino = orc_f.forward(M, scale, x.reshape(op.K, -1).T)   # (R, My, K)
        return np.einsum("ryk,rkj->ryj", sino, pf)

    def adj(y):                                                  # y (R, My, CP)
        z = (op.N_Omega / np.pi) * np.einsum("ryj,rkj->ryk", y, pf)
        return orc_f.backward(M, op.angle_weight, z).T.reshape(op.K, op.Ny, op.Nx)
    return op, fwd, adj


orc_f = orc


@pytest.mark.parametrize("name", ["al5_small", "adj_0_360"])
def test_operator_with_fourier_projector_matches_oracle(golden, name):
    op, fwd, adj = _fft_operator_and_reference(golden, name)
    rng = np.random.default_rng(2)
    x = rng.random(op.coeff_shape).astype(np.float32)
    y = rng.random(op.data_shape).astype(np.float32)
    ax = op.direct(torch.as_tensor(x, device="cuda")).cpu().numpy()
    aty = op.adjoint(torch.as_tensor(y, device="cuda")).cpu().numpy()
    rf, ra = fwd(x), adj(y)
    assert np.abs(ax - rf).max() <= 1e-4 * np.abs(rf).max()
    assert np.abs(aty - ra).max() <= 1e-4 * np.abs(ra).max()
    # the subset form gives the subset's rows (the same bits as the full forward's rows need not hold: the subset's
    # projector has its own polar samples; to the NUFFT's accuracy)
    op.set_omega_subsets(3)
    d = torch.zeros(op.data_shape, device="cuda")
    op.direct_cl(torch.as_tensor(x, device="cuda"), d, subset=1)
    rows = op.omega_subsets[1]
    assert np.abs(d.cpu().numpy()[rows] - rf[rows]).max() <= 1e-4 * np.abs(rf).max()
    assert not d.cpu().numpy()[np.setdiff1d(np.arange(op.N_Omega), rows)].any()


def test_spdhg_with_fourier_projector_runs(golden):
    """SPDHG with projector "fft" (backprojection, then the primal step as its own kernel): the deviance falls, the
    iterates stay non-negative and inside the support."""
    from diffractom_b200 import SPDHGPoisson
    op, fwd, adj = _fft_operator_and_reference(golden, "al5_small")
    rng = np.random.default_rng(9)
    x_true = (rng.random(op.coeff_shape) * (rng.random(op.coeff_shape) < 0.2) * op.support_mask()[None]
              ).astype(np.float32)
    b = rng.poisson(np.maximum(fwd(x_true), 0) * 50).astype(np.float32)
    sp = SPDHGPoisson(op, subsets=3, seed=1)
    x = sp.run(torch.zeros(op.coeff_shape, device="cuda"), b, 4, diagnostics_interval=2).cpu().numpy()
    f = [s["f"] for s in sp.iter_stats if s["f"] is not None]
    assert len(f) == 2 and np.isfinite(f).all() and f[1] < f[0]
    assert np.all(x[:, ~op.support_mask()] == 0) and x.min() >= 0


def test_bf16_contraction_with_fourier_projector(golden):
    """precision "bf16" with projector "fft": the Fourier-slice transforms run in float32 and their output is
    rounded to BF16 once for the tensor-core PF products (PF stored or generated per subset). Forward, adjoint and a
    subset's rows within 1e-2 of the float32 operator's; SPDHG with T streamed (x and z resident, host arrays
    through the staging buffers) gives the resident run's iterates, deviances and state bit for bit, and its
    deviances stay within 1e-3 of the float32 run's; with T stored in BF16 (steps rounded toward zero) within 5e-3."""
    from conftest import case_inputs
    from diffractom_b200 import SinglePhaseForwardOperator, SPDHGPoisson
    d = golden("al5_small")
    cfg, mat, grid = case_inputs(d)
    mk = lambda **kw: SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"],
                                                 projector="fft", **kw)
    op32 = mk()
    rng = np.random.default_rng(4)
    x = rng.random(op32.coeff_shape).astype(np.float32)
    y = rng.random(op32.data_shape).astype(np.float32)
    xt, yt = torch.as_tensor(x, device="cuda"), torch.as_tensor(y, device="cuda")
    f32, a32 = op32.direct(xt).cpu().numpy(), op32.adjoint(yt).cpu().numpy()
    op32.set_omega_subsets(3)
    s32 = torch.zeros(op32.data_shape, device="cuda")
    op32.direct_cl(xt, s32, subset=2)
    for bf16_pf in ("stored", "generated"):
        op = mk(precision="bf16", bf16_pf=bf16_pf)
        assert op.projector == "fft" and op.precision == "bf16" and not op.tc_forward
        assert np.abs(op.direct(xt).cpu().numpy() - f32).max() <= 1e-2 * np.abs(f32).max()
        assert np.abs(op.adjoint(yt).cpu().numpy() - a32).max() <= 1e-2 * np.abs(a32).max()
        op.set_omega_subsets(3)
        s = torch.zeros(op.data_shape, device="cuda")
        op.direct_cl(xt, s, subset=2)
        rows = op.omega_subsets[2]
        assert np.abs((s - s32).cpu().numpy()[rows]).max() <= 1e-2 * np.abs(f32).max()
        assert not s.cpu().numpy()[np.setdiff1d(np.arange(op.N_Omega), rows)].any()

    op = mk(precision="bf16")
    x_true = (rng.random(op.coeff_shape) * (rng.random(op.coeff_shape) < 0.2) * op.support_mask()[None]
              ).astype(np.float32)
    b = rng.poisson(np.maximum(op32.direct(torch.as_tensor(x_true, device="cuda")).cpu().numpy(), 0) * 50
                    ).astype(np.float32)
    runs = {}
    for key, o, resident in (("f32", op32, "all"), ("all", op, "all"), ("xz", op, ["x", "z"]), ("t16", op, "all")):
        sp = SPDHGPoisson(o, subsets=3, seed=1, resident=resident)
        sp.bf16_T = key == "t16"
        xr = sp.run(np.zeros(op.coeff_shape, np.float32), b, 4, diagnostics_interval=1)
        runs[key] = (xr, [st["f"] for st in sp.iter_stats], sp.state, sp.final_stats["resident"])
        assert sp.final_stats["T_bf16"] == (key == "t16")
    assert runs["xz"][3] == ("x", "z")
    assert np.array_equal(runs["xz"][0], runs["all"][0]) and runs["xz"][1] == runs["all"][1]
    assert np.array_equal(runs["xz"][2]["z"], runs["all"][2]["z"])
    assert np.array_equal(runs["xz"][2]["y"], runs["all"][2]["y"])
    np.testing.assert_allclose(runs["all"][1], runs["f32"][1], rtol=1e-3)
    # T rounded toward zero in BF16: steps up to 2^-8 (on average 2^-9) smaller, so the early epochs descend a little
    # slower (0.26 % higher deviance after the first epoch of this case, 0.21 % after the fourth)
    np.testing.assert_allclose(runs["t16"][1], runs["f32"][1], rtol=5e-3)
    assert runs["t16"][1][-1] < runs["t16"][1][0]
    f = runs["all"][1]
    assert np.isfinite(f).all() and f[-1] < f[0]
