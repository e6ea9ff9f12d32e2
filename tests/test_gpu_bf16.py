"""The BF16 tensor-core precision path of the operator and of SPDHGPoisson against the float64 oracle: operator
values within the BF16 bound, subset rows, angle-chunked products, and the SPDHG deviance within 1e-3 relative of
the float64 run of the same loop (same subsets, schedule and step sizes); the side-stream residual against the
in-line one."""
import numpy as np
import pytest

from conftest import case_inputs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

# BF16 operands (8-bit significands) with float32 accumulation: the operator's values stay within a few 2^-9 of the
# largest value; this bound is checked, not assumed
OP_TOL = 1e-2
DEV_TOL = 1e-3


def make_operator(d, **kw):
    from diffractom_b200 import SinglePhaseForwardOperator
    cfg, mat, grid = case_inputs(d)
    kw.setdefault("max_gb", 1e-5)
    return SinglePhaseForwardOperator(cfg, mat, grid, normalized=True, quadrature=d["quadrature"],
                                      radon_kernel=d["kernel"], **kw)


def rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / np.abs(b).max())


@pytest.mark.parametrize("name", ["al5_small", "ti8_small", "adj_0_360"])
def test_bf16_operator_matches_oracle(golden, name):
    from oracle.oracle import OracleOperator
    d = golden(name)
    op = make_operator(d, precision="bf16")
    assert op.precision == "bf16" and len(op.batches) > 1
    orc = OracleOperator.from_operator(op, precision="f64")
    c = torch.as_tensor(d["c"], device="cuda")
    r = torch.as_tensor(d["r"], device="cuda")
    fwd = op.direct(c).cpu().numpy()
    adj = op.adjoint(r).cpu().numpy()
    ef, ea = rel(fwd, orc.forward(d["c"])), rel(adj, orc.adjoint(d["r"]))
    assert ef < OP_TOL and ea < OP_TOL, (ef, ea)
    # the float32 operator of the same object is untouched by the precision switch
    op.precision = "fp32"
    assert rel(op.direct(c).cpu().numpy(), orc.forward(d["c"])) < 1e-5


def test_bf16_subsets_and_angle_chunks(golden):
    d = golden("adj_0_360")
    op = make_operator(d, precision="bf16")
    R = op.N_Omega
    subs = op.set_omega_subsets(4)
    rng = np.random.default_rng(2)
    x = torch.as_tensor((rng.random(op.coeff_shape) * op.support_mask()[None]).astype(np.float32), device="cuda")
    y = torch.as_tensor(rng.random(op.data_shape).astype(np.float32), device="cuda")
    full = op.direct(x)
    adj = op.adjoint(y)
    for m, s in enumerate(subs):
        dd = torch.full(op.data_shape, -7.0, device="cuda")
        op.direct_cl(x, dd, subset=m)
        sel = torch.as_tensor(s, device="cuda")
        assert torch.equal(dd[sel], full[sel])                      # same tensor-core sums row by row
        rest = torch.as_tensor(np.setdiff1d(np.arange(R), s), device="cuda")
        assert torch.all(dd[rest] == -7.0)
    # angles in several chunks of the Z buffer: the same rows, and the backprojections summed over the chunks
    op.build_dense_bf16_pf(max_z_gb=3 * 2 * op.My * op.Ktot / 1024 ** 3)
    assert op._bf16_chunk == 3 < R
    assert torch.equal(op.direct(x), full)
    a2 = op.adjoint(y)
    assert rel(a2.cpu().numpy(), adj.cpu().numpy().astype(np.float64)) < 1e-5


def test_bf16_spdhg_deviance_within_1e3_of_float64(golden):
    from diffractom_b200 import SinglePhaseForwardOperator, SPDHGPoisson
    from oracle.oracle import OracleOperator, spdhg_reference
    d = golden("al5_small")
    cfg, mat, grid = case_inputs(d)
    op = SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"],
                                    precision="bf16")
    rng = np.random.default_rng(11)
    x_true = (rng.random(op.coeff_shape) * (rng.random(op.coeff_shape) < 0.2) * op.support_mask()[None]
              ).astype(np.float32)
    op.precision = "fp32"
    b = rng.poisson(op.direct(x_true) * 50).astype(np.float32)
    op.precision = "bf16"
    n_ep = 6
    sp = SPDHGPoisson(op, subsets=3, seed=1)
    x = sp.run(torch.zeros(op.coeff_shape, device="cuda"), b, n_ep, diagnostics_interval=n_ep).cpu().numpy()
    f_bf16 = sp.iter_stats[-1]["f"]
    orc = OracleOperator.from_operator(op, precision="f64")
    xr, yr, zr, devs, rho = spdhg_reference(orc, op.omega_subsets, b, n_ep, support=op.support_mask(), seed=1,
                                            diagnostics_interval=n_ep)
    f64 = devs[-1]
    dev_err = abs(f_bf16 - f64) / f64
    coef_err = float(np.linalg.norm(x - xr) / np.linalg.norm(xr))
    assert dev_err <= DEV_TOL, (dev_err, coef_err)
    assert coef_err < 5e-2, coef_err


def test_side_stream_residual_matches_the_inline_one(golden):
    """The residual of every diagnostics epoch run on a side stream from a copy of x (SPDHGPoisson.overlap_residual,
    run()'s default with a BF16 operator): every epoch's objective is filled in, and the objectives and the final x
    agree with those of the in-line residual, whose rows also serve the next subset (where the BF16 forward's rows do
    otherwise), to the BF16 path's 1e-3 (measured: 1.7e-4) and 5e-3."""
    from diffractom_b200 import SPDHGPoisson
    d = golden("al5_small")
    op = make_operator(d, precision="bf16")
    assert len(op.batches) > 2
    rng = np.random.default_rng(12)
    x_true = (rng.random(op.coeff_shape) * (rng.random(op.coeff_shape) < 0.2) * op.support_mask()[None]
              ).astype(np.float32)
    op.precision = "fp32"
    b = rng.poisson(op.direct(x_true) * 50).astype(np.float32)
    op.precision = "bf16"
    out = {}
    for overlap in (False, True):
        sp = SPDHGPoisson(op, subsets=3, seed=1)
        sp.overlap_residual = overlap
        x = sp.run(np.zeros(op.coeff_shape, np.float32), b, 5, diagnostics_interval=1)
        out[overlap] = (x, [st["f"] for st in sp.iter_stats], sp.final_stats["final_f"])
    (x0, f0, l0), (x1, f1, l1) = out[False], out[True]
    assert all(f is not None for f in f1) and l1 == f1[-1]
    assert f1[0] == f0[0]                 # the first epoch's iterations are the same; later ones differ in BF16
    np.testing.assert_allclose(f1, f0, rtol=1e-3)
    assert np.linalg.norm(x1 - x0) <= 5e-3 * np.linalg.norm(x0)


def _tc_vs_simt(geo, R, nx, ny, ns, kb, kernel_id, n_taps, seed=8):
    """Runs the SIMT and the tensor-core backprojection with the fused SPDHG step on the same BF16 sinogram and
    state and checks: z (= the backprojection, from z = 0) within 2e-5 of its maximum, x from the same formula, and
    the BF16 copy of x exactly x rounded."""
    import ctypes
    from diffractom_b200 import _lib
    rng = np.random.default_rng(seed)
    npix = nx * ny
    ks = -(-max(kb, 16) // 16) * 16
    sld = ks + 16
    sino = torch.as_tensor(rng.standard_normal((R, ns, sld)).astype(np.float32), device="cuda").to(torch.bfloat16)
    T = torch.as_tensor((rng.random((npix, ks)) * (rng.random((npix, ks)) < 0.9)).astype(np.float32), device="cuda")
    T[:, kb:] = 0
    x0 = torch.full((npix, ks), 50.0, device="cuda")
    x0[:, kb:] = 0
    stream = torch.cuda.current_stream().cuda_stream
    out = {}
    for name_fn in ("dfx_radon_backward_spdhg_bf16", "dfx_radon_backward_spdhg_tc"):
        x, z = x0.clone(), torch.zeros((npix, ks), device="cuda")
        xb = torch.zeros((npix, ks), dtype=torch.bfloat16, device="cuda")
        _lib.call(name_fn, sino.data_ptr(), sld, geo.data_ptr(), R, nx, ny, ns, ks, kb, kernel_id, n_taps,
                  x.data_ptr(), z.data_ptr(), T.data_ptr(), 3.0, 0.1, xb.data_ptr(), stream)
        out[name_fn] = (x, z, xb)
    torch.cuda.synchronize()
    xs, zs, xbs = out["dfx_radon_backward_spdhg_bf16"]
    xt, zt, xbt = out["dfx_radon_backward_spdhg_tc"]
    zmax = float(zs.abs().max())
    assert zmax > 0
    assert float((zt - zs).abs().max()) <= 2e-5 * zmax
    assert float((xt - xs).abs().max()) <= 1e-4 * float(xs.abs().max())
    assert torch.equal(xbt[:, :kb], xt[:, :kb].to(torch.bfloat16))
    assert torch.equal(xbs[:, :kb], xs[:, :kb].to(torch.bfloat16))
    # channels past the batch are left alone
    assert torch.equal(xt[:, kb:], x0[:, kb:]) and not bool(zt[:, kb:].any())
    f = ctypes.c_uint(0)
    _lib.check(_lib.lib().dfx_tc_status(ctypes.byref(f), 1))
    assert f.value == 0


@pytest.mark.parametrize("name", ["al5_small", "adj_0_360", "diff_midpoint_hat"])
def test_tc_backprojection_update_matches_simt(golden, name):
    """The tensor-core backprojection with the fused SPDHG step against the SIMT one on the reference's test
    geometries (one tile per CTA)."""
    d = golden(name)
    op = make_operator(d)
    assert op.Kstride > 0
    _tc_vs_simt(op.geo_gpu, op.N_Omega, op.Nx, op.Ny, op.My, op.batches[0]["K_batch"], op._kernel_id,
                int(op.radon_geo.n_taps))


@pytest.mark.parametrize("kernel", ["trapezoid", "hat"])
def test_tc_backprojection_many_tiles_per_cta(kernel):
    """A ragged image (130 x 124 pixels: partial 16 x 8 tiles on both edges) and 1200 channels (a partial last
    256-channel block): 720 tiles, so each persistent CTA walks several tiles and both tensor-memory accumulators
    go through several phases."""
    from diffractom_b200.geometry import radon_geometry
    nx, ny, ns, R = 130, 124, 190, 30
    ang = np.linspace(0.0, np.pi, R, endpoint=False) + 0.013
    g = radon_geometry(ang, nx, ny, ns, float(max(nx, ny)), float(ns), 0.37, np.pi / R, kernel=kernel)
    geo = torch.as_tensor(g.geo, device="cuda")
    _tc_vs_simt(geo, R, nx, ny, ns, 1200, 1 if kernel == "trapezoid" else 0, int(g.n_taps), seed=3)


def test_generated_bf16_pf_equals_the_stored_one(golden):
    """bf16_pf="generated" (no PF of all angles kept; each tensor-core product generates the PF of its angles into
    one of two buffers) computes the stored PF's operator bit for bit: full and subset products, and a BF16 SPDHG
    run (the same iterates, deviances and state)."""
    from diffractom_b200 import SinglePhaseForwardOperator, SPDHGPoisson
    d = golden("al5_small")
    cfg, mat, grid = case_inputs(d)
    ops = [SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"],
                                      precision="bf16", bf16_pf=mode) for mode in ("stored", "generated")]
    assert ops[0].bf16_pf_storage == "stored" and ops[1].bf16_pf_storage == "generated" and ops[1].pf_bf16 is None
    rng = np.random.default_rng(8)
    x = torch.as_tensor(rng.random(ops[0].coeff_shape).astype(np.float32), device="cuda")
    y = torch.as_tensor(rng.random(ops[0].data_shape).astype(np.float32), device="cuda")
    outs = []
    for op in ops:
        op.set_omega_subsets(3)
        r = []
        for sub in (None, 0, 2, 0):
            fx, ay = torch.zeros_like(y), torch.empty_like(x)
            op.direct_cl(x, fx, subset=sub)
            op.adjoint_cl(y, ay, subset=sub)
            r += [fx.cpu(), ay.cpu()]
        outs.append(r)
    for a, b in zip(*outs):
        assert torch.equal(a, b)
    b = np.random.default_rng(3).poisson(np.abs(outs[0][0].numpy()) * 50).astype(np.float32)
    runs = []
    for op in ops:
        sp = SPDHGPoisson(op, subsets=3, seed=4)
        xr = sp.run(torch.zeros(op.coeff_shape, device="cuda"), b, 3, diagnostics_interval=1).cpu().numpy()
        runs.append((xr, [s["f"] for s in sp.iter_stats], sp.state["y"]))
    assert np.array_equal(runs[0][0], runs[1][0]) and runs[0][1] == runs[1][1]
    assert np.array_equal(runs[0][2], runs[1][2])
