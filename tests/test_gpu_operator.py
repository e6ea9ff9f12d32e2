"""The CUDA operator against the CPU oracle (same geometry, same batches) and against the reference's fixtures:
forward / adjoint values, the sparse PF structure bit for bit, the adjoint identity over the reference's angle
ranges, the omega-subset forms in both PF storage modes, NumPy streaming, and reproducibility."""
import numpy as np
import pytest

from conftest import CASES, case_inputs

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def make_operator(d, **kw):
    from diffractom_b200 import SinglePhaseForwardOperator
    cfg, mat, grid = case_inputs(d)
    kw.setdefault("max_gb", 1e-5)
    return SinglePhaseForwardOperator(cfg, mat, grid, normalized=True, quadrature=d["quadrature"],
                                      radon_kernel=d["kernel"], **kw)


def oracle_of(op):
    from oracle.oracle import OracleOperator
    return OracleOperator.from_operator(op)


def rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / np.abs(b).max())


@pytest.mark.parametrize("name", CASES)
def test_forward_adjoint_match_oracle_and_reference(golden, name):
    d = golden(name)
    op = make_operator(d)
    assert len(op.batches) > 1
    orc = oracle_of(op)
    c = torch.as_tensor(d["c"], device="cuda")
    r = torch.as_tensor(d["r"], device="cuda")
    fwd = op.direct(c).cpu().numpy()
    adj = op.adjoint(r).cpu().numpy()
    assert rel(fwd, orc.forward(d["c"])) < 1e-5
    assert rel(adj, orc.adjoint(d["r"])) < 1e-5
    # the reference's own tolerance against its float64 model (tests/test_differentiable.py:39)
    assert rel(fwd, d["fwd"]) < 2e-5
    assert rel(adj * np.float64(d["scale"]), d["adj"]) < 2e-5


@pytest.mark.parametrize("name", ["diff_auto_trapezoid", "al5_small", "ti8_small"])
def test_sparse_pf_structure_is_bit_exact(golden, name):
    d = golden(name)
    op = make_operator(d, pf_mode="sparse")
    orc = oracle_of(op)
    for sb, b in zip(op.sparse_batches, op.batches):
        ref = orc.csr(b["k_start"], b["K_batch"])
        nnz = ref["nnz"]
        assert sb["nnz"] == nnz
        for dev_key, ref_key in (("row_ptr_a", "row_ptr_a"), ("row_ptr_f", "row_ptr_f")):
            assert np.array_equal(sb[dev_key].cpu().numpy(), ref[ref_key])
        assert np.array_equal(sb["col_j"].cpu().numpy()[:nnz].view(np.uint16), ref["col_j"])
        assert np.array_equal(sb["col_k"].cpu().numpy()[:nnz].view(np.uint16), ref["col_k"])
        for key in ("val_a", "val_f"):
            v = sb[key].cpu().numpy()[:nnz].astype(np.float64)
            np.testing.assert_allclose(v, ref[key], rtol=2e-6, atol=0)   # float32 exp: a few ulp


@pytest.mark.parametrize("name", ["adj_0_180", "adj_0_360", "adj_0_90", "adj_180_0"])
def test_adjoint_is_transpose(golden, name):
    d = golden(name)
    op = make_operator(d)
    rng = np.random.default_rng(1)
    x = (rng.random(op.coeff_shape) * op.support_mask()[None]).astype(np.float32)
    y = rng.random(op.data_shape).astype(np.float32)
    ax = op.direct(torch.as_tensor(x, device="cuda")).cpu().numpy()
    aty = op.adjoint(torch.as_tensor(y, device="cuda")).cpu().numpy()
    lhs = float(np.dot(x.ravel().astype(np.float64), aty.ravel()))
    rhs = float(np.dot(ax.ravel().astype(np.float64), y.ravel()))
    assert rhs > 0 and abs(lhs / rhs - 1) < 1e-5


@pytest.mark.parametrize("pf_mode", ["sparse", "generated"])
@pytest.mark.parametrize("subsets", [4, "blocks"])
def test_subset_forward_and_adjoint(golden, pf_mode, subsets):
    d = golden("adj_0_360")
    op = make_operator(d, pf_mode=pf_mode)
    assert op.pf_mode == pf_mode and len(op.batches) > 1
    R = op.N_Omega
    subs = op.set_omega_subsets(4 if subsets == 4 else [np.arange(0, 7), np.arange(7, 20), np.arange(20, R)])
    rng = np.random.default_rng(6)
    x = (rng.random(op.coeff_shape) * op.support_mask()[None]).astype(np.float32)
    y = rng.random(op.data_shape).astype(np.float32)
    xd, yd = torch.as_tensor(x, device="cuda"), torch.as_tensor(y, device="cuda")
    full = op.direct(xd).cpu().numpy()
    adj = op.adjoint(yd).cpu().numpy()
    adj_sum = np.zeros_like(adj)
    for m, s in enumerate(subs):
        dd = torch.full(op.data_shape, -7.0, device="cuda")
        op.direct_cl(xd, dd, subset=m)
        dd = dd.cpu().numpy()
        np.testing.assert_allclose(dd[s], full[s], rtol=1e-5, atol=1e-6 * np.abs(full).max())
        assert np.all(dd[np.setdiff1d(np.arange(R), s)] == -7.0)
        a_m = torch.empty(op.coeff_shape, device="cuda")
        op.adjoint_cl(yd, a_m, subset=m)
        a_m = a_m.cpu().numpy()
        adj_sum += a_m
        lhs = float(np.dot(dd[s].ravel().astype(np.float64), y[s].ravel()))
        rhs = float(np.dot(x.ravel().astype(np.float64), a_m.ravel()))
        assert abs(lhs / rhs - 1) < 1e-5
    np.testing.assert_allclose(adj_sum, adj, rtol=1e-4, atol=1e-5 * np.abs(adj).max())


def test_generated_equals_stored(golden):
    d = golden("al5_small")
    a, b = make_operator(d, pf_mode="sparse"), make_operator(d, pf_mode="generated")
    c = torch.as_tensor(d["c"], device="cuda")
    r = torch.as_tensor(d["r"], device="cuda")
    assert torch.equal(a.direct(c), b.direct(c))
    assert torch.equal(a.adjoint(r), b.adjoint(r))


def test_numpy_streaming_equals_device_and_is_reproducible(golden):
    d = golden("ti8_small")
    op = make_operator(d)
    c_dev = op.direct(torch.as_tensor(d["c"], device="cuda")).cpu().numpy()
    assert np.array_equal(op.direct(d["c"]), c_dev)
    a_dev = op.adjoint(torch.as_tensor(d["r"], device="cuda")).cpu().numpy()
    assert np.array_equal(op.adjoint(d["r"]), a_dev)
    assert np.array_equal(op.direct(d["c"]), c_dev)          # same bits every call


def test_fused_backprojection_update_equals_unfused(golden):
    """dfx_radon_backward_spdhg (backprojection + SPDHG primal step in one kernel) gives bitwise the result of the
    backprojection followed by dfx_spdhg_primal_update; channel-fastest batches round-trip through the gathers."""
    from diffractom_b200 import _lib
    d = golden("al5_small")
    op = make_operator(d)
    op.set_omega_subsets(3)
    rng = np.random.default_rng(4)
    be = op.batch_elems()
    data = torch.as_tensor(rng.random(op.data_shape).astype(np.float32), device="cuda")
    coeffs = torch.as_tensor(rng.random(op.coeff_shape).astype(np.float32), device="cuda")
    xk = torch.empty(len(op.batches) * be, device="cuda")
    op.to_batches(coeffs, xk)
    back = torch.empty(op.coeff_shape, device="cuda")
    op.from_batches(xk, back)
    assert torch.equal(back, coeffs)
    zk = torch.as_tensor(rng.normal(0, 1, xk.numel()).astype(np.float32), device="cuda")
    Tk = torch.as_tensor((rng.random(xk.numel()) * (rng.random(xk.numel()) < 0.8)).astype(np.float32),
                         device="cuda")
    x1, z1 = xk.clone(), zk.clone()
    dz = torch.empty(be, device="cuda")
    for ib in range(len(op.batches)):
        off = ib * be
        op._adjoint_batch_k(data, ib, dz.data_ptr(), subset=1)
        _lib.call("dfx_spdhg_primal_update", x1.data_ptr() + 4 * off, z1.data_ptr() + 4 * off,
                  Tk.data_ptr() + 4 * off, dz.data_ptr(), 3.0, 0.25, be, op._s())
        op._adjoint_update_batch(data, ib, 1, xk.data_ptr() + 4 * off, zk.data_ptr() + 4 * off,
                                 Tk.data_ptr() + 4 * off, 3.0, 0.25)
    assert torch.equal(x1, xk) and torch.equal(z1, zk)


def test_argument_errors(golden):
    d = golden("diff_midpoint_hat")
    op = make_operator(d, pf_mode="sparse")
    with pytest.raises(TypeError):
        op.direct_cl(np.zeros(op.coeff_shape, np.float32), torch.empty(op.data_shape, device="cuda"))
    with pytest.raises(ValueError):
        op.direct_cl(torch.zeros((1, 2, 3), device="cuda"), torch.empty(op.data_shape, device="cuda"))
    with pytest.raises(TypeError):
        op.direct_cl(torch.zeros(op.coeff_shape, device="cuda", dtype=torch.float64),
                     torch.empty(op.data_shape, device="cuda"))
    with pytest.raises(ValueError):
        op.zero_subset_rows(torch.empty(op.data_shape, device="cuda"), 0)     # no subsets yet
    with pytest.raises(ValueError):
        op.set_omega_subsets([np.array([0, op.N_Omega])])


@pytest.mark.parametrize("name", ["ti8_small", "adj_0_90", "diff_midpoint_hat"])
def test_ray_table_forward_equals_footprint_forward(golden, name):
    """The table-driven forward projection (the operator's) gives the bits of the footprint-evaluating one, for all
    angles and for a subset's angle list, in float32 and BF16 sinograms; the grouped table gives the per-bin
    table's."""
    from diffractom_b200 import _lib
    d = golden(name)
    op = make_operator(d)
    rng = np.random.default_rng(5)
    kb = op.batches[0]["K_batch"]
    img = torch.as_tensor(rng.random((op.npix, op.Kstride)).astype(np.float32), device="cuda")
    img[:, kb:] = 0
    s = op._s()
    R, ns, ks = op.N_Omega, op.My, op.Kstride
    a = torch.empty((R, ns, ks), device="cuda")
    b = torch.empty((R, ns, ks), device="cuda")
    _lib.call("dfx_radon_forward", img.data_ptr(), a.data_ptr(), op.geo_gpu.data_ptr(), R, op.Nx, op.Ny, ns, ks, kb,
              op._kernel_id, float(op.radon_geo.scale), s)
    op._radon_fwd(img.data_ptr(), b.data_ptr(), None, R, kb)
    assert torch.equal(a, b)
    om = torch.arange(1, R, 3, dtype=torch.int32, device="cuda")
    c = torch.empty((om.numel(), ns, ks), device="cuda")
    op._radon_fwd(img.data_ptr(), c.data_ptr(), om, om.numel(), kb)
    assert torch.equal(c, a[om.long()])
    zb = torch.empty((R, ns, ks + 8), dtype=torch.bfloat16, device="cuda")
    op._radon_fwd(img.data_ptr(), zb.data_ptr(), None, R, kb, sld=ks + 8)
    assert torch.equal(zb[:, :, :ks], a.to(torch.bfloat16))
    assert op.ray_taps == int(op._ray_rp[-1].item()) > 0
    # the float32 forward of many angles reads the grouped table (four bins per pixel load): the per-bin table's
    # bits, for all angles, a subset's angles, and a support's tables (the kernel called directly)
    assert op._ray_grp is not None

    def grouped(src, rows, tabs):
        n = R if rows is None else rows.numel()
        out = torch.empty((n, ns, ks), device="cuda")
        _lib.call("dfx_radon_forward_gtable", src.data_ptr(), out.data_ptr(), tabs[0].data_ptr(), tabs[1].data_ptr(),
                  tabs[2].data_ptr(), None if rows is None else rows.data_ptr(), n, ns, ks, kb,
                  float(op.radon_geo.scale), s)
        return out

    assert torch.equal(grouped(img, None, op._ray_grp), a)
    assert torch.equal(grouped(img, om, op._ray_grp), a[om.long()])
    supp = torch.as_tensor(op.support_mask().ravel().astype(np.uint8), device="cuda")
    ray = op.support_ray_table(supp)
    assert len(ray) == 4 and int(ray[3][0][-1].item()) <= int(op._ray_grp[0][-1].item())
    imgs = img * supp.float()[:, None]
    t = torch.empty((om.numel(), ns, ks), device="cuda")
    _lib.call("dfx_radon_forward_table", imgs.data_ptr(), t.data_ptr(), ray[0].data_ptr(), ray[1].data_ptr(),
              om.data_ptr(), om.numel(), ns, ks, kb, float(op.radon_geo.scale), s)
    assert torch.equal(grouped(imgs, om, ray[3]), t)


def test_operator_on_its_own_queue_equals_current_stream(golden):
    """An operator built with queue=<a stream that is not current> gives the bits of one on the current stream: its
    build, forward, adjoint (device and NumPy) and an SPDHG run order themselves against the caller's stream."""
    from diffractom_b200 import SPDHGPoisson
    d = golden("al5_small")
    op = make_operator(d)
    opq = make_operator(d, queue=torch.cuda.Stream())
    assert opq.stream() != torch.cuda.current_stream()
    rng = np.random.default_rng(4)
    c = torch.as_tensor(rng.random(op.coeff_shape).astype(np.float32), device="cuda")
    fwd, fwdq = op.direct(c), opq.direct(c)
    assert torch.equal(fwd, fwdq)
    assert torch.equal(op.adjoint(fwd), opq.adjoint(fwdq))
    assert np.array_equal(op.direct(c.cpu().numpy()), opq.direct(c.cpu().numpy()))
    b = np.random.default_rng(5).poisson(fwd.cpu().numpy() * 20).astype(np.float32)
    xs = []
    for o in (op, opq):
        sp = SPDHGPoisson(o, subsets=3, seed=2)
        xs.append(sp.run(torch.zeros(o.coeff_shape, device="cuda"), b, 2, diagnostics_interval=1).cpu().numpy())
    assert np.array_equal(xs[0], xs[1])


def test_estimate_L_power_streamed(golden):
    """The streamed power iteration: with the serial start it is estimate_L_power; with the parallel start (other
    random numbers) it converges to the same largest eigenvalue of A^T A."""
    from diffractom_b200 import estimate_L_power, estimate_L_power_streamed
    op = make_operator(golden("diff_auto_trapezoid"))
    L = estimate_L_power(op, niter=40, verbose=0)
    assert estimate_L_power_streamed(op, niter=40, verbose=0, parallel_start=False) == L
    Lp = estimate_L_power_streamed(op, niter=40, verbose=0)
    assert abs(Lp / L - 1) < 1e-2


def test_dense_pf_mode_gemm_products(golden):
    """pf_mode "dense" (the reference's float32 GEMM path, SPFO:2063-2127): the batch's PF generated in every call and
    applied by batched SGEMMs, forward and adjoint within 1e-5 of the sparse products and of the oracle; "auto" takes
    it above max_fill (SPFO:1249-1263); omega subsets need a sparse mode (NotImplementedError, as the reference)."""
    d = golden("diff_auto_trapezoid")
    dense = make_operator(d, pf_mode="dense")
    sparse = make_operator(d, pf_mode="sparse")
    auto = make_operator(d)                                # 59 % fill > 30 %
    assert dense.pf_mode == "dense" and auto.pf_mode == "dense" and sparse.pf_mode == "sparse"
    assert len(dense.batches) > 1
    orc = oracle_of(dense)
    c = torch.as_tensor(d["c"], device="cuda")
    r = torch.as_tensor(d["r"], device="cuda")
    fd, fs = dense.direct(c).cpu().numpy(), sparse.direct(c).cpu().numpy()
    ad, as_ = dense.adjoint(r).cpu().numpy(), sparse.adjoint(r).cpu().numpy()
    assert rel(fd, fs) < 1e-5 and rel(ad, as_) < 1e-5
    assert rel(fd, orc.forward(d["c"])) < 1e-5 and rel(ad, orc.adjoint(d["r"])) < 1e-5
    assert np.array_equal(dense.direct(d["c"]), fd)        # NumPy (streamed batches) path, same bits
    with pytest.raises(NotImplementedError):
        dense.set_omega_subsets(3)


def test_pf_storage_modes_compute_the_same_operator(golden):
    """The PF storage preferences of build_sparse_pf (SPFO:1207-1373): both CSR copies, the adjoint copies only (the
    forward copy generated in every call), the adjoint copies of the first batches (mode "auto" within a budget that
    holds only some; the others generated in every call), nothing stored; full and subset products are the same bits
    in every mode. Mode "sparse" with a budget below the adjoint copies raises MemoryError."""
    d = golden("al5_small")
    ref = make_operator(d, pf_mode="sparse")
    assert ref.pf_storage == "both" and len(ref.batches) >= 3
    both, adj, ptr_f, batch_adj = ref.sparse_estimates(ref.sparse_fill_first)
    gb = 1024.0 ** 3
    part = (len(ref.batches) * ptr_f + batch_adj[0] + batch_adj[1] + 1) / gb   # room for two batches' adjoints
    # the storage preferences alone: the reference's dense switch above max_fill_partial (when the sparse matrix does
    # not fit) turned off; with it on, this case's fill takes the dense path
    nodense = dict(sparse_max_fill=1.0, sparse_max_fill_partial=1.0)
    ops = {"adjoint": make_operator(d, pf_mode="auto", sparse_max_gb=(adj + 1) / gb, **nodense),
           "partial": make_operator(d, pf_mode="auto", sparse_max_gb=part, **nodense),
           "generated": make_operator(d, pf_mode="generated")}
    if ref.sparse_fill_first > 0.1:
        assert make_operator(d, pf_mode="auto", sparse_max_gb=(adj + 1) / gb).pf_mode == "dense"
    assert ops["adjoint"].pf_storage == "adjoint"
    assert ops["partial"].pf_storage == f"adjoint, 2 of {len(ref.batches)} batches"
    assert ops["generated"].pf_storage == "none"
    rng = np.random.default_rng(2)
    x = torch.as_tensor(rng.random(ref.coeff_shape).astype(np.float32), device="cuda")
    y = torch.as_tensor(rng.random(ref.data_shape).astype(np.float32), device="cuda")
    outs = {}
    for name, op in [("both", ref)] + list(ops.items()):
        assert [b["K_batch"] for b in op.batches] == [b["K_batch"] for b in ref.batches]
        op.set_omega_subsets(3)
        fx, ay = torch.empty_like(y), torch.empty_like(x)
        op.direct_cl(x, fx)
        op.adjoint_cl(y, ay)
        fs, as_ = torch.zeros_like(y), torch.empty_like(x)
        op.direct_cl(x, fs, subset=1)
        op.adjoint_cl(y, as_, subset=2)
        outs[name] = [t.cpu().numpy() for t in (fx, ay, fs, as_)]
    for name in ops:
        for a, b in zip(outs[name], outs["both"]):
            assert np.array_equal(a, b), name
    with pytest.raises(MemoryError):
        make_operator(d, pf_mode="sparse", sparse_max_gb=part)


@pytest.mark.parametrize("pf_mode", ["sparse", "generated"])
def test_channel_constant_forward_equals_batch_by_batch(golden, pf_mode):
    """_direct_channel_constant (one Radon transform of an image that is the same in every channel, read by every
    batch's PF product; the step sizes' row sums A 1_S) gives the bits of the forward batch by batch, with the full
    ray table and with a support's table, for batches of different widths."""
    d = golden("al5_small")
    op = make_operator(d, pf_mode=pf_mode)
    widths = [b["K_batch"] for b in op.batches]
    assert len(widths) > 1
    kbm = max(widths)
    npix, ks = op.Nx * op.Ny, op.Kstride
    rng = np.random.default_rng(11)
    supp = torch.as_tensor(op.support_mask().ravel().astype(np.uint8), device="cuda")
    pattern = torch.as_tensor(rng.random(npix).astype(np.float32), device="cuda") * supp.float()
    for ray in (None, op.support_ray_table(supp)):
        img = torch.zeros((npix, ks), device="cuda")
        img[:, :kbm] = pattern[:, None]
        one = torch.zeros(op.data_shape, device="cuda")
        torch.cuda.synchronize()
        op._direct_channel_constant(img.data_ptr(), kbm, one, ray=ray)
        torch.cuda.synchronize()
        each = torch.zeros(op.data_shape, device="cuda")
        for ib, kb in enumerate(widths):
            imb = torch.zeros((npix, ks), device="cuda")
            imb[:, :kb] = pattern[:, None]
            torch.cuda.synchronize()
            op._direct_batch_k(imb.data_ptr(), ib, each, ray=ray)
            torch.cuda.synchronize()
        assert torch.equal(one, each)
        assert float(one.abs().max()) > 0
