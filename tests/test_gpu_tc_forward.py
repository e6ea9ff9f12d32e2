"""The tensor-core forward projection (dfx_radon_forward_tc: tcgen05, 8 x 8 pixel tiles, BF16 image, weights as BF16
hi + lo parts, float32 accumulation) against the table-driven forward of the same image (dfx_radon_forward_table on
the image widened to float32, exactly): float32 outputs within 2e-5 of the largest value, for the trapezoid and the
hat kernel, every angle of the golden geometries and of a 256 x 256, 360-angle scan; a tile list that skips the
tiles outside a support equals the full projection of an image that is zero there; BF16 output rows in a wider
sinogram; the weight-table variant gives the same bits; no tensor-core wait ran out and no tap left its window;
BF16 SPDHG with and without it; the float32 grouped-table forward of the same 360-angle scan."""
import ctypes

import numpy as np
import pytest

from conftest import case_inputs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _flags(lib):
    f = ctypes.c_uint(0)
    assert lib.dfx_tc_status(ctypes.byref(f), 1) == 0
    return f.value


def _project(op, img_bf16, tiles=None, out_bf16_ld=None):
    """(tensor-core output (R, My, Kstride) float32, table output of the widened image)."""
    from diffractom_b200 import _lib
    lib = _lib.lib()
    R, My, ks = op.N_Omega, op.My, op.Kstride
    s = op._s()
    tc = torch.full((R, My, ks), -9.0, dtype=torch.float32, device="cuda")
    tp, nt = (None, 0) if tiles is None else (tiles.data_ptr(), int(tiles.numel()))
    _lib.call("dfx_radon_forward_tc", img_bf16.data_ptr(), tc.data_ptr(), ks, 1, op.geo_gpu.data_ptr(), R, op.Nx,
              op.Ny, My, ks, op._kernel_id, int(op.radon_geo.n_taps), float(op.radon_geo.scale), tp, nt, s)
    ref = torch.empty((R, My, ks), dtype=torch.float32, device="cuda")
    img32 = img_bf16.float().contiguous()
    _lib.call("dfx_radon_forward_table", img32.data_ptr(), ref.data_ptr(), op._ray_rp.data_ptr(),
              op._ray_ent.data_ptr(), None, R, My, ks, ks, float(op.radon_geo.scale), s)
    torch.cuda.synchronize()
    return tc, ref


def _image(op, seed, supp=None):
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.rand((op.Ny * op.Nx, op.Kstride), generator=g, device="cuda")
    if supp is not None:
        x *= torch.as_tensor(supp.reshape(-1, 1), device="cuda")
    return x.to(torch.bfloat16).contiguous()


@pytest.mark.parametrize("name", ["al5_small", "diff_midpoint_hat", "adj_0_360", "ti8_small"])
def test_tc_forward_matches_table_forward(golden, name):
    from diffractom_b200 import SinglePhaseForwardOperator, _lib
    d = golden(name)
    cfg, mat, grid = case_inputs(d)
    op = SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"],
                                    radon_kernel=d["kernel"], precision="bf16")
    assert op.tc_forward
    _flags(_lib.lib())
    tc, ref = _project(op, _image(op, 3))
    err = float((tc - ref).abs().max() / ref.abs().max())
    assert err <= 2e-5, err
    assert _flags(_lib.lib()) == 0


def _ti256_operator(K=120):
    from diffractom_b200 import Grid, Material, SinglePhaseForwardOperator
    cfg = dict(Nx=256, Ny=256, My=263, N_Omega=360, angle_range=[0, 180], cor_offset=0.0, N_eta=360,
               eta_angle_range=[0, 360], energy=12.398 / 0.3, k_direction_0=[0, 0, 1], p_direction_0=[1, 0, 0],
               detector_direction_origin=[0, -1, 0], detector_direction_positive_90=[0, 0, -1])
    mat = Material.from_lattice_parameters(a=2.95, c=4.68, gamma=120, symmetry_group="hexagonal", wavelength_A=0.3,
                                           hkl_list=[[1, 0, 0], [0, 0, 2], [1, 0, 1]])
    grid = Grid.from_random_fundamental_zone(K, mat.crystal_system, np.deg2rad(2.0), seed=1)
    return SinglePhaseForwardOperator(cfg, mat, grid, 0.5, normalized=True, precision="bf16")


def test_tc_forward_full_scan_support_tiles_and_bf16_rows():
    from diffractom_b200 import _lib
    op = _ti256_operator()
    assert op.tc_forward and op.Kstride % 64 == 0
    lib = _lib.lib()
    _flags(lib)
    supp = op.support_mask()
    img = _image(op, 5, supp)
    tc, ref = _project(op, img)
    err = float((tc - ref).abs().max() / ref.abs().max())
    assert err <= 2e-5, err
    tiles = op.support_tiles(torch.as_tensor(supp.ravel().astype(np.uint8), device="cuda"))
    assert 0 < tiles.numel() < (-(-op.Ny // 8)) * (-(-op.Nx // 8))
    tc_t, _ = _project(op, img, tiles=tiles)
    assert torch.equal(tc_t, tc)                       # skipped tiles hold zeros only
    # BF16 rows at a column offset of a wider sinogram (the Z buffer of all batches)
    ld = 3 * op.Kstride
    z = torch.zeros((op.N_Omega, op.My, ld), dtype=torch.bfloat16, device="cuda")
    _lib.call("dfx_radon_forward_tc", img.data_ptr(), z.data_ptr() + 2 * op.Kstride, ld, 0, op.geo_gpu.data_ptr(),
              op.N_Omega, op.Nx, op.Ny, op.My, op.Kstride, op._kernel_id, int(op.radon_geo.n_taps),
              float(op.radon_geo.scale), None, 0, op._s())
    torch.cuda.synchronize()
    assert torch.equal(z[:, :, op.Kstride:2 * op.Kstride], tc.to(torch.bfloat16))
    assert not z[:, :, :op.Kstride].any() and not z[:, :, 2 * op.Kstride:].any()
    assert _flags(lib) == 0


def test_grouped_table_forward_of_a_full_scan():
    """The float32 forward through the grouped table (dfx_radon_forward_gtable) at 360 angles and 256 x 256 pixels,
    and for a subset's 18 angles: the per-bin table's bits."""
    from diffractom_b200 import _lib
    op = _ti256_operator()
    assert op._ray_grp is not None
    R, My, ks, s = op.N_Omega, op.My, op.Kstride, op._s()
    kb = op.batches[0]["K_batch"]
    g = torch.Generator(device="cuda").manual_seed(7)
    img = torch.rand((op.npix, ks), generator=g, device="cuda")
    img[:, kb:] = 0
    om = torch.arange(3, R, 20, dtype=torch.int32, device="cuda")
    for rows in (None, om):
        n = R if rows is None else rows.numel()
        rp = None if rows is None else rows.data_ptr()
        a = torch.empty((n, My, ks), device="cuda")
        b = torch.empty((n, My, ks), device="cuda")
        _lib.call("dfx_radon_forward_table", img.data_ptr(), a.data_ptr(), op._ray_rp.data_ptr(),
                  op._ray_ent.data_ptr(), rp, n, My, ks, kb, float(op.radon_geo.scale), s)
        grp = op._ray_grp
        _lib.call("dfx_radon_forward_gtable", img.data_ptr(), b.data_ptr(), grp[0].data_ptr(), grp[1].data_ptr(),
                  grp[2].data_ptr(), rp, n, My, ks, kb, float(op.radon_geo.scale), s)
        torch.cuda.synchronize()
        assert torch.equal(a, b)


@pytest.mark.parametrize("case", ["al5_small", "ti256"])
def test_tc_forward_from_the_weight_table_equals_the_built_weights(golden, case):
    """dfx_radon_forward_tc_table (weight tiles precomputed per geometry by dfx_radon_tc_weights, loaded beside the
    image tiles) gives dfx_radon_forward_tc's bits: all angles, a subset's angle rows with a support tile list, BF16
    rows in a wider sinogram."""
    from diffractom_b200 import SinglePhaseForwardOperator, _lib
    if case == "ti256":
        op = _ti256_operator()
    else:
        d = golden(case)
        cfg, mat, grid = case_inputs(d)
        op = SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"],
                                        precision="bf16")
    assert op.tc_forward
    lib = _lib.lib()
    _flags(lib)
    R, My, ks, s = op.N_Omega, op.My, op.Kstride, op._s()
    w, win = op._tc_weight_table()
    assert w.numel() == lib.dfx_radon_tc_weights_bytes(R, op.Nx, op.Ny)
    supp = op.support_mask()
    img = _image(op, 8, supp)
    tiles = op.support_tiles(torch.as_tensor(supp.ravel().astype(np.uint8), device="cuda"))
    om = torch.arange(2, R, 5, dtype=torch.int32, device="cuda")
    geo_sub = op.geo_gpu[om.long()].contiguous()
    for rows, geo, tl in ((None, op.geo_gpu, None), (om, geo_sub, tiles)):
        n = R if rows is None else rows.numel()
        tp, nt = (None, 0) if tl is None else (tl.data_ptr(), int(tl.numel()))
        ref = torch.full((n, My, 2 * ks), 7.0, dtype=torch.bfloat16, device="cuda")
        got = torch.full((n, My, 2 * ks), 7.0, dtype=torch.bfloat16, device="cuda")
        _lib.call("dfx_radon_forward_tc", img.data_ptr(), ref.data_ptr() + 2 * ks, 2 * ks, 0, geo.data_ptr(), n,
                  op.Nx, op.Ny, My, ks, op._kernel_id, int(op.radon_geo.n_taps), float(op.radon_geo.scale), tp, nt, s)
        _lib.call("dfx_radon_forward_tc_table", img.data_ptr(), got.data_ptr() + 2 * ks, 2 * ks, 0, w.data_ptr(),
                  win.data_ptr(), None if rows is None else rows.data_ptr(), n, op.Nx, op.Ny, My, ks,
                  float(op.radon_geo.scale), tp, nt, s)
        torch.cuda.synchronize()
        assert torch.equal(got, ref)
        assert torch.all(got[:, :, :ks] == 7.0)
    assert _flags(lib) == 0


def test_bf16_spdhg_with_and_without_the_tc_forward(golden):
    from diffractom_b200 import SinglePhaseForwardOperator, SPDHGPoisson
    d = golden("al5_small")
    cfg, mat, grid = case_inputs(d)
    op = SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"],
                                    precision="bf16")
    rng = np.random.default_rng(9)
    x_true = (rng.random(op.coeff_shape) * (rng.random(op.coeff_shape) < 0.2) * op.support_mask()[None]
              ).astype(np.float32)
    b = rng.poisson(op.direct(torch.as_tensor(x_true, device="cuda")).cpu().numpy() * 50).astype(np.float32)
    out = []
    for use in (True, False):
        op.use_tc_forward = use
        sp = SPDHGPoisson(op, subsets=3, seed=1)
        x = sp.run(torch.zeros(op.coeff_shape, device="cuda"), b, 4, diagnostics_interval=1).cpu().numpy()
        out.append((x, [s["f"] for s in sp.iter_stats]))
    op.use_tc_forward = True
    (x1, f1), (x0, f0) = out
    np.testing.assert_allclose(f1, f0, rtol=1e-4)
    assert np.linalg.norm(x1 - x0) <= 1e-2 * np.linalg.norm(x0)
