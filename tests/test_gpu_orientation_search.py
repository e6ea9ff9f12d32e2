"""The multi-RHS adjoint (adjoint_multi_cl: one PF matrix per batch for several data arrays and angle-row masks,
whole images or a pixel list) against adjoint_cl of the row-masked arrays, bitwise; score_candidates (chunked
operators, the score on the device, top-k per pixel) against the score computed from adjoint_cl per chunk."""
import numpy as np
import pytest

from conftest import case_inputs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _op(golden, name="al5_small", grid=None, pf_mode="auto"):
    from diffractom_b200 import SinglePhaseForwardOperator
    d = golden(name)
    cfg, mat, g = case_inputs(d)
    return SinglePhaseForwardOperator(cfg, mat, grid if grid is not None else g, 1e-5, normalized=True,
                                      quadrature=d["quadrature"], pf_mode=pf_mode)


@pytest.mark.parametrize("pf_mode", ["sparse", "generated"])
def test_adjoint_multi_equals_masked_adjoints(golden, pf_mode):
    op = _op(golden, pf_mode=pf_mode)
    assert len(op.batches) > 1
    rng = np.random.default_rng(4)
    datas = [torch.as_tensor(rng.standard_normal(op.data_shape).astype(np.float32), device="cuda") for _ in range(3)]
    mask = rng.random(op.N_Omega) < 0.6
    masks = [None, mask, np.zeros(op.N_Omega, bool)]
    pixels = np.sort(rng.choice(op.npix, 57, replace=False))
    for pix in (None, pixels):
        got = {}

        def consume(i, s, k0, Kb, block):
            if pix is None:
                got[(i, s, k0)] = block[:, :Kb].T.cpu().numpy().reshape(Kb, op.Ny, op.Nx).copy()
            else:
                got[(i, s, k0)] = block[:Kb].cpu().numpy().copy()

        done = []
        op.adjoint_multi_cl(datas, consume, row_masks=masks, pixels=pix, nrhs=2,
                            batch_done=lambda k0, Kb: done.append((k0, Kb)))
        assert done == [(b["k_start"], b["K_batch"]) for b in op.batches]
        for i, d in enumerate(datas):
            for s, m in enumerate(masks):
                dm = d.clone()
                if m is not None:
                    dm[torch.as_tensor(~m, device="cuda")] = 0
                ref = op.adjoint(dm).cpu().numpy()
                for b in op.batches:
                    k0, Kb = b["k_start"], b["K_batch"]
                    want = ref[k0:k0 + Kb]
                    if pix is not None:
                        want = want.reshape(Kb, -1)[:, pix]
                    assert np.array_equal(got[(i, s, k0)], want), (i, s, k0)


def test_score_candidates_equals_direct_scores(golden):
    from diffractom_b200.grid import Grid, MatrixGrid
    from diffractom_b200.orientation_search import poisson_score_inputs, scramble_eta, score_candidates
    d = golden("al5_small")
    cand = Grid.from_random_fundamental_zone(40, "cubic", float(np.asarray(d["sigma64"]).ravel()[0]), seed=3)
    rots, sig = cand.leaf_arrays()
    base = _op(golden)
    rng = np.random.default_rng(6)
    mu = (rng.random(base.data_shape) * 5 + 0.5).astype(np.float32)
    b = rng.poisson(mu * 1.3).astype(np.float32)
    e, dd = poisson_score_inputs(b, mu, 1.0, np.ones(base.N_seg, np.float32))
    e2 = scramble_eta(e, base.N_eta, base.N_peaks, block=3, margin=2)
    inputs = [(torch.as_tensor(e, device="cuda"), torch.as_tensor(dd, device="cuda")),
              (torch.as_tensor(e2, device="cuda"), torch.as_tensor(dd, device="cuda"))]
    held = np.zeros(base.N_Omega, bool)
    held[::3] = True
    masks = [~held, held]
    pixels = np.flatnonzero(base.support_mask().ravel())[::2]
    make = lambda r: _op(golden, grid=MatrixGrid(r, sig[:len(r)]))
    top_k, chunk = 5, 16
    out = score_candidates(make, rots, inputs, masks, pixels, top_k=top_k, chunk=chunk)
    for j, (E, D) in enumerate(inputs):
        z = [[] for _ in masks]
        for c0 in range(0, len(rots), chunk):
            op = make(rots[c0:c0 + chunk])
            for s, m in enumerate(masks):
                sel = torch.as_tensor(~m, device="cuda")
                Em, Dm = E.clone(), D.clone()
                Em[sel] = 0
                Dm[sel] = 0
                ae = op.adjoint(Em).cpu().numpy().reshape(op.K, -1)[:, pixels]
                ad = op.adjoint(Dm).cpu().numpy().reshape(op.K, -1)[:, pixels]
                zz = ae / np.sqrt(np.maximum(ad, np.float32(1e-30)))
                zz[ad <= 0] = 0
                z[s].append(zz)
        z = [np.concatenate(zs, 0) for zs in z]                      # (K, npix)
        order = np.argsort(-z[0], axis=0, kind="stable")[:top_k].T    # (npix, top_k)
        assert np.array_equal(np.sort(out[j]["idx"], 1), np.sort(order, 1))
        for s in range(len(masks)):
            assert np.array_equal(out[j]["z"][s], np.take_along_axis(z[s].T, out[j]["idx"], 1))
        assert np.all(np.diff(out[j]["z"][0], axis=1) <= 0)


def test_refine_candidates_moves_a_candidate_to_the_missing_crystal():
    """A crystal missing from the model (data = its forward plus a flat background, prediction = the background) and a
    candidate on its tiles started 3 deg away: refine_candidates (two rotation lattices, scores through a local-basis
    operator's adjoint on the fitted angles) brings it within 0.6 deg of the truth."""
    from scipy.spatial.transform import Rotation

    from diffractom_b200 import Material, SinglePhaseForwardOperator
    from diffractom_b200.grid import MatrixGrid
    from diffractom_b200.local import LocalSinglePhaseForwardOperator, LocalSupport
    from diffractom_b200.orientation_search import Candidates, poisson_score_inputs, refine_candidates
    cfg = dict(Nx=24, Ny=24, My=27, N_Omega=60, angle_range=[0, 180], cor_offset=0.0, N_eta=72,
               eta_angle_range=[0, 360], energy=12.398 / 0.3, k_direction_0=[0, 0, 1], p_direction_0=[1, 0, 0],
               detector_direction_origin=[0, -1, 0], detector_direction_positive_90=[0, 0, -1])
    mat = Material.from_lattice_parameters(a=4.05, symmetry_group="cubic", wavelength_A=0.3,
                                           hkl_list=[[1, 1, 1], [2, 0, 0], [2, 2, 0], [3, 1, 1]])
    U = Rotation.from_euler("zxz", [30, 40, 50], degrees=True).as_matrix()[None]
    truth = SinglePhaseForwardOperator(cfg, mat, MatrixGrid(U, np.deg2rad([1.0])), 0.1, normalized=True)
    x = np.zeros(truth.coeff_shape, np.float32)
    x[0, 8:16, 4:12] = 1.0                                     # the grain: tiles (2..3, 1..2) of 4-voxel tiles
    bg = np.float32(0.5)
    mu_true = truth.direct(torch.as_tensor(x, device="cuda")).cpu().numpy() * 200 + bg
    b = np.random.default_rng(3).poisson(mu_true).astype(np.float32)
    mu = np.full(b.shape, bg, np.float32)
    e, d = poisson_score_inputs(b, mu, 1.0, np.ones(truth.N_seg, np.float32))
    off = Rotation.from_rotvec(np.deg2rad([2.0, -1.5, 1.2])).as_matrix()
    cand = Candidates((U[0] @ off)[None], np.array([1.0]), [np.array([13, 14, 19, 20])], (6, 6))
    rows = np.ones(truth.N_Omega, bool)
    rows[::5] = False

    def make(rots, sigs, k, iy, ix):
        sup = LocalSupport(k, iy, ix, len(rots), (cfg["Ny"], cfg["Nx"]))
        return LocalSinglePhaseForwardOperator(cfg, mat, MatrixGrid(rots, sigs), 0.1, sup, normalized=True)

    out = refine_candidates(make, cand, e, d, rows, 4, (cfg["Ny"], cfg["Nx"]))
    mis = np.degrees(Rotation.from_matrix(U[0].T @ out.rotations[0]).magnitude())
    start = np.degrees(Rotation.from_matrix(U[0].T @ cand.rotations[0]).magnitude())
    assert mis < 0.6 < start, (start, mis)
    assert out.tiles is cand.tiles and np.array_equal(out.score, cand.score)
