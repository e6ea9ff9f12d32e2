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
