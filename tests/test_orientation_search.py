"""The orientation search's candidate workflow on the CPU against the reference's own outputs
(tests/golden/search_candidates.npz, made by tests/golden/make_search_golden.py from the reference's
select_candidates, candidate_support, orientation_weights and prune_added on seeded synthetic top lists): the
candidates (orientations, scores, tiles) under three selection settings, the support of the strict candidates, the
orientation weights and the pruning masks, exactly."""
import numpy as np
import pytest

from conftest import GOLDEN


@pytest.fixture(scope="module")
def fx():
    return dict(np.load(GOLDEN / "search_candidates.npz"))


@pytest.mark.parametrize("name,kw", [("strict", {}), ("liberal", dict(ratio=1.5, min_tiles=1)),
                                     ("narrow", dict(sep_deg=3.0, link_deg=2.0, max_per_tile=2))])
def test_select_candidates_equals_the_reference(fx, name, kw):
    from diffractom_b200.orientation_search import select_candidates
    real = {"idx": fx["real_idx"], "z": fx["real_z"]}
    null = {"idx": fx["real_idx"], "z": fx["null_z"]}
    c = select_candidates(real, null, fx["rotations"], fx["pixels"], tuple(fx["tile_shape"]), fx["sym"], **kw)
    assert len(c) == len(fx[f"{name}_score"]) > 0
    assert np.array_equal(c.rotations, fx[f"{name}_rot"])
    np.testing.assert_allclose(c.score, fx[f"{name}_score"], rtol=1e-12)
    assert [len(t) for t in c.tiles] == list(fx[f"{name}_ntiles"])
    assert np.array_equal(np.concatenate(c.tiles), fx[f"{name}_tiles"])
    sub = c.subset(np.arange(len(c)) % 2 == 0)
    assert len(sub) == (len(c) + 1) // 2 and np.array_equal(sub.rotations, c.rotations[::2])


def test_support_weights_and_pruning_equal_the_reference(fx):
    from diffractom_b200.orientation_search import (candidate_support, orientation_weights, prune_added,
                                                    select_candidates)
    real = {"idx": fx["real_idx"], "z": fx["real_z"]}
    null = {"idx": fx["real_idx"], "z": fx["null_z"]}
    c = select_candidates(real, null, fx["rotations"], fx["pixels"], tuple(fx["tile_shape"]), fx["sym"])
    k, iy, ix = candidate_support(c, 4, tuple(fx["support_shape"]), dilate=2, mask=fx["support_mask"])
    for a, key in ((k, "support_k"), (iy, "support_iy"), (ix, "support_ix")):
        assert np.array_equal(a, fx[key])
    np.testing.assert_allclose(orientation_weights(fx["coeff"]), fx["weights_dense"], rtol=1e-13)
    np.testing.assert_allclose(orientation_weights(fx["coo_v"], k=fx["coo_k"]), fx["weights_coo"], rtol=1e-13)
    assert np.array_equal(prune_added(fx["weights_dense"], 4, rel=0.3), fx["prune"])
    w = np.r_[fx["weights_dense"][:4], np.zeros(5)]
    assert np.array_equal(prune_added(w, 4), fx["prune_none"])


def test_no_qualifying_peak_gives_no_candidate(fx):
    from diffractom_b200.orientation_search import select_candidates
    real = {"idx": fx["real_idx"], "z": fx["real_z"] * 0}
    null = {"idx": fx["real_idx"], "z": fx["null_z"]}
    c = select_candidates(real, null, fx["rotations"], fx["pixels"], tuple(fx["tile_shape"]), fx["sym"])
    assert len(c) == 0 and c.rotations.shape == (0, 3, 3)
