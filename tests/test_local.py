"""The local basis on the CPU: LocalSupport (sorting, dilation, restriction, union, masks) and build_patches (one box
per orientation, clusters of scattered voxels, merged boxes, the flat coefficient layout and its mask)."""
import numpy as np
import pytest

from diffractom_b200.local import LocalSupport, _merge_boxes, build_patches


def test_support_is_sorted_unique_and_converts():
    s = LocalSupport([2, 0, 2, 0], [1, 3, 1, 0], [4, 2, 4, 1], 3, (5, 6))
    assert s.n_pairs == 3 and list(s.k) == [0, 0, 2] and list(s.iy) == [0, 3, 1]
    m = s.to_mask()
    assert m.sum() == 3 and LocalSupport.from_mask(m).n_pairs == 3
    assert LocalSupport.everywhere(2, (3, 4)).n_pairs == 24
    d = s.dilate(1)
    assert d.to_mask()[s.k, s.iy, s.ix].all() and d.n_pairs > s.n_pairs
    r = d.restrict(np.arange(30).reshape(5, 6) % 2 == 0)
    assert np.all((r.iy * 6 + r.ix) % 2 == 0)
    assert s.union(d).n_pairs == d.n_pairs and s.per_voxel().sum() == 3
    with pytest.raises(ValueError):
        LocalSupport([3], [0], [0], 3, (5, 6))


def test_patches_cover_the_pairs_once():
    rng = np.random.default_rng(0)
    K, shape = 6, (40, 44)
    mask = np.zeros((K,) + shape, bool)
    mask[0, 5:12, 7:20] = True                                  # one compact block
    mask[1, 2:6, 3:8] = True                                    # two far apart blocks: split into two patches
    mask[1, 30:36, 35:41] = True
    mask[2] = rng.random(shape) < 0.02                          # scattered voxels
    mask[4, 10, 10] = True
    s = LocalSupport.from_mask(mask)
    P = build_patches(s.k, s.iy, s.ix, K)
    assert (P["pk"] == 1).sum() == 2 and (P["pk"] == 0).sum() == 1 and (P["pk"] == 4).sum() == 1
    assert np.all(np.diff(P["pk"]) >= 0) and int(P["mask"].sum()) == s.n_pairs
    # every pair's coefficient lies in its orientation's patch at its position
    for j in range(s.n_pairs):
        c = P["pair_index"][j]
        p = np.searchsorted(P["coff"], c, side="right") - 1
        off = c - P["coff"][p]
        assert P["pk"][p] == s.k[j]
        assert P["y0"][p] + off // P["w"][p] == s.iy[j] and P["x0"][p] + off % P["w"][p] == s.ix[j]
    one = build_patches(s.k, s.iy, s.ix, K, split=False)
    assert len(one["pk"]) == len(s.orientations_used()) and one["n_coef"] >= P["n_coef"]


def test_merge_boxes_merges_overlaps():
    out = sorted(_merge_boxes([[0, 4, 0, 4], [3, 8, 3, 8], [20, 21, 20, 21], [7, 9, 0, 1]]))
    assert out == [[0, 9, 0, 8], [20, 21, 20, 21]]


def test_split_regions():
    """Components, tiles and both: every region of an orientation becomes a copy (parent), the copies' voxels are
    exactly the original pairs, regions below min_pairs are dropped."""
    from diffractom_b200.local import LocalSupport, split_regions
    K, Ny, Nx = 3, 12, 10
    m = np.zeros((K, Ny, Nx), bool)
    m[0, 1:3, 1:3] = True          # two 8-connected components
    m[0, 7:10, 6:9] = True
    m[1, 2, 2] = m[1, 3, 3] = True  # diagonal neighbours: one component
    m[2, 0:12, 4] = True           # a column crossing tiles
    sup = LocalSupport.from_mask(m)
    mats = np.stack([np.eye(3) * (i + 1) for i in range(K)])
    sig = np.arange(K, dtype=np.float64) + 0.1
    m2, s2, sp, parent = split_regions(mats, sig, sup, mode="components")
    assert list(parent) == [0, 0, 1, 2] and np.array_equal(m2, mats[parent]) and np.array_equal(s2, sig[parent])
    back = np.zeros_like(m)
    for k2, y, x in zip(sp.k, sp.iy, sp.ix):
        back[parent[k2], y, x] = True
    assert np.array_equal(back, m)
    # 4 x 4 tiles: orientation 0's blobs cover tile (0, 0) and tiles (1..2, 1..2); orientation 2's column 3 tiles
    _, _, sp_t, par_t = split_regions(mats, sig, sup, mode="tiles", tile=4)
    assert list(par_t) == [0] * 5 + [1] + [2] * 3
    _, _, sp_c, par_c = split_regions(mats, sig, sup, mode="components+tiles", tile=4)
    assert list(par_c) == [0] * 5 + [1] + [2] * 3
    assert sp_c.n_pairs == sup.n_pairs
    _, _, sp_m, par_m = split_regions(mats, sig, sup, mode="components", min_pairs=3)
    assert list(par_m) == [0, 0, 2]
    with pytest.raises(ValueError):
        split_regions(mats, sig, sup, mode="rings")
