"""OrientationTree (the nested cells of the hierarchical total variation) as the reference's
tests/test_tree_tv.py:18-35 checks it: a symmetric copy of an orientation falls in its cell at every level, the cells
nest, edges and leaf edge follow the radii; and the node-pixel arrays the solver's tree kernels use against a
construction pixel by pixel and against the explicit penalty rows. CPU only."""
import numpy as np
import pytest

pytest.importorskip("scipy")


def _rotations(n=40, seed=0):
    from scipy.spatial.transform import Rotation
    rng = np.random.default_rng(seed)
    base = Rotation.random(n, random_state=seed + 1)
    return (base * Rotation.from_rotvec(np.radians(rng.normal(0, 1.0, (n, 3))))).as_matrix()


def _four_fold():
    from scipy.spatial.transform import Rotation
    return Rotation.from_euler("z", np.array([[0.0], [90.0], [180.0], [270.0]]), degrees=True).as_matrix()


def test_cells_nest_and_respect_symmetry():
    from diffractom_b200 import OrientationTree
    R = _rotations()
    S = _four_fold()
    R2 = np.concatenate([R, (R[0] @ S[1])[None]])          # a symmetric copy of the first orientation
    t = OrientationTree(R2, S, (30.0, 10.0, 3.0))
    assert [len(c) for c in t.nodes] == [41] * 3
    for cell in t.nodes:
        assert cell[0] == cell[-1]
    for fine, coarse in zip(t.nodes[1:], t.nodes[:-1]):
        assert all(len(np.unique(coarse[fine == c])) == 1 for c in np.unique(fine))
    assert t.edges == [0.0, 10.0, 3.5] and t.leaf_edge == 1.5
    assert t.n_nodes[0] <= t.n_nodes[1] <= t.n_nodes[2]
    assert [lv[1] for lv in t.levels()] == [10.0, 3.5]
    for cell, m in zip(t.nodes, t.n_nodes):                 # labels 0..m-1, all used
        assert np.array_equal(np.unique(cell), np.arange(m))


def test_cells_have_the_radius():
    """Every orientation lies within twice the radius of its cell's other members' centre: two members of a cell are
    at most 2 r apart (through symmetry); without symmetry far orientations never share a cell of a small radius."""
    from scipy.spatial.transform import Rotation
    from diffractom_b200 import OrientationTree
    R = _rotations(60, seed=3)
    t = OrientationTree(R, None, (20.0, 5.0))
    rot = Rotation.from_matrix(R)
    for cell, r in zip(t.nodes, t.radii):
        for c in np.unique(cell):
            ids = np.flatnonzero(cell == c)
            d = np.degrees((rot[ids[:, None]].inv() * rot[ids[None, :]]).magnitude()) if len(ids) > 1 else 0
            assert np.max(d) <= 2 * r + 1e-9


def test_single_radius_has_no_levels_and_bad_radii_raise():
    from diffractom_b200 import OrientationTree
    R = _rotations(10)
    t = OrientationTree(R, None, (4.0,))
    assert t.levels() == [] and t.leaf_edge == 2.0
    assert len(OrientationTree(R, None, (4.0,), top_edge=1.0).levels()) == 1
    for radii in ((), (3.0, 3.0), (2.0, 5.0), (-1.0,)):
        with pytest.raises(ValueError):
            OrientationTree(R, None, radii)
    with pytest.raises(ValueError):
        OrientationTree(R[:, :2], None, (4.0,))


def test_tree_level_arrays_against_pixelwise_construction():
    from diffractom_b200 import OrientationTree
    from diffractom_b200.orientation_tree import tree_level_arrays
    rng = np.random.default_rng(5)
    K, Ny, Nx = 12, 7, 9
    R = _rotations(K, seed=7)
    tree = OrientationTree(R, None, (150.0, 90.0, 40.0), top_edge=2.0)
    mask = rng.random((K, Ny, Nx)) < 0.4
    k, iy, ix = np.nonzero(mask)
    pi = rng.permutation(len(k))                            # flat positions in some patch order
    n = len(k) + 3                                          # padding coefficients outside every node-pixel
    T = rng.random(n).astype(np.float32)
    levels = tree_level_arrays(k, iy, ix, pi, Ny, Nx, n, T, tree)
    assert [lv["edge"] for lv in levels] == [e for _, e in tree.levels()]
    for lev, (cell, _) in zip(levels, tree.levels()):
        members = {}
        for kk, yy, xx, j in zip(k, iy, ix, pi):
            members.setdefault((int(cell[kk]), int(yy), int(xx)), []).append(int(j))
        keys = sorted(members)
        assert lev["n"] == len(keys)
        pos = {key: i for i, key in enumerate(keys)}
        for i, key in enumerate(keys):
            js = lev["idx"][lev["ptr"][i]:lev["ptr"][i + 1]]
            assert list(js) == members[key]                 # the support's pair order
            assert np.all(lev["map"][js] == i)
            assert lev["A"][i] == np.float32(np.sum(T[members[key]].astype(np.float64)))
            c, y, x = key
            for name, (dy, dx) in (("right", (0, 1)), ("down", (1, 0)), ("left", (0, -1)), ("up", (-1, 0))):
                assert lev[name][i] == pos.get((c, y + dy, x + dx), -1), (name, key)
        assert np.count_nonzero(lev["map"] >= 0) == len(k)
        for a in ("ptr", "idx", "map", "right", "down", "left", "up"):
            assert lev[a].dtype == np.int32


def test_level_arrays_give_the_explicit_penalty():
    """The penalty of the tree levels computed on the node-pixel arrays (sums over the CSR lists, differences to the
    right / down neighbours, edge-weighted norms) equals the norms of the explicit penalty rows of the GPU test, on
    random coefficients with every coefficient free."""
    from test_gpu_tree_tv import _tree_rows
    from diffractom_b200 import OrientationTree
    from diffractom_b200.orientation_tree import tree_level_arrays
    rng = np.random.default_rng(11)
    K, Ny, Nx = 10, 6, 7
    tree = OrientationTree(_rotations(K, seed=2), None, (150.0, 80.0, 30.0))
    mask = rng.random((K, Ny, Nx)) < 0.5
    k, iy, ix = np.nonzero(mask)
    n = len(k)
    pi = rng.permutation(n)
    x = rng.random(n)
    levels = tree_level_arrays(k, iy, ix, pi, Ny, Nx, n, np.ones(n, np.float32), tree)
    got = 0.0
    for lev in levels:
        s = np.array([x[lev["idx"][lev["ptr"][j]:lev["ptr"][j + 1]]].sum() for j in range(lev["n"])])
        gx = np.where(lev["right"] >= 0, s[np.maximum(lev["right"], 0)] - s, 0.0)
        gy = np.where(lev["down"] >= 0, s[np.maximum(lev["down"], 0)] - s, 0.0)
        got += lev["edge"] * np.hypot(gx, gy).sum()
    D = _tree_rows(k, iy, ix, pi, Ny, Nx, n, tree, np.ones(n, bool))
    leaf_rows = 2 * K * Ny * Nx                              # the leaf level's rows come first
    g = (D @ x)[leaf_rows:].reshape(-1, 2)
    assert abs(np.hypot(g[:, 0], g[:, 1]).sum() - got) <= 1e-12 * got
