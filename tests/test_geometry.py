"""Host set-up of the operator against the reference's own host code (golden fixtures): quadrature rule and nodes,
ring two-theta, probed directions, pole axes and counts, rotated poles, kernel factors, projector geometry and
field-of-view mask, bit for bit; the package's Material against the reference's for the benchmark materials."""
import numpy as np
import pytest

from conftest import CASES, GOLDEN, case_geometry


@pytest.mark.parametrize("name", CASES)
def test_geometry_matches_reference(golden, name):
    d = golden(name)
    g = case_geometry(d)
    r = g.quadrature
    assert [r.p_omega, r.k_omega, r.p_eta, r.k_eta] == d["rule"].tolist()
    assert np.array_equal(g.angles_subdivided, d["angles_sub"])
    assert np.array_equal(g.eta_angles_subdivided, d["eta_sub"])
    if d["quad_w"].size == 0:
        assert g.quad_weights_cpu is None
    else:
        assert np.array_equal(g.quad_weights_cpu, d["quad_w"])
    assert np.array_equal(g.two_theta_peaks, d["two_theta"])
    assert np.array_equal(g.coords_cpu, d["coords"])
    assert np.array_equal(g.pole_axes_cpu, d["axes"])
    assert np.array_equal(g.axis_count_cpu, d["counts"])
    assert np.array_equal(g.axis_start_cpu, d["start"])
    assert np.array_equal(g.poles_cpu, d["poles"])
    assert np.array_equal(g.inv_sigma2_cpu, d["inv_sigma2"])
    assert np.array_equal(g.norm_factor_cpu, d["norm"])
    assert np.array_equal(g.radon_geo.geo, d["geo"])
    assert g.radon_geo.scale == d["scale"] and g.radon_geo.n_taps == int(d["n_taps"])
    assert np.array_equal(g.support_mask(), d["support"])


MATS = {
    "al5": dict(a=4.05, symmetry_group="cubic", wavelength_A=0.3,
                hkl_list=[[1, 1, 1], [2, 0, 0], [2, 2, 0], [3, 1, 1], [2, 2, 2]]),
    "al3": dict(a=4.05, symmetry_group="cubic", wavelength_A=0.35, hkl_list=[[1, 1, 1], [2, 0, 0], [2, 2, 0]]),
    "ti8": dict(a=2.95, c=4.68, gamma=120, symmetry_group="hexagonal", wavelength_A=0.3,
                hkl_list=[[1, 0, 0], [0, 0, 2], [1, 0, 1], [1, 0, 2], [1, 1, 0], [1, 0, 3], [2, 0, 0], [1, 1, 2]]),
    "fe5": dict(a=2.87, symmetry_group="cubic", wavelength_A=0.3,
                hkl_list=[[1, 1, 0], [2, 0, 0], [2, 1, 1], [2, 2, 0], [3, 1, 0]]),
    "ni6": dict(a=3.52, symmetry_group="cubic", wavelength_A=0.3,
                hkl_list=[[1, 1, 1], [2, 0, 0], [2, 2, 0], [3, 1, 1], [2, 2, 2], [4, 0, 0]]),
}


@pytest.mark.parametrize("name", sorted(MATS))
def test_material_matches_reference(name):
    from diffractom_b200.geometry import pole_axes
    from diffractom_b200.material import Material, group_reflections_into_rings
    ref = np.load(GOLDEN / "materials.npz")
    mat = Material.from_lattice_parameters(**MATS[name])
    rings = group_reflections_into_rings(mat)
    pa = pole_axes(mat, rings, [np.ones(len(r)) for r in rings])
    assert {tuple(np.round(m, 6)) for m in ref[f"{name}_point_group"]} == \
        {tuple(np.round(m, 6)) for m in mat.point_group_matrices}
    assert np.array_equal(pa.axes, ref[f"{name}_axes"])
    assert np.array_equal(pa.counts, ref[f"{name}_counts"])
    assert np.array_equal(pa.start, ref[f"{name}_start"])
    assert np.allclose(np.asarray(mat.h_vecs, np.float32)[[r[0] for r in rings]], ref[f"{name}_h_first"])


def test_group_orders_and_closure():
    from diffractom_b200.material import hkl_group, rotation_group
    for system, order in (("triclinic", 1), ("monoclinic", 2), ("orthorhombic", 4), ("tetragonal", 8),
                          ("trigonal", 6), ("hexagonal", 12), ("cubic", 24)):
        G = rotation_group(system)
        assert len(G) == order and len(hkl_group(system)) == order
        assert np.allclose(np.einsum("gij,gkj->gik", G, G), np.eye(3))          # orthogonal
        assert np.allclose(np.linalg.det(G), 1.0)                                # proper


def test_interleaved_subsets_and_errors():
    from diffractom_b200.geometry import interleaved_subsets
    s = interleaved_subsets(10, 3)
    assert [list(a) for a in s] == [[0, 3, 6, 9], [1, 4, 7], [2, 5, 8]]
    with pytest.raises(ValueError):
        interleaved_subsets(4, 5)


def test_reflection_two_theta_geometry_matches_reference(golden):
    """reflection_two_theta with windows of reflections at different Bragg angles: the probed u and w, every axis's
    Bragg angle and the windows' mean two-theta equal the reference's."""
    import json
    from diffractom_b200.geometry import OperatorGeometry
    from diffractom_b200.grid import MatrixGrid
    from diffractom_b200.material import Material
    d = golden("refl_windows")
    rings = [(ix, w) for ix, w in json.loads(str(d["rings"]))]
    mat = Material.from_lattice_parameters(**d["material"])
    g = OperatorGeometry(d["cfg"], mat, MatrixGrid(d["rot"], d["sigma64"]), normalized=True,
                         quadrature=d["quadrature"], radon_kernel=d["kernel"], rings=rings,
                         reflection_two_theta=True)
    assert np.array_equal(g.two_theta_peaks, d["two_theta"])
    assert np.abs(g.coords_cpu - d["coords"]).max() <= 2e-7 and np.abs(g.w_cpu - d["w"]).max() <= 2e-7
    assert np.array_equal(g.axis_start_cpu, d["start"]) and np.allclose(g.pole_axes_cpu, d["axes"], atol=1e-12)
    assert np.allclose(g.axis_two_theta_cpu, d["axis_two_theta"], rtol=0, atol=1e-14)
    assert len(np.unique(np.round(g.axis_two_theta_cpu[d["start"][0]:d["start"][1]], 9))) == 2   # two angles in a window
