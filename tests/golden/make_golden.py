"""Generate the golden fixtures of the parity tests from the reference implementation (diffractom).

Usage: python tests/golden/make_golden.py <path of the reference's source tree> (required). The fixtures it writes
(tests/golden/*.npz) are committed, so the tests never need the reference.

The reference's device code is OpenCL (pyopencl), which is not installed here. Its host code is plain NumPy, so
the pyopencl modules are replaced by stubs and an operator object is assembled from the reference's own host
methods (SinglePhaseForwardOperator.__init__ steps: quadrature, material upload, detector_coordinates, grid upload,
transfer_pole_axes_to_gpu). The float64 ReferenceModel (diffractom/differentiable/reference.py) then gives the
pole-figure matrix, the forward model and its transpose. What is recorded per case:

  inputs   cfg, material description, rotation matrices and sigmas of the orientations, seeded coefficients c and
           data-shaped r
  geometry the reference's quadrature rule and nodes, probed directions (coords), pole axes / counts / starts,
           rotated poles, 1/sigma^2, norm factors, ring two-theta and intensities, projector geometry (X, Y, T0,
           weights, scale, taps) and the field-of-view support mask
  outputs  ReferenceModel.pf (R, K, C, P) float64, forward(c) and the coefficient gradient of <r, forward(c)>
           (= the adjoint applied to r); the gradients of <r, forward(c)> with respect to the PF parameters (rot,
           sigma, eta_offset, axis_tilt, two_theta) and the projector's (shift, cor), the probed directions'
           derivatives, and the forward at moved PF and projector parameters (the checks of the parameter updates)

Material fixtures record, for the materials of the benchmark configurations, the ring two-theta, the pole axes and
their counts, which the package's own Material must reproduce.
"""
import json
import sys
import warnings
from pathlib import Path
from unittest import mock

import numpy as np

if len(sys.argv) < 2:
    sys.exit("usage: make_golden.py <path of the reference's source tree (the directory holding src/diffractom)>")
REF = Path(sys.argv[1])
OUT = Path(__file__).resolve().parent

for m in ["pyopencl", "pyopencl.array", "pyopencl.tools", "pyopencl.scan", "pyopencl.elementwise",
          "pyopencl.reduction", "pyopencl.clrandom", "pyopencl.cltypes", "pyopencl.clmath", "pyopencl.characterize",
          "gratopy", "pyclblast", "pyvkfft", "pyvkfft.opencl", "h5py"]:
    sys.modules[m] = mock.MagicMock()
# host copies in place of device arrays: every "upload" of the reference's host code returns the array itself
sys.modules["pyopencl.array"].to_device = lambda queue, a, *args, **kw: np.array(a)
sys.modules["pyopencl"].array = sys.modules["pyopencl.array"]
sys.path.insert(0, str(REF / "src"))
warnings.filterwarnings("ignore")

from diffractom import Grid, Material  # noqa: E402
from diffractom.crystallography.intensity import as_intensity_model, group_reflections_into_rings  # noqa: E402
from diffractom.differentiable.reference import ReferenceModel  # noqa: E402
from diffractom.operators.parallel_radon import ParallelRadon  # noqa: E402
from diffractom.operators.quadrature import grid_sigma_min, setup_quadrature  # noqa: E402
from diffractom.operators.single_phase_forward_operator import SinglePhaseForwardOperator  # noqa: E402
from diffractom.utils.support import fov_support_mask  # noqa: E402


def host_operator(cfg, mat, grid, quadrature="auto", kernel="trapezoid", pf_cutoff_sigma=4.0, rings=None,
                  reflection_two_theta=False):
    """A SinglePhaseForwardOperator with its host state only (the steps of __init__ that run on the host)."""
    op = SinglePhaseForwardOperator.__new__(SinglePhaseForwardOperator)
    op.reserve_coefficient_arrays = 3
    op.pf_cutoff_sigma = pf_cutoff_sigma
    op.sparse_batch_max = 1024
    op.pf_cut_options = []
    op.ctx, op.queue = mock.MagicMock(), mock.MagicMock()
    op.queue.device.max_mem_alloc_size = 1 << 40
    op.cfg = dict(cfg)
    op.normalized = True
    op.intensity_model = as_intensity_model(None)
    op.material, op.grid, op.verbose = mat, grid, False
    op.N_eta = op.cfg["N_eta"]
    if rings is None:
        op.ring_reflections = group_reflections_into_rings(mat)
        op.ring_overlap = [np.ones(len(r)) for r in op.ring_reflections]
    else:
        op.ring_reflections = [np.asarray(ix, dtype=np.int64) for ix, _ in rings]
        op.ring_overlap = [np.asarray(w, dtype=np.float64) for _, w in rings]
    op._custom_rings, op._ring_two_theta = rings is not None, None
    op.reflection_two_theta = bool(reflection_two_theta)
    op.N_peaks = len(op.ring_reflections)
    op.N_seg = op.N_peaks * op.N_eta
    op.Nx, op.Ny, op.My, op.N_Omega = cfg["Nx"], cfg["Ny"], cfg["My"], cfg["N_Omega"]
    op.cor_offset = cfg["cor_offset"]
    op.voxel_size, op.image_width = None, float(op.Nx)
    op.angle_range = np.array(cfg["angle_range"]) / 180 * np.pi
    delta = (op.angle_range[1] - op.angle_range[0]) / op.N_Omega
    op.angles = np.linspace(op.angle_range[0], op.angle_range[1], op.N_Omega, endpoint=False) + delta / 2
    op.eta_angle_range = np.array(cfg.get("eta_angle_range", [0, 360])) / 180 * np.pi
    ed = (op.eta_angle_range[1] - op.eta_angle_range[0]) / op.N_eta
    op.eta_angles = np.linspace(op.eta_angle_range[0], op.eta_angle_range[1], op.N_eta, endpoint=False) + ed / 2
    setup_quadrature(op, quadrature, 0.05, grid_sigma_min(grid))
    op.transfer_material_parameters_to_gpu()
    op.detector_coordinates()
    op.transfer_grid_parameters_to_gpu()
    op.transfer_pole_axes_to_gpu()
    op.projector, op.radon_kernel = "native", kernel
    return op


def radon_geometry(op):
    """The reference ParallelRadon's geometry for the operator's arguments (SinglePhaseForwardOperator:478-490):
    geo (R, 4) = (X, Y, T0, angle weight) float32, the forward scale and the number of taps."""
    pr = ParallelRadon(op.queue, (op.Nx, op.Ny), op.angles, op.My, image_width=op.image_width, detector_width=op.My,
                       detector_shift=op.cor_offset, angle_weights=np.pi / op.N_Omega, bins_per_item=3,
                       tiled=False, kernel=op.radon_kernel)
    return np.asarray(pr.geo_gpu, np.float32), np.float32(pr.scale), int(pr.n_taps)


def material_record(mat, cfg_energy):
    """The pole axes of every ring as the reference's operator builds them."""
    cfg = {"Nx": 4, "Ny": 4, "My": 5, "N_Omega": 4, "angle_range": [0, 180], "cor_offset": 0.0, "N_eta": 8,
           "eta_angle_range": [0, 360], "energy": cfg_energy, "k_direction_0": [0, 0, 1], "p_direction_0": [1, 0, 0],
           "detector_direction_origin": [0, -1, 0], "detector_direction_positive_90": [0, 0, -1]}
    grid = Grid.from_rotation_matrices(np.eye(3)[None], np.deg2rad(3.0))
    op = host_operator(cfg, mat, grid, quadrature="midpoint")
    return dict(two_theta=np.asarray(op.two_theta_peaks, np.float32), axes=np.asarray(op.pole_axes_cpu, np.float64),
                counts=np.asarray(op.axis_count_cpu, np.float32), start=np.asarray(op.axis_start_cpu, np.int32),
                point_group=np.asarray(mat.point_group_matrices, np.float32),
                h_first=np.asarray(op.h_cpu, np.float32))


def case(name, cfg, mat_spec, n_orient, sigma_deg, grid_seed, quadrature="auto", kernel="trapezoid", seed=0,
         probed=False, with_moved=True):
    mat = Material.from_lattice_parameters(**mat_spec)
    np.random.seed(grid_seed)
    grid = Grid.from_random_fundamental_zone(n_orient, mat_spec["symmetry_group"], np.deg2rad(sigma_deg))
    op = host_operator(cfg, mat, grid, quadrature, kernel)
    ref = ReferenceModel(op)
    prm = ref.params0()
    rng = np.random.default_rng(seed)
    K, Ny, Nx = op.K, op.Ny, op.Nx
    supp = fov_support_mask(Nx, Ny, op.My, angles=op.angles, image_width=op.image_width, detector_width=op.My,
                            detector_shift=op.cor_offset)
    c = (rng.random((K, Ny, Nx)) * supp[None]).astype(np.float32)
    r = rng.random((op.N_Omega, op.My, op.N_seg)).astype(np.float32)
    pf = ref.pf(prm)
    fwd = ref.forward(c, prm)
    adj = ref.vjp(c, prm, r, groups=("c",))["c"]
    pf_groups = ("rot", "sigma", "eta_offset", "axis_tilt", "two_theta")
    grads = ref.vjp(c, prm, r, groups=pf_groups + ("shift", "cor"))
    dv = ref.probed_derivatives(prm)
    moved = ref.params0()
    moved["rot"] = rng.normal(0, 0.02, (K, 3))
    moved["sigma"] = moved["sigma"] * 1.1
    moved["two_theta"] = moved["two_theta"] + 0.001
    moved["eta_offset"] = 0.01
    moved["axis_tilt"] = np.array([0.01, -0.02])
    fwd_pf_moved = ref.forward(c, moved)
    proj = ref.params0()
    proj["cor"] = proj["cor"] + 0.3
    proj["shift"] = rng.normal(0, 0.4, op.N_Omega)
    fwd_proj_moved = ref.forward(c, proj)
    geo, scale, n_taps = radon_geometry(op)
    rule = op.quadrature
    mat_json = {k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in mat_spec.items()}
    out = dict(
        cfg=json.dumps(cfg), material=json.dumps(mat_json), kernel=kernel, quadrature=quadrature,
        rot=np.asarray(op.grid_rot_cpu, np.float64), sigma=np.asarray(op.sigma_cpu, np.float32),
        sigma64=np.array([n.sigma for n in grid.nodes], np.float64),
        c=c, r=r,
        rule=np.array([rule.p_omega, rule.k_omega, rule.p_eta, rule.k_eta], np.int32),
        angles_sub=np.asarray(op.angles_subdivided, np.float64), eta_sub=np.asarray(op.eta_angles_subdivided, np.float64),
        quad_w=(np.zeros(0, np.float32) if op.quad_weights_cpu is None else np.asarray(op.quad_weights_cpu, np.float32)),
        coords=np.asarray(op.coords_cpu, np.float32), two_theta=np.asarray(op.two_theta_peaks, np.float32),
        axes=np.asarray(op.pole_axes_cpu, np.float64), counts=np.asarray(op.axis_count_cpu, np.float32),
        start=np.asarray(op.axis_start_cpu, np.int32),
        poles=np.asarray(op.poles_gpu, np.float32),
        inv_sigma2=(1.0 / (op.sigma_cpu * op.sigma_cpu)).astype(np.float32),
        norm=(1.0 / (8.0 * np.pi * op.sigma_cpu * op.sigma_cpu)).astype(np.float32),
        intens=np.asarray(op.intens_cpu, np.float32),
        geo=geo, scale=np.float32(scale), n_taps=np.int32(n_taps), support=supp,
        pf=pf, fwd=fwd, adj=adj,
        g_rot=grads["rot"], g_sigma=grads["sigma"], g_eta_offset=np.float64(grads["eta_offset"]),
        g_axis_tilt=grads["axis_tilt"], g_two_theta=grads["two_theta"], g_shift=grads["shift"],
        g_cor=np.float64(grads["cor"]),
    )
    if with_moved:      # the forward at moved parameters, float32 (the checks' tolerance is 2e-5 of the maximum)
        out.update(moved_rot=moved["rot"], moved_sigma=moved["sigma"], moved_two_theta=moved["two_theta"],
                   fwd_pf_moved=fwd_pf_moved.astype(np.float32), moved_cor=np.float64(proj["cor"]),
                   moved_shift=proj["shift"], fwd_proj_moved=fwd_proj_moved.astype(np.float32))
    if probed:          # the probed directions' derivatives (coords-shaped), float32 as they reach the device
        out.update(dv_eta=dv["eta_offset"].astype(np.float32), dv_tilt0=dv[("axis_tilt", 0)].astype(np.float32),
                   dv_tilt1=dv[("axis_tilt", 1)].astype(np.float32), dv_tth=dv["two_theta"].astype(np.float32))
    np.savez_compressed(OUT / f"{name}.npz", **out)
    print(f"{name}: K={K} R={op.N_Omega} My={op.My} C={op.N_eta} P={op.N_peaks} rule={rule} "
          f"fill={np.mean(pf != 0):.3f}")


BASE = {"k_direction_0": [0, 0, 1], "p_direction_0": [1, 0, 0], "detector_direction_origin": [0, -1, 0],
        "detector_direction_positive_90": [0, 0, -1], "eta_angle_range": [0, 360]}
AL3 = dict(a=4.05, b=4.05, c=4.05, alpha=90, beta=90, gamma=90, symmetry_group="cubic", wavelength_A=0.35,
           hkl_list=np.array([[1, 1, 1], [2, 0, 0], [2, 2, 0]]))
AL5 = dict(a=4.05, b=4.05, c=4.05, alpha=90, beta=90, gamma=90, symmetry_group="cubic", wavelength_A=0.3,
           hkl_list=np.array([[1, 1, 1], [2, 0, 0], [2, 2, 0], [3, 1, 1], [2, 2, 2]]))
TI8 = dict(a=2.95, b=2.95, c=4.68, alpha=90, beta=90, gamma=120, symmetry_group="hexagonal", wavelength_A=0.3,
           hkl_list=np.array([[1, 0, 0], [0, 0, 2], [1, 0, 1], [1, 0, 2], [1, 1, 0], [1, 0, 3], [2, 0, 0],
                              [1, 1, 2]]))
FE5 = dict(a=2.87, b=2.87, c=2.87, alpha=90, beta=90, gamma=90, symmetry_group="cubic", wavelength_A=0.3,
           hkl_list=np.array([[1, 1, 0], [2, 0, 0], [2, 1, 1], [2, 2, 0], [3, 1, 0]]))
NI6 = dict(a=3.52, b=3.52, c=3.52, alpha=90, beta=90, gamma=90, symmetry_group="cubic", wavelength_A=0.3,
           hkl_list=np.array([[1, 1, 1], [2, 0, 0], [2, 2, 0], [3, 1, 1], [2, 2, 2], [4, 0, 0]]))


def main():
    # the geometry of the reference's tests/test_differentiable.py (two quadrature / kernel variants)
    diff = {**BASE, "Nx": 14, "Ny": 12, "My": 17, "N_Omega": 16, "angle_range": [0, 360], "cor_offset": 0.7,
            "N_eta": 24, "energy": 12.398 / 0.35}
    case("diff_auto_trapezoid", diff, AL3, 12, 6.0, 5, "auto", "trapezoid", seed=0, probed=True)
    case("diff_midpoint_hat", diff, AL3, 12, 6.0, 5, "midpoint", "hat", seed=0)
    # the geometry of tests/test_adjoint.py, every angle range it tests (a decreasing one too)
    for lo, hi in ((0, 180), (0, 360), (0, 90), (180, 0)):
        adj = {**BASE, "Nx": 16, "Ny": 16, "My": 17, "N_Omega": 30, "angle_range": [lo, hi], "cor_offset": 0.5,
               "N_eta": 36, "energy": 12.398 / 0.35}
        case(f"adj_{lo}_{hi}", adj, AL3, 12, 4.0, 0, "auto", "trapezoid", seed=1)
    # a reduced version of the cubic-Al configuration (5 rings, half rotation, sigma 3 deg, midpoint rule)
    al = {**BASE, "Nx": 33, "Ny": 33, "My": 35, "N_Omega": 60, "angle_range": [0, 180], "cor_offset": 0.0,
          "N_eta": 60, "energy": 12.398 / 0.3}
    case("al5_small", al, AL5, 16, 3.0, 3, "auto", "trapezoid", seed=2, with_moved=False)
    # non-square image, hexagonal Ti, pixels smaller than the bins do not occur here (image width = Nx bins)
    ti = {**BASE, "Nx": 20, "Ny": 26, "My": 27, "N_Omega": 24, "angle_range": [0, 180], "cor_offset": -0.3,
          "N_eta": 48, "energy": 12.398 / 0.3}
    case("ti8_small", ti, TI8, 10, 5.0, 4, "auto", "trapezoid", seed=3, probed=True)

    mats = {}
    for name, spec in (("al5", AL5), ("ti8", TI8), ("fe5", FE5), ("ni6", NI6), ("al3", AL3)):
        rec = material_record(Material.from_lattice_parameters(**spec), 12.398 / spec["wavelength_A"])
        for k, v in rec.items():
            mats[f"{name}_{k}"] = v
    np.savez_compressed(OUT / "materials.npz", **mats)
    print("materials:", sorted({k.split("_")[0] for k in mats}))




def axis_case(name="refl_windows"):
    """reflection_two_theta with windows of reflections of different Bragg angles (the geometry and material of the
    reference's tests/test_reflection_two_theta.py): the operator model's PF, forward and adjoint, and the probed
    u, w and axis angles."""
    from scipy.spatial.transform import Rotation
    from diffractom import MatrixGrid
    cfg = {**BASE, "Nx": 14, "Ny": 12, "My": 17, "N_Omega": 16, "angle_range": [0, 360], "cor_offset": 0.7,
           "N_eta": 36, "energy": 12.398 / 0.35}
    spec = dict(a=8.1, b=12.8, c=7.1, alpha=94, beta=116, gamma=88, crystal_system="triclinic", wavelength_A=0.35,
                hkl_list=np.array([[1, 0, 0], [0, 1, 0], [1, 1, 0], [1, -1, 0], [0, 0, 1], [1, 0, 1]]))
    windows = [([0, 1], [1.0, 0.6]), ([2, 3], [0.5, 1.0]), ([4], [1.0])]
    mat = Material.from_lattice_parameters(**spec)
    rot = Rotation.random(10, random_state=5).as_matrix()
    grid = MatrixGrid(rot, np.full(10, np.deg2rad(3.0)))
    op = host_operator(cfg, mat, grid, "auto", "trapezoid", rings=windows, reflection_two_theta=True)
    ref = ReferenceModel(op)
    prm = ref.params0()
    rng = np.random.default_rng(7)
    supp = fov_support_mask(op.Nx, op.Ny, op.My, angles=op.angles, image_width=op.image_width, detector_width=op.My,
                            detector_shift=op.cor_offset)
    c = (rng.random((op.K, op.Ny, op.Nx)) * supp[None]).astype(np.float32)
    r = rng.random((op.N_Omega, op.My, op.N_seg)).astype(np.float32)
    rule = op.quadrature
    mat_json = {k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in spec.items()}
    out = dict(cfg=json.dumps(cfg), material=json.dumps(mat_json), rings=json.dumps(windows), kernel="trapezoid",
               quadrature="auto", rot=np.asarray(op.grid_rot_cpu, np.float64), sigma=np.asarray(op.sigma_cpu, np.float32),
               sigma64=np.full(10, np.deg2rad(3.0)), c=c, r=r,
               rule=np.array([rule.p_omega, rule.k_omega, rule.p_eta, rule.k_eta], np.int32),
               coords=np.asarray(op.coords_cpu, np.float32), w=np.asarray(op.w_cpu, np.float32),
               two_theta=np.asarray(op.two_theta_peaks, np.float32),
               axis_two_theta=np.asarray(op.axis_two_theta_cpu, np.float64),
               axes=np.asarray(op.pole_axes_cpu, np.float64), counts=np.asarray(op.axis_count_cpu, np.float32),
               start=np.asarray(op.axis_start_cpu, np.int32), support=supp,
               pf=ref.pf(prm), fwd=ref.forward(c, prm), adj=ref.vjp(c, prm, r, groups=("c",))["c"])
    grads = ref.vjp(c, prm, r, groups=("rot", "sigma", "eta_offset", "axis_tilt", "two_theta"))
    out.update(g_rot=grads["rot"], g_sigma=grads["sigma"], g_eta_offset=np.float64(grads["eta_offset"]),
               g_axis_tilt=grads["axis_tilt"], g_two_theta=grads["two_theta"])
    np.savez_compressed(OUT / f"{name}.npz", **out)
    print(f"{name}: K={op.K} R={op.N_Omega} C={op.N_eta} P={op.N_peaks} axes={op.N_axes}")



if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[2] == "axis":       # only the reflection_two_theta case
        axis_case()
    else:
        main()
        axis_case()
