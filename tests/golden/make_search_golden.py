"""Golden fixture of the orientation search's candidate workflow (tests/golden/search_candidates.npz).

Usage: python tests/golden/make_search_golden.py <path of the reference's source tree> (required). The reference's
select_candidates, candidate_support, orientation_weights and prune_added are NumPy / SciPy code; they run here with
the pyopencl modules stubbed, on seeded synthetic top lists (a real and a null input over a 12 x 10 tile image, 60
candidate orientations of cubic symmetry, some planted near-duplicates so that the separation and linking rules act).
The fixture holds the inputs and the reference's outputs; the tests never read the reference.
"""
import sys
from pathlib import Path
from unittest import mock

import numpy as np

if len(sys.argv) < 2:
    sys.exit("usage: make_search_golden.py <path of the reference's source tree (the directory holding src/diffractom)>")
REF = Path(sys.argv[1])
OUT = Path(__file__).resolve().parent
for m in ["pyopencl", "pyopencl.array", "pyopencl.tools", "pyopencl.scan", "pyopencl.elementwise",
          "pyopencl.reduction", "pyopencl.clrandom", "pyopencl.cltypes", "pyopencl.clmath", "pyopencl.characterize",
          "gratopy", "pyclblast", "pyvkfft", "pyvkfft.opencl", "h5py"]:
    sys.modules[m] = mock.MagicMock()
sys.path.insert(0, str(REF / "src"))

from scipy.spatial.transform import Rotation  # noqa: E402

from diffractom import orientation_search as ref  # noqa: E402


def cubic_rotations():
    """The 24 proper rotations of the cubic point group as matrices."""
    mats = []
    for perm in ([0, 1, 2], [1, 2, 0], [2, 0, 1], [1, 0, 2], [0, 2, 1], [2, 1, 0]):
        for signs in np.array(np.meshgrid([1, -1], [1, -1], [1, -1])).T.reshape(-1, 3):
            m = np.zeros((3, 3))
            m[np.arange(3), perm] = signs
            if np.linalg.det(m) > 0:
                mats.append(m)
    return np.array(mats)


def main():
    rng = np.random.default_rng(42)
    Ny, Nx, top_k = 12, 10, 6
    base = Rotation.random(40, random_state=7).as_matrix()
    near = base[:20] @ Rotation.from_rotvec(np.deg2rad(rng.normal(0, 1.5, (20, 3)))).as_matrix()
    sym = cubic_rotations()
    # symmetry equivalents of some: the same orientation on the crystal side
    eqv = base[:4] @ sym[[5, 9, 13, 17]]
    rotations = np.concatenate([base, near, eqv])
    n_c = len(rotations)
    pixels = np.arange(Ny * Nx)
    idx = np.stack([rng.choice(n_c, top_k, replace=False) for _ in pixels]).astype(np.int32)
    z = rng.gamma(2.0, 1.0, (2, len(pixels), top_k)).astype(np.float32)
    # three planted crystals over blocks of tiles: strong fitted and held-out z of nearby orientations
    for c, (y0, x0, h, w) in enumerate([(1, 1, 3, 3), (6, 5, 2, 4), (9, 0, 2, 2)]):
        for y in range(y0, y0 + h):
            for x in range(x0, x0 + w):
                t = y * Nx + x
                choice = [c, 40 + c, 60 + c] if c < 3 else [c]
                idx[t, 0] = choice[(y + x) % len(choice)]
                z[0, t, 0] = 20 + 5 * c + rng.random()
                z[1, t, 0] = 8 + rng.random()
    idx[5, 2] = -1
    o = np.argsort(-z[0], axis=1, kind="stable")
    idx = np.take_along_axis(idx, o, 1)
    z = np.stack([np.take_along_axis(a, o, 1) for a in z])
    null_z = rng.gamma(2.0, 1.0, (2, len(pixels), top_k)).astype(np.float32)
    real, null = {"idx": idx, "z": z}, {"idx": idx.copy(), "z": null_z}
    out = {"rotations": rotations, "sym": sym, "real_idx": idx, "real_z": z, "null_z": null_z,
           "pixels": pixels, "tile_shape": np.array([Ny, Nx])}
    for name, kw in (("strict", {}), ("liberal", dict(ratio=1.5, min_tiles=1)),
                     ("narrow", dict(sep_deg=3.0, link_deg=2.0, max_per_tile=2))):
        c = ref.select_candidates(real, null, rotations, pixels, (Ny, Nx), sym, **kw)
        out[f"{name}_rot"] = c.rotations
        out[f"{name}_score"] = c.score
        out[f"{name}_ntiles"] = np.array([len(t) for t in c.tiles])
        out[f"{name}_tiles"] = np.concatenate(c.tiles) if len(c) else np.zeros(0, np.int64)
        if name == "strict":
            strict = c
    shape = (Ny * 4 - 3, Nx * 4 - 1)
    mask = np.ones(shape, bool)
    mask[:5, :7] = False
    k, iy, ix = ref.candidate_support(strict, 4, shape, dilate=2, mask=mask)
    out.update(support_k=k, support_iy=iy, support_ix=ix, support_shape=np.array(shape), support_mask=mask)
    coeff = rng.standard_normal((9, 5, 6))
    coeff[7] = np.abs(coeff[7]) * 1e-4
    out["coeff"] = coeff
    out["weights_dense"] = ref.orientation_weights(coeff)
    kk = rng.integers(0, 9, 200)
    vv = rng.standard_normal(200)
    out.update(coo_k=kk, coo_v=vv, weights_coo=ref.orientation_weights(vv, k=kk))
    out["prune"] = ref.prune_added(out["weights_dense"], 4, rel=0.3)
    out["prune_none"] = ref.prune_added(np.r_[out["weights_dense"][:4], np.zeros(5)], 4)
    np.savez_compressed(OUT / "search_candidates.npz", **out)
    print("wrote", OUT / "search_candidates.npz", {k: v.shape for k, v in out.items() if hasattr(v, "shape")})


if __name__ == "__main__":
    main()
