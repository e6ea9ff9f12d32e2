"""Local basis: orientation k has coefficients only where a LocalSupport allows it (diffractom's
operators/local_support.py and operators/local_forward_operator.py).

LocalSupport holds the allowed (orientation, voxel) pairs; build_patches groups them into rectangular patches (one
bounding box per orientation, or per cluster of its voxels when they are scattered); the coefficients are a flat
float32 vector of the patches' cells (row-major per patch), held at zero outside the support.

LocalSinglePhaseForwardOperator is SinglePhaseForwardOperator over the orientations the support uses (numbered along
a Z-order curve through their voxels, so that a batch covers one part of the slice), with the flat coefficients: a
batch's patches are scattered into its channel-fastest image before the forward projection and gathered after the
backprojection (dfx_local_scatter / dfx_local_gather), so the coefficient arrays scale with the support while the
projections and PF products run through the operator's dense kernels. Its values are those of the inner operator
applied to the zero-extended coefficients, bit for bit, for any patch split.
"""
from __future__ import annotations

import numpy as np
import torch

from .arrays import as_host, check_device, on_op_stream
from .geometry import fov_support_mask
from .grid import MatrixGrid
from .operator import SinglePhaseForwardOperator


def _disk(radius):
    """Offsets (dy, dx) of a disc of the given radius in voxels (0: the voxel itself)."""
    r = int(np.ceil(radius))
    dy, dx = np.mgrid[-r:r + 1, -r:r + 1]
    keep = dy ** 2 + dx ** 2 <= radius ** 2 + 0.5
    return dy[keep], dx[keep]


class LocalSupport:
    """Sorted, unique (orientation k, voxel (iy, ix)) pairs of a basis of K orientations on an Ny x Nx grid
    (local_support.py:29-188)."""

    def __init__(self, k, iy, ix, K, shape):
        self.K = int(K)
        self.Ny, self.Nx = (int(n) for n in shape)
        k, iy, ix = (np.asarray(a, dtype=np.int64).ravel() for a in (k, iy, ix))
        if not (len(k) == len(iy) == len(ix)):
            raise ValueError("k, iy and ix must have the same length")
        ok = (k >= 0) & (k < self.K) & (iy >= 0) & (iy < self.Ny) & (ix >= 0) & (ix < self.Nx)
        if not ok.all():
            raise ValueError(f"{int((~ok).sum())} pairs outside the basis (K = {self.K}) or the grid "
                             f"({self.Ny} x {self.Nx})")
        lin = np.unique((k * self.Ny + iy) * self.Nx + ix)
        self.k, rem = np.divmod(lin, self.Ny * self.Nx)
        self.iy, self.ix = np.divmod(rem, self.Nx)

    @classmethod
    def from_mask(cls, mask):
        """From a boolean (K, Ny, Nx) array."""
        mask = np.asarray(mask, dtype=bool)
        if mask.ndim != 3:
            raise ValueError("mask must have shape (K, Ny, Nx)")
        k, iy, ix = np.nonzero(mask)
        return cls(k, iy, ix, mask.shape[0], mask.shape[1:])

    @classmethod
    def everywhere(cls, K, shape):
        """Every orientation in every voxel (the global basis)."""
        k, iy, ix = np.meshgrid(np.arange(K), np.arange(shape[0]), np.arange(shape[1]), indexing="ij")
        return cls(k, iy, ix, K, shape)

    def dilate(self, radius):
        """Every orientation's voxels grown by a disc of the given radius."""
        dy, dx = _disk(radius)
        k = np.repeat(self.k, len(dy))
        iy = (self.iy[:, None] + dy[None]).ravel()
        ix = (self.ix[:, None] + dx[None]).ravel()
        ok = (iy >= 0) & (iy < self.Ny) & (ix >= 0) & (ix < self.Nx)
        return LocalSupport(k[ok], iy[ok], ix[ok], self.K, (self.Ny, self.Nx))

    def restrict(self, mask):
        """Only the voxels where the (Ny, Nx) mask is True."""
        mask = np.asarray(mask, dtype=bool)
        if mask.shape != (self.Ny, self.Nx):
            raise ValueError(f"mask shape {mask.shape} != {(self.Ny, self.Nx)}")
        keep = mask[self.iy, self.ix]
        return LocalSupport(self.k[keep], self.iy[keep], self.ix[keep], self.K, (self.Ny, self.Nx))

    def union(self, other):
        if (other.K, other.Ny, other.Nx) != (self.K, self.Ny, self.Nx):
            raise ValueError("supports of different bases or grids")
        return LocalSupport(np.r_[self.k, other.k], np.r_[self.iy, other.iy], np.r_[self.ix, other.ix], self.K,
                            (self.Ny, self.Nx))

    def to_mask(self):
        m = np.zeros((self.K, self.Ny, self.Nx), dtype=bool)
        m[self.k, self.iy, self.ix] = True
        return m

    @property
    def n_pairs(self):
        return len(self.k)

    @property
    def fill(self):
        return self.n_pairs / float(self.K * self.Ny * self.Nx)

    def orientations_used(self):
        return np.unique(self.k)

    def per_voxel(self):
        return np.bincount(self.iy * self.Nx + self.ix, minlength=self.Ny * self.Nx).reshape(self.Ny, self.Nx)

    def __repr__(self):
        return (f"LocalSupport({self.n_pairs} pairs, {len(self.orientations_used())} of {self.K} orientations, "
                f"{self.Ny} x {self.Nx} voxels, fill {100 * self.fill:.2f} %)")


def _merge_boxes(boxes):
    """Overlapping boxes [y0, y1, x0, x1] (inclusive) merged until none overlap."""
    boxes = [list(b) for b in boxes]
    merged = True
    while merged and len(boxes) > 1:
        merged = False
        out = []
        while boxes:
            b = boxes.pop()
            i = 0
            while i < len(boxes):
                c = boxes[i]
                if b[0] <= c[1] and c[0] <= b[1] and b[2] <= c[3] and c[2] <= b[3]:
                    b = [min(b[0], c[0]), max(b[1], c[1]), min(b[2], c[2]), max(b[3], c[3])]
                    boxes.pop(i)
                    merged = True
                else:
                    i += 1
            out.append(b)
        boxes = out
    return boxes


def build_patches(k, iy, ix, K, split=True, merge_gap=2, min_box_fill=0.5):
    """Rectangular patches of sorted, unique (k, iy, ix) pairs (local_support.py:209-283): one bounding box per
    orientation, unless split and its voxels fill less than min_box_fill of it; then its voxels are clustered
    (connected after growing by merge_gap voxels), each cluster gets its bounding box and overlapping boxes are merged.
    Patches are ordered by orientation, then position. Returns pk, y0, x0, h, w, coff (offset of a patch's
    coefficients, row-major in its box), n_coef, mask (uint8, 1 where a pair is) and pair_index (every pair's
    coefficient, in the pairs' order)."""
    from scipy.ndimage import binary_dilation, label
    k, iy, ix = (np.asarray(a, dtype=np.int64) for a in (k, iy, ix))
    n = len(k)
    if n == 0:
        raise ValueError("empty support")
    starts = np.flatnonzero(np.r_[True, k[1:] != k[:-1]])
    ends = np.r_[starts[1:], n]
    ymin, ymax = np.minimum.reduceat(iy, starts), np.maximum.reduceat(iy, starts)
    xmin, xmax = np.minimum.reduceat(ix, starts), np.maximum.reduceat(ix, starts)
    count = ends - starts
    area = (ymax - ymin + 1) * (xmax - xmin + 1)
    sparse = split & (count < min_box_fill * area)
    pk, py0, px0, ph, pw = [], [], [], [], []
    pair_patch = np.empty(n, dtype=np.int64)
    conn = np.ones((3, 3), dtype=bool)
    grow = np.ones((2 * merge_gap + 1, 2 * merge_gap + 1), dtype=bool) if merge_gap > 0 else None
    for g in range(len(starts)):
        s, e = starts[g], ends[g]
        if not sparse[g]:
            pair_patch[s:e] = len(pk)
            pk.append(k[s]); py0.append(ymin[g]); px0.append(xmin[g])
            ph.append(ymax[g] - ymin[g] + 1); pw.append(xmax[g] - xmin[g] + 1)
            continue
        y, x = iy[s:e] - ymin[g], ix[s:e] - xmin[g]
        m = np.zeros((ymax[g] - ymin[g] + 1, xmax[g] - xmin[g] + 1), dtype=bool)
        m[y, x] = True
        lab, nl = label(binary_dilation(m, grow) if grow is not None else m, structure=conn)
        lv = lab[y, x]
        boxes = [[y[lv == c].min(), y[lv == c].max(), x[lv == c].min(), x[lv == c].max()]
                 for c in range(1, nl + 1) if (lv == c).any()]
        for b in sorted(_merge_boxes(boxes)):
            inside = (y >= b[0]) & (y <= b[1]) & (x >= b[2]) & (x <= b[3])
            pair_patch[s:e][inside] = len(pk)
            pk.append(k[s]); py0.append(ymin[g] + b[0]); px0.append(xmin[g] + b[2])
            ph.append(b[1] - b[0] + 1); pw.append(b[3] - b[2] + 1)
    pk, py0, px0, ph, pw = (np.asarray(a, dtype=np.int64) for a in (pk, py0, px0, ph, pw))
    sizes = ph * pw
    coff = np.r_[0, np.cumsum(sizes)[:-1]].astype(np.int64)
    n_coef = int(sizes.sum())
    pair_index = coff[pair_patch] + (iy - py0[pair_patch]) * pw[pair_patch] + (ix - px0[pair_patch])
    mask = np.zeros(n_coef, dtype=np.uint8)
    mask[pair_index] = 1
    if int(mask.sum()) != n:
        raise RuntimeError("patches overlap")
    return dict(pk=pk, y0=py0, x0=px0, h=ph, w=pw, coff=coff, n_coef=n_coef, mask=mask, pair_index=pair_index)


def split_regions(mats, sigmas, support: LocalSupport, mode: str = "components", tile: int = 8, min_pairs: int = 1):
    """Copies of the orientations, one per region of their support (differentiable/local_basis.py:17-61), so that a
    refinement can turn every region's copy on its own (orientation gradients inside a grain).

    mode "components": every 8-connected component of an orientation's voxels is a region; "tiles": the voxels are
    grouped by tile x tile blocks of the grid; "components+tiles": components cut by the tiles. Regions of fewer
    than min_pairs voxels are dropped. Returns (mats, sigmas, support, parent), parent[k'] the orientation that the new
    orientation k' copies; the new orientations are numbered by parent, then region label."""
    from scipy import ndimage
    if mode not in ("components", "tiles", "components+tiles"):
        raise ValueError(f"mode: 'components', 'tiles' or 'components+tiles', not {mode!r}")
    Ny, Nx = support.Ny, support.Nx
    n_tx = -(-Nx // tile)
    order = np.argsort(support.k, kind="stable")
    k, iy, ix = support.k[order], support.iy[order], support.ix[order]
    bounds = np.searchsorted(k, np.arange(support.K + 1))
    out_k, out_y, out_x, parent = [], [], [], []
    for kk in range(support.K):
        a, b = bounds[kk], bounds[kk + 1]
        if a == b:
            continue
        y, x = iy[a:b], ix[a:b]
        tiles = (y // tile) * n_tx + x // tile
        if mode == "tiles":
            lab = tiles
        else:
            y0, x0 = y.min(), x.min()
            img = np.zeros((y.max() - y0 + 1, x.max() - x0 + 1), bool)
            img[y - y0, x - x0] = True
            comp, _ = ndimage.label(img, structure=np.ones((3, 3), bool))
            lab = comp[y - y0, x - x0].astype(np.int64)
            if mode == "components+tiles":
                lab = lab * (Ny * Nx) + tiles
        uniq, inv = np.unique(lab, return_inverse=True)
        keep = np.bincount(inv, minlength=len(uniq)) >= min_pairs
        new_id = np.full(len(uniq), -1, np.int64)
        new_id[keep] = len(parent) + np.arange(int(keep.sum()))
        sel = new_id[inv] >= 0
        out_k.append(new_id[inv][sel])
        out_y.append(y[sel])
        out_x.append(x[sel])
        parent.extend([kk] * int(keep.sum()))
    parent = np.asarray(parent, np.int64)
    cat = lambda parts: np.concatenate(parts) if parts else np.zeros(0, np.int64)
    sup = LocalSupport(cat(out_k), cat(out_y), cat(out_x), len(parent), (Ny, Nx))
    return np.asarray(mats)[parent], np.asarray(sigmas)[parent], sup, parent


def spatial_moments(k, iy, ix, v, K):
    """Per orientation (K of them) the weighted mean (col, row) and covariance (col-col, col-row, row-row) of its
    voxels (v: weights, default 1; local_forward_operator.py:77-92): the positions of the window_parallax option.
    Orientations without weight get the origin and no spread."""
    k = np.asarray(k, np.int64)
    x, y = np.asarray(ix, np.float64), np.asarray(iy, np.float64)
    w = np.ones(len(k)) if v is None else np.clip(np.asarray(v, np.float64), 0, None)
    W = np.bincount(k, w, minlength=K)
    Wn = np.maximum(W, 1e-300)
    mx, my = np.bincount(k, w * x, minlength=K) / Wn, np.bincount(k, w * y, minlength=K) / Wn
    dx, dy = x - mx[k], y - my[k]
    cov = np.stack([np.bincount(k, w * dx * dx, minlength=K), np.bincount(k, w * dx * dy, minlength=K),
                    np.bincount(k, w * dy * dy, minlength=K)], 1) / Wn[:, None]
    pos = np.stack([mx, my], 1)
    pos[W <= 0] = 0.0
    cov[W <= 0] = 0.0
    return pos, cov


def _morton(y, x):
    """Z-order code of non-negative integer coordinates below 2^16 (bits of y and x interleaved)."""
    def spread(v):
        v = np.asarray(v, dtype=np.uint64) & np.uint64(0xFFFF)
        for shift, m in ((8, 0x00FF00FF), (4, 0x0F0F0F0F), (2, 0x33333333), (1, 0x55555555)):
            v = (v | (v << np.uint64(shift))) & np.uint64(m)
        return v
    return (spread(y) << np.uint64(1)) | spread(x)


class LocalSinglePhaseForwardOperator(SinglePhaseForwardOperator):
    """data = PF @ Radon(coeffs) with a local basis (local_forward_operator.py:93-532): coefficients are a flat
    float32 vector of length n_coef (coeff_shape (n_coef,)); to_dense / from_dense / to_coo / coefficient_mask
    convert in the grid's orientation order. Omega subsets as SinglePhaseForwardOperator's.

    Arguments besides SinglePhaseForwardOperator's: support (LocalSupport of the grid's orientations; restricted to
    the field of view unless restrict_to_fov=False; orientations without voxels are left out), split_patches,
    merge_gap, min_box_fill (build_patches), spatial_order (number the orientations along a Z-order curve through
    their voxels; the coefficients use the grid's order either way), pf_chunk (accepted). Native projector, FP32,
    sparse PF modes."""

    coefficient_layout = "local"

    def __init__(self, cfg, material, grid, max_gb, support: LocalSupport, verbose=False, split_patches=True,
                 merge_gap=2, min_box_fill=0.5, restrict_to_fov=True, spatial_order=True, pf_chunk=None, **kwargs):
        if kwargs.pop("projector", "native") not in ("native", "auto"):
            raise ValueError("LocalSinglePhaseForwardOperator uses the native projector")
        if kwargs.get("pf_mode", "auto") == "dense":
            raise ValueError("LocalSinglePhaseForwardOperator needs a sparse PF mode ('auto', 'sparse', 'generated')")
        kwargs.setdefault("sparse_max_fill", 1.0)          # never the dense path (local_forward_operator.py:134-135)
        kwargs.setdefault("sparse_max_fill_partial", 1.0)
        if kwargs.get("precision", "fp32") != "fp32":
            raise NotImplementedError("LocalSinglePhaseForwardOperator computes in float32")
        if not isinstance(support, LocalSupport):
            raise TypeError("support must be a LocalSupport")
        c = {**cfg, **kwargs}
        Nx, Ny, My = int(c["Nx"]), int(c["Ny"]), int(c["My"])
        if hasattr(grid, "leaf_arrays"):
            mats, sig = (np.asarray(a) for a in grid.leaf_arrays())
        else:
            from .grid import grid_arrays
            mats, sig = grid_arrays(grid)
        if support.K != len(mats) or (support.Ny, support.Nx) != (Ny, Nx):
            raise ValueError(f"support is for K = {support.K} on {support.Ny} x {support.Nx}; the grid has "
                             f"{len(mats)} orientations, the geometry {Ny} x {Nx} voxels")
        if restrict_to_fov:
            n_om = int(c["N_Omega"])
            rng = np.array(c["angle_range"], dtype=np.float64) / 180 * np.pi
            delta = (rng[1] - rng[0]) / n_om
            angles = np.linspace(rng[0], rng[1], n_om, endpoint=False) + delta / 2
            vs = c.get("voxel_size")
            fov = fov_support_mask(Nx, Ny, My, angles=angles,
                                   image_width=Nx if vs is None else float(vs) * max(Nx, Ny), detector_width=My,
                                   detector_shift=c.get("cor_offset", 0.0))
            support = support.restrict(fov)
        if support.n_pairs == 0:
            raise ValueError("the support is empty (inside the field of view)")
        self.support = support
        self.K_basis = len(mats)
        used = support.orientations_used()
        k_used = np.searchsorted(used, support.k)
        if spatial_order:
            cnt = np.bincount(k_used, minlength=len(used))
            cy = np.bincount(k_used, weights=support.iy, minlength=len(used)) / cnt
            cx = np.bincount(k_used, weights=support.ix, minlength=len(used)) / cnt
            order = np.argsort(_morton(cy.astype(np.int64), cx.astype(np.int64)), kind="stable")
        else:
            order = np.arange(len(used))
        rank = np.empty(len(used), dtype=np.int64)
        rank[order] = np.arange(len(used))
        self.orientation_index = used[order]                 # operator orientation -> grid orientation
        k_int = rank[k_used]
        perm = np.lexsort((support.ix, support.iy, k_int))
        P = build_patches(k_int[perm], support.iy[perm], support.ix[perm], len(used), split=split_patches,
                          merge_gap=merge_gap, min_box_fill=min_box_fill)
        pair_index = np.empty_like(P["pair_index"])
        pair_index[perm] = P["pair_index"]                  # in the order of the support's pairs
        P["pair_index"] = pair_index
        self._patches = P
        self.n_coef = int(P["n_coef"])
        self.n_patches = len(P["pk"])
        self._pf_chunk = pf_chunk
        inner = MatrixGrid(mats[self.orientation_index], sig[self.orientation_index])
        if kwargs.get("window_parallax") is not None:            # positions in grid order -> operator order
            wp = dict(kwargs["window_parallax"])
            if wp.get("positions") is None:                      # default: the support's centroid and spread
                wp["positions"], wp["covariances"] = spatial_moments(support.k, support.iy, support.ix, None,
                                                                     self.K_basis)
            pos = np.asarray(wp["positions"], np.float64).reshape(self.K_basis, 2)[self.orientation_index]
            cov = (None if wp.get("covariances") is None else
                   np.asarray(wp["covariances"], np.float64).reshape(self.K_basis, 3)[self.orientation_index])
            kwargs["window_parallax"] = {**wp, "positions": pos, "covariances": cov}
        super().__init__(cfg, material, inner, max_gb, verbose=verbose, projector="native", **kwargs)
        self._setup_local()

    def _setup_local(self):
        """Per orientation batch: its patch table, and the compact image of the pixels where the batch has
        coefficients (support pixels, ascending): the pixel -> row map, the pixel list for the backprojection and the
        ray table restricted to those pixels with its pixel indices turned into rows. The projections of a batch then
        cost its support, not the image."""
        P = self._patches
        bounds = np.searchsorted(P["pk"], [b["k_start"] for b in self.batches] + [self.K])
        dev = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a, dtype=dt), device=self.device)
        _, iy, ix, pi = self._pairs()
        pix_of_coef = np.full(self.n_coef, -1, np.int64)
        pix_of_coef[pi] = iy * self.Nx + ix
        npix = self.Nx * self.Ny
        self.local_batches = []
        n_max = 0
        for ib, b in enumerate(self.batches):
            p0, p1 = int(bounds[ib]), int(bounds[ib + 1])
            if p1 == p0:
                self.local_batches.append(None)
                continue
            chan = P["pk"][p0:p1] - b["k_start"]
            if chan.min() < 0 or chan.max() >= b["K_batch"]:
                raise RuntimeError("a patch outside its batch")
            box = np.stack([P["y0"][p0:p1], P["x0"][p0:p1], P["h"][p0:p1], P["w"][p0:p1]], 1)
            c0, c1 = int(P["coff"][p0]), int(P["coff"][p1]) if p1 < len(P["coff"]) else self.n_coef
            pix = np.unique(pix_of_coef[c0:c1])
            pix = pix[pix >= 0]
            row = np.full(npix, -1, np.int32)
            row[pix] = np.arange(len(pix), dtype=np.int32)
            lb = dict(n=p1 - p0, box=dev(box, np.int32), coff=dev(P["coff"][p0:p1], np.int64),
                      chan=dev(chan, np.int32), n_pix=len(pix), plist=dev(pix, np.int32), pix_row=dev(row, np.int32))
            if self.projector == "native":
                supp = torch.zeros(npix, dtype=torch.uint8, device=self.device)
                supp[lb["plist"].long()] = 1
                rp, ent, taps = self._build_ray_table(supp)
                e = ent[:2 * taps].view(-1, 2)
                e[:, 0] = lb["pix_row"][e[:, 0].long()]
                lb["ray"] = (rp, ent, taps)
            n_max = max(n_max, len(pix))
            self.local_batches.append(lb)
        self._mask = dev(P["mask"], np.uint8)
        self._img_c = torch.empty(max(n_max, 1) * self.Kstride, dtype=torch.float32, device=self.device)

    @property
    def coeff_shape(self):
        return (self.n_coef,) if hasattr(self, "n_coef") and hasattr(self, "_mask") else super().coeff_shape

    def _scatter(self, lb, coeffs, img, compact=False):
        """The batch's patches into a batch image (zero elsewhere: the caller clears it): the whole image, or the
        compact image of the batch's support pixels."""
        self._call("dfx_local_scatter", coeffs.data_ptr(), self._mask.data_ptr(), lb["box"].data_ptr(),
                   lb["coff"].data_ptr(), lb["chan"].data_ptr(), lb["n"], self.Nx, self.Ny, self.Kstride,
                   lb["pix_row"].data_ptr() if compact else None, img.data_ptr(), self._s())

    def _gather(self, lb, img, coeffs, compact=False):
        self._call("dfx_local_gather", img.data_ptr(), self._mask.data_ptr(), lb["box"].data_ptr(),
                   lb["coff"].data_ptr(), lb["chan"].data_ptr(), lb["n"], self.Nx, self.Ny, self.Kstride,
                   lb["pix_row"].data_ptr() if compact else None, coeffs.data_ptr(), self._s())

    def _project_local(self, coeffs, ib, subset=None):
        """Radon of batch ib's patches into the batch sinogram (its support pixels only, through the batch's
        compact image and restricted ray table); returns (om, n_ang, Kb, m) of the angles projected."""
        lb = self.local_batches[ib]
        Kb = self.batches[ib]["K_batch"]
        img = self._img_c[:lb["n_pix"] * self.Kstride]
        self._fill(img, 0.0)
        self._scatter(lb, coeffs, img, compact=True)
        geo, n_ang, om, m = self._geo_of(subset)
        self._radon_fwd(img.data_ptr(), self.coeffs_sino_C.data_ptr(), om, n_ang, Kb, ray=lb["ray"], m=m)
        return om, n_ang, Kb, m

    @on_op_stream
    def direct_cl(self, coeffs, data, subset=None):
        """data = PF @ Radon(coeffs) in place (subset=m: only the rows of subset m, the others left as they are)."""
        check_device(coeffs, self.coeff_shape, "coeffs")
        check_device(data, self.data_shape, "data")
        if subset is None:
            self._fill(data, 0.0)
        else:
            self.zero_subset_rows(data, subset)
        for ib, lb in enumerate(self.local_batches):
            if lb is None:
                continue
            om, n_ang, Kb, m = self._project_local(coeffs, ib, subset)
            self._pf_forward_product(ib, m, self.coeffs_sino_C.data_ptr(), data, om, n_ang, Kb)

    @on_op_stream
    def adjoint_cl(self, data, coeffs, subset=None):
        """coeffs = A^T data in place (zero outside the support); subset=m: A_m^T."""
        check_device(data, self.data_shape, "data")
        check_device(coeffs, self.coeff_shape, "coeffs")
        for ib, lb in enumerate(self.local_batches):         # every patch is in one batch: all coefficients written
            if lb is None:
                continue
            geo, n_ang, Kb = self._pf_adjoint_to_sino(data, ib, subset)
            img = self._img_c[:lb["n_pix"] * self.Kstride]
            self._call("dfx_radon_backward_pixels", self.coeffs_sino_C.data_ptr(), img.data_ptr(), geo.data_ptr(),
                       n_ang, self.Nx, self.Ny, self.My, self.Kstride, Kb, self._kernel_id,
                       int(self.radon_geo.n_taps), lb["plist"].data_ptr(), lb["n_pix"], self._s())
            self._gather(lb, img, coeffs, compact=True)

    @on_op_stream
    def direct(self, coeffs):
        """NumPy (n_coef,) -> NumPy data, or CUDA tensor -> CUDA tensor."""
        if isinstance(coeffs, torch.Tensor):
            data = torch.empty(self.data_shape, dtype=torch.float32, device=self.device)
            self.direct_cl(coeffs, data)
            return data
        x = torch.as_tensor(as_host(coeffs, self.coeff_shape, "coeffs"), device=self.device)
        data = torch.empty(self.data_shape, dtype=torch.float32, device=self.device)
        self.direct_cl(x, data)
        return data.cpu().numpy()

    @on_op_stream
    def adjoint(self, data):
        """NumPy data -> NumPy (n_coef,), or CUDA tensor -> CUDA tensor."""
        if isinstance(data, torch.Tensor):
            coeffs = torch.empty(self.coeff_shape, dtype=torch.float32, device=self.device)
            self.adjoint_cl(data, coeffs)
            return coeffs
        d = torch.as_tensor(as_host(data, self.data_shape, "data"), device=self.device)
        coeffs = torch.empty(self.coeff_shape, dtype=torch.float32, device=self.device)
        self.adjoint_cl(d, coeffs)
        return coeffs.cpu().numpy()

    def adjoint_batches_cl(self, *args, **kwargs):
        raise NotImplementedError("the local-basis operator has no batched adjoint")

    def adjoint_multi_cl(self, *args, **kwargs):
        raise NotImplementedError("the local-basis operator has no multi-RHS adjoint")

    # ---- coefficients
    def _pairs(self):
        s = self.support
        return s.k, s.iy, s.ix, self._patches["pair_index"]

    def to_dense(self, x):
        """(K, Ny, Nx) float32 array in the grid's orientation order (zero outside the support)."""
        x = x.cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)
        k, iy, ix, pi = self._pairs()
        out = np.zeros((self.K_basis, self.Ny, self.Nx), dtype=np.float32)
        out[k, iy, ix] = x[pi]
        return out

    def from_dense(self, coeffs):
        """The flat coefficients of a (K, Ny, Nx) array (values outside the support dropped)."""
        coeffs = np.asarray(coeffs)
        if coeffs.shape != (self.K_basis, self.Ny, self.Nx):
            raise ValueError(f"coeffs must have shape {(self.K_basis, self.Ny, self.Nx)}, not {coeffs.shape}")
        k, iy, ix, pi = self._pairs()
        x = np.zeros(self.n_coef, dtype=np.float32)
        x[pi] = coeffs[k, iy, ix]
        return x

    def to_coo(self, x):
        """(k, iy, ix, value) of every allowed pair (k in the grid's orientation order)."""
        x = x.cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)
        k, iy, ix, pi = self._pairs()
        return k.copy(), iy.copy(), ix.copy(), x[pi].astype(np.float32)

    def coefficient_mask(self, mask=None):
        """(n_coef,) float32: 1 for the allowed coefficients (and, given an (Ny, Nx) mask, only where it is True)."""
        m = self._patches["mask"].astype(np.float32)
        if mask is not None:
            mask = np.asarray(mask, dtype=bool)
            k, iy, ix, pi = self._pairs()
            m[pi[~mask[iy, ix]]] = 0.0
        return m

    def device_bytes(self):
        n = super().device_bytes()
        for lb in getattr(self, "local_batches", None) or []:
            if lb is not None:
                n += sum(v.numel() * v.element_size() for v in lb.values() if isinstance(v, torch.Tensor))
                n += sum(t.numel() * t.element_size() for t in lb.get("ray", ())[:2])
        for t in (getattr(self, "_mask", None), getattr(self, "_img_c", None)):
            n += 0 if t is None else t.numel() * t.element_size()
        return n

    def free_memory(self):
        self.local_batches = None
        self._mask = self._img_c = None
        super().free_memory()
