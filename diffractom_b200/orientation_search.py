"""Residual orientation search (diffractom's orientation_search.py): which orientations missing from a basis the data
still ask for, and where.

A fit with counts b, prediction mu, gain g and weights w leaves the score e = w / g (b / mu - 1) and the Fisher
information d = w / (g mu) in data space. For a candidate orientation k and a pixel p the score test of adding a
coefficient c_kp is z_kp = (A^T e)_kp / sqrt((A^T d)_kp) (orientation_search.py:1-20). score_candidates scores a list
of candidates in chunks, one operator per chunk, for several (e, d) pairs (e.g. the real residual and one with its
azimuths scrambled, the null) and several angle-row sets (e.g. fitted and held-out angles), and keeps per pixel the
top_k candidates with the largest z on the first row set. Each chunk's operator applies its PF matrix once for all
inputs and back-projects only the scored pixels (SinglePhaseForwardOperator.adjoint_multi_cl); z is computed on the
device with correctly rounded division and square root (dfx_score_z), so it equals the host's float32 expression
bitwise, and only z crosses to the host.

The candidate workflow around the scores (orientation_search.py:232-470): select_candidates turns the per-pixel top
lists of the real and the null inputs into Candidates (tile peaks that beat the null, linked across neighbouring tiles
by misorientation under the crystal symmetry), refine_candidates moves each candidate to the best orientation of finer
rotation lattices around it (the score test summed over its tiles, through a local-basis operator's adjoint),
candidate_support gives the (orientation, voxel) pairs of a local basis for them, and orientation_weights /
prune_added drop added orientations that a joint fit left (almost) empty.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .arrays import check_device

__all__ = ["poisson_score_inputs", "scramble_eta", "score_candidates", "Candidates", "select_candidates",
           "refine_candidates", "candidate_support", "orientation_weights", "prune_added"]


def poisson_score_inputs(b, mu, gain, weights, floor=0.25):
    """e = w / g (b / mu - 1) and d = w / (g mu) (float32, the data's shape) with mu >= floor x g; cells of weight 0
    give 0 (orientation_search.py:58-67). NumPy arrays (broadcastable gain and weights)."""
    b = np.asarray(b, np.float32)
    g = np.asarray(gain, np.float32)
    w = np.asarray(weights, np.float32)
    m = np.maximum(np.maximum(np.asarray(mu, np.float32), 0), floor * g)
    e = np.where(w > 0, w / g * (b / m - 1), 0).astype(np.float32)
    d = np.where(w > 0, w / (g * m), 0).astype(np.float32)
    return e, d


def scramble_eta(a, n_eta, n_channels, block=12, seed=1, margin=10, mask=None):
    """The null of the search (orientation_search.py:70-90): a (N_Omega, My, n_eta * n_channels) array (segment =
    eta * n_channels + channel) with the azimuth of every channel turned by a random number of bins (margin ..
    n_eta - margin) per block of ``block`` rotation angles; mask (optional) is multiplied in."""
    a = np.asarray(a)
    n_omega = a.shape[0]
    shifts = np.random.default_rng(seed).integers(margin, n_eta - margin, size=(n_omega // block + 1, n_channels))
    out = np.empty_like(a)
    eta = np.arange(n_eta)
    for b0 in range(0, n_omega, block):
        sh = shifts[b0 // block]
        perm = np.empty(n_eta * n_channels, np.int64)
        for r in range(n_channels):
            perm[eta * n_channels + r] = ((eta + sh[r]) % n_eta) * n_channels + r
        out[b0:b0 + block] = a[b0:b0 + block][:, :, perm]
        if mask is not None:
            out[b0:b0 + block] *= mask
    return out


def _merge(top, z_new, K, c0, top_k):
    """The kept top_k of every pixel merged with a chunk's candidates c0 .. c0+K-1 (z_new: per row set (K, npix))."""
    idx, zs = top
    npix = idx.shape[0]
    cand_i = np.concatenate([idx, np.broadcast_to(np.arange(c0, c0 + K, dtype=np.int32), (npix, K))], axis=1)
    cand_z = [np.concatenate([zs[s], z_new[s][:K].T], axis=1) for s in range(len(zs))]
    o = np.argpartition(-cand_z[0], top_k - 1, axis=1)[:, :top_k]
    return (np.take_along_axis(cand_i, o, 1).astype(np.int32),
            [np.take_along_axis(cz, o, 1).astype(np.float32) for cz in cand_z])


def score_candidates(make_operator, rotations, inputs, row_masks, pixels, top_k=64, chunk=30000, verbose=False,
                     reuse_operator=True, nrhs=4, rows_per_group=16, gpu_scores=True):
    """Score test of candidate orientations per pixel; keep the best top_k per pixel (orientation_search.py:93-238).

    make_operator(rotations (n, 3, 3)) -> SinglePhaseForwardOperator (pf_mode "sparse" or "generated", native
    projector) for a chunk of candidates (all chunks: the same image grid and data shape); inputs: list of (E, D)
    pairs of CUDA data arrays; row_masks: list of (N_Omega,) bool arrays (the first ranks); pixels: (npix,) flat pixel
    indices. reuse_operator, rows_per_group: accepted (this implementation builds one operator per chunk; the scores do
    not depend on it); gpu_scores False: E and D go to the host and z is computed there (same values).

    Returns one dict per input pair: "idx" (npix, top_k) int32 candidate indices (-1: none), "z" (n_rows, npix, top_k)
    float32, sorted by z[0] descending."""
    rotations = np.asarray(rotations, np.float64)
    K_all = len(rotations)
    pixels = np.asarray(pixels, np.int32)
    npix, nr, ni = len(pixels), len(row_masks), len(inputs)
    top = [(np.full((npix, top_k), -1, np.int32),
            [np.full((npix, top_k), -np.inf, np.float32)] + [np.zeros((npix, top_k), np.float32)
                                                             for _ in range(nr - 1)]) for _ in range(ni)]
    t0 = time.perf_counter()
    for c0 in range(0, K_all, chunk):
        rc = rotations[c0:c0 + chunk]
        K = len(rc)
        op = make_operator(rc)
        datas = [a for pair in inputs for a in pair]
        for a in datas:
            check_device(a, op.data_shape, "input")
        s = op._s()
        n_max = op.K_batch_max * npix
        if gpu_scores:
            host = [[np.empty((op.K, npix), np.float32) for _ in range(nr)] for _ in range(ni)]
            e_keep = [torch.empty(n_max, dtype=torch.float32, device=op.device) for _ in range(nr)]
            zbuf = torch.empty(n_max, dtype=torch.float32, device=op.device)

            def consume(i, si, k0, Kb, block, host=host):
                n = Kb * npix
                if i % 2 == 0:               # E: kept until its D arrives (the block is reused)
                    _lib.call("dfx_copy_f32", block.data_ptr(), e_keep[si].data_ptr(), n, s)
                    return
                _lib.call("dfx_score_z", e_keep[si].data_ptr(), block.data_ptr(), zbuf.data_ptr(), n, s)
                host[i // 2][si][k0:k0 + Kb] = zbuf[:n].view(Kb, npix).cpu().numpy()
        else:
            host = [[np.empty((op.K, npix), np.float32) for _ in range(nr)] for _ in datas]

            def consume(i, si, k0, Kb, block, host=host):
                host[i][si][k0:k0 + Kb] = block[:Kb].cpu().numpy()

        op.adjoint_multi_cl(datas, consume, row_masks=row_masks, pixels=pixels, nrhs=nrhs,
                            rows_per_group=rows_per_group)
        for j in range(ni):
            if gpu_scores:
                z = [host[j][si] for si in range(nr)]
            else:
                z = []
                for si in range(nr):
                    e_, d_ = host[2 * j][si], host[2 * j + 1][si]
                    zz = e_ / np.sqrt(np.maximum(d_, np.float32(1e-30)))
                    zz[d_ <= 0] = 0
                    z.append(zz)
            top[j] = _merge(top[j], z, K, c0, top_k)
        op.free_memory()
        del op
        if verbose:
            print(f"  candidates {c0}..{c0 + K} scored ({time.perf_counter() - t0:.0f} s)", flush=True)
    out = []
    for idx, zs in top:
        o = np.argsort(-zs[0], axis=1, kind="stable")
        out.append({"idx": np.take_along_axis(idx, o, 1), "z": np.stack([np.take_along_axis(a, o, 1) for a in zs])})
    return out


# ------------------------------------------------------------------------------------------------ candidates
@dataclass
class Candidates:
    """Orientations the search proposes (orientation_search.py:232-246): rotations (n, 3, 3), score (n,) (the summed
    fitted z of their tile peaks), tiles (n arrays of flat indices x + Nx y of the scoring image) and tile_shape
    (Ny, Nx) of that image."""
    rotations: np.ndarray
    score: np.ndarray
    tiles: list
    tile_shape: tuple

    def __len__(self):
        return len(self.rotations)

    def subset(self, keep):
        """The candidates selected by a bool mask or an index array."""
        keep = np.asarray(keep)
        sel = np.flatnonzero(keep) if keep.dtype == bool else keep.astype(np.int64)
        return Candidates(self.rotations[sel], self.score[sel], [self.tiles[i] for i in sel], self.tile_shape)


def _quat_xyzw(mats):
    """Unit quaternions (x, y, z, w) of rotation matrices (n, 3, 3), float64."""
    from scipy.spatial.transform import Rotation
    return Rotation.from_matrix(np.asarray(mats, np.float64).reshape(-1, 3, 3)).as_quat()


def _symmetry_quats(symmetry):
    """(G, 4) quaternions of the proper rotations of a point group: matrices (G, 3, 3) (improper ones dropped) or a
    scipy Rotation."""
    from scipy.spatial.transform import Rotation
    if isinstance(symmetry, Rotation):
        return symmetry.as_quat()
    m = np.asarray(symmetry, np.float64).reshape(-1, 3, 3)
    return _quat_xyzw(m[np.linalg.det(m) > 0])


def _crystal_side(q, S):
    """(n, G, 4): every q (n, 4) composed with every symmetry rotation S (G, 4) on the crystal side, q * s."""
    a = q[:, None, :]
    b = S[None, :, :]
    ax, ay, az, aw = (a[..., i] for i in range(4))
    bx, by, bz, bw = (b[..., i] for i in range(4))
    return np.stack([aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw,
                     aw * bw - ax * bx - ay * by - az * bz], axis=-1)


def _within(qa, eq_b, angle_deg):
    """(len(qa), len(eq_b)) bool: misorientation of qa[i] and the orientation whose symmetry equivalents are eq_b[j]
    below angle_deg (|<q_a, q_b s>| above cos(angle / 2) for some s)."""
    c = np.cos(np.deg2rad(angle_deg) / 2.0)
    return np.abs(np.einsum("ic,jgc->ijg", qa, eq_b)).max(axis=2) > c


class _Links:
    """Union-find over n nodes; components(): the component of every node, numbered in the order of their smallest
    node."""

    def __init__(self, n):
        self.up = np.arange(n)

    def root(self, i):
        while self.up[i] != i:
            self.up[i] = self.up[self.up[i]]
            i = self.up[i]
        return i

    def join(self, i, j):
        a, b = self.root(i), self.root(j)
        if a != b:
            self.up[max(a, b)] = min(a, b)

    def components(self):
        roots = np.array([self.root(i) for i in range(len(self.up))], np.int64)
        _, label = np.unique(roots, return_inverse=True)       # roots are each component's smallest node
        return label


def select_candidates(real, null, rotations, pixels, tile_shape, symmetry, ratio=2.0, sep_deg=8.0, link_deg=5.0,
                      max_per_tile=3, min_tiles=2):
    """Candidates from the per-pixel top lists of score_candidates (orientation_search.py:271-350).

    A peak (a candidate in a tile's top list) qualifies when its fitted z (row set 0) reaches ratio x the null's best z
    in that tile and its held-out z (row set 1) reaches the null's best there. A tile keeps its qualifying peaks in
    rank order, at most max_per_tile, each sep_deg from those kept before it. Kept peaks of 8-neighbouring tiles within
    link_deg are linked; a connected group over at least min_tiles tiles is a candidate with its strongest peak's
    orientation and the sum of its peaks' fitted z as score. real, null: score_candidates dicts ("idx" (npix, top_k),
    "z" (n_rows, npix, top_k)); rotations: the scored list; pixels: (npix,) flat indices of the scoring image of shape
    tile_shape = (Ny, Nx); symmetry: the crystal's proper rotations (matrices or a scipy Rotation). Returns
    Candidates, the largest score first."""
    rotations = np.asarray(rotations, np.float64)
    pixels = np.asarray(pixels, np.int64)
    Ny, Nx = (int(v) for v in tile_shape)
    idx, z_fit, z_held = real["idx"], real["z"][0], real["z"][1]
    floor_fit = null["z"][0].max(axis=1)[:, None]
    floor_held = null["z"][1].max(axis=1)[:, None]
    good = (idx >= 0) & (z_fit >= ratio * floor_fit) & (z_held >= floor_held)
    none = Candidates(np.zeros((0, 3, 3)), np.zeros(0), [], (Ny, Nx))
    if not good.any():
        return none
    used, col = np.unique(idx[good], return_inverse=True)        # the candidate list entries that occur
    slot = np.full(idx.shape, -1, np.int64)
    slot[good] = col
    q = _quat_xyzw(rotations[used])
    eq = _crystal_side(q, _symmetry_quats(symmetry))
    # the kept peaks of every tile, tiles in the order of the scored pixels
    node_u, node_z, node_tile, first_of = [], [], [], {}
    for t in np.flatnonzero(good.any(axis=1)):
        ranks = np.flatnonzero(good[t])
        u = slot[t, ranks]
        near = _within(q[u], eq[u], sep_deg)
        kept = []
        for i in range(len(ranks)):
            if kept and near[i, kept].any():
                continue
            kept.append(i)
            if len(kept) == max_per_tile:
                break
        first_of[int(pixels[t])] = len(node_u)
        node_u.extend(u[kept])
        node_z.extend(z_fit[t, ranks[kept]])
        node_tile.extend([int(pixels[t])] * len(kept))
    node_u = np.asarray(node_u, np.int64)
    node_z = np.asarray(node_z, np.float64)
    node_tile = np.asarray(node_tile, np.int64)
    links = _Links(len(node_u))
    tiles = list(first_of)
    count = {p: int(np.count_nonzero(node_tile == p)) for p in tiles}
    for p in tiles:                       # each neighbour pair once: right, and the three below
        y, x = divmod(p, Nx)
        a0 = first_of[p]
        ua = node_u[a0:a0 + count[p]]
        for dy, dx in ((0, 0), (0, 1), (1, -1), (1, 0), (1, 1)):
            y2, x2 = y + dy, x + dx
            p2 = y2 * Nx + x2
            if not (0 <= y2 < Ny and 0 <= x2 < Nx) or p2 not in first_of:
                continue
            b0 = first_of[p2]
            ub = node_u[b0:b0 + count[p2]]
            for i, j in zip(*np.nonzero(_within(q[ua], eq[ub], link_deg))):
                links.join(a0 + i, b0 + j)
    label = links.components()
    rot, score, cand_tiles = [], [], []
    for c in range(label.max() + 1):
        members = np.flatnonzero(label == c)
        ts = np.unique(node_tile[members])
        if len(ts) < min_tiles:
            continue
        best = members[np.argmax(node_z[members])]
        rot.append(used[node_u[best]])
        score.append(float(node_z[members].sum()))
        cand_tiles.append(ts)
    if not rot:
        return none
    order = np.argsort(-np.asarray(score), kind="stable")
    return Candidates(rotations[np.asarray(rot)[order]], np.asarray(score)[order], [cand_tiles[i] for i in order],
                      (Ny, Nx))


def _voxels_of_tiles(tiles, tile_shape, tile_size, shape):
    """(iy, ix) of the image voxels covered by tiles (flat indices of the scoring image, tile_size voxels per edge),
    tile by tile, row-major inside a tile, cut to the image shape (Ny, Nx)."""
    tiles = np.asarray(tiles, np.int64)
    ty, tx = np.divmod(tiles, int(tile_shape[1]))
    dy, dx = np.divmod(np.arange(tile_size * tile_size), tile_size)
    iy = (ty[:, None] * tile_size + dy[None]).ravel()
    ix = (tx[:, None] * tile_size + dx[None]).ravel()
    inside = (iy < shape[0]) & (ix < shape[1])
    return iy[inside], ix[inside]


DEFAULT_LEVELS = ((1.25, 6.0, 1.0), (0.4, 1.6, 0.4))


def refine_candidates(make_local_operator, candidates, e, d, row_mask, tile_size, shape, levels=DEFAULT_LEVELS,
                      verbose=False):
    """Each candidate moved to the best orientation of finer rotation lattices around it (orientation_search.py:
    366-429). Per level (spacing, radius, sigma; degrees): the rotation vectors of the cubic lattice of that spacing
    within the radius, applied on the crystal side, are scored with z = sum E / sqrt(sum D) over the candidate's voxels
    on the fitted angles (E, D: the adjoints of e and d restricted to row_mask), and the best becomes the candidate's
    orientation. make_local_operator(rotations, sigmas (radians), k, iy, ix) -> a LocalSinglePhaseForwardOperator with
    those orientations on the pairs (k, iy, ix); e, d: NumPy data arrays; tile_size: voxels per tile edge of the
    scoring image; shape: (Ny, Nx). Returns Candidates with the same tiles and scores."""
    n = len(candidates)
    if n == 0:
        return candidates
    R = np.asarray(candidates.rotations, np.float64).copy()
    rows = np.asarray(row_mask, np.float32).reshape(-1, 1, 1)
    e_fit = np.ascontiguousarray(np.asarray(e, np.float32) * rows)
    d_fit = np.ascontiguousarray(np.asarray(d, np.float32) * rows)
    vox = [_voxels_of_tiles(t, candidates.tile_shape, tile_size, shape) for t in candidates.tiles]
    from scipy.spatial.transform import Rotation

    def lattice_scores(rots, sigma, owner):
        """z of every trial orientation (owner[i]: its candidate) over its candidate's voxels."""
        ks, iys, ixs = [], [], []
        for j in range(n):
            trials = np.flatnonzero(owner == j)
            iy, ix = vox[j]
            ks.append(np.repeat(trials, len(iy)))
            iys.append(np.tile(iy, len(trials)))
            ixs.append(np.tile(ix, len(trials)))
        k, iy, ix = (np.concatenate(a) for a in (ks, iys, ixs))
        op = make_local_operator(rots, np.full(len(rots), np.deg2rad(sigma)), k, iy, ix)
        sums = []
        for arr in (e_fit, d_fit):
            out = torch.zeros(op.coeff_shape, dtype=torch.float32, device=op.device)
            op.adjoint_cl(torch.as_tensor(arr, device=op.device), out)
            kk, _, _, v = op.to_coo(out.cpu().numpy())
            sums.append(np.bincount(kk, weights=np.asarray(v, np.float64), minlength=len(rots)))
        op.free_memory()
        return sums[0] / np.sqrt(np.maximum(sums[1], 1e-30))

    for spacing, radius, sigma in levels:
        m = int(np.ceil(radius / spacing))
        steps = np.arange(-m, m + 1) * spacing
        vecs = np.stack(np.meshgrid(steps, steps, steps, indexing="ij"), -1).reshape(-1, 3)
        vecs = vecs[np.linalg.norm(vecs, axis=1) <= radius + 1e-9]
        turns = Rotation.from_rotvec(np.deg2rad(vecs)).as_matrix()
        trials = np.einsum("nij,tjk->ntik", R, turns).reshape(-1, 3, 3)
        owner = np.repeat(np.arange(n), len(vecs))
        z = lattice_scores(trials, sigma, owner).reshape(n, len(vecs))
        R = trials.reshape(n, len(vecs), 3, 3)[np.arange(n), np.argmax(z, axis=1)]
        if verbose:
            print(f"  lattice {spacing} deg within {radius} deg (sigma {sigma} deg): {len(trials)} orientations",
                  flush=True)
    return Candidates(R, candidates.score, candidates.tiles, candidates.tile_shape)


def candidate_support(candidates, tile_size, shape, dilate=0, mask=None):
    """(k, iy, ix) int64 arrays of the voxels of every candidate (k its index): its tiles' voxels, grown by dilate
    steps of a binary dilation with the 4-neighbour cross (scipy.ndimage's default structure) and cut to the (Ny, Nx)
    bool mask if given (orientation_search.py:432-449); the arguments of a LocalSupport."""
    from scipy import ndimage
    parts = []
    for j, t in enumerate(candidates.tiles):
        iy, ix = _voxels_of_tiles(t, candidates.tile_shape, tile_size, shape)
        img = np.zeros(shape, bool)
        img[iy, ix] = True
        if dilate:
            img = ndimage.binary_dilation(img, iterations=int(dilate))
        if mask is not None:
            img &= np.asarray(mask, bool)
        y, x = np.nonzero(img)
        parts.append((np.full(len(y), j, np.int64), y.astype(np.int64), x.astype(np.int64)))
    if not parts:
        return tuple(np.zeros(0, np.int64) for _ in range(3))
    return tuple(np.concatenate([p[i] for p in parts]) for i in range(3))


def orientation_weights(coefficients, k=None):
    """The total (non-negative part of the) coefficient of every orientation: from a dense (K, Ny, Nx) array, or from
    a local basis's values with their orientation indices k (to_coo) (orientation_search.py:452-458)."""
    c = np.maximum(np.asarray(coefficients, np.float64), 0.0)
    if k is not None:
        return np.bincount(np.asarray(k, np.int64), weights=c)
    return c.reshape(c.shape[0], -1).sum(axis=1)


def prune_added(weights, n_old, rel=0.1):
    """Bool keep-mask: the first n_old orientations, and the added ones whose weight reaches rel x the median weight
    of the added ones that received any (none if no added one did) (orientation_search.py:461-470)."""
    w = np.asarray(weights, np.float64)
    keep = np.ones(len(w), bool)
    added = w[n_old:]
    got = added[added > 0]
    keep[n_old:] = added >= rel * np.median(got) if got.size else False
    return keep
