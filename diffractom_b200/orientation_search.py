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
"""
from __future__ import annotations

import time

import numpy as np
import torch

from . import _lib
from .arrays import check_device

__all__ = ["poisson_score_inputs", "scramble_eta", "score_candidates"]


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
