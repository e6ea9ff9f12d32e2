"""Fourier-slice parallel-beam projector (diffractom's FourierRadon, operators/fourier_radon.py), tables on the host.

The geometry and conventions are those of the native projector (detector coordinate t = X x + Y y + T0 in bins,
forward scaled by delta_x^2 / delta_s, backward = the transpose weighted by the angle weights). For angle a and bin
s the forward projection is the Fourier slice theorem on an L-point detector line,

    P f [a, s] = 1/L sum_{j = -L/2+1}^{L/2} fhat(w_j X_a, w_j Y_a) e^{-i w_j T_a} h(w_j) e^{i w_j s},

w_j = 2 pi j / L, h(w) = sinc^2(w / 2 pi) the transform of the bin's hat, T_a the detector coordinate of pixel
(cx, cy) = (Nx // 2, Ny // 2), fhat the discrete-time transform of the pixels about (cx, cy). fhat at the polar
samples is a type-2 non-uniform FFT with the "exponential of semicircle" kernel phi(z) = exp(beta (sqrt(1 - z^2) -
1)) of W taps (Barnett, Magland, af Klinteberg, SIAM J. Sci. Comput. 41 (2019), FINUFFT): pixels divided by the
kernel's transform psi, zero-padded to an oversampled grid (sigma = 1.5), a 2-D real FFT, and per sample a W x W
interpolation. The backward projection is the transpose of the same float32 steps (spreading as a gather over the
grid's tiles). The numbers that fix the method (sigma 1.5, W 7, beta = 0.97 pi (1 - 1 / (2 sigma)) W, L = the
smallest 7-smooth even length >= 1.25 x the span of the projections, the 4001-point quadrature of psi, 16 x 16
spreading tiles) are diffractom's (fourier_radon.py:101-209), so that the two implementations compute the same
approximation.

This module builds the float32 tables (per angle set: the full scan, or one omega subset) and uploads them; the
device work is dfx_fr_forward / dfx_fr_backward (csrc/fourier.cu: the pad, slice, line, spread and crop kernels
around cuFFT plans).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

SIGMA, W_TAPS, L_FACTOR, TILE, PIECE = 1.5, 7, 1.25, 16, 512


def smooth_length(n, even=True):
    """The smallest m >= n whose prime factors are 2, 3, 5, 7 (an efficient FFT length), even if asked."""
    m = int(np.ceil(n))
    while True:
        k = m
        for p in (2, 3, 5, 7):
            while k % p == 0:
                k //= p
        if k == 1 and (not even or m % 2 == 0):
            return m
        m += 1


def es_kernel(z, beta):
    """phi(z) = exp(beta (sqrt(1 - z^2) - 1)) for |z| < 1, else 0."""
    z = np.asarray(z, np.float64)
    out = np.zeros_like(z)
    inside = np.abs(z) < 1
    out[inside] = np.exp(beta * (np.sqrt(1.0 - z[inside] ** 2) - 1.0))
    return out


def deapodisation(n, c, M, W, beta):
    """1 / psi(x - c) for x = 0 .. n-1, psi(x) = int phi(2 kappa / W) cos(2 pi kappa x / M) dkappa over
    [-W/2, W/2] (a 4001-point Riemann sum), float32."""
    kap = np.linspace(-W / 2, W / 2, 4001)
    phi = es_kernel(2 * kap / W, beta)
    x = np.arange(n, dtype=np.float64) - c
    psi = (phi[None, :] * np.cos(2 * np.pi * kap[None, :] * x[:, None] / M)).sum(1) * (kap[1] - kap[0])
    return (1.0 / psi).astype(np.float32)


class FourierTables:
    """The float32 tables of one angle set (host arrays): per polar sample (angle a, frequency j = 0 .. H-1) the
    first tap (k1, k2) on the oversampled grid, the W tap weights per dimension, the phase / bin response filt; the
    spreading tiles; the angle weights."""

    def __init__(self, X, Y, T, angle_weights, Mx, My, L, W, beta):
        R = len(X)
        H = L // 2 + 1
        self.R, self.H, self.RH = R, H, R * H
        om = 2 * np.pi * np.arange(H) / L
        filt = (np.sinc(om / (2 * np.pi)) ** 2)[None, :] * np.exp(-1j * om[None, :] * T[:, None]) / L
        self.filt = np.ascontiguousarray(filt.astype(np.complex64).ravel())
        ku = (Mx * om[None, :] * X[:, None] / (2 * np.pi)).ravel()
        kv = (My * om[None, :] * Y[:, None] / (2 * np.pi)).ravel()
        k1b = (np.floor(ku - W / 2) + 1).astype(np.int64)
        k2b = (np.floor(kv - W / 2) + 1).astype(np.int64)
        taps = np.arange(W)
        self.w1 = np.ascontiguousarray(es_kernel(2 * (ku[:, None] - (k1b[:, None] + taps)) / W, beta), np.float32)
        self.w2 = np.ascontiguousarray(es_kernel(2 * (kv[:, None] - (k2b[:, None] + taps)) / W, beta), np.float32)
        self.kb = np.ascontiguousarray(np.stack([k1b, k2b], 1), np.int32)
        # spreading as a gather: for every TILE x TILE tile of the half grid (rows k2, columns k1 <= Mx/2), the
        # samples with a tap on it directly (k) or through the Hermitian mirror (-k), sorted by (tile, mirror,
        # sample); a mirrored sample is stored as -(sample + 1)
        Hx = Mx // 2 + 1
        self.n_tx = -(-Hx // TILE)
        n_ty = -(-My // TILE)
        self.n_tiles = self.n_tx * n_ty
        RH = self.RH
        k1 = np.broadcast_to((k1b[:, None] + taps)[:, None, :], (RH, W, W))      # [sample, l, i] -> k1b + i
        k2 = np.broadcast_to((k2b[:, None] + taps)[:, :, None], (RH, W, W))      # [sample, l, i] -> k2b + l
        smp = np.broadcast_to(np.arange(RH)[:, None, None], (RH, W, W))
        keys = []
        for sgn, mir in ((1, 0), (-1, 1)):
            c1, c2 = (sgn * k1) % Mx, (sgn * k2) % My
            ok = c1 <= Mx // 2
            tile = (c2[ok] // TILE) * self.n_tx + c1[ok] // TILE
            keys.append((tile * 2 + mir) * RH + smp[ok])
        keys = np.unique(np.concatenate(keys))
        tile, mir, s = keys // (2 * RH), (keys // RH) % 2, keys % RH
        tile_ptr = np.zeros(self.n_tiles + 1, np.int64)
        np.cumsum(np.bincount(tile, minlength=self.n_tiles), out=tile_ptr[1:])
        if tile_ptr[-1] >= 2 ** 31:
            raise ValueError("too many spreading entries for 32-bit indices")
        self.tile_ptr = tile_ptr.astype(np.int32)
        self.tile_smp = np.where(mir == 1, -s - 1, s).astype(np.int32)
        # the lists are very uneven (the tiles at the origin collect the low frequencies of every angle): a list is
        # cut into pieces of at most PIECE samples, one block each; a tile's first piece writes the spectrum, the
        # others partial tiles (slots) that are added to it afterwards in the pieces' order
        cnt = np.diff(tile_ptr)
        n_pc = np.maximum(1, -(-cnt // PIECE))
        first = np.concatenate([[0], np.cumsum(n_pc)[:-1]])
        tile_of = np.repeat(np.arange(self.n_tiles), n_pc)
        k = np.arange(len(tile_of)) - first[tile_of]                 # piece number within its tile
        e0 = tile_ptr[tile_of] + k * PIECE
        e1 = np.minimum(e0 + PIECE, tile_ptr[tile_of + 1])
        extra = np.maximum(0, n_pc - 1)
        self.tile_xptr = np.concatenate([[0], np.cumsum(extra)]).astype(np.int32)
        slot = np.where(k == 0, -1, self.tile_xptr[tile_of] + k - 1)
        self.pieces = np.ascontiguousarray(np.stack([tile_of, e0, e1, slot], 1), np.int32)
        self.n_slots = int(self.tile_xptr[-1])
        self.wa = np.ascontiguousarray(np.broadcast_to(np.asarray(angle_weights, np.float64), (R,)), np.float32)


class FRGeometry(ctypes.Structure):
    """dfx_fr_geometry (include/diffractom_b200.h): device pointers of one angle set's tables and the sizes."""
    _fields_ = [("inv_dx", ctypes.c_void_p), ("inv_dy", ctypes.c_void_p), ("filt", ctypes.c_void_p),
                ("kb", ctypes.c_void_p), ("w1", ctypes.c_void_p), ("w2", ctypes.c_void_p),
                ("tile_ptr", ctypes.c_void_p), ("tile_smp", ctypes.c_void_p), ("wa", ctypes.c_void_p),
                ("pieces", ctypes.c_void_p), ("tile_xptr", ctypes.c_void_p),
                ("Nx", ctypes.c_int32), ("Ny", ctypes.c_int32), ("Ns", ctypes.c_int32), ("R", ctypes.c_int32),
                ("L", ctypes.c_int32), ("H", ctypes.c_int32), ("Mx", ctypes.c_int32), ("My", ctypes.c_int32),
                ("W", ctypes.c_int32), ("cx", ctypes.c_int32), ("cy", ctypes.c_int32), ("n_tx", ctypes.c_int32),
                ("n_tiles", ctypes.c_int32), ("n_pieces", ctypes.c_int32), ("n_slots", ctypes.c_int32),
                ("scale", ctypes.c_float)]


class FourierHost:
    """The host side of the projector of a geometry: sizes (L, Mx, My, W, beta, cx, cy, scale), per-angle X, Y, T
    and the deapodisation (float32 host arrays); tables(idx) gives the FourierTables of the angles idx."""

    def __init__(self, angles, Nx, Ny, Ns, image_width, detector_width, detector_shift, angle_weights, W=W_TAPS,
                 sigma=SIGMA, L_factor=L_FACTOR):
        angles = np.asarray(angles, np.float64)
        self.Nx, self.Ny, self.Ns = int(Nx), int(Ny), int(Ns)
        R = len(angles)
        self.weights_all = np.broadcast_to(np.asarray(angle_weights, np.float64), (R,)).copy()
        delta_x = image_width / float(max(self.Nx, self.Ny))
        delta_s = float(detector_width) / self.Ns
        rho = delta_s / delta_x
        X = np.cos(angles - 0.5 * np.pi) / rho
        Y = np.sin(angles - 0.5 * np.pi) / rho
        T0 = ((self.Ns - 1) / 2.0 - X * (self.Nx - 1) / 2.0 - Y * (self.Ny - 1) / 2.0
              - np.asarray(detector_shift, np.float64) / delta_s)
        self.scale = np.float32(delta_x * delta_x / delta_s)
        self.cx, self.cy = self.Nx // 2, self.Ny // 2
        self.XYT_all = (X, Y, T0 + X * self.cx + Y * self.cy)
        corners = np.array([[0, 0], [self.Nx - 1, 0], [0, self.Ny - 1], [self.Nx - 1, self.Ny - 1]], float)
        t = corners[:, :1] * X[None, :] + corners[:, 1:] * Y[None, :] + T0[None, :]
        span = max(t.max(), self.Ns - 1) - min(t.min(), 0.0) + 4
        self.L = smooth_length(L_factor * span)
        self.W = int(W)
        if self.W not in (6, 7):
            raise ValueError("the interpolation kernel has 6 or 7 taps")
        self.beta = 0.97 * np.pi * (1 - 1 / (2 * sigma)) * self.W
        self.Mx, self.My = smooth_length(sigma * self.Nx), smooth_length(sigma * self.Ny)
        self.inv_dx = deapodisation(self.Nx, self.cx, self.Mx, self.W, self.beta)
        self.inv_dy = deapodisation(self.Ny, self.cy, self.My, self.W, self.beta)

    def tables(self, idx=None):
        idx = np.arange(len(self.weights_all)) if idx is None else np.asarray(idx, np.int64)
        X, Y, T = (a[idx] for a in self.XYT_all)
        return FourierTables(X, Y, T, self.weights_all[idx], self.Mx, self.My, self.L, self.W, self.beta)


class FourierProjector:
    """The Fourier-slice projector of a geometry on the device; subset(idx) gives the projector of some angles
    (their own polar samples and spreading tiles, the same grid and deapodisation)."""

    def __init__(self, host: FourierHost, device, idx=None, _inv=None):
        self.host, self.device = host, device
        for k in ("Nx", "Ny", "Ns", "scale", "cx", "cy", "L", "W", "Mx", "My"):
            setattr(self, k, getattr(host, k))
        dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=device)
        self.inv_dx, self.inv_dy = _inv if _inv is not None else (dev(host.inv_dx), dev(host.inv_dy))
        tab = host.tables(idx)
        self.R, self.H, self.RH = tab.R, tab.H, tab.RH
        self.filt = dev(tab.filt.view(np.float32))
        self.kb = dev(tab.kb)
        self.w1, self.w2 = dev(tab.w1), dev(tab.w2)
        self.tile_ptr, self.tile_smp = dev(tab.tile_ptr), dev(tab.tile_smp)
        self.wa = dev(tab.wa)
        self.pieces, self.tile_xptr = dev(tab.pieces), dev(tab.tile_xptr)
        self.geom = FRGeometry(self.inv_dx.data_ptr(), self.inv_dy.data_ptr(), self.filt.data_ptr(),
                               self.kb.data_ptr(), self.w1.data_ptr(), self.w2.data_ptr(), self.tile_ptr.data_ptr(),
                               self.tile_smp.data_ptr(), self.wa.data_ptr(), self.pieces.data_ptr(),
                               self.tile_xptr.data_ptr(), self.Nx, self.Ny, self.Ns, self.R, self.L, self.H, self.Mx,
                               self.My, self.W, self.cx, self.cy, tab.n_tx, tab.n_tiles, len(tab.pieces),
                               tab.n_slots, float(self.scale))

    def subset(self, idx):
        return FourierProjector(self.host, self.device, idx, _inv=(self.inv_dx, self.inv_dy))

    def nbytes(self):
        return sum(t.numel() * t.element_size() for t in (self.filt, self.kb, self.w1, self.w2, self.tile_ptr,
                                                           self.tile_smp, self.wa, self.pieces, self.tile_xptr))

    def scratch_bytes(self, channels):
        n = int(_lib.lib().dfx_fr_scratch_bytes(ctypes.byref(self.geom), int(channels)))
        if n == 0:
            raise RuntimeError(_lib.lib().dfx_last_error().decode(errors="replace") or "fr_scratch_bytes failed")
        return n

    def forward(self, img_k, sino, kstride, kb, channels, scratch, nbytes, stream):
        """sino (R, Ns, kstride) channels 0 .. kb-1 = forward projections of the channel-fastest batch img_k
        (npix, kstride); padding channels 0. img_k, sino, scratch: device addresses."""
        _lib.call("dfx_fr_forward", ctypes.byref(self.geom), img_k, sino, int(kstride), int(kb), int(channels),
                  scratch, int(nbytes), stream)

    def backward(self, sino, img_k, kstride, kb, channels, scratch, nbytes, stream):
        """img_k (npix, kstride) channels 0 .. kb-1 = the backward projection (transpose, angle weights) of sino;
        padding channels 0."""
        _lib.call("dfx_fr_backward", ctypes.byref(self.geom), sino, img_k, int(kstride), int(kb), int(channels),
                  scratch, int(nbytes), stream)
