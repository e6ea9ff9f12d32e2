"""Oracle (test infrastructure only) of the Fourier-slice projector: the exact projection that the type-2 NUFFT of
diffractom's FourierRadon (operators/fourier_radon.py:1-30) approximates to about 1e-5, in float64.

For angle a, bin s and a pixel at detector coordinate t = X_a x + Y_a y + T0_a (the native projector's coordinate,
parallel_radon.py:106-124), the projection through the Fourier slice theorem on an L-point line with the bin
response h(w) = sinc^2(w / 2 pi), w_j = 2 pi j / L, is

    M[a, s, pixel] = 1/L (h_0 + 2 sum_{j=1}^{L/2-1} h_j cos(w_j (s - t)) + h_{L/2} cos(pi (s - t)))

(the real line of the Hermitian sum over j = -L/2+1 .. L/2; at the Nyquist frequency its real part, as the
reference's fr_slices keeps, fourier_radon.cl:78-82). forward = scale M f, backward = sum_a w_a M^T (no scale),
the conventions of the native projector. L is the reference's padded line length: the smallest even 2,3,5,7-smooth
length >= 1.25 x (the span of the projections + 4 bins) (fourier_radon.py:120-124). Dense: small geometries only.
The reference's own output (VkFFT through pyopencl) cannot be produced here, so parity for this projector rests on
this exact formula, on the adjoint identity and on the agreement with the native projector that the reference
documents (about 1 %).
"""
from __future__ import annotations

import numpy as np


def _smooth(n):
    m = int(np.ceil(n))
    while True:
        k = m
        for p in (2, 3, 5, 7):
            while k % p == 0:
                k //= p
        if k == 1 and m % 2 == 0:
            return m
        m += 1


def fourier_slice_matrix(angles, Nx, Ny, Ns, image_width, detector_width, detector_shift=0.0, L_factor=1.25):
    """(M (R, Ns, Nx*Ny) float64, scale, L): the exact Fourier-slice projection of the geometry (pixel p = x + Nx y)."""
    angles = np.asarray(angles, np.float64)
    delta_x = image_width / float(max(Nx, Ny))
    delta_s = float(detector_width) / Ns
    rho = delta_s / delta_x
    X = np.cos(angles - 0.5 * np.pi) / rho
    Y = np.sin(angles - 0.5 * np.pi) / rho
    T0 = (Ns - 1) / 2.0 - X * (Nx - 1) / 2.0 - Y * (Ny - 1) / 2.0 - np.asarray(detector_shift, np.float64) / delta_s
    corners = np.array([[0, 0], [Nx - 1, 0], [0, Ny - 1], [Nx - 1, Ny - 1]], float)
    tc = corners[:, :1] * X[None, :] + corners[:, 1:] * Y[None, :] + T0[None, :]
    L = _smooth(L_factor * (max(tc.max(), Ns - 1) - min(tc.min(), 0.0) + 4))
    yy, xx = np.mgrid[:Ny, :Nx]
    t = X[:, None] * xx.ravel()[None, :] + Y[:, None] * yy.ravel()[None, :] + T0[:, None]      # (R, npix)
    d = np.arange(Ns, dtype=np.float64)[None, :, None] - t[:, None, :]                         # (R, Ns, npix)
    M = np.ones(d.shape)                                                                       # j = 0: h_0 = 1
    for j in range(1, L // 2):
        M += 2 * np.sinc(j / L) ** 2 * np.cos(2 * np.pi * j / L * d)
    M += np.sinc(0.5) ** 2 * np.cos(np.pi * d)
    M /= L
    return M, float(np.float32(delta_x * delta_x / delta_s)), L


def forward(M, scale, img):
    """sino (R, Ns, C) = scale M img, img (npix, C) channel-fastest."""
    R, Ns, npix = M.shape
    return scale * (M.reshape(R * Ns, npix) @ np.asarray(img, np.float64)).reshape(R, Ns, -1)


def backward(M, weights, sino):
    """img (npix, C) = sum_a w_a M[a]^T sino[a], sino (R, Ns, C)."""
    R, Ns, npix = M.shape
    ws = np.asarray(sino, np.float64) * np.broadcast_to(np.asarray(weights, np.float64), (R,))[:, None, None]
    return M.reshape(R * Ns, npix).T @ ws.reshape(R * Ns, -1)
