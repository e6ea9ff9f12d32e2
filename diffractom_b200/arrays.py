"""Array conventions of the operators and solvers (diffractom/utils/arrays.py:1-47), with torch CUDA tensors in place
of pyopencl arrays.

  coefficients  (K, Ny, Nx) float32, C-contiguous: coeffs[k] is the image of orientation k
  data          (N_Omega, My, N_seg), N_seg = N_eta * N_rings, segment j = eta_bin * N_rings + ring
  weights etc.  N_seg, My * N_seg or data-shaped (periodic, see solvers)
  support       (Ny, Nx) bool
"""
from __future__ import annotations

import numpy as np
import torch


def is_device(a) -> bool:
    return isinstance(a, torch.Tensor) and a.is_cuda


def check_device(a, shape, name):
    """A CUDA tensor of the given shape, float32 and contiguous; TypeError / ValueError otherwise."""
    if not isinstance(a, torch.Tensor) or not a.is_cuda:
        raise TypeError(f"{name} must be a CUDA torch tensor (or a NumPy array where accepted), not "
                        f"{type(a).__name__}{'' if not isinstance(a, torch.Tensor) else ' on ' + str(a.device)}")
    if a.dtype != torch.float32:
        raise TypeError(f"{name} must be float32, not {a.dtype}")
    if tuple(a.shape) != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}, not {tuple(a.shape)}")
    if not a.is_contiguous():
        raise ValueError(f"{name} must be contiguous (e.g. tensor.contiguous())")
    return a


def as_host(a, shape, name):
    """A C-contiguous float32 NumPy array of the given shape: a itself if it already is one, else a converted copy."""
    out = np.ascontiguousarray(a, dtype=np.float32)
    if out.shape != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}, not {out.shape}")
    return out


def ptr(t) -> int | None:
    """Device address of a tensor (None for None)."""
    return None if t is None else t.data_ptr()
