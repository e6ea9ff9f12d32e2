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


def as_host(a, shape, name, writeable=False):
    """A C-contiguous float32 NumPy array of the given shape: a itself if it already is one, else a converted copy.
    writeable: the caller writes its result into the array (a solver's x0), so a read-only array (a read-only memory
    map, a view of bytes) is copied as well; the copy is what the solver returns."""
    out = np.ascontiguousarray(a, dtype=np.float32)
    if out.shape != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}, not {out.shape}")
    if writeable and not out.flags.writeable:
        out = out.copy()
    return out


def ptr(t) -> int | None:
    """Device address of a tensor (None for None)."""
    return None if t is None else t.data_ptr()


class stream_scope:
    """Runs a block with an operator's stream current (operators built with queue=<torch.cuda.Stream>). The stream
    first waits for the caller's current stream (inputs written there), and the caller's stream waits for it at the
    end (results visible there), so torch work and the operator's kernels stay ordered whichever stream the caller
    uses. Without a queue, or when the queue is already current, nothing changes."""

    def __init__(self, op):
        self.q = getattr(op, "queue", None)
        self.dev = op.device
        self.cur = None
        self.ctx = None

    def __enter__(self):
        if self.q is None:
            return self
        cur = torch.cuda.current_stream(self.dev)
        if cur == self.q:
            return self
        self.cur = cur
        self.q.wait_stream(cur)
        self.ctx = torch.cuda.stream(self.q)
        self.ctx.__enter__()
        return self

    def __exit__(self, *exc):
        if self.ctx is not None:
            self.ctx.__exit__(*exc)
            self.cur.wait_stream(self.q)
            self.ctx = self.cur = None
        return False


def on_op_stream(method):
    """Decorator: the method of an operator (self) or of a solver (self.op) runs inside stream_scope."""
    import functools

    @functools.wraps(method)
    def wrapper(self, *args, **kwargs):
        op = self.op if hasattr(self, "op") and not hasattr(self, "batches") else self
        with stream_scope(op):
            return method(self, *args, **kwargs)
    return wrapper
