"""Coefficient arrays in host memory, streamed through the GPU batch by batch (diffractom/optimization/streaming.py).

A batch goes host -> pinned staging buffer (a CPU copy) -> device slot (an async copy on the upload stream), is used
by the compute stream, and results go device slot -> pinned (download stream) -> host. Two slots per direction:
batch ib + 1 is uploaded while batch ib is computed. Ordering between the streams uses CUDA events only; the host
waits for an event only before it reuses a pinned buffer.
"""
from __future__ import annotations

import weakref

import numpy as np
import torch


class Streamer:
    """Double-buffered host <-> device transfers of (K, Ny, Nx) coefficient batches of one operator."""

    def __init__(self, op):
        self.op = weakref.proxy(op)
        self.device = op.device
        self.npix = op.Nx * op.Ny
        n = self.npix * op.K_batch_max
        self.n = n
        self.up_stream = torch.cuda.Stream(self.device)
        self.dn_stream = torch.cuda.Stream(self.device)
        self.slots = [torch.empty(n, dtype=torch.float32, device=self.device) for _ in range(2)]
        self.pin_up = [torch.empty(n, dtype=torch.float32, pin_memory=True) for _ in range(2)]
        self.pin_dn = [torch.empty(n, dtype=torch.float32, pin_memory=True) for _ in range(2)]
        self._up_done = [None, None]    # event: upload from pin_up[s] finished (pinned buffer reusable)
        self._slot_free = [None, None]  # event: compute on slot s finished

    def release(self):
        self.slots = self.pin_up = self.pin_dn = []

    def _view(self, flat, ib):
        b = self.op.batches[ib]
        return flat[self.npix * b["k_start"]:self.npix * (b["k_start"] + b["K_batch"])]

    def _upload(self, host_view, s):
        if self._up_done[s] is not None:
            self._up_done[s].synchronize()
        n = host_view.size
        np.copyto(self.pin_up[s].numpy()[:n], host_view)
        with torch.cuda.stream(self.up_stream):
            if self._slot_free[s] is not None:
                self.up_stream.wait_event(self._slot_free[s])
            self.slots[s][:n].copy_(self.pin_up[s][:n], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.up_stream)
        self._up_done[s] = ev
        return ev

    def forward(self, src_flat, data):
        """data = A src for a host coefficient array (flattened (K, Ny, Nx))."""
        op = self.op
        comp = op.stream()
        op._fill(data, 0.0)
        ev = self._upload(self._view(src_flat, 0), 0)
        for ib in range(len(op.batches)):
            s = ib % 2
            comp.wait_event(ev)
            if ib + 1 < len(op.batches):
                ev_next = self._upload(self._view(src_flat, ib + 1), 1 - s)
            op._direct_batch(self.slots[s], 0, op.K_batch_max, ib, data)
            done = torch.cuda.Event()
            done.record(comp)
            self._slot_free[s] = done
            if ib + 1 < len(op.batches):
                ev = ev_next

    def adjoint_to_host(self, data, out_flat):
        """out = A^T data, written batch by batch into a host array (flattened (K, Ny, Nx))."""
        op = self.op
        comp = op.stream()
        pending = []
        for ib in range(len(op.batches)):
            s = ib % 2
            if len(pending) == 2:
                self._finish_download(*pending.pop(0))
            if self._slot_free[s] is not None:
                comp.wait_event(self._slot_free[s])
            op._adjoint_batch(data, ib, self.slots[s], 0, op.K_batch_max)
            done = torch.cuda.Event()
            done.record(comp)
            n = self.npix * op.batches[ib]["K_batch"]
            with torch.cuda.stream(self.dn_stream):
                self.dn_stream.wait_event(done)
                self.pin_dn[s][:n].copy_(self.slots[s][:n], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.dn_stream)
            self._slot_free[s] = ev
            pending.append((ev, s, self._view(out_flat, ib)))
        while pending:
            self._finish_download(*pending.pop(0))

    def _finish_download(self, ev, s, host_view):
        ev.synchronize()
        np.copyto(host_view, self.pin_dn[s].numpy()[:host_view.size])


def streamer_for(op) -> Streamer:
    """The operator's streamer, made on first use and kept (op.release_streamer frees it)."""
    if op._streamer is None:
        op._streamer = Streamer(op)
    return op._streamer
