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


# ---------------------------------------------------------------------------------------------- solver state
# A solver's coefficient-sized state (x, z, T of SPDHG) is kept in the operator's channel-fastest batch layout, batch
# ib at element ib * npix * Kstride. An array that does not stay on the device lives in pinned host memory in that
# same layout, so a batch crosses the host link as one contiguous copy in each direction, and two device slots hold
# the batches in use (spdhg_poisson.py:287-296, streaming.py:255-309 of diffractom).

class CoeffArray:
    """One coefficient-sized state array: resident (one flat device array) or streamed (pinned host array + two
    device slots). ptr(ib, s) is the device address of batch ib while it sits in slot s."""

    def __init__(self, op, name, resident, dtype=torch.float32):
        self.name = name
        self.be = op.batch_elems()
        self.n_batches = len(op.batches)
        self.esize = torch.empty(0, dtype=dtype).element_size()
        n = self.n_batches * self.be
        if resident:
            self.dev = torch.empty(n, dtype=dtype, device=op.device)
            self.host = self.slots = None
        else:
            self.dev = None
            self.host = torch.empty(n, dtype=dtype, pin_memory=True)
            self.slots = [torch.empty(self.be, dtype=dtype, device=op.device) for _ in range(2)]
        self.host_ready = [None] * self.n_batches    # event: the last download of batch ib into host has finished

    @property
    def resident(self):
        return self.dev is not None

    def ptr(self, ib, s):
        if self.dev is not None:
            return self.dev.data_ptr() + self.esize * ib * self.be
        return self.slots[s].data_ptr()

    def host_batch(self, ib):
        return self.host[ib * self.be:(ib + 1) * self.be]

    def nbytes_device(self):
        t = [self.dev] if self.dev is not None else self.slots
        return sum(x.numel() * x.element_size() for x in t)


class BatchPipeline:
    """Runs a pass over the orientation batches with the streamed state arrays moving through their two slots:
    batch ib + 1 is uploaded (upload stream) while batch ib is computed (the operator's stream), and the updated
    arrays of batch ib go back to host memory on the download stream. Ordering is by CUDA events only: an upload into
    a slot waits for the compute and the download of the batch that used it before, and the upload of a batch waits
    for the previous download of that batch's host memory; the host never waits."""

    def __init__(self, op):
        self.op = op
        self.up = torch.cuda.Stream(op.device)
        self.dn = torch.cuda.Stream(op.device)
        self.slot_free = [None, None]

    def _upload(self, arrays, ib):
        s = ib % 2
        if not arrays:
            return None
        with torch.cuda.stream(self.up):
            if self.slot_free[s] is not None:
                self.up.wait_event(self.slot_free[s])
            for c in arrays:
                if c.host_ready[ib] is not None:
                    self.up.wait_event(c.host_ready[ib])
                c.slots[s].copy_(c.host_batch(ib), non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.up)
        return ev

    def run(self, ups, dns, compute):
        """compute(ib, s) launches batch ib's work on the operator's stream with the arrays of ups in slot s; the
        arrays of dns are written back to host memory afterwards. Resident arrays in ups / dns are ignored."""
        ups = [c for c in ups if not c.resident]
        dns = [c for c in dns if not c.resident]
        nbt = len(self.op.batches)
        if not ups and not dns:
            for ib in range(nbt):
                compute(ib, ib % 2)
            return
        comp = self.op.stream()
        ev = self._upload(ups, 0)
        for ib in range(nbt):
            s = ib % 2
            nxt = self._upload(ups, ib + 1) if ib + 1 < nbt else None
            if ev is not None:
                comp.wait_event(ev)
            elif self.slot_free[s] is not None:
                comp.wait_event(self.slot_free[s])
            compute(ib, s)
            done = torch.cuda.Event()
            done.record(comp)
            if dns:
                with torch.cuda.stream(self.dn):
                    self.dn.wait_event(done)
                    for c in dns:
                        c.host_batch(ib).copy_(c.slots[s], non_blocking=True)
                    done = torch.cuda.Event()
                    done.record(self.dn)
                for c in dns:
                    c.host_ready[ib] = done
            self.slot_free[s] = done
            ev = nxt

    def synchronize(self):
        """Waits for every copy issued so far (before the host reads or writes a streamed array)."""
        self.op.stream().synchronize()
        self.up.synchronize()
        self.dn.synchronize()


class KMajorStaging:
    """Conversions between a host (K, Ny, Nx) float32 array and a state array in the batch layout, one batch at a
    time through a pinned buffer and a device buffer (set-up and results only)."""

    def __init__(self, op):
        self.op = op
        n = op.npix * op.K_batch_max
        self.pin = torch.empty(n, dtype=torch.float32, pin_memory=True)
        self.dev = torch.empty(n, dtype=torch.float32, device=op.device)

    def load(self, host_k, coeff, pipe, post=None):
        """coeff <- host_k (flattened (K, Ny, Nx)); post(ib, ptr) runs on the batch on the device before it is
        stored (e.g. the support projection)."""
        op = self.op
        comp = op.stream()
        pipe.synchronize()
        for ib, b in enumerate(op.batches):
            n = op.npix * b["K_batch"]
            k0 = op.npix * b["k_start"]
            np.copyto(self.pin.numpy()[:n], host_k[k0:k0 + n])
            with torch.cuda.stream(comp):
                self.dev[:n].copy_(self.pin[:n], non_blocking=True)
            dst = coeff.ptr(ib, 0)
            op._call("dfx_gather_channels", self.dev.data_ptr(), dst, op.npix, 0, b["K_batch"], op.Kstride, op._s())
            if post is not None:
                post(ib, dst)
            if not coeff.resident:
                with torch.cuda.stream(comp):
                    coeff.host_batch(ib).copy_(coeff.slots[0], non_blocking=True)
            comp.synchronize()          # the pinned buffer and slot 0 are reused by the next batch
        pipe.slot_free = [None, None]
        coeff.host_ready = [None] * coeff.n_batches

    def store(self, coeff, host_k, pipe):
        """host_k (flattened (K, Ny, Nx)) <- coeff."""
        op = self.op
        comp = op.stream()
        pipe.synchronize()
        for ib, b in enumerate(op.batches):
            n = op.npix * b["K_batch"]
            k0 = op.npix * b["k_start"]
            if not coeff.resident:
                with torch.cuda.stream(comp):
                    coeff.slots[0].copy_(coeff.host_batch(ib), non_blocking=True)
            op._call("dfx_scatter_channels", coeff.ptr(ib, 0), self.dev.data_ptr(), op.npix, 0, b["K_batch"],
                     op.Kstride, op._s())
            with torch.cuda.stream(comp):
                self.pin[:n].copy_(self.dev[:n], non_blocking=True)
            comp.synchronize()
            np.copyto(host_k[k0:k0 + n], self.pin.numpy()[:n])
        pipe.slot_free = [None, None]


# ---------------------------------------------------------------------------------------------- host copies
# Host arrays of the public API (NumPy x0, b, and the returned x, y, z) are pageable memory: a plain copy from or to
# the device runs at a few GB/s there. These copies go through pinned chunks instead: the DMA of one chunk overlaps
# the CPU copies of others, which run on a few threads (NumPy's copy releases the GIL).

_COPY_CHUNK = 64 << 20          # bytes per pinned chunk
_COPY_BUFS = 16                 # pinned chunks in flight = host threads: on a 16-core B200 host, 4 -> 16 threads took
                                # downloads into fresh (page-faulting) NumPy memory from 14 to 34 GB/s (warm 39 -> 51)


class HostCopier:
    """Chunked, pipelined copies between pageable NumPy arrays and contiguous device tensors (float32 or any dtype
    of equal size on both sides)."""

    def __init__(self):
        import threading
        from concurrent.futures import ThreadPoolExecutor
        self.lock = threading.Lock()        # one copy at a time per process (the pinned chunks are shared)
        self.pool = ThreadPoolExecutor(_COPY_BUFS, thread_name_prefix="dfx-copy")
        self.pins = [torch.empty(_COPY_CHUNK, dtype=torch.uint8, pin_memory=True) for _ in range(_COPY_BUFS)]

    @staticmethod
    def _bytes(a: np.ndarray):
        return a.reshape(-1).view(np.uint8)

    def prefault(self, host: np.ndarray, keep: bool):
        """Touches every 4 KB page of host (C-contiguous) on the copy threads, so that a later download into it runs
        at the copy rate of mapped memory instead of the page-fault rate of fresh memory; keep: write back each
        touched byte (the contents stay), else write 0. Returns the futures; a later copy into host must wait for
        them (a run does this work while the device computes)."""
        if not host.flags.writeable:
            raise ValueError("prefault: the host array is read-only (its pages cannot be prepared for a download)")
        v = self._bytes(host)
        page = 4096

        def touch(o, m):
            sl = v[o:o + m:page]
            if keep:
                sl[...] = sl.copy()
            else:
                sl[...] = 0
        return [self.pool.submit(touch, o, min(_COPY_CHUNK, v.size - o)) for o in range(0, v.size, _COPY_CHUNK)]

    def to_device(self, host: np.ndarray, dev: torch.Tensor, stream=None):
        """dev <- host (C-contiguous, same number of bytes); returns after the copies are enqueued on stream (the
        pinned buffers are not reused before their DMA has finished)."""
        with self.lock:
            self._to_device(host, dev, stream)

    def _to_device(self, host, dev, stream):
        src = self._bytes(np.ascontiguousarray(host))
        dst = dev.view(-1).view(torch.uint8)
        assert src.size == dst.numel()
        stream = stream or torch.cuda.current_stream(dev.device)
        n, nb = src.size, len(self.pins)
        starts = list(range(0, n, _COPY_CHUNK))
        done = [None] * nb
        staged = {}

        def stage(i):
            o = starts[i]
            m = min(_COPY_CHUNK, n - o)
            np.copyto(self.pins[i % nb].numpy()[:m], src[o:o + m])
            return m

        for i in range(min(nb, len(starts))):
            staged[i] = self.pool.submit(stage, i)
        for i, o in enumerate(starts):
            m = staged.pop(i).result()
            b = i % nb
            with torch.cuda.stream(stream):
                dst[o:o + m].copy_(self.pins[b][:m], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(stream)
            done[b] = ev
            j = i + nb
            if j < len(starts):
                def restage(j=j, ev=ev):
                    ev.synchronize()          # the DMA out of this pinned buffer has finished
                    return stage(j)
                staged[j] = self.pool.submit(restage)
        for ev in done:
            if ev is not None:
                ev.synchronize()

    def to_host(self, dev: torch.Tensor, host: np.ndarray, stream=None):
        """host (C-contiguous, same number of bytes) <- dev, after the work queued on stream; returns when host
        holds the data."""
        with self.lock:
            self._to_host(dev, host, stream)

    def _to_host(self, dev, host, stream):
        dst = self._bytes(host)
        src = dev.reshape(-1).view(torch.uint8)
        assert dst.size == src.numel()
        stream = stream or torch.cuda.current_stream(dev.device)
        n, nb = dst.size, len(self.pins)
        starts = list(range(0, n, _COPY_CHUNK))
        futs = [None] * nb
        for i, o in enumerate(starts):
            m = min(_COPY_CHUNK, n - o)
            b = i % nb
            if futs[b] is not None:
                futs[b].result()              # the CPU copy out of this pinned buffer has finished
            with torch.cuda.stream(stream):
                self.pins[b][:m].copy_(src[o:o + m], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(stream)

            def unstage(o=o, m=m, b=b, ev=ev):
                ev.synchronize()
                np.copyto(dst[o:o + m], self.pins[b].numpy()[:m])
            futs[b] = self.pool.submit(unstage)
        for f in futs:
            if f is not None:
                f.result()


_copier = None


def host_copier() -> HostCopier:
    """The process's copier (made on first use: a few pinned chunks and threads)."""
    global _copier
    if _copier is None:
        _copier = HostCopier()
    return _copier
