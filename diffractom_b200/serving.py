"""Serving of slice reconstructions: continuous batching of SPDHGPoisson requests on one GPU.

    server = ReconstructionServer(device=0, max_slots=4, hbm_budget_gb=120)
    server.start()
    server.submit(Request(cfg, material, grid, counts, subsets=10))      # any time, from any thread
    server.wait_all()
    server.stats()      # {"p50_s", "p99_s", "throughput_rps", ...}
    server.stop()

Requests arrive with their own geometry (pixels, angles, eta bins, rings), material and orientation set, i.e.
uneven sizes. The scheduler admits the oldest waiting request as soon as a slot is free and its estimated device
memory fits in the HBM budget next to the requests already running (and in the device's free memory). An admitted
request gets its own CUDA stream and worker thread; its operator, primal (x, z, T) and dual (y, S, D) state stay on
the device until it finishes. The workers run SPDHG epochs concurrently, so the kernels of different requests
overlap on the GPU; a request ends when the relative change of its deviance between epochs falls below its tol (or
after max_epochs), its coefficients are copied to the host and its memory is released for the next admission.
Every request is computed exactly as it would be alone (same kernels, same order on its own stream): results do not
depend on the mix. Latency = finish - arrival (queueing included).

No reference counterpart (diffractom reconstructs one slice per call); each request runs diffractom's SPDHGPoisson
loop (optimization/spdhg_poisson.py:513-751) through SinglePhaseForwardOperator.
"""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field
from typing import Any, Callable, Optional

import numpy as np

__all__ = ["Request", "ReconstructionServer", "Scheduler", "estimate_request_bytes"]


@dataclass
class Request:
    """One slice reconstruction: operator inputs, counts (N_Omega, My, N_eta * N_rings) and solver settings."""
    cfg: dict
    material: Any
    grid: Any
    counts: Any
    subsets: int = 8
    max_epochs: int = 100
    tol: float = 1e-3
    precision: str = "bf16"      # the BF16 tensor-core path (float32 step sizes and residual); "fp32" for float32
    max_gb: float = 2.0
    seed: int = 0
    id: int = 0
    # replay the SPDHG iterations as CUDA graphs from the second epoch on; off by default: a capture on one request's
    # stream is invalidated when another request's thread synchronises the device meanwhile (an operator build does)
    graphs: bool = False
    # filled in by the server
    arrival: float = 0.0
    admitted: float = 0.0
    finished: float = 0.0
    epochs: int = 0
    deviance: list = field(default_factory=list)
    timings: dict = field(default_factory=dict)   # build / setup / epochs / finish seconds of the worker
    stage: str = "queued"        # queued, build, setup, epochs, finish, done (progress of a running request)
    result: Optional[np.ndarray] = None
    error: Optional[str] = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def estimate_request_bytes(cfg, K, n_rings, fill=0.15, precision="fp32") -> int:
    """Device memory of a request, estimated before its operator exists: SPDHG's coefficient arrays (x, z, T in the
    batch layout and x in the (K, Ny, Nx) layout), its data arrays (b, y, S, D), both sparse PF copies at the given
    fill (12 bytes per non-zero, plus the eta-blocked forward copy, ~6 more), the ray tables (per-bin and grouped, for
    the whole image and the support) and the batch buffers;
    with precision "bf16" also the dense BF16 PF (2 bytes per entry), the BF16 copies of x and of the data rows and
    the Radon output of the subset angles. n_rings: an upper bound (the reflections)."""
    npix = int(cfg["Nx"]) * int(cfg["Ny"])
    R, My = int(cfg["N_Omega"]), int(cfg["My"])
    CP = int(cfg["N_eta"]) * int(n_rings)
    coeff = 4 * K * npix
    data = 4 * R * My * CP
    n = 4 * coeff + 4 * data + 18 * fill * R * K * CP + 90 * R * npix + 8 * 1024 * (R * My + npix) + (1 << 28)
    if precision == "bf16":
        n += 2 * R * K * CP + coeff // 2 + data // 2 + 2 * R * My * K
    return int(n)


class Scheduler:
    """Admission policy (host logic only): FIFO, at most max_slots running, the sum of the running requests'
    reservations within budget_bytes; admit() starts queued requests while the oldest one fits."""

    def __init__(self, max_slots: int, budget_bytes: int):
        if max_slots < 1 or budget_bytes <= 0:
            raise ValueError("max_slots must be >= 1 and the budget positive")
        self.max_slots, self.budget = int(max_slots), int(budget_bytes)
        self.running = {}                   # id -> reserved bytes
        self.queue = []                     # (id, bytes) in arrival order

    def enqueue(self, rid, nbytes):
        if nbytes > self.budget:
            raise MemoryError(f"request {rid} needs {nbytes / 1e9:.1f} GB, more than the budget "
                              f"{self.budget / 1e9:.1f} GB")
        self.queue.append((rid, int(nbytes)))

    def used(self) -> int:
        return sum(self.running.values())

    def admit(self, free_bytes: Optional[int] = None):
        """Ids of the queued requests that start now, oldest first; stops at the first that does not fit."""
        out = []
        while self.queue and len(self.running) < self.max_slots:
            rid, nb = self.queue[0]
            if self.used() + nb > self.budget or (free_bytes is not None and nb > free_bytes):
                break
            self.queue.pop(0)
            self.running[rid] = nb
            if free_bytes is not None:
                free_bytes -= nb
            out.append(rid)
        return out

    def release(self, rid):
        self.running.pop(rid, None)


class ReconstructionServer:
    """Continuous batching of SPDHG reconstructions on one GPU (module docstring)."""

    def __init__(self, device=0, max_slots: int = 4, hbm_budget_gb: float = 120.0,
                 on_finish: Optional[Callable[[Request], None]] = None):
        import torch
        self.torch = torch
        self.device = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
        self.sched = Scheduler(max_slots, int(hbm_budget_gb * 1e9))
        self.on_finish = on_finish
        self.requests = {}
        self.done = []
        self._lock = threading.Condition()
        self._stop = False
        self._thread = None
        self._workers = []
        self._t0 = None
        self._next_id = 0

    # ---------------------------------------------------------------- client side
    def start(self):
        self._t0 = time.perf_counter()
        self._thread = threading.Thread(target=self._loop, name="dfx-scheduler", daemon=True)
        self._thread.start()
        return self

    def now(self) -> float:
        return time.perf_counter() - self._t0

    def submit(self, req: Request) -> int:
        with self._lock:
            hkl = getattr(req.material, "hkl", None)
            nbytes = estimate_request_bytes(req.cfg, len(req.grid), len(hkl) if hkl is not None else 8,
                                            precision=req.precision)
            self.sched.enqueue(self._next_id, nbytes)       # MemoryError if it can never fit
            req.id = self._next_id
            self._next_id += 1
            req.arrival = self.now()
            self.requests[req.id] = req
            self._lock.notify_all()
        return req.id

    def wait_all(self, timeout: Optional[float] = None) -> bool:
        end = None if timeout is None else time.perf_counter() + timeout
        with self._lock:
            while len(self.done) < len(self.requests):
                left = None if end is None else end - time.perf_counter()
                if left is not None and left <= 0:
                    return False
                self._lock.wait(timeout=left)
        return True

    def stop(self):
        with self._lock:
            self._stop = True
            self._lock.notify_all()
        if self._thread is not None:
            self._thread.join()
        for w in self._workers:
            w.join()

    def stats(self) -> dict:
        lat = np.array([r.latency for r in self.done if r.error is None])
        if lat.size == 0:
            return {"requests": 0}
        span = max(r.finished for r in self.done) - min(r.arrival for r in self.done)
        ok = [r for r in self.done if r.error is None]
        parts = {k: float(np.sum([r.timings.get(k, 0.0) for r in ok])) for k in ("build", "setup", "epochs", "finish")}
        queued = [r.admitted - r.arrival for r in ok]
        done_ids = {r.id for r in self.done}
        pending = [r for r in self.requests.values() if r.id not in done_ids]
        return {"requests": int(lat.size), "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
                "throughput_rps": float(lat.size / span) if span > 0 else None,
                "epochs": int(sum(r.epochs for r in self.done)),
                "failed": int(sum(r.error is not None for r in self.done)),
                "worker_s": {k: round(v, 1) for k, v in parts.items()},
                "queued_s_p50": float(np.percentile(queued, 50)) if queued else None,
                "makespan_s": float(span),
                "unfinished": [(r.id, r.stage, r.epochs) for r in pending][:16]}

    # ---------------------------------------------------------------- server side
    def _loop(self):
        torch = self.torch
        while True:
            with self._lock:
                if self._stop:
                    return
                try:
                    # free device memory plus what this process's allocator holds cached (finished requests' buffers,
                    # which the next request's tensors reuse)
                    free = (int(torch.cuda.mem_get_info(self.device)[0]) + int(torch.cuda.memory_reserved(self.device))
                            - int(torch.cuda.memory_allocated(self.device)) - (1 << 30))
                except RuntimeError:            # a query failing now and then must not end the admissions
                    free = None
                if not self.sched.running and self.sched.queue and free is not None and self.sched.queue[0][1] > free:
                    # nothing runs and the oldest request still does not fit: it never will
                    rid, nb = self.sched.queue.pop(0)
                    req = self.requests[rid]
                    req.error = (f"MemoryError: request needs {nb / 1e9:.1f} GB, more than the device's "
                                 f"{max(free, 0) / 1e9:.1f} GB free")
                    req.admitted = req.finished = self.now()
                    self.done.append(req)
                    self._lock.notify_all()
                for rid in self.sched.admit(free_bytes=free):
                    req = self.requests[rid]
                    req.admitted = self.now()
                    w = threading.Thread(target=self._work, args=(req,), name=f"dfx-request-{rid}", daemon=True)
                    self._workers.append(w)
                    w.start()
                self._lock.wait(timeout=0.05)

    def _work(self, req: Request):
        torch = self.torch
        try:
            torch.cuda.set_device(self.device)
            stream = torch.cuda.Stream(self.device)
            with torch.cuda.stream(stream):
                req.result, req.epochs, req.deviance = run_request(req, self.device, stream)
        except Exception as e:                      # reported per request; the server keeps serving
            req.error = f"{type(e).__name__}: {e}"
        finally:
            req.finished = self.now()
            with self._lock:
                self.sched.release(req.id)
                self.done.append(req)
                self._lock.notify_all()
            if self.on_finish is not None:
                self.on_finish(req)


def run_request(req: Request, device, stream):
    """One request on its stream: operator, SPDHG set-up, epochs until the relative deviance change is below tol.
    Returns (x (K, Ny, Nx) NumPy, epochs, deviance per epoch)."""
    import torch
    from .operator import SinglePhaseForwardOperator
    from .spdhg import SPDHGPoisson
    t0 = time.perf_counter()
    req.stage = "build"
    # SPDHG runs over omega subsets, which need a sparse PF mode: "auto" with the dense switch off (the sparse
    # matrix stored as far as memory allows, the rest generated in every call)
    op = SinglePhaseForwardOperator(req.cfg, req.material, req.grid, req.max_gb, normalized=True, ctx=device,
                                    queue=stream, precision=req.precision, sparse_max_fill=1.0,
                                    sparse_max_fill_partial=1.0)
    t1 = time.perf_counter()
    try:
        sp = SPDHGPoisson(op, subsets=req.subsets, seed=req.seed)
        sp.use_graphs = req.graphs
        x0 = torch.zeros(op.coeff_shape, dtype=torch.float32, device=device)
        req.stage = "setup"
        sp._setup(x0, req.counts)
        stream.synchronize()
        t2 = time.perf_counter()
        devs = []
        req.stage = "epochs"
        for e in range(req.max_epochs):
            last = e + 1 == req.max_epochs
            sp._iterate(1, diagnostics_interval=1, final=last)
            devs.append(float(sp._f))
            req.epochs = len(devs)
            if len(devs) > 1 and abs(devs[-2] - devs[-1]) <= req.tol * abs(devs[-1]):
                break
        t3 = time.perf_counter()
        req.stage = "finish"
        x = sp._finish()
        out = x.cpu().numpy()
        req.timings = {"build": t1 - t0, "setup": t2 - t1, "epochs": t3 - t2, "finish": time.perf_counter() - t3}
        req.stage = "done"
        return out, len(devs), devs
    finally:
        op.free_memory()
