"""Benchmark of the reconstruction hot path: SPDHG epochs per second on the B200 (diffractom's SPDHGPoisson with the
single-phase forward operator), with the CPU oracle timed beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload ti256|al99]

A step is one SPDHG epoch (M subset iterations, each a pass over all orientation batches: adjoint of the subset's
dual change, primal update, forward of the next subset). Workloads are seeded synthetic stand-ins with the shapes
of the benchmark configurations (no dataset exists for them):

  ti256  256 x 256 pixels, 360 rotation angles over 180 deg, 263 translations, 360 eta bins, 8 rings of hexagonal Ti
         (a 2.95, c 4.68 A), K = 20000 orientations (sigma 2 deg, random in the fundamental zone), 200 Voronoi grains
         plus 10 % fine-grained random background, Poisson counts with mean 50, 20 subsets        (the default)
  al99   99 x 99 pixels, 180 angles over 180 deg, 103 translations, 180 eta bins, 5 rings of cubic Al, K = 1000
         (sigma 3 deg), 30 grains, mean 100 counts, 10 subsets

Output: one JSON line (rank 0). value = epochs/s of the whole job on device-resident inputs (CUDA events around
exactly `steps` epochs after `warmup` untimed ones; inputs are larger than L2, which is not flushed); e2e = the same
metric through the public API (SPDHGPoisson.run on NumPy arrays: uploads, set-up, epochs, downloads); roofline of the
dominant kernel from CUDA events around its launches inside the timed region; cpu_baseline = the CPU oracle
(oracle/oracle.c, float32, all host threads) on a bounded sample of the same epoch.

With --gpus N > 1 (torchrun, NCCL) the orientations are sharded: the grid holds N x K orientations and each rank
builds the operator of its K (weak scaling: per-GPU work fixed); the only exchange is the all-reduce of the data rows
each forward pass writes (diffractom_b200.sharding). value = N x epochs / (max over ranks of the time), i.e. epochs
of K orientations per second summed over the GPUs, as at N = 1.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "SPDHG epochs/s BF16-TC vs FP32 at ≤1e-3 FP64 deviance err; serve p50/p99"

WORKLOADS = {
    "ti256": dict(cfg=dict(Nx=256, Ny=256, My=263, N_Omega=360, angle_range=[0, 180], cor_offset=0.0, N_eta=360,
                           eta_angle_range=[0, 360], energy=12.398 / 0.3, k_direction_0=[0, 0, 1],
                           p_direction_0=[1, 0, 0], detector_direction_origin=[0, -1, 0],
                           detector_direction_positive_90=[0, 0, -1]),
                  material=dict(a=2.95, c=4.68, gamma=120, symmetry_group="hexagonal", wavelength_A=0.3,
                                hkl_list=[[1, 0, 0], [0, 0, 2], [1, 0, 1], [1, 0, 2], [1, 1, 0], [1, 0, 3],
                                          [2, 0, 0], [1, 1, 2]]),
                  K=20000, sigma_deg=2.0, grains=200, background=0.10, mean_counts=50.0, subsets=20, epochs=30,
                  max_gb=3.9),
    "al99": dict(cfg=dict(Nx=99, Ny=99, My=103, N_Omega=180, angle_range=[0, 180], cor_offset=0.0, N_eta=180,
                          eta_angle_range=[0, 360], energy=12.398 / 0.3, k_direction_0=[0, 0, 1],
                          p_direction_0=[1, 0, 0], detector_direction_origin=[0, -1, 0],
                          detector_direction_positive_90=[0, 0, -1]),
                 material=dict(a=4.05, symmetry_group="cubic", wavelength_A=0.3,
                               hkl_list=[[1, 1, 1], [2, 0, 0], [2, 2, 0], [3, 1, 1], [2, 2, 2]]),
                 K=1000, sigma_deg=3.0, grains=30, background=0.0, mean_counts=100.0, subsets=10, epochs=20,
                 max_gb=2.0),
}


# ----------------------------------------------------------------------------------------------- workload
def make_problem(name, seed=0, K=None):
    """(cfg, Material, Grid, workload dict): seeded orientations (K: fewer orientations than the workload's, for
    profiling captures of the same geometry on a few GB)."""
    from diffractom_b200 import Grid, Material
    w = dict(WORKLOADS[name])
    if K:
        w["K"] = int(K)
        w["grains"] = min(w["grains"], w["K"])
    mat = Material.from_lattice_parameters(**w["material"])
    grid = Grid.from_random_fundamental_zone(w["K"], mat.crystal_system, np.deg2rad(w["sigma_deg"]), seed=seed)
    return dict(w["cfg"]), mat, grid, w


def phantom(op, w, seed=1):
    """x_true (K, Ny, Nx) on the device: Voronoi grains in the field of view, one orientation each (weight 1), plus
    a fraction of the pixels with one more random orientation (weight 0.5)."""
    import torch
    rng = np.random.default_rng(seed)
    supp = op.support_mask()
    ys, xs = np.nonzero(supp)
    seeds = rng.choice(len(ys), w["grains"], replace=False)
    sy, sx = ys[seeds].astype(np.float64), xs[seeds].astype(np.float64)
    grain_k = rng.choice(op.K, w["grains"], replace=False)
    yy, xx = np.mgrid[:op.Ny, :op.Nx]
    d2 = (yy.ravel()[:, None] - sy[None]) ** 2 + (xx.ravel()[:, None] - sx[None]) ** 2
    owner = grain_k[np.argmin(d2, axis=1)]
    inside = supp.ravel()
    x = torch.zeros((op.K, op.Ny * op.Nx), dtype=torch.float32, device=op.device)
    pix = np.nonzero(inside)[0]
    x[torch.as_tensor(owner[pix], device=op.device), torch.as_tensor(pix, device=op.device)] = 1.0
    if w["background"] > 0:
        bg = rng.choice(pix, int(w["background"] * len(pix)), replace=False)
        kb = rng.integers(0, op.K, len(bg))
        x[torch.as_tensor(kb, device=op.device), torch.as_tensor(bg, device=op.device)] += 0.5
    return x.reshape(op.coeff_shape)


def counts(op, x_true, mean, seed=2, dist=None):
    """Poisson counts with the given mean of the prediction A x_true (scaled); with orientation shards the prediction
    is summed over the ranks and rank 0's counts are broadcast."""
    import torch
    ax = op.direct(x_true)
    if dist is not None:
        dist.all_reduce(ax)
    lam = (ax * (mean / float(ax.double().mean().item()))).clamp_min_(0.0)
    g = torch.Generator(device=op.device)
    g.manual_seed(seed)
    b = torch.poisson(lam, generator=g)
    if dist is not None:
        dist.broadcast(b, 0)
    return b


# ----------------------------------------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi samples of this GPU's SM clock and throttle reasons while the timed region runs."""

    def __init__(self, index):
        self.rows = []
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(index), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def stop(self):
        if self.proc is not None:
            time.sleep(0.3)
            self.proc.terminate()
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[3:]) if v.lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ----------------------------------------------------------------------------------------------- CPU oracle
def dense_batches(geom, max_gb):
    """The operator's orientation batches for a geometry without a device (SPFO:1026-1094: as many orientations as a
    dense PF batch of max_gb holds)."""
    per_k = geom.N_Omega * geom.N_eta * geom.N_peaks * 4
    kb = min(max(int(max_gb * 1024 ** 3 // per_k), 1), geom.K)
    return [(k0, min(kb, geom.K - k0)) for k0 in range(0, geom.K, kb)]


class CpuSubsetIterations:
    """The CPU oracle (oracle/: the reference's kernels restated in C, float32 like the reference's, OpenMP over all
    host threads) running whole SPDHG subset iterations of a workload: the dual step on one subset's rows, then for
    every orientation batch that subset's adjoint (PF product, backprojection), the primal update of the batch and
    the next subset's forward (projection, PF product) added into its rows. One step is exactly 1 / M of an epoch's
    work (every subset has the same number of angles); nothing is extrapolated over batches. The PF matrix of the two
    subsets' angles is built before the steps (not timed), as the reference builds its sparse PF at construction."""

    def __init__(self, geom, w, batches, seed=0):
        from oracle.oracle import OracleOperator, lib
        self.L = lib()
        M = w["subsets"]
        R = geom.N_Omega
        sub_a, sub_f = np.arange(0, R, M), np.arange(1, R, M)
        rows = np.union1d(sub_a, sub_f)
        self.ia = np.searchsorted(rows, sub_a)
        self.jf = np.searchsorted(rows, sub_f)
        self.om = np.ascontiguousarray(self.ia, np.int32)
        full = OracleOperator.from_operator(geom, precision="f32", batches=batches)
        self.parts = []
        t0 = time.perf_counter()
        for k0, kb in full.batches:
            o = OracleOperator(coords=full.coords[rows], poles=full.poles[k0:k0 + kb], axis_start=full.axis_start,
                               axis_count=full.axis_count, inv_sigma2=full.inv_sigma2[k0:k0 + kb],
                               norm=full.norm[k0:k0 + kb], quad_w=full.quad_w, intens=full.intens,
                               geo=full.geo[rows], scale=full.scale, n_taps=full.n_taps, kernel=full.kernel,
                               Nx=geom.Nx, Ny=geom.Ny, My=geom.My, cut=full.cut, batches=[(0, kb)], precision="f32")
            o.csr(0, kb)
            self.parts.append((k0, kb, o))
        self.setup_s = time.perf_counter() - t0
        rng = np.random.default_rng(seed)
        npix = geom.Nx * geom.Ny
        shape = (len(rows), geom.My, geom.N_seg)
        self.D = rng.random(shape).astype(np.float32)
        self.b = rng.poisson(50, shape).astype(np.float32)
        self.y = np.zeros(shape, np.float32)
        self.sig = np.full(shape, 1e-3, np.float32)
        self.x = rng.random((geom.K, npix)).astype(np.float32)
        self.z = np.zeros_like(self.x)
        self.T = np.full_like(self.x, 1e-3)
        self.M = M
        self.row = geom.My * geom.N_seg
        self.threads = int(self.L.orc_num_threads())
        self.n_batches = len(self.parts)
        self.K = geom.K

    def step(self):
        """One subset iteration; returns its wall-clock seconds."""
        from oracle.oracle import _p
        L = self.L
        t0 = time.perf_counter()
        L.orc_dual_update_sub(_p(self.y), _p(self.D), _p(self.sig), _p(self.b), None, 0, None, 0, None, 0, 1e-3,
                              _p(self.om), self.row, len(self.om) * self.row)
        self.D[self.jf] = 0.0
        for k0, kb, o in self.parts:
            dz = np.ascontiguousarray(o.adjoint(self.D, subset=self.ia).reshape(kb, -1))
            xb, zb, Tb = self.x[k0:k0 + kb], self.z[k0:k0 + kb], self.T[k0:k0 + kb]
            L.orc_spdhg_update(_p(xb), _p(zb), _p(Tb), _p(dz), float(self.M), 0.0, xb.size)
            o.forward(xb, subset=self.jf, data=self.D, accumulate=True)
        return time.perf_counter() - t0

    def describe(self, n):
        return (f"{n} whole SPDHG subset iteration(s) (1 / {self.M} epoch each: dual step, adjoint, primal update "
                f"and next subset's forward over all {self.n_batches} batches of the {self.K} orientations), "
                f"float32 oracle on {self.threads} threads; PF of the two subsets' angles built before ("
                f"{self.setup_s:.1f} s)")


def precision_errors_al99():
    """The precision of the float32 and BF16 paths against the float64 oracle loop at the al99 configuration (99 x 99
    pixels, 180 angles, K 1000, 10 subsets, 20 epochs): SPDHGPoisson on the device (float32; BF16 with the float32
    residual and step sizes; BF16 with the BF16 ones) and oracle.spdhg_reference64 (every operand float64, the same
    schedule) on the host. Returns relative deviance (final epoch, and the largest over the epochs) and coefficient
    (2-norm) errors. The oracle is the checker here."""
    import torch
    from diffractom_b200 import SinglePhaseForwardOperator, SPDHGPoisson
    from oracle.oracle import OracleOperator, spdhg_reference64
    cfg, mat, grid, w = make_problem("al99")
    op = SinglePhaseForwardOperator(cfg, mat, grid, w["max_gb"], normalized=True, precision="bf16")
    op.precision = "fp32"
    b = counts(op, phantom(op, w, seed=1), w["mean_counts"]).cpu().numpy()
    M, E = w["subsets"], w["epochs"]
    runs = {}
    for name, prec, fast in (("fp32", "fp32", False), ("bf16", "bf16", False), ("bf16_fast_passes", "bf16", True)):
        op.precision = prec
        sp = SPDHGPoisson(op, subsets=M, seed=0)
        sp.bf16_steps = sp.bf16_diagnostics = fast
        x = sp.run(torch.zeros(op.coeff_shape, device=op.device), b, E, diagnostics_interval=1).cpu().numpy()
        runs[name] = (x, np.array([st["f"] for st in sp.iter_stats]))
    op.precision = "fp32"
    t0 = time.perf_counter()
    orc = OracleOperator.from_operator(op, precision="f64io")
    x64, _, _, devs64, _, _ = spdhg_reference64(orc, op.omega_subsets, b, E, support=op.support_mask(), seed=0)
    t64 = time.perf_counter() - t0
    devs64 = np.asarray(devs64)
    out = {"workload": f"al99 (99x99, 180 angles, K {op.K}, {M} subsets, {E} epochs, diagnostics every epoch)",
           "f64_oracle_s": round(t64, 1)}
    for name, (x, devs) in runs.items():
        e = np.abs(devs - devs64) / devs64
        out[f"deviance_rel_err_{name}_vs_f64"] = float(e[-1])
        out[f"deviance_rel_err_{name}_vs_f64_max_epoch"] = float(e.max())
        out[f"coef_rel_err_{name}_vs_f64"] = float(np.linalg.norm(x - x64) / np.linalg.norm(x64))
    op.free_memory()
    return out


# ----------------------------------------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="ti256", choices=sorted(WORKLOADS) + ["ni512"],
                    help="ni512: the large tailored-grid slice (Fourier-slice projector, BF16 contraction, streamed "
                    "T); its own JSON line")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the short serving run of the default line")
    ap.add_argument("--serve", action="store_true", help="only the serving benchmark (64 requests, Poisson "
                    "arrivals at 2/s, sizes of the serving configuration); its own JSON line")
    ap.add_argument("--projectors", action="store_true", help="only the projector comparison (native vs "
                    "Fourier-slice) at the large-slice geometry; its own JSON line")
    ap.add_argument("--extras", action="store_true", help="only the solvers and tools around the operator (FISTA, "
                    "OSEM, PDHG, parameter gradients, orientation search) at the ti256 geometry; its own JSON line")
    ap.add_argument("--local", action="store_true", help="only the local-basis comparison (local vs dense operator "
                    "over the same orientations) at the ti256 geometry; its own JSON line")
    ap.add_argument("--K", type=int, default=None, help="orientations (default: the workload's)")
    ap.add_argument("--precision", default="both", choices=["both", "bf16", "fp32"],
                    help="both: the BF16 tensor-core path (the value) and the float32 path (for the ratio)")
    ap.add_argument("--no-errors", action="store_true", help="skip the al99 precision check against the float64 "
                    "oracle loop")
    ap.add_argument("--tc-forward", default="auto", choices=["auto", "on", "builder", "off"],
                    help="the BF16 passes' forward projection on the tensor cores (on: weights from the per-geometry "
                    "table, dfx_radon_forward_tc_table; builder: weights built per CTA, dfx_radon_forward_tc) or "
                    "through the ray table (off); auto: the operator's default")
    ap.add_argument("--no-generated", action="store_true", help="skip the arms with the PF generated on the fly "
                    "(no PF stored: the float32 CSR generated per batch, the BF16 PF per subset)")
    a = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    if a.impl == "reference":
        return run_reference(a, rank)
    torch.cuda.set_device(local)
    if a.workload == "ni512":
        if rank == 0:
            print(json.dumps(ni512_run(a.steps, a.warmup, a.K)), flush=True)
        return 0
    if a.projectors:
        if rank == 0:
            print(json.dumps(projector_run(a.K or 256, a.steps, a.warmup)), flush=True)
        return 0
    if a.extras:
        if rank == 0:
            print(json.dumps(extras_run(a.K or 2000, a.steps, a.warmup)), flush=True)
        return 0
    if a.local:
        if rank == 0:
            print(json.dumps(local_run(a.K or 2000, a.steps, a.warmup)), flush=True)
        return 0
    if a.serve:
        if rank == 0:
            st = serving_run(**SERVE_FULL)
            print(json.dumps({"metric": "serving latency p50/p99 (SPDHG to 1e-3 relative deviance change)",
                              "value": st["p99_s"], "unit": "s", "higher_is_better": False, "n_gpus": 1,
                              "data": "synthetic", "serve": st}), flush=True)
        return 0
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    from diffractom_b200 import SinglePhaseForwardOperator
    from diffractom_b200.sharding import ShardSum, shard_grid
    k_per = a.K or WORKLOADS[a.workload]["K"]
    cfg, mat, grid, w = make_problem(a.workload, K=k_per * world if world > 1 else a.K)
    shards = None
    if world > 1:
        grid = shard_grid(grid, rank, world)
        shards = ShardSum()
    t_build = time.perf_counter()
    op = SinglePhaseForwardOperator(cfg, mat, grid, w["max_gb"], normalized=True,
                                    precision="bf16" if a.precision in ("bf16", "both") else "fp32")
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t_build
    if a.tc_forward != "auto":
        op.use_tc_forward = a.tc_forward in ("on", "builder")
        if a.tc_forward == "builder":
            op.tc_weight_table_max_frac = 0.0
    op.precision = "fp32"
    x_true = phantom(op, dict(w, grains=min(w["grains"], op.K)), seed=1 + rank)
    b = counts(op, x_true, w["mean_counts"], dist=dist)
    del x_true
    torch.cuda.empty_cache()

    # arms: (name, operator precision, per-epoch diagnostics, full forward of the diagnostics on the BF16 path)
    arm_list = []
    if a.precision in ("fp32", "both"):
        arm_list.append(("fp32", "fp32", True, False))
    if a.precision in ("bf16", "both"):
        arm_list += [("bf16", "bf16", True, False), ("bf16_bf16_residual", "bf16", True, True),
                     ("bf16_no_diagnostics", "bf16", False, True)]
    arms = {}
    for name, prec, diag, bf16_res in arm_list:
        arms[name] = timed_epochs(op, w, b, a, prec, dist, local, world, shards, diagnostics=diag,
                                  bf16_residual=bf16_res)
    head = arms["bf16" if "bf16" in arms else "fp32"]

    e2e = None
    if not a.no_e2e:
        op.precision = "bf16" if "bf16" in arms else "fp32"
        e2e = measure_e2e(op, w, b, a.steps, dist, world, shards)
        op.precision = "fp32"
    cpu = None
    errors = None
    if rank == 0 and not a.no_cpu:
        # the CPU leg: the oracle timed on whole subset iterations of this workload (the CPU baseline), and the
        # float64 oracle loop as the checker of the precision paths at al99
        t0 = time.perf_counter()
        batches = [(bt["k_start"], bt["K_batch"]) for bt in op.batches]
        cpu_it = CpuSubsetIterations(op, w, batches)
        n_cpu = 1
        secs = [cpu_it.step() for _ in range(n_cpu)]
        per_epoch = w["subsets"] * float(np.mean(secs))
        cpu = {"value": 1.0 / per_epoch, "unit": "epochs/s", "cores": cpu_it.threads, "kind": "port",
               "sample": cpu_it.describe(n_cpu) + f"; {time.perf_counter() - t0:.1f} s in all"}
        del cpu_it
        if not a.no_errors:
            errors = precision_errors_al99()
    if rank == 0:
        cfg_line = {"workload": a.workload + (f" (K {a.K})" if a.K else ""), "K": op.K * world, "K_per_gpu": op.K,
                    "pixels": f"{op.Nx}x{op.Ny}", "N_Omega": op.N_Omega,
                    "My": op.My, "N_eta": op.N_eta, "rings": op.N_peaks, "subsets": w["subsets"],
                    "batches": len(op.batches), "K_batch_max": op.K_batch_max, "pf_mode": op.pf_mode,
                    "pf_nnz": op.sparse_nnz, "precision_path": "bf16-tc" if "bf16" in arms else "fp32",
                    "l2": "inputs larger than L2, no flush",
                    "parallelism": "single GPU" if world == 1 else
                    f"orientation shards x{world} (NCCL all-reduce of the forward's data rows)",
                    "operator_build_s": round(t_build, 2),
                    "epoch": "M subset iterations (dual step, adjoint with the fused primal step, next subset's "
                             "forward) + diagnostics every epoch: full forward A x (the residual) and the float64 "
                             "deviance",
                    "arms": {"fp32": "float32 operator throughout (the drop-in path)",
                             "bf16": "value: Radon and PF contraction in BF16 with float32 accumulation; the residual "
                                     "recomputed with the float32 operator once per epoch; float64 deviance",
                             "bf16_bf16_residual": "as bf16, the per-epoch residual through the BF16 path",
                             "bf16_no_diagnostics": "as bf16, no per-epoch residual or deviance"}}
        for name, r in arms.items():
            cfg_line[f"{name}_epochs_per_s"] = r["value"]
            cfg_line[f"{name}_final_deviance_f64"] = r["f"]
        if "fp32" in arms and "bf16" in arms:
            xf = arms["fp32"]["x"]
            cfg_line["bf16_speedup_vs_fp32"] = arms["bf16"]["value"] / arms["fp32"]["value"]
            for name in arms:
                if name == "fp32":
                    continue
                xb = arms[name]["x"]
                cfg_line[f"deviance_rel_err_{name}_vs_fp32"] = (abs(arms[name]["f"] - arms["fp32"]["f"]) /
                                                              arms["fp32"]["f"])
                cfg_line[f"coef_rel_err_{name}_vs_fp32"] = float((xb - xf).double().norm() / xf.double().norm())
            cfg_line["deviance_note"] = ("deviance of each run's final iterate: float32 forward, float64 sum; errors "
                                         "against float64 from the oracle's float64 loop at al99 (precision_vs_f64)")
            cfg_line["fp32_roofline"] = arms["fp32"]["roof"]
        if errors is not None:
            cfg_line["precision_vs_f64"] = errors
            for k in ("deviance_rel_err_bf16_vs_f64", "coef_rel_err_bf16_vs_f64", "deviance_rel_err_fp32_vs_f64",
                      "coef_rel_err_fp32_vs_f64"):
                cfg_line[k] = errors[k]
    gen = {}
    if not a.no_generated:
        # the same problem with no PF stored: an operator whose float32 products generate the CSR of each batch in
        # every call and whose BF16 products generate the PF of each subset's angles when they use it
        op.free_memory()
        del op
        torch.cuda.empty_cache()
        op = SinglePhaseForwardOperator(cfg, mat, grid, w["max_gb"], normalized=True, precision="bf16",
                                        bf16_pf="generated", pf_mode="generated")
        for name, prec in (("fp32_generated_pf", "fp32"), ("bf16_generated_pf", "bf16")):
            if prec == "bf16" and a.precision == "fp32" or prec == "fp32" and a.precision == "bf16":
                continue
            gen[name] = timed_epochs(op, w, b, a, prec, dist, local, world, shards, diagnostics=True)
    if rank == 0 and gen:
        cfg_line["arms"]["fp32_generated_pf"] = ("as fp32 with no PF stored: the CSR of every batch generated in "
                                                 "every product (pf_mode 'generated')")
        cfg_line["arms"]["bf16_generated_pf"] = ("as bf16 with no PF stored: the BF16 PF of a subset's angles "
                                                 "generated when a product uses it (bf16_pf 'generated'), the float32 "
                                                 "residual through generated CSRs")
        for name, r in gen.items():
            cfg_line[f"{name}_epochs_per_s"] = r["value"]
            cfg_line[f"{name}_final_deviance_f64"] = r["f"]
            ref = arms.get(name.split("_")[0])
            if ref is not None:
                cfg_line[f"deviance_rel_err_{name}_vs_stored"] = abs(r["f"] - ref["f"]) / ref["f"]
        gen.clear()
    serve = None
    if not a.no_serve and rank == 0:
        op.free_memory()
        del op, b
        torch.cuda.empty_cache()
        serve = serving_run(**SERVE_SHORT)
    if rank == 0:
        line = {
            "metric": METRIC, "value": head["value"], "unit": "epochs/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": head["t_max"] / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16" if "bf16" in arms else "f32",
            "data": "synthetic (seeded phantom, Poisson counts)", "config": cfg_line,
            "roofline": head["roof"], "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(head["launches"]),
            "clocks": head["clk"], "serve": serve,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def timed_epochs(op, w, b, a, precision, dist, local, world, shards=None, diagnostics=True, bf16_residual=False):
    """warmup untimed + steps timed SPDHG epochs with the operator in the given precision; diagnostics: every epoch
    ends with the full forward (the residual; bf16_residual: through the BF16 path, else the float32 operator) and
    the float64 deviance, as run() with diagnostics_interval=1. Returns the rate and the deviance of the final
    iterate with the float32 operator (float64 sum)."""
    import torch
    from diffractom_b200 import SPDHGPoisson, _lib
    op.precision = precision
    sp = SPDHGPoisson(op, subsets=w["subsets"], seed=0, shards=shards)
    sp.bf16_diagnostics = bool(bf16_residual)
    x0 = torch.zeros(op.coeff_shape, dtype=torch.float32, device=op.device)
    sp._setup(x0, b)
    interval = 1 if diagnostics else 1 << 30
    sp._iterate(a.warmup, diagnostics_interval=interval, final=False, async_diagnostics=True)
    stream = op.stream()
    timers = KernelTimers(op)
    stream.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = Clocks(local)
    n0 = _lib.lib().dfx_launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    timers.on()
    sp._iterate(a.steps, diagnostics_interval=interval, final=False, async_diagnostics=True)
    timers.off()
    end.record(stream)
    end.synchronize()
    launches = _lib.lib().dfx_launch_count() - n0 - timers.n_extra
    clk = clocks.stop()
    ms = start.elapsed_time(end)
    t_max = ms
    if dist is not None:
        tt = torch.tensor([ms], device=op.device, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
        dist.barrier()
    value = world * a.steps / (t_max / 1e3)
    x = sp.x
    sp._finish()
    op.precision = "fp32"
    D = torch.empty(op.data_shape, dtype=torch.float32, device=op.device)
    op.direct_cl(x, D)
    if shards is not None:
        shards.all(D, op.stream())
    sp.b, sp.w, sp.pw, sp.g, sp.pg, sp.bg, sp.pbg = b, None, 0, None, 0, None, 0
    f_final = sp._deviance(D)
    del D
    roof = timers.roofline(op)
    return {"value": value, "t_max": t_max, "f": f_final, "x": x, "roof": roof, "launches": launches, "clk": clk}


class KernelTimers:
    """CUDA events around the launches of chosen kernels inside the timed region (same stream), for the roofline."""

    def __init__(self, op):
        from diffractom_b200 import _lib
        self.op = op
        self._lib = _lib
        self.events, self.args = {}, {}
        self.n_extra = 0
        self._orig_op, self._orig_lib = op._call, _lib.call

    def _wrap(self, orig):
        import torch
        op = self.op

        def call(name, *args):
            s = op.stream()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            orig(name, *args)
            e1.record(s)
            self.events.setdefault(name, []).append((e0, e1))
            self.args.setdefault(name, []).append(args)
        return call

    def on(self):
        """Every entry point the operator or the solvers call (all launch on the operator's stream) is timed."""
        self.op._call = self._wrap(self._orig_op)
        self._lib.call = self._wrap(self._orig_lib)

    def off(self):
        self.op._call = self._orig_op
        self._lib.call = self._orig_lib

    def roofline(self, op):
        """The dominant kernel (largest share of the timed kernels' device time) against its roofline: tensor-core
        products against the measured sustained BF16 GEMM rate (they run inside a seconds-long loop), the rest
        against the measured HBM copy bandwidth; every kernel's share and achieved rates under "kernels"."""
        import torch
        torch.cuda.synchronize()
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() \
            else {}
        hbm = float(peaks.get("hbm_gbs", 6650.0))
        tc = float(peaks.get("bf16_tflops_sustained", 1400.0))
        src = "MEASURED_PEAKS.json" if peaks else "fallback"
        fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12          # FP32 FMA lanes x 2 flops x max SM clock (TFLOP/s)
        per = {n: [e0.elapsed_time(e1) for e0, e1 in evs] for n, evs in self.events.items() if evs}
        tot = {n: sum(v) for n, v in per.items()}
        total = sum(tot.values())
        kernels = {}
        for n in sorted(tot, key=lambda n: -tot[n]):
            ms = float(np.mean(per[n]))
            nbytes, flops = algorithmic_work(op, n, self.args[n])
            entry = {"share": round(tot[n] / total, 4), "launches": len(per[n]), "mean_ms": round(ms, 4),
                     "gbs": round(nbytes / (ms / 1e3) / 1e9, 1)}
            if flops:
                entry["tflops"] = round(flops / (ms / 1e3) / 1e12, 2)
            kernels[n] = entry
        dom = max(tot, key=tot.get)
        ms = float(np.mean(per[dom]))
        nbytes, flops = algorithmic_work(op, dom, self.args[dom])
        if dom.startswith("dfx_pf_tc"):
            achieved = flops / (ms / 1e3) / 1e12
            out = {"kernel": dom, "bound": "tensor", "achieved": achieved, "peak": tc, "unit": "TFLOP/s",
                   "frac": achieved / tc, "peak_source": f"{src} bf16_tflops_sustained (of measured)"}
        else:
            achieved = nbytes / (ms / 1e3) / 1e9
            out = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                   "frac": achieved / hbm, "peak_source": f"{src} hbm_gbs (of measured)"}
            if flops:
                out["fp32_tflops"] = flops / (ms / 1e3) / 1e12
                out["fp32_frac_of_nominal"] = out["fp32_tflops"] / fp32_peak
        out.update({"traffic": profiled_traffic(dom), "mean_launch_ms": ms, "launches": len(per[dom]),
                    "kernels": kernels})
        return out


def profiled_traffic(kernel):
    """DRAM bytes per launch of a kernel from the committed ncu summary of this workload (profiles/traffic.json),
    or None when none was captured."""
    f = ROOT / "profiles" / "traffic.json"
    if not f.exists():
        return None
    return json.loads(f.read_text()).get(kernel, {}).get("dram_bytes_per_launch")


def algorithmic_work(op, name, args_list):
    """(bytes, flops) per launch (mean over the recorded launches) of a kernel: its own inputs + outputs once, and the
    multiply-adds of its non-zero taps / entries (an FMA = 2 flops); the tensor-core products count the dense
    multiply-adds they perform."""
    nb, nf = [], []
    npix = op.Nx * op.Ny
    My = op.My
    for args in args_list:
        if name in ("dfx_radon_forward", "dfx_radon_backward"):
            n_ang, kb = args[3], args[8]
            nb.append(4 * kb * (npix + n_ang * My))
            nf.append(2 * 2 * npix * n_ang * kb)            # ~2 taps per pixel and angle
        elif name == "dfx_radon_forward_bf16":
            n_ang, kb = args[4], args[9]
            nb.append(4 * kb * npix + 2 * kb * n_ang * My)
            nf.append(2 * 2 * npix * n_ang * kb)
        elif name == "dfx_radon_forward_gtable":
            n_ang, kb = args[6], args[9]
            nb.append(4 * kb * (npix + n_ang * My))
            nf.append(2 * 2 * npix * n_ang * kb)
        elif name == "dfx_radon_forward_tc":
            # BF16 image in, sinogram rows out (BF16, or float32 when out_f32); the MMAs count the taps' FMAs
            n_ang, kst, osz = args[5], args[9], 4 if args[3] else 2
            nb.append(2 * kst * npix + osz * kst * n_ang * My)
            nf.append(2 * 2 * npix * n_ang * kst)
        elif name == "dfx_radon_forward_table":
            n_ang, kb = args[5], args[8]
            nb.append(4 * kb * (npix + n_ang * My))
            nf.append(2 * 2 * npix * n_ang * kb)
        elif name == "dfx_radon_forward_table_bf16":
            n_ang, kb = args[6], args[9]
            nb.append(4 * kb * npix + 2 * kb * n_ang * My)
            nf.append(2 * 2 * npix * n_ang * kb)
        elif name == "dfx_radon_forward_table_bf16_bf16":
            n_ang, kb = args[6], args[9]
            nb.append(2 * kb * npix + 2 * kb * n_ang * My)
            nf.append(2 * 2 * npix * n_ang * kb)
        elif name == "dfx_radon_backward_spdhg":
            n_ang, kstride, kb = args[2], args[6], args[7]
            nb.append(4 * kb * n_ang * My + 4 * 5 * npix * kstride)      # sino; x, z, T read; x, z written
            nf.append(2 * 2 * npix * n_ang * kb)
        elif name == "dfx_radon_backward_spdhg_bf16":
            n_ang, kstride, kb = args[3], args[7], args[8]
            nb.append(2 * kb * n_ang * My + (4 * 5 + (2 if args[16] else 0)) * npix * kstride)   # + BF16 x copy
            nf.append(2 * 2 * npix * n_ang * kb)
        elif name == "dfx_radon_backward_spdhg_tc":
            # BF16 Z rows of the batch's channels; x, z, T read, x, z written (float32) and the BF16 copy of x
            n_ang, kb = args[3], args[8]
            nb.append(2 * kb * n_ang * My + (4 * 5 + (2 if args[16] else 0)) * npix * kb)
            nf.append(2 * 2 * npix * n_ang * kb)
        elif name in ("dfx_spmm_pf_forward_blocked", "dfx_spmm_pf_forward_blocked_zt"):
            # the transposed copy of the Radon output is not algorithmic traffic
            n_sub, kb = (args[7], args[12]) if name == "dfx_spmm_pf_forward_blocked" else (args[9], args[14])
            frac = n_sub / op.N_Omega
            nnz = sum(sb["nnz"] for sb in op.sparse_batches) / len(op.sparse_batches) * frac
            nb.append(4 * n_sub * My * (kb + 2 * op.N_seg) + 6 * nnz)
            nf.append(2 * nnz * My)
        elif name in ("dfx_spmm_pf_forward", "dfx_spmm_pf_adjoint", "dfx_spmm_pf_adjoint_zt"):
            # (the transposed copy of the data rows of dfx_spmm_pf_adjoint_zt is not algorithmic traffic)
            if name == "dfx_spmm_pf_adjoint_zt":
                n_sub, kb = args[8], args[10]
            else:
                n_sub = args[6]
                kb = args[10] if name == "dfx_spmm_pf_forward" else args[8]
            frac = n_sub / op.N_Omega
            nnz = sum(sb["nnz"] for sb in op.sparse_batches) / len(op.sparse_batches) * frac
            nb.append(4 * n_sub * My * (kb + 2 * op.N_seg) + 6 * nnz)
            nf.append(2 * nnz * My)
        elif name == "dfx_pf_tc_forward":
            kn, cp, cp_pad, n_sub, my, acc = args[3], args[4], args[5], args[9], args[10], args[12]
            nb.append(2 * n_sub * kn * cp_pad + 2 * n_sub * my * kn + 4 * n_sub * my * cp * (2 if acc else 1))
            nf.append(2 * n_sub * my * kn * cp)
        elif name == "dfx_pf_tc_adjoint":
            kn, cp, cp_pad, n_sub, my = args[3], args[4], args[5], args[9], args[10]
            nb.append(2 * n_sub * kn * cp_pad + 2 * n_sub * my * cp_pad + 2 * n_sub * my * kn)
            nf.append(2 * n_sub * my * kn * cp)
        elif name == "dfx_rows_to_bf16":
            n_sub, my, cp, cp_pad = args[3], args[4], args[5], args[6]
            nb.append(n_sub * my * (4 * cp + 2 * cp_pad))
            nf.append(0)
        elif name in ("dfx_fr_forward", "dfx_fr_backward"):
            # the channel-fastest images in or out and the sinogram rows out or in (the transforms' intermediates
            # are not algorithmic traffic)
            n_ang, kb = args[0]._obj.R, args[4]
            nb.append(4 * kb * (npix + n_ang * My))
            nf.append(0)
        elif name == "dfx_pf_dense_bf16_rows":
            n_rows, kb, cp_pad = args[2], args[4], args[7]
            nb.append(2 * n_rows * kb * cp_pad)
            nf.append(0)
        elif name == "dfx_convert_rows":
            nb.append(6 * args[5] * args[6])
            nf.append(0)
        elif name in ("dfx_gather_channels", "dfx_scatter_channels"):
            nb.append(2 * 4 * npix * args[4])
            nf.append(0)
        elif name == "dfx_spdhg_primal_update":
            nb.append(4 * 6 * args[6])
            nf.append(0)
        elif name == "dfx_spdhg_dual_update":
            nb.append(4 * 7 * args[12] * args[13])
            nf.append(0)
        else:
            nb.append(0)
            nf.append(0)
    return float(np.mean(nb)), float(np.mean(nf))


SERVE_FULL = dict(n=64, rate=2.0, px=(48, 200), omega=(90, 360), eta=(90, 360), rings=(3, 8), K=(500, 10000),
                  slots=8, budget_gb=120.0, max_epochs=100, seed=0,
                  scenario="64 requests, Poisson arrivals 2/s, pixels 48^2-200^2, omega 90-360, eta 90-360, rings 3-8, "
                           "K 500-10000, cubic or hexagonal, SPDHG to 1e-3 relative deviance change, 120 GB budget")
SERVE_SHORT = dict(n=12, rate=2.0, px=(48, 128), omega=(90, 240), eta=(90, 240), rings=(3, 8), K=(500, 2000),
                   slots=8, budget_gb=120.0, max_epochs=150, seed=0,
                   scenario="12 requests, Poisson arrivals 2/s, pixels 48^2-128^2, omega 90-240, eta 90-240, rings "
                            "3-8, K 500-2000 (the serving configuration's ranges, capped to keep the run short), "
                            "SPDHG to 1e-3 relative deviance change, 120 GB budget")


LARGE_SLICE = dict(cfg=dict(Nx=512, Ny=512, My=520, N_Omega=720, angle_range=[0, 180], cor_offset=0.0, N_eta=360,
                             eta_angle_range=[0, 360], energy=12.398 / 0.3, k_direction_0=[0, 0, 1],
                             p_direction_0=[1, 0, 0], detector_direction_origin=[0, -1, 0],
                             detector_direction_positive_90=[0, 0, -1]),
                   material=dict(a=3.52, symmetry_group="cubic", wavelength_A=0.3,
                                 hkl_list=[[1, 1, 1], [2, 0, 0], [2, 2, 0], [3, 1, 1], [2, 2, 2], [4, 0, 0]]),
                   sigma_deg=1.0, subsets=36)


def clustered_grid(K, clusters, sigma, symmetry, seed=0):
    """K orientations in seeded clusters (a tailored grid around candidate orientations): uniformly random centres,
    each member rotated from its centre about a uniformly random axis by |N(0, sigma)|, reduced to the fundamental
    zone; the clusters are contiguous in the grid's order (so that orientation batches hold whole clusters)."""
    from diffractom_b200.grid import Grid, random_rotations, reduce_to_fundamental_zone
    rng = np.random.default_rng(seed)
    centres = random_rotations(clusters, rng)
    owner = np.sort(np.arange(K) % clusters)
    ax = rng.standard_normal((K, 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    ang = np.abs(rng.standard_normal(K)) * sigma
    S = np.zeros((K, 3, 3))
    S[:, 0, 1], S[:, 0, 2], S[:, 1, 2] = -ax[:, 2], ax[:, 1], -ax[:, 0]
    S[:, 1, 0], S[:, 2, 0], S[:, 2, 1] = ax[:, 2], -ax[:, 1], ax[:, 0]
    R = (np.eye(3)[None] + np.sin(ang)[:, None, None] * S
         + (1 - np.cos(ang))[:, None, None] * np.einsum("nij,njk->nik", S, S))           # Rodrigues
    return Grid.from_rotation_matrices(reduce_to_fundamental_zone(np.einsum("nij,njk->nik", R, centres[owner]),
                                                                  symmetry), sigma)


def counts_batched(op, grains, mean, seed=1):
    """Poisson counts of a Voronoi-grain phantom (one orientation per grain, weight 1) computed batch by batch in the
    channel-fastest layout: no (K, Ny, Nx) array of the phantom is made (it would not fit beside the state at the
    large-slice size)."""
    import torch
    rng = np.random.default_rng(seed)
    supp = op.support_mask().ravel()
    pix = np.flatnonzero(supp)
    seeds = rng.choice(len(pix), grains, replace=False)
    sy, sx = (pix[seeds] // op.Nx).astype(np.float32), (pix[seeds] % op.Nx).astype(np.float32)
    grain_k = rng.choice(op.K, grains, replace=False)
    py, px = (pix // op.Nx).astype(np.float32), (pix % op.Nx).astype(np.float32)
    owner = np.empty(len(pix), np.int64)
    for a in range(0, len(pix), 8192):
        d2 = (py[a:a + 8192, None] - sy[None]) ** 2 + (px[a:a + 8192, None] - sx[None]) ** 2
        owner[a:a + 8192] = grain_k[np.argmin(d2, axis=1)]
    with torch.cuda.stream(op.stream()):              # the batch kernels run on the operator's stream
        D = torch.zeros(op.data_shape, dtype=torch.float32, device=op.device)
        buf = torch.zeros(op.batch_elems(), dtype=torch.float32, device=op.device)
        for ib, bt in enumerate(op.batches):
            sel = (owner >= bt["k_start"]) & (owner < bt["k_start"] + bt["K_batch"])
            if not sel.any():
                continue
            buf.zero_()
            idx = torch.as_tensor(pix[sel] * op.Kstride + (owner[sel] - bt["k_start"]), device=op.device)
            buf[idx] = 1.0
            op._direct_batch_k(buf.data_ptr(), ib, D)
        # the Fourier-slice projection of a non-negative image can dip slightly below zero (the interpolation's
        # ringing): Poisson rates are clamped at 0
        lam = (D * (mean / float(D.double().mean().item()))).clamp_min_(0.0)
        g = torch.Generator(device=op.device)
        g.manual_seed(seed + 1)
        b = torch.poisson(lam, generator=g)
    op.stream().synchronize()
    return b


NI512 = dict(LARGE_SLICE, K=50000, clusters=500, grains=500, mean_counts=50.0, epochs=10, max_gb=2.0)


def ni512_run(steps, warmup, K=None):
    """The large tailored-grid slice: 512 x 512 pixels, 720 angles over 180 deg, 520 translations, 360 eta bins, 6
    rings of cubic Ni, K = 50000 orientations in 500 seeded clusters (sigma 1 deg), 36 subsets; the Fourier-slice
    projector (float32 transforms), the PF contraction in BF16 on the tensor cores with the PF of each subset
    generated when it is used (no stored PF), x and z resident in float32, T resident in BF16 (rounded toward zero)
    when it does not fit in float32 beside them, the host x0 moved through the staging buffers, the residual
    recomputed with the float32 operator (its PF rows generated per batch) once per epoch and the deviance in float64.
    A step is one epoch; CUDA events around `steps` epochs after `warmup`."""
    import torch
    from diffractom_b200 import Material, SinglePhaseForwardOperator, SPDHGPoisson, _lib
    w = dict(NI512)
    if K:
        w["K"] = int(K)
        w["clusters"] = min(w["clusters"], w["K"])
        w["grains"] = min(w["grains"], w["K"])
    mat = Material.from_lattice_parameters(**w["material"])
    grid = clustered_grid(w["K"], w["clusters"], np.deg2rad(w["sigma_deg"]), mat.crystal_system, seed=0)
    t0 = time.perf_counter()
    op = SinglePhaseForwardOperator(dict(w["cfg"]), mat, grid, w["max_gb"], normalized=True, projector="fft",
                                    precision="bf16", bf16_pf="generated", pf_mode="generated")
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t0
    gib = lambda: round(torch.cuda.memory_allocated(op.device) / 1024 ** 3, 1)
    mem = {"operator": gib()}
    b = counts_batched(op, w["grains"], w["mean_counts"])
    torch.cuda.empty_cache()
    mem["counts"] = gib()
    sp = SPDHGPoisson(op, subsets=w["subsets"], seed=0, resident="auto")
    x0 = np.zeros(op.coeff_shape, np.float32)
    t0 = time.perf_counter()
    sp._setup(x0, b)
    op.stream().synchronize()
    t_setup = time.perf_counter() - t0
    mem["setup"] = gib()
    sp._iterate(warmup, diagnostics_interval=1, final=False)
    stream = op.stream()
    stream.synchronize()
    timers = KernelTimers(op)
    clocks = Clocks(torch.cuda.current_device())
    n0 = _lib.lib().dfx_launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    timers.on()
    sp._iterate(steps, diagnostics_interval=1, final=False)
    timers.off()
    end.record(stream)
    end.synchronize()
    launches = _lib.lib().dfx_launch_count() - n0 - timers.n_extra
    clk = clocks.stop()
    ms = start.elapsed_time(end)
    f = [st["f"] for st in sp.iter_stats]
    peak = torch.cuda.max_memory_allocated(op.device)
    roof = timers.roofline(op)
    return {"metric": "SPDHG epochs/s (large tailored-grid slice, Fourier-slice projector, BF16 contraction)",
            "value": steps / (ms / 1e3), "unit": "epochs/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
            "ms_per_step": ms / steps, "higher_is_better": True, "dtype": "bf16", "vs_baseline": None,
            "data": "synthetic (seeded clustered grid, Voronoi phantom, Poisson counts)",
            "config": {"workload": "ni512", "pixels": f"{op.Nx}x{op.Ny}", "N_Omega": op.N_Omega, "My": op.My,
                       "N_eta": op.N_eta, "rings": op.N_peaks, "K": op.K, "clusters": w["clusters"],
                       "subsets": w["subsets"], "batches": len(op.batches), "K_batch_max": op.K_batch_max,
                       "projector": op.projector, "fft_channels_per_slice": op._fft_channels,
                       "pf": "BF16 PF of each subset generated when used (two subset buffers); float32 PF rows "
                             "generated per batch for the residual and the step sizes",
                       "resident": sp.resident_used, "T_bf16": sp._t16,
                       "streamed": [n for n in ("x", "z", "T") if n not in sp.resident_used],
                       "operator_build_s": round(t_build, 1), "setup_s": round(t_setup, 1),
                       "deviance_f64_per_epoch": f, "device_gib": {**mem, "max": round(peak / 1024 ** 3, 1)},
                       "epoch": "36 subset iterations + the float32 residual and float64 deviance every epoch",
                       "l2": "inputs larger than L2, no flush"},
            "roofline": roof, "gpu_launches": int(launches), "clocks": clk}


def extras_run(K, steps, warmup):
    """The solvers and tools around the operator at the ti256 geometry with K orientations (FP32, state on the
    device): a FISTAL2 and a FISTAHuber iteration, an OSEM epoch (20 subsets), a PDHG iteration (each the difference
    of a longer and a 1-iteration run), PFGradient (all parameter groups; with the Gauss-Newton blocks), ProjGradient
    (the mean of `steps` synchronised calls after `warmup`), and the orientation search (score_candidates of 4 K
    candidates, 2 input pairs x 2 angle-row sets, every 4th field-of-view pixel; one call). Wall clock."""
    import torch
    from diffractom_b200 import (FISTAHuber, FISTAL2, Grid, OSEMPoisson, PDHGPoisson, SinglePhaseForwardOperator,
                                 estimate_L_power)
    from diffractom_b200.differentiable import PFGradient, ProjGradient
    from diffractom_b200.grid import MatrixGrid
    from diffractom_b200.orientation_search import poisson_score_inputs, score_candidates
    cfg, mat, grid, w = make_problem("ti256", K=K)
    op = SinglePhaseForwardOperator(cfg, mat, grid, w["max_gb"], normalized=True)
    x_true = phantom(op, dict(w, grains=min(w["grains"], op.K)), seed=1)
    b = counts(op, x_true, w["mean_counts"])
    del x_true
    out = {}

    def timed(f, n=steps, w_=warmup):
        for _ in range(w_):
            f()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(n):
            f()
        torch.cuda.synchronize()
        return round(1000 * (time.perf_counter() - t0) / n, 2)

    x = torch.zeros(op.coeff_shape, device="cuda")
    L = estimate_L_power(op, niter=5, verbose=0)

    def per_iteration(run, n):
        """(wall clock of run(1 + n) - that of run(1)) / n: the set-up and the closing work cancel."""
        run(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        run(1)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        run(1 + n)
        torch.cuda.synchronize()
        return round(1000 * ((time.perf_counter() - t1) - (t1 - t0)) / n, 2)

    for name, cls in (("fista_l2", FISTAL2), ("fista_huber", FISTAHuber)):
        out[f"{name}_iteration_ms"] = per_iteration(lambda it, cls=cls: cls(op, L=L).run(x, b, it), steps)
    out["osem_epoch_ms"] = per_iteration(lambda it: OSEMPoisson(op, subsets=20, seed=0).run(
        torch.full(op.coeff_shape, 0.01, device="cuda"), b, it, diagnostics_interval=0), max(1, steps // 2))
    out["pdhg_iteration_ms"] = per_iteration(lambda it: PDHGPoisson(op).run(x, b, it), steps)
    xs = torch.rand(op.coeff_shape, device="cuda")
    r = torch.randn(op.data_shape, device="cuda")
    pg, ph, pj = PFGradient(op), PFGradient(op, hessian=True), ProjGradient(op)
    out["pf_gradient_ms"] = timed(lambda: pg(xs, r))
    out["pf_gradient_hessian_ms"] = timed(lambda: ph(xs, r, groups=("rot", "sigma"), curv=torch.ones_like(r)))
    out["proj_gradient_ms"] = timed(lambda: pj(xs, r))
    mu = torch.clamp(op.direct(xs), min=0.1)
    e, dd = poisson_score_inputs(b.cpu().numpy(), mu.cpu().numpy(), 1.0, np.ones(op.N_seg, np.float32))
    inputs = [(torch.as_tensor(e, device="cuda"), torch.as_tensor(dd, device="cuda"))] * 2
    held = np.zeros(op.N_Omega, bool)
    held[::10] = True
    pixels = np.flatnonzero(op.support_mask().ravel())[::4]
    cand = Grid.from_random_fundamental_zone(4 * K, mat.crystal_system, np.deg2rad(w["sigma_deg"]), seed=9)
    rots, sig = cand.leaf_arrays()
    make = lambda rr: SinglePhaseForwardOperator(cfg, mat, MatrixGrid(rr, sig[:len(rr)]), w["max_gb"],
                                                 normalized=True, pf_mode="generated")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    score_candidates(make, rots, inputs, [~held, held], pixels, top_k=16, chunk=K)
    torch.cuda.synchronize()
    out["search_s"] = round(time.perf_counter() - t0, 2)
    out["search_candidates_per_s"] = round(4 * K / out["search_s"], 1)
    return {"metric": "solvers and tools around the operator (ms per call)", "unit": "ms", "higher_is_better": False,
            "config": {"workload": f"ti256 geometry, {K} orientations, FP32, state on the device",
                       "search": f"{4 * K} candidates in chunks of {K}, 2 input pairs x 2 angle-row sets, "
                                 f"{len(pixels)} pixels, top 16"},
            "steps": steps, "warmup": warmup, "data": "synthetic (seeded phantom, Poisson counts)", "extras": out}


def projector_run(K, steps, warmup):
    """The native and the Fourier-slice projector at the large-slice geometry (512 x 512 pixels, 720 angles over 180
    deg, 520 bins, cubic Ni): forward and backward projection of one batch of K orientations, for the full scan and
    for one of 36 subsets; CUDA events, mean over `steps` launches after `warmup`."""
    import torch
    from diffractom_b200 import Grid, Material, SinglePhaseForwardOperator
    w = LARGE_SLICE
    mat = Material.from_lattice_parameters(**w["material"])
    grid = Grid.from_random_fundamental_zone(K, mat.crystal_system, np.deg2rad(w["sigma_deg"]), seed=0)
    out = {}
    for proj in ("native", "fft"):
        op = SinglePhaseForwardOperator(dict(w["cfg"]), mat, grid, 2.0, normalized=True, projector=proj,
                                        pf_mode="generated")
        op.set_omega_subsets(w["subsets"])
        kb = op.batches[0]["K_batch"]
        img = torch.rand(op.npix * op.Kstride, device=op.device)
        res = torch.empty_like(img)
        st = op.stream()
        for tag, m in (("full", None), ("subset", 0)):
            om, n = (None, op.N_Omega) if m is None else (op._sub[m]["omegas"], op._sub[m]["n"])
            geo = op.geo_gpu if m is None else op._sub[m]["geo"]
            calls = {"forward": lambda: op._radon_fwd(img.data_ptr(), op.coeffs_sino_C.data_ptr(), om, n, kb, m=m),
                     "backward": lambda: op._radon_bwd(op.coeffs_sino_C.data_ptr(), res.data_ptr(), geo, n, kb, m)}
            for name, f in calls.items():
                for _ in range(max(1, warmup)):
                    f()
                st.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                for _ in range(steps):
                    f()
                e1.record(st)
                e1.synchronize()
                out[f"{proj}_{tag}_{name}_us_per_orientation"] = round(1000 * e0.elapsed_time(e1) / steps / kb, 2)
        if proj == "fft":
            out["fft_channels_per_slice"] = op._fft_channels
        op.free_memory()
        del op
        torch.cuda.empty_cache()
    return {"metric": "projector time per orientation (us)", "unit": "us", "higher_is_better": False,
            "config": {"workload": "large slice 512x512, 720 angles over 180 deg, 520 bins, 36 subsets",
                       "K_batch": K}, "steps": steps, "warmup": warmup, "data": "synthetic (random images)",
            "projectors": out}


def local_run(K, steps, warmup, blob=12):
    """The local basis against the dense operator over the same orientations, at the ti256 geometry (256 x 256
    pixels, 360 angles, 263 bins, 360 eta bins, 8 Ti rings): K orientations, each allowed in a seeded disc of radius
    blob pixels (inside the field of view). direct_cl / adjoint_cl of the full scan and of one of 20 subsets (CUDA
    events, mean over `steps` after `warmup`), and one SPDHG epoch (20 subsets; wall clock of a run of 1 + steps / 2
    epochs less that of a 1-epoch run)."""
    import torch
    from diffractom_b200 import SinglePhaseForwardOperator, SPDHGPoisson
    from diffractom_b200.grid import MatrixGrid
    from diffractom_b200.local import LocalSinglePhaseForwardOperator, LocalSupport
    cfg, mat, grid, w = make_problem("ti256", K=K)
    rng = np.random.default_rng(5)
    Ny, Nx = cfg["Ny"], cfg["Nx"]
    yy, xx = np.mgrid[:Ny, :Nx]
    cy, cx = rng.uniform(blob, Ny - blob, K), rng.uniform(blob, Nx - blob, K)
    mask = (yy[None] - cy[:, None, None]) ** 2 + (xx[None] - cx[:, None, None]) ** 2 <= blob ** 2
    loc = LocalSinglePhaseForwardOperator(cfg, mat, grid, w["max_gb"], LocalSupport.from_mask(mask), normalized=True)
    mats, sig = grid.leaf_arrays()
    oi = loc.orientation_index
    dense = SinglePhaseForwardOperator(cfg, mat, MatrixGrid(mats[oi], sig[oi]), w["max_gb"], normalized=True,
                                       pf_mode=loc.pf_mode)
    x = torch.as_tensor(rng.random(loc.n_coef).astype(np.float32) * loc.coefficient_mask(), device="cuda")
    xd = torch.as_tensor(loc.to_dense(x.cpu().numpy())[oi], device="cuda")
    out = {"fill": loc.n_coef / (loc.K * Nx * Ny), "n_coef": loc.n_coef, "patches": loc.n_patches,
           "batches": len(loc.batches), "K_batch_max": loc.K_batch_max}
    for op in (loc, dense):
        op.set_omega_subsets(20)
    data = torch.empty(loc.data_shape, device="cuda")

    def timed(op, f):
        st = op.stream()
        for _ in range(max(1, warmup)):
            f()
        st.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            f()
        e1.record(st)
        e1.synchronize()
        return round(e0.elapsed_time(e1) / steps, 3)

    for name, op, c in (("local", loc, x), ("dense", dense, xd)):
        g = torch.empty_like(c)
        out[f"{name}_direct_ms"] = timed(op, lambda: op.direct_cl(c, data))
        out[f"{name}_adjoint_ms"] = timed(op, lambda: op.adjoint_cl(data, g))
        out[f"{name}_direct_subset_ms"] = timed(op, lambda: op.direct_cl(c, data, subset=3))
        out[f"{name}_adjoint_subset_ms"] = timed(op, lambda: op.adjoint_cl(data, g, subset=3))
    b = torch.poisson(torch.clamp(dense.direct(xd) * 20.0, min=0.0)).contiguous()
    n_ep = max(1, steps // 2)

    def run_time(op, c, epochs):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        SPDHGPoisson(op, subsets=20, seed=0).run(torch.zeros_like(c), b, epochs, diagnostics_interval=epochs)
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    for name, op, c in (("local", loc, x), ("dense", dense, xd)):
        run_time(op, c, 1)
        # an epoch: the difference of two runs (set-up, final deviance and state download cancel)
        out[f"{name}_spdhg_epoch_ms"] = round(1000 * (run_time(op, c, 1 + n_ep) - run_time(op, c, 1)) / n_ep, 2)
    return {"metric": "local basis vs dense operator (ms per call)", "unit": "ms", "higher_is_better": False,
            "config": {"workload": f"ti256 geometry, {K} orientations, each in a disc of radius {blob} px",
                       "subsets": 20}, "steps": steps, "warmup": warmup, "data": "synthetic", "local": out}


def serving_run(n, rate, px, omega, eta, rings, K, slots, budget_gb, max_epochs, seed, scenario, precision="bf16"):
    """Requests of random size drawn uniformly from the ranges (cubic Al or hexagonal Ti, the first `rings`
    reflections), seeded phantoms and Poisson counts made beforehand, then submitted to a ReconstructionServer at
    Poisson arrival times; returns its latency statistics."""
    import torch
    from diffractom_b200 import Grid, Material, SinglePhaseForwardOperator
    from diffractom_b200.serving import ReconstructionServer, Request
    rng = np.random.default_rng(seed)
    cub = [[1, 1, 1], [2, 0, 0], [2, 2, 0], [3, 1, 1], [2, 2, 2], [4, 0, 0], [3, 3, 1], [4, 2, 0]]
    reqs = []
    t_prep = time.perf_counter()
    for i in range(n):
        p = int(rng.integers(px[0], px[1] + 1))
        cfg = dict(Nx=p, Ny=p, My=p + 4 + p // 40, N_Omega=int(rng.integers(omega[0], omega[1] + 1)),
                   angle_range=[0, 180], cor_offset=0.0, N_eta=int(rng.integers(eta[0], eta[1] + 1)),
                   eta_angle_range=[0, 360], energy=12.398 / 0.3, k_direction_0=[0, 0, 1], p_direction_0=[1, 0, 0],
                   detector_direction_origin=[0, -1, 0], detector_direction_positive_90=[0, 0, -1])
        nr = int(rng.integers(rings[0], rings[1] + 1))
        if rng.random() < 0.5:
            mat = Material.from_lattice_parameters(a=4.05, symmetry_group="cubic", wavelength_A=0.3,
                                                   hkl_list=cub[:nr])
        else:
            mat = Material.from_lattice_parameters(**{**WORKLOADS["ti256"]["material"],
                                                      "hkl_list": WORKLOADS["ti256"]["material"]["hkl_list"][:nr]})
        k = int(rng.integers(K[0], K[1] + 1))
        grid = Grid.from_random_fundamental_zone(k, mat.crystal_system, np.deg2rad(3.0), seed=seed + i)
        op = SinglePhaseForwardOperator(cfg, mat, grid, 1.0, normalized=True)
        x = phantom(op, {"grains": 10, "background": 0.0}, seed=seed + i)
        b = counts(op, x, 50.0, seed=seed + i).cpu().numpy()
        op.free_memory()
        del op, x
        reqs.append(Request(cfg, mat, grid, b, subsets=8, max_epochs=max_epochs, tol=1e-3, precision=precision))
    torch.cuda.empty_cache()
    t_prep = time.perf_counter() - t_prep
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
    srv = ReconstructionServer(device=torch.cuda.current_device(), max_slots=slots, hbm_budget_gb=budget_gb).start()
    t0 = time.perf_counter()
    for r, t in zip(reqs, arrivals):
        delay = t - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        srv.submit(r)
    finished = srv.wait_all(timeout=1800)
    srv.stop()
    st = srv.stats()
    st.update({"scenario": scenario, "slots": slots, "all_finished": bool(finished), "precision": precision,
               "input_preparation_s": round(t_prep, 1),
               "converged": int(sum(1 for r in reqs if r.error is None and r.epochs < max_epochs)),
               "epochs_p50": float(np.median([r.epochs for r in reqs])),
               "deviance_first_request": [float("%.6g" % f) for f in reqs[0].deviance[:12]],
               "errors": [r.error for r in reqs if r.error][:3]})
    return st


def measure_e2e(op, w, b_dev, steps, dist=None, world=1, shards=None):
    """The metric through the public API on host arrays: SPDHGPoisson.run(NumPy x0, NumPy b, steps epochs); with
    orientation shards every rank runs it on its shard, the time is the maximum over the ranks."""
    import torch
    from diffractom_b200 import SPDHGPoisson
    b_host = torch.empty(b_dev.shape, dtype=torch.float32, pin_memory=True)
    b_host.copy_(b_dev)
    b_np = b_host.numpy()
    x0 = np.zeros(op.coeff_shape, np.float32)
    sp = SPDHGPoisson(op, subsets=w["subsets"], seed=0, shards=shards)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    x = sp.run(x0, b_np, steps, diagnostics_interval=1)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    if dist is not None:
        tt = torch.tensor([dt], dtype=torch.float64, device=op.device)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        dt = float(tt.item())
    h2d = b_np.nbytes + x0.nbytes
    d2h = x.nbytes + sp.state["y"].nbytes + sp.state["z"].nbytes
    return {"value": world * steps / dt, "unit": "epochs/s", "h2d_bytes_per_step": h2d // steps,
            "d2h_bytes_per_step": d2h // steps,
            "includes": "upload of x0 and b, step sizes S and T (1 forward + M subset adjoints), epochs with the "
                        "diagnostics of every epoch (residual and deviance), download of x, y, z"}


def run_reference(a, rank):
    """The reference arm: diffractom's path on the host cores. The reference is Python + OpenCL and no OpenCL runtime
    or pyopencl exists here, so the reference's kernels as restated in oracle/ (float32 like the reference's, OpenMP
    over all host threads) are timed on this arm's workload and configuration. A step is one whole SPDHG subset
    iteration over all orientation batches (CpuSubsetIterations: 1 / M of an epoch's work, nothing extrapolated);
    value = epochs/s = 1 / (M x the mean step time). The steps and warm-up steps asked for are run as long as the
    timed steps stay within REFERENCE_BUDGET_S; the line reports how many ran."""
    if rank != 0:
        return 0
    from diffractom_b200.geometry import OperatorGeometry
    cfg, mat, grid, w = make_problem(a.workload, K=a.K)
    geom = OperatorGeometry(cfg, mat, grid, normalized=True)
    t0 = time.perf_counter()
    it = CpuSubsetIterations(geom, w, dense_batches(geom, w["max_gb"]))
    for _ in range(min(a.warmup, 1)):
        it.step()
    secs = []
    while len(secs) < max(1, a.steps) and sum(secs) < REFERENCE_BUDGET_S:
        secs.append(it.step())
    step_s = float(np.mean(secs))
    value = 1.0 / (w["subsets"] * step_s)
    desc = it.describe(len(secs))
    line = {"metric": METRIC, "value": value, "unit": "epochs/s", "n_gpus": 0, "steps": len(secs),
            "warmup": min(a.warmup, 1), "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": a.workload + (f" (K {a.K})" if a.K else ""), "K": geom.K,
                       "pixels": f"{geom.Nx}x{geom.Ny}", "subsets": w["subsets"],
                       "step": f"one SPDHG subset iteration = 1/{w['subsets']} epoch",
                       "steps_asked": a.steps, "warmup_asked": a.warmup,
                       "wall_s": round(time.perf_counter() - t0, 1)},
            "cpu_baseline": {"value": value, "unit": "epochs/s", "cores": it.threads, "kind": "port",
                             "sample": desc},
            "e2e": {"value": value, "unit": "epochs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "diffractom runs its path as OpenCL kernels (pyopencl); no OpenCL runtime or pyopencl is "
                    "installed on this host, so the timed reference is its CPU restatement in oracle/ (float32, "
                    "OpenMP)"}
    print(json.dumps(line), flush=True)
    return 0


REFERENCE_BUDGET_S = 240.0


if __name__ == "__main__":
    sys.exit(main())
