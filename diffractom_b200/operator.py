"""SinglePhaseForwardOperator: the single-phase texture-tomography forward operator and its adjoint on a B200.

Drop-in for diffractom's SinglePhaseForwardOperator (operators/single_phase_forward_operator.py, "SPFO" below): the
same constructor signature, cfg keys, batching (max_gb), array layouts and methods used by the solvers, with CUDA
torch tensors in place of pyopencl arrays. The model (SPFO:158-164):

    data = PF @ Radon(coeffs),   coeffs (K, Ny, Nx),   data (N_Omega, My, N_eta * N_rings)

computed batch by batch over the orientations: the Radon transform of every orientation's image (channel-fastest,
the batch's orientations are the channels), then per rotation angle the product of the sinogram (My x Kb) with the
sparse pole-figure matrix (Kb x N_eta * N_rings). The adjoint is the exact transpose: the transposed products
(scaled by N_Omega / pi) and the backprojection with angle weights pi / N_Omega.

All device work goes through the C ABI of diffractom_b200/_lib/libdfx_b200.so (hand-written sm_100a kernels); torch
only holds the device memory and provides the stream. Host set-up (quadrature, probed directions, pole axes,
projector geometry) is float64 NumPy, uploaded as float32 (geometry.py).
"""
from __future__ import annotations

import ctypes
import math
import time
import warnings
from typing import Any, Mapping

import numpy as np
import torch

from . import _lib
from .arrays import as_host, check_device, is_device, on_op_stream, stream_scope
from .geometry import OperatorGeometry, interleaved_subsets
from .quadrature import DEFAULT_TOL

SPARSE_BATCH_MAX = 1024   # largest orientation batch of the sparse modes (SPFO:134)
AUTO_FFT_PIXELS = 400 * 400   # projector="auto": the Fourier-slice projector for grids of more pixels (SPFO:27)
SPARSE_MIN_BATCHES = 4    # sparse modes: at least this many batches (SPFO:135)
CAND_BYTES = 2 + 4 + 4 + 4 + 4          # per candidate / non-zero scratch of the reference's generator
NNZ_BYTES = 2 + 4 + 4 + 2 + 4 + 2 + 4   # (pf_generate.py:29-30), used by the batch-size rule
GTABLE_MIN_ANGLES = 64                   # float32 forwards of this many angles read the grouped table
KSTRIDE_ALIGN = 16                       # channel stride of the batch buffers (16 channels per tensor-memory load)


def _stream_handle(stream) -> ctypes.c_void_p:
    return ctypes.c_void_p(stream.cuda_stream)


class SinglePhaseForwardOperator:
    """Single-material pole-figure forward operator (SPFO:158)."""

    coefficient_layout = "dense"
    _pf_forward_csr = True
    # True: BF16 images are projected on the tensor cores (dfx_radon_forward_tc) where the geometry admits it. Off by
    # default: at 256 x 256 pixels, 18 angles and 1024 channels a launch took 0.54 ms against 0.25 ms for the ray
    # table's gather (dfx_radon_forward_table_bf16_bf16)
    use_tc_forward = False
    # with both CSR copies stored, the forward products run over an eta-blocked copy of the forward CSR (four
    # neighbouring eta bins of a ring per entry; the same sums bit for bit); False: over the forward CSR itself
    forward_blocks = True
    # the blocked forward products read the Radon output transposed to detector lines fastest (one warp per block
    # row, whole 128-byte segments of a Z column per entry; dfx_spmm_pf_forward_blocked_zt, the same bits) through a
    # buffer of up to zt_max_angles angles of a batch; False: dfx_spmm_pf_forward_blocked on the channel-fastest output
    forward_lines_fastest = True
    # the adjoint products read the data rows transposed to detector lines fastest (one warp per orientation row,
    # whole 128-byte segments of a data column per entry; dfx_spmm_pf_adjoint_zt, the same bits) through the same
    # buffer; False: dfx_spmm_pf_adjoint on the segment-fastest rows
    adjoint_lines_fastest = True
    zt_max_angles = 64                   # angles per transpose chunk at most
    zt_max_bytes = 256 * 1024 ** 2       # the transpose buffer at most (at least one angle)
    zt_max_groups = 0

    def __init__(self, cfg: Mapping[str, Any], material, grid, max_gb: float, verbose: bool = False,
                 normalized: bool = False, ctx=None, queue=None, pf_mode: str = "auto", sparse_max_fill: float = 0.3,
                 sparse_max_fill_partial: float = 0.1, sparse_max_gb: float | None = None, projector: str = "auto",
                 radon_kernel: str | None = None, fft_max_gb: float = 1.5, reserve_coefficient_arrays: int = 3,
                 pf_cutoff_sigma: float | None = 4.0, quadrature="auto", quadrature_tol: float = DEFAULT_TOL,
                 intensity_model=None, sparse_batch_max: int = SPARSE_BATCH_MAX, rings=None, ring_two_theta=None,
                 reflection_two_theta: bool = False, window_parallax=None, ring_intensities=None,
                 precision: str = "fp32", bf16_pf: str = "auto", **kwargs):
        """Arguments as diffractom's (SPFO:169-197). ctx: None, a torch.device or a CUDA device index (the GPU);
        queue: None (the current torch stream at every call) or a torch.cuda.Stream. ring_intensities: with
        normalized=False, the integrated intensity of every ring (diffractom computes them from structure factors,
        which this package does not model). projector: "native" (the ray-driven / pixel-driven pair), "fft" (the
        Fourier-slice projector, fourier.py; fft_max_gb bounds its scratch per channel slice) or "auto" (the
        Fourier-slice one for grids of more than 400 x 400 pixels at float32 precision, SPFO:448-449).

        precision: "fp32" (the reference's arithmetic) or "bf16": direct_cl / adjoint_cl on device tensors then run
        the Radon output through BF16 and the pole-figure products on the tensor cores (dense BF16 PF, float32
        accumulation); the float32 sparse PF stays available (NumPy (streamed) calls stay float32). bf16_pf: "stored"
        (the BF16 PF of all angles kept), "generated" (the PF of each product's angles generated when it runs) or
        "auto" (stored if it takes at most half of the free device memory). reflection_two_theta: every pole axis
        probes at its reflections' own Bragg angle (the windows of rings= then hold reflections of different angles;
        SPFO:236-244).

        pf_mode "dense" applies the float32 PF by batched SGEMMs (no omega subsets, as the reference). Not provided
        (NotImplementedError): projector "gratopy"."""
        lib = _lib.lib()                                    # fails loudly without the CUDA library
        if not torch.cuda.is_available():
            raise RuntimeError("SinglePhaseForwardOperator needs a CUDA device")
        if isinstance(ctx, torch.device):
            self.device = ctx
        elif isinstance(ctx, int):
            self.device = torch.device("cuda", ctx)
        else:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self._lib = lib
        self.queue = queue if isinstance(queue, torch.cuda.Stream) else None
        self.ctx = self.device
        self.verbose = verbose
        self.reserve_coefficient_arrays = int(reserve_coefficient_arrays)
        self.pf_cutoff_sigma = pf_cutoff_sigma
        self.sparse_batch_max = int(sparse_batch_max)
        self.cfg = {**cfg, **kwargs}
        self.material, self.grid = material, grid
        if projector not in ("auto", "native", "fft", "gratopy"):
            raise ValueError(f"projector must be 'auto', 'native', 'fft' or 'gratopy', not {projector!r}")
        if projector == "gratopy":
            raise NotImplementedError("projector 'gratopy' is not provided (the native and 'fft' projectors are)")
        if pf_mode not in ("dense", "sparse", "generated", "auto"):
            raise ValueError(f"pf_mode must be 'dense', 'sparse', 'generated' or 'auto', not {pf_mode!r}")
        # the native projector's geometry is made in any case (the Fourier-slice projector shares its conventions)
        geom_kernel = "trapezoid" if projector == "fft" or radon_kernel is None else radon_kernel

        # ---- host set-up (SPFO:376-494): rings, quadrature, probed directions, poles, projector geometry
        geom = OperatorGeometry(self.cfg, material, grid, normalized=normalized, quadrature=quadrature,
                                quadrature_tol=quadrature_tol, pf_cutoff_sigma=pf_cutoff_sigma,
                                radon_kernel=geom_kernel, rings=rings, ring_two_theta=ring_two_theta,
                                ring_intensities=ring_intensities, reflection_two_theta=reflection_two_theta)
        self.__dict__.update({k: v for k, v in vars(geom).items() if k != "cfg"})
        self.geometry = geom
        self.pf_batch_max_gb = float(max_gb)
        if projector == "auto":
            projector = ("fft" if self.Nx * self.Ny > AUTO_FFT_PIXELS and radon_kernel in (None, "hat")
                         else "native")
        if radon_kernel is None:
            radon_kernel = "trapezoid" if projector == "native" else "hat"
        if radon_kernel != "hat" and projector != "native":
            raise ValueError(f"radon_kernel={radon_kernel!r} needs the native projector (projector is {projector!r})")
        self.projector = projector
        self.radon_kernel = radon_kernel
        self._kernel_id = 1 if geom_kernel == "trapezoid" else 0
        self.fft_max_gb = float(fft_max_gb)

        with stream_scope(self):          # device work of the build on the operator's stream
            # ---- device copies
            dev = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=self.device)
            self.coords_gpu = dev(self.coords_cpu)
            self.poles_gpu = dev(self.poles_cpu)
            self.axis_start_gpu = dev(self.axis_start_cpu, torch.int32)
            self.axis_count_gpu = dev(self.axis_count_cpu)
            self.inv_sigma2_gpu = dev(self.inv_sigma2_cpu)
            self.norm_factor_gpu = dev(self.norm_factor_cpu)
            self.quad_weights_gpu = None if self.quad_weights_cpu is None else dev(self.quad_weights_cpu)
            self.intens_gpu = None if self.normalized else dev(self.intens_cpu)
            self.geo_gpu = dev(self.radon_geo.geo)
            self._upload_axis_theta()
            self.window_parallax = None
            self._wp = None
            if window_parallax is not None:
                self.set_window_parallax(**dict(window_parallax), _build=False)
            self._pf_version = 0
            self._sub_version = 0
            self._make_pfg()
            self._scratch = torch.empty(0, dtype=torch.uint8, device=self.device)
            self._zt = None
            self._ray_supp = {}
            self._supp_tiles = {}
            self._fft = None
            if self.projector == "fft":
                self._ray_rp = self._ray_ent = self._ray_grp = None
                self.ray_taps = 0
                self._build_fourier()
            else:
                self._ray_rp, self._ray_ent, self.ray_taps = self._build_ray_table()
                self._ray_grp = self._build_group_table()
            self.omega_subsets = None
            self._sub = []
            self._streamer = None

            if precision not in ("fp32", "bf16"):
                raise ValueError(f"precision must be 'fp32' or 'bf16', not {precision!r}")
            self.precision = precision
            # ---- batches and the sparse PF matrix (SPFO:1026-1094, 1207-1373)
            self.get_pf_batches_for_material()
            self.pf_mode = pf_mode
            self.sparse_batches = None
            self.pf_storage = None
            if sparse_max_gb is None:
                sparse_max_gb = self.default_sparse_budget_gb()
            self._pf_build = dict(mode=pf_mode, max_fill=sparse_max_fill, max_gb=sparse_max_gb,
                                  max_fill_partial=sparse_max_fill_partial)
            self.build_sparse_pf(**self._pf_build)
            self.pf_bf16 = None
            self.bf16_pf = bf16_pf
            if precision == "bf16":
                self.build_dense_bf16_pf()

    # ------------------------------------------------------------------ small helpers
    def _upload_axis_theta(self):
        """reflection_two_theta: the rotated p0 and every pole axis's sin / cos of theta on the device (None
        otherwise)."""
        if not self.reflection_two_theta:
            self.w_gpu = self.axis_sin_gpu = self.axis_cos_gpu = None
            return
        dev = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32), device=self.device)
        self.w_gpu, self.axis_sin_gpu, self.axis_cos_gpu = dev(self.w_cpu), dev(self.axis_sin_cpu), dev(self.axis_cos_cpu)

    def _make_pfg(self):
        """The PF kernels' view of the device parameters (dfx_pf_geometry), made again after they change."""
        self._pfg = _lib.PFGeometry(
            self.coords_gpu.data_ptr(), self.poles_gpu.data_ptr(), self.axis_start_gpu.data_ptr(),
            self.axis_count_gpu.data_ptr(), self.inv_sigma2_gpu.data_ptr(), self.norm_factor_gpu.data_ptr(),
            None if self.quad_weights_gpu is None else self.quad_weights_gpu.data_ptr(),
            None if self.intens_gpu is None else self.intens_gpu.data_ptr(),
            self.N_Omega, self.N_eta, self.N_peaks, self.N_axes, self.N_Omega_subdivisions, self.N_eta_subdivisions,
            self.K, float(self.pf_cut),
            *((None, None, None) if self.w_gpu is None else
              (self.w_gpu.data_ptr(), self.axis_sin_gpu.data_ptr(), self.axis_cos_gpu.data_ptr())),
            *((None,) * 5 + (0.0, 0.0) if self._wp is None else
              tuple(self._wp[k].data_ptr() for k in ("pos", "cov", "b", "ax", "ch")) + (self._wp["invD"],
                                                                                      self._wp["eta"])))

    def set_window_parallax(self, windows, sigma, distance, positions=None, covariances=None, lorentz=0.0,
                            gamma=None, _build=True):
        """Window fractions with sample parallax (SPFO:704-734, the window_parallax option): channels are
        integration windows (windows (P, 2) two-theta limits, rad) that cut the reflections' radial profiles (width
        sigma, rad: scalar, per channel or per pole axis), and an orientation's depth x along the beam shifts its
        rings by -(x / distance) sin 2t cos 2t (distance in translation steps); positions (K, 2) / covariances
        (K, 3): the orientations' mean (col, row) and spatial covariance in pixels (default the image centre, no
        spread); lorentz, gamma: a pseudo-Voigt profile's Lorentzian share and half width (default sigma
        sqrt(2 ln 2)). The sparse PF matrix is rebuilt (a call after construction)."""
        from .geometry import image_direction
        P, A, K = self.N_peaks, self.N_axes, self.K
        win = np.asarray(windows, np.float64).reshape(P, 2)
        st = np.asarray(self.axis_start_cpu)
        ch = np.repeat(np.arange(P), np.diff(st))
        tth = (np.asarray(self.axis_two_theta_built, np.float64) if self.reflection_two_theta
               else np.asarray(self.two_theta_peaks, np.float64)[ch])
        sig = np.asarray(sigma, np.float64)
        sig_a = (np.broadcast_to(sig, (A,)) if sig.ndim == 0 or (sig.size == A and sig.size != P)
                 else sig.reshape(P)[ch])
        px = self.image_width / max(self.Nx, self.Ny)
        cxy = np.array([(self.Nx - 1) / 2, (self.Ny - 1) / 2])
        pos = np.zeros((K, 2)) if positions is None else (np.asarray(positions, np.float64).reshape(K, 2) - cxy) * px
        cov = np.zeros((K, 3)) if covariances is None else np.asarray(covariances, np.float64).reshape(K, 3) * px ** 2
        b = image_direction(np.asarray(self.cfg["p_direction_0"], np.float64)[:2], np.asarray(self.angles))
        gam = (np.sqrt(2 * np.log(2)) * sig_a if gamma is None
               else np.broadcast_to(np.asarray(gamma, np.float64), (A,)))
        dev = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32).reshape(-1), device=self.device)
        self.window_parallax = dict(windows=win, sigma=sig_a, distance=float(distance), positions=positions,
                                    covariances=covariances, lorentz=float(lorentz), gamma=gamma)
        self._wp = {"pos": dev(pos), "cov": dev(np.concatenate([cov, np.zeros((K, 1))], 1)), "b": dev(b),
                    "ax": dev(np.stack([tth, np.sin(tth) * np.cos(tth), sig_a ** 2, gam], 1)), "ch": dev(win),
                    "invD": float(np.float32(1.0 / float(distance))), "eta": float(np.float32(lorentz))}
        self._make_pfg()
        if _build:
            self.release_omega_subsets()
            self.build_sparse_pf(**self._pf_build)
            if self.precision == "bf16":
                self.pf_bf16 = None
                self.build_dense_bf16_pf()
            self._pf_version += 1

    def stream(self) -> torch.cuda.Stream:
        return self.queue if self.queue is not None else torch.cuda.current_stream(self.device)

    def _s(self):
        return _stream_handle(self.stream())

    def _call(self, name, *args):
        _lib.check(getattr(self._lib, name)(*args))

    def scratch(self, nbytes: int) -> torch.Tensor:
        """A device scratch buffer of at least nbytes (reused; grows on demand)."""
        if self._scratch.numel() < nbytes:
            self._scratch = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=self.device)
        return self._scratch

    def detector_shifts(self):
        return self.geometry.detector_shifts()

    def _build_ray_table(self, supp=None):
        """The projector's non-zero taps per (angle, bin) (dfx_radon_table_*): the forward projection then reads
        (pixel, weight) pairs instead of evaluating the footprint of every candidate pixel in every call. supp (a
        uint8 (Ny * Nx) device mask): the taps of the support's pixels only. Returns (row_ptr, entries, taps)."""
        R, ns = self.N_Omega, self.My
        n = R * ns
        s = self._s()
        sp = None if supp is None else supp.data_ptr()
        rp = torch.empty(n + 1, dtype=torch.int32, device=self.device)
        self._call("dfx_radon_table_count", self.geo_gpu.data_ptr(), R, self.Nx, self.Ny, ns, self._kernel_id, sp,
                   rp.data_ptr(), s)
        self.stream().synchronize()
        cnt64 = rp[:n].to(torch.int64).sum()
        total = int(cnt64.item())
        if total >= 2 ** 31:
            raise ValueError(f"the projector has {total} taps, more than 2^31 - 1")
        nb = self._lib.dfx_scan_scratch_bytes(n)
        scr = self.scratch(nb)
        self._call("dfx_scan_exclusive_i32", rp.data_ptr(), rp.data_ptr(), n, scr.data_ptr(), nb, s)
        ent = torch.empty(2 * max(total, 1), dtype=torch.int32, device=self.device)
        self._call("dfx_radon_table_fill", self.geo_gpu.data_ptr(), R, self.Nx, self.Ny, ns, self._kernel_id, sp,
                   rp.data_ptr(), ent.data_ptr(), s)
        return rp, ent, total

    def _build_group_table(self, supp=None):
        """The grouped ray table of the float32 forward of many angles (dfx_radon_gtable_*): per (angle, four bins)
        the pixels that reach them with their four weights, so that each pixel's channels are loaded once per group;
        the sums are the per-bin table's bits. Returns (row_ptr, pixels, weights)."""
        R, ns = self.N_Omega, self.My
        n = R * (-(-ns // 4))
        s = self._s()
        sp = None if supp is None else supp.data_ptr()
        rp = torch.empty(n + 1, dtype=torch.int32, device=self.device)
        self._call("dfx_radon_gtable_count", self.geo_gpu.data_ptr(), R, self.Nx, self.Ny, ns, self._kernel_id, sp,
                   rp.data_ptr(), s)
        self.stream().synchronize()
        total = int(rp[:n].to(torch.int64).sum().item())
        if total >= 2 ** 31:
            raise ValueError(f"the grouped projector table has {total} entries, more than 2^31 - 1")
        nb = self._lib.dfx_scan_scratch_bytes(n)
        scr = self.scratch(nb)
        self._call("dfx_scan_exclusive_i32", rp.data_ptr(), rp.data_ptr(), n, scr.data_ptr(), nb, s)
        pix = torch.empty(max(total, 1), dtype=torch.int32, device=self.device)
        w = torch.empty((max(total, 1), 4), dtype=torch.float32, device=self.device)
        self._call("dfx_radon_gtable_fill", self.geo_gpu.data_ptr(), R, self.Nx, self.Ny, ns, self._kernel_id, sp,
                   rp.data_ptr(), pix.data_ptr(), w.data_ptr(), s)
        return rp, pix, w

    @on_op_stream
    def support_ray_table(self, supp):
        """The ray table restricted to a support mask (uint8 (Ny * Nx) device tensor), built once per mask content
        and kept: the solvers' forward projections of iterates that are zero outside the support read it (same
        bits, fewer taps)."""
        if self.projector == "fft":
            return None                     # the Fourier-slice projector reads every pixel in any case
        key = bytes(supp.cpu().numpy())
        hit = self._ray_supp.get(key)
        if hit is None:
            hit = self._build_ray_table(supp) + (self._build_group_table(supp),)
            self._ray_supp[key] = hit
        return hit

    def _build_fourier(self):
        """The Fourier-slice projector of the geometry (fourier.py) and its channel slice: as many channels as fit
        fft_max_gb of scratch (at most 256, at least 1), SPFO:469-481."""
        from .fourier import FourierHost, FourierProjector
        host = FourierHost(self.angles, self.Nx, self.Ny, self.My, self.image_width, self.My, self.detector_shifts(),
                           self.angle_weight)
        self._fft = FourierProjector(host, self.device)
        per = self._fft.scratch_bytes(1)
        self._fft_channels = int(max(1, min(256, self.fft_max_gb * 1024 ** 3 // per)))

    def _fft_of(self, m):
        return self._fft if m is None else self._sub[m]["fft"]

    def _fft_run(self, forward, m, src_ptr, dst_ptr, kb):
        fp = self._fft_of(m)
        ch = self._fft_channels
        nb = fp.scratch_bytes(min(ch, max(kb, 1)))
        scr = self.scratch(nb)
        (fp.forward if forward else fp.backward)(src_ptr, dst_ptr, self.Kstride, kb, ch, scr.data_ptr(), nb, self._s())

    def _radon_bwd(self, sino_ptr, out_ptr, geo, n_ang, kb, m):
        """Backward projection of a (n_ang, My, Kstride) sinogram into a channel-fastest batch (angles of subset m,
        None: all)."""
        if self.projector == "fft":
            self._fft_run(False, m, sino_ptr, out_ptr, kb)
            return
        self._call("dfx_radon_backward", sino_ptr, out_ptr, geo.data_ptr(), n_ang, self.Nx, self.Ny, self.My,
                   self.Kstride, kb, self._kernel_id, int(self.radon_geo.n_taps), self._s())

    def _radon_fwd(self, src_ptr, dst_ptr, om, n_ang, kb, sld=None, ray=None, m=None):
        """Forward projection of a channel-fastest batch through the ray table (ray: (row_ptr, entries, taps) of a
        support table, None: the full one): angles om (int32 device tensor of angle indices, None: all) into float32
        (sld None) or BF16 (row stride sld) sinogram rows."""
        if self.projector == "fft":
            if sld is not None:
                raise NotImplementedError("BF16 sinograms need the native projector")
            self._fft_run(True, m, src_ptr, dst_ptr, kb)
            return
        om_ptr = None if om is None else om.data_ptr()
        rp, ent = (self._ray_rp, self._ray_ent) if ray is None else ray[:2]
        grp = self._ray_grp if ray is None else (ray[3] if len(ray) > 3 else None)
        # the grouped table has a quarter of the warps: for a few angles (a subset) the per-bin one fills the GPU
        # better (at 256 x 256, 1024 channels and 18 angles: 0.56 ms per-bin, 0.63 to 0.67 ms grouped)
        if sld is None and grp is not None and n_ang >= GTABLE_MIN_ANGLES:
            self._call("dfx_radon_forward_gtable", src_ptr, dst_ptr, grp[0].data_ptr(), grp[1].data_ptr(),
                       grp[2].data_ptr(), om_ptr, n_ang, self.My, self.Kstride, kb, float(self.radon_geo.scale),
                       self._s())
        elif sld is None:
            self._call("dfx_radon_forward_table", src_ptr, dst_ptr, rp.data_ptr(), ent.data_ptr(),
                       om_ptr, n_ang, self.My, self.Kstride, kb, float(self.radon_geo.scale), self._s())
        else:
            self._call("dfx_radon_forward_table_bf16", src_ptr, dst_ptr, sld, rp.data_ptr(),
                       ent.data_ptr(), om_ptr, n_ang, self.My, self.Kstride, kb,
                       float(self.radon_geo.scale), self._s())

    @property
    def coeff_shape(self):
        return (self.K, self.Ny, self.Nx)

    @property
    def data_shape(self):
        return (self.N_Omega, self.My, self.N_seg)

    @property
    def npix(self) -> int:
        return self.Nx * self.Ny

    def support_mask(self):
        """(Ny, Nx) bool mask of the pixels inside the field of view at every projection angle (SPFO:544-547)."""
        return self.geometry.support_mask()

    # ------------------------------------------------------------------ batching
    def get_pf_batches_for_material(self, K_batch=None):
        """Orientation batches: K_batch each, or as many as a dense PF batch of max_gb holds (SPFO:1026-1094);
        K_batch_max rounded up to a multiple of 4, 2^31 element limits of the batch buffers."""
        R, C, P, K = self.N_Omega, self.N_eta, self.N_peaks, self.K
        bytes_per_K = R * C * P * 4
        max_bytes = self.pf_batch_max_gb * (1024 ** 3)
        if K_batch is not None:
            kbm = max(1, min(int(K_batch), K))
        elif bytes_per_K > 0.01:
            kbm = min(max(int(max_bytes // bytes_per_K), 1), K)
        else:
            kbm = 1
        if getattr(self, "precision", "fp32") == "bf16" and 64 < kbm < K:
            kbm = kbm // 64 * 64        # whole 64-channel image boxes: no padding channels in the BF16 batches
        self.batches = [{"k_start": k0, "k_end": min(k0 + kbm, K), "K_batch": min(k0 + kbm, K) - k0}
                        for k0 in range(0, K, kbm)]
        self.K_batch_max = -(-max(b["K_batch"] for b in self.batches) // 4) * 4
        checks = [("sinogram batch (N_Omega, My, K_batch)", R * self.My * self.K_batch_max),
                  ("image batch (Nx, Ny, K_batch)", self.Nx * self.Ny * self.K_batch_max)]
        if K_batch is None:
            checks.append(("PF batch (N_Omega, K_batch, N_eta, N_rings)", R * self.K_batch_max * C * P))
        for name, n in checks:
            if n >= 2 ** 31:
                raise ValueError(f"The {name} has {n} elements, more than 2^31 - 1; lower max_gb.")
        # BF16 runs pad the channels to the 64-channel image boxes of the tensor-core forward projection
        align = 64 if getattr(self, "precision", "fp32") == "bf16" else KSTRIDE_ALIGN
        self.Kstride = -(-self.K_batch_max // align) * align
        self._alloc_batch_buffers()
        return self.batches

    def _alloc_batch_buffers(self):
        self.coeffs_sino_C = torch.empty((self.N_Omega, self.My, self.Kstride), dtype=torch.float32,
                                         device=self.device)
        self._img_k = torch.empty((self.npix, self.Kstride), dtype=torch.float32, device=self.device)

    def sparse_batch_size(self, fill):
        """Orientations per batch of the sparse modes (SPFO:1377-1397)."""
        R, CP, npix = self.N_Omega, self.N_seg, self.Nx * self.Ny
        nnz_per_k = 1.1 * fill * R * CP
        bytes_per_k = 4 * (R * self.My + 6 * npix) + 8 * R + (CAND_BYTES + NNZ_BYTES) * nnz_per_k
        kb = int(self.pf_batch_max_gb * 1024 ** 3 // bytes_per_k)
        limit = min(self.sparse_batch_max, (2 ** 31 - 1) // max(R * self.My, npix, int(nnz_per_k) + 1, R))
        return max(self.K_batch_max, min(kb, limit, -(-self.K // SPARSE_MIN_BATCHES)))

    def default_sparse_budget_gb(self):
        """Half of the free device memory after a solver's reserve (SPFO:1180-1203)."""
        coeff_bytes = 4 * self.Nx * self.Ny * self.K
        data_bytes = 4 * self.N_Omega * self.My * self.N_seg
        buffers = 4 * self.K_batch_max * (self.N_Omega * self.My + self.Nx * self.Ny)
        free, total = torch.cuda.mem_get_info(self.device)
        free = free - self.reserve_coefficient_arrays * coeff_bytes - 2 * data_bytes - buffers - 1024 ** 3
        return 0.5 * max(free, 0) / 1024 ** 3

    # ------------------------------------------------------------------ sparse PF matrix
    def _csr(self, k0, kb, fwd, rows=None, n_rows=None, row_ptr=None, out=None):
        """Count (and scan) or fill one CSR of a batch: returns (row_ptr, nnz) when counting, fills `out` (col, val)
        when row_ptr is given. rows: int32 device tensor of angle indices (None: all)."""
        n_rows = self.N_Omega if rows is None else int(rows.numel())
        n = n_rows * (self.N_seg if fwd else kb)
        rp = rows.data_ptr() if rows is not None else None
        s = self._s()
        if row_ptr is None:
            cnt = torch.empty(n + 1, dtype=torch.int32, device=self.device)
            self._call("dfx_pf_csr_count", ctypes.byref(self._pfg), rp, n_rows, k0, kb, int(fwd), cnt.data_ptr(), s)
            nb = self._lib.dfx_scan_scratch_bytes(n)
            scr = self.scratch(nb)
            self._call("dfx_scan_exclusive_i32", cnt.data_ptr(), cnt.data_ptr(), n, scr.data_ptr(), nb, s)
            return cnt, int(cnt[n].item())
        col, val = out
        self._call("dfx_pf_csr_fill", ctypes.byref(self._pfg), rp, n_rows, k0, kb, int(fwd), row_ptr.data_ptr(),
                   col.data_ptr(), val.data_ptr(), s)

    def _make_csr(self, k0, kb, fwd, rows=None):
        rp, nnz = self._csr(k0, kb, fwd, rows)
        n = max(nnz, 1)
        col = torch.empty(n, dtype=torch.int16, device=self.device)        # uint16 bit pattern
        val = torch.empty(n, dtype=torch.float32, device=self.device)
        self._csr(k0, kb, fwd, rows, row_ptr=rp, out=(col, val))
        return rp, col, val, nnz

    def _make_fblock(self, rpf, ck, vf):
        """The eta-blocked copy of a batch's stored forward CSR (dfx_pf_fblock_*): (fb_ptr, fb_k, fb_v, fb_mask);
        the forward products over it are those over the CSR bit for bit, with a staged Z column feeding four
        outputs."""
        R, P, C = self.N_Omega, self.N_peaks, self.N_eta
        s = self._s()
        n = int(self._lib.dfx_pf_fblock_rows(R, P, C))
        cnt = torch.empty(n + 1, dtype=torch.int32, device=self.device)
        mask = torch.empty(n, dtype=torch.uint8, device=self.device)
        self._call("dfx_pf_fblock_count", rpf.data_ptr(), ck.data_ptr(), R, P, C, cnt.data_ptr(), mask.data_ptr(), s)
        nb = self._lib.dfx_scan_scratch_bytes(n)
        scr = self.scratch(nb)
        self._call("dfx_scan_exclusive_i32", cnt.data_ptr(), cnt.data_ptr(), n, scr.data_ptr(), nb, s)
        total = max(int(cnt[n].item()), 1)
        fk = torch.empty(total, dtype=torch.int16, device=self.device)         # uint16 bit pattern
        fv = torch.empty((total, 4), dtype=torch.float32, device=self.device)
        self._call("dfx_pf_fblock_fill", rpf.data_ptr(), ck.data_ptr(), vf.data_ptr(), R, P, C, cnt.data_ptr(),
                   fk.data_ptr(), fv.data_ptr(), s)
        return dict(fb_ptr=cnt, fb_k=fk, fb_v=fv, fb_mask=mask)

    def _pf_forward_product(self, ib, m, sino_ptr, data, om, n_ang, kb):
        """data rows += the forward PF product of batch ib's Radon output at sino_ptr (angles om, subset m): over the
        eta-blocked copy when the batch stores it, else over the (stored or generated) forward CSR."""
        if self.pf_mode == "dense":
            if m is not None:
                raise NotImplementedError("omega subsets need pf_mode 'sparse' or 'generated'")
            self._dense_pf_product(ib, False, sino_ptr, data.data_ptr())
            return
        sb = self.sparse_batches[ib]
        s = self._s()
        om_ptr = None if om is None else om.data_ptr()
        if sb.get("fb_ptr") is not None and self.forward_lines_fastest and self.N_peaks <= 32:
            zt = self._zt_buffer()
            self._call("dfx_spmm_pf_forward_blocked_zt", sino_ptr, zt.data_ptr(), zt.numel(), sb["fb_ptr"].data_ptr(),
                       sb["fb_k"].data_ptr(), sb["fb_v"].data_ptr(), sb["fb_mask"].data_ptr(), data.data_ptr(),
                       om_ptr, n_ang, self.My, self.N_peaks, self.N_eta, self.Kstride, kb, int(self.zt_max_groups), s)
            return
        if sb.get("fb_ptr") is not None:
            self._call("dfx_spmm_pf_forward_blocked", sino_ptr, sb["fb_ptr"].data_ptr(), sb["fb_k"].data_ptr(),
                       sb["fb_v"].data_ptr(), sb["fb_mask"].data_ptr(), data.data_ptr(), om_ptr, n_ang, self.My,
                       self.N_peaks, self.N_eta, self.Kstride, kb, s)
            return
        rp, col, val, compact = self._pf_batch(ib, True, m)
        self._call("dfx_spmm_pf_forward", sino_ptr, rp.data_ptr(), col.data_ptr(), val.data_ptr(), data.data_ptr(),
                   om_ptr, n_ang, self.My, self.N_seg, self.Kstride, kb, compact, s)

    def _zt_floats(self):
        kmax = max(b["K_batch"] for b in self.batches)
        per = 0                                          # floats per angle of the widest use
        if self.forward_lines_fastest:
            per = int(self._lib.dfx_spmm_pf_forward_zt_floats(1, self.My, kmax))
        if self.adjoint_lines_fastest:
            per = max(per, int(self._lib.dfx_spmm_pf_adjoint_zt_floats(1, self.My, self.N_seg)))
        na = min(int(self.zt_max_angles), self.N_Omega, int(self.zt_max_bytes) // max(4 * per, 1))
        return max(1, na) * per

    def _zt_buffer(self):
        """The lines-fastest copy of the Radon output the blocked forward reads, or of the data rows the adjoint
        reads (zt_max_angles angles; allocated on first use)."""
        need = self._zt_floats()
        if self._zt is None or self._zt.numel() < need:
            self._zt = None
            self._zt = torch.empty(need, dtype=torch.float32, device=self.device)
        return self._zt

    def build_sparse_pf(self, mode="auto", max_fill=0.3, max_gb=None, max_fill_partial=0.1):
        """The sparse PF matrix per orientation batch (SPFO:1207-1373). The fill fraction of the first (dense-sized)
        batch sets the sparse batch size. Then, within max_gb, in the reference's order of preference:
          "both"      both CSR copies of every batch;
          "adjoint"   the adjoint CSR of every batch, the forward copy generated again in every call;
          partial     (mode "auto") the adjoint CSRs of the first batches that fit, the other batches generated in
                      every call; mode "sparse" raises MemoryError instead;
        mode "generated" stores nothing. Row pointers are always kept (4 bytes per row). A generated copy is the
        stored one bit for bit: the structure and values are pure functions of the float32 entries (dfx_pf_csr_*).
        An allocation that fails while storing (less free memory than the budget assumed) keeps half of what fitted
        in mode "auto", as the reference does."""
        t0 = time.perf_counter()
        R, CP = self.N_Omega, self.N_seg
        auto = mode == "auto"
        if mode == "dense":
            self._use_dense_pf()
            return
        if self.K_batch_max > 65535 or CP > 65535:
            if auto:
                self._use_dense_pf(f"K_batch_max = {self.K_batch_max} or N_eta * N_rings = {CP} exceeds the 16-bit "
                                   "index range")
                return
            raise ValueError(f"K_batch_max = {self.K_batch_max} or N_eta * N_rings = {CP} exceeds the 16-bit index "
                             "range of the sparse PF matrix; use pf_mode='dense' or a smaller max_gb")
        b0 = self.batches[0]
        _, nnz0 = self._csr(b0["k_start"], b0["K_batch"], False)
        fill = nnz0 / (R * b0["K_batch"] * CP)
        self.sparse_fill_first = fill
        # mode "auto" applies the dense matrix above max_fill, or above max_fill_partial when the whole sparse
        # matrix would not fit in max_gb (SPFO:1249-1263)
        if auto and fill > max_fill:
            self._use_dense_pf(f"fill fraction {100 * fill:.2f} % > {100 * max_fill:.2f} %")
            return
        if auto and fill > max_fill_partial and max_gb is not None:
            nb_est = -(-self.K // self.sparse_batch_size(fill))
            both_est = 12 * fill * R * self.K * CP + 4 * (nb_est * (R * CP + 1) + R * self.K + nb_est)
            if both_est > max_gb * 1024 ** 3:
                self._use_dense_pf(f"fill fraction {100 * fill:.2f} % > {100 * max_fill_partial:.2f} % and the "
                                   f"whole sparse matrix ({both_est / 1024 ** 3:.1f} GB) does not fit in "
                                   f"{max_gb:.1f} GB")
                return
        self.get_pf_batches_for_material(K_batch=self.sparse_batch_size(fill))
        nb = len(self.batches)
        both, adj, ptr_f, batch_adj = self.sparse_estimates(fill)
        budget = np.inf if max_gb is None else max_gb * 1024 ** 3
        if mode == "generated":
            store, n_fit = None, 0
        elif both <= budget and self._pf_forward_csr:
            store, n_fit = "both", nb
        elif adj <= budget:
            store, n_fit = "adjoint", nb
        elif not auto:
            raise MemoryError(f"Sparse PF matrix: estimated size {adj / 1024 ** 3:.1f} GB (adjoint CSR only) > "
                              f"{max_gb:.1f} GB; use pf_mode='generated' or 'auto', or raise sparse_max_gb.")
        else:                                           # the adjoint CSRs of the first batches that fit
            store, used_est, n_fit = "adjoint", nb * ptr_f, 0
            for ib in range(nb):
                used_est += batch_adj[ib]
                if used_est > budget:
                    break
                n_fit += 1
        self.sparse_batches = []
        nnz_total = 0
        stored_bytes = 0
        for ib, b in enumerate(self.batches):
            k0, kb = b["k_start"], b["K_batch"]
            sb = None
            if store is not None and ib < n_fit:
                try:
                    rpa, cj, va, nnz = self._make_csr(k0, kb, False)
                    sb = dict(row_ptr_a=rpa, col_j=cj, val_a=va, nnz=nnz)
                    if store == "both":
                        rpf, ck, vf, nnz_f = self._make_csr(k0, kb, True)
                        assert nnz_f == nnz, (nnz, nnz_f)
                        sb.update(row_ptr_f=rpf, col_k=ck, val_f=vf)
                        if self.forward_blocks:
                            sb.update(self._make_fblock(rpf, ck, vf))
                    else:
                        sb["row_ptr_f"], _ = self._csr(k0, kb, True)
                    torch.cuda.synchronize(self.device)
                except torch.cuda.OutOfMemoryError:
                    if not auto:
                        raise
                    # less free memory than the budget assumed: keep half of what fitted, generate the rest
                    sb = None
                    keep = ib // 2
                    for j in range(keep, ib):
                        self.sparse_batches[j] = self._generated_entry(j)
                    n_fit = keep
                    torch.cuda.empty_cache()
            if sb is None:
                sb = self._generated_entry(ib)
            self.sparse_batches.append(sb)
            nnz_total += sb["nnz"]
        self._gen_cap = max([sb["nnz"] for sb in self.sparse_batches
                             if not (self._stored(sb, True) and self._stored(sb, False))] or [0])
        self._gen_col = self._gen_val = None
        if self._gen_cap:
            n = max(self._gen_cap, 1)
            self._gen_col = torch.empty(n, dtype=torch.int16, device=self.device)
            self._gen_val = torch.empty(n, dtype=torch.float32, device=self.device)
        stored = [ib for ib, sb in enumerate(self.sparse_batches) if sb.get("col_j") is not None]
        for sb in self.sparse_batches:
            stored_bytes += sum(t.numel() * t.element_size() for k, t in sb.items() if torch.is_tensor(t))
        self.pf_mode = "sparse" if len(stored) == nb else "generated"
        if not stored:
            self.pf_storage = "none"
        else:
            self.pf_storage = store + (f", {len(stored)} of {nb} batches" if len(stored) < nb else "")
        self.pf_stored_bytes = stored_bytes
        self.sparse_nnz = nnz_total
        self.sparse_fill = nnz_total / (R * self.K * CP)
        self.pf_setup_s = time.perf_counter() - t0
        if self.verbose:
            print(f"Sparse PF matrix: {nnz_total} non-zeros (fill {100 * self.sparse_fill:.3f} %), {nb} batches of up "
                  f"to {self.K_batch_max}, stored: {self.pf_storage} ({stored_bytes / 1024 ** 2:.1f} MB); set up in "
                  f"{self.pf_setup_s:.2f} s")

    def _use_dense_pf(self, reason=None):
        """pf_mode "dense" (SPFO:1207-1263, 2063-2127): the float32 PF of a batch is generated in every call into a
        buffer of the dense batch size and applied by batched SGEMMs over the angles (dfx_pf_dense_products); omega
        subsets are not available, as in the reference."""
        R, CP = self.N_Omega, self.N_seg
        self.pf_mode = "dense"
        self.pf_storage = "none"
        self.sparse_batches = None
        self.sparse_nnz = None
        self._pf_dense = torch.empty((R, self.K_batch_max, CP), dtype=torch.float32, device=self.device)
        if reason is not None and self.verbose:
            print(f"Sparse PF matrix: {reason}, using the dense PF path")

    def _dense_pf_product(self, ib, adjoint, src_ptr, dst_ptr, alpha=1.0):
        """The dense-mode PF product of batch ib over all angles: the batch's float32 PF generated, then forward
        data (+)= PF^T Z or adjoint Z = alpha PF D by batched SGEMMs."""
        b = self.batches[ib]
        s = self._s()
        self._call("dfx_pf_dense", ctypes.byref(self._pfg), b["k_start"], b["K_batch"], self._pf_dense.data_ptr(), s)
        self._call("dfx_pf_dense_products", int(adjoint), self._pf_dense.data_ptr(), self.N_Omega, b["K_batch"],
                   self.N_seg, src_ptr, dst_ptr, self.My, self.Kstride, float(alpha), s)

    def sparse_estimates(self, fill):
        """Estimated bytes of the sparse PF matrix at a fill fraction, for the current batches: (both CSR copies,
        the adjoint copies only, the forward row pointers of one batch, [adjoint copy of batch ib: row pointers +
        6 bytes per non-zero]); every copy includes its row pointers (4 bytes per row)."""
        R, CP = self.N_Omega, self.N_seg
        est = [int(math.ceil(1.02 * fill * R * b["K_batch"] * CP)) + 16 for b in self.batches]
        nb = len(self.batches)
        ptr_f = 4 * (R * CP + 1)
        ptr_a = [4 * (R * b["K_batch"] + 1) for b in self.batches]
        batch_adj = [pa + 6 * n for pa, n in zip(ptr_a, est)]
        both = sum(12 * n for n in est) + nb * ptr_f + sum(ptr_a)
        return both, sum(batch_adj) + nb * ptr_f, ptr_f, batch_adj

    def _generated_entry(self, ib):
        """A batch whose CSR copies are generated in every call: its row pointers and non-zero count."""
        b = self.batches[ib]
        rpa, nnz = self._csr(b["k_start"], b["K_batch"], False)
        rpf, _ = self._csr(b["k_start"], b["K_batch"], True)
        return dict(row_ptr_a=rpa, row_ptr_f=rpf, nnz=nnz)

    @staticmethod
    def _stored(sb, forward):
        return sb.get("col_k" if forward else "col_j") is not None

    def _pf_batch(self, ib, forward, m=None):
        """(row_ptr, col, val, compact) of batch ib for the forward or adjoint product; m: subset (its rows). A copy
        that is not stored is generated into the operator's scratch (the subset's rows only, for a subset)."""
        sb = self.sparse_batches[ib]
        b = self.batches[ib]
        key = "f" if forward else "a"
        if self._stored(sb, forward):
            return sb["row_ptr_" + key], sb["col_k" if forward else "col_j"], sb["val_" + key], 0
        if m is None:
            rp, rows, compact = sb["row_ptr_" + key], None, 0
        else:
            rp, rows, compact = self._sub[m]["row_ptr"][ib][key], self._sub[m]["omegas"], 1
        self._csr(b["k_start"], b["K_batch"], forward, rows, row_ptr=rp, out=(self._gen_col, self._gen_val))
        return rp, self._gen_col, self._gen_val, compact

    # ------------------------------------------------------------------ BF16 tensor-core path
    def build_dense_bf16_pf(self, max_z_gb: float = 2.0):
        """The dense BF16 PF of all orientation batches, (N_Omega, Ktot, CPpad) with batch ib at rows ib * Kstride
        (padding rows and columns 0), and the BF16 work buffers of the tensor-core products: Z (angles, My, Ktot),
        the Radon output of all batches side by side, for up to max_z_gb of angles at a time, and D's BF16 copy.
        bf16_pf "generated" (or "auto" when the PF of all angles would take more than half of the free device memory):
        no PF of all angles is kept; every tensor-core product generates the PF of its angles (dfx_pf_dense_bf16_rows)
        into one of two buffers, which keep the last two angle lists (an SPDHG iteration's adjoint subset and next
        forward subset)."""
        R, CP = self.N_Omega, self.N_seg
        self.Ktot = len(self.batches) * self.Kstride
        self.cp_pad = -(-CP // 8) * 8
        nbytes = 2 * R * self.Ktot * self.cp_pad
        free, _ = torch.cuda.mem_get_info(self.device)
        mode = self.bf16_pf
        if mode not in ("auto", "stored", "generated"):
            raise ValueError(f"bf16_pf must be 'auto', 'stored' or 'generated', not {mode!r}")
        if mode == "auto":
            mode = "stored" if nbytes <= 0.5 * free else "generated"
        if mode == "stored" and nbytes > 0.9 * free:
            raise MemoryError(f"dense BF16 PF of {nbytes / 1024 ** 3:.1f} GB does not fit in the free device memory "
                              f"({free / 1024 ** 3:.1f} GB); use bf16_pf='generated'")
        self.bf16_pf_storage = mode
        t0 = time.perf_counter()
        per_angle = 2 * self.My * self.Ktot
        self._bf16_chunk = max(1, min(R, int(max_z_gb * 1024 ** 3 // per_angle)))
        self._pf_gen_slots = []
        if mode == "stored":
            self.pf_bf16 = torch.zeros((R, self.Ktot, self.cp_pad), dtype=torch.bfloat16, device=self.device)
            for ib, b in enumerate(self.batches):
                self._call("dfx_pf_dense_bf16", ctypes.byref(self._pfg), b["k_start"], b["K_batch"],
                           ib * self.Kstride, self.Ktot, self.cp_pad, self.pf_bf16.data_ptr(), self._s())
        else:
            self.pf_bf16 = None
            self._pf_gen_max = self._bf16_chunk
        self._d_bf16 = torch.zeros((R, self.My, self.cp_pad), dtype=torch.bfloat16, device=self.device)
        self._z_bf16 = torch.empty(0, dtype=torch.bfloat16, device=self.device)
        self._all_omegas = torch.arange(R, dtype=torch.int32, device=self.device)
        # the tensor-core backprojection covers a 16 x 8 pixel tile with a 32-bin window per angle
        g = np.abs(np.asarray(self.radon_geo.geo, np.float64))
        hw = (1.0 + np.maximum(g[:, 0], g[:, 1])) / 2.0 if self._kernel_id == 1 else np.ones(R)
        span = 15.0 * g[:, 0] + 7.0 * g[:, 1] + 2.0 * hw + 2.0
        self.tc_backprojection = bool(np.all(span <= 32.0)) and self.Kstride % 16 == 0
        # the tensor-core forward projection: 8 x 8 pixel tiles on 32-bin windows that start at a multiple of 16
        # (taps within 17 bins of the tile's first), every bin of an angle in tensor memory (My + 31 <= 512 columns)
        span_f = 7.0 * (g[:, 0] + g[:, 1]) + 2.0 * hw + 2.0
        self.tc_forward = (bool(np.all(span_f <= 17.0)) and self.Kstride % 64 == 0 and self.My + 31 <= 512
                           and self.projector == "native")
        self.pf_bf16_setup_s = time.perf_counter() - t0

    def _z(self, n):
        """The BF16 Radon output buffer for n angles, (n, My, Ktot)."""
        need = n * self.My * self.Ktot
        if self._z_bf16.numel() < need:
            # zeros: the padding channels of a batch whose columns a projection writes for its K_batch channels only
            # stay finite (they meet zero PF rows in the products)
            self._z_bf16 = torch.zeros(need, dtype=torch.bfloat16, device=self.device)
        return self._z_bf16[:need].view(n, self.My, self.Ktot)

    def _bf16_chunks(self, subset):
        """(geo, n, omegas, first) pieces of the angles of subset m (or of all angles), each at most the Z buffer's
        size; first: the piece's first position in the angle list."""
        if subset is None:
            geo, om = self.geo_gpu, self._all_omegas
        else:
            e = self._sub[self._subset(subset)]
            geo, om = e["geo"], e["omegas"]
        n = om.numel()
        c = max(self._bf16_chunk, self._max_subset()) if subset is not None else self._bf16_chunk
        return [(geo[a:a + c], min(c, n - a), om[a:a + c], a) for a in range(0, n, c)]

    def lazy_bytes(self) -> int:
        """Device memory the operator allocates on first use during a solver's iterations (the BF16 Radon output of
        the largest subset, the generated BF16 PF buffers, the Fourier-slice scratch), for callers that size their
        own arrays beforehand."""
        n = 0
        if self.precision == "bf16":
            ns = self._max_subset() if self._sub else self._bf16_chunk
            n += 2 * ns * self.My * self.Ktot
            if self.pf_bf16 is None:
                n += 2 * 2 * ns * self.Ktot * self.cp_pad
        if self.projector == "fft":
            n += int(self.fft_max_gb * 1024 ** 3)
        if self._zt is None and self.pf_mode != "dense" and (self.adjoint_lines_fastest or (
                self.forward_lines_fastest and self.sparse_batches
                and any(sb.get("fb_ptr") is not None for sb in self.sparse_batches))):
            n += 4 * self._zt_floats()
        return int(n)

    def _max_subset(self):
        return max((e["n"] for e in self._sub), default=1)

    def _radon_forward_bf16(self, src_ptr, ib, z, om, n, m=None, row0=0):
        """Radon transform of channel-fastest batch ib (float32 at src_ptr) into its columns of Z (BF16): the n angles
        om, which are subset m's, or (m None) angles row0 .. row0 + n - 1 of all. The Fourier-slice projector
        transforms every angle of the subset (or of all angles) into the float32 batch sinogram, whose rows are then
        rounded to BF16 (its padding channels are zeros)."""
        if self.projector == "fft":
            self._fft_run(True, m, src_ptr, self.coeffs_sino_C.data_ptr(), self.batches[ib]["K_batch"])
            self._call("dfx_convert_rows", 1, self.coeffs_sino_C.data_ptr() + 4 * row0 * self.My * self.Kstride,
                       self.Kstride, z.data_ptr() + 2 * ib * self.Kstride, self.Ktot, n * self.My, self.Kstride,
                       self._s())
            return
        self._radon_fwd(src_ptr, z.data_ptr() + 2 * ib * self.Kstride, om, n, self.batches[ib]["K_batch"],
                        sld=self.Ktot)

    def _pf_of(self, om, n):
        """(PF tensor, compact flag) for the tensor-core products over the n angles om: the stored PF of all angles,
        or the PF of these angles generated into one of two kept buffers (reused while the same angle list comes
        again: an iteration's adjoint and the next one's forward of the same subset)."""
        if self.pf_bf16 is not None:
            return self.pf_bf16, 0
        key = (om.data_ptr(), int(n), self._pf_version, self._sub_version)
        for slot in self._pf_gen_slots:
            if slot["key"] == key:
                return slot["pf"][:n], 1
        if n > self._pf_gen_max:
            self._pf_gen_max = n
            self._pf_gen_slots = []
        if len(self._pf_gen_slots) < 2:
            buf = torch.zeros((self._pf_gen_max, self.Ktot, self.cp_pad), dtype=torch.bfloat16, device=self.device)
            slot = {"pf": buf, "key": None}
            self._pf_gen_slots.append(slot)
        else:
            slot = self._pf_gen_slots.pop(0)                  # the older list's buffer
            self._pf_gen_slots.append(slot)
        slot["key"] = key
        for ib, b in enumerate(self.batches):
            self._call("dfx_pf_dense_bf16_rows", ctypes.byref(self._pfg), om.data_ptr(), int(n), b["k_start"],
                       b["K_batch"], ib * self.Kstride, self.Ktot, self.cp_pad, slot["pf"].data_ptr(), self._s())
        return slot["pf"][:n], 1

    def _pf_tc_forward(self, z, om, n, data, k0=0, kn=None, accumulate=0):
        """data rows om (+)= PF Z on the tensor cores (the stored PF, or the PF of these angles generated)."""
        src, compact = self._pf_of(om, n)
        self._call("dfx_pf_tc_forward", src.data_ptr(), self.Ktot, k0, self.Ktot if kn is None else kn,
                   self.N_seg, self.cp_pad, self.N_Omega, z.data_ptr(), om.data_ptr(), n, self.My, data.data_ptr(),
                   accumulate, compact, self._s())

    def _pf_tc_adjoint(self, om, n, z, k0=0, kn=None):
        """Z = alpha PF^T D for the angles om (D's BF16 copy must hold their rows); the PF as in _pf_tc_forward."""
        alpha = float(np.float32(self.N_Omega / np.pi))
        src, compact = self._pf_of(om, n)
        self._call("dfx_pf_tc_adjoint", src.data_ptr(), self.Ktot, k0, self.Ktot if kn is None else kn,
                   self.N_seg, self.cp_pad, self.N_Omega, self._d_bf16.data_ptr(), om.data_ptr(), n, self.My, alpha,
                   z.data_ptr(), compact, self._s())

    def _rows_to_bf16(self, data, om, n):
        self._call("dfx_rows_to_bf16", data.data_ptr(), self._d_bf16.data_ptr(), om.data_ptr(), n, self.My,
                   self.N_seg, self.cp_pad, self._s())

    def _direct_bf16(self, coeffs, data, subset):
        m = None if subset is None else self._subset(subset)
        for geo, n, om, a in self._bf16_chunks(subset):
            z = self._z(n)
            for ib, b in enumerate(self.batches):
                self._call("dfx_gather_channels", coeffs.data_ptr(), self._img_k.data_ptr(), self.npix, b["k_start"],
                           b["K_batch"], self.Kstride, self._s())
                self._radon_forward_bf16(self._img_k.data_ptr(), ib, z, om, n, m=m, row0=a)
            self._pf_tc_forward(z, om, n, data)

    def _adjoint_bf16(self, data, coeffs, subset):
        chunks = self._bf16_chunks(subset)
        for geo, n, om, _ in chunks:
            self._rows_to_bf16(data, om, n)
        fft = self.projector == "fft"
        for ib, b in enumerate(self.batches):
            k0, kb = ib * self.Kstride, b["K_batch"]
            for ic, (geo, n, om, a) in enumerate(chunks):
                z = self._z(n)
                self._pf_tc_adjoint(om, n, z, k0, self.Kstride)
                if fft:     # the pieces' rows widened into the float32 batch sinogram, transformed once complete
                    self._call("dfx_convert_rows", 0, self.coeffs_sino_C.data_ptr() + 4 * a * self.My * self.Kstride,
                               self.Kstride, z.data_ptr() + 2 * k0, self.Ktot, n * self.My, kb, self._s())
                    continue
                # over several angle chunks the backprojections of the chunks are summed in the batch buffer
                dst = self._img_k if ic == 0 else self._img_acc()
                self._call("dfx_radon_backward_bf16", z.data_ptr() + 2 * k0, self.Ktot, dst.data_ptr(),
                           geo.data_ptr(), n, self.Nx, self.Ny, self.My, self.Kstride, kb, self._kernel_id,
                           int(self.radon_geo.n_taps), self._s())
                if ic > 0:
                    with torch.cuda.stream(self.stream()):
                        self._img_k.add_(dst)
            if fft:
                self._fft_run(False, None if subset is None else self._subset(subset), self.coeffs_sino_C.data_ptr(),
                              self._img_k.data_ptr(), kb)
            self._call("dfx_scatter_channels", self._img_k.data_ptr(), coeffs.data_ptr(), self.npix, b["k_start"],
                       kb, self.Kstride, self._s())

    def _img_acc(self):
        if getattr(self, "_img_k2", None) is None:
            self._img_k2 = torch.empty_like(self._img_k)
        return self._img_k2

    # ---- BF16 SPDHG pass pieces (channel-fastest batches)
    def _bf16_adjoint_sino(self, data, subset):
        """Z = alpha PF^T data for the angles of subset m, all batches (one tensor-core launch); returns (geo, n, z)."""
        e = self._sub[self._subset(subset)]
        z = self._z(e["n"])
        self._rows_to_bf16(data, e["omegas"], e["n"])
        self._pf_tc_adjoint(e["omegas"], e["n"], z)
        return e["geo"], e["n"], z

    def _bf16_update_batch(self, ib, geo, n, z, x_ptr, z_ptr, T_ptr, inv_p, lam, xb_ptr=None, subset=None,
                           t_bf16=False):
        """SPDHG's update of batch ib from its columns of Z (the n angles of subset m): the backprojection with the
        primal step fused (and the BF16 copy of the new x written to xb_ptr). The Fourier-slice projector
        backprojects the columns widened to float32, and the primal step follows as its own kernel (t_bf16: T stored
        in BF16)."""
        if self.projector == "fft":
            kb, s = self.batches[ib]["K_batch"], self._s()
            self._call("dfx_convert_rows", 0, self.coeffs_sino_C.data_ptr(), self.Kstride,
                       z.data_ptr() + 2 * ib * self.Kstride, self.Ktot, n * self.My, kb, s)
            self._fft_run(False, self._subset(subset), self.coeffs_sino_C.data_ptr(), self._img_k.data_ptr(), kb)
            self._call("dfx_spdhg_primal_update_t16" if t_bf16 else "dfx_spdhg_primal_update", x_ptr, z_ptr, T_ptr,
                       self._img_k.data_ptr(), float(inv_p), float(lam), self.batch_elems(), s)
            if xb_ptr is not None:
                self._call("dfx_f32_to_bf16", x_ptr, xb_ptr, self.batch_elems(), s)
            return
        if t_bf16:
            raise ValueError("T in BF16 needs the Fourier-slice projector")
        name = "dfx_radon_backward_spdhg_tc" if self.tc_backprojection else "dfx_radon_backward_spdhg_bf16"
        self._call(name, z.data_ptr() + 2 * ib * self.Kstride, self.Ktot, geo.data_ptr(), n, self.Nx, self.Ny,
                   self.My, self.Kstride, self.batches[ib]["K_batch"], self._kernel_id, int(self.radon_geo.n_taps),
                   x_ptr, z_ptr, T_ptr, float(inv_p), float(lam), xb_ptr, self._s())

    def _bf16_forward_sino(self, subset, ib, src_ptr, src_bf16=False, ray=None, tiles=None):
        """Radon transform of batch ib (channel-fastest at src_ptr, float32 or BF16) for the angles of subset m into
        Z (ray, tiles: a support ray table and the support's tile list, for images that are zero outside the
        support)."""
        m = self._subset(subset)
        e = self._sub[m]
        if not src_bf16:
            self._radon_forward_bf16(src_ptr, ib, self._z(e["n"]), e["omegas"], e["n"], m=m)
            return
        if self.projector == "fft":
            raise ValueError("the Fourier-slice projector transforms float32 images only")
        z = self._z(e["n"])
        self._radon_bf16_image(src_ptr, z.data_ptr() + 2 * ib * self.Kstride, e["geo"], e["omegas"], e["n"],
                               self.batches[ib]["K_batch"], ray=ray, tiles=tiles)

    def _radon_bf16_image(self, src_ptr, dst_ptr, geo, om, n, kb, ray=None, tiles=None):
        """The Radon output (BF16, row stride Ktot) of a BF16 channel-fastest batch at src_ptr for the n angles om
        (geo: their geometry rows): on the tensor cores (dfx_radon_forward_tc) when the geometry admits them and
        use_tc_forward is set, else through the ray table (ray: a support table; tiles: the support's tile list; an
        image that is zero outside the support may skip the other tiles)."""
        if self.use_tc_forward and getattr(self, "tc_forward", False):
            tp, nt = (None, 0) if tiles is None else (tiles.data_ptr(), int(tiles.numel()))
            tab = self._tc_weight_table()
            if tab is not None:
                self._call("dfx_radon_forward_tc_table", src_ptr, dst_ptr, self.Ktot, 0, tab[0].data_ptr(),
                           tab[1].data_ptr(), om.data_ptr(), n, self.Nx, self.Ny, self.My, self.Kstride,
                           float(self.radon_geo.scale), tp, nt, self._s())
                return
            self._call("dfx_radon_forward_tc", src_ptr, dst_ptr, self.Ktot, 0, geo.data_ptr(), n, self.Nx, self.Ny,
                       self.My, self.Kstride, self._kernel_id, int(self.radon_geo.n_taps),
                       float(self.radon_geo.scale), tp, nt, self._s())
            return
        rp, ent = (self._ray_rp, self._ray_ent) if ray is None else ray[:2]
        self._call("dfx_radon_forward_table_bf16_bf16", src_ptr, dst_ptr, self.Ktot, rp.data_ptr(), ent.data_ptr(),
                   om.data_ptr(), n, self.My, self.Kstride, kb, float(self.radon_geo.scale), self._s())

    # the tensor-core forward reads its weight tiles from a table built once per geometry (8 KB per angle and 8 x 8
    # pixel tile) when that takes at most this fraction of the free device memory; else each CTA builds them
    tc_weight_table_max_frac = 0.1

    def _tc_weight_table(self):
        """(weights, windows) of dfx_radon_tc_weights for every angle, built on first use, or None."""
        tab = getattr(self, "_tcf_tab", None)
        if tab is not None:
            return tab or None
        R = self.N_Omega
        nb = int(self._lib.dfx_radon_tc_weights_bytes(R, self.Nx, self.Ny))
        free, _ = torch.cuda.mem_get_info(self.device)
        if nb <= 0 or nb > self.tc_weight_table_max_frac * free:
            self._tcf_tab = ()
            return None
        n_tiles = (-(-self.Nx // 8)) * (-(-self.Ny // 8))
        w = torch.empty(nb, dtype=torch.uint8, device=self.device)
        win = torch.empty(R * n_tiles, dtype=torch.int32, device=self.device)
        self._call("dfx_radon_tc_weights", self.geo_gpu.data_ptr(), R, self.Nx, self.Ny, self.My, self._kernel_id,
                   int(self.radon_geo.n_taps), w.data_ptr(), win.data_ptr(), self._s())
        self._tcf_tab = (w, win)
        return self._tcf_tab

    def support_tiles(self, supp):
        """int32 device tensor of the 8 x 8 pixel tiles (row-major over the tile grid) holding at least one pixel of
        a support mask (uint8 (Ny * Nx) device tensor); kept per mask content."""
        key = bytes(supp.cpu().numpy())
        hit = self._supp_tiles.get(key)
        if hit is None:
            m = supp.cpu().numpy().reshape(self.Ny, self.Nx).astype(bool)
            ty, tx = -(-self.Ny // 8), -(-self.Nx // 8)
            pad = np.zeros((ty * 8, tx * 8), bool)
            pad[:self.Ny, :self.Nx] = m
            any_ = pad.reshape(ty, 8, tx, 8).any(axis=(1, 3)).ravel()
            hit = torch.as_tensor(np.flatnonzero(any_).astype(np.int32), device=self.device)
            self._supp_tiles[key] = hit
        return hit

    def _bf16_forward_rows(self, subset, data):
        """data rows of subset m = PF Z over all orientations (the rows are overwritten)."""
        e = self._sub[self._subset(subset)]
        self._pf_tc_forward(self._z(e["n"]), e["omegas"], e["n"], data)

    # ------------------------------------------------------------------ omega subsets
    @on_op_stream
    def set_omega_subsets(self, subsets):
        """Subsets of the rotation angles for the subset forms direct_cl / adjoint_cl(subset=m) (SPFO:1541-1599):
        an int M (angle i in subset i % M) or a list of index arrays; returns the sorted index arrays."""
        if self.pf_mode not in ("sparse", "generated"):
            raise NotImplementedError(f"omega subsets need pf_mode 'sparse' or 'generated' (this operator: "
                                      f"{self.pf_mode!r})")
        R = self.N_Omega
        if np.isscalar(subsets):
            subsets = interleaved_subsets(R, int(subsets))
        out = []
        for s in subsets:
            s = np.unique(np.asarray(s, dtype=np.int64))
            if s.size == 0 or s[0] < 0 or s[-1] >= R:
                raise ValueError(f"every subset must hold angle indices in 0 .. {R - 1}")
            out.append(s)
        old = self.omega_subsets
        if old is not None and len(old) == len(out) and all(np.array_equal(a, b) for a, b in zip(old, out)):
            return out
        self.release_omega_subsets()
        self.omega_subsets = out
        for s in out:
            om = torch.as_tensor(s.astype(np.int32), device=self.device)
            geo = self.geo_gpu[torch.as_tensor(s, device=self.device)].contiguous()
            entry = dict(omegas=om, geo=geo, n=len(s), row_ptr=None)
            if self.projector == "fft":
                entry["fft"] = self._fft.subset(s)
            if any(not (self._stored(sb, True) and self._stored(sb, False)) for sb in self.sparse_batches):
                entry["row_ptr"] = []
                for b in self.batches:
                    rpa, nnz = self._csr(b["k_start"], b["K_batch"], False, om)
                    rpf, _ = self._csr(b["k_start"], b["K_batch"], True, om)
                    entry["row_ptr"].append({"a": rpa, "f": rpf})
            self._sub.append(entry)
        return out

    def release_omega_subsets(self):
        self._sub = []
        self.omega_subsets = None
        self._sub_version += 1          # angle lists held by the generated-PF buffers are stale now

    @property
    def _sub_omegas(self):
        return [e["omegas"] for e in self._sub]

    def _subset(self, subset):
        if self.omega_subsets is None:
            raise ValueError("no omega subsets defined: call set_omega_subsets first")
        return int(subset)

    @on_op_stream
    def zero_subset_rows(self, data, subset):
        """data rows of the angles of subset m <- 0 (SPFO:1638-1644)."""
        m = self._subset(subset)
        e = self._sub[m]
        self._call("dfx_zero_rows", data.data_ptr(), e["omegas"].data_ptr(), e["n"], self.My * self.N_seg, self._s())

    def _fill(self, t: torch.Tensor, value: float = 0.0):
        self._call("dfx_fill_f32", t.data_ptr(), float(value), t.numel(), self._s())

    # ------------------------------------------------------------------ forward / adjoint
    @on_op_stream
    def direct_cl(self, coeffs, data, subset=None):
        """In-place forward operator data = PF @ Radon(coeffs) (SPFO:1646-1662); subset=m: only the rows of the angles
        of subset m are written (the other rows are left as they are)."""
        check_device(coeffs, self.coeff_shape, "coeffs")
        check_device(data, self.data_shape, "data")
        if self.precision == "bf16":
            self._direct_bf16(coeffs, data, subset)
            return
        if subset is None:
            self._fill(data, 0.0)
        else:
            self.zero_subset_rows(data, subset)
        for ib, b in enumerate(self.batches):
            self._direct_batch(coeffs, b["k_start"], self.K, ib, data, subset)

    def _direct_batch(self, src, k_src, K_src, ib, data, subset=None):
        """Add the forward projection of batch ib to data; its coefficients are orientations k_src .. k_src+Kb-1 of
        src, a (K_src, Ny, Nx) array (SPFO:1664-1728)."""
        b = self.batches[ib]
        Kb = b["K_batch"]
        s = self._s()
        if subset is None:
            geo, n_ang, om, m = self.geo_gpu, self.N_Omega, None, None
        else:
            m = self._subset(subset)
            e = self._sub[m]
            geo, n_ang, om = e["geo"], e["n"], e["omegas"]
        self._call("dfx_gather_channels", src.data_ptr(), self._img_k.data_ptr(), self.npix, k_src, Kb, self.Kstride, s)
        self._radon_fwd(self._img_k.data_ptr(), self.coeffs_sino_C.data_ptr(), om, n_ang, Kb, m=m)
        self._pf_forward_product(ib, m, self.coeffs_sino_C.data_ptr(), data, om, n_ang, Kb)

    @on_op_stream
    def adjoint_cl(self, data, coeffs, subset=None):
        """In-place adjoint coeffs = A^T data (SPFO:1800-1817); subset=m: A_m^T (rows of subset m only)."""
        check_device(data, self.data_shape, "data")
        check_device(coeffs, self.coeff_shape, "coeffs")
        if self.precision == "bf16":
            self._adjoint_bf16(data, coeffs, subset)
            return
        for ib, b in enumerate(self.batches):
            self._adjoint_batch(data, ib, coeffs, b["k_start"], self.K, subset)

    def _adjoint_batch(self, data, ib, target, k_target, K_target, subset=None):
        """A^T data of batch ib into orientations k_target .. k_target+Kb-1 of target (SPFO:1966-2033)."""
        s = self._s()
        geo, n_ang, Kb = self._pf_adjoint_to_sino(data, ib, subset)
        m = None if subset is None else self._subset(subset)
        self._radon_bwd(self.coeffs_sino_C.data_ptr(), self._img_k.data_ptr(), geo, n_ang, Kb, m)
        self._call("dfx_scatter_channels", self._img_k.data_ptr(), target.data_ptr(), self.npix, k_target, Kb,
                   self.Kstride, s)

    # ---- channel-fastest batches: the solvers keep their coefficient state in the layout the kernels use, batch ib
    # at element offset ib * npix * Kstride of a flat array (no gather / scatter pass per iteration)
    def batch_elems(self) -> int:
        return self.npix * self.Kstride

    def _geo_of(self, subset):
        if subset is None:
            return self.geo_gpu, self.N_Omega, None, None
        m = self._subset(subset)
        e = self._sub[m]
        return e["geo"], e["n"], e["omegas"], m

    def _direct_batch_k(self, src_ptr, ib, data, subset=None, ray=None):
        """Add the forward projection of batch ib, given channel-fastest at device address src_ptr, to data (ray: a
        support ray table for images that are zero outside the support)."""
        Kb = self.batches[ib]["K_batch"]
        s = self._s()
        geo, n_ang, om, m = self._geo_of(subset)
        self._radon_fwd(src_ptr, self.coeffs_sino_C.data_ptr(), om, n_ang, Kb, ray=ray, m=m)
        self._pf_forward_product(ib, m, self.coeffs_sino_C.data_ptr(), data, om, n_ang, Kb)

    def _direct_channel_constant(self, src_ptr, kb_src, data, ray=None):
        """Add to data the forward projection, through every batch, of an image that is the same in every channel:
        src_ptr holds it channel-fastest for kb_src >= every batch's K_batch channels. Its Radon transform is computed
        once and every batch's PF product reads its own channels of it; per channel the Radon output does not depend
        on the batch (the native projector: the same taps in the same order), so data gets the bits of
        _direct_batch_k batch by batch."""
        if self.projector != "native" or kb_src < max(b["K_batch"] for b in self.batches):
            raise ValueError("_direct_channel_constant needs the native projector and the widest batch's channels")
        geo, n_ang, om, m = self._geo_of(None)
        sino = self.coeffs_sino_C.data_ptr()
        self._radon_fwd(src_ptr, sino, om, n_ang, kb_src, ray=ray, m=m)
        for ib, b in enumerate(self.batches):
            self._pf_forward_product(ib, m, sino, data, om, n_ang, b["K_batch"])

    def _pf_adjoint_to_sino(self, data, ib, subset):
        Kb = self.batches[ib]["K_batch"]
        geo, n_ang, om, m = self._geo_of(subset)
        alpha = float(np.float32(self.N_Omega / np.pi))
        if self.pf_mode == "dense":
            if m is not None:
                raise NotImplementedError("omega subsets need pf_mode 'sparse' or 'generated'")
            self._dense_pf_product(ib, True, data.data_ptr(), self.coeffs_sino_C.data_ptr(), alpha)
            return geo, n_ang, Kb
        rp, col, val, compact = self._pf_batch(ib, False, m)
        self._pf_adjoint_product(data.data_ptr(), rp, col, val, self.coeffs_sino_C.data_ptr(), om, n_ang, Kb, alpha,
                                 compact, self._s())
        return geo, n_ang, Kb

    def _pf_adjoint_product(self, data_ptr, rp, col, val, out_ptr, om, n_ang, kb, alpha, compact, s):
        """out (Radon input, n_ang x My x Kstride) = alpha PF^T data rows over the adjoint CSR (rp, col, val): through
        the lines-fastest copy of the data rows (dfx_spmm_pf_adjoint_zt) when adjoint_lines_fastest is set, else
        dfx_spmm_pf_adjoint; the same bits."""
        om_ptr = None if om is None else om.data_ptr()
        if self.adjoint_lines_fastest:
            zt = self._zt_buffer()
            self._call("dfx_spmm_pf_adjoint_zt", data_ptr, zt.data_ptr(), zt.numel(), rp.data_ptr(), col.data_ptr(),
                       val.data_ptr(), out_ptr, om_ptr, n_ang, self.My, kb, self.N_seg, self.Kstride, alpha, compact,
                       int(self.zt_max_groups), s)
            return
        self._call("dfx_spmm_pf_adjoint", data_ptr, rp.data_ptr(), col.data_ptr(), val.data_ptr(), out_ptr, om_ptr,
                   n_ang, self.My, kb, self.N_seg, self.Kstride, alpha, compact, s)

    def _adjoint_batch_k(self, data, ib, out_ptr, subset=None):
        """A^T data of batch ib into a channel-fastest batch at device address out_ptr."""
        geo, n_ang, Kb = self._pf_adjoint_to_sino(data, ib, subset)
        self._radon_bwd(self.coeffs_sino_C.data_ptr(), out_ptr, geo, n_ang, Kb,
                        None if subset is None else self._subset(subset))

    def _adjoint_update_batch(self, data, ib, subset, x_ptr, z_ptr, T_ptr, inv_p, lam):
        """SPDHG's update of batch ib: dz = A_m^T data (batch ib), z += dz, x = max(0, x - T (z + inv_p dz + lam)),
        on channel-fastest batches, the primal step fused into the backprojection."""
        geo, n_ang, Kb = self._pf_adjoint_to_sino(data, ib, subset)
        if self.projector == "fft":         # backprojection into the batch buffer, then the primal step
            self._radon_bwd(self.coeffs_sino_C.data_ptr(), self._img_k.data_ptr(), geo, n_ang, Kb,
                            None if subset is None else self._subset(subset))
            self._call("dfx_spdhg_primal_update", x_ptr, z_ptr, T_ptr, self._img_k.data_ptr(), float(inv_p),
                       float(lam), self.batch_elems(), self._s())
            return
        self._call("dfx_radon_backward_spdhg", self.coeffs_sino_C.data_ptr(), geo.data_ptr(), n_ang, self.Nx,
                   self.Ny, self.My, self.Kstride, Kb, self._kernel_id, int(self.radon_geo.n_taps), x_ptr, z_ptr,
                   T_ptr, float(inv_p), float(lam), self._s())

    def to_batches(self, coeffs, out_k, stream=None):
        """coeffs (K, Ny, Nx) -> channel-fastest batches (flat, batch ib at ib * npix * Kstride; on stream, default
        the operator's)."""
        s = self._s() if stream is None else _stream_handle(stream)
        for ib, b in enumerate(self.batches):
            self._call("dfx_gather_channels", coeffs.data_ptr(), out_k.data_ptr() + 4 * ib * self.batch_elems(),
                       self.npix, b["k_start"], b["K_batch"], self.Kstride, s)

    def from_batches(self, in_k, coeffs, stream=None):
        """Channel-fastest batches -> coeffs (K, Ny, Nx) (on stream, default the operator's)."""
        s = self._s() if stream is None else _stream_handle(stream)
        for ib, b in enumerate(self.batches):
            self._call("dfx_scatter_channels", in_k.data_ptr() + 4 * ib * self.batch_elems(), coeffs.data_ptr(),
                       self.npix, b["k_start"], b["K_batch"], self.Kstride, s)

    @on_op_stream
    def adjoint_batches_cl(self, data, out_batch, update):
        """The adjoint one batch at a time into the first Kb * Ny * Nx elements of out_batch, then update(k0, Kb)
        (SPFO:1819-1838)."""
        check_device(data, self.data_shape, "data")
        assert out_batch.dtype == torch.float32 and out_batch.numel() >= self.npix * self.K_batch_max
        for ib, b in enumerate(self.batches):
            self._adjoint_batch(data, ib, out_batch, 0, self.K_batch_max)
            update(b["k_start"], b["K_batch"])

    @on_op_stream
    def adjoint_multi_cl(self, datas, consume, row_masks=(None,), batch_done=None, pixels=None, nrhs=4,
                         rows_per_group=12):
        """Several adjoints in one pass over the orientation batches, sharing each batch's PF matrix (SPFO:1840-1964).

        For every batch the PF matrix is made once (stored, or generated once) and its transpose applied to every
        array of ``datas`` for the rows of every entry of ``row_masks`` (None: all rows, else an (N_Omega,) bool array
        of the rows that count); each product is back-projected over those rows and handed to
        ``consume(i, s, k0, Kb, block)`` (data array i, row mask s); ``batch_done(k0, Kb)`` follows every batch.

        pixels None: block = the batch image, a (Nx*Ny, Kstride) view of the operator's batch buffer (block[p, k],
        pixel p = x + Nx*y; columns k < Kb valid). pixels = (npix,) flat pixel indices: only these pixels are
        back-projected, block = (K_batch_max, npix) orientation-major (rows k < Kb valid). Blocks are overwritten by
        later calls of consume. The values are those adjoint_cl gives for datas[i] with the rows outside mask s set to
        zero, bitwise: the product of an angle row depends on that row only, and the skipped rows would add exact
        zeros to the backprojection. nrhs: data arrays per group of blocks (each group member keeps its own blocks
        while the group is consumed); rows_per_group is accepted (a launch-shape option of the reference).

        Needs pf_mode "sparse" or "generated" and the native projector."""
        if self.pf_mode not in ("sparse", "generated") or self.projector != "native":
            raise NotImplementedError("adjoint_multi_cl needs pf_mode 'sparse' or 'generated' and the native projector")
        for d in datas:
            check_device(d, self.data_shape, "data")
        R = self.N_Omega
        sets = []
        for m in row_masks:
            if m is None:
                sets.append((None, self.geo_gpu, R))
                continue
            m = np.asarray(m, dtype=bool).reshape(-1)
            if m.size != R:
                raise ValueError(f"a row mask needs {R} entries (one per rotation angle), not {m.size}")
            rows = np.nonzero(m)[0]
            sets.append((torch.as_tensor(rows.astype(np.int32), device=self.device),
                         self.geo_gpu[torch.as_tensor(rows, device=self.device)].contiguous(), len(rows)))
        nrhs = max(1, min(int(nrhs), len(datas))) if datas else 1
        s = self._s()
        alpha = float(np.float32(self.N_Omega / np.pi))
        Kmax, npix_img = self.K_batch_max, self.npix
        if pixels is not None:
            pix_h = np.asarray(pixels, dtype=np.int64).reshape(-1)
            if pix_h.size == 0 or pix_h.min() < 0 or pix_h.max() >= npix_img:
                raise ValueError(f"pixels must be flat indices in 0 .. {npix_img - 1}")
            pix = torch.as_tensor(pix_h.astype(np.int32), device=self.device)
            npl = int(pix_h.size)
            tmp = torch.empty(npl * self.Kstride, dtype=torch.float32, device=self.device)
            blocks = [[torch.empty((Kmax, npl), dtype=torch.float32, device=self.device) for _ in sets]
                      for _ in range(nrhs)]
        image = self._img_k.view(npix_img, self.Kstride)
        for ib, b in enumerate(self.batches):
            k0, Kb = b["k_start"], b["K_batch"]
            rp, col, val, compact = self._pf_batch(ib, False, None)       # once for every data array and mask
            for g0 in range(0, len(datas), nrhs):
                for n, i in enumerate(range(g0, min(g0 + nrhs, len(datas)))):
                    for si, (om, geo, n_ang) in enumerate(sets):
                        if n_ang == 0:              # no rows count: the adjoint is zero
                            blk = blocks[n][si] if pixels is not None else image
                            self._fill(blk, 0.0)
                            consume(i, si, k0, Kb, blk)
                            continue
                        self._pf_adjoint_product(datas[i].data_ptr(), rp, col, val, self.coeffs_sino_C.data_ptr(), om,
                                                 n_ang, Kb, alpha, compact, s)
                        if pixels is None:
                            self._call("dfx_radon_backward", self.coeffs_sino_C.data_ptr(), self._img_k.data_ptr(),
                                       geo.data_ptr(), n_ang, self.Nx, self.Ny, self.My, self.Kstride, Kb,
                                       self._kernel_id, int(self.radon_geo.n_taps), s)
                            consume(i, si, k0, Kb, image)
                        else:
                            self._call("dfx_radon_backward_pixels", self.coeffs_sino_C.data_ptr(), tmp.data_ptr(),
                                       geo.data_ptr(), n_ang, self.Nx, self.Ny, self.My, self.Kstride, Kb,
                                       self._kernel_id, int(self.radon_geo.n_taps), pix.data_ptr(), npl, s)
                            self._call("dfx_scatter_channels", tmp.data_ptr(), blocks[n][si].data_ptr(), npl, 0, Kb,
                                       self.Kstride, s)
                            consume(i, si, k0, Kb, blocks[n][si])
            if batch_done is not None:
                batch_done(k0, Kb)

    @on_op_stream
    def direct(self, coeffs):
        """Forward operator allocating its output: a CUDA tensor for a CUDA tensor; for a NumPy array (K, Ny, Nx) the
        coefficients are streamed to the GPU batch by batch and a NumPy array is returned (SPFO:1107-1127)."""
        if is_device(coeffs):
            data = torch.empty(self.data_shape, dtype=torch.float32, device=self.device)
            self.direct_cl(coeffs, data)
            return data
        x = as_host(coeffs, self.coeff_shape, "coeffs")
        data = torch.empty(self.data_shape, dtype=torch.float32, device=self.device)
        from .streaming import streamer_for
        streamer_for(self).forward(x.reshape(-1), data)
        return data.cpu().numpy()

    @on_op_stream
    def adjoint(self, data):
        """Adjoint allocating its output (SPFO:1777-1796): CUDA tensor in, CUDA tensor out; NumPy in, NumPy out with
        the coefficients streamed to the host batch by batch."""
        if is_device(data):
            coeffs = torch.empty(self.coeff_shape, dtype=torch.float32, device=self.device)
            self.adjoint_cl(data, coeffs)
            return coeffs
        d = torch.as_tensor(as_host(data, self.data_shape, "data"), device=self.device)
        out = np.empty(self.coeff_shape, np.float32)
        from .streaming import streamer_for
        streamer_for(self).adjoint_to_host(d, out.reshape(-1))
        return out

    # ------------------------------------------------------------------ memory
    def device_bytes(self):
        """Device memory held by the operator (batch buffers, sparse PF matrix, geometry)."""
        n = 0
        for t in (self.coeffs_sino_C, self._img_k, self.coords_gpu, self.poles_gpu, self._scratch):
            n += t.numel() * t.element_size()
        for sb in self.sparse_batches or []:
            n += sum(v.numel() * v.element_size() for v in sb.values() if isinstance(v, torch.Tensor))
        for t in (getattr(self, "_gen_col", None), getattr(self, "_gen_val", None), self.pf_bf16,
                  getattr(self, "_d_bf16", None), getattr(self, "_z_bf16", None), getattr(self, "_img_k2", None),
                  getattr(self, "_pf_dense", None)):
            if t is not None:
                n += t.numel() * t.element_size()
        return n

    def release_streamer(self):
        if self._streamer is not None:
            self._streamer.release()
            self._streamer = None

    @on_op_stream
    def free_memory(self):
        """Release the operator's device buffers (SPFO:957-1020)."""
        self.release_omega_subsets()
        self.release_streamer()
        self._ray_supp = {}
        self._ray_grp = None
        self._tcf_tab = None
        self._supp_tiles = {}
        self._fft = None
        self.sparse_batches = None
        self.coeffs_sino_C = self._img_k = None
        self._gen_col = self._gen_val = None
        self._pf_dense = None
        self.pf_bf16 = self._d_bf16 = self._z_bf16 = self._img_k2 = None
        self._scratch = torch.empty(0, dtype=torch.uint8, device=self.device)
        self._zt = None
        self.stream().synchronize()          # this operator's work only (other streams keep running)


def estimate_L_power(op, niter: int = 20, seed: int = 0, eps: float = 1e-30, verbose: int = 1) -> float:
    """Lipschitz constant ||A^T A|| by power iteration (SPFO:2136-2206); the start vector is the reference's
    (a standard normal (Nx, Ny, K) draw stored pixel-fastest; a draw of the coefficient shape for a local-basis
    operator) and the dot products are float64 (dfx_dot_f64)."""
    with stream_scope(op):
        return _estimate_L_power(op, niter, seed, eps, verbose)


def _estimate_L_power(op, niter, seed, eps, verbose):
    if niter < 1:
        raise ValueError("niter must be >= 1")
    rng = np.random.default_rng(seed)
    if getattr(op, "coefficient_layout", "dense") == "dense":
        x_host = np.ascontiguousarray(rng.standard_normal((op.Nx, op.Ny, op.K)).astype(np.float32).transpose(2, 1, 0))
    else:                                       # flat coefficients (local basis): drawn in their own shape
        x_host = rng.standard_normal(tuple(op.coeff_shape)).astype(np.float32)
    x = torch.as_tensor(x_host, device=op.device)
    Ax = torch.empty(op.data_shape, dtype=torch.float32, device=op.device)
    z = torch.empty(op.coeff_shape, dtype=torch.float32, device=op.device)
    out = torch.zeros(1, dtype=torch.float64, device=op.device)
    lib = op._lib

    def dot(a, b=None):
        nb = lib.dfx_reduce_scratch_bytes(a.numel())
        scr = op.scratch(nb)
        _lib.call("dfx_dot_f64", a.data_ptr(), None if b is None else b.data_ptr(), a.numel(), out.data_ptr(),
                  scr.data_ptr(), nb, op._s())
        return float(out.item())

    x.mul_(float(np.float32(1.0 / (np.sqrt(dot(x, x)) + eps))))
    L_est = 0.0
    for it in range(niter):
        op.direct_cl(x, Ax)
        op.adjoint_cl(Ax, z)
        L_est = dot(x, z) / (dot(x, x) + eps)
        zn = np.sqrt(dot(z, z)) + eps
        z.mul_(float(np.float32(1.0 / zn)))
        x, z = z, x
        if verbose:
            print(f"[power {it + 1:02d}] L_est={L_est:.6e}  ||z||={zn:.6e}")
    return float(L_est)


def _host_dot(a, b, pool, chunk=1 << 24):
    """float64 dot product of two float32 host vectors, chunk by chunk, the chunks' sums added in order."""
    parts = [(i, min(i + chunk, a.size)) for i in range(0, a.size, chunk)]
    return float(sum(pool.map(lambda c: float(np.dot(a[c[0]:c[1]].astype(np.float64), b[c[0]:c[1]])), parts)))


def parallel_random_start(K, Ny, Nx, seed, threads=16):
    """The parallel random start of estimate_L_power_streamed (streaming.py:363-372): x3 (K, Ny, Nx) float32 with column
    ix (x3[:, :, ix]) the transposed (Ny, K) standard-normal draw of default_rng([seed, ix])."""
    from concurrent.futures import ThreadPoolExecutor
    x3 = np.empty((K, Ny, Nx), np.float32)

    def col(ix):
        x3[:, :, ix] = np.random.default_rng([seed, ix]).standard_normal((Ny, K)).astype(np.float32).T

    with ThreadPoolExecutor(threads) as p:
        list(p.map(col, range(Nx)))
    return x3


def estimate_L_power_streamed(op, niter: int = 20, seed: int = 0, eps: float = 1e-30, verbose: int = 1,
                              parallel_start: bool = True) -> float:
    """estimate_L_power with the two coefficient-sized vectors in host memory (streaming.py:398-432): the forward and
    adjoint stream them through the device batch by batch (the operator's NumPy path), the dot products are float64
    on the host. parallel_start (default): a column of the start from its own random stream (parallel_random_start),
    fast, but not the numbers of estimate_L_power; False: the start of estimate_L_power, and its estimate (computed on
    the device). Local-basis operators: estimate_L_power."""
    if getattr(op, "coefficient_layout", "dense") != "dense" or not parallel_start:
        return estimate_L_power(op, niter=niter, seed=seed, eps=eps, verbose=verbose)
    if niter < 1:
        raise ValueError("niter must be >= 1")
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(16) as pool:
        x = parallel_random_start(op.K, op.Ny, op.Nx, seed).reshape(-1)
        x *= np.float32(1.0 / (np.sqrt(_host_dot(x, x, pool)) + eps))
        L_est = 0.0
        for it in range(niter):
            z = np.ascontiguousarray(op.adjoint(op.direct(x.reshape(op.coeff_shape))), np.float32).reshape(-1)
            L_est = _host_dot(x, z, pool) / (_host_dot(x, x, pool) + eps)
            zn = float(np.sqrt(_host_dot(z, z, pool))) + eps
            z *= np.float32(1.0 / zn)
            x = z
            if verbose:
                print(f"[power {it + 1:02d}] L_est={L_est:.6e}  ||z||={zn:.6e}")
    return float(L_est)
