/*
 * diffractom_b200 — C ABI of the sm_100a kernels of diffractom's reconstruction hot path.
 *
 * Every entry point enqueues work on the CUDA stream it is given (a cudaStream_t passed as void *, NULL = the legacy
 * default stream) and returns at once; it allocates nothing: buffers, including scratch, are passed in by the caller
 * (sizes from the *_scratch_bytes queries). Device pointers are plain CUDA device addresses. Layouts follow the
 * reference: coefficients (K, Ny, Nx) float32 C order, data (N_Omega, My, N_eta * N_rings) with segment
 * j = eta_bin * N_rings + ring, channel-fastest batch buffers img_k (Nx * Ny, Kstride) and sino_k (angles, My, Kstride).
 *
 * Return value: DFX_OK, or an error code; dfx_last_error() then describes it (per host thread). No C++ exception
 * crosses this interface.
 *
 * Each declaration names the reference code it replaces (file:line within msaca-okse/diffractom, src/diffractom/
 * abbreviated): OpenCL kernels launched through pyopencl, which are the reference's only "foreign" interface on this
 * path; the Python methods that launch them are mirrored by the package diffractom_b200 on top of this ABI.
 */
#ifndef DIFFRACTOM_B200_H
#define DIFFRACTOM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DFX_OK 0
#define DFX_EINVAL 1     /* bad argument (size, alignment, null pointer, out-of-range option) */
#define DFX_ENOMEM 2     /* scratch too small */
#define DFX_ELAUNCH 3    /* a kernel launch failed */
#define DFX_ETIMEOUT 4   /* a bounded device-side wait ran out */
#define DFX_ECUDA 5      /* another CUDA runtime error */

#define DFX_ABI_VERSION 1

int dfx_abi_version(void);
const char *dfx_last_error(void);
/* Number of kernels this library has launched since it was loaded (all host threads); no reference counterpart
 * (instrumentation for benchmarks). */
uint64_t dfx_launch_count(void);

/* ---------------------------------------------------------------- parallel-beam Radon transform
 * geo: (n_angles, 4) float32 device array (X, Y, T0, angle weight), operators/parallel_radon.py:106-124.
 * kernel: 0 hat, 1 trapezoid (pixel footprint). Channels k < kb of kstride are computed, kstride % 8 == 0,
 * channels kb .. kstride-1 of the output are written as 0. */

/* replaces gather_channels_k_fastest (operators/radon_kernels.cl:222-244; ParallelRadon.gather, parallel_radon.py:221-229):
 * img_k[p, k] = coeffs[k0 + k, p] for k < kb, 0 for kb <= k < kstride. */
int dfx_gather_channels(const float *coeffs, float *img_k, int64_t npix, int k0, int kb, int kstride, void *stream);

/* replaces scatter_channels_k_fastest (radon_kernels.cl:192-215; ParallelRadon.scatter, parallel_radon.py:231-236):
 * coeffs[k0 + k, p] = img_k[p, k] for k < kb. */
int dfx_scatter_channels(const float *img_k, float *coeffs, int64_t npix, int k0, int kb, int kstride, void *stream);

/* replaces radon_forward_k / radon_forward_tiled (radon_kernels.cl:44-101, 262-372; ParallelRadon.forward,
 * parallel_radon.py:283-301): sino_k[a, s, k] = scale * sum_pixels K(t_a(pixel) - s) img_k[pixel, k]. */
int dfx_radon_forward(const float *img_k, float *sino_k, const float *geo, int n_angles, int nx, int ny, int n_det,
                      int kstride, int kb, int kernel, float scale, void *stream);

/* replaces radon_backward_k / radon_backward_tiled (radon_kernels.cl:106-141, 378-449; ParallelRadon.backward,
 * parallel_radon.py:303-318): img_k[pixel, k] = sum_a w_a sum_s K(t_a(pixel) - s) sino_k[a, s, k], pixel-driven, no
 * atomics. n_taps: the most bins a pixel touches (ParallelRadon.n_taps). */
int dfx_radon_backward(const float *sino_k, float *img_k, const float *geo, int n_angles, int nx, int ny, int n_det,
                       int kstride, int kb, int kernel, int n_taps, void *stream);
/* dfx_radon_backward for the pixels pixels[0 .. n_pix-1] (flat indices x + nx y, each checked by the caller to lie in
 * the image) only: img_k row r (n_pix rows of kstride) = the backprojection at pixel pixels[r], the same arithmetic
 * as the whole-image call (replaces ParallelRadon.backward_list, operators/parallel_radon.py:320-340, used by
 * adjoint_multi_cl with pixels, SPFO:1840-1964). */
int dfx_radon_backward_pixels(const float *sino_k, float *img_k, const float *geo, int n_angles, int nx, int ny,
                              int n_det, int kstride, int kb, int kernel, int n_taps, const int32_t *pixels,
                              int64_t n_pix, void *stream);

/* replaces, in one kernel, radon_backward_k + scatter_channels_k_fastest + spdhg_update (radon_kernels.cl:106-141,
 * 192-215; spdhg_poisson.py:95-106) for the fused SPDHG pass (spdhg_poisson.py:430-484): the backprojection dz of
 * sino_k is applied to channel-fastest coefficient batches x_k, z_k, T_k (npix, kstride):
 * z += dz; x = T > 0 ? max(0, x - T (z + inv_p dz + lam)) : 0 (dz = 0 on padding channels kb .. kstride-1). */
int dfx_radon_backward_spdhg(const float *sino_k, const float *geo, int n_angles, int nx, int ny, int n_det,
                             int kstride, int kb, int kernel, int n_taps, float *x_k, float *z_k, const float *T_k,
                             float inv_p, float lam, void *stream);

/* The three Radon entry points above for the BF16 precision path: the sinogram is BF16 with sino_ld elements between
 * consecutive bins (sino_ld >= kstride, a multiple of 8: the batches of all orientations side by side, the layout of
 * the Z operand of dfx_pf_tc_forward / dfx_pf_tc_adjoint). The forward accumulates in float32 and rounds to BF16 on
 * store; the backward widens BF16 exactly and accumulates in float32. Same references as above. */
int dfx_radon_forward_bf16(const float *img_k, void *sino_bf16, int64_t sino_ld, const float *geo, int n_angles,
                           int nx, int ny, int n_det, int kstride, int kb, int kernel, float scale, void *stream);
int dfx_radon_backward_bf16(const void *sino_bf16, int64_t sino_ld, float *img_k, const float *geo, int n_angles,
                            int nx, int ny, int n_det, int kstride, int kb, int kernel, int n_taps, void *stream);
/* x_bf16 (or NULL): also writes the new x rounded to BF16 there (same layout as x_k), the input of
 * dfx_radon_forward_table_bf16_bf16 for the next forward projection. */
int dfx_radon_backward_spdhg_bf16(const void *sino_bf16, int64_t sino_ld, const float *geo, int n_angles, int nx,
                                  int ny, int n_det, int kstride, int kb, int kernel, int n_taps, float *x_k,
                                  float *z_k, const float *T_k, float inv_p, float lam, void *x_bf16, void *stream);

/* dfx_radon_backward_spdhg_bf16 on the tensor cores (same arguments, same references; kstride a multiple of 16):
 * per 16 x 8 pixel tile and angle, the tap weights on a 32-bin window (float32 weights as BF16 hi + lo) times the
 * window's BF16 rows, float32 accumulation in tensor memory; the primal step as in the SIMT kernel. The geometry must
 * keep a tile within the window: |X| * 15 + |Y| * 7 + 2 hw + 2 <= 32 for every angle (X, Y the first two columns of
 * geo, hw the footprint half width, 1 for the hat); taps outside it are skipped and flagged (DFX_TC_WINDOW). */
int dfx_radon_backward_spdhg_tc(const void *sino_bf16, int64_t sino_ld, const float *geo, int n_angles, int nx,
                                int ny, int n_det, int kstride, int kb, int kernel, int n_taps, float *x_k, float *z_k,
                                const float *T_k, float inv_p, float lam, void *x_bf16, void *stream);

/* Ray table of a projector geometry (no reference counterpart: the reference evaluates the taps in every call): the
 * non-zero taps of every (angle a, bin s), row a * n_det + s, as int32 pairs (pixel index, float32 weight bits) in
 * the order the forward projection sums them. count: counts[row] = taps of the row (row_ptr = exclusive scan, at
 * most 2^31 - 1 in total); fill: entries (2 int32 per tap, 8-byte aligned) at row_ptr[row] .. row_ptr[row + 1].
 * supp (NULL: all pixels): one byte per pixel (index x + nx y); only the taps of pixels with supp != 0 are listed, so
 * that the forward of an image that is zero outside the support skips terms that are exactly zero. */
int dfx_radon_table_count(const float *geo, int n_angles, int nx, int ny, int n_det, int kernel, const uint8_t *supp,
                          int32_t *counts, void *stream);
int dfx_radon_table_fill(const float *geo, int n_angles, int nx, int ny, int n_det, int kernel, const uint8_t *supp,
                         const int32_t *row_ptr, int32_t *entries, void *stream);
/* dfx_radon_forward / dfx_radon_forward_bf16 through the ray table (same references): angle a of the launch is row
 * block angles[a] of the table (angles NULL: a); the same taps, weights and summation order, hence the same bits. */
int dfx_radon_forward_table(const float *img_k, float *sino_k, const int32_t *row_ptr, const int32_t *entries,
                            const int32_t *angles, int n_angles, int n_det, int kstride, int kb, float scale,
                            void *stream);
int dfx_radon_forward_table_bf16(const float *img_k, void *sino_bf16, int64_t sino_ld, const int32_t *row_ptr,
                                 const int32_t *entries, const int32_t *angles, int n_angles, int n_det, int kstride,
                                 int kb, float scale, void *stream);
/* The same with a BF16 image batch (the BF16 copy of the coefficients), widened exactly; float32 sums. */
int dfx_radon_forward_table_bf16_bf16(const void *img_bf16, void *sino_bf16, int64_t sino_ld, const int32_t *row_ptr,
                                      const int32_t *entries, const int32_t *angles, int n_angles, int n_det,
                                      int kstride, int kb, float scale, void *stream);

/* Grouped ray table (no reference counterpart): row a * ceil(n_det / 4) + g lists, in the per-bin rows' order, every
 * pixel that reaches one of the bins 4 g .. 4 g + 3 of angle a, as an int32 pixel index and a float4 of its weights
 * on those four bins (0 where the per-bin row has no entry; 16-byte aligned); count / fill / supp as for the per-bin
 * table. dfx_radon_forward_gtable: dfx_radon_forward_table over it (float32 sinogram rows of stride kstride): each
 * pixel's channels are loaded once per group of four bins, and each bin sums its per-bin row's taps in the same
 * order, so the result is dfx_radon_forward_table's, bit for bit. */
int dfx_radon_gtable_count(const float *geo, int n_angles, int nx, int ny, int n_det, int kernel, const uint8_t *supp,
                           int32_t *counts, void *stream);
int dfx_radon_gtable_fill(const float *geo, int n_angles, int nx, int ny, int n_det, int kernel, const uint8_t *supp,
                          const int32_t *row_ptr, int32_t *pixels, float *weights, void *stream);
int dfx_radon_forward_gtable(const float *img_k, float *sino_k, const int32_t *row_ptr, const int32_t *pixels,
                             const float *weights, const int32_t *angles, int n_angles, int n_det, int kstride,
                             int kb, float scale, void *stream);

/* replaces support_ones / project_support / tmin (fista_poisson.py:256-263, 277-281; spdhg_poisson.py:259-265) on a
 * channel-fastest batch (npix, kstride) with padding channels kb .. kstride-1 (supp (npix) uint8 or NULL):
 * mode 0: x = 1 on live channels of support pixels, else 0; mode 1: x = 0 outside them or where negative;
 * mode 2: x = min(x, c / colsum) on live channels of support pixels where colsum > 0; mode 3: x = 0 outside them
 * (apply_support, prox.py:75-99). */
int dfx_batch_support(float *x_k, const float *colsum_k, const uint8_t *supp, int64_t npix, int kstride, int kb,
                      float c, int mode, void *stream);

/* ---------------------------------------------------------------- pole-figure matrix
 * The PF entry of (angle r, orientation k, eta bin c, ring p) is pf_entry of operators/pf_generate.cl:62-140
 * (== pfmatrix_eval_poles, operators/create_pfo_matrix.py:108-199), times the ring intensity unless normalized. */
typedef struct dfx_pf_geometry {
    const float *coords;       /* (R, S, C, S_eta, P, 3) probed directions */
    const float *poles;        /* (K, A, 3) pole axes rotated by every orientation */
    const int32_t *axis_start; /* (P + 1) */
    const float *axis_count;   /* (A) */
    const float *inv_sigma2;   /* (K) */
    const float *norm;         /* (K) 1 / (8 pi sigma^2) */
    const float *quad_w;       /* (S * S_eta) product weights, NULL: the midpoint rule (mean over the nodes) */
    const float *intens;       /* (P) ring intensities, NULL: normalized (every ring weight 1) */
    int32_t R, C, P, A, S, S_eta, K;
    float cut;                 /* exponent at which the Gaussian is cut (pf_cutoff_sigma^2 / 2) */
    /* reflection_two_theta (SPFO:581-591, pf_generate.cl:37-43, 82-100), all NULL otherwise: every pole axis has its
     * own Bragg angle theta_a; coords then holds u (R, S, C, S_eta, 3), without the ring index, and the entry uses
     * v = cos(theta_a) u - sin(theta_a) w. */
    const float *axis_w;       /* (R * S, 3) the rotated p0 */
    const float *axis_sin;     /* (A) sin(theta_a) */
    const float *axis_cos;     /* (A) cos(theta_a) */
    /* window_parallax (SPFO:704-734, pf_generate.cl:45-57, 103-121), wp_ax NULL otherwise: every axis's weight times
     * the fraction of its radial profile inside its channel's window at the parallax-shifted angle, for the
     * orientation's mean depth at this rotation angle (a Gaussian of variance sigma^2 + (sin 2t cos 2t / D)^2 var(x),
     * optionally a pseudo-Voigt with Lorentzian share wp_eta). */
    const float *wp_pos;       /* (K, 2) mean (col, row) position relative to the rotation axis, translation steps */
    const float *wp_cov;       /* (K, 4) covariance (cc, cr, rr, 0), steps^2 */
    const float *wp_b;         /* (R, 2) the beam direction in the image plane per angle */
    const float *wp_ax;        /* (A, 4) (2 theta, sin 2t cos 2t, sigma^2, Lorentzian half width) per axis */
    const float *wp_ch;        /* (P, 2) the windows' (lo, hi) two-theta */
    float wp_invD, wp_eta;     /* 1 / sample-detector distance (steps), Lorentzian share */
} dfx_pf_geometry;

/* replaces pfmatrix_eval_poles + SCALE_PF_BY_INTENSITY_INPLACE (create_pfo_matrix.py:108-199, pf_kernels.cl:450-465;
 * SPFO:1130-1164): dense batch out (R, kb, C, P) of orientations k0 .. k0+kb-1. */
int dfx_pf_dense(const dfx_pf_geometry *g, int k0, int kb, float *out, void *stream);

/* Sparse PF of a batch of orientations k0 .. k0+kb-1, restricted to the angles rows[0 .. n_rows-1] (rows NULL: all R
 * angles). Replaces the generator pf_gen_* (pf_generate.cl:146-377, pf_generate.py:218-303) and the dense-batch CSR
 * build pf_count_rows_* / pf_fill_rows_* (pf_kernels.cl:482-548): the CSR is the one of the dense batch, bit for bit
 * in its structure.
 *   forward_rows = 0: adjoint rows (s, k) = s * kb + k listing eta/ring segments j ascending (col: j)
 *   forward_rows = 1: forward rows (s, j) = s * C * P + j listing orientations k ascending (col: k)
 * count: counts[row] = non-zeros of the row (row_ptr = exclusive scan of counts, dfx_scan_exclusive_i32);
 * fill:  col (uint16) and val at row_ptr[row] .. row_ptr[row + 1]. */
int dfx_pf_csr_count(const dfx_pf_geometry *g, const int32_t *rows, int n_rows, int k0, int kb, int forward_rows,
                     int32_t *counts, void *stream);
int dfx_pf_csr_fill(const dfx_pf_geometry *g, const int32_t *rows, int n_rows, int k0, int kb, int forward_rows,
                    const int32_t *row_ptr, uint16_t *col, float *val, void *stream);

/* Exclusive prefix sum of n int32 (out may alias in), replaces pyopencl's ExclusiveScanKernel (pf_generate.py:69):
 * out[0] = 0, out[i] = in[0] + ... + in[i - 1] for i <= n (out has n + 1 entries; in is read for i < n). */
size_t dfx_scan_scratch_bytes(int64_t n);
int dfx_scan_exclusive_i32(const int32_t *in, int32_t *out, int64_t n, void *scratch, size_t scratch_bytes,
                           void *stream);

/* The same exclusive scan for callers that cannot allocate device memory; it has no counterpart in the reference.
 * Some callers own every byte of the GPU through their own pool or budget and may not call cudaMalloc (a host
 * application that hands this library fixed buffers, or a loop that must not synchronise the device on an
 * allocation); they cannot provide dfx_scan_exclusive_i32's scratch. This entry point takes inputs and outputs only:
 * its scratch (one int32 per 2048 elements) is a fixed array inside the library, present on every GPU that loads it
 * until the process exits (256 KiB per device). Limits and rules:
 *   n <= DFX_SCAN_STATIC_MAX_N, else DFX_EINVAL with a message (the other entry point has no such limit);
 *   every call looks up the array's address in the calling thread's current context (nothing is cached, so a
 *   context that was reset and made again is handled); the first lookup on a device may load the library's module
 *   there, so make the first call on each device before any stream capture;
 *   all calls on a device share the array: calls that overlap on the GPU (other streams, other threads) race and
 *   corrupt each other's result; serialise them. Nothing has to be cleared between calls (each call writes every
 *   slot it later reads). */
#define DFX_SCAN_STATIC_MAX_N (65536LL * 2048LL)
int dfx_scan_exclusive_i32_static(const int32_t *in, int32_t *out, int64_t n, void *stream);

/* replaces spmm_pf_forward_c / spmm_pf_forward_sub (pf_kernels.cl:597-641, SPFO:38-80): for the n_sub angles
 * omegas (NULL: all, n_sub = R): data[omegas[s], y, j] += sum_k val * sino[s, y, k] over the forward CSR; rows of the
 * CSR are s * CP + j if compact, else omegas[s] * CP + j. Empty CSR rows leave data untouched. */
int dfx_spmm_pf_forward(const float *sino, const int32_t *row_ptr, const uint16_t *col_k, const float *val,
                        float *data, const int32_t *omegas, int n_sub, int my, int cp, int kstride, int kb,
                        int compact, void *stream);

/* replaces spmm_pf_adjoint_c / spmm_pf_adjoint_sub (pf_kernels.cl:644-687, SPFO:82-123):
 * sino[s, y, k] = alpha * sum_j val * data[omegas[s], y, j] for k < kb over the adjoint CSR (rows s * kb + k if
 * compact, else omegas[s] * kb + k); channels kb .. kstride-1 of sino are set to 0. */
int dfx_spmm_pf_adjoint(const float *data, const int32_t *row_ptr, const uint16_t *col_j, const float *val,
                        float *sino, const int32_t *omegas, int n_sub, int my, int kb, int cp, int kstride,
                        float alpha, int compact, void *stream);

/* The forward CSR of a batch regrouped into eta blocks (used by dfx_spmm_pf_forward_blocked in place of
 * spmm_pf_forward_c, pf_kernels.cl:597-641): block row g = r * P * ncb + cb * P + p (ncb = ceil(C / 4)) merges the
 * forward rows of the eta bins c = 4 cb .. 4 cb + 3 of ring p (j = c * P + p) into one list of orientations k
 * ascending, each entry holding k (uint16) and four values (float4; 0 where that bin's row has no entry k).
 * dfx_pf_fblock_rows: the number of block rows; dfx_pf_fblock_count: counts[g] (entries) and mask[g] (bit u: the row
 * of bin 4 cb + u has entries); after an exclusive scan of counts into fb_ptr (rows + 1 entries), dfx_pf_fblock_fill
 * writes fb_k and fb_v (16-byte aligned). */
int64_t dfx_pf_fblock_rows(int n_angles, int P, int C);
int dfx_pf_fblock_count(const int32_t *row_ptr_f, const uint16_t *col_k, int n_angles, int P, int C, int32_t *counts,
                        uint8_t *mask, void *stream);
int dfx_pf_fblock_fill(const int32_t *row_ptr_f, const uint16_t *col_k, const float *val_f, int n_angles, int P, int C,
                       const int32_t *fb_ptr, uint16_t *fb_k, float *fb_v, void *stream);

/* replaces spmm_pf_forward_c / spmm_pf_forward_sub (pf_kernels.cl:597-641, SPFO:38-80) over the eta-blocked rows of a
 * batch: data[omegas[s], y, j] += sum_k val * sino[s, y, k] for the n_sub angles omegas (NULL: all), C eta bins and P
 * rings; the bins whose forward row is empty are left untouched. The same sums as dfx_spmm_pf_forward on the batch's
 * forward CSR, bit for bit (over k ascending from 0, fused multiply-adds; a zero value adds exactly 0). */
int dfx_spmm_pf_forward_blocked(const float *sino, const int32_t *fb_ptr, const uint16_t *fb_k, const float *fb_v,
                                const uint8_t *fb_mask, float *data, const int32_t *omegas, int n_sub, int my, int P,
                                int C, int kstride, int kb, void *stream);

/* The same product as dfx_spmm_pf_forward_blocked, bit for bit (the same sums in the same order), through the
 * Radon output transposed to detector lines fastest: per chunk of angles, zt[s][k][y] (line stride 32 ceil(my / 32))
 * is written from sino, then each warp takes block rows (a block's rows longest first) and, per row, reads each entry
 * once and Z column k as whole 128-byte segments, 32 lines per lane group. zt holds zt_floats floats, at least dfx_spmm_pf_forward_zt_floats(1, my, kb) (one angle); the
 * angles run in chunks of what fits. max_groups: 32-line groups per warp at most (1 .. 9; 0: 9). P <= 32 rings. */
int64_t dfx_spmm_pf_forward_zt_floats(int n_angles, int my, int kb);
int dfx_spmm_pf_forward_blocked_zt(const float *sino, float *zt, int64_t zt_floats, const int32_t *fb_ptr,
                                   const uint16_t *fb_k, const float *fb_v, const uint8_t *fb_mask, float *data,
                                   const int32_t *omegas, int n_sub, int my, int P, int C, int kstride, int kb,
                                   int max_groups, void *stream);

/* The same product as dfx_spmm_pf_adjoint, bit for bit, through the data rows transposed to detector lines fastest:
 * per chunk of angles, dt[s][j][y] (line stride 32 ceil(my / 32)) is written from the rows omegas[s] (NULL: s) of
 * data, then one warp per orientation row and 32 lines reads each entry once and data column j as whole 128-byte
 * segments; the outputs (alpha times the sums; 0 for kb <= k < kstride) are written as whole row segments. dt holds
 * dt_floats floats, at least dfx_spmm_pf_adjoint_zt_floats(1, my, cp); max_groups as in
 * dfx_spmm_pf_forward_blocked_zt. cp <= 65536. */
int64_t dfx_spmm_pf_adjoint_zt_floats(int n_angles, int my, int cp);
int dfx_spmm_pf_adjoint_zt(const float *data, float *dt, int64_t dt_floats, const int32_t *row_ptr,
                           const uint16_t *col_j, const float *val, float *sino, const int32_t *omegas, int n_sub,
                           int my, int kb, int cp, int kstride, float alpha, int compact, int max_groups,
                           void *stream);

/* replaces batched_gemm_clblast / batched_gemm_clblast_adj (SPFO:2063-2127), the products of pf_mode "dense": pf is
 * the batch's float32 PF (n_omega, kb, cp) (dfx_pf_dense); adjoint 0: out = data (n_omega, my, cp) += in (n_omega, my,
 * kstride: the Radon output) . PF per angle; adjoint 1: out (n_omega, my, kstride) = alpha in (data) . PF^T per angle,
 * channels kb .. kstride-1 set to 0. One strided batched cuBLAS SGEMM over the angles in float32 (pedantic math: no
 * TF32); the cuBLAS handle is made on the first call of each host thread on each device. */
int dfx_pf_dense_products(int adjoint, const float *pf, int n_omega, int kb, int cp, const float *in, float *out,
                          int my, int kstride, float alpha, void *stream);

/* replaces zero_rows (SPFO:126-132): data rows omegas[s] (row_len floats each) <- 0. */
int dfx_zero_rows(float *data, const int32_t *omegas, int n_sub, int64_t row_len, void *stream);

/* replaces data.fill(0.0) of the pyopencl arrays (SPFO:1658 and the solvers): x[0 .. n-1] = value. */
int dfx_fill_f32(float *x, float value, int64_t n, void *stream);

/* ---------------------------------------------------------------- Poisson solvers
 * Periodic arrays (weights w, gain g, background bg): element i uses a[i % period]; period 0: the constant 1, 1, 0
 * (fista_poisson.py:287-308). */

/* replaces dual_update_sub (optimization/spdhg_poisson.py:69-91): on the rows of the angles omegas (row_len data
 * points each), d holds A x on entry and the dual change on exit; y <- prox_{sigma F*}(y + sigma A x), float64 math. */
int dfx_spdhg_dual_update(float *y, float *d, const float *sig, const float *b, const float *w, int64_t pw,
                          const float *g, int64_t pg, const float *bg, int64_t pbg, float eps,
                          const int32_t *omegas, int n_sub, int64_t row_len, void *stream);

/* replaces spdhg_update (spdhg_poisson.py:95-106): z += dz; x = T > 0 ? max(0, x - T (z + inv_p dz + lam)) : 0. */
int dfx_spdhg_primal_update(float *x, float *z, const float *T, const float *dz, float inv_p, float lam, int64_t n,
                            void *stream);
/* The same step with T stored in BF16 (widened exactly when read). */
int dfx_spdhg_primal_update_t16(float *x, float *z, const void *T_bf16, const float *dz, float inv_p, float lam,
                                int64_t n, void *stream);
/* out[i] = bf16(in[i]) rounded toward zero (stored step sizes never above their float32 values). */
int dfx_f32_to_bf16_rz(const float *in, void *out, int64_t n, void *stream);

/* replaces dual_steps (optimization/pdhg_poisson.py:79-84): sig = w != 0 && rowsum > 0 ? sigma0 / rowsum : 0. */
int dfx_dual_steps(float *sig, const float *rowsum, const float *w, int64_t pw, float sigma0, int64_t n, void *stream);

/* replaces set_mask_ones (pdhg_poisson.py:113-116): u = w != 0 ? 1 : 0. */
int dfx_set_mask_ones(float *u, const float *w, int64_t pw, int64_t n, void *stream);

/* replaces tinit / tmin / tfinal (spdhg_poisson.py:252-272), on n elements of a batch of whole images (npix pixels
 * each, supp (npix) uint8 or NULL): T = +inf; T = min(T, c / colsum) where inside and colsum > 0; T = 0 where +inf. */
int dfx_tinit(float *T, int64_t n, void *stream);
int dfx_tmin(float *T, const float *colsum, const uint8_t *supp, int64_t npix, float c, int64_t n, void *stream);
int dfx_tfinal(float *T, int64_t n, void *stream);

/* replaces support_ones / project_support (fista_poisson.py:256-263, 277-281): x = inside ? 1 : 0;
 * x = 0 where outside or x < 0. */
int dfx_support_ones(float *x, const uint8_t *supp, int64_t npix, int64_t n, void *stream);
int dfx_project_support(float *x, const uint8_t *supp, int64_t npix, int64_t n, void *stream);

/* FP64 reductions. Each writes its sums (float64) to out on the device; the partials go through scratch
 * (dfx_reduce_scratch_bytes(n) bytes). */
size_t dfx_reduce_scratch_bytes(int64_t n);

/* replaces poisson_value_grad (fista_poisson.py:72-113) with write_grad and mode: out[0] = sum_i w/g [m - b + b log(b/m)]
 * (mode 0, m = max(mu, 0) + bg + eps g) or its quadratic approximation at the data (mode 1); write_grad: mu <- df/dmu. */
int dfx_poisson_value_grad(float *mu, const float *b, const float *w, int64_t pw, const float *g, int64_t pg,
                           const float *bg, int64_t pbg, float eps, int write_grad, int mode, float floor_counts,
                           int64_t n, double *out, void *scratch, size_t scratch_bytes, void *stream);

/* replaces mean_counted (pdhg_poisson.py:97-111): out[0] = sum of b over w != 0, out[1] = their number. */
int dfx_mean_counted(const float *b, const float *w, int64_t pw, int64_t n, double *out, void *scratch,
                     size_t scratch_bytes, void *stream);

/* sums of x (and of x^2, x * y) in float64 for diagnostics and power iterations (replaces clarray.sum / vdot,
 * SPFO:2169-2185): out[0] = sum x_i y_i (y NULL: sum x_i). */
int dfx_dot_f64(const float *x, const float *y, int64_t n, double *out, void *scratch, size_t scratch_bytes,
                void *stream);

/* ---------------------------------------------------------------- BF16 tensor-core precision path
 * Dense BF16 PF (R, ktot, cp_pad), segments fastest: the batch k0 .. k0+kb-1 fills rows koff .. koff+kb-1 of every
 * angle (columns CP .. cp_pad-1 and rows outside the batch are left as they are: zero them once). The entries are the
 * float32 pf_entry values (dfx_pf_dense) rounded to nearest-even BF16. */
int dfx_pf_dense_bf16(const dfx_pf_geometry *g, int k0, int kb, int64_t koff, int64_t ktot, int cp_pad, void *out,
                      void *stream);
/* The same entries for the n_rows angles rows[s] only: out (n_rows, ktot, cp_pad), plane s = angle rows[s] (the PF of
 * one omega subset, generated for every pass in place of a stored dense PF of all angles). */
int dfx_pf_dense_bf16_rows(const dfx_pf_geometry *g, const int32_t *rows, int n_rows, int k0, int kb, int64_t koff,
                           int64_t ktot, int cp_pad, void *out, void *stream);

/* replaces batched_gemm_clblast (SPFO:2063-2098) and, in the BF16 path, spmm_pf_forward_c (pf_kernels.cl:597-641):
 * for the n_sub angles r = omegas[s] (omegas NULL: r = s), data[r, y, j] (+)= sum_k PF[r, k, j] Z[s, y, k] over the
 * orientations k = k0 .. k0+kn-1 of the ktot, with tcgen05 BF16 MMAs and float32 accumulation. pf_bf16 (n_omega,
 * ktot, cp_pad), z_bf16 (n_sub, my, ktot) BF16, data (n_omega, my, cp) float32; accumulate = 0 overwrites the rows.
 * ktot, k0 and cp_pad multiples of 8, both BF16 arrays 16-byte aligned. pf_compact: pf_bf16 holds the n_sub listed
 * angles only, (n_sub, ktot, cp_pad), angle s at row s (a PF generated for one subset). */
int dfx_pf_tc_forward(const void *pf_bf16, int64_t ktot, int64_t k0, int64_t kn, int cp, int cp_pad, int n_omega,
                      const void *z_bf16, const int32_t *omegas, int n_sub, int my, float *data, int accumulate,
                      int pf_compact, void *stream);
/* replaces batched_gemm_clblast_adj (SPFO:2100-2127) and, in the BF16 path, spmm_pf_adjoint_c (pf_kernels.cl:644-687):
 * Z[s, y, k] = alpha sum_j PF[r, k, j] D[r, y, j] for k = k0 .. k0+kn-1 (BF16 out, float32 accumulation), d_bf16
 * (n_omega, my, cp_pad); the other orientations of Z are left as they are; pf_compact as above. */
int dfx_pf_tc_adjoint(const void *pf_bf16, int64_t ktot, int64_t k0, int64_t kn, int cp, int cp_pad, int n_omega,
                      const void *d_bf16, const int32_t *omegas, int n_sub, int my, float alpha, void *z_bf16,
                      int pf_compact, void *stream);
/* Strided row conversion between float32 and BF16 (the Fourier-slice projector's float32 sinogram and the BF16
 * Radon output of the tensor-core products): to_bf16 1: b16[r * ld_b16 + c] = bf16(f32[r * ld_f32 + c]) (nearest-
 * even); 0: f32[...] = b16[...] (exact), for r < rows, c < cols. */
int dfx_convert_rows(int to_bf16, float *f32, int64_t ld_f32, void *b16, int64_t ld_b16, int64_t rows, int cols,
                     void *stream);

/* Forward projection of a BF16 channel-fastest batch on the tensor cores (tcgen05; the BF16 path's replacement of
 * radon_forward_k, radon_kernels.cl:44-101): sino[a, s, k] = scale * sum_p K(t_a(p) - s) img[p, k] for the n_angles
 * rows of geo (the launch's angles), float32 accumulation, written as BF16 (out_f32 0) or float32 with row stride
 * sino_ld. 8 x 8 pixel tiles against 32-bin windows starting at a multiple of 16 bins, weights as BF16 hi + lo parts;
 * admissible when every tile's taps span at most 17 bins (7 (|X| + |Y|) + 2 hw + 2 <= 17 per angle), n_det + 31 <=
 * 512 and kstride is a multiple of 64; taps outside a window are skipped and flagged (DFX_TC_WINDOW). tiles (NULL: all
 * tiles): the n_tiles tile indices (row-major over ceil(ny / 8) x ceil(nx / 8)) to project; the others must be zero. */
int dfx_radon_forward_tc(const void *img_bf16, void *sino, int64_t sino_ld, int out_f32, const float *geo,
                         int n_angles, int nx, int ny, int n_det, int kstride, int kernel, int n_taps, float scale,
                         const int32_t *tiles, int n_tiles, void *stream);
/* The weight tiles of dfx_radon_forward_tc precomputed per geometry (no reference counterpart): for every angle a of
 * geo and 8 x 8 pixel tile t (row-major over the tile grid), 8192 bytes at weights + (a * n_tiles + t) * 8192 (the
 * tap weights of the tile's pixels on its 32-bin window as BF16 hi and lo parts, in the MMA operand's layout) and
 * the window's first bin at windows[a * n_tiles + t]; weights 16-byte aligned, dfx_radon_tc_weights_bytes long.
 * dfx_radon_forward_tc_table: dfx_radon_forward_tc reading them (launch angle i = row angle_rows[i] of the table,
 * angle_rows NULL: i), the same products in the same order, hence the same bits. */
int64_t dfx_radon_tc_weights_bytes(int n_angles, int nx, int ny);
int dfx_radon_tc_weights(const float *geo, int n_angles, int nx, int ny, int n_det, int kernel, int n_taps,
                         void *weights, int32_t *windows, void *stream);
int dfx_radon_forward_tc_table(const void *img_bf16, void *sino, int64_t sino_ld, int out_f32, const void *weights,
                               const int32_t *windows, const int32_t *angle_rows, int n_angles, int nx, int ny,
                               int n_det, int kstride, float scale, const int32_t *tiles, int n_tiles, void *stream);

/* Bits of device-side waits of the tensor-core kernels that ran out since the last reset (DFX_TC_TIMEOUT); the
 * kernels return early on expiry and leave their outputs undefined. Synchronous; no reference counterpart. */
#define DFX_TC_TIMEOUT 1u
#define DFX_TC_WINDOW 2u   /* a tap outside the tensor-core backprojection's 32-bin window (skipped) */
int dfx_tc_status(unsigned int *flags, int reset);

/* BF16 copy of the data rows of the n_sub angles omegas[s] (omegas NULL: all n_omega rows): out (n_omega, my, cp_pad)
 * = in (n_omega, my, cp) rounded to nearest-even, padding columns set to 0. The data side of the adjoint product. */
int dfx_rows_to_bf16(const float *in, void *out, const int32_t *omegas, int n_sub, int my, int cp, int cp_pad,
                     void *stream);

/* out = in rounded to nearest-even BF16, n a multiple of 4 (in 16-byte, out 8-byte aligned); no reference
 * counterpart (the BF16 copies of the precision path). */
int dfx_f32_to_bf16(const float *in, void *out, int64_t n, void *stream);

/* FISTAPoisson (optimization/fista_poisson.py), all float32 element-wise with float64 sums:
 * replaces times_curvature (:115-144): u <- u * c, c the curvature of the data term at mu (mode 0 Poisson, 1 the
 * weighted least squares of the start); out[0] = sum c u_old^2. */
int dfx_times_curvature(float *u, const float *mu, const float *b, const float *w, int64_t pw, const float *g,
                        int64_t pg, const float *bg, int64_t pbg, float floor_counts, int mode, int64_t n, double *out,
                        void *scratch, size_t scratch_bytes, void *stream);
/* replaces support_sum (:146-159): out[0] = sum of x over the support (supp (npix) uint8 or NULL). */
int dfx_support_sum(const float *x, const uint8_t *supp, int64_t npix, int64_t n, double *out, void *scratch,
                    size_t scratch_bytes, void *stream);
/* replaces weighted_sums (:161-180): out = (sum w b, sum w mu). */
int dfx_weighted_sums(const float *mu, const float *b, const float *w, int64_t pw, int64_t n, double *out,
                      void *scratch, size_t scratch_bytes, void *stream);
/* replaces step_sums (:230-258): out = (<grad, xn - y>, sum (xn - y)^2 / D over D > 0, sum xn). */
int dfx_step_sums(const float *xn, const float *y, const float *grad, const float *D, int64_t n, double *out,
                  void *scratch, size_t scratch_bytes, void *stream);
/* replaces invert_metric (:201-209): D = inside && d > 0 ? 1 / d : 0. */
int dfx_invert_metric(float *D, const float *d, const uint8_t *supp, int64_t npix, int64_t n, void *stream);
/* replaces metric_step (:219-225): xn = D > 0 ? max(0, y - th D (grad + lam)) : 0. */
int dfx_metric_step(float *xn, const float *y, const float *grad, const float *D, float th, float lam, int64_t n,
                    void *stream);
/* replaces extrapolate (:260-266): out = a + beta (a - c). */
int dfx_extrapolate(float *out, const float *a, const float *c, float beta, int64_t n, void *stream);
/* replaces copy_buf / scale_buf (:268-275, :195-198): dst = src (both 16-byte aligned); x *= a. */
int dfx_copy_f32(const float *src, float *dst, int64_t n, void *stream);
int dfx_scale_f32(float *x, float a, int64_t n, void *stream);

/* FISTAL2 / FISTAHuber (optimization/fista_l2.py, fista_huber.py, fused_update.py), float32 element-wise with float64
 * sums. replaces residual_sumsq (fista_huber.py:80-105): r = w (Ax - b) in place (w periodic with period pw, pw = 0:
 * unweighted), then clipped to [-delta, delta] if clip; out[0] = sum r^2 before the clip. */
int dfx_ls_residual(float *ax, const float *b, const float *w, int64_t pw, int clip, float delta, int64_t n,
                    double *out, void *scratch, size_t scratch_bytes, void *stream);
/* replaces fista_fused_update (fused_update.py:22-49) for one orientation batch in the channel-fastest layout
 * (npix x kstride, kb live channels): v = prox(y - tau g) (prox 0 nonneg, 1 soft threshold lt, 2 nonneg soft
 * threshold), v = 0 outside supp (NULL: no support) and on padding channels, y = v + beta (v - x), x = v. Writes
 * dfx_fista_ls_blocks() x 3 float64 partial sums (sum g^2, sum v^2, sum |v|) to part; dfx_sum_partials adds the
 * partials of several launches in a fixed order (n_sums of 1, 2 or 3 per partial). */
int dfx_fista_ls_blocks(void);
int dfx_fista_ls_update(const float *g, float *x, float *y, const uint8_t *supp, int64_t npix, int kstride, int kb,
                        float tau, float beta, float lt, int prox, double *part, void *stream);
int dfx_sum_partials(const double *part, int n_part, int n_sums, double *out, void *stream);

/* Fourier-slice projector (replaces FourierRadon.forward / backward, operators/fourier_radon.py:248-297, with their
 * OpenCL kernels fourier_radon.cl:10-217 around the VkFFT transforms). The tables of one angle set (the full scan or
 * a subset), built on the host: deapodisation inv_dx (Nx), inv_dy (Ny); per polar sample (angle a, frequency
 * j < H = L/2 + 1; R*H samples): filt (2 floats: phase, bin response, 1/L), kb (2 int32: the first tap on the
 * oversampled Mx x My grid), w1 and w2 (W floats each); the spreading tiles of the half grid (16 x 16 cells,
 * n_tx per row of tiles): tile_ptr (n_tiles + 1) and tile_smp (sample, or -(sample + 1) through the Hermitian
 * mirror); wa (R) the angle weights; the lists cut into n_pieces pieces (4 int32 each: tile, first and end entry,
 * partial slot or -1 for a tile's first piece) with tile_xptr (n_tiles + 1) the slots of each tile's later pieces
 * (n_slots in all); scale the forward factor. */
typedef struct dfx_fr_geometry {
    const float *inv_dx, *inv_dy;
    const void *filt;
    const int32_t *kb;
    const float *w1, *w2;
    const int32_t *tile_ptr, *tile_smp;
    const float *wa;
    const int32_t *pieces, *tile_xptr;
    int32_t Nx, Ny, Ns, R, L, H, Mx, My, W, cx, cy, n_tx, n_tiles, n_pieces, n_slots;
    float scale;
} dfx_fr_geometry;
/* Scratch for channel slices of at most `channels` (grid, spectrum, lines and the cuFFT work area); 0 on bad input
 * (dfx_last_error says why). cuFFT plans are made on first use per size and kept by the library. */
size_t dfx_fr_scratch_bytes(const dfx_fr_geometry *g, int channels);
/* sino (R, Ns, kstride): channels 0 .. kb-1 = scale x the projections of the channel-fastest batch img_k
 * (Nx*Ny, kstride), channels kb .. kstride-1 = 0; the batch goes through in equal slices of at most `channels`. */
int dfx_fr_forward(const dfx_fr_geometry *g, const float *img_k, float *sino, int kstride, int kb, int channels,
                   void *scratch, size_t scratch_bytes, void *stream);
/* img_k channels 0 .. kb-1 = the transpose of the unscaled projection applied to sino, weighted by wa; padding
 * channels 0. */
int dfx_fr_backward(const dfx_fr_geometry *g, const float *sino, float *img_k, int kstride, int kb, int channels,
                    void *scratch, size_t scratch_bytes, void *stream);

/* replaces score_z (orientation_search.py:41-54): Z = E / sqrt(max(D, 1e-30)) (a NaN D kept), 0 where D <= 0, with
 * correctly rounded division and square root (the float32 NumPy values, bitwise). */
int dfx_score_z(const float *E, const float *D, float *Z, int64_t n, void *stream);

/* Local basis (replaces the strip kernels local_radon_forward / local_radon_backward of
 * operators/local_kernels.cl:38-181 around the dense projections): the patches of one orientation batch, box
 * (y0, x0, h, w) int32 x 4 per patch (16-byte aligned), coff int64 (offset of its coefficients, row-major), chan
 * int32 (its orientation's channel in the batch, < kstride), mask (uint8 per coefficient: 1 where the voxel is
 * allowed). scatter: img_k (Nx*Ny, kstride) channel-fastest, at the patches' voxels = coeffs where allowed, 0 at
 * their other voxels (the caller zeroes the rest of the batch image first); gather: coeffs of the patches = img_k at
 * the allowed voxels, 0 at the others. pix_row (NULL: whole images): the row of every pixel (nx * ny int32) in a
 * compact batch image of the batch's support pixels, -1 for the others (cells there are skipped / read as 0). */
int dfx_local_scatter(const float *coeffs, const uint8_t *mask, const int32_t *box, const int64_t *coff,
                      const int32_t *chan, int n_patches, int nx, int ny, int kstride, const int32_t *pix_row,
                      float *img_k, void *stream);
int dfx_local_gather(const float *img_k, const uint8_t *mask, const int32_t *box, const int64_t *coff,
                     const int32_t *chan, int n_patches, int nx, int ny, int kstride, const int32_t *pix_row,
                     float *coeffs, void *stream);

/* replaces tv_dual_dense / tv_adjoint_dense + spdhg_update / tv_value_dense (optimization/spdhg_poisson.py:110-186)
 * on one channel-fastest batch (nx * ny pixels x kstride channels; T = 0 on padding channels): SPDHG's total-variation
 * block. dfx_tv_dual: q <- proj_{|q| <= lam}(q + s D x) with forward differences to the right and down between
 * coefficients with T > 0, s = ps / (4 max(T_j + T_neighbour)), dq = q' - q (batch-sized). dfx_tv_adjoint_update:
 * dz = D^T dq, z += dz, x = T > 0 ? max(0, x - T (z + inv_p dz + lam)) : 0. dfx_tv_value: out[0] = sum |D x| (float64
 * sum; scratch of dfx_reduce_scratch_bytes(nx * ny * kstride)). */
int dfx_tv_dual(const float *x, const float *T, float *qx, float *qy, float *dqx, float *dqy, int nx, int ny,
                int kstride, float lam, float ps, void *stream);
int dfx_tv_adjoint_update(const float *dqx, const float *dqy, float *x, float *z, const float *T, int nx, int ny,
                          int kstride, float inv_p, float lam, void *stream);
int dfx_tv_value(const float *x, const float *T, int nx, int ny, int kstride, double *out, void *scratch,
                 size_t scratch_bytes, void *stream);

/* replaces tv_dual_local / tv_adjoint_local + spdhg_update / tv_value_local (spdhg_poisson.py:188-230): the TV block
 * on a local basis's n flat coefficients, the differences to the right / down neighbours within each patch (index
 * arrays right, down, left, up; -1: none), the arithmetic of dfx_tv_dual / dfx_tv_adjoint_update / dfx_tv_value. */
int dfx_tv_dual_local(const float *x, const float *T, float *qx, float *qy, float *dqx, float *dqy,
                      const int32_t *right, const int32_t *down, float lam, float ps, int64_t n, void *stream);
int dfx_tv_adjoint_update_local(const float *dqx, const float *dqy, float *x, float *z, const float *T,
                                const int32_t *left, const int32_t *up, float inv_p, float lam, int64_t n,
                                void *stream);
int dfx_tv_value_local(const float *x, const float *T, const int32_t *right, const int32_t *down, int64_t n,
                       double *out, void *scratch, size_t scratch_bytes, void *stream);

/* replaces tv_adjoint_local / tree_sums / tree_scatter (spdhg_poisson.py:188-249): the hierarchical total variation's
 * pieces. dfx_tv_adjoint_local writes w = D^T dq (the adjoint of dfx_tv_dual_local's differences, no primal step);
 * dfx_tree_sums writes s_j = the float32 sum of x[idx[p]], p in [ptr[j], ptr[j+1]) (a node-pixel's coefficients);
 * dfx_tree_scatter adds w[map[i]] to dz[i] where map[i] >= 0. */
int dfx_tv_adjoint_local(const float *dqx, const float *dqy, float *w, const int32_t *left, const int32_t *up,
                         int64_t n, void *stream);
int dfx_tree_sums(const float *x, const int32_t *ptr, const int32_t *idx, float *s, int64_t n, void *stream);
int dfx_tree_scatter(const float *w, const int32_t *map, float *dz, int64_t n, void *stream);

/* replaces osem_update (optimization/osem_poisson.py:80-84): x = outside the support (mask periodic with period pm,
 * 0: no mask) ? 0 : (sens > 0 ? x back / (sens + lam) : x). */
int dfx_osem_update(float *x, const float *back, const float *sens, const uint8_t *mask, int64_t pm, float lam,
                    int64_t n, void *stream);

/* replaces PDHGPoisson's dual_update, primal_update, average, primal_steps (optimization/pdhg_poisson.py:33-94):
 * y <- prox_{sig F*}(y + sig Axb) in float64 (0 where w = 0 or sig = 0); x_new = T > 0 ? max(0, x - T (grad + lam)) :
 * 0, xb = 2 x_new - x, x = x_new; Ax = (Axb + Ax) / 2; T = tau0 / colsum inside the support (period npix) where
 * colsum > 0, else 0. */
int dfx_pdhg_dual_update(float *y, const float *Axb, const float *sig, const float *b, const float *w, int64_t pw,
                         const float *g, int64_t pg, const float *bg, int64_t pbg, float eps, int64_t n, void *stream);
int dfx_pdhg_primal_update(float *x, float *xb, const float *grad, const float *T, float lam, int64_t n, void *stream);
int dfx_pdhg_average(float *Ax, const float *Axb, int64_t n, void *stream);
int dfx_pdhg_primal_steps(float *T, const float *colsum, const uint8_t *supp, int64_t npix, float tau0, int64_t n,
                          void *stream);

/* replaces PoissonTerm's pt_grad_curv / pt_ratio / pt_wg (optimization/poisson_term.py:52-58), mu = max(pred, 0) +
 * bg + eps g, on points of weight != 0 (0 elsewhere): mode 0 r = w/g (1 - b/mu), c = w / (g max(mu, floor g)) (c may
 * be NULL); mode 1 r = w b / (g mu); mode 2 r = w / g (pred unused). */
int dfx_poisson_term(const float *pred, const float *b, const float *w, int64_t pw, const float *g, int64_t pg,
                     const float *bg, int64_t pbg, float eps, float floor_counts, int mode, float *r, float *c,
                     int64_t n, void *stream);

/* ---------------------------------------------------------------- parameter gradients
 * replaces pf_param_vjp (differentiable/pf_grad.cl:48-176, launched by PFGradient.__call__,
 * differentiable/gradients.py:112-174): for every non-zero (r, k, j) of a batch's adjoint CSR (orientations
 * k0 .. k0+kb-1), G = sum_y res[r, y, j] sino[r, y, k] times the derivative of the PF entry with respect to the
 * rotation (3), the width (1), the eta offset, the axis tilt (2) and the ring's two-theta, summed per row r * kb + k
 * into rows (R * kb, nq doubles; nq = dfx_pf_param_nq(P, hess); float32 entries, float64 sums); hess: also the
 * upper triangle of
 * sum_y curv S^2 q q^T (10 floats after the width), q the derivative of the entry with respect to (rot, sigma).
 * flags: 1 eta offset, 2 axis tilt, 4 two-theta (each needs its probed directions' derivatives, coords-shaped).
 * With reflection_two_theta (g->axis_w set; pf_grad.cl AXIS_THETA) dv_* are the derivatives of u, dw_t1 / dw_t2 those
 * of w ((R * S, 3)) for the tilt, and the Bragg angle's derivative needs none (dv_tth unused).
 * At most 16 rings; my floats + 2 nq doubles of shared memory (<= 48 KB). */
int dfx_pf_param_nq(int n_rings, int hess);
int dfx_pf_param_vjp(const dfx_pf_geometry *g, const int32_t *row_ptr, const uint16_t *col_j, const float *res,
                     const float *curv, const float *sino, int my, int kstride, int k0, int kb, int flags,
                     const float *dv_eta, const float *dv_t1, const float *dv_t2, const float *dv_tth,
                     const float *dw_t1, const float *dw_t2, int hess, double *rows, void *stream);
/* replaces rows_to_orientations (pf_grad.cl:179-187): out (kb, nq) = rows summed over the n_angles angles. */
int dfx_pf_rows_sum(const double *rows, int n_angles, int kb, int nq, double *out, void *stream);

/* replaces radon_dforward_k (differentiable/proj_grad.cl:12-63): the ray table (row pointers of
 * dfx_radon_table_count without support) with the weights K'(t - s), the derivative of every tap with respect to a
 * detector shift; dfx_radon_forward_table through it gives dS. */
int dfx_radon_dtable_fill(const float *geo, int n_angles, int nx, int ny, int n_det, int kernel,
                          const int32_t *row_ptr, int32_t *entries, void *stream);
/* replaces shift_dot (proj_grad.cl:66-87): out[a] = sum_{y < n_det, k < kb} Z[a, y, k] dS[a, y, k]. */
int dfx_angle_dot(const float *Z, const float *dS, int n_angles, int n_det, int kstride, int kb, float *out,
                  void *stream);

#ifdef __cplusplus
}
#endif
#endif
