// Parallel-beam Radon transform of a batch of channel-fastest images (the orientations of a batch are the channels),
// sm_100a, FP32. Semantics: operators/radon_kernels.cl of diffractom (ParallelRadon), tap weights as in
// dfx_common.cuh (and the CPU oracle, oracle/oracle_core.h).
//
// Forward (ray-driven): a thread owns NB neighbouring detector bins of one angle and 8 channels (two float4), loops
// over the image rows and over the pixels of each row whose footprint reaches its bins, and accumulates in
// registers; no atomics, each output written once. Backward (pixel-driven): a thread owns one pixel and 8 channels
// and loops over the angles and the taps of its footprint. Both read the image / sinogram through L1 (__ldg).
#include "dfx_common.cuh"

namespace dfx {

constexpr int CPT = 8;              // channels per thread (two float4)
constexpr int FWD_CG = 16;          // channel groups per forward block (128 channels)
constexpr int FWD_BG = 8;           // bin groups per forward block
constexpr int BWD_CG = 16;          // channel groups per backward block
constexpr int BWD_PX = 16;          // pixels per backward block

__device__ __forceinline__ void ld8(const float *p, float4 &a, float4 &b) {
    a = __ldg(reinterpret_cast<const float4 *>(p));
    b = __ldg(reinterpret_cast<const float4 *>(p) + 1);
}

template <int KERNEL, int NB>
__global__ void __launch_bounds__(FWD_CG *FWD_BG) radon_forward_kernel(
    const float *__restrict__ img, float *__restrict__ sino, const float4 *__restrict__ geo, int nx, int ny, int ns,
    int kstride, int kb, float scale)
{
    const int a = blockIdx.z;
    const int k = (blockIdx.y * FWD_CG + threadIdx.x) * CPT;
    const int s0 = (blockIdx.x * FWD_BG + threadIdx.y) * NB;
    if (k >= kstride || s0 >= ns) return;
    const AngleGeo g = load_geo(geo, a);
    const int nu = g.rows_are_y ? nx : ny, nv = g.rows_are_y ? ny : nx;
    const int64_t du = g.rows_are_y ? 1 : nx, dv = g.rows_are_y ? nx : 1;   // pixel strides of u, v
    const bool live = k < kb;             // kb is a multiple of 8 or the tail group is fully masked below
    float acc[NB][CPT];
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[j][c] = 0.0f;

    const float half = KERNEL == 1 ? g.hw : 1.0f;
    const float inv = __frcp_rn(g.A);
    const float *base = img + k;
    if (live) {
        for (int v = 0; v < nv; ++v) {
            const float c = __fmaf_rn(g.B, (float)v, g.T0);
            // pixels whose t lies in (s0 - half, s0 + NB - 1 + half): u between these, in either order
            const float e1 = (s0 - half - c) * inv, e2 = (s0 + NB - 1 + half - c) * inv;
            // (a margin of 1e-3 pixel covers the rounding of e1, e2; the tap weights decide membership)
            const int u0 = max((int)floorf(fminf(e1, e2) - 1e-3f), 0);
            const int u1 = min((int)ceilf(fmaxf(e1, e2) + 1e-3f), nu - 1);
            const float *row = base + (int64_t)v * dv * kstride;
            for (int u = u0; u <= u1; ++u) {
                const float t = __fmaf_rn(g.A, (float)u, c);
                float4 p0, p1;
                ld8(row + (int64_t)u * du * kstride, p0, p1);
#pragma unroll
                for (int j = 0; j < NB; ++j) {
                    const float w = tap_weight<KERNEL>(g, __fsub_rn(t, (float)(s0 + j)));
                    acc[j][0] = __fmaf_rn(w, p0.x, acc[j][0]);
                    acc[j][1] = __fmaf_rn(w, p0.y, acc[j][1]);
                    acc[j][2] = __fmaf_rn(w, p0.z, acc[j][2]);
                    acc[j][3] = __fmaf_rn(w, p0.w, acc[j][3]);
                    acc[j][4] = __fmaf_rn(w, p1.x, acc[j][4]);
                    acc[j][5] = __fmaf_rn(w, p1.y, acc[j][5]);
                    acc[j][6] = __fmaf_rn(w, p1.z, acc[j][6]);
                    acc[j][7] = __fmaf_rn(w, p1.w, acc[j][7]);
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        if (s0 + j >= ns) break;
        float *o = sino + ((int64_t)a * ns + s0 + j) * kstride + k;
        float4 r0, r1;
        float r[CPT];
#pragma unroll
        for (int c = 0; c < CPT; ++c) r[c] = (k + c < kb) ? scale * acc[j][c] : 0.0f;   // padding channels: 0
        r0 = make_float4(r[0], r[1], r[2], r[3]);
        r1 = make_float4(r[4], r[5], r[6], r[7]);
        reinterpret_cast<float4 *>(o)[0] = r0;
        reinterpret_cast<float4 *>(o)[1] = r1;
    }
}

template <int KERNEL>
__global__ void __launch_bounds__(BWD_CG *BWD_PX) radon_backward_kernel(
    const float *__restrict__ sino, float *__restrict__ img, const float4 *__restrict__ geo, int n_angles, int nx,
    int ny, int ns, int kstride, int kb, int n_taps)
{
    const int k = (blockIdx.y * BWD_CG + threadIdx.x) * CPT;
    const int64_t p = (int64_t)blockIdx.x * BWD_PX + threadIdx.y;
    if (k >= kstride || p >= (int64_t)nx * ny) return;
    const int x = (int)(p % nx), y = (int)(p / nx);
    float acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = 0.0f;
    if (k < kb) {
        const float *col = sino + k;
        for (int a = 0; a < n_angles; ++a) {
            const AngleGeo g = load_geo(geo, a);
            const float u = (float)(g.rows_are_y ? x : y), v = (float)(g.rows_are_y ? y : x);
            const float t = __fmaf_rn(g.A, u, __fmaf_rn(g.B, v, g.T0));
            const int s_lo = KERNEL == 1 ? (int)floorf(__fsub_rn(t, g.hw)) : (int)floorf(t);
            const int n = KERNEL == 1 ? n_taps + 1 : 2;
            for (int i = 0; i < n; ++i) {
                const int s = s_lo + i;
                if (s < 0 || s >= ns) continue;
                const float w = tap_weight<KERNEL>(g, __fsub_rn(t, (float)s));
                if (w == 0.0f) continue;
                const float ww = __fmul_rn(g.w, w);
                float4 q0, q1;
                ld8(col + ((int64_t)a * ns + s) * kstride, q0, q1);
                acc[0] = __fmaf_rn(ww, q0.x, acc[0]);
                acc[1] = __fmaf_rn(ww, q0.y, acc[1]);
                acc[2] = __fmaf_rn(ww, q0.z, acc[2]);
                acc[3] = __fmaf_rn(ww, q0.w, acc[3]);
                acc[4] = __fmaf_rn(ww, q1.x, acc[4]);
                acc[5] = __fmaf_rn(ww, q1.y, acc[5]);
                acc[6] = __fmaf_rn(ww, q1.z, acc[6]);
                acc[7] = __fmaf_rn(ww, q1.w, acc[7]);
            }
        }
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c)
        if (k + c >= kb) acc[c] = 0.0f;                     // padding channels: 0
    float4 *o = reinterpret_cast<float4 *>(img + p * kstride + k);
    o[0] = make_float4(acc[0], acc[1], acc[2], acc[3]);
    o[1] = make_float4(acc[4], acc[5], acc[6], acc[7]);
}

// (Ktot, npix) <-> (npix, kstride) channel transposes through a 32 x 33 shared tile.
constexpr int TT = 32;

__global__ void __launch_bounds__(TT * 8) gather_kernel(const float *__restrict__ coeffs, float *__restrict__ img,
                                                        int64_t npix, int k0, int kb, int kstride)
{
    __shared__ float tile[TT][TT + 1];
    const int64_t p0 = (int64_t)blockIdx.x * TT;
    const int q0 = blockIdx.y * TT;
    for (int j = threadIdx.y; j < TT; j += 8) {            // read: pixels contiguous
        const int64_t p = p0 + threadIdx.x;
        const int q = q0 + j;
        tile[j][threadIdx.x] = (p < npix && q < kb) ? coeffs[(int64_t)(k0 + q) * npix + p] : 0.0f;
    }
    __syncthreads();
    for (int j = threadIdx.y; j < TT; j += 8) {            // write: channels contiguous
        const int64_t p = p0 + j;
        const int q = q0 + threadIdx.x;
        if (p < npix && q < kstride) img[p * kstride + q] = tile[threadIdx.x][j];
    }
}

__global__ void __launch_bounds__(TT * 8) scatter_kernel(const float *__restrict__ img, float *__restrict__ coeffs,
                                                         int64_t npix, int k0, int kb, int kstride)
{
    __shared__ float tile[TT][TT + 1];
    const int64_t p0 = (int64_t)blockIdx.x * TT;
    const int q0 = blockIdx.y * TT;
    for (int j = threadIdx.y; j < TT; j += 8) {            // read: channels contiguous
        const int64_t p = p0 + j;
        const int q = q0 + threadIdx.x;
        tile[j][threadIdx.x] = (p < npix && q < kstride) ? img[p * kstride + q] : 0.0f;
    }
    __syncthreads();
    for (int j = threadIdx.y; j < TT; j += 8) {            // write: pixels contiguous
        const int64_t p = p0 + threadIdx.x;
        const int q = q0 + j;
        if (p < npix && q < kb) coeffs[(int64_t)(k0 + q) * npix + p] = tile[threadIdx.x][j];
    }
}

static int check_radon_args(const void *in, const void *out, const void *geo, int n_angles, int nx, int ny,
                            int n_det, int kstride, int kb, int kernel)
{
    DFX_REQUIRE(in && out && geo, "radon: null pointer");
    DFX_REQUIRE(n_angles >= 0 && nx > 0 && ny > 0 && n_det > 0, "radon: bad sizes (angles %d, %d x %d, %d bins)",
                n_angles, nx, ny, n_det);
    DFX_REQUIRE(kstride > 0 && kstride % CPT == 0 && kb >= 0 && kb <= kstride,
                "radon: kstride (%d) must be a positive multiple of %d and kb (%d) <= kstride", kstride, CPT, kb);
    DFX_REQUIRE(kernel == 0 || kernel == 1, "radon: kernel must be 0 (hat) or 1 (trapezoid)");
    DFX_REQUIRE(((uintptr_t)in % 16) == 0 && ((uintptr_t)out % 16) == 0 && ((uintptr_t)geo % 16) == 0,
                "radon: arrays must be 16-byte aligned");
    DFX_REQUIRE((int64_t)nx * ny * kstride < ((int64_t)1 << 40), "radon: image batch too large");
    return DFX_OK;
}

}  // namespace dfx

using namespace dfx;

extern "C" int dfx_radon_forward(const float *img_k, float *sino_k, const float *geo, int n_angles, int nx, int ny,
                                 int n_det, int kstride, int kb, int kernel, float scale, void *stream)
{
    int st = check_radon_args(img_k, sino_k, geo, n_angles, nx, ny, n_det, kstride, kb, kernel);
    if (st) return st;
    if (n_angles == 0) return DFX_OK;
    constexpr int NB = 2;
    DFX_REQUIRE(n_angles <= 65535, "radon: at most 65535 angles per launch");
    dim3 block(FWD_CG, FWD_BG);
    dim3 grid((unsigned)cdiv(n_det, FWD_BG * NB), (unsigned)cdiv(kstride, FWD_CG * CPT), (unsigned)n_angles);
    cudaStream_t s = (cudaStream_t)stream;
    const float4 *g4 = reinterpret_cast<const float4 *>(geo);
    if (kernel == 1)
        radon_forward_kernel<1, NB><<<grid, block, 0, s>>>(img_k, sino_k, g4, nx, ny, n_det, kstride, kb, scale);
    else
        radon_forward_kernel<0, NB><<<grid, block, 0, s>>>(img_k, sino_k, g4, nx, ny, n_det, kstride, kb, scale);
    return launch_status("radon_forward");
}

extern "C" int dfx_radon_backward(const float *sino_k, float *img_k, const float *geo, int n_angles, int nx, int ny,
                                  int n_det, int kstride, int kb, int kernel, int n_taps, void *stream)
{
    int st = check_radon_args(sino_k, img_k, geo, n_angles, nx, ny, n_det, kstride, kb, kernel);
    if (st) return st;
    DFX_REQUIRE(n_taps >= 2 && n_taps <= 64, "radon: n_taps (%d) out of range", n_taps);
    const int64_t npix = (int64_t)nx * ny;
    dim3 block(BWD_CG, BWD_PX);
    dim3 grid((unsigned)cdiv(npix, BWD_PX), (unsigned)cdiv(kstride, BWD_CG * CPT));
    DFX_REQUIRE(grid.x < 2147483647u && grid.y <= 65535u, "radon: batch too large for one launch");
    cudaStream_t s = (cudaStream_t)stream;
    const float4 *g4 = reinterpret_cast<const float4 *>(geo);
    if (kernel == 1)
        radon_backward_kernel<1><<<grid, block, 0, s>>>(sino_k, img_k, g4, n_angles, nx, ny, n_det, kstride, kb, n_taps);
    else
        radon_backward_kernel<0><<<grid, block, 0, s>>>(sino_k, img_k, g4, n_angles, nx, ny, n_det, kstride, kb, n_taps);
    return launch_status("radon_backward");
}

extern "C" int dfx_gather_channels(const float *coeffs, float *img_k, int64_t npix, int k0, int kb, int kstride,
                                   void *stream)
{
    DFX_REQUIRE(coeffs && img_k, "gather: null pointer");
    DFX_REQUIRE(npix > 0 && k0 >= 0 && kb >= 0 && kb <= kstride, "gather: bad sizes");
    dim3 grid((unsigned)cdiv(npix, TT), (unsigned)cdiv(kstride, TT));
    DFX_REQUIRE(grid.y <= 65535u, "gather: kstride too large");
    gather_kernel<<<grid, dim3(TT, 8), 0, (cudaStream_t)stream>>>(coeffs, img_k, npix, k0, kb, kstride);
    return launch_status("gather_channels");
}

extern "C" int dfx_scatter_channels(const float *img_k, float *coeffs, int64_t npix, int k0, int kb, int kstride,
                                    void *stream)
{
    DFX_REQUIRE(coeffs && img_k, "scatter: null pointer");
    DFX_REQUIRE(npix > 0 && k0 >= 0 && kb >= 0 && kb <= kstride, "scatter: bad sizes");
    dim3 grid((unsigned)cdiv(npix, TT), (unsigned)cdiv(kb, TT));
    if (kb == 0) return DFX_OK;
    DFX_REQUIRE(grid.y <= 65535u, "scatter: kb too large");
    scatter_kernel<<<grid, dim3(TT, 8), 0, (cudaStream_t)stream>>>(img_k, coeffs, npix, k0, kb, kstride);
    return launch_status("scatter_channels");
}
