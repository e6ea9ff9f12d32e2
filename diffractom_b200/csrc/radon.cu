// Parallel-beam Radon transform of a batch of channel-fastest images (the orientations of a batch are the channels),
// sm_100a, FP32. Semantics: operators/radon_kernels.cl of diffractom (ParallelRadon); tap weights as in
// dfx_common.cuh, which the CPU oracle (oracle/oracle_core.h) restates bit for bit.
//
// Work split: the 32 lanes of a warp own 8 channels each (256 channels per warp), so everything that depends on the
// geometry only (detector coordinate, tap bins and weights) is the same for the whole warp: one warp instruction
// serves 256 channels, and a zero weight skips its FMAs with a branch all lanes take.
//
// Forward (ray-driven gather, no atomics): a warp owns one bin of one angle; per image row it reads the two to four
// pixels whose footprint reaches the bin. The grid is ordered so that one channel block of the image stays in L2
// while all angles and bins of the launch read it.
//
// Backward (pixel-driven, no atomics): a warp owns one pixel. The per-angle constants are computed once per block
// into shared memory; per angle the warp evaluates the pixel's taps and reads 8 channels of each tap's sinogram bin
// per lane. A fused variant applies SPDHG's primal step in the epilogue (no dz array).
//
// The sinogram is float32 or, in the BF16 precision path, BF16 with its own row stride (bins of all orientation
// batches side by side): loads widen BF16 to float32 exactly, the forward rounds its float32 sums once on store.
#include <cuda_bf16.h>

#include "dfx_common.cuh"

namespace dfx {

constexpr int WARPS = 8;        // warps per block
constexpr int CPL = 8;          // channels per lane
constexpr int CPW = 32 * CPL;   // channels per warp

__device__ __forceinline__ void ld8(const float *p, float4 &a, float4 &b)
{
    a = __ldg(reinterpret_cast<const float4 *>(p));
    b = __ldg(reinterpret_cast<const float4 *>(p) + 1);
}

__device__ __forceinline__ float bf_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf_hi(uint32_t u) { return __uint_as_float(u & 0xFFFF0000u); }

__device__ __forceinline__ void ld8(const __nv_bfloat16 *p, float4 &a, float4 &b)
{
    const uint4 u = __ldg(reinterpret_cast<const uint4 *>(p));
    a = make_float4(bf_lo(u.x), bf_hi(u.x), bf_lo(u.y), bf_hi(u.y));
    b = make_float4(bf_lo(u.z), bf_hi(u.z), bf_lo(u.w), bf_hi(u.w));
}

__device__ __forceinline__ void st8(float *p, const float (&r)[CPL])
{
    reinterpret_cast<float4 *>(p)[0] = make_float4(r[0], r[1], r[2], r[3]);
    reinterpret_cast<float4 *>(p)[1] = make_float4(r[4], r[5], r[6], r[7]);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&h);
}

__device__ __forceinline__ void st8(__nv_bfloat16 *p, const float (&r)[CPL])
{
    *reinterpret_cast<uint4 *>(p) = make_uint4(pack_bf16(r[0], r[1]), pack_bf16(r[2], r[3]), pack_bf16(r[4], r[5]),
                                               pack_bf16(r[6], r[7]));
}

// a += w p on 8 channels: four paired FMAs (FFMA2, sm_100), each lane of a pair rounded once as fmaf does
__device__ __forceinline__ void acc8(float (&a)[CPL], float w, const float4 &p0, const float4 &p1)
{
    const float2 ww = make_float2(w, w);
    float2 r0 = __ffma2_rn(ww, make_float2(p0.x, p0.y), make_float2(a[0], a[1]));
    float2 r1 = __ffma2_rn(ww, make_float2(p0.z, p0.w), make_float2(a[2], a[3]));
    float2 r2 = __ffma2_rn(ww, make_float2(p1.x, p1.y), make_float2(a[4], a[5]));
    float2 r3 = __ffma2_rn(ww, make_float2(p1.z, p1.w), make_float2(a[6], a[7]));
    a[0] = r0.x; a[1] = r0.y; a[2] = r1.x; a[3] = r1.y;
    a[4] = r2.x; a[5] = r2.y; a[6] = r3.x; a[7] = r3.y;
}

// bins strictly inside a pixel's footprint (t - hw, t + hw) at this angle: at most ceil(1 + |A|) for the trapezoid
// (2 for the hat), never more than the caller's bound n_taps
__device__ __forceinline__ int taps_of(const AngleGeo &g, int kernel, int n_taps)
{
    if (kernel != 1) return 2;
    const int t = max(2, (int)ceilf(1.0f + fabsf(g.A) - 1e-6f));
    return min(t, n_taps);
}

// first bin that can get a non-zero weight from a pixel at detector coordinate t
template <int KERNEL>
__device__ __forceinline__ int first_tap(const AngleGeo &g, float t)
{
    return KERNEL == 1 ? (int)floorf(__fsub_rn(t, g.hw)) + 1 : (int)floorf(t);
}

// ------------------------------------------------------------------------------------------------ forward
// Ray-driven gather: a warp owns one bin s of one angle and 256 channels. Per image row it evaluates the pixels whose
// footprint can reach s (two to four), skips zero weights (a branch the whole warp takes) and accumulates the
// weighted channels in registers: no shared memory, no atomics, a fixed summation order. The grid runs
// channel-block-major (blockIdx.z), so the columns of one channel block (npix x 256) are read from L2 by every
// angle and bin while they are resident.
template <int KERNEL, typename ST>
__global__ void __launch_bounds__(32 * WARPS) radon_forward_v4(
    const float *__restrict__ img, ST *__restrict__ sino, int64_t sld, const float4 *__restrict__ geo, int nx, int ny,
    int ns, int kstride, int kb, float scale)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int s = blockIdx.x * WARPS + warp;
    const int a = blockIdx.y;
    const int k = blockIdx.z * CPW + lane * CPL;
    if (s >= ns) return;                                   // whole warps
    const bool live = k < kstride;
    if (blockIdx.z * CPW >= kb) {                          // padding channels only
        const float zero[CPL] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (live) st8(sino + ((int64_t)a * ns + s) * sld + k, zero);
        return;
    }
    const bool load = k < kb;
    const AngleGeo g = load_geo(geo, a);
    const int nu = g.rows_are_y ? nx : ny, nv = g.rows_are_y ? ny : nx;
    const int64_t du = (g.rows_are_y ? 1 : (int64_t)nx) * kstride, dv = (g.rows_are_y ? (int64_t)nx : 1) * kstride;
    const float half = KERNEL == 1 ? g.hw : 1.0f;
    const float inv = __frcp_rn(g.A);
    const float fs = (float)s;
    float acc[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c) acc[c] = 0.0f;
    const float *base = img + (live ? k : 0);
#pragma unroll 2
    for (int v = 0; v < nv; ++v) {
        const float c = __fmaf_rn(g.B, (float)v, g.T0);
        const float e1 = (fs - half - c) * inv, e2 = (fs + half - c) * inv;
        // a margin of 1e-3 pixel covers the rounding of e1, e2; the tap weights decide membership
        const int u0 = max((int)floorf(fminf(e1, e2) - 1e-3f), 0);
        const int u1 = min((int)ceilf(fmaxf(e1, e2) + 1e-3f), nu - 1);
        const float *row = base + (int64_t)v * dv;
        for (int u = u0; u <= u1; ++u) {
            const float w = tap_weight<KERNEL>(g, __fsub_rn(__fmaf_rn(g.A, (float)u, c), fs));
            if (w == 0.0f) continue;
            float4 p0 = make_float4(0.f, 0.f, 0.f, 0.f), p1 = p0;
            if (load) ld8(row + (int64_t)u * du, p0, p1);
            acc8(acc, w, p0, p1);
        }
    }
    if (!live) return;
    float r[CPL];
#pragma unroll
    for (int q = 0; q < CPL; ++q) r[q] = (k + q < kb) ? __fmul_rn(scale, acc[q]) : 0.0f;   // padding channels: 0
    st8(sino + ((int64_t)a * ns + s) * sld + k, r);
}

// ---- ray table: the non-zero taps of every (angle, bin) in the order radon_forward_v4 visits them (rows v, then
// pixels u ascending), as (pixel index, weight bits). The geometry of an operator is fixed, so the table is built
// once; the table-driven forward then spends its instructions on loads and FMAs only, with many taps in flight.
// supp (optional, one byte per pixel): only the taps of pixels inside the support; for images that are zero outside
// it (a solver's iterates projected onto the support) the forward through this table adds exactly the same terms
// minus zeros, so it gives the same bits.
// DERIV: the same taps with the weights K'(t - s) (tap_dweight), the table of the projections' derivative with
// respect to a detector shift of every angle.
template <int KERNEL, bool DERIV = false>
__global__ void ray_table_kernel(const float4 *__restrict__ geo, int n_angles, int nx, int ny, int ns,
                                 const uint8_t *__restrict__ supp, int32_t *__restrict__ counts,
                                 const int32_t *__restrict__ row_ptr, int2 *__restrict__ entries)
{
    const int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;      // a * ns + s
    if (row >= (int64_t)n_angles * ns) return;
    const int a = (int)(row / ns), s = (int)(row % ns);
    const AngleGeo g = load_geo(geo, a);
    const int nu = g.rows_are_y ? nx : ny, nv = g.rows_are_y ? ny : nx;
    const float half = KERNEL == 1 ? g.hw : 1.0f;
    const float inv = __frcp_rn(g.A);
    const float fs = (float)s;
    int n = 0;
    int64_t pos = row_ptr ? row_ptr[row] : 0;
    for (int v = 0; v < nv; ++v) {
        const float c = __fmaf_rn(g.B, (float)v, g.T0);
        const float e1 = (fs - half - c) * inv, e2 = (fs + half - c) * inv;
        const int u0 = max((int)floorf(fminf(e1, e2) - 1e-3f), 0);
        const int u1 = min((int)ceilf(fmaxf(e1, e2) + 1e-3f), nu - 1);
        for (int u = u0; u <= u1; ++u) {
            const float d = __fsub_rn(__fmaf_rn(g.A, (float)u, c), fs);
            const float w = tap_weight<KERNEL>(g, d);
            if (w == 0.0f) continue;
            const int pix = g.rows_are_y ? u + nx * v : v + nx * u;
            if (supp && !supp[pix]) continue;
            if (row_ptr) entries[pos++] = make_int2(pix, __float_as_int(DERIV ? tap_dweight<KERNEL>(g, d) : w));
            ++n;
        }
    }
    if (!row_ptr) counts[row] = n;
}

// Raw channel loads of the table-driven forward: 8 channels kept as loaded (2 x float4, or 8 BF16 in a uint4) until
// their FMAs, so that a warp can hold many taps' loads in flight in few registers.
template <typename IT> struct Raw8;
template <> struct Raw8<float> { float4 a, b; };
template <> struct Raw8<__nv_bfloat16> { uint4 u; };

__device__ __forceinline__ void ldraw(const float *p, Raw8<float> &r) { ld8(p, r.a, r.b); }
__device__ __forceinline__ void ldraw(const __nv_bfloat16 *p, Raw8<__nv_bfloat16> &r)
{
    r.u = __ldg(reinterpret_cast<const uint4 *>(p));
}
__device__ __forceinline__ void zraw(Raw8<float> &r) { r.a = r.b = make_float4(0.f, 0.f, 0.f, 0.f); }
__device__ __forceinline__ void zraw(Raw8<__nv_bfloat16> &r) { r.u = make_uint4(0, 0, 0, 0); }
__device__ __forceinline__ void accraw(float (&a)[CPL], float w, const Raw8<float> &r) { acc8(a, w, r.a, r.b); }
__device__ __forceinline__ void accraw(float (&a)[CPL], float w, const Raw8<__nv_bfloat16> &r)
{
    acc8(a, w, make_float4(bf_lo(r.u.x), bf_hi(r.u.x), bf_lo(r.u.y), bf_hi(r.u.y)),
         make_float4(bf_lo(r.u.z), bf_hi(r.u.z), bf_lo(r.u.w), bf_hi(r.u.w)));
}

// Table-driven forward: warp per (angle, bin, 256 channels), angle a of the launch = angles[a] of the table (angles
// NULL: a); the same taps, weights and summation order as radon_forward_v4, so the same bits. U taps are loaded
// before their FMAs (16 for a BF16 image: 0.32 -> 0.28 ms per ti256 launch of 18 angles x 1012 channels).
template <typename ST, typename IT>
__global__ void __launch_bounds__(32 * WARPS) radon_forward_table(
    const IT *__restrict__ img, ST *__restrict__ sino, int64_t sld, const int32_t *__restrict__ row_ptr,
    const int2 *__restrict__ entries, const int32_t *__restrict__ angles, int ns, int kstride, int kb, float scale)
{
    constexpr int U = sizeof(IT) == 2 ? 16 : 8;   // taps in flight: 16 x 16 bytes (BF16), 8 x 32 bytes (float32)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int s = blockIdx.x * WARPS + warp;
    const int al = blockIdx.y;
    const int k = blockIdx.z * CPW + lane * CPL;
    if (s >= ns) return;
    const bool live = k < kstride;
    ST *out = sino + ((int64_t)al * ns + s) * sld + k;
    if (blockIdx.z * CPW >= kb) {
        const float zero[CPL] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (live) st8(out, zero);
        return;
    }
    const bool load = k < kb;
    const int a = angles ? __ldg(angles + al) : al;
    const int64_t r = (int64_t)a * ns + s;
    int e = __ldg(row_ptr + r);
    const int e1 = __ldg(row_ptr + r + 1);
    const IT *base = img + (load ? k : 0);
    float acc[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c) acc[c] = 0.0f;
    for (; e + U <= e1; e += U) {
        int2 t[U];
        Raw8<IT> q[U];
#pragma unroll
        for (int i = 0; i < U; ++i) t[i] = __ldg(entries + e + i);
#pragma unroll
        for (int i = 0; i < U; ++i) {
            zraw(q[i]);
            if (load) ldraw(base + (int64_t)t[i].x * kstride, q[i]);
        }
#pragma unroll
        for (int i = 0; i < U; ++i) accraw(acc, __int_as_float(t[i].y), q[i]);
    }
    for (; e < e1; ++e) {
        const int2 t = __ldg(entries + e);
        Raw8<IT> q;
        zraw(q);
        if (load) ldraw(base + (int64_t)t.x * kstride, q);
        accraw(acc, __int_as_float(t.y), q);
    }
    if (!live) return;
    float o[CPL];
#pragma unroll
    for (int q = 0; q < CPL; ++q) o[q] = (k + q < kb) ? __fmul_rn(scale, acc[q]) : 0.0f;
    st8(out, o);
}

// ------------------------------------------------------------------------------------------------ grouped table
// The float32 forward reads each pixel of a row about twice per angle through the per-bin table: a pixel's footprint
// covers two bins (more for steep trapezoids), and every bin's warp loads it again. The grouped table lists, per
// (angle, group of GB consecutive bins), every pixel that reaches one of the group's bins, with its weight on each
// of them (0 where the per-bin row has no entry), in the per-bin rows' order (image row v, then u): one warp loads a
// pixel's channels once for the whole group, and every bin still adds exactly its per-bin row's taps in its order,
// so the sums are the per-bin forward's bits.
constexpr int GB = 4;           // bins per group

template <int KERNEL>
__global__ void ray_gtable_kernel(const float4 *__restrict__ geo, int n_angles, int nx, int ny, int ns,
                                  const uint8_t *__restrict__ supp, int32_t *__restrict__ counts,
                                  const int32_t *__restrict__ row_ptr, int32_t *__restrict__ pix_out,
                                  float4 *__restrict__ w_out)
{
    const int ng = (ns + GB - 1) / GB;
    const int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;      // a * ng + g
    if (row >= (int64_t)n_angles * ng) return;
    const int a = (int)(row / ng), s0 = (int)(row % ng) * GB;
    const AngleGeo g = load_geo(geo, a);
    const int nu = g.rows_are_y ? nx : ny, nv = g.rows_are_y ? ny : nx;
    const float half = KERNEL == 1 ? g.hw : 1.0f;
    const float inv = __frcp_rn(g.A);
    int n = 0;
    int64_t pos = row_ptr ? row_ptr[row] : 0;
    for (int v = 0; v < nv; ++v) {
        const float c = __fmaf_rn(g.B, (float)v, g.T0);
        int u0[GB], u1[GB];
        int lo = nu, hi = -1;
#pragma unroll
        for (int j = 0; j < GB; ++j) {                    // each bin's candidate range, as the per-bin table's
            const float fs = (float)(s0 + j);
            const float e1 = (fs - half - c) * inv, e2 = (fs + half - c) * inv;
            u0[j] = max((int)floorf(fminf(e1, e2) - 1e-3f), 0);
            u1[j] = min((int)ceilf(fmaxf(e1, e2) + 1e-3f), nu - 1);
            if (s0 + j >= ns) u1[j] = -1;
            if (u0[j] <= u1[j]) {
                lo = min(lo, u0[j]);
                hi = max(hi, u1[j]);
            }
        }
        for (int u = lo; u <= hi; ++u) {
            float w[GB];
            bool any = false;
#pragma unroll
            for (int j = 0; j < GB; ++j) {
                w[j] = 0.0f;
                if (u < u0[j] || u > u1[j]) continue;
                const float d = __fsub_rn(__fmaf_rn(g.A, (float)u, c), (float)(s0 + j));
                w[j] = tap_weight<KERNEL>(g, d);
                any |= w[j] != 0.0f;
            }
            if (!any) continue;
            const int pix = g.rows_are_y ? u + nx * v : v + nx * u;
            if (supp && !supp[pix]) continue;
            if (row_ptr) {
                pix_out[pos] = pix;
                w_out[pos++] = make_float4(w[0], w[1], w[2], w[3]);
            }
            ++n;
        }
    }
    if (!row_ptr) counts[row] = n;
}

// Grouped-table forward (float32 image and sinogram rows): warp per (angle, GB bins, 256 channels); U pixels in
// flight, each pixel's FMAs into the bins whose weight is not 0 (a branch the whole warp takes).
__global__ void __launch_bounds__(32 * WARPS) radon_forward_gtable(
    const float *__restrict__ img, float *__restrict__ sino, const int32_t *__restrict__ row_ptr,
    const int32_t *__restrict__ pix, const float4 *__restrict__ wts, const int32_t *__restrict__ angles, int ns,
    int kstride, int kb, float scale)
{
    constexpr int U = 4;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ng = (ns + GB - 1) / GB;
    const int grp = blockIdx.x * WARPS + warp;
    const int al = blockIdx.y;
    const int k = blockIdx.z * CPW + lane * CPL;
    if (grp >= ng) return;
    const bool live = k < kstride;
    const int s0 = grp * GB;
    float *out = sino + ((int64_t)al * ns + s0) * kstride + k;
    const int nb = min(GB, ns - s0);
    if (blockIdx.z * CPW >= kb) {
        const float zero[CPL] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (live)
            for (int j = 0; j < nb; ++j) st8(out + (int64_t)j * kstride, zero);
        return;
    }
    const bool load = k < kb;
    const int a = angles ? __ldg(angles + al) : al;
    const int64_t r = (int64_t)a * ng + grp;
    int e = __ldg(row_ptr + r);
    const int e1 = __ldg(row_ptr + r + 1);
    const float *base = img + (load ? k : 0);
    float acc[GB][CPL];
#pragma unroll
    for (int j = 0; j < GB; ++j)
#pragma unroll
        for (int c = 0; c < CPL; ++c) acc[j][c] = 0.0f;
    for (; e + U <= e1; e += U) {
        int p[U];
        float4 w[U];
        Raw8<float> q[U];
#pragma unroll
        for (int i = 0; i < U; ++i) {
            p[i] = __ldg(pix + e + i);
            w[i] = __ldg(wts + e + i);
        }
#pragma unroll
        for (int i = 0; i < U; ++i) {
            zraw(q[i]);
            if (load) ldraw(base + (int64_t)p[i] * kstride, q[i]);
        }
#pragma unroll
        for (int i = 0; i < U; ++i) {
            if (w[i].x != 0.0f) accraw(acc[0], w[i].x, q[i]);
            if (w[i].y != 0.0f) accraw(acc[1], w[i].y, q[i]);
            if (w[i].z != 0.0f) accraw(acc[2], w[i].z, q[i]);
            if (w[i].w != 0.0f) accraw(acc[3], w[i].w, q[i]);
        }
    }
    for (; e < e1; ++e) {
        const int p = __ldg(pix + e);
        const float4 w = __ldg(wts + e);
        Raw8<float> q;
        zraw(q);
        if (load) ldraw(base + (int64_t)p * kstride, q);
        if (w.x != 0.0f) accraw(acc[0], w.x, q);
        if (w.y != 0.0f) accraw(acc[1], w.y, q);
        if (w.z != 0.0f) accraw(acc[2], w.z, q);
        if (w.w != 0.0f) accraw(acc[3], w.w, q);
    }
    if (!live) return;
#pragma unroll
    for (int j = 0; j < GB; ++j) {
        if (j >= nb) break;
        float o[CPL];
#pragma unroll
        for (int q = 0; q < CPL; ++q) o[q] = (k + q < kb) ? __fmul_rn(scale, acc[j][q]) : 0.0f;
        st8(out + (int64_t)j * kstride, o);
    }
}

// ------------------------------------------------------------------------------------------------ backward
// SPDHG primal step of one coefficient: the operations of primal_update_kernel (solver.cu), bitwise
__device__ __forceinline__ void primal_step(float &x, float &z, float t, float dz, float inv_p, float lam)
{
    const float zi = __fadd_rn(z, dz);
    z = zi;
    const float zb = __fadd_rn(zi, __fmul_rn(inv_p, dz));
    x = t > 0.0f ? fmaxf(0.0f, __fsub_rn(x, __fmul_rn(t, __fadd_rn(zb, lam)))) : 0.0f;
}

// MODE 0: img (npix, kstride) = backprojection; MODE 1: the backprojection dz is applied to x, z (T the steps):
// z += dz; x = T > 0 ? max(0, x - T (z + inv_p dz + lam)) : 0. plist (MODE 0, optional): only the pixels plist[0 ..
// n_out-1], output row r for pixel plist[r] (the same arithmetic per pixel as the whole image).
// P channel groups of 256 per warp (lane: channels k, k + 256, ...): the pixel's taps and weights are computed once for
// P x 8 channels per lane, which halves the geometry work per FMA at P = 2; every channel sums the same terms in the
// same order whatever P is.
template <int KERNEL, int MODE, typename ST, int P>
__global__ void __launch_bounds__(32 * WARPS) radon_backward_v3(
    const ST *__restrict__ sino, int64_t sld, float *__restrict__ img, const float4 *__restrict__ geo, int n_angles, int nx,
    int ny, int ns, int kstride, int kb, int n_taps, float *__restrict__ z, const float *__restrict__ T, float inv_p,
    float lam, __nv_bfloat16 *__restrict__ xb, const int32_t *__restrict__ plist, int64_t n_out)
{
    extern __shared__ AngleParams prm[];                   // the constants of every angle
    for (int i = threadIdx.x; i < n_angles; i += blockDim.x) prm[i] = pack_geo(load_geo(geo, i));
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t p = (int64_t)blockIdx.x * WARPS + warp;     // output row
    const int kblk = blockIdx.y * CPW * P;
    if (p >= n_out || kblk + lane * CPL >= kstride) return;
    // group h: channels kblk + h CPW + lane CPL (+0..7); live: inside kstride; data: not a block of padding only
    bool live[P], data[P];
#pragma unroll
    for (int h = 0; h < P; ++h) {
        live[h] = kblk + h * CPW + lane * CPL < kstride;
        data[h] = live[h] && kblk + h * CPW < kb;
    }
    const int64_t pix = plist ? (int64_t)__ldg(plist + p) : p;
    if (!data[0]) {                        // padding channels only: the backprojection is 0 there
        if (MODE == 0) {
            const float zero[CPL] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int h = 0; h < P; ++h)
                if (live[h]) st8(img + p * kstride + kblk + h * CPW + lane * CPL, zero);
        }
        return;                            // MODE 1: dz = 0 leaves z, and x (0 on padding channels), unchanged
    }
    const int px = (int)(pix % nx), py = (int)(pix / nx);
    const float fx = (float)px, fy = (float)py;
    float acc[P][CPL];
#pragma unroll
    for (int h = 0; h < P; ++h)
#pragma unroll
        for (int c = 0; c < CPL; ++c) acc[h][c] = 0.0f;
    const ST *col = sino + kblk + lane * CPL;
    const int64_t angle_stride = (int64_t)ns * sld;
    for (int a = 0; a < n_angles; ++a, col += angle_stride) {
        const AngleGeo g = unpack_geo(prm[a]);
        const float t = __fmaf_rn(g.A, g.rows_are_y ? fx : fy, __fmaf_rn(g.B, g.rows_are_y ? fy : fx, g.T0));
        const int sf = first_tap<KERNEL>(g, t);
        const int ntap = taps_of(g, KERNEL, n_taps);
        if (ntap == 2 && sf >= 0 && sf + 1 < ns) {        // the common case: two taps inside the detector
            const float w0 = __fmul_rn(g.w, tap_weight<KERNEL>(g, __fsub_rn(t, (float)sf)));
            const float w1 = __fmul_rn(g.w, tap_weight<KERNEL>(g, __fsub_rn(t, (float)(sf + 1))));
#pragma unroll
            for (int h = 0; h < P; ++h) {
                if (!data[h]) continue;
                float4 a0, a1, b0, b1;
                ld8(col + h * CPW + (int64_t)sf * sld, a0, a1);
                ld8(col + h * CPW + (int64_t)(sf + 1) * sld, b0, b1);
                acc8(acc[h], w0, a0, a1);
                acc8(acc[h], w1, b0, b1);
            }
            continue;
        }
        for (int i = 0; i < ntap; ++i) {
            const int s = sf + i;
            if (s < 0 || s >= ns) continue;
            const float w = tap_weight<KERNEL>(g, __fsub_rn(t, (float)s));
            if (w == 0.0f) continue;
            const float ww = __fmul_rn(g.w, w);
#pragma unroll
            for (int h = 0; h < P; ++h) {
                if (!data[h]) continue;
                float4 q0, q1;
                ld8(col + h * CPW + (int64_t)s * sld, q0, q1);
                acc8(acc[h], ww, q0, q1);
            }
        }
    }
#pragma unroll
    for (int h = 0; h < P; ++h) {
        const int k = kblk + h * CPW + lane * CPL;
        const int64_t o = p * kstride + k;
        if (MODE == 0) {
            if (!live[h]) continue;
            float r[CPL];
#pragma unroll
            for (int c = 0; c < CPL; ++c) r[c] = (data[h] && k + c < kb) ? acc[h][c] : 0.0f;   // padding: 0
            float4 *d = reinterpret_cast<float4 *>(img + o);
            d[0] = make_float4(r[0], r[1], r[2], r[3]);
            d[1] = make_float4(r[4], r[5], r[6], r[7]);
        } else {
            if (!data[h]) continue;
            float xn[CPL];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                float4 *xp = reinterpret_cast<float4 *>(img + o) + q;
                float4 *zp = reinterpret_cast<float4 *>(z + o) + q;
                float4 xv = *xp, zv = *zp;
                const float4 tv = __ldg(reinterpret_cast<const float4 *>(T + o) + q);
                primal_step(xv.x, zv.x, tv.x, (k + 4 * q + 0 < kb) ? acc[h][4 * q + 0] : 0.0f, inv_p, lam);
                primal_step(xv.y, zv.y, tv.y, (k + 4 * q + 1 < kb) ? acc[h][4 * q + 1] : 0.0f, inv_p, lam);
                primal_step(xv.z, zv.z, tv.z, (k + 4 * q + 2 < kb) ? acc[h][4 * q + 2] : 0.0f, inv_p, lam);
                primal_step(xv.w, zv.w, tv.w, (k + 4 * q + 3 < kb) ? acc[h][4 * q + 3] : 0.0f, inv_p, lam);
                *xp = xv;
                *zp = zv;
                xn[4 * q] = xv.x; xn[4 * q + 1] = xv.y; xn[4 * q + 2] = xv.z; xn[4 * q + 3] = xv.w;
            }
            if (xb) st8(xb + o, xn);       // the BF16 copy of x the next forward projection reads
        }
    }
}

// ------------------------------------------------------------------------------------------------ batch helpers
// Element-wise on channel-fastest batches (npix, kstride) whose channels kb .. kstride-1 are padding:
// mode 0: x = 1 inside the support on live channels, else 0 (support_ones); mode 1: x = 0 outside the support, on
// padding channels or where negative (project_support); mode 2: T = min(T, c / colsum) inside the support where
// colsum > 0 (tmin).
__global__ void batch_support_kernel(float *__restrict__ x, const float *__restrict__ colsum,
                                     const uint8_t *__restrict__ supp, int64_t npix, int kstride, int kb, float c,
                                     int mode)
{
    const int64_t n = npix * kstride;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = i / kstride;
        const int k = (int)(i - p * kstride);
        const bool inside = (supp ? __ldg(supp + p) != 0 : true) && k < kb;
        if (mode == 0) {
            x[i] = inside ? 1.0f : 0.0f;
        } else if (mode == 1) {
            if (!inside || x[i] < 0.0f) x[i] = 0.0f;
        } else if (mode == 3) {
            if (!inside) x[i] = 0.0f;
        } else {
            const float cs = colsum[i];
            if (inside && cs > 0.0f) x[i] = fminf(x[i], __fdiv_rn(c, cs));
        }
    }
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
    DFX_REQUIRE(kstride > 0 && kstride % CPL == 0 && kb >= 0 && kb <= kstride,
                "radon: kstride (%d) must be a positive multiple of %d and kb (%d) <= kstride", kstride, CPL, kb);
    DFX_REQUIRE(kernel == 0 || kernel == 1, "radon: kernel must be 0 (hat) or 1 (trapezoid)");
    DFX_REQUIRE(((uintptr_t)in % 16) == 0 && ((uintptr_t)out % 16) == 0 && ((uintptr_t)geo % 16) == 0,
                "radon: arrays must be 16-byte aligned");
    DFX_REQUIRE((int64_t)nx * ny * kstride < ((int64_t)1 << 40), "radon: image batch too large");
    return DFX_OK;
}

template <typename Kernel>
static int allow_smem(Kernel kernel, size_t bytes)
{
    if (bytes <= 48 * 1024) return DFX_OK;
    const cudaError_t e = allow_max_dynamic_smem(kernel);
    if (e != cudaSuccess) {
        set_error("radon: %zu bytes of shared memory: %s", bytes, cudaGetErrorString(e));
        return DFX_ECUDA;
    }
    return DFX_OK;
}

template <int KERNEL, int MODE, typename ST>
static int launch_backward(const ST *sino, int64_t sld, float *img, const float *geo, int n_angles, int nx, int ny,
                           int n_det, int kstride, int kb, int n_taps, float *z, const float *T, float inv_p, float lam,
                           __nv_bfloat16 *xb, void *stream, const int32_t *plist = nullptr, int64_t n_list = 0)
{
    const int64_t npix = plist ? n_list : (int64_t)nx * ny;
    // two channel groups per warp once the batch has more than one (fewer, longer warps: the taps of a pixel are
    // evaluated once for 16 channels per lane)
    const bool pair = kstride > CPW;
    dim3 grid((unsigned)cdiv(npix, WARPS), (unsigned)cdiv(kstride, pair ? 2 * CPW : CPW));
    DFX_REQUIRE(grid.x < 2147483647u && grid.y <= 65535u, "radon: batch too large for one launch");
    const size_t smem = sizeof(AngleParams) * (size_t)(n_angles > 0 ? n_angles : 1);
    DFX_REQUIRE(smem <= 200 * 1024, "radon: %d angles exceed the shared memory of one launch", n_angles);
    int st = pair ? allow_smem(radon_backward_v3<KERNEL, MODE, ST, 2>, smem)
                  : allow_smem(radon_backward_v3<KERNEL, MODE, ST, 1>, smem);
    if (st) return st;
    if (pair)
        radon_backward_v3<KERNEL, MODE, ST, 2><<<grid, 32 * WARPS, smem, (cudaStream_t)stream>>>(
            sino, sld, img, reinterpret_cast<const float4 *>(geo), n_angles, nx, ny, n_det, kstride, kb, n_taps, z, T,
            inv_p, lam, xb, plist, npix);
    else
        radon_backward_v3<KERNEL, MODE, ST, 1><<<grid, 32 * WARPS, smem, (cudaStream_t)stream>>>(
            sino, sld, img, reinterpret_cast<const float4 *>(geo), n_angles, nx, ny, n_det, kstride, kb, n_taps, z, T,
            inv_p, lam, xb, plist, npix);
    return launch_status(MODE ? "radon_backward_spdhg" : "radon_backward");
}

}  // namespace dfx

using namespace dfx;

template <typename ST>
static int radon_forward_any(const float *img_k, ST *sino, int64_t sld, const float *geo, int n_angles, int nx, int ny,
                             int n_det, int kstride, int kb, int kernel, float scale, void *stream)
{
    int st = check_radon_args(img_k, sino, geo, n_angles, nx, ny, n_det, kstride, kb, kernel);
    if (st) return st;
    DFX_REQUIRE(sld >= kstride && sld % CPL == 0, "radon: sinogram row stride (%lld) must be a multiple of %d >= "
                "kstride", (long long)sld, CPL);
    if (n_angles == 0) return DFX_OK;
    DFX_REQUIRE(n_angles <= 65535, "radon: at most 65535 angles per launch");
    DFX_REQUIRE(cdiv(kstride, CPW) <= 65535, "radon: kstride too large for one launch");
    dim3 grid((unsigned)cdiv(n_det, WARPS), (unsigned)n_angles, (unsigned)cdiv(kstride, CPW));
    if (kernel == 1)
        radon_forward_v4<1, ST><<<grid, 32 * WARPS, 0, (cudaStream_t)stream>>>(
            img_k, sino, sld, reinterpret_cast<const float4 *>(geo), nx, ny, n_det, kstride, kb, scale);
    else
        radon_forward_v4<0, ST><<<grid, 32 * WARPS, 0, (cudaStream_t)stream>>>(
            img_k, sino, sld, reinterpret_cast<const float4 *>(geo), nx, ny, n_det, kstride, kb, scale);
    return launch_status("radon_forward");
}

template <typename ST, typename IT>
static int radon_forward_table_any(const IT *img_k, ST *sino, int64_t sld, const int32_t *row_ptr,
                                   const int32_t *entries, const int32_t *angles, int n_angles, int n_det,
                                   int kstride, int kb, float scale, void *stream)
{
    DFX_REQUIRE(img_k && sino && row_ptr && entries, "radon_forward_table: null pointer");
    DFX_REQUIRE(((uintptr_t)img_k % 16) == 0 && ((uintptr_t)sino % 16) == 0 && ((uintptr_t)entries % 8) == 0,
                "radon_forward_table: misaligned arrays");
    DFX_REQUIRE(n_angles >= 0 && n_angles <= 65535 && n_det > 0, "radon_forward_table: bad sizes");
    DFX_REQUIRE(kstride > 0 && kstride % CPL == 0 && kb >= 0 && kb <= kstride && cdiv(kstride, CPW) <= 65535,
                "radon_forward_table: kstride (%d) must be a positive multiple of %d and kb (%d) <= kstride",
                kstride, CPL, kb);
    DFX_REQUIRE(sld >= kstride && sld % CPL == 0, "radon_forward_table: sinogram row stride (%lld) must be a "
                "multiple of %d >= kstride", (long long)sld, CPL);
    if (n_angles == 0) return DFX_OK;
    dim3 grid((unsigned)cdiv(n_det, WARPS), (unsigned)n_angles, (unsigned)cdiv(kstride, CPW));
    radon_forward_table<ST, IT><<<grid, 32 * WARPS, 0, (cudaStream_t)stream>>>(
        img_k, sino, sld, row_ptr, reinterpret_cast<const int2 *>(entries), angles, n_det, kstride, kb, scale);
    return launch_status("radon_forward_table");
}

template <int MODE, typename ST>
static int radon_backward_any(const ST *sino, int64_t sld, float *img_k, const float *geo, int n_angles, int nx,
                              int ny, int n_det, int kstride, int kb, int kernel, int n_taps, float *z_k,
                              const float *T_k, float inv_p, float lam, void *stream,
                              __nv_bfloat16 *xb = nullptr)
{
    int st = check_radon_args(sino, img_k, geo, n_angles, nx, ny, n_det, kstride, kb, kernel);
    if (st) return st;
    DFX_REQUIRE(sld >= kstride && sld % CPL == 0, "radon: sinogram row stride (%lld) must be a multiple of %d >= "
                "kstride", (long long)sld, CPL);
    DFX_REQUIRE(MODE == 0 || (z_k && T_k && ((uintptr_t)z_k % 16) == 0 && ((uintptr_t)T_k % 16) == 0),
                "radon_backward_spdhg: z and T must be 16-byte aligned device arrays");
    DFX_REQUIRE(n_taps >= 2 && n_taps <= 64, "radon: n_taps (%d) out of range", n_taps);
    if (kernel == 1)
        return launch_backward<1, MODE, ST>(sino, sld, img_k, geo, n_angles, nx, ny, n_det, kstride, kb, n_taps, z_k,
                                            T_k, inv_p, lam, xb, stream);
    return launch_backward<0, MODE, ST>(sino, sld, img_k, geo, n_angles, nx, ny, n_det, kstride, kb, n_taps, z_k, T_k,
                                        inv_p, lam, xb, stream);
}

extern "C" int dfx_radon_forward(const float *img_k, float *sino_k, const float *geo, int n_angles, int nx, int ny,
                                 int n_det, int kstride, int kb, int kernel, float scale, void *stream)
{
    return radon_forward_any(img_k, sino_k, (int64_t)kstride, geo, n_angles, nx, ny, n_det, kstride, kb, kernel,
                             scale, stream);
}

extern "C" int dfx_radon_forward_bf16(const float *img_k, void *sino_bf16, int64_t sino_ld, const float *geo,
                                      int n_angles, int nx, int ny, int n_det, int kstride, int kb, int kernel,
                                      float scale, void *stream)
{
    return radon_forward_any(img_k, reinterpret_cast<__nv_bfloat16 *>(sino_bf16), sino_ld, geo, n_angles, nx, ny,
                             n_det, kstride, kb, kernel, scale, stream);
}

extern "C" int dfx_radon_backward_pixels(const float *sino_k, float *img_k, const float *geo, int n_angles, int nx,
                                         int ny, int n_det, int kstride, int kb, int kernel, int n_taps,
                                         const int32_t *pixels, int64_t n_pix, void *stream)
{
    int st = check_radon_args(sino_k, img_k, geo, n_angles, nx, ny, n_det, kstride, kb, kernel);
    if (st) return st;
    DFX_REQUIRE(pixels && n_pix > 0 && n_pix <= (int64_t)nx * ny, "radon_backward_pixels: bad pixel list");
    DFX_REQUIRE(n_taps >= 2 && n_taps <= 64, "radon: n_taps (%d) out of range", n_taps);
    if (kernel == 1)
        return launch_backward<1, 0, float>(sino_k, (int64_t)kstride, img_k, geo, n_angles, nx, ny, n_det, kstride, kb,
                                            n_taps, nullptr, nullptr, 0.0f, 0.0f, nullptr, stream, pixels, n_pix);
    return launch_backward<0, 0, float>(sino_k, (int64_t)kstride, img_k, geo, n_angles, nx, ny, n_det, kstride, kb,
                                        n_taps, nullptr, nullptr, 0.0f, 0.0f, nullptr, stream, pixels, n_pix);
}

extern "C" int dfx_radon_backward(const float *sino_k, float *img_k, const float *geo, int n_angles, int nx, int ny,
                                  int n_det, int kstride, int kb, int kernel, int n_taps, void *stream)
{
    return radon_backward_any<0>(sino_k, (int64_t)kstride, img_k, geo, n_angles, nx, ny, n_det, kstride, kb, kernel,
                                 n_taps, nullptr, nullptr, 0.0f, 0.0f, stream);
}

extern "C" int dfx_radon_backward_bf16(const void *sino_bf16, int64_t sino_ld, float *img_k, const float *geo,
                                       int n_angles, int nx, int ny, int n_det, int kstride, int kb, int kernel,
                                       int n_taps, void *stream)
{
    return radon_backward_any<0>(reinterpret_cast<const __nv_bfloat16 *>(sino_bf16), sino_ld, img_k, geo, n_angles, nx,
                                 ny, n_det, kstride, kb, kernel, n_taps, nullptr, nullptr, 0.0f, 0.0f, stream);
}

extern "C" int dfx_radon_backward_spdhg(const float *sino_k, const float *geo, int n_angles, int nx, int ny, int n_det,
                                        int kstride, int kb, int kernel, int n_taps, float *x_k, float *z_k,
                                        const float *T_k, float inv_p, float lam, void *stream)
{
    return radon_backward_any<1>(sino_k, (int64_t)kstride, x_k, geo, n_angles, nx, ny, n_det, kstride, kb, kernel,
                                 n_taps, z_k, T_k, inv_p, lam, stream);
}

extern "C" int dfx_radon_backward_spdhg_bf16(const void *sino_bf16, int64_t sino_ld, const float *geo, int n_angles,
                                             int nx, int ny, int n_det, int kstride, int kb, int kernel, int n_taps,
                                             float *x_k, float *z_k, const float *T_k, float inv_p, float lam,
                                             void *x_bf16, void *stream)
{
    DFX_REQUIRE(((uintptr_t)x_bf16 % 16) == 0, "radon_backward_spdhg_bf16: x_bf16 must be 16-byte aligned");
    return radon_backward_any<1>(reinterpret_cast<const __nv_bfloat16 *>(sino_bf16), sino_ld, x_k, geo, n_angles, nx,
                                 ny, n_det, kstride, kb, kernel, n_taps, z_k, T_k, inv_p, lam, stream,
                                 reinterpret_cast<__nv_bfloat16 *>(x_bf16));
}

extern "C" int dfx_radon_table_count(const float *geo, int n_angles, int nx, int ny, int n_det, int kernel,
                                     const uint8_t *supp, int32_t *counts, void *stream)
{
    DFX_REQUIRE(geo && counts && ((uintptr_t)geo % 16) == 0, "radon_table: null or misaligned pointer");
    DFX_REQUIRE(n_angles > 0 && nx > 0 && ny > 0 && n_det > 0 && (kernel == 0 || kernel == 1),
                "radon_table: bad sizes or kernel");
    const int64_t rows = (int64_t)n_angles * n_det;
    DFX_REQUIRE(cdiv(rows, 128) < 2147483647LL, "radon_table: too many rows");
    if (kernel == 1)
        ray_table_kernel<1><<<(unsigned)cdiv(rows, 128), 128, 0, (cudaStream_t)stream>>>(
            reinterpret_cast<const float4 *>(geo), n_angles, nx, ny, n_det, supp, counts, nullptr, nullptr);
    else
        ray_table_kernel<0><<<(unsigned)cdiv(rows, 128), 128, 0, (cudaStream_t)stream>>>(
            reinterpret_cast<const float4 *>(geo), n_angles, nx, ny, n_det, supp, counts, nullptr, nullptr);
    return launch_status("radon_table_count");
}

extern "C" int dfx_radon_table_fill(const float *geo, int n_angles, int nx, int ny, int n_det, int kernel,
                                    const uint8_t *supp, const int32_t *row_ptr, int32_t *entries, void *stream)
{
    DFX_REQUIRE(geo && row_ptr && entries && ((uintptr_t)geo % 16) == 0 && ((uintptr_t)entries % 8) == 0,
                "radon_table: null or misaligned pointer");
    DFX_REQUIRE(n_angles > 0 && nx > 0 && ny > 0 && n_det > 0 && (kernel == 0 || kernel == 1),
                "radon_table: bad sizes or kernel");
    const int64_t rows = (int64_t)n_angles * n_det;
    int2 *e = reinterpret_cast<int2 *>(entries);
    if (kernel == 1)
        ray_table_kernel<1><<<(unsigned)cdiv(rows, 128), 128, 0, (cudaStream_t)stream>>>(
            reinterpret_cast<const float4 *>(geo), n_angles, nx, ny, n_det, supp, nullptr, row_ptr, e);
    else
        ray_table_kernel<0><<<(unsigned)cdiv(rows, 128), 128, 0, (cudaStream_t)stream>>>(
            reinterpret_cast<const float4 *>(geo), n_angles, nx, ny, n_det, supp, nullptr, row_ptr, e);
    return launch_status("radon_table_fill");
}

extern "C" int dfx_radon_gtable_count(const float *geo, int n_angles, int nx, int ny, int n_det, int kernel,
                                      const uint8_t *supp, int32_t *counts, void *stream)
{
    DFX_REQUIRE(geo && counts && ((uintptr_t)geo % 16) == 0, "radon_gtable: null or misaligned pointer");
    DFX_REQUIRE(n_angles > 0 && nx > 0 && ny > 0 && n_det > 0 && (kernel == 0 || kernel == 1),
                "radon_gtable: bad sizes or kernel");
    const int64_t rows = (int64_t)n_angles * cdiv(n_det, GB);
    DFX_REQUIRE(cdiv(rows, 128) < 2147483647LL, "radon_gtable: too many rows");
    if (kernel == 1)
        ray_gtable_kernel<1><<<(unsigned)cdiv(rows, 128), 128, 0, (cudaStream_t)stream>>>(
            reinterpret_cast<const float4 *>(geo), n_angles, nx, ny, n_det, supp, counts, nullptr, nullptr, nullptr);
    else
        ray_gtable_kernel<0><<<(unsigned)cdiv(rows, 128), 128, 0, (cudaStream_t)stream>>>(
            reinterpret_cast<const float4 *>(geo), n_angles, nx, ny, n_det, supp, counts, nullptr, nullptr, nullptr);
    return launch_status("radon_gtable_count");
}

extern "C" int dfx_radon_gtable_fill(const float *geo, int n_angles, int nx, int ny, int n_det, int kernel,
                                     const uint8_t *supp, const int32_t *row_ptr, int32_t *pixels, float *weights,
                                     void *stream)
{
    DFX_REQUIRE(geo && row_ptr && pixels && weights && ((uintptr_t)geo % 16) == 0 && ((uintptr_t)weights % 16) == 0,
                "radon_gtable: null or misaligned pointer");
    DFX_REQUIRE(n_angles > 0 && nx > 0 && ny > 0 && n_det > 0 && (kernel == 0 || kernel == 1),
                "radon_gtable: bad sizes or kernel");
    const int64_t rows = (int64_t)n_angles * cdiv(n_det, GB);
    float4 *w = reinterpret_cast<float4 *>(weights);
    if (kernel == 1)
        ray_gtable_kernel<1><<<(unsigned)cdiv(rows, 128), 128, 0, (cudaStream_t)stream>>>(
            reinterpret_cast<const float4 *>(geo), n_angles, nx, ny, n_det, supp, nullptr, row_ptr, pixels, w);
    else
        ray_gtable_kernel<0><<<(unsigned)cdiv(rows, 128), 128, 0, (cudaStream_t)stream>>>(
            reinterpret_cast<const float4 *>(geo), n_angles, nx, ny, n_det, supp, nullptr, row_ptr, pixels, w);
    return launch_status("radon_gtable_fill");
}

extern "C" int dfx_radon_forward_gtable(const float *img_k, float *sino_k, const int32_t *row_ptr,
                                        const int32_t *pixels, const float *weights, const int32_t *angles,
                                        int n_angles, int n_det, int kstride, int kb, float scale, void *stream)
{
    DFX_REQUIRE(img_k && sino_k && row_ptr && pixels && weights, "radon_forward_gtable: null pointer");
    DFX_REQUIRE(((uintptr_t)img_k % 16) == 0 && ((uintptr_t)sino_k % 16) == 0 && ((uintptr_t)weights % 16) == 0,
                "radon_forward_gtable: misaligned arrays");
    DFX_REQUIRE(n_angles >= 0 && n_angles <= 65535 && n_det > 0, "radon_forward_gtable: bad sizes");
    DFX_REQUIRE(kstride > 0 && kstride % CPL == 0 && kb >= 0 && kb <= kstride && cdiv(kstride, CPW) <= 65535,
                "radon_forward_gtable: kstride (%d) must be a positive multiple of %d and kb (%d) <= kstride",
                kstride, CPL, kb);
    if (n_angles == 0) return DFX_OK;
    dim3 grid((unsigned)cdiv(cdiv(n_det, GB), WARPS), (unsigned)n_angles, (unsigned)cdiv(kstride, CPW));
    radon_forward_gtable<<<grid, 32 * WARPS, 0, (cudaStream_t)stream>>>(
        img_k, sino_k, row_ptr, pixels, reinterpret_cast<const float4 *>(weights), angles, n_det, kstride, kb, scale);
    return launch_status("radon_forward_gtable");
}

extern "C" int dfx_radon_dtable_fill(const float *geo, int n_angles, int nx, int ny, int n_det, int kernel,
                                     const int32_t *row_ptr, int32_t *entries, void *stream)
{
    DFX_REQUIRE(geo && row_ptr && entries && ((uintptr_t)geo % 16) == 0 && ((uintptr_t)entries % 8) == 0,
                "radon_dtable: null or misaligned pointer");
    DFX_REQUIRE(n_angles > 0 && nx > 0 && ny > 0 && n_det > 0 && (kernel == 0 || kernel == 1),
                "radon_dtable: bad sizes or kernel");
    const int64_t rows = (int64_t)n_angles * n_det;
    int2 *e = reinterpret_cast<int2 *>(entries);
    if (kernel == 1)
        ray_table_kernel<1, true><<<(unsigned)cdiv(rows, 128), 128, 0, (cudaStream_t)stream>>>(
            reinterpret_cast<const float4 *>(geo), n_angles, nx, ny, n_det, nullptr, nullptr, row_ptr, e);
    else
        ray_table_kernel<0, true><<<(unsigned)cdiv(rows, 128), 128, 0, (cudaStream_t)stream>>>(
            reinterpret_cast<const float4 *>(geo), n_angles, nx, ny, n_det, nullptr, nullptr, row_ptr, e);
    return launch_status("radon_dtable_fill");
}

extern "C" int dfx_radon_forward_table(const float *img_k, float *sino_k, const int32_t *row_ptr,
                                       const int32_t *entries, const int32_t *angles, int n_angles, int n_det,
                                       int kstride, int kb, float scale, void *stream)
{
    return radon_forward_table_any(img_k, sino_k, (int64_t)kstride, row_ptr, entries, angles, n_angles, n_det,
                                   kstride, kb, scale, stream);
}

extern "C" int dfx_radon_forward_table_bf16(const float *img_k, void *sino_bf16, int64_t sino_ld,
                                            const int32_t *row_ptr, const int32_t *entries, const int32_t *angles,
                                            int n_angles, int n_det, int kstride, int kb, float scale, void *stream)
{
    return radon_forward_table_any(img_k, reinterpret_cast<__nv_bfloat16 *>(sino_bf16), sino_ld, row_ptr, entries,
                                   angles, n_angles, n_det, kstride, kb, scale, stream);
}

extern "C" int dfx_radon_forward_table_bf16_bf16(const void *img_bf16, void *sino_bf16, int64_t sino_ld,
                                                 const int32_t *row_ptr, const int32_t *entries, const int32_t *angles,
                                                 int n_angles, int n_det, int kstride, int kb, float scale, void *stream)
{
    return radon_forward_table_any(reinterpret_cast<const __nv_bfloat16 *>(img_bf16),
                                   reinterpret_cast<__nv_bfloat16 *>(sino_bf16), sino_ld, row_ptr, entries, angles,
                                   n_angles, n_det, kstride, kb, scale, stream);
}

extern "C" int dfx_batch_support(float *x_k, const float *colsum_k, const uint8_t *supp, int64_t npix, int kstride,
                                 int kb, float c, int mode, void *stream)
{
    DFX_REQUIRE(x_k && npix > 0 && kstride > 0 && kb >= 0 && kb <= kstride && mode >= 0 && mode <= 3,
                "batch_support: bad arguments");
    DFX_REQUIRE(mode != 2 || colsum_k, "batch_support: tmin needs the column sums");
    const int64_t blocks = cdiv(npix * kstride, 256);
    batch_support_kernel<<<(unsigned)(blocks < 148 * 32 ? blocks : 148 * 32), 256, 0, (cudaStream_t)stream>>>(
        x_k, colsum_k, supp, npix, kstride, kb, c, mode);
    return launch_status("batch_support");
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
    if (kb == 0) return DFX_OK;
    dim3 grid((unsigned)cdiv(npix, TT), (unsigned)cdiv(kb, TT));
    DFX_REQUIRE(grid.y <= 65535u, "scatter: kb too large");
    scatter_kernel<<<grid, dim3(TT, 8), 0, (cudaStream_t)stream>>>(img_k, coeffs, npix, k0, kb, kstride);
    return launch_status("scatter_channels");
}
