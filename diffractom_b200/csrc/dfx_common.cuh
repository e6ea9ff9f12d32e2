// Shared pieces of the sm_100a kernels of diffractom_b200: status codes, the per-thread error message, launch
// checks and the float32 arithmetic conventions that the CPU oracle restates bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "../../include/diffractom_b200.h"

namespace dfx {

// Last error message of the calling host thread (dfx_last_error returns it).
void set_error(const char *fmt, ...);

// Status of the launch just issued on the calling thread (cudaGetLastError), with the kernel's name.
int launch_status(const char *what);

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Allows a kernel the device's whole opt-in shared memory (less its static shared memory) as dynamic shared memory.
// The same value on every call, so that host threads launching the kernel with different sizes concurrently (the
// serving loop) never lower the limit under another thread's launch; occupancy follows each launch's actual size.
template <typename Kernel>
inline cudaError_t allow_max_dynamic_smem(Kernel kernel)
{
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    int dev = 0, optin = 0;
    e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

#define DFX_REQUIRE(cond, ...)                  \
    do {                                        \
        if (!(cond)) {                          \
            ::dfx::set_error(__VA_ARGS__);      \
            return DFX_EINVAL;                  \
        }                                       \
    } while (0)

// ---- detector coordinate and tap weight of the parallel-beam projector (the oracle's convention) ----
// Rows run along the image axis with the larger coefficient |X| or |Y| (A); t = A u + (B v + T0) with two
// correctly rounded fused multiply-adds, so forward and backward projection see the same t and the same weights.
struct AngleGeo {
    float A, B, T0, w;     // row-axis coefficient, column coefficient, offset, angle weight
    int rows_are_y;        // 1: u = x (rows of constant y), 0: u = y
    float hw, top, iw;     // trapezoid: half width (1 + |A|) / 2, plateau min(1, |A|), 1 / |A|
};

__device__ __forceinline__ AngleGeo load_geo(const float4 *geo, int a) {
    const float4 g = __ldg(geo + a);
    AngleGeo o;
    o.rows_are_y = fabsf(g.x) >= fabsf(g.y);
    o.A = o.rows_are_y ? g.x : g.y;
    o.B = o.rows_are_y ? g.y : g.x;
    o.T0 = g.z;
    o.w = g.w;
    const float aA = fabsf(o.A);
    o.hw = __fmul_rn(0.5f, __fadd_rn(1.0f, aA));
    o.top = fminf(1.0f, aA);
    o.iw = __frcp_rn(aA);
    return o;
}

// The per-angle constants packed for shared memory: (A, B, T0, w) and (hw, top, iw, rows_are_y).
struct __align__(16) AngleParams {
    float4 abtw;
    float4 htir;
};

__device__ __forceinline__ AngleParams pack_geo(const AngleGeo &g)
{
    AngleParams p;
    p.abtw = make_float4(g.A, g.B, g.T0, g.w);
    p.htir = make_float4(g.hw, g.top, g.iw, g.rows_are_y ? 1.0f : 0.0f);
    return p;
}

__device__ __forceinline__ AngleGeo unpack_geo(const AngleParams &p)
{
    AngleGeo g;
    g.A = p.abtw.x;
    g.B = p.abtw.y;
    g.T0 = p.abtw.z;
    g.w = p.abtw.w;
    g.hw = p.htir.x;
    g.top = p.htir.y;
    g.iw = p.htir.z;
    g.rows_are_y = p.htir.w != 0.0f;
    return g;
}

// K(d) for d = t - s: trapezoid (kernel 1) or hat (kernel 0).
template <int KERNEL>
__device__ __forceinline__ float tap_weight(const AngleGeo &g, float d) {
    if (KERNEL == 1) return __fmul_rn(fminf(fmaxf(__fsub_rn(g.hw, fabsf(d)), 0.0f), g.top), g.iw);
    return fmaxf(__fsub_rn(1.0f, fabsf(d)), 0.0f);
}

// K'(d): the derivative of the tap weight with respect to the detector coordinate (0 at the kinks' outer side:
// non-zero only where K is); the derivative of a projection with respect to a detector shift.
template <int KERNEL>
__device__ __forceinline__ float tap_dweight(const AngleGeo &g, float d) {
    if (KERNEL == 1) {
        const float q = __fsub_rn(g.hw, fabsf(d));
        return (q > 0.0f && q < g.top) ? -copysignf(g.iw, d) : 0.0f;
    }
    return fabsf(d) < 1.0f ? -copysignf(1.0f, d) : 0.0f;
}

// window_parallax: the fraction of axis a's radial profile inside channel p's window at angle r for orientation kg
// (pf_generate.cl:103-121); the caller checks g.wp_ax != nullptr
__device__ __forceinline__ float wp_fraction(const dfx_pf_geometry &g, int r, int kg, int p, int a)
{
    const float bx = __ldg(g.wp_b + 2 * r), by = __ldg(g.wp_b + 2 * r + 1);
    const float qx = __ldg(g.wp_pos + 2 * kg), qy = __ldg(g.wp_pos + 2 * kg + 1);
    const float cxx = __ldg(g.wp_cov + 4 * kg), cxy = __ldg(g.wp_cov + 4 * kg + 1), cyy = __ldg(g.wp_cov + 4 * kg + 2);
    const float wx = qx * bx + qy * by;                               // mean depth along the beam
    const float wvar = cxx * bx * bx + 2.0f * cxy * bx * by + cyy * by * by;
    const float lo = __ldg(g.wp_ch + 2 * p), hi = __ldg(g.wp_ch + 2 * p + 1);
    const float tt = __ldg(g.wp_ax + 4 * a), scs = __ldg(g.wp_ax + 4 * a + 1), s2 = __ldg(g.wp_ax + 4 * a + 2),
                gam = __ldg(g.wp_ax + 4 * a + 3);
    const float sh = tt - wx * g.wp_invD * scs;                       // the shifted two-theta
    const float gg = scs * g.wp_invD;
    const float is = rsqrtf(2.0f * (s2 + gg * gg * wvar));
    const float zh = (hi - sh) * is, zl = (lo - sh) * is;             // erfc in the tails
    float fr = zl > 0.0f ? 0.5f * (erfcf(zl) - erfcf(zh))
                         : (zh < 0.0f ? 0.5f * (erfcf(-zh) - erfcf(-zl)) : 0.5f * (erff(zh) - erff(zl)));
    if (g.wp_eta > 0.0f)
        fr = (1.0f - g.wp_eta) * fr + g.wp_eta * (atanf((hi - sh) / gam) - atanf((lo - sh) / gam)) * 0.31830988618f;
    return fr;
}

}  // namespace dfx
