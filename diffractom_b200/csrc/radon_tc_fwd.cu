// Forward projection on the tensor cores (tcgen05, sm_100a) for the BF16 precision path: the Radon output of a batch
// of BF16 channel-fastest images, float32 accumulation, written as BF16 (or float32) sinogram rows.
//
// For one angle a and 128 channels (the tensor-memory lanes) the projection Z[s, k] = scale sum_p K(t_a(p) - s) X[p, k]
// is a sum over 8 x 8 pixel tiles of products  D[k, window] += X_tile^T (128 x 64) . W_tile (64 x 32): X_tile holds
// the tile's 64 pixel rows of the 128 channels (a TMA box per 64-channel half, 128-byte swizzle), W_tile the tap
// weights of those pixels on a 32-bin window that starts at a multiple of 16 bins at or below the tile's first tap
// (so every accumulator address is 16-column aligned; a tile's taps span at most 17 bins at the geometries the host
// admits). The weights are float32 split into BF16 hi + lo parts and applied by two MMAs, so they keep float32
// accuracy; the image is BF16 already. D covers all bins of the angle (ns + 31 <= 512 columns), stays in tensor
// memory over the whole image and is written once at the end: no partial sums leave the SM, no atomics.
//
// One CTA per (angle, 128 channels); warp roles:
//   warp 0      lane 0 streams the image tiles through a 4-stage ring (TMA);
//   warps 1-2   build the weight tiles (thread m: pixel m of the tile) into a 4-deep ring of (hi, lo) pairs, each warp
//               zeroing the 16-byte rows of its own 32 pixels first (so only a warp sync orders zeros and taps);
//   warp 3      lane 0 issues a tile's MMAs once its weights (64 arrivals) and its image tile are in place;
//   warps 4-7   zero the accumulator before the first MMA and, after the last, read it (tensor-memory lane quarter
//               w % 4 each), scale, round and store the sinogram rows (channels contiguous).
// Replaces, on the BF16 path, radon_forward_k (radon_kernels.cl:44-101) as dfx_radon_forward_table_bf16_bf16 does.
//
// Every mbarrier wait is bounded (2 s) and also ends once another role of the CTA has given up; on expiry the CTA
// records DFX_TC_TIMEOUT, stops issuing work, lets its copies and MMAs in flight land, frees its tensor memory and
// returns. A tap outside its tile's window (a geometry the host check did not cover) records DFX_TC_WINDOW.

#include "tc_common.cuh"

namespace dfx {

unsigned int tcf_status(unsigned int reset);

namespace {

using namespace tc;

constexpr int TF_T = 8;                        // pixel tile: 8 x 8 = 64 pixels = the MMA contraction of one tile
constexpr int TF_PX = TF_T * TF_T;
constexpr int TF_NW = 32;                      // bins per tile window (MMA N)
constexpr int TF_CH = 128;                     // channels per CTA (MMA M = tensor-memory lanes)
constexpr int TF_STAGES = 4;                   // image tiles in the ring
constexpr int TF_WBUF = 4;                     // weight tiles in the ring
constexpr int TF_X_BYTES = TF_PX * TF_CH * 2;  // 16 KB: two boxes of 64 pixels x 64 channels (128-byte rows)
constexpr int TF_W_BYTES = TF_NW * TF_PX * 2;  // 4 KB: one weight tile (hi or lo)
constexpr int TF_THREADS = 256;
constexpr int TF_EPI0 = 4;                     // first epilogue warp

__device__ unsigned int g_tcf_flags;

struct TfArgs {
    int n_angles, nx, ny, ns, kstride, n_tiles, tiles_x, tmem_cols;
    const int32_t *tiles;                      // tile indices (row-major over the tile grid); NULL: all
    void *out;
    int64_t sld;                               // sinogram row stride (elements)
    float scale;
    int out_f32;
};

// K-major weight tile: row n (bin), column k (pixel) in interleaved 8 x 8 core matrices (16 bytes: 8 pixels of a bin)
__device__ __forceinline__ uint32_t w_offset(int n, int k)
{
    return (uint32_t)((n >> 3) * 1024 + (k >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ void tmem_st16_zero(uint32_t taddr)
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, "
        "%1};" ::"r"(taddr),
        "r"(0u)
        : "memory");
}

__device__ __forceinline__ bool wait_or_abort(uint32_t bar, uint32_t parity, volatile int *abort)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (*abort) return false;
        if (now_ns() - t0 > WAIT_NS) {
            atomicOr(&g_tcf_flags, DFX_TC_TIMEOUT);
            *abort = 1;
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tile_xy(const TfArgs &p, int i, int &px0, int &py0)
{
    const int t = p.tiles ? __ldg(p.tiles + i) : i;
    px0 = (t % p.tiles_x) * TF_T;
    py0 = (t / p.tiles_x) * TF_T;
}

// The tile's window start: its smallest detector coordinate's first tap, clamped to the detector, rounded down to 16.
template <int KERNEL>
__device__ __forceinline__ int window16(const AngleGeo &g, int px0, int py0, int ns)
{
    float tmin = 3.0e38f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float fx = (float)(px0 + (c & 1) * (TF_T - 1)), fy = (float)(py0 + (c >> 1) * (TF_T - 1));
        const float t = __fmaf_rn(g.A, g.rows_are_y ? fx : fy, __fmaf_rn(g.B, g.rows_are_y ? fy : fx, g.T0));
        tmin = fminf(tmin, t);
    }
    const int sf = KERNEL == 1 ? (int)floorf(__fsub_rn(tmin, g.hw)) + 1 : (int)floorf(tmin);
    return min(max(sf, 0), ns - 1) & ~15;
}

template <int KERNEL>
__global__ void __launch_bounds__(TF_THREADS, 1) tc_forward(const __grid_constant__ CUtensorMap xmap,
                                                           const float4 *__restrict__ geo, int n_taps, TfArgs p)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    uint8_t *xtile = smem;                                        // [STAGES][16 KB]
    uint8_t *wtile = xtile + TF_STAGES * TF_X_BYTES;              // [WBUF][hi 4 KB | lo 4 KB]
    uint64_t *bars = reinterpret_cast<uint64_t *>(wtile + TF_WBUF * 2 * TF_W_BYTES);
    // full[S], empty[S], wready[WB], wfree[WB], done
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * TF_STAGES + 2 * TF_WBUF + 1);
    int *n_issued = reinterpret_cast<int *>(tmem_slot + 1), *n_used = n_issued + 1;
    volatile int *abort = n_issued + 2;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int a = blockIdx.x, k0 = blockIdx.y * TF_CH;
    const uint32_t full0 = smem_u32(bars), empty0 = full0 + 8 * TF_STAGES, wready0 = empty0 + 8 * TF_STAGES;
    const uint32_t wfree0 = wready0 + 8 * TF_WBUF, done = wfree0 + 8 * TF_WBUF;
    const AngleGeo ga = load_geo(geo, a);

    if (tid == 0) {
        for (int s = 0; s < TF_STAGES; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        for (int b = 0; b < TF_WBUF; ++b) {
            mbar_init(wready0 + 8 * b, TF_PX);
            mbar_init(wfree0 + 8 * b, 1);
        }
        mbar_init(done, 1);
        *n_issued = *n_used = 0;
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&xmap)) : "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"((uint32_t)p.tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    if (warp >= TF_EPI0) {
        // zero the accumulator (this warp's 32 lanes, every column the windows can reach)
        const uint32_t lanes = (uint32_t)(32 * (warp & 3)) << 16;
        for (int c = 0; c < p.tmem_cols; c += 16) tmem_st16_zero(tmem + lanes + (uint32_t)c);
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    const int n_tiles = p.n_tiles;
    if (warp == 0) {
        // ---- producer: the image tiles, up to TF_STAGES ahead of the MMAs
        if (lane == 0) {
            int issued = 0;
            for (int i = 0; i < n_tiles; ++i) {
                const int st = i % TF_STAGES;
                if (i >= TF_STAGES && !wait_or_abort(empty0 + 8 * st, ((i - TF_STAGES) / TF_STAGES) & 1, abort))
                    break;
                int px0, py0;
                tile_xy(p, i, px0, py0);
                const uint32_t fb = full0 + 8 * st;
                mbar_expect_tx(fb, (uint32_t)TF_X_BYTES);
                tma_load_3d(smem_u32(xtile + st * TF_X_BYTES), &xmap, fb, k0, px0, py0);
                tma_load_3d(smem_u32(xtile + st * TF_X_BYTES + TF_X_BYTES / 2), &xmap, fb, k0 + 64, px0, py0);
                issued = i + 1;
            }
            *n_issued = issued;
        }
    } else if (warp == 1 || warp == 2) {
        // ---- builders: thread m = pixel m of the tile; warp 1 owns pixels 0-31, warp 2 pixels 32-63
        const int m = tid - 32, wg = warp - 1;
        for (int i = 0; i < n_tiles; ++i) {
            const int wb = i % TF_WBUF;
            if (*abort) break;
            // weight buffer wb is free once the MMAs of tile i - TF_WBUF have completed
            if (i >= TF_WBUF && !wait_or_abort(wfree0 + 8 * wb, ((i - TF_WBUF) / TF_WBUF) & 1, abort)) break;
            int px0, py0;
            tile_xy(p, i, px0, py0);
            const int sw = window16<KERNEL>(ga, px0, py0, p.ns);
            uint8_t *wh = wtile + wb * 2 * TF_W_BYTES, *wl = wh + TF_W_BYTES;
            // this warp's pixels are the core-matrix columns 4 wg .. 4 wg + 3: lane n zeroes bin row n of them
#pragma unroll
            for (int g = 0; g < 4; ++g) {
                const uint32_t off = (uint32_t)((lane >> 3) * 1024 + (4 * wg + g) * 128 + (lane & 7) * 16);
                *reinterpret_cast<uint4 *>(wh + off) = make_uint4(0, 0, 0, 0);
                *reinterpret_cast<uint4 *>(wl + off) = make_uint4(0, 0, 0, 0);
            }
            __syncwarp();
            const int px = px0 + (m & (TF_T - 1)), py = py0 + (m >> 3);
            if (px < p.nx && py < p.ny) {
                const float fx = (float)px, fy = (float)py;
                const float tt =
                    __fmaf_rn(ga.A, ga.rows_are_y ? fx : fy, __fmaf_rn(ga.B, ga.rows_are_y ? fy : fx, ga.T0));
                const int sf = KERNEL == 1 ? (int)floorf(__fsub_rn(tt, ga.hw)) + 1 : (int)floorf(tt);
                const int nt = KERNEL == 1 ? min(max(2, (int)ceilf(1.0f + fabsf(ga.A) - 1e-6f)), n_taps) : 2;
                for (int q = 0; q < nt; ++q) {
                    const int s = sf + q;
                    if (s < 0 || s >= p.ns) continue;
                    const float w = tap_weight<KERNEL>(ga, __fsub_rn(tt, (float)s));
                    if (w == 0.0f) continue;
                    const int n = s - sw;
                    if (n < 0 || n >= TF_NW) {
                        atomicOr(&g_tcf_flags, DFX_TC_WINDOW);
                        continue;
                    }
                    const __nv_bfloat16 hi = __float2bfloat16_rn(w);
                    const __nv_bfloat16 lo = __float2bfloat16_rn(__fsub_rn(w, __bfloat162float(hi)));
                    *reinterpret_cast<__nv_bfloat16 *>(wh + w_offset(n, m)) = hi;
                    *reinterpret_cast<__nv_bfloat16 *>(wl + w_offset(n, m)) = lo;
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // generic writes -> tensor core
            mbar_arrive(wready0 + 8 * wb);
        }
    } else if (warp == 3) {
        // ---- MMA issuer
        if (lane == 0) {
            const uint32_t idesc = instr_desc(TF_NW, 1, 0);      // A (image) channels-major, B (weights) K-major
            for (int i = 0; i < n_tiles; ++i) {
                const int st = i % TF_STAGES, wb = i % TF_WBUF;
                if (!wait_or_abort(wready0 + 8 * wb, (i / TF_WBUF) & 1, abort)) break;
                if (!wait_or_abort(full0 + 8 * st, (i / TF_STAGES) & 1, abort)) break;
                *n_used = i + 1;
                tc_fence_after();
                int px0, py0;
                tile_xy(p, i, px0, py0);
                const uint32_t dcol = tmem + (uint32_t)window16<KERNEL>(ga, px0, py0, p.ns);
                const uint32_t xb = smem_u32(xtile + st * TF_X_BYTES);
                const uint32_t hb = smem_u32(wtile + wb * 2 * TF_W_BYTES), lb = hb + TF_W_BYTES;
#pragma unroll
                for (int kk = 0; kk < TF_PX / 16; ++kk) {
                    const uint64_t ad = smem_desc(xb + kk * 2048, TF_X_BYTES / 2, 1024, SW_128B);
                    mma_bf16(dcol, ad, smem_desc(hb + kk * 256, 128, 1024, SW_NONE), idesc, 1);
                    mma_bf16(dcol, ad, smem_desc(lb + kk * 256, 128, 1024, SW_NONE), idesc, 1);
                }
                mma_commit(empty0 + 8 * st);                      // image tile free once these are done
                mma_commit(wfree0 + 8 * wb);                      // weight tiles free likewise
            }
            mma_commit(done);                                     // tracks every MMA this thread issued
        }
    } else if (warp >= TF_EPI0) {
        // ---- epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31 = channels k0 + 32 (w % 4) + lane
        bool ok = wait_or_abort(done, 0, abort);
        ok = __all_sync(0xffffffffu, ok && !*abort);              // tcgen05.ld below is warp-collective
        tc_fence_after();
        const int q4 = warp & 3;
        const int k = k0 + 32 * q4 + lane;
        if (ok) {
            const uint32_t lanes = (uint32_t)(32 * q4) << 16;
            for (int c0 = 0; c0 < p.ns; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + lanes + (uint32_t)c0, v);
                if (k < p.kstride) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int s = c0 + j;
                        if (s >= p.ns) break;
                        const int64_t o = ((int64_t)a * p.ns + s) * p.sld + k;
                        const float val = __fmul_rn(p.scale, v[j]);
                        if (p.out_f32)
                            reinterpret_cast<float *>(p.out)[o] = val;
                        else
                            reinterpret_cast<__nv_bfloat16 *>(p.out)[o] = __float2bfloat16_rn(val);
                    }
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (tid == 96) mbar_wait(done, 0, DFX_TC_TIMEOUT, &g_tcf_flags);     // every MMA has completed
    if (tid == 64) {
        // tiles loaded but never consumed (only after an expired wait): let them land before the CTA exits
        for (int i = *n_used; i < *n_issued; ++i)
            if (!mbar_wait(full0 + 8 * (i % TF_STAGES), (i / TF_STAGES) & 1, DFX_TC_TIMEOUT, &g_tcf_flags)) break;
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)p.tmem_cols));
    }
}

// ---------------------------------------------------------------------------------------------- weight-table variant
// The weight tiles depend on (angle, tile) only, not on the channels: built once per geometry into a table (hi and lo
// tiles in the B operand's shared-memory layout, 8 KB per (angle, tile), and the window start), they are loaded by
// the producer with the image tile (a bulk copy beside the TMA), so the MMA warp waits for copies only.
constexpr int TW_W_BYTES = 2 * TF_W_BYTES;                  // hi | lo
constexpr int TW_STAGE_BYTES = TF_X_BYTES + TW_W_BYTES;     // 24 KB: image tile, then its weights
constexpr int TW_STAGES = 6;
constexpr int TW_THREADS = 192;                             // warp 0 loads, warp 1 MMAs, warps 2-5 epilogue

template <int KERNEL>
__global__ void __launch_bounds__(TF_PX) tcf_weights_kernel(const float4 *__restrict__ geo, int nx, int ny, int ns,
                                                           int n_taps, int tiles_x, int n_tiles_img,
                                                           uint8_t *__restrict__ weights, int32_t *__restrict__ windows)
{
    const int t = blockIdx.x, a = blockIdx.y, m = threadIdx.x;
    const AngleGeo ga = load_geo(geo, a);
    const int px0 = (t % tiles_x) * TF_T, py0 = (t / tiles_x) * TF_T;
    const int sw = window16<KERNEL>(ga, px0, py0, ns);
    const int64_t row = (int64_t)a * n_tiles_img + t;
    uint8_t *wh = weights + row * TW_W_BYTES, *wl = wh + TF_W_BYTES;
    uint4 *w4 = reinterpret_cast<uint4 *>(wh);
    for (int i = m; i < TW_W_BYTES / 16; i += TF_PX) w4[i] = make_uint4(0, 0, 0, 0);
    if (m == 0) windows[row] = sw;
    __syncthreads();
    const int px = px0 + (m & (TF_T - 1)), py = py0 + (m >> 3);
    if (px >= nx || py >= ny) return;
    const float fx = (float)px, fy = (float)py;
    const float tt = __fmaf_rn(ga.A, ga.rows_are_y ? fx : fy, __fmaf_rn(ga.B, ga.rows_are_y ? fy : fx, ga.T0));
    const int sf = KERNEL == 1 ? (int)floorf(__fsub_rn(tt, ga.hw)) + 1 : (int)floorf(tt);
    const int nt = KERNEL == 1 ? min(max(2, (int)ceilf(1.0f + fabsf(ga.A) - 1e-6f)), n_taps) : 2;
    for (int q = 0; q < nt; ++q) {
        const int s = sf + q;
        if (s < 0 || s >= ns) continue;
        const float w = tap_weight<KERNEL>(ga, __fsub_rn(tt, (float)s));
        if (w == 0.0f) continue;
        const int n = s - sw;
        if (n < 0 || n >= TF_NW) {
            atomicOr(&g_tcf_flags, DFX_TC_WINDOW);
            continue;
        }
        const __nv_bfloat16 hi = __float2bfloat16_rn(w);
        const __nv_bfloat16 lo = __float2bfloat16_rn(__fsub_rn(w, __bfloat162float(hi)));
        *reinterpret_cast<__nv_bfloat16 *>(wh + w_offset(n, m)) = hi;
        *reinterpret_cast<__nv_bfloat16 *>(wl + w_offset(n, m)) = lo;
    }
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(bar)
                 : "memory");
}

struct TwArgs {
    const uint8_t *weights;
    const int32_t *windows;
    const int32_t *angle_rows;                  // table row of each launch angle (NULL: the launch angle)
    int n_tiles_img;
};

__global__ void __launch_bounds__(TW_THREADS, 1) tc_forward_tab(const __grid_constant__ CUtensorMap xmap, TfArgs p,
                                                               TwArgs q)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + TW_STAGES * TW_STAGE_BYTES);   // full[S], empty[S], done
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * TW_STAGES + 1);
    int *n_issued = reinterpret_cast<int *>(tmem_slot + 1), *n_used = n_issued + 1;
    volatile int *abort = n_issued + 2;
    // the launch's tile sequence and each tile's window start, read from global memory once per CTA (the MMA
    // issuer would otherwise wait for a global load before every tile's MMAs)
    int32_t *s_tile = reinterpret_cast<int32_t *>(n_issued + 4), *s_win = s_tile + p.n_tiles;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int a = blockIdx.x, k0 = blockIdx.y * TF_CH;
    const int arow = q.angle_rows ? __ldg(q.angle_rows + a) : a;
    const uint32_t full0 = smem_u32(bars), empty0 = full0 + 8 * TW_STAGES, done = empty0 + 8 * TW_STAGES;

    if (tid == 0) {
        for (int st = 0; st < TW_STAGES; ++st) {
            mbar_init(full0 + 8 * st, 1);
            mbar_init(empty0 + 8 * st, 1);
        }
        mbar_init(done, 1);
        *n_issued = *n_used = 0;
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&xmap)) : "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"((uint32_t)p.tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    if (warp >= 2) {
        const uint32_t lanes = (uint32_t)(32 * (warp & 3)) << 16;
        for (int c = 0; c < p.tmem_cols; c += 16) tmem_st16_zero(tmem + lanes + (uint32_t)c);
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    const int n_tiles = p.n_tiles;
    const uint8_t *wrow = q.weights + (int64_t)arow * q.n_tiles_img * TW_W_BYTES;
    const int32_t *winrow = q.windows + (int64_t)arow * q.n_tiles_img;
    for (int i = tid; i < n_tiles; i += TW_THREADS) {
        const int t = p.tiles ? __ldg(p.tiles + i) : i;
        s_tile[i] = t;
        s_win[i] = __ldg(winrow + t);
    }
    __syncthreads();
    if (warp == 0) {
        // ---- producer: image tile (TMA) and its weight tiles (bulk copy), up to TW_STAGES ahead of the MMAs
        if (lane == 0) {
            int issued = 0;
            for (int i = 0; i < n_tiles; ++i) {
                const int st = i % TW_STAGES;
                if (i >= TW_STAGES && !wait_or_abort(empty0 + 8 * st, ((i - TW_STAGES) / TW_STAGES) & 1, abort))
                    break;
                const int t = s_tile[i];
                const int px0 = (t % p.tiles_x) * TF_T, py0 = (t / p.tiles_x) * TF_T;
                const uint32_t fb = full0 + 8 * st, xs = smem_u32(smem + st * TW_STAGE_BYTES);
                mbar_expect_tx(fb, (uint32_t)TW_STAGE_BYTES);
                tma_load_3d(xs, &xmap, fb, k0, px0, py0);
                tma_load_3d(xs + TF_X_BYTES / 2, &xmap, fb, k0 + 64, px0, py0);
                bulk_load(xs + TF_X_BYTES, wrow + (int64_t)t * TW_W_BYTES, (uint32_t)TW_W_BYTES, fb);
                issued = i + 1;
            }
            *n_issued = issued;
        }
    } else if (warp == 1) {
        // ---- MMA issuer
        if (lane == 0) {
            const uint32_t idesc = instr_desc(TF_NW, 1, 0);
            for (int i = 0; i < n_tiles; ++i) {
                const int st = i % TW_STAGES;
                if (!wait_or_abort(full0 + 8 * st, (i / TW_STAGES) & 1, abort)) break;
                *n_used = i + 1;
                tc_fence_after();
                const uint32_t dcol = tmem + (uint32_t)s_win[i];
                const uint32_t xb = smem_u32(smem + st * TW_STAGE_BYTES);
                const uint32_t hb = xb + TF_X_BYTES, lb = hb + TF_W_BYTES;
#pragma unroll
                for (int kk = 0; kk < TF_PX / 16; ++kk) {
                    const uint64_t ad = smem_desc(xb + kk * 2048, TF_X_BYTES / 2, 1024, SW_128B);
                    mma_bf16(dcol, ad, smem_desc(hb + kk * 256, 128, 1024, SW_NONE), idesc, 1);
                    mma_bf16(dcol, ad, smem_desc(lb + kk * 256, 128, 1024, SW_NONE), idesc, 1);
                }
                mma_commit(empty0 + 8 * st);
            }
            mma_commit(done);
        }
    } else {
        // ---- epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31 = channels k0 + 32 (w % 4) + lane
        bool ok = wait_or_abort(done, 0, abort);
        ok = __all_sync(0xffffffffu, ok && !*abort);
        tc_fence_after();
        const int q4 = warp & 3;
        const int k = k0 + 32 * q4 + lane;
        if (ok) {
            const uint32_t lanes = (uint32_t)(32 * q4) << 16;
            for (int c0 = 0; c0 < p.ns; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + lanes + (uint32_t)c0, v);
                if (k < p.kstride) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int s = c0 + j;
                        if (s >= p.ns) break;
                        const int64_t o = ((int64_t)a * p.ns + s) * p.sld + k;
                        const float val = __fmul_rn(p.scale, v[j]);
                        if (p.out_f32)
                            reinterpret_cast<float *>(p.out)[o] = val;
                        else
                            reinterpret_cast<__nv_bfloat16 *>(p.out)[o] = __float2bfloat16_rn(val);
                    }
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (tid == 32) mbar_wait(done, 0, DFX_TC_TIMEOUT, &g_tcf_flags);      // every MMA has completed
    if (tid == 64) {
        // loads issued but never consumed (only after an expired wait): let them land before the CTA exits
        for (int i = *n_used; i < *n_issued; ++i)
            if (!mbar_wait(full0 + 8 * (i % TW_STAGES), (i / TW_STAGES) & 1, DFX_TC_TIMEOUT, &g_tcf_flags)) break;
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)p.tmem_cols));
    }
}

size_t tw_smem_bytes(int n_tiles) { return 1024 + (size_t)TW_STAGES * TW_STAGE_BYTES + 256 + 8 * (size_t)n_tiles; }

size_t tf_smem_bytes() { return 1024 + (size_t)TF_STAGES * TF_X_BYTES + (size_t)TF_WBUF * 2 * TF_W_BYTES + 256; }

// 3-D BF16 image batch (channels, x, y) with a box of 64 channels x 8 x 8 pixels, 128-byte swizzle
int make_image_map(CUtensorMap *map, const void *img, int kstride, int nx, int ny)
{
    EncodeTiledFn enc = encoder();
    DFX_REQUIRE(enc != nullptr, "radon_forward_tc: cuTensorMapEncodeTiled is not available from the driver");
    DFX_REQUIRE(((uintptr_t)img % 16) == 0 && kstride % 64 == 0,
                "radon_forward_tc: the image must be 16-byte aligned with kstride a multiple of 64");
    const cuuint64_t dims[3] = {(cuuint64_t)kstride, (cuuint64_t)nx, (cuuint64_t)ny};
    const cuuint64_t strides[2] = {(cuuint64_t)kstride * 2, (cuuint64_t)kstride * nx * 2};
    const cuuint32_t box[3] = {64, TF_T, TF_T};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult rc = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void *>(img), dims, strides, box,
                            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    DFX_REQUIRE(rc == CUDA_SUCCESS, "radon_forward_tc: tensor map of the image rejected (CUresult %d)", (int)rc);
    return DFX_OK;
}

}  // namespace

unsigned int tcf_status(unsigned int reset)
{
    unsigned int f = 0;
    cudaMemcpyFromSymbol(&f, g_tcf_flags, sizeof(f));
    if (reset) {
        const unsigned int zero = 0;
        cudaMemcpyToSymbol(g_tcf_flags, &zero, sizeof(zero));
    }
    return f;
}

}  // namespace dfx

using namespace dfx;

extern "C" int64_t dfx_radon_tc_weights_bytes(int n_angles, int nx, int ny)
{
    if (n_angles <= 0 || nx <= 0 || ny <= 0) return 0;
    return (int64_t)n_angles * cdiv(nx, TF_T) * cdiv(ny, TF_T) * TW_W_BYTES;
}

extern "C" int dfx_radon_tc_weights(const float *geo, int n_angles, int nx, int ny, int n_det, int kernel, int n_taps,
                                    void *weights, int32_t *windows, void *stream)
{
    DFX_REQUIRE(geo && weights && windows, "radon_tc_weights: null pointer");
    DFX_REQUIRE(((uintptr_t)geo % 16) == 0 && ((uintptr_t)weights % 16) == 0, "radon_tc_weights: misaligned arrays");
    DFX_REQUIRE(n_angles > 0 && n_angles <= 65535 && nx > 0 && ny > 0 && n_det > 0, "radon_tc_weights: bad sizes");
    DFX_REQUIRE(kernel == 0 || kernel == 1, "radon_tc_weights: kernel must be 0 or 1");
    DFX_REQUIRE(n_taps >= 2 && n_taps <= 64, "radon_tc_weights: n_taps (%d) out of range", n_taps);
    const int tiles_x = (int)cdiv(nx, TF_T), n_tiles = tiles_x * (int)cdiv(ny, TF_T);
    const dim3 grid((unsigned)n_tiles, (unsigned)n_angles);
    if (kernel == 1)
        tcf_weights_kernel<1><<<grid, TF_PX, 0, (cudaStream_t)stream>>>(
            reinterpret_cast<const float4 *>(geo), nx, ny, n_det, n_taps, tiles_x, n_tiles,
            reinterpret_cast<uint8_t *>(weights), windows);
    else
        tcf_weights_kernel<0><<<grid, TF_PX, 0, (cudaStream_t)stream>>>(
            reinterpret_cast<const float4 *>(geo), nx, ny, n_det, n_taps, tiles_x, n_tiles,
            reinterpret_cast<uint8_t *>(weights), windows);
    return launch_status("radon_tc_weights");
}

extern "C" int dfx_radon_forward_tc_table(const void *img_bf16, void *sino, int64_t sino_ld, int out_f32,
                                          const void *weights, const int32_t *windows, const int32_t *angle_rows,
                                          int n_angles, int nx, int ny, int n_det, int kstride, float scale,
                                          const int32_t *tiles, int n_tiles, void *stream)
{
    DFX_REQUIRE(img_bf16 && sino && weights && windows, "radon_forward_tc_table: null pointer");
    DFX_REQUIRE(((uintptr_t)weights % 16) == 0, "radon_forward_tc_table: weights must be 16-byte aligned");
    DFX_REQUIRE(n_angles >= 0 && n_angles <= 65535 && nx > 0 && ny > 0 && n_det > 0,
                "radon_forward_tc_table: bad sizes (angles %d, %d x %d, %d bins)", n_angles, nx, ny, n_det);
    DFX_REQUIRE(kstride > 0 && kstride % 64 == 0, "radon_forward_tc_table: kstride (%d) must be a multiple of 64",
                kstride);
    DFX_REQUIRE(sino_ld >= kstride && sino_ld % 8 == 0, "radon_forward_tc_table: bad sinogram row stride");
    const int tiles_x = (int)cdiv(nx, TF_T), tiles_img = tiles_x * (int)cdiv(ny, TF_T);
    DFX_REQUIRE(tiles == nullptr ? true : (n_tiles >= 0 && n_tiles <= tiles_img),
                "radon_forward_tc_table: bad tile list");
    int cols = 32;
    while (cols < n_det + TF_NW - 1) cols *= 2;
    DFX_REQUIRE(cols <= 512, "radon_forward_tc_table: %d bins exceed the tensor memory of one CTA", n_det);
    if (n_angles == 0) return DFX_OK;
    CUtensorMap xmap;
    int st = make_image_map(&xmap, img_bf16, kstride, nx, ny);
    if (st) return st;
    TfArgs a{};
    a.n_angles = n_angles;
    a.nx = nx;
    a.ny = ny;
    a.ns = n_det;
    a.kstride = kstride;
    a.tiles = tiles;
    a.n_tiles = tiles ? n_tiles : tiles_img;
    a.tiles_x = tiles_x;
    a.tmem_cols = cols;
    a.out = sino;
    a.sld = sino_ld;
    a.scale = scale;
    a.out_f32 = out_f32 ? 1 : 0;
    TwArgs q{reinterpret_cast<const uint8_t *>(weights), windows, angle_rows, tiles_img};
    const size_t smem = tw_smem_bytes(a.n_tiles);
    DFX_REQUIRE(smem <= 227 * 1024, "radon_forward_tc_table: %d tiles exceed the shared memory of one CTA", a.n_tiles);
    const cudaError_t e = allow_max_dynamic_smem(tc_forward_tab);
    if (e != cudaSuccess) {
        set_error("radon_forward_tc_table: shared memory attribute: %s", cudaGetErrorString(e));
        return DFX_ELAUNCH;
    }
    const dim3 grid((unsigned)n_angles, (unsigned)cdiv(kstride, TF_CH));
    tc_forward_tab<<<grid, TW_THREADS, smem, (cudaStream_t)stream>>>(xmap, a, q);
    return launch_status("radon_forward_tc_table");
}

extern "C" int dfx_radon_forward_tc(const void *img_bf16, void *sino, int64_t sino_ld, int out_f32, const float *geo,
                                    int n_angles, int nx, int ny, int n_det, int kstride, int kernel, int n_taps,
                                    float scale, const int32_t *tiles, int n_tiles, void *stream)
{
    DFX_REQUIRE(img_bf16 && sino && geo, "radon_forward_tc: null pointer");
    DFX_REQUIRE(((uintptr_t)geo % 16) == 0, "radon_forward_tc: geo must be 16-byte aligned");
    DFX_REQUIRE(n_angles >= 0 && n_angles <= 65535 && nx > 0 && ny > 0 && n_det > 0,
                "radon_forward_tc: bad sizes (angles %d, %d x %d, %d bins)", n_angles, nx, ny, n_det);
    DFX_REQUIRE(kstride > 0 && kstride % 64 == 0, "radon_forward_tc: kstride (%d) must be a multiple of 64", kstride);
    DFX_REQUIRE(sino_ld >= kstride && sino_ld % 8 == 0, "radon_forward_tc: bad sinogram row stride");
    DFX_REQUIRE(kernel == 0 || kernel == 1, "radon_forward_tc: kernel must be 0 or 1");
    DFX_REQUIRE(n_taps >= 2 && n_taps <= 64, "radon_forward_tc: n_taps (%d) out of range", n_taps);
    const int tiles_x = (int)cdiv(nx, TF_T), tiles_y = (int)cdiv(ny, TF_T);
    DFX_REQUIRE(tiles == nullptr ? true : (n_tiles >= 0 && n_tiles <= tiles_x * tiles_y),
                "radon_forward_tc: bad tile list");
    int cols = 32;
    while (cols < n_det + TF_NW - 1) cols *= 2;
    DFX_REQUIRE(cols <= 512, "radon_forward_tc: %d bins exceed the tensor memory of one CTA", n_det);
    if (n_angles == 0) return DFX_OK;
    CUtensorMap xmap;
    int st = make_image_map(&xmap, img_bf16, kstride, nx, ny);
    if (st) return st;
    TfArgs a{};
    a.n_angles = n_angles;
    a.nx = nx;
    a.ny = ny;
    a.ns = n_det;
    a.kstride = kstride;
    a.tiles = tiles;
    a.n_tiles = tiles ? n_tiles : tiles_x * tiles_y;
    a.tiles_x = tiles_x;
    a.tmem_cols = cols;
    a.out = sino;
    a.sld = sino_ld;
    a.scale = scale;
    a.out_f32 = out_f32 ? 1 : 0;
    // one CTA per SM when the accumulator takes more than half of the tensor memory: more than half of the SM's
    // shared memory is requested then, so that no second CTA waits in tcgen05.alloc on the same SM
    const size_t smem = cols > 256 ? (size_t)120 * 1024 : tf_smem_bytes();
    static_assert(TF_STAGES * TF_X_BYTES + TF_WBUF * 2 * TF_W_BYTES + 1024 + 256 <= 120 * 1024, "ring fits");
    const dim3 grid((unsigned)n_angles, (unsigned)cdiv(kstride, TF_CH));
    cudaError_t e;
    if (kernel == 1) {
        e = allow_max_dynamic_smem(tc_forward<1>);
        if (e == cudaSuccess)
            tc_forward<1><<<grid, TF_THREADS, smem, (cudaStream_t)stream>>>(xmap, (const float4 *)geo, n_taps, a);
    } else {
        e = allow_max_dynamic_smem(tc_forward<0>);
        if (e == cudaSuccess)
            tc_forward<0><<<grid, TF_THREADS, smem, (cudaStream_t)stream>>>(xmap, (const float4 *)geo, n_taps, a);
    }
    if (e != cudaSuccess) {
        set_error("radon_forward_tc: shared memory attribute: %s", cudaGetErrorString(e));
        return DFX_ELAUNCH;
    }
    return launch_status("radon_forward_tc");
}
