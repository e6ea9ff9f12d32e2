// Backprojection on the tensor cores (tcgen05, sm_100a) for the BF16 precision path, with SPDHG's primal step in the
// epilogue.
//
// For a tile of 128 pixels (16 x 8) and 256 channels the backprojection img[p, k] = sum_a w_a sum_s K(t_a(p) - s)
// Z[a, s, k] is a sum over the launch's angles of GEMMs  D (128 x 256) += W_a (128 x 32) . Z_a (32 x 256):  W_a holds
// the tap weights of the tile's pixels on a window of 32 bins that covers all of them at angle a (two or three
// non-zeros per row, float32 weights split into BF16 hi + lo parts, two MMAs, so the weights keep float32 accuracy),
// Z_a the window's rows of the BF16 Radon output, fetched by TMA (128-byte swizzle, channels fastest).
//
// The kernel is persistent: one CTA per SM walks the tiles (pixel tile, channel block) blockIdx.x, + gridDim.x, ...
// with two float32 accumulators in tensor memory (2 x 256 of the SM's 512 columns), so that the epilogue of one tile,
// which moves the SPDHG state through HBM, overlaps the MMAs of the next. Warp roles:
//   warps 0-3   build W_a in shared memory (thread m: row m; interleaved 8 x 16-byte core matrices, two buffers);
//               warp 0 lane 0 issues the MMAs of an angle once its weights and Z window are in place;
//   warp 4      lane 0 streams the Z windows through a four-stage ring, across tile boundaries;
//   warps 5-12  epilogue: per half of the 256 channels the accumulator goes through shared memory, then each warp
//               walks 16 pixel rows with channel-contiguous loads and stores of x, z, T and the BF16 copy of x:
//                   z += dz;  x = T > 0 ? max(0, x - T (z + inv_p dz + lam)) : 0;  x_bf16 = bf16(x)
//               exactly as the SIMT kernel radon_backward_v3<MODE 1> does.
// Replaces, like dfx_radon_backward_spdhg_bf16, radon_backward_k + spdhg_update (radon_kernels.cl:106-141;
// spdhg_poisson.py:95-106).
//
// Every mbarrier wait is bounded (2 s) and also ends when another role of the CTA has given up; on expiry the CTA
// records DFX_TC_TIMEOUT, stops issuing work, lets its copies and MMAs in flight land, frees its tensor memory and
// returns (tiles not yet finished keep their old x and z). A tap outside the 32-bin window (a geometry whose 16 x 8
// tile spans more bins; the host checks this before launching) records DFX_TC_WINDOW.

#include "tc_common.cuh"

namespace dfx {

unsigned int tcb_status(unsigned int reset);

namespace {

using namespace tc;

constexpr int TB_TX = 16, TB_TY = 8;           // pixel tile: 128 pixels = tensor-memory lanes
constexpr int TB_KW = 32;                      // bins per angle window
constexpr int TB_N = 256;                      // channels per CTA = accumulator columns
constexpr int TB_STAGES = 4;                   // Z windows in the ring
constexpr int TB_A_BYTES = 128 * TB_KW * 2;    // one weight tile (hi or lo): 8 KB
constexpr int TB_B_BYTES = TB_KW * TB_N * 2;   // one Z window: 16 KB (four 64-channel boxes of 4 KB)

__device__ unsigned int g_tcb_flags;

struct TbArgs {
    int n_angles, nx, ny, ns, kstride, kb, n_taps, tiles_x, n_ptiles, n_tiles;
    float *x, *z;
    const float *T;
    __nv_bfloat16 *xb;
    float inv_p, lam;
};

__device__ __forceinline__ uint32_t a_offset(int m, int j)      // interleaved K-major core matrices
{
    return (uint32_t)((m >> 3) * 512 + (j >> 3) * 128 + (m & 7) * 16 + (j & 7) * 2);
}

__device__ __forceinline__ void primal_step_tc(float &x, float &z, float t, float dz, float inv_p, float lam)
{
    const float zi = __fadd_rn(z, dz);
    z = zi;
    const float zb = __fadd_rn(zi, __fmul_rn(inv_p, dz));
    x = t > 0.0f ? fmaxf(0.0f, __fsub_rn(x, __fmul_rn(t, __fadd_rn(zb, lam)))) : 0.0f;
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&h);
}

// OR of v over the 128 threads of warps 0-3 (named barrier 1), which also orders their shared-memory writes
__device__ __forceinline__ bool builders_or(bool v)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, 1, 128, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)v)
        : "memory");
    return r != 0;
}

template <int KERNEL>
__device__ __forceinline__ int window_start(const AngleGeo &g, int px0, int py0, int ns)
{
    // the tile's smallest detector coordinate is at a corner; its first tap is the tile's first tap
    float tmin = 3.0e38f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float fx = (float)(px0 + (c & 1) * (TB_TX - 1)), fy = (float)(py0 + (c >> 1) * (TB_TY - 1));
        const float t = __fmaf_rn(g.A, g.rows_are_y ? fx : fy, __fmaf_rn(g.B, g.rows_are_y ? fy : fx, g.T0));
        tmin = fminf(tmin, t);
    }
    const int sf = KERNEL == 1 ? (int)floorf(__fsub_rn(tmin, g.hw)) + 1 : (int)floorf(tmin);
    // taps outside the detector get no weight, so the window may start at bin 0 (or the last bin) instead
    return min(max(sf, 0), ns - 1);
}

constexpr int PREFETCH_ROUNDS = 1;             // epilogue: L2 prefetch of x, z, T this many rounds ahead (2: slower)
constexpr int TP_EPI0 = 5;                     // first epilogue warp
constexpr int TP_EPI_WARPS = 8;
constexpr int TP_THREADS = (TP_EPI0 + TP_EPI_WARPS) * 32;   // 416
constexpr int TP_LD = 129;                     // staging row stride in floats (128 channels + 1: no bank conflicts)
constexpr int TP_STAGE_BYTES = 128 * TP_LD * 4;

// Bounded wait on an mbarrier phase that also gives up once another role of the CTA has set *abort; an expiry
// records DFX_TC_TIMEOUT and sets *abort.
__device__ __forceinline__ bool wait_or_abort(uint32_t bar, uint32_t parity, volatile int *abort)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (*abort) return false;
        if (now_ns() - t0 > WAIT_NS) {
            atomicOr(&g_tcb_flags, DFX_TC_TIMEOUT);
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

// AND of v over the 256 epilogue threads (named barrier 2), which also orders their shared-memory accesses
__device__ __forceinline__ bool epilogue_and(bool v)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, 2, 256, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)v)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void epilogue_sync() { asm volatile("bar.sync 2, 256;" ::: "memory"); }

__device__ __forceinline__ void tile_origin(const TbArgs &p, int t, int &px0, int &py0, int &k0)
{
    const int pt = t % p.n_ptiles, cb = t / p.n_ptiles;
    px0 = (pt % p.tiles_x) * TB_TX;
    py0 = (pt / p.tiles_x) * TB_TY;
    k0 = cb * TB_N;
}

// L2 prefetch of one epilogue round: the rows of x, z and T of the 4 pixels px .. px + 3 of image row qy, 128
// channels from kc (48 lines of 128 B; lane l takes lines l and l + 32); pixels and channels outside are skipped
__device__ __forceinline__ void prefetch_round(const TbArgs &p, int qy, int px, int kc, int lane)
{
    if (qy >= p.ny) return;
    const int nv = min(4, p.nx - px);
    const int64_t nb = ((int64_t)qy * p.nx + px) * p.kstride + kc;
    for (int L = lane; L < 48; L += 32) {
        const int u = L / 12, arr = (L >> 2) % 3, c = L & 3;
        if (u < nv && kc + 32 * c < p.kb) {
            const float *src = arr == 0 ? p.x : (arr == 1 ? p.z : p.T);
            asm volatile("prefetch.global.L2 [%0];" ::"l"(src + nb + (int64_t)u * p.kstride + 32 * c));
        }
    }
}

template <int KERNEL>
__global__ void __launch_bounds__(TP_THREADS, 1) tc_backproject_spdhg(const __grid_constant__ CUtensorMap zmap,
                                                                    const float4 *__restrict__ geo, TbArgs p)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    uint8_t *btile = smem;                                        // [TB_STAGES][16 KB] Z windows
    uint8_t *atile = btile + TB_STAGES * TB_B_BYTES;              // [2][hi 8 KB | lo 8 KB] weights
    float *stage = reinterpret_cast<float *>(atile + 4 * TB_A_BYTES);    // epilogue: 128 rows x TP_LD floats
    AngleParams *prm = reinterpret_cast<AngleParams *>(atile + 4 * TB_A_BYTES + TP_STAGE_BYTES);
    uint64_t *bars = reinterpret_cast<uint64_t *>(prm + p.n_angles);    // full[S], empty[S], tfull[2], tempty[2], done
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * TB_STAGES + 5);
    int *n_issued = reinterpret_cast<int *>(tmem_slot + 1), *n_used = n_issued + 1;
    volatile int *abort = n_issued + 2;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n_ang = p.n_angles, n_tiles = p.n_tiles;
    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + TB_STAGES);
    const uint32_t tfull0 = smem_u32(bars + 2 * TB_STAGES), tempty0 = tfull0 + 16, done = tfull0 + 32;

    for (int i = tid; i < n_ang; i += blockDim.x) prm[i] = pack_geo(load_geo(geo, i));
    if (tid == 0) {
        for (int s = 0; s < TB_STAGES; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(tfull0 + 8 * b, 1);
            mbar_init(tempty0 + 8 * b, TP_EPI_WARPS);
        }
        mbar_init(done, 1);
        *n_issued = *n_used = 0;
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&zmap)) : "memory");
    }
    if (warp == 0) {
        // both accumulators: all 512 columns (one CTA per SM: the shared memory of a CTA exceeds half the SM's)
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 4) {
        // ---- producer: the Z windows of every (tile, angle) in order, up to TB_STAGES ahead of the MMAs
        if (lane == 0) {
            int g = 0, issued = 0;
            bool stop = false;
            for (int t = blockIdx.x; t < n_tiles && !stop; t += gridDim.x) {
                int px0, py0, k0;
                tile_origin(p, t, px0, py0, k0);
                int boxes = 0;                                    // 64-channel boxes inside the batch's columns
                for (int i = 0; i < TB_N / 64; ++i) boxes += (k0 + 64 * i < p.kstride);
                for (int a = 0; a < n_ang; ++a, ++g) {
                    const int st = g % TB_STAGES;
                    if (g >= TB_STAGES &&
                        !wait_or_abort(empty0 + 8 * st, ((g - TB_STAGES) / TB_STAGES) & 1, abort)) {
                        stop = true;
                        break;
                    }
                    const int sw = window_start<KERNEL>(unpack_geo(prm[a]), px0, py0, p.ns);
                    const uint32_t fb = full0 + 8 * st;
                    mbar_expect_tx(fb, (uint32_t)boxes * 4096u);
                    for (int i = 0; i < boxes; ++i)
                        tma_load_3d(smem_u32(btile + st * TB_B_BYTES + 4096 * i), &zmap, fb, k0 + 64 * i, sw, a);
                    issued = g + 1;
                }
            }
            *n_issued = issued;
        }
    } else if (warp < 4) {
        // ---- builders (thread m: row m of W_a) and the MMA issuer (thread 32)
        const int m = tid;
        const uint32_t idesc = instr_desc(TB_N, 0, 1);            // A (weights) K-major, B (Z) channels-major
        int g = 0, it = 0;
        bool failed = false;
        for (int t = blockIdx.x; t < n_tiles && !failed; t += gridDim.x, ++it) {
            int px0, py0, k0;
            tile_origin(p, t, px0, py0, k0);
            const int px = px0 + (m & (TB_TX - 1)), py = py0 + (m / TB_TX);
            const bool valid = px < p.nx && py < p.ny;
            const uint32_t dcol = tmem + (uint32_t)((it & 1) * TB_N);
            for (int a = 0; a < n_ang; ++a, ++g) {
                const int st = g % TB_STAGES;
                const AngleGeo ga = unpack_geo(prm[a]);
                const int sw = window_start<KERNEL>(ga, px0, py0, p.ns);
                bool bad = *abort != 0;
                // the weight buffer g & 1 is free once the MMAs of step g - 2 have completed
                if (!bad && g >= 2 &&
                    !wait_or_abort(empty0 + 8 * ((g - 2) % TB_STAGES), ((g - 2) / TB_STAGES) & 1, abort))
                    bad = true;
                uint8_t *ah = atile + (g & 1) * 2 * TB_A_BYTES, *al = ah + TB_A_BYTES;
                if (!bad) {
#pragma unroll
                    for (int c = 0; c < TB_KW / 8; ++c) {
                        const uint32_t off = (uint32_t)((m >> 3) * 512 + c * 128 + (m & 7) * 16);
                        *reinterpret_cast<uint4 *>(ah + off) = make_uint4(0, 0, 0, 0);
                        *reinterpret_cast<uint4 *>(al + off) = make_uint4(0, 0, 0, 0);
                    }
                    if (valid) {
                        const float fx = (float)px, fy = (float)py;
                        const float tt =
                            __fmaf_rn(ga.A, ga.rows_are_y ? fx : fy, __fmaf_rn(ga.B, ga.rows_are_y ? fy : fx, ga.T0));
                        const int sf = KERNEL == 1 ? (int)floorf(__fsub_rn(tt, ga.hw)) + 1 : (int)floorf(tt);
                        const int nt =
                            KERNEL == 1 ? min(max(2, (int)ceilf(1.0f + fabsf(ga.A) - 1e-6f)), p.n_taps) : 2;
                        for (int i = 0; i < nt; ++i) {
                            const int s = sf + i;
                            if (s < 0 || s >= p.ns) continue;
                            const float w = __fmul_rn(ga.w, tap_weight<KERNEL>(ga, __fsub_rn(tt, (float)s)));
                            if (w == 0.0f) continue;
                            const int j = s - sw;
                            if (j < 0 || j >= TB_KW) {
                                atomicOr(&g_tcb_flags, DFX_TC_WINDOW);
                                continue;
                            }
                            const __nv_bfloat16 hi = __float2bfloat16_rn(w);
                            const __nv_bfloat16 lo = __float2bfloat16_rn(__fsub_rn(w, __bfloat162float(hi)));
                            *reinterpret_cast<__nv_bfloat16 *>(ah + a_offset(m, j)) = hi;
                            *reinterpret_cast<__nv_bfloat16 *>(al + a_offset(m, j)) = lo;
                        }
                    }
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // generic writes -> tensor core
                }
                if (builders_or(bad)) {                           // the same decision in all 128 builder threads
                    failed = true;
                    break;
                }
                if (tid == 32) {
                    // the first MMA of a tile overwrites its accumulator: the epilogue of tile it - 2 must be done
                    bool ok = a != 0 || it < 2 || wait_or_abort(tempty0 + 8 * (it & 1), ((it - 2) >> 1) & 1, abort);
                    ok = ok && wait_or_abort(full0 + 8 * st, (g / TB_STAGES) & 1, abort);
                    if (ok) {                                     // otherwise *abort is set: the builders stop next
                        *n_used = g + 1;
                        tc_fence_after();
                        const uint32_t b_base = smem_u32(btile + st * TB_B_BYTES);
                        const uint32_t ah_base = smem_u32(ah), al_base = smem_u32(al);
#pragma unroll
                        for (int kk = 0; kk < TB_KW / 16; ++kk) {
                            const uint64_t bd = smem_desc(b_base + kk * 2048, 4096, 1024, SW_128B);
                            mma_bf16(dcol, smem_desc(ah_base + kk * 256, 128, 512, SW_NONE), bd, idesc,
                                     (a | kk) != 0);
                            mma_bf16(dcol, smem_desc(al_base + kk * 256, 128, 512, SW_NONE), bd, idesc, 1);
                        }
                        mma_commit(empty0 + 8 * st);              // weights and window free once these are done
                        if (a == n_ang - 1) mma_commit(tfull0 + 8 * (it & 1));    // accumulator complete
                    }
                }
            }
        }
        if (tid == 32) mma_commit(done);                          // tracks every MMA this thread issued
    } else {
        // ---- epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31 (its access restriction), half of the
        // 128 columns of a channel half; then walks 16 staging rows (pixels) with lane l on channels 4 l .. 4 l + 3
        const int ew = warp - TP_EPI0, lg = warp & 3, cw = (ew >> 2) * 64;
        int it = 0;
        for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++it) {
            int px0, py0, k0;
            tile_origin(p, t, px0, py0, k0);
            const bool ok = wait_or_abort(tfull0 + 8 * (it & 1), (it >> 1) & 1, abort);
            if (!epilogue_and(ok)) break;
            tc_fence_after();
            const uint32_t dcol = tmem + (uint32_t)((it & 1) * TB_N);
            const int nh = (k0 + 128 < p.kb) ? 2 : 1;
            for (int h = 0; h < nh; ++h) {
#pragma unroll
                for (int c = 0; c < 64; c += 16) {
                    float v[16];
                    tmem_ld16(dcol + ((uint32_t)(32 * lg) << 16) + (uint32_t)(h * 128 + cw + c), v);
                    float *row = stage + (32 * lg + lane) * TP_LD + cw + c;
#pragma unroll
                    for (int i = 0; i < 16; ++i) row[i] = v[i];
                }
                if (h == nh - 1) {                                // accumulator read: the MMAs may reuse it
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(tempty0 + 8 * (it & 1));
                }
                epilogue_sync();
                // warp ew owns the 16 staging rows of image row py0 + ew (pixels px0 .. px0 + 15, TB_TX = 16)
                const int k = k0 + h * 128 + 4 * lane;
                const int qy = py0 + ew;
                if (k < p.kb && qy < p.ny) {
                    const int64_t ks = p.kstride;
#pragma unroll 1
                    for (int r0 = 0; r0 < 16; r0 += 4) {
                        const int nv = min(4, p.nx - (px0 + r0));     // pixels of these 4 rows inside the image
                        const int64_t base = ((int64_t)qy * p.nx + px0 + r0) * ks + k;
                        if (PREFETCH_ROUNDS > 0) {
                            // the rows of x, z and T of the round PREFETCH_ROUNDS ahead into L2 while these are
                            // loaded and stepped: 4 pixels further, else in the next channel half, else in the CTA's
                            // next tile
                            int rr = r0 / 4 + PREFETCH_ROUNDS, hh = h, tt = t, tx0 = px0, ty0 = py0, tk0 = k0,
                                tnh = nh;
                            while (rr >= 4 && tt < n_tiles) {
                                rr -= 4;
                                if (++hh >= tnh) {
                                    hh = 0;
                                    tt += gridDim.x;
                                    if (tt < n_tiles) {
                                        tile_origin(p, tt, tx0, ty0, tk0);
                                        tnh = (tk0 + 128 < p.kb) ? 2 : 1;
                                    }
                                }
                            }
                            if (tt < n_tiles) prefetch_round(p, ty0 + ew, tx0 + 4 * rr, tk0 + hh * 128, lane);
                        }
                        float4 xv[4], zv[4], tv[4];
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            if (u < nv) {
                                xv[u] = __ldcs(reinterpret_cast<const float4 *>(p.x + base + u * ks));
                                zv[u] = __ldcs(reinterpret_cast<const float4 *>(p.z + base + u * ks));
                                tv[u] = __ldcs(reinterpret_cast<const float4 *>(p.T + base + u * ks));
                            }
                        }
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            if (u >= nv) continue;
                            const float *d = stage + (ew * 16 + r0 + u) * TP_LD + 4 * lane;
                            primal_step_tc(xv[u].x, zv[u].x, tv[u].x, (k + 0 < p.kb) ? d[0] : 0.0f, p.inv_p, p.lam);
                            primal_step_tc(xv[u].y, zv[u].y, tv[u].y, (k + 1 < p.kb) ? d[1] : 0.0f, p.inv_p, p.lam);
                            primal_step_tc(xv[u].z, zv[u].z, tv[u].z, (k + 2 < p.kb) ? d[2] : 0.0f, p.inv_p, p.lam);
                            primal_step_tc(xv[u].w, zv[u].w, tv[u].w, (k + 3 < p.kb) ? d[3] : 0.0f, p.inv_p, p.lam);
                            __stcs(reinterpret_cast<float4 *>(p.x + base + u * ks), xv[u]);
                            __stcs(reinterpret_cast<float4 *>(p.z + base + u * ks), zv[u]);
                            if (p.xb)
                                *reinterpret_cast<uint2 *>(p.xb + base + u * ks) =
                                    make_uint2(pack2(xv[u].x, xv[u].y), pack2(xv[u].z, xv[u].w));
                        }
                    }
                }
                epilogue_sync();                                  // staging read before it is written again
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (tid == 32) mbar_wait(done, 0, DFX_TC_TIMEOUT, &g_tcb_flags);     // every MMA has completed
    if (tid == 128) {
        // windows loaded but never consumed (only after an expired wait): let them land before the CTA exits
        for (int g = *n_used; g < *n_issued; ++g)
            if (!mbar_wait(full0 + 8 * (g % TB_STAGES), (g / TB_STAGES) & 1, DFX_TC_TIMEOUT, &g_tcb_flags)) break;
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    }
}

size_t tb_smem_bytes(int n_angles)
{
    return 1024 + (size_t)TB_STAGES * TB_B_BYTES + 4 * TB_A_BYTES + TP_STAGE_BYTES +
           sizeof(AngleParams) * (size_t)n_angles + (2 * TB_STAGES + 5) * 8 + 16;
}

}  // namespace

unsigned int tcb_status(unsigned int reset)
{
    unsigned int f = 0;
    cudaMemcpyFromSymbol(&f, g_tcb_flags, sizeof(f));
    if (reset) {
        const unsigned int zero = 0;
        cudaMemcpyToSymbol(g_tcb_flags, &zero, sizeof(zero));
    }
    return f;
}

}  // namespace dfx

using namespace dfx;

extern "C" int dfx_radon_backward_spdhg_tc(const void *sino_bf16, int64_t sino_ld, const float *geo, int n_angles,
                                           int nx, int ny, int n_det, int kstride, int kb, int kernel, int n_taps,
                                           float *x_k, float *z_k, const float *T_k, float inv_p, float lam,
                                           void *x_bf16, void *stream)
{
    DFX_REQUIRE(sino_bf16 && geo && x_k && z_k && T_k, "radon_backward_spdhg_tc: null pointer");
    DFX_REQUIRE(((uintptr_t)sino_bf16 % 16) == 0 && ((uintptr_t)geo % 16) == 0 && ((uintptr_t)x_k % 16) == 0 &&
                    ((uintptr_t)z_k % 16) == 0 && ((uintptr_t)T_k % 16) == 0 && ((uintptr_t)x_bf16 % 16) == 0,
                "radon_backward_spdhg_tc: arrays must be 16-byte aligned");
    DFX_REQUIRE(n_angles >= 0 && n_angles <= 1024 && nx > 0 && ny > 0 && n_det > 0,
                "radon_backward_spdhg_tc: bad sizes (angles %d, %d x %d, %d bins)", n_angles, nx, ny, n_det);
    DFX_REQUIRE(kstride > 0 && kstride % 16 == 0 && kb >= 0 && kb <= kstride,
                "radon_backward_spdhg_tc: kstride (%d) must be a positive multiple of 16 and kb (%d) <= kstride",
                kstride, kb);
    DFX_REQUIRE(sino_ld >= kstride && sino_ld % 8 == 0, "radon_backward_spdhg_tc: bad sinogram row stride");
    DFX_REQUIRE(kernel == 0 || kernel == 1, "radon_backward_spdhg_tc: kernel must be 0 or 1");
    DFX_REQUIRE(n_taps >= 2 && n_taps <= 64, "radon_backward_spdhg_tc: n_taps (%d) out of range", n_taps);
    if (n_angles == 0 || kb == 0) return DFX_OK;
    CUtensorMap zmap;
    int st = tc::make_map(&zmap, sino_bf16, (uint64_t)kstride, (uint64_t)n_det, (uint64_t)n_angles,
                          (uint64_t)sino_ld, (uint64_t)sino_ld * n_det, 64, TB_KW, "Z");
    if (st) return st;
    TbArgs a{};
    a.n_angles = n_angles;
    a.nx = nx;
    a.ny = ny;
    a.ns = n_det;
    a.kstride = kstride;
    a.kb = kb;
    a.n_taps = n_taps;
    a.tiles_x = (int)cdiv(nx, TB_TX);
    a.x = x_k;
    a.z = z_k;
    a.T = T_k;
    a.xb = reinterpret_cast<__nv_bfloat16 *>(x_bf16);
    a.inv_p = inv_p;
    a.lam = lam;
    const int64_t ptiles = (int64_t)a.tiles_x * cdiv(ny, TB_TY);
    const int64_t n_tiles = ptiles * cdiv(kb, TB_N);
    DFX_REQUIRE(n_tiles < 2147483647LL, "radon_backward_spdhg_tc: batch too large");
    a.n_ptiles = (int)ptiles;
    a.n_tiles = (int)n_tiles;
    const size_t smem = tb_smem_bytes(n_angles);
    DFX_REQUIRE(smem <= 227 * 1024, "radon_backward_spdhg_tc: %d angles exceed the shared memory of one launch",
                n_angles);
    // one CTA per SM (a second one could not get tensor memory for both accumulators): its shared memory is more
    // than half of an SM's, so no two CTAs share an SM
    static_assert(2 * (4 * TB_B_BYTES + 4 * TB_A_BYTES + TP_STAGE_BYTES) > 228 * 1024, "one CTA per SM");
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                  cudaSuccess || sms <= 0) {
        set_error("radon_backward_spdhg_tc: cannot query the SM count");
        return DFX_ECUDA;
    }
    const dim3 grid((unsigned)(n_tiles < sms ? n_tiles : sms));
    cudaError_t e;
    if (kernel == 1) {
        e = allow_max_dynamic_smem(tc_backproject_spdhg<1>);
        if (e == cudaSuccess)
            tc_backproject_spdhg<1><<<grid, TP_THREADS, smem, (cudaStream_t)stream>>>(zmap, (const float4 *)geo, a);
    } else {
        e = allow_max_dynamic_smem(tc_backproject_spdhg<0>);
        if (e == cudaSuccess)
            tc_backproject_spdhg<0><<<grid, TP_THREADS, smem, (cudaStream_t)stream>>>(zmap, (const float4 *)geo, a);
    }
    if (e != cudaSuccess) {
        set_error("radon_backward_spdhg_tc: shared memory attribute: %s", cudaGetErrorString(e));
        return DFX_ELAUNCH;
    }
    return launch_status("radon_backward_spdhg_tc");
}
