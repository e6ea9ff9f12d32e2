// Sparse PF products (FP32), sm_100a.
//
// Both products are "CSR rows x dense lines": output row q (a segment j of the forward product, an orientation k of
// the adjoint) of one rotation angle is the sum over the row's entries (c, v) of v * X[y, c], for SP_TY detector
// lines y at once. A block owns one angle, SP_TY lines and SP_ROWS rows (one per thread). It stages X[y0 .. y0+TY,
// a chunk of columns] in shared memory transposed (the TY values of one column contiguous, read as float4); every
// thread walks its row's entries in groups of four, loading the next group while it applies the current one, and
// uses each entry TY times from a register. Rows are sorted by column, so a thread keeps its place from one chunk to
// the next. No atomics: every output is written by one thread. The adjoint launches spmm_adjoint8_kernel (eight lines
// per thread, the whole data row staged at once); the forward over stored copies runs over eta blocks
// (spmm_forward_b4_kernel), the CSR kernel serving generated copies. The lines-fastest forms turn the work around:
// the dense operand (the Radon output for the forward, the data rows for the adjoint) is first transposed to detector
// lines fastest, then a warp walks one row's entries with its lanes on the lines, reading every entry once and a
// whole 128-byte segment of the column per 32 lines (spmm_forward_zt_kernel, spmm_adjoint_zt_kernel); their sums
// are the kernels' above bit for bit.
#include "dfx_common.cuh"

#include <algorithm>

namespace dfx {

constexpr int SP_ROWS = 256;              // CSR rows per block
constexpr int SP_TY = 16;                 // detector lines per block
constexpr int SP_TYP = SP_TY + 4;         // padded column (float4 alignment, fewer bank conflicts)
constexpr int SP_CHUNK = 512;             // columns staged per pass: 512 * 20 * 4 B = 40 KB (5 blocks per SM)

struct Group {
    int c[4];
    float v[4];
};

__device__ __forceinline__ void load_group(Group &g, const uint16_t *__restrict__ col, const float *__restrict__ val,
                                           int i, int e)
{
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const bool ok = i + u < e;
        g.c[u] = ok ? (int)__ldg(col + i + u) : 0x7fffffff;
        g.v[u] = ok ? __ldg(val + i + u) : 0.0f;
    }
}

__device__ __forceinline__ void fma_col(float (&acc)[SP_TY], const float *tile, int c, float v)
{
    const float4 *t4 = reinterpret_cast<const float4 *>(tile + c * SP_TYP);
#pragma unroll
    for (int q = 0; q < SP_TY / 4; ++q) {
        const float4 z = t4[q];
        acc[4 * q + 0] = __fmaf_rn(v, z.x, acc[4 * q + 0]);
        acc[4 * q + 1] = __fmaf_rn(v, z.y, acc[4 * q + 1]);
        acc[4 * q + 2] = __fmaf_rn(v, z.z, acc[4 * q + 2]);
        acc[4 * q + 3] = __fmaf_rn(v, z.w, acc[4 * q + 3]);
    }
}

// Applies the entries i, i+1, ... of a row (ending at e) whose columns are below c_end; g holds the group starting
// at i on entry and the group starting at the returned index on exit.
__device__ __forceinline__ int walk_row(float (&acc)[SP_TY], const float *tile, const uint16_t *__restrict__ col,
                                        const float *__restrict__ val, int i, int e, Group &g, int c_begin,
                                        int c_end)
{
    while (i < e) {
        if (g.c[3] < c_end) {                     // the whole group lies in this chunk (or past e: c = max)
            Group n;
            load_group(n, col, val, i + 4, e);    // in flight while the current group is applied
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (i + u < e) fma_col(acc, tile, g.c[u] - c_begin, g.v[u]);
            g = n;
            i += 4;
        } else {                                  // the chunk ends inside the group: entry by entry
            int u = 0;
            while (u < 4 && i + u < e && g.c[u] < c_end) {
                fma_col(acc, tile, g.c[u] - c_begin, g.v[u]);
                ++u;
            }
            if (u < 4 && i + u < e) {             // stopped at the chunk boundary: realign the group
                i += u;
                load_group(g, col, val, i, e);
                return i;
            }
            i += u;
            load_group(g, col, val, i, e);
        }
    }
    return i;
}

// stage lines line0 .. line0+ny of X (stride ld) at columns c_begin .. c_begin+cn into tile[c][t]
__device__ __forceinline__ void stage(float *tile, const float *__restrict__ X, int64_t line0, int64_t ld, int ny,
                                      int c_begin, int cn)
{
    for (int idx = threadIdx.x; idx < SP_TY * cn; idx += blockDim.x) {
        const int t = idx / cn, c = idx - t * cn;
        tile[c * SP_TYP + t] = t < ny ? __ldg(X + (line0 + t) * ld + c_begin + c) : 0.0f;
    }
}

// forward: data[r, y, j] += sum_k PF[k, j] sino[s, y, k]   (rows j over the forward CSR)
__global__ void __launch_bounds__(SP_ROWS) spmm_forward_kernel(
    const float *__restrict__ sino, const int32_t *__restrict__ row_ptr, const uint16_t *__restrict__ col_k,
    const float *__restrict__ val, float *__restrict__ data, const int32_t *__restrict__ omegas, int my, int cp,
    int kstride, int kb, int compact)
{
    __shared__ __align__(16) float tile[SP_CHUNK * SP_TYP];
    const int j = blockIdx.x * SP_ROWS + threadIdx.x;
    const int y0 = blockIdx.y * SP_TY;
    const int s = blockIdx.z;
    const int r = omegas ? __ldg(omegas + s) : s;
    const int ny = min(SP_TY, my - y0);
    int i = 0, e = 0;
    if (j < cp) {
        const int64_t rr = (int64_t)(compact ? s : r) * cp + j;
        i = __ldg(row_ptr + rr);
        e = __ldg(row_ptr + rr + 1);
    }
    const bool nonempty = i < e;
    Group g;
    load_group(g, col_k, val, i, e);
    float acc[SP_TY];
#pragma unroll
    for (int t = 0; t < SP_TY; ++t) acc[t] = 0.0f;
    for (int c0 = 0; c0 < kb; c0 += SP_CHUNK) {
        const int cn = min(SP_CHUNK, kb - c0);
        if (c0) __syncthreads();
        stage(tile, sino, (int64_t)s * my + y0, kstride, ny, c0, cn);
        __syncthreads();
        i = walk_row(acc, tile, col_k, val, i, e, g, c0, c0 + cn);
    }
    if (j < cp && nonempty) {
        // all old values loaded before the first store (one round trip, not one per line)
        float *dl = data + ((int64_t)r * my + y0) * cp + j;
        float old[SP_TY];
#pragma unroll
        for (int t = 0; t < SP_TY; ++t) old[t] = t < ny ? dl[(int64_t)t * cp] : 0.0f;
#pragma unroll
        for (int t = 0; t < SP_TY; ++t)
            if (t < ny) dl[(int64_t)t * cp] = old[t] + acc[t];
    }
}

// ---- adjoint with eight lines per thread ----
// adjoint: sino[s, y, k] = alpha sum_j PF[k, j] data[r, y, j] (rows k over the adjoint CSR), per row k over its
// entries j ascending, fmaf from 0, times alpha, with the
// work laid out for the adjoint's shape: a block owns AJ_ROWS orientations of one angle and AJ_TY detector lines and
// stages those lines of the data row as wide as shared memory allows (the whole row for CP <= AJ_MAX_CHUNK), so a thread
// walks its row in one pass with no chunk boundaries. The staged lines are split in two halves of four (half h of
// column c at float4 index h * cn + c): the two 16-byte loads of an entry fall on bank groups that depend on c alone,
// spreading a warp's random columns over all eight groups.
constexpr int AJ_TY = 8;
constexpr int AJ_ROWS = 512;
constexpr int AJ_MAX_CHUNK = 3072;        // 3072 columns x 8 lines x 4 B = 96 KB (two blocks per SM)

__global__ void __launch_bounds__(AJ_ROWS) spmm_adjoint8_kernel(
    const float *__restrict__ data, const int32_t *__restrict__ row_ptr, const uint16_t *__restrict__ col_j,
    const float *__restrict__ val, float *__restrict__ sino, const int32_t *__restrict__ omegas, int my, int kb,
    int cp, int kstride, float alpha, int compact, int chunk)
{
    extern __shared__ __align__(16) float4 tile4[];
    float *tile = reinterpret_cast<float *>(tile4);
    const int k = blockIdx.x * AJ_ROWS + threadIdx.x;
    const int y0 = blockIdx.y * AJ_TY;
    const int s = blockIdx.z;
    const int r = omegas ? __ldg(omegas + s) : s;
    const int ny = min(AJ_TY, my - y0);
    int i = 0, e = 0;
    if (k < kb) {
        const int64_t rr = (int64_t)(compact ? s : r) * kb + k;
        i = __ldg(row_ptr + rr);
        e = __ldg(row_ptr + rr + 1);
    }
    Group g;
    load_group(g, col_j, val, i, e);
    float acc[AJ_TY];
#pragma unroll
    for (int t = 0; t < AJ_TY; ++t) acc[t] = 0.0f;
    const int64_t line0 = (int64_t)r * my + y0;
    if (chunk == cp) {
        // the whole row in one pass: entries loaded four at a time (8-byte columns, 16-byte values) once the row
        // position is a multiple of four, the same entries in the same order as the general loop below
        for (int idx = threadIdx.x; idx < AJ_TY * cp; idx += blockDim.x) {
            const int t = idx / cp, c = idx - t * cp;
            tile[((t >> 2) * cp + c) * 4 + (t & 3)] = t < ny ? __ldg(data + (line0 + t) * cp + c) : 0.0f;
        }
        __syncthreads();
        const bool vec = ((reinterpret_cast<uintptr_t>(col_j) & 7) == 0) &&
                         ((reinterpret_cast<uintptr_t>(val) & 15) == 0);
        auto apply = [&](int c, float v) {
            const float4 z0 = tile4[c], z1 = tile4[cp + c];
            acc[0] = __fmaf_rn(v, z0.x, acc[0]);
            acc[1] = __fmaf_rn(v, z0.y, acc[1]);
            acc[2] = __fmaf_rn(v, z0.z, acc[2]);
            acc[3] = __fmaf_rn(v, z0.w, acc[3]);
            acc[4] = __fmaf_rn(v, z1.x, acc[4]);
            acc[5] = __fmaf_rn(v, z1.y, acc[5]);
            acc[6] = __fmaf_rn(v, z1.z, acc[6]);
            acc[7] = __fmaf_rn(v, z1.w, acc[7]);
        };
        if (vec) {
            for (; i < e && (i & 3); ++i) apply(__ldg(col_j + i), __ldg(val + i));
            if (i + 4 <= e) {
                uint2 cc = __ldg(reinterpret_cast<const uint2 *>(col_j + i));
                float4 vv = __ldg(reinterpret_cast<const float4 *>(val + i));
                for (; i + 4 <= e; i += 4) {
                    uint2 cn_ = cc;
                    float4 vn_ = vv;
                    if (i + 8 <= e) {              // the next four in flight while these are applied
                        cn_ = __ldg(reinterpret_cast<const uint2 *>(col_j + i + 4));
                        vn_ = __ldg(reinterpret_cast<const float4 *>(val + i + 4));
                    }
                    apply((int)(cc.x & 0xffffu), vv.x);
                    apply((int)(cc.x >> 16), vv.y);
                    apply((int)(cc.y & 0xffffu), vv.z);
                    apply((int)(cc.y >> 16), vv.w);
                    cc = cn_;
                    vv = vn_;
                }
            }
        }
        for (; i < e; ++i) apply(__ldg(col_j + i), __ldg(val + i));
    }
    for (int c0 = 0; c0 < cp && chunk < cp; c0 += chunk) {
        const int cn = min(chunk, cp - c0);
        if (c0) __syncthreads();
        for (int idx = threadIdx.x; idx < AJ_TY * cn; idx += blockDim.x) {
            const int t = idx / cn, c = idx - t * cn;
            tile[((t >> 2) * cn + c) * 4 + (t & 3)] = t < ny ? __ldg(data + (line0 + t) * cp + c0 + c) : 0.0f;
        }
        __syncthreads();
        const int c_end = c0 + cn;
        while (i < e && g.c[0] < c_end) {
            Group n;
            const bool whole = g.c[3] < c_end;             // the group lies in this chunk (or ends the row)
            if (whole) load_group(n, col_j, val, i + 4, e);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (i + u >= e || g.c[u] >= c_end) break;
                const int c = g.c[u] - c0;
                const float4 z0 = tile4[c], z1 = tile4[cn + c];
                const float v = g.v[u];
                acc[0] = __fmaf_rn(v, z0.x, acc[0]);
                acc[1] = __fmaf_rn(v, z0.y, acc[1]);
                acc[2] = __fmaf_rn(v, z0.z, acc[2]);
                acc[3] = __fmaf_rn(v, z0.w, acc[3]);
                acc[4] = __fmaf_rn(v, z1.x, acc[4]);
                acc[5] = __fmaf_rn(v, z1.y, acc[5]);
                acc[6] = __fmaf_rn(v, z1.z, acc[6]);
                acc[7] = __fmaf_rn(v, z1.w, acc[7]);
            }
            if (whole) {
                g = n;
                i += 4;
            } else {                                        // the chunk ends inside the group: realign at its end
                int u = 0;
                while (u < 4 && i + u < e && g.c[u] < c_end) ++u;
                i += u;
                load_group(g, col_j, val, i, e);
            }
        }
    }
    if (k < kstride) {
        float *zl = sino + ((int64_t)s * my + y0) * kstride + k;
#pragma unroll
        for (int t = 0; t < AJ_TY; ++t)
            if (t < ny) zl[(int64_t)t * kstride] = k < kb ? alpha * acc[t] : 0.0f;
    }
}

// ---- eta-blocked forward rows ----
// The forward CSR of a batch (rows r * CP + j, j = c * P + p, each listing its orientations k ascending) regrouped
// into block rows (r, cb, p), q = cb * P + p: the rows of the eta bins c = 4 cb .. 4 cb + 3 of ring p merged into one
// list of k ascending whose entries carry four values (0 where that bin's row has no entry k). Neighbouring eta bins
// of a ring share most orientations (a kernel's pole figure crosses a ring over several bins), so an entry's Z column
// is staged once for four outputs. mask bit u: the row of bin 4 cb + u has entries (its output is written). Rings run
// fastest, so the 32 threads of a warp (eight rings of four eta blocks) store to four 32-byte sectors per line.
constexpr int FB_W = 4;

__device__ __forceinline__ int fb_heads(const int32_t *__restrict__ row_ptr, int64_t row0, int P, int C, int cb,
                                        int (&b)[FB_W], int (&e)[FB_W])
{
    int m = 0;
#pragma unroll
    for (int u = 0; u < FB_W; ++u) {
        const int c = FB_W * cb + u;
        b[u] = e[u] = 0;
        if (c < C) {
            const int64_t row = row0 + (int64_t)c * P;
            b[u] = __ldg(row_ptr + row);
            e[u] = __ldg(row_ptr + row + 1);
        }
        m |= (b[u] < e[u]) << u;
    }
    return m;
}

// FILL 0: counts[q] = entries of block row q, mask[q]; FILL 1: the entries at fb_ptr[q] ...
template <int FILL>
__global__ void fb_build_kernel(const int32_t *__restrict__ row_ptr, const uint16_t *__restrict__ col_k,
                                const float *__restrict__ val, int64_t n_blocks, int P, int C, int ncb,
                                int32_t *__restrict__ counts, uint8_t *__restrict__ mask,
                                const int32_t *__restrict__ fb_ptr, uint16_t *__restrict__ fb_k,
                                float4 *__restrict__ fb_v)
{
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_blocks) return;
    const int64_t per_angle = (int64_t)P * ncb;
    const int64_t r = g / per_angle;
    const int q = (int)(g - r * per_angle), cb = q / P, p = q - (q / P) * P;
    int b[FB_W], e[FB_W];
    const int m = fb_heads(row_ptr, r * (int64_t)C * P + p, P, C, cb, b, e);
    int head[FB_W];
#pragma unroll
    for (int u = 0; u < FB_W; ++u) head[u] = b[u] < e[u] ? (int)__ldg(col_k + b[u]) : 0x10000;
    int n = 0;
    int64_t o = FILL ? __ldg(fb_ptr + g) : 0;
    while (true) {
        int k = 0x10000;
#pragma unroll
        for (int u = 0; u < FB_W; ++u) k = min(k, head[u]);
        if (k == 0x10000) break;
        float v[FB_W];
#pragma unroll
        for (int u = 0; u < FB_W; ++u) {
            v[u] = 0.0f;
            if (head[u] == k) {
                if (FILL) v[u] = __ldg(val + b[u]);
                ++b[u];
                head[u] = b[u] < e[u] ? (int)__ldg(col_k + b[u]) : 0x10000;
            }
        }
        if (FILL) {
            fb_k[o] = (uint16_t)k;
            fb_v[o] = make_float4(v[0], v[1], v[2], v[3]);
            ++o;
        }
        ++n;
    }
    if (!FILL) {
        counts[g] = n;
        mask[g] = (uint8_t)m;
    }
}

// forward over the blocked rows: data[r, y, (4 cb + u) P + p] += sum_k v_u sino[s, y, k] for the bins with entries.
// A thread owns one block row and SP_TY lines (4 x SP_TY accumulators); per entry one staged column of SP_TY values
// feeds 4 SP_TY fused multiply-adds. The sums run over k ascending from 0 with fmaf, as spmm_forward_kernel's: a zero
// value adds exactly 0, so the results are that kernel's bit for bit.
__global__ void __launch_bounds__(SP_ROWS) spmm_forward_b4_kernel(
    const float *__restrict__ sino, const int32_t *__restrict__ fb_ptr, const uint16_t *__restrict__ fb_k,
    const float4 *__restrict__ fb_v, const uint8_t *__restrict__ fb_mask, float *__restrict__ data,
    const int32_t *__restrict__ omegas, int my, int P, int C, int ncb, int kstride, int kb)
{
    __shared__ __align__(16) float tile[SP_CHUNK * SP_TYP];
    const int per_angle = P * ncb;
    const int q = blockIdx.x * SP_ROWS + threadIdx.x;
    const int y0 = blockIdx.y * SP_TY;
    const int s = blockIdx.z;
    const int r = omegas ? __ldg(omegas + s) : s;
    const int ny = min(SP_TY, my - y0);
    int i = 0, e = 0, m = 0;
    if (q < per_angle) {
        const int64_t g = (int64_t)r * per_angle + q;
        i = __ldg(fb_ptr + g);
        e = __ldg(fb_ptr + g + 1);
        m = __ldg(fb_mask + g);
    }
    int kn = i < e ? (int)__ldg(fb_k + i) : 0x7fffffff;
    float4 vn = i < e ? __ldg(fb_v + i) : make_float4(0.f, 0.f, 0.f, 0.f);
    float acc[FB_W][SP_TY];
#pragma unroll
    for (int u = 0; u < FB_W; ++u)
#pragma unroll
        for (int t = 0; t < SP_TY; ++t) acc[u][t] = 0.0f;
    for (int c0 = 0; c0 < kb; c0 += SP_CHUNK) {
        const int cn = min(SP_CHUNK, kb - c0);
        if (c0) __syncthreads();
        stage(tile, sino, (int64_t)s * my + y0, kstride, ny, c0, cn);
        __syncthreads();
        while (kn < c0 + cn) {
            const int k = kn;
            const float4 v = vn;
            ++i;
            kn = i < e ? (int)__ldg(fb_k + i) : 0x7fffffff;
            vn = i < e ? __ldg(fb_v + i) : make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 *t4 = reinterpret_cast<const float4 *>(tile + (k - c0) * SP_TYP);
#pragma unroll
            for (int w = 0; w < SP_TY / 4; ++w) {
                const float4 z = t4[w];
                const float zz[4] = {z.x, z.y, z.z, z.w};
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    acc[0][4 * w + h] = __fmaf_rn(v.x, zz[h], acc[0][4 * w + h]);
                    acc[1][4 * w + h] = __fmaf_rn(v.y, zz[h], acc[1][4 * w + h]);
                    acc[2][4 * w + h] = __fmaf_rn(v.z, zz[h], acc[2][4 * w + h]);
                    acc[3][4 * w + h] = __fmaf_rn(v.w, zz[h], acc[3][4 * w + h]);
                }
            }
        }
    }
    if (q < per_angle && m) {
        const int cb = q / P, p = q - cb * P;
        const int cp = C * P;
        float *dl = data + ((int64_t)r * my + y0) * cp + p;
#pragma unroll
        for (int u = 0; u < FB_W; ++u) {
            if (!((m >> u) & 1)) continue;
            float *d = dl + (int64_t)(FB_W * cb + u) * P;
#pragma unroll
            for (int t = 0; t < SP_TY; ++t)
                if (t < ny) d[(int64_t)t * cp] += acc[u][t];
        }
    }
}

// ---- blocked forward over the lines-fastest sinogram ----
// zt[s][k][y] (line stride ly = 32 * groups, lines my .. ly - 1 zero) is the Radon output of one launch's angles with
// the detector lines fastest. A warp applies one block row (four eta bins of one ring) of one angle at a time to up
// to 32 ZT_G lines: lane l holds the lines y0 + l + 32 t. Per entry the warp reads the entry once (the same address in
// every lane) and one coalesced 128-byte segment of Z column k per 32 lines, four entries in flight, and applies the
// entry's four values with paired fused multiply-adds (fma.rn.f32x2: two IEEE fmaf in one instruction, lines t and
// t + 1). A block of 8 warps owns the block rows of nb consecutive eta blocks, all rings (nb * P <= 16 rows; one eta
// block above 16 rings), whose outputs j = 4 cb P .. 4 (cb + nb) P - 1 are contiguous in a data row. The rows differ
// in length, so the warps take them longest first from a shared counter instead of one row each: the block no longer
// waits for its longest row with most warps idle. The sums go to shared memory; the block's data row segments, put in
// L2 by a prefetch when the block starts, are then read a batch of lines at a time and written back whole. The sums
// per output run over the block row's entries in order with fmaf, each added once to the data row, as in
// spmm_forward_b4_kernel: the results are that kernel's (and the CSR kernel's) bit for bit.
constexpr int ZT_G = 9;                  // 32-line groups per warp at most (288 lines)
constexpr int ZT_U = 4;                  // entries in flight per warp
constexpr int ZT_TR = 32;                // transpose tile

// zt[s][k][y] = sino[s][y][k] (k < kb, y < my; zero for my <= y < ly)
__global__ void __launch_bounds__(256) zt_transpose_kernel(const float *__restrict__ sino, float *__restrict__ zt,
                                                           int my, int ly, int kstride, int kb)
{
    __shared__ float tile[ZT_TR][ZT_TR + 1];
    const int s = blockIdx.z, k0 = blockIdx.x * ZT_TR, y0 = blockIdx.y * ZT_TR;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int yy = ty; yy < ZT_TR; yy += 8) {
        const int y = y0 + yy, k = k0 + tx;
        tile[yy][tx] = (y < my && k < kb) ? __ldg(sino + ((int64_t)s * my + y) * kstride + k) : 0.0f;
    }
    __syncthreads();
    for (int kk = ty; kk < ZT_TR; kk += 8) {
        const int k = k0 + kk;
        if (k < kb) zt[((int64_t)s * kb + k) * ly + y0 + tx] = tile[tx][kk];
    }
}

// a0 = fmaf(v, z0, a0), a1 = fmaf(v, z1, a1) in one instruction (same rounding as two fmaf)
__device__ __forceinline__ void fma_pair(float &a0, float &a1, float v, float z0, float z1)
{
    const float2 r = __ffma2_rn(make_float2(v, v), make_float2(z0, z1), make_float2(a0, a1));
    a0 = r.x;
    a1 = r.y;
}

constexpr int ZT_ROWS_MAX = 32;         // block rows per block at most (one eta block of 32 rings)
constexpr int ZT_NB_LINES = 9;           // data row lines read per batch in the write-back

template <int MT>
__global__ void __launch_bounds__(256, 2) spmm_forward_zt_kernel(
    const float *__restrict__ zt, const int32_t *__restrict__ fb_ptr, const uint16_t *__restrict__ fb_k,
    const float4 *__restrict__ fb_v, const uint8_t *__restrict__ fb_mask, float *__restrict__ data,
    const int32_t *__restrict__ omegas, int r0, int my, int ly, int P, int C, int ncb, int nb, int kb)
{
    extern __shared__ __align__(16) float s_out[];    // [32 MT][width + 1]: the block's sums
    __shared__ uint8_t s_own[FB_W * ZT_ROWS_MAX];      // output j of the block written (its bin's row has entries)
    __shared__ int s_order[ZT_ROWS_MAX];               // the block's rows, longest first
    __shared__ int s_next;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int s = blockIdx.z;
    const int r = omegas ? __ldg(omegas + s) : r0 + s;
    const int ngroups = ly >> 5;
    const int g0 = blockIdx.y * MT;                   // first 32-line group of the block
    const int y0 = g0 * 32;
    const int cb0 = blockIdx.x * nb;
    const int nrows = nb * P;                         // row q: eta block cb0 + q / P, ring q % P
    const int width = FB_W * nb * P, wp = width + 1;
    const int cp = C * P;
    const int j0 = FB_W * cb0 * P;                    // first output of the block in a data row
    const int wj = min(width, cp - j0);
    const int ny = min(32 * MT, my - y0);
    float *drow = data + ((int64_t)r * my + y0) * cp + j0;
    // the data row segments into L2 while the rows are summed (read and written back at the end)
    const int lines = (wj + 31) >> 5;
    for (int idx = tid; idx < ny * lines; idx += blockDim.x) {
        const int yl = idx / lines, c = idx - yl * lines;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(drow + (int64_t)yl * cp + 32 * c));
    }
    for (int t = tid; t < width; t += blockDim.x) s_own[t] = 0;
    if (warp == 0) {                                  // rank of every row by length (ties: lower row first)
        int len = -1;
        if (lane < nrows) {
            const int cb = cb0 + lane / P, p = lane - (lane / P) * P;
            if (cb < ncb) {
                const int64_t g = (int64_t)r * P * ncb + (int64_t)cb * P + p;
                len = __ldg(fb_ptr + g + 1) - __ldg(fb_ptr + g);
            }
        }
        int rank = 0;
        for (int j = 0; j < nrows; ++j) {
            const int lj = __shfl_sync(0xffffffffu, len, j);
            rank += (lj > len || (lj == len && j < lane)) ? 1 : 0;
        }
        if (lane < nrows) s_order[rank] = lane;
        if (lane == 0) s_next = 0;
    }
    __syncthreads();
    const float *zs = zt + (int64_t)s * kb * ly + y0 + lane;
    while (true) {
        int idx = 0;
        if (lane == 0) idx = atomicAdd(&s_next, 1);
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (idx >= nrows) break;
        const int q = s_order[idx], cbw = q / P, p = q - cbw * P, cb = cb0 + cbw;
        if (cb >= ncb) continue;
        const int64_t g = (int64_t)r * P * ncb + (int64_t)cb * P + p;
        int i = __ldg(fb_ptr + g);
        const int e = __ldg(fb_ptr + g + 1);
        const int m = __ldg(fb_mask + g);
        float acc[FB_W][MT];
#pragma unroll
        for (int u = 0; u < FB_W; ++u)
#pragma unroll
            for (int t = 0; t < MT; ++t) acc[u][t] = 0.0f;
        int kq[ZT_U];
        float4 vq[ZT_U];
#pragma unroll
        for (int qq = 0; qq < ZT_U; ++qq) {
            kq[qq] = i + qq < e ? __ldg(fb_k + i + qq) : 0;
            vq[qq] = i + qq < e ? __ldg(fb_v + i + qq) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        for (; i < e; i += ZT_U) {
            float4 vc[ZT_U];
            float z[ZT_U][MT];
#pragma unroll
            for (int qq = 0; qq < ZT_U; ++qq) {
                vc[qq] = vq[qq];
                const float *zc = zs + (int64_t)kq[qq] * ly;
#pragma unroll
                for (int t = 0; t < MT; ++t) z[qq][t] = g0 + t < ngroups ? __ldg(zc + 32 * t) : 0.0f;
            }
#pragma unroll
            for (int qq = 0; qq < ZT_U; ++qq) {        // the next entries' loads go out while these are applied
                kq[qq] = i + ZT_U + qq < e ? __ldg(fb_k + i + ZT_U + qq) : 0;
                vq[qq] = i + ZT_U + qq < e ? __ldg(fb_v + i + ZT_U + qq) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int qq = 0; qq < ZT_U; ++qq) {
                if (i + qq < e) {
#pragma unroll
                    for (int t = 0; t + 1 < MT; t += 2) {
                        fma_pair(acc[0][t], acc[0][t + 1], vc[qq].x, z[qq][t], z[qq][t + 1]);
                        fma_pair(acc[1][t], acc[1][t + 1], vc[qq].y, z[qq][t], z[qq][t + 1]);
                        fma_pair(acc[2][t], acc[2][t + 1], vc[qq].z, z[qq][t], z[qq][t + 1]);
                        fma_pair(acc[3][t], acc[3][t + 1], vc[qq].w, z[qq][t], z[qq][t + 1]);
                    }
                    if (MT & 1) {
                        acc[0][MT - 1] = __fmaf_rn(vc[qq].x, z[qq][MT - 1], acc[0][MT - 1]);
                        acc[1][MT - 1] = __fmaf_rn(vc[qq].y, z[qq][MT - 1], acc[1][MT - 1]);
                        acc[2][MT - 1] = __fmaf_rn(vc[qq].z, z[qq][MT - 1], acc[2][MT - 1]);
                        acc[3][MT - 1] = __fmaf_rn(vc[qq].w, z[qq][MT - 1], acc[3][MT - 1]);
                    }
                }
            }
        }
        const int jl = FB_W * cbw * P + p;            // local j of bin u: (4 cbw + u) P + p
#pragma unroll
        for (int u = 0; u < FB_W; ++u) {
#pragma unroll
            for (int t = 0; t < MT; ++t) s_out[(lane + 32 * t) * wp + jl + u * P] = acc[u][t];
            if (lane == 0) s_own[jl + u * P] = (uint8_t)((m >> u) & 1);
        }
    }
    __syncthreads();
    // write-back: per pass rows_per_pass lines of the segment, the old values of ZT_NB_LINES passes loaded first
    const int rows_per_pass = blockDim.x / width;     // at least 2: width <= 128
    const int tj = tid % width, ty = tid / width;
    if (ty < rows_per_pass && s_own[tj]) {
        for (int yb = ty; yb < ny; yb += ZT_NB_LINES * rows_per_pass) {
            float old[ZT_NB_LINES];
#pragma unroll
            for (int n = 0; n < ZT_NB_LINES; ++n) {
                const int yl = yb + n * rows_per_pass;
                old[n] = yl < ny ? drow[(int64_t)yl * cp + tj] : 0.0f;
            }
#pragma unroll
            for (int n = 0; n < ZT_NB_LINES; ++n) {
                const int yl = yb + n * rows_per_pass;
                if (yl < ny) drow[(int64_t)yl * cp + tj] = old[n] + s_out[yl * wp + tj];
            }
        }
    }
}

// ---- adjoint over the lines-fastest data rows ----
// dt[s][j][y] (line stride ly, lines my .. ly - 1 zero): the data rows of one launch's angles with the detector lines
// fastest. A warp owns kw (1, 2 or 4) consecutive orientation rows k of one angle, one after the other, and up to
// 32 ZT_G lines (lane l: lines y0 + l + 32 t); per entry (j, v) of a row it reads the entry once and one coalesced
// 128-byte segment of column j per 32 lines, four entries in flight, paired fused multiply-adds. A block's 8 warps
// hold 8 kw consecutive orientations, written as whole row segments of the Radon input through shared memory (kw is
// the largest that still gives the launch a few waves of blocks). Per output the sum runs over the row's entries in
// order with fmaf from 0 and is scaled by alpha: spmm_adjoint8_kernel's bits.
constexpr int AZ_KW = 4;                 // orientation rows per warp at most
constexpr int AZ_WARPS = 8;

// dt[s][j][y] = data[r(s)][y][j] (j < cp, y < my; zero for my <= y < ly), r(s) = omegas[s] or r0 + s
__global__ void __launch_bounds__(256) dt_transpose_kernel(const float *__restrict__ data, float *__restrict__ dt,
                                                           const int32_t *__restrict__ omegas, int r0, int my, int ly,
                                                           int cp)
{
    __shared__ float tile[ZT_TR][ZT_TR + 1];
    const int s = blockIdx.z, j0 = blockIdx.x * ZT_TR, y0 = blockIdx.y * ZT_TR;
    const int r = omegas ? __ldg(omegas + s) : r0 + s;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int yy = ty; yy < ZT_TR; yy += 8) {
        const int y = y0 + yy, j = j0 + tx;
        tile[yy][tx] = (y < my && j < cp) ? __ldg(data + ((int64_t)r * my + y) * cp + j) : 0.0f;
    }
    __syncthreads();
    for (int jj = ty; jj < ZT_TR; jj += 8) {
        const int j = j0 + jj;
        if (j < cp) dt[((int64_t)s * cp + j) * ly + y0 + tx] = tile[tx][jj];
    }
}

template <int MT>
__global__ void __launch_bounds__(32 * AZ_WARPS, 3) spmm_adjoint_zt_kernel(
    const float *__restrict__ dt, const int32_t *__restrict__ row_ptr, const uint16_t *__restrict__ col_j,
    const float *__restrict__ val, float *__restrict__ sino, const int32_t *__restrict__ omegas, int r0, int my,
    int ly, int kb, int cp, int kstride, float alpha, int compact, int kw)
{
    extern __shared__ float s_outk[];                 // [32 MT][8 kw + 1]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.z;
    const int r = omegas ? __ldg(omegas + s) : r0 + s;
    const int ngroups = ly >> 5;
    const int g0 = blockIdx.y * MT;
    const int y0 = g0 * 32;
    const int nk = AZ_WARPS * kw, ldk = nk + 1;
    const int k0 = blockIdx.x * nk;
    const float *ds = dt + (int64_t)s * cp * ly + y0 + lane;
    for (int kk = 0; kk < kw; ++kk) {
        const int kl = warp * kw + kk, k = k0 + kl;
        int i = 0, e = 0;
        if (k < kb) {
            const int64_t rr = (int64_t)(compact ? s : r) * kb + k;
            i = __ldg(row_ptr + rr);
            e = __ldg(row_ptr + rr + 1);
        }
        float acc[MT];
#pragma unroll
        for (int t = 0; t < MT; ++t) acc[t] = 0.0f;
        int jq[ZT_U];
        float vq[ZT_U];
#pragma unroll
        for (int q = 0; q < ZT_U; ++q) {
            jq[q] = i + q < e ? __ldg(col_j + i + q) : 0;
            vq[q] = i + q < e ? __ldg(val + i + q) : 0.0f;
        }
        for (; i < e; i += ZT_U) {
            float vc[ZT_U];
            float z[ZT_U][MT];
#pragma unroll
            for (int q = 0; q < ZT_U; ++q) {
                vc[q] = vq[q];
                const float *zc = ds + (int64_t)jq[q] * ly;
#pragma unroll
                for (int t = 0; t < MT; ++t) z[q][t] = g0 + t < ngroups ? __ldg(zc + 32 * t) : 0.0f;
            }
#pragma unroll
            for (int q = 0; q < ZT_U; ++q) {
                jq[q] = i + ZT_U + q < e ? __ldg(col_j + i + ZT_U + q) : 0;
                vq[q] = i + ZT_U + q < e ? __ldg(val + i + ZT_U + q) : 0.0f;
            }
#pragma unroll
            for (int q = 0; q < ZT_U; ++q) {
                if (i + q < e) {
#pragma unroll
                    for (int t = 0; t + 1 < MT; t += 2) fma_pair(acc[t], acc[t + 1], vc[q], z[q][t], z[q][t + 1]);
                    if (MT & 1) acc[MT - 1] = __fmaf_rn(vc[q], z[q][MT - 1], acc[MT - 1]);
                }
            }
        }
#pragma unroll
        for (int t = 0; t < MT; ++t) s_outk[(lane + 32 * t) * ldk + kl] = k < kb ? alpha * acc[t] : 0.0f;
    }
    __syncthreads();
    const int ny = min(32 * MT, my - y0);
    const int kl = threadIdx.x % nk, ty = threadIdx.x / nk;
    const int k = k0 + kl;
    if (k < kstride) {
        float *zl = sino + ((int64_t)s * my + y0) * kstride + k;
        for (int yl = ty; yl < ny; yl += (32 * AZ_WARPS) / nk) zl[(int64_t)yl * kstride] = s_outk[yl * ldk + kl];
    }
}

}  // namespace dfx

using namespace dfx;

extern "C" int dfx_spmm_pf_forward(const float *sino, const int32_t *row_ptr, const uint16_t *col_k, const float *val,
                                   float *data, const int32_t *omegas, int n_sub, int my, int cp, int kstride, int kb,
                                   int compact, void *stream)
{
    DFX_REQUIRE(sino && row_ptr && col_k && val && data, "spmm_forward: null pointer");
    DFX_REQUIRE(n_sub > 0 && my > 0 && cp > 0 && kb > 0 && kb <= kstride, "spmm_forward: bad sizes");
    DFX_REQUIRE(n_sub <= 65535 && cdiv(my, SP_TY) <= 65535, "spmm_forward: grid too large");
    dim3 grid((unsigned)cdiv(cp, SP_ROWS), (unsigned)cdiv(my, SP_TY), (unsigned)n_sub);
    spmm_forward_kernel<<<grid, SP_ROWS, 0, (cudaStream_t)stream>>>(sino, row_ptr, col_k, val, data, omegas, my, cp,
                                                                    kstride, kb, compact);
    return launch_status("spmm_pf_forward");
}

extern "C" int dfx_spmm_pf_adjoint(const float *data, const int32_t *row_ptr, const uint16_t *col_j, const float *val,
                                   float *sino, const int32_t *omegas, int n_sub, int my, int kb, int cp, int kstride,
                                   float alpha, int compact, void *stream)
{
    DFX_REQUIRE(sino && row_ptr && col_j && val && data, "spmm_adjoint: null pointer");
    DFX_REQUIRE(n_sub > 0 && my > 0 && cp > 0 && kb > 0 && kb <= kstride, "spmm_adjoint: bad sizes");
    DFX_REQUIRE(n_sub <= 65535 && cdiv(my, SP_TY) <= 65535, "spmm_adjoint: grid too large");
    DFX_REQUIRE(cdiv(my, AJ_TY) <= 65535, "spmm_adjoint: grid too large");
    const int chunk = cp < AJ_MAX_CHUNK ? cp : AJ_MAX_CHUNK;
    const size_t smem = (size_t)AJ_TY * chunk * sizeof(float);
    const cudaError_t e = allow_max_dynamic_smem(spmm_adjoint8_kernel);
    if (e != cudaSuccess) {
        set_error("spmm_adjoint: shared memory attribute: %s", cudaGetErrorString(e));
        return DFX_ELAUNCH;
    }
    dim3 grid((unsigned)cdiv(kstride, AJ_ROWS), (unsigned)cdiv(my, AJ_TY), (unsigned)n_sub);
    spmm_adjoint8_kernel<<<grid, AJ_ROWS, smem, (cudaStream_t)stream>>>(data, row_ptr, col_j, val, sino, omegas, my,
                                                                        kb, cp, kstride, alpha, compact, chunk);
    return launch_status("spmm_pf_adjoint");
}

extern "C" int64_t dfx_pf_fblock_rows(int n_angles, int P, int C)
{
    return (int64_t)n_angles * P * cdiv(C, FB_W);
}

extern "C" int dfx_pf_fblock_count(const int32_t *row_ptr_f, const uint16_t *col_k, int n_angles, int P, int C,
                                   int32_t *counts, uint8_t *mask, void *stream)
{
    DFX_REQUIRE(row_ptr_f && col_k && counts && mask, "pf_fblock_count: null pointer");
    DFX_REQUIRE(n_angles > 0 && P > 0 && C > 0, "pf_fblock_count: bad sizes");
    const int ncb = (int)cdiv(C, FB_W);
    const int64_t n = dfx_pf_fblock_rows(n_angles, P, C);
    DFX_REQUIRE(cdiv(n, 256) < 2147483647LL, "pf_fblock_count: too many rows");
    fb_build_kernel<0><<<(unsigned)cdiv(n, 256), 256, 0, (cudaStream_t)stream>>>(
        row_ptr_f, col_k, nullptr, n, P, C, ncb, counts, mask, nullptr, nullptr, nullptr);
    return launch_status("pf_fblock_count");
}

extern "C" int dfx_pf_fblock_fill(const int32_t *row_ptr_f, const uint16_t *col_k, const float *val_f, int n_angles,
                                  int P, int C, const int32_t *fb_ptr, uint16_t *fb_k, float *fb_v, void *stream)
{
    DFX_REQUIRE(row_ptr_f && col_k && val_f && fb_ptr && fb_k && fb_v, "pf_fblock_fill: null pointer");
    DFX_REQUIRE(((uintptr_t)fb_v % 16) == 0, "pf_fblock_fill: the values must be 16-byte aligned");
    DFX_REQUIRE(n_angles > 0 && P > 0 && C > 0, "pf_fblock_fill: bad sizes");
    const int ncb = (int)cdiv(C, FB_W);
    const int64_t n = dfx_pf_fblock_rows(n_angles, P, C);
    fb_build_kernel<1><<<(unsigned)cdiv(n, 256), 256, 0, (cudaStream_t)stream>>>(
        row_ptr_f, col_k, val_f, n, P, C, ncb, nullptr, nullptr, fb_ptr, fb_k, reinterpret_cast<float4 *>(fb_v));
    return launch_status("pf_fblock_fill");
}

extern "C" int dfx_spmm_pf_forward_blocked(const float *sino, const int32_t *fb_ptr, const uint16_t *fb_k,
                                           const float *fb_v, const uint8_t *fb_mask, float *data,
                                           const int32_t *omegas, int n_sub, int my, int P, int C, int kstride, int kb,
                                           void *stream)
{
    DFX_REQUIRE(sino && fb_ptr && fb_k && fb_v && fb_mask && data, "spmm_forward_blocked: null pointer");
    DFX_REQUIRE(((uintptr_t)fb_v % 16) == 0, "spmm_forward_blocked: the values must be 16-byte aligned");
    DFX_REQUIRE(n_sub > 0 && my > 0 && P > 0 && C > 0 && kb > 0 && kb <= kstride, "spmm_forward_blocked: bad sizes");
    const int ncb = (int)cdiv(C, FB_W);
    DFX_REQUIRE(n_sub <= 65535 && cdiv(my, SP_TY) <= 65535, "spmm_forward_blocked: grid too large");
    dim3 grid((unsigned)cdiv((int64_t)P * ncb, SP_ROWS), (unsigned)cdiv(my, SP_TY), (unsigned)n_sub);
    spmm_forward_b4_kernel<<<grid, SP_ROWS, 0, (cudaStream_t)stream>>>(
        sino, fb_ptr, fb_k, reinterpret_cast<const float4 *>(fb_v), fb_mask, data, omegas, my, P, C, ncb, kstride,
        kb);
    return launch_status("spmm_pf_forward_blocked");
}

extern "C" int64_t dfx_spmm_pf_forward_zt_floats(int n_angles, int my, int kb)
{
    if (n_angles <= 0 || my <= 0 || kb <= 0) return -1;
    return (int64_t)n_angles * kb * (cdiv(my, 32) * 32);
}

template <int MT>
static int launch_zt(const float *zt, const int32_t *fb_ptr, const uint16_t *fb_k, const float *fb_v,
                     const uint8_t *fb_mask, float *data, const int32_t *omegas, int r0, int na, int my, int ly,
                     int nyb, int P, int C, int ncb, int nb, int kb, cudaStream_t st)
{
    const cudaError_t err = allow_max_dynamic_smem(spmm_forward_zt_kernel<MT>);
    if (err != cudaSuccess) {
        set_error("spmm_forward_blocked_zt: shared memory attribute: %s", cudaGetErrorString(err));
        return DFX_ELAUNCH;
    }
    const int width = FB_W * nb * P;
    const size_t smem = (size_t)32 * MT * (width + 1) * sizeof(float);
    dim3 grid((unsigned)cdiv(ncb, nb), (unsigned)nyb, (unsigned)na);
    spmm_forward_zt_kernel<MT><<<grid, 256, smem, st>>>(zt, fb_ptr, fb_k, reinterpret_cast<const float4 *>(fb_v),
                                                        fb_mask, data, omegas, r0, my, ly, P, C, ncb, nb, kb);
    return launch_status("spmm_pf_forward_blocked_zt");
}

extern "C" int dfx_spmm_pf_forward_blocked_zt(const float *sino, float *zt, int64_t zt_floats, const int32_t *fb_ptr,
                                              const uint16_t *fb_k, const float *fb_v, const uint8_t *fb_mask,
                                              float *data, const int32_t *omegas, int n_sub, int my, int P, int C,
                                              int kstride, int kb, int max_groups, void *stream)
{
    DFX_REQUIRE(sino && zt && fb_ptr && fb_k && fb_v && fb_mask && data, "spmm_forward_blocked_zt: null pointer");
    DFX_REQUIRE(((uintptr_t)fb_v % 16) == 0, "spmm_forward_blocked_zt: the values must be 16-byte aligned");
    DFX_REQUIRE(n_sub > 0 && my > 0 && P > 0 && C > 0 && kb > 0 && kb <= kstride,
                "spmm_forward_blocked_zt: bad sizes");
    DFX_REQUIRE(P <= 32, "spmm_forward_blocked_zt: more than 32 rings");
    const int64_t per_angle = dfx_spmm_pf_forward_zt_floats(1, my, kb);
    DFX_REQUIRE(zt_floats >= per_angle, "spmm_forward_blocked_zt: the transpose buffer holds less than one angle");
    const int ly = (int)(cdiv(my, 32) * 32), ngroups = ly / 32;
    DFX_REQUIRE(max_groups >= 0 && max_groups <= ZT_G, "spmm_forward_blocked_zt: max_groups outside 0 .. 9");
    const int gmax = max_groups ? max_groups : ZT_G;
    const int nyb = (int)cdiv(ngroups, gmax), mt = (int)cdiv(ngroups, nyb);
    // blocks of nb eta blocks x all rings: at most 16 rows (one eta block above 16 rings)
    const int nb = P >= 16 ? 1 : 16 / P;
    const int ncb = (int)cdiv(C, FB_W);
    DFX_REQUIRE(nyb <= 65535 && cdiv(kb, ZT_TR) <= 2147483647LL, "spmm_forward_blocked_zt: grid too large");
    const int chunk = (int)std::min<int64_t>(std::min<int64_t>(n_sub, zt_floats / per_angle), 65535);
    cudaStream_t st = (cudaStream_t)stream;
    for (int s0 = 0; s0 < n_sub; s0 += chunk) {
        const int na = std::min(chunk, n_sub - s0);
        dim3 tg((unsigned)cdiv(kb, ZT_TR), (unsigned)(ly / ZT_TR), (unsigned)na);
        zt_transpose_kernel<<<tg, 256, 0, st>>>(sino + (int64_t)s0 * my * kstride, zt, my, ly, kstride, kb);
        int rc = launch_status("spmm_pf_forward_blocked_zt: transpose");
        if (rc) return rc;
        const int32_t *om = omegas ? omegas + s0 : nullptr;
        switch (mt) {
#define DFX_ZT_CASE(M)                                                                                                 \
    case M:                                                                                                            \
        rc = launch_zt<M>(zt, fb_ptr, fb_k, fb_v, fb_mask, data, om, s0, na, my, ly, nyb, P, C, ncb, nb, kb, st);       \
        break;
            DFX_ZT_CASE(1)
            DFX_ZT_CASE(2)
            DFX_ZT_CASE(3)
            DFX_ZT_CASE(4)
            DFX_ZT_CASE(5)
            DFX_ZT_CASE(6)
            DFX_ZT_CASE(7)
            DFX_ZT_CASE(8)
            DFX_ZT_CASE(9)
#undef DFX_ZT_CASE
        default:
            set_error("spmm_forward_blocked_zt: %d line groups per warp", mt);
            return DFX_EINVAL;
        }
        if (rc) return rc;
    }
    return DFX_OK;
}

extern "C" int64_t dfx_spmm_pf_adjoint_zt_floats(int n_angles, int my, int cp)
{
    if (n_angles <= 0 || my <= 0 || cp <= 0) return -1;
    return (int64_t)n_angles * cp * (cdiv(my, 32) * 32);
}

template <int MT>
static int launch_az(const float *dt, const int32_t *row_ptr, const uint16_t *col_j, const float *val, float *sino,
                     const int32_t *omegas, int r0, int na, int my, int ly, int nyb, int kb, int cp, int kstride,
                     float alpha, int compact, cudaStream_t st)
{
    const cudaError_t err = allow_max_dynamic_smem(spmm_adjoint_zt_kernel<MT>);
    if (err != cudaSuccess) {
        set_error("spmm_adjoint_zt: shared memory attribute: %s", cudaGetErrorString(err));
        return DFX_ELAUNCH;
    }
    // orientation rows per warp: the most (of 4, 2, 1) that still gives the launch about four waves of blocks (three
    // blocks of 8 warps per SM)
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int kw = AZ_KW;
    while (kw > 1 && cdiv(kstride, AZ_WARPS * kw) * nyb * na < 4LL * 3 * nsm) kw >>= 1;
    const size_t smem = (size_t)32 * MT * (AZ_WARPS * kw + 1) * sizeof(float);
    dim3 grid((unsigned)cdiv(kstride, AZ_WARPS * kw), (unsigned)nyb, (unsigned)na);
    spmm_adjoint_zt_kernel<MT><<<grid, 32 * AZ_WARPS, smem, st>>>(dt, row_ptr, col_j, val, sino, omegas, r0, my, ly,
                                                                  kb, cp, kstride, alpha, compact, kw);
    return launch_status("spmm_pf_adjoint_zt");
}

extern "C" int dfx_spmm_pf_adjoint_zt(const float *data, float *dt, int64_t dt_floats, const int32_t *row_ptr,
                                      const uint16_t *col_j, const float *val, float *sino, const int32_t *omegas,
                                      int n_sub, int my, int kb, int cp, int kstride, float alpha, int compact,
                                      int max_groups, void *stream)
{
    DFX_REQUIRE(data && dt && row_ptr && col_j && val && sino, "spmm_adjoint_zt: null pointer");
    DFX_REQUIRE(n_sub > 0 && my > 0 && cp > 0 && kb > 0 && kb <= kstride, "spmm_adjoint_zt: bad sizes");
    DFX_REQUIRE(cp <= 65536, "spmm_adjoint_zt: more than 65536 segments per data row");
    DFX_REQUIRE(max_groups >= 0 && max_groups <= ZT_G, "spmm_adjoint_zt: max_groups outside 0 .. 9");
    const int64_t per_angle = dfx_spmm_pf_adjoint_zt_floats(1, my, cp);
    DFX_REQUIRE(dt_floats >= per_angle, "spmm_adjoint_zt: the transpose buffer holds less than one angle");
    const int ly = (int)(cdiv(my, 32) * 32), ngroups = ly / 32;
    const int gmax = max_groups ? max_groups : ZT_G;
    const int nyb = (int)cdiv(ngroups, gmax), mt = (int)cdiv(ngroups, nyb);
    DFX_REQUIRE(nyb <= 65535 && cdiv(kstride, AZ_WARPS) <= 2147483647LL, "spmm_adjoint_zt: grid too large");
    const int chunk = (int)std::min<int64_t>(std::min<int64_t>(n_sub, dt_floats / per_angle), 65535);
    cudaStream_t st = (cudaStream_t)stream;
    for (int s0 = 0; s0 < n_sub; s0 += chunk) {
        const int na = std::min(chunk, n_sub - s0);
        const int32_t *om = omegas ? omegas + s0 : nullptr;
        dim3 tg((unsigned)cdiv(cp, ZT_TR), (unsigned)(ly / ZT_TR), (unsigned)na);
        dt_transpose_kernel<<<tg, 256, 0, st>>>(data, dt, om, s0, my, ly, cp);
        int rc = launch_status("spmm_pf_adjoint_zt: transpose");
        if (rc) return rc;
        // compact rows are numbered by the position in the subset: the chunk's rows start at s0 * kb
        const int32_t *rp = compact ? row_ptr + (int64_t)s0 * kb : row_ptr;
        float *out = sino + (int64_t)s0 * my * kstride;
        switch (mt) {
#define DFX_AZ_CASE(M)                                                                                                 \
    case M:                                                                                                            \
        rc = launch_az<M>(dt, rp, col_j, val, out, om, s0, na, my, ly, nyb, kb, cp, kstride, alpha, compact, st);      \
        break;
            DFX_AZ_CASE(1)
            DFX_AZ_CASE(2)
            DFX_AZ_CASE(3)
            DFX_AZ_CASE(4)
            DFX_AZ_CASE(5)
            DFX_AZ_CASE(6)
            DFX_AZ_CASE(7)
            DFX_AZ_CASE(8)
            DFX_AZ_CASE(9)
#undef DFX_AZ_CASE
        default:
            set_error("spmm_adjoint_zt: %d line groups per warp", mt);
            return DFX_EINVAL;
        }
        if (rc) return rc;
    }
    return DFX_OK;
}
