// Sparse PF products (FP32), sm_100a.
//
// Both products are "CSR rows x dense lines": output row q (a segment j of the forward product, an orientation k of
// the adjoint) of one rotation angle is the sum over the row's entries (c, v) of v * X[y, c], for SP_TY detector
// lines y at once. A block owns one angle, SP_TY lines and SP_ROWS rows (one per thread). It stages X[y0 .. y0+TY,
// a chunk of columns] in shared memory transposed (the TY values of one column contiguous, read as float4); every
// thread walks its row's entries in groups of four, loading the next group while it applies the current one, and
// uses each entry TY times from a register. Rows are sorted by column, so a thread keeps its place from one chunk to
// the next. No atomics: every output is written by one thread.
#include "dfx_common.cuh"

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
        float *dl = data + ((int64_t)r * my + y0) * cp + j;
#pragma unroll
        for (int t = 0; t < SP_TY; ++t)
            if (t < ny) dl[(int64_t)t * cp] += acc[t];
    }
}

// adjoint: sino[s, y, k] = alpha sum_j PF[k, j] data[r, y, j]   (rows k over the adjoint CSR)
__global__ void __launch_bounds__(SP_ROWS) spmm_adjoint_kernel(
    const float *__restrict__ data, const int32_t *__restrict__ row_ptr, const uint16_t *__restrict__ col_j,
    const float *__restrict__ val, float *__restrict__ sino, const int32_t *__restrict__ omegas, int my, int kb,
    int cp, int kstride, float alpha, int compact)
{
    __shared__ __align__(16) float tile[SP_CHUNK * SP_TYP];
    const int k = blockIdx.x * SP_ROWS + threadIdx.x;
    const int y0 = blockIdx.y * SP_TY;
    const int s = blockIdx.z;
    const int r = omegas ? __ldg(omegas + s) : s;
    const int ny = min(SP_TY, my - y0);
    int i = 0, e = 0;
    if (k < kb) {
        const int64_t rr = (int64_t)(compact ? s : r) * kb + k;
        i = __ldg(row_ptr + rr);
        e = __ldg(row_ptr + rr + 1);
    }
    Group g;
    load_group(g, col_j, val, i, e);
    float acc[SP_TY];
#pragma unroll
    for (int t = 0; t < SP_TY; ++t) acc[t] = 0.0f;
    for (int c0 = 0; c0 < cp; c0 += SP_CHUNK) {
        const int cn = min(SP_CHUNK, cp - c0);
        if (c0) __syncthreads();
        stage(tile, data, (int64_t)r * my + y0, cp, ny, c0, cn);
        __syncthreads();
        i = walk_row(acc, tile, col_j, val, i, e, g, c0, c0 + cn);
    }
    if (k < kstride) {
        float *zl = sino + ((int64_t)s * my + y0) * kstride + k;
#pragma unroll
        for (int t = 0; t < SP_TY; ++t)
            if (t < ny) zl[(int64_t)t * kstride] = k < kb ? alpha * acc[t] : 0.0f;
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
    dim3 grid((unsigned)cdiv(kstride, SP_ROWS), (unsigned)cdiv(my, SP_TY), (unsigned)n_sub);
    spmm_adjoint_kernel<<<grid, SP_ROWS, 0, (cudaStream_t)stream>>>(data, row_ptr, col_j, val, sino, omegas, my, kb,
                                                                    cp, kstride, alpha, compact);
    return launch_status("spmm_pf_adjoint");
}
