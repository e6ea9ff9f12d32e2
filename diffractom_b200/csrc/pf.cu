// Pole-figure (PF) matrix of the single-phase operator on sm_100a: entry evaluation and CSR construction (the sparse
// products with the channel-fastest sinogram batch are in spmm.cu).
//
// CSR construction: one warp per CSR row. The lanes evaluate the row's 32 next entries in column order, a ballot
// orders the non-zeros, so every row is written in ascending column order and the structure is a pure function of
// the float32 entry values: the CSR of the dense batch, bit for bit, with no sort and no atomics. Adjoint rows
// (angle, orientation) run over the segments j = c * P + p; forward rows (angle, segment) over the orientations.

#include <cuda_bf16.h>

#include "dfx_common.cuh"

namespace dfx {

__device__ __forceinline__ float pf_entry(const dfx_pf_geometry &g, int r, int kg, int c, int p)
{
    const int a0 = __ldg(g.axis_start + p), a1 = __ldg(g.axis_start + p + 1);
    const float *pole = g.poles + (int64_t)kg * g.A * 3;
    const float inv = __ldg(g.inv_sigma2 + kg);
    float w_total = 0.0f;
    const bool axis_theta = g.axis_w != nullptr;
    const bool wp = g.wp_ax != nullptr;
    int wp_last = -1;                                  // window_parallax: the fraction depends on the axis only here
    float wp_fr = 1.0f;
    for (int s = 0; s < g.S; ++s)
        for (int se = 0; se < g.S_eta; ++se) {
            const float *v = axis_theta
                                 ? g.coords + (((int64_t)(r * g.S + s) * g.C + c) * g.S_eta + se) * 3
                                 : g.coords + ((((int64_t)(r * g.S + s) * g.C + c) * g.S_eta + se) * g.P + p) * 3;
            const float vx = __ldg(v), vy = __ldg(v + 1), vz = __ldg(v + 2);
            float wx = 0.0f, wy = 0.0f, wz = 0.0f;
            if (axis_theta) {
                const float *wv = g.axis_w + (int64_t)(r * g.S + s) * 3;
                wx = __ldg(wv);
                wy = __ldg(wv + 1);
                wz = __ldg(wv + 2);
            }
            float w_node = 0.0f;
            for (int a = a0; a < a1; ++a) {
                const float nx = __ldg(pole + 3 * a), ny = __ldg(pole + 3 * a + 1), nz = __ldg(pole + 3 * a + 2);
                const float du = __fmaf_rn(nz, vz, __fmaf_rn(ny, vy, __fmul_rn(nx, vx)));
                // reflection_two_theta: n . v = cos(theta_a) (n . u) - sin(theta_a) (n . w)
                const float d = axis_theta
                                    ? fabsf(__fsub_rn(__fmul_rn(__ldg(g.axis_cos + a), du),
                                                      __fmul_rn(__ldg(g.axis_sin + a),
                                                                __fmaf_rn(nz, wz, __fmaf_rn(ny, wy, __fmul_rn(nx, wx))))))
                                    : fabsf(du);
                float t = 0.0f;
                const float e1 = __fmul_rn(__fsub_rn(1.0f, d), inv);
                if (e1 < g.cut) t = __fadd_rn(t, expf(-e1));
                const float e2 = __fmul_rn(__fadd_rn(1.0f, d), inv);
                if (e2 < g.cut) t = __fadd_rn(t, expf(-e2));
                if (wp && t > 0.0f) {
                    if (a != wp_last) {
                        wp_fr = wp_fraction(g, r, kg, p, a);
                        wp_last = a;
                    }
                    t = __fmul_rn(t, wp_fr);
                }
                w_node = __fmaf_rn(__ldg(g.axis_count + a), t, w_node);
            }
            if (g.quad_w) w_total = __fmaf_rn(__ldg(g.quad_w + s * g.S_eta + se), w_node, w_total);
            else w_total = __fadd_rn(w_total, w_node);
        }
    const float norm = __ldg(g.norm + kg);
    float val = g.quad_w ? __fmul_rn(w_total, norm) : __fmul_rn(__fdiv_rn(w_total, (float)(g.S * g.S_eta)), norm);
    if (g.intens) val = __fmul_rn(val, __ldg(g.intens + p));
    return val;
}

__global__ void pf_dense_kernel(dfx_pf_geometry g, int k0, int kb, float *__restrict__ out)
{
    const int64_t total = (int64_t)g.R * kb * g.C * g.P;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int p = (int)(i % g.P);
        int64_t t = i / g.P;
        const int c = (int)(t % g.C);
        t /= g.C;
        const int k = (int)(t % kb);
        const int r = (int)(t / kb);
        out[i] = pf_entry(g, r, k0 + k, c, p);
    }
}

// Dense BF16 batch: rows koff .. koff+kb-1 of (n_rows, ktot, cp_pad), the float32 entry rounded to nearest-even;
// angle plane s holds angle rows[s] (rows NULL: all R angles, plane r = angle r).
__global__ void pf_dense_bf16_kernel(dfx_pf_geometry g, const int32_t *__restrict__ rows, int n_rows, int k0, int kb,
                                     int64_t koff, int64_t ktot, int cp_pad, __nv_bfloat16 *__restrict__ out)
{
    const int CP = g.C * g.P;
    const int64_t total = (int64_t)n_rows * kb * CP;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(i % CP);
        const int64_t t = i / CP;
        const int k = (int)(t % kb);
        const int s = (int)(t / kb);
        const int r = rows ? __ldg(rows + s) : s;
        out[((int64_t)s * ktot + koff + k) * cp_pad + j] = __float2bfloat16_rn(pf_entry(g, r, k0 + k, j / g.P, j % g.P));
    }
}

// One warp per CSR row: FILL = 0 counts the row's non-zeros, FILL = 1 writes them in column order.
template <int FWD, int FILL>
__global__ void __launch_bounds__(256) pf_csr_kernel(dfx_pf_geometry g, const int32_t *__restrict__ rows, int n_rows,
                                                     int k0, int kb, int32_t *__restrict__ counts,
                                                     const int32_t *__restrict__ row_ptr, uint16_t *__restrict__ col,
                                                     float *__restrict__ val)
{
    const int lane = threadIdx.x & 31;
    const int CP = g.C * g.P;
    const int64_t n_csr = (int64_t)n_rows * (FWD ? CP : kb);
    const int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= n_csr) return;
    const int s = (int)(row / (FWD ? CP : kb));
    const int q = (int)(row % (FWD ? CP : kb));        // orientation (adjoint rows) or segment (forward rows)
    const int r = rows ? __ldg(rows + s) : s;
    const int n_cols = FWD ? kb : CP;
    int pos = FILL ? __ldg(row_ptr + row) : 0;
    const int end = FILL ? __ldg(row_ptr + row + 1) : 0;   // writes stay inside the row whatever happens
    int n = 0;
    for (int base = 0; base < n_cols; base += 32) {
        const int col_i = base + lane;
        float v = 0.0f;
        if (col_i < n_cols) {
            if (FWD) v = pf_entry(g, r, k0 + col_i, q / g.P, q % g.P);
            else v = pf_entry(g, r, k0 + q, col_i / g.P, col_i % g.P);
        }
        const unsigned m = __ballot_sync(0xffffffffu, v != 0.0f);
        if (FILL && v != 0.0f) {
            const int o = pos + __popc(m & ((1u << lane) - 1u));
            if (o < end) {
                col[o] = (uint16_t)col_i;
                val[o] = v;
            }
        }
        pos += __popc(m);
        n += __popc(m);
    }
    if (!FILL && lane == 0) counts[row] = n;
}

// ---- exclusive scan of int32 (three passes: tile sums, scan of the tile sums, tile scans) ----
constexpr int SCAN_THREADS = 256, SCAN_PER = 8, SCAN_TILE = SCAN_THREADS * SCAN_PER;

__device__ __forceinline__ int block_exclusive(int x, int *sh, int *total)
{
    // exclusive scan over the block of one value per thread
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) sh[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int w = lane < (SCAN_THREADS >> 5) ? sh[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < (SCAN_THREADS >> 5)) sh[lane] = wi - w;
        if (lane == (SCAN_THREADS >> 5) - 1) *total = wi;
    }
    __syncthreads();
    const int r = sh[wid] + inc - x;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_tile_sums(const int32_t *__restrict__ in, int64_t n,
                                                              int32_t *__restrict__ sums)
{
    __shared__ int sh[32];
    __shared__ int tot;
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_PER;
    int s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_PER; ++i) s += (base + i < n) ? in[base + i] : 0;
    block_exclusive(s, sh, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_sums(int32_t *__restrict__ sums, int64_t n_tiles,
                                                         int32_t *__restrict__ out_total)
{
    __shared__ int sh[32];
    __shared__ int tot;
    int carry = 0;
    for (int64_t b = 0; b < n_tiles; b += SCAN_THREADS) {
        const int64_t i = b + threadIdx.x;
        const int x = i < n_tiles ? sums[i] : 0;
        const int e = block_exclusive(x, sh, &tot);
        if (i < n_tiles) sums[i] = carry + e;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *out_total = carry;
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_tiles(const int32_t *in, int64_t n,
                                                          const int32_t *__restrict__ sums, int32_t *out)
{
    __shared__ int sh[32];
    __shared__ int tot;
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_PER;
    int v[SCAN_PER];
    int s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_PER; ++i) {
        v[i] = (base + i < n) ? in[base + i] : 0;
        s += v[i];
    }
    int e = block_exclusive(s, sh, &tot) + sums[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SCAN_PER; ++i) {
        if (base + i < n) out[base + i] = e;
        e += v[i];
    }
}

__global__ void zero_rows_kernel(float *__restrict__ data, const int32_t *__restrict__ omegas, int n_sub,
                                 int64_t row_len)
{
    const int64_t n = (int64_t)n_sub * row_len;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = i / row_len;
        data[(int64_t)__ldg(omegas + s) * row_len + (i - s * row_len)] = 0.0f;
    }
}

static int check_geometry(const dfx_pf_geometry *g)
{
    DFX_REQUIRE(g && g->coords && g->poles && g->axis_start && g->axis_count && g->inv_sigma2 && g->norm,
                "pf: geometry has null pointers");
    DFX_REQUIRE(g->R > 0 && g->C > 0 && g->P > 0 && g->A > 0 && g->S > 0 && g->S_eta > 0 && g->K > 0,
                "pf: bad geometry sizes");
    DFX_REQUIRE((g->axis_w == nullptr) == (g->axis_sin == nullptr) && (g->axis_w == nullptr) == (g->axis_cos == nullptr),
                "pf: reflection_two_theta needs axis_w, axis_sin and axis_cos together");
    DFX_REQUIRE(!g->wp_ax || (g->wp_pos && g->wp_cov && g->wp_b && g->wp_ch), "pf: incomplete window_parallax arrays");
    return DFX_OK;
}

static unsigned grid_for(int64_t n, int threads)
{
    const int64_t b = cdiv(n, threads);
    return (unsigned)(b < 148 * 64 ? (b > 0 ? b : 1) : 148 * 64);
}

}  // namespace dfx

using namespace dfx;

extern "C" int dfx_pf_dense(const dfx_pf_geometry *g, int k0, int kb, float *out, void *stream)
{
    int st = check_geometry(g);
    if (st) return st;
    DFX_REQUIRE(out && k0 >= 0 && kb > 0 && k0 + kb <= g->K, "pf_dense: bad batch");
    const int64_t n = (int64_t)g->R * kb * g->C * g->P;
    pf_dense_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(*g, k0, kb, out);
    return launch_status("pf_dense");
}

extern "C" int dfx_pf_dense_bf16(const dfx_pf_geometry *g, int k0, int kb, int64_t koff, int64_t ktot, int cp_pad,
                                 void *out, void *stream)
{
    int st = check_geometry(g);
    if (st) return st;
    DFX_REQUIRE(out && k0 >= 0 && kb > 0 && k0 + kb <= g->K, "pf_dense_bf16: bad batch");
    DFX_REQUIRE(koff >= 0 && koff + kb <= ktot && cp_pad >= g->C * g->P, "pf_dense_bf16: batch rows %lld + %d outside "
                "ktot %lld, or cp_pad %d < CP", (long long)koff, kb, (long long)ktot, cp_pad);
    const int64_t n = (int64_t)g->R * kb * g->C * g->P;
    pf_dense_bf16_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
        *g, nullptr, g->R, k0, kb, koff, ktot, cp_pad, reinterpret_cast<__nv_bfloat16 *>(out));
    return launch_status("pf_dense_bf16");
}

extern "C" int dfx_pf_dense_bf16_rows(const dfx_pf_geometry *g, const int32_t *rows, int n_rows, int k0, int kb,
                                      int64_t koff, int64_t ktot, int cp_pad, void *out, void *stream)
{
    int st = check_geometry(g);
    if (st) return st;
    DFX_REQUIRE(out && rows && n_rows > 0 && k0 >= 0 && kb > 0 && k0 + kb <= g->K, "pf_dense_bf16_rows: bad batch");
    DFX_REQUIRE(koff >= 0 && koff + kb <= ktot && cp_pad >= g->C * g->P, "pf_dense_bf16_rows: batch rows %lld + %d "
                "outside ktot %lld, or cp_pad %d < CP", (long long)koff, kb, (long long)ktot, cp_pad);
    const int64_t n = (int64_t)n_rows * kb * g->C * g->P;
    pf_dense_bf16_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
        *g, rows, n_rows, k0, kb, koff, ktot, cp_pad, reinterpret_cast<__nv_bfloat16 *>(out));
    return launch_status("pf_dense_bf16_rows");
}

static int pf_csr(const dfx_pf_geometry *g, const int32_t *rows, int n_rows, int k0, int kb, int fwd, int fill,
                  int32_t *counts, const int32_t *row_ptr, uint16_t *col, float *val, void *stream)
{
    int st = check_geometry(g);
    if (st) return st;
    DFX_REQUIRE(n_rows > 0 && k0 >= 0 && kb > 0 && k0 + kb <= g->K, "pf_csr: bad batch (rows %d, k0 %d, kb %d, K %d)",
                n_rows, k0, kb, g->K);
    DFX_REQUIRE(kb <= 65536 && (int64_t)g->C * g->P <= 65536, "pf_csr: columns exceed the 16-bit index range");
    DFX_REQUIRE(fill ? (row_ptr && col && val) : (counts != nullptr), "pf_csr: null output");
    const int64_t n_csr = (int64_t)n_rows * (fwd ? (int64_t)g->C * g->P : kb);
    const int warps = 8;
    const int64_t blocks = cdiv(n_csr, warps);
    DFX_REQUIRE(blocks < 2147483647, "pf_csr: too many rows");
    cudaStream_t s = (cudaStream_t)stream;
    if (fwd && fill)
        pf_csr_kernel<1, 1><<<(unsigned)blocks, 32 * warps, 0, s>>>(*g, rows, n_rows, k0, kb, counts, row_ptr, col, val);
    else if (fwd)
        pf_csr_kernel<1, 0><<<(unsigned)blocks, 32 * warps, 0, s>>>(*g, rows, n_rows, k0, kb, counts, row_ptr, col, val);
    else if (fill)
        pf_csr_kernel<0, 1><<<(unsigned)blocks, 32 * warps, 0, s>>>(*g, rows, n_rows, k0, kb, counts, row_ptr, col, val);
    else
        pf_csr_kernel<0, 0><<<(unsigned)blocks, 32 * warps, 0, s>>>(*g, rows, n_rows, k0, kb, counts, row_ptr, col, val);
    return launch_status(fill ? "pf_csr_fill" : "pf_csr_count");
}

extern "C" int dfx_pf_csr_count(const dfx_pf_geometry *g, const int32_t *rows, int n_rows, int k0, int kb,
                                int forward_rows, int32_t *counts, void *stream)
{
    return pf_csr(g, rows, n_rows, k0, kb, forward_rows ? 1 : 0, 0, counts, nullptr, nullptr, nullptr, stream);
}

extern "C" int dfx_pf_csr_fill(const dfx_pf_geometry *g, const int32_t *rows, int n_rows, int k0, int kb,
                               int forward_rows, const int32_t *row_ptr, uint16_t *col, float *val, void *stream)
{
    return pf_csr(g, rows, n_rows, k0, kb, forward_rows ? 1 : 0, 1, nullptr, row_ptr, col, val, stream);
}

extern "C" size_t dfx_scan_scratch_bytes(int64_t n)
{
    return (size_t)(cdiv(n > 0 ? n : 1, SCAN_TILE) + 1) * sizeof(int32_t);
}

extern "C" int dfx_scan_exclusive_i32(const int32_t *in, int32_t *out, int64_t n, void *scratch,
                                      size_t scratch_bytes, void *stream)
{
    DFX_REQUIRE(in && out && scratch && n >= 0, "scan: bad arguments");
    if (scratch_bytes < dfx_scan_scratch_bytes(n)) {
        set_error("scan: scratch of %zu bytes, %zu needed", scratch_bytes, dfx_scan_scratch_bytes(n));
        return DFX_ENOMEM;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t tiles = cdiv(n > 0 ? n : 1, SCAN_TILE);
    DFX_REQUIRE(tiles < 2147483647, "scan: too long");
    int32_t *sums = (int32_t *)scratch;
    scan_tile_sums<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(in, n, sums);
    int st = launch_status("scan_tile_sums");
    if (st) return st;
    scan_sums<<<1, SCAN_THREADS, 0, s>>>(sums, tiles, out + n);
    st = launch_status("scan_sums");
    if (st) return st;
    if (n == 0) return DFX_OK;
    scan_tiles<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(in, n, sums, out);
    return launch_status("scan_tiles");
}

// ---- the exclusive scan without caller scratch ----
// Its tile sums live in this array, which the CUDA runtime places in the memory of every device that loads this
// library and keeps there until the process exits. Host code only knows a stand-in for its name: the device address
// comes from cudaGetSymbolAddress, looked up on every call with the caller's device current. No address is cached,
// so a context that was destroyed and made again (cudaDeviceReset, another driver context) never sees a stale one.
static __device__ __align__(256) int32_t g_scan_tile_sums[DFX_SCAN_STATIC_MAX_N / SCAN_TILE + 1];

extern "C" int dfx_scan_exclusive_i32_static(const int32_t *in, int32_t *out, int64_t n, void *stream)
{
    static_assert(DFX_SCAN_STATIC_MAX_N % SCAN_TILE == 0, "the maximum is a whole number of tiles");
    DFX_REQUIRE(in && out, "scan_static: null pointer");
    DFX_REQUIRE(n >= 0 && n <= DFX_SCAN_STATIC_MAX_N,
                "scan_static: n = %lld is beyond the %lld elements its built-in scratch covers; use "
                "dfx_scan_exclusive_i32 with scratch of dfx_scan_scratch_bytes(n) bytes", (long long)n,
                (long long)DFX_SCAN_STATIC_MAX_N);
    // the array's address in the current context (the first lookup on a device may load this library's module
    // there; the later ones only read a table)
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scan_tile_sums);
    if (e != cudaSuccess) {
        set_error("scan_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        return DFX_ECUDA;
    }
    int32_t *sums = static_cast<int32_t *>(p);
    // every slot the later passes read is written by the first pass of this call: nothing to clear
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t tiles = cdiv(n > 0 ? n : 1, SCAN_TILE);
    scan_tile_sums<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(in, n, sums);
    int st = launch_status("scan_static_tile_sums");
    if (st) return st;
    scan_sums<<<1, SCAN_THREADS, 0, s>>>(sums, tiles, out + n);
    st = launch_status("scan_static_sums");
    if (st) return st;
    if (n == 0) return DFX_OK;
    scan_tiles<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(in, n, sums, out);
    return launch_status("scan_static_tiles");
}

extern "C" int dfx_zero_rows(float *data, const int32_t *omegas, int n_sub, int64_t row_len, void *stream)
{
    DFX_REQUIRE(data && omegas && n_sub >= 0 && row_len > 0, "zero_rows: bad arguments");
    if (n_sub == 0) return DFX_OK;
    zero_rows_kernel<<<grid_for((int64_t)n_sub * row_len, 256), 256, 0, (cudaStream_t)stream>>>(data, omegas, n_sub,
                                                                                                 row_len);
    return launch_status("zero_rows");
}
