// Fourier-slice parallel-beam projector (diffractom's FourierRadon: operators/fourier_radon.py, fourier_radon.cl) on
// sm_100a: the kernels around cuFFT.
//
// Forward, per slice of C channels of a channel-fastest batch (npix, kstride):
//   pad       image / deapodisation -> oversampled grid (C, My, Mx), pixel (x, y) at ((x - cx) mod Mx, (y - cy) mod My)
//   cuFFT     real-to-complex 2-D: G (C, My, Mx/2+1)
//   slices    per polar sample (angle a, frequency j): W x W taps of G (Hermitian mirror beyond the half) times the
//             phase / bin response: spec (C, R*H)
//   cuFFT     complex-to-real 1-D of length L per (channel, angle): lines (C, R, L)
//   lines_out sino[a, s, k] = scale * lines[k, a, s]  (32 x 32 tiles through shared memory: both sides coalesced)
// Backward (the transpose, angle weights): lines_in, cuFFT real-to-complex 1-D, unfilter (conjugate response),
// spread (the transposed interpolation as a gather: a block owns a 16 x 16 tile of the half grid and walks the
// samples with a tap on it, deterministic), cuFFT complex-to-real 2-D, crop.
// Scratch (grid, G, spec, lines, cuFFT work area) is the caller's; cuFFT plans are made once per size and kept.
#include <cufft.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

#include "dfx_common.cuh"

namespace dfx {
namespace {

constexpr int FR_TS = 16;     // spreading tile (cells per side)
constexpr int FR_SB = 64;     // samples staged per round of the spread
constexpr int FR_CCS = 16;    // channels per spreading block

__device__ __forceinline__ int wrap(int v, int m)
{
    int r = v % m;
    return r < 0 ? r + m : r;
}

// image slice (channel-fastest, channels c0 .. c0+cb-1 of img_k) -> grid (C, My, Mx); a block: 32 grid columns x 32
// channels of one grid row
__global__ void __launch_bounds__(256) fr_pad_kernel(const float *__restrict__ img, int kstride, int c0, int cb,
                                                     float *__restrict__ grid, const float *__restrict__ inv_dx,
                                                     const float *__restrict__ inv_dy, int Nx, int Ny, int Mx, int My,
                                                     int cx, int cy, int C)
{
    __shared__ float t[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int gy = blockIdx.y, gx0 = blockIdx.x * 32, cc0 = blockIdx.z * 32;
    const int y = (gy < My / 2 ? gy : gy - My) + cy;
    const bool yin = y >= 0 && y < Ny;
    for (int r = ty; r < 32; r += 8) {
        const int gx = gx0 + r, c = cc0 + tx;
        const int x = (gx < Mx / 2 ? gx : gx - Mx) + cx;
        float v = 0.0f;
        if (yin && gx < Mx && x >= 0 && x < Nx && c < cb)
            v = __fmul_rn(__fmul_rn(__ldg(img + ((int64_t)y * Nx + x) * kstride + c0 + c), __ldg(inv_dx + x)),
                          __ldg(inv_dy + y));
        t[r][tx] = v;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int c = cc0 + r, gx = gx0 + tx;
        if (c < C && gx < Mx) grid[((int64_t)c * My + gy) * Mx + gx] = t[tx][r];
    }
}

// polar samples: spec[c, smp] = filt[smp] * sum_{l, i} w2[l] w1[i] G[k2b + l, k1b + i]; imaginary parts of the
// frequencies 0 and L/2 (real for a real line) set to 0
template <int W>
__global__ void __launch_bounds__(128) fr_slices_kernel(const float2 *__restrict__ G, const int2 *__restrict__ kb,
                                                        const float *__restrict__ w1s, const float *__restrict__ w2s,
                                                        const float2 *__restrict__ filt, float2 *__restrict__ spec,
                                                        int Mx, int My, int RH, int H)
{
    const int smp = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
    if (smp >= RH) return;
    const int Hx = Mx / 2 + 1;
    const float2 *Gc = G + (int64_t)c * My * Hx;
    const int2 b = __ldg(kb + smp);
    float w1[W], w2[W];
    int col[W], row_d[W], row_m[W];
    bool cj[W];
#pragma unroll
    for (int i = 0; i < W; ++i) {
        w1[i] = __ldg(w1s + (int64_t)smp * W + i);
        w2[i] = __ldg(w2s + (int64_t)smp * W + i);
        const int k1 = wrap(b.x + i, Mx);
        cj[i] = k1 > Mx / 2;
        col[i] = cj[i] ? Mx - k1 : k1;
        const int k2 = wrap(b.y + i, My);
        row_d[i] = k2;
        row_m[i] = k2 == 0 ? 0 : My - k2;
    }
    float ar = 0.0f, ai = 0.0f;
#pragma unroll
    for (int l = 0; l < W; ++l) {
#pragma unroll
        for (int i = 0; i < W; ++i) {
            const float w = __fmul_rn(w2[l], w1[i]);
            const float2 g = __ldg(Gc + (int64_t)(cj[i] ? row_m[l] : row_d[l]) * Hx + col[i]);
            ar = __fmaf_rn(w, g.x, ar);
            ai = __fmaf_rn(w, cj[i] ? -g.y : g.y, ai);
        }
    }
    const float2 f = __ldg(filt + smp);
    float2 out = make_float2(__fsub_rn(__fmul_rn(ar, f.x), __fmul_rn(ai, f.y)),
                             __fadd_rn(__fmul_rn(ar, f.y), __fmul_rn(ai, f.x)));
    const int j = smp % H;
    if (j == 0 || j == H - 1) out.y = 0.0f;
    spec[(int64_t)c * RH + smp] = out;
}

// lines (C, R, L) -> sino (R, Ns, kstride) channels c0 .. c0+cb-1, times scale; a block: 32 bins x 32 channels of
// one angle
__global__ void __launch_bounds__(256) fr_lines_out_kernel(const float *__restrict__ lines, float *__restrict__ sino,
                                                           int R, int Ns, int L, int kstride, int c0, int cb,
                                                           float scale)
{
    __shared__ float t[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int s0 = blockIdx.x * 32, cc0 = blockIdx.y * 32, a = blockIdx.z;
    for (int r = ty; r < 32; r += 8) {
        const int c = cc0 + r, s = s0 + tx;
        t[r][tx] = (c < cb && s < Ns) ? lines[((int64_t)c * R + a) * L + s] : 0.0f;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int s = s0 + r, c = cc0 + tx;
        if (s < Ns && c < cb) sino[((int64_t)a * Ns + s) * kstride + c0 + c] = __fmul_rn(scale, t[tx][r]);
    }
}

// sino channels c0 .. c0+cb-1 -> weighted lines (C, R, L), zero past Ns and for c >= cb
__global__ void __launch_bounds__(256) fr_lines_in_kernel(const float *__restrict__ sino, float *__restrict__ lines,
                                                          const float *__restrict__ wa, int R, int Ns, int L,
                                                          int kstride, int c0, int cb, int C)
{
    __shared__ float t[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int s0 = blockIdx.x * 32, cc0 = blockIdx.y * 32, a = blockIdx.z;
    const float w = __ldg(wa + a);
    for (int r = ty; r < 32; r += 8) {
        const int s = s0 + r, c = cc0 + tx;
        t[r][tx] = (s < Ns && c < cb) ? __fmul_rn(w, sino[((int64_t)a * Ns + s) * kstride + c0 + c]) : 0.0f;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int c = cc0 + r, s = s0 + tx;
        if (c < C && s < L) lines[((int64_t)c * R + a) * L + s] = t[tx][r];
    }
}

__global__ void fr_unfilter_kernel(float2 *__restrict__ spec, const float2 *__restrict__ filt, int RH, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 f = __ldg(filt + i % RH), v = spec[i];
        spec[i] = make_float2(__fadd_rn(__fmul_rn(v.x, f.x), __fmul_rn(v.y, f.y)),
                              __fsub_rn(__fmul_rn(v.y, f.x), __fmul_rn(v.x, f.y)));
    }
}

// The transposed interpolation as a gather over the half grid. A block owns one piece of a FR_TS x FR_TS tile's
// sample list (rows k2, columns k1 <= Mx/2) and FR_CCS channels; every thread adds, for its cell q, half * w2[l]
// w1[i] * spec (conjugated through the mirror) of each tap of each listed sample that lands on q, in the list's
// order (half = 1/2 for the frequencies 0 and L/2, counted once by the real line). The tap offsets need no division:
// each staged sample carries its first tap reduced modulo the grid (or its mirror's), so d = q - b (or b - q) is one
// conditional wrap away. A tile's first piece writes the spectrum, its later pieces their own partial tiles, which
// fr_spread_finish adds in order: deterministic.
template <int W>
__global__ void __launch_bounds__(FR_TS *FR_TS) fr_spread_kernel(
    const float2 *__restrict__ spec, const int4 *__restrict__ pieces, const int32_t *__restrict__ tile_smp,
    const int2 *__restrict__ kb, const float *__restrict__ w1s, const float *__restrict__ w2s, float2 *__restrict__ Q,
    float2 *__restrict__ part, int Mx, int My, int RH, int H, int n_tx, int C)
{
    __shared__ int lb1[FR_SB], lb2[FR_SB], lmir[FR_SB];
    __shared__ float lw1[FR_SB][W], lw2[FR_SB][W], lhalf[FR_SB];
    __shared__ float2 lv[FR_CCS][FR_SB];
    const int4 pc = __ldg(pieces + blockIdx.x);                   // tile, first entry, end entry, slot
    const int tile = pc.x, cg = blockIdx.y * FR_CCS;
    const int lx = threadIdx.x, ly = threadIdx.y, lid = ly * FR_TS + lx;
    const int Hx = Mx / 2 + 1;
    const int q1 = (tile % n_tx) * FR_TS + lx, q2 = (tile / n_tx) * FR_TS + ly;
    float2 acc[FR_CCS];
#pragma unroll
    for (int c = 0; c < FR_CCS; ++c) acc[c] = make_float2(0.0f, 0.0f);
    for (int b0 = pc.y; b0 < pc.z; b0 += FR_SB) {
        const int nb = min(FR_SB, pc.z - b0);
        __syncthreads();
        if (lid < nb) {
            const int sm = __ldg(tile_smp + b0 + lid);
            const int smp = sm >= 0 ? sm : -sm - 1;
            const bool mir = sm < 0;
            const int2 b = __ldg(kb + smp);
            lmir[lid] = mir;
            lb1[lid] = wrap(mir ? -b.x : b.x, Mx);                // tap offset d = q - b, or b - q through the mirror
            lb2[lid] = wrap(mir ? -b.y : b.y, My);
            const int j = smp % H;
            lhalf[lid] = (j == 0 || j == H - 1) ? 0.5f : 1.0f;
#pragma unroll
            for (int i = 0; i < W; ++i) {
                lw1[lid][i] = __ldg(w1s + (int64_t)smp * W + i);
                lw2[lid][i] = __ldg(w2s + (int64_t)smp * W + i);
            }
        }
        for (int i = lid; i < nb * FR_CCS; i += FR_TS * FR_TS) {
            const int t = i % nb, c = i / nb;                     // consecutive threads: consecutive samples
            const int sm = __ldg(tile_smp + b0 + t);
            lv[c][t] = cg + c < C ? spec[(int64_t)(cg + c) * RH + (sm >= 0 ? sm : -sm - 1)] : make_float2(0.0f, 0.0f);
        }
        __syncthreads();
        if (q1 < Hx && q2 < My) {
            for (int t = 0; t < nb; ++t) {
                const bool mir = lmir[t] != 0;
                int d1 = mir ? lb1[t] - q1 : q1 - lb1[t];
                int d2 = mir ? lb2[t] - q2 : q2 - lb2[t];
                d1 += d1 < 0 ? Mx : 0;
                d2 += d2 < 0 ? My : 0;
                if (d1 < W && d2 < W) {
                    const float w = __fmul_rn(__fmul_rn(lw2[t][d2], lw1[t][d1]), lhalf[t]);
#pragma unroll
                    for (int c = 0; c < FR_CCS; ++c) {
                        acc[c].x = __fmaf_rn(w, lv[c][t].x, acc[c].x);
                        acc[c].y = __fmaf_rn(w, mir ? -lv[c][t].y : lv[c][t].y, acc[c].y);
                    }
                }
            }
        }
    }
    if (q1 < Hx && q2 < My) {
#pragma unroll
        for (int c = 0; c < FR_CCS; ++c) {
            if (cg + c >= C) break;
            if (pc.w < 0)
                Q[((int64_t)(cg + c) * My + q2) * Hx + q1] = acc[c];
            else
                part[((int64_t)pc.w * C + cg + c) * (FR_TS * FR_TS) + lid] = acc[c];
        }
    }
}

// Q += the partial tiles of a tile's later pieces, in their order (one block per tile, thread = cell)
__global__ void __launch_bounds__(FR_TS *FR_TS) fr_spread_finish_kernel(float2 *__restrict__ Q,
                                                                        const float2 *__restrict__ part,
                                                                        const int32_t *__restrict__ tile_xptr, int Mx,
                                                                        int My, int n_tx, int C)
{
    const int tile = blockIdx.x;
    const int s0 = __ldg(tile_xptr + tile), s1 = __ldg(tile_xptr + tile + 1);
    if (s0 == s1) return;
    const int lid = threadIdx.y * FR_TS + threadIdx.x, Hx = Mx / 2 + 1;
    const int q1 = (tile % n_tx) * FR_TS + threadIdx.x, q2 = (tile / n_tx) * FR_TS + threadIdx.y;
    if (q1 >= Hx || q2 >= My) return;
    for (int c = 0; c < C; ++c) {
        float2 *q = Q + ((int64_t)c * My + q2) * Hx + q1;
        float2 v = *q;
        for (int sl = s0; sl < s1; ++sl) {
            const float2 pv = part[((int64_t)sl * C + c) * (FR_TS * FR_TS) + lid];
            v.x = __fadd_rn(v.x, pv.x);
            v.y = __fadd_rn(v.y, pv.y);
        }
        *q = v;
    }
}

// grid (C, My, Mx) -> image slice (channel-fastest, channels c0 .. c0+cb-1 of img_k) / deapodisation; a block: 32
// pixels of one image row x 32 channels
__global__ void __launch_bounds__(256) fr_crop_kernel(const float *__restrict__ grid, float *__restrict__ img,
                                                      int kstride, int c0, int cb, const float *__restrict__ inv_dx,
                                                      const float *__restrict__ inv_dy, int Nx, int Ny, int Mx,
                                                      int My, int cx, int cy)
{
    __shared__ float t[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int y = blockIdx.y, x0 = blockIdx.x * 32, cc0 = blockIdx.z * 32;
    const int gy = wrap(y - cy, My);
    for (int r = ty; r < 32; r += 8) {
        const int c = cc0 + r, x = x0 + tx;
        float v = 0.0f;
        if (c < cb && x < Nx)
            v = __fmul_rn(__fmul_rn(grid[((int64_t)c * My + gy) * Mx + wrap(x - cx, Mx)], __ldg(inv_dx + x)),
                          __ldg(inv_dy + y));
        t[r][tx] = v;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int x = x0 + r, c = cc0 + tx;
        if (x < Nx && c < cb) img[((int64_t)y * Nx + x) * kstride + c0 + c] = t[tx][r];
    }
}

// channels k0 .. kstride-1 of n_lines lines of stride kstride set to 0 (the padding of a batch)
__global__ void fr_zero_channels_kernel(float *__restrict__ a, int64_t n_lines, int kstride, int k0)
{
    const int w = kstride - k0;
    const int64_t n = n_lines * w;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        a[(i / w) * kstride + k0 + i % w] = 0.0f;
}

// ---- cuFFT plans, made once per (device, kind, sizes, batch) and kept; set-stream / work-area / exec of a plan run
// under one lock, so callers on different streams (with their own work areas) may share it
struct Plan {
    cufftHandle h;
    size_t work;
};

std::mutex g_plan_lock;
std::map<std::tuple<int, int, int, int, int>, Plan> g_plans;   // (device, type, n0, n1 (0: 1-D), batch)

int get_plan(int type, int n0, int n1, int batch, Plan *out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        set_error("fourier: cannot query the device");
        return DFX_ECUDA;
    }
    const auto key = std::make_tuple(dev, type, n0, n1, batch);
    auto it = g_plans.find(key);
    if (it != g_plans.end()) {
        *out = it->second;
        return DFX_OK;
    }
    Plan p{};
    if (cufftCreate(&p.h) != CUFFT_SUCCESS) {
        set_error("fourier: cufftCreate failed");
        return DFX_ECUDA;
    }
    cufftSetAutoAllocation(p.h, 0);
    int n[2] = {n0, n1};
    const cufftResult r =
        cufftMakePlanMany(p.h, n1 ? 2 : 1, n, nullptr, 1, 0, nullptr, 1, 0, (cufftType)type, batch, &p.work);
    if (r != CUFFT_SUCCESS) {
        cufftDestroy(p.h);
        set_error("fourier: cufftMakePlanMany (%d x %d, batch %d) failed: %d", n0, n1, batch, (int)r);
        return DFX_ECUDA;
    }
    g_plans[key] = p;
    *out = p;
    return DFX_OK;
}

int run_plan(int type, int n0, int n1, int batch, void *in, void *outp, void *work, size_t work_bytes,
             cudaStream_t s)
{
    std::lock_guard<std::mutex> lk(g_plan_lock);
    Plan p;
    int st = get_plan(type, n0, n1, batch, &p);
    if (st) return st;
    if (p.work > work_bytes) {
        set_error("fourier: cuFFT work area of %zu bytes > the %zu bytes left in the scratch", p.work, work_bytes);
        return DFX_ENOMEM;
    }
    cufftResult r = cufftSetStream(p.h, s);
    if (r == CUFFT_SUCCESS) r = cufftSetWorkArea(p.h, work);
    if (r == CUFFT_SUCCESS) {
        if (type == CUFFT_R2C)
            r = cufftExecR2C(p.h, (cufftReal *)in, (cufftComplex *)outp);
        else
            r = cufftExecC2R(p.h, (cufftComplex *)in, (cufftReal *)outp);
    }
    if (r != CUFFT_SUCCESS) {
        set_error("fourier: cuFFT execution failed: %d", (int)r);
        return DFX_ELAUNCH;
    }
    return DFX_OK;
}

struct Layout {
    size_t grid, G, spec, lines, part, work, total;
};

size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

int layout(const dfx_fr_geometry *g, int C, Layout *L)
{
    const size_t Hx = (size_t)g->Mx / 2 + 1;
    L->grid = 0;
    L->G = L->grid + al256((size_t)C * g->My * g->Mx * 4);
    L->spec = L->G + al256((size_t)C * g->My * Hx * 8);
    L->lines = L->spec + al256((size_t)C * g->R * g->H * 8);
    L->part = L->lines + al256((size_t)C * g->R * g->L * 4);
    L->work = L->part + al256((size_t)g->n_slots * C * FR_TS * FR_TS * 8);
    size_t w = 0;
    std::lock_guard<std::mutex> lk(g_plan_lock);
    const int kinds[4][4] = {{CUFFT_R2C, g->My, g->Mx, C},
                             {CUFFT_C2R, g->My, g->Mx, C},
                             {CUFFT_R2C, g->L, 0, C * g->R},
                             {CUFFT_C2R, g->L, 0, C * g->R}};
    for (auto &k : kinds) {
        Plan p;
        int st = get_plan(k[0], k[1], k[2], k[3], &p);
        if (st) return st;
        w = p.work > w ? p.work : w;
    }
    L->total = L->work + al256(w);
    return DFX_OK;
}

int check_geometry(const dfx_fr_geometry *g, const char *what)
{
    DFX_REQUIRE(g && g->inv_dx && g->inv_dy && g->filt && g->kb && g->w1 && g->w2 && g->tile_ptr && g->tile_smp &&
                    g->wa,
                "%s: incomplete geometry", what);
    DFX_REQUIRE(g->Nx > 0 && g->Ny > 0 && g->Ns > 0 && g->R > 0 && g->R <= 65535 && g->L >= 2 && g->L % 2 == 0 &&
                    g->H == g->L / 2 + 1 && g->Mx >= 2 && g->My >= 2 && g->My <= 65535 && (g->W == 6 || g->W == 7) &&
                    g->n_tx > 0 && g->n_tiles > 0,
                "%s: bad geometry sizes", what);
    DFX_REQUIRE((int64_t)g->R * g->H < 2147483647LL, "%s: too many polar samples", what);
    DFX_REQUIRE(g->pieces && g->tile_xptr && g->n_pieces >= g->n_tiles && g->n_slots >= 0,
                "%s: bad spreading pieces", what);
    return DFX_OK;
}

// Equal channel slices of at most `channels` (the plans' batch is the slice size cs; the last slice may be smaller)
int slice_size(int kb, int channels)
{
    const int n = (kb + channels - 1) / channels;
    return (kb + n - 1) / n;
}

}  // namespace
}  // namespace dfx

using namespace dfx;

extern "C" size_t dfx_fr_scratch_bytes(const dfx_fr_geometry *g, int channels)
{
    if (check_geometry(g, "fr_scratch_bytes") != DFX_OK || channels <= 0) return 0;
    Layout L;
    if (layout(g, channels, &L) != DFX_OK) return 0;
    return L.total;
}

extern "C" int dfx_fr_forward(const dfx_fr_geometry *g, const float *img_k, float *sino, int kstride, int kb,
                              int channels, void *scratch, size_t scratch_bytes, void *stream)
{
    int st = check_geometry(g, "fr_forward");
    if (st) return st;
    DFX_REQUIRE(img_k && sino && scratch && channels > 0 && kstride > 0 && kb >= 0 && kb <= kstride,
                "fr_forward: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    if (kb > 0) {
        const int cs = slice_size(kb, channels);
        DFX_REQUIRE(cdiv(cs, 32) <= 65535, "fr_forward: too many channels per slice");
        Layout L;
        if ((st = layout(g, cs, &L))) return st;
        DFX_REQUIRE(scratch_bytes >= L.total, "fr_forward: scratch of %zu bytes < %zu", scratch_bytes, L.total);
        char *base = (char *)scratch;
        float *grid = (float *)(base + L.grid);
        float2 *G = (float2 *)(base + L.G), *spec = (float2 *)(base + L.spec);
        float *lines = (float *)(base + L.lines);
        const int RH = g->R * g->H;
        for (int c0 = 0; c0 < kb; c0 += cs) {
            const int cb = kb - c0 < cs ? kb - c0 : cs;
            fr_pad_kernel<<<dim3((unsigned)cdiv(g->Mx, 32), (unsigned)g->My, (unsigned)cdiv(cs, 32)), dim3(32, 8), 0,
                            s>>>(img_k, kstride, c0, cb, grid, g->inv_dx, g->inv_dy, g->Nx, g->Ny, g->Mx, g->My,
                                 g->cx, g->cy, cs);
            if ((st = launch_status("fr_pad"))) return st;
            if ((st = run_plan(CUFFT_R2C, g->My, g->Mx, cs, grid, G, base + L.work, scratch_bytes - L.work, s)))
                return st;
            const dim3 sg((unsigned)cdiv(RH, 128), (unsigned)cs);
            if (g->W == 7)
                fr_slices_kernel<7><<<sg, 128, 0, s>>>(G, (const int2 *)g->kb, g->w1, g->w2, (const float2 *)g->filt,
                                                       spec, g->Mx, g->My, RH, g->H);
            else
                fr_slices_kernel<6><<<sg, 128, 0, s>>>(G, (const int2 *)g->kb, g->w1, g->w2, (const float2 *)g->filt,
                                                       spec, g->Mx, g->My, RH, g->H);
            if ((st = launch_status("fr_slices"))) return st;
            if ((st = run_plan(CUFFT_C2R, g->L, 0, cs * g->R, spec, lines, base + L.work, scratch_bytes - L.work, s)))
                return st;
            fr_lines_out_kernel<<<dim3((unsigned)cdiv(g->Ns, 32), (unsigned)cdiv(cb, 32), (unsigned)g->R),
                                  dim3(32, 8), 0, s>>>(lines, sino, g->R, g->Ns, g->L, kstride, c0, cb, g->scale);
            if ((st = launch_status("fr_lines_out"))) return st;
        }
    }
    if (kb < kstride) {
        const int64_t n_lines = (int64_t)g->R * g->Ns;
        fr_zero_channels_kernel<<<(unsigned)std::min<int64_t>(cdiv(n_lines * (kstride - kb), 256), 148 * 32), 256, 0,
                                  s>>>(sino, n_lines, kstride, kb);
        if ((st = launch_status("fr_zero_channels"))) return st;
    }
    return DFX_OK;
}

extern "C" int dfx_fr_backward(const dfx_fr_geometry *g, const float *sino, float *img_k, int kstride, int kb,
                               int channels, void *scratch, size_t scratch_bytes, void *stream)
{
    int st = check_geometry(g, "fr_backward");
    if (st) return st;
    DFX_REQUIRE(img_k && sino && scratch && channels > 0 && kstride > 0 && kb >= 0 && kb <= kstride,
                "fr_backward: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    if (kb > 0) {
        const int cs = slice_size(kb, channels);
        DFX_REQUIRE(cdiv(cs, 32) <= 65535, "fr_backward: too many channels per slice");
        Layout L;
        if ((st = layout(g, cs, &L))) return st;
        DFX_REQUIRE(scratch_bytes >= L.total, "fr_backward: scratch of %zu bytes < %zu", scratch_bytes, L.total);
        char *base = (char *)scratch;
        float *grid = (float *)(base + L.grid);
        float2 *Q = (float2 *)(base + L.G), *spec = (float2 *)(base + L.spec);
        float *lines = (float *)(base + L.lines);
        const int RH = g->R * g->H;
        for (int c0 = 0; c0 < kb; c0 += cs) {
            const int cb = kb - c0 < cs ? kb - c0 : cs;
            fr_lines_in_kernel<<<dim3((unsigned)cdiv(g->L, 32), (unsigned)cdiv(cs, 32), (unsigned)g->R), dim3(32, 8),
                                 0, s>>>(sino, lines, g->wa, g->R, g->Ns, g->L, kstride, c0, cb, cs);
            if ((st = launch_status("fr_lines_in"))) return st;
            if ((st = run_plan(CUFFT_R2C, g->L, 0, cs * g->R, lines, spec, base + L.work, scratch_bytes - L.work, s)))
                return st;
            const int64_t nsp = (int64_t)cs * RH;
            fr_unfilter_kernel<<<(unsigned)std::min<int64_t>(cdiv(nsp, 256), 148 * 32), 256, 0, s>>>(
                spec, (const float2 *)g->filt, RH, nsp);
            if ((st = launch_status("fr_unfilter"))) return st;
            const dim3 sg((unsigned)g->n_pieces, (unsigned)cdiv(cs, FR_CCS));
            DFX_REQUIRE(sg.y <= 65535u, "fr_backward: too many channels per slice");
            float2 *part = (float2 *)(base + L.part);
            if (g->W == 7)
                fr_spread_kernel<7><<<sg, dim3(FR_TS, FR_TS), 0, s>>>(spec, (const int4 *)g->pieces, g->tile_smp,
                                                                     (const int2 *)g->kb, g->w1, g->w2, Q, part,
                                                                     g->Mx, g->My, RH, g->H, g->n_tx, cs);
            else
                fr_spread_kernel<6><<<sg, dim3(FR_TS, FR_TS), 0, s>>>(spec, (const int4 *)g->pieces, g->tile_smp,
                                                                     (const int2 *)g->kb, g->w1, g->w2, Q, part,
                                                                     g->Mx, g->My, RH, g->H, g->n_tx, cs);
            if ((st = launch_status("fr_spread"))) return st;
            if (g->n_slots > 0) {
                fr_spread_finish_kernel<<<(unsigned)g->n_tiles, dim3(FR_TS, FR_TS), 0, s>>>(Q, part, g->tile_xptr,
                                                                                             g->Mx, g->My, g->n_tx, cs);
                if ((st = launch_status("fr_spread_finish"))) return st;
            }
            if ((st = run_plan(CUFFT_C2R, g->My, g->Mx, cs, Q, grid, base + L.work, scratch_bytes - L.work, s)))
                return st;
            fr_crop_kernel<<<dim3((unsigned)cdiv(g->Nx, 32), (unsigned)g->Ny, (unsigned)cdiv(cb, 32)), dim3(32, 8), 0,
                             s>>>(grid, img_k, kstride, c0, cb, g->inv_dx, g->inv_dy, g->Nx, g->Ny, g->Mx, g->My,
                                  g->cx, g->cy);
            if ((st = launch_status("fr_crop"))) return st;
        }
    }
    if (kb < kstride) {
        const int64_t n_lines = (int64_t)g->Nx * g->Ny;
        fr_zero_channels_kernel<<<(unsigned)std::min<int64_t>(cdiv(n_lines * (kstride - kb), 256), 148 * 32), 256, 0,
                                  s>>>(img_k, n_lines, kstride, kb);
        if ((st = launch_status("fr_zero_channels"))) return st;
    }
    return DFX_OK;
}
