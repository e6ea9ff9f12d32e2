// BF16 tensor-core contraction of the Radon output with the dense pole-figure matrix (tcgen05, sm_100a).
//
// Per angle r of a subset the contraction is a GEMM with float32 accumulation in tensor memory:
//   forward  data[r, y, j]  (+)=     sum_k PF[r, k, j] Z[r, y, k]   D^T (j x y) = PF^T (j x k) . Z^T (k x y)
//   adjoint  Z[r, y, k]      = alpha sum_j PF[r, k, j] D[r, y, j]   Z^T (k x y) = PF   (k x j) . D^T (j x y)
// PF is stored densely in BF16 as (R, Ktot, CPpad) (segments fastest); Z, the channel-fastest Radon output of all
// orientation batches of the subset, as (n_sub, My, Ktot) BF16; D's BF16 copy as (R, My, CPpad). One CTA computes a
// 128 x NT tile (M = segments or orientations, N = translations y) of one angle: TMA streams 64-wide K slices of
// both operands (128-byte swizzle) into a ring of shared-memory stages, one thread issues tcgen05.mma (M = 128,
// K = 16 per instruction) into a 128-lane x NT-column float32 accumulator in tensor memory, tcgen05.commit frees a
// stage when the MMAs reading it are done, and after the last slice four warps move the accumulator to registers
// (tcgen05.ld) and write it with coalesced stores. Two CTAs fit an SM, so one CTA's epilogue overlaps the other's
// main loop. Every wait on an mbarrier is bounded in time: on expiry the kernel records DFX_TC_TIMEOUT in a device
// flag, stops issuing, waits (bounded) for its copies in flight, frees its tensor memory and returns.
//
// Replaces the dense batched GEMMs batched_gemm_clblast / _adj of the reference (SPFO:2063-2127) and, in the BF16
// precision path, the sparse products spmm_pf_forward_c / spmm_pf_adjoint_c (pf_kernels.cl:597-687).

#include <cuda.h>
#include <cuda_bf16.h>

#include <mutex>

#include "tc_common.cuh"

namespace dfx {
namespace {

using namespace tc;

constexpr int TC_M = 128;              // tile rows = tensor-memory lanes
constexpr int TC_BK = 64;              // K elements per stage: one 128-byte swizzle row of BF16
constexpr int TC_THREADS = 128;
constexpr int A_STAGE_BYTES = TC_M * TC_BK * 2;

__device__ unsigned int g_tc_flags;    // DFX_TC_* bits of expired waits since the last dfx_tc_status reset

struct TcArgs {
    const int32_t *omegas;   // subset angles (n_sub), NULL: angle = subset index
    int n_sub, m_extent, n_extent, nt, k_chunks, stages;
    float *out_f32;          // forward: data (R, My, CP)
    __nv_bfloat16 *out_bf16; // adjoint: Z (n_sub, My, Ktot)
    int64_t out_ld;          // forward: CP; adjoint: Ktot
    float alpha;
    int accumulate;
    int pf_compact;          // the PF holds the subset's angles only: its angle coordinate is the subset index
};

constexpr uint32_t TMEM_COLS = 256;    // NT <= 256 float32 columns

// DIR 0: forward (A = PF^T, MN-major; out float32 data), DIR 1: adjoint (A = PF, K-major; out BF16 Z).
template <int DIR>
__global__ void __launch_bounds__(TC_THREADS) pf_tc_kernel(const __grid_constant__ CUtensorMap map_a,
                                                           const __grid_constant__ CUtensorMap map_b, TcArgs p)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);     // swizzle atoms: 1024-byte aligned offsets
    const int S = p.stages;
    const uint32_t b_stage_bytes = (uint32_t)p.nt * TC_BK * 2;
    uint8_t *a_tiles = smem;
    uint8_t *b_tiles = smem + (size_t)S * A_STAGE_BYTES;
    uint64_t *bars = reinterpret_cast<uint64_t *>(b_tiles + (size_t)S * b_stage_bytes);   // full[S], empty[S], done
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * S + 1);
    int *progress = reinterpret_cast<int *>(tmem_slot + 1);                                  // issued, consumed

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rl = blockIdx.z;
    const int r = p.omegas ? __ldg(p.omegas + rl) : rl;
    const int rp = p.pf_compact ? rl : r;                        // the PF's angle coordinate
    const int m0 = blockIdx.y * TC_M, n0 = blockIdx.x * p.nt;
    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + S), done = smem_u32(bars + 2 * S);

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        mbar_init(done, 1);
        progress[0] = progress[1] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_a)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_b)) : "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (threadIdx.x == 0) {
        // producer: TMA slices of A and B into the stage ring
        const bool a_hi = DIR == 0 && m0 + 64 < p.m_extent;      // forward: second 64-segment box of the tile
        const uint32_t tx = (DIR == 0 ? (a_hi ? 2u : 1u) * (A_STAGE_BYTES / 2) : (uint32_t)A_STAGE_BYTES) +
                            b_stage_bytes;
        int kc = 0;
        for (; kc < p.k_chunks; ++kc) {
            const int s = kc % S;
            if (kc >= S && !mbar_wait(empty0 + 8 * s, ((kc / S) & 1) ^ 1, DFX_TC_TIMEOUT, &g_tc_flags)) break;
            const uint32_t fb = full0 + 8 * s;
            mbar_expect_tx(fb, tx);
            const uint32_t a_dst = smem_u32(a_tiles + (size_t)s * A_STAGE_BYTES);
            const uint32_t b_dst = smem_u32(b_tiles + (size_t)s * b_stage_bytes);
            if (DIR == 0) {
                tma_load_3d(a_dst, &map_a, fb, m0, kc * TC_BK, rp);
                if (a_hi) tma_load_3d(a_dst + A_STAGE_BYTES / 2, &map_a, fb, m0 + 64, kc * TC_BK, rp);
                tma_load_3d(b_dst, &map_b, fb, kc * TC_BK, n0, rl);
            } else {
                tma_load_3d(a_dst, &map_a, fb, kc * TC_BK, m0, rp);
                tma_load_3d(b_dst, &map_b, fb, kc * TC_BK, n0, r);
            }
        }
        progress[0] = kc;
    } else if (threadIdx.x == 32) {
        // MMA issuer
        const uint32_t idesc = instr_desc(p.nt, DIR == 0 ? 1 : 0);
        int kc = 0;
        for (; kc < p.k_chunks; ++kc) {
            const int s = kc % S;
            if (!mbar_wait(full0 + 8 * s, (kc / S) & 1, DFX_TC_TIMEOUT, &g_tc_flags)) break;
            tc_fence_after();
            const uint32_t a_base = smem_u32(a_tiles + (size_t)s * A_STAGE_BYTES);
            const uint32_t b_base = smem_u32(b_tiles + (size_t)s * b_stage_bytes);
#pragma unroll
            for (int kk = 0; kk < TC_BK / 16; ++kk) {
                // A: MN-major K step = 16 rows of 128 B (two 8-row groups); K-major = 32 B inside the swizzle row
                const uint64_t ad = DIR == 0 ? smem_desc(a_base + kk * 2048, A_STAGE_BYTES / 2, 1024)
                                             : smem_desc(a_base + kk * 32, 16, 1024);
                const uint64_t bd = smem_desc(b_base + kk * 32, 16, 1024);
                mma_bf16(tmem, ad, bd, idesc, (kc | kk) != 0);
            }
            mma_commit(empty0 + 8 * s);         // the stage is free once these MMAs have read it
        }
        progress[1] = kc;
        mma_commit(done);                       // accumulator complete
    }
    __syncwarp();

    // epilogue: lane i of warp w holds row m0 + 32 w + i of the tile
    const bool ok = mbar_wait(done, 0, DFX_TC_TIMEOUT, &g_tc_flags);
    tc_fence_after();
    const int m = m0 + 32 * warp + lane;
    const bool row_live = m < p.m_extent;
    if (ok) {
        for (int c = 0; c < p.nt; c += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c, v);
            if (!row_live) continue;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int n = n0 + c + i;
                if (n >= p.n_extent) break;
                if (DIR == 0) {
                    float *o = p.out_f32 + ((int64_t)r * p.n_extent + n) * p.out_ld + m;
                    *o = p.accumulate ? __fadd_rn(*o, v[i]) : v[i];
                } else {
                    p.out_bf16[((int64_t)rl * p.n_extent + n) * p.out_ld + m] =
                        __float2bfloat16_rn(__fmul_rn(p.alpha, v[i]));
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0) {
        // copies issued but never consumed (only after an expired wait): let them land before the CTA exits
        for (int kc = progress[1]; kc < progress[0]; ++kc)
            if (!mbar_wait(full0 + 8 * (kc % S), (kc / S) & 1, DFX_TC_TIMEOUT, &g_tc_flags)) break;
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

// BF16 copy of data rows: one block-stride loop over (row, y, column of cp_pad) of the listed angles.
__global__ void rows_to_bf16_kernel(const float *__restrict__ in, __nv_bfloat16 *__restrict__ out,
                                    const int32_t *__restrict__ omegas, int n_sub, int my, int cp, int cp_pad)
{
    const int64_t per = (int64_t)my * cp_pad, total = per * n_sub;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int s = (int)(i / per);
        const int64_t q = i % per;
        const int y = (int)(q / cp_pad), j = (int)(q % cp_pad);
        const int64_t r = omegas ? __ldg(omegas + s) : s;
        const float v = j < cp ? __ldg(in + (r * my + y) * cp + j) : 0.0f;
        out[(r * my + y) * cp_pad + j] = __float2bfloat16_rn(v);
    }
}

__global__ void f32_to_bf16_kernel(const float4 *__restrict__ in, uint2 *__restrict__ out, int64_t n4)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
        const float4 v = __ldg(in + i);
        const __nv_bfloat162 a = __floats2bfloat162_rn(v.x, v.y), b = __floats2bfloat162_rn(v.z, v.w);
        out[i] = make_uint2(*reinterpret_cast<const uint32_t *>(&a), *reinterpret_cast<const uint32_t *>(&b));
    }
}

// Strided row conversions between a float32 sinogram (rows of ld_f32) and BF16 rows (ld_bf16): TO_BF16 rounds to
// nearest-even, the other way widens exactly. rows x cols elements; one thread per element.
template <int TO_BF16>
__global__ void convert_rows_kernel(float *__restrict__ f32, int64_t ld_f32, __nv_bfloat16 *__restrict__ b16,
                                    int64_t ld_b16, int64_t rows, int cols)
{
    const int64_t total = rows * cols;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / cols;
        const int c = (int)(i - r * cols);
        if (TO_BF16)
            b16[r * ld_b16 + c] = __float2bfloat16_rn(f32[r * ld_f32 + c]);
        else
            f32[r * ld_f32 + c] = __bfloat162float(b16[r * ld_b16 + c]);
    }
}

// ---------------------------------------------------------------------------------------------- host side
// N tile: the translations split into the fewest tiles of at most 256, each a multiple of 16.
int n_tile(int my)
{
    const int tiles = (int)cdiv(my, 256);
    return (int)(cdiv(cdiv(my, tiles), 16) * 16);
}

size_t smem_bytes(int nt, int stages)
{
    return 1024 + (size_t)stages * (A_STAGE_BYTES + (size_t)nt * TC_BK * 2) + (2 * stages + 1) * 8 + 16;
}

int pick_stages(int nt)
{
    // two CTAs per SM (228 KB of shared memory, 1 KB reserved per CTA) when four stages or fewer fit
    for (int s = 4; s >= 2; --s)
        if (smem_bytes(nt, s) <= 112 * 1024) return s;
    return 2;
}

template <int DIR>
int launch(const CUtensorMap &ma, const CUtensorMap &mb, TcArgs a, int m_tiles, cudaStream_t stream)
{
    const size_t smem = smem_bytes(a.nt, a.stages);
    const cudaError_t e = allow_max_dynamic_smem(pf_tc_kernel<DIR>);
    if (e != cudaSuccess) {
        set_error("pf_tc: shared memory attribute: %s", cudaGetErrorString(e));
        return DFX_ELAUNCH;
    }
    dim3 grid((unsigned)cdiv(a.n_extent, a.nt), (unsigned)m_tiles, (unsigned)a.n_sub);
    pf_tc_kernel<DIR><<<grid, TC_THREADS, smem, stream>>>(ma, mb, a);
    return launch_status(DIR == 0 ? "pf_tc_forward" : "pf_tc_adjoint");
}

int check_common(const void *pf, int64_t ktot, int64_t k0, int64_t kn, int cp, int cp_pad, int n_sub, int my,
                 int n_omega)
{
    DFX_REQUIRE(pf != nullptr, "pf_tc: null PF");
    DFX_REQUIRE(ktot > 0 && ktot % 8 == 0 && ktot <= 2147483647LL, "pf_tc: Ktot (%lld) must be a positive multiple "
                "of 8", (long long)ktot);
    DFX_REQUIRE(k0 >= 0 && k0 % 8 == 0 && kn > 0 && k0 + kn <= ktot, "pf_tc: orientation range %lld + %lld outside "
                "Ktot %lld (start a multiple of 8)", (long long)k0, (long long)kn, (long long)ktot);
    DFX_REQUIRE(cp > 0 && cp_pad >= cp && cp_pad % 8 == 0, "pf_tc: CPpad (%d) must be a multiple of 8 >= CP (%d)",
                cp_pad, cp);
    DFX_REQUIRE(n_sub > 0 && n_sub <= 65535 && n_omega > 0, "pf_tc: bad angle counts");
    DFX_REQUIRE(my > 0 && my <= 65535, "pf_tc: bad number of translations (%d)", my);
    return DFX_OK;
}

}  // namespace
}  // namespace dfx

using namespace dfx;

extern "C" int dfx_pf_tc_forward(const void *pf_bf16, int64_t ktot, int64_t k0, int64_t kn, int cp, int cp_pad,
                                 int n_omega, const void *z_bf16, const int32_t *omegas, int n_sub, int my, float *data,
                                 int accumulate, int pf_compact, void *stream)
{
    int st = check_common(pf_bf16, ktot, k0, kn, cp, cp_pad, n_sub, my, n_omega);
    if (st) return st;
    DFX_REQUIRE(z_bf16 && data, "pf_tc_forward: null pointer");
    const __nv_bfloat16 *pf = reinterpret_cast<const __nv_bfloat16 *>(pf_bf16) + k0 * cp_pad;
    const __nv_bfloat16 *z = reinterpret_cast<const __nv_bfloat16 *>(z_bf16) + k0;
    CUtensorMap ma, mb;
    TcArgs a{};
    a.omegas = omegas;
    a.n_sub = n_sub;
    a.m_extent = cp;
    a.n_extent = my;
    a.nt = n_tile(my);
    a.k_chunks = (int)cdiv(kn, TC_BK);
    a.stages = pick_stages(a.nt);
    a.out_f32 = data;
    a.out_ld = cp;
    a.alpha = 1.0f;
    a.accumulate = accumulate != 0;
    a.pf_compact = pf_compact != 0;
    if ((st = make_map(&ma, pf, (uint64_t)cp_pad, (uint64_t)kn, (uint64_t)(pf_compact ? n_sub : n_omega),
                       (uint64_t)cp_pad, (uint64_t)ktot * cp_pad, 64, 64, "PF")))
        return st;
    if ((st = make_map(&mb, z, (uint64_t)kn, (uint64_t)my, (uint64_t)n_sub, (uint64_t)ktot, (uint64_t)ktot * my, 64,
                       (uint32_t)a.nt, "Z")))
        return st;
    return launch<0>(ma, mb, a, (int)cdiv(cp, TC_M), (cudaStream_t)stream);
}

extern "C" int dfx_pf_tc_adjoint(const void *pf_bf16, int64_t ktot, int64_t k0, int64_t kn, int cp, int cp_pad,
                                 int n_omega, const void *d_bf16, const int32_t *omegas, int n_sub, int my,
                                 float alpha, void *z_bf16, int pf_compact, void *stream)
{
    int st = check_common(pf_bf16, ktot, k0, kn, cp, cp_pad, n_sub, my, n_omega);
    if (st) return st;
    DFX_REQUIRE(z_bf16 && d_bf16, "pf_tc_adjoint: null pointer");
    const __nv_bfloat16 *pf = reinterpret_cast<const __nv_bfloat16 *>(pf_bf16) + k0 * cp_pad;
    CUtensorMap ma, mb;
    TcArgs a{};
    a.omegas = omegas;
    a.n_sub = n_sub;
    a.m_extent = (int)kn;
    a.n_extent = my;
    a.nt = n_tile(my);
    a.k_chunks = (int)cdiv(cp_pad, TC_BK);
    a.stages = pick_stages(a.nt);
    a.out_bf16 = reinterpret_cast<__nv_bfloat16 *>(z_bf16) + k0;
    a.out_ld = ktot;
    a.alpha = alpha;
    a.pf_compact = pf_compact != 0;
    if ((st = make_map(&ma, pf, (uint64_t)cp_pad, (uint64_t)kn, (uint64_t)(pf_compact ? n_sub : n_omega),
                       (uint64_t)cp_pad, (uint64_t)ktot * cp_pad, 64, TC_M, "PF")))
        return st;
    if ((st = make_map(&mb, d_bf16, (uint64_t)cp_pad, (uint64_t)my, (uint64_t)n_omega, (uint64_t)cp_pad,
                       (uint64_t)cp_pad * my, 64, (uint32_t)a.nt, "D")))
        return st;
    return launch<1>(ma, mb, a, (int)cdiv(kn, TC_M), (cudaStream_t)stream);
}

namespace dfx {
unsigned int tcb_status(unsigned int reset);    // the flags of the tensor-core backprojection (radon_tc.cu)
unsigned int tcf_status(unsigned int reset);    // the flags of the tensor-core forward projection (radon_tc_fwd.cu)
}

extern "C" int dfx_tc_status(unsigned int *flags, int reset)
{
    DFX_REQUIRE(flags != nullptr, "tc_status: null output");
    cudaError_t e = cudaMemcpyFromSymbol(flags, g_tc_flags, sizeof(unsigned int));
    *flags |= dfx::tcb_status(reset ? 1u : 0u);
    *flags |= dfx::tcf_status(reset ? 1u : 0u);
    if (e == cudaSuccess && reset) {
        const unsigned int zero = 0;
        e = cudaMemcpyToSymbol(g_tc_flags, &zero, sizeof(unsigned int));
    }
    if (e != cudaSuccess) {
        set_error("tc_status: %s", cudaGetErrorString(e));
        return DFX_ELAUNCH;
    }
    return DFX_OK;
}

extern "C" int dfx_rows_to_bf16(const float *in, void *out, const int32_t *omegas, int n_sub, int my, int cp,
                                int cp_pad, void *stream)
{
    DFX_REQUIRE(in && out, "rows_to_bf16: null pointer");
    DFX_REQUIRE(n_sub > 0 && my > 0 && cp > 0 && cp_pad >= cp, "rows_to_bf16: bad sizes");
    const int64_t n = (int64_t)n_sub * my * cp_pad;
    const int64_t blocks = cdiv(n, 256);
    rows_to_bf16_kernel<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, (cudaStream_t)stream>>>(
        in, reinterpret_cast<__nv_bfloat16 *>(out), omegas, n_sub, my, cp, cp_pad);
    return launch_status("rows_to_bf16");
}

extern "C" int dfx_f32_to_bf16(const float *in, void *out, int64_t n, void *stream)
{
    DFX_REQUIRE(in && out && n >= 0 && n % 4 == 0, "f32_to_bf16: null pointer or n not a multiple of 4");
    DFX_REQUIRE(((uintptr_t)in % 16) == 0 && ((uintptr_t)out % 8) == 0, "f32_to_bf16: misaligned arrays");
    if (n == 0) return DFX_OK;
    const int64_t blocks = cdiv(n / 4, 256);
    f32_to_bf16_kernel<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const float4 *>(in), reinterpret_cast<uint2 *>(out), n / 4);
    return launch_status("f32_to_bf16");
}

extern "C" int dfx_convert_rows(int to_bf16, float *f32, int64_t ld_f32, void *b16, int64_t ld_b16, int64_t rows,
                                int cols, void *stream)
{
    DFX_REQUIRE(f32 && b16, "convert_rows: null pointer");
    DFX_REQUIRE(rows >= 0 && cols >= 0 && ld_f32 >= cols && ld_b16 >= cols, "convert_rows: bad sizes");
    const int64_t n = rows * cols;
    if (n == 0) return DFX_OK;
    const int64_t blocks = cdiv(n, 256);
    const unsigned g = (unsigned)(blocks < 148 * 16 ? blocks : 148 * 16);
    auto *b = reinterpret_cast<__nv_bfloat16 *>(b16);
    if (to_bf16)
        convert_rows_kernel<1><<<g, 256, 0, (cudaStream_t)stream>>>(f32, ld_f32, b, ld_b16, rows, cols);
    else
        convert_rows_kernel<0><<<g, 256, 0, (cudaStream_t)stream>>>(f32, ld_f32, b, ld_b16, rows, cols);
    return launch_status("convert_rows");
}
