// Element-wise and reduction kernels of the Poisson solvers (SPDHGPoisson, FISTAPoisson) on sm_100a.
//
// Element-wise kernels are grid-stride loops over 64-bit indices (one pass over HBM, vectorised where the layout
// allows). Reductions sum in float64: every block reduces its grid-stride share with warp shuffles into one partial
// in the caller's scratch, and one block sums the partials in a fixed order, so the result does not depend on
// timing (bitwise reproducible for a given launch shape).
#include <cuda_bf16.h>

#include "dfx_common.cuh"

namespace dfx {

constexpr int EW_THREADS = 256;
constexpr int RED_THREADS = 256;
constexpr int RED_BLOCKS_MAX = 148 * 8;

static unsigned ew_grid(int64_t n)
{
    const int64_t b = cdiv(n, EW_THREADS);
    return (unsigned)(b < 148 * 32 ? (b > 0 ? b : 1) : 148 * 32);
}

static int red_blocks(int64_t n)
{
    const int64_t b = cdiv(n, RED_THREADS * 4);
    return (int)(b < RED_BLOCKS_MAX ? (b > 0 ? b : 1) : RED_BLOCKS_MAX);
}

__device__ __forceinline__ float periodic(const float *a, int64_t period, int64_t i, float dflt)
{
    return period ? __ldg(a + (i % period)) : dflt;
}

// sum over the block of NS doubles per thread, written by thread 0 to out[0 .. NS-1]
template <int NS>
__device__ __forceinline__ void block_sum(double (&v)[NS], double *out)
{
    __shared__ double sh[NS][RED_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NS; ++q) {
        double x = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[q][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            double s = 0.0;
            for (int w = 0; w < RED_THREADS / 32; ++w) s += sh[q][w];
            out[q] = s;
        }
    }
}

// out[q] = sum of the nb partials part[b * NS + q] (one block, fixed order)
template <int NS>
__global__ void __launch_bounds__(RED_THREADS) finish_sums(const double *__restrict__ part, int nb, double *out)
{
    double v[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nb; b += RED_THREADS) s += part[(int64_t)b * NS + q];
        v[q] = s;
    }
    block_sum<NS>(v, out);
}


// ---- FISTA for least squares and Huber (FISTAL2 / FISTAHuber) ----
constexpr int FU_BLOCKS = 148 * 4;    // blocks of one fused update launch = its partial sums

// r = w (Ax - b) (w periodic, pw = 0: 1) in place, clipped to [-delta, delta] if clip; partial sums of r^2 before
// the clip (fista_huber.py / fista_l2.py residual_sumsq)
__global__ void __launch_bounds__(RED_THREADS) ls_residual_kernel(float *__restrict__ ax, const float *__restrict__ b,
                                                                  const float *__restrict__ w, int64_t pw, int clip,
                                                                  float delta, int64_t n, double *part)
{
    double v[1] = {0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float r = __fsub_rn(ax[i], b[i]);
        if (pw) r = __fmul_rn(periodic(w, pw, i, 1.0f), r);
        v[0] += (double)r * (double)r;
        if (clip) r = fminf(fmaxf(r, -delta), delta);
        ax[i] = r;
    }
    block_sum<1>(v, part + blockIdx.x);
}

// The FISTA step of one orientation batch in the channel-fastest layout (npix x kstride, kb live channels), from its
// gradient g: v = prox(y - tau g) (0: max(v, 0); 1: soft threshold lt; 2: max(v - lt, 0)), 0 outside the support and
// on padding channels; y = v + beta (v - x); x = v (fused_update.py:22-49). Per-block partials of g^2, v^2, |v|.
__global__ void __launch_bounds__(RED_THREADS) fista_ls_update_kernel(
    const float4 *__restrict__ g, float4 *__restrict__ x, float4 *__restrict__ y, const uint8_t *__restrict__ supp,
    int64_t npix, int kq, int kb, float tau, float beta, float lt, int prox, double *part)
{
    double acc[3] = {0.0, 0.0, 0.0};
    const int64_t n4 = npix * kq;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n4; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pix = t / kq;
        const int k = (int)(t - pix * kq) * 4;
        const bool in = supp == nullptr || supp[pix] != 0;
        const float4 gv = g[t], xv = x[t], yv = y[t];
        const float gg[4] = {gv.x, gv.y, gv.z, gv.w}, xo[4] = {xv.x, xv.y, xv.z, xv.w};
        const float yy[4] = {yv.x, yv.y, yv.z, yv.w};
        float xn[4], yn[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float v = __fsub_rn(yy[c], __fmul_rn(tau, gg[c]));
            if (prox == 0) {
                v = v < 0.0f ? 0.0f : v;
            } else if (prox == 1) {
                const float a = __fsub_rn(fabsf(v), lt);
                v = a > 0.0f ? copysignf(a, v) : 0.0f;
            } else {
                const float d = __fsub_rn(v, lt);
                v = d > 0.0f ? d : 0.0f;
            }
            if (!in || k + c >= kb) v = 0.0f;
            xn[c] = v;
            yn[c] = __fadd_rn(v, __fmul_rn(beta, __fsub_rn(v, xo[c])));
            acc[0] += (double)gg[c] * (double)gg[c];
            acc[1] += (double)v * (double)v;
            acc[2] += (double)fabsf(v);
        }
        x[t] = make_float4(xn[0], xn[1], xn[2], xn[3]);
        y[t] = make_float4(yn[0], yn[1], yn[2], yn[3]);
    }
    block_sum<3>(acc, part + 3 * (int64_t)blockIdx.x);
}


// ---- SPDHG's total-variation block on a channel-fastest batch (npix x kstride, kb live channels): forward
// differences to the right (+1 pixel) and down (+nx pixels) between free coefficients (T > 0 at both ends), the dual
// q = (qx, qy) per coefficient projected onto |q| <= lam after the step s = ps / (4 max(T_j + T_right, T_j + T_down))
// (spdhg_poisson.py:110-165). The float32 operations are correctly rounded, in the reference's order.
__device__ __forceinline__ void tv_dual_core(float tj, float tr, float td, bool vr0, bool vd0, float xj, float xr,
                                             float xd, float ox, float oy, float lam, float ps, float &nx, float &ny)
{
    const bool vr = vr0 && tj > 0.0f && tr > 0.0f;
    const bool vd = vd0 && tj > 0.0f && td > 0.0f;
    float m = 0.0f;
    if (vr) m = fmaxf(m, __fadd_rn(tj, tr));
    if (vd) m = fmaxf(m, __fadd_rn(tj, td));
    float ax = 0.0f, ay = 0.0f;
    if (m > 0.0f) {
        const float st = __fdiv_rn(ps, __fmul_rn(4.0f, m));
        if (vr) ax = __fadd_rn(ox, __fmul_rn(st, __fsub_rn(xr, xj)));
        if (vd) ay = __fadd_rn(oy, __fmul_rn(st, __fsub_rn(xd, xj)));
        const float nrm = __fsqrt_rn(__fadd_rn(__fmul_rn(ax, ax), __fmul_rn(ay, ay)));
        if (nrm > lam) {
            const float c = __fdiv_rn(lam, nrm);
            ax = __fmul_rn(ax, c);
            ay = __fmul_rn(ay, c);
        }
    }
    nx = ax;
    ny = ay;
}

// q <- proj(q + s D x), dq = q' - q (dq batch-sized)
__global__ void tv_dual_kernel(const float *__restrict__ x, const float *__restrict__ T, float *__restrict__ qx,
                               float *__restrict__ qy, float *__restrict__ dqx, float *__restrict__ dqy, int nx, int ny,
                               int kstride, float lam, float ps, int64_t n)
{
    const int64_t row = (int64_t)nx * kstride;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pix = i / kstride;
        const int ix = (int)(pix % nx), iy = (int)(pix / nx);
        const bool vr0 = ix + 1 < nx, vd0 = iy + 1 < ny;
        const float tr = vr0 ? T[i + kstride] : 0.0f, td = vd0 ? T[i + row] : 0.0f;
        const float xr = vr0 ? x[i + kstride] : 0.0f, xd = vd0 ? x[i + row] : 0.0f;
        const float ox = qx[i], oy = qy[i];
        float nxv, nyv;
        tv_dual_core(T[i], tr, td, vr0, vd0, x[i], xr, xd, ox, oy, lam, ps, nxv, nyv);
        qx[i] = nxv;
        qy[i] = nyv;
        dqx[i] = __fsub_rn(nxv, ox);
        dqy[i] = __fsub_rn(nyv, oy);
    }
}

// dz = D^T dq, then the primal step of SPDHG with it: z += dz; x = T > 0 ? max(0, x - T (z + inv_p dz + lam)) : 0
__global__ void tv_adjoint_update_kernel(const float *__restrict__ dqx, const float *__restrict__ dqy,
                                         float *__restrict__ x, float *__restrict__ z, const float *__restrict__ T,
                                         int nx, int kstride, float inv_p, float lam, int64_t n)
{
    const int64_t row = (int64_t)nx * kstride;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pix = i / kstride;
        const int ix = (int)(pix % nx);
        float v = __fsub_rn(-dqx[i], dqy[i]);
        if (ix > 0) v = __fadd_rn(v, dqx[i - kstride]);
        if (pix >= nx) v = __fadd_rn(v, dqy[i - row]);
        const float zi = __fadd_rn(z[i], v);
        z[i] = zi;
        const float zb = __fadd_rn(zi, __fmul_rn(inv_p, v));
        const float t = T[i];
        x[i] = t > 0.0f ? fmaxf(0.0f, __fsub_rn(x[i], __fmul_rn(t, __fadd_rn(zb, lam)))) : 0.0f;
    }
}

// sum of |D x| over the coefficients (float32 norms, float64 sum)
__global__ void __launch_bounds__(RED_THREADS) tv_value_kernel(const float *__restrict__ x,
                                                               const float *__restrict__ T, int nx, int ny,
                                                               int kstride, int64_t n, double *__restrict__ part)
{
    const int64_t row = (int64_t)nx * kstride;
    double v[1] = {0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pix = i / kstride;
        const int ix = (int)(pix % nx), iy = (int)(pix / nx);
        const bool vr0 = ix + 1 < nx, vd0 = iy + 1 < ny;
        const float tj = T[i];
        const float gx = (vr0 && tj > 0.0f && T[i + kstride] > 0.0f) ? __fsub_rn(x[i + kstride], x[i]) : 0.0f;
        const float gy = (vd0 && tj > 0.0f && T[i + row] > 0.0f) ? __fsub_rn(x[i + row], x[i]) : 0.0f;
        v[0] += (double)__fsqrt_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)));
    }
    block_sum<1>(v, part + blockIdx.x);
}

// ---- the TV block on a local basis's flat coefficients (spdhg_poisson.py:188-230): the differences to the right and
// down neighbours within a coefficient's patch (index arrays, -1: none); the same arithmetic as the dense kernels
__global__ void tv_dual_local_kernel(const float *__restrict__ x, const float *__restrict__ T, float *__restrict__ qx,
                                     float *__restrict__ qy, float *__restrict__ dqx, float *__restrict__ dqy,
                                     const int32_t *__restrict__ right, const int32_t *__restrict__ down, float lam,
                                     float ps, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int r = right[i], d = down[i];
        const bool vr0 = r >= 0, vd0 = d >= 0;
        const float ox = qx[i], oy = qy[i];
        float nxv, nyv;
        tv_dual_core(T[i], vr0 ? T[r] : 0.0f, vd0 ? T[d] : 0.0f, vr0, vd0, x[i], vr0 ? x[r] : 0.0f,
                     vd0 ? x[d] : 0.0f, ox, oy, lam, ps, nxv, nyv);
        qx[i] = nxv;
        qy[i] = nyv;
        dqx[i] = __fsub_rn(nxv, ox);
        dqy[i] = __fsub_rn(nyv, oy);
    }
}

// (D^T dq)_i within the patches: -dqx_i - dqy_i + dqx_left + dqy_up
__device__ __forceinline__ float tv_adjoint_local_at(const float *__restrict__ dqx, const float *__restrict__ dqy,
                                                     const int32_t *__restrict__ left, const int32_t *__restrict__ up,
                                                     int64_t i)
{
    float v = __fsub_rn(-dqx[i], dqy[i]);
    const int l = left[i], u = up[i];
    if (l >= 0) v = __fadd_rn(v, dqx[l]);
    if (u >= 0) v = __fadd_rn(v, dqy[u]);
    return v;
}

__global__ void tv_adjoint_update_local_kernel(const float *__restrict__ dqx, const float *__restrict__ dqy,
                                               float *__restrict__ x, float *__restrict__ z,
                                               const float *__restrict__ T, const int32_t *__restrict__ left,
                                               const int32_t *__restrict__ up, float inv_p, float lam, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = tv_adjoint_local_at(dqx, dqy, left, up, i);
        const float zi = __fadd_rn(z[i], v);
        z[i] = zi;
        const float zb = __fadd_rn(zi, __fmul_rn(inv_p, v));
        const float t = T[i];
        x[i] = t > 0.0f ? fmaxf(0.0f, __fsub_rn(x[i], __fmul_rn(t, __fadd_rn(zb, lam)))) : 0.0f;
    }
}

__global__ void __launch_bounds__(RED_THREADS) tv_value_local_kernel(const float *__restrict__ x,
                                                                     const float *__restrict__ T,
                                                                     const int32_t *__restrict__ right,
                                                                     const int32_t *__restrict__ down, int64_t n,
                                                                     double *__restrict__ part)
{
    double v[1] = {0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int r = right[i], d = down[i];
        const float tj = T[i];
        const float gx = (r >= 0 && tj > 0.0f && T[r] > 0.0f) ? __fsub_rn(x[r], x[i]) : 0.0f;
        const float gy = (d >= 0 && tj > 0.0f && T[d] > 0.0f) ? __fsub_rn(x[d], x[i]) : 0.0f;
        v[0] += (double)__fsqrt_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)));
    }
    block_sum<1>(v, part + blockIdx.x);
}

// ---- the hierarchical total variation on a local basis (spdhg_poisson.py:232-249): the node-pixels of a level of the
// orientation tree (a cell of orientations in one pixel), their sums s over the cell's coefficients (CSR ptr / idx
// into the flat coefficients, float32 in the list's order), D^T dq on the node-pixels, and its scatter back onto the
// coefficients (map: a coefficient's node-pixel, -1: none)
__global__ void tree_sums_kernel(const float *__restrict__ x, const int32_t *__restrict__ ptr,
                                 const int32_t *__restrict__ idx, float *__restrict__ s, int64_t n)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        float a = 0.0f;
        for (int p = ptr[j], e = ptr[j + 1]; p < e; ++p) a = __fadd_rn(a, x[idx[p]]);
        s[j] = a;
    }
}

__global__ void tv_adjoint_local_kernel(const float *__restrict__ dqx, const float *__restrict__ dqy,
                                        float *__restrict__ w, const int32_t *__restrict__ left,
                                        const int32_t *__restrict__ up, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        w[i] = tv_adjoint_local_at(dqx, dqy, left, up, i);
}

__global__ void tree_scatter_kernel(const float *__restrict__ w, const int32_t *__restrict__ map,
                                    float *__restrict__ dz, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int m = map[i];
        if (m >= 0) dz[i] = __fadd_rn(dz[i], w[m]);
    }
}

// ---- OSEM's multiplicative update (optimization/osem_poisson.py:80-84): x = outside ? 0 : (s > 0 ? x back / (s + lam)
// : x), the support mask periodic with period pm (0: none)
__global__ void osem_update_kernel(float *__restrict__ x, const float *__restrict__ back,
                                   const float *__restrict__ sens, const uint8_t *__restrict__ mask, int64_t pm,
                                   float lam, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const bool ok = pm ? mask[i % pm] != 0 : true;
        const float sv = sens[i];
        x[i] = !ok ? 0.0f : (sv > 0.0f ? __fdiv_rn(__fmul_rn(x[i], back[i]), __fadd_rn(sv, lam)) : x[i]);
    }
}

// ---- PDHG (optimization/pdhg_poisson.py:33-94). Dual: y <- prox_{sig F*}(y + sig Axb), F_i(z) = s (z + r - b log(z +
// r)), s = w / g, r = bg + eps g: y = (v + s - sqrt((v - s)^2 + 4 sig s b)) / 2, v = y + sig Axb + sig r (float64);
// 0 where w = 0 or sig = 0
__global__ void pdhg_dual_kernel(float *__restrict__ y, const float *__restrict__ Axb, const float *__restrict__ sig,
                                 const float *__restrict__ b, const float *__restrict__ w, int64_t pw,
                                 const float *__restrict__ g, int64_t pg, const float *__restrict__ bg, int64_t pbg,
                                 float eps, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float wi = periodic(w, pw, i, 1.0f);
        const float si = sig[i];
        if (wi == 0.0f || si == 0.0f) {
            y[i] = 0.0f;
            continue;
        }
        const float gi = periodic(g, pg, i, 1.0f);
        const double sd = (double)wi / (double)gi;
        const double r = (double)periodic(bg, pbg, i, 0.0f) + (double)eps * gi;
        const double v = (double)y[i] + (double)si * Axb[i] + (double)si * r;
        const double d = v - sd;
        y[i] = (float)(0.5 * (v + sd - sqrt(d * d + 4.0 * (double)si * sd * (double)b[i])));
    }
}

// primal: x_new = T > 0 ? max(0, x - T (grad + lam)) : 0; xb = 2 x_new - x; x = x_new
__global__ void pdhg_primal_kernel(float *__restrict__ x, float *__restrict__ xb, const float *__restrict__ grad,
                                   const float *__restrict__ T, float lam, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float t = T[i];
        const float xo = x[i];
        const float xn = t > 0.0f ? fmaxf(0.0f, __fsub_rn(xo, __fmul_rn(t, __fadd_rn(grad[i], lam)))) : 0.0f;
        xb[i] = __fsub_rn(__fmul_rn(2.0f, xn), xo);
        x[i] = xn;
    }
}

// Ax <- (Axb + Ax) / 2 (A x_k from A x_bar_k = 2 A x_k - A x_(k-1))
__global__ void pdhg_average_kernel(float *__restrict__ Ax, const float *__restrict__ Axb, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        Ax[i] = __fmul_rn(0.5f, __fadd_rn(Axb[i], Ax[i]));
}

// T = tau0 / colsum on the support (mask periodic with period npix, 0: none) where colsum > 0, else 0
__global__ void pdhg_primal_steps_kernel(float *__restrict__ T, const float *__restrict__ colsum,
                                         const uint8_t *__restrict__ supp, int64_t npix, float tau0, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const bool inside = npix ? supp[i % npix] != 0 : true;
        const float c = colsum[i];
        T[i] = (inside && c > 0.0f) ? __fdiv_rn(tau0, c) : 0.0f;
    }
}

// ---- the Poisson data term of a prediction (optimization/poisson_term.py:36-58), mu = max(pred, 0) + bg + eps g, on
// the points of weight != 0 (0 elsewhere; the fitted angles are the caller's weights):
//   mode 0: r = w/g (1 - b/mu), c = w / (g max(mu, floor g))     (gradient and Fisher curvature; c may be NULL)
//   mode 1: r = w/g b/mu                                          (the EM ratio)
//   mode 2: r = w/g                                               (the EM sensitivity's data)
__global__ void poisson_term_kernel(const float *__restrict__ pred, const float *__restrict__ b,
                                    const float *__restrict__ w, int64_t pw, const float *__restrict__ g, int64_t pg,
                                    const float *__restrict__ bg, int64_t pbg, float eps, float floor_counts, int mode,
                                    float *__restrict__ r, float *__restrict__ c, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float wi = periodic(w, pw, i, 1.0f);
        const float gi = periodic(g, pg, i, 1.0f);
        float ri = 0.0f, ci = 0.0f;
        if (wi != 0.0f) {
            const float wg = __fdiv_rn(wi, gi);
            if (mode == 2) {
                ri = wg;
            } else {
                const float mu = __fadd_rn(__fadd_rn(fmaxf(pred[i], 0.0f), periodic(bg, pbg, i, 0.0f)),
                                           __fmul_rn(eps, gi));
                const float q = __fdiv_rn(b[i], mu);
                ri = mode == 1 ? __fmul_rn(wg, q) : __fmul_rn(wg, __fsub_rn(1.0f, q));
                ci = __fdiv_rn(wi, __fmul_rn(gi, fmaxf(mu, __fmul_rn(floor_counts, gi))));
            }
        }
        r[i] = ri;
        if (c) c[i] = ci;
    }
}

// ---- orientation search: z = E / sqrt(max(D, 1e-30)) (NaN kept), 0 where D <= 0, with correctly rounded division
// and square root: the float32 NumPy expression of the reference's host path, bitwise (orientation_search.py:41-54)
__global__ void score_z_kernel(const float *__restrict__ E, const float *__restrict__ D, float *__restrict__ Z,
                               int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float d = D[i];
        const float m = d != d ? d : fmaxf(d, 1e-30f);
        const float z = __fdiv_rn(E[i], __fsqrt_rn(m));
        Z[i] = d <= 0.0f ? 0.0f : z;
    }
}

// ---- SPDHG ----
// The closed-form Poisson conjugate prox of one data point in float64 arithmetic (spdhg_poisson.py:69-91):
// y' = (v + sc - sqrt((v - sc)^2 + 4 s sc b)) / 2, v = y + s (A x) + s (bg + eps g), sc = w / g; 0 where w = 0 or s = 0.
__device__ __forceinline__ float dual_prox(float yo, float ax, float si, float bi, float wi, float gi, float bgi,
                                           float eps)
{
    if (wi == 0.0f || si == 0.0f) return 0.0f;
    const double sc = __ddiv_rn((double)wi, (double)gi);
    const double rr = __dadd_rn((double)bgi, __dmul_rn((double)eps, (double)gi));
    const double v = __dadd_rn(__dadd_rn((double)yo, __dmul_rn((double)si, (double)ax)), __dmul_rn((double)si, rr));
    const double dd = __dsub_rn(v, sc);
    const double disc = __dadd_rn(__dmul_rn(dd, dd), __dmul_rn(__dmul_rn(__dmul_rn(4.0, (double)si), sc), (double)bi));
    return (float)__dmul_rn(0.5, __dsub_rn(__dadd_rn(v, sc), __dsqrt_rn(disc)));
}

__global__ void dual_update_kernel(float *__restrict__ y, float *__restrict__ d, const float *__restrict__ sig,
                                   const float *__restrict__ b, const float *__restrict__ w, int64_t pw,
                                   const float *__restrict__ g, int64_t pg, const float *__restrict__ bg, int64_t pbg,
                                   float eps, const int32_t *__restrict__ omegas, int64_t row)
{
    // blockIdx.y: the subset's angle (one data row of row elements), no division per element
    const int64_t base = (int64_t)__ldg(omegas + blockIdx.y) * row;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < row; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + j;
        const float yo = y[i];
        const float yn = dual_prox(yo, d[i], sig[i], b[i], periodic(w, pw, i, 1.0f), periodic(g, pg, i, 1.0f),
                                   periodic(bg, pbg, i, 0.0f), eps);
        d[i] = yn - yo;
        y[i] = yn;
    }
}

// The same step four points at a time with 16-byte loads and stores (rows of a multiple of 4 points, arrays 16-byte
// aligned): more bytes in flight per thread. PLAIN (no weights, gain or background): w = g = 1, bg = 0 without loads.
template <bool PLAIN>
__global__ void dual_update4_kernel(float4 *__restrict__ y, float4 *__restrict__ d, const float4 *__restrict__ sig,
                                    const float4 *__restrict__ b, const float *__restrict__ w, int64_t pw,
                                    const float *__restrict__ g, int64_t pg, const float *__restrict__ bg, int64_t pbg,
                                    float eps, const int32_t *__restrict__ omegas, int64_t row4)
{
    const int64_t base = (int64_t)__ldg(omegas + blockIdx.y) * row4;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < row4; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = base + j;
        const float4 yo = __ldcs(y + q), ax = d[q], si = __ldcs(sig + q), bi = __ldcs(b + q);
        const float yv[4] = {yo.x, yo.y, yo.z, yo.w}, av[4] = {ax.x, ax.y, ax.z, ax.w};
        const float sv[4] = {si.x, si.y, si.z, si.w}, bv[4] = {bi.x, bi.y, bi.z, bi.w};
        float yn[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t i = 4 * q + u;
            yn[u] = PLAIN ? dual_prox(yv[u], av[u], sv[u], bv[u], 1.0f, 1.0f, 0.0f, eps)
                          : dual_prox(yv[u], av[u], sv[u], bv[u], periodic(w, pw, i, 1.0f), periodic(g, pg, i, 1.0f),
                                      periodic(bg, pbg, i, 0.0f), eps);
        }
        d[q] = make_float4(yn[0] - yv[0], yn[1] - yv[1], yn[2] - yv[2], yn[3] - yv[3]);   // read next: kept in L2
        __stcs(y + q, make_float4(yn[0], yn[1], yn[2], yn[3]));
    }
}

// The same step with T held in BF16 (widened exactly): the step sizes of a run whose x, z and T do not all fit in
// float32 (T rounded toward zero when stored, so never above its float32 value).
__global__ void primal_update_t16_kernel(float *__restrict__ x, float *__restrict__ z,
                                         const __nv_bfloat16 *__restrict__ T, const float *__restrict__ dz, float inv_p,
                                         float lam, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float di = dz[i];
        const float zi = __fadd_rn(z[i], di);
        z[i] = zi;
        const float zb = __fadd_rn(zi, __fmul_rn(inv_p, di));
        const float t = __bfloat162float(T[i]);
        x[i] = t > 0.0f ? fmaxf(0.0f, __fsub_rn(x[i], __fmul_rn(t, __fadd_rn(zb, lam)))) : 0.0f;
    }
}

__global__ void f32_to_bf16_rz_kernel(const float *__restrict__ in, __nv_bfloat16 *__restrict__ out, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = __float2bfloat16_rz(in[i]);
}

__global__ void primal_update_kernel(float *__restrict__ x, float *__restrict__ z, const float *__restrict__ T,
                                     const float *__restrict__ dz, float inv_p, float lam, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float di = dz[i];
        const float zi = __fadd_rn(z[i], di);
        z[i] = zi;
        const float zb = __fadd_rn(zi, __fmul_rn(inv_p, di));
        const float t = T[i];
        x[i] = t > 0.0f ? fmaxf(0.0f, __fsub_rn(x[i], __fmul_rn(t, __fadd_rn(zb, lam)))) : 0.0f;
    }
}

__global__ void dual_steps_kernel(float *__restrict__ sig, const float *__restrict__ rowsum,
                                  const float *__restrict__ w, int64_t pw, float sigma0, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float rs = rowsum[i];
        sig[i] = (periodic(w, pw, i, 1.0f) != 0.0f && rs > 0.0f) ? __fdiv_rn(sigma0, rs) : 0.0f;
    }
}

__global__ void set_mask_ones_kernel(float *__restrict__ u, const float *__restrict__ w, int64_t pw, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        u[i] = periodic(w, pw, i, 1.0f) != 0.0f ? 1.0f : 0.0f;
}

__global__ void fill_kernel(float *__restrict__ x, float value, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = value;
}

__global__ void tinit_kernel(float *__restrict__ T, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        T[i] = __int_as_float(0x7f800000);
}

__global__ void tmin_kernel(float *__restrict__ T, const float *__restrict__ colsum, const uint8_t *__restrict__ supp,
                            int64_t npix, float c, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const bool inside = supp ? __ldg(supp + (i % npix)) != 0 : true;
        const float cs = colsum[i];
        if (inside && cs > 0.0f) T[i] = fminf(T[i], __fdiv_rn(c, cs));
    }
}

__global__ void tfinal_kernel(float *__restrict__ T, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (isinf(T[i])) T[i] = 0.0f;
}

__global__ void support_ones_kernel(float *__restrict__ x, const uint8_t *__restrict__ supp, int64_t npix, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = (supp ? __ldg(supp + (i % npix)) != 0 : true) ? 1.0f : 0.0f;
}

__global__ void project_support_kernel(float *__restrict__ x, const uint8_t *__restrict__ supp, int64_t npix,
                                       int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if ((supp && __ldg(supp + (i % npix)) == 0) || x[i] < 0.0f) x[i] = 0.0f;
}

// ---- reductions ----
__global__ void __launch_bounds__(RED_THREADS) poisson_value_grad_kernel(
    float *__restrict__ mu, const float *__restrict__ b, const float *__restrict__ w, int64_t pw,
    const float *__restrict__ g, int64_t pg, const float *__restrict__ bg, int64_t pbg, float eps, int write_grad,
    int mode, float floor_counts, int64_t n, double *__restrict__ part)
{
    double v[1] = {0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float wi = periodic(w, pw, i, 1.0f);
        float gr = 0.0f;
        if (wi != 0.0f) {
            const float gi = periodic(g, pg, i, 1.0f);
            const double bi = (double)b[i];
            const double sc = (double)wi / (double)gi;
            if (mode == 0) {
                const double m = (double)fmaxf(mu[i], 0.0f) + (double)periodic(bg, pbg, i, 0.0f) + (double)eps * gi;
                double val = m - bi;
                if (bi > 0.0) val += bi * log(bi / m);
                v[0] += sc * val;
                gr = (float)(sc * (1.0 - bi / m));
            } else {
                const double r = (double)mu[i] + (double)periodic(bg, pbg, i, 0.0f) - bi;
                const double c = sc / fmax(bi, (double)floor_counts * gi);
                v[0] += 0.5 * c * r * r;
                gr = (float)(c * r);
            }
        }
        if (write_grad) mu[i] = gr;
    }
    block_sum<1>(v, part + blockIdx.x);
}

__global__ void __launch_bounds__(RED_THREADS) mean_counted_kernel(const float *__restrict__ b,
                                                                   const float *__restrict__ w, int64_t pw, int64_t n,
                                                                   double *__restrict__ part)
{
    double v[2] = {0.0, 0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (periodic(w, pw, i, 1.0f) != 0.0f) {
            v[0] += (double)b[i];
            v[1] += 1.0;
        }
    block_sum<2>(v, part + 2 * blockIdx.x);
}

__global__ void __launch_bounds__(RED_THREADS) dot_kernel(const float *__restrict__ x, const float *__restrict__ y,
                                                          int64_t n, double *__restrict__ part)
{
    double v[1] = {0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[0] += y ? (double)x[i] * (double)y[i] : (double)x[i];
    block_sum<1>(v, part + blockIdx.x);
}

// ---- FISTAPoisson (fista_poisson.py:115-282) ----
__global__ void __launch_bounds__(RED_THREADS) times_curvature_kernel(
    float *__restrict__ u, const float *__restrict__ mu, const float *__restrict__ b, const float *__restrict__ w,
    int64_t pw, const float *__restrict__ g, int64_t pg, const float *__restrict__ bg, int64_t pbg, float floor_counts,
    int mode, int64_t n, double *__restrict__ part)
{
    double v[1] = {0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float wi = periodic(w, pw, i, 1.0f);
        const float gi = periodic(g, pg, i, 1.0f);
        const float r = u[i];
        float c;
        if (mode == 0) {
            const float m = fmaxf(__fadd_rn(fmaxf(mu[i], 0.0f), periodic(bg, pbg, i, 0.0f)), __fmul_rn(floor_counts, gi));
            c = wi != 0.0f ? __fmul_rn(__fdiv_rn(wi, gi), __fdiv_rn(fmaxf(b[i], m), __fmul_rn(m, m))) : 0.0f;
        } else {
            c = wi != 0.0f ? __fdiv_rn(wi, __fmul_rn(gi, fmaxf(b[i], __fmul_rn(floor_counts, gi)))) : 0.0f;
        }
        u[i] = __fmul_rn(r, c);
        v[0] += (double)c * (double)r * (double)r;
    }
    block_sum<1>(v, part + blockIdx.x);
}

__global__ void __launch_bounds__(RED_THREADS) support_sum_kernel(const float *__restrict__ x,
                                                                  const uint8_t *__restrict__ supp, int64_t npix,
                                                                  int64_t n, double *__restrict__ part)
{
    double v[1] = {0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (!supp || __ldg(supp + (i % npix))) v[0] += (double)x[i];
    block_sum<1>(v, part + blockIdx.x);
}

__global__ void __launch_bounds__(RED_THREADS) weighted_sums_kernel(const float *__restrict__ mu,
                                                                    const float *__restrict__ b,
                                                                    const float *__restrict__ w, int64_t pw, int64_t n,
                                                                    double *__restrict__ part)
{
    double v[2] = {0.0, 0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float wi = periodic(w, pw, i, 1.0f);
        v[0] += (double)wi * b[i];
        v[1] += (double)wi * mu[i];
    }
    block_sum<2>(v, part + 2 * blockIdx.x);
}

__global__ void invert_metric_kernel(float *__restrict__ D, const float *__restrict__ d,
                                     const uint8_t *__restrict__ supp, int64_t npix, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const bool inside = supp ? __ldg(supp + (i % npix)) != 0 : true;
        const float di = d[i];
        D[i] = (inside && di > 0.0f) ? __frcp_rn(di) : 0.0f;
    }
}

__global__ void metric_step_kernel(float *__restrict__ xn, const float *__restrict__ y,
                                   const float *__restrict__ grad, const float *__restrict__ D, float th, float lam,
                                   int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float Di = D[i];
        xn[i] = Di > 0.0f ? fmaxf(0.0f, __fsub_rn(y[i], __fmul_rn(__fmul_rn(th, Di), __fadd_rn(grad[i], lam)))) : 0.0f;
    }
}

__global__ void __launch_bounds__(RED_THREADS) step_sums_kernel(const float *__restrict__ xn,
                                                                const float *__restrict__ y,
                                                                const float *__restrict__ grad,
                                                                const float *__restrict__ D, int64_t n,
                                                                double *__restrict__ part)
{
    double v[3] = {0.0, 0.0, 0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double d = (double)xn[i] - (double)y[i];
        v[0] += (double)grad[i] * d;
        const float Di = D[i];
        if (Di > 0.0f) v[1] += d * d / (double)Di;
        v[2] += (double)xn[i];
    }
    block_sum<3>(v, part + 3 * blockIdx.x);
}

__global__ void extrapolate_kernel(float *__restrict__ out, const float *__restrict__ a, const float *__restrict__ c,
                                   float beta, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float ai = a[i];
        out[i] = __fadd_rn(ai, __fmul_rn(beta, __fsub_rn(ai, c[i])));
    }
}

__global__ void copy_kernel(const float *__restrict__ src, float *__restrict__ dst, int64_t n)
{
    // float4 body (both arrays 16-byte aligned, checked by the caller) and a scalar tail
    const int64_t n4 = n / 4;
    const float4 *s4 = reinterpret_cast<const float4 *>(src);
    float4 *d4 = reinterpret_cast<float4 *>(dst);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x)
        d4[i] = s4[i];
    for (int64_t i = 4 * n4 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

__global__ void scale_kernel(float *__restrict__ x, float a, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = __fmul_rn(x[i], a);
}

static int check_scratch(void *scratch, size_t bytes, int64_t n, int ns)
{
    const size_t need = (size_t)red_blocks(n) * ns * sizeof(double);
    if (!scratch || bytes < need) {
        set_error("reduction: scratch of %zu bytes, %zu needed", bytes, need);
        return DFX_ENOMEM;
    }
    return DFX_OK;
}

}  // namespace dfx

using namespace dfx;

#define EW_LAUNCH(kernel, n, stream, ...)                                                                   \
    do {                                                                                                    \
        kernel<<<ew_grid(n), EW_THREADS, 0, (cudaStream_t)(stream)>>>(__VA_ARGS__);                         \
        return launch_status(#kernel);                                                                      \
    } while (0)

extern "C" int dfx_tv_dual(const float *x, const float *T, float *qx, float *qy, float *dqx, float *dqy, int nx,
                           int ny, int kstride, float lam, float ps, void *stream)
{
    DFX_REQUIRE(x && T && qx && qy && dqx && dqy && nx > 0 && ny > 0 && kstride > 0, "tv_dual: bad arguments");
    const int64_t n = (int64_t)nx * ny * kstride;
    EW_LAUNCH(tv_dual_kernel, n, stream, x, T, qx, qy, dqx, dqy, nx, ny, kstride, lam, ps, n);
}

extern "C" int dfx_tv_adjoint_update(const float *dqx, const float *dqy, float *x, float *z, const float *T, int nx,
                                     int ny, int kstride, float inv_p, float lam, void *stream)
{
    DFX_REQUIRE(dqx && dqy && x && z && T && nx > 0 && ny > 0 && kstride > 0, "tv_adjoint_update: bad arguments");
    const int64_t n = (int64_t)nx * ny * kstride;
    EW_LAUNCH(tv_adjoint_update_kernel, n, stream, dqx, dqy, x, z, T, nx, kstride, inv_p, lam, n);
}

extern "C" int dfx_tv_value(const float *x, const float *T, int nx, int ny, int kstride, double *out, void *scratch,
                            size_t scratch_bytes, void *stream)
{
    DFX_REQUIRE(x && T && out && nx > 0 && ny > 0 && kstride > 0, "tv_value: bad arguments");
    const int64_t n = (int64_t)nx * ny * kstride;
    int st = check_scratch(scratch, scratch_bytes, n, 1);
    if (st) return st;
    const int nb = red_blocks(n);
    cudaStream_t s = (cudaStream_t)stream;
    tv_value_kernel<<<nb, RED_THREADS, 0, s>>>(x, T, nx, ny, kstride, n, (double *)scratch);
    st = launch_status("tv_value");
    if (st) return st;
    finish_sums<1><<<1, RED_THREADS, 0, s>>>((const double *)scratch, nb, out);
    return launch_status("finish_sums");
}

extern "C" int dfx_tv_dual_local(const float *x, const float *T, float *qx, float *qy, float *dqx, float *dqy,
                                 const int32_t *right, const int32_t *down, float lam, float ps, int64_t n,
                                 void *stream)
{
    DFX_REQUIRE(x && T && qx && qy && dqx && dqy && right && down && n >= 0, "tv_dual_local: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(tv_dual_local_kernel, n, stream, x, T, qx, qy, dqx, dqy, right, down, lam, ps, n);
}

extern "C" int dfx_tv_adjoint_update_local(const float *dqx, const float *dqy, float *x, float *z, const float *T,
                                           const int32_t *left, const int32_t *up, float inv_p, float lam, int64_t n,
                                           void *stream)
{
    DFX_REQUIRE(dqx && dqy && x && z && T && left && up && n >= 0, "tv_adjoint_update_local: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(tv_adjoint_update_local_kernel, n, stream, dqx, dqy, x, z, T, left, up, inv_p, lam, n);
}

extern "C" int dfx_tv_adjoint_local(const float *dqx, const float *dqy, float *w, const int32_t *left,
                                    const int32_t *up, int64_t n, void *stream)
{
    DFX_REQUIRE(dqx && dqy && w && left && up && n >= 0, "tv_adjoint_local: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(tv_adjoint_local_kernel, n, stream, dqx, dqy, w, left, up, n);
}

extern "C" int dfx_tree_sums(const float *x, const int32_t *ptr, const int32_t *idx, float *s, int64_t n,
                             void *stream)
{
    DFX_REQUIRE(x && ptr && idx && s && n >= 0, "tree_sums: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(tree_sums_kernel, n, stream, x, ptr, idx, s, n);
}

extern "C" int dfx_tree_scatter(const float *w, const int32_t *map, float *dz, int64_t n, void *stream)
{
    DFX_REQUIRE(w && map && dz && n >= 0, "tree_scatter: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(tree_scatter_kernel, n, stream, w, map, dz, n);
}

extern "C" int dfx_tv_value_local(const float *x, const float *T, const int32_t *right, const int32_t *down,
                                  int64_t n, double *out, void *scratch, size_t scratch_bytes, void *stream)
{
    DFX_REQUIRE(x && T && right && down && out && n > 0, "tv_value_local: bad arguments");
    int st = check_scratch(scratch, scratch_bytes, n, 1);
    if (st) return st;
    const int nb = red_blocks(n);
    cudaStream_t s = (cudaStream_t)stream;
    tv_value_local_kernel<<<nb, RED_THREADS, 0, s>>>(x, T, right, down, n, (double *)scratch);
    st = launch_status("tv_value_local");
    if (st) return st;
    finish_sums<1><<<1, RED_THREADS, 0, s>>>((const double *)scratch, nb, out);
    return launch_status("finish_sums");
}

extern "C" int dfx_osem_update(float *x, const float *back, const float *sens, const uint8_t *mask, int64_t pm,
                               float lam, int64_t n, void *stream)
{
    DFX_REQUIRE(x && back && sens && n >= 0 && (!pm || mask), "osem_update: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(osem_update_kernel, n, stream, x, back, sens, mask, pm, lam, n);
}

extern "C" int dfx_pdhg_dual_update(float *y, const float *Axb, const float *sig, const float *b, const float *w,
                                    int64_t pw, const float *g, int64_t pg, const float *bg, int64_t pbg, float eps,
                                    int64_t n, void *stream)
{
    DFX_REQUIRE(y && Axb && sig && b && n >= 0 && (!pw || w) && (!pg || g) && (!pbg || bg),
                "pdhg_dual_update: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(pdhg_dual_kernel, n, stream, y, Axb, sig, b, w, pw, g, pg, bg, pbg, eps, n);
}

extern "C" int dfx_pdhg_primal_update(float *x, float *xb, const float *grad, const float *T, float lam, int64_t n,
                                      void *stream)
{
    DFX_REQUIRE(x && xb && grad && T && n >= 0, "pdhg_primal_update: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(pdhg_primal_kernel, n, stream, x, xb, grad, T, lam, n);
}

extern "C" int dfx_pdhg_average(float *Ax, const float *Axb, int64_t n, void *stream)
{
    DFX_REQUIRE(Ax && Axb && n >= 0, "pdhg_average: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(pdhg_average_kernel, n, stream, Ax, Axb, n);
}

extern "C" int dfx_pdhg_primal_steps(float *T, const float *colsum, const uint8_t *supp, int64_t npix, float tau0,
                                     int64_t n, void *stream)
{
    DFX_REQUIRE(T && colsum && n >= 0 && (!npix || supp), "pdhg_primal_steps: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(pdhg_primal_steps_kernel, n, stream, T, colsum, supp, npix, tau0, n);
}

extern "C" int dfx_poisson_term(const float *pred, const float *b, const float *w, int64_t pw, const float *g, int64_t pg,
                                const float *bg, int64_t pbg, float eps, float floor_counts, int mode, float *r,
                                float *c, int64_t n, void *stream)
{
    DFX_REQUIRE(b && r && n >= 0 && (mode == 2 || pred) && mode >= 0 && mode <= 2 && (!pw || w) && (!pg || g) &&
                    (!pbg || bg),
                "poisson_term: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(poisson_term_kernel, n, stream, pred, b, w, pw, g, pg, bg, pbg, eps, floor_counts, mode, r, c, n);
}

extern "C" int dfx_spdhg_dual_update(float *y, float *d, const float *sig, const float *b, const float *w, int64_t pw,
                                     const float *g, int64_t pg, const float *bg, int64_t pbg, float eps,
                                     const int32_t *omegas, int n_sub, int64_t row_len, void *stream)
{
    DFX_REQUIRE(y && d && sig && b && omegas && n_sub >= 0 && row_len > 0, "dual_update: bad arguments");
    DFX_REQUIRE((!pw || w) && (!pg || g) && (!pbg || bg), "dual_update: periodic array missing");
    DFX_REQUIRE(n_sub <= 65535, "dual_update: at most 65535 angles per call");
    if (n_sub == 0) return DFX_OK;
    const bool vec4 = row_len % 4 == 0 && (((uintptr_t)y | (uintptr_t)d | (uintptr_t)sig | (uintptr_t)b) % 16) == 0;
    if (vec4) {
        const int64_t row4 = row_len / 4;
        const dim3 grid((unsigned)std::min<int64_t>(cdiv(row4, (int64_t)EW_THREADS), 65535), (unsigned)n_sub);
        auto *y4 = reinterpret_cast<float4 *>(y), *d4 = reinterpret_cast<float4 *>(d);
        auto *s4 = reinterpret_cast<const float4 *>(sig), *b4 = reinterpret_cast<const float4 *>(b);
        if (pw == 0 && pg == 0 && pbg == 0)
            dual_update4_kernel<true><<<grid, EW_THREADS, 0, (cudaStream_t)stream>>>(y4, d4, s4, b4, w, pw, g, pg,
                                                                                    bg, pbg, eps, omegas, row4);
        else
            dual_update4_kernel<false><<<grid, EW_THREADS, 0, (cudaStream_t)stream>>>(y4, d4, s4, b4, w, pw, g, pg,
                                                                                     bg, pbg, eps, omegas, row4);
        return launch_status("dual_update4_kernel");
    }
    const dim3 grid((unsigned)std::min<int64_t>(cdiv(row_len, (int64_t)EW_THREADS * 4), 65535), (unsigned)n_sub);
    dual_update_kernel<<<grid, EW_THREADS, 0, (cudaStream_t)stream>>>(y, d, sig, b, w, pw, g, pg, bg, pbg, eps,
                                                                      omegas, row_len);
    return launch_status("dual_update_kernel");
}

extern "C" int dfx_spdhg_primal_update(float *x, float *z, const float *T, const float *dz, float inv_p, float lam,
                                       int64_t n, void *stream)
{
    DFX_REQUIRE(x && z && T && dz && n >= 0, "primal_update: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(primal_update_kernel, n, stream, x, z, T, dz, inv_p, lam, n);
}

extern "C" int dfx_spdhg_primal_update_t16(float *x, float *z, const void *T_bf16, const float *dz, float inv_p,
                                           float lam, int64_t n, void *stream)
{
    DFX_REQUIRE(x && z && T_bf16 && dz && n >= 0, "primal_update_t16: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(primal_update_t16_kernel, n, stream, x, z, reinterpret_cast<const __nv_bfloat16 *>(T_bf16), dz, inv_p,
              lam, n);
}

extern "C" int dfx_f32_to_bf16_rz(const float *in, void *out, int64_t n, void *stream)
{
    DFX_REQUIRE(in && out && n >= 0, "f32_to_bf16_rz: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(f32_to_bf16_rz_kernel, n, stream, in, reinterpret_cast<__nv_bfloat16 *>(out), n);
}

extern "C" int dfx_dual_steps(float *sig, const float *rowsum, const float *w, int64_t pw, float sigma0, int64_t n,
                              void *stream)
{
    DFX_REQUIRE(sig && rowsum && (!pw || w) && n >= 0, "dual_steps: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(dual_steps_kernel, n, stream, sig, rowsum, w, pw, sigma0, n);
}

extern "C" int dfx_set_mask_ones(float *u, const float *w, int64_t pw, int64_t n, void *stream)
{
    DFX_REQUIRE(u && (!pw || w) && n >= 0, "set_mask_ones: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(set_mask_ones_kernel, n, stream, u, w, pw, n);
}

extern "C" int dfx_fill_f32(float *x, float value, int64_t n, void *stream)
{
    DFX_REQUIRE(x && n >= 0, "fill: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(fill_kernel, n, stream, x, value, n);
}

extern "C" int dfx_tinit(float *T, int64_t n, void *stream)
{
    DFX_REQUIRE(T && n >= 0, "tinit: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(tinit_kernel, n, stream, T, n);
}

extern "C" int dfx_tmin(float *T, const float *colsum, const uint8_t *supp, int64_t npix, float c, int64_t n,
                        void *stream)
{
    DFX_REQUIRE(T && colsum && n >= 0 && (!supp || npix > 0), "tmin: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(tmin_kernel, n, stream, T, colsum, supp, npix, c, n);
}

extern "C" int dfx_tfinal(float *T, int64_t n, void *stream)
{
    DFX_REQUIRE(T && n >= 0, "tfinal: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(tfinal_kernel, n, stream, T, n);
}

extern "C" int dfx_support_ones(float *x, const uint8_t *supp, int64_t npix, int64_t n, void *stream)
{
    DFX_REQUIRE(x && n >= 0 && (!supp || npix > 0), "support_ones: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(support_ones_kernel, n, stream, x, supp, npix, n);
}

extern "C" int dfx_project_support(float *x, const uint8_t *supp, int64_t npix, int64_t n, void *stream)
{
    DFX_REQUIRE(x && n >= 0 && (!supp || npix > 0), "project_support: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(project_support_kernel, n, stream, x, supp, npix, n);
}

extern "C" size_t dfx_reduce_scratch_bytes(int64_t n) { return (size_t)red_blocks(n) * 4 * sizeof(double); }

extern "C" int dfx_poisson_value_grad(float *mu, const float *b, const float *w, int64_t pw, const float *g,
                                      int64_t pg, const float *bg, int64_t pbg, float eps, int write_grad, int mode,
                                      float floor_counts, int64_t n, double *out, void *scratch, size_t scratch_bytes,
                                      void *stream)
{
    DFX_REQUIRE(mu && b && out && n >= 0 && (!pw || w) && (!pg || g) && (!pbg || bg), "poisson_value_grad: bad args");
    int st = check_scratch(scratch, scratch_bytes, n, 1);
    if (st) return st;
    const int nb = red_blocks(n);
    cudaStream_t s = (cudaStream_t)stream;
    double *part = (double *)scratch;
    poisson_value_grad_kernel<<<nb, RED_THREADS, 0, s>>>(mu, b, w, pw, g, pg, bg, pbg, eps, write_grad, mode,
                                                         floor_counts, n, part);
    st = launch_status("poisson_value_grad");
    if (st) return st;
    finish_sums<1><<<1, RED_THREADS, 0, s>>>(part, nb, out);
    return launch_status("finish_sums");
}

extern "C" int dfx_mean_counted(const float *b, const float *w, int64_t pw, int64_t n, double *out, void *scratch,
                                size_t scratch_bytes, void *stream)
{
    DFX_REQUIRE(b && out && n >= 0 && (!pw || w), "mean_counted: bad arguments");
    int st = check_scratch(scratch, scratch_bytes, n, 2);
    if (st) return st;
    const int nb = red_blocks(n);
    cudaStream_t s = (cudaStream_t)stream;
    mean_counted_kernel<<<nb, RED_THREADS, 0, s>>>(b, w, pw, n, (double *)scratch);
    st = launch_status("mean_counted");
    if (st) return st;
    finish_sums<2><<<1, RED_THREADS, 0, s>>>((const double *)scratch, nb, out);
    return launch_status("finish_sums");
}

extern "C" int dfx_dot_f64(const float *x, const float *y, int64_t n, double *out, void *scratch, size_t scratch_bytes,
                           void *stream)
{
    DFX_REQUIRE(x && out && n >= 0, "dot: bad arguments");
    int st = check_scratch(scratch, scratch_bytes, n, 1);
    if (st) return st;
    const int nb = red_blocks(n);
    cudaStream_t s = (cudaStream_t)stream;
    dot_kernel<<<nb, RED_THREADS, 0, s>>>(x, y, n, (double *)scratch);
    st = launch_status("dot");
    if (st) return st;
    finish_sums<1><<<1, RED_THREADS, 0, s>>>((const double *)scratch, nb, out);
    return launch_status("finish_sums");
}

// ---- FISTAPoisson entry points ----
template <int NS, typename Launch>
static int reduce_launch(int64_t n, void *scratch, size_t bytes, double *out, void *stream, const char *what,
                         Launch launch)
{
    int st = check_scratch(scratch, bytes, n, NS);
    if (st) return st;
    const int nb = red_blocks(n);
    cudaStream_t s = (cudaStream_t)stream;
    launch(nb, s, (double *)scratch);
    st = launch_status(what);
    if (st) return st;
    finish_sums<NS><<<1, RED_THREADS, 0, s>>>((const double *)scratch, nb, out);
    return launch_status("finish_sums");
}

extern "C" int dfx_times_curvature(float *u, const float *mu, const float *b, const float *w, int64_t pw,
                                   const float *g, int64_t pg, const float *bg, int64_t pbg, float floor_counts,
                                   int mode, int64_t n, double *out, void *scratch, size_t scratch_bytes, void *stream)
{
    DFX_REQUIRE(u && mu && b && out && n >= 0 && (!pw || w) && (!pg || g) && (!pbg || bg), "times_curvature: bad args");
    return reduce_launch<1>(n, scratch, scratch_bytes, out, stream, "times_curvature",
                            [&](int nb, cudaStream_t s, double *part) {
                                times_curvature_kernel<<<nb, RED_THREADS, 0, s>>>(u, mu, b, w, pw, g, pg, bg, pbg,
                                                                                  floor_counts, mode, n, part);
                            });
}

extern "C" int dfx_support_sum(const float *x, const uint8_t *supp, int64_t npix, int64_t n, double *out,
                               void *scratch, size_t scratch_bytes, void *stream)
{
    DFX_REQUIRE(x && out && n >= 0 && (!supp || npix > 0), "support_sum: bad arguments");
    return reduce_launch<1>(n, scratch, scratch_bytes, out, stream, "support_sum",
                            [&](int nb, cudaStream_t s, double *part) {
                                support_sum_kernel<<<nb, RED_THREADS, 0, s>>>(x, supp, npix, n, part);
                            });
}

extern "C" int dfx_weighted_sums(const float *mu, const float *b, const float *w, int64_t pw, int64_t n, double *out,
                                 void *scratch, size_t scratch_bytes, void *stream)
{
    DFX_REQUIRE(mu && b && out && n >= 0 && (!pw || w), "weighted_sums: bad arguments");
    return reduce_launch<2>(n, scratch, scratch_bytes, out, stream, "weighted_sums",
                            [&](int nb, cudaStream_t s, double *part) {
                                weighted_sums_kernel<<<nb, RED_THREADS, 0, s>>>(mu, b, w, pw, n, part);
                            });
}

extern "C" int dfx_step_sums(const float *xn, const float *y, const float *grad, const float *D, int64_t n,
                             double *out, void *scratch, size_t scratch_bytes, void *stream)
{
    DFX_REQUIRE(xn && y && grad && D && out && n >= 0, "step_sums: bad arguments");
    return reduce_launch<3>(n, scratch, scratch_bytes, out, stream, "step_sums",
                            [&](int nb, cudaStream_t s, double *part) {
                                step_sums_kernel<<<nb, RED_THREADS, 0, s>>>(xn, y, grad, D, n, part);
                            });
}

extern "C" int dfx_invert_metric(float *D, const float *d, const uint8_t *supp, int64_t npix, int64_t n, void *stream)
{
    DFX_REQUIRE(D && d && n >= 0 && (!supp || npix > 0), "invert_metric: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(invert_metric_kernel, n, stream, D, d, supp, npix, n);
}

extern "C" int dfx_metric_step(float *xn, const float *y, const float *grad, const float *D, float th, float lam,
                               int64_t n, void *stream)
{
    DFX_REQUIRE(xn && y && grad && D && n >= 0, "metric_step: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(metric_step_kernel, n, stream, xn, y, grad, D, th, lam, n);
}

extern "C" int dfx_extrapolate(float *out, const float *a, const float *c, float beta, int64_t n, void *stream)
{
    DFX_REQUIRE(out && a && c && n >= 0, "extrapolate: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(extrapolate_kernel, n, stream, out, a, c, beta, n);
}

extern "C" int dfx_copy_f32(const float *src, float *dst, int64_t n, void *stream)
{
    DFX_REQUIRE(src && dst && n >= 0, "copy: bad arguments");
    DFX_REQUIRE(((uintptr_t)src % 16) == 0 && ((uintptr_t)dst % 16) == 0, "copy: 16-byte aligned arrays");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(copy_kernel, cdiv(n, 4), stream, src, dst, n);
}

extern "C" int dfx_scale_f32(float *x, float a, int64_t n, void *stream)
{
    DFX_REQUIRE(x && n >= 0, "scale: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(scale_kernel, n, stream, x, a, n);
}


// ---- FISTAL2 / FISTAHuber entry points ----
extern "C" int dfx_ls_residual(float *ax, const float *b, const float *w, int64_t pw, int clip, float delta,
                               int64_t n, double *out, void *scratch, size_t scratch_bytes, void *stream)
{
    DFX_REQUIRE(ax && b && out && n >= 0 && (!pw || w) && pw >= 0, "ls_residual: bad arguments");
    DFX_REQUIRE(!clip || delta >= 0.0f, "ls_residual: the Huber delta must be >= 0");
    return reduce_launch<1>(n, scratch, scratch_bytes, out, stream, "ls_residual", [&](int nb, cudaStream_t s,
                                                                                         double *part) {
        ls_residual_kernel<<<nb, RED_THREADS, 0, s>>>(ax, b, w, pw, clip, delta, n, part);
    });
}

extern "C" int dfx_fista_ls_blocks(void) { return FU_BLOCKS; }

extern "C" int dfx_fista_ls_update(const float *g, float *x, float *y, const uint8_t *supp, int64_t npix, int kstride,
                                   int kb, float tau, float beta, float lt, int prox, double *part, void *stream)
{
    DFX_REQUIRE(g && x && y && part && npix > 0, "fista_ls_update: bad arguments");
    DFX_REQUIRE(kstride > 0 && kstride % 4 == 0 && kb >= 0 && kb <= kstride,
                "fista_ls_update: kstride (%d) must be a positive multiple of 4 and kb (%d) <= kstride", kstride, kb);
    DFX_REQUIRE(prox >= 0 && prox <= 2, "fista_ls_update: prox must be 0 (nonneg), 1 (l1) or 2 (nonneg_l1)");
    DFX_REQUIRE(((uintptr_t)g % 16) == 0 && ((uintptr_t)x % 16) == 0 && ((uintptr_t)y % 16) == 0,
                "fista_ls_update: arrays must be 16-byte aligned");
    fista_ls_update_kernel<<<FU_BLOCKS, RED_THREADS, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const float4 *>(g), reinterpret_cast<float4 *>(x), reinterpret_cast<float4 *>(y), supp,
        npix, kstride / 4, kb, tau, beta, lt, prox, part);
    return launch_status("fista_ls_update");
}

extern "C" int dfx_sum_partials(const double *part, int n_part, int n_sums, double *out, void *stream)
{
    DFX_REQUIRE(part && out && n_part > 0 && n_sums >= 1 && n_sums <= 3, "sum_partials: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    if (n_sums == 1)
        finish_sums<1><<<1, RED_THREADS, 0, s>>>(part, n_part, out);
    else if (n_sums == 2)
        finish_sums<2><<<1, RED_THREADS, 0, s>>>(part, n_part, out);
    else
        finish_sums<3><<<1, RED_THREADS, 0, s>>>(part, n_part, out);
    return launch_status("finish_sums");
}

extern "C" int dfx_score_z(const float *E, const float *D, float *Z, int64_t n, void *stream)
{
    DFX_REQUIRE(E && D && Z && n >= 0, "score_z: bad arguments");
    if (n == 0) return DFX_OK;
    EW_LAUNCH(score_z_kernel, n, stream, E, D, Z, n);
}
