// Vector-Jacobian products of the forward model with respect to its PF and projector parameters (diffractom's
// differentiable/gradients.py with pf_grad.cl and proj_grad.cl; model of differentiable/reference.py).
//
// PF parameters. For every non-zero (r, k, j) of a batch's adjoint CSR (rows r * kb + k listing segments
// j = c P + p), with S the batch's projections (R, My, kstride) and res = dL/d data:
//     G  = sum_y res[r, y, j] S[r, y, k],      Hs = sum_y curv[r, y, j] S[r, y, k]^2   (hess only)
// times the derivative of the entry PF[r, k, j] = f sum_nodes w sum_{axes h of ring p} m_h g(n_kh . v; sigma_k),
// g(d) = exp(-(1 - |d|) / sigma^2) + exp(-(1 + |d|) / sigma^2), each term cut at the operator's cut, f = N(sigma_k) I_p:
//     d/d rot_k   = f sum w m g'(d) (n x v)          (left increment U_k <- exp([rot]x) U_k)
//     d/d sigma_k = f sum w m (-2/sigma g - 2/sigma^3 dg/ds),  s = 1 / sigma^2
//     d/d eta, tilt_1, tilt_2, 2theta_p = f sum w m g'(d) (n . dv)   (dv: the probed directions' derivatives)
// summed per row (the quantities of a row, NQ values: rot 3, sigma 1, [the upper triangle of q q^T Hs, 10], eta 1,
// tilt 2, two-theta P), then per orientation over the angles in fixed order. The entries are float32 (as the
// operator's PF); their sums are float64: the global parameters' gradients are sums over every (angle, orientation,
// segment) whose terms cancel to 1e-3 of their absolute sum, beyond a float32 accumulator.
//
// Projector parameters: dS = the forward projection through the derivative ray table (K' weights), and per angle
// sum_{y, k < kb} Z[r, y, k] dS[r, y, k] with Z = PF^T res.
#include "dfx_common.cuh"

namespace dfx {
namespace {

constexpr int PG_THREADS = 64;
constexpr int PG_PMAX = 16;          // rings (two-theta accumulators per thread)

template <int HESS>
struct PGLayout {
    static constexpr int NH = HESS ? 10 : 0;
    static constexpr int Q_ETA = 4 + NH;
    static constexpr int Q_TILT = Q_ETA + 1;
    static constexpr int Q_TTH = Q_TILT + 2;
};

__device__ __forceinline__ float dot3(const float *a, float x, float y, float z)
{
    return fmaf(a[0], x, fmaf(a[1], y, a[2] * z));
}

template <int HESS>
__global__ void __launch_bounds__(PG_THREADS) pf_param_vjp_kernel(
    dfx_pf_geometry g, const int32_t *__restrict__ row_ptr, const uint16_t *__restrict__ col_j,
    const float *__restrict__ res, const float *__restrict__ curv, const float *__restrict__ sino, int my,
    int kstride, int k0, int kb, int flags, const float *__restrict__ dv_eta, const float *__restrict__ dv_t1,
    const float *__restrict__ dv_t2, const float *__restrict__ dv_tth, const float *__restrict__ dw_t1,
    const float *__restrict__ dw_t2, double *__restrict__ rows, int nq)
{
    using L = PGLayout<HESS>;
    extern __shared__ float lS[];                         // my floats, then the warps' partial sums
    const int row = blockIdx.x;
    const int r = row / kb, k = row - r * kb, kg = k0 + k;
    const int P = g.P, C = g.C, A = g.A, S = g.S, Se = g.S_eta, CP = C * P;
    for (int y = threadIdx.x; y < my; y += PG_THREADS) lS[y] = sino[((int64_t)r * my + y) * kstride + k];
    __syncthreads();

    const float sinv = g.inv_sigma2[kg];
    const float sig = __frsqrt_rn(sinv);
    const float fk = g.norm[kg];
    const float w_mid = 1.0f / (float)(S * Se);
    const bool w_eta = flags & 1, w_tilt = flags & 2, w_tth = flags & 4;
    // reflection_two_theta: coords = u without the ring index, v = cos(theta_a) u - sin(theta_a) w per axis; the
    // derivatives of u (dv_*) and of w (dw_*) are given, the Bragg angle's is formed here (pf_grad.cl:100-122)
    const bool axis_theta = g.axis_w != nullptr;
    double acc[L::Q_TTH];
    double att[PG_PMAX];
#pragma unroll
    for (int q = 0; q < L::Q_TTH; ++q) acc[q] = 0.0;
#pragma unroll
    for (int q = 0; q < PG_PMAX; ++q) att[q] = 0.0;

    for (int i = row_ptr[row] + threadIdx.x; i < row_ptr[row + 1]; i += PG_THREADS) {
        const int j = col_j[i];
        const int c = j / P, p = j - c * P;
        const float *rr = res + (int64_t)r * my * CP + j;
        float G = 0.0f, Hs = 0.0f;
        for (int y = 0; y < my; ++y) {
            G = fmaf(rr[(int64_t)y * CP], lS[y], G);
            if (HESS) Hs = fmaf(curv[(int64_t)r * my * CP + (int64_t)y * CP + j], lS[y] * lS[y], Hs);
        }
        const float f = fk * (g.intens ? g.intens[p] : 1.0f);
        const int a0 = g.axis_start[p], a1 = g.axis_start[p + 1];
        float dr0 = 0.f, dr1 = 0.f, dr2 = 0.f, gs = 0.f, dgs = 0.f, de = 0.f, dt1 = 0.f, dt2 = 0.f, dtt = 0.f;
        for (int s = 0; s < S; ++s) {
            for (int se = 0; se < Se; ++se) {
                const float w = g.quad_w ? g.quad_w[s * Se + se] : w_mid;
                const int64_t cb = axis_theta ? (((int64_t)(r * S + s) * C + c) * Se + se) * 3
                                              : ((((int64_t)(r * S + s) * C + c) * Se + se) * P + p) * 3;
                const int64_t wb = (int64_t)(r * S + s) * 3;
                const float ux = g.coords[cb], uy = g.coords[cb + 1], uz = g.coords[cb + 2];
                const float wx = axis_theta ? g.axis_w[wb] : 0.0f, wy = axis_theta ? g.axis_w[wb + 1] : 0.0f,
                            wz = axis_theta ? g.axis_w[wb + 2] : 0.0f;
                for (int a = a0; a < a1; ++a) {
                    const float *n = g.poles + ((int64_t)kg * A + a) * 3;
                    const float nx = n[0], ny = n[1], nz = n[2];
                    const float ct = axis_theta ? g.axis_cos[a] : 1.0f, st = axis_theta ? g.axis_sin[a] : 0.0f;
                    const float vx = axis_theta ? ct * ux - st * wx : ux, vy = axis_theta ? ct * uy - st * wy : uy,
                                vz = axis_theta ? ct * uz - st * wz : uz;
                    // n . v near 1 for the terms that count: formed in float64 so that 1 - |n . v| keeps its
                    // digits (in float32 the exponent (1 - |d|) / sigma^2 of a narrow kernel loses up to 1e-4)
                    const double du = fma((double)nx, (double)ux, fma((double)ny, (double)uy, (double)nz * uz));
                    const double Dd = axis_theta
                                          ? (double)ct * du -
                                                (double)st * fma((double)nx, (double)wx,
                                                                 fma((double)ny, (double)wy, (double)nz * wz))
                                          : du;
                    const float D = (float)Dd;
                    const double add = fabs(Dd);
                    const float ad = (float)add;
                    const float x1 = (float)((1.0 - add) * sinv), x2 = (float)((1.0 + add) * sinv);
                    const float e1 = x1 < g.cut ? expf(-x1) : 0.0f;
                    const float e2 = x2 < g.cut ? expf(-x2) : 0.0f;
                    // window_parallax: the weight carries the window fraction (its own derivatives are not taken)
                    const float cw = w * g.axis_count[a] * (g.wp_ax && (e1 != 0.0f || e2 != 0.0f)
                                                                ? wp_fraction(g, r, kg, p, a) : 1.0f);
                    const float gd = cw * copysignf(sinv, D) * (e1 - e2);
                    dr0 = fmaf(gd, ny * vz - nz * vy, dr0);
                    dr1 = fmaf(gd, nz * vx - nx * vz, dr1);
                    dr2 = fmaf(gd, nx * vy - ny * vx, dr2);
                    gs = fmaf(cw, e1 + e2, gs);
                    dgs = fmaf(cw, -(1.0f - ad) * e1 - (1.0f + ad) * e2, dgs);
                    if (axis_theta) {
                        if (w_eta) de = fmaf(gd * ct, dot3(dv_eta + cb, nx, ny, nz), de);
                        if (w_tilt) {
                            dt1 = fmaf(gd, ct * dot3(dv_t1 + cb, nx, ny, nz) - st * dot3(dw_t1 + wb, nx, ny, nz), dt1);
                            dt2 = fmaf(gd, ct * dot3(dv_t2 + cb, nx, ny, nz) - st * dot3(dw_t2 + wb, nx, ny, nz), dt2);
                        }
                        if (w_tth)
                            dtt = fmaf(gd, 0.5f * (-st * dot3(g.coords + cb, nx, ny, nz) -
                                                   ct * dot3(g.axis_w + wb, nx, ny, nz)), dtt);
                    } else {
                        if (w_eta) de = fmaf(gd, dot3(dv_eta + cb, nx, ny, nz), de);
                        if (w_tilt) {
                            dt1 = fmaf(gd, dot3(dv_t1 + cb, nx, ny, nz), dt1);
                            dt2 = fmaf(gd, dot3(dv_t2 + cb, nx, ny, nz), dt2);
                        }
                        if (w_tth) dtt = fmaf(gd, dot3(dv_tth + cb, nx, ny, nz), dtt);
                    }
                }
            }
        }
        const float q0 = f * dr0, q1 = f * dr1, q2 = f * dr2;
        const float q3 = f * (-2.0f / sig * gs - 2.0f / (sig * sig * sig) * dgs);
        const double Gd = G, Gf = (double)G * f;
        acc[0] += Gd * q0;
        acc[1] += Gd * q1;
        acc[2] += Gd * q2;
        acc[3] += Gd * q3;
        if (HESS) {
            const double qv[4] = {q0, q1, q2, q3};
            int t = 4;
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = u; v < 4; ++v) acc[t++] += (double)Hs * qv[u] * qv[v];
        }
        acc[L::Q_ETA] += Gf * de;
        acc[L::Q_TILT] += Gf * dt1;
        acc[L::Q_TILT + 1] += Gf * dt2;
#pragma unroll
        for (int pp = 0; pp < PG_PMAX; ++pp)
            if (pp == p) att[pp] += Gf * dtt;
    }

    // block sum in a fixed order: lanes by shuffles, then the warps in order
    double *part = reinterpret_cast<double *>(lS + ((my + 1) & ~1));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < nq; ++q) {
        double v = 0.0;
#pragma unroll
        for (int u = 0; u < L::Q_TTH; ++u)
            if (u == q) v = acc[u];
#pragma unroll
        for (int u = 0; u < PG_PMAX; ++u)
            if (L::Q_TTH + u == q) v = att[u];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) part[warp * nq + q] = v;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nq; q += PG_THREADS) {
        double v = 0.0;
        for (int w = 0; w < PG_THREADS / 32; ++w) v += part[w * nq + q];
        rows[(int64_t)row * nq + q] = v;
    }
}

// per orientation of the batch: the rows (r, k) summed over r ascending
__global__ void pf_rows_sum_kernel(const double *__restrict__ rows, double *__restrict__ out, int R, int kb, int nq)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= kb * nq) return;
    const int k = t / nq, q = t - k * nq;
    double s = 0.0;
    for (int r = 0; r < R; ++r) s += rows[((int64_t)r * kb + k) * nq + q];
    out[t] = s;
}

// per angle: sum_{y < ns, k < kb} Z dS, a block per angle, fixed order
constexpr int AD_THREADS = 256;
__global__ void __launch_bounds__(AD_THREADS) angle_dot_kernel(const float *__restrict__ Z,
                                                               const float *__restrict__ dS, float *__restrict__ out,
                                                               int ns, int kstride, int kb)
{
    const int a = blockIdx.x;
    const int64_t n = (int64_t)ns * kb;
    float s = 0.0f;
    for (int64_t t = threadIdx.x; t < n; t += AD_THREADS) {
        const int64_t y = t / kb, k = t - y * kb;
        const int64_t i = ((int64_t)a * ns + y) * kstride + k;
        s = fmaf(Z[i], dS[i], s);
    }
    __shared__ float sh[AD_THREADS / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float v = 0.0f;
        for (int w = 0; w < AD_THREADS / 32; ++w) v += sh[w];
        out[a] = v;
    }
}

}  // namespace
}  // namespace dfx

using namespace dfx;

extern "C" int dfx_pf_param_nq(int n_rings, int hess) { return 4 + (hess ? 10 : 0) + 3 + n_rings; }

extern "C" int dfx_pf_param_vjp(const dfx_pf_geometry *g, const int32_t *row_ptr, const uint16_t *col_j,
                                const float *res, const float *curv, const float *sino, int my, int kstride, int k0,
                                int kb, int flags, const float *dv_eta, const float *dv_t1, const float *dv_t2,
                                const float *dv_tth, const float *dw_t1, const float *dw_t2, int hess, double *rows,
                                void *stream)
{
    DFX_REQUIRE(g && row_ptr && col_j && res && sino && rows, "pf_param_vjp: null pointer");
    DFX_REQUIRE(g->coords && g->poles && g->axis_start && g->axis_count && g->inv_sigma2 && g->norm,
                "pf_param_vjp: incomplete PF geometry");
    DFX_REQUIRE(g->P >= 1 && g->P <= PG_PMAX, "pf_param_vjp: %d rings (at most %d)", g->P, PG_PMAX);
    DFX_REQUIRE(my > 0 && kb > 0 && kstride >= kb && k0 >= 0 && k0 + kb <= g->K && g->R > 0,
                "pf_param_vjp: bad sizes");
    DFX_REQUIRE(!hess || curv, "pf_param_vjp: the Hessian blocks need curv");
    DFX_REQUIRE(!(flags & 1) || dv_eta, "pf_param_vjp: eta offset requested without its derivatives");
    DFX_REQUIRE(!(flags & 2) || (dv_t1 && dv_t2), "pf_param_vjp: axis tilt requested without its derivatives");
    const bool axis_theta = g->axis_w != nullptr;
    DFX_REQUIRE(!(flags & 4) || dv_tth || axis_theta, "pf_param_vjp: two-theta requested without its derivatives");
    DFX_REQUIRE(!(flags & 2) || !axis_theta || (dw_t1 && dw_t2),
                "pf_param_vjp: axis tilt with reflection_two_theta needs the derivatives of w");
    DFX_REQUIRE(!axis_theta || (g->axis_sin && g->axis_cos), "pf_param_vjp: incomplete axis Bragg angles");
    const int64_t n_rows = (int64_t)g->R * kb;
    DFX_REQUIRE(n_rows < 2147483647LL, "pf_param_vjp: too many rows");
    const int nq = dfx_pf_param_nq(g->P, hess);
    const size_t smem = sizeof(float) * (size_t)((my + 1) & ~1) + sizeof(double) * (size_t)(PG_THREADS / 32) * nq;
    DFX_REQUIRE(smem <= 48 * 1024, "pf_param_vjp: %d detector bins exceed the shared-memory column", my);
    cudaStream_t s = (cudaStream_t)stream;
    if (hess)
        pf_param_vjp_kernel<1><<<(unsigned)n_rows, PG_THREADS, smem, s>>>(
            *g, row_ptr, col_j, res, curv, sino, my, kstride, k0, kb, flags, dv_eta, dv_t1, dv_t2, dv_tth, dw_t1,
            dw_t2, rows, nq);
    else
        pf_param_vjp_kernel<0><<<(unsigned)n_rows, PG_THREADS, smem, s>>>(
            *g, row_ptr, col_j, res, curv, sino, my, kstride, k0, kb, flags, dv_eta, dv_t1, dv_t2, dv_tth, dw_t1,
            dw_t2, rows, nq);
    return launch_status("pf_param_vjp");
}

extern "C" int dfx_pf_rows_sum(const double *rows, int n_angles, int kb, int nq, double *out, void *stream)
{
    DFX_REQUIRE(rows && out && n_angles > 0 && kb > 0 && nq > 0, "pf_rows_sum: bad arguments");
    const int n = kb * nq;
    pf_rows_sum_kernel<<<(unsigned)cdiv(n, 128), 128, 0, (cudaStream_t)stream>>>(rows, out, n_angles, kb, nq);
    return launch_status("pf_rows_sum");
}

extern "C" int dfx_angle_dot(const float *Z, const float *dS, int n_angles, int n_det, int kstride, int kb,
                             float *out, void *stream)
{
    DFX_REQUIRE(Z && dS && out && n_angles > 0 && n_det > 0 && kb > 0 && kstride >= kb, "angle_dot: bad arguments");
    angle_dot_kernel<<<(unsigned)n_angles, AD_THREADS, 0, (cudaStream_t)stream>>>(Z, dS, out, n_det, kstride, kb);
    return launch_status("angle_dot");
}
