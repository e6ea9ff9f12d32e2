/*
 * CPU restatement of diffractom's reconstruction hot path, TEST INFRASTRUCTURE ONLY (the checker of the CUDA
 * kernels and the timed CPU baseline; never linked into or called by the product). Built by oracle/Makefile into
 * oracle/_build/liboracle.so (gcc, -O3 -fopenmp -ffp-contract=off) and loaded with ctypes by oracle/oracle.py.
 *
 * Parity pins: tests/test_oracle.py checks these functions against the golden fixtures made from the reference's
 * own host code and its float64 ReferenceModel (tests/golden/make_golden.py).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ACC double
#define SUFFIX _f64
#include "oracle_core.h"
#undef ACC
#undef SUFFIX
#define ACC float
#define SUFFIX _f32
#include "oracle_core.h"
#undef ACC
#undef SUFFIX
#undef IO
#define ACC double
#define IO double
#define SUFFIX _f64io
#include "oracle_core.h"
#undef ACC
#undef IO
#undef SUFFIX

/* One pole-figure entry, pf_generate.cl:62-140 (pf_entry) == create_pfo_matrix.py:108-199 (pfmatrix_eval_poles):
 * PF[r, k, c, p] = norm_k * mean over the (omega, eta) quadrature nodes of
 *     sum_{axes a of ring p} count_a [exp(-(1 - |n.v|) s_k) [< cut] + exp(-(1 + |n.v|) s_k) [< cut]],
 * n = poles[kg, a], v = coords[r, s, c, se, p], s_k = 1 / sigma_k^2; quad_w == NULL: the midpoint rule (equal
 * sub-bins, averaged), else the product weights qw[s * S_eta + se] (Gauss-Legendre, weights summing to 1).
 * The dot product is fmaf(pz, vz, fmaf(py, vy, px * vx)) and each exponent (1 -+ d) * s_k is rounded twice, as in
 * the CUDA kernel, so the zero pattern (which exponents pass the cut) is the same bit for bit. */
static float pf_entry(const float *coords, const float *poles, const int32_t *axis_start, const float *axis_count,
                      const float *qw, float inv_sig2, float norm, int r, int kg, int c, int p, int S, int C,
                      int S_eta, int P, int A, float cut)
{
    const int a0 = axis_start[p], a1 = axis_start[p + 1];
    const float *pole = poles + (size_t)kg * A * 3;
    float w_total = 0.0f;
    for (int s = 0; s < S; ++s)
        for (int se = 0; se < S_eta; ++se) {
            const float *v = coords + ((((size_t)(r * S + s) * C + c) * S_eta + se) * P + p) * 3;
            float w_node = 0.0f;
            for (int a = a0; a < a1; ++a) {
                const float *n = pole + 3 * a;
                const float d = fabsf(fmaf(n[2], v[2], fmaf(n[1], v[1], n[0] * v[0])));
                float t = 0.0f;
                const float e1 = (1.0f - d) * inv_sig2;
                if (e1 < cut) t += expf(-e1);
                const float e2 = (1.0f + d) * inv_sig2;
                if (e2 < cut) t += expf(-e2);
                w_node = fmaf(axis_count[a], t, w_node);
            }
            if (qw) w_total = fmaf(qw[s * S_eta + se], w_node, w_total);
            else w_total += w_node;
        }
    return qw ? w_total * norm : (w_total / (float)(S * S_eta)) * norm;
}

/* Dense PF batch of orientations k0 .. k0+Kb-1: out (R, Kb, C, P), scaled by the ring intensity unless normalized
 * (SCALE_PF_BY_INTENSITY_INPLACE, pf_kernels.cl:450-465). */
void orc_pf_dense(const float *coords, const float *poles, const int32_t *axis_start, const float *axis_count,
                  const float *inv_sigma2, const float *norm_factor, const float *qw, const float *intens,
                  float *out, int R, int k0, int Kb, int C, int P, int A, int S, int S_eta, float cut, int normalized)
{
    #pragma omp parallel for collapse(2) schedule(static)
    for (int r = 0; r < R; ++r)
        for (int k = 0; k < Kb; ++k) {
            const int kg = k0 + k;
            for (int c = 0; c < C; ++c)
                for (int p = 0; p < P; ++p) {
                    float v = pf_entry(coords, poles, axis_start, axis_count, qw, inv_sigma2[kg], norm_factor[kg],
                                       r, kg, c, p, S, C, S_eta, P, A, cut);
                    if (!normalized) v *= intens[p];
                    out[(((size_t)r * Kb + k) * C + c) * P + p] = v;
                }
        }
}

/* Row lengths of the two CSR copies of a dense batch pf (R, Kb, CP), pf_kernels.cl:482-548: adjoint rows r * Kb + k
 * (non-zero j ascending), forward rows r * CP + j (non-zero k ascending). */
void orc_csr_counts(const float *pf, int R, int Kb, int CP, int32_t *cnt_adj, int32_t *cnt_fwd)
{
    for (size_t i = 0; i < (size_t)R * CP; ++i) cnt_fwd[i] = 0;
    for (int r = 0; r < R; ++r)
        for (int k = 0; k < Kb; ++k) {
            int n = 0;
            const float *row = pf + ((size_t)r * Kb + k) * CP;
            for (int j = 0; j < CP; ++j)
                if (row[j] != 0.0f) { ++n; ++cnt_fwd[(size_t)r * CP + j]; }
            cnt_adj[(size_t)r * Kb + k] = n;
        }
}

void orc_csr_fill(const float *pf, int R, int Kb, int CP, const int32_t *ptr_adj, uint16_t *col_j, float *val_a,
                  const int32_t *ptr_fwd, uint16_t *col_k, float *val_f)
{
    for (int r = 0; r < R; ++r) {
        for (int k = 0; k < Kb; ++k) {
            int i = ptr_adj[(size_t)r * Kb + k];
            const float *row = pf + ((size_t)r * Kb + k) * CP;
            for (int j = 0; j < CP; ++j)
                if (row[j] != 0.0f) { col_j[i] = (uint16_t)j; val_a[i] = row[j]; ++i; }
        }
        for (int j = 0; j < CP; ++j) {
            int i = ptr_fwd[(size_t)r * CP + j];
            for (int k = 0; k < Kb; ++k) {
                const float v = pf[((size_t)r * Kb + k) * CP + j];
                if (v != 0.0f) { col_k[i] = (uint16_t)k; val_f[i] = v; ++i; }
            }
        }
    }
}

/* Channel gather / scatter between the coefficients (Ktot, Npix) and the channel-fastest batch (Npix, Kstride),
 * radon_kernels.cl:192-244. */
void orc_gather(const float *coeffs, float *img, int Npix, int k0, int Kb, int Kstride)
{
    for (int p = 0; p < Npix; ++p)
        for (int k = 0; k < Kstride; ++k)
            img[(size_t)p * Kstride + k] = k < Kb ? coeffs[(size_t)(k0 + k) * Npix + p] : 0.0f;
}

void orc_scatter(const float *img, float *coeffs, int Npix, int k0, int Kb, int Kstride)
{
    for (int k = 0; k < Kb; ++k)
        for (int p = 0; p < Npix; ++p)
            coeffs[(size_t)(k0 + k) * Npix + p] = img[(size_t)p * Kstride + k];
}

/* dst (cols, rows) = src (rows, cols)^T, blocked and spread over the threads: the layout changes between the
 * coefficients (K, Npix) and the channel-fastest batch (Npix, K) that the reference's gather / scatter kernels do on
 * the device (radon_kernels.cl:192-244). src_ld / dst_ld: row strides in elements. */
#define TRANSPOSE(NAME, T)                                                                                         \
    void NAME(const T *src, T *dst, int64_t rows, int64_t cols, int64_t src_ld, int64_t dst_ld)                   \
    {                                                                                                              \
        const int64_t B = 64;                                                                                      \
        _Pragma("omp parallel for collapse(2) schedule(static)")                                                  \
        for (int64_t r0 = 0; r0 < rows; r0 += B)                                                                   \
            for (int64_t c0 = 0; c0 < cols; c0 += B) {                                                             \
                const int64_t r1 = r0 + B < rows ? r0 + B : rows, c1 = c0 + B < cols ? c0 + B : cols;            \
                for (int64_t c = c0; c < c1; ++c)                                                                  \
                    for (int64_t r = r0; r < r1; ++r) dst[c * dst_ld + r] = src[r * src_ld + c];                   \
            }                                                                                                      \
    }
TRANSPOSE(orc_transpose_f32, float)
TRANSPOSE(orc_transpose_f64, double)
#undef TRANSPOSE

static inline float pv(const float *a, uint64_t period, uint64_t i, float dflt) { return period ? a[i % period] : dflt; }

/* SPDHG dual step on the rows of the angles omegas (spdhg_poisson.py:69-91, dual_update_sub): on entry d holds A x
 * there, on exit the dual change; y' = prox_{sigma F*}(y + sigma (A x + r)) in closed form, float64 arithmetic,
 * r = bg + eps g, sc = w / g; y' = 0 where w = 0 or sigma = 0. */
void orc_dual_update_sub(float *y, float *d, const float *sig, const float *b, const float *w, uint64_t pw,
                         const float *g, uint64_t pg, const float *bg, uint64_t pbg, float eps,
                         const int32_t *omegas, uint64_t row, uint64_t n)
{
    #pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < (int64_t)n; ++t) {
        const uint64_t s = (uint64_t)t / row;
        const uint64_t i = (uint64_t)omegas[s] * row + ((uint64_t)t - s * row);
        const float wi = pv(w, pw, i, 1.0f), si = sig[i];
        float yn = 0.0f;
        if (wi != 0.0f && si != 0.0f) {
            const float gi = pv(g, pg, i, 1.0f);
            const double sc = (double)wi / (double)gi;
            const double rr = (double)pv(bg, pbg, i, 0.0f) + (double)eps * gi;
            const double v = (double)y[i] + (double)si * d[i] + (double)si * rr;
            const double dd = v - sc;
            yn = (float)(0.5 * (v + sc - sqrt(dd * dd + 4.0 * (double)si * sc * (double)b[i])));
        }
        d[i] = yn - y[i];
        y[i] = yn;
    }
}

/* SPDHG primal step of one batch (spdhg_poisson.py:95-106): z += dz; x = max(0, x - T (z + dz / p + lam)), 0 where
 * T = 0. */
void orc_spdhg_update(float *x, float *z, const float *T, const float *dz, float inv_p, float lam, uint64_t n)
{
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const float zi = z[i] + dz[i];
        z[i] = zi;
        const float zb = zi + inv_p * dz[i];
        const float t = T[i];
        x[i] = t > 0.0f ? fmaxf(0.0f, x[i] - t * (zb + lam)) : 0.0f;
    }
}

/* Poisson deviance in float64 (fista_poisson.py:72-113, mode 0, without the gradient):
 * sum_i w_i / g_i [m_i - b_i + b_i log(b_i / m_i)], m = max(mu, 0) + bg + eps g. */
double orc_deviance(const float *mu, const float *b, const float *w, uint64_t pw, const float *g, uint64_t pg,
                    const float *bg, uint64_t pbg, float eps, uint64_t n)
{
    double s = 0.0;
    #pragma omp parallel for reduction(+ : s) schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const float wi = pv(w, pw, i, 1.0f);
        if (wi == 0.0f) continue;
        const float gi = pv(g, pg, i, 1.0f);
        const double bi = (double)b[i];
        const double sc = (double)wi / (double)gi;
        const double m = (double)fmaxf(mu[i], 0.0f) + (double)pv(bg, pbg, i, 0.0f) + (double)eps * gi;
        double v = m - bi;
        if (bi > 0.0) v += bi * log(bi / m);
        s += sc * v;
    }
    return s;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}
