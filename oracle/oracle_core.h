/*
 * CPU restatement of the reconstruction hot path of diffractom (msaca-okse/diffractom), TEST INFRASTRUCTURE ONLY:
 * the checker of the CUDA kernels in diffractom_b200/csrc and the timed CPU baseline. Nothing in the product
 * imports, links or calls it.
 *
 * This header is compiled three times by oracle.c: with ACC = double (suffix _f64, the checker: float32 inputs and
 * tap weights, float64 sums), with ACC = float (suffix _f32, the CPU baseline, float32 like the reference's kernels)
 * and with ACC = IO = double (suffix _f64io: the same float32 geometry and weights, float64 images, sinograms and
 * data, for float64 finite differences of the forward model).
 *
 * Conventions shared with the CUDA kernels (they make the float32 tap weights of both identical bit for bit; the C
 * side is compiled with -ffp-contract=off and writes every fused multiply-add as fmaf):
 *   geo[a] = (X, Y, T0, w): pixel (x, y) lands at detector coordinate t (bins), with rows along the image axis whose
 *   coefficient is larger in magnitude: A = rows_are_y ? X : Y, B = the other, (u, v) = rows_are_y ? (x, y) : (y, x),
 *       t = fmaf(A, u, fmaf(B, v, T0))
 *   and adds weight K(t - s) to bin s. Trapezoid (distance-driven): K(d) = min(max(hw - |d|, 0), top) * iw with
 *   hw = (1 + |A|) / 2, top = min(1, |A|), iw = 1 / |A|; hat: K(d) = max(1 - |d|, 0).
 *   The reference computes the same kernel with t evaluated per strip of bins (radon_kernels.cl:44-101) or per pixel
 *   (radon_kernels.cl:106-141); both are the same real number t, rounded differently in float32.
 */
#include <math.h>
#include <stdint.h>
#include <stddef.h>

#ifndef ACC
#error "define ACC"
#endif
#ifndef IO
#define IO float
#endif
#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SUFFIX)

/* Forward projection, radon_kernels.cl:44-101 (radon_forward_k): sino[a, s, k] = scale * sum_pix K(t - s) img[pix, k]
 * for angles a < R (the rows of geo), channels k < Kb of a (Npix, Kstride) / (R, Ns, Kstride) channel-fastest
 * layout; channels Kb .. Kstride-1 of sino are set to 0 (the reference leaves its padding channels to the zero
 * padding of the image). kernel: 0 hat, 1 trapezoid. */
void FN(orc_radon_forward)(const IO *img, IO *sino, const float *geo, int R, int Nx, int Ny, int Ns,
                           int Kstride, int Kb, int kernel, float scale)
{
    #pragma omp parallel for schedule(dynamic, 1)
    for (int a = 0; a < R; ++a) {
        const float X = geo[4 * a], Y = geo[4 * a + 1], T0 = geo[4 * a + 2];
        const int rows_are_y = fabsf(X) >= fabsf(Y);
        const float A = rows_are_y ? X : Y, B = rows_are_y ? Y : X;
        const int Nu = rows_are_y ? Nx : Ny, Nv = rows_are_y ? Ny : Nx;
        const float aA = fabsf(A);
        const float hw = 0.5f * (1.0f + aA), top = fminf(1.0f, aA), iw = 1.0f / aA;
        ACC *acc = (ACC *)calloc((size_t)Ns * Kb, sizeof(ACC));
        for (int v = 0; v < Nv; ++v) {
            const float c = fmaf(B, (float)v, T0);
            for (int u = 0; u < Nu; ++u) {
                const float t = fmaf(A, (float)u, c);
                const int p = rows_are_y ? (u + Nx * v) : (v + Nx * u);
                const IO *row = img + (size_t)p * Kstride;
                int s_lo, s_hi;
                if (kernel == 1) { s_lo = (int)floorf(t - hw); s_hi = (int)ceilf(t + hw); }   /* a superset: */
                else { s_lo = (int)floorf(t); s_hi = s_lo + 1; }                           /* K decides */
                if (s_lo < 0) s_lo = 0;
                if (s_hi > Ns - 1) s_hi = Ns - 1;
                for (int s = s_lo; s <= s_hi; ++s) {
                    const float d = t - (float)s;
                    const float w = kernel == 1 ? fminf(fmaxf(hw - fabsf(d), 0.0f), top) * iw
                                                : fmaxf(1.0f - fabsf(d), 0.0f);
                    if (w == 0.0f) continue;
                    ACC *o = acc + (size_t)s * Kb;
                    for (int k = 0; k < Kb; ++k) o[k] += (ACC)w * (ACC)row[k];
                }
            }
        }
        for (int s = 0; s < Ns; ++s) {
            IO *o = sino + ((size_t)a * Ns + s) * Kstride;
            for (int k = 0; k < Kb; ++k) o[k] = (IO)((ACC)scale * acc[(size_t)s * Kb + k]);
            for (int k = Kb; k < Kstride; ++k) o[k] = 0.0f;
        }
        free(acc);
    }
}

/* Backward projection, radon_kernels.cl:106-141 (radon_backward_k): img[pix, k] = sum_a w_a sum_s K(t - s) sino[a, s, k],
 * no atomics (pixel-driven); channels Kb .. Kstride-1 of img are set to 0. */
void FN(orc_radon_backward)(const IO *sino, IO *img, const float *geo, int R, int Nx, int Ny, int Ns,
                            int Kstride, int Kb, int kernel)
{
    const int Npix = Nx * Ny;
    #pragma omp parallel for schedule(static)
    for (int p = 0; p < Npix; ++p) {
        const int x = p % Nx, y = p / Nx;
        ACC *acc = (ACC *)calloc((size_t)Kb, sizeof(ACC));
        for (int a = 0; a < R; ++a) {
            const float X = geo[4 * a], Y = geo[4 * a + 1], T0 = geo[4 * a + 2], wa = geo[4 * a + 3];
            const int rows_are_y = fabsf(X) >= fabsf(Y);
            const float A = rows_are_y ? X : Y, B = rows_are_y ? Y : X;
            const float u = (float)(rows_are_y ? x : y), v = (float)(rows_are_y ? y : x);
            const float t = fmaf(A, u, fmaf(B, v, T0));
            const float aA = fabsf(A);
            const float hw = 0.5f * (1.0f + aA), top = fminf(1.0f, aA), iw = 1.0f / aA;
            int s_lo, s_hi;
            if (kernel == 1) { s_lo = (int)floorf(t - hw); s_hi = (int)ceilf(t + hw); }
            else { s_lo = (int)floorf(t); s_hi = s_lo + 1; }
            if (s_lo < 0) s_lo = 0;
            if (s_hi > Ns - 1) s_hi = Ns - 1;
            for (int s = s_lo; s <= s_hi; ++s) {
                const float d = t - (float)s;
                const float w = kernel == 1 ? fminf(fmaxf(hw - fabsf(d), 0.0f), top) * iw
                                            : fmaxf(1.0f - fabsf(d), 0.0f);
                if (w == 0.0f) continue;
                const IO *src = sino + ((size_t)a * Ns + s) * Kstride;
                const ACC ww = (ACC)wa * (ACC)w;
                for (int k = 0; k < Kb; ++k) acc[k] += ww * (ACC)src[k];
            }
        }
        IO *o = img + (size_t)p * Kstride;
        for (int k = 0; k < Kb; ++k) o[k] = (IO)acc[k];
        for (int k = Kb; k < Kstride; ++k) o[k] = 0.0f;
        free(acc);
    }
}

/* Forward PF product on a forward CSR (rows r * CP + j listing k), pf_kernels.cl:597-641 and its subset form
 * SPFO:38-80: data[omegas[rs], y, j] += sum_k val * sino[rs, y, k] for the Rm subset angles (omegas NULL: all R
 * angles, rs = r). compact: the CSR holds the subset's rows only (row rs * CP + j); otherwise row omegas[rs] * CP + j.
 * An empty row leaves its data untouched (the reference skips its read-modify-write). */
void FN(orc_spmm_forward)(const IO *sino, const int32_t *row_ptr, const uint16_t *col_k, const float *val,
                          IO *data, const int32_t *omegas, int Rm, int My, int CP, int Kstride, int compact)
{
    #pragma omp parallel for collapse(2) schedule(static)
    for (int rs = 0; rs < Rm; ++rs)
        for (int y = 0; y < My; ++y) {
            const int r = omegas ? omegas[rs] : rs;
            const int rr = compact ? rs : r;
            const IO *zl = sino + ((size_t)rs * My + y) * Kstride;
            IO *dl = data + ((size_t)r * My + y) * CP;
            for (int j = 0; j < CP; ++j) {
                const int b = row_ptr[(size_t)rr * CP + j], e = row_ptr[(size_t)rr * CP + j + 1];
                if (b == e) continue;
                ACC s = 0;
                for (int i = b; i < e; ++i) s += (ACC)val[i] * (ACC)zl[col_k[i]];
                dl[j] = (IO)((ACC)dl[j] + s);
            }
        }
}

/* Adjoint PF product on an adjoint CSR (rows r * Kb + k listing j), pf_kernels.cl:644-687 and SPFO:82-123:
 * sino[rs, y, k] = alpha * sum_j val * data[omegas[rs], y, j] for k < Kb (channels Kb .. Kstride-1 untouched). */
void FN(orc_spmm_adjoint)(const IO *data, const int32_t *row_ptr, const uint16_t *col_j, const float *val,
                          IO *sino, const int32_t *omegas, int Rm, int My, int Kb, int CP, int Kstride,
                          float alpha, int compact)
{
    #pragma omp parallel for collapse(2) schedule(static)
    for (int rs = 0; rs < Rm; ++rs)
        for (int y = 0; y < My; ++y) {
            const int r = omegas ? omegas[rs] : rs;
            const int rr = compact ? rs : r;
            const IO *dl = data + ((size_t)r * My + y) * CP;
            IO *zl = sino + ((size_t)rs * My + y) * Kstride;
            for (int k = 0; k < Kb; ++k) {
                const int b = row_ptr[(size_t)rr * Kb + k], e = row_ptr[(size_t)rr * Kb + k + 1];
                ACC s = 0;
                for (int i = b; i < e; ++i) s += (ACC)val[i] * (ACC)dl[col_j[i]];
                zl[k] = (IO)((ACC)alpha * s);
            }
        }
}

#undef FN
#undef CAT
#undef CAT_
