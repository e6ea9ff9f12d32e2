// Local basis (diffractom's LocalSinglePhaseForwardOperator, operators/local_forward_operator.py): the coefficients
// of an orientation batch are rectangular patches (flat, row-major per patch, a 0/1 mask for the allowed voxels).
// The B200 operator projects a batch through the dense channel-fastest kernels: the patches are scattered into the
// batch image (zero elsewhere) before the forward projection and gathered from it after the backprojection, so the
// solvers' coefficient arrays scale with the support while the projections run at the full-image kernels' speed.
//
// Patch table of a batch (n_patches entries): box (y0, x0, h, w) int32 x 4, coff int64 (offset of the patch's
// coefficients), chan int32 (the orientation's channel in the batch). A block per patch, threads over its cells.
// pix_row (optional, nx * ny int32): the row of every pixel in a compact batch image that holds only the pixels of
// the batch's support (-1: not there); NULL: the whole image, row = pixel.
#include "dfx_common.cuh"

namespace dfx {
namespace {

__device__ __forceinline__ int64_t pixel_row(const int32_t *pix_row, int64_t pix)
{
    return pix_row ? (int64_t)__ldg(pix_row + pix) : pix;
}

__global__ void local_scatter_kernel(const float *__restrict__ coeffs, const uint8_t *__restrict__ mask,
                                     const int4 *__restrict__ box, const int64_t *__restrict__ coff,
                                     const int32_t *__restrict__ chan, const int32_t *__restrict__ pix_row,
                                     float *__restrict__ img, int nx, int ny, int kstride)
{
    const int4 b = __ldg(box + blockIdx.x);                // y0, x0, h, w
    const int64_t base = __ldg(coff + blockIdx.x);
    const int c = __ldg(chan + blockIdx.x);
    const int n = b.z * b.w;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int dy = i / b.w, y = b.x + dy, x = b.y + (i - dy * b.w);
        if (y < 0 || y >= ny || x < 0 || x >= nx) continue;
        const int64_t row = pixel_row(pix_row, (int64_t)y * nx + x);
        if (row < 0) continue;
        img[row * kstride + c] = __ldg(mask + base + i) ? coeffs[base + i] : 0.0f;
    }
}

__global__ void local_gather_kernel(const float *__restrict__ img, const uint8_t *__restrict__ mask,
                                    const int4 *__restrict__ box, const int64_t *__restrict__ coff,
                                    const int32_t *__restrict__ chan, const int32_t *__restrict__ pix_row,
                                    float *__restrict__ coeffs, int nx, int ny, int kstride)
{
    const int4 b = __ldg(box + blockIdx.x);
    const int64_t base = __ldg(coff + blockIdx.x);
    const int c = __ldg(chan + blockIdx.x);
    const int n = b.z * b.w;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int dy = i / b.w, y = b.x + dy, x = b.y + (i - dy * b.w);
        const bool in = y >= 0 && y < ny && x >= 0 && x < nx && __ldg(mask + base + i);
        const int64_t row = in ? pixel_row(pix_row, (int64_t)y * nx + x) : -1;
        coeffs[base + i] = row >= 0 ? img[row * kstride + c] : 0.0f;
    }
}

int check_local(const void *a, const void *b, const uint8_t *mask, const int32_t *box, const int64_t *coff,
                const int32_t *chan, int n_patches, int nx, int ny, int kstride, const char *what)
{
    DFX_REQUIRE(a && b && mask && box && coff && chan, "%s: null pointer", what);
    DFX_REQUIRE(n_patches >= 0 && nx > 0 && ny > 0 && kstride > 0, "%s: bad sizes", what);
    DFX_REQUIRE(((uintptr_t)box % 16) == 0 && ((uintptr_t)coff % 8) == 0, "%s: misaligned patch table", what);
    return DFX_OK;
}

}  // namespace
}  // namespace dfx

using namespace dfx;

extern "C" int dfx_local_scatter(const float *coeffs, const uint8_t *mask, const int32_t *box, const int64_t *coff,
                                 const int32_t *chan, int n_patches, int nx, int ny, int kstride,
                                 const int32_t *pix_row, float *img_k, void *stream)
{
    int st = check_local(coeffs, img_k, mask, box, coff, chan, n_patches, nx, ny, kstride, "local_scatter");
    if (st) return st;
    if (n_patches == 0) return DFX_OK;
    local_scatter_kernel<<<(unsigned)n_patches, 128, 0, (cudaStream_t)stream>>>(
        coeffs, mask, reinterpret_cast<const int4 *>(box), coff, chan, pix_row, img_k, nx, ny, kstride);
    return launch_status("local_scatter");
}

extern "C" int dfx_local_gather(const float *img_k, const uint8_t *mask, const int32_t *box, const int64_t *coff,
                                const int32_t *chan, int n_patches, int nx, int ny, int kstride,
                                const int32_t *pix_row, float *coeffs, void *stream)
{
    int st = check_local(img_k, coeffs, mask, box, coff, chan, n_patches, nx, ny, kstride, "local_gather");
    if (st) return st;
    if (n_patches == 0) return DFX_OK;
    local_gather_kernel<<<(unsigned)n_patches, 128, 0, (cudaStream_t)stream>>>(
        img_k, mask, reinterpret_cast<const int4 *>(box), coff, chan, pix_row, coeffs, nx, ny, kstride);
    return launch_status("local_gather");
}
