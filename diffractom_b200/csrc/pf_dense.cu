// The dense pole-figure products of pf_mode "dense" (FP32): per orientation batch the float32 PF of every angle is
// generated (dfx_pf_dense) and applied by one strided batched SGEMM over the angles, as the reference applies its
// dense batch with CLBlast's batched GEMM above 30 % fill (SPFO:2063-2127, batched_gemm_clblast / _adj):
//   forward  data[r] (My x CP) += Z[r] (My x Kb) . PF[r] (Kb x CP)         (beta = 1: batches add into the rows)
//   adjoint  Z[r] (My x Kb)     = alpha D[r] (My x CP) . PF[r]^T (CP x Kb)
// Row-major arrays are handed to cuBLAS as their column-major transposes. The handle is made once per host thread and
// device and runs in float32 (CUBLAS_PEDANTIC_MATH: no TF32, no reduced-precision reductions).
#include <cublas_v2.h>

#include <map>

#include "dfx_common.cuh"

namespace dfx {
namespace {

cublasHandle_t handle_for_current_device(int &status)
{
    thread_local std::map<int, cublasHandle_t> handles;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        status = DFX_ECUDA;
        return nullptr;
    }
    auto it = handles.find(dev);
    if (it != handles.end()) return it->second;
    cublasHandle_t h = nullptr;
    if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS || cublasSetMathMode(h, CUBLAS_PEDANTIC_MATH) != CUBLAS_STATUS_SUCCESS) {
        status = DFX_ECUDA;
        return nullptr;
    }
    handles[dev] = h;
    return h;
}

}  // namespace
}  // namespace dfx

using namespace dfx;

extern "C" int dfx_pf_dense_products(int adjoint, const float *pf, int n_omega, int kb, int cp, const float *in,
                                     float *out, int my, int kstride, float alpha, void *stream)
{
    DFX_REQUIRE(pf && in && out, "pf_dense_products: null pointer");
    DFX_REQUIRE(n_omega > 0 && kb > 0 && cp > 0 && my > 0 && kstride >= kb,
                "pf_dense_products: bad sizes (angles %d, Kb %d, CP %d, My %d, kstride %d)", n_omega, kb, cp, my,
                kstride);
    int status = DFX_OK;
    cublasHandle_t h = handle_for_current_device(status);
    if (!h) {
        set_error("pf_dense_products: no cuBLAS handle");
        return status ? status : DFX_ECUDA;
    }
    if (cublasSetStream(h, (cudaStream_t)stream) != CUBLAS_STATUS_SUCCESS) {
        set_error("pf_dense_products: cublasSetStream failed");
        return DFX_ECUDA;
    }
    const long long s_pf = (long long)kb * cp, s_sino = (long long)my * kstride, s_data = (long long)my * cp;
    cublasStatus_t rc;
    if (!adjoint) {
        // data^T (CP x My, ld CP) += PF^T (CP x Kb, ld CP) . Z^T (Kb x My, ld kstride)
        const float one = 1.0f;
        rc = cublasSgemmStridedBatched(h, CUBLAS_OP_N, CUBLAS_OP_N, cp, my, kb, &one, pf, cp, s_pf, in, kstride,
                                       s_sino, &one, out, cp, s_data, n_omega);
    } else {
        // Z^T (Kb x My, ld kstride) = alpha PF (Kb x CP) . D^T (CP x My, ld CP); the padding channels Kb.. set to 0
        if (kb < kstride) {
            const cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float) * (size_t)s_sino * n_omega,
                                                  (cudaStream_t)stream);
            if (e != cudaSuccess) {
                set_error("pf_dense_products: %s", cudaGetErrorString(e));
                return DFX_ECUDA;
            }
        }
        const float zero = 0.0f;
        rc = cublasSgemmStridedBatched(h, CUBLAS_OP_T, CUBLAS_OP_N, kb, my, cp, &alpha, pf, cp, s_pf, in, cp, s_data,
                                       &zero, out, kstride, s_sino, n_omega);
    }
    if (rc != CUBLAS_STATUS_SUCCESS) {
        set_error("pf_dense_products: cuBLAS status %d", (int)rc);
        return DFX_ELAUNCH;
    }
    return launch_status("pf_dense_products");
}
