// aclblasSgetrsAdjointBatched: reverse-mode derivative of the batched solve X = A^{-1} B.
//
// No counterpart in the reference (an extension next to the drop-in chain). Given the LU
// factors and pivots of A (aclblasSgetrfBatched), the forward solution X and the upstream
// gradient dX:
//   dB = A^{-T} dX      -- the transposed solve on the stored factors (trans T of
//                          aclblasSgetrsBatched's kernels), overwriting dX in place;
//   dA = -dB * X^T      -- a rank-nrhs outer product per matrix, by the batched GEMM kernel
//                          with alpha = -1 and beta = 0 fused in its epilogue.
// Both run on the handle's stream; nothing is allocated or copied to the host.
#include <cuda_runtime.h>

#include "internal.h"

using namespace opsblas;

extern "C" aclblasStatus_t aclblasSgetrsAdjointBatched(
    aclblasHandle_t handle, int n, int nrhs, const float* const LUarray[], int lda, const int* devIpiv,
    const float* const Xarray[], int ldx, float* const dXarray[], int lddx, float* const dAarray[], int ldda,
    int batchCount)
{
    static const char* kApi = "aclblasSgetrsAdjointBatched";
    if (handle == nullptr) {
        log_error(kApi, "handle is nullptr");
        return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    }
    if (n < 0 || nrhs < 0 || nrhs > 256 || batchCount < 0) {
        log_error(kApi, "invalid sizes n=%d nrhs=%d batchCount=%d (nrhs <= 256)", n, nrhs, batchCount);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (lda < max1(n) || ldx < max1(n) || lddx < max1(n) || (dAarray != nullptr && ldda < max1(n))) {
        log_error(kApi, "leading dimensions must be >= max(1, n)");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (n == 0 || nrhs == 0 || batchCount == 0) return ACLBLAS_STATUS_SUCCESS;
    if (LUarray == nullptr || Xarray == nullptr || dXarray == nullptr) {
        log_error(kApi, "LUarray, Xarray and dXarray must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    cudaStream_t st = handle->stream;
    cudaError_t err = getrs_launch(st, true, n, nrhs, LUarray, lda, devIpiv, dXarray, lddx, batchCount);
    if (err == cudaSuccess && dAarray != nullptr)
        err = gemm_f32_launch(st, false, true, n, n, nrhs, -1.0f, const_cast<const float* const*>(dXarray), lddx,
                              Xarray, ldx, 0.0f, dAarray, ldda, batchCount, 0);
    return launch_status(kApi, err);
}
