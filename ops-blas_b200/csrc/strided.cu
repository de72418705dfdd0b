// Pointer-array builder and strided-batch entry points (extensions; the reference has only the
// pointer-array API and builds its internal arrays with a kernel of its own,
// blas/matinv_batched/arch35/init_ptr_array_kernel.cpp). A strided batch is `batchSize`
// matrices at base + i * stride elements. The strided calls write their pointer arrays into the
// handle's workspace on the handle's stream and then run the batched entry points, so the results
// are those of the pointer-array calls bit for bit; successive calls on one handle reuse the
// workspace in stream order.
#include <cuda_runtime.h>

#include "internal.h"

namespace opsblas {

__global__ void build_ptr_array_kernel(const char* base, long long stride_bytes, int count, void** out)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = const_cast<char*>(base) + i * stride_bytes;
}

static cudaError_t build_ptrs(cudaStream_t st, const void* base, long long stride_bytes, int count, void** out)
{
    if (count <= 0) return cudaSuccess;
    build_ptr_array_kernel<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(static_cast<const char*>(base),
                                                                          stride_bytes, count, out);
    return cudaGetLastError();
}

// Pointer arrays for `arrays` strided operands in the handle's workspace (256-byte aligned each).
static aclblasStatus_t strided_ptrs(const char* api, aclblasHandle_t handle, int count, int arrays, void*** out)
{
    const size_t each = (((size_t)count * sizeof(void*)) + 255) & ~(size_t)255;
    if (handle->workspace == nullptr || handle->workspace_size < each * arrays) {
        log_error(api, "workspace required %zu bytes for the pointer arrays, but only %zu available", each * arrays,
                  handle->workspace_size);
        return ACLBLAS_STATUS_EXECUTION_FAILED;
    }
    for (int a = 0; a < arrays; a++) out[a] = reinterpret_cast<void**>(static_cast<char*>(handle->workspace) + a * each);
    return ACLBLAS_STATUS_SUCCESS;
}

}  // namespace opsblas

using namespace opsblas;

extern "C" aclblasStatus_t aclblasBuildPointerArray(aclblasHandle_t handle, const void* base, long long strideBytes,
                                                    int count, void** ptrArray)
{
    static const char* kApi = "aclblasBuildPointerArray";
    if (handle == nullptr) {
        log_error(kApi, "handle is nullptr");
        return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    }
    if (count < 0) {
        log_error(kApi, "count must be >= 0, got %d", count);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (count == 0) return ACLBLAS_STATUS_SUCCESS;
    if (base == nullptr || ptrArray == nullptr) {
        log_error(kApi, "base and ptrArray must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    return launch_status(kApi, build_ptrs(handle->stream, base, strideBytes, count, ptrArray));
}

extern "C" aclblasStatus_t aclblasSgetrfStridedBatched(aclblasHandle_t handle, int n, float* A, int lda,
                                                       long long strideA, int* PivotArray, int* infoArray,
                                                       int batchSize)
{
    static const char* kApi = "aclblasSgetrfStridedBatched";
    // arguments the batched call rejects or treats as a no-op go straight to it: it returns before
    // reading any array, with the status and info it gives the same arguments
    if (handle == nullptr || n <= 0 || batchSize <= 0 || A == nullptr || lda < max1(n) ||
        (PivotArray != nullptr && infoArray == nullptr))
        return aclblasSgetrfBatched(handle, n, reinterpret_cast<float* const*>(A), lda, PivotArray, infoArray,
                                    batchSize);
    void** p[1];
    aclblasStatus_t s = strided_ptrs(kApi, handle, batchSize, 1, p);
    if (s != ACLBLAS_STATUS_SUCCESS) return s;
    s = launch_status(kApi, build_ptrs(handle->stream, A, strideA * (long long)sizeof(float), batchSize, p[0]));
    if (s != ACLBLAS_STATUS_SUCCESS) return s;
    // the blocked factorisation's stop codes after the pointer array, when the workspace holds them
    const size_t each = (((size_t)batchSize * sizeof(void*)) + 255) & ~(size_t)255;
    int* stat = handle->workspace_size >= each + sizeof(int) * (size_t)batchSize
                    ? reinterpret_cast<int*>(static_cast<char*>(handle->workspace) + each)
                    : nullptr;
    return getrf_batched_impl(handle, n, reinterpret_cast<float* const*>(p[0]), lda, PivotArray, infoArray, batchSize,
                              stat);
}

extern "C" aclblasStatus_t aclblasSgetrsStridedBatched(aclblasHandle_t handle, aclblasOperation_t trans, int n,
                                                       int nrhs, const float* A, int lda, long long strideA,
                                                       const int* devIpiv, float* B, int ldb, long long strideB,
                                                       int* info, int batchCount)
{
    static const char* kApi = "aclblasSgetrsStridedBatched";
    const bool op_ok = trans == ACLBLAS_OP_N || trans == ACLBLAS_OP_T || trans == ACLBLAS_OP_C;
    if (handle == nullptr || !op_ok || n <= 0 || nrhs <= 0 || nrhs > 256 || batchCount <= 0 || A == nullptr ||
        B == nullptr || lda < max1(n) || ldb < max1(n) || info == nullptr)
        return aclblasSgetrsBatched(handle, trans, n, nrhs, reinterpret_cast<const float* const*>(A), lda, devIpiv,
                                    reinterpret_cast<float* const*>(B), ldb, info, batchCount);
    void** p[2];
    aclblasStatus_t s = strided_ptrs(kApi, handle, batchCount, 2, p);
    if (s != ACLBLAS_STATUS_SUCCESS) return s;
    s = launch_status(kApi, build_ptrs(handle->stream, A, strideA * (long long)sizeof(float), batchCount, p[0]));
    if (s == ACLBLAS_STATUS_SUCCESS)
        s = launch_status(kApi, build_ptrs(handle->stream, B, strideB * (long long)sizeof(float), batchCount, p[1]));
    if (s != ACLBLAS_STATUS_SUCCESS) return s;
    return aclblasSgetrsBatched(handle, trans, n, nrhs, reinterpret_cast<const float* const*>(p[0]), lda, devIpiv,
                                reinterpret_cast<float* const*>(p[1]), ldb, info, batchCount);
}

extern "C" aclblasStatus_t aclblasSgetriStridedBatched(aclblasHandle_t handle, int n, const float* A, int lda,
                                                       long long strideA, const int* PivotArray, float* C, int ldc,
                                                       long long strideC, int* infoArray, int batchSize)
{
    static const char* kApi = "aclblasSgetriStridedBatched";
    if (handle == nullptr || n <= 0 || batchSize <= 0 || A == nullptr || C == nullptr || infoArray == nullptr ||
        lda < max1(n) || ldc < max1(n))
        return aclblasSgetriBatched(handle, n, reinterpret_cast<const float* const*>(A), lda, PivotArray,
                                    reinterpret_cast<float* const*>(C), ldc, infoArray, batchSize);
    void** p[2];
    aclblasStatus_t s = strided_ptrs(kApi, handle, batchSize, 2, p);
    if (s != ACLBLAS_STATUS_SUCCESS) return s;
    s = launch_status(kApi, build_ptrs(handle->stream, A, strideA * (long long)sizeof(float), batchSize, p[0]));
    if (s == ACLBLAS_STATUS_SUCCESS)
        s = launch_status(kApi, build_ptrs(handle->stream, C, strideC * (long long)sizeof(float), batchSize, p[1]));
    if (s != ACLBLAS_STATUS_SUCCESS) return s;
    return aclblasSgetriBatched(handle, n, reinterpret_cast<const float* const*>(p[0]), lda, PivotArray,
                                reinterpret_cast<float* const*>(p[1]), ldc, infoArray, batchSize);
}
