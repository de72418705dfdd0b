// aclblasSgetriBatched: inverse from the LU factors of aclblasSgetrfBatched, out of place.
//
// Replaces blas/getri_batched/arch35/getri_batched_host.cpp:27-127 (host) and
// getri_batched_kernel.cpp:39-308 (device). Per matrix, column by column of C:
// C = I, row interchanges, unit-L forward solve, U backward solve j = n-1..0 that stops at the
// first zero U(j,j) it meets (so info is the highest zero diagonal index + 1). On that stop
// the reference leaves C as the forward-solve result for n <= 8 (its register path,
// :163-168) and partially back-substituted for n > 8; both are kept.
// B200 kernels:
//   n <= 32 : getri_small_kernel. LU of each matrix is staged in shared memory (cp.async),
//             lane c of a warp segment solves column c of C in registers (two rows per packed
//             f32x2 FMA) reading L/U with broadcast 16-byte loads, and C leaves through shared
//             memory as coalesced column stores.
//   n  > 32 : getri_generic_kernel, thread per column of C in global memory.
#include <cuda_runtime.h>

#include "internal.h"
#include "getri_small.cuh"
#include "small_common.cuh"

namespace opsblas {

template <int N>
__global__ void __launch_bounds__(kSmallWarps * 32, N > 16 ? 3 : 4)
getri_small_kernel(const float* const* __restrict__ Aarray, int lda, const int* __restrict__ ipiv,
                   float* const* __restrict__ Carray, int ldc, int* __restrict__ info, int batch)
{
    using S = SmallShape<N>;
    constexpr int NP = S::NP;
    constexpr int NC = S::NC;
    constexpr int NPAIR = NP / 2;
    // Per matrix: N columns of NP floats. LU is staged column-major (16-byte aligned columns
    // for the float4 broadcast reads). C is staged in the same space with the 16-byte chunks
    // of column c rotated by c (chunk q of column c at slot (q + c) % NC), so that the 32
    // lanes writing their columns chunk-wise hit distinct banks. Matrices are 16 bytes apart
    // modulo 128 so that the broadcast reads of different segments use different banks.
    constexpr int MAT = N * NP + 4;
    __shared__ __align__(16) float lu_s[kSmallWarps][S::MPW][MAT];
    __shared__ __align__(16) int pbuf[kSmallWarps][32];

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int seg = lane / S::SEG;
    const int r = lane % S::SEG;
    const long long m = ((long long)blockIdx.x * kSmallWarps + warp) * S::MPW + seg;
    const bool mvalid = m < batch;
    const bool cvalid = mvalid && r < N;
    float* sm = lu_s[warp][seg];

    if (mvalid) {
        const float* A = Aarray[m];
        if (N % 4 == 0 && (lda & 3) == 0 && (reinterpret_cast<uintptr_t>(A) & 15) == 0) {
            for (int e = r; e < N * NC; e += S::SEG) {
                const int q = e % NC, j = e / NC;
                cp_async16(sm + 4 * q + j * NP, A + 4 * q + (long long)j * lda);
            }
        } else {
            for (int e = r; e < N * N; e += S::SEG) {
                const int i = e % N, j = e / N;
                cp_async4(sm + i + j * NP, A + i + (long long)j * lda);
            }
        }
    }
    int* pv = &pbuf[warp][seg * S::SEG];
    if (r < N) pv[r] = (ipiv != nullptr && mvalid) ? ipiv[m * N + r] : r + 1;
    cp_async_wait_all();
    __syncwarp();

    float2 x2[NPAIR];
    const int inf = getri_small_solve<N>(sm, pv, r, cvalid, x2);
    getri_small_store<N>(sm, x2, r, cvalid, mvalid, mvalid ? Carray[m] : nullptr, ldc);
    if (mvalid && r == 0) info[m] = inf;
}

// n > 32: thread per column of C, the reference's column-parallel structure, in global memory.
// Several CTAs share one matrix along the columns (grid.y).
constexpr int kGenericThreads = 256;

__global__ void __launch_bounds__(kGenericThreads)
getri_generic_kernel(const float* const* __restrict__ Aarray, int n, int lda, const int* __restrict__ ipiv,
                     float* const* __restrict__ Carray, int ldc, int* __restrict__ info)
{
    const long long m = blockIdx.x;
    const float* A = Aarray[m];
    float* C = Carray[m];
    const int* p = ipiv ? ipiv + m * n : nullptr;
    int inf = 0;
    for (int j = n - 1; j >= 0; j--) {
        if (A[j + (long long)j * lda] == 0.0f) {
            inf = j + 1;
            break;
        }
    }
    const int col = blockIdx.y * kGenericThreads + threadIdx.x;
    if (col < n) {
        float* x = C + (long long)col * ldc;
        for (int i = 0; i < n; i++) x[i] = (i == col) ? 1.0f : 0.0f;
        if (p) {
            for (int k = 0; k < n; k++) {
                const int pk = p[k] - 1;
                if (pk >= 0 && pk < n && pk != k) {
                    const float t = x[k];
                    x[k] = x[pk];
                    x[pk] = t;
                }
            }
        }
        for (int j = 0; j < n; j++) {
            const float xj = x[j];
            const float* lj = A + (long long)j * lda;
            for (int i = j + 1; i < n; i++) x[i] = fmaf(-lj[i], xj, x[i]);
        }
        for (int j = n - 1; j >= 0; j--) {
            const float* uj = A + (long long)j * lda;
            const float ujj = uj[j];
            if (ujj == 0.0f) break;
            const float xj = x[j] / ujj;
            x[j] = xj;
            for (int i = 0; i < j; i++) x[i] = fmaf(-uj[i], xj, x[i]);
        }
    }
    if (blockIdx.y == 0 && threadIdx.x == 0) info[m] = inf;
}

}  // namespace opsblas

using namespace opsblas;

extern "C" aclblasStatus_t aclblasSgetriBatched(
    aclblasHandle_t handle, int n, const float* const Aarray[], int lda, const int* PivotArray,
    float* const Carray[], int ldc, int* infoArray, int batchSize)
{
    static const char* kApi = "aclblasSgetriBatched";
    if (handle == nullptr) {
        log_error(kApi, "handle is nullptr");
        return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    }
    // Validation order of ValidateGetriBatchedParams (getri_batched_host.cpp:27-64).
    if (n < 0) {
        log_error(kApi, "n must be >= 0, got %d", n);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (batchSize < 0) {
        log_error(kApi, "batchSize must be >= 0, got %d", batchSize);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (lda < max1(n)) {
        log_error(kApi, "lda must be >= max(1, n), got lda=%d, n=%d", lda, n);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (ldc < max1(n)) {
        log_error(kApi, "ldc must be >= max(1, n), got ldc=%d, n=%d", ldc, n);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (n == 0 || batchSize == 0) return ACLBLAS_STATUS_SUCCESS;
    if (Aarray == nullptr) {
        log_error(kApi, "Aarray must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (Carray == nullptr) {
        log_error(kApi, "Carray must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (infoArray == nullptr) {
        log_error(kApi, "infoArray must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }

    cudaStream_t st = handle->stream;
    if (n <= 32) {
        switch (n) {
#define OPSBLAS_GETRI_CASE(NN)                                                                                      \
    case NN: {                                                                                                      \
        constexpr int per_cta = kSmallWarps * SmallShape<NN>::MPW;                                                  \
        const unsigned grid = (unsigned)((batchSize + per_cta - 1) / per_cta);                                      \
        getri_small_kernel<NN><<<grid, kSmallWarps * 32, 0, st>>>(Aarray, lda, PivotArray, Carray, ldc, infoArray,  \
                                                                  batchSize);                                       \
        break;                                                                                                      \
    }
            OPSBLAS_FOR_N_1_32(OPSBLAS_GETRI_CASE)
#undef OPSBLAS_GETRI_CASE
            default:
                break;
        }
    } else {
        dim3 grid((unsigned)batchSize, (unsigned)((n + kGenericThreads - 1) / kGenericThreads));
        getri_generic_kernel<<<grid, kGenericThreads, 0, st>>>(Aarray, n, lda, PivotArray, Carray, ldc, infoArray);
    }
    return launch_status(kApi, cudaGetLastError());
}
