// aclblasSgetrsBatched: solve op(A) X = B from the LU factors of aclblasSgetrfBatched.
//
// Replaces blas/getrs_batched/arch35/sgetrs_batched_host.cpp:29-185 (host validation with the
// LAPACK -position info convention) and sgetrs_batched_kernel.cpp:83-446 (device). Per matrix:
//   N  : row interchanges k = 0..n-1, unit-L forward solve, U backward solve with division;
//   T/C: U^T forward solve with division, unit L^T backward solve, interchanges k = n-1..0.
// B200 kernels:
//   n <= 32, trans N, nrhs == 1 : getrs_small_kernel, rows of LU in registers, shuffle broadcasts;
//   n <= 32, otherwise : getrs_rhs_kernel, one lane per right-hand side, LU staged in shared
//                        memory by cp.async;
//   n  > 32, trans N   : getrs_trhs_kernel<false> (getrs_trhs.cu), one thread per right-hand side,
//                        for n <= 128 with at least 65536 right-hand sides in the batch; otherwise
//                        getrs_blk_kernel (getrs_blk.cu), blocked, right-hand sides in shared memory;
//   n  > 32, trans T/C : getrs_trhs_kernel (getrs_trhs.cu), one thread per right-hand side;
//   larger n than either handles: getrs_generic_kernel, one CTA per matrix in global memory.
#include <cuda_runtime.h>

#include "internal.h"
#include "getrs_small.cuh"

namespace opsblas {

// n > 32: one CTA per matrix, global memory. The row interchanges and the L^T sweep run one
// thread per right-hand side (the reference's order); the other sweeps run in parallel over
// (row, rhs) with one barrier per pivot step.
constexpr int kGenericThreads = 256;

__global__ void __launch_bounds__(kGenericThreads)
getrs_generic_kernel(const float* const* __restrict__ Aarray, int n, int lda, const int* __restrict__ ipiv,
                     float* const* __restrict__ Barray, int ldb, int nrhs, int trans)
{
    const long long m = blockIdx.x;
    const float* A = Aarray[m];
    float* B = Barray[m];
    if (B == nullptr) return;  // a NULL right-hand side skips the matrix
    const int* p = ipiv ? ipiv + m * n : nullptr;
    const int tid = threadIdx.x;
    __shared__ float sx[256];
    auto at = [&](int i, int j) { return A[i + (long long)j * lda]; };
    auto bb = [&](int i, int c) -> float& { return B[i + (long long)c * ldb]; };

    auto swap_rows = [&](bool reverse) {
        if (!p) return;
        for (int c = tid; c < nrhs; c += kGenericThreads) {
            for (int t = 0; t < n; t++) {
                const int k = reverse ? n - 1 - t : t;
                const int pk = p[k] - 1;
                if (pk >= 0 && pk < n && pk != k) {
                    const float tmp = bb(k, c);
                    bb(k, c) = bb(pk, c);
                    bb(pk, c) = tmp;
                }
            }
        }
    };

    if (trans == 0) {
        swap_rows(false);
        __syncthreads();
        for (int j = 0; j < n - 1; j++) {
            const int rows = n - 1 - j;
            const int total = rows * nrhs;
            const float* lj = A + (long long)j * lda;
            for (int idx = tid; idx < total; idx += kGenericThreads) {
                const int c = idx / rows;
                const int i = j + 1 + idx % rows;
                bb(i, c) = fmaf(-lj[i], bb(j, c), bb(i, c));
            }
            __syncthreads();
        }
        for (int j = n - 1; j >= 0; j--) {
            const float ujj = at(j, j);
            for (int c = tid; c < nrhs; c += kGenericThreads) {
                const float v = bb(j, c) / ujj;
                bb(j, c) = v;
                sx[c] = v;
            }
            __syncthreads();
            const int total = j * nrhs;
            const float* uj = A + (long long)j * lda;
            for (int idx = tid; idx < total; idx += kGenericThreads) {
                const int c = idx / j;
                const int i = idx % j;
                bb(i, c) = fmaf(-uj[i], sx[c], bb(i, c));
            }
            __syncthreads();
        }
    } else {
        for (int j = 0; j < n; j++) {
            const float ujj = at(j, j);
            for (int c = tid; c < nrhs; c += kGenericThreads) {
                const float v = bb(j, c) / ujj;
                bb(j, c) = v;
                sx[c] = v;
            }
            __syncthreads();
            const int rows = n - 1 - j;
            const int total = rows * nrhs;
            for (int idx = tid; idx < total; idx += kGenericThreads) {
                const int c = idx / rows;
                const int i = j + 1 + idx % rows;
                bb(i, c) = fmaf(-at(j, i), sx[c], bb(i, c));
            }
            __syncthreads();
        }
        for (int c = tid; c < nrhs; c += kGenericThreads) {
            for (int j = n - 1; j >= 0; j--) {
                float s = bb(j, c);
                const float* lj = A + (long long)j * lda;
                for (int i = j + 1; i < n; i++) s = fmaf(-lj[i], bb(i, c), s);
                bb(j, c) = s;
            }
        }
        __syncthreads();
        swap_rows(true);
    }
}

}  // namespace opsblas

namespace opsblas {

cudaError_t getrs_launch(cudaStream_t st, bool tr, int n, int nrhs, const float* const* Aarray, int lda,
                         const int* devIpiv, float* const* Barray, int ldb, int batchCount)
{
    if (n <= 32) {
        if (tr)
            getrs_small_dispatch_t(n, st, Aarray, lda, devIpiv, Barray, ldb, nrhs, batchCount);
        else
            getrs_small_dispatch_n(n, st, Aarray, lda, devIpiv, Barray, ldb, nrhs, batchCount);
    } else if (!tr && getrs_nrhs_preferred(n, nrhs, batchCount)) {
        return getrs_nrhs_launch(st, n, nrhs, Aarray, lda, devIpiv, Barray, ldb, batchCount);
    } else if (!tr && getrs_blk_supported(n)) {
        return getrs_blk_launch(st, n, nrhs, Aarray, lda, devIpiv, Barray, ldb, batchCount);
    } else if (tr && getrs_trhs_supported(n)) {
        return getrs_trhs_launch(st, n, nrhs, Aarray, lda, devIpiv, Barray, ldb, batchCount);
    } else {
        getrs_generic_kernel<<<(unsigned)batchCount, kGenericThreads, 0, st>>>(Aarray, n, lda, devIpiv, Barray, ldb,
                                                                               nrhs, tr ? 1 : 0);
    }
    return cudaGetLastError();
}

}  // namespace opsblas

using namespace opsblas;

namespace {

// LAPACK argument positions of aclblasSgetrsBatched (sgetrs_batched_host.cpp:29-40).
constexpr int kPosTrans = 2, kPosN = 3, kPosNrhs = 4, kPosAarray = 5, kPosLda = 6, kPosBarray = 8, kPosLdb = 9,
              kPosBatch = 11;
constexpr int kMaxNrhs = 256;

inline void set_info(int* info, int v)
{
    if (info) *info = v;
}

}  // namespace

extern "C" aclblasStatus_t aclblasSgetrsBatched(
    aclblasHandle_t handle, aclblasOperation_t trans, int n, int nrhs, const float* const Aarray[], int lda,
    const int* devIpiv, float* const Barray[], int ldb, int* info, int batchCount)
{
    static const char* kApi = "aclblasSgetrsBatched";
    if (handle == nullptr) {
        log_error(kApi, "handle is nullptr");
        return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    }
    // Validation order of ValidateSgetrsBatchedParams (sgetrs_batched_host.cpp:49-95).
    if (trans != ACLBLAS_OP_N && trans != ACLBLAS_OP_T && trans != ACLBLAS_OP_C) {
        log_error(kApi, "trans must be OP_N(111), OP_T(112) or OP_C(113), got %d", (int)trans);
        set_info(info, -kPosTrans);
        return ACLBLAS_STATUS_INVALID_ENUM;
    }
    if (n < 0) {
        log_error(kApi, "n must be >= 0, got %d", n);
        set_info(info, -kPosN);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (nrhs < 0 || nrhs > kMaxNrhs) {
        log_error(kApi, "nrhs must be in [0, %d], got %d", kMaxNrhs, nrhs);
        set_info(info, -kPosNrhs);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (n > 0 && nrhs > 0 && batchCount > 0 && Aarray == nullptr) {
        log_error(kApi, "Aarray must not be nullptr");
        set_info(info, -kPosAarray);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (lda < max1(n)) {
        log_error(kApi, "lda must be >= max(1, n), got lda=%d, n=%d", lda, n);
        set_info(info, -kPosLda);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (n > 0 && nrhs > 0 && batchCount > 0 && Barray == nullptr) {
        log_error(kApi, "Barray must not be nullptr");
        set_info(info, -kPosBarray);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (ldb < max1(n)) {
        log_error(kApi, "ldb must be >= max(1, n), got ldb=%d, n=%d", ldb, n);
        set_info(info, -kPosLdb);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (batchCount < 0) {
        log_error(kApi, "batchCount must be >= 0, got %d", batchCount);
        set_info(info, -kPosBatch);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    set_info(info, 0);
    if (n == 0 || nrhs == 0 || batchCount == 0) return ACLBLAS_STATUS_SUCCESS;

    return launch_status(kApi, getrs_launch(handle->stream, trans != ACLBLAS_OP_N, n, nrhs, Aarray, lda, devIpiv,
                                            Barray, ldb, batchCount));
}
