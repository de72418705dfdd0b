// aclblasSmatinvBatched: the inverse of every matrix of a batch, n <= 32, in one launch.
//
// Replaces blas/matinv_batched/arch35/matinv_batched_host.cpp:44-257 of the reference, which runs
// five launches on the stream: build a pointer array into the handle's workspace, copy A to
// Ainv, getrf in place on Ainv (pivots into the workspace), copy the factors to the workspace,
// getri from the workspace into Ainv -- the getri writes its info over the getrf's. Here one
// warp segment per matrix does the same work without leaving the chip: it loads A into registers
// (one row per lane), factors it with small_getrf_core (the batched getrf's arithmetic), stages
// LU at the rows' final positions and the pivots in shared memory, solves the columns of the
// inverse with getri_small_solve (the batched getri's arithmetic) and stores Ainv once. Ainv and
// info are bit-identical to aclblasSgetrfBatched followed by aclblasSgetriBatched on a copy of A
// (singular matrices included: info is then the getri's, the highest zero U(j,j) + 1, and Ainv
// holds what that getri leaves). HBM traffic is one read of A and one write of Ainv, where the
// reference's sequence moves every matrix eight times. No workspace is used, so the reference's
// workspace-size failure (EXECUTION_FAILED) cannot occur; A may be the same matrices as Ainv when
// lda == lda_inv (A is read completely before Ainv is written).
#include <cuda_runtime.h>

#include "getri_small.cuh"
#include "internal.h"
#include "lu_core.cuh"
#include "small_common.cuh"

namespace opsblas {

template <int N>
__global__ void __launch_bounds__(kSmallWarps * 32, N > 16 ? 3 : 4)
matinv_small_kernel(const float* const* __restrict__ Aarray, int lda, float* const* __restrict__ Carray, int ldc,
                    int* __restrict__ info, int batch)
{
    using S = SmallShape<N>;
    constexpr int NC = S::NC;
    constexpr int NP = S::NP;
    constexpr int MAT = N * NP + 4;  // staged LU of one matrix (columns of NP floats)
    __shared__ __align__(16) float lu_s[kSmallWarps][S::MPW][MAT];
    __shared__ __align__(16) float rowbuf[kSmallWarps][2][32];
    __shared__ __align__(16) int pbuf[kSmallWarps][32];

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int seg = lane / S::SEG;
    const int r = lane % S::SEG;
    const long long m = ((long long)blockIdx.x * kSmallWarps + warp) * S::MPW + seg;
    const bool mvalid = m < batch;
    const bool rvalid = mvalid && r < N;

    // row r in registers (coalesced column-wise loads), then the getrf
    float4 a4[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) a4[c] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (rvalid) {
        const float* Ar = Aarray[m] + r;
#pragma unroll
        for (int j = 0; j < N; j++) qset<N>(a4, j, Ar[(long long)j * lda]);
    }
    int pos, mypiv, inf;
    small_getrf_core<N, true, S::SEG>(a4, pos, mypiv, inf, &rowbuf[warp][0][0], seg, r, mvalid, rvalid);

    // LU at the rows' final positions (what the getrf stores), column-major with stride NP;
    // the pivots as the getrf writes them (0 after a zero pivot)
    float* sm = lu_s[warp][seg];
    if (rvalid) {
#pragma unroll
        for (int j = 0; j < N; j++) sm[pos + j * NP] = qget<N>(a4, j);
    }
    int* pv = &pbuf[warp][seg * S::SEG];
    if (r < N) pv[r] = mypiv;
    __syncwarp();

    float2 x2[NP / 2];
    const int inf2 = getri_small_solve<N>(sm, pv, r, rvalid, x2);
    getri_small_store<N>(sm, x2, r, rvalid, mvalid, mvalid ? Carray[m] : nullptr, ldc);
    if (mvalid && r == 0) info[m] = inf2;
}

}  // namespace opsblas

using namespace opsblas;

extern "C" aclblasStatus_t aclblasSmatinvBatched(aclblasHandle_t handle, int n, const float* const A[], int lda,
                                                 float* const Ainv[], int lda_inv, int* info, int batchSize)
{
    static const char* kApi = "aclblasSmatinvBatched";
    if (handle == nullptr) {
        log_error(kApi, "handle is nullptr");
        return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    }
    // Validation order of ValidateSmatinvBatchedParams (matinv_batched_host.cpp:44-87).
    if (n < 0) {
        log_error(kApi, "n must be >= 0, got %d", n);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (n > 32) {
        log_error(kApi, "n must be <= 32, got %d", n);
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
    if (lda_inv < max1(n)) {
        log_error(kApi, "lda_inv must be >= max(1, n), got lda_inv=%d, n=%d", lda_inv, n);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (n == 0 || batchSize == 0) return ACLBLAS_STATUS_SUCCESS;
    if (A == nullptr) {
        log_error(kApi, "A must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (Ainv == nullptr) {
        log_error(kApi, "Ainv must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (info == nullptr) {
        log_error(kApi, "info must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }

    cudaStream_t st = handle->stream;
    switch (n) {
#define OPSBLAS_MATINV_CASE(NN)                                                                                     \
    case NN: {                                                                                                      \
        constexpr int per_cta = kSmallWarps * SmallShape<NN>::MPW;                                                  \
        const unsigned grid = (unsigned)((batchSize + per_cta - 1) / per_cta);                                      \
        matinv_small_kernel<NN><<<grid, kSmallWarps * 32, 0, st>>>(A, lda, Ainv, lda_inv, info, batchSize);         \
        break;                                                                                                      \
    }
        OPSBLAS_FOR_N_1_32(OPSBLAS_MATINV_CASE)
#undef OPSBLAS_MATINV_CASE
        default:
            break;
    }
    return launch_status(kApi, cudaGetLastError());
}
