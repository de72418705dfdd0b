// aclblasSgetrsBatched: solve op(A) X = B from the LU factors of aclblasSgetrfBatched.
//
// Replaces blas/getrs_batched/arch35/sgetrs_batched_host.cpp:29-185 (host validation with the
// LAPACK -position info convention) and sgetrs_batched_kernel.cpp:83-446 (device). Per matrix:
//   N  : row interchanges k = 0..n-1, unit-L forward solve, U backward solve with division;
//   T/C: U^T forward solve with division, unit L^T backward solve, interchanges k = n-1..0.
// B200 kernels:
//   n <= 32 : getrs_small_kernel. Lane r of a warp segment holds row r (N) or column r (T) of
//             LU in registers and row r of a chunk of RC right-hand sides; the interchanges
//             are folded into the row the lane loads (N) or stores (T); solution entries are
//             broadcast through a shuffle (RC == 1) or shared memory (RC == 4).
//   n  > 32 : getrs_generic_kernel, one CTA per matrix in global memory.
#include <cuda_runtime.h>

#include "internal.h"
#include "small_common.cuh"

namespace opsblas {

// Broadcast chunk x (RC floats) of lane `src` of this segment to every lane of the segment.
template <int SEG, int RC>
__device__ __forceinline__ void seg_bcast(const float (&x)[RC], float (&out)[RC], int seg, int r, int src,
                                          float* slot)
{
    if constexpr (RC == 1) {
        out[0] = __shfl_sync(0xffffffffu, x[0], seg * SEG + src);
    } else {
        if (r == src) *reinterpret_cast<float4*>(slot) = make_float4(x[0], x[1], x[2], x[3]);
        __syncwarp();
        const float4 v = *reinterpret_cast<const float4*>(slot);
        out[0] = v.x;
        out[1] = v.y;
        out[2] = v.z;
        out[3] = v.w;
    }
}

template <int N, int RC, bool TRANS>
__global__ void __launch_bounds__(kSmallWarps * 32)
getrs_small_kernel(const float* const* __restrict__ Aarray, int lda, const int* __restrict__ ipiv,
                   float* const* __restrict__ Barray, int ldb, int nrhs, int batch)
{
    using S = SmallShape<N>;
    static_assert(RC == 1 || RC == 4, "chunk of 1 or 4 right-hand sides");
    __shared__ __align__(16) float xbuf[kSmallWarps][2][S::MPW][4];
    __shared__ int pbuf[kSmallWarps][32];

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int seg = lane / S::SEG;
    const int r = lane % S::SEG;
    const long long m = ((long long)blockIdx.x * kSmallWarps + warp) * S::MPW + seg;
    const bool mvalid = m < batch;
    const bool rvalid = mvalid && r < N;

    const float* A = mvalid ? Aarray[m] : nullptr;
    float* B = mvalid ? Barray[m] : nullptr;

    float lu[N];
#pragma unroll
    for (int j = 0; j < N; j++) lu[j] = 0.0f;
    if (rvalid) {
#pragma unroll
        for (int j = 0; j < N; j++) lu[j] = TRANS ? A[j + (long long)r * lda] : A[r + (long long)j * lda];
    }

    int* pv = &pbuf[warp][seg * S::SEG];
    if (r < N) pv[r] = (ipiv != nullptr && mvalid) ? ipiv[m * N + r] : r + 1;
    __syncwarp();
    const int prow = rvalid ? trace_backward<N>(pv, r) : r;

    for (int c0 = 0; c0 < nrhs; c0 += RC) {
        float x[RC];
#pragma unroll
        for (int t = 0; t < RC; t++) {
            const int c = c0 + t;
            x[t] = (rvalid && c < nrhs) ? B[(TRANS ? r : prow) + (long long)c * ldb] : 0.0f;
        }
        int step = 0;
        float xj[RC];
        if (!TRANS) {
#pragma unroll
            for (int j = 0; j < N; j++, step++) {
                seg_bcast<S::SEG, RC>(x, xj, seg, r, j, xbuf[warp][step & 1][seg]);
                if (r > j) {
#pragma unroll
                    for (int t = 0; t < RC; t++) x[t] = fmaf(-lu[j], xj[t], x[t]);
                }
            }
#pragma unroll
            for (int j = N - 1; j >= 0; j--, step++) {
                if (r == j) {
#pragma unroll
                    for (int t = 0; t < RC; t++) x[t] = x[t] / lu[j];
                }
                seg_bcast<S::SEG, RC>(x, xj, seg, r, j, xbuf[warp][step & 1][seg]);
                if (r < j) {
#pragma unroll
                    for (int t = 0; t < RC; t++) x[t] = fmaf(-lu[j], xj[t], x[t]);
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < N; j++, step++) {
                if (r == j) {
#pragma unroll
                    for (int t = 0; t < RC; t++) x[t] = x[t] / lu[j];
                }
                seg_bcast<S::SEG, RC>(x, xj, seg, r, j, xbuf[warp][step & 1][seg]);
                if (r > j) {
#pragma unroll
                    for (int t = 0; t < RC; t++) x[t] = fmaf(-lu[j], xj[t], x[t]);
                }
            }
#pragma unroll
            for (int i = N - 1; i >= 0; i--, step++) {
                seg_bcast<S::SEG, RC>(x, xj, seg, r, i, xbuf[warp][step & 1][seg]);
                if (r < i) {
#pragma unroll
                    for (int t = 0; t < RC; t++) x[t] = fmaf(-lu[i], xj[t], x[t]);
                }
            }
        }
#pragma unroll
        for (int t = 0; t < RC; t++) {
            const int c = c0 + t;
            if (rvalid && c < nrhs) B[(TRANS ? prow : r) + (long long)c * ldb] = x[t];
        }
        __syncwarp();
    }
}

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

    cudaStream_t st = handle->stream;
    const bool tr = trans != ACLBLAS_OP_N;
    if (n <= 32) {
        switch (n) {
#define OPSBLAS_GETRS_LAUNCH(NN, RCV, TRV)                                                                          \
    getrs_small_kernel<NN, RCV, TRV><<<grid, kSmallWarps * 32, 0, st>>>(Aarray, lda, devIpiv, Barray, ldb, nrhs,    \
                                                                        batchCount)
#define OPSBLAS_GETRS_CASE(NN)                                                                                      \
    case NN: {                                                                                                      \
        constexpr int per_cta = kSmallWarps * SmallShape<NN>::MPW;                                                  \
        const unsigned grid = (unsigned)((batchCount + per_cta - 1) / per_cta);                                     \
        if (nrhs == 1) {                                                                                            \
            if (tr)                                                                                                 \
                OPSBLAS_GETRS_LAUNCH(NN, 1, true);                                                                  \
            else                                                                                                    \
                OPSBLAS_GETRS_LAUNCH(NN, 1, false);                                                                 \
        } else {                                                                                                    \
            if (tr)                                                                                                 \
                OPSBLAS_GETRS_LAUNCH(NN, 4, true);                                                                  \
            else                                                                                                    \
                OPSBLAS_GETRS_LAUNCH(NN, 4, false);                                                                 \
        }                                                                                                           \
        break;                                                                                                      \
    }
            OPSBLAS_FOR_N_1_32(OPSBLAS_GETRS_CASE)
#undef OPSBLAS_GETRS_CASE
#undef OPSBLAS_GETRS_LAUNCH
            default:
                break;
        }
    } else {
        getrs_generic_kernel<<<(unsigned)batchCount, kGenericThreads, 0, st>>>(Aarray, n, lda, devIpiv, Barray, ldb,
                                                                               nrhs, tr ? 1 : 0);
    }
    return launch_status(kApi, cudaGetLastError());
}
