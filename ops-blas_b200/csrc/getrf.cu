// aclblasSgetrfBatched: batched LU factorisation with partial pivoting, FP32, column-major.
//
// Replaces blas/getrf_batched/arch35/sgetrf_batched_host.cpp:32-118 (host) and
// sgetrf_batched_kernel.cpp:38-221 (device) of the reference. The arithmetic is the
// reference's unblocked right-looking LU: first-maximum pivot search (FindPivotRow :52-79),
// full-row interchange (SwapRows :81-91), multipliers by true division (ComputeMultipliers
// :93-104), rank-1 update (Rank1Update :38-50), stop at the first exactly-zero pivot
// (:127-137). The B200 kernels are:
//   n <= 32 : getrf_small_kernel, one warp segment per matrix, rows in registers;
//   32 < n <= 128 : getrf_reg_kernel (getrf_reg.cu), matrix in registers across the CTA;
//   128 < n <= 1024 : the blocked LU on a by-rows copy made in place (getrf_blocked_tc.cu:
//                     panel kernels and a tiled trailing update), given 4 bytes of handle
//                     workspace per matrix; without them getrf_large_kernel (getrf_large.cu,
//                     n <= 640, blocked, one CTA per matrix in global memory);
//   otherwise : getrf_generic_kernel, one CTA per matrix, unblocked in global memory.
#include <cuda_runtime.h>

#include "internal.h"
#include "lu_core.cuh"
#include "small_common.cuh"

namespace opsblas {

// ---------------------------------------------------------------------------------------
// n <= 32: one warp segment per matrix, rows in registers (small_getrf_core, lu_core.cuh).
// The lane of row r loads it with coalesced column-wise loads and stores it at its final
// position. LD = N compiles the contiguous case (lda == n) with constant strides; with one
// matrix per warp (n > 16) a warp past the batch leaves at once, so no per-lane validity state
// is carried through the factorisation.
// ---------------------------------------------------------------------------------------
template <int N, bool PIVOT, int LD>
__global__ void __launch_bounds__(kSmallWarps * 32, N > 16 ? 4 : (N > 8 ? 5 : 6))
getrf_small_kernel(float* const* __restrict__ Aarray, int lda_rt, int* __restrict__ piv, int* __restrict__ info,
                   int batch)
{
    using S = SmallShape<N>;
    constexpr int NC = S::NC;
    __shared__ __align__(16) float rowbuf[kSmallWarps][2][32];

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int seg = lane / S::SEG;
    const int r = lane % S::SEG;
    const long long m = ((long long)blockIdx.x * kSmallWarps + warp) * S::MPW + seg;
    if (S::SEG == 32 && m >= batch) return;  // warp-uniform: the warp's only matrix is past the batch
    const bool mvalid = S::SEG == 32 ? true : m < batch;
    const bool rvalid = mvalid && r < N;
    const int lda = LD > 0 ? LD : lda_rt;

    // Row r in registers as float4 chunks (contiguous quads: published with one 16-byte store,
    // updated two columns per packed fma); padding entries stay zero.
    float* A = mvalid ? Aarray[m] : nullptr;
    float4 a4[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) a4[c] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (rvalid) {
        const float* Ar = A + r;
#pragma unroll
        for (int j = 0; j < N; j++) qset<N>(a4, j, Ar[(long long)j * lda]);
    }

    int pos, mypiv, inf;
    small_getrf_core<N, PIVOT, S::SEG>(a4, pos, mypiv, inf, &rowbuf[warp][0][0], seg, r, mvalid, rvalid);

    if (rvalid) {
        float* Ap = A + pos;
#pragma unroll
        for (int j = 0; j < N; j++) Ap[(long long)j * lda] = qget<N>(a4, j);
        if (PIVOT) piv[m * N + r] = mypiv;
        if (r == 0 && info != nullptr) info[m] = inf;
    }
}

// ---------------------------------------------------------------------------------------
// n > 32: one CTA per matrix working in global memory (L1/L2 resident). Warp 0 searches the
// pivot, the CTA swaps rows, forms multipliers, and applies the rank-1 update with one thread
// per trailing row (coalesced along the column).
// ---------------------------------------------------------------------------------------
constexpr int kGenericThreads = 256;

template <bool PIVOT>
__global__ void __launch_bounds__(kGenericThreads)
getrf_generic_kernel(float* const* __restrict__ Aarray, int n, int lda, int* __restrict__ piv, int* __restrict__ info)
{
    const long long m = blockIdx.x;
    float* A = Aarray[m];
    int* pm = PIVOT ? piv + m * n : nullptr;
    __shared__ int s_prow;
    __shared__ float s_pv;
    const int tid = threadIdx.x;
    int inf = 0;
    int k;
    for (k = 0; k < n; k++) {
        const float* colk = A + (long long)k * lda;
        if (PIVOT) {
            if (tid < 32) {
                float best = 0.0f;
                int brow = k;
                for (int rr = k + tid; rr < n; rr += 32) {
                    const float v = fabsf(colk[rr]);
                    if (v > best) {
                        best = v;
                        brow = rr;
                    }
                }
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    const float ob = __shfl_xor_sync(0xffffffffu, best, off);
                    const int orow = __shfl_xor_sync(0xffffffffu, brow, off);
                    if (ob > best || (ob == best && orow < brow)) {
                        best = ob;
                        brow = orow;
                    }
                }
                if (tid == 0) {
                    s_prow = brow;
                    s_pv = colk[brow];
                }
            }
        } else if (tid == 0) {
            s_prow = k;
            s_pv = colk[k];
        }
        __syncthreads();
        const int p = s_prow;
        const float pv = s_pv;
        if (PIVOT && tid == 0) pm[k] = p + 1;
        if (pv == 0.0f) {
            inf = k + 1;
            break;
        }
        if (p != k) {
            for (int c = tid; c < n; c += kGenericThreads) {
                float* col = A + (long long)c * lda;
                const float t = col[k];
                col[k] = col[p];
                col[p] = t;
            }
        }
        __syncthreads();
        float* ck = A + (long long)k * lda;
        for (int i = k + 1 + tid; i < n; i += kGenericThreads) {
            const float l = ck[i] / pv;
            ck[i] = l;
            for (int j = k + 1; j < n; j++) {
                float* cj = A + (long long)j * lda;
                cj[i] = fmaf(-l, cj[k], cj[i]);
            }
        }
        __syncthreads();
    }
    if (PIVOT && inf) {
        for (int kk = k + 1 + tid; kk < n; kk += kGenericThreads) pm[kk] = 0;
    }
    if (tid == 0 && info != nullptr) info[m] = inf;
}

}  // namespace opsblas

using namespace opsblas;

// The body of aclblasSgetrfBatched; stat: batchSize ints of device scratch for the blocked path
// (nullptr: that path is not taken).
aclblasStatus_t opsblas::getrf_batched_impl(aclblasHandle_t handle, int n, float* const Aarray[], int lda,
                                            int* PivotArray, int* infoArray, int batchSize, int* stat)
{
    static const char* kApi = "aclblasSgetrfBatched";
    if (handle == nullptr) {
        log_error(kApi, "handle is nullptr");
        return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    }
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
    if (n == 0 || batchSize == 0) return ACLBLAS_STATUS_SUCCESS;
    if (Aarray == nullptr) {
        log_error(kApi, "Aarray must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (PivotArray != nullptr && infoArray == nullptr) {
        log_error(kApi, "infoArray must not be nullptr when PivotArray is provided");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }

    cudaStream_t st = handle->stream;
    const bool pivot = PivotArray != nullptr;
    if (n <= 32) {
        switch (n) {
#define OPSBLAS_GETRF_CASE(NN)                                                                                      \
    case NN: {                                                                                                      \
        constexpr int per_cta = kSmallWarps * SmallShape<NN>::MPW;                                                  \
        const unsigned grid = (unsigned)((batchSize + per_cta - 1) / per_cta);                                      \
        constexpr int ld_c = NN > 16 ? NN : 0; /* contiguous variant for one matrix per warp */                      \
        if (ld_c > 0 && lda == NN) {                                                                                \
            if (pivot)                                                                                              \
                getrf_small_kernel<NN, true, ld_c><<<grid, kSmallWarps * 32, 0, st>>>(Aarray, lda, PivotArray,      \
                                                                                     infoArray, batchSize);         \
            else                                                                                                    \
                getrf_small_kernel<NN, false, ld_c><<<grid, kSmallWarps * 32, 0, st>>>(Aarray, lda, nullptr,        \
                                                                                      infoArray, batchSize);        \
        } else if (pivot)                                                                                           \
            getrf_small_kernel<NN, true, 0><<<grid, kSmallWarps * 32, 0, st>>>(Aarray, lda, PivotArray, infoArray,  \
                                                                               batchSize);                          \
        else                                                                                                        \
            getrf_small_kernel<NN, false, 0><<<grid, kSmallWarps * 32, 0, st>>>(Aarray, lda, nullptr, infoArray,    \
                                                                                batchSize);                         \
        break;                                                                                                      \
    }
            OPSBLAS_FOR_N_1_32(OPSBLAS_GETRF_CASE)
#undef OPSBLAS_GETRF_CASE
            default:
                break;
        }
    } else if (getrf_reg_supported(n)) {
        int rows, warps;
        reg_default_shape(n, rows, warps);
        return launch_status(kApi, getrf_reg_launch(st, Aarray, n, lda, PivotArray, infoArray, batchSize, rows,
                                                    warps));
    } else if (getrf_rows_supported(n, batchSize) && stat != nullptr) {
        return launch_status(kApi, getrf_rows_launch(st, Aarray, n, lda, PivotArray, infoArray, stat, batchSize));
    } else if (getrf_large_supported(n)) {
        return launch_status(kApi, getrf_large_launch(st, Aarray, n, lda, PivotArray, infoArray, batchSize));
    } else {
        if (pivot)
            getrf_generic_kernel<true><<<(unsigned)batchSize, kGenericThreads, 0, st>>>(Aarray, n, lda, PivotArray,
                                                                                      infoArray);
        else
            getrf_generic_kernel<false><<<(unsigned)batchSize, kGenericThreads, 0, st>>>(Aarray, n, lda, nullptr,
                                                                                       infoArray);
    }
    return launch_status(kApi, cudaGetLastError());
}

extern "C" aclblasStatus_t aclblasSgetrfBatched(
    aclblasHandle_t handle, int n, float* const Aarray[], int lda, int* PivotArray, int* infoArray, int batchSize)
{
    // the blocked path keeps the matrices' stop codes in the first 4 * batchSize workspace bytes
    int* stat = nullptr;
    if (handle != nullptr && batchSize > 0 && handle->workspace != nullptr &&
        handle->workspace_size >= sizeof(int) * (size_t)batchSize)
        stat = static_cast<int*>(handle->workspace);
    return getrf_batched_impl(handle, n, Aarray, lda, PivotArray, infoArray, batchSize, stat);
}
