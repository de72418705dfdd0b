// aclblasSgeqrfBatched: batched Householder QR, FP32, column-major, LAPACK storage (R in the
// upper triangle, the Householder vectors below the diagonal with an implicit unit head, tau).
//
// Replaces blas/geqrf_batched/arch35/sgeqrf_batched_host.cpp:19-141 (host) and
// sgeqrf_batched_kernel.cpp:44-190 (device) of the reference. Its arithmetic, per column i:
// sigma = sum_{r>i} A(r,i)^2; sigma == 0 gives tau = 0 and no update; otherwise
// alpha = -sign(x1) sqrt(sigma + x1^2), tau = (alpha - x1) / alpha, v = A(i+1:, i) / (x1 - alpha),
// A(i,i) = alpha, and every column c > i gets dot = A(i,c) + v . A(i+1:, c), coef = tau * dot,
// A(i+1:, c) -= coef v, A(i,c) -= coef. The reference sums by thread trees; these kernels sum in
// row order with every product rounded before it is added (no contraction), the order of the
// CPU oracle they match bit for bit. Parity with the reference is its own test rule:
// MIXED_TOLERANCE against LAPACK sgeqrf_.
//   m, n <= 32 : geqrf_col_kernel<M>, one warp per matrix, lane c = column c in registers (every
//                sum local, in row order), the reflector published through shared memory with
//                its divisions one row per lane, the column update in packed f32x2 operations;
//   otherwise  : geqrf_generic_kernel, one CTA per matrix in global memory (correctness path):
//                thread 0 forms the reflector, thread t updates columns i+1+t, i+1+t+256, ...
#include <cuda_runtime.h>

#include <utility>

#include "internal.h"
#include "small_common.cuh"

namespace opsblas {

constexpr int kQrWarps = 8;

// Reflector I of the warp's matrix. Lane c holds column c (rows in registers, M = m rows); every
// sum runs locally in row order, so the arithmetic is the row-order restatement's. The reflector's
// divisions are shared out one row per lane through the warp's shared-memory column buffer.
template <int M, int I>
__device__ __forceinline__ void qr_col_step(float (&col)[M], float& mytau, float* vb, int lane, int n)
{
    // sigma = sum_{r>I} A(r,I)^2 (every lane forms it for its own column; lane I's is used)
    float sigma = 0.0f;
#pragma unroll
    for (int r = I + 1; r < M; r++) sigma = __fadd_rn(sigma, __fmul_rn(col[r], col[r]));
    sigma = __shfl_sync(0xffffffffu, sigma, I);
    const float x1 = __shfl_sync(0xffffffffu, col[I], I);
    float t, alpha;
    if (sigma == 0.0f) {
        t = 0.0f;
        alpha = x1;
    } else {
        const float normx = sqrtf(__fadd_rn(sigma, __fmul_rn(x1, x1)));
        alpha = x1 >= 0.0f ? -normx : normx;
        t = __fdiv_rn(__fsub_rn(alpha, x1), alpha);
    }
    if (lane == I) mytau = t;
    if (t == 0.0f) return;  // uniform: A(I,I) stays x1 == alpha, no update
    const float vscale = __fsub_rn(x1, alpha);
    // v_r = A(r,I) / vscale for r > I: lane I publishes its column, lane r divides row r
    if (lane == I) {
#pragma unroll
        for (int r = I + 1; r < M; r++) vb[r] = col[r];
    }
    __syncwarp();
    if (lane > I && lane < M) vb[lane] = __fdiv_rn(vb[lane], vscale);
    __syncwarp();
    float v[M];
#pragma unroll
    for (int r = I + 1; r < M; r++) v[r] = vb[r];
    if (lane == I) {
        col[I] = alpha;
#pragma unroll
        for (int r = I + 1; r < M; r++) col[r] = v[r];
    } else if (lane > I && lane < n) {
        // dot = A(I,c) + sum_{r>I} v_r A(r,c) in row order, then A(r,c) -= coef v_r, A(I,c) -= coef
        float dot = col[I];
#pragma unroll
        for (int r = I + 1; r < M; r++) dot = __fadd_rn(dot, __fmul_rn(v[r], col[r]));
        const float coef = __fmul_rn(t, dot);
        const float2 cc = make_float2(coef, coef);
        int r = I + 1;
#pragma unroll
        for (; r + 1 < M; r += 2) {
            const float2 p = __fmul2_rn(cc, make_float2(v[r], v[r + 1]));
            const float2 q = __fadd2_rn(make_float2(col[r], col[r + 1]), make_float2(-p.x, -p.y));
            col[r] = q.x;
            col[r + 1] = q.y;
        }
        if (r < M) col[r] = __fsub_rn(col[r], __fmul_rn(coef, v[r]));
        col[I] = __fsub_rn(col[I], coef);
    }
    __syncwarp();  // the buffer is read before the next reflector writes it
}

// Reflectors 0 .. min(m, n) - 1, one instantiation per row index.
template <int M, int... I>
__device__ __forceinline__ void qr_col_all(float (&col)[M], float& mytau, float* vb, int lane, int n,
                                           std::integer_sequence<int, I...>)
{
    ((I < n ? qr_col_step<M, I>(col, mytau, vb, lane, n) : void()), ...);
}

template <int M>
__global__ void __launch_bounds__(kQrWarps * 32)
geqrf_col_kernel(float* const* __restrict__ Aarray, int n, int lda, float* const* __restrict__ TauArray, int batch)
{
    __shared__ float vbuf[kQrWarps][32];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long b = (long long)blockIdx.x * kQrWarps + warp;
    if (b >= batch) return;  // warp-uniform
    float* A = Aarray[b];
    float* tau = TauArray[b];
    const bool cv = lane < n;
    float col[M];
    const float* Ac = A + (long long)lane * lda;
#pragma unroll
    for (int r = 0; r < M; r++) col[r] = cv ? Ac[r] : 0.0f;
    float mytau = 0.0f;
    qr_col_all<M>(col, mytau, vbuf[warp], lane, n, std::make_integer_sequence<int, M>{});
    if (cv) {
        float* Aw = A + (long long)lane * lda;
#pragma unroll
        for (int r = 0; r < M; r++) Aw[r] = col[r];
    }
    if (lane < M && lane < n) tau[lane] = mytau;
}

constexpr int kQrThreads = 256;

__global__ void __launch_bounds__(kQrThreads)
geqrf_generic_kernel(float* const* __restrict__ Aarray, int m, int n, int lda, float* const* __restrict__ TauArray)
{
    __shared__ float s_par[3];  // tau, alpha, x1 - alpha
    float* A = Aarray[blockIdx.x];
    float* tau = TauArray[blockIdx.x];
    const int tid = threadIdx.x;
    const int k = m < n ? m : n;
    for (int i = 0; i < k; i++) {
        float* ci = A + (long long)i * lda;
        if (tid == 0) {
            float sigma = 0.0f;
            for (int r = i + 1; r < m; r++) sigma = __fadd_rn(sigma, __fmul_rn(ci[r], ci[r]));
            const float x1 = ci[i];
            float t, alpha;
            if (sigma == 0.0f) {
                t = 0.0f;
                alpha = x1;
            } else {
                const float normx = sqrtf(__fadd_rn(sigma, __fmul_rn(x1, x1)));
                alpha = x1 >= 0.0f ? -normx : normx;
                t = __fdiv_rn(__fsub_rn(alpha, x1), alpha);
            }
            tau[i] = t;
            s_par[0] = t;
            s_par[1] = alpha;
            s_par[2] = __fsub_rn(x1, alpha);
        }
        __syncthreads();
        const float t = s_par[0], alpha = s_par[1], vscale = s_par[2];
        if (t != 0.0f) {
            for (int r = i + 1 + tid; r < m; r += kQrThreads) ci[r] = __fdiv_rn(ci[r], vscale);
            __syncthreads();
            for (int c = i + 1 + tid; c < n; c += kQrThreads) {
                float* cc = A + (long long)c * lda;
                float dot = cc[i];
                for (int r = i + 1; r < m; r++) dot = __fadd_rn(dot, __fmul_rn(ci[r], cc[r]));
                const float coef = __fmul_rn(t, dot);
                for (int r = i + 1; r < m; r++) cc[r] = __fsub_rn(cc[r], __fmul_rn(coef, ci[r]));
                cc[i] = __fsub_rn(cc[i], coef);
            }
            if (tid == 0) ci[i] = alpha;
        }
        __syncthreads();  // s_par and column i+1 ready for the next step
    }
}

}  // namespace opsblas

using namespace opsblas;

extern "C" aclblasStatus_t aclblasSgeqrfBatched(aclblasHandle_t handle, int m, int n, float* const Aarray[], int lda,
                                                float* const TauArray[], int* info, int batchSize)
{
    static const char* kApi = "aclblasSgeqrfBatched";
    if (handle == nullptr) {
        log_error(kApi, "handle is nullptr");
        return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    }
    if (info == nullptr) {
        log_error(kApi, "info must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    // ValidateGeqrfBatchedParams (sgeqrf_batched_host.cpp:21-58): LAPACK-style -position in the
    // host info, counting m=1, n=2, Aarray=3, lda=4, TauArray=5, batchSize=6.
    if (m < 0) {
        log_error(kApi, "m must be >= 0, got %d", m);
        *info = ACLBLAS_LAPACK_INFO_ARG_1;
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (n < 0) {
        log_error(kApi, "n must be >= 0, got %d", n);
        *info = ACLBLAS_LAPACK_INFO_ARG_2;
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (lda < max1(m)) {
        log_error(kApi, "lda must be >= max(1, m), got lda=%d, m=%d", lda, m);
        *info = ACLBLAS_LAPACK_INFO_ARG_4;
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (batchSize < 0) {
        log_error(kApi, "batchSize must be >= 0, got %d", batchSize);
        *info = ACLBLAS_LAPACK_INFO_ARG_6;
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (batchSize > 0 && Aarray == nullptr) {
        log_error(kApi, "Aarray must not be nullptr when batchSize > 0");
        *info = ACLBLAS_LAPACK_INFO_ARG_3;
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (batchSize > 0 && m > 0 && n > 0 && TauArray == nullptr) {
        log_error(kApi, "TauArray must not be nullptr when batchSize > 0 and min(m,n) > 0");
        *info = ACLBLAS_LAPACK_INFO_ARG_5;
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (m == 0 || n == 0 || batchSize == 0) {
        *info = ACLBLAS_LAPACK_INFO_OK;
        return ACLBLAS_STATUS_SUCCESS;
    }

    cudaStream_t st = handle->stream;
    if (m <= 32 && n <= 32) {
        const unsigned grid = (unsigned)((batchSize + kQrWarps - 1) / kQrWarps);
        switch (m) {
#define OPSBLAS_GEQRF_CASE(MM)                                                                                      \
    case MM:                                                                                                        \
        geqrf_col_kernel<MM><<<grid, kQrWarps * 32, 0, st>>>(Aarray, n, lda, TauArray, batchSize);                  \
        break;
            OPSBLAS_FOR_N_1_32(OPSBLAS_GEQRF_CASE)
#undef OPSBLAS_GEQRF_CASE
            default:
                break;
        }
    } else {
        geqrf_generic_kernel<<<(unsigned)batchSize, kQrThreads, 0, st>>>(Aarray, m, n, lda, TauArray);
    }
    const aclblasStatus_t status = launch_status(kApi, cudaGetLastError());
    if (status == ACLBLAS_STATUS_SUCCESS) *info = ACLBLAS_LAPACK_INFO_OK;
    return status;
}
