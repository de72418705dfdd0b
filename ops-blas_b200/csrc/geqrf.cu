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
//   m, n <= 32 : geqrf_warp_kernel<N>, one warp per matrix, lane = row, the row in registers;
//                the column sums go through a per-warp shared-memory transpose (lane c sums
//                column c), the divisions run one per lane;
//   otherwise  : geqrf_generic_kernel, one CTA per matrix in global memory (correctness path):
//                thread 0 forms the reflector, thread t updates columns i+1+t, i+1+t+256, ...
#include <cuda_runtime.h>

#include <utility>

#include "internal.h"
#include "small_common.cuh"

namespace opsblas {

constexpr int kQrWarps = 8;
constexpr int kQrStride = 33;  // row stride of the per-warp transpose buffer (conflict-free columns)

// Reflector i of the warp's matrix (lane = row, the row in a[]); I is a template parameter so that
// every register index is a compile-time constant.
template <int N, int I>
__device__ __forceinline__ void qr_warp_step(float (&a)[N], float& mytau, float* xw, float* cw, int lane, int m,
                                             bool rv)
{
    // sigma = sum_{r>i} A(r,i)^2 in row order (lane i)
    cw[lane] = a[I];
    __syncwarp();
    float sigma = 0.0f;
    if (lane == I) {
        for (int r = I + 1; r < m; r++) {
            const float x = cw[r];
            sigma = __fadd_rn(sigma, __fmul_rn(x, x));
        }
    }
    sigma = __shfl_sync(0xffffffffu, sigma, I);
    const float x1 = __shfl_sync(0xffffffffu, a[I], I);
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
    __syncwarp();  // column i read before the buffer is reused
    if (t == 0.0f) return;  // A(i,i) stays x1 == alpha, no update
    const float vscale = __fsub_rn(x1, alpha);
    const bool below = rv && lane > I;
    if (below) a[I] = __fdiv_rn(a[I], vscale);
    if (lane == I) a[I] = alpha;
    const float v = a[I];
    // dot_c = A(i,c) + sum_{r>i} v_r A(r,c): row r's term at xw[r][c], lane c sums its column
#pragma unroll
    for (int c = I + 1; c < N; c++) xw[lane * kQrStride + c] = below ? __fmul_rn(v, a[c]) : (lane == I ? a[c] : 0.0f);
    __syncwarp();
    float coef = 0.0f;
    if (lane > I && lane < N) {
        float dot = xw[I * kQrStride + lane];
        for (int r = I + 1; r < m; r++) dot = __fadd_rn(dot, xw[r * kQrStride + lane]);
        coef = __fmul_rn(t, dot);
    }
#pragma unroll
    for (int c = I + 1; c < N; c++) {
        const float cc = __shfl_sync(0xffffffffu, coef, c);
        if (below)
            a[c] = __fsub_rn(a[c], __fmul_rn(cc, v));
        else if (lane == I)
            a[c] = __fsub_rn(a[c], cc);
    }
    __syncwarp();  // sums read before the next step writes the buffer
}

// Reflectors 0 .. min(m, n) - 1, one instantiation per column index.
template <int N, int... I>
__device__ __forceinline__ void qr_warp_all(float (&a)[N], float& mytau, float* xw, float* cw, int lane, int m, bool rv,
                                            std::integer_sequence<int, I...>)
{
    ((I < m ? qr_warp_step<N, I>(a, mytau, xw, cw, lane, m, rv) : void()), ...);
}

template <int N>
__global__ void __launch_bounds__(kQrWarps * 32)
geqrf_warp_kernel(float* const* __restrict__ Aarray, int m, int lda, float* const* __restrict__ TauArray, int batch)
{
    __shared__ float xs[kQrWarps][32 * kQrStride];  // products of the current step, [row][column]
    __shared__ float cs[kQrWarps][32];              // column i of the current step
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long b = (long long)blockIdx.x * kQrWarps + warp;
    if (b >= batch) return;  // warp-uniform
    float* A = Aarray[b];
    float* tau = TauArray[b];
    float* xw = xs[warp];
    float* cw = cs[warp];
    const bool rv = lane < m;

    float a[N];
#pragma unroll
    for (int c = 0; c < N; c++) a[c] = rv ? A[lane + (long long)c * lda] : 0.0f;
    float mytau = 0.0f;

    qr_warp_all<N>(a, mytau, xw, cw, lane, m, rv, std::make_integer_sequence<int, N>{});

    if (rv) {
#pragma unroll
        for (int c = 0; c < N; c++) A[lane + (long long)c * lda] = a[c];
    }
    if (lane < m && lane < N) tau[lane] = mytau;
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
        switch (n) {
#define OPSBLAS_GEQRF_CASE(NN)                                                                                      \
    case NN:                                                                                                        \
        geqrf_warp_kernel<NN><<<grid, kQrWarps * 32, 0, st>>>(Aarray, m, lda, TauArray, batchSize);                 \
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
