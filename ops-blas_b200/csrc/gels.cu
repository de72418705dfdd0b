// aclblasSgelsBatched: batched least squares / minimum-norm solutions by Householder QR or LQ.
//
// Replaces blas/gels_batched/arch35/sgels_batched_host.cpp:23-190 (host) and
// sgels_batched_kernel.cpp:25-400 (device) of the reference. Per matrix (trans T first transposes A
// in place into an n x m matrix of leading dimension n), with (M, N) the effective shape:
//   M >= N: QR by column reflectors -- xnorm = ||A(k+1:,k)||, a reflector is skipped (tau = 0)
//           when xnorm < 1e-30 and A(k,k) >= 0, else nm = sc sqrt((akk/sc)^2 + (xnorm/sc)^2) with
//           sc = max(|akk|, xnorm), beta = -sign(akk) nm, tau = (beta - akk) / beta,
//           v *= 1 / (akk - beta), A(k,k) = beta, and every later column takes w = v.a + a(k),
//           a(k) -= tau w, a += (-tau w) v; Q^T is applied to C the same way; back substitution
//           R x = c with a zero R(i,i) setting info = i + 1 and stopping the solve;
//   M <  N: LQ by row reflectors, forward substitution L y = c (same stop rule), rows M..N-1 of C
//           zeroed, Q^T applied in reverse reflector order.
// info is per matrix (device array), as the reference kernel writes it (its CPU golden keeps one
// value for the batch). Small QR-path systems run a warp per system (gels_warp_kernel); the rest
// one CTA per matrix: thread 0 forms each reflector, threads take the independent columns / rows /
// right-hand sides of every step. Every sum runs in index order with each product rounded before
// it is added -- bit for bit the CPU oracle's restatement, on both paths.
// Parity with the reference is its tests' rule (MERE_MARE on the solution against LAPACK sgels_).
#include <cuda_runtime.h>

#include <utility>

#include "internal.h"
#include "small_common.cuh"

namespace opsblas {

constexpr int kGelsThreads = 128;
constexpr size_t kGelsMaxSmem = 200 * 1024;

__device__ __forceinline__ float gels_dot_strided(const float* v, int vstride, const float* a, int astride, int len)
{
    float w = 0.0f;
    for (int i = 0; i < len; i++) w = __fadd_rn(w, __fmul_rn(v[(long long)i * vstride], a[(long long)i * astride]));
    return w;
}

// a(-astride) and a(i * astride), i < len, reflected by (v, t).
__device__ __forceinline__ void gels_apply(const float* v, int vstride, float* a, int astride, int len, float t)
{
    const float w = __fadd_rn(gels_dot_strided(v, vstride, a, astride, len), a[-(long long)astride]);
    a[-(long long)astride] = __fsub_rn(a[-(long long)astride], __fmul_rn(t, w));
    const float alpha = -__fmul_rn(t, w);
    for (int i = 0; i < len; i++)
        a[(long long)i * astride] = __fadd_rn(a[(long long)i * astride], __fmul_rn(alpha, v[(long long)i * vstride]));
}

// Thread 0: reflector of column/row k from A(k,k) and the tail v (stride vs, length len). Returns
// through shared memory: p[0] = tau (0: skipped), p[1] = scale of v.
__device__ __forceinline__ void gels_reflector(float* A, long long kk_index, const float* v, int vs, int len,
                                               float* tau_k, float* p)
{
    float ss = 0.0f;
    for (int i = 0; i < len; i++) ss = __fadd_rn(ss, __fmul_rn(v[(long long)i * vs], v[(long long)i * vs]));
    const float xnorm = sqrtf(ss);
    const float akk = A[kk_index];
    if (xnorm < 1.0e-30f && akk >= 0.0f) {
        *tau_k = 0.0f;
        p[0] = 0.0f;
        return;
    }
    const float na = fabsf(akk);
    const float sc = na > xnorm ? na : xnorm;
    const float sa = __fdiv_rn(akk, sc), sx = __fdiv_rn(xnorm, sc);
    const float nm = __fmul_rn(sc, sqrtf(__fadd_rn(__fmul_rn(sa, sa), __fmul_rn(sx, sx))));
    const float beta = akk >= 0.0f ? -nm : nm;
    const float t = __fdiv_rn(__fsub_rn(beta, akk), beta);
    *tau_k = t;
    A[kk_index] = beta;
    p[0] = t;
    p[1] = __fdiv_rn(1.0f, __fsub_rn(akk, beta));
}

__global__ void __launch_bounds__(kGelsThreads)
gels_kernel(int trans, int m, int n, int nrhs, float* const* __restrict__ Aarray, int lda,
            float* const* __restrict__ Carray, int ldc, int* __restrict__ info)
{
    extern __shared__ __align__(16) float sm[];  // tau[min(M,N)], then (trans) a copy of A
    __shared__ float p[2];
    __shared__ int s_stop;
    const int tid = threadIdx.x;
    float* A = Aarray[blockIdx.x];
    float* C = Carray[blockIdx.x];
    int* inf = info + blockIdx.x;
    int M = m, N = n, ld = lda;
    const int k = m < n ? m : n;
    float* tau = sm;
    if (trans) {
        float* scr = sm + ((k + 3) & ~3);
        for (long long e = tid; e < (long long)lda * n; e += kGelsThreads) scr[e] = A[e];
        __syncthreads();
        for (long long e = tid; e < (long long)m * n; e += kGelsThreads) {
            const int col = (int)(e / n), row = (int)(e % n);
            A[(long long)col * n + row] = scr[(long long)row * lda + col];
        }
        __syncthreads();
        M = n;
        N = m;
        ld = n;
    }

    if (M >= N) {
        for (int kk = 0; kk < N; kk++) {
            const int tail = M - kk - 1;
            float* v = A + (long long)kk * ld + kk + 1;
            if (tid == 0) gels_reflector(A, (long long)kk * ld + kk, v, 1, tail, &tau[kk], p);
            __syncthreads();
            const float t = p[0], scalev = p[1];
            if (t != 0.0f) {  // uniform: read from shared memory by every thread
                for (int i = tid; i < tail; i += kGelsThreads) v[i] = __fmul_rn(v[i], scalev);
                __syncthreads();
                for (int j = kk + 1 + tid; j < N; j += kGelsThreads) gels_apply(v, 1, A + (long long)j * ld + kk + 1, 1, tail, t);
            }
            __syncthreads();
        }
        for (int kk = 0; kk < N; kk++) {
            const float t = tau[kk];
            if (t == 0.0f) continue;
            const float* v = A + (long long)kk * ld + kk + 1;
            for (int j = tid; j < nrhs; j += kGelsThreads) gels_apply(v, 1, C + (long long)j * ldc + kk + 1, 1, M - kk - 1, t);
            __syncthreads();
        }
        // back substitution; the highest zero R(i,i) stops the first right-hand side there and
        // leaves the others untouched
        if (tid == 0) {
            int stop = -1;
            for (int i = N - 1; i >= 0; i--)
                if (A[(long long)i * ld + i] == 0.0f) {
                    stop = i;
                    break;
                }
            s_stop = stop;
        }
        __syncthreads();
        const int stop = s_stop;
        const int jmax = stop >= 0 ? 1 : nrhs;
        for (int j = tid; j < jmax; j += kGelsThreads) {
            float* c = C + (long long)j * ldc;
            for (int i = N - 1; i > stop; i--) {
                float sum = 0.0f;
                for (int q = i + 1; q < N; q++) sum = __fadd_rn(sum, __fmul_rn(A[(long long)q * ld + i], c[q]));
                c[i] = __fdiv_rn(__fsub_rn(c[i], sum), A[(long long)i * ld + i]);
            }
        }
        if (tid == 0) *inf = stop >= 0 ? stop + 1 : 0;
    } else {
        for (int kk = 0; kk < M; kk++) {
            const int tail = N - kk - 1;
            float* v = A + (long long)(kk + 1) * ld + kk;
            if (tid == 0) gels_reflector(A, (long long)kk * ld + kk, v, ld, tail, &tau[kk], p);
            __syncthreads();
            const float t = p[0], scalev = p[1];
            if (t != 0.0f) {
                for (int i = tid; i < tail; i += kGelsThreads) v[(long long)i * ld] = __fmul_rn(v[(long long)i * ld], scalev);
                __syncthreads();
                for (int ii = kk + 1 + tid; ii < M; ii += kGelsThreads)
                    gels_apply(v, ld, A + (long long)(kk + 1) * ld + ii, ld, tail, t);
            }
            __syncthreads();
        }
        // forward substitution; the lowest zero L(i,i) stops the first right-hand side there,
        // leaves the others untouched and skips the rest of the solve
        if (tid == 0) {
            int stop = -1;
            for (int i = 0; i < M; i++)
                if (A[(long long)i * ld + i] == 0.0f) {
                    stop = i;
                    break;
                }
            s_stop = stop;
        }
        __syncthreads();
        const int stop = s_stop;
        const int jmax = stop >= 0 ? 1 : nrhs;
        const int imax = stop >= 0 ? stop : M;
        for (int j = tid; j < jmax; j += kGelsThreads) {
            float* c = C + (long long)j * ldc;
            for (int i = 0; i < imax; i++) {
                float sum = 0.0f;
                for (int q = 0; q < i; q++) sum = __fadd_rn(sum, __fmul_rn(A[(long long)q * ld + i], c[q]));
                c[i] = __fdiv_rn(__fsub_rn(c[i], sum), A[(long long)i * ld + i]);
            }
        }
        if (tid == 0) *inf = stop >= 0 ? stop + 1 : 0;
        if (stop >= 0) return;  // uniform
        __syncthreads();
        for (int j = tid; j < nrhs; j += kGelsThreads)
            for (int i = M; i < N; i++) C[(long long)j * ldc + i] = 0.0f;
        __syncthreads();
        for (int kk = M - 1; kk >= 0; kk--) {
            const float t = tau[kk];
            if (t == 0.0f) continue;
            const float* v = A + (long long)(kk + 1) * ld + kk;
            for (int j = tid; j < nrhs; j += kGelsThreads)
                gels_apply(v, ld, C + (long long)j * ldc + kk + 1, 1, N - kk - 1, t);
            __syncthreads();
        }
    }
}

// Fast path, effective M >= N, M <= 32, N + nrhs <= 32: one warp per system. Lane c < N holds
// column c of the (transposed, for trans T) matrix, lane N + j holds right-hand side j, rows in
// registers. Reflector k is formed by lane k (norm, scale of v), published through shared memory
// and applied by every later column lane and every right-hand-side lane in the same step -- the
// reference applies Q^T to C after the factorisation, but each reflector meets the same column
// state either way, so the bits agree. R then goes to shared memory and each right-hand-side lane
// solves R x = c in row order (same stop rule as the CTA kernel).
constexpr int kGelsWarps = 4;

template <int M, int K>
__device__ __forceinline__ void gels_warp_step(float (&col)[M], float* vb, int lane, int ncols, float& tau_k)
{
    // xnorm = ||A(K+1:, K)||, row order, formed by every lane for its own column (lane K's is used)
    float ss = 0.0f;
#pragma unroll
    for (int r = K + 1; r < M; r++) ss = __fadd_rn(ss, __fmul_rn(col[r], col[r]));
    const float xnorm = sqrtf(__shfl_sync(0xffffffffu, ss, K));
    const float akk = __shfl_sync(0xffffffffu, col[K], K);
    if (xnorm < 1.0e-30f && akk >= 0.0f) {
        tau_k = 0.0f;
        return;  // uniform
    }
    const float na = fabsf(akk);
    const float sc = na > xnorm ? na : xnorm;
    const float sa = __fdiv_rn(akk, sc), sx = __fdiv_rn(xnorm, sc);
    const float nm = __fmul_rn(sc, sqrtf(__fadd_rn(__fmul_rn(sa, sa), __fmul_rn(sx, sx))));
    const float beta = akk >= 0.0f ? -nm : nm;
    const float t = __fdiv_rn(__fsub_rn(beta, akk), beta);
    const float scalev = __fdiv_rn(1.0f, __fsub_rn(akk, beta));
    tau_k = t;
    if (lane == K) {
        col[K] = beta;
#pragma unroll
        for (int r = K + 1; r < M; r++) {
            col[r] = __fmul_rn(col[r], scalev);
            vb[r] = col[r];
        }
    }
    __syncwarp();
    if (lane > K && lane < ncols) {
        // w = v . a + a(K); a(K) -= t w; a += (-t w) v
        float w = 0.0f;
#pragma unroll
        for (int r = K + 1; r < M; r++) w = __fadd_rn(w, __fmul_rn(vb[r], col[r]));
        w = __fadd_rn(w, col[K]);
        col[K] = __fsub_rn(col[K], __fmul_rn(t, w));
        const float alpha = -__fmul_rn(t, w);
#pragma unroll
        for (int r = K + 1; r < M; r++) col[r] = __fadd_rn(col[r], __fmul_rn(alpha, vb[r]));
    }
    __syncwarp();  // v read before the next reflector writes it
}

template <int M, int... K>
__device__ __forceinline__ void gels_warp_all(float (&col)[M], float* vb, int lane, int ncols, int N, float* tau,
                                              std::integer_sequence<int, K...>)
{
    ((K < N ? gels_warp_step<M, K>(col, vb, lane, ncols, tau[K]) : void()), ...);
}

template <int M>
__global__ void __launch_bounds__(kGelsWarps * 32)
gels_warp_kernel(int trans, int m, int n, int nrhs, float* const* __restrict__ Aarray, int lda,
                 float* const* __restrict__ Carray, int ldc, int* __restrict__ info, int batch)
{
    __shared__ float vbuf[kGelsWarps][32];
    __shared__ float rbuf[kGelsWarps][32 * 33];  // R (N x N), column c at rbuf[c * 33]
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long b = (long long)blockIdx.x * kGelsWarps + warp;
    if (b >= batch) return;  // warp-uniform
    float* A = Aarray[b];
    float* C = Carray[b];
    const int N = trans ? m : n;  // effective columns (M = effective rows)
    const int ncols = N + nrhs;
    float col[M];
    if (lane < N) {
#pragma unroll
        for (int r = 0; r < M; r++) col[r] = trans ? A[lane + (long long)r * lda] : A[r + (long long)lane * lda];
    } else if (lane < ncols) {
        const float* c = C + (long long)(lane - N) * ldc;
#pragma unroll
        for (int r = 0; r < M; r++) col[r] = c[r];
    } else {
#pragma unroll
        for (int r = 0; r < M; r++) col[r] = 0.0f;
    }
    float tau[32];
    gels_warp_all<M>(col, vbuf[warp], lane, ncols, N, tau, std::make_integer_sequence<int, M>{});
    // factors back (trans: the n x m transpose with leading dimension n, as the reference leaves it)
    if (lane < N) {
        if (trans) {
            __syncwarp();  // every lane has read its row of A before any lane writes the transpose
#pragma unroll
            for (int r = 0; r < M; r++) A[r + (long long)lane * M] = col[r];
        } else {
#pragma unroll
            for (int r = 0; r < M; r++) A[r + (long long)lane * lda] = col[r];
        }
    } else if (trans) {
        __syncwarp();
    }
    // R to shared memory; the highest zero diagonal stops the first right-hand side there
    float* R = rbuf[warp];
    if (lane < N) {
#pragma unroll
        for (int r = 0; r < M; r++)
            if (r < N) R[lane * 33 + r] = col[r];
    }
    __syncwarp();
    int stop = -1;
    for (int i = N - 1; i >= 0; i--)
        if (R[i * 33 + i] == 0.0f) {
            stop = i;
            break;
        }
    const int j = lane - N;
    if (j >= 0 && j < (stop >= 0 ? 1 : nrhs)) {
#pragma unroll
        for (int i = M - 1; i >= 0; i--) {
            if (i < N && i > stop) {
                float sum = 0.0f;
#pragma unroll
                for (int q = i + 1; q < M; q++)
                    if (q < N) sum = __fadd_rn(sum, __fmul_rn(R[q * 33 + i], col[q]));
                col[i] = __fdiv_rn(__fsub_rn(col[i], sum), R[i * 33 + i]);
            }
        }
    }
    if (j >= 0 && j < nrhs) {
        float* c = C + (long long)j * ldc;
#pragma unroll
        for (int r = 0; r < M; r++) c[r] = col[r];
    }
    if (lane == 0) info[b] = stop >= 0 ? stop + 1 : 0;
}

size_t gels_smem_bytes(int trans, int m, int n, int lda)
{
    const int k = m < n ? m : n;
    return (size_t)((k + 3) & ~3) * 4 + (trans ? (size_t)lda * n * 4 : 0);
}

}  // namespace opsblas

using namespace opsblas;

extern "C" aclblasStatus_t aclblasSgelsBatched(aclblasHandle_t handle, aclblasOperation_t trans, int m, int n,
                                               int nrhs, float* const Aarray[], int lda, float* const Carray[],
                                               int ldc, int* devInfo, int batchSize)
{
    static const char* kApi = "aclblasSgelsBatched";
    if (handle == nullptr) {
        log_error(kApi, "handle is nullptr");
        return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    }
    // ValidateSgelsBatchedParams (sgels_batched_host.cpp:23-68)
    if (trans != ACLBLAS_OP_N && trans != ACLBLAS_OP_T) {
        log_error(kApi, "trans must be OP_N(111) or OP_T(112), got %d", (int)trans);
        return ACLBLAS_STATUS_INVALID_ENUM;
    }
    if (m < 0 || n < 0 || nrhs < 0 || batchSize < 0) {
        log_error(kApi, "invalid sizes (m=%d n=%d nrhs=%d batch=%d)", m, n, nrhs, batchSize);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (lda < max1(m)) {
        log_error(kApi, "lda must be >= max(1, m), got lda=%d, m=%d", lda, m);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (ldc < max1(m > n ? m : n)) {
        log_error(kApi, "ldc must be >= max(1, m, n), got ldc=%d, m=%d, n=%d", ldc, m, n);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (batchSize > 0 && (Aarray == nullptr || Carray == nullptr)) {
        log_error(kApi, "Aarray and Carray must not be nullptr when batchSize > 0");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (devInfo == nullptr) {
        log_error(kApi, "devInfo must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (m == 0 || n == 0 || nrhs == 0 || batchSize == 0) return ACLBLAS_STATUS_SUCCESS;

    const int t = trans == ACLBLAS_OP_T ? 1 : 0;
    const int effM = t ? n : m, effN = t ? m : n;
    if (effM >= effN && effM <= 32 && effN + nrhs <= 32) {
        const unsigned grid = (unsigned)((batchSize + kGelsWarps - 1) / kGelsWarps);
        switch (effM) {
#define OPSBLAS_GELS_CASE(MM)                                                                                       \
    case MM:                                                                                                        \
        gels_warp_kernel<MM><<<grid, kGelsWarps * 32, 0, handle->stream>>>(t, m, n, nrhs, Aarray, lda, Carray, ldc,  \
                                                                           devInfo, batchSize);                     \
        break;
            OPSBLAS_FOR_N_1_32(OPSBLAS_GELS_CASE)
#undef OPSBLAS_GELS_CASE
            default:
                break;
        }
        return launch_status(kApi, cudaGetLastError());
    }
    const size_t smem = gels_smem_bytes(t, m, n, lda);
    if (smem > kGelsMaxSmem) {
        log_error(kApi, "the transposed solve needs lda*n <= %zu floats of shared memory, got lda=%d n=%d",
                  kGelsMaxSmem / 4, lda, n);
        return ACLBLAS_STATUS_NOT_SUPPORTED;
    }
    const cudaError_t e = ensure_smem_limit(gels_kernel, (int)kGelsMaxSmem);
    if (e != cudaSuccess) return launch_status(kApi, e);
    gels_kernel<<<(unsigned)batchSize, kGelsThreads, smem, handle->stream>>>(t, m, n, nrhs, Aarray, lda, Carray, ldc,
                                                                             devInfo);
    return launch_status(kApi, cudaGetLastError());
}
