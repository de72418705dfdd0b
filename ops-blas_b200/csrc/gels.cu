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
// value for the batch). One CTA per matrix: thread 0 forms each reflector, threads take the
// independent columns / rows / right-hand sides of every step, and every sum runs in index order
// with each product rounded before it is added -- bit for bit the CPU oracle's restatement.
// Parity with the reference is its tests' rule (MERE_MARE on the solution against LAPACK sgels_).
#include <cuda_runtime.h>

#include "internal.h"

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
    const size_t smem = gels_smem_bytes(t, m, n, lda);
    if (smem > kGelsMaxSmem) {
        log_error(kApi, "the transposed solve needs lda*n <= %zu floats of shared memory, got lda=%d n=%d",
                  kGelsMaxSmem / 4, lda, n);
        return ACLBLAS_STATUS_NOT_SUPPORTED;
    }
    static int configured_device = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (configured_device != dev) {
        cudaError_t e = cudaFuncSetAttribute(gels_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGelsMaxSmem);
        if (e != cudaSuccess) return launch_status(kApi, e);
        configured_device = dev;
    }
    gels_kernel<<<(unsigned)batchSize, kGelsThreads, smem, handle->stream>>>(t, m, n, nrhs, Aarray, lda, Carray, ldc,
                                                                             devInfo);
    return launch_status(kApi, cudaGetLastError());
}
