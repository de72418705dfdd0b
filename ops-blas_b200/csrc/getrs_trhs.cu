// aclblasSgetrsBatched, n > 32: one thread per (matrix, right-hand side) -- trans T / C always,
// trans N for small orders with many right-hand sides (getrs_nrhs_preferred).
//
// The reference's transposed solve (sgetrs_batched_kernel.cpp:202-388) runs, per right-hand
// side: the U^T forward sweep x_j /= U(j,j), x_i -= U(j,i) x_j (i > j), then the L^T backward
// sweep as dot products s = x_j - sum_{i>j} L(i,j) x_i accumulated in increasing i, then the
// interchanges in reverse order. The dot-product order makes every element depend on the whole
// chain before it, so this kernel keeps the reference's thread-per-right-hand-side structure:
// thread g solves column g % nrhs of matrix g / nrhs with its x vector in shared memory (row
// stride n rounded up to 4, plus 4: 16-byte aligned, and eight threads' 16-byte reads cover the 32
// banks), reading LU through L1/L2 down its columns (the threads of one matrix read the same
// addresses), four elements per load where LU is 16-byte aligned. Bit-identical to the reference
// order: every accumulation stays one fmaf per element in increasing index.
#include <cuda_runtime.h>

#include <cstdint>

#include "internal.h"

namespace opsblas {

constexpr int kTrThreads = 128;

static int trhs_stride(int n) { return ((n + 3) & ~3) + 4; }

// Trans N (TR false), same thread-per-right-hand-side layout: the reference's sequence
// (sgetrs_batched_kernel.cpp:83-200) is right-looking -- interchanges k = 0..n-1, then
// x_i -= L(i,j) x_j for i > j, j ascending, then x_j /= U(j,j) and x_i -= U(i,j) x_j for i < j,
// j descending -- so each step walks column j of LU (contiguous) and updates x in shared memory,
// four elements per step where LU is 16-byte aligned.
template <bool TR>
__global__ void __launch_bounds__(kTrThreads)
getrs_trhs_kernel(const float* const* __restrict__ Aarray, int n, int lda, const int* __restrict__ ipiv,
                  float* const* __restrict__ Barray, int ldb, int nrhs, long long chains, int stride)
{
    extern __shared__ __align__(16) float xs_all[];
    const long long g = (long long)blockIdx.x * kTrThreads + threadIdx.x;
    if (g >= chains) return;
    const long long m = g / nrhs;
    const int c = (int)(g % nrhs);
    float* B = Barray[m];
    if (B == nullptr) return;  // a NULL right-hand side skips the matrix
    const float* A = Aarray[m];
    float* x = xs_all + (size_t)threadIdx.x * stride;
    float* bc = B + (long long)c * ldb;
    for (int i = 0; i < n; i++) x[i] = bc[i];
    const bool vec = (lda & 3) == 0 && (reinterpret_cast<uintptr_t>(A) & 15) == 0;

    if (!TR) {
        if (ipiv != nullptr) {  // interchanges k = 0..n-1 (out-of-range or self pivots skipped)
            const int* p = ipiv + m * n;
            for (int k = 0; k < n; k++) {
                const int q = p[k] - 1;
                if ((unsigned)q < (unsigned)n && q != k) {
                    const float t = x[k];
                    x[k] = x[q];
                    x[q] = t;
                }
            }
        }
        for (int j = 0; j + 1 < n; j++) {  // unit L, column j
            const float* lcol = A + (long long)j * lda;
            const float xj = x[j];
            int i = j + 1;
            if (vec) {
                for (; i < n && (i & 3) != 0; i++) x[i] = fmaf(-lcol[i], xj, x[i]);
                for (; i + 4 <= n; i += 4) {
                    const float4 l = *reinterpret_cast<const float4*>(lcol + i);
                    float4 xv = *reinterpret_cast<const float4*>(x + i);
                    xv.x = fmaf(-l.x, xj, xv.x);
                    xv.y = fmaf(-l.y, xj, xv.y);
                    xv.z = fmaf(-l.z, xj, xv.z);
                    xv.w = fmaf(-l.w, xj, xv.w);
                    *reinterpret_cast<float4*>(x + i) = xv;
                }
            }
            for (; i < n; i++) x[i] = fmaf(-lcol[i], xj, x[i]);
        }
        for (int j = n - 1; j >= 0; j--) {  // U, column j
            const float* ucol = A + (long long)j * lda;
            const float xj = x[j] / ucol[j];
            x[j] = xj;
            int i = 0;
            if (vec) {
                for (; i + 4 <= j; i += 4) {
                    const float4 u = *reinterpret_cast<const float4*>(ucol + i);
                    float4 xv = *reinterpret_cast<const float4*>(x + i);
                    xv.x = fmaf(-u.x, xj, xv.x);
                    xv.y = fmaf(-u.y, xj, xv.y);
                    xv.z = fmaf(-u.z, xj, xv.z);
                    xv.w = fmaf(-u.w, xj, xv.w);
                    *reinterpret_cast<float4*>(x + i) = xv;
                }
            }
            for (; i < j; i++) x[i] = fmaf(-ucol[i], xj, x[i]);
        }
        for (int i = 0; i < n; i++) bc[i] = x[i];
        return;
    }

    // U^T forward sweep. The reference runs it right-looking (x_j /= U(j,j), then x_i -= U(j,i) x_j
    // for i > j); every x_i receives its updates in increasing j and is divided last, which is the
    // same sequence as the left-looking form used here -- x_i = (x_i - sum_{j<i} U(j,i) x_j, one
    // fmaf per j in increasing j) / U(i,i) -- and that form walks column i of U (contiguous).
    for (int i = 0; i < n; i++) {
        const float* ucol = A + (long long)i * lda;
        float s = x[i];
        int j = 0;
        if (vec) {
            for (; j + 4 <= i; j += 4) {
                const float4 u = *reinterpret_cast<const float4*>(ucol + j);
                const float4 xv = *reinterpret_cast<const float4*>(x + j);
                s = fmaf(-u.x, xv.x, s);
                s = fmaf(-u.y, xv.y, s);
                s = fmaf(-u.z, xv.z, s);
                s = fmaf(-u.w, xv.w, s);
            }
        }
        for (; j < i; j++) s = fmaf(-ucol[j], x[j], s);
        x[i] = s / ucol[i];
    }
    // L^T backward sweep (column j of L: A[i + j*lda], i > j), dot products in increasing i
    for (int j = n - 1; j >= 0; j--) {
        const float* lcol = A + (long long)j * lda;
        float s = x[j];
        int i = j + 1;
        if (vec) {
            for (; i < n && (i & 3) != 0; i++) s = fmaf(-lcol[i], x[i], s);
            for (; i + 4 <= n; i += 4) {
                const float4 l = *reinterpret_cast<const float4*>(lcol + i);
                const float4 xv = *reinterpret_cast<const float4*>(x + i);
                s = fmaf(-l.x, xv.x, s);
                s = fmaf(-l.y, xv.y, s);
                s = fmaf(-l.z, xv.z, s);
                s = fmaf(-l.w, xv.w, s);
            }
        }
        for (; i < n; i++) s = fmaf(-lcol[i], x[i], s);
        x[j] = s;
    }
    // interchanges in reverse (sgetrs_batched_kernel.cpp:94-100 semantics: invalid pivots skipped)
    if (ipiv != nullptr) {
        const int* p = ipiv + m * n;
        for (int k = n - 1; k >= 0; k--) {
            const int q = p[k] - 1;
            if ((unsigned)q < (unsigned)n && q != k) {
                const float t = x[k];
                x[k] = x[q];
                x[q] = t;
            }
        }
    }
    for (int i = 0; i < n; i++) bc[i] = x[i];
}

bool getrs_trhs_supported(int n) { return n > 32 && (size_t)kTrThreads * trhs_stride(n) * 4 <= 200 * 1024; }

template <bool TR>
static cudaError_t thread_rhs_launch(cudaStream_t st, int n, int nrhs, const float* const* Aarray, int lda,
                                     const int* ipiv, float* const* Barray, int ldb, int batch)
{
    const cudaError_t e = ensure_smem_limit(getrs_trhs_kernel<TR>, 200 * 1024);
    if (e != cudaSuccess) return e;
    const long long chains = (long long)batch * nrhs;
    const long long blocks = (chains + kTrThreads - 1) / kTrThreads;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    const int stride = trhs_stride(n);
    getrs_trhs_kernel<TR><<<(unsigned)blocks, kTrThreads, (size_t)kTrThreads * stride * 4, st>>>(
        Aarray, n, lda, ipiv, Barray, ldb, nrhs, chains, stride);
    return cudaGetLastError();
}

cudaError_t getrs_trhs_launch(cudaStream_t st, int n, int nrhs, const float* const* Aarray, int lda, const int* ipiv,
                              float* const* Barray, int ldb, int batch)
{
    return thread_rhs_launch<true>(st, n, nrhs, Aarray, lda, ipiv, Barray, ldb, batch);
}

// Trans N, one thread per right-hand side: chosen over the CTA-per-matrix blocked kernel when there
// are enough independent right-hand sides to fill the GPU and the orders are small.
bool getrs_nrhs_preferred(int n, int nrhs, int batch)
{
    return getrs_trhs_supported(n) && n <= 128 && (long long)batch * nrhs >= 65536;
}

cudaError_t getrs_nrhs_launch(cudaStream_t st, int n, int nrhs, const float* const* Aarray, int lda, const int* ipiv,
                              float* const* Barray, int ldb, int batch)
{
    return thread_rhs_launch<false>(st, n, nrhs, Aarray, lda, ipiv, Barray, ldb, batch);
}

}  // namespace opsblas
