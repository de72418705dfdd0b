// aclblasSgetrfsRefineBatchedEx: factor + solve + iterative refinement, one call.
//
// No counterpart in the reference (an extension next to the drop-in chain). Per matrix:
//   LU = A (copy; A is kept for the residual), P*LU = A factored by aclblasSgetrfBatched's
//   kernels -- plain FP32 for ACLBLAS_COMPUTE_32F; for ACLBLAS_COMPUTE_32F_FAST_TF32 / _FAST_16BF
//   with the split TF32 / BF16 trailing update on the tensor cores, the matrix resident in TMEM
//   (getrf_tmem.cu, 32 < n <= 256); for TF32 with 256 < n <= 1024 the blocked LU with FP32
//   panels and the tensor-core trailing update (getrf_blocked_tc.cu), when the workspace also
//   holds its scratch; other cases factor in plain FP32, after which refinement converges at once;
//   X = LU \ B (aclblasSgetrsBatched's kernels);
//   repeat up to maxIter times: r = B - A X in FP64 on the GPU, backward error
//     berr = max_c ||r_c||_inf / (||A||_inf ||x_c||_inf + ||b_c||_inf) in FP64;
//     matrices with berr <= tol stop; the others solve LU d = r (FP32) and set X += d.
// Convergence is tracked on the device (no host synchronisation inside the call), so the
// call can be captured in a CUDA graph. berrArray / iterArray / infoArray are device arrays.
#include <cuda_runtime.h>

#include <mutex>

#include "internal.h"

namespace opsblas {

__global__ void init_ptr_array_kernel(float** out, float* base, long long stride, int count)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x)
        out[i] = base + i * stride;
}

// dst[b](i, j) = src[b](i, j), i < rows, j < cols. One CTA per matrix, a warp per column at a
// time, 16-byte accesses when both columns are 16-byte aligned.
__global__ void copy_batched_kernel(const float* const* src, int lds, float* const* dst, int ldd, int rows, int cols)
{
    const float* s = src[blockIdx.x];
    float* d = dst[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const bool vec = ((reinterpret_cast<uintptr_t>(s) | reinterpret_cast<uintptr_t>(d)) & 15) == 0 && lds % 4 == 0 &&
                     ldd % 4 == 0;
    for (int j = warp; j < cols; j += nw) {
        const float* sc = s + (long long)j * lds;
        float* dc = d + (long long)j * ldd;
        int i = 0;
        if (vec) {
            for (; i + 128 <= rows; i += 128)
                reinterpret_cast<float4*>(dc + i)[lane] = reinterpret_cast<const float4*>(sc + i)[lane];
        }
        for (i += lane; i < rows; i += 32) dc[i] = sc[i];
    }
}

constexpr int kResThreads = 256;
constexpr int kResMaxRhs = 16;  // right-hand sides per pass

// One CTA per matrix. FP64 residual r = b - A x and normwise backward error; on the last check
// (final != 0) only the error is recorded. d receives r in FP32; Dact[m] is set to d, or to NULL
// when the matrix has converged, so that the correction solve and update skip it.
__global__ void __launch_bounds__(kResThreads, 2)
refine_residual_kernel(int n, int nrhs, const float* const* Aarray, int lda, const float* const* Barray, int ldb,
                       const float* const* Xarray, int ldx, float* const* Darray, int ldd, float** Dact, double tol,
                       int it, int final_check, int* __restrict__ done, double* __restrict__ berr,
                       int* __restrict__ iters)
{
    extern __shared__ double xs[];  // [n + 16][kResMaxRhs]
    __shared__ double s_anorm;
    const long long m = blockIdx.x;
    const float* A = Aarray[m];
    const float* B = Barray[m];
    const float* X = Xarray[m];
    float* D = Darray[m];
    const int tid = threadIdx.x;
    const bool was_done = done[m] != 0;
    if (was_done) {  // converged earlier: error and step count are recorded, no correction
        if (tid == 0 && !final_check) Dact[m] = nullptr;
        return;
    }
    const int lane = tid & 31, warp = tid >> 5;
    // block maxima of K values per thread at once: shuffles within the warp, one row of K per warp
    // in shared memory, then a thread per value across the warps -- two barriers for all K
    __shared__ double red[kResThreads / 32][2 * kResMaxRhs + 1];
    __shared__ double s_max[2 * kResMaxRhs + 1];
    auto block_max_all = [&](auto& v) {
        constexpr int K = (int)(sizeof(v) / sizeof(double));
        static_assert(K <= 2 * kResMaxRhs + 1, "reduction width");
#pragma unroll
        for (int q = 0; q < K; q++) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v[q] = fmax(v[q], __shfl_xor_sync(0xffffffffu, v[q], off));
        }
        if (lane == 0) {
#pragma unroll
            for (int q = 0; q < K; q++) red[warp][q] = v[q];
        }
        __syncthreads();
        if (tid < K) {
            double r = red[0][tid];
            for (int w = 1; w < kResThreads / 32; w++) r = fmax(r, red[w][tid]);
            s_max[tid] = r;
        }
        __syncthreads();
    };
    // r = b - A x per right-hand-side chunk; the row sums of |A| (for ||A||_inf) are gathered in
    // the first chunk's pass over A, so A is read once per chunk. The column maxima of |x| and |b|
    // are reduced first (into shared memory) so that the row loop keeps only r and max |r| live.
    __shared__ double s_xn[kResMaxRhs], s_bn[kResMaxRhs];
    double worst = 0.0;
    double rowmax = 0.0;
    for (int c0 = 0; c0 < nrhs; c0 += kResMaxRhs) {
        const int cw = min(kResMaxRhs, nrhs - c0);
        __syncthreads();
        // X chunk into shared memory as FP64, eight loads in flight before their stores
        const int total = (n + 16) * kResMaxRhs;  // 16 zero rows of padding
        for (int base = tid; base < total; base += 8 * kResThreads) {
            float v[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int e = base + u * kResThreads, i = e / kResMaxRhs, c = e % kResMaxRhs;
                v[u] = (e < total && c < cw && i < n) ? X[i + (long long)(c0 + c) * ldx] : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < 8; u++)
                if (base + u * kResThreads < total) xs[base + u * kResThreads] = (double)v[u];
        }
        __syncthreads();
        {  // column maxima of |x| and |b| (FP32 values: their maxima are exact)
            double v[2 * kResMaxRhs];
#pragma unroll
            for (int q = 0; q < 2 * kResMaxRhs; q++) v[q] = 0.0;
            for (int i = tid; i < n; i += kResThreads) {
                float bv[kResMaxRhs];
#pragma unroll
                for (int c = 0; c < kResMaxRhs; c++) bv[c] = c < cw ? B[i + (long long)(c0 + c) * ldb] : 0.0f;
#pragma unroll
                for (int c = 0; c < kResMaxRhs; c++) {
                    v[c] = fmax(v[c], fabs(xs[i * kResMaxRhs + c]));
                    v[kResMaxRhs + c] = fmax(v[kResMaxRhs + c], (double)fabsf(bv[c]));
                }
            }
            block_max_all(v);
            if (tid < kResMaxRhs) {
                s_xn[tid] = s_max[tid];
                s_bn[tid] = s_max[kResMaxRhs + tid];
            }
        }
        double rmaxs[kResMaxRhs + 1];  // [kResMaxRhs]: the row sums' maximum (first chunk)
#pragma unroll
        for (int c = 0; c <= kResMaxRhs; c++) rmaxs[c] = 0.0;
        for (int i = tid; i < n; i += kResThreads) {
            double r[kResMaxRhs];
#pragma unroll
            for (int c = 0; c < kResMaxRhs; c++) r[c] = c < cw ? (double)B[i + (long long)(c0 + c) * ldb] : 0.0;
            double asum = 0.0;
            for (int j0 = 0; j0 < n; j0 += 16) {
                float av[16];  // sixteen independent loads in flight before the FMAs that use them
#pragma unroll
                for (int u = 0; u < 16; u++) av[u] = j0 + u < n ? A[i + (long long)(j0 + u) * lda] : 0.0f;
#pragma unroll
                for (int u = 0; u < 16; u++) {
                    const double a = (double)av[u];
                    asum += fabs(a);
                    const double2* xr = reinterpret_cast<const double2*>(xs + (j0 + u) * kResMaxRhs);
#pragma unroll
                    for (int q = 0; q < kResMaxRhs / 2; q++) {
                        const double2 v = xr[q];  // rows n..n+15 are zero padding
                        r[2 * q] = fma(-a, v.x, r[2 * q]);
                        r[2 * q + 1] = fma(-a, v.y, r[2 * q + 1]);
                    }
                }
            }
            rmaxs[kResMaxRhs] = fmax(rmaxs[kResMaxRhs], asum);
#pragma unroll
            for (int c = 0; c < kResMaxRhs; c++) {
                if (c < cw) {
                    rmaxs[c] = fmax(rmaxs[c], fabs(r[c]));
                    if (!final_check) D[i + (long long)(c0 + c) * ldd] = (float)r[c];
                }
            }
        }
        block_max_all(rmaxs);
        if (c0 == 0) {
            rowmax = s_max[kResMaxRhs];
            if (tid == 0) s_anorm = rowmax;
        }
        __syncthreads();
        for (int c = 0; c < cw; c++) {
            const double rn = s_max[c];
            const double den = s_anorm * s_xn[c] + s_bn[c];
            const double e = den > 0.0 ? rn / den : (rn > 0.0 ? INFINITY : 0.0);
            worst = fmax(worst, e);
        }
    }
    __syncthreads();
    const bool conv = worst <= tol;
    if (tid == 0) {
        berr[m] = worst;
        if (!was_done && (conv || final_check)) {
            done[m] = conv ? 1 : 0;
            iters[m] = it;
        }
        if (conv && !final_check) done[m] = 1;
        if (!final_check) Dact[m] = conv ? nullptr : D;
    }
}

__global__ void axpy_batched_kernel(int n, int nrhs, const float* const* Darray, int ldd, float* const* Xarray, int ldx)
{
    const float* D = Darray[blockIdx.x];  // one CTA per matrix; NULL: converged, nothing to add
    if (D == nullptr) return;
    float* X = Xarray[blockIdx.x];
    for (long long e = threadIdx.x; e < (long long)n * nrhs; e += blockDim.x) {
        const long long i = e % n, c = e / n;
        X[i + c * ldx] += D[i + c * ldd];
    }
}

__global__ void fill_int_kernel(int* p, int v, int count)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) p[i] = v;
}

}  // namespace opsblas

using namespace opsblas;

extern "C" aclblasStatus_t aclblasSgetrfsRefineBatchedEx(
    aclblasHandle_t handle, int n, int nrhs, const float* const Aarray[], int lda, float* const LUarray[], int ldlu,
    int* PivotArray, const float* const Barray[], int ldb, float* const Xarray[], int ldx,
    aclblasComputeType_t computeType, int maxIter, double tol, double* berrArray, int* iterArray, int* infoArray,
    int batchCount)
{
    static const char* kApi = "aclblasSgetrfsRefineBatchedEx";
    if (handle == nullptr) {
        log_error(kApi, "handle is nullptr");
        return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    }
    if (n < 0 || nrhs < 0 || batchCount < 0 || maxIter < 0 || !(tol >= 0.0)) {
        log_error(kApi, "invalid size or control argument (n=%d nrhs=%d batch=%d maxIter=%d)", n, nrhs, batchCount,
                  maxIter);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (lda < max1(n) || ldlu < max1(n) || ldb < max1(n) || ldx < max1(n)) {
        log_error(kApi, "leading dimensions must be >= max(1, n)");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    int mode;
    switch (computeType) {
        case ACLBLAS_COMPUTE_32F: mode = 0; break;
        case ACLBLAS_COMPUTE_32F_FAST_TF32: mode = 1; break;
        case ACLBLAS_COMPUTE_32F_FAST_16BF: mode = 2; break;
        default:
            log_error(kApi, "computeType must be 32F, 32F_FAST_TF32 or 32F_FAST_16BF, got %d", (int)computeType);
            return ACLBLAS_STATUS_NOT_SUPPORTED;
    }
    if (n == 0 || batchCount == 0) return ACLBLAS_STATUS_SUCCESS;
    if (!Aarray || !LUarray || !PivotArray || !Barray || !Xarray || !berrArray || !iterArray || !infoArray) {
        log_error(kApi, "array arguments must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    // workspace: correction block D (n x nrhs per matrix), its two pointer arrays, done flags
    const size_t dbytes = ((size_t)n * nrhs * 4 + 255) / 256 * 256;
    const size_t need = dbytes * batchCount + (size_t)batchCount * 16 + (size_t)batchCount * 4 + 512;
    if (handle->workspace_size < need) {
        log_error(kApi, "workspace required %zu bytes, but only %zu available; call aclblasSetWorkspace", need,
                  handle->workspace_size);
        return ACLBLAS_STATUS_EXECUTION_FAILED;
    }
    // TF32 above n = 256: the blocked tensor-core LU when the workspace also holds its scratch
    // (after the refinement's part, 256-byte aligned); else plain FP32 factors
    const size_t bt_off = (need + 255) / 256 * 256;
    const bool blocked = mode == 1 && getrf_blocked_tc_supported(n) &&
                         handle->workspace_size >= bt_off + getrf_blocked_tc_scratch_bytes(n, batchCount);
    char* ws = static_cast<char*>(handle->workspace);
    float* dbase = reinterpret_cast<float*>(ws);
    float** dptr = reinterpret_cast<float**>(ws + dbytes * batchCount);
    float** dact = dptr + batchCount;  // dptr, or NULL for converged matrices
    int* done = reinterpret_cast<int*>(reinterpret_cast<char*>(dact) + (size_t)batchCount * 8);
    cudaStream_t st = handle->stream;
    const unsigned bgrid = (unsigned)((batchCount + 255) / 256 < 4096 ? (batchCount + 255) / 256 : 4096);

    init_ptr_array_kernel<<<bgrid, 256, 0, st>>>(dptr, dbase, (long long)(dbytes / 4), batchCount);
    fill_int_kernel<<<bgrid, 256, 0, st>>>(done, 0, batchCount);
    fill_int_kernel<<<bgrid, 256, 0, st>>>(iterArray, maxIter, batchCount);
    const bool tmem = mode != 0 && getrf_tmem_supported(n);  // reads A, writes LU: no copy
    if (!tmem && !blocked) copy_batched_kernel<<<(unsigned)batchCount, 256, 0, st>>>(Aarray, lda, LUarray, ldlu, n, n);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return launch_status(kApi, err);
    if (tmem) {
        err = getrf_tmem_launch(st, Aarray, lda, LUarray, n, ldlu, PivotArray, infoArray, batchCount, mode,
                                handle->dstatus);
    } else if (blocked) {  // reads A, writes LU
        err = getrf_blocked_tc_launch(st, Aarray, lda, LUarray, n, ldlu, PivotArray, infoArray, batchCount,
                                      ws + bt_off, handle->dstatus, handle->tmslots);
    } else {  // plain FP32 factors: the batched getrf's kernels (stop codes after the refinement's part)
        int* stat = handle->workspace_size >= bt_off + sizeof(int) * (size_t)batchCount
                        ? reinterpret_cast<int*>(ws + bt_off)
                        : nullptr;
        aclblasStatus_t s = getrf_batched_impl(handle, n, LUarray, ldlu, PivotArray, infoArray, batchCount, stat);
        if (s != ACLBLAS_STATUS_SUCCESS) return s;
    }
    if (err != cudaSuccess || nrhs == 0) return launch_status(kApi, err);
    copy_batched_kernel<<<(unsigned)batchCount, 256, 0, st>>>(Barray, ldb, Xarray, ldx, n, nrhs);
    err = getrs_launch(st, false, n, nrhs, LUarray, ldlu, PivotArray, Xarray, ldx, batchCount);
    if (err != cudaSuccess) return launch_status(kApi, err);
    const int rhs_chunk = nrhs < kResMaxRhs ? nrhs : kResMaxRhs;
    (void)rhs_chunk;
    const size_t rsm = (size_t)(n + 16) * kResMaxRhs * 8;
    if (rsm > 200 * 1024) {
        log_error(kApi, "n=%d exceeds the residual kernel's shared-memory limit", n);
        return ACLBLAS_STATUS_NOT_SUPPORTED;
    }
    err = ensure_smem_limit(refine_residual_kernel, 200 * 1024);
    if (err != cudaSuccess) return launch_status(kApi, err);
    for (int it = 0; it < maxIter; it++) {
        refine_residual_kernel<<<(unsigned)batchCount, kResThreads, rsm, st>>>(
            n, nrhs, Aarray, lda, Barray, ldb, Xarray, ldx, dptr, n, dact, tol, it, 0, done, berrArray, iterArray);
        err = getrs_launch(st, false, n, nrhs, LUarray, ldlu, PivotArray, dact, n, batchCount);
        if (err != cudaSuccess) return launch_status(kApi, err);
        axpy_batched_kernel<<<(unsigned)batchCount, 256, 0, st>>>(n, nrhs, dact, n, Xarray, ldx);
    }
    refine_residual_kernel<<<(unsigned)batchCount, kResThreads, rsm, st>>>(
        n, nrhs, Aarray, lda, Barray, ldb, Xarray, ldx, dptr, n, dact, tol, maxIter, 1, done, berrArray, iterArray);
    return launch_status(kApi, cudaGetLastError());
}

// ----------------------------------------------------------------------------------------------
// aclblasSgetrfsRefineBatchedStaticScratch: aclblasSgetrfsRefineBatchedEx with its scratch taken
// from a fixed array in the library's device image instead of the handle workspace.
//
// Some callers cannot hand the library device memory: a plugin inside a host application that
// owns every device allocation (a caching allocator with all memory reserved, or a hard memory
// budget), or code that must not call cudaMalloc/cudaFree because those synchronise the device.
// This entry point needs no workspace and allocates nothing. Its scratch (correction blocks D,
// their pointer array, per-matrix convergence flags; the same layout as the workspace of
// aclblasSgetrfsRefineBatchedEx) is kRefineStaticScratchBytes of static device memory; a request
// that needs more is rejected with ACLBLAS_STATUS_INVALID_VALUE before anything is launched.
//
// Set-up: the first call on each device (with that device current) looks up the scratch address
// with cudaGetSymbolAddress and sets the residual kernel's shared-memory limit; later calls reuse
// the cached address. Make that first call before any stream capture. The cached address does not
// survive a cudaDeviceReset (the module is reloaded elsewhere): do not use the entry point on a
// device after resetting it.
//
// Only the convergence flags must start at zero; every call clears them on its stream before use,
// so the scratch may hold anything a previous call left there. There is one scratch array per
// device, shared by every handle and stream in the process: calls that overlap in time on the
// same device (different streams, or different host threads) race on it and give wrong results.
// Calls issued one after another on the same stream are safe.
namespace opsblas {

constexpr size_t kRefineStaticScratchBytes = ACLBLAS_REFINE_STATIC_SCRATCH_BYTES;
constexpr int kStaticMaxDevices = 64;

static __device__ __align__(256) unsigned char g_refine_static_scratch[kRefineStaticScratchBytes];

static std::mutex g_static_mu;
static char* g_static_base[kStaticMaxDevices];  // per device ordinal, nullptr until set up

// The scratch address on the current device; the first call per device does the set-up.
static aclblasStatus_t static_scratch_base(const char* api, int device, char** base)
{
    if (device < 0 || device >= kStaticMaxDevices) {
        log_error(api, "device ordinal %d is beyond the %d devices this entry point supports", device,
                  kStaticMaxDevices);
        return ACLBLAS_STATUS_NOT_SUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (g_static_base[device] == nullptr) {
        void* p = nullptr;
        cudaError_t err = cudaGetSymbolAddress(&p, g_refine_static_scratch);
        if (err != cudaSuccess || p == nullptr) {
            log_error(api, "cannot resolve the static scratch on device %d: %s", device, cudaGetErrorString(err));
            return launch_status(api, err != cudaSuccess ? err : cudaErrorInvalidSymbol);
        }
        err = ensure_smem_limit(refine_residual_kernel, 200 * 1024);
        if (err != cudaSuccess) return launch_status(api, err);
        g_static_base[device] = static_cast<char*>(p);
    }
    *base = g_static_base[device];
    return ACLBLAS_STATUS_SUCCESS;
}

}  // namespace opsblas

extern "C" aclblasStatus_t aclblasSgetrfsRefineBatchedStaticScratch(
    aclblasHandle_t handle, int n, int nrhs, const float* const Aarray[], int lda, float* const LUarray[], int ldlu,
    int* PivotArray, const float* const Barray[], int ldb, float* const Xarray[], int ldx,
    aclblasComputeType_t computeType, int maxIter, double tol, double* berrArray, int* iterArray, int* infoArray,
    int batchCount)
{
    static const char* kApi = "aclblasSgetrfsRefineBatchedStaticScratch";
    if (handle == nullptr) {
        log_error(kApi, "handle is nullptr");
        return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    }
    if (n < 0 || nrhs < 0 || batchCount < 0 || maxIter < 0 || !(tol >= 0.0)) {
        log_error(kApi, "invalid size or control argument (n=%d nrhs=%d batch=%d maxIter=%d)", n, nrhs, batchCount,
                  maxIter);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (lda < max1(n) || ldlu < max1(n) || ldb < max1(n) || ldx < max1(n)) {
        log_error(kApi, "leading dimensions must be >= max(1, n)");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    int mode;
    switch (computeType) {
        case ACLBLAS_COMPUTE_32F: mode = 0; break;
        case ACLBLAS_COMPUTE_32F_FAST_TF32: mode = 1; break;
        case ACLBLAS_COMPUTE_32F_FAST_16BF: mode = 2; break;
        default:
            log_error(kApi, "computeType must be 32F, 32F_FAST_TF32 or 32F_FAST_16BF, got %d", (int)computeType);
            return ACLBLAS_STATUS_NOT_SUPPORTED;
    }
    if (n == 0 || batchCount == 0) return ACLBLAS_STATUS_SUCCESS;
    if (!Aarray || !LUarray || !PivotArray || !Barray || !Xarray || !berrArray || !iterArray || !infoArray) {
        log_error(kApi, "array arguments must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    // scratch: correction block D (n x nrhs per matrix, 256-byte rounded), its two pointer arrays, flags
    const size_t cap = kRefineStaticScratchBytes;
    if ((size_t)n * (size_t)nrhs > cap / 4) {
        log_error(kApi, "n*nrhs=%zu needs more than the %zu bytes of static scratch", (size_t)n * nrhs, cap);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    const size_t dbytes = ((size_t)n * nrhs * 4 + 255) / 256 * 256;
    if ((size_t)batchCount > (cap - 512) / (dbytes + 20)) {
        log_error(kApi,
                  "scratch required %zu bytes, but the static scratch holds %zu; split the batch or use "
                  "aclblasSgetrfsRefineBatchedEx with a workspace",
                  (dbytes + 20) * (size_t)batchCount + 512, cap);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    const size_t rsm = (size_t)(n + 16) * kResMaxRhs * 8;
    if (rsm > 200 * 1024) {
        log_error(kApi, "n=%d exceeds the residual kernel's shared-memory limit", n);
        return ACLBLAS_STATUS_NOT_SUPPORTED;
    }
    int device = -1;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) return launch_status(kApi, err);
    if (device != handle->device) {
        log_error(kApi, "the handle belongs to device %d but device %d is current", handle->device, device);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    char* ws = nullptr;
    aclblasStatus_t s = static_scratch_base(kApi, device, &ws);
    if (s != ACLBLAS_STATUS_SUCCESS) return s;

    float* dbase = reinterpret_cast<float*>(ws);
    float** dptr = reinterpret_cast<float**>(ws + dbytes * batchCount);
    float** dact = dptr + batchCount;  // dptr, or NULL for converged matrices
    int* done = reinterpret_cast<int*>(reinterpret_cast<char*>(dact) + (size_t)batchCount * 8);
    cudaStream_t st = handle->stream;
    const unsigned bgrid = (unsigned)((batchCount + 255) / 256 < 4096 ? (batchCount + 255) / 256 : 4096);

    init_ptr_array_kernel<<<bgrid, 256, 0, st>>>(dptr, dbase, (long long)(dbytes / 4), batchCount);
    fill_int_kernel<<<bgrid, 256, 0, st>>>(done, 0, batchCount);
    fill_int_kernel<<<bgrid, 256, 0, st>>>(iterArray, maxIter, batchCount);
    const bool tmem = mode != 0 && getrf_tmem_supported(n);  // reads A, writes LU: no copy
    // the blocked tensor-core LU (TF32 above n = 256) when the static scratch also holds its scratch,
    // after the refinement's part -- as the workspace entry point decides with its workspace
    const size_t used = ((dbytes + 20) * (size_t)batchCount + 512 + 255) / 256 * 256;
    const bool blocked = mode == 1 && getrf_blocked_tc_supported(n) &&
                         used + getrf_blocked_tc_scratch_bytes(n, batchCount) <= cap;
    if (!tmem && !blocked) copy_batched_kernel<<<(unsigned)batchCount, 256, 0, st>>>(Aarray, lda, LUarray, ldlu, n, n);
    err = cudaGetLastError();
    if (err != cudaSuccess) return launch_status(kApi, err);
    if (tmem) {
        err = getrf_tmem_launch(st, Aarray, lda, LUarray, n, ldlu, PivotArray, infoArray, batchCount, mode,
                                handle->dstatus);
    } else if (blocked) {  // reads A, writes LU
        err = getrf_blocked_tc_launch(st, Aarray, lda, LUarray, n, ldlu, PivotArray, infoArray, batchCount, ws + used,
                                      handle->dstatus, handle->tmslots);
    } else {  // plain FP32 factors: the batched getrf's kernels (stop codes in the static scratch)
        int* stat = used + sizeof(int) * (size_t)batchCount <= cap ? reinterpret_cast<int*>(ws + used) : nullptr;
        s = getrf_batched_impl(handle, n, LUarray, ldlu, PivotArray, infoArray, batchCount, stat);
        if (s != ACLBLAS_STATUS_SUCCESS) return s;
    }
    if (err != cudaSuccess || nrhs == 0) return launch_status(kApi, err);
    copy_batched_kernel<<<(unsigned)batchCount, 256, 0, st>>>(Barray, ldb, Xarray, ldx, n, nrhs);
    err = getrs_launch(st, false, n, nrhs, LUarray, ldlu, PivotArray, Xarray, ldx, batchCount);
    if (err != cudaSuccess) return launch_status(kApi, err);
    for (int it = 0; it < maxIter; it++) {
        refine_residual_kernel<<<(unsigned)batchCount, kResThreads, rsm, st>>>(
            n, nrhs, Aarray, lda, Barray, ldb, Xarray, ldx, dptr, n, dact, tol, it, 0, done, berrArray, iterArray);
        err = getrs_launch(st, false, n, nrhs, LUarray, ldlu, PivotArray, dact, n, batchCount);
        if (err != cudaSuccess) return launch_status(kApi, err);
        axpy_batched_kernel<<<(unsigned)batchCount, 256, 0, st>>>(n, nrhs, dact, n, Xarray, ldx);
    }
    refine_residual_kernel<<<(unsigned)batchCount, kResThreads, rsm, st>>>(
        n, nrhs, Aarray, lda, Barray, ldb, Xarray, ldx, dptr, n, dact, tol, maxIter, 1, done, berrArray, iterArray);
    return launch_status(kApi, cudaGetLastError());
}
