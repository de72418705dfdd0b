/*
 * aclblas C API for the batched LU chain, B200 (sm_100a) build.
 *
 * Every entry point keeps the name, argument order, argument meaning, status codes and
 * validation order of the hicann/ops-blas function it replaces (cited per declaration), so that
 * code written against the reference's include/cann_ops_blas.h links against
 * libopsblas_b200.so unchanged. `aclrtStream` is a CUDA stream (include/acl/acl.h).
 *
 * Conventions shared by every batched routine:
 *   - matrices are FP32, column-major, element (i, j) at A[i + j * lda];
 *   - `Aarray` / `Barray` / `Carray` are DEVICE arrays of DEVICE pointers, one per matrix;
 *   - pivot and info arrays are DEVICE memory unless stated otherwise;
 *   - calls are asynchronous on the handle's stream: they never synchronise, never copy
 *     between host and device and never allocate, so they can be captured in a CUDA graph.
 */
#ifndef OPSBLAS_B200_CANN_OPS_BLAS_H
#define OPSBLAS_B200_CANN_OPS_BLAS_H

#include <stddef.h>
#include <stdint.h>
#include "acl/acl.h"
#include "cann_ops_blas_common.h"

#if defined(__GNUC__)
#define ACLBLAS_EXPORT __attribute__((visibility("default")))
#else
#define ACLBLAS_EXPORT
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct _aclblas_handle* aclblasHandle_t;
typedef void (*aclblasLogCallback)(const char*);

/* ---------------------------------------------------------------- handle and runtime --- */

/* Replaces aclblasCreate (include/cann_ops_blas.h:41; blas/common/helper/aclblas_auxiliary.cpp:24-48).
 * *handle must be NULL on entry. Allocates the 32 MiB default device workspace on the current
 * device. HANDLE_IS_NULLPTR if handle is NULL, INVALID_VALUE if *handle is not NULL,
 * ALLOC_FAILED if the workspace cannot be allocated. */
ACLBLAS_EXPORT aclblasStatus_t aclblasCreate(aclblasHandle_t* handle);

/* Replaces aclblasDestroy (include/cann_ops_blas.h:54; aclblas_auxiliary.cpp:50-71).
 * Synchronises the bound stream, frees the library workspace, never frees user workspace.
 * EXECUTION_FAILED if the stream synchronisation fails. */
ACLBLAS_EXPORT aclblasStatus_t aclblasDestroy(aclblasHandle_t handle);

/* Replaces aclblasSetStream (include/cann_ops_blas.h:66; aclblas_auxiliary.cpp:73-90).
 * Switching streams reverts the handle to the library workspace. */
ACLBLAS_EXPORT aclblasStatus_t aclblasSetStream(aclblasHandle_t handle, aclrtStream stream);

/* Replaces aclblasGetStream (include/cann_ops_blas.h:76; aclblas_auxiliary.cpp:92-104). */
ACLBLAS_EXPORT aclblasStatus_t aclblasGetStream(aclblasHandle_t handle, aclrtStream* stream);

/* Replaces aclblasSetWorkspace (include/cann_ops_blas.h:93; aclblas_auxiliary.cpp:106-137).
 * Borrows user device memory; grow-only (a smaller size than the current user workspace is
 * ignored). INVALID_VALUE if workspace is NULL or workspaceSize is 0. */
ACLBLAS_EXPORT aclblasStatus_t aclblasSetWorkspace(aclblasHandle_t handle, void* workspace, size_t workspaceSize);

/* Replaces aclblasGetVersion (include/cann_ops_blas.h:105; aclblas_auxiliary.cpp:139-148).
 * MAJOR*10000 + MINOR*100 + PATCH; handle may be NULL. */
ACLBLAS_EXPORT aclblasStatus_t aclblasGetVersion(aclblasHandle_t handle, int* version);

/* Replace the logger trio (include/cann_ops_blas.h:116-133;
 * blas/common/helper/aclblas_logger_manager.cpp:19-48). Unlike the reference, whose
 * configuration is stored but never consumed, messages of this library (validation failures,
 * launch errors) are delivered to the callback, stdout, stderr and/or the file. */
ACLBLAS_EXPORT aclblasStatus_t aclblasLoggerConfigure(int logIsOn, int logToStdOut, int logToStdErr, const char* logFile);
ACLBLAS_EXPORT aclblasStatus_t aclblasSetLoggerCallback(aclblasLogCallback userCallback);
ACLBLAS_EXPORT aclblasStatus_t aclblasGetLoggerCallback(aclblasLogCallback* userCallback);

/* Extension (no counterpart in the reference, whose kernels have no waits that can give up).
 * Every wait inside this library's kernels (on a bulk copy or on tensor-core MMAs) is bounded;
 * a kernel whose wait gives up stops its work, lets its copies in flight land and sets a bit in
 * the handle's device status word instead of faulting or hanging. This call synchronises the
 * handle's stream, returns the bits set since the previous call in *flags and clears them:
 * bit 0 a getrf bulk copy, bit 1 the mixed-precision TMEM LU, bit 2 the tcgen05 GEMM. It
 * returns ACLBLAS_STATUS_EXECUTION_FAILED when any bit was set (the results of the calls since
 * the previous check are then incomplete), else ACLBLAS_STATUS_SUCCESS. */
ACLBLAS_EXPORT aclblasStatus_t aclblasGetDeviceStatus(aclblasHandle_t handle, unsigned int* flags);

/* ------------------------------------------------------------------ batched LU chain --- */

/* Replaces aclblasSgetrfBatched (include/cann_ops_blas.h:403;
 * blas/getrf_batched/arch35/sgetrf_batched_host.cpp:66-118, kernel sgetrf_batched_kernel.cpp:106-197).
 * In-place P*A = L*U with partial pivoting; PivotArray == NULL selects no pivoting.
 * PivotArray: n ints per matrix, 1-based. infoArray: one int per matrix, 0 or the 1-based
 * column of the first exactly-zero pivot; factorisation of that matrix stops there.
 * Validation order (sgetrf_batched_host.cpp:32-64): n < 0, batchSize < 0, lda < max(1,n)
 * -> INVALID_VALUE; n == 0 or batchSize == 0 -> SUCCESS with nothing touched;
 * Aarray == NULL, or PivotArray != NULL with infoArray == NULL -> INVALID_VALUE.
 * Deliberate strengthening: for a singular matrix (info = k > 0) PivotArray[k..n-1] is
 * written as 0, the value the reference's golden model expects
 * (test/getrf_batched/sgetrf_batched/sgetrf_batched_golden.h:78-82) and its test wrapper
 * only gets by pre-zeroing. For 128 < n <= 1024 the factorisation is blocked and uses the first
 * 4 * batchSize bytes of the handle workspace (the reference's kernel uses none); with a smaller
 * workspace it takes an unblocked-order kernel with the same results (n <= 640) or the generic
 * one. Results are bit-identical either way. */
ACLBLAS_EXPORT aclblasStatus_t aclblasSgetrfBatched(
    aclblasHandle_t handle, int n, float* const Aarray[], int lda, int* PivotArray, int* infoArray, int batchSize);

/* Replaces aclblasSgetrsBatched (include/cann_ops_blas.h:457;
 * blas/getrs_batched/arch35/sgetrs_batched_host.cpp:49-185, kernel sgetrs_batched_kernel.cpp:83-388).
 * Solves op(A) X = B with the LU factors and pivots of aclblasSgetrfBatched; B is overwritten
 * by X. devIpiv == NULL means no pivoting. `info` is a HOST pointer (may be NULL) that receives
 * 0, or -position of the first invalid argument (trans=2, n=3, nrhs=4, Aarray=5, lda=6,
 * Barray=8, ldb=9, batchCount=11). An invalid trans returns INVALID_ENUM; nrhs is limited to
 * 0..256 as in the reference. */
ACLBLAS_EXPORT aclblasStatus_t aclblasSgetrsBatched(
    aclblasHandle_t handle, aclblasOperation_t trans, int n, int nrhs, const float* const Aarray[], int lda,
    const int* devIpiv, float* const Barray[], int ldb, int* info, int batchCount);

/* Replaces aclblasSgetriBatched (include/cann_ops_blas.h:430;
 * blas/getri_batched/arch35/getri_batched_host.cpp:27-127, kernel getri_batched_kernel.cpp:39-308).
 * Carray[i] = inverse of the matrix whose LU factors are in Aarray[i] (out of place; C must
 * not alias A). PivotArray == NULL means no pivoting. infoArray (required) receives 0, or j+1
 * for the highest-index j with U(j,j) == 0 (the reference's backward sweep stops there). */
ACLBLAS_EXPORT aclblasStatus_t aclblasSgetriBatched(
    aclblasHandle_t handle, int n, const float* const Aarray[], int lda, const int* PivotArray,
    float* const Carray[], int ldc, int* infoArray, int batchSize);

/* Extension (no counterpart): ptrArray[i] = (char*)base + i * strideBytes for i < count, written
 * on the handle's stream by a kernel (ptrArray is device memory with count entries). */
ACLBLAS_EXPORT aclblasStatus_t aclblasBuildPointerArray(
    aclblasHandle_t handle, const void* base, long long strideBytes, int count, void** ptrArray);

/* Extensions (no counterpart): strided-batch forms of aclblasSgetrfBatched / SgetrsBatched /
 * SgetriBatched -- matrix i at base + i * stride (elements). The pointer arrays are built in the
 * handle's workspace (8 bytes per matrix and operand, 256-byte aligned; EXECUTION_FAILED when it
 * is too small) and the batched entry points run on them: same validation, same results. */
ACLBLAS_EXPORT aclblasStatus_t aclblasSgetrfStridedBatched(
    aclblasHandle_t handle, int n, float* A, int lda, long long strideA, int* PivotArray, int* infoArray,
    int batchSize);
ACLBLAS_EXPORT aclblasStatus_t aclblasSgetrsStridedBatched(
    aclblasHandle_t handle, aclblasOperation_t trans, int n, int nrhs, const float* A, int lda, long long strideA,
    const int* devIpiv, float* B, int ldb, long long strideB, int* info, int batchCount);
ACLBLAS_EXPORT aclblasStatus_t aclblasSgetriStridedBatched(
    aclblasHandle_t handle, int n, const float* A, int lda, long long strideA, const int* PivotArray, float* C,
    int ldc, long long strideC, int* infoArray, int batchSize);

/* Replaces aclblasSgeqrfBatched (include/cann_ops_blas.h:399;
 * blas/geqrf_batched/arch35/sgeqrf_batched_host.cpp:19-141). Householder QR of every
 * m x n matrix in place (R above, the reflectors below the diagonal), TauArray[i] receives
 * min(m,n) scalars. info is HOST memory: 0, or the LAPACK-style -position of the first invalid
 * argument (m=1, n=2, Aarray=3, lda=4, TauArray=5, batchSize=6). */
ACLBLAS_EXPORT aclblasStatus_t aclblasSgeqrfBatched(
    aclblasHandle_t handle, int m, int n, float* const Aarray[], int lda, float* const TauArray[], int* info,
    int batchSize);

/* Replaces aclblasSgelsBatched (include/cann_ops_blas.h:405;
 * blas/gels_batched/arch35/sgels_batched_host.cpp:23-190). Least squares (m >= n after op) or
 * minimum-norm (m < n) solutions of op(A[i]) X = C[i] by Householder QR / LQ, trans N or T;
 * C[i] (ldc >= max(m, n)) receives the solutions, A[i] the factors (for T: of A^T, stored n x m
 * with leading dimension n). devInfo[i] (device, one per matrix) is 0 or i+1 for a zero
 * triangular diagonal. trans T needs lda * n <= 51200 (shared-memory transpose), otherwise
 * NOT_SUPPORTED. */
ACLBLAS_EXPORT aclblasStatus_t aclblasSgelsBatched(
    aclblasHandle_t handle, aclblasOperation_t trans, int m, int n, int nrhs, float* const Aarray[], int lda,
    float* const Carray[], int ldc, int* devInfo, int batchSize);

/* Replaces aclblasSgemmBatched (include/cann_ops_blas.h:415;
 * blas/gemm_batched/arch35/gemm_batched_host.cpp:397-435). C[i] = alpha * op(A[i]) * op(B[i]) +
 * beta * C[i] in FP32 (plain FP32 products and accumulation), alpha and beta host floats. k == 0
 * or alpha == 0 scales C by beta (beta == 1: C untouched); an operation outside N/T/C is
 * INVALID_VALUE. */
ACLBLAS_EXPORT aclblasStatus_t aclblasSgemmBatched(
    aclblasHandle_t handle, aclblasOperation_t transa, aclblasOperation_t transb, int m, int n, int k,
    const float* alpha, const float* const Aarray[], int lda, const float* const Barray[], int ldb,
    const float* beta, float* const Carray[], int ldc, int batchCount);

/* Replaces aclblasCgemmBatched (include/cann_ops_blas.h:423;
 * blas/gemm_batched/arch35/gemm_batched_host.cpp:462-508, 767-819). C[i] = alpha * op(A[i]) *
 * op(B[i]) + beta * C[i] in single-precision complex, op N, T or C (conjugate transpose), alpha
 * and beta host values. The reference's decomposition: four FP32 sums T1 = sum Ar Br,
 * T2 = sum Ai Bi, T3 = sum Ar Bi, T4 = sum Ai Br, then P = (T1 - T2, T3 + T4) and
 * C = alpha P (+ beta C when beta != 0), each product and sum rounded separately. k == 0 or
 * alpha == 0 takes P = 0 (beta == 1: C untouched). A null C[i] skips matrix i. Matrix pointers
 * are 8-byte aligned (as cuComplex). Validation order of ValidateCgemmBatchedParams; every
 * failure is INVALID_VALUE except the null handle. */
ACLBLAS_EXPORT aclblasStatus_t aclblasCgemmBatched(
    aclblasHandle_t handle, aclblasOperation_t transa, aclblasOperation_t transb, int m, int n, int k,
    const aclblasComplex* alpha, const aclblasComplex* const Aarray[], int lda, const aclblasComplex* const Barray[],
    int ldb, const aclblasComplex* beta, aclblasComplex* const Carray[], int ldc, int batchCount);

/* Replaces aclblasSmatinvBatched (include/cann_ops_blas.h:434;
 * blas/matinv_batched/arch35/matinv_batched_host.cpp:44-257). Ainv[i] = inverse of A[i] for
 * n <= 32, as aclblasSgetrfBatched on a copy of A followed by aclblasSgetriBatched (bit for
 * bit), in one launch and without workspace. info (required, device) receives 0, or the getri's
 * j+1 for the highest-index j with U(j,j) == 0 when A is singular. n > 32 is INVALID_VALUE. */
ACLBLAS_EXPORT aclblasStatus_t aclblasSmatinvBatched(
    aclblasHandle_t handle, int n, const float* const A[], int lda, float* const Ainv[], int lda_inv, int* info,
    int batchSize);

/* Replaces aclblasGemmBatchedEx (include/cann_ops_blas.h:409;
 * blas/gemm_batched_ex/arch35/gemm_batched_ex_host.cpp:156-581). C[i] = alpha*op(A[i])*op(B[i]) +
 * beta*C[i]; alpha and beta are HOST pointers to float. Validation order: handle, alpha/beta
 * (INVALID_VALUE), m/n/k/trans/batchCount (INVALID_VALUE), lda/ldb/ldc (INVALID_VALUE), algo !=
 * DEFAULT (NOT_SUPPORTED), dtype combination (NOT_SUPPORTED), NULL arrays when batchCount > 0
 * (INVALID_VALUE). Dtype combinations: the reference's FP16/BF16/FP8 table
 * (gemm_batched_ex_host.cpp:87-118) plus FP32/FP32/FP32 with ACLBLAS_COMPUTE_32F_PEDANTIC (plain
 * FP32), ACLBLAS_COMPUTE_32F_FAST_TF32 or ACLBLAS_COMPUTE_32F_FAST_16BF (FP32 under
 * ACLBLAS_COMPUTE_32F stays NOT_SUPPORTED, as in the reference). No workspace, no host copy. */
ACLBLAS_EXPORT aclblasStatus_t aclblasGemmBatchedEx(
    aclblasHandle_t handle, aclblasOperation_t transa, aclblasOperation_t transb, int m, int n, int k,
    const void* alpha, const void* const Aarray[], aclDataType Atype, int lda, const void* const Barray[],
    aclDataType Btype, int ldb, const void* beta, void* const Carray[], aclDataType Ctype, int ldc, int batchCount,
    aclblasComputeType_t computeType, aclblasGemmAlgo_t algo);

/* ------------------------------------------------------------------------ extensions --- */

/* Factor, solve and refine in one call; no counterpart in the reference. Aarray (kept
 * unchanged) is copied to LUarray and factored (PivotArray, infoArray as for
 * aclblasSgetrfBatched); computeType ACLBLAS_COMPUTE_32F factors in plain FP32,
 * ACLBLAS_COMPUTE_32F_FAST_TF32 / _FAST_16BF use a split (hi + lo) TF32 / BF16 trailing update.
 * X = LU \ B, then up to maxIter refinement steps: r = B - A X and the normwise backward error
 * max_c ||r_c||inf / (||A||inf ||x_c||inf + ||b_c||inf) are computed in FP64 on the GPU;
 * matrices whose error is <= tol stop, the others add LU \ r to X. berrArray (double),
 * iterArray (refinement steps used; maxIter if not converged) and infoArray are device arrays.
 * Needs n*nrhs*4 (rounded up to 256) + 20 bytes per matrix (+ 512) of handle workspace
 * (aclblasSetWorkspace); EXECUTION_FAILED if it is smaller. With _FAST_TF32 and 256 < n <= 1024
 * the factorization is blocked (FP32 panels of 32 columns, split-TF32 tensor-core trailing
 * updates) when the workspace holds, after that amount rounded up to 256, another P + 16 bytes
 * per matrix + 512, P = 2*(n-32)*128 rounded up to 256, twice;
 * with less, and for _FAST_16BF above n = 256, the factors are plain FP32. */
ACLBLAS_EXPORT aclblasStatus_t aclblasSgetrfsRefineBatchedEx(
    aclblasHandle_t handle, int n, int nrhs, const float* const Aarray[], int lda, float* const LUarray[], int ldlu,
    int* PivotArray, const float* const Barray[], int ldb, float* const Xarray[], int ldx,
    aclblasComputeType_t computeType, int maxIter, double tol, double* berrArray, int* iterArray, int* infoArray,
    int batchCount);

/* Bytes of device scratch that aclblasSgetrfsRefineBatchedStaticScratch can use. */
#define ACLBLAS_REFINE_STATIC_SCRATCH_BYTES ((size_t)8 << 20)

/* aclblasSgetrfsRefineBatchedEx without a workspace; no counterpart in the reference. For callers
 * that cannot give the library device memory (the host application owns it all, or must not
 * call cudaMalloc/cudaFree, which synchronise the device): the call allocates nothing and
 * leaves the handle workspace alone. Its scratch is a fixed array of
 * ACLBLAS_REFINE_STATIC_SCRATCH_BYTES in the library's device image, one per device; a call
 * needs (n*nrhs*4 rounded up to 256 + 20) * batchCount + 512 bytes of it, and a larger request
 * returns ACLBLAS_STATUS_INVALID_VALUE without launching anything. With _FAST_TF32 and
 * 256 < n <= 1024 the factorization is blocked when the rest of the scratch holds the blocked LU's
 * part (as aclblasSgetrfsRefineBatchedEx decides with its workspace), else plain FP32. The first call on each device
 * (with the handle's device current) sets up the scratch address; make it before any stream
 * capture. The address is kept for the life of the process, so the entry point must not be used
 * on a device after a cudaDeviceReset of that device. The scratch is shared by all handles and streams of the process: calls that overlap
 * in time on one device race on it; calls one after another on one stream are safe. Arguments,
 * results and status codes are otherwise those of aclblasSgetrfsRefineBatchedEx. */
ACLBLAS_EXPORT aclblasStatus_t aclblasSgetrfsRefineBatchedStaticScratch(
    aclblasHandle_t handle, int n, int nrhs, const float* const Aarray[], int lda, float* const LUarray[], int ldlu,
    int* PivotArray, const float* const Barray[], int ldb, float* const Xarray[], int ldx,
    aclblasComputeType_t computeType, int maxIter, double tol, double* berrArray, int* iterArray, int* infoArray,
    int batchCount);

/* Adjoint of the batched solve X = A^{-1} B; no counterpart in the reference. With the LU
 * factors / pivots of aclblasSgetrfBatched, the solution X and the upstream gradient dX:
 * dX is overwritten by dB = A^{-T} dX (transposed solve on the stored factors) and, when
 * dAarray is not NULL, dA = -dB X^T is written (overwritten, not accumulated). nrhs <= 256. */
ACLBLAS_EXPORT aclblasStatus_t aclblasSgetrsAdjointBatched(
    aclblasHandle_t handle, int n, int nrhs, const float* const LUarray[], int lda, const int* devIpiv,
    const float* const Xarray[], int ldx, float* const dXarray[], int lddx, float* const dAarray[], int ldda,
    int batchCount);

/* Grouped factor + solve of matrices of different orders; no counterpart in the reference.
 * A plan describes groupCount groups (host arrays): group g has groupSizeArray[g] instances of
 * order nArray[g], nrhsArray[g] right-hand sides (0: factor only), leading dimensions
 * ldaArray[g] / ldbArray[g]. Instances are numbered group by group. configArray is NULL or holds
 * 3 ints per group {lanes per matrix (n <= 32: 4/8/16/32), warps per matrix (n > 32: 2, 4 or 8),
 * rows per lane (n > 32: 2, 3 or 4, with 32 * rows >= n; 2 warps only with 2 rows, 4 rows need
 * 8 warps)}, 0 = take the tuning table's choice; the table is the file
 * named by OPSBLAS_GROUPED_TUNING, else grouped_tuning.txt beside the library, else built-in
 * defaults. Invalid choices are replaced; aclblasSgetrfGetrsGroupedPlanGetConfig returns the
 * ones in use. Creating a plan allocates and uploads its task lists (synchronously). */
typedef struct _aclblas_grouped_plan* aclblasGroupedPlan_t;

ACLBLAS_EXPORT aclblasStatus_t aclblasSgetrfGetrsGroupedPlanCreate(
    aclblasHandle_t handle, int groupCount, const int nArray[], const int nrhsArray[], const int ldaArray[],
    const int ldbArray[], const int groupSizeArray[], const int* configArray, aclblasGroupedPlan_t* plan);

ACLBLAS_EXPORT aclblasStatus_t aclblasSgetrfGetrsGroupedPlanGetConfig(aclblasGroupedPlan_t plan, int* configArray);

ACLBLAS_EXPORT aclblasStatus_t aclblasSgetrfGetrsGroupedPlanDestroy(aclblasGroupedPlan_t plan);

/* Executes a plan on the handle's stream: for every instance i, Aarray[i] is factored in place
 * (P*A = L*U, pivots at PivotArray + sum of the orders of the instances before i, infoArray[i]
 * as aclblasSgetrfBatched) and Barray[i] (n x nrhs) is overwritten by the solution X of A X = B
 * (as aclblasSgetrsBatched with trans N); the results equal those two calls bit for bit.
 * Instances with n <= 128 run in one persistent launch; larger ones use the batched kernels.
 * No allocation and no host synchronisation. Executions of one plan must not overlap in time
 * (they share the plan's work counters). */
ACLBLAS_EXPORT aclblasStatus_t aclblasSgetrfGetrsGroupedBatched(
    aclblasHandle_t handle, aclblasGroupedPlan_t plan, float* const Aarray[], int* PivotArray, int* infoArray,
    float* const Barray[]);

#ifdef __cplusplus
}
#endif

#endif /* OPSBLAS_B200_CANN_OPS_BLAS_H */
