/*
 * CPU oracle for the batched LU chain -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C, the arithmetic of the reference's device kernels for
 * aclblasSgetrfBatched / aclblasSgetrsBatched / aclblasSgetriBatched (hicann/ops-blas,
 * AscendC SIMT kernels). It is the checker the tests and the bench's CPU-baseline leg compare
 * the CUDA kernels against; the library never links, loads or calls it.
 *
 * Arithmetic model. Every update `x -= a * b` of the reference source is evaluated as one
 * fused multiply-add fmaf(-a, b, x) (a contraction the C++ source permits and the CUDA
 * kernels perform), every multiplier and every triangular-solve pivot step uses true IEEE
 * division, and loops run in the reference's order. With that model the CUDA register-resident
 * kernels for n <= 32 agree with this oracle bit for bit, which the GPU tests check.
 *
 * Parity pin. This restatement is checked against the reference's own golden path (LAPACK
 * sgetrf_/sgetrs_/sgetri_ called by the reference's test headers, compiled in place by
 * oracle/build_oracle.py into oracle/_ref/) on the reference's CSV test cases; see
 * tests/test_oracle_pin.py.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define ORACLE_API __attribute__((visibility("default")))

/* Pivot search of FindPivotRow (blas/getrf_batched/arch35/sgetrf_batched_kernel.cpp:52-79):
 * the first row r >= col with the largest |A(r,col)| strictly greater than zero; when every
 * candidate is zero or NaN the result is col. Also returns the relative gap between the two
 * largest candidate magnitudes, the tie measure used by the tests. */
static int find_pivot(const float* A, int lda, int col, int n, double* gap)
{
    float best = 0.0f, second = 0.0f;
    int row = col;
    for (int r = col; r < n; r++) {
        float v = fabsf(A[r + (int64_t)col * lda]);
        if (v > best) {
            second = best;
            best = v;
            row = r;
        } else if (v > second) {
            second = v; /* an exact tie with best lands here and gives gap 0 */
        }
    }
    if (gap) *gap = (best > 0.0f) ? ((double)best - (double)second) / (double)best : 0.0;
    return row;
}

/* GetrfSimtPivot (sgetrf_batched_kernel.cpp:106-150): unblocked right-looking LU, full-row
 * swaps (SwapRows :81-91), multipliers by division (ComputeMultipliers :93-104), rank-1
 * update (Rank1Update :38-50). On the first exactly-zero pivot: piv[col] is written, info =
 * col+1, and the factorisation stops before the swap. piv[k] for k > col is set to 0 (the
 * golden contract, sgetrf_batched_golden.h:78-82). min_gap (may be NULL) receives the
 * smallest relative pivot gap over the steps taken. */
ORACLE_API void oracle_sgetrf(int n, float* A, int lda, int* piv, int* info, double* min_gap)
{
    int inf = 0;
    double mg = 1.0;
    int col;
    for (col = 0; col < n; col++) {
        double g;
        int p = find_pivot(A, lda, col, n, &g);
        if (g < mg) mg = g;
        float pv = A[p + (int64_t)col * lda];
        piv[col] = p + 1;
        if (pv == 0.0f) {
            inf = col + 1;
            break;
        }
        if (p != col) {
            for (int c = 0; c < n; c++) {
                float t = A[col + (int64_t)c * lda];
                A[col + (int64_t)c * lda] = A[p + (int64_t)c * lda];
                A[p + (int64_t)c * lda] = t;
            }
        }
        float d = A[col + (int64_t)col * lda];
        for (int r = col + 1; r < n; r++) A[r + (int64_t)col * lda] = A[r + (int64_t)col * lda] / d;
        for (int c = col + 1; c < n; c++) {
            float u = A[col + (int64_t)c * lda];
            for (int r = col + 1; r < n; r++) {
                float l = A[r + (int64_t)col * lda];
                A[r + (int64_t)c * lda] = fmaf(-l, u, A[r + (int64_t)c * lda]);
            }
        }
    }
    if (inf) {
        for (int k = col + 1; k < n; k++) piv[k] = 0;
    }
    *info = inf;
    if (min_gap) *min_gap = mg;
}

/* GetrfSimtNoPivot (sgetrf_batched_kernel.cpp:152-197). */
ORACLE_API void oracle_sgetrf_nopiv(int n, float* A, int lda, int* info)
{
    int inf = 0;
    for (int col = 0; col < n; col++) {
        float d = A[col + (int64_t)col * lda];
        if (d == 0.0f) {
            inf = col + 1;
            break;
        }
        for (int r = col + 1; r < n; r++) A[r + (int64_t)col * lda] = A[r + (int64_t)col * lda] / d;
        for (int c = col + 1; c < n; c++) {
            float u = A[col + (int64_t)c * lda];
            for (int r = col + 1; r < n; r++) {
                float l = A[r + (int64_t)col * lda];
                A[r + (int64_t)c * lda] = fmaf(-l, u, A[r + (int64_t)c * lda]);
            }
        }
    }
    if (info) *info = inf;
}

/* Strided batch driver: matrix b starts at A + b*strideA (elements). */
ORACLE_API void oracle_sgetrf_batched(
    int n, float* A, int64_t strideA, int lda, int* piv, int* info, double* min_gap, int batch)
{
    for (int b = 0; b < batch; b++) {
        float* Ab = A + (int64_t)b * strideA;
        if (piv) {
            oracle_sgetrf(n, Ab, lda, piv + (int64_t)b * n, info + b, min_gap ? min_gap + b : 0);
        } else {
            oracle_sgetrf_nopiv(n, Ab, lda, info ? info + b : 0);
            if (min_gap) min_gap[b] = 1.0;
        }
    }
}

/* Row interchanges of ApplyPermutationNrhs (sgetrs_batched_kernel.cpp:83-120), forward order,
 * and ApplyInversePermutationNrhs (:123-163), reverse order. Out-of-range and self pivots
 * (including the zeros written for singular matrices) are skipped. */
static void laswp(float* B, int ldb, int n, int nrhs, const int* piv, int reverse)
{
    for (int t = 0; t < n; t++) {
        int k = reverse ? n - 1 - t : t;
        int p = piv[k] - 1;
        if (p >= 0 && p < n && p != k) {
            for (int c = 0; c < nrhs; c++) {
                float tmp = B[k + (int64_t)c * ldb];
                B[k + (int64_t)c * ldb] = B[p + (int64_t)c * ldb];
                B[p + (int64_t)c * ldb] = tmp;
            }
        }
    }
}

/* GetrsSimtPivot / GetrsSimtNoPivot (sgetrs_batched_kernel.cpp:365-410) for one matrix.
 * trans: 0 = N, 1 = T, 2 = C (real data, so C == T). N: laswp, unit-L forward
 * (ForwardSolveNrhs :167-202), U backward with division (BackwardSolveNrhs :205-259).
 * T/C: U^T forward with division (:263-315), unit L^T backward (:319-362), reverse laswp. */
ORACLE_API void oracle_sgetrs(
    int trans, int n, int nrhs, const float* LU, int lda, const int* piv, float* B, int ldb)
{
    if (trans == 0) {
        if (piv) laswp(B, ldb, n, nrhs, piv, 0);
        for (int c = 0; c < nrhs; c++) {
            float* x = B + (int64_t)c * ldb;
            for (int j = 0; j < n; j++) {
                float xj = x[j];
                for (int i = j + 1; i < n; i++) x[i] = fmaf(-LU[i + (int64_t)j * lda], xj, x[i]);
            }
            for (int j = n - 1; j >= 0; j--) {
                float xj = x[j] / LU[j + (int64_t)j * lda];
                x[j] = xj;
                for (int i = 0; i < j; i++) x[i] = fmaf(-LU[i + (int64_t)j * lda], xj, x[i]);
            }
        }
    } else {
        for (int c = 0; c < nrhs; c++) {
            float* x = B + (int64_t)c * ldb;
            for (int j = 0; j < n; j++) {
                float xj = x[j] / LU[j + (int64_t)j * lda];
                x[j] = xj;
                for (int i = j + 1; i < n; i++) x[i] = fmaf(-LU[j + (int64_t)i * lda], xj, x[i]);
            }
            for (int j = n - 1; j >= 0; j--) {
                float s = x[j];
                for (int i = j + 1; i < n; i++) s = fmaf(-LU[i + (int64_t)j * lda], x[i], s);
                x[j] = s;
            }
        }
        if (piv) laswp(B, ldb, n, nrhs, piv, 1);
    }
}

ORACLE_API void oracle_sgetrs_batched(
    int trans, int n, int nrhs, const float* LU, int64_t strideA, int lda, const int* piv, float* B,
    int64_t strideB, int ldb, int batch)
{
    for (int b = 0; b < batch; b++) {
        oracle_sgetrs(trans, n, nrhs, LU + (int64_t)b * strideA, lda, piv ? piv + (int64_t)b * n : 0,
                      B + (int64_t)b * strideB, ldb);
    }
}

/* GetriSimtPivot / GetriSimtNoPivot (blas/getri_batched/arch35/getri_batched_kernel.cpp:211-274)
 * for one matrix: C = I (InitIdentity :39-47), row interchanges (ApplyPermutation :52-88),
 * unit-L forward solve (ForwardSolve :95-128), U backward solve (BackwardSolve :131-208).
 * The backward sweep runs j = n-1..0 and stops at the first U(j,j) == 0 it meets, so info is
 * the HIGHEST zero diagonal index + 1. On that stop the reference leaves C as follows: for
 * n <= 8 (register path, :163-168) C holds the forward-solve result; for n > 8 C holds the
 * partially updated columns. Both are restated. */
ORACLE_API void oracle_sgetri(int n, const float* LU, int lda, const int* piv, float* C, int ldc, int* info)
{
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) C[i + (int64_t)j * ldc] = (i == j) ? 1.0f : 0.0f;
    if (piv) laswp(C, ldc, n, n, piv, 0);
    for (int c = 0; c < n; c++) {
        float* x = C + (int64_t)c * ldc;
        for (int j = 0; j < n; j++) {
            float xj = x[j];
            for (int i = j + 1; i < n; i++) x[i] = fmaf(-LU[i + (int64_t)j * lda], xj, x[i]);
        }
    }
    int inf = 0;
    for (int j = n - 1; j >= 0; j--) {
        if (LU[j + (int64_t)j * lda] == 0.0f) {
            inf = j + 1;
            break;
        }
    }
    if (inf && n <= 8) {
        *info = inf; /* register path: forward result stays in C */
        return;
    }
    for (int j = n - 1; j >= 0; j--) {
        float ujj = LU[j + (int64_t)j * lda];
        if (ujj == 0.0f) break;
        for (int c = 0; c < n; c++) {
            float* x = C + (int64_t)c * ldc;
            float xj = x[j] / ujj;
            x[j] = xj;
            for (int i = 0; i < j; i++) x[i] = fmaf(-LU[i + (int64_t)j * lda], xj, x[i]);
        }
    }
    *info = inf;
}

ORACLE_API void oracle_sgetri_batched(
    int n, const float* LU, int64_t strideA, int lda, const int* piv, float* C, int64_t strideC, int ldc, int* info,
    int batch)
{
    for (int b = 0; b < batch; b++) {
        oracle_sgetri(n, LU + (int64_t)b * strideA, lda, piv ? piv + (int64_t)b * n : 0, C + (int64_t)b * strideC,
                      ldc, info + b);
    }
}
