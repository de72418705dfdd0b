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
 * largest candidate magnitudes, the tie measure used by the tests.
 *
 * Exact ties above n = 256. The reference searches with 256 threads, thread t striding over
 * rows col+t, col+t+256, ..., and its tree reduction keeps the lower THREAD index on an exact
 * tie of magnitudes. For n <= 256 every thread holds at most one row and that equals the
 * lower row; above n = 256 a tie between rows col+t+256 and col+u (t < u) goes to the higher
 * row col+t+256. This function keeps the first row in every case. The tests compare pivots only
 * for matrices whose two largest candidates differ by more than 1e-5 relative at every step, so
 * the difference never reaches a comparison. */
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

/* aclblasSgeqrfBatched (blas/geqrf_batched/arch35/sgeqrf_batched_kernel.cpp:44-190): unblocked
 * Householder QR, for i = 0 .. min(m,n)-1:
 *   sigma = sum_{r>i} A(r,i)^2 (ComputeSigma :94-111), x1 = A(i,i);
 *   sigma == 0: tau = 0, A(i,i) unchanged, no update (ComputeTauAndNormalize :113-149);
 *   else normX = sqrt(sigma + x1*x1), alpha = x1 >= 0 ? -normX : normX, tau = (alpha - x1) / alpha,
 *        A(r,i) /= (x1 - alpha) for r > i, A(i,i) = alpha;
 *   then for every column c > i (ComputeCoefficients :44-60, ApplyUpdate :62-83):
 *        dot = A(i,c) + sum_{r>i} A(r,i) A(r,c), coef = tau * dot,
 *        A(r,c) -= coef * A(r,i) for r > i, A(i,c) = A(i,c) - coef.
 * The reference's sums are thread-tree reductions; this restatement (and the CUDA kernels,
 * which follow it bit for bit) sums in row order with every product rounded before the add.
 * Parity with the reference is by its own test rule: MIXED_TOLERANCE against LAPACK sgeqrf_
 * (tests/test_geqrf_oracle.py). */
/* a product rounded on its own (the file is compiled with -ffp-contract=off) */
static inline float rmul(float a, float b) { return a * b; }

static void oracle_sgeqrf(int m, int n, float* A, int lda, float* tau)
{
    const int k = m < n ? m : n;
    for (int i = 0; i < k; i++) {
        float* ci = A + (int64_t)i * lda;
        float sigma = 0.0f;
        for (int r = i + 1; r < m; r++) sigma = sigma + rmul(ci[r], ci[r]);
        const float x1 = ci[i];
        float t, alpha;
        if (sigma == 0.0f) {
            t = 0.0f;
            alpha = x1;
        } else {
            const float normX = sqrtf(sigma + rmul(x1, x1));
            alpha = (x1 >= 0.0f) ? -normX : normX;
            t = (alpha - x1) / alpha;
        }
        tau[i] = t;
        if (t == 0.0f) {
            ci[i] = alpha;
            continue;
        }
        const float vscale = x1 - alpha;
        for (int r = i + 1; r < m; r++) ci[r] = ci[r] / vscale;
        ci[i] = alpha;
        for (int c = i + 1; c < n; c++) {
            float* cc = A + (int64_t)c * lda;
            float dot = cc[i];
            for (int r = i + 1; r < m; r++) dot = dot + rmul(ci[r], cc[r]);
            const float coef = rmul(t, dot);
            for (int r = i + 1; r < m; r++) cc[r] = cc[r] - rmul(coef, ci[r]);
            cc[i] = cc[i] - coef;
        }
    }
}

ORACLE_API void oracle_sgeqrf_batched(int m, int n, float* A, int64_t strideA, int lda, float* tau,
                                      int64_t strideTau, int batch)
{
    for (int b = 0; b < batch; b++) oracle_sgeqrf(m, n, A + (int64_t)b * strideA, lda, tau + (int64_t)b * strideTau);
}

/* aclblasSgelsBatched (blas/gels_batched/arch35/sgels_batched_kernel.cpp:25-400), per matrix:
 * trans T first transposes A in place into an n x m matrix of leading dimension n
 * (SgelsTransposeSimt); then with (M, N) the effective shape:
 *   M >= N: Householder QR (column reflectors: xnorm = ||A(k+1:,k)||; xnorm < 1e-30 with
 *           A(k,k) >= 0 gives tau = 0; else the scaled norm nm = sc sqrt((akk/sc)^2 + (xnorm/sc)^2),
 *           beta = -sign(akk) nm, tau = (beta - akk)/beta, v *= 1/(akk - beta), A(k,k) = beta,
 *           columns j > k: w = v.a + a(k), a(k) -= tau w, a += (-tau w) v), Q^T applied to C the
 *           same way, then back substitution R x = c per right-hand side; a zero R(i,i) sets
 *           info = i + 1 and stops (the right-hand sides after the current one stay untouched);
 *   M <  N: LQ with row reflectors, forward substitution L y = c (same stop rule), C rows M..N-1
 *           zeroed, Q^T applied in reverse reflector order (the minimum-norm solution).
 * Sums run in index order with each product rounded before the add, as in the CUDA kernel. */
static float gels_norm(const float* v, int len, int stride)
{
    float ss = 0.0f;
    for (int i = 0; i < len; i++) ss = ss + rmul(v[(int64_t)i * stride], v[(int64_t)i * stride]);
    return sqrtf(ss);
}

/* Reflector k: returns 0 (tau = 0, no reflection) or 1 with tau and the scale of v. */
static int gels_reflector(float akk, float xnorm, float* tau, float* beta, float* scalev)
{
    if (xnorm < 1.0e-30f && akk >= 0.0f) {
        *tau = 0.0f;
        return 0;
    }
    const float na = fabsf(akk);
    const float sc = na > xnorm ? na : xnorm;
    const float sa = akk / sc, sx = xnorm / sc;
    const float nm = rmul(sc, sqrtf(rmul(sa, sa) + rmul(sx, sx)));
    *beta = akk >= 0.0f ? -nm : nm;
    *tau = (*beta - akk) / *beta;
    *scalev = 1.0f / (akk - *beta);
    return 1;
}

/* a(-stride) and a(0..len-1)*stride updated with the reflector (v, tau) */
static void gels_apply(const float* v, int vstride, float* a, int astride, int len, float t)
{
    float w = 0.0f;
    for (int i = 0; i < len; i++) w = w + rmul(v[(int64_t)i * vstride], a[(int64_t)i * astride]);
    w = w + a[-(int64_t)astride];
    a[-(int64_t)astride] = a[-(int64_t)astride] - rmul(t, w);
    const float alpha = -rmul(t, w);
    for (int i = 0; i < len; i++) a[(int64_t)i * astride] = a[(int64_t)i * astride] + rmul(alpha, v[(int64_t)i * vstride]);
}

static void oracle_sgels(int trans, int m, int n, int nrhs, float* A, int lda, float* C, int ldc, int* info,
                         float* scratch)
{
    int M = m, N = n, ld = lda;
    if (trans) {
        memcpy(scratch, A, sizeof(float) * (size_t)lda * n);
        for (int col = 0; col < m; col++)
            for (int row = 0; row < n; row++) A[(int64_t)col * n + row] = scratch[(int64_t)row * lda + col];
        M = n;
        N = m;
        ld = n;
    }
    const int k = M < N ? M : N;
    float tau[4096];
    if (M >= N) {
        for (int kk = 0; kk < N; kk++) {
            const int tail = M - kk - 1;
            float* v = A + (int64_t)kk * ld + kk + 1;
            const float akk = A[(int64_t)kk * ld + kk];
            float beta = 0.0f, scalev = 0.0f;
            if (!gels_reflector(akk, gels_norm(v, tail, 1), &tau[kk], &beta, &scalev)) continue;
            A[(int64_t)kk * ld + kk] = beta;
            for (int i = 0; i < tail; i++) v[i] = rmul(v[i], scalev);
            for (int j = kk + 1; j < N; j++) gels_apply(v, 1, A + (int64_t)j * ld + kk + 1, 1, tail, tau[kk]);
        }
        for (int kk = 0; kk < k; kk++) {
            if (tau[kk] == 0.0f) continue;
            const float* v = A + (int64_t)kk * ld + kk + 1;
            for (int j = 0; j < nrhs; j++) gels_apply(v, 1, C + (int64_t)j * ldc + kk + 1, 1, M - kk - 1, tau[kk]);
        }
        for (int j = 0; j < nrhs; j++) {
            for (int i = N - 1; i >= 0; i--) {
                const float rii = A[(int64_t)i * ld + i];
                if (rii == 0.0f) {
                    *info = i + 1;
                    return;
                }
                float sum = 0.0f;
                for (int p = i + 1; p < N; p++) sum = sum + rmul(A[(int64_t)p * ld + i], C[(int64_t)j * ldc + p]);
                C[(int64_t)j * ldc + i] = (C[(int64_t)j * ldc + i] - sum) / rii;
            }
        }
        *info = 0;
    } else {
        for (int kk = 0; kk < M; kk++) {
            const int tail = N - kk - 1;
            float* v = A + (int64_t)(kk + 1) * ld + kk;
            const float akk = A[(int64_t)kk * ld + kk];
            float beta = 0.0f, scalev = 0.0f;
            if (!gels_reflector(akk, gels_norm(v, tail, ld), &tau[kk], &beta, &scalev)) continue;
            A[(int64_t)kk * ld + kk] = beta;
            for (int i = 0; i < tail; i++) v[(int64_t)i * ld] = rmul(v[(int64_t)i * ld], scalev);
            for (int ii = kk + 1; ii < M; ii++) gels_apply(v, ld, A + (int64_t)(kk + 1) * ld + ii, ld, tail, tau[kk]);
        }
        *info = 0;
        for (int j = 0; j < nrhs; j++) {
            for (int i = 0; i < M; i++) {
                const float lii = A[(int64_t)i * ld + i];
                if (lii == 0.0f) {
                    *info = i + 1;
                    return;
                }
                float sum = 0.0f;
                for (int p = 0; p < i; p++) sum = sum + rmul(A[(int64_t)p * ld + i], C[(int64_t)j * ldc + p]);
                C[(int64_t)j * ldc + i] = (C[(int64_t)j * ldc + i] - sum) / lii;
            }
        }
        for (int j = 0; j < nrhs; j++)
            for (int i = M; i < N; i++) C[(int64_t)j * ldc + i] = 0.0f;
        for (int kk = M - 1; kk >= 0; kk--) {
            if (tau[kk] == 0.0f) continue;
            const float* v = A + (int64_t)(kk + 1) * ld + kk;
            for (int j = 0; j < nrhs; j++) gels_apply(v, ld, C + (int64_t)j * ldc + kk + 1, 1, N - kk - 1, tau[kk]);
        }
    }
}

ORACLE_API void oracle_sgels_batched(int trans, int m, int n, int nrhs, float* A, int64_t strideA, int lda, float* C,
                                     int64_t strideC, int ldc, int* info, int batch, float* scratch)
{
    for (int b = 0; b < batch; b++)
        oracle_sgels(trans, m, n, nrhs, A + (int64_t)b * strideA, lda, C + (int64_t)b * strideC, ldc, info + b,
                     scratch);
}

/* aclblasCgemmBatched (blas/gemm_batched/arch35/gemm_batched_host.cpp:438-819,
 * gemm_batched_kernel.cpp:848-1110). Complex values are interleaved (real, imaginary) float
 * pairs; op 0 = N, 1 = T, 2 = C (conjugate transpose: the imaginary part negated on the
 * de-interleave). Per output the four real sums T1 = sum Ar Br, T2 = sum Ai Bi, T3 = sum Ar Bi,
 * T4 = sum Ai Br (one fmaf per product, k in order, as this project's device kernel), then the
 * reference's combine with every product and sum rounded on its own:
 *   Pr = T1 - T2, Pi = T3 + T4, Cr = Pr aR - Pi aI, Ci = Pi aR + Pr aI;
 *   beta != 0: Cr += Cor bR, Ci += Coi bR, Cr -= Coi bI, Ci += Cor bI.
 * k == 0 or alpha == 0 combines zero sums (LaunchCgemmEarlyExit); with beta == 1 as well nothing
 * is written. A null C pointer skips the matrix. m, n, batch == 0 return at once. */
static void cg_elem(int op, const float* X, int ld, int r, int c, float* re, float* im)
{
    const int64_t idx = op == 0 ? (int64_t)r + (int64_t)c * ld : (int64_t)c + (int64_t)r * ld;
    *re = X[2 * idx];
    *im = op == 2 ? -X[2 * idx + 1] : X[2 * idx + 1];
}

ORACLE_API void oracle_cgemm_batched(int opa, int opb, int m, int n, int k, float alpha_re, float alpha_im,
                                     float beta_re, float beta_im, const float* const* A, int lda,
                                     const float* const* B, int ldb, float* const* C, int ldc, int batch)
{
    if (m == 0 || n == 0 || batch == 0) return;
    const int zero_product = k == 0 || (alpha_re == 0.0f && alpha_im == 0.0f);
    if (zero_product && beta_re == 1.0f && beta_im == 0.0f) return;
    const int keff = zero_product ? 0 : k;
    const int has_beta = beta_re != 0.0f || beta_im != 0.0f;
    for (int b = 0; b < batch; b++) {
        float* Cb = C[b];
        if (Cb == NULL) continue;
        for (int j = 0; j < n; j++)
            for (int i = 0; i < m; i++) {
                float t1 = 0.0f, t2 = 0.0f, t3 = 0.0f, t4 = 0.0f;
                for (int p = 0; p < keff; p++) {
                    float ar, ai, br, bi;
                    cg_elem(opa, A[b], lda, i, p, &ar, &ai);
                    cg_elem(opb, B[b], ldb, p, j, &br, &bi);
                    t1 = fmaf(ar, br, t1);
                    t2 = fmaf(ai, bi, t2);
                    t3 = fmaf(ar, bi, t3);
                    t4 = fmaf(ai, br, t4);
                }
                const float pr = t1 - t2, pi = t3 + t4;
                float cr = pr * alpha_re - pi * alpha_im;
                float ci = pi * alpha_re + pr * alpha_im;
                float* c = Cb + 2 * ((int64_t)i + (int64_t)j * ldc);
                if (has_beta) {
                    const float cor = c[0], coi = c[1];
                    cr = cr + cor * beta_re;
                    ci = ci + coi * beta_re;
                    cr = cr - coi * beta_im;
                    ci = ci + cor * beta_im;
                }
                c[0] = cr;
                c[1] = ci;
            }
    }
}
