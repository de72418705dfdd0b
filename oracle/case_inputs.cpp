/*
 * Input generators of the reference's batched-LU test suites -- TEST INFRASTRUCTURE ONLY.
 *
 * Restates, with the same engine (std::mt19937), the same distributions
 * (std::uniform_real_distribution<float>) and the same draw order, the matrices the reference
 * tests build, so that the tests here run the reference's CSV cases on the reference's own
 * inputs:
 *   makeBlasLapackMatrix           test/frame/fill.h:587-740 (getrs / getri suites)
 *   generateMatrix                 test/getrf_batched/sgetrf_batched/arch35/sgetrf_batched_test.cpp:29-141
 *                                  (same draws as makeBlasLapackMatrix for the types it has)
 *   GenerateBMatrix                test/getrs_batched/arch35/getrs_batched_test.cpp:31-47
 * Seeds: matrix b of a batch uses seed + b*1000; right-hand sides use seed + b*1000 + 500.
 */
#include <algorithm>
#include <cstdint>
#include <random>

#define ORACLE_API extern "C" __attribute__((visibility("default")))

enum CaseMatrixType {
    CASE_RANDOM_NONSINGULAR = 0, /* U(0,1) entries, n added to the diagonal */
    CASE_IDENTITY = 1,
    CASE_DIAGONALLY_DOMINANT = 2, /* U(0,1) entries, diagonal set to n */
    CASE_ILL_CONDITIONED = 3,     /* Hilbert matrix 1/(i+j+1) */
    CASE_DIAGONAL = 4,            /* diagonal U(0.1,10) */
    CASE_UPPER_TRIANGULAR = 5,    /* off-diagonal U(0,1), diagonal U(0.5,2) */
    CASE_LOWER_TRIANGULAR = 6,
    CASE_SINGULAR_ZERO_COL = 7,   /* random nonsingular, column 0 zeroed */
    CASE_SINGULAR_DEPENDENT_ROW = 8, /* random nonsingular, row min(n-1,2) = 2 * row 0 */
    CASE_MIXED = 9                /* random nonsingular, column 0 zeroed on odd batch indices */
};

static void random_nonsingular(float* m, int n, int lda, std::mt19937& rng, std::uniform_real_distribution<float>& u01)
{
    for (int j = 0; j < n; j++) {
        for (int i = 0; i < n; i++) m[(int64_t)j * lda + i] = u01(rng);
        m[(int64_t)j * lda + j] += static_cast<float>(n);
    }
}

/* Fills one lda x n column-major matrix (storage must be zeroed by the caller). */
ORACLE_API void case_matrix(float* m, int n, int lda, int type, uint32_t seed, int batch_idx)
{
    if (n <= 0) return;
    std::mt19937 rng(seed + static_cast<uint32_t>(batch_idx) * 1000u);
    std::uniform_real_distribution<float> u01(0.0f, 1.0f);
    switch (type) {
        case CASE_IDENTITY:
            for (int j = 0; j < n; j++) m[(int64_t)j * lda + j] = 1.0f;
            break;
        case CASE_DIAGONALLY_DOMINANT:
            for (int j = 0; j < n; j++) {
                for (int i = 0; i < n; i++) m[(int64_t)j * lda + i] = u01(rng);
                m[(int64_t)j * lda + j] = static_cast<float>(n);
            }
            break;
        case CASE_ILL_CONDITIONED:
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n; i++) m[(int64_t)j * lda + i] = 1.0f / static_cast<float>(i + j + 1);
            break;
        case CASE_DIAGONAL: {
            std::uniform_real_distribution<float> d(0.1f, 10.0f);
            for (int j = 0; j < n; j++) m[(int64_t)j * lda + j] = d(rng);
            break;
        }
        case CASE_UPPER_TRIANGULAR:
        case CASE_LOWER_TRIANGULAR: {
            const bool upper = (type == CASE_UPPER_TRIANGULAR);
            std::uniform_real_distribution<float> d(0.5f, 2.0f);
            std::uniform_real_distribution<float> off(0.0f, 1.0f);
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n; i++) {
                    const bool is_off = upper ? (i < j) : (i > j);
                    if (is_off)
                        m[(int64_t)j * lda + i] = off(rng);
                    else if (i == j)
                        m[(int64_t)j * lda + i] = d(rng);
                }
            break;
        }
        case CASE_SINGULAR_ZERO_COL:
            random_nonsingular(m, n, lda, rng, u01);
            for (int i = 0; i < n; i++) m[i] = 0.0f;
            break;
        case CASE_SINGULAR_DEPENDENT_ROW: {
            random_nonsingular(m, n, lda, rng, u01);
            const int dep = std::min(n - 1, 2);
            if (dep > 0)
                for (int j = 0; j < n; j++) m[(int64_t)j * lda + dep] = 2.0f * m[(int64_t)j * lda];
            break;
        }
        case CASE_MIXED:
            random_nonsingular(m, n, lda, rng, u01);
            if (batch_idx % 2 == 1)
                for (int i = 0; i < n; i++) m[i] = 0.0f;
            break;
        case CASE_RANDOM_NONSINGULAR:
        default:
            random_nonsingular(m, n, lda, rng, u01);
            break;
    }
}

/* A batch of matrices with stride lda*n (the reference's per-matrix vectors laid end to end). */
ORACLE_API void case_matrix_batch(float* m, int n, int lda, int type, uint32_t seed, int batch)
{
    for (int b = 0; b < batch; b++) case_matrix(m + (int64_t)b * lda * n, n, lda, type, seed, b);
}

/* Right-hand sides of the getrs suite: ldb x nrhs per matrix, U(-1,1) in column order. */
ORACLE_API void case_rhs_batch(float* B, int n, int nrhs, int ldb, uint32_t seed, int batch)
{
    for (int b = 0; b < batch; b++) {
        float* m = B + (int64_t)b * ldb * nrhs;
        std::mt19937 rng(seed + static_cast<uint32_t>(b) * 1000u + 500u);
        std::uniform_real_distribution<float> u(-1.0f, 1.0f);
        for (int j = 0; j < nrhs; j++)
            for (int i = 0; i < n; i++) m[(int64_t)j * ldb + i] = u(rng);
    }
}
