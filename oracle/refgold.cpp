/*
 * The reference's own CPU golden path, built in place -- TEST INFRASTRUCTURE ONLY.
 *
 * This translation unit includes, unmodified and by include path from the reference tree,
 *   test/getrf_batched/sgetrf_batched/sgetrf_batched_golden.h  (aclblasSgetrfBatched_cpu)
 *   test/getrs_batched/sgetrs_batched_golden.h                 (aclblasSgetrsBatched_cpu)
 *   test/getri_batched/sgetri_batched/sgetri_batched_golden.h  (aclblasSgetriBatched_cpu)
 * and exports flat C entry points over strided host batches. Those headers call system
 * LAPACK (sgetrf_/sgetrs_/sgetri_); here the symbols are forwarded to the OpenBLAS (config string "0.3.31.dev")
 * that ships inside scipy 1.18.1 (scipy_sgetrf_ etc.), loaded with dlopen at first use.
 * OpenBLAS runs single-threaded; batch parallelism is OpenMP over contiguous chunks, each
 * chunk one call of the golden function on its sub-batch, as the reference's golden loops
 * are serial over the batch (sgetrf_batched_golden.h:73-89).
 *
 * Built by oracle/build_oracle.py into oracle/_ref/librefgold.so; never part of the library.
 */
#include <dlfcn.h>
#include <omp.h>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "sgetrf_batched_golden.h"
#include "sgetrs_batched_golden.h"
#include "sgetri_batched_golden.h"
#include "sgeqrf_batched_golden.h"
#include "sgels_batched_golden.h"

namespace {

using getrf_fn = void (*)(const int*, const int*, float*, const int*, int*, int*);
using getrs_fn = void (*)(const char*, const int*, const int*, const float*, const int*, const int*, float*,
                          const int*, int*);
using getri_fn = void (*)(const int*, float*, const int*, int*, float*, const int*, int*);
using geqrf_fn = void (*)(const int*, const int*, float*, const int*, float*, float*, const int*, int*);
using gels_fn = void (*)(const char*, const int*, const int*, const int*, float*, const int*, float*, const int*,
                        float*, const int*, int*);
using nthreads_fn = void (*)(int);
using config_fn = char* (*)();

struct Lapack {
    getrf_fn getrf = nullptr;
    getrs_fn getrs = nullptr;
    getri_fn getri = nullptr;
    geqrf_fn geqrf = nullptr;
    gels_fn gels = nullptr;
    config_fn config = nullptr;
    bool ok = false;
};

Lapack& lapack()
{
    static Lapack L = [] {
        Lapack l;
        const char* path = std::getenv("OPSBLAS_ORACLE_OPENBLAS");
        if (!path) path = OPENBLAS_DEFAULT_PATH;
        void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
        if (!h) {
            std::fprintf(stderr, "refgold: cannot dlopen %s: %s\n", path, dlerror());
            return l;
        }
        l.getrf = reinterpret_cast<getrf_fn>(dlsym(h, "scipy_sgetrf_"));
        l.getrs = reinterpret_cast<getrs_fn>(dlsym(h, "scipy_sgetrs_"));
        l.getri = reinterpret_cast<getri_fn>(dlsym(h, "scipy_sgetri_"));
        l.geqrf = reinterpret_cast<geqrf_fn>(dlsym(h, "scipy_sgeqrf_"));
        l.gels = reinterpret_cast<gels_fn>(dlsym(h, "scipy_sgels_"));
        l.config = reinterpret_cast<config_fn>(dlsym(h, "scipy_openblas_get_config"));
        auto setn = reinterpret_cast<nthreads_fn>(dlsym(h, "scipy_openblas_set_num_threads"));
        if (setn) setn(1);
        l.ok = l.getrf && l.getrs && l.getri && l.geqrf && l.gels;
        return l;
    }();
    return L;
}

int g_dummy_handle_storage = 0;
aclblasHandle_t dummy_handle() { return reinterpret_cast<aclblasHandle_t>(&g_dummy_handle_storage); }

template <typename F>
void for_chunks(int batch, int nthreads, F&& f)
{
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    if (nthreads > batch) nthreads = batch > 0 ? batch : 1;
    const int per = (batch + nthreads - 1) / nthreads;
#pragma omp parallel for num_threads(nthreads) schedule(static, 1)
    for (int t = 0; t < nthreads; t++) {
        int b0 = t * per;
        int cnt = batch - b0 < per ? batch - b0 : per;
        if (cnt > 0) f(b0, cnt);
    }
}

} // namespace

/* LAPACK symbols the golden headers declare, forwarded to scipy's OpenBLAS. */
extern "C" {
void sgetrf_(const int* m, const int* n, float* a, const int* lda, int* ipiv, int* info)
{
    lapack().getrf(m, n, a, lda, ipiv, info);
}
void sgetrs_(const char* trans, const int* n, const int* nrhs, const float* a, const int* lda, const int* ipiv,
             float* b, const int* ldb, int* info)
{
    lapack().getrs(trans, n, nrhs, a, lda, ipiv, b, ldb, info);
}
void sgetri_(const int* n, float* a, const int* lda, int* ipiv, float* work, const int* lwork, int* info)
{
    lapack().getri(n, a, lda, ipiv, work, lwork, info);
}
void sgeqrf_(const int* m, const int* n, float* a, const int* lda, float* tau, float* work, const int* lwork,
             int* info)
{
    lapack().geqrf(m, n, a, lda, tau, work, lwork, info);
}
void sgels_(const char* trans, const int* m, const int* n, const int* nrhs, float* a, const int* lda, float* b,
            const int* ldb, float* work, const int* lwork, int* info)
{
    lapack().gels(trans, m, n, nrhs, a, lda, b, ldb, work, lwork, info);
}
}

#define REF_API extern "C" __attribute__((visibility("default")))

REF_API int ref_available() { return lapack().ok ? 1 : 0; }

REF_API const char* ref_openblas_config() { return lapack().config ? lapack().config() : "unknown"; }

REF_API int ref_max_threads() { return omp_get_max_threads(); }

/* aclblasSgetrfBatched_cpu over a strided batch. piv may be NULL (no-pivot golden). */
REF_API int ref_sgetrf_batched(int n, float* A, long long strideA, int lda, int* piv, int* info, int batch,
                               int nthreads)
{
    if (!lapack().ok) return -1;
    int status = 0;
    for_chunks(batch, nthreads, [&](int b0, int cnt) {
        std::vector<float*> ptrs(cnt);
        for (int i = 0; i < cnt; i++) ptrs[i] = A + (long long)(b0 + i) * strideA;
        aclblasStatus_t st = aclblasSgetrfBatched_cpu(dummy_handle(), n, ptrs.data(), lda,
                                                      piv ? piv + (long long)b0 * n : nullptr, info + b0, cnt);
        if (st != ACLBLAS_STATUS_SUCCESS) status = static_cast<int>(st);
    });
    return status;
}

/* LAPACK sgetrf (or the golden no-pivot loop) without the golden's pivot zeroing: the
 * factorisation the reference's getrs/getri tests feed to the solve (sgetrs_batched_golden.h:164-180). */
REF_API int ref_sgetrf_for_solve(int n, float* A, long long strideA, int lda, int* piv, int* info, int batch,
                                 int nthreads)
{
    if (!lapack().ok) return -1;
    for_chunks(batch, nthreads, [&](int b0, int cnt) {
        std::vector<float*> ptrs(cnt);
        for (int i = 0; i < cnt; i++) ptrs[i] = A + (long long)(b0 + i) * strideA;
        aclblasSgetrfBatched_cpu_for_getrs(n, ptrs.data(), lda, piv ? piv + (long long)b0 * n : nullptr, info + b0,
                                           cnt, piv != nullptr);
    });
    return 0;
}

/* aclblasSgetrsBatched_cpu over a strided batch. trans: 111/112/113. */
REF_API int ref_sgetrs_batched(int trans, int n, int nrhs, const float* LU, long long strideA, int lda,
                               const int* piv, float* B, long long strideB, int ldb, int batch, int nthreads)
{
    if (!lapack().ok) return -1;
    int status = 0;
    for_chunks(batch, nthreads, [&](int b0, int cnt) {
        std::vector<const float*> ap(cnt);
        std::vector<float*> bp(cnt);
        for (int i = 0; i < cnt; i++) {
            ap[i] = LU + (long long)(b0 + i) * strideA;
            bp[i] = B + (long long)(b0 + i) * strideB;
        }
        int info = 0;
        aclblasStatus_t st = aclblasSgetrsBatched_cpu(dummy_handle(), static_cast<aclblasOperation_t>(trans), n,
                                                      nrhs, ap.data(), lda, piv ? piv + (long long)b0 * n : nullptr,
                                                      bp.data(), ldb, &info, cnt);
        if (st != ACLBLAS_STATUS_SUCCESS) status = static_cast<int>(st);
    });
    return status;
}

/* aclblasSgetriBatched_cpu over a strided batch. */
REF_API int ref_sgetri_batched(int n, const float* LU, long long strideA, int lda, const int* piv, float* C,
                               long long strideC, int ldc, int* info, int batch, int nthreads)
{
    if (!lapack().ok) return -1;
    int status = 0;
    for_chunks(batch, nthreads, [&](int b0, int cnt) {
        std::vector<const float*> ap(cnt);
        std::vector<float*> cp(cnt);
        for (int i = 0; i < cnt; i++) {
            ap[i] = LU + (long long)(b0 + i) * strideA;
            cp[i] = C + (long long)(b0 + i) * strideC;
        }
        aclblasStatus_t st = aclblasSgetriBatched_cpu(dummy_handle(), n, ap.data(), lda,
                                                      piv ? piv + (long long)b0 * n : nullptr, cp.data(), ldc,
                                                      info + b0, cnt);
        if (st != ACLBLAS_STATUS_SUCCESS) status = static_cast<int>(st);
    });
    return status;
}

/* aclblasSgeqrfBatched_cpu over a strided batch; returns its status, *info its LAPACK-style info. */
REF_API int ref_sgeqrf_batched(int m, int n, float* A, long long strideA, int lda, float* tau, long long strideTau,
                               int* info, int batch, int nthreads)
{
    if (!lapack().ok) return -1;
    int status = 0;
    *info = 0;
    for_chunks(batch, nthreads, [&](int b0, int cnt) {
        std::vector<float*> ap(cnt), tp(cnt);
        for (int i = 0; i < cnt; i++) {
            ap[i] = A + (long long)(b0 + i) * strideA;
            tp[i] = tau + (long long)(b0 + i) * strideTau;
        }
        int inf = 0;
        aclblasStatus_t st = aclblasSgeqrfBatched_cpu(dummy_handle(), m, n, ap.data(), lda, tp.data(), &inf, cnt);
        if (st != ACLBLAS_STATUS_SUCCESS) status = static_cast<int>(st);
    });
    return status;
}

/* aclblasSgelsBatched_cpu one matrix at a time (its info is one value per call), over a strided
 * batch; info receives each matrix's LAPACK info. */
REF_API int ref_sgels_batched(int trans, int m, int n, int nrhs, float* A, long long strideA, int lda, float* C,
                              long long strideC, int ldc, int* info, int batch, int nthreads)
{
    if (!lapack().ok) return -1;
    int status = 0;
    for_chunks(batch, nthreads, [&](int b0, int cnt) {
        for (int i = 0; i < cnt; i++) {
            float* a = A + (long long)(b0 + i) * strideA;
            float* c = C + (long long)(b0 + i) * strideC;
            aclblasStatus_t st = aclblasSgelsBatched_cpu(dummy_handle(), static_cast<aclblasOperation_t>(trans), m, n,
                                                         nrhs, &a, lda, &c, ldc, info + b0 + i, 1);
            if (st != ACLBLAS_STATUS_SUCCESS) status = static_cast<int>(st);
        }
    });
    return status;
}
