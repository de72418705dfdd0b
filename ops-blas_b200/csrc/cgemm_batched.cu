// aclblasCgemmBatched: single-precision complex batched GEMM on the FP32 CUDA cores.
//
// The reference (blas/gemm_batched/arch35/gemm_batched_host.cpp:438-819) splits A and B into
// real and imaginary planes in workspace, runs four real FP32 GEMMs T1 = Ar Br, T2 = Ai Bi,
// T3 = Ar Bi, T4 = Ai Br into four temporary matrices, and combines them in a fifth pass
// (gemm_batched_kernel.cpp:1029-1110): Pr = T1 - T2, Pi = T3 + T4, Cr = Pr aR - Pi aI,
// Ci = Pi aR + Pr aI, then, when beta != 0, Cr += Cor bR, Ci += Coi bR, Cr -= Coi bI,
// Ci += Cor bI -- every product and sum rounded on its own. Here one kernel does all of it: each
// CTA owns a 64 x 64 complex tile and walks k in slices of 8, staging op(A) and op(B) slices in
// shared memory as separate real and imaginary planes (the de-interleave, conjugation for op C
// included, happens on the load; the next slice is fetched into registers during the multiply and
// stored into the second of two stages), keeps the four sums of its 4 x 4 complex outputs per
// thread in registers (one fmaf per product, k in order), and applies the combine in the
// reference's operation order in the epilogue. No workspace, one launch, C read once (only when
// beta != 0) and written once.
#include <climits>
#include <cuda_runtime.h>

#include "internal.h"

namespace opsblas {

constexpr int kCgBM = 64, kCgBN = 64, kCgBK = 8, kCgThreads = 256;

// Element (r, c) of op(X) for op code OP (0 = N, 1 = T, 2 = C): X(r, c), X(c, r), conj(X(c, r)).
template <int OP>
__device__ __forceinline__ float2 cg_load_op(const float2* X, int ld, int r, int c)
{
    float2 v = OP == 0 ? X[r + (long long)c * ld] : X[c + (long long)r * ld];
    if (OP == 2) v.y = -v.y;
    return v;
}

struct CgAcc {
    float t1[4][4], t2[4][4], t3[4][4], t4[4][4];
};

// One k step of the 4 x 4 complex outputs of thread (tx, ty).
__device__ __forceinline__ void cg_step(const float (*Ar)[kCgBM + 4], const float (*Ai)[kCgBM + 4],
                                        const float (*Br)[kCgBN + 4], const float (*Bi)[kCgBN + 4], int kk, int tx,
                                        int ty, CgAcc& s)
{
    const float4 ar4 = *reinterpret_cast<const float4*>(&Ar[kk][tx * 4]);
    const float4 ai4 = *reinterpret_cast<const float4*>(&Ai[kk][tx * 4]);
    const float4 br4 = *reinterpret_cast<const float4*>(&Br[kk][ty * 4]);
    const float4 bi4 = *reinterpret_cast<const float4*>(&Bi[kk][ty * 4]);
    const float ar[4] = {ar4.x, ar4.y, ar4.z, ar4.w}, ai[4] = {ai4.x, ai4.y, ai4.z, ai4.w};
    const float br[4] = {br4.x, br4.y, br4.z, br4.w}, bi[4] = {bi4.x, bi4.y, bi4.z, bi4.w};
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            s.t1[i][j] = fmaf(ar[i], br[j], s.t1[i][j]);
            s.t2[i][j] = fmaf(ai[i], bi[j], s.t2[i][j]);
            s.t3[i][j] = fmaf(ar[i], bi[j], s.t3[i][j]);
            s.t4[i][j] = fmaf(ai[i], br[j], s.t4[i][j]);
        }
}

constexpr int kCgLoads = kCgBM * kCgBK / kCgThreads;  // elements per thread and operand slice
static_assert(kCgBM * kCgBK == kCgBK * kCgBN, "both operand slices hold the same element count");

// Loads this thread's elements of the operand slices starting at k0 (zero outside the matrix).
// The fast index follows the operand's contiguous dimension (coalesced loads).
template <int OPA, int OPB>
__device__ __forceinline__ void cg_fetch(const float2* A, int lda, const float2* B, int ldb, int m, int n, int k,
                                         int m0, int n0, int k0, int tid, float2 (&pa)[kCgLoads],
                                         float2 (&pb)[kCgLoads])
{
#pragma unroll
    for (int r = 0; r < kCgLoads; r++) {
        const int e = tid + r * kCgThreads;
        const int i = OPA == 0 ? e % kCgBM : e / kCgBK;
        const int kk = OPA == 0 ? e / kCgBM : e % kCgBK;
        const int gi = m0 + i, gk = k0 + kk;
        pa[r] = (gi < m && gk < k) ? cg_load_op<OPA>(A, lda, gi, gk) : make_float2(0.0f, 0.0f);
        const int kb = OPB == 0 ? e % kCgBK : e / kCgBN;
        const int j = OPB == 0 ? e / kCgBK : e % kCgBN;
        const int gj = n0 + j, gkb = k0 + kb;
        pb[r] = (gj < n && gkb < k) ? cg_load_op<OPB>(B, ldb, gkb, gj) : make_float2(0.0f, 0.0f);
    }
}

// Stores this thread's fetched elements into one stage of the shared-memory planes.
template <int OPA, int OPB>
__device__ __forceinline__ void cg_store(float (*Ar)[kCgBM + 4], float (*Ai)[kCgBM + 4], float (*Br)[kCgBN + 4],
                                         float (*Bi)[kCgBN + 4], int tid, const float2 (&pa)[kCgLoads],
                                         const float2 (&pb)[kCgLoads])
{
#pragma unroll
    for (int r = 0; r < kCgLoads; r++) {
        const int e = tid + r * kCgThreads;
        const int i = OPA == 0 ? e % kCgBM : e / kCgBK;
        const int kk = OPA == 0 ? e / kCgBM : e % kCgBK;
        Ar[kk][i] = pa[r].x;
        Ai[kk][i] = pa[r].y;
        const int kb = OPB == 0 ? e % kCgBK : e / kCgBN;
        const int j = OPB == 0 ? e / kCgBK : e % kCgBN;
        Br[kb][j] = pb[r].x;
        Bi[kb][j] = pb[r].y;
    }
}

// grid.x = (row tile, matrix) pairs, grid.y = column tiles. k == 0 computes P = 0 (the
// reference's alpha == 0 / k == 0 path) without reading A or B.
template <int OPA, int OPB>
__global__ void __launch_bounds__(kCgThreads, 2)
cgemm_batched_kernel(int m, int n, int k, float2 alpha, float2 beta, const float2* const* Aarray, int lda,
                     const float2* const* Barray, int ldb, float2* const* Carray, int ldc)
{
    // two stages of the operand slices: the multiply reads one while the next is stored into the other
    __shared__ __align__(16) float Ar[2][kCgBK][kCgBM + 4];
    __shared__ __align__(16) float Ai[2][kCgBK][kCgBM + 4];
    __shared__ __align__(16) float Br[2][kCgBK][kCgBN + 4];
    __shared__ __align__(16) float Bi[2][kCgBK][kCgBN + 4];
    const int tiles_m = (m + kCgBM - 1) / kCgBM;
    const long long b = blockIdx.x / tiles_m;
    float2* C = Carray[b];
    if (C == nullptr) return;  // the whole CTA leaves before its first barrier
    const int m0 = (int)(blockIdx.x % tiles_m) * kCgBM, n0 = blockIdx.y * kCgBN;
    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    CgAcc s;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) s.t1[i][j] = s.t2[i][j] = s.t3[i][j] = s.t4[i][j] = 0.0f;

    if (k > 0) {
        const float2* A = Aarray[b];
        const float2* B = Barray[b];
        // This thread's elements of the next operand slice are fetched into registers while the
        // current one is multiplied from shared memory, then stored into the other stage; one
        // barrier per slice (the barrier that ends slice t also ends every read of the stage that
        // slice t + 1 stores into).
        float2 pa[kCgLoads], pb[kCgLoads];
        cg_fetch<OPA, OPB>(A, lda, B, ldb, m, n, k, m0, n0, 0, tid, pa, pb);
        cg_store<OPA, OPB>(Ar[0], Ai[0], Br[0], Bi[0], tid, pa, pb);
        __syncthreads();
        int cur = 0;
        for (int k0 = 0; k0 < k; k0 += kCgBK) {
            const bool more = k0 + kCgBK < k;
            if (more) cg_fetch<OPA, OPB>(A, lda, B, ldb, m, n, k, m0, n0, k0 + kCgBK, tid, pa, pb);
            const int kn = min(kCgBK, k - k0);
            if (kn == kCgBK) {
#pragma unroll
                for (int kk = 0; kk < kCgBK; kk++) cg_step(Ar[cur], Ai[cur], Br[cur], Bi[cur], kk, tx, ty, s);
            } else {
                // the last slice runs only its kn steps, so every sum holds exactly k products
                for (int kk = 0; kk < kn; kk++) cg_step(Ar[cur], Ai[cur], Br[cur], Bi[cur], kk, tx, ty, s);
            }
            if (more) cg_store<OPA, OPB>(Ar[cur ^ 1], Ai[cur ^ 1], Br[cur ^ 1], Bi[cur ^ 1], tid, pa, pb);
            __syncthreads();
            cur ^= 1;
        }
    }

    const bool has_beta = beta.x != 0.0f || beta.y != 0.0f;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int gi = m0 + tx * 4 + i;
        if (gi >= m) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int gj = n0 + ty * 4 + j;
            if (gj >= n) continue;
            const long long idx = gi + (long long)gj * ldc;
            const float pr = __fsub_rn(s.t1[i][j], s.t2[i][j]);
            const float pi = __fadd_rn(s.t3[i][j], s.t4[i][j]);
            float cr = __fsub_rn(__fmul_rn(pr, alpha.x), __fmul_rn(pi, alpha.y));
            float ci = __fadd_rn(__fmul_rn(pi, alpha.x), __fmul_rn(pr, alpha.y));
            if (has_beta) {
                const float2 c = C[idx];
                cr = __fadd_rn(cr, __fmul_rn(c.x, beta.x));
                ci = __fadd_rn(ci, __fmul_rn(c.y, beta.x));
                cr = __fsub_rn(cr, __fmul_rn(c.y, beta.y));
                ci = __fadd_rn(ci, __fmul_rn(c.x, beta.y));
            }
            C[idx] = make_float2(cr, ci);
        }
    }
}

using CgKernel = void (*)(int, int, int, float2, float2, const float2* const*, int, const float2* const*, int,
                          float2* const*, int);

static CgKernel cg_kernel(int opa, int opb)
{
    static const CgKernel table[3][3] = {
        {cgemm_batched_kernel<0, 0>, cgemm_batched_kernel<0, 1>, cgemm_batched_kernel<0, 2>},
        {cgemm_batched_kernel<1, 0>, cgemm_batched_kernel<1, 1>, cgemm_batched_kernel<1, 2>},
        {cgemm_batched_kernel<2, 0>, cgemm_batched_kernel<2, 1>, cgemm_batched_kernel<2, 2>},
    };
    return table[opa][opb];
}

static int op_code(aclblasOperation_t t) { return t == ACLBLAS_OP_N ? 0 : (t == ACLBLAS_OP_T ? 1 : 2); }

}  // namespace opsblas

using namespace opsblas;

extern "C" aclblasStatus_t aclblasCgemmBatched(aclblasHandle_t handle, aclblasOperation_t transa,
                                               aclblasOperation_t transb, int m, int n, int k,
                                               const aclblasComplex* alpha, const aclblasComplex* const Aarray[],
                                               int lda, const aclblasComplex* const Barray[], int ldb,
                                               const aclblasComplex* beta, aclblasComplex* const Carray[], int ldc,
                                               int batchCount)
{
    static const char* kApi = "aclblasCgemmBatched";
    // ValidateCgemmBatchedParams (gemm_batched_host.cpp:462-508), in its order
    if (handle == nullptr) {
        log_error(kApi, "handle is nullptr");
        return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    }
    if (alpha == nullptr || beta == nullptr) {
        log_error(kApi, "%s must not be nullptr", alpha == nullptr ? "alpha" : "beta");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (m < 0 || n < 0 || k < 0 || batchCount < 0) {
        log_error(kApi, "invalid dimensions (m=%d n=%d k=%d batch=%d)", m, n, k, batchCount);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    const auto op_ok = [](aclblasOperation_t t) {
        return t == ACLBLAS_OP_N || t == ACLBLAS_OP_T || t == ACLBLAS_OP_C;
    };
    if (!op_ok(transa) || !op_ok(transb)) {
        log_error(kApi, "invalid transa=%d or transb=%d", (int)transa, (int)transb);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    const bool ta = transa != ACLBLAS_OP_N, tb = transb != ACLBLAS_OP_N;
    if (lda < max1(ta ? k : m) || ldb < max1(tb ? n : k) || ldc < max1(m)) {
        log_error(kApi, "invalid leading dimension (lda=%d ldb=%d ldc=%d)", lda, ldb, ldc);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (batchCount > 0 && (Aarray == nullptr || Barray == nullptr || Carray == nullptr)) {
        log_error(kApi, "Aarray, Barray and Carray must not be nullptr when batchCount > 0");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (m == 0 || n == 0 || batchCount == 0) return ACLBLAS_STATUS_SUCCESS;

    const aclblasComplex a = *alpha, bt = *beta;
    // k == 0 or alpha == 0: the combine over zero sums (LaunchCgemmEarlyExit), nothing when beta == 1
    const bool zero_product = k == 0 || (a.real == 0.0f && a.imag == 0.0f);
    if (zero_product && bt.real == 1.0f && bt.imag == 0.0f) return ACLBLAS_STATUS_SUCCESS;
    const int keff = zero_product ? 0 : k;

    const int tiles_m = (m + kCgBM - 1) / kCgBM, tiles_n = (n + kCgBN - 1) / kCgBN;
    if (tiles_n > 65535) {
        log_error(kApi, "n=%d exceeds the supported %d columns", n, 65535 * kCgBN);
        return ACLBLAS_STATUS_NOT_SUPPORTED;
    }
    const CgKernel kern = keff == 0 ? cg_kernel(0, 0) : cg_kernel(op_code(transa), op_code(transb));
    const float2 fa = make_float2(a.real, a.imag), fb = make_float2(bt.real, bt.imag);
    auto A = reinterpret_cast<const float2* const*>(Aarray);
    auto B = reinterpret_cast<const float2* const*>(Barray);
    auto Cp = reinterpret_cast<float2* const*>(Carray);
    // grid.x carries (row tile, matrix) pairs: batches beyond its range go in several launches
    const int per_launch = (int)((long long)INT_MAX / tiles_m);
    for (int b0 = 0; b0 < batchCount; b0 += per_launch) {
        const int nb = batchCount - b0 < per_launch ? batchCount - b0 : per_launch;
        dim3 grid((unsigned)((long long)tiles_m * nb), (unsigned)tiles_n);
        kern<<<grid, kCgThreads, 0, handle->stream>>>(m, n, keff, fa, fb, A + b0, lda, B + b0, ldb, Cp + b0, ldc);
        const cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) return launch_status(kApi, err);
    }
    return ACLBLAS_STATUS_SUCCESS;
}
