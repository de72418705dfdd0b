// aclblasGemmBatchedEx: C[i] = alpha * op(A[i]) * op(B[i]) + beta * C[i] over pointer arrays.
//
// Replaces blas/gemm_batched_ex/arch35/gemm_batched_ex_host.cpp:87-581 (host) and the cube
// kernels of gemm_batched_ex_kernel.cpp:386-978. Validation order, status codes and the
// dtype table follow gemm_batched_ex_host.cpp:87-118,156-244: FP16/FP16/FP16 with COMPUTE_16F
// or COMPUTE_32F, BF16/BF16/BF16 and the four FP8 E4M3/E5M2 pairs with FP16 output under
// COMPUTE_32F. Added for the LU trailing update: FP32/FP32/FP32 with COMPUTE_32F_PEDANTIC (plain
// FP32 FMA), COMPUTE_32F_FAST_TF32 and COMPUTE_32F_FAST_16BF (operands rounded to TF32 / BF16,
// FP32 accumulation); FP32 under COMPUTE_32F stays NOT_SUPPORTED as in the reference. alpha and beta are host floats, as in the reference
// (gemm_batched_ex_host.cpp:79-85). Unlike the reference (which runs a second alpha/beta
// kernel on a workspace copy of C filled through a host-to-device memcpy, :493-523), alpha
// and beta are applied in the epilogue of the one kernel: no workspace, no copy, capturable.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include "internal.h"

namespace opsblas {

template <GemmElem T>
__device__ __forceinline__ float load_elem(const void* p, long long idx)
{
    if constexpr (T == GemmElem::F32) return static_cast<const float*>(p)[idx];
    if constexpr (T == GemmElem::F16) return __half2float(static_cast<const __half*>(p)[idx]);
    if constexpr (T == GemmElem::BF16) return __bfloat162float(static_cast<const __nv_bfloat16*>(p)[idx]);
    if constexpr (T == GemmElem::E4M3) return float(static_cast<const __nv_fp8_e4m3*>(p)[idx]);
    if constexpr (T == GemmElem::E5M2) return float(static_cast<const __nv_fp8_e5m2*>(p)[idx]);
    return 0.0f;
}

template <GemmElem T>
__device__ __forceinline__ void store_elem(void* p, long long idx, float v)
{
    if constexpr (T == GemmElem::F32) static_cast<float*>(p)[idx] = v;
    if constexpr (T == GemmElem::F16) static_cast<__half*>(p)[idx] = __float2half_rn(v);
    if constexpr (T == GemmElem::BF16) static_cast<__nv_bfloat16*>(p)[idx] = __float2bfloat16_rn(v);
}

// Operand rounding of the FAST compute types: TF32 keeps 10 mantissa bits, BF16 keeps 7
// (round to nearest even on the dropped bits; non-finite values pass through).
enum class OperandRound { None, TF32, BF16 };

template <OperandRound R>
__device__ __forceinline__ float round_operand(float x)
{
    if constexpr (R == OperandRound::TF32) {
        unsigned u = __float_as_uint(x);
        if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x0fffu + ((u >> 13) & 1u)) & 0xffffe000u;
        return __uint_as_float(u);
    } else if constexpr (R == OperandRound::BF16) {
        return __bfloat162float(__float2bfloat16_rn(x));
    }
    return x;
}

constexpr int kGemmBM = 64, kGemmBN = 64, kGemmBK = 16, kGemmThreads = 256;

// 64x64 output tile per CTA, 4x4 per thread, K staged through shared memory in slices of 16.
template <GemmElem TA, GemmElem TB, GemmElem TC, OperandRound R>
__global__ void __launch_bounds__(kGemmThreads)
gemm_batched_simt_kernel(bool transA, bool transB, int m, int n, int k, float alpha, const void* const* Aarray,
                         int lda, const void* const* Barray, int ldb, float beta, void* const* Carray, int ldc)
{
    __shared__ __align__(16) float As[kGemmBK][kGemmBM + 4];
    __shared__ __align__(16) float Bs[kGemmBK][kGemmBN + 4];
    // grid.x enumerates (row tile, matrix) pairs so that the batch is not limited by grid.y/z
    const int tiles_m = (m + kGemmBM - 1) / kGemmBM;
    const long long b = blockIdx.x / tiles_m;
    const void* A = Aarray[b];
    const void* B = Barray[b];
    void* C = Carray[b];
    const int m0 = (int)(blockIdx.x % tiles_m) * kGemmBM, n0 = blockIdx.y * kGemmBN;
    const int tid = threadIdx.x;
    const int tx = tid % 16, ty = tid / 16;  // thread computes rows m0+tx*4.., cols n0+ty*4..
    float acc[4][4] = {};

    for (int k0 = 0; k0 < k; k0 += kGemmBK) {
        // op(A) tile: rows m0..m0+63, cols k0..k0+15 ; op(B) tile: rows k0.., cols n0.. -- the
        // fast index follows each operand's contiguous dimension (coalesced loads)
        for (int e = tid; e < kGemmBM * kGemmBK; e += kGemmThreads) {
            const int i = transA ? e / kGemmBK : e % kGemmBM, kk = transA ? e % kGemmBK : e / kGemmBM;
            const int gi = m0 + i, gk = k0 + kk;
            float v = 0.0f;
            if (gi < m && gk < k) v = load_elem<TA>(A, transA ? (gk + (long long)gi * lda) : (gi + (long long)gk * lda));
            As[kk][i] = round_operand<R>(v);
        }
        for (int e = tid; e < kGemmBN * kGemmBK; e += kGemmThreads) {
            const int kk = transB ? e / kGemmBN : e % kGemmBK, j = transB ? e % kGemmBN : e / kGemmBK;
            const int gj = n0 + j, gk = k0 + kk;
            float v = 0.0f;
            if (gj < n && gk < k) v = load_elem<TB>(B, transB ? (gj + (long long)gk * ldb) : (gk + (long long)gj * ldb));
            Bs[kk][j] = round_operand<R>(v);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kGemmBK; kk++) {
            const float4 a = *reinterpret_cast<const float4*>(&As[kk][tx * 4]);
            const float4 bv = *reinterpret_cast<const float4*>(&Bs[kk][ty * 4]);
            const float av[4] = {a.x, a.y, a.z, a.w};
            const float bw[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(av[i], bw[j], acc[i][j]);
        }
        __syncthreads();
    }
    // The tile goes through shared memory so that C is read and written column by column (each
    // warp a contiguous run of rows); the per-element epilogue is unchanged.
    __shared__ float Cs[kGemmBN][kGemmBM + 1];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) Cs[ty * 4 + j][tx * 4 + i] = acc[i][j];
    __syncthreads();
    for (int e = tid; e < kGemmBM * kGemmBN; e += kGemmThreads) {
        const int i = e % kGemmBM, j = e / kGemmBM;
        const int gi = m0 + i, gj = n0 + j;
        if (gi < m && gj < n) {
            const long long idx = gi + (long long)gj * ldc;
            float v = alpha * Cs[j][i];
            if (beta != 0.0f) v = fmaf(beta, load_elem<TC>(C, idx), v);
            store_elem<TC>(C, idx, v);
        }
    }
}

// k == 0 or alpha == 0: C = beta * C. GemmBatchedEx writes zeros for beta == 0, as its
// reference early-exit kernel (gemm_batched_ex_host.cpp:462-491); SgemmBatched multiplies
// unconditionally, as its reference (gemm_batched_host.cpp:350-390, GemmBatchedEarlyExitOp in
// gemm_batched_kernel.cpp:682-760: Muls by beta), so 0 * Inf or NaN stays NaN there.
template <GemmElem TC, bool ZERO_ON_BETA0 = true>
__global__ void gemm_batched_scale_kernel(int m, int n, float beta, void* const* Carray, int ldc)
{
    void* C = Carray[blockIdx.x];  // one CTA per matrix
    for (long long e = threadIdx.x; e < (long long)m * n; e += blockDim.x) {
        const long long i = e % m, j = e / m;
        const long long idx = i + j * ldc;
        store_elem<TC>(C, idx, (ZERO_ON_BETA0 && beta == 0.0f) ? 0.0f : beta * load_elem<TC>(C, idx));
    }
}

}  // namespace opsblas

using namespace opsblas;

namespace {

enum class Combo { Invalid, F16_F16_F16, BF16_BF16_BF16, E4M3_E4M3_F16, E5M2_E5M2_F16, E4M3_E5M2_F16,
                   E5M2_E4M3_F16, F32_F32_F32 };

Combo combo_of(aclDataType a, aclDataType b, aclDataType c, aclblasComputeType_t ct)
{
    const bool c32 = ct == ACLBLAS_COMPUTE_32F;
    if (a == ACL_FLOAT16 && b == ACL_FLOAT16 && c == ACL_FLOAT16 && (ct == ACLBLAS_COMPUTE_16F || c32))
        return Combo::F16_F16_F16;
    if (!c32 && a != ACL_FLOAT) return Combo::Invalid;
    if (a == ACL_BF16 && b == ACL_BF16 && c == ACL_BF16) return Combo::BF16_BF16_BF16;
    if (c == ACL_FLOAT16 && a == ACL_FLOAT8_E4M3FN && b == ACL_FLOAT8_E4M3FN) return Combo::E4M3_E4M3_F16;
    if (c == ACL_FLOAT16 && a == ACL_FLOAT8_E5M2 && b == ACL_FLOAT8_E5M2) return Combo::E5M2_E5M2_F16;
    if (c == ACL_FLOAT16 && a == ACL_FLOAT8_E4M3FN && b == ACL_FLOAT8_E5M2) return Combo::E4M3_E5M2_F16;
    if (c == ACL_FLOAT16 && a == ACL_FLOAT8_E5M2 && b == ACL_FLOAT8_E4M3FN) return Combo::E5M2_E4M3_F16;
    // FP32 operands: the reference rejects them under COMPUTE_32F (its test row L0_36 expects
    // NOT_SUPPORTED), so plain FP32 is requested with COMPUTE_32F_PEDANTIC instead.
    if (a == ACL_FLOAT && b == ACL_FLOAT && c == ACL_FLOAT &&
        (ct == ACLBLAS_COMPUTE_32F_PEDANTIC || ct == ACLBLAS_COMPUTE_32F_FAST_TF32 ||
         ct == ACLBLAS_COMPUTE_32F_FAST_16BF))
        return Combo::F32_F32_F32;
    return Combo::Invalid;
}

bool valid_op(aclblasOperation_t t) { return t == ACLBLAS_OP_N || t == ACLBLAS_OP_T || t == ACLBLAS_OP_C; }

template <GemmElem TA, GemmElem TB, GemmElem TC, OperandRound R>
cudaError_t run_gemm(cudaStream_t st, bool ta, bool tb, int m, int n, int k, float alpha, const void* const* A,
                     int lda, const void* const* B, int ldb, float beta, void* const* C, int ldc, int batch)
{
    dim3 grid((unsigned)((long long)((m + kGemmBM - 1) / kGemmBM) * batch), (unsigned)((n + kGemmBN - 1) / kGemmBN));
    gemm_batched_simt_kernel<TA, TB, TC, R><<<grid, kGemmThreads, 0, st>>>(ta, tb, m, n, k, alpha, A, lda, B, ldb,
                                                                          beta, C, ldc);
    return cudaGetLastError();
}

}  // namespace

namespace opsblas {

cudaError_t gemm_f32_launch(cudaStream_t st, bool transA, bool transB, int m, int n, int k, float alpha,
                            const float* const* A, int lda, const float* const* B, int ldb, float beta,
                            float* const* C, int ldc, int batch, int round)
{
    using E = GemmElem;
    auto a = reinterpret_cast<const void* const*>(A);
    auto b = reinterpret_cast<const void* const*>(B);
    auto c = reinterpret_cast<void* const*>(C);
    if (round == 1)
        return run_gemm<E::F32, E::F32, E::F32, OperandRound::TF32>(st, transA, transB, m, n, k, alpha, a, lda, b,
                                                                     ldb, beta, c, ldc, batch);
    if (round == 2)
        return run_gemm<E::F32, E::F32, E::F32, OperandRound::BF16>(st, transA, transB, m, n, k, alpha, a, lda, b,
                                                                     ldb, beta, c, ldc, batch);
    return run_gemm<E::F32, E::F32, E::F32, OperandRound::None>(st, transA, transB, m, n, k, alpha, a, lda, b, ldb,
                                                                 beta, c, ldc, batch);
}

}  // namespace opsblas

extern "C" aclblasStatus_t aclblasGemmBatchedEx(
    aclblasHandle_t handle, aclblasOperation_t transa, aclblasOperation_t transb, int m, int n, int k,
    const void* alpha, const void* const Aarray[], aclDataType Atype, int lda, const void* const Barray[],
    aclDataType Btype, int ldb, const void* beta, void* const Carray[], aclDataType Ctype, int ldc, int batchCount,
    aclblasComputeType_t computeType, aclblasGemmAlgo_t algo)
{
    static const char* kApi = "aclblasGemmBatchedEx";
    if (handle == nullptr) {
        log_error(kApi, "handle is nullptr");
        return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    }
    if (alpha == nullptr || beta == nullptr) {
        log_error(kApi, "alpha and beta must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (m < 0 || n < 0 || k < 0 || !valid_op(transa) || !valid_op(transb) || batchCount < 0) {
        log_error(kApi, "invalid dimensions or operation (m=%d n=%d k=%d batch=%d)", m, n, k, batchCount);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    const bool ta = transa != ACLBLAS_OP_N, tb = transb != ACLBLAS_OP_N;
    if (lda < max1(ta ? k : m) || ldb < max1(tb ? n : k) || ldc < max1(m)) {
        log_error(kApi, "invalid leading dimension (lda=%d ldb=%d ldc=%d)", lda, ldb, ldc);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (algo != ACLBLAS_GEMM_DEFAULT) {
        log_error(kApi, "unsupported algo=%d", (int)algo);
        return ACLBLAS_STATUS_NOT_SUPPORTED;
    }
    const Combo cb = combo_of(Atype, Btype, Ctype, computeType);
    if (cb == Combo::Invalid) {
        log_error(kApi, "invalid dtype combination: Atype=%d, Btype=%d, Ctype=%d, computeType=%d", (int)Atype,
                  (int)Btype, (int)Ctype, (int)computeType);
        return ACLBLAS_STATUS_NOT_SUPPORTED;
    }
    if (batchCount > 0 && (Aarray == nullptr || Barray == nullptr || Carray == nullptr)) {
        log_error(kApi, "Aarray, Barray and Carray must not be nullptr when batchCount > 0");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    const float a = *static_cast<const float*>(alpha);
    const float b = *static_cast<const float*>(beta);
    if (m == 0 || n == 0 || batchCount == 0) return ACLBLAS_STATUS_SUCCESS;

    cudaStream_t st = handle->stream;
    if (k == 0 || a == 0.0f) {
        if (b == 1.0f) return ACLBLAS_STATUS_SUCCESS;
        const unsigned grid = (unsigned)batchCount;
        if (Ctype == ACL_FLOAT)
            gemm_batched_scale_kernel<GemmElem::F32><<<grid, 256, 0, st>>>(m, n, b, Carray, ldc);
        else if (Ctype == ACL_BF16)
            gemm_batched_scale_kernel<GemmElem::BF16><<<grid, 256, 0, st>>>(m, n, b, Carray, ldc);
        else
            gemm_batched_scale_kernel<GemmElem::F16><<<grid, 256, 0, st>>>(m, n, b, Carray, ldc);
        return launch_status(kApi, cudaGetLastError());
    }

    // Every dtype of the reference's table runs on the tcgen05 tensor cores with FP32 accumulation
    // (its cube unit's arithmetic); FP32 operands with COMPUTE_32F_PEDANTIC stay on the FP32
    // CUDA-core kernel (plain FP32 products).
    cudaError_t err = cudaSuccess;
    using E = GemmElem;
    auto tc = [&](TcIn ka, TcIn kb, E kc) {
        return gemm_tc_typed_launch(st, ka, kb, kc, false, ta, tb, m, n, k, a, Aarray, 0, lda, Barray, 0, ldb, b,
                                    Carray, 0, ldc, batchCount, handle->dstatus, handle->tmslots);
    };
    switch (cb) {
        case Combo::F16_F16_F16: err = tc(TcIn::F16, TcIn::F16, E::F16); break;
        case Combo::BF16_BF16_BF16: err = tc(TcIn::BF16, TcIn::BF16, E::BF16); break;
        case Combo::E4M3_E4M3_F16: err = tc(TcIn::E4M3, TcIn::E4M3, E::F16); break;
        case Combo::E5M2_E5M2_F16: err = tc(TcIn::E5M2, TcIn::E5M2, E::F16); break;
        case Combo::E4M3_E5M2_F16: err = tc(TcIn::E4M3, TcIn::E5M2, E::F16); break;
        case Combo::E5M2_E4M3_F16: err = tc(TcIn::E5M2, TcIn::E4M3, E::F16); break;
        case Combo::F32_F32_F32:
            if (computeType == ACLBLAS_COMPUTE_32F_FAST_TF32)
                err = tc(TcIn::F32_TF32, TcIn::F32_TF32, E::F32);
            else if (computeType == ACLBLAS_COMPUTE_32F_FAST_16BF)
                err = tc(TcIn::F32_BF16, TcIn::F32_BF16, E::F32);
            else
                err = run_gemm<E::F32, E::F32, E::F32, OperandRound::None>(st, ta, tb, m, n, k, a, Aarray, lda, Barray,
                                                                          ldb, b, Carray, ldc, batchCount);
            break;
        default:
            return ACLBLAS_STATUS_NOT_SUPPORTED;
    }
    return launch_status(kApi, err);
}

// aclblasSgemmBatched (include/cann_ops_blas.h:415; gemm_batched_host.cpp:397-435): FP32 batched
// GEMM with plain FP32 products (the reference disables HF32), on the same FP32 CUDA-core kernel
// as GemmBatchedEx with COMPUTE_32F operands; alpha and beta are host floats applied in the
// kernel's epilogue. Validation order of ValidateSgemmBatchedParams (:53-98); an operation value
// outside N/T/C is INVALID_VALUE there (not INVALID_ENUM).
extern "C" aclblasStatus_t aclblasSgemmBatched(aclblasHandle_t handle, aclblasOperation_t transa,
                                               aclblasOperation_t transb, int m, int n, int k, const float* alpha,
                                               const float* const Aarray[], int lda, const float* const Barray[],
                                               int ldb, const float* beta, float* const Carray[], int ldc,
                                               int batchCount)
{
    using namespace opsblas;
    static const char* kApi = "aclblasSgemmBatched";
    if (handle == nullptr) {
        log_error(kApi, "handle is nullptr");
        return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    }
    if (alpha == nullptr || beta == nullptr) {
        log_error(kApi, "alpha and beta must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (m < 0 || n < 0 || k < 0 || batchCount < 0) {
        log_error(kApi, "invalid dimensions (m=%d n=%d k=%d batch=%d)", m, n, k, batchCount);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (!valid_op(transa) || !valid_op(transb)) {
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
    const float a = *alpha, b = *beta;
    cudaStream_t st = handle->stream;
    if (k == 0 || a == 0.0f) {
        if (b == 1.0f) return ACLBLAS_STATUS_SUCCESS;
        gemm_batched_scale_kernel<GemmElem::F32, false><<<(unsigned)batchCount, 256, 0, st>>>(
            m, n, b, reinterpret_cast<void* const*>(Carray), ldc);
        return launch_status(kApi, cudaGetLastError());
    }
    return launch_status(kApi, gemm_f32_launch(st, ta, tb, m, n, k, a, Aarray, lda, Barray, ldb, b, Carray, ldc,
                                               batchCount, 0));
}
