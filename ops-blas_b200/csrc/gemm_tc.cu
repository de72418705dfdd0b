// Batched FP32 GEMM on the 5th-generation tensor cores (tcgen05, kind::tf32):
//   C[b] = alpha * op(A[b]) * op(B[b]) + beta * C[b]   (column-major, element offsets applied)
// One CTA (4 warps) per 128 x 128 tile of C. Per K slice of 32, the CTA stages op(A) (128 x 32)
// and op(B)^T (128 x 32) in shared memory in the K-major no-swizzle layout (tc_common.cuh),
// split into TF32 high and low parts when split = 1; thread 0 issues the MMAs (4 K-steps x 1 or
// 3 products: hi*hi [+ hi*lo + lo*hi]) into a 128 x 128 FP32 accumulator in TMEM and commits them
// to an mbarrier; after the last slice each warp reads its 32 accumulator rows with tcgen05.ld and
// applies alpha / beta to C with coalesced column accesses.
//
// split = 0 is TF32 arithmetic (ACLBLAS_COMPUTE_32F_FAST_TF32); split = 1 carries about 21 bits of
// each operand (the products of the low parts are dropped), enough for the mixed-precision LU's
// trailing update to stay at FP32 accuracy. The wait on the mbarrier is bounded: on time-out the
// tile is filled with NaN and g_tc_timeouts counts it, and the TMEM is still released.
#include <cuda_runtime.h>

#include "internal.h"
#include "tc_common.cuh"

namespace opsblas {

constexpr int kTcTile = 128;      // M and N of a tile (one MMA: 128 x 128 x 8)
constexpr int kTcK = 32;          // K slice staged per round
constexpr int kTcThreads = 128;
constexpr int kTcSlice = kTcTile * kTcK;  // floats of one staged operand part
constexpr uint32_t kTcWaitLimit = 1u << 24;

__device__ unsigned int g_tc_timeouts;

struct TcSmem {
    float a_hi[kTcSlice];
    float a_lo[kTcSlice];
    float b_hi[kTcSlice];
    float b_lo[kTcSlice];
    uint64_t mbar;
    uint32_t taddr;
};

__device__ __forceinline__ int tc_off(int r, int k)
{
    return (r >> 3) * (kTcK * 8) + (k >> 2) * 32 + (r & 7) * 4 + (k & 3);
}

__global__ void __launch_bounds__(kTcThreads)
gemm_tc_kernel(int M, int N, int K, float alpha, const float* const* __restrict__ Aarr, long long a_off, int lda,
               int tA, const float* const* __restrict__ Barr, long long b_off, int ldb, int tB, float beta,
               float* const* __restrict__ Carr, long long c_off, int ldc, int tiles_m, int tiles_n, int split)
{
    extern __shared__ __align__(1024) unsigned char smraw[];
    TcSmem& S = *reinterpret_cast<TcSmem*>(smraw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles = tiles_m * tiles_n;
    const long long bidx = blockIdx.x / tiles;
    const int tile = blockIdx.x % tiles;
    const int m0 = (tile % tiles_m) * kTcTile, n0 = (tile / tiles_m) * kTcTile;
    const float* A = Aarr[bidx] + a_off;
    const float* B = Barr[bidx] + b_off;
    float* C = Carr[bidx] + c_off;

    if (warp == 0) {
        tmem_alloc(&S.taddr, kTcTile);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(&S.mbar, 1);
        fence_mbar_init();
    }
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tacc = S.taddr;
    constexpr uint32_t idesc = umma_idesc(kTcTile, kTcTile, 2);
    bool ok = true;
    uint32_t phase = 0;

    for (int k0 = 0; k0 < K; k0 += kTcK) {
        // ---- stage op(A) rows m0.., op(B)^T rows n0.. (zero outside the matrices) ----
        for (int e = tid; e < kTcSlice; e += kTcThreads) {
            const int r = e % kTcTile, k = e / kTcTile;
            const int gi = m0 + r, gk = k0 + k;
            float x = 0.0f;
            if (gi < M && gk < K) x = tA ? A[gk + (long long)gi * lda] : A[gi + (long long)gk * lda];
            const float hi = tf32_rne(x);
            S.a_hi[tc_off(r, k)] = hi;
            if (split) S.a_lo[tc_off(r, k)] = tf32_rne(x - hi);
        }
        for (int e = tid; e < kTcSlice; e += kTcThreads) {
            const int k = e % kTcK, r = e / kTcK;
            const int gj = n0 + r, gk = k0 + k;
            float x = 0.0f;
            if (gj < N && gk < K) x = tB ? B[gj + (long long)gk * ldb] : B[gk + (long long)gj * ldb];
            const float hi = tf32_rne(x);
            S.b_hi[tc_off(r, k)] = hi;
            if (split) S.b_lo[tc_off(r, k)] = tf32_rne(x - hi);
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after_sync();
            const uint32_t sbo = kTcK * 32;  // bytes between 8-row groups
#pragma unroll
            for (int s = 0; s < kTcK / 8; s++) {
                const uint32_t step = s * 256;  // 2 core matrices along K
                const uint64_t ah = umma_smem_desc(smem_u32(S.a_hi) + step, 128, sbo);
                const uint64_t bh = umma_smem_desc(smem_u32(S.b_hi) + step, 128, sbo);
                umma_tf32(tacc, ah, bh, idesc, (k0 > 0 || s > 0) ? 1 : 0);
                if (split) {
                    const uint64_t al = umma_smem_desc(smem_u32(S.a_lo) + step, 128, sbo);
                    const uint64_t bl = umma_smem_desc(smem_u32(S.b_lo) + step, 128, sbo);
                    umma_tf32(tacc, ah, bl, idesc, 1);
                    umma_tf32(tacc, al, bh, idesc, 1);
                }
            }
            umma_commit(&S.mbar);
        }
        // every thread waits for the MMAs before the operands are restaged or TMEM is read
        if (!mbar_wait_bounded(&S.mbar, phase, kTcWaitLimit)) ok = false;
        phase ^= 1u;
        tc_fence_after_sync();
        __syncthreads();
    }

    if (!ok && tid == 0) atomicAdd(&g_tc_timeouts, 1u);
    // ---- epilogue: warp w holds accumulator rows 32w..32w+31 ----
    const int gi = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < kTcTile; c0 += 16) {
        if (n0 + c0 >= N) break;
        float v[16];
        tmem_ld16(tacc + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
        if (gi < M) {
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const int gj = n0 + c0 + j;
                if (gj < N) {
                    float* cp = C + gi + (long long)gj * ldc;
                    const float d = K <= 0 ? 0.0f : (ok ? v[j] : __int_as_float(0x7fc00000));
                    *cp = (beta == 0.0f) ? alpha * d : fmaf(alpha, d, beta * *cp);
                }
            }
        }
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tacc, kTcTile);
}

size_t gemm_tc_smem_bytes() { return sizeof(TcSmem); }

cudaError_t gemm_tc_launch(cudaStream_t st, bool transA, bool transB, int m, int n, int k, float alpha,
                           const float* const* A, long long a_off, int lda, const float* const* B, long long b_off,
                           int ldb, float beta, float* const* C, long long c_off, int ldc, int batch, int split)
{
    if (m <= 0 || n <= 0 || batch <= 0) return cudaSuccess;
    const cudaError_t e = ensure_smem_limit(gemm_tc_kernel, (int)gemm_tc_smem_bytes());
    if (e != cudaSuccess) return e;
    const int tm = (m + kTcTile - 1) / kTcTile, tn = (n + kTcTile - 1) / kTcTile;
    const long long blocks = (long long)tm * tn * batch;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    gemm_tc_kernel<<<(unsigned)blocks, kTcThreads, gemm_tc_smem_bytes(), st>>>(
        m, n, k, alpha, A, a_off, lda, transA ? 1 : 0, B, b_off, ldb, transB ? 1 : 0, beta, C, c_off, ldc, tm, tn,
        split);
    return cudaGetLastError();
}

}  // namespace opsblas
