// Batched GEMM on the 5th-generation tensor cores (tcgen05), the engine behind aclblasGemmBatchedEx
// for every dtype the reference supports and for the mixed-precision LU's trailing update:
//   C[b] = alpha * op(A[b]) * op(B[b]) + beta * C[b]   (column-major, pointer arrays, element
//   offsets a_off / b_off / c_off added to every matrix pointer)
//
// One CTA per 128 x 128 tile of C, five warps:
//   * warps 0-3 produce: per K tile (128 bytes of K: 64 FP16/BF16, 128 FP8 or 32 TF32 values) they
//     fill a pipeline stage with op(A) rows m0..m0+127 and op(B)^T rows n0..n0+127 in the
//     canonical no-swizzle UMMA layout of the operand's own orientation in global memory, so that
//     every 16-byte run of the source is one 16-byte shared-memory row of a core matrix:
//       K-major source (K contiguous: A with op T, B with op N): core matrix = 8 MN-rows x 16 B
//         of K; K-adjacent core matrices 128 B apart (LBO), 8-row groups 1024 B apart (SBO);
//       MN-major source (A with op N, B with op T): core matrix = 8 K-rows x 16 B of MN;
//         MN-adjacent core matrices 128 B apart (SBO), 8-row K groups 128 * (16 B groups along
//         MN) apart (LBO) -- except TF32 operands, which are always staged K-major.
//     Native FP16 / BF16 / FP8 operands whose matrix and leading dimension are 16-byte aligned
//     move by cp.async (16 bytes per copy, zero fill at the edges, no registers held); FP32
//     operands (rounded to TF32 or BF16, or split into TF32 high and low parts) and unaligned
//     matrices go through registers. A stage is handed over with an mbarrier (full[s]);
//   * warp 4 issues the MMAs (one elected thread): per stage four K steps of 32 bytes,
//     tcgen05.mma kind::f16 / kind::f8f6f4 / kind::tf32 into a 128 x 128 FP32 accumulator in
//     TMEM (three products hi*hi + hi*lo + lo*hi with SPLIT), then tcgen05.commit frees the stage
//     (empty[s]) when its MMAs are done; a last commit signals the epilogue;
//   * warps 0-3 then read their 32 accumulator rows each (tcgen05.ld) and apply alpha / beta to C
//     in C's type, coalesced along the columns.
// Every mbarrier wait is bounded. A wait that gives up sets the CTA's abort flag and
// kStatusTcGemmTimeout in the handle's status word; no further loads or MMAs are issued, the
// copies and MMAs already in flight are waited for (bounded), C is left as it was and the TMEM is
// released.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include "internal.h"
#include "small_common.cuh"
#include "tc_common.cuh"

namespace opsblas {

constexpr int kTcTile = 128;                       // M and N of a CTA tile (one MMA: 128 x 128)
constexpr int kTcProducers = 128;                  // warps 0-3
constexpr int kTcThreads = kTcProducers + 32;      // + the MMA warp
constexpr int kTcOperandBytes = kTcTile * 128;     // one operand tile of one stage: 16 KB
constexpr unsigned kTcWaitPolls = 1u << 24;

// shared-memory element of each operand kind, and the MMA kind / format fields
__host__ __device__ constexpr int tc_esize(TcIn t)
{
    return t == TcIn::F32_TF32 ? 4 : ((t == TcIn::E4M3 || t == TcIn::E5M2) ? 1 : 2);
}
__host__ __device__ constexpr uint32_t tc_format(TcIn t)
{
    switch (t) {
        case TcIn::F16: return 0;
        case TcIn::BF16: return 1;
        case TcIn::F32_BF16: return 1;
        case TcIn::F32_TF32: return 2;
        case TcIn::E4M3: return 0;
        case TcIn::E5M2: return 1;
    }
    return 0;
}

// Instruction descriptor: F32 accumulator, A/B formats, A/B major (0 = K, 1 = MN), N >> 3, M >> 4.
__host__ __device__ constexpr uint32_t tc_idesc(uint32_t afmt, uint32_t bfmt, uint32_t amn, uint32_t bmn, int m, int n)
{
    return (1u << 4) | (afmt << 7) | (bfmt << 10) | (amn << 15) | (bmn << 16) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

template <TcIn T>
__device__ __forceinline__ void umma_issue(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, int acc)
{
    if constexpr (T == TcIn::E4M3 || T == TcIn::E5M2) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
            "l"(a), "l"(b), "r"(idesc), "r"(acc)
            : "memory");
    } else if constexpr (T == TcIn::F32_TF32) {
        umma_tf32(d, a, b, idesc, acc);
    } else {
        umma_f16(d, a, b, idesc, acc);
    }
}

// Byte offset of 16-byte chunk `c16` (along the contiguous dimension) of line `ln` (the other
// dimension) in an operand tile, and the descriptor fields, for each source orientation.
//   K-major:  line = MN row (0..127), chunk = 16 B of K (0..7)
//   MN-major: line = K index (0..BK-1), chunk = 16 B of MN (0..8*es-1)
template <int ES>
struct TcLayout {
    static constexpr int BK = 128 / ES;                // K values per stage
    static constexpr int MN_CHUNKS = kTcTile * ES / 16;  // 16-byte groups along MN
    static constexpr uint32_t MN_LBO = MN_CHUNKS * 128;  // bytes between 8-row K groups
    __device__ static __forceinline__ uint32_t kmaj(int row, int c16) { return (row >> 3) * 1024 + c16 * 128 + (row & 7) * 16; }
    __device__ static __forceinline__ uint32_t mnmaj(int k, int c16) { return c16 * 128 + (k >> 3) * MN_LBO + (k & 7) * 16; }
    // descriptor of K step s (32 bytes of K)
    __device__ static __forceinline__ uint64_t desc(uint32_t base, bool mn, int s)
    {
        return mn ? umma_smem_desc(base + (uint32_t)s * (4 / ES > 0 ? 4 / ES : 1) * MN_LBO, MN_LBO, 128)
                  : umma_smem_desc(base + (uint32_t)s * 256, 128, 1024);
    }
};

template <TcIn T>
struct TcSrc;  // storage type of a source element
template <> struct TcSrc<TcIn::F16> { using type = __half; };
template <> struct TcSrc<TcIn::BF16> { using type = __nv_bfloat16; };
template <> struct TcSrc<TcIn::E4M3> { using type = __nv_fp8_e4m3; };
template <> struct TcSrc<TcIn::E5M2> { using type = __nv_fp8_e5m2; };
template <> struct TcSrc<TcIn::F32_TF32> { using type = float; };
template <> struct TcSrc<TcIn::F32_BF16> { using type = float; };

// Register path: 16 bytes of shared-memory operand from the source elements x[0..16/ES) (the
// element at index i lies at src + i * step; `n` of them exist, the rest are zero). hi / lo receive
// the operand (lo only for the TF32 split).
template <TcIn T, bool SPLIT>
__device__ __forceinline__ void tc_chunk_regs(const typename TcSrc<T>::type* src, long long step, int n, uint4& hi,
                                              uint4& lo)
{
    constexpr int ES = tc_esize(T);
    constexpr int NE = 16 / ES;
    uint32_t w[4] = {0u, 0u, 0u, 0u}, wl[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int i = 0; i < NE; i++) {
        if (i < n) {
            const auto v = src[i * step];
            uint32_t bits, lbits = 0;
            if constexpr (T == TcIn::F32_TF32) {
                const float x = v;
                const float h = tf32_rne(x);
                bits = __float_as_uint(h);
                if (SPLIT) lbits = __float_as_uint(tf32_rne(x - h));
            } else if constexpr (T == TcIn::F32_BF16) {
                const __nv_bfloat16 h = __float2bfloat16_rn(v);
                bits = *reinterpret_cast<const unsigned short*>(&h);
            } else if constexpr (ES == 2) {
                bits = *reinterpret_cast<const unsigned short*>(&v);
            } else {
                bits = *reinterpret_cast<const unsigned char*>(&v);
            }
            const int sh = (i * ES * 8) & 31;
            w[(i * ES) >> 2] |= bits << sh;
            if (SPLIT) wl[(i * ES) >> 2] |= lbits << sh;
        }
    }
    hi = make_uint4(w[0], w[1], w[2], w[3]);
    lo = make_uint4(wl[0], wl[1], wl[2], wl[3]);
}

__device__ __forceinline__ void cp_async16_zfill(uint32_t saddr, const void* gmem, int src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(gmem), "r"(src_bytes) : "memory");
}

__device__ __forceinline__ void cp_async_mbar_arrive(uint64_t* mbar)
{
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* mbar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(mbar)) : "memory");
}

template <GemmElem TC>
__device__ __forceinline__ float tc_load_c(const void* C, long long idx)
{
    if constexpr (TC == GemmElem::F32) return static_cast<const float*>(C)[idx];
    if constexpr (TC == GemmElem::F16) return __half2float(static_cast<const __half*>(C)[idx]);
    return __bfloat162float(static_cast<const __nv_bfloat16*>(C)[idx]);
}

template <GemmElem TC>
__device__ __forceinline__ void tc_store_c(void* C, long long idx, float v)
{
    if constexpr (TC == GemmElem::F32) static_cast<float*>(C)[idx] = v;
    if constexpr (TC == GemmElem::F16) static_cast<__half*>(C)[idx] = __float2half_rn(v);
    if constexpr (TC == GemmElem::BF16) static_cast<__nv_bfloat16*>(C)[idx] = __float2bfloat16_rn(v);
}

template <bool SPLIT>
struct TcStages {
    static constexpr int S = SPLIT ? 2 : 3;
    static constexpr int PARTS = SPLIT ? 2 : 1;                     // hi (+ lo)
    static constexpr int STAGE_BYTES = 2 * PARTS * kTcOperandBytes;  // A and B
    static constexpr size_t SMEM = (size_t)S * STAGE_BYTES + 256;  // + barriers, flags, alignment slack
};

// Fills stage `st` with K tile kt of one operand (rows r0.. of op(X), X's leading dimension ld).
// mn: the source is MN-major (contiguous along rows of op(X)). Returns true when the copies were
// cp.async (the caller tracks their completion), false when they were stores from registers.
// TF32 operands are always staged K-major: an MN-major TF32 tile in this layout gave wrong products
// on B200 (measured), so an MN-major FP32 source is read along K (stride ld) into K-major chunks.
template <TcIn T>
__device__ __forceinline__ bool tc_smem_mn(bool src_mn)
{
    return src_mn && T != TcIn::F32_TF32;
}

template <TcIn T, bool SPLIT>
__device__ __forceinline__ bool tc_fill_operand(uint32_t s_hi, uint32_t s_lo, const typename TcSrc<T>::type* X,
                                                long long ld, bool src_mn, int rows, int K, int r0, int k0, bool vec,
                                                int tid)
{
    constexpr int ES = tc_esize(T);
    constexpr int NE = 16 / ES;  // elements per 16-byte chunk
    using L = TcLayout<ES>;
    const int lane = tid & 31, warp = tid >> 5;
    const bool native = T != TcIn::F32_TF32 && T != TcIn::F32_BF16;
    const bool mn = tc_smem_mn<T>(src_mn);          // shared-memory orientation
    const bool across = src_mn && !mn;              // K-major chunks read across an MN-major source
#pragma unroll
    for (int it = 0; it < 8; it++) {
        const int combo = warp * 8 + it;  // 32 combos of (high line, high chunk) over the 4 warps
        int ln, c16;
        if (!mn) {  // line = row (0..127), chunk along K (0..7): lanes cover 8 rows x 4 chunks
            ln = (combo >> 1) * 8 + (lane & 7);
            c16 = (combo & 1) * 4 + (lane >> 3);
        } else {  // line = k (0..BK-1), chunk along MN (0..MN_CHUNKS-1): lanes cover 8 k x 4 chunks
            constexpr int CH_HI = L::MN_CHUNKS / 4;
            ln = (combo / CH_HI) * 8 + (lane & 7);
            c16 = (combo % CH_HI) * 4 + (lane >> 3);
        }
        const uint32_t off = mn ? L::mnmaj(ln, c16) : L::kmaj(ln, c16);
        // the chunk's first element: (row, k) of op(X)
        const int row = mn ? r0 + c16 * NE : r0 + ln;
        const int k = mn ? k0 + ln : k0 + c16 * NE;
        const bool line_ok = mn ? (k < K) : (row < rows);
        const int left = mn ? rows - row : K - k;  // elements left along the chunk's dimension
        const int n = line_ok ? (left < 0 ? 0 : (left > NE ? NE : left)) : 0;
        const long long gidx = src_mn ? (row + (long long)k * ld) : (k + (long long)row * ld);
        if (native && vec) {
            cp_async16_zfill(s_hi + off, n > 0 ? (const void*)(X + gidx) : (const void*)X, n * ES);
        } else {
            uint4 h, l;
            tc_chunk_regs<T, SPLIT>(X + (n > 0 ? gidx : 0), across ? ld : 1, n, h, l);
            asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(s_hi + off), "r"(h.x), "r"(h.y), "r"(h.z),
                         "r"(h.w)
                         : "memory");
            if (SPLIT)
                asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(s_lo + off), "r"(l.x), "r"(l.y),
                             "r"(l.z), "r"(l.w)
                             : "memory");
        }
    }
    return native && vec;
}

template <TcIn TA, TcIn TB, GemmElem TC, bool SPLIT>
__global__ void __launch_bounds__(kTcThreads)
gemm_tc_kernel(int M, int N, int K, float alpha, const void* const* __restrict__ Aarr, long long a_off, int lda,
               int tA, const void* const* __restrict__ Barr, long long b_off, int ldb, int tB, float beta,
               void* const* __restrict__ Carr, long long c_off, int ldc, int tiles_m, int tiles_n,
               unsigned* __restrict__ status, unsigned polls)
{
    static_assert(tc_esize(TA) == tc_esize(TB), "A and B share the MMA kind");
    constexpr int ES = tc_esize(TA);
    using L = TcLayout<ES>;
    using ST = TcStages<SPLIT>;
    constexpr int S = ST::S;
    using SA = typename TcSrc<TA>::type;
    using SB = typename TcSrc<TB>::type;

    // no-swizzle operand layouts need 16-byte alignment only; 128 keeps every tile on its own lines
    extern __shared__ __align__(128) unsigned char smraw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~(uintptr_t)127);
    uint64_t* full = reinterpret_cast<uint64_t*>(sm + S * ST::STAGE_BYTES);
    uint64_t* empty = full + S;
    uint64_t* done = empty + S;
    uint32_t* taddr_s = reinterpret_cast<uint32_t*>(done + 1);
    int* abort_s = reinterpret_cast<int*>(taddr_s + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles = tiles_m * tiles_n;
    const long long bidx = blockIdx.x / tiles;
    const int tile = blockIdx.x % tiles;
    const int m0 = (tile % tiles_m) * kTcTile, n0 = (tile / tiles_m) * kTcTile;
    const SA* A = static_cast<const SA*>(Aarr[bidx]) + a_off;
    const SB* B = static_cast<const SB*>(Barr[bidx]) + b_off;
    const bool amn = tA == 0;  // op(A) = A: M contiguous
    const bool bmn = tB != 0;  // op(B)^T rows = B's columns when transposed: N contiguous
    const bool amn_s = tc_smem_mn<TA>(amn), bmn_s = tc_smem_mn<TB>(bmn);  // orientation in shared memory
    const int KT = (K + L::BK - 1) / L::BK;

    if (warp == 0) {
        tmem_alloc(taddr_s, kTcTile);
        tmem_relinquish();
    }
    if (tid == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(&full[s], kTcProducers);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        *abort_s = 0;
        fence_mbar_init();
    }
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tacc = *taddr_s;
    const uint32_t sbase = smem_u32(sm);
    auto a_hi = [&](int s) { return sbase + (uint32_t)(s * ST::STAGE_BYTES); };
    auto b_hi = [&](int s) { return sbase + (uint32_t)(s * ST::STAGE_BYTES + kTcOperandBytes); };
    auto a_lo = [&](int s) { return sbase + (uint32_t)(s * ST::STAGE_BYTES + 2 * kTcOperandBytes); };
    auto b_lo = [&](int s) { return sbase + (uint32_t)(s * ST::STAGE_BYTES + 3 * kTcOperandBytes); };

    if (warp < 4) {
        // ---------------------------------------------------------------- producers
        const bool avec = (reinterpret_cast<uintptr_t>(A) & 15) == 0 && ((long long)lda * ES) % 16 == 0;
        const bool bvec = (reinterpret_cast<uintptr_t>(B) & 15) == 0 && ((long long)ldb * ES) % 16 == 0;
        bool pending = false;  // cp.async group of the previous tile not yet handed over
        int prev_s = 0;
        for (int kt = 0; kt < KT; kt++) {
            const int s = kt % S;
            if (kt >= S) {
                const bool ok = mbar_wait_or_abort(&empty[s], (uint32_t)((kt / S - 1) & 1), polls, abort_s);
                if (!ok) atomicExch(abort_s, 1);
            }
            if (*(volatile int*)abort_s) break;
            const bool ca = tc_fill_operand<TA, SPLIT>(a_hi(s), a_lo(s), A, lda, amn, M, K, m0, kt * L::BK, avec, tid);
            const bool cb = tc_fill_operand<TB, SPLIT>(b_hi(s), b_lo(s), B, ldb, bmn, N, K, n0, kt * L::BK, bvec, tid);
            if (ca || cb) {
                cp_async_commit();
                if (pending) {  // hand over the previous stage once its copies have landed
                    cp_async_wait_group<1>();
                    fence_async_smem();
                    mbar_arrive(&full[prev_s]);
                }
                pending = true;
                prev_s = s;
            } else {
                if (pending) {
                    cp_async_wait_all();
                    fence_async_smem();
                    mbar_arrive(&full[prev_s]);
                    pending = false;
                }
                fence_async_smem();
                mbar_arrive(&full[s]);
            }
        }
        if (pending) {
            cp_async_wait_all();
            fence_async_smem();
            mbar_arrive(&full[prev_s]);
        }
        cp_async_wait_all();  // nothing of this thread is still writing shared memory
    } else if (lane == 0) {
        // ---------------------------------------------------------------- MMA issue
        const uint32_t idesc =
            tc_idesc(tc_format(TA), tc_format(TB), amn_s ? 1u : 0u, bmn_s ? 1u : 0u, kTcTile, kTcTile);
        for (int kt = 0; kt < KT; kt++) {
            const int s = kt % S;
            if (!mbar_wait_or_abort(&full[s], (uint32_t)((kt / S) & 1), polls, abort_s)) {
                atomicExch(abort_s, 1);
                break;
            }
            tc_fence_after_sync();
#pragma unroll
            for (int st = 0; st < 4; st++) {
                const uint64_t ah = L::desc(a_hi(s), amn_s, st), bh = L::desc(b_hi(s), bmn_s, st);
                umma_issue<TA>(tacc, ah, bh, idesc, (kt > 0 || st > 0) ? 1 : 0);
                if (SPLIT) {
                    const uint64_t al = L::desc(a_lo(s), amn_s, st), bl = L::desc(b_lo(s), bmn_s, st);
                    umma_issue<TA>(tacc, ah, bl, idesc, 1);
                    umma_issue<TA>(tacc, al, bh, idesc, 1);
                }
            }
            umma_commit(&empty[s]);
        }
        umma_commit(done);  // completes when every MMA issued above has
    }
    if (warp == 4) __syncwarp();

    // ---------------------------------------------------------------- epilogue (warps 0-3)
    if (warp < 4) {
        bool ok = mbar_wait_bounded(done, 0, polls);
        if (!ok) {
            atomicExch(abort_s, 1);
            ok = mbar_wait_bounded(done, 0, kTcWaitPolls);  // the MMAs in flight finish first
        }
        tc_fence_after_sync();
        const bool skip = *(volatile int*)abort_s != 0 || K <= 0;
        void* C = static_cast<void*>(static_cast<char*>(Carr[bidx]) + c_off * (TC == GemmElem::F32 ? 4 : 2));
        const int gi = m0 + warp * 32 + lane;
        for (int c0 = 0; c0 < kTcTile; c0 += 16) {
            if (n0 + c0 >= N) break;
            float v[16];
            tmem_ld16(tacc + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (!skip && gi < M) {
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int gj = n0 + c0 + j;
                    if (gj < N) {
                        const long long idx = gi + (long long)gj * ldc;
                        const float d = alpha * v[j];
                        tc_store_c<TC>(C, idx, beta == 0.0f ? d : fmaf(beta, tc_load_c<TC>(C, idx), d));
                    }
                }
            }
        }
    }
    tc_fence_before_sync();
    __syncthreads();
    if (tid == 0 && *(volatile int*)abort_s) atomicOr(status, kStatusTcGemmTimeout);
    if (warp == 0) tmem_dealloc(tacc, kTcTile);
}

template <TcIn TA, TcIn TB, GemmElem TC, bool SPLIT>
static cudaError_t tc_launch_t(cudaStream_t st, bool transA, bool transB, int m, int n, int k, float alpha,
                               const void* const* A, long long a_off, int lda, const void* const* B, long long b_off,
                               int ldb, float beta, void* const* C, long long c_off, int ldc, int batch,
                               unsigned* status)
{
    const size_t smem = TcStages<SPLIT>::SMEM;
    const cudaError_t e = ensure_smem_limit(gemm_tc_kernel<TA, TB, TC, SPLIT>, (int)smem);
    if (e != cudaSuccess) return e;
    const int tm = (m + kTcTile - 1) / kTcTile, tn = (n + kTcTile - 1) / kTcTile;
    const long long blocks = (long long)tm * tn * batch;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    gemm_tc_kernel<TA, TB, TC, SPLIT><<<(unsigned)blocks, kTcThreads, smem, st>>>(
        m, n, k, alpha, A, a_off, lda, transA ? 1 : 0, B, b_off, ldb, transB ? 1 : 0, beta, C, c_off, ldc, tm, tn,
        status, wait_limit(kTcWaitPolls));
    return cudaGetLastError();
}

cudaError_t gemm_tc_typed_launch(cudaStream_t st, TcIn ta_kind, TcIn tb_kind, GemmElem tc_kind, bool split,
                                 bool transA, bool transB, int m, int n, int k, float alpha, const void* const* A,
                                 long long a_off, int lda, const void* const* B, long long b_off, int ldb, float beta,
                                 void* const* C, long long c_off, int ldc, int batch, unsigned* status)
{
    if (m <= 0 || n <= 0 || batch <= 0) return cudaSuccess;
#define OPSBLAS_TC(TA_, TB_, TC_, SP_)                                                                               \
    return tc_launch_t<TA_, TB_, TC_, SP_>(st, transA, transB, m, n, k, alpha, A, a_off, lda, B, b_off, ldb, beta, C, \
                                           c_off, ldc, batch, status)
    using E = GemmElem;
    if (ta_kind == TcIn::F32_TF32) {
        if (tc_kind != E::F32) return cudaErrorInvalidValue;
        if (split) OPSBLAS_TC(TcIn::F32_TF32, TcIn::F32_TF32, E::F32, true);
        OPSBLAS_TC(TcIn::F32_TF32, TcIn::F32_TF32, E::F32, false);
    }
    if (ta_kind == TcIn::F32_BF16 && tc_kind == E::F32) OPSBLAS_TC(TcIn::F32_BF16, TcIn::F32_BF16, E::F32, false);
    if (ta_kind == TcIn::F16 && tc_kind == E::F16) OPSBLAS_TC(TcIn::F16, TcIn::F16, E::F16, false);
    if (ta_kind == TcIn::BF16 && tc_kind == E::BF16) OPSBLAS_TC(TcIn::BF16, TcIn::BF16, E::BF16, false);
    if (tc_kind == E::F16) {
        if (ta_kind == TcIn::E4M3 && tb_kind == TcIn::E4M3) OPSBLAS_TC(TcIn::E4M3, TcIn::E4M3, E::F16, false);
        if (ta_kind == TcIn::E4M3 && tb_kind == TcIn::E5M2) OPSBLAS_TC(TcIn::E4M3, TcIn::E5M2, E::F16, false);
        if (ta_kind == TcIn::E5M2 && tb_kind == TcIn::E4M3) OPSBLAS_TC(TcIn::E5M2, TcIn::E4M3, E::F16, false);
        if (ta_kind == TcIn::E5M2 && tb_kind == TcIn::E5M2) OPSBLAS_TC(TcIn::E5M2, TcIn::E5M2, E::F16, false);
    }
#undef OPSBLAS_TC
    return cudaErrorInvalidValue;
}

cudaError_t gemm_tc_launch(cudaStream_t st, bool transA, bool transB, int m, int n, int k, float alpha,
                           const float* const* A, long long a_off, int lda, const float* const* B, long long b_off,
                           int ldb, float beta, float* const* C, long long c_off, int ldc, int batch, int split,
                           unsigned* status)
{
    return gemm_tc_typed_launch(st, TcIn::F32_TF32, TcIn::F32_TF32, GemmElem::F32, split != 0, transA, transB, m, n,
                                k, alpha, reinterpret_cast<const void* const*>(A), a_off, lda,
                                reinterpret_cast<const void* const*>(B), b_off, ldb, beta,
                                reinterpret_cast<void* const*>(C), c_off, ldc, batch, status);
}

}  // namespace opsblas
