// Batched GEMM on the 5th-generation tensor cores (tcgen05), the engine behind aclblasGemmBatchedEx
// for every dtype the reference supports and for the mixed-precision LU's trailing update:
//   C[b] = alpha * op(A[b]) * op(B[b]) + beta * C[b]   (column-major, pointer arrays, element
//   offsets a_off / b_off / c_off added to every matrix pointer)
//
// Persistent: one CTA per SM walks the 128 x 128 tiles of C (tile t, t + #CTAs, ...: the CTAs
// work on neighbouring tiles of the same matrices at the same time, which share operands in L2;
// or, for the LU's update, one contiguous range of tiles per CTA, so that consecutive tiles keep
// their matrix's tensor maps), nine warps:
//   * warps 0-3 produce: per K tile (128 bytes of K: 64 FP16/BF16, 128 FP8 or 32 TF32 values) they
//     fill a stage of a ring that runs across tile boundaries with op(A) rows m0..m0+127 and
//     op(B)^T rows n0..n0+127 in the 128-byte swizzled canonical UMMA layout of the operand's
//     own orientation in global memory (TcLayout below): K-major for a K-contiguous source (A
//     with op T, B with op N), MN-major for an MN-contiguous one (A with op N, B with op T) --
//     except TF32 operands, which are always staged K-major.
//     With the handle's tensor-map slots, warp 0 loads each stage by TMA: every CTA keeps its
//     per-matrix maps in a global slot and rewrites their base address when it moves to another
//     matrix (tensormap.replace + a release / acquire proxy fence). FP32 operands arrive by TMA
//     when both are K-contiguous and are rounded to TF32 in shared memory by warps 1-3, or arrive
//     already split into TF32 high and low planes (the LU's update). Otherwise the producers copy
//     by cp.async (16 bytes per copy, zero fill at the edges) or, for unaligned matrices and FP32
//     conversions, through registers;
//   * warp 4 issues the MMAs (one elected thread): per stage four K steps of 32 bytes,
//     tcgen05.mma kind::f16 / kind::f8f6f4 / kind::tf32 (three products hi*hi + hi*lo + lo*hi
//     with SPLIT) into one of two 128 x 128 FP32 accumulators in TMEM (256 columns), alternating
//     per tile; tcgen05.commit frees each stage (empty[s]) and, after a tile's last stage, hands
//     the accumulator to the epilogue (acc_full[b]);
//   * warps 5-8 drain the other accumulator meanwhile, in 128 x 32 chunks: each reads its TMEM
//     lane quarter (tcgen05.ld, 32 rows), releases the accumulator (acc_empty[b]) after the last
//     chunk, and applies alpha / beta in C's type. With a tensor map for C the chunks of C are
//     loaded by TMA into a ring of staging buffers before the accumulator is ready (the LU plan:
//     eight buffers, the next tile's chunks loaded while this tile is combined), combined in
//     place and stored by TMA; without one, C is read and written with coalesced loads and
//     stores, the next chunk's values loaded while the current one is stored.
// Every mbarrier wait is bounded. A wait that gives up sets the CTA's abort flag (every role then
// stops) and kStatusTcGemmTimeout in the handle's status word; the copies and MMAs already in
// flight are waited for (bounded) before the TMEM is released, and the tiles not finished keep
// their old C.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <mutex>
#include <type_traits>

#include "internal.h"
#include "small_common.cuh"
#include "tc_common.cuh"

namespace opsblas {

constexpr int kTcTile = 128;                       // M and N of a CTA tile (one MMA: 128 x 128)
constexpr int kTcProducers = 128;                  // warps 0-3
constexpr int kTcEpilogue = 128;                   // warps 5-8
constexpr int kTcThreads = kTcProducers + 32 + kTcEpilogue;  // + the MMA warp (warp 4)
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

// Operand tiles use the 128-byte swizzled canonical UMMA layouts (1024-byte atoms of 8 lines x
// 128 bytes, the 16-byte chunk c of line r stored at chunk position c ^ (r % 8)), so that a warp
// copies four whole 128-byte lines of the source per instruction without bank conflicts.
//   K-major:  line = MN row (0..127), chunk = 16 B of K (0..7): atoms of 8 rows 1024 B apart
//             (SBO); a K step of 32 bytes moves the start address by 32 bytes inside the atom;
//   MN-major: line = K index (0..BK-1), chunk = 16 B of MN (0..8*es-1): 8-row K groups 1024 B
//             apart (SBO), 128-byte MN atoms (BK / 8) * 1024 B apart (LBO).
template <int ES>
struct TcLayout {
    static constexpr int BK = 128 / ES;                  // K values per stage
    static constexpr int MN_CHUNKS = kTcTile * ES / 16;  // 16-byte chunks along MN
    static constexpr uint32_t MN_LBO = (BK / 8) * 1024;  // bytes between 128-byte MN atoms
    __device__ static __forceinline__ uint32_t kmaj(int row, int c16)
    {
        return (row >> 3) * 1024 + (row & 7) * 128 + ((c16 ^ (row & 7)) << 4);
    }
    __device__ static __forceinline__ uint32_t mnmaj(int k, int c16)
    {
        return (c16 >> 3) * MN_LBO + (k >> 3) * 1024 + (k & 7) * 128 + (((c16 & 7) ^ (k & 7)) << 4);
    }
    // descriptor of K step s (32 bytes of K)
    __device__ static __forceinline__ uint64_t desc(uint32_t base, bool mn, int s)
    {
        constexpr uint64_t kSw128 = (uint64_t)2 << 61;
        return mn ? (umma_smem_desc(base + (uint32_t)s * (4 / ES > 0 ? 4 / ES : 1) * 1024, MN_LBO, 1024) | kSw128)
                  : (umma_smem_desc(base + (uint32_t)s * 32, 16, 1024) | kSw128);
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

// q = t / tiles, r = t % tiles, in 32-bit arithmetic when t fits (64-bit division is a long
// instruction sequence on the epilogue's critical path)
__device__ __forceinline__ void tile_split(long long t, int tiles, long long& q, int& r)
{
    if (t >= 0 && t <= 0xffffffffLL) {
        const unsigned tu = (unsigned)t, qq = tu / (unsigned)tiles;
        q = qq;
        r = (int)(tu - qq * (unsigned)tiles);
    } else {
        q = t / tiles;
        r = (int)(t % tiles);
    }
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

// Four C values of column gj at rows src.x..src.w (n of them exist): one vector load when vec
// (a 16-byte (FP32) or 8-byte (FP16 / BF16) aligned run of consecutive rows), else one at a time.
template <GemmElem TC>
__device__ __forceinline__ float4 tc_load_run(const void* C, int4 src, int gj, int ldc, int n, bool vec)
{
    const long long col = (long long)gj * ldc;
    if (vec && n == 4) {
        if constexpr (TC == GemmElem::F32) {
            return *reinterpret_cast<const float4*>(static_cast<const float*>(C) + src.x + col);
        } else {
            using H = typename std::conditional<TC == GemmElem::F16, __half, __nv_bfloat16>::type;
            const uint2 w = *reinterpret_cast<const uint2*>(static_cast<const H*>(C) + src.x + col);
            const H* h = reinterpret_cast<const H*>(&w);
            return make_float4(tc_load_c<TC>(h, 0), tc_load_c<TC>(h, 1), tc_load_c<TC>(h, 2), tc_load_c<TC>(h, 3));
        }
    }
    const int sr[4] = {src.x, src.y, src.z, src.w};
    float v[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int e = 0; e < 4; e++)
        if (e < n) v[e] = tc_load_c<TC>(C, sr[e] + col);
    return make_float4(v[0], v[1], v[2], v[3]);
}

// C[idx .. idx + n) = r[0 .. n) in C's type: one vector store when vec and n == 4.
template <GemmElem TC>
__device__ __forceinline__ void tc_store_vals(void* C, long long idx, const float4& r, int n, bool vec)
{
    if (vec && n == 4) {
        if constexpr (TC == GemmElem::F32) {
            *reinterpret_cast<float4*>(static_cast<float*>(C) + idx) = r;
        } else {
            using H = typename std::conditional<TC == GemmElem::F16, __half, __nv_bfloat16>::type;
            uint2 ow;
            H* oh = reinterpret_cast<H*>(&ow);
            tc_store_c<TC>(oh, 0, r.x);
            tc_store_c<TC>(oh, 1, r.y);
            tc_store_c<TC>(oh, 2, r.z);
            tc_store_c<TC>(oh, 3, r.w);
            *reinterpret_cast<uint2*>(static_cast<H*>(C) + idx) = ow;
        }
        return;
    }
    const float rv[4] = {r.x, r.y, r.z, r.w};
    for (int e = 0; e < n && e < 4; e++) tc_store_c<TC>(C, idx + e, rv[e]);
}

// Shared-memory plan. LU: the LU trailing update (K = 32, one K tile a tile): one operand stage,
// and a ring of eight C chunks so that the next tile's C is loaded while this one is combined.
template <bool SPLIT, bool LU = false>
struct TcStages {
    static constexpr int S = LU ? 1 : (SPLIT ? 2 : 4);
    static constexpr int RING = LU ? 8 : 5;                         // TMA epilogue staging buffers
    static constexpr int PARTS = SPLIT ? 2 : 1;                     // hi (+ lo)
    static constexpr int STAGE_BYTES = 2 * PARTS * kTcOperandBytes;  // A and B
    // epilogue staging: a ring of RING 128 x 32 FP32 chunks of C (the TMA epilogue), or 4 KB per warp
    static constexpr int EPI_BYTES = RING * kTcTile * 32 * 4;
    // stages | barriers (0..511) | tensor maps (512..895) | staging (from 1024) | alignment slack
    static constexpr size_t SMEM = (size_t)S * STAGE_BYTES + 1024 + EPI_BYTES + 1024;
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
    const bool copy = native && vec;
    uint4 hv[8], lv[8];
    uint32_t offs[8];
    // phase 1: every chunk's copy is issued (cp.async) or its elements are loaded into registers
    // before anything is stored, so that the loads of all chunks are in flight together
#pragma unroll
    for (int it = 0; it < 8; it++) {
        const int combo = warp * 8 + it;  // 32 combos of (high line, high chunk) over the 4 warps
        int ln, c16;
        if (!mn) {  // line = row (0..127), chunk along K (0..7): a warp copies 4 whole rows
            ln = combo * 4 + (lane >> 3);
            c16 = lane & 7;
        } else {  // line = k (0..BK-1), chunk along MN: a warp copies one 128-byte atom row of 4 k
            constexpr int ATOMS = L::MN_CHUNKS / 8;
            ln = (combo / ATOMS) * 4 + (lane >> 3);
            c16 = (combo % ATOMS) * 8 + (lane & 7);
        }
        offs[it] = mn ? L::mnmaj(ln, c16) : L::kmaj(ln, c16);
        // the chunk's first element: (row, k) of op(X)
        const int row = mn ? r0 + c16 * NE : r0 + ln;
        const int k = mn ? k0 + ln : k0 + c16 * NE;
        const bool line_ok = mn ? (k < K) : (row < rows);
        const int left = mn ? rows - row : K - k;  // elements left along the chunk's dimension
        const int n = line_ok ? (left < 0 ? 0 : (left > NE ? NE : left)) : 0;
        const long long gidx = src_mn ? (row + (long long)k * ld) : (k + (long long)row * ld);
        if (copy)
            cp_async16_zfill(s_hi + offs[it], n > 0 ? (const void*)(X + gidx) : (const void*)X, n * ES);
        else
            tc_chunk_regs<T, SPLIT>(X + (n > 0 ? gidx : 0), across ? ld : 1, n, hv[it], lv[it]);
    }
    // phase 2: register chunks into shared memory
    if (!copy) {
#pragma unroll
        for (int it = 0; it < 8; it++) {
            asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(s_hi + offs[it]), "r"(hv[it].x),
                         "r"(hv[it].y), "r"(hv[it].z), "r"(hv[it].w)
                         : "memory");
            if (SPLIT)
                asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(s_lo + offs[it]), "r"(lv[it].x),
                             "r"(lv[it].y), "r"(lv[it].z), "r"(lv[it].w)
                             : "memory");
        }
    }
    return copy;
}

__device__ __forceinline__ void sts_v4(uint32_t a, uint32_t x, uint32_t y, uint32_t z, uint32_t w)
{
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(a), "r"(x), "r"(y), "r"(z), "r"(w) : "memory");
}

__device__ __forceinline__ void sts_v2(uint32_t a, uint32_t x, uint32_t y)
{
    asm volatile("st.shared.v2.b32 [%0], {%1, %2};" ::"r"(a), "r"(x), "r"(y) : "memory");
}

__device__ __forceinline__ uint32_t bf16x2_bits(float a, float b)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);  // a in the low half (lower address)
    return *reinterpret_cast<const uint32_t*>(&h);
}

// FP32 operands (TF32 rounding / TF32 high + low split / BF16 conversion): the stage is moved in
// blocks of 4 rows x 4 K values per thread, read with 16-byte loads along the source's contiguous
// dimension (transposed in registers when that is MN) and written as 16-byte (TF32) or 8-byte
// (BF16) shared-memory rows of the operand layout. Blocks that cross the matrix edge, and matrices
// that are not 16-byte aligned (vec4 false), are read element by element.
template <TcIn T, bool SPLIT>
__device__ __forceinline__ void tc_fill_f32(uint32_t s_hi, uint32_t s_lo, const float* X, long long ld, bool src_mn,
                                            int rows, int K, int r0, int k0, bool vec4, int tid)
{
    constexpr int ES = tc_esize(T);  // 4 (TF32) or 2 (BF16)
    using L = TcLayout<ES>;
    constexpr int BK = L::BK;
    constexpr int KB = BK / 4;           // 4-wide K blocks per stage
    constexpr int NB = (kTcTile / 4) * KB;  // blocks per operand tile
    const bool smn = tc_smem_mn<T>(src_mn);
    float v[NB / kTcProducers][4][4];  // [block][row][k]
#pragma unroll
    for (int i = 0; i < NB / kTcProducers; i++) {
        const int bi = tid + i * kTcProducers;
        // consecutive threads walk the source's contiguous dimension
        const int rb = src_mn ? bi % (kTcTile / 4) : bi / KB;
        const int kb = src_mn ? bi / (kTcTile / 4) : bi % KB;
        const int row = r0 + rb * 4, k = k0 + kb * 4;
        if (vec4 && row + 3 < rows && k + 3 < K) {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float4 f = src_mn ? *reinterpret_cast<const float4*>(X + row + (long long)(k + j) * ld)
                                        : *reinterpret_cast<const float4*>(X + k + (long long)(row + j) * ld);
                const float e[4] = {f.x, f.y, f.z, f.w};
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    if (src_mn)
                        v[i][q][j] = e[q];
                    else
                        v[i][j][q] = e[q];
                }
            }
        } else {
#pragma unroll
            for (int rr = 0; rr < 4; rr++)
#pragma unroll
                for (int kk = 0; kk < 4; kk++) {
                    const bool ok = row + rr < rows && k + kk < K;
                    const long long idx = src_mn ? (row + rr + (long long)(k + kk) * ld) : (k + kk + (long long)(row + rr) * ld);
                    v[i][rr][kk] = ok ? X[idx] : 0.0f;
                }
        }
    }
#pragma unroll
    for (int i = 0; i < NB / kTcProducers; i++) {
        const int bi = tid + i * kTcProducers;
        const int rb = src_mn ? bi % (kTcTile / 4) : bi / KB;
        const int kb = src_mn ? bi / (kTcTile / 4) : bi % KB;
        if constexpr (T == TcIn::F32_TF32) {  // K-major, one 16-byte chunk row per block row
#pragma unroll
            for (int rr = 0; rr < 4; rr++) {
                uint32_t h[4], l[4];
#pragma unroll
                for (int kk = 0; kk < 4; kk++) {
                    const float x = v[i][rr][kk];
                    const float hi = tf32_rne(x);
                    h[kk] = __float_as_uint(hi);
                    l[kk] = __float_as_uint(tf32_rne(x - hi));
                }
                const uint32_t off = L::kmaj(rb * 4 + rr, kb);
                sts_v4(s_hi + off, h[0], h[1], h[2], h[3]);
                if (SPLIT) sts_v4(s_lo + off, l[0], l[1], l[2], l[3]);
            }
        } else if (!smn) {  // BF16, K-major: half a chunk row (4 K values) per block row
#pragma unroll
            for (int rr = 0; rr < 4; rr++)
                sts_v2(s_hi + L::kmaj(rb * 4 + rr, kb >> 1) + (kb & 1) * 8, bf16x2_bits(v[i][rr][0], v[i][rr][1]),
                       bf16x2_bits(v[i][rr][2], v[i][rr][3]));
        } else {  // BF16, MN-major: half a chunk row (4 MN values) per block K value
#pragma unroll
            for (int kk = 0; kk < 4; kk++)
                sts_v2(s_hi + L::mnmaj(kb * 4 + kk, rb >> 1) + (rb & 1) * 8, bf16x2_bits(v[i][0][kk], v[i][1][kk]),
                       bf16x2_bits(v[i][2][kk], v[i][3][kk]));
        }
    }
}

// ---- TMA with per-matrix tensor maps ----
__device__ __forceinline__ void tma_load_2d(uint32_t smem_dst, const CUtensorMap* map, int c0, int c1, uint64_t* mbar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_dst),
        "l"(map), "r"(c0), "r"(c1), "r"(smem_u32(mbar))
        : "memory");
}

// Points the tensor map held in shared memory at another matrix.
__device__ __forceinline__ void tmap_replace_address(CUtensorMap* smap, const void* ptr)
{
    asm volatile("tensormap.replace.tile.global_address.shared::cta.b1024.b64 [%0], %1;" ::"r"(smem_u32(smap)),
                 "l"(ptr)
                 : "memory");
}

// Copies a tensor map from shared to global memory with the release fence the TMA unit needs
// (whole warp, converged).
__device__ __forceinline__ void tmap_publish(CUtensorMap* gmap, const CUtensorMap* smap)
{
    asm volatile(
        "tensormap.cp_fenceproxy.global.shared::cta.tensormap::generic.release.gpu.sync.aligned [%0], [%1], 128;" ::"l"(
            gmap),
        "r"(smem_u32(smap))
        : "memory");
}

__device__ __forceinline__ void tmap_acquire(const CUtensorMap* gmap)
{
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(gmap) : "memory");
}

// OR of p over the 128 producer threads (named barrier 1); every producer thread must call it.
__device__ __forceinline__ bool producers_any(bool p)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred q, o;\n\tsetp.ne.b32 q, %1, 0;\n\tbarrier.red.or.pred o, 1, %2, q;\n\tselp.b32 %0, 1, 0, o;\n\t}"
        : "=r"(r)
        : "r"((int)p), "n"(kTcProducers)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void producers_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kTcProducers) : "memory"); }

// Shared -> global tile copies of the TMA epilogue (bulk groups of the issuing thread).
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int c0, int c1, uint32_t smem_src)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(map),
                 "r"(c0), "r"(c1), "r"(smem_src)
                 : "memory");
}

// Until at most N of this thread's committed bulk stores have not yet read their source.
template <int N>
__device__ __forceinline__ void bulk_wait_read_n()
{
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

// OR over the four epilogue warps (5-8, named barrier 3) / their barrier.
__device__ __forceinline__ bool epilogue_any(bool p)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred q, o;\n\tsetp.ne.b32 q, %1, 0;\n\tbarrier.red.or.pred o, 3, %2, q;\n\tselp.b32 %0, 1, 0, o;\n\t}"
        : "=r"(r)
        : "r"((int)p), "n"(kTcEpilogue)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void epilogue_sync() { asm volatile("bar.sync 3, %0;" ::"n"(kTcEpilogue) : "memory"); }

// The same over the three converter warps (1-3) of an FP32 TMA tile (named barrier 2).
__device__ __forceinline__ bool converters_any(bool p)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred q, o;\n\tsetp.ne.b32 q, %1, 0;\n\tbarrier.red.or.pred o, 2, %2, q;\n\tselp.b32 %0, 1, 0, o;\n\t}"
        : "=r"(r)
        : "r"((int)p), "n"(kTcProducers - 32)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void converters_sync()
{
    asm volatile("bar.sync 2, %0;" ::"n"(kTcProducers - 32) : "memory");
}

template <TcIn TA, TcIn TB, GemmElem TC, bool SPLIT, bool LU>
__global__ void __launch_bounds__(kTcThreads, 1)
gemm_tc_kernel(int M, int N, int K, float alpha, const void* const* __restrict__ Aarr, long long a_off, int lda,
               int tA, const void* const* __restrict__ Barr, long long b_off, int ldb, int tB, float beta,
               void* const* __restrict__ Carr, long long c_off, int ldc, int tiles_m, int tiles_n, long long total,
               unsigned* __restrict__ status, unsigned polls, const __grid_constant__ CUtensorMap tmA,
               const __grid_constant__ CUtensorMap tmB, CUtensorMap* __restrict__ gslots, int use_tma,
               int presplit, int a_lo_rows, int b_lo_rows,
               const __grid_constant__ CUtensorMap tmC, int epi_mode, int contig)
{
    static_assert(tc_esize(TA) == tc_esize(TB), "A and B share the MMA kind");
    constexpr int ES = tc_esize(TA);
    using L = TcLayout<ES>;
    using ST = TcStages<SPLIT, LU>;
    constexpr int S = ST::S;
    constexpr int R = ST::RING;
    using SA = typename TcSrc<TA>::type;
    using SB = typename TcSrc<TB>::type;

    // swizzled operand tiles start on 1024-byte boundaries (the swizzle pattern's period)
    extern __shared__ __align__(1024) unsigned char smraw[];
    unsigned char* sm =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(sm + S * ST::STAGE_BYTES);
    uint64_t* empty = full + S;
    uint64_t* ready = empty + S;  // FP32 operands: the stage converted to TF32 (high and low parts)
    uint64_t* acc_full = ready + S;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* drain = acc_empty + 2;
    uint64_t* cload = drain + 1;  // TMA epilogue: the staging buffers' loads of C
    uint32_t* taddr_s = reinterpret_cast<uint32_t*>(cload + R);
    int* abort_s = reinterpret_cast<int*>(taddr_s + 1);
    CUtensorMap* smap = reinterpret_cast<CUtensorMap*>(sm + S * ST::STAGE_BYTES + 512);  // A, B, C (128-aligned)
    float* epi = reinterpret_cast<float*>(sm + S * ST::STAGE_BYTES + 1024);             // epilogue staging

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles = tiles_m * tiles_n;
    // the CTA's tiles: every gridDim.x-th one, or (contig) one contiguous range, so that
    // consecutive tiles mostly belong to the same matrix and keep its tensor maps
    const long long t_first = contig ? (long long)blockIdx.x * total / gridDim.x : (long long)blockIdx.x;
    const long long t_last = contig ? ((long long)blockIdx.x + 1) * total / gridDim.x : total;
    const long long t_step = contig ? 1 : (long long)gridDim.x;
    const bool amn = tA == 0;  // op(A) = A: M contiguous
    const bool bmn = tB != 0;  // op(B)^T rows = B's columns when transposed: N contiguous
    const bool amn_s = tc_smem_mn<TA>(amn), bmn_s = tc_smem_mn<TB>(bmn);  // orientation in shared memory
    const int KT = (K + L::BK - 1) / L::BK;
    // FP32 operands arriving by TMA are converted in shared memory (round to TF32, low parts)
    // before the MMAs: the MMA warp then waits on ready[] instead of full[]
    // (operands that arrive already split into TF32 high and low planes, presplit, need nothing)
    const bool CONVERT = TA == TcIn::F32_TF32 && !presplit;
    uint64_t* hand = CONVERT ? ready : full;

    if (warp == 0) {
        tmem_alloc(taddr_s, 2 * kTcTile);
        tmem_relinquish();
    }
    if (tid == 0) {
        for (int q = 0; q < S; q++) {
            mbar_init(&full[q], 1);  // one arrival: the TMA issuer's expect_tx, or producer 0 after a sync
            mbar_init(&empty[q], 1);
            mbar_init(&ready[q], 1);
        }
        for (int q = 0; q < 2; q++) {
            mbar_init(&acc_full[q], 1);
            mbar_init(&acc_empty[q], kTcEpilogue);
        }
        mbar_init(drain, 1);
        for (int q = 0; q < R; q++) mbar_init(&cload[q], 1);
        *abort_s = 0;
        fence_mbar_init();
    }
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tacc = *taddr_s;
    const uint32_t sbase = smem_u32(sm);
    auto a_hi = [&](int q) { return sbase + (uint32_t)(q * ST::STAGE_BYTES); };
    auto b_hi = [&](int q) { return sbase + (uint32_t)(q * ST::STAGE_BYTES + kTcOperandBytes); };
    auto a_lo = [&](int q) { return sbase + (uint32_t)(q * ST::STAGE_BYTES + 2 * kTcOperandBytes); };
    auto b_lo = [&](int q) { return sbase + (uint32_t)(q * ST::STAGE_BYTES + 3 * kTcOperandBytes); };
    auto aborted = [&]() { return *(volatile int*)abort_s != 0; };
    auto give_up = [&]() { atomicExch(abort_s, 1); };

    if (warp < 4) {
        // ---------------------------------------------------------------- producers
        CUtensorMap* gA = gslots + 3 * (long long)blockIdx.x;
        CUtensorMap* gB = gA + 1;
        if (use_tma && tid == 0) {  // the templates into shared memory, to be pointed at each matrix
            const uint4* pa = reinterpret_cast<const uint4*>(&tmA);
            const uint4* pb = reinterpret_cast<const uint4*>(&tmB);
            uint4* da = reinterpret_cast<uint4*>(&smap[0]);
            uint4* db = reinterpret_cast<uint4*>(&smap[1]);
#pragma unroll
            for (int i = 0; i < 8; i++) {
                da[i] = pa[i];
                db[i] = pb[i];
            }
        }
        long long g = 0;          // K tiles issued by this CTA (the ring position)
        long long issued = 0;     // K tiles whose loads were actually issued (warp 0 tracks it)
        long long mapped = -1;    // the matrix the global maps point at
        for (long long t = t_first; t < t_last; t += t_step) {
            // every producer thread takes the same path through every tile (named barrier 1)
            if (producers_any(aborted())) break;
            long long bidx;
            int tile;
            tile_split(t, tiles, bidx, tile);
            const int m0 = (tile % tiles_m) * kTcTile, n0 = (tile / tiles_m) * kTcTile;
            const SA* A = static_cast<const SA*>(Aarr[bidx]) + a_off;
            const SB* B = static_cast<const SB*>(Barr[bidx]) + b_off;
            const bool avec = (reinterpret_cast<uintptr_t>(A) & 15) == 0 && ((long long)lda * ES) % 16 == 0;
            const bool bvec = (reinterpret_cast<uintptr_t>(B) & 15) == 0 && ((long long)ldb * ES) % 16 == 0;
            const bool tma = use_tma && avec && bvec;
            if (tma) {
                // one thread of warp 0 issues a TMA load per operand (two for 16-bit MN-major A or B)
                if (warp == 0) {
                    if (bidx != mapped) {
                        if (lane == 0) {
                            tmap_replace_address(&smap[0], A);
                            tmap_replace_address(&smap[1], B);
                            // loads still in flight must have read the maps before they change
                            bulk_commit();
                            bulk_wait_read_all();
                        }
                        __syncwarp();
                        tmap_publish(gA, &smap[0]);
                        tmap_publish(gB, &smap[1]);
                        tmap_acquire(gA);
                        tmap_acquire(gB);
                        mapped = bidx;
                    }
                    long long gl = g;
                    for (int kt = 0; kt < KT; kt++, gl++) {
                        const int q = (int)(gl % S);
                        bool ok = gl < S || mbar_wait_or_abort(&empty[q], (uint32_t)((gl / S - 1) & 1), polls, abort_s);
                        ok = __all_sync(0xffffffffu, ok && !aborted());
                        if (!ok) {
                            if (lane == 0) give_up();
                            break;
                        }
                        if (lane == 0 && presplit) {  // high and low planes of both operands
                            const int k0 = kt * L::BK;
                            mbar_arrive_expect_tx(&full[q], 4 * kTcOperandBytes);
                            tma_load_2d(a_hi(q), gA, k0, m0, &full[q]);
                            tma_load_2d(a_lo(q), gA, k0, m0 + a_lo_rows, &full[q]);
                            tma_load_2d(b_hi(q), gB, k0, n0, &full[q]);
                            tma_load_2d(b_lo(q), gB, k0, n0 + b_lo_rows, &full[q]);
                        } else if (lane == 0) {
                            const int k0 = kt * L::BK;
                            mbar_arrive_expect_tx(&full[q], 2 * kTcOperandBytes);
                            if (amn_s) {
                                for (int a = 0; a < ES; a++)
                                    tma_load_2d(a_hi(q) + a * L::MN_LBO, gA, m0 + a * (128 / ES), k0, &full[q]);
                            } else {
                                tma_load_2d(a_hi(q), gA, k0, m0, &full[q]);
                            }
                            if (bmn_s) {
                                for (int a = 0; a < ES; a++)
                                    tma_load_2d(b_hi(q) + a * L::MN_LBO, gB, n0 + a * (128 / ES), k0, &full[q]);
                            } else {
                                tma_load_2d(b_hi(q), gB, k0, n0, &full[q]);
                            }
                        }
                        __syncwarp();
                    }
                    issued = gl;
                } else if (CONVERT && warp > 0) {
                    // warps 1-3: each landed stage to TF32 in place (round to nearest even), plus
                    // the low parts x - hi with SPLIT, then hand it to the MMA warp
                    const int ctid = tid - 32;
                    long long gl = g;
                    for (int kt = 0; kt < KT; kt++, gl++) {
                        const int q = (int)(gl % S);
                        const bool ok = mbar_wait_or_abort(&full[q], (uint32_t)((gl / S) & 1), polls, abort_s);
                        if (converters_any(!ok || aborted())) {
                            if (ctid == 0) give_up();
                            break;
                        }
                        for (int c = ctid; c < 2 * kTcOperandBytes / 16; c += kTcProducers - 32) {
                            const uint32_t off = (uint32_t)(c % (kTcOperandBytes / 16)) * 16;
                            const uint32_t hi_a = (c < kTcOperandBytes / 16 ? a_hi(q) : b_hi(q)) + off;
                            const uint32_t lo_a = (c < kTcOperandBytes / 16 ? a_lo(q) : b_lo(q)) + off;
                            uint32_t x[4];
                            asm volatile("ld.shared.v4.b32 {%0, %1, %2, %3}, [%4];"
                                         : "=r"(x[0]), "=r"(x[1]), "=r"(x[2]), "=r"(x[3])
                                         : "r"(hi_a));
                            uint32_t h[4], l[4];
#pragma unroll
                            for (int e = 0; e < 4; e++) {
                                const float f = __uint_as_float(x[e]);
                                const float hf = tf32_rne(f);
                                h[e] = __float_as_uint(hf);
                                l[e] = __float_as_uint(tf32_rne(f - hf));
                            }
                            sts_v4(hi_a, h[0], h[1], h[2], h[3]);
                            if (SPLIT) sts_v4(lo_a, l[0], l[1], l[2], l[3]);
                        }
                        fence_async_smem();
                        converters_sync();
                        if (ctid == 0) mbar_arrive(&ready[q]);
                    }
                }
                g += KT;
                continue;
            }
            for (int kt = 0; kt < KT; kt++, g++) {
                const int q = (int)(g % S);
                const bool ok = g < S || mbar_wait_or_abort(&empty[q], (uint32_t)((g / S - 1) & 1), polls, abort_s);
                if (producers_any(!ok || aborted())) {
                    give_up();
                    break;
                }
                bool ca = false, cb = false;
                if constexpr (TA == TcIn::F32_TF32 || TA == TcIn::F32_BF16) {
                    const bool a4 = (reinterpret_cast<uintptr_t>(A) & 15) == 0 && lda % 4 == 0;
                    const bool b4 = (reinterpret_cast<uintptr_t>(B) & 15) == 0 && ldb % 4 == 0;
                    tc_fill_f32<TA, SPLIT>(a_hi(q), a_lo(q), reinterpret_cast<const float*>(A), lda, amn, M, K, m0,
                                           kt * L::BK, a4, tid);
                    tc_fill_f32<TB, SPLIT>(b_hi(q), b_lo(q), reinterpret_cast<const float*>(B), ldb, bmn, N, K, n0,
                                           kt * L::BK, b4, tid);
                } else {
                    ca = tc_fill_operand<TA, SPLIT>(a_hi(q), a_lo(q), A, lda, amn, M, K, m0, kt * L::BK, avec, tid);
                    cb = tc_fill_operand<TB, SPLIT>(b_hi(q), b_lo(q), B, ldb, bmn, N, K, n0, kt * L::BK, bvec, tid);
                }
                // hand the stage over once every producer's copies and stores are in place
                if (ca || cb) cp_async_wait_all();
                fence_async_smem();
                producers_sync();
                if (tid == 0) mbar_arrive(&hand[q]);
                issued = g + 1;
            }
        }
        cp_async_wait_all();  // nothing of this thread is still writing shared memory
        if (use_tma && tid == 0) {
            // no TMA load may still be writing shared memory when the CTA ends (after a give-up
            // some stages were never consumed): wait for the last phase of every stage used
            for (long long gg = issued > S ? issued - S : 0; gg < issued; gg++)
                mbar_wait_bounded(&full[gg % S], (uint32_t)((gg / S) & 1), kTcWaitPolls);
        }
    } else if (warp == 4) {
        // ---------------------------------------------------------------- MMA issue
        if (lane == 0) {
            const uint32_t idesc =
                tc_idesc(tc_format(TA), tc_format(TB), amn_s ? 1u : 0u, bmn_s ? 1u : 0u, kTcTile, kTcTile);
            long long g = 0;
            long long i = 0;  // local tile count
            for (long long t = t_first; t < t_last; t += t_step, i++) {
                const int b = (int)(i & 1);
                if (i >= 2 && !mbar_wait_or_abort(&acc_empty[b], (uint32_t)((i / 2 - 1) & 1), polls, abort_s)) {
                    give_up();
                    break;
                }
                const uint32_t dacc = tacc + (uint32_t)(b * kTcTile);
                bool ok = true;
                for (int kt = 0; kt < KT; kt++, g++) {
                    const int q = (int)(g % S);
                    if (!mbar_wait_or_abort(&hand[q], (uint32_t)((g / S) & 1), polls, abort_s)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after_sync();
#pragma unroll
                    for (int st = 0; st < 4; st++) {
                        const uint64_t ah = L::desc(a_hi(q), amn_s, st), bh = L::desc(b_hi(q), bmn_s, st);
                        umma_issue<TA>(dacc, ah, bh, idesc, (kt > 0 || st > 0) ? 1 : 0);
                        if (SPLIT) {
                            const uint64_t al = L::desc(a_lo(q), amn_s, st), bl = L::desc(b_lo(q), bmn_s, st);
                            umma_issue<TA>(dacc, ah, bl, idesc, 1);
                            umma_issue<TA>(dacc, al, bh, idesc, 1);
                        }
                    }
                    umma_commit(&empty[q]);
                }
                if (!ok) {
                    give_up();
                    break;
                }
                umma_commit(&acc_full[b]);
            }
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------------- epilogue (warps 5-8)
        const int quarter = warp & 3;  // TMEM lane quarter this warp may read
        float* stg = epi + quarter * 32 * 32;  // this warp's 32 columns x 32 rows, column-major
        constexpr int CES = TC == GemmElem::F32 ? 4 : 2;
        CUtensorMap* gC = gslots + 3 * (long long)blockIdx.x + 2;
        const int issuer = kTcProducers + 32;  // warp 5, lane 0: every TMA store of C
        long long mapped_c = -1;
        bool prev_tma = false;
        long long gch = 0;      // TMA epilogue chunks so far (the staging buffer ring position)
        long long gis = 0;      // issuer: chunks whose loads of C were issued (runs ahead of gch)
        void* pre_c = nullptr;  // the next tile's matrix pointer, read ahead
        uint32_t cphase = 0;    // bit k: the phase to wait for on cload[k]
        if (epi_mode != 0 && tid == issuer) {
            const uint4* pc = reinterpret_cast<const uint4*>(&tmC);
            uint4* dc = reinterpret_cast<uint4*>(&smap[2]);
#pragma unroll
            for (int k = 0; k < 8; k++) dc[k] = pc[k];
        }
        long long i = 0;
        for (long long t = t_first; t < t_last; t += t_step, i++) {
            const int b = (int)(i & 1);
            long long bidx;
            int tile;
            tile_split(t, tiles, bidx, tile);
            const int m0 = (tile % tiles_m) * kTcTile, n0 = (tile / tiles_m) * kTcTile;
            void* C = static_cast<void*>(static_cast<char*>(i > 0 ? pre_c : Carr[bidx]) + c_off * CES);
            // the next tile's matrix pointer: its load's latency hides behind this tile
            long long bnx = bidx;
            int tlx = tile;
            if (t + t_step < t_last) {
                tile_split(t + t_step, tiles, bnx, tlx);
                pre_c = Carr[bnx];
            }
            const bool cvec = (reinterpret_cast<uintptr_t>(C) & (4 * CES - 1)) == 0 && ((long long)ldc * CES) % (4 * CES) == 0;
            if (epi_mode != 0 && (reinterpret_cast<uintptr_t>(C) & 15) == 0) {
                // ---- TMA epilogue in 128 x 32 chunks through a ring of R staging buffers:
                // beta = 0: alpha * D staged and stored by TMA; otherwise every chunk of the tile's
                // C is loaded by TMA before the accumulator is ready (up to 64 KB in flight; with
                // the LU's ring of eight, each chunk of the CTA's next tile of the same matrix is
                // loaded as soon as this tile's chunk is stored), combined in place
                // (beta * C + alpha * D) and stored.
                if (bidx != mapped_c) {
                    if (warp == kTcProducers / 32 + 1) {
                        if (lane == 0) {
                            tmap_replace_address(&smap[2], C);
                            bulk_commit();
                            bulk_wait_read_all();  // earlier stores must have read the old map
                        }
                        __syncwarp();
                        tmap_publish(gC, &smap[2]);
                        tmap_acquire(gC);
                    }
                    mapped_c = bidx;
                }
                const int nchunks = (N - n0) < kTcTile ? (N - n0 + 31) / 32 : kTcTile / 32;
                epilogue_sync();
                // chunk g's load of C goes to buffer g % R, whose last store was chunk g - R's. The
                // tile's chunks not issued ahead (g = gch + c, c < 4): stores are committed up to
                // chunk gch - 1, so at most R - 4 of them may still be reading their buffers.
                auto issue_load = [&](long long g, int lm0, int ln0) {  // issuer only
                    const int bf = (int)(g % R);
                    mbar_arrive_expect_tx(&cload[bf], (uint32_t)(kTcTile * 32 * CES));
                    tma_load_2d(smem_u32(epi) + (uint32_t)(bf * kTcTile * 32 * 4), gC, lm0, ln0, &cload[bf]);
                };
                if (epi_mode == 2 && tid == issuer && gis < gch + nchunks) {
                    bulk_wait_read_n<R - 4>();
                    for (; gis < gch + nchunks; gis++) issue_load(gis, m0, n0 + (int)(gis - gch) * 32);
                }
                // the CTA's next tile, when it belongs to the same matrix (same tensor map): its
                // chunks are loaded ahead, one after each of this tile's stores (LU ring only)
                const bool ahead = R >= 8 && epi_mode == 2 && t + t_step < t_last && bnx == bidx;
                const int m2 = (tlx % tiles_m) * kTcTile, n2 = (tlx / tiles_m) * kTcTile;
                const int nchunks2 = (N - n2) < kTcTile ? (N - n2 + 31) / 32 : kTcTile / 32;
                // after a give-up: the loads of C issued from chunk g0 on land before the CTA ends
                auto drain_loads = [&](long long g0) {
                    for (long long g = g0; g < gis; g++) {
                        const int bf = (int)(g % R);
                        mbar_wait_bounded(&cload[bf], (cphase >> bf) & 1u, kTcWaitPolls);
                    }
                };
                const long long gch0 = gch;
                const bool ok = mbar_wait_or_abort(&acc_full[b], (uint32_t)((i / 2) & 1), polls, abort_s);
                if (epilogue_any(!ok)) {
                    if (tid == issuer) {
                        give_up();
                        if (epi_mode == 2) drain_loads(gch0);
                    }
                    break;
                }
                tc_fence_after_sync();
                const uint32_t row_addr = tacc + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * kTcTile);
                bool stop = false;
                for (int c = 0; c < nchunks; c++) {
                    const int c0 = c * 32;
                    const int bf = (int)((gch0 + c) % R);
                    float v[32];
                    tmem_ld32(row_addr + (uint32_t)c0, v);
                    if (c + 1 == nchunks) {
                        tc_fence_before_sync();
                        mbar_arrive(&acc_empty[b]);
                    }
                    if (epi_mode == 2) {
                        const bool okc = mbar_wait_or_abort(&cload[bf], (cphase >> bf) & 1u, polls, abort_s);
                        if (epilogue_any(!okc)) {
                            if (tid == issuer) {
                                give_up();
                                drain_loads(gch0 + c);
                            }
                            stop = true;
                            break;
                        }
                        cphase ^= 1u << bf;
                    } else {
                        // the store of chunk gch0 + c - R has read the buffer (R - 1 later ones may be reading)
                        if (tid == issuer) bulk_wait_read_n<R - 1>();
                        epilogue_sync();
                    }
                    const int row = quarter * 32 + lane;
                    if constexpr (TC == GemmElem::F32) {
                        float* buf = epi + bf * kTcTile * 32;
                        if (epi_mode == 2) {
#pragma unroll
                            for (int j = 0; j < 32; j++) {
                                float* e = &buf[j * kTcTile + row];
                                *e = fmaf(beta, *e, alpha * v[j]);
                            }
                        } else {
#pragma unroll
                            for (int j = 0; j < 32; j++) buf[j * kTcTile + row] = alpha * v[j];
                        }
                    } else {
                        using H = typename std::conditional<TC == GemmElem::F16, __half, __nv_bfloat16>::type;
                        H* buf = reinterpret_cast<H*>(epi + bf * kTcTile * 32);
                        if (epi_mode == 2) {
#pragma unroll
                            for (int j = 0; j < 32; j++) {
                                const int e = j * kTcTile + row;
                                tc_store_c<TC>(buf, e, fmaf(beta, tc_load_c<TC>(buf, e), alpha * v[j]));
                            }
                        } else {
#pragma unroll
                            for (int j = 0; j < 32; j++) tc_store_c<TC>(buf, j * kTcTile + row, alpha * v[j]);
                        }
                    }
                    fence_async_smem();
                    epilogue_sync();
                    if (tid == issuer) {
                        tma_store_2d(gC, m0, n0 + c0, smem_u32(epi) + (uint32_t)(bf * kTcTile * 32 * 4));
                        bulk_commit();
                        // the next tile's chunk c: g = gch0 + nchunks + c, its buffer's last store is
                        // chunk g - R <= gch0 + c + 4 - R, with stores committed up to chunk gch0 + c
                        if (ahead && c < nchunks2 && gis == gch0 + nchunks + c) {
                            bulk_wait_read_n<R - 4>();
                            issue_load(gis, m2, n2 + c0);
                            gis++;
                        }
                    }
                }
                gch = gch0 + nchunks;
                if (stop) break;
                prev_tma = true;
                continue;
            }
            if (prev_tma) {  // the staging buffers become the per-warp areas: TMA stores must be done
                if (tid == issuer) bulk_wait_read_all();
                epilogue_sync();
                prev_tma = false;
            }
            // Lane l handles, for every 32-column chunk, the 4-row runs idx = l + 32 i (i < 8):
            // column jj = idx / 8, rows rg * 4 .. + 3 (rg = idx % 8) of this warp's quarter. C's
            // values do not depend on the MMAs: the first chunk's are
            // loaded before the accumulator is ready, each next chunk's while the current one is
            // stored, so a chunk waits for no DRAM round trip of its own.
            auto load_chunk = [&](int c0, float4 (&cv)[8]) {
#pragma unroll
                for (int r = 0; r < 8; r++) {
                    cv[r] = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (beta == 0.0f || K <= 0) continue;
                    const int idx = lane + 32 * r;
                    const int gj = n0 + c0 + (idx >> 3);
                    const int gr = m0 + quarter * 32 + (idx & 7) * 4;
                    if (gj >= N || gr >= M) continue;
                    const int nr = M - gr < 4 ? M - gr : 4;
                    cv[r] = tc_load_run<TC>(C, make_int4(gr, gr + 1, gr + 2, gr + 3), gj, ldc, nr, cvec);
                }
            };
            float4 cv[8], cn[8];
            load_chunk(0, cn);
            const bool okw = mbar_wait_or_abort(&acc_full[b], (uint32_t)((i / 2) & 1), polls, abort_s);
            // (with TMA tiles in this launch the epilogue warps must stay in step: uniform decision)
            if (epi_mode != 0 ? epilogue_any(!okw) : !okw) {
                give_up();
                break;
            }
            tc_fence_after_sync();
            const uint32_t row_addr = tacc + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * kTcTile);
            for (int c0 = 0; c0 < kTcTile; c0 += 32) {
                if (n0 + c0 >= N) break;  // uniform
#pragma unroll
                for (int r = 0; r < 8; r++) cv[r] = cn[r];
                float v[32];
                tmem_ld32(row_addr + (uint32_t)c0, v);
                const bool last = c0 + 32 >= kTcTile || n0 + c0 + 32 >= N;
                if (last) {
                    // the accumulator is in registers: the MMA warp may start the next tile here
                    tc_fence_before_sync();
                    mbar_arrive(&acc_empty[b]);
                } else {
                    load_chunk(c0 + 32, cn);
                }
                // lane = row: stage alpha * D column by column, then every lane writes its runs
#pragma unroll
                for (int j = 0; j < 32; j++) stg[j * 32 + lane] = alpha * v[j];
                __syncwarp();
                if (K > 0) {
#pragma unroll
                    for (int r = 0; r < 8; r++) {
                        const int idx = lane + 32 * r;
                        const int jj = idx >> 3, rg = idx & 7;
                        const int gj = n0 + c0 + jj;
                        const int gr = m0 + quarter * 32 + rg * 4;
                        if (gj >= N || gr >= M) continue;
                        const int nr = M - gr < 4 ? M - gr : 4;
                        const float4 a = *reinterpret_cast<const float4*>(&stg[jj * 32 + rg * 4]);
                        const float4 res = beta == 0.0f
                                               ? a
                                               : make_float4(fmaf(beta, cv[r].x, a.x), fmaf(beta, cv[r].y, a.y),
                                                             fmaf(beta, cv[r].z, a.z), fmaf(beta, cv[r].w, a.w));
                        tc_store_vals<TC>(C, gr + (long long)gj * ldc, res, nr, cvec);
                    }
                }
                __syncwarp();
            }
        }
        if (tid == issuer) bulk_wait_all();  // C is written before the CTA ends
    }

    // ---------------------------------------------------------------- teardown
    if (tid == 4 * 32) umma_commit(drain);  // completes once every MMA issued by this CTA has
    __syncthreads();
    if (!mbar_wait_bounded(drain, 0, kTcWaitPolls)) give_up();
    tc_fence_after_sync();
    __syncthreads();
    if (tid == 0 && aborted()) atomicOr(status, kStatusTcGemmTimeout);
    if (warp == 0) tmem_dealloc(tacc, 2 * kTcTile);
}

using TmapEncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static TmapEncodeFn tmap_encoder()
{
    static TmapEncodeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<TmapEncodeFn>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// Template tensor map of one operand: 2D, 128-byte swizzle, zero fill outside, the box of one TMA
// load (K-major: BK x 128 rows; MN-major: 128 bytes of MN x BK). The base address is a placeholder
// that every CTA replaces with the matrix it loads from.
template <TcIn T>
static bool tmap_encode(CUtensorMap* map, void* placeholder, bool mn, int rows, int K, int ld)
{
    constexpr int ES = tc_esize(T);
    TmapEncodeFn enc = tmap_encoder();
    if (enc == nullptr || ((long long)ld * ES) % 16 != 0) return false;
    const CUtensorMapDataType dt = ES == 1 ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                           : ES == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                                     : (T == TcIn::BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                                        : CU_TENSOR_MAP_DATA_TYPE_FLOAT16);
    const cuuint64_t dims[2] = {(cuuint64_t)(mn ? rows : K), (cuuint64_t)(mn ? K : rows)};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * ES};
    const cuuint32_t box[2] = {(cuuint32_t)(mn ? 128 / ES : 128 / ES), (cuuint32_t)(mn ? 128 / ES : kTcTile)};
    const cuuint32_t estr[2] = {1, 1};
    return enc(map, dt, 2, placeholder, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Template tensor map of C for the TMA epilogue: box 128 rows x 32 columns, no swizzle.
template <GemmElem TC>
static bool tmap_encode_c(CUtensorMap* map, void* placeholder, int m, int n, int ldc)
{
    constexpr int CES = TC == GemmElem::F32 ? 4 : 2;
    TmapEncodeFn enc = tmap_encoder();
    if (enc == nullptr || ((long long)ldc * CES) % 16 != 0) return false;
    const CUtensorMapDataType dt = TC == GemmElem::F32   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                   : TC == GemmElem::F16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                         : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    const cuuint64_t dims[2] = {(cuuint64_t)m, (cuuint64_t)n};
    const cuuint64_t strides[1] = {(cuuint64_t)ldc * CES};
    const cuuint32_t box[2] = {(cuuint32_t)kTcTile, 32};
    const cuuint32_t estr[2] = {1, 1};
    return enc(map, dt, 2, placeholder, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// presplit > 0 (FP32 operands, transA and not transB): op(A) and op(B)^T arrive as TF32 high
// planes whose low planes start presplit rows further down the same arrays.
template <TcIn TA, TcIn TB, GemmElem TC, bool SPLIT, bool LU = false>
static cudaError_t tc_launch_t(cudaStream_t st, bool transA, bool transB, int m, int n, int k, float alpha,
                               const void* const* A, long long a_off, int lda, const void* const* B, long long b_off,
                               int ldb, float beta, void* const* C, long long c_off, int ldc, int batch,
                               unsigned* status, void* tmslots, int presplit = 0)
{
    const size_t smem = TcStages<SPLIT, LU>::SMEM;
    const cudaError_t e = ensure_smem_limit(gemm_tc_kernel<TA, TB, TC, SPLIT, LU>, (int)smem);
    if (e != cudaSuccess) return e;
    const int tm = (m + kTcTile - 1) / kTcTile, tn = (n + kTcTile - 1) / kTcTile;
    const long long total = (long long)tm * tn * batch;
    const long long grid = total < sm_count() ? total : sm_count();  // persistent: one CTA per SM
    CUtensorMap ma{}, mb{}, mc{};
    bool use_tma = false;
    constexpr bool native = TA != TcIn::F32_TF32 && TA != TcIn::F32_BF16;
    // FP32 operands by TMA only when both are K-contiguous (A transposed, B not): they are staged
    // K-major, and converted to TF32 in shared memory (or arrive split, presplit)
    constexpr bool tf32 = TA == TcIn::F32_TF32;
    const bool slots = tmslots != nullptr && grid * 3 * sizeof(CUtensorMap) <= kTensorMapSlotBytes;
    if ((native || (tf32 && transA && !transB)) && slots) {
        // op(A) rows = M (MN-major when A is not transposed); op(B)^T rows = N (MN-major when B is)
        use_tma = tmap_encode<TA>(&ma, tmslots, !transA, presplit + m, k, lda) &&
                  tmap_encode<TB>(&mb, tmslots, transB, presplit + n, k, ldb);
    }
    if (presplit > 0 && !use_tma) return cudaErrorInvalidValue;  // pre-split operands need TMA
    // the TMA epilogue: beta = 0 stores alpha * D, otherwise loads C, combines and stores
    int epi_mode = beta == 0.0f ? 1 : 2;
    if (epi_mode != 0 && !(slots && tmap_encode_c<TC>(&mc, tmslots, m, n, ldc))) epi_mode = 0;
    gemm_tc_kernel<TA, TB, TC, SPLIT, LU><<<(unsigned)grid, kTcThreads, smem, st>>>(
        m, n, k, alpha, A, a_off, lda, transA ? 1 : 0, B, b_off, ldb, transB ? 1 : 0, beta, C, c_off, ldc, tm, tn,
        total, status, wait_limit(kTcWaitPolls), ma, mb, static_cast<CUtensorMap*>(tmslots), use_tma ? 1 : 0,
        presplit > 0 ? 1 : 0, presplit, presplit, mc, epi_mode, LU ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t gemm_tc_typed_launch(cudaStream_t st, TcIn ta_kind, TcIn tb_kind, GemmElem tc_kind, bool split,
                                 bool transA, bool transB, int m, int n, int k, float alpha, const void* const* A,
                                 long long a_off, int lda, const void* const* B, long long b_off, int ldb, float beta,
                                 void* const* C, long long c_off, int ldc, int batch, unsigned* status, void* tmslots)
{
    if (m <= 0 || n <= 0 || batch <= 0) return cudaSuccess;
#define OPSBLAS_TC(TA_, TB_, TC_, SP_)                                                                               \
    return tc_launch_t<TA_, TB_, TC_, SP_>(st, transA, transB, m, n, k, alpha, A, a_off, lda, B, b_off, ldb, beta, C, \
                                           c_off, ldc, batch, status, tmslots)
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
                           unsigned* status, void* tmslots)
{
    return gemm_tc_typed_launch(st, TcIn::F32_TF32, TcIn::F32_TF32, GemmElem::F32, split != 0, transA, transB, m, n,
                                k, alpha, reinterpret_cast<const void* const*>(A), a_off, lda,
                                reinterpret_cast<const void* const*>(B), b_off, ldb, beta,
                                reinterpret_cast<void* const*>(C), c_off, ldc, batch, status, tmslots);
}

cudaError_t gemm_tc_lu_update(cudaStream_t st, int m, const float* const* Aop, const float* const* Bop,
                              float* const* C, long long c_off, int ldc, int batch, int lo_rows, unsigned* status,
                              void* tmslots)
{
    if (m <= 0 || batch <= 0) return cudaSuccess;
    return tc_launch_t<TcIn::F32_TF32, TcIn::F32_TF32, GemmElem::F32, true, true>(
        st, true, false, m, m, 32, -1.0f, reinterpret_cast<const void* const*>(Aop), 0, 32,
        reinterpret_cast<const void* const*>(Bop), 0, 32, 1.0f, reinterpret_cast<void* const*>(C), c_off, ldc, batch,
        status, tmslots, lo_rows);
}

}  // namespace opsblas
