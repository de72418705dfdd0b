// Device helpers shared by the register-resident kernels for n <= 32.
//
// Layout: a warp is split into 32/SEG segments of SEG lanes (SEG = 4, 8, 16 or 32, the
// smallest power of two >= n, at least 4); each segment works on one matrix, and lane r of a
// segment owns row r (getrf, getrs) or column r (getri) of it in registers.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace opsblas {

constexpr int kSmallWarps = 8;  // warps per CTA of the small kernels

template <int N>
struct SmallShape {
    static constexpr int SEG = N <= 4 ? 4 : (N <= 8 ? 8 : (N <= 16 ? 16 : 32));
    static constexpr int MPW = 32 / SEG;   // matrices per warp
    static constexpr int NC = (N + 3) / 4;  // float4 chunks per padded row
    static constexpr int NP = NC * 4;       // padded row length (<= SEG)
};

__device__ __forceinline__ float f4get(const float4& v, int i)
{
    return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

// Element j of a row held as float2 pairs (j compile-time after unrolling).
template <int NPAIR>
__device__ __forceinline__ float pget(const float2 (&v)[NPAIR], int j)
{
    return (j & 1) ? v[j >> 1].y : v[j >> 1].x;
}

template <int NPAIR>
__device__ __forceinline__ void pset(float2 (&v)[NPAIR], int j, float x)
{
    if (j & 1)
        v[j >> 1].y = x;
    else
        v[j >> 1].x = x;
}

// Asynchronous global -> shared copies (cp.async, sm_80+): no registers held while in flight.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}

// Closes the current group of cp.async copies / waits until at most N groups are pending.
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Waits for this thread's outstanding cp.async copies; a __syncwarp()/__syncthreads() must
// follow before other threads read the data.
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Per-segment max of `key` over the lanes of each segment, then the minimum `cand` among the
// lanes whose key equals that max. Full-warp redux.sync per segment, other lanes contribute
// the identity, so the result never mixes segments. Must be called by all 32 lanes.
template <int SEG>
__device__ __forceinline__ unsigned seg_argmax(unsigned key, unsigned cand, int seg)
{
    if constexpr (SEG == 32) {
        const unsigned mx = __reduce_max_sync(0xffffffffu, key);
        return __reduce_min_sync(0xffffffffu, key == mx ? cand : 0xffffffffu);
    } else {
        constexpr int MPW = 32 / SEG;
        unsigned mx = 0;
#pragma unroll
        for (int s = 0; s < MPW; s++) {
            const unsigned v = __reduce_max_sync(0xffffffffu, seg == s ? key : 0u);
            if (seg == s) mx = v;
        }
        const unsigned c = key == mx ? cand : 0xffffffffu;
        unsigned best = 0xffffffffu;
#pragma unroll
        for (int s = 0; s < MPW; s++) {
            const unsigned v = __reduce_min_sync(0xffffffffu, seg == s ? c : 0xffffffffu);
            if (seg == s) best = v;
        }
        return best;
    }
}

// Applies the row interchanges of a pivot vector to a row index. `pv` holds the 1-based
// pivots in shared memory (16-byte aligned); out-of-range and self pivots are skipped as in the
// reference (sgetrs_batched_kernel.cpp:94-100). FORWARD = true applies k = 0..n-1 in order
// (the row that row r moves to under LAPACK laswp); FORWARD = false applies k = n-1..0 (the
// source row of position r after laswp, equivalently where row r goes under the reverse
// interchanges).
template <int N, bool FORWARD>
__device__ __forceinline__ int trace_pivots(const int* pv, int r)
{
    constexpr int NC = (N + 3) / 4;
    int4 q[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) q[c] = reinterpret_cast<const int4*>(pv)[c];
    int pos = r;
#pragma unroll
    for (int t = 0; t < N; t++) {
        const int k = FORWARD ? t : N - 1 - t;
        const int4& qc = q[k / 4];
        const int p = ((k % 4) == 0 ? qc.x : (k % 4) == 1 ? qc.y : (k % 4) == 2 ? qc.z : qc.w) - 1;
        if ((unsigned)p < (unsigned)N && p != k) pos = (pos == k) ? p : (pos == p ? k : pos);
    }
    return pos;
}

template <int N>
__device__ __forceinline__ int trace_forward(const int* pv, int r)
{
    return trace_pivots<N, true>(pv, r);
}

template <int N>
__device__ __forceinline__ int trace_backward(const int* pv, int r)
{
    return trace_pivots<N, false>(pv, r);
}

}  // namespace opsblas

// Dispatch helper: expands CASE(n) for n = 1..32.
#define OPSBLAS_FOR_N_1_32(CASE)                                                                                     \
    CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9) CASE(10) CASE(11) CASE(12) CASE(13)    \
    CASE(14) CASE(15) CASE(16) CASE(17) CASE(18) CASE(19) CASE(20) CASE(21) CASE(22) CASE(23) CASE(24) CASE(25)     \
    CASE(26) CASE(27) CASE(28) CASE(29) CASE(30) CASE(31) CASE(32)
