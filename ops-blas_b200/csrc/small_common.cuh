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

// Position that row `r` takes after the row interchanges k = 0..n-1 of a pivot vector
// (LAPACK laswp forward order) -- equivalently the source row of position r after the
// interchanges applied in reverse order. `pv` holds the 1-based pivots in shared memory;
// out-of-range and self pivots are skipped as in the reference (sgetrs_batched_kernel.cpp:94-100).
template <int N>
__device__ __forceinline__ int trace_forward(const int* pv, int r)
{
    int pos = r;
#pragma unroll
    for (int k = 0; k < N; k++) {
        const int p = pv[k] - 1;
        if (p >= 0 && p < N && p != k) pos = (pos == k) ? p : (pos == p ? k : pos);
    }
    return pos;
}

// Same interchanges traced in reverse order (k = n-1..0).
template <int N>
__device__ __forceinline__ int trace_backward(const int* pv, int r)
{
    int pos = r;
#pragma unroll
    for (int k = N - 1; k >= 0; k--) {
        const int p = pv[k] - 1;
        if (p >= 0 && p < N && p != k) pos = (pos == k) ? p : (pos == p ? k : pos);
    }
    return pos;
}

}  // namespace opsblas

// Dispatch helper: expands CASE(n) for n = 1..32.
#define OPSBLAS_FOR_N_1_32(CASE)                                                                                     \
    CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9) CASE(10) CASE(11) CASE(12) CASE(13)    \
    CASE(14) CASE(15) CASE(16) CASE(17) CASE(18) CASE(19) CASE(20) CASE(21) CASE(22) CASE(23) CASE(24) CASE(25)     \
    CASE(26) CASE(27) CASE(28) CASE(29) CASE(30) CASE(31) CASE(32)
