// The column solve and the store of aclblasSgetriBatched for n <= 32, shared by
// getri_small_kernel (getri.cu) and the fused inverse of aclblasSmatinvBatched (matinv.cu).
//
// The reference's getri (getri_batched_kernel.cpp:39-308), per column of C: C = I, row
// interchanges, unit-L forward solve, U backward solve j = n-1..0 that stops at the first zero
// U(j,j) it meets (info = the highest zero diagonal index + 1). On that stop the reference keeps
// C as the forward-solve result for n <= 8 (its register path, :163-168) and partially
// back-substituted for n > 8; both are kept. Lane r of a warp segment solves column r in
// registers (two rows per packed f32x2 FMA) reading L/U from shared memory with broadcast
// 16-byte loads.
#pragma once

#include <cuda_runtime.h>

#include "small_common.cuh"

namespace opsblas {

// Solves column r of C from the LU staged column-major in sm (column stride NP, 16-byte
// aligned) and the 1-based pivots pv of the segment; x2 receives the column (pairs of rows).
// Returns info (uniform within the segment). All 32 lanes of the warp call this.
template <int N>
__device__ __forceinline__ int getri_small_solve(const float* sm, const int* pv, int r, bool cvalid,
                                                 float2 (&x2)[SmallShape<N>::NP / 2])
{
    using S = SmallShape<N>;
    constexpr int NP = S::NP;
    constexpr int NC = S::NC;
    constexpr int NPAIR = NP / 2;
    // Column r of P*I is the unit vector at the position row r moves to.
    const int d = cvalid ? trace_forward<N>(pv, r) : -1;
#pragma unroll
    for (int p = 0; p < NPAIR; p++) x2[p] = make_float2(2 * p == d ? 1.0f : 0.0f, 2 * p + 1 == d ? 1.0f : 0.0f);

    // Unit-L forward solve: x[i] -= L[i][j] * x[j] for i > j; L column j read as float4
    // chunks (broadcast within the segment); fma(L, -x_j, x) == fma(-L, x_j, x) exactly.
#pragma unroll
    for (int j = 0; j < N - 1; j++) {
        const float xj = pget(x2, j);
        const float2 nx = make_float2(-xj, -xj);
        const float* lj = sm + j * NP;
#pragma unroll
        for (int c = j / 4; c < NC; c++) {
            const float4 l4 = *reinterpret_cast<const float4*>(lj + 4 * c);
            // pair 2c = rows 4c, 4c+1; pair 2c+1 = rows 4c+2, 4c+3
            if (4 * c > j) {
                x2[2 * c] = __ffma2_rn(make_float2(l4.x, l4.y), nx, x2[2 * c]);
            } else if (4 * c + 1 > j) {
                x2[2 * c].y = fmaf(l4.y, -xj, x2[2 * c].y);
            }
            if (4 * c + 2 > j && 4 * c + 2 < N) {
                x2[2 * c + 1] = __ffma2_rn(make_float2(l4.z, l4.w), nx, x2[2 * c + 1]);
            } else if (4 * c + 3 > j && 4 * c + 3 < N) {
                x2[2 * c + 1].y = fmaf(l4.w, -xj, x2[2 * c + 1].y);
            }
        }
    }

    // U backward sweep j = n-1..0; it stops at the first zero U(j,j) it meets, so info is the
    // highest zero diagonal + 1. For n <= 8 the reference keeps the forward result in C on a
    // stop, so the diagonal is scanned first; for n > 8 the sweep detects the zero itself.
    int inf = 0;
    if (N <= 8) {
#pragma unroll
        for (int j = N - 1; j >= 0; j--)
            if (inf == 0 && sm[j + j * NP] == 0.0f) inf = j + 1;
    }
    if (!(N <= 8 && inf != 0)) {
#pragma unroll
        for (int j = N - 1; j >= 0; j--) {
            const float* uj = sm + j * NP;
            const float4 dj = *reinterpret_cast<const float4*>(uj + 4 * (j / 4));
            const float ujj = f4get(dj, j % 4);
            if (N > 8) {
                if (S::MPW == 1) {
                    if (ujj == 0.0f) {  // warp-uniform
                        inf = j + 1;
                        break;
                    }
                } else {
                    if (inf == 0 && ujj == 0.0f) inf = j + 1;
                    if (inf != 0) continue;
                }
            }
            const float xj = pget(x2, j) / ujj;
            pset(x2, j, xj);
            const float2 nx = make_float2(-xj, -xj);
#pragma unroll
            for (int c = 0; c <= j / 4; c++) {
                const float4 u4 = (c == j / 4) ? dj : *reinterpret_cast<const float4*>(uj + 4 * c);
                if (4 * c + 1 < j) {
                    x2[2 * c] = __ffma2_rn(make_float2(u4.x, u4.y), nx, x2[2 * c]);
                } else if (4 * c < j) {
                    x2[2 * c].x = fmaf(u4.x, -xj, x2[2 * c].x);
                }
                if (4 * c + 3 < j) {
                    x2[2 * c + 1] = __ffma2_rn(make_float2(u4.z, u4.w), nx, x2[2 * c + 1]);
                } else if (4 * c + 2 < j) {
                    x2[2 * c + 1].x = fmaf(u4.z, -xj, x2[2 * c + 1].x);
                }
            }
        }
    }
    return inf;
}

// Writes the segment's columns to Cm (leading dimension ldc) through sm, which is overwritten:
// column r is staged with its 16-byte chunks rotated by r (chunk q at slot (q + r) % NC) so that
// the lanes hit distinct banks, then the segment stores coalesced columns. All 32 lanes call this.
template <int N>
__device__ __forceinline__ void getri_small_store(float* sm, const float2 (&x2)[SmallShape<N>::NP / 2], int r,
                                                  bool cvalid, bool mvalid, float* Cm, int ldc)
{
    using S = SmallShape<N>;
    constexpr int NP = S::NP;
    constexpr int NC = S::NC;
    // Stage column r of C (rotated chunks), then store coalesced.
    __syncwarp();
    if (cvalid) {
#pragma unroll
        for (int q = 0; q < NC; q++)
            *reinterpret_cast<float4*>(sm + r * NP + 4 * ((q + r) % NC)) =
                make_float4(x2[2 * q].x, x2[2 * q].y, x2[2 * q + 1].x, x2[2 * q + 1].y);
    }
    __syncwarp();
    if (mvalid) {
        if (N % 4 == 0 && (ldc & 3) == 0 && (reinterpret_cast<uintptr_t>(Cm) & 15) == 0) {
            for (int e = r; e < N * NC; e += S::SEG) {
                const int q = e % NC, j = e / NC;
                *reinterpret_cast<float4*>(Cm + 4 * q + (long long)j * ldc) =
                    *reinterpret_cast<const float4*>(sm + j * NP + 4 * ((q + j) % NC));
            }
        } else {
            for (int e = r; e < N * N; e += S::SEG) {
                const int i = e % N, j = e / N;
                Cm[i + (long long)j * ldc] = sm[j * NP + 4 * ((i / 4 + j) % NC) + (i % 4)];
            }
        }
    }
}

}  // namespace opsblas
