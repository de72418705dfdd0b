// LU building blocks shared by the batched kernels (getrf.cu, getrf_reg.cu) and the grouped
// persistent kernel (grouped.cu). Each block restates the reference's unblocked right-looking
// LU (sgetrf_batched_kernel.cpp:106-150): first-maximum pivot, whole-row interchange,
// multipliers by true division, one fmaf per update in column order, stop at the first
// exactly-zero pivot. Whatever kernel runs them, the factors are the same bits.
#pragma once

#include <cuda_runtime.h>

#include "small_common.cuh"

namespace opsblas {

// =============================================================================================
// Register LU for n <= 32: one warp segment per matrix (SEG lanes, 32/SEG matrices per warp).
// Lane r of a segment holds row r of its matrix in registers a4 (float4 chunks, zero padded).
// Pivoting is implicit: rows never move between lanes; `pos` is the row index the lane's row
// has in the reference's in-place matrix at the current step. Per column k:
//   1. argmax of |a[k]| over lanes with pos >= k (redux.sync), ties to the lowest pos --
//      the reference's first-maximum rule; zero and NaN are never chosen;
//   2. the pivot lane publishes its row (from column k on) in shared memory; every lane
//      reads it back with broadcast 16-byte loads;
//   3. lanes below the pivot form l = a[k] / pivot and update a[j] -= l * u[j], j > k.
// =============================================================================================
template <int N>
__device__ __forceinline__ float qget(const float4 (&v)[(N + 3) / 4], int j)
{
    return f4get(v[j >> 2], j & 3);
}

template <int N>
__device__ __forceinline__ void qset(float4 (&v)[(N + 3) / 4], int j, float x)
{
    float4& c = v[j >> 2];
    if ((j & 3) == 0) c.x = x;
    else if ((j & 3) == 1) c.y = x;
    else if ((j & 3) == 2) c.z = x;
    else c.w = x;
}

// a[j] -= l * u[j] on the pairs (x, y) / (z, w) of a float4 chunk, one packed fma per pair;
// fma(u, -l, a) == fma(-l, u, a) exactly.
__device__ __forceinline__ void ffma2_lo(float4& a, float ux, float uy, float2 nl)
{
    const float2 r = __ffma2_rn(make_float2(ux, uy), nl, make_float2(a.x, a.y));
    a.x = r.x;
    a.y = r.y;
}

__device__ __forceinline__ void ffma2_hi(float4& a, float uz, float uw, float2 nl)
{
    const float2 r = __ffma2_rn(make_float2(uz, uw), nl, make_float2(a.z, a.w));
    a.z = r.x;
    a.w = r.y;
}

// Factors the segment's matrix held in a4. rowbuf: this warp's 2 x 32 floats of shared memory
// (16-byte aligned). On return: pos = the lane row's final row index, mypiv = 1-based pivot of
// column r (0 when r >= info), inf = info (uniform within the segment).
template <int N, bool PIVOT, int SEG>
__device__ __forceinline__ void small_getrf_core(float4 (&a4)[(N + 3) / 4], int& pos, int& mypiv, int& inf,
                                                 float* rowbuf, int seg, int r, bool mvalid, bool rvalid)
{
    constexpr int NC = (N + 3) / 4;
    constexpr bool UNIFORM = SEG == 32;  // one matrix per warp: segment state is warp-uniform
    pos = r;
    mypiv = 0;
    inf = 0;
#pragma unroll
    for (int k = 0; k < N; k++) {
        float* buf = rowbuf + (k & 1) * 32 + seg * SEG;
        const bool live = UNIFORM ? rvalid : (rvalid && inf == 0);
        const float ak = qget<N>(a4, k);
        int prow = k;
        bool ispiv;
        if (PIVOT) {
            const bool elig = live && pos >= k;
            const float v = fabsf(ak);
            const unsigned key = (elig && v > 0.0f) ? __float_as_uint(v) : 0u;
            prow = (int)seg_argmax<SEG>(key, elig ? (unsigned)pos : 0xffffffffu, seg);
            ispiv = elig && pos == prow;
        } else {
            ispiv = live && pos == k;
        }
        if (ispiv) {
#pragma unroll
            for (int c = k / 4; c < NC; c++) reinterpret_cast<float4*>(buf)[c] = a4[c];
        }
        __syncwarp();
        const float4 ck = reinterpret_cast<const float4*>(buf)[k / 4];
        const float pv = f4get(ck, k % 4);
        if (UNIFORM) {
            if (PIVOT && r == k) mypiv = prow + 1;
            if (pv == 0.0f) {  // warp-uniform: every lane read the same pivot
                inf = k + 1;
                break;
            }
        } else if (mvalid && inf == 0) {
            if (PIVOT && r == k) mypiv = prow + 1;
            if (pv == 0.0f) inf = k + 1;
        }
        if (UNIFORM ? live : (live && inf == 0)) {
            if (ispiv)
                pos = k;
            else if (pos == k)
                pos = prow;
            if (pos > k) {
                // Multiplier by true division, then a[j] -= l * u[j] for j > k, one fma each.
                const float l = ak / pv;
                qset<N>(a4, k, l);
                const float2 nl = make_float2(-l, -l);
#pragma unroll
                for (int c = k / 4; c < NC; c++) {
                    const float4 u = (c == k / 4) ? ck : reinterpret_cast<const float4*>(buf)[c];
                    // columns 4c..4c+3 that lie right of k
                    if (4 * c > k) {
                        ffma2_lo(a4[c], u.x, u.y, nl);
                    } else if (4 * c + 1 > k) {
                        a4[c].y = fmaf(-l, u.y, a4[c].y);
                    }
                    if (4 * c + 2 > k && 4 * c + 2 < N) {
                        ffma2_hi(a4[c], u.z, u.w, nl);
                    } else if (4 * c + 3 > k && 4 * c + 3 < N) {
                        a4[c].w = fmaf(-l, u.w, a4[c].w);
                    }
                }
            }
        }
    }
}

// Solves one right-hand side with the factors left in registers by small_getrf_core, in the
// reference getrs's order (sgetrs_batched_kernel.cpp:83-200, trans N): b permuted by the row
// interchanges, unit-L forward sweep j = 0..n-1, U backward sweep j = n-1..0 with x_j = y_j /
// U(j,j), one fmaf per update. The lane of original row r enters with y = b[r] (b[r] sits at
// position pos after the interchanges) and leaves with y = x[pos]. owner: this segment's SEG
// ints of shared memory, filled here with the lane of each position. All 32 lanes call this.
template <int N, int SEG>
__device__ __forceinline__ float small_solve_core(const float4 (&a4)[(N + 3) / 4], int pos, bool rvalid, int seg,
                                                  int r, int* owner, float y)
{
    if (rvalid) owner[pos] = r;
    __syncwarp();
    const int base = seg * SEG;
#pragma unroll
    for (int k = 0; k < N; k++) {
        const float yk = __shfl_sync(0xffffffffu, y, base + owner[k]);
        if (rvalid && pos > k) y = fmaf(-qget<N>(a4, k), yk, y);
    }
#pragma unroll
    for (int k = N - 1; k >= 0; k--) {
        const float t = (rvalid && pos == k) ? y / qget<N>(a4, k) : 0.0f;
        const float xk = __shfl_sync(0xffffffffu, t, base + owner[k]);
        if (rvalid) {
            if (pos == k)
                y = xk;
            else if (pos < k)
                y = fmaf(-qget<N>(a4, k), xk, y);
        }
    }
    __syncwarp();
    return y;
}

// Barrier over the team: bar < 0 means the team is the whole CTA; a one-warp team needs only
// the warp barrier.
template <int NT>
__device__ __forceinline__ void team_sync(int bar)
{
    if (NT == 32)
        __syncwarp();
    else if (bar < 0)
        __syncthreads();
    else
        asm volatile("bar.sync %0, %1;\n" ::"r"(bar), "n"(NT) : "memory");
}

// =============================================================================================
// Register LU for 32 < n <= 128, run by a team of NW warps. The matrix lives in registers:
// lane l of every warp holds rows p = l + 32 t (t < R, R = ceil(n / 32)), and warp w holds the
// columns j = s * NW + w (slot s < CW = 32 R / NW), so every warp sees every row and the columns
// are dealt out cyclically (all warps stay busy until the last columns). Pivoting is implicit as
// in small_getrf_core: `pos` (replicated in every warp) is the row's index in the reference's
// in-place matrix; rows never move. Per column k (owner warp k % NW, slot k / NW):
//   A. the owner warp finds the first-maximum pivot (lane-local over t, then redux.sync),
//      forms l = a / pivot for the rows that end below the pivot (true division) and publishes
//      the pivot position, the pivot value and the multipliers in shared memory;
//   B. one team barrier; every warp applies the interchange to `pos`, broadcasts the pivot row's
//      entries of its own columns through shared memory, and updates a(i, j) -= l_i * u_j for
//      its columns j > k and rows below the pivot -- one fmaf per element, column order.
// On an exactly-zero pivot every warp stops (the reference's early exit).
// =============================================================================================
template <int R, int NW>
struct RegShape {
    static constexpr int NMAX = 32 * R;
    static constexpr int CW = NMAX / NW;  // column slots per warp
    static_assert(NMAX % NW == 0 && CW % 4 == 0, "columns must deal out evenly, in float4 chunks");
};

// Shared state of one team.
struct __align__(16) RegTeamSmem {
    float l[2][128];               // multipliers of the current column by physical row (double buffered)
    float u[128];                  // the pivot row's entries; warp w's columns at u[w * CW]
    int lmap[128];                 // after factoring: logical row -> physical row
    int ppos[2];
    float pv[2];
};

// Loads matrix A (n x n, leading dimension lda) into the team's registers.
template <int R, int NW>
__device__ __forceinline__ void reg_load(float (&a)[R][RegShape<R, NW>::CW], const float* A, int lda, int n,
                                         int warp, int lane)
{
    constexpr int CW = RegShape<R, NW>::CW;
#pragma unroll
    for (int s = 0; s < CW; s++) {
        const int j = s * NW + warp;
#pragma unroll
        for (int t = 0; t < R; t++) {
            const int p = lane + 32 * t;
            a[t][s] = (p < n && j < n) ? A[p + (long long)j * lda] : 0.0f;
        }
    }
}

// Stores the factors: row p goes to its final position pos.
template <int R, int NW>
__device__ __forceinline__ void reg_store(const float (&a)[R][RegShape<R, NW>::CW], const int (&pos)[R], float* A,
                                          int lda, int n, int warp, int lane)
{
    constexpr int CW = RegShape<R, NW>::CW;
#pragma unroll
    for (int s = 0; s < CW; s++) {
        const int j = s * NW + warp;
#pragma unroll
        for (int t = 0; t < R; t++) {
            const int p = lane + 32 * t;
            if (p < n && j < n) A[pos[t] + (long long)j * lda] = a[t][s];
        }
    }
}

// Factors the team's matrix. pos must start as the physical row (lane + 32 t); pm (when
// pivoting) must be zero for the whole team before the call (a team barrier after zeroing).
// Returns info.
template <int R, int NW, bool PIVOT>
__device__ __forceinline__ int reg_getrf_core(float (&a)[R][RegShape<R, NW>::CW], int (&pos)[R], int n,
                                              RegTeamSmem& S, int* pm, int warp, int lane, int bar)
{
    constexpr int CW = RegShape<R, NW>::CW;
    int info = 0;
    bool stop = false;
#pragma unroll
    for (int c = 0; c < CW; c++) {
        if (stop) break;
        for (int w = 0; w < NW; w++) {
            const int k = c * NW + w;
            if (k >= n) {
                stop = true;
                break;
            }
            const int buf = k & 1;
            if (warp == w) {
                // ---- A: pivot, multipliers (owner warp) ----
                int ppos = k;
                if (PIVOT) {
                    unsigned bkey = 0, bpos = 0xffffffffu;
#pragma unroll
                    for (int t = 0; t < R; t++) {
                        const bool elig = pos[t] < n && pos[t] >= k;
                        const float v = fabsf(a[t][c]);
                        const unsigned key = (elig && v > 0.0f) ? __float_as_uint(v) : 0u;
                        if (elig && (key > bkey || (key == bkey && (unsigned)pos[t] < bpos))) {
                            bkey = key;
                            bpos = (unsigned)pos[t];
                        }
                    }
                    ppos = (int)seg_argmax<32>(bkey, bpos, 0);
                }
                float cand = 0.0f;
                bool own = false;
#pragma unroll
                for (int t = 0; t < R; t++) {
                    if (pos[t] == ppos) {
                        cand = a[t][c];
                        own = true;
                    }
                }
                const unsigned bal = __ballot_sync(0xffffffffu, own);
                const float pv = __shfl_sync(0xffffffffu, cand, __ffs(bal) - 1);
                if (pv != 0.0f) {
#pragma unroll
                    for (int t = 0; t < R; t++) {
                        const int np = pos[t] == ppos ? k : (pos[t] == k ? ppos : pos[t]);
                        if (np > k && np < n) {
                            const float l = a[t][c] / pv;
                            a[t][c] = l;
                            if (NW > 1) S.l[buf][lane + 32 * t] = l;
                        }
                    }
                }
                if (lane == 0) {
                    S.ppos[buf] = ppos;
                    S.pv[buf] = pv;
                    if (PIVOT) pm[k] = ppos + 1;
                }
            }
            team_sync<NW * 32>(bar);
            // ---- B: interchange, pivot-row broadcast, update (every warp) ----
            const int ppos = S.ppos[buf];
            if (S.pv[buf] == 0.0f) {
                info = k + 1;
                stop = true;
                break;
            }
#pragma unroll
            for (int t = 0; t < R; t++) pos[t] = pos[t] == ppos ? k : (pos[t] == k ? ppos : pos[t]);
            float l[R];
            bool below[R];
#pragma unroll
            for (int t = 0; t < R; t++) {
                below[t] = pos[t] > k && pos[t] < n;
                l[t] = below[t] ? (NW == 1 ? a[t][c] : S.l[buf][lane + 32 * t]) : 0.0f;
            }
            // the lane holding logical row k publishes its slots (from chunk c/4 on) as float4s
            float4* ub4 = reinterpret_cast<float4*>(S.u + warp * CW);
#pragma unroll
            for (int t = 0; t < R; t++) {
                if (pos[t] == k) {
#pragma unroll
                    for (int q = c / 4; q < CW / 4; q++)
                        ub4[q] = make_float4(a[t][4 * q], a[t][4 * q + 1], a[t][4 * q + 2], a[t][4 * q + 3]);
                }
            }
            __syncwarp();
            // update, one float4 chunk of the pivot row at a time (slot c only for warps after the
            // owner; slots > c always), two slots per packed fma; fma(u, -l, a) == fma(-l, u, a)
#pragma unroll
            for (int q = c / 4; q < CW / 4; q++) {
                const float4 v = ub4[q];
                const float uu[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int e = 0; e < 4; e += 2) {
                    const int s0 = 4 * q + e;
                    if (s0 > c) {
#pragma unroll
                        for (int t = 0; t < R; t++) {
                            if (below[t]) {
                                const float2 r2 = __ffma2_rn(make_float2(uu[e], uu[e + 1]), make_float2(-l[t], -l[t]),
                                                             make_float2(a[t][s0], a[t][s0 + 1]));
                                a[t][s0] = r2.x;
                                a[t][s0 + 1] = r2.y;
                            }
                        }
                    } else {
#pragma unroll
                        for (int h = 0; h < 2; h++) {
                            const int sl = s0 + h;
                            if (sl > c || (sl == c && warp > w)) {
#pragma unroll
                                for (int t = 0; t < R; t++)
                                    if (below[t]) a[t][sl] = fmaf(-l[t], uu[e + h], a[t][sl]);
                            }
                        }
                    }
                }
            }
        }
    }
    return info;
}

// =============================================================================================
// Triangular solve from factors held in shared memory (32 < n <= 128; the grouped kernel stages
// its register-resident factors there for the right-hand sides).
// =============================================================================================
constexpr int kMedMaxN = 128;
constexpr int kMedRows = kMedMaxN / 32;  // rows per lane

// Solves right-hand-side column y (n values, logical order after the interchanges: the lane's
// rows i = lane + 32 t enter with y[t] = b[rmap[i]]) with the factors held in shared memory at
// sa (physical row p, column j at sa[p + j * ld]; logical row i is physical row rmap[i]), in the reference
// getrs's order (trans N): unit-L forward sweep, then U backward sweep with x_j = y_j / U(j,j).
// Run by one warp; y[t] leaves as x[lane + 32 t].
__device__ __forceinline__ void med_solve_core(const float* sa, const int* rmap, int n, int ld, int lane,
                                               float (&y)[kMedRows])
{
    int ph[kMedRows];
#pragma unroll
    for (int t = 0; t < kMedRows; t++) ph[t] = (lane + 32 * t < n) ? rmap[lane + 32 * t] : 0;
#pragma unroll
    for (int kq = 0; kq < kMedRows; kq++) {
        for (int kl = 0; kl < 32; kl++) {
            const int k = kq * 32 + kl;
            if (k >= n) break;
            const float yk = __shfl_sync(0xffffffffu, y[kq], kl);
#pragma unroll
            for (int t = 0; t < kMedRows; t++) {
                const int i = lane + 32 * t;
                if (t >= kq && i > k && i < n) y[t] = fmaf(-sa[ph[t] + k * ld], yk, y[t]);
            }
        }
    }
#pragma unroll
    for (int kq = kMedRows - 1; kq >= 0; kq--) {
        for (int kl = 31; kl >= 0; kl--) {
            const int k = kq * 32 + kl;
            if (k >= n) continue;
            const float t0 = (lane == kl) ? y[kq] / sa[ph[kq] + k * ld] : 0.0f;
            const float xk = __shfl_sync(0xffffffffu, t0, kl);
#pragma unroll
            for (int t = 0; t < kMedRows; t++) {
                const int i = lane + 32 * t;
                if (t <= kq) {
                    if (i == k)
                        y[t] = xk;
                    else if (i < k)
                        y[t] = fmaf(-sa[ph[t] + k * ld], xk, y[t]);
                }
            }
        }
    }
}

}  // namespace opsblas
