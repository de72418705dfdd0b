// Register/shared-memory kernels of aclblasSgetrsBatched for n <= 32 (see getrs.cu).
#pragma once

#include <cuda_runtime.h>

#include "small_common.cuh"

namespace opsblas {

// ---------------------------------------------------------------------------------------
// nrhs == 1, n <= 32, trans N: lane r of a warp segment holds row r of LU in registers and
// entry r of the right-hand side; the interchanges are folded into the row the lane loads;
// solution entries are broadcast by shuffles. Each x[i] takes its updates in the reference's
// order (j ascending in the L sweep, descending in the U sweep). Trans T / C goes to
// getrs_rhs_kernel instead: the reference's L^T sweep adds x[j]'s terms with i ascending,
// which a lane per column can only follow one position at a time.
// ---------------------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(kSmallWarps * 32)
getrs_small_kernel(const float* const* __restrict__ Aarray, int lda, const int* __restrict__ ipiv,
                   float* const* __restrict__ Barray, int ldb, int batch)
{
    using S = SmallShape<N>;
    __shared__ __align__(16) int pbuf[kSmallWarps][32];

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int seg = lane / S::SEG;
    const int r = lane % S::SEG;
    const long long m = ((long long)blockIdx.x * kSmallWarps + warp) * S::MPW + seg;
    const bool mvalid = m < batch && Barray[m] != nullptr;  // a NULL right-hand side skips the matrix
    const bool rvalid = mvalid && r < N;

    const float* A = mvalid ? Aarray[m] : nullptr;
    float* B = mvalid ? Barray[m] : nullptr;

    float lu[N];
#pragma unroll
    for (int j = 0; j < N; j++) lu[j] = 0.0f;
    if (rvalid) {
#pragma unroll
        for (int j = 0; j < N; j++) lu[j] = A[r + (long long)j * lda];
    }

    int* pv = &pbuf[warp][seg * S::SEG];
    if (r < N) pv[r] = (ipiv != nullptr && mvalid) ? ipiv[m * N + r] : r + 1;
    __syncwarp();
    const int prow = rvalid ? trace_backward<N>(pv, r) : r;
    const int base = seg * S::SEG;

    float x = rvalid ? B[prow] : 0.0f;
#pragma unroll
    for (int j = 0; j < N; j++) {
        const float xj = __shfl_sync(0xffffffffu, x, base + j);
        if (r > j) x = fmaf(-lu[j], xj, x);
    }
#pragma unroll
    for (int j = N - 1; j >= 0; j--) {
        if (r == j) x = x / lu[j];
        const float xj = __shfl_sync(0xffffffffu, x, base + j);
        if (r < j) x = fmaf(-lu[j], xj, x);
    }
    if (rvalid) B[r] = x;
}

// ---------------------------------------------------------------------------------------
// n <= 32 with nrhs >= 2, or trans T / C with any nrhs: the reference's
// thread-per-right-hand-side structure (sgetrs_batched_kernel.cpp:365-388) with B200
// staging. A warp holds 32/LPM matrices; the LPM
// lanes of a segment own right-hand sides c = q, q+LPM, ... of one matrix and keep that
// column in registers. The matrix's LU is staged in shared memory by cp.async and read as
// broadcast 16-byte column chunks; the interchanges become a row map computed once per
// matrix (x[i] = B[map[i]] for N, B[map[j]] = x[j] for T).
//   N: right-looking unit-L forward and U backward sweeps over L/U columns, two rows per
//      packed f32x2 FMA -- the reference's per-element operation order;
//   T: U^T forward and L^T backward as dot products over LU columns, again in the
//      reference's per-element order (:263-362).
// ---------------------------------------------------------------------------------------
template <int N, int LPM>
struct RhsShape {
    static constexpr int NP = (N + 3) / 4 * 4;
    static constexpr int NC = NP / 4;
    static constexpr int MPW = 32 / LPM;
    static constexpr int MAT = N * NP + 4;       // floats of one staged matrix (16-byte stagger)
    static constexpr int SLOT = MAT + 64;        // + pivots and row map (32 ints each)
    static constexpr int BCOL = NP;              // staged right-hand-side column per lane
    static constexpr int WARP_WORDS = MPW * SLOT + 32 * BCOL;
    static constexpr int W0 = 9216 / WARP_WORDS;  // about 36 KiB per CTA: several CTAs per SM
    static constexpr int WARPS = W0 < 1 ? 1 : (W0 > 8 ? 8 : W0);
    static constexpr size_t SMEM = (size_t)WARPS * WARP_WORDS * 4;
};

template <int N, int LPM, bool TRANS>
__global__ void __launch_bounds__(RhsShape<N, LPM>::WARPS * 32)
getrs_rhs_kernel(const float* const* __restrict__ Aarray, int lda, const int* __restrict__ ipiv,
                 float* const* __restrict__ Barray, int ldb, int nrhs, int batch)
{
    using R = RhsShape<N, LPM>;
    constexpr int NP = R::NP, NC = R::NC, NPAIR = NP / 2;
    extern __shared__ __align__(16) float dsm[];

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int seg = lane / LPM;
    const int q = lane % LPM;
    const long long m = ((long long)blockIdx.x * R::WARPS + warp) * R::MPW + seg;
    const bool mvalid = m < batch && Barray[m] != nullptr;  // a NULL right-hand side skips the matrix
    float* wbase = dsm + warp * R::WARP_WORDS;
    float* sm = wbase + seg * R::SLOT;
    int* pv = reinterpret_cast<int*>(sm + R::MAT);
    int* map = pv + 32;
    float* bs = wbase + R::MPW * R::SLOT + lane * R::BCOL;  // this lane's right-hand side

    const float* A = mvalid ? Aarray[m] : nullptr;
    float* B = mvalid ? Barray[m] : nullptr;
    const bool bvec = N % 4 == 0 && (ldb & 3) == 0 && (reinterpret_cast<uintptr_t>(B) & 15) == 0;

    // Issue every global read of the first right-hand side up front: LU and B by cp.async,
    // the pivots as plain loads; the row map is built while the copies are in flight.
    auto stage_rhs = [&](int c) {
        const float* Bc = B + (long long)c * ldb;
        if (bvec) {
#pragma unroll
            for (int t = 0; t < NC; t++) cp_async16(bs + 4 * t, Bc + 4 * t);
        } else {
#pragma unroll
            for (int i = 0; i < N; i++) cp_async4(bs + i, Bc + i);
        }
    };
    if (mvalid) {
        if (N % 4 == 0 && (lda & 3) == 0 && (reinterpret_cast<uintptr_t>(A) & 15) == 0) {
            for (int e = q; e < N * NC; e += LPM) {
                const int c = e % NC, j = e / NC;
                cp_async16(sm + 4 * c + j * NP, A + 4 * c + (long long)j * lda);
            }
        } else {
            for (int e = q; e < N * N; e += LPM) {
                const int i = e % N, j = e / N;
                cp_async4(sm + i + j * NP, A + i + (long long)j * lda);
            }
        }
        if (q < nrhs) stage_rhs(q);
        for (int k = q; k < N; k += LPM) {
            pv[k] = ipiv != nullptr ? ipiv[m * N + k] : k + 1;
            map[k] = k;
        }
    }
    __syncwarp();
    if (mvalid && q == 0 && ipiv != nullptr) {
        // The interchanges k = 0..n-1 applied to the identity row map.
        for (int k = 0; k < N; k++) {
            const int p = pv[k] - 1;
            if ((unsigned)p < (unsigned)N && p != k) {
                const int t = map[k];
                map[k] = map[p];
                map[p] = t;
            }
        }
    }
    cp_async_wait_all();
    __syncwarp();
    if (!mvalid) return;

    for (int c = q; c < nrhs; c += LPM) {
        float* Bc = B + (long long)c * ldb;
        if (c != q) {  // later right-hand sides of this lane (nrhs > LPM)
            stage_rhs(c);
            cp_async_wait_all();
        }
        float2 x2[NPAIR];
#pragma unroll
        for (int p = 0; p < NPAIR; p++) x2[p] = make_float2(0.0f, 0.0f);
        if (!TRANS) {
#pragma unroll
            for (int t = 0; t < NC; t++) {
                const int4 mp = reinterpret_cast<const int4*>(map)[t];
                if (4 * t + 0 < N) x2[2 * t].x = bs[mp.x];
                if (4 * t + 1 < N) x2[2 * t].y = bs[mp.y];
                if (4 * t + 2 < N) x2[2 * t + 1].x = bs[mp.z];
                if (4 * t + 3 < N) x2[2 * t + 1].y = bs[mp.w];
            }
            // unit-L forward: x[i] -= L[i][j] * x[j], i > j
#pragma unroll
            for (int j = 0; j < N - 1; j++) {
                const float xj = pget(x2, j);
                const float2 nx = make_float2(-xj, -xj);
                const float* lj = sm + j * NP;
#pragma unroll
                for (int t = j / 4; t < NC; t++) {
                    const float4 l4 = *reinterpret_cast<const float4*>(lj + 4 * t);
                    if (4 * t > j)
                        x2[2 * t] = __ffma2_rn(make_float2(l4.x, l4.y), nx, x2[2 * t]);
                    else if (4 * t + 1 > j)
                        x2[2 * t].y = fmaf(l4.y, -xj, x2[2 * t].y);
                    if (4 * t + 2 > j && 4 * t + 2 < N)
                        x2[2 * t + 1] = __ffma2_rn(make_float2(l4.z, l4.w), nx, x2[2 * t + 1]);
                    else if (4 * t + 3 > j && 4 * t + 3 < N)
                        x2[2 * t + 1].y = fmaf(l4.w, -xj, x2[2 * t + 1].y);
                }
            }
            // U backward: x[j] /= U[j][j]; x[i] -= U[i][j] * x[j], i < j
#pragma unroll
            for (int j = N - 1; j >= 0; j--) {
                const float* uj = sm + j * NP;
                const float4 dj = *reinterpret_cast<const float4*>(uj + 4 * (j / 4));
                const float xj = pget(x2, j) / f4get(dj, j % 4);
                pset(x2, j, xj);
                const float2 nx = make_float2(-xj, -xj);
#pragma unroll
                for (int t = 0; t <= j / 4; t++) {
                    const float4 u4 = (t == j / 4) ? dj : *reinterpret_cast<const float4*>(uj + 4 * t);
                    if (4 * t + 1 < j)
                        x2[2 * t] = __ffma2_rn(make_float2(u4.x, u4.y), nx, x2[2 * t]);
                    else if (4 * t < j)
                        x2[2 * t].x = fmaf(u4.x, -xj, x2[2 * t].x);
                    if (4 * t + 3 < j)
                        x2[2 * t + 1] = __ffma2_rn(make_float2(u4.z, u4.w), nx, x2[2 * t + 1]);
                    else if (4 * t + 2 < j)
                        x2[2 * t + 1].x = fmaf(u4.z, -xj, x2[2 * t + 1].x);
                }
            }
            if (bvec) {
#pragma unroll
                for (int t = 0; t < NC; t++)
                    *reinterpret_cast<float4*>(Bc + 4 * t) = make_float4(x2[2 * t].x, x2[2 * t].y, x2[2 * t + 1].x,
                                                                         x2[2 * t + 1].y);
            } else {
#pragma unroll
                for (int i = 0; i < N; i++) Bc[i] = pget(x2, i);
            }
        } else {
#pragma unroll
            for (int t = 0; t < NC; t++) {
                const float4 v = *reinterpret_cast<const float4*>(bs + 4 * t);
                x2[2 * t] = make_float2(v.x, v.y);
                x2[2 * t + 1] = make_float2(v.z, v.w);
            }
            // U^T forward: x[i] = (x[i] - sum_{j<i} U[j][i] x[j]) / U[i][i], j ascending
#pragma unroll
            for (int i = 0; i < N; i++) {
                const float* ui = sm + i * NP;
                float sacc = pget(x2, i);
#pragma unroll
                for (int t = 0; t <= i / 4; t++) {
                    const float4 u4 = *reinterpret_cast<const float4*>(ui + 4 * t);
#pragma unroll
                    for (int e = 0; e < 4; e++)
                        if (4 * t + e < i) sacc = fmaf(-f4get(u4, e), pget(x2, 4 * t + e), sacc);
                    if (t == i / 4) sacc = sacc / f4get(u4, i % 4);
                }
                pset(x2, i, sacc);
            }
            // L^T backward: x[j] -= sum_{i>j} L[i][j] x[i], i ascending
#pragma unroll
            for (int j = N - 2; j >= 0; j--) {
                const float* lj = sm + j * NP;
                float sacc = pget(x2, j);
#pragma unroll
                for (int t = j / 4; t < NC; t++) {
                    const float4 l4 = *reinterpret_cast<const float4*>(lj + 4 * t);
#pragma unroll
                    for (int e = 0; e < 4; e++)
                        if (4 * t + e > j && 4 * t + e < N) sacc = fmaf(-f4get(l4, e), pget(x2, 4 * t + e), sacc);
                }
                pset(x2, j, sacc);
            }
#pragma unroll
            for (int t = 0; t < NC; t++) {
                const int4 mp = reinterpret_cast<const int4*>(map)[t];
                if (4 * t + 0 < N) Bc[mp.x] = x2[2 * t].x;
                if (4 * t + 1 < N) Bc[mp.y] = x2[2 * t].y;
                if (4 * t + 2 < N) Bc[mp.z] = x2[2 * t + 1].x;
                if (4 * t + 3 < N) Bc[mp.w] = x2[2 * t + 1].y;
            }
        }
    }
}

template <int N, int LPM, bool TRANS>
inline void launch_getrs_rhs(cudaStream_t st, const float* const* Aarray, int lda, const int* ipiv,
                             float* const* Barray, int ldb, int nrhs, int batch)
{
    using R = RhsShape<N, LPM>;
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(getrs_rhs_kernel<N, LPM, TRANS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)R::SMEM);
        configured = true;
    }
    constexpr int per_cta = R::WARPS * R::MPW;
    const unsigned grid = (unsigned)((batch + per_cta - 1) / per_cta);
    getrs_rhs_kernel<N, LPM, TRANS><<<grid, R::WARPS * 32, R::SMEM, st>>>(Aarray, lda, ipiv, Barray, ldb, nrhs,
                                                                         batch);
}

template <int N, bool TRANS>
inline void launch_getrs_n(cudaStream_t st, const float* const* Aarray, int lda, const int* ipiv,
                           float* const* Barray, int ldb, int nrhs, int batch)
{
    if (!TRANS && nrhs == 1) {
        using S = SmallShape<N>;
        constexpr int per_cta = kSmallWarps * S::MPW;
        const unsigned grid = (unsigned)((batch + per_cta - 1) / per_cta);
        getrs_small_kernel<N><<<grid, kSmallWarps * 32, 0, st>>>(Aarray, lda, ipiv, Barray, ldb, batch);
    } else if (nrhs <= 4) {
        launch_getrs_rhs<N, 4, TRANS>(st, Aarray, lda, ipiv, Barray, ldb, nrhs, batch);
    } else {
        launch_getrs_rhs<N, 32, TRANS>(st, Aarray, lda, ipiv, Barray, ldb, nrhs, batch);
    }
}

// One translation unit per transpose instantiates the 32 sizes (getrs_small_n.cu, _t.cu).
void getrs_small_dispatch_n(int n, cudaStream_t st, const float* const* Aarray, int lda, const int* ipiv,
                            float* const* Barray, int ldb, int nrhs, int batch);
void getrs_small_dispatch_t(int n, cudaStream_t st, const float* const* Aarray, int lda, const int* ipiv,
                            float* const* Barray, int ldb, int nrhs, int batch);

}  // namespace opsblas
