// aclblasSgetrfBatched for 128 < n <= 1024 and the mixed-precision factorisation: one CTA per
// matrix, blocked right-looking LU with the matrix in global memory (L2 resident per CTA).
//
// Per panel of PB columns:
//   1. the panel (rows k0..n-1) is staged in shared memory and factored by the whole CTA:
//      first-maximum pivot search (per warp, then across warps), physical row swap inside
//      the panel, multipliers by true division, rank-1 update of the remaining panel columns;
//   2. the panel's interchanges are applied to the columns left and right of the panel
//      (whole-row swaps, as the reference's SwapRows, sgetrf_batched_kernel.cpp:81-91);
//   3. U12 (panel rows, right of the panel) by forward substitution with the unit L11;
//   4. A22 -= L21 * U12 with 4x4 register tiles.
// In the plain mode every element receives its updates one fmaf at a time in increasing
// column order -- the reference's operation sequence, so results match it bit for bit. In the
// mixed modes the L21 / U12 operands of step 4 (the dense trailing update, ~90% of the flops)
// are split into a high and a low part of reduced precision (TF32 or BF16, x = hi + lo) and
// the update accumulates hi*hi + hi*lo + lo*hi in FP32 -- the error-compensated three-product
// scheme, which keeps the factorisation close to FP32 accuracy so that iterative refinement
// converges for condition numbers up to ~1e6; the panel and U12 stay FP32.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "internal.h"
#include "small_common.cuh"

namespace opsblas {

constexpr int kLgThreads = 256;
constexpr int kLgWarps = kLgThreads / 32;
constexpr int kLgPB = 16;
constexpr int kLgMaxN = 640;  // mixed-mode staging keeps shared memory under 227 KiB
constexpr int kLgPS = kLgPB + 1;  // panel row stride in shared memory (odd: conflict-free)

__device__ __forceinline__ float lg_round(float x, int mode)
{
    if (mode == 1) {  // TF32: keep 10 mantissa bits, round to nearest even
        unsigned u = __float_as_uint(x);
        if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x0fffu + ((u >> 13) & 1u)) & 0xffffe000u;
        return __uint_as_float(u);
    }
    if (mode == 2) return __bfloat162float(__float2bfloat16_rn(x));
    return x;
}

struct LgLayout {
    int lsd;
    size_t bytes;
    __host__ __device__ LgLayout(int n, int mode = 0)
    {
        lsd = (n + 3) & ~3;
        bytes = (size_t)n * kLgPS * 4                        // panel
                + (size_t)(mode ? 4 : 2) * kLgPB * lsd * 4     // staged L21 (transposed) and U12 (+ low parts)
                + (size_t)kLgPB * 2 * 4           // recorded interchanges
                + (size_t)kLgWarps * 2 * 4 + 64;  // per-warp argmax, scalars
    }
};

template <bool PIVOT, int MODE>
__global__ void __launch_bounds__(kLgThreads)
getrf_large_kernel(float* const* __restrict__ Aarray, int n, int lda, int* __restrict__ piv, int* __restrict__ info)
{
    extern __shared__ __align__(16) float smem[];
    const LgLayout L(n, MODE);
    const int lsd = L.lsd;
    float* l21 = smem;                           // [PB][lsd] (negated)
    float* u12 = l21 + kLgPB * lsd;              // [PB][lsd]
    float* l21lo = MODE ? u12 + kLgPB * lsd : nullptr;     // low parts (mixed modes)
    float* u12lo = MODE ? l21lo + kLgPB * lsd : nullptr;
    float* pb_s = u12 + (MODE ? 3 : 1) * kLgPB * lsd;  // [n][PS]: panel row i-k0 at pb_s[(i-k0)*PS]
    int* swaps = reinterpret_cast<int*>(pb_s + (size_t)n * kLgPS);  // [PB] pivot rows (logical)
    float* wv = reinterpret_cast<float*>(swaps + 2 * kLgPB);          // per-warp best value
    int* wr = reinterpret_cast<int*>(wv + kLgWarps);                  // per-warp best row
    int* sc = wr + kLgWarps;                                          // [0] info [1] width [2] pivot row

    const long long mi = blockIdx.x;
    float* A = Aarray[mi];
    int* pm = PIVOT ? piv + mi * n : nullptr;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    auto at = [&](int i, int j) -> float& { return A[i + (long long)j * lda]; };

    if (PIVOT)
        for (int i = tid; i < n; i += kLgThreads) pm[i] = 0;
    if (tid == 0) sc[0] = 0;

    for (int k0 = 0; k0 < n; k0 += kLgPB) {
        const int pb = min(kLgPB, n - k0);
        const int prows = n - k0;
        // ----------------------------------------------------------- 1. panel --
        for (int e = tid; e < prows * pb; e += kLgThreads) {
            const int ii = e % prows, c = e / prows;
            pb_s[ii * kLgPS + c] = at(k0 + ii, k0 + c);
        }
        __syncthreads();
        int w = pb;
        for (int c = 0; c < pb; c++) {
            const int k = k0 + c;
            int p = k;
            if (PIVOT) {
                float best = 0.0f;
                int brow = k;
                for (int i = k + tid; i < n; i += kLgThreads) {
                    const float v = fabsf(pb_s[(i - k0) * kLgPS + c]);
                    if (v > best) {
                        best = v;
                        brow = i;
                    }
                }
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    const float ob = __shfl_xor_sync(0xffffffffu, best, off);
                    const int orow = __shfl_xor_sync(0xffffffffu, brow, off);
                    if (ob > best || (ob == best && orow < brow)) {
                        best = ob;
                        brow = orow;
                    }
                }
                if (lane == 0) {
                    wv[warp] = best;
                    wr[warp] = brow;
                }
                __syncthreads();
                if (tid == 0) {
                    float b = wv[0];
                    int r = wr[0];
                    for (int q = 1; q < kLgWarps; q++)
                        if (wv[q] > b || (wv[q] == b && wr[q] < r)) {
                            b = wv[q];
                            r = wr[q];
                        }
                    sc[2] = r;
                }
                __syncthreads();
                p = sc[2];
            }
            const float pv = pb_s[(p - k0) * kLgPS + c];
            if (tid == 0) {
                if (PIVOT) pm[k] = p + 1;
                swaps[c] = p;
            }
            if (pv == 0.0f) {  // uniform: every thread read the same value
                if (tid == 0) sc[0] = k + 1;
                w = c;
                break;
            }
            __syncthreads();  // every thread has read pv before the pivot row moves
            if (p != k && tid < kLgPB) {
                const float t = pb_s[(k - k0) * kLgPS + tid];
                pb_s[(k - k0) * kLgPS + tid] = pb_s[(p - k0) * kLgPS + tid];
                pb_s[(p - k0) * kLgPS + tid] = t;
            }
            __syncthreads();
            for (int i = k + 1 + tid; i < n; i += kLgThreads) {
                float* row = pb_s + (i - k0) * kLgPS;
                const float* prow = pb_s + (k - k0) * kLgPS;
                const float l = row[c] / pv;
                row[c] = l;
                for (int cc = c + 1; cc < pb; cc++) row[cc] = fmaf(-l, prow[cc], row[cc]);
            }
            __syncthreads();
        }
        // panel back to global memory (rows in their swapped order)
        for (int e = tid; e < prows * pb; e += kLgThreads) {
            const int ii = e % prows, c = e / prows;
            at(k0 + ii, k0 + c) = pb_s[ii * kLgPS + c];
        }
        // -------------------------------------- 2. interchanges outside the panel --
        const int nsw = (w < pb) ? w + 1 : pb;  // a zero pivot records its row but does not swap
        for (int c = 0; c < w; c++) {
            const int k = k0 + c, p = swaps[c];
            if (p != k) {
                for (int j = tid; j < n; j += kLgThreads) {
                    if (j >= k0 && j < k0 + pb) continue;
                    const float t = at(k, j);
                    at(k, j) = at(p, j);
                    at(p, j) = t;
                }
            }
            __syncthreads();
        }
        (void)nsw;
        const int j0 = k0 + pb, r0 = k0 + w, rest = n - j0, rows = n - r0;
        if (w > 0 && rest > 0) {
            // ------------------------------------------------------- 3. U12 --
            for (int jj = tid; jj < rest; jj += kLgThreads) {
                const int j = j0 + jj;
                float u[kLgPB];
#pragma unroll
                for (int r = 0; r < kLgPB; r++) u[r] = r < w ? at(k0 + r, j) : 0.0f;
#pragma unroll
                for (int mm = 0; mm < kLgPB; mm++) {
                    if (mm < w) {
#pragma unroll
                        for (int r = mm + 1; r < kLgPB; r++)
                            if (r < w) u[r] = fmaf(-pb_s[r * kLgPS + mm], u[mm], u[r]);
                    }
                }
#pragma unroll
                for (int r = 0; r < kLgPB; r++) {
                    if (r < w) {
                        at(k0 + r, j) = u[r];
                        const float hi = lg_round(u[r], MODE);
                        u12[r * lsd + jj] = hi;
                        if (MODE) u12lo[r * lsd + jj] = lg_round(u[r] - hi, MODE);
                    }
                }
            }
            for (int e = tid; e < rows * w; e += kLgThreads) {
                const int ii = e % rows, mm = e / rows;
                const float v = pb_s[(r0 - k0 + ii) * kLgPS + mm];
                const float hi = lg_round(v, MODE);
                l21[mm * lsd + ii] = -hi;
                if (MODE) l21lo[mm * lsd + ii] = -lg_round(v - hi, MODE);
            }
            __syncthreads();
            // ------------------------------------------- 4. A22 -= L21 * U12 --
            const int tr = (rows + 3) / 4, tc = (rest + 3) / 4;
            const bool vec = ((lda & 3) == 0) && ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && ((r0 & 3) == 0);
            for (int tile = tid; tile < tr * tc; tile += kLgThreads) {
                const int bi = (tile % tr) * 4, bj = (tile / tr) * 4;
                const int gi = r0 + bi;
                float acc[4][4];
                const bool full = vec && bi + 4 <= rows;
#pragma unroll
                for (int b = 0; b < 4; b++) {
                    const int gj = j0 + bj + b;
                    if (gj < n && full) {
                        const float4 v = *reinterpret_cast<const float4*>(&at(gi, gj));
                        acc[0][b] = v.x;
                        acc[1][b] = v.y;
                        acc[2][b] = v.z;
                        acc[3][b] = v.w;
                    } else {
#pragma unroll
                        for (int a = 0; a < 4; a++) acc[a][b] = (gj < n && bi + a < rows) ? at(gi + a, gj) : 0.0f;
                    }
                }
                for (int mm = 0; mm < w; mm++) {
                    const float4 lv = *reinterpret_cast<const float4*>(l21 + mm * lsd + bi);
                    const float4 uv = *reinterpret_cast<const float4*>(u12 + mm * lsd + bj);
                    const float la[4] = {lv.x, lv.y, lv.z, lv.w};
                    const float ub[4] = {uv.x, uv.y, uv.z, uv.w};
                    if (MODE) {
                        // small terms first: hi*lo + lo*hi, then hi*hi
                        const float4 lw = *reinterpret_cast<const float4*>(l21lo + mm * lsd + bi);
                        const float4 uw = *reinterpret_cast<const float4*>(u12lo + mm * lsd + bj);
                        const float ll[4] = {lw.x, lw.y, lw.z, lw.w};
                        const float ul[4] = {uw.x, uw.y, uw.z, uw.w};
                        float t[4][4];
#pragma unroll
                        for (int a = 0; a < 4; a++)
#pragma unroll
                            for (int b = 0; b < 4; b++) t[a][b] = fmaf(la[a], ul[b], ll[a] * ub[b]);
#pragma unroll
                        for (int a = 0; a < 4; a++)
#pragma unroll
                            for (int b = 0; b < 4; b++) acc[a][b] = fmaf(la[a], ub[b], acc[a][b] + t[a][b]);
                    } else {
#pragma unroll
                        for (int a = 0; a < 4; a++)
#pragma unroll
                            for (int b = 0; b < 4; b++) acc[a][b] = fmaf(la[a], ub[b], acc[a][b]);
                    }
                }
#pragma unroll
                for (int b = 0; b < 4; b++) {
                    const int gj = j0 + bj + b;
                    if (gj >= n) continue;
                    if (full) {
                        *reinterpret_cast<float4*>(&at(gi, gj)) = make_float4(acc[0][b], acc[1][b], acc[2][b], acc[3][b]);
                    } else {
#pragma unroll
                        for (int a = 0; a < 4; a++)
                            if (bi + a < rows) at(gi + a, gj) = acc[a][b];
                    }
                }
            }
        }
        __syncthreads();
        if (sc[0] != 0) break;
    }
    if (tid == 0 && info != nullptr) info[mi] = sc[0];
}

bool getrf_large_supported(int n) { return n > 32 && n <= kLgMaxN; }

cudaError_t getrf_large_launch(cudaStream_t st, float* const* Aarray, int n, int lda, int* piv, int* info, int batch,
                               int mode)
{
    const LgLayout L(n, piv ? mode : 0);
    static bool configured = false;
    if (!configured) {
        const int big = (int)LgLayout(kLgMaxN, 1).bytes;
        cudaFuncSetAttribute(getrf_large_kernel<true, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(getrf_large_kernel<false, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(getrf_large_kernel<true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(getrf_large_kernel<true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        configured = true;
    }
    const unsigned grid = (unsigned)batch;
    if (piv == nullptr) {
        getrf_large_kernel<false, 0><<<grid, kLgThreads, L.bytes, st>>>(Aarray, n, lda, nullptr, info);
    } else if (mode == 1) {
        getrf_large_kernel<true, 1><<<grid, kLgThreads, L.bytes, st>>>(Aarray, n, lda, piv, info);
    } else if (mode == 2) {
        getrf_large_kernel<true, 2><<<grid, kLgThreads, L.bytes, st>>>(Aarray, n, lda, piv, info);
    } else {
        getrf_large_kernel<true, 0><<<grid, kLgThreads, L.bytes, st>>>(Aarray, n, lda, piv, info);
    }
    return cudaGetLastError();
}

}  // namespace opsblas
