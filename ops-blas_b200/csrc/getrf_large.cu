// aclblasSgetrfBatched for 128 < n <= 640: one CTA per matrix, blocked right-looking LU with the
// matrix in global memory (L2 resident per CTA).
//
// Per panel of PB columns:
//   1. the panel (rows k0..n-1) is staged in shared memory and factored by the whole CTA:
//      first-maximum pivot search (per warp, then across warps), physical row swap inside
//      the panel, multipliers by true division, rank-1 update of the remaining panel columns;
//   2. the panel's interchanges are applied to the columns left and right of the panel
//      (whole-row swaps, as the reference's SwapRows, sgetrf_batched_kernel.cpp:81-91);
//   3. U12 (panel rows, right of the panel) by forward substitution with the unit L11;
//   4. A22 -= L21 * U12 with 4x4 register tiles.
// Every element receives its updates one fmaf at a time in increasing column order -- the
// reference's operation sequence, so results match it bit for bit. (A variant that split the
// step-4 operands into TF32 / BF16 high and low parts on the CUDA cores was measured slower than
// this plain kernel at n = 512 and removed; the mixed modes use the tensor-memory kernel up to
// n = 256 and these plain factors above.)
#include <cuda_runtime.h>

#include "internal.h"
#include "small_common.cuh"

namespace opsblas {

constexpr int kLgThreads = 256;
constexpr int kLgWarps = kLgThreads / 32;
constexpr int kLgPB = 16;
constexpr int kLgMaxN = 640;
constexpr int kLgPS = kLgPB + 1;  // panel row stride in shared memory (odd: conflict-free)

struct LgLayout {
    int lsd;
    size_t bytes;
    __host__ __device__ explicit LgLayout(int n)
    {
        lsd = (n + 3) & ~3;
        bytes = (size_t)n * kLgPS * 4             // panel
                + (size_t)2 * kLgPB * lsd * 4     // staged L21 (transposed) and U12
                + (size_t)kLgPB * 2 * 4           // recorded interchanges
                + (size_t)kLgWarps * 2 * 4 + 64;  // per-warp argmax, scalars
    }
};

template <bool PIVOT>
__global__ void __launch_bounds__(kLgThreads)
getrf_large_kernel(float* const* __restrict__ Aarray, int n, int lda, int* __restrict__ piv, int* __restrict__ info)
{
    extern __shared__ __align__(16) float smem[];
    const LgLayout L(n);
    const int lsd = L.lsd;
    float* l21 = smem;                           // [PB][lsd] (negated)
    float* u12 = l21 + kLgPB * lsd;              // [PB][lsd]
    float* pb_s = u12 + kLgPB * lsd;             // [n][PS]: panel row i-k0 at pb_s[(i-k0)*PS]
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
                        u12[r * lsd + jj] = u[r];
                    }
                }
            }
            for (int e = tid; e < rows * w; e += kLgThreads) {
                const int ii = e % rows, mm = e / rows;
                l21[mm * lsd + ii] = -pb_s[(r0 - k0 + ii) * kLgPS + mm];
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
#pragma unroll
                    for (int a = 0; a < 4; a++)
#pragma unroll
                        for (int b = 0; b < 4; b++) acc[a][b] = fmaf(la[a], ub[b], acc[a][b]);
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

cudaError_t getrf_large_launch(cudaStream_t st, float* const* Aarray, int n, int lda, int* piv, int* info, int batch)
{
    const LgLayout L(n);
    const int big = (int)LgLayout(kLgMaxN).bytes;
    const cudaError_t e = piv == nullptr ? ensure_smem_limit(getrf_large_kernel<false>, big)
                                         : ensure_smem_limit(getrf_large_kernel<true>, big);
    if (e != cudaSuccess) return e;
    const unsigned grid = (unsigned)batch;
    if (piv == nullptr)
        getrf_large_kernel<false><<<grid, kLgThreads, L.bytes, st>>>(Aarray, n, lda, nullptr, info);
    else
        getrf_large_kernel<true><<<grid, kLgThreads, L.bytes, st>>>(Aarray, n, lda, piv, info);
    return cudaGetLastError();
}

}  // namespace opsblas
