// aclblasSgetrfBatched for 32 < n <= 128: one CTA per matrix, matrix resident in shared memory,
// blocked right-looking LU that keeps the reference's per-element arithmetic.
//
// The reference factors column by column (sgetrf_batched_kernel.cpp:106-150): each element
// a(i,j) receives a(i,j) -= l(i,m) * u(m,j) for m = 0, 1, ... in order, multipliers are formed
// by true division, and rows are swapped whole. This kernel reorganises the same arithmetic
// into panels of PB columns so that most of it runs as a register-tiled update:
//   1. panel: one warp factors columns k0..k0+PB-1 of the rows k0..n-1, up to 4 rows per lane
//      in registers, first-maximum pivots by redux.sync, multipliers by division;
//   2. U12: rows k0..k0+PB-1 right of the panel, forward substitution with the panel's unit
//      L11 in order m = 0..PB-1 (what the reference's rank-1 updates do to those rows);
//   3. A22 -= L21 * U12 with 4x4 register tiles whose accumulators start from A22 and add
//      the PB products in order -- one fmaf per product, exactly the reference sequence.
// Rows never move in shared memory: pivoting only updates a logical-to-physical row map,
// which the final store applies. On an exactly-zero pivot at column k the panel's columns
// before k are still applied to the trailing columns (steps 2-3 with a narrower panel), so a
// singular matrix ends in the reference's state too.
#include <cuda_runtime.h>

#include "internal.h"
#include "small_common.cuh"

namespace opsblas {

constexpr int kMedThreads = 128;   // 4 warps
constexpr int kMedPB = 16;         // panel width
constexpr int kMedMaxN = 128;
constexpr int kMedRows = kMedMaxN / 32;  // panel rows per lane

struct MedLayout {
    int ld;       // column stride of the resident matrix (odd: conflict-free row access)
    int ls_ld;    // row stride of the staged L21 / U12 blocks (multiple of 4)
    int mat;      // floats reserved for the matrix (multiple of 4: 16-byte aligned staging)
    size_t bytes;
    __host__ __device__ MedLayout(int n)
    {
        ld = n | 1;
        ls_ld = (n + 3) & ~3;
        mat = (ld * n + 3) & ~3;
        bytes = (size_t)mat * 4                  // matrix
                + (size_t)2 * kMedPB * ls_ld * 4  // staged L21 (transposed) and U12
                + (size_t)n * 4                   // row map
                + (size_t)2 * 32 * 4              // pivot row broadcast (double buffered)
                + 64;                             // scalars
    }
};

template <bool PIVOT>
__global__ void __launch_bounds__(kMedThreads)
getrf_medium_kernel(float* const* __restrict__ Aarray, int n, int lda, int* __restrict__ piv, int* __restrict__ info)
{
    extern __shared__ __align__(16) float smem[];
    const MedLayout L(n);
    const int ld = L.ld, lsd = L.ls_ld;
    float* sa = smem;                                  // resident matrix, column-major, ld
    float* l21 = sa + L.mat;                           // [PB][lsd]: l21[m*lsd + i'] = L(r0+i', k0+m)
    float* u12 = l21 + kMedPB * lsd;                   // [PB][lsd]: u12[m*lsd + j'] = U(k0+m, j0+j')
    int* rmap = reinterpret_cast<int*>(u12 + kMedPB * lsd);  // logical row -> physical row
    float* prow = reinterpret_cast<float*>(rmap + n);        // 2 x 32 floats
    int* sc = reinterpret_cast<int*>(prow + 64);             // scalars: [0] info, [1] panel width done

    const long long m = blockIdx.x;
    float* A = Aarray[m];
    int* pm = PIVOT ? piv + m * n : nullptr;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    for (int e = tid; e < n * n; e += kMedThreads) {
        const int i = e % n, j = e / n;
        sa[i + j * ld] = A[i + (long long)j * lda];
    }
    for (int i = tid; i < n; i += kMedThreads) rmap[i] = i;
    if (PIVOT)
        for (int i = tid; i < n; i += kMedThreads) pm[i] = 0;
    if (tid == 0) sc[0] = 0;
    __syncthreads();

    for (int k0 = 0; k0 < n; k0 += kMedPB) {
        const int pb = min(kMedPB, n - k0);
        // ---------------------------------------------------------------- 1. panel --
        if (warp == 0) {
            float pr[kMedRows][kMedPB];
            int pos[kMedRows], phys[kMedRows];
#pragma unroll
            for (int t = 0; t < kMedRows; t++) {
                const int i = k0 + lane + 32 * t;
                pos[t] = i;
                phys[t] = i < n ? rmap[i] : 0;
#pragma unroll
                for (int c = 0; c < kMedPB; c++) pr[t][c] = (i < n && c < pb) ? sa[phys[t] + (k0 + c) * ld] : 0.0f;
            }
            int done = pb;
            int inf = 0;
#pragma unroll
            for (int c = 0; c < kMedPB; c++) {
                if (c >= pb) break;
                const int k = k0 + c;
                float* buf = prow + 32 * (c & 1);
                int ppos = k;
                if (PIVOT) {
                    // lane-local first maximum (ties to the lowest logical row), then warp-wide
                    unsigned bkey = 0, bpos = 0xffffffffu;
#pragma unroll
                    for (int t = 0; t < kMedRows; t++) {
                        const bool elig = pos[t] < n && pos[t] >= k;
                        const float v = fabsf(pr[t][c]);
                        const unsigned key = (elig && v > 0.0f) ? __float_as_uint(v) : 0u;
                        if (elig && (key > bkey || (key == bkey && (unsigned)pos[t] < bpos))) {
                            bkey = key;
                            bpos = (unsigned)pos[t];
                        }
                    }
                    ppos = (int)seg_argmax<32>(bkey, bpos, 0);
                }
                // the pivot row's owner publishes it
#pragma unroll
                for (int t = 0; t < kMedRows; t++) {
                    if (pos[t] == ppos) {
#pragma unroll
                        for (int cc = 0; cc < kMedPB; cc++) buf[cc] = pr[t][cc];
                    }
                }
                __syncwarp();
                const float pv = buf[c];
                if (PIVOT && lane == 0) pm[k] = ppos + 1;
                if (pv == 0.0f) {
                    inf = k + 1;
                    done = c;
                    break;
                }
#pragma unroll
                for (int t = 0; t < kMedRows; t++) {
                    if (pos[t] == ppos)
                        pos[t] = k;
                    else if (pos[t] == k)
                        pos[t] = ppos;
                }
#pragma unroll
                for (int t = 0; t < kMedRows; t++) {
                    if (pos[t] < n && pos[t] > k) {
                        const float l = pr[t][c] / pv;
                        pr[t][c] = l;
#pragma unroll
                        for (int cc = c + 1; cc < kMedPB; cc++) pr[t][cc] = fmaf(-l, buf[cc], pr[t][cc]);
                    }
                }
            }
            // write the panel back in place, record the new logical order
#pragma unroll
            for (int t = 0; t < kMedRows; t++) {
                if (k0 + lane + 32 * t < n) {
#pragma unroll
                    for (int c = 0; c < kMedPB; c++)
                        if (c < pb) sa[phys[t] + (k0 + c) * ld] = pr[t][c];
                }
            }
            __syncwarp();
#pragma unroll
            for (int t = 0; t < kMedRows; t++)
                if (k0 + lane + 32 * t < n) rmap[pos[t]] = phys[t];
            if (lane == 0) {
                sc[0] = inf;
                sc[1] = done;
            }
        }
        __syncthreads();
        const int w = sc[1];   // panel columns to apply (pb, or fewer after a zero pivot)
        const int j0 = k0 + pb;  // first column right of the panel
        const int r0 = k0 + w;   // first row of the trailing block
        const int rest = n - j0;
        if (w > 0 && rest > 0) {
            // ------------------------------------------------ 2. U12 (+ staging) --
            for (int jj = tid; jj < rest; jj += kMedThreads) {
                const int j = j0 + jj;
                float u[kMedPB];
#pragma unroll
                for (int r = 0; r < kMedPB; r++) u[r] = r < w ? sa[rmap[k0 + r] + j * ld] : 0.0f;
#pragma unroll
                for (int mm = 0; mm < kMedPB; mm++) {
                    if (mm < w) {
#pragma unroll
                        for (int r = mm + 1; r < kMedPB; r++)
                            if (r < w) u[r] = fmaf(-sa[rmap[k0 + r] + (k0 + mm) * ld], u[mm], u[r]);
                    }
                }
#pragma unroll
                for (int r = 0; r < kMedPB; r++) {
                    if (r < w) {
                        sa[rmap[k0 + r] + j * ld] = u[r];
                        u12[r * lsd + jj] = u[r];
                    }
                }
            }
            const int rows = n - r0;  // rows below the applied panel columns
            for (int e = tid; e < rows * w; e += kMedThreads) {
                const int ii = e % rows, mm = e / rows;
                l21[mm * lsd + ii] = sa[rmap[r0 + ii] + (k0 + mm) * ld];
            }
            __syncthreads();
            // ------------------------------------------- 3. A22 -= L21 * U12 --
            const int tr = (rows + 3) / 4, tc = (rest + 3) / 4;
            for (int tile = tid; tile < tr * tc; tile += kMedThreads) {
                const int bi = (tile % tr) * 4, bj = (tile / tr) * 4;
                float acc[4][4];
                int pr4[4];
#pragma unroll
                for (int a = 0; a < 4; a++) pr4[a] = (bi + a < rows) ? rmap[r0 + bi + a] : -1;
#pragma unroll
                for (int a = 0; a < 4; a++)
#pragma unroll
                    for (int b = 0; b < 4; b++)
                        acc[a][b] = (pr4[a] >= 0 && bj + b < rest) ? sa[pr4[a] + (j0 + bj + b) * ld] : 0.0f;
                for (int mm = 0; mm < w; mm++) {
                    const float4 lv = *reinterpret_cast<const float4*>(l21 + mm * lsd + bi);
                    const float4 uv = *reinterpret_cast<const float4*>(u12 + mm * lsd + bj);
                    const float la[4] = {-lv.x, -lv.y, -lv.z, -lv.w};
                    const float ub[4] = {uv.x, uv.y, uv.z, uv.w};
#pragma unroll
                    for (int a = 0; a < 4; a++)
#pragma unroll
                        for (int b = 0; b < 4; b++) acc[a][b] = fmaf(la[a], ub[b], acc[a][b]);
                }
#pragma unroll
                for (int a = 0; a < 4; a++)
#pragma unroll
                    for (int b = 0; b < 4; b++)
                        if (pr4[a] >= 0 && bj + b < rest) sa[pr4[a] + (j0 + bj + b) * ld] = acc[a][b];
            }
        }
        __syncthreads();
        if (sc[0] != 0) break;
    }

    // store: logical row i of the result is physical row rmap[i]
    for (int e = tid; e < n * n; e += kMedThreads) {
        const int i = e % n, j = e / n;
        A[i + (long long)j * lda] = sa[rmap[i] + j * ld];
    }
    if (tid == 0 && info != nullptr) info[m] = sc[0];
}

bool getrf_medium_supported(int n) { return n > 32 && n <= kMedMaxN; }

cudaError_t getrf_medium_launch(cudaStream_t st, float* const* Aarray, int n, int lda, int* piv, int* info,
                                int batch)
{
    const MedLayout L(n);
    static bool configured = false;
    if (!configured) {
        const MedLayout big(kMedMaxN);
        cudaFuncSetAttribute(getrf_medium_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)big.bytes);
        cudaFuncSetAttribute(getrf_medium_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)big.bytes);
        configured = true;
    }
    if (piv)
        getrf_medium_kernel<true><<<(unsigned)batch, kMedThreads, L.bytes, st>>>(Aarray, n, lda, piv, info);
    else
        getrf_medium_kernel<false><<<(unsigned)batch, kMedThreads, L.bytes, st>>>(Aarray, n, lda, nullptr, info);
    return cudaGetLastError();
}

}  // namespace opsblas
