// aclblasSgetrsBatched, trans N, n > 32: one CTA per matrix, blocked substitution with the
// right-hand sides resident in shared memory.
//
// The reference solve (sgetrs_batched_kernel.cpp:83-200) is laswp, then the unit-L forward sweep
// x_i -= L(i,j) x_j for j = 0..n-1, then the U backward sweep x_j /= U(j,j), x_i -= U(i,j) x_j
// for j = n-1..0. Every element x_i receives its updates in j order, so the sweeps can be blocked
// by 32 rows without changing a bit:
//   * interchanges: the swap sequence is applied to an index array once, then B is gathered;
//   * forward, per 32-row block: the diagonal block is solved by warps (one right-hand side per
//     warp at a time, lane = row, shuffles), then every row below subtracts the block's
//     contributions in j order (one thread per row, 16 right-hand sides in registers);
//   * backward, per block from the bottom: diagonal solve with true division, then the rows above
//     subtract the block's contributions in descending j order.
// Right-hand sides are processed 16 at a time.
#include <cuda_runtime.h>

#include "internal.h"
#include "small_common.cuh"

namespace opsblas {

constexpr int kBsThreads = 256;
constexpr int kBsRC = 16;  // right-hand sides per pass
constexpr int kBsB = 32;   // block rows
constexpr int kBsLd = 36;  // row stride of a staged diagonal block (16-byte rows for cp.async)

// xs, two diagonal-block buffers, perm and pivots
size_t getrs_blk_smem(int n) { return (size_t)n * kBsRC * 4 + 2 * kBsB * kBsLd * 4 + (size_t)n * 4 * 2 + 16; }

__global__ void __launch_bounds__(kBsThreads)
getrs_blk_kernel(const float* const* __restrict__ Aarray, int n, int lda, const int* __restrict__ ipiv,
                 float* const* __restrict__ Barray, int ldb, int nrhs)
{
    extern __shared__ __align__(16) float sm[];
    float* xs = sm;                                              // [n][kBsRC]
    float* blks = xs + (size_t)n * kBsRC;                        // 2 x [kBsB][kBsLd]: blk[j * kBsLd + i]
    int* perm = reinterpret_cast<int*>(blks + 2 * kBsB * kBsLd);  // [n]: source row of position i
    int* pv = perm + n;                                      // [n]: pivots
    const long long m = blockIdx.x;
    float* B = Barray[m];
    if (B == nullptr) return;  // a NULL right-hand side skips the matrix
    const float* A = Aarray[m];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    auto at = [&](int i, int j) { return A[i + (long long)j * lda]; };
    const bool vec = (reinterpret_cast<uintptr_t>(A) & 15) == 0 && (lda & 3) == 0;
    // the diagonal block at (r0, r0) into buffer `buf`: by cp.async (one 16-byte copy a thread)
    // when the matrix is 16-byte aligned and the block whole, else element-wise; the caller
    // waits (cp_async_wait_all) and syncs before reading it
    auto stage_blk = [&](int r0, int buf) {
        float* blk = blks + buf * kBsB * kBsLd;
        const int bs = min(kBsB, n - r0);
        if (vec && bs == kBsB) {
            const int j = tid >> 3, iq = (tid & 7) * 4;  // 256 threads = 32 columns x 8 quads
            cp_async16(blk + j * kBsLd + iq, A + (r0 + iq) + (long long)(r0 + j) * lda);
            cp_async_commit();
        } else {
            for (int e = tid; e < kBsB * kBsB; e += kBsThreads) {
                const int j = e / kBsB, i = e % kBsB;
                blk[j * kBsLd + i] = (i < bs && j < bs) ? at(r0 + i, r0 + j) : 0.0f;
            }
        }
    };

    // ---- interchanges (sgetrs_batched_kernel.cpp:94-100: out-of-range or zero pivots skipped) ----
    for (int i = tid; i < n; i += kBsThreads) pv[i] = ipiv ? ipiv[m * n + i] - 1 : i;
    __syncthreads();
    // perm[i] = the row that the swap sequence k = 0..n-1 brings to position i: i traced back
    // through the swaps in reverse order, every position in parallel (instead of one thread
    // applying the n swaps in turn)
    for (int i = tid; i < n; i += kBsThreads) {
        int x = i;
#pragma unroll 8
        for (int k = n - 1; k >= 0; k--) {
            const int p = pv[k];
            const bool sw = (unsigned)p < (unsigned)n && p != k;
            x = (sw && x == k) ? p : ((sw && x == p) ? k : x);
        }
        perm[i] = x;
    }
    __syncthreads();

    for (int c0 = 0; c0 < nrhs; c0 += kBsRC) {
        const int cw = min(kBsRC, nrhs - c0);
        // B gathered through the interchanges, eight loads in flight before their stores
        for (int base = tid; base < n * kBsRC; base += 8 * kBsThreads) {
            float v[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int e = base + u * kBsThreads, i = e % n, c = e / n;
                v[u] = (e < n * kBsRC && c < cw) ? B[perm[i] + (long long)(c0 + c) * ldb] : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int e = base + u * kBsThreads;
                if (e < n * kBsRC) xs[(e % n) * kBsRC + e / n] = v[u];
            }
        }
        __syncthreads();

        // ------------------------------------------------------------ forward, unit L --
        // the next block's diagonal is staged while the rows below the current one update
        stage_blk(0, 0);
        for (int r0 = 0, bi = 0; r0 < n; r0 += kBsB, bi ^= 1) {
            const int bs = min(kBsB, n - r0);
            const float* blk = blks + bi * kBsB * kBsLd;
            cp_async_wait_all();
            __syncthreads();
            if (bs == kBsB) {
                // a whole block: warp 0 alone, lane = right-hand side, the block's 32 unknowns in
                // registers, x_i -= L(i,j) x_j for j < i in turn (each element's updates in j order,
                // as the shuffle form below); a third of the instructions of that form
                if (warp == 0 && lane < cw) {
                    float x[kBsB];
#pragma unroll
                    for (int i = 0; i < kBsB; i++) x[i] = xs[(r0 + i) * kBsRC + lane];
#pragma unroll
                    for (int i = 1; i < kBsB; i++)
#pragma unroll
                        for (int j = 0; j < kBsB; j++)
                            if (j < i) x[i] = fmaf(-blk[j * kBsLd + i], x[j], x[i]);
#pragma unroll
                    for (int i = 0; i < kBsB; i++) xs[(r0 + i) * kBsRC + lane] = x[i];
                }
            } else {
            // two right-hand sides per warp, their dependency chains interleaved
            for (int c = warp; c < cw; c += 2 * (kBsThreads / 32)) {
                const int c1 = c + kBsThreads / 32;
                const bool two = c1 < cw;
                float y0 = lane < bs ? xs[(r0 + lane) * kBsRC + c] : 0.0f;
                float y1 = (two && lane < bs) ? xs[(r0 + lane) * kBsRC + c1] : 0.0f;
                if (two) {
                    for (int j = 0; j < bs; j++) {
                        const float l = -blk[j * kBsLd + lane];
                        const float yj0 = __shfl_sync(0xffffffffu, y0, j);
                        const float yj1 = __shfl_sync(0xffffffffu, y1, j);
                        if (lane > j && lane < bs) {
                            y0 = fmaf(l, yj0, y0);
                            y1 = fmaf(l, yj1, y1);
                        }
                    }
                } else {
                    for (int j = 0; j < bs; j++) {
                        const float l = -blk[j * kBsLd + lane];
                        const float yj0 = __shfl_sync(0xffffffffu, y0, j);
                        if (lane > j && lane < bs) y0 = fmaf(l, yj0, y0);
                    }
                }
                if (lane < bs) {
                    xs[(r0 + lane) * kBsRC + c] = y0;
                    if (two) xs[(r0 + lane) * kBsRC + c1] = y1;
                }
            }
            }
            __syncthreads();
            if (r0 + kBsB < n) stage_blk(r0 + kBsB, bi ^ 1);
            for (int i = r0 + bs + tid; i < n; i += kBsThreads) {
                float4 acc[kBsRC / 4];
#pragma unroll
                for (int q = 0; q < kBsRC / 4; q++) acc[q] = reinterpret_cast<const float4*>(xs + i * kBsRC)[q];
                for (int jb = 0; jb < bs; jb += 16) {
                    float lv[16];  // sixteen of the row's L values in flight: two round trips a block
#pragma unroll
                    for (int u = 0; u < 16; u++) lv[u] = jb + u < bs ? at(i, r0 + jb + u) : 0.0f;
#pragma unroll
                    for (int u = 0; u < 16; u++) {
                        if (jb + u >= bs) break;
                        const float nl = -lv[u];
#pragma unroll
                        for (int q = 0; q < kBsRC / 4; q++) {
                            const float4 xj = reinterpret_cast<const float4*>(xs + (r0 + jb + u) * kBsRC)[q];
                            acc[q].x = fmaf(nl, xj.x, acc[q].x);
                            acc[q].y = fmaf(nl, xj.y, acc[q].y);
                            acc[q].z = fmaf(nl, xj.z, acc[q].z);
                            acc[q].w = fmaf(nl, xj.w, acc[q].w);
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < kBsRC / 4; q++) reinterpret_cast<float4*>(xs + i * kBsRC)[q] = acc[q];
            }
            __syncthreads();
        }

        // ---------------------------------------------------------------- backward, U --
        const int nblk = (n + kBsB - 1) / kBsB;
        __syncthreads();  // the forward sweep's last reads of both buffers are done
        stage_blk((nblk - 1) * kBsB, 0);
        for (int kb = nblk - 1, bi = 0; kb >= 0; kb--, bi ^= 1) {
            const int r0 = kb * kBsB;
            const int bs = min(kBsB, n - r0);
            const float* blk = blks + bi * kBsB * kBsLd;
            cp_async_wait_all();
            __syncthreads();
            if (bs == kBsB) {
                // a whole block: warp 0 alone, lane = right-hand side; for j from the bottom,
                // x_j /= U(j,j), then x_i -= U(i,j) x_j for i < j (the reference's order)
                if (warp == 0 && lane < cw) {
                    float x[kBsB];
#pragma unroll
                    for (int i = 0; i < kBsB; i++) x[i] = xs[(r0 + i) * kBsRC + lane];
#pragma unroll
                    for (int j = kBsB - 1; j >= 0; j--) {
                        x[j] = x[j] / blk[j * kBsLd + j];
#pragma unroll
                        for (int i = 0; i < kBsB; i++)
                            if (i < j) x[i] = fmaf(-blk[j * kBsLd + i], x[j], x[i]);
                    }
#pragma unroll
                    for (int i = 0; i < kBsB; i++) xs[(r0 + i) * kBsRC + lane] = x[i];
                }
            } else {
            // two right-hand sides per warp; every lane divides (no divergence), lane j's quotient
            // x_j = y_j / U(j,j) is the one broadcast
            for (int c = warp; c < cw; c += 2 * (kBsThreads / 32)) {
                const int c1 = c + kBsThreads / 32;
                const bool two = c1 < cw;
                float y0 = lane < bs ? xs[(r0 + lane) * kBsRC + c] : 0.0f;
                float y1 = (two && lane < bs) ? xs[(r0 + lane) * kBsRC + c1] : 0.0f;
                if (two) {
                    for (int j = bs - 1; j >= 0; j--) {
                        const float ujj = blk[j * kBsLd + j];
                        const float u = -blk[j * kBsLd + lane];
                        const float xj0 = __shfl_sync(0xffffffffu, y0 / ujj, j);
                        const float xj1 = __shfl_sync(0xffffffffu, y1 / ujj, j);
                        if (lane == j) {
                            y0 = xj0;
                            y1 = xj1;
                        } else if (lane < j) {
                            y0 = fmaf(u, xj0, y0);
                            y1 = fmaf(u, xj1, y1);
                        }
                    }
                } else {
                    for (int j = bs - 1; j >= 0; j--) {
                        const float ujj = blk[j * kBsLd + j];
                        const float u = -blk[j * kBsLd + lane];
                        const float xj0 = __shfl_sync(0xffffffffu, y0 / ujj, j);
                        if (lane == j)
                            y0 = xj0;
                        else if (lane < j)
                            y0 = fmaf(u, xj0, y0);
                    }
                }
                if (lane < bs) {
                    xs[(r0 + lane) * kBsRC + c] = y0;
                    if (two) xs[(r0 + lane) * kBsRC + c1] = y1;
                }
            }
            }
            __syncthreads();
            if (kb > 0) stage_blk(r0 - kBsB, bi ^ 1);
            for (int i = tid; i < r0; i += kBsThreads) {
                float4 acc[kBsRC / 4];
#pragma unroll
                for (int q = 0; q < kBsRC / 4; q++) acc[q] = reinterpret_cast<const float4*>(xs + i * kBsRC)[q];
                for (int jt = bs; jt > 0; jt -= 16) {  // j = jt-1 down to jt-16, descending
                    float uv[16];  // sixteen of the row's U values in flight
#pragma unroll
                    for (int u = 0; u < 16; u++) uv[u] = jt - 1 - u >= 0 ? at(i, r0 + jt - 1 - u) : 0.0f;
#pragma unroll
                    for (int u = 0; u < 16; u++) {
                        const int j = jt - 1 - u;
                        if (j < 0) break;
                        const float nu = -uv[u];
#pragma unroll
                        for (int q = 0; q < kBsRC / 4; q++) {
                            const float4 xj = reinterpret_cast<const float4*>(xs + (r0 + j) * kBsRC)[q];
                            acc[q].x = fmaf(nu, xj.x, acc[q].x);
                            acc[q].y = fmaf(nu, xj.y, acc[q].y);
                            acc[q].z = fmaf(nu, xj.z, acc[q].z);
                            acc[q].w = fmaf(nu, xj.w, acc[q].w);
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < kBsRC / 4; q++) reinterpret_cast<float4*>(xs + i * kBsRC)[q] = acc[q];
            }
            __syncthreads();
        }

        for (int e = tid; e < n * cw; e += kBsThreads) {
            const int i = e % n, c = e / n;
            B[i + (long long)(c0 + c) * ldb] = xs[i * kBsRC + c];
        }
        __syncthreads();
    }
}

bool getrs_blk_supported(int n) { return n > 32 && getrs_blk_smem(n) <= 200 * 1024; }

cudaError_t getrs_blk_launch(cudaStream_t st, int n, int nrhs, const float* const* Aarray, int lda, const int* ipiv,
                             float* const* Barray, int ldb, int batch)
{
    const cudaError_t e = ensure_smem_limit(getrs_blk_kernel, 200 * 1024);
    if (e != cudaSuccess) return e;
    getrs_blk_kernel<<<(unsigned)batch, kBsThreads, getrs_blk_smem(n), st>>>(Aarray, n, lda, ipiv, Barray, ldb, nrhs);
    return cudaGetLastError();
}

}  // namespace opsblas
