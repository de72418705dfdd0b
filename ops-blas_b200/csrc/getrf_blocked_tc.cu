// Blocked batched LU on the matrix stored by rows, panels of 32 columns, two variants:
//   * plain FP32 getrf for 128 < n <= 1024 (aclblasSgetrfBatched, getrf_rows_launch): the
//     reference's arithmetic -- first-maximum pivot on exact magnitudes, true division, stop at
//     the first exactly-zero pivot -- and a tiled CUDA-core trailing update that applies the
//     rank-1 updates one fmaf at a time in the reference's order: bit-identical to it;
//   * mixed precision for 256 < n <= 1024 (aclblasSgetrfsRefineBatchedEx with
//     ACLBLAS_COMPUTE_32F_FAST_TF32, once the matrix no longer fits one SM's tensor memory:
//     getrf_tmem.cu covers n <= 256; getrf_blocked_tc_launch): the trailing update on the tcgen05
//     tensor cores in split TF32.
// Both work on the matrix stored by rows (T(i, j) at LU[j + i * ldlu]): a row is contiguous, so
// pivot rows, interchanges and the panel's rows are whole cache lines, where by columns every row
// element is a separate sector. The steps below describe the mixed variant; the plain one differs
// where lu_panel_kernel's EXACT says and runs lu_rows_update_kernel as its update.
//   0. lu_rows_in_kernel: A (by columns) into LU by rows, 32 x 32 tiles through shared memory.
//   Per panel k0 = 0, 32, ...:
//   1. lu_panel_kernel, one CTA per matrix, two panel rows a thread:
//      * factors the panel (rows k0..n-1, columns k0..k0+31) in FP32 in registers with implicit
//        pivoting (`pos` tracks the reference's in-place order): pivot = the largest magnitude
//        compared on the exponent and 14 mantissa bits (ties to the lowest position), multipliers
//        by an approximate reciprocal -- the refinement absorbs both --, one CTA barrier per
//        column; 1-based pivots in LAPACK's sequential-swap convention;
//      * writes the factored panel at the final positions and moves the rest of every row whose
//        position changed (at most 64 rows: the whole-row interchanges of the reference,
//        SwapRows, applied once per panel);
//      * L21 (rows below the diagonal block, K-contiguous) and U12 = L11^-1 * (the pivot rows'
//        trailing entries) into scratch as TF32 high and low planes; U12 also into its final rows;
//   2. gemm_tc_lu_update: T22 -= L21 * U12 on the tensor cores (split TF32, three products, FP32
//      accumulation), as the column-major product U12^T * L21^T on the by-rows storage;
//   and lu_rows_out_kernel transposes LU in place back to columns. On an exactly-zero pivot the
//   matrix stops (info = column + 1); its later updates change nothing.
#include <cuda_runtime.h>

#include "internal.h"
#include "small_common.cuh"
#include "tc_common.cuh"

namespace opsblas {

constexpr int kBpW = 32;  // panel width = the update's K

struct __align__(16) BpSmem {
    float crow[2][32][kBpW];  // per column parity and warp: the warp's pivot candidate row
    // per column (mod 3) the CTA's best pivot candidate: key << 5 | warp, by atomicMax; the
    // exact search keys on the magnitude bits and then the position, the mixed one on its
    // 32-bit approximate key
    unsigned long long pkey[3];
    float l11[kBpW][kBpW + 1];
    int mv_src[2 * kBpW];     // rows whose position changed: memory row and destination row
    int mv_dst[2 * kBpW];
    int mv_cnt;
};

// Scratch per matrix (byte offsets): L21 (n - 32 rows x 32, row-major) as its TF32 high plane
// followed by its low plane; U12 (32 x (n - 32), column-major: n - 32 "rows" of 32) the same way.
// A plane is (n - 32) x 32 floats, so each low plane starts n - 32 rows after its high plane.
struct BpScratch {
    long long plane, l21, u12, per_matrix;
    explicit BpScratch(int n)
    {
        plane = (long long)(n - kBpW) * kBpW * 4;
        l21 = 0;
        u12 = (2 * plane + 255) / 256 * 256;
        per_matrix = u12 + (2 * plane + 255) / 256 * 256;
    }
};

// 16-byte cp.async that reads src_bytes (0 or 16) and zero-fills the rest.
__device__ __forceinline__ void cp_async16_zf(uint32_t saddr, const void* gmem, int src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(gmem), "r"(src_bytes) : "memory");
}

// hi = x rounded to TF32 (nearest even), lo = (x - hi) rounded to TF32.
__device__ __forceinline__ void tf32_split(float x, float& hi, float& lo)
{
    hi = tf32_rne(x);
    lo = tf32_rne(x - hi);
}

// The transposes move 64 x 64 tiles with 256 threads: each thread has four 16-byte loads (or
// sixteen 4-byte loads when rows are not 16-byte aligned) of a tile in flight, the tile is
// re-read across from shared memory (row stride 65: conflict-free) and written as columns.
constexpr int kTpT = 64;

// tile (r0, c0) of the column-major matrix X (ld) into s[c][r] (r, c < 64, zeros outside n x n)
__device__ __forceinline__ void tp_load(float (*s)[kTpT + 1], const float* X, long long ld, int r0, int c0, int n,
                                        bool vec)
{
    const int tid = threadIdx.x;
    if (vec && r0 + kTpT <= n) {
        constexpr int K = kTpT * kTpT / 4 / 256;
        float4 v[K];  // every load in flight before the first store
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int e = tid + 256 * k, c = e / (kTpT / 4), rq = (e % (kTpT / 4)) * 4;
            v[k] = c0 + c < n ? *reinterpret_cast<const float4*>(X + (r0 + rq) + (long long)(c0 + c) * ld)
                              : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int e = tid + 256 * k, c = e / (kTpT / 4), rq = (e % (kTpT / 4)) * 4;
            s[c][rq] = v[k].x;
            s[c][rq + 1] = v[k].y;
            s[c][rq + 2] = v[k].z;
            s[c][rq + 3] = v[k].w;
        }
    } else {
        constexpr int K = kTpT * kTpT / 256;
        float v[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int e = tid + 256 * k, c = e / kTpT, r = e % kTpT;
            v[k] = (r0 + r < n && c0 + c < n) ? X[(r0 + r) + (long long)(c0 + c) * ld] : 0.0f;
        }
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int e = tid + 256 * k;
            s[e / kTpT][e % kTpT] = v[k];
        }
    }
}

// Y(r0 + r, c0 + c) = s[r][c] (the transpose of the tile s holds), column-major Y (ld)
__device__ __forceinline__ void tp_store(const float (*s)[kTpT + 1], float* Y, long long ld, int r0, int c0, int n,
                                         bool vec)
{
    const int tid = threadIdx.x;
    if (vec && r0 + kTpT <= n) {
#pragma unroll
        for (int k = 0; k < kTpT * kTpT / 4 / 256; k++) {
            const int e = tid + 256 * k, c = e / (kTpT / 4), rq = (e % (kTpT / 4)) * 4;
            if (c0 + c < n)
                *reinterpret_cast<float4*>(Y + (r0 + rq) + (long long)(c0 + c) * ld) =
                    make_float4(s[rq][c], s[rq + 1][c], s[rq + 2][c], s[rq + 3][c]);
        }
    } else {
#pragma unroll
        for (int k = 0; k < kTpT * kTpT / 256; k++) {
            const int e = tid + 256 * k, c = e / kTpT, r = e % kTpT;
            if (r0 + r < n && c0 + c < n) Y[(r0 + r) + (long long)(c0 + c) * ld] = s[r][c];
        }
    }
}

// T(i, j) = A(i, j): A by columns (lda) into LU by rows (ldt), i.e. the storage of T is the
// transpose of A's. One 64 x 64 tile (blockIdx.y) of one matrix (blockIdx.x).
__global__ void __launch_bounds__(256)
lu_rows_in_kernel(const float* const* __restrict__ Aarr, int lda, float* const* __restrict__ Tarr, int ldt, int n)
{
    __shared__ float tile[kTpT][kTpT + 1];
    const int nt = (n + kTpT - 1) / kTpT;
    const int i0 = (int)(blockIdx.y % nt) * kTpT, j0 = (int)(blockIdx.y / nt) * kTpT;
    const float* A = Aarr[blockIdx.x];
    float* T = Tarr[blockIdx.x];
    const bool vec = (reinterpret_cast<uintptr_t>(A) & 15) == 0 && (lda & 3) == 0 &&
                     (reinterpret_cast<uintptr_t>(T) & 15) == 0 && (ldt & 3) == 0;
    tp_load(tile, A, lda, i0, j0, n, vec);  // tile[c][r] = A(i0 + r, j0 + c)
    __syncthreads();
    tp_store(tile, T, ldt, j0, i0, n, vec);  // storage (j0 + r, i0 + c) = tile[r][c] = A(i0 + c, j0 + r)
}

// In-place transpose of the n x n storage matrix S(r, c) = LU[r + c * ld]: the by-rows factors
// become the by-columns LU (and back). One pair of 64 x 64 tiles (I, J), I <= J, per CTA
// (blockIdx.y).
__global__ void __launch_bounds__(256)
lu_rows_out_kernel(float* const* __restrict__ LUarr, int ld, int n)
{
    __shared__ float ta[kTpT][kTpT + 1], tb[kTpT][kTpT + 1];
    const int nt = (n + kTpT - 1) / kTpT;
    int p = (int)blockIdx.y, I = 0;
    while (p >= nt - I) {
        p -= nt - I;
        I++;
    }
    const int J = I + p;
    float* S = LUarr[blockIdx.x];
    const bool vec = (reinterpret_cast<uintptr_t>(S) & 15) == 0 && (ld & 3) == 0;
    const int a0 = I * kTpT, b0 = J * kTpT;
    tp_load(ta, S, ld, a0, b0, n, vec);                 // ta[c][r] = S(a0 + r, b0 + c)
    if (I != J) tp_load(tb, S, ld, b0, a0, n, vec);     // tb[c][r] = S(b0 + r, a0 + c)
    __syncthreads();
    if (I != J) tp_store(tb, S, ld, a0, b0, n, vec);    // S'(a0 + r, b0 + c) = tb[r][c] = S(b0 + c, a0 + r)
    tp_store(ta, S, ld, b0, a0, n, vec);                // S'(b0 + r, a0 + c) = ta[r][c] = S(a0 + c, b0 + r)
}

// Rows moved a round by the panel kernel's interchange step: 64 rows x MVC columns (128, or 64
// for the small CTAs, so that their shared memory lets more of them share an SM).
template <int NT>
struct PanelMv {
    static constexpr int MVC = NT >= 128 ? 64 : 32;  // two buffers of 64 x MVC floats
};

// One CTA per matrix; thread t holds memory rows k0 + t + r * NT (r < RPT) of the panel. NT x RPT
// covers the panel's rows; 128 registers a thread, so that 512 / NT CTAs share an SM.
// EXACT (the plain FP32 factorisation): the reference's arithmetic -- first maximum of the exact
// magnitudes, true division, and after a stop at column kk of the panel only the U rows above kk
// (the trailing update then takes rows from kk on with K = kk - k0); no TF32 planes (the update
// reads L21 and U12 from LU). Otherwise (mixed): the approximate pivot key and reciprocal, TF32
// planes, and a stop zeroes the update. PIVOT = false: no pivoting (the reference's no-pivot
// variant). st[m]: the matrix's info code so far (0, or the stop column + 1); info, when not
// nullptr, receives the same.
template <int NT, int RPT, bool EXACT, bool PIVOT>
__global__ void __launch_bounds__(NT, 512 / NT)
lu_panel_kernel(float* const* __restrict__ LUarr, int n, int ldt, int k0, int* __restrict__ piv,
                int* __restrict__ info, int* __restrict__ st, char* __restrict__ scratch, long long l21_off,
                long long u12_off, long long per_matrix)
{
    constexpr int NW = NT / 32;
    __shared__ BpSmem S;
    constexpr int kMvCols = PanelMv<NT>::MVC;
    __shared__ __align__(16) float mvbuf[2][2 * kBpW * kMvCols];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long m = blockIdx.x;
    float* T = LUarr[m];  // by rows: T(i, j) = T[j + i * ldt]
    int* pm = PIVOT ? piv + m * n : nullptr;
    const int mp = n - k0;                      // panel rows
    const int pw = mp < kBpW ? mp : kBpW;       // panel columns
    const int ntr = n - k0 - kBpW;              // trailing rows and columns
    const long long lo = (long long)(n - kBpW) * kBpW;  // floats from a high plane to its low plane
    float* L21 = EXACT ? nullptr : reinterpret_cast<float*>(scratch + m * per_matrix + l21_off);
    float* U12 = EXACT ? nullptr : reinterpret_cast<float*>(scratch + m * per_matrix + u12_off);
    const int inf0 = st[m];
    // whole rows as float4 when every row start is 16-byte aligned (uniform per matrix)
    const bool vec = (reinterpret_cast<uintptr_t>(T) & 15) == 0 && (ldt & 3) == 0 && pw == kBpW;

    if (tid == 0) {
        S.mv_cnt = 0;
        S.pkey[0] = 0ull;
        S.pkey[1] = 0ull;
    }
    if (inf0 != 0) {  // stopped at an earlier zero pivot
        if (!EXACT) {  // this step's update must change nothing
            for (int e = tid; e < (ntr > 0 ? ntr : 0) * kBpW; e += NT) {
                L21[e] = 0.0f;
                L21[lo + e] = 0.0f;
                U12[e] = 0.0f;
                U12[lo + e] = 0.0f;
            }
        }
        return;
    }

    // 1. this thread's panel rows (zeros outside the matrix)
    bool valid[RPT];
    int pos[RPT];
    float p[RPT][kBpW];
#pragma unroll
    for (int r = 0; r < RPT; r++) {
        valid[r] = tid + r * NT < mp;
        pos[r] = k0 + tid + r * NT;
#pragma unroll
        for (int c = 0; c < kBpW; c++) p[r][c] = 0.0f;
        if (valid[r]) {
            const float* row = T + (long long)pos[r] * ldt + k0;
            if (vec) {
#pragma unroll
                for (int q = 0; q < kBpW / 4; q++) {
                    const float4 v = reinterpret_cast<const float4*>(row)[q];
                    p[r][4 * q] = v.x;
                    p[r][4 * q + 1] = v.y;
                    p[r][4 * q + 2] = v.z;
                    p[r][4 * q + 3] = v.w;
                }
            } else {
#pragma unroll
                for (int c = 0; c < kBpW; c++)
                    if (c < pw) p[r][c] = row[c];
            }
        }
    }
    __syncthreads();

    // 2. factor, one CTA barrier per column
    int done = pw;
#pragma unroll
    for (int c = 0; c < kBpW; c++) {
        if (c >= pw) break;
        const int k = k0 + c;
        const int buf = c & 1;
        int ppos;
        const float* prow;
        bool nocand = false;  // (mixed search) no candidate key at all: treated as a zero pivot
        if (!PIVOT) {  // the row at position k
#pragma unroll
            for (int r = 0; r < RPT; r++)
                if (valid[r] && pos[r] == k) {
                    float4* dst = reinterpret_cast<float4*>(S.crow[buf][0]);
#pragma unroll
                    for (int q = 0; q < kBpW / 4; q++)
                        dst[q] = make_float4(p[r][4 * q], p[r][4 * q + 1], p[r][4 * q + 2], p[r][4 * q + 3]);
                }
            __syncthreads();
            ppos = k;
            prow = S.crow[buf][0];
        } else if (EXACT) {
            // first maximum of |x| over the positions >= k: the largest magnitude (as its bits; NaN
            // counts as zero and never wins), then the lowest position among equals
            unsigned bm = 0u;
            int bp = 0x7fffffff;
#pragma unroll
            for (int r = 0; r < RPT; r++) {
                if (!(valid[r] && pos[r] >= k)) continue;
                const float av = fabsf(p[r][c]);
                const unsigned mag = av == av ? __float_as_uint(av) : 0u;
                if (mag > bm || (mag == bm && pos[r] < bp)) {
                    bm = mag;
                    bp = pos[r];
                }
            }
            const unsigned wm = __reduce_max_sync(0xffffffffu, bm);
            const int wp = (int)__reduce_min_sync(0xffffffffu, bm == wm ? (unsigned)bp : 0x7fffffffu);
            // the warp's best into the CTA's: magnitude, then the lower position, then the warp
            if (lane == 0 && wp != 0x7fffffff)
                atomicMax(&S.pkey[c % 3], ((unsigned long long)wm << 32) |
                                              ((unsigned long long)(1023 - (wp - k0)) << 5) | (unsigned)warp);
#pragma unroll
            for (int r = 0; r < RPT; r++)
                if (valid[r] && pos[r] == wp && bp == wp) {
                    float4* dst = reinterpret_cast<float4*>(S.crow[buf][warp]);
#pragma unroll
                    for (int q = 0; q < kBpW / 4; q++)
                        dst[q] = make_float4(p[r][4 * q], p[r][4 * q + 1], p[r][4 * q + 2], p[r][4 * q + 3]);
                }
            if (tid == 0) S.pkey[(c + 1) % 3] = 0ull;  // read last at column c - 2, before this barrier
            __syncthreads();
            const unsigned long long key = S.pkey[c % 3];  // (position k is always a candidate)
            ppos = k0 + 1023 - (int)((key >> 5) & 1023u);
            prow = S.crow[buf][(int)(key & 31u)];
        } else {
            unsigned best = 0u;  // this thread's best candidate key (0: none)
#pragma unroll
            for (int r = 0; r < RPT; r++) {
                const float av = fabsf(p[r][c]);
                const unsigned mag = (av == av) ? (__float_as_uint(av) >> 9) : 0u;  // NaN never wins
                const unsigned key =
                    (valid[r] && pos[r] >= k) ? ((mag << 10) | (1023u - (unsigned)(pos[r] - k0))) : 0u;
                best = key > best ? key : best;
            }
            const unsigned wkey = __reduce_max_sync(0xffffffffu, best);
            if (lane == 0 && wkey != 0u) atomicMax(&S.pkey[c % 3], ((unsigned long long)wkey << 5) | (unsigned)warp);
            if (best != 0u && best == wkey) {  // keys are unique: one writer a warp
                float4* dst = reinterpret_cast<float4*>(S.crow[buf][warp]);
#pragma unroll
                for (int r = 0; r < RPT; r++) {
                    const float av = fabsf(p[r][c]);
                    const unsigned mag = (av == av) ? (__float_as_uint(av) >> 9) : 0u;
                    const unsigned key =
                        (valid[r] && pos[r] >= k) ? ((mag << 10) | (1023u - (unsigned)(pos[r] - k0))) : 0u;
                    if (key == best) {
#pragma unroll
                        for (int q = 0; q < kBpW / 4; q++)
                            dst[q] = make_float4(p[r][4 * q], p[r][4 * q + 1], p[r][4 * q + 2], p[r][4 * q + 3]);
                    }
                }
            }
            if (tid == 0) S.pkey[(c + 1) % 3] = 0ull;  // read last at column c - 2, before this barrier
            __syncthreads();
            const unsigned long long key = S.pkey[c % 3];
            const unsigned bk = (unsigned)(key >> 5);
            nocand = bk == 0u;
            ppos = nocand ? k : k0 + 1023 - (int)(bk & 1023u);
            prow = S.crow[buf][(int)(key & 31u)];
        }
        const float pv = prow[c];
        if (PIVOT && tid == 0) pm[k] = ppos + 1;
        if (pv == 0.0f || nocand) {  // exactly-zero pivot: stop here, before the interchange (uniform)
            if (tid == 0) {
                st[m] = k + 1;
                if (info != nullptr && info != st) info[m] = k + 1;
            }
            done = c;
            break;
        }
        float rinv = 0.0f;
        if (!EXACT) asm("rcp.approx.f32 %0, %1;" : "=f"(rinv) : "f"(pv));
        float l[RPT];
        bool upd[RPT];  // rows below the pivot position take the update
#pragma unroll
        for (int r = 0; r < RPT; r++) {
            if (PIVOT) {
                if (pos[r] == ppos)
                    pos[r] = k;
                else if (pos[r] == k)
                    pos[r] = ppos;
            }
            upd[r] = valid[r] && pos[r] > k;
            l[r] = EXACT ? p[r][c] / pv : p[r][c] * rinv;
            if (upd[r]) p[r][c] = l[r];
        }
        // p[j] -= l * u[j] for j > c: packed f32x2 fmas on the column pairs right of c (each lane
        // an IEEE fma, fma(u, -l, p) == fmaf(-l, u, p) bit for bit)
#pragma unroll
        for (int j = 0; j < kBpW; j += 2) {
            if (j > c) {
                const float2 u = make_float2(prow[j], prow[j + 1]);
#pragma unroll
                for (int r = 0; r < RPT; r++)
                    if (upd[r]) {
                        const float2 q = __ffma2_rn(u, make_float2(-l[r], -l[r]), make_float2(p[r][j], p[r][j + 1]));
                        p[r][j] = q.x;
                        p[r][j + 1] = q.y;
                    }
            } else if (j + 1 > c) {
                const float u = prow[j + 1];
#pragma unroll
                for (int r = 0; r < RPT; r++)
                    if (upd[r]) p[r][j + 1] = fmaf(-l[r], u, p[r][j + 1]);
            }
        }
    }
    const bool stopped = done < pw;

    // 3. the panel at its final rows; L21 (zero after a stop: the update then changes nothing) and
    //    L11; the rows whose position changed
#pragma unroll
    for (int r = 0; r < RPT; r++) {
        if (!valid[r]) continue;
        float* row = T + (long long)pos[r] * ldt + k0;
        if (vec) {
#pragma unroll
            for (int q = 0; q < kBpW / 4; q++)
                reinterpret_cast<float4*>(row)[q] =
                    make_float4(p[r][4 * q], p[r][4 * q + 1], p[r][4 * q + 2], p[r][4 * q + 3]);
        } else {
#pragma unroll
            for (int c = 0; c < kBpW; c++)
                if (c < pw) row[c] = p[r][c];
        }
        if (PIVOT && pos[r] != k0 + tid + r * NT) {
            const int q = atomicAdd(&S.mv_cnt, 1);
            S.mv_src[q] = k0 + tid + r * NT;
            S.mv_dst[q] = pos[r];
        }
        if (!EXACT && ntr > 0 && pos[r] >= k0 + kBpW) {
            float4* dh = reinterpret_cast<float4*>(L21 + (long long)(pos[r] - k0 - kBpW) * kBpW);
            float4* dl = reinterpret_cast<float4*>(L21 + lo + (long long)(pos[r] - k0 - kBpW) * kBpW);
#pragma unroll
            for (int q = 0; q < kBpW / 4; q++) {
                float h[4], lw[4];
#pragma unroll
                for (int e = 0; e < 4; e++) tf32_split(stopped ? 0.0f : p[r][4 * q + e], h[e], lw[e]);
                dh[q] = make_float4(h[0], h[1], h[2], h[3]);
                dl[q] = make_float4(lw[0], lw[1], lw[2], lw[3]);
            }
        }
        if (pos[r] < k0 + kBpW) {
#pragma unroll
            for (int c = 0; c < kBpW; c++) S.l11[pos[r] - k0][c] = p[r][c];
        }
    }
    __syncthreads();

    // 4. the rest of each moved row (columns 0..k0-1 and k0+pw..n-1) to its destination row,
    //    kMvCols columns a round staged in shared memory by cp.async: a round reads all its values
    //    before any is written (the moves form cycles)
    const int cnt = S.mv_cnt;  // <= 64: each of the panel's interchanges moves two rows
    if (cnt > 0) {
        const int nx = n - pw;  // columns outside the panel
        const int rounds = (nx + kMvCols - 1) / kMvCols;
        auto col_of = [&](int x) { return x < k0 ? x : x + pw; };
        // round rd: columns rd * kMvCols .. of every moved row into buffer rd & 1 (one cp.async group)
        auto fetch = [&](int rd) {
            const int x0 = rd * kMvCols;
            float* b = mvbuf[rd & 1];
            for (int e = tid; e < cnt * (kMvCols / 4); e += NT) {
                const int r = e / (kMvCols / 4), xq = x0 + (e % (kMvCols / 4)) * 4;
                float* d = b + r * kMvCols + (xq - x0);
                const float* srow = T + (long long)S.mv_src[r] * ldt;
                if (vec && xq + 3 < nx) {
                    cp_async16(d, srow + col_of(xq));  // four columns on the same side of the panel
                } else {
#pragma unroll
                    for (int u = 0; u < 4; u++)
                        if (xq + u < nx) cp_async4(d + u, srow + col_of(xq + u));
                }
            }
            cp_async_commit();
        };
        // two rounds in flight: a round's values are all read (into its buffer) before any of them
        // is written; rounds cover disjoint columns
        fetch(0);
        if (rounds > 1) fetch(1);
        for (int rd = 0; rd < rounds; rd++) {
            if (rd + 1 < rounds)
                cp_async_wait_group<1>();
            else
                cp_async_wait_group<0>();
            __syncthreads();
            const int x0 = rd * kMvCols;
            const float* b = mvbuf[rd & 1];
            for (int e = tid; e < cnt * (kMvCols / 4); e += NT) {
                const int r = e / (kMvCols / 4), xq = x0 + (e % (kMvCols / 4)) * 4;
                const float* sv = b + r * kMvCols + (xq - x0);
                float* drow = T + (long long)S.mv_dst[r] * ldt;
                if (vec && xq + 3 < nx) {
                    *reinterpret_cast<float4*>(drow + col_of(xq)) = *reinterpret_cast<const float4*>(sv);
                } else {
#pragma unroll
                    for (int u = 0; u < 4; u++)
                        if (xq + u < nx) drow[col_of(xq + u)] = sv[u];
                }
            }
            __syncthreads();
            if (rd + 2 < rounds) fetch(rd + 2);
        }
    }
    if (ntr <= 0) return;  // last panel: no trailing block

    // 5. U12 = L11^-1 * (the pivot rows' trailing entries, now in rows k0..k0+31), one thread per
    //    trailing column, in the reference's order (row i takes columns 0..i-1 in turn): the final U
    //    rows (above the stop column only, EXACT) and the TF32 planes of the update (mixed)
    const int urows = EXACT ? done : kBpW;
    for (int jj = tid; jj < ntr; jj += NT) {
        const int col = k0 + kBpW + jj;
        float u[kBpW];
#pragma unroll
        for (int i = 0; i < kBpW; i++) u[i] = (stopped && !EXACT) ? 0.0f : T[(long long)(k0 + i) * ldt + col];
#pragma unroll
        for (int i = 1; i < kBpW; i++)
#pragma unroll
            for (int c = 0; c < kBpW; c++)
                if (c < i && i < urows) u[i] = fmaf(-S.l11[i][c], u[c], u[i]);
        if (EXACT || !stopped) {
#pragma unroll
            for (int i = 1; i < kBpW; i++)
                if (i < urows) T[(long long)(k0 + i) * ldt + col] = u[i];
        }
        if (!EXACT) {
            float4* dh = reinterpret_cast<float4*>(U12 + (long long)jj * kBpW);
            float4* dl = reinterpret_cast<float4*>(U12 + lo + (long long)jj * kBpW);
#pragma unroll
            for (int q = 0; q < kBpW / 4; q++) {
                float h[4], lw[4];
#pragma unroll
                for (int e = 0; e < 4; e++) tf32_split(u[4 * q + e], h[e], lw[e]);
                dh[q] = make_float4(h[0], h[1], h[2], h[3]);
                dl[q] = make_float4(lw[0], lw[1], lw[2], lw[3]);
            }
        }
    }
}

// Trailing update of the plain factorisation, by rows: T(i, j) -= sum_k T(i, k0 + k) T(k0 + k, j)
// for rows i from r0 = k0 + 32 (or the stop column) and columns j from k0 + 32, K = 32 (or the
// columns before the stop), one fmaf at a time in increasing k -- the reference's sequence of
// rank-1 updates, so the result is bit-identical to it. A CTA of 128 threads computes a 64 x 128
// tile, each thread an 8 x 8 block (rows ty + 8 a, columns 8 tx ..): L (row-major, row stride 36
// floats: the eight row values of a step are conflict-free broadcasts) and U arrive in shared
// memory by cp.async while the thread's C block is loaded into registers, so a tile waits for one
// memory round trip; 144 registers, three CTAs an SM. st[m]: the matrix's info code (the update
// is skipped for a matrix stopped earlier). The grid's row tiles cover n - k0 rows (a stop adds up
// to 31 rows to the block).
constexpr int kRuRows = 64, kRuCols = 128, kRuLd = 36;

__global__ void __launch_bounds__(128, 3)
lu_rows_update_kernel(float* const* __restrict__ LUarr, int n, int ldt, int k0, const int* __restrict__ st,
                      int tiles_m, int tiles_n)
{
    __shared__ __align__(16) float Ls[kRuRows][kRuLd];    // Ls[row][k]
    __shared__ __align__(16) float Us[kBpW][kRuCols];     // Us[k][col]
    const int tiles = tiles_m * tiles_n;
    const long long m = blockIdx.x / tiles;
    const int tile = (int)(blockIdx.x % tiles);
    const int code = st[m];
    int r0 = k0 + kBpW, K = kBpW;
    if (code != 0) {
        if (code - 1 < k0) return;  // stopped in an earlier panel: no more updates
        K = code - 1 - k0;          // stopped in this panel at column k0 + K
        r0 = k0 + K;
        if (K == 0) return;
    }
    const int c0 = k0 + kBpW;
    const int rows = n - r0, cols = n - c0;
    const int tr = (tile % tiles_m) * kRuRows, tc = (tile / tiles_m) * kRuCols;
    if (tr >= rows || tc >= cols) return;
    float* T = LUarr[m];
    const bool vec = (reinterpret_cast<uintptr_t>(T) & 15) == 0 && (ldt & 3) == 0;
    const int tid = threadIdx.x;
    // L: rows r0 + tr + i, columns k0 .. k0 + K - 1; U: rows k0 .. k0 + K - 1, columns c0 + tc + j
    if (vec) {
#pragma unroll
        for (int u = 0; u < kRuRows * kBpW / 4 / 128; u++) {
            const int e = tid + 128 * u, i = e / (kBpW / 4), kq = (e % (kBpW / 4)) * 4;
            const bool ok = tr + i < rows && kq < K;
            cp_async16_zf(smem_u32(&Ls[i][kq]), T + (long long)(ok ? r0 + tr + i : r0) * ldt + k0 + kq, ok ? 16 : 0);
        }
#pragma unroll
        for (int u = 0; u < kRuCols * kBpW / 4 / 128; u++) {
            const int e = tid + 128 * u, k = e / (kRuCols / 4), jq = (e % (kRuCols / 4)) * 4;
            const bool ok = k < K && tc + jq + 3 < cols;
            if (ok || tc + jq >= cols || k >= K) {
                cp_async16_zf(smem_u32(&Us[k][jq]), T + (long long)(k0 + (k < K ? k : 0)) * ldt + c0 + (ok ? tc + jq : 0),
                                 ok ? 16 : 0);
            } else {  // the ragged right edge
#pragma unroll
                for (int q = 0; q < 4; q++)
                    Us[k][jq + q] = tc + jq + q < cols ? T[(long long)(k0 + k) * ldt + c0 + tc + jq + q] : 0.0f;
            }
        }
        cp_async_commit();
    } else {
        for (int e = tid; e < kRuRows * kBpW; e += 128) {
            const int i = e / kBpW, k = e % kBpW;
            Ls[i][k] = (tr + i < rows && k < K) ? T[(long long)(r0 + tr + i) * ldt + k0 + k] : 0.0f;
        }
        for (int e = tid; e < kRuCols * kBpW; e += 128) {
            const int k = e / kRuCols, j = e % kRuCols;
            Us[k][j] = (tc + j < cols && k < K) ? T[(long long)(k0 + k) * ldt + c0 + tc + j] : 0.0f;
        }
    }
    const int tx = tid & 15, ty = tid >> 4;  // 16 x 8 threads
    const int jb = tc + 8 * tx;
    const bool full = vec && jb + 7 < cols;
    float acc[8][8];
#pragma unroll
    for (int a = 0; a < 8; a++) {
        const int i = tr + ty + 8 * a;
        const float* src = T + (long long)(r0 + i) * ldt + c0 + jb;
        if (i >= rows) {
#pragma unroll
            for (int b = 0; b < 8; b++) acc[a][b] = 0.0f;
        } else if (full) {
            const float4 x = reinterpret_cast<const float4*>(src)[0], y = reinterpret_cast<const float4*>(src)[1];
            acc[a][0] = x.x, acc[a][1] = x.y, acc[a][2] = x.z, acc[a][3] = x.w;
            acc[a][4] = y.x, acc[a][5] = y.y, acc[a][6] = y.z, acc[a][7] = y.w;
        } else {
#pragma unroll
            for (int b = 0; b < 8; b++) acc[a][b] = jb + b < cols ? src[b] : 0.0f;
        }
    }
    if (vec) cp_async_wait_all();
    __syncthreads();
    // one step of k: acc -= l * u, as packed f32x2 fmas (each lane an IEEE fma: fma(u, -l, acc)
    // == fmaf(-l, u, acc) bit for bit)
    auto step = [&](int k) {
        float lv[8];
#pragma unroll
        for (int a = 0; a < 8; a++) lv[a] = Ls[ty + 8 * a][k];
        const float4 u0 = *reinterpret_cast<const float4*>(&Us[k][8 * tx]);
        const float4 u1 = *reinterpret_cast<const float4*>(&Us[k][8 * tx + 4]);
        const float2 up[4] = {make_float2(u0.x, u0.y), make_float2(u0.z, u0.w), make_float2(u1.x, u1.y),
                              make_float2(u1.z, u1.w)};
#pragma unroll
        for (int a = 0; a < 8; a++) {
            const float2 nl = make_float2(-lv[a], -lv[a]);
#pragma unroll
            for (int b = 0; b < 4; b++) {
                const float2 r = __ffma2_rn(up[b], nl, make_float2(acc[a][2 * b], acc[a][2 * b + 1]));
                acc[a][2 * b] = r.x;
                acc[a][2 * b + 1] = r.y;
            }
        }
    };
    if (K == kBpW) {
#pragma unroll 4
        for (int k = 0; k < kBpW; k++) step(k);
    } else {
        for (int k = 0; k < K; k++) step(k);
    }
#pragma unroll
    for (int a = 0; a < 8; a++) {
        const int i = tr + ty + 8 * a;
        if (i >= rows) continue;
        float* dst = T + (long long)(r0 + i) * ldt + c0 + jb;
        if (full) {
            reinterpret_cast<float4*>(dst)[0] = make_float4(acc[a][0], acc[a][1], acc[a][2], acc[a][3]);
            reinterpret_cast<float4*>(dst)[1] = make_float4(acc[a][4], acc[a][5], acc[a][6], acc[a][7]);
        } else {
#pragma unroll
            for (int b = 0; b < 8; b++)
                if (jb + b < cols) dst[b] = acc[a][b];
        }
    }
}

// The panel kernel's CTA shape by panel rows: two rows a thread, small CTAs share an SM.
template <bool EXACT, bool PIVOT>
static cudaError_t panel_launch(cudaStream_t st, float* const* T, int n, int ldt, int k0, int* piv, int* info,
                                int* stat, char* scratch, long long l21_off, long long u12_off, long long per_matrix,
                                int batch)
{
    const int mp = n - k0;
    const unsigned g = (unsigned)batch;
    if (mp <= 128)
        lu_panel_kernel<64, 2, EXACT, PIVOT><<<g, 64, 0, st>>>(T, n, ldt, k0, piv, info, stat, scratch, l21_off,
                                                                u12_off, per_matrix);
    else if (mp <= 256)
        lu_panel_kernel<128, 2, EXACT, PIVOT><<<g, 128, 0, st>>>(T, n, ldt, k0, piv, info, stat, scratch, l21_off,
                                                                  u12_off, per_matrix);
    else if (mp <= 512)
        lu_panel_kernel<256, 2, EXACT, PIVOT><<<g, 256, 0, st>>>(T, n, ldt, k0, piv, info, stat, scratch, l21_off,
                                                                  u12_off, per_matrix);
    else
        lu_panel_kernel<512, 2, EXACT, PIVOT><<<g, 512, 0, st>>>(T, n, ldt, k0, piv, info, stat, scratch, l21_off,
                                                                  u12_off, per_matrix);
    return cudaGetLastError();
}

bool getrf_rows_supported(int n, int batch)
{
    if (n <= 128 || n > 1024) return false;
    // the update's grid (batch x its tiles) must fit a 31-bit grid dimension
    const long long max_tiles = (long long)((n + kRuRows - 1) / kRuRows) * ((n - kBpW + kRuCols - 1) / kRuCols);
    return (long long)batch * max_tiles <= 0x7fffffffLL;
}

cudaError_t getrf_rows_launch(cudaStream_t st, float* const* Aarray, int n, int lda, int* piv, int* info, int* stat,
                              int batch)
{
    if (batch <= 0 || !getrf_rows_supported(n, batch)) return cudaErrorInvalidValue;
    cudaError_t err = cudaMemsetAsync(stat, 0, sizeof(int) * (size_t)batch, st);
    if (err == cudaSuccess && info != nullptr) err = cudaMemsetAsync(info, 0, sizeof(int) * (size_t)batch, st);
    if (err == cudaSuccess && piv != nullptr) err = cudaMemsetAsync(piv, 0, sizeof(int) * (size_t)n * batch, st);
    if (err != cudaSuccess) return err;
    const int nt = (n + kTpT - 1) / kTpT;
    const dim3 tgrid((unsigned)batch, (unsigned)(nt * (nt + 1) / 2));
    lu_rows_out_kernel<<<tgrid, 256, 0, st>>>(Aarray, lda, n);  // in place: by columns -> by rows
    for (int k0 = 0; k0 < n; k0 += kBpW) {
        err = piv != nullptr ? panel_launch<true, true>(st, Aarray, n, lda, k0, piv, info, stat, nullptr, 0, 0, 0, batch)
                             : panel_launch<true, false>(st, Aarray, n, lda, k0, nullptr, info, stat, nullptr, 0, 0, 0,
                                                         batch);
        if (err != cudaSuccess) return err;
        if (n - k0 - kBpW > 0) {
            const int tm = (n - k0 + kRuRows - 1) / kRuRows, tn = (n - k0 - kBpW + kRuCols - 1) / kRuCols;
            lu_rows_update_kernel<<<(unsigned)((long long)batch * tm * tn), 128, 0, st>>>(Aarray, n, lda, k0, stat, tm,
                                                                                          tn);
            err = cudaGetLastError();
            if (err != cudaSuccess) return err;
        }
    }
    lu_rows_out_kernel<<<tgrid, 256, 0, st>>>(Aarray, lda, n);  // by rows -> by columns
    return cudaGetLastError();
}

bool getrf_blocked_tc_supported(int n) { return n > 256 && n <= 1024; }

size_t getrf_blocked_tc_scratch_bytes(int n, int batch)
{
    return (size_t)BpScratch(n).per_matrix * (size_t)batch + (size_t)batch * 16 + 512;
}

cudaError_t getrf_blocked_tc_launch(cudaStream_t st, const float* const* Aarray, int lda, float* const* LUarray, int n,
                                    int ldlu, int* piv, int* info, int batch, void* scratch, unsigned* status,
                                    void* tmslots)
{
    if (!getrf_blocked_tc_supported(n) || batch <= 0) return cudaErrorInvalidValue;
    const BpScratch L(n);
    char* base = static_cast<char*>(scratch);
    float** l21p = reinterpret_cast<float**>(base + L.per_matrix * batch);
    float** u12p = l21p + batch;
    cudaError_t err = cudaMemsetAsync(info, 0, sizeof(int) * (size_t)batch, st);
    if (err == cudaSuccess) err = cudaMemsetAsync(piv, 0, sizeof(int) * (size_t)n * batch, st);
    if (err != cudaSuccess) return err;
    const unsigned bgrid = (unsigned)((batch + 255) / 256);
    init_ptr_array_kernel<<<bgrid, 256, 0, st>>>(l21p, reinterpret_cast<float*>(base + L.l21),
                                                 L.per_matrix / 4, batch);
    init_ptr_array_kernel<<<bgrid, 256, 0, st>>>(u12p, reinterpret_cast<float*>(base + L.u12),
                                                 L.per_matrix / 4, batch);
    const int nt = (n + kTpT - 1) / kTpT;
    lu_rows_in_kernel<<<dim3((unsigned)batch, (unsigned)(nt * nt)), 256, 0, st>>>(Aarray, lda, LUarray, ldlu, n);
    for (int k0 = 0; k0 < n; k0 += kBpW) {
        err = panel_launch<false, true>(st, LUarray, n, ldlu, k0, piv, info, info, base, L.l21, L.u12, L.per_matrix,
                                        batch);
        if (err != cudaSuccess) return err;
        const int mt = n - k0 - kBpW;
        if (mt > 0) {
            // by rows T22 -= L21 * U12 is, on the storage, C -= U12^T * L21^T (m x m, K = 32)
            err = gemm_tc_lu_update(st, mt, u12p, l21p, LUarray, (long long)(k0 + kBpW) * (1 + (long long)ldlu), ldlu,
                                    batch, n - kBpW, status, tmslots);
            if (err != cudaSuccess) return err;
        }
    }
    lu_rows_out_kernel<<<dim3((unsigned)batch, (unsigned)(nt * (nt + 1) / 2)), 256, 0, st>>>(LUarray, ldlu, n);
    return cudaGetLastError();
}

}  // namespace opsblas
