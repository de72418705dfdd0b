// Mixed-precision batched LU for 32 < n <= 256 with the matrix resident in tensor memory (TMEM).
//
// Used by aclblasSgetrfsRefineBatchedEx with ACLBLAS_COMPUTE_32F_FAST_TF32. One CTA of 256 threads
// per matrix; thread t owns physical row t. TMEM (all 512 columns of the SM) holds the matrix:
// rows 0..127 in lanes 0..127 at columns 0..255, rows 128..255 in the same lanes at columns
// 256..511, so warp w reaches its rows 32w..32w+31 through its lane quarter (w % 4). Rows never
// move; `pos` (the row's index in the reference's in-place matrix) records the interchanges.
// Per panel of 32 columns k0..k0+31:
//   1. every thread reads its row's panel columns from TMEM and the CTA factors the panel in FP32
//      by the reference's unblocked right-looking steps (one fmaf per update), with two
//      relaxations that the refinement absorbs: the pivot is the largest magnitude to 15 mantissa
//      bits and the multipliers use an approximate reciprocal; one CTA barrier per column;
//   2. the panel goes back to TMEM; the rows that became this panel's pivot rows publish their
//      unit-lower L11 part, and the rows below publish -L21 split into TF32 high and low parts
//      in the UMMA shared-memory layout (the MMA's A operand);
//   3. the pivot rows' trailing entries are read from TMEM, U12 = L11^-1 * A12 is formed in FP32
//      (one thread per column, reference order) and staged split into TF32 parts as the B operand;
//      the final U12 rows are written to global memory while the MMAs of step 4 run;
//   4. one thread issues A22 += (-L21) * U12 as tcgen05.mma (kind::tf32, hi*hi + hi*lo + lo*hi)
//      accumulating straight into the TMEM-resident trailing matrix, and commits to an mbarrier
//      that the CTA waits on (bounded) before the next panel reads TMEM. If that wait gives up,
//      the CTA waits (bounded) for the MMAs in flight, sets kStatusTmemLuTimeout in the handle's
//      status word and info = -1, and stops.
// At the end every row is written to global memory at its final position: the columns left of
// and inside its pivot panel from TMEM, the rest was written in step 3. HBM traffic is one read
// and one write of the matrix. Rows that are not below a panel get zero A-operand rows, so the MMA
// leaves them unchanged. On an exactly-zero pivot the factorisation stops (info = column + 1) and
// the trailing columns keep the state of the last completed panel.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "internal.h"
#include "small_common.cuh"
#include "tc_common.cuh"

namespace opsblas {

constexpr int kTmThreads = 256;
constexpr int kTmWarps = kTmThreads / 32;
constexpr int kTmMaxN = 256;
constexpr int kTmPB = 32;                // panel width = the MMA's K slice
constexpr int kTmPart = 128 * kTmPB;     // floats of one 128-row operand part
constexpr uint32_t kTmWaitLimit = 1u << 24;

struct TmSmem {
    float a_hi[2][kTmPart];  // -L21, rows of block b (physical rows 128b..), K-major UMMA layout
    float a_lo[2][kTmPart];
    float b_hi[2 * kTmPart];  // U12^T: 256 trailing columns x 32, K-major
    float b_lo[2 * kTmPart];
    float u12[kTmPB][kTmMaxN + 1];  // pivot rows' trailing entries, then U12
    float l11[kTmPB][kTmPB];        // unit-lower L11 of the panel (row = position - k0)
    float crow[2][kTmWarps][kTmPB]; // per column parity and warp: the warp's pivot candidate row
    unsigned ckey[2][kTmWarps];     //   its key (magnitude and position)
    int info;
    uint64_t mbar;
    uint32_t taddr;
};

__device__ __forceinline__ int tm_off(int r, int k)
{
    return (r >> 3) * (kTmPB * 8) + (k >> 2) * 32 + (r & 7) * 4 + (k & 3);
}

// BF16 operands: the same core-matrix layout with 8 values per 16-byte row. Float offset of the
// 16-byte chunk holding k = 8q..8q+7 of row r (SBO = 4 chunks x 128 B = 512 B).
__device__ __forceinline__ int tm_off16(int r, int q) { return (r >> 3) * 128 + q * 32 + (r & 7) * 4; }

__device__ __forceinline__ uint32_t bf16_pair(float a, float b)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);  // a in the low half (lower address)
    return *reinterpret_cast<const uint32_t*>(&h);
}

// Splits x into hi = bf16(x) and lo = bf16(x - hi).
__device__ __forceinline__ void bf16_split(float x, float& hi, float& lo)
{
    hi = __bfloat162float(__float2bfloat16_rn(x));
    lo = x - hi;
}

// Stages 32 values v (K index 0..31) of operand row r: TF32 (PREC 1) or BF16 (PREC 2) hi/lo parts.
template <int PREC>
__device__ __forceinline__ void tm_stage_row(float* hi_base, float* lo_base, int r, const float (&v)[kTmPB])
{
    if (PREC == 1) {
#pragma unroll
        for (int q = 0; q < kTmPB / 4; q++) {
            float hi[4], lo[4];
#pragma unroll
            for (int e = 0; e < 4; e++) {
                hi[e] = tf32_cvt(v[4 * q + e]);
                lo[e] = tf32_cvt(v[4 * q + e] - hi[e]);
            }
            *reinterpret_cast<float4*>(&hi_base[tm_off(r, 4 * q)]) = make_float4(hi[0], hi[1], hi[2], hi[3]);
            *reinterpret_cast<float4*>(&lo_base[tm_off(r, 4 * q)]) = make_float4(lo[0], lo[1], lo[2], lo[3]);
        }
    } else {
#pragma unroll
        for (int q = 0; q < kTmPB / 8; q++) {
            float hi[8], lo[8];
#pragma unroll
            for (int e = 0; e < 8; e++) bf16_split(v[8 * q + e], hi[e], lo[e]);
            *reinterpret_cast<uint4*>(&hi_base[tm_off16(r, q)]) =
                make_uint4(bf16_pair(hi[0], hi[1]), bf16_pair(hi[2], hi[3]), bf16_pair(hi[4], hi[5]),
                           bf16_pair(hi[6], hi[7]));
            *reinterpret_cast<uint4*>(&lo_base[tm_off16(r, q)]) =
                make_uint4(bf16_pair(lo[0], lo[1]), bf16_pair(lo[2], lo[3]), bf16_pair(lo[4], lo[5]),
                           bf16_pair(lo[6], lo[7]));
        }
    }
}

// Factors the panel held in p (this thread's row, 32 columns). Returns false when a zero pivot
// stopped the factorisation (S.info set). One CTA barrier per column: every warp publishes its
// best candidate (key, position and the whole panel row), double buffered by column parity, and
// after the barrier every thread picks the same winner and reads the pivot row from there.
__device__ __forceinline__ bool tm_panel(float (&p)[kTmPB], int& pos, bool valid, int n, int k0, int* pm, TmSmem& S,
                                         int tid, int warp, int lane)
{
#pragma unroll
    for (int c = 0; c < kTmPB; c++) {
        const int k = k0 + c;
        if (k >= n) break;
        const int buf = c & 1;
        // pivot: largest |a(., k)| over the rows at positions >= k, compared on the exponent and
        // 15 mantissa bits, ties to the lowest position -- one 32-bit key (magnitude << 9 |
        // 511 - position, never zero for an eligible row; NaN counts as zero) and a single
        // redux.sync per level. (The factors feed iterative refinement, so an equally good
        // pivot suffices; the plain kernels keep the reference's exact first-maximum rule.)
        const bool elig = valid && pos >= k;
        const float av = fabsf(p[c]);
        const unsigned mag = (av == av) ? (__float_as_uint(av) >> 8) : 0u;
        const unsigned key = elig ? ((mag << 9) | (511u - (unsigned)pos)) : 0u;
        const unsigned wkey = __reduce_max_sync(0xffffffffu, key);
        if (lane == 0) S.ckey[buf][warp] = wkey;
        if (elig && key == wkey) {  // the pivot row from column c's 16-byte chunk on
            float4* dst = reinterpret_cast<float4*>(S.crow[buf][warp]);
#pragma unroll
            for (int q = c / 4; q < kTmPB / 4; q++)
                dst[q] = make_float4(p[4 * q], p[4 * q + 1], p[4 * q + 2], p[4 * q + 3]);
        }
        __syncthreads();
        const unsigned qk = lane < kTmWarps ? S.ckey[buf][lane] : 0u;
        const unsigned bk = __reduce_max_sync(0xffffffffu, qk);
        const int bw = __ffs(__ballot_sync(0xffffffffu, lane < kTmWarps && qk == bk)) - 1;
        const int ppos = 511 - (int)(bk & 511u);
        const float* prow = S.crow[buf][bw];
        const float pv = prow[c];
        if (tid == 0 && pm) pm[k] = ppos + 1;
        if (pv == 0.0f) {
            if (tid == 0) S.info = k + 1;
            return false;
        }
        if (pos == ppos)
            pos = k;
        else if (pos == k)
            pos = ppos;
        if (valid && pos > k) {
            // multiplier by the approximate reciprocal (refinement absorbs its last-bit error),
            // then a(., j) -= l * u(j) two columns per packed fma
            float rinv;
            asm("rcp.approx.f32 %0, %1;" : "=f"(rinv) : "f"(pv));
            const float l = p[c] * rinv;
            p[c] = l;
            const float2 nl = make_float2(-l, -l);
#pragma unroll
            for (int q = c / 4; q < kTmPB / 4; q++) {
                const float4 u = reinterpret_cast<const float4*>(prow)[q];
                if (4 * q > c) {
                    const float2 r = __ffma2_rn(make_float2(u.x, u.y), nl, make_float2(p[4 * q], p[4 * q + 1]));
                    p[4 * q] = r.x;
                    p[4 * q + 1] = r.y;
                } else if (4 * q + 1 > c) {
                    p[4 * q + 1] = fmaf(-l, u.y, p[4 * q + 1]);
                }
                if (4 * q + 2 > c) {
                    const float2 r = __ffma2_rn(make_float2(u.z, u.w), nl, make_float2(p[4 * q + 2], p[4 * q + 3]));
                    p[4 * q + 2] = r.x;
                    p[4 * q + 3] = r.y;
                } else if (4 * q + 3 > c) {
                    p[4 * q + 3] = fmaf(-l, u.w, p[4 * q + 3]);
                }
            }
        }
    }
    return true;
}

template <int PREC>
__global__ void __launch_bounds__(kTmThreads, 1)
getrf_tmem_kernel(const float* const* __restrict__ Ain, int lda, float* const* __restrict__ LUarr, int n, int ldlu,
                  int* __restrict__ piv, int* __restrict__ info, unsigned* __restrict__ status, unsigned polls)
{
    extern __shared__ __align__(1024) unsigned char smraw[];
    TmSmem& S = *reinterpret_cast<TmSmem*>(smraw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long m = blockIdx.x;
    const float* A = Ain[m];
    float* LU = LUarr[m];
    int* pm = piv ? piv + m * n : nullptr;
    const int row = tid;  // physical row
    const bool valid = row < n;

    if (warp == 0) {
        tmem_alloc(&S.taddr, 512);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(&S.mbar, 1);
        fence_mbar_init();
        S.info = 0;
    }
    if (pm)
        for (int i = tid; i < n; i += kTmThreads) pm[i] = 0;
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tbase = S.taddr;
    // this thread's row at column 0: lane quarter of the warp, column half of the row block
    const uint32_t trow = tbase + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)((row >> 7) * 256);

    // ---- load: the whole row block, zeros outside the matrix ----
    {
        float v[16], w[16];  // the next chunk's loads are in flight while this chunk is stored
#pragma unroll
        for (int i = 0; i < 16; i++) v[i] = (valid && i < n) ? A[row + (long long)i * lda] : 0.0f;
        for (int j0 = 0; j0 < kTmMaxN; j0 += 16) {
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const int j = j0 + 16 + i;
                w[i] = (valid && j < n) ? A[row + (long long)j * lda] : 0.0f;
            }
            tmem_st16(trow + j0, v);
#pragma unroll
            for (int i = 0; i < 16; i++) v[i] = w[i];
        }
        tmem_wait_st();
    }

    int pos = row;
    int upanel = -1;  // first column of the panel in which this row became a pivot row
    uint32_t phase = 0;
    for (int k0 = 0; k0 < n; k0 += kTmPB) {
        // ---- 1. panel ----
        float p[kTmPB];
        {
            float v[16];
            tmem_ld16(trow + k0, v);
#pragma unroll
            for (int i = 0; i < 16; i++) p[i] = v[i];
            tmem_ld16(trow + k0 + 16, v);
#pragma unroll
            for (int i = 0; i < 16; i++) p[16 + i] = v[i];
        }
        const bool go = tm_panel(p, pos, valid, n, k0, pm, S, tid, warp, lane);
        // ---- 2. panel back to TMEM; L11 and -L21 operands ----
        {
            float v[16];
#pragma unroll
            for (int i = 0; i < 16; i++) v[i] = p[i];
            tmem_st16(trow + k0, v);
#pragma unroll
            for (int i = 0; i < 16; i++) v[i] = p[16 + i];
            tmem_st16(trow + k0 + 16, v);
            tmem_wait_st();
        }
        if (!go) break;  // zero pivot (uniform)
        const int kend = min(k0 + kTmPB, n);
        const int j0 = k0 + kTmPB;
        const int rest = n - j0;
        const bool pivot_row = valid && pos >= k0 && pos < kend;
        if (pivot_row) {
            upanel = k0;
#pragma unroll
            for (int q = 0; q < kTmPB / 4; q++)
                reinterpret_cast<float4*>(S.l11[pos - k0])[q] = make_float4(p[4 * q], p[4 * q + 1], p[4 * q + 2],
                                                                            p[4 * q + 3]);
        }
        if (rest <= 0) break;
        {
            const int b = row >> 7, r = row & 127;
            const bool below = valid && pos >= kend;
            float x[kTmPB];
#pragma unroll
            for (int cc = 0; cc < kTmPB; cc++) x[cc] = (below && k0 + cc < n) ? -p[cc] : 0.0f;
            tm_stage_row<PREC>(S.a_hi[b], S.a_lo[b], r, x);
        }
        __syncthreads();
        // ---- 3. U12 = L11^-1 * A12 ----
        for (int jc = j0; jc < n; jc += 16) {
            float v[16];
            tmem_ld16(trow + jc, v);
            if (pivot_row) {
#pragma unroll
                for (int i = 0; i < 16; i++)
                    if (jc + i < n) S.u12[pos - k0][jc - j0 + i] = v[i];
            }
        }
        __syncthreads();
        const int nr = kend - k0;  // pivot rows of this panel
        const int npad = (rest + 15) & ~15;
        for (int jj = tid; jj < npad; jj += kTmThreads) {
            float u[kTmPB];
#pragma unroll
            for (int r = 0; r < kTmPB; r++) u[r] = (jj < rest && r < nr) ? S.u12[r][jj] : 0.0f;
#pragma unroll
            for (int r = 1; r < kTmPB; r++) {
                if (r < nr) {
#pragma unroll
                    for (int q = 0; q < (r + 3) / 4; q++) {
                        const float4 lv = reinterpret_cast<const float4*>(S.l11[r])[q];
                        const float ll[4] = {lv.x, lv.y, lv.z, lv.w};
#pragma unroll
                        for (int e = 0; e < 4; e++)
                            if (4 * q + e < r) u[r] = fmaf(-ll[e], u[4 * q + e], u[r]);
                    }
                }
            }
            if (jj < rest) {
#pragma unroll
                for (int r = 0; r < kTmPB; r++) S.u12[r][jj] = u[r];  // written out after the MMA issue
            }
            tm_stage_row<PREC>(S.b_hi, S.b_lo, jj, u);
        }
        fence_async_smem();
        tc_fence_before_sync();
        __syncthreads();
        // ---- 4. A22 += (-L21) * U12 on the tensor cores, into the resident matrix ----
        if (tid == 0) {
            tc_fence_after_sync();
            const uint32_t idesc = umma_idesc(128, npad, PREC == 1 ? 2u : 1u);
            const uint32_t sbo = PREC == 1 ? kTmPB * 32 : kTmPB * 16;  // bytes between 8-row groups
            for (int b = 0; b < 2; b++) {
                if (128 * b >= n) break;
                const uint32_t d = tbase + (uint32_t)(b * 256 + j0);
#pragma unroll
                for (int s = 0; s < (PREC == 1 ? kTmPB / 8 : kTmPB / 16); s++) {
                    const uint32_t step = s * 256;  // two core matrices along K
                    const uint64_t ah = umma_smem_desc(smem_u32(S.a_hi[b]) + step, 128, sbo);
                    const uint64_t al = umma_smem_desc(smem_u32(S.a_lo[b]) + step, 128, sbo);
                    const uint64_t bh = umma_smem_desc(smem_u32(S.b_hi) + step, 128, sbo);
                    const uint64_t bl = umma_smem_desc(smem_u32(S.b_lo) + step, 128, sbo);
                    if (PREC == 1) {
                        umma_tf32(d, ah, bl, idesc, 1);
                        umma_tf32(d, al, bh, idesc, 1);
                        umma_tf32(d, ah, bh, idesc, 1);
                    } else {
                        umma_f16(d, ah, bl, idesc, 1);
                        umma_f16(d, al, bh, idesc, 1);
                        umma_f16(d, ah, bh, idesc, 1);
                    }
                }
            }
            umma_commit(&S.mbar);
        }
        // the final U12 rows go to global memory while the tensor cores run (coalesced columns)
        for (int jj = warp; jj < rest; jj += kTmWarps)
            if (lane < nr) LU[(k0 + lane) + (long long)(j0 + jj) * ldlu] = S.u12[lane][jj];
        const bool waited = mbar_wait_bounded(&S.mbar, phase, polls);
        if (__syncthreads_or(!waited)) {
            // give up: the MMAs in flight finish first (bounded), the status word reports it
            mbar_wait_bounded(&S.mbar, phase, kTmWaitLimit);
            tc_fence_after_sync();
            if (tid == 0) {
                atomicOr(status, kStatusTmemLuTimeout);
                S.info = -1;
            }
            break;
        }
        phase ^= 1u;
        tc_fence_after_sync();
    }

    // ---- store: row at its final position; columns right of its pivot panel were written as U12 ----
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const int lim = upanel >= 0 ? upanel + kTmPB : n;
    for (int jc = 0; jc < n; jc += 16) {
        float v[16];
        tmem_ld16(trow + jc, v);
        if (valid) {
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const int j = jc + i;
                if (j < n && j < lim) LU[pos + (long long)j * ldlu] = v[i];
            }
        }
    }
    if (tid == 0 && info != nullptr) info[m] = S.info;
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tbase, 512);
}

bool getrf_tmem_supported(int n) { return n > 32 && n <= kTmMaxN; }

cudaError_t getrf_tmem_launch(cudaStream_t st, const float* const* Aarray, int lda, float* const* LUarray, int n,
                              int ldlu, int* piv, int* info, int batch, int prec, unsigned* status)
{
    const unsigned polls = wait_limit(kTmWaitLimit);
    const cudaError_t e = prec == 2 ? ensure_smem_limit(getrf_tmem_kernel<2>, (int)sizeof(TmSmem))
                                    : ensure_smem_limit(getrf_tmem_kernel<1>, (int)sizeof(TmSmem));
    if (e != cudaSuccess) return e;
    if (prec == 2)
        getrf_tmem_kernel<2><<<(unsigned)batch, kTmThreads, sizeof(TmSmem), st>>>(Aarray, lda, LUarray, n, ldlu, piv,
                                                                                 info, status, polls);
    else
        getrf_tmem_kernel<1><<<(unsigned)batch, kTmThreads, sizeof(TmSmem), st>>>(Aarray, lda, LUarray, n, ldlu, piv,
                                                                                 info, status, polls);
    return cudaGetLastError();
}

}  // namespace opsblas
