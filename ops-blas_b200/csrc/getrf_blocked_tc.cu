// Mixed-precision batched LU for 256 < n <= 1024: blocked right-looking, panels of 32 columns,
// the trailing update on the tcgen05 tensor cores.
//
// Used by aclblasSgetrfsRefineBatchedEx with ACLBLAS_COMPUTE_32F_FAST_TF32 when the matrix no
// longer fits one SM's tensor memory (getrf_tmem.cu covers n <= 256). Per panel k0 = 0, 32, ...:
//   1. lu_panel_kernel, one CTA per matrix, thread t = panel row k0 + t:
//      * writes the previous panel's U12 (kept in scratch) into its final rows k0-32..k0-1;
//      * factors the panel (rows k0..n-1, columns k0..k0+31) in FP32 in registers with implicit
//        pivoting (rows never move; `pos` tracks the reference's in-place order): pivot = the
//        largest magnitude compared on the exponent and 14 mantissa bits (ties to the lowest
//        position), multipliers by an approximate reciprocal -- the refinement absorbs both --,
//        one CTA barrier per column; 1-based pivots in LAPACK's sequential-swap convention;
//      * writes the factored panel at the final positions, L21 (rows below the diagonal block,
//        K-contiguous) and U12 = L11^-1 * (the pivot rows' trailing entries) into scratch, both
//        already split into TF32 high and low planes (plus U12 in FP32 for the final U), and the
//        row map of the trailing block: position r's trailing data still sits in memory row
//        src(r) (a row that left the top 32 rows for a pivot row's place keeps its data there);
//   2. gemm_tc_lu_update: A22(r, :) = A22(src(r), :) - L21(r, :) * U12 on the tensor cores
//      (split TF32, three products, FP32 accumulation), the four operand planes by TMA, the
//      result added to A22 by TMA reduce-add; the few rows whose data moved are written from
//      their source rows -- the row interchanges of the trailing block, with no swap pass;
// and at the end lu_lgather_kernel applies each panel's later interchanges to its L columns (a
// gather through shared memory per 32-column block). On an exactly-zero pivot the matrix stops
// (info = column + 1); its later updates change nothing.
#include <cuda_runtime.h>

#include "internal.h"
#include "tc_common.cuh"

namespace opsblas {

constexpr int kBpW = 32;  // panel width = the update's K

struct __align__(16) BpSmem {
    float crow[2][32][kBpW];  // per column parity and warp: the warp's pivot candidate row
    unsigned ckey[2][32];     //   its key
    float l11[kBpW][kBpW + 1];
    int prow[kBpW];           // memory row of the pivot row of U row i (position k0 + i)
    int info;
};

// Scratch per matrix (byte offsets): L21 (n - 32 rows x 32, row-major) as its TF32 high plane
// followed by its low plane; U12 (32 x (n - 32), column-major: n - 32 "rows" of 32) as high plane,
// low plane and the FP32 values (the final U rows); the row map (n ints). A plane is
// (n - 32) x 32 floats, so each low plane starts n - 32 rows after its high plane.
struct BpScratch {
    long long plane, l21, u12, src, per_matrix;
    explicit BpScratch(int n)
    {
        plane = (long long)(n - kBpW) * kBpW * 4;
        l21 = 0;
        u12 = (2 * plane + 255) / 256 * 256;
        src = u12 + (3 * plane + 255) / 256 * 256;
        per_matrix = src + ((long long)n * 4 + 255) / 256 * 256;
    }
};

// hi = x rounded to TF32 (nearest even), lo = (x - hi) rounded to TF32.
__device__ __forceinline__ void tf32_split(float x, float& hi, float& lo)
{
    hi = tf32_rne(x);
    lo = tf32_rne(x - hi);
}

template <int NT>
__global__ void __launch_bounds__(NT, 1)
lu_panel_kernel(float* const* __restrict__ LUarr, int n, int ldlu, int k0, int* __restrict__ piv,
                int* __restrict__ info, char* __restrict__ scratch, long long l21_off, long long u12_off,
                long long src_off, long long per_matrix)
{
    constexpr int NW = NT / 32;
    __shared__ BpSmem S;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long m = blockIdx.x;
    float* LU = LUarr[m];
    char* base = scratch + m * per_matrix;
    float* L21 = reinterpret_cast<float*>(base + l21_off);
    float* U12 = reinterpret_cast<float*>(base + u12_off);
    int* src = reinterpret_cast<int*>(base + src_off);
    int* pm = piv + m * n;
    const int mp = n - k0;                      // panel rows
    const int pw = mp < kBpW ? mp : kBpW;       // panel columns
    const int ntr = n - k0 - kBpW;              // trailing rows and columns
    const long long lo = (long long)(n - kBpW) * kBpW;  // floats from a high plane to its low plane
    const int inf0 = info[m];

    // 1. the previous panel's U12 (FP32 plane) into its final rows (k0 - 32 .. k0 - 1, columns
    //    k0 .. n - 1)
    if (k0 > 0 && inf0 == 0) {
        const int cols = n - k0;
        for (int e = tid; e < cols * kBpW; e += NT) {
            const int j = e / kBpW, i = e % kBpW;
            LU[(k0 - kBpW + i) + (long long)(k0 + j) * ldlu] = U12[2 * lo + j * kBpW + i];
        }
    }
    if (tid == 0) S.info = inf0;
    __syncthreads();
    if (inf0 != 0) {  // stopped at an earlier zero pivot: this step's update must change nothing
        for (int e = tid; e < (ntr > 0 ? ntr : 0) * kBpW; e += NT) {
            L21[e] = 0.0f;
            L21[lo + e] = 0.0f;
            U12[e] = 0.0f;
            U12[lo + e] = 0.0f;
        }
        for (int r = tid; r < ntr; r += NT) src[r] = r;
        return;
    }

    // 2. the panel row of this thread (zeros outside the matrix)
    const bool valid = tid < mp;
    float p[kBpW];
#pragma unroll
    for (int c = 0; c < kBpW; c++) p[c] = (valid && c < pw) ? LU[(k0 + tid) + (long long)(k0 + c) * ldlu] : 0.0f;
    int pos = k0 + tid;

    // 3. factor, one CTA barrier per column
    int done = pw;
#pragma unroll
    for (int c = 0; c < kBpW; c++) {
        if (c >= pw) break;
        const int k = k0 + c;
        const int buf = c & 1;
        const bool elig = valid && pos >= k;
        const float av = fabsf(p[c]);
        const unsigned mag = (av == av) ? (__float_as_uint(av) >> 9) : 0u;  // NaN never wins
        const unsigned key = elig ? ((mag << 10) | (1023u - (unsigned)(pos - k0))) : 0u;
        const unsigned wkey = __reduce_max_sync(0xffffffffu, key);
        if (lane == 0) S.ckey[buf][warp] = wkey;
        if (elig && key == wkey) {
            float4* dst = reinterpret_cast<float4*>(S.crow[buf][warp]);
#pragma unroll
            for (int q = 0; q < kBpW / 4; q++) dst[q] = make_float4(p[4 * q], p[4 * q + 1], p[4 * q + 2], p[4 * q + 3]);
        }
        __syncthreads();
        const unsigned qk = lane < NW ? S.ckey[buf][lane] : 0u;
        const unsigned bk = __reduce_max_sync(0xffffffffu, qk);
        const int bw = __ffs(__ballot_sync(0xffffffffu, lane < NW && qk == bk)) - 1;
        const int ppos = k0 + 1023 - (int)(bk & 1023u);
        const float* prow = S.crow[buf][bw];
        const float pv = prow[c];
        if (tid == 0) pm[k] = ppos + 1;
        if (pv == 0.0f || bk == 0u) {  // exactly-zero pivot column: stop here (uniform)
            if (tid == 0) {
                S.info = k + 1;
                info[m] = k + 1;
            }
            done = c;
            break;
        }
        if (pos == ppos)
            pos = k;
        else if (pos == k)
            pos = ppos;
        if (valid && pos > k) {
            float rinv;
            asm("rcp.approx.f32 %0, %1;" : "=f"(rinv) : "f"(pv));
            const float l = p[c] * rinv;
            p[c] = l;
#pragma unroll
            for (int j = 0; j < kBpW; j++)
                if (j > c) p[j] = fmaf(-l, prow[j], p[j]);
        }
    }
    const bool stopped = done < pw;

    // 4. the panel at its final positions
    if (valid) {
#pragma unroll
        for (int c = 0; c < kBpW; c++)
            if (c < pw) LU[pos + (long long)(k0 + c) * ldlu] = p[c];
    }
    if (ntr <= 0) return;  // last panel: no trailing block
    // 5. L21 (zero after a stop: the update then changes nothing), the row map, L11 and pivot rows
    if (valid && pos >= k0 + kBpW) {
        float4* dh = reinterpret_cast<float4*>(L21 + (long long)(pos - k0 - kBpW) * kBpW);
        float4* dl = reinterpret_cast<float4*>(L21 + lo + (long long)(pos - k0 - kBpW) * kBpW);
#pragma unroll
        for (int q = 0; q < kBpW / 4; q++) {
            float h[4], l[4];
#pragma unroll
            for (int e = 0; e < 4; e++) tf32_split(stopped ? 0.0f : p[4 * q + e], h[e], l[e]);
            dh[q] = make_float4(h[0], h[1], h[2], h[3]);
            dl[q] = make_float4(l[0], l[1], l[2], l[3]);
        }
        src[pos - k0 - kBpW] = stopped ? pos - k0 - kBpW : tid - kBpW;
    }
    if (valid && pos < k0 + kBpW) {
        const int i = pos - k0;
        S.prow[i] = k0 + tid;
#pragma unroll
        for (int c = 0; c < kBpW; c++) S.l11[i][c] = p[c];
    }
    __syncthreads();
    // 6. U12 = L11^-1 * (the pivot rows' trailing entries), one thread per trailing column
    for (int jj = tid; jj < ntr; jj += NT) {
        const long long col = (long long)(k0 + kBpW + jj) * ldlu;
        float u[kBpW];
#pragma unroll
        for (int i = 0; i < kBpW; i++) u[i] = stopped ? 0.0f : LU[S.prow[i] + col];
#pragma unroll
        for (int i = 1; i < kBpW; i++)
#pragma unroll
            for (int c = 0; c < kBpW; c++)
                if (c < i) u[i] = fmaf(-S.l11[i][c], u[c], u[i]);
        float4* dh = reinterpret_cast<float4*>(U12 + (long long)jj * kBpW);
        float4* dl = reinterpret_cast<float4*>(U12 + lo + (long long)jj * kBpW);
        float4* df = reinterpret_cast<float4*>(U12 + 2 * lo + (long long)jj * kBpW);
#pragma unroll
        for (int q = 0; q < kBpW / 4; q++) {
            float h[4], l[4];
#pragma unroll
            for (int e = 0; e < 4; e++) tf32_split(u[4 * q + e], h[e], l[e]);
            dh[q] = make_float4(h[0], h[1], h[2], h[3]);
            dl[q] = make_float4(l[0], l[1], l[2], l[3]);
            df[q] = make_float4(u[4 * q], u[4 * q + 1], u[4 * q + 2], u[4 * q + 3]);
        }
    }
}

// After the last panel: the rows of each 32-column block below its diagonal block take their
// final order. The interchanges of the later panels (applied to every column by the reference's
// whole-row swaps) are traced back from each final position i to the position that held the row
// when the block was factored (undoing each later panel's swaps in reverse), and the block is
// gathered through shared memory. One CTA per matrix, thread = row (up to 1024 rows).
__global__ void __launch_bounds__(1024, 1)
lu_lgather_kernel(float* const* __restrict__ LUarr, int n, int ldlu, const int* __restrict__ piv)
{
    extern __shared__ float blk[];  // (n - 32) x 32, row i - 32 (p + 1) at blk[... * 33]
    const int tid = threadIdx.x;
    const long long m = blockIdx.x;
    float* LU = LUarr[m];
    const int* pm = piv + m * n;
    const int P = (n + kBpW - 1) / kBpW;
    int pos = tid;  // for row tid: where its row sat after panel p
    for (int p = P - 2; p >= 0; p--) {
        // undo panel p + 1's interchanges (in reverse order)
        const int s0 = (p + 1) * kBpW;
        const int s1 = min(n, s0 + kBpW);
        for (int k = s1 - 1; k >= s0; k--) {
            const int r = pm[k] - 1;
            if (r < 0 || r == k) continue;  // no interchange (after a stop the pivots are 0)
            if (pos == k)
                pos = r;
            else if (pos == r)
                pos = k;
        }
        const int r0 = (p + 1) * kBpW;  // first row below block p's diagonal block
        const int rows = n - r0;
        const int c0 = p * kBpW;
        __syncthreads();
        if (tid >= r0 && tid < n) {
#pragma unroll 4
            for (int c = 0; c < kBpW; c++) blk[(tid - r0) * (kBpW + 1) + c] = LU[pos + (long long)(c0 + c) * ldlu];
        }
        __syncthreads();
        for (int e = tid; e < rows * kBpW; e += blockDim.x) {
            const int c = e / rows, i = e % rows;  // coalesced along the column
            LU[(r0 + i) + (long long)(c0 + c) * ldlu] = blk[i * (kBpW + 1) + c];
        }
    }
}

bool getrf_blocked_tc_supported(int n) { return n > 256 && n <= 1024; }

size_t getrf_blocked_tc_scratch_bytes(int n, int batch)
{
    return (size_t)BpScratch(n).per_matrix * (size_t)batch + (size_t)batch * 16 + 512;
}

cudaError_t getrf_blocked_tc_launch(cudaStream_t st, float* const* LUarray, int n, int ldlu, int* piv, int* info,
                                    int batch, void* scratch, unsigned* status, void* tmslots)
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
    const int* srcmap = reinterpret_cast<const int*>(base + L.src);
    for (int k0 = 0; k0 < n; k0 += kBpW) {
        if (n - k0 <= 512)
            lu_panel_kernel<512><<<(unsigned)batch, 512, 0, st>>>(LUarray, n, ldlu, k0, piv, info, base, L.l21, L.u12,
                                                                  L.src, L.per_matrix);
        else
            lu_panel_kernel<1024><<<(unsigned)batch, 1024, 0, st>>>(LUarray, n, ldlu, k0, piv, info, base, L.l21,
                                                                    L.u12, L.src, L.per_matrix);
        err = cudaGetLastError();
        if (err != cudaSuccess) return err;
        const int mt = n - k0 - kBpW;
        if (mt > 0) {
            err = gemm_tc_lu_update(st, mt, l21p, u12p, LUarray, (long long)(k0 + kBpW) * (1 + (long long)ldlu), ldlu,
                                    batch, srcmap, L.per_matrix / 4, n - kBpW, status, tmslots);
            if (err != cudaSuccess) return err;
        }
    }
    const size_t gsm = (size_t)(n - kBpW) * (kBpW + 1) * 4;
    err = ensure_smem_limit(lu_lgather_kernel, (int)gsm);
    if (err != cudaSuccess) return err;
    lu_lgather_kernel<<<(unsigned)batch, 1024, gsm, st>>>(LUarray, n, ldlu, piv);
    return cudaGetLastError();
}

}  // namespace opsblas
