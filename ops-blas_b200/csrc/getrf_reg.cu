// aclblasSgetrfBatched for 32 < n <= 128: one CTA per matrix, the matrix in registers
// (reg_getrf_core, lu_core.cuh). Rows are spread over the lanes (R = ceil(n/32) rows per lane,
// the same rows in every warp) and columns are dealt out cyclically over NW warps, so all warps
// update until the last columns; one CTA barrier per column hands the pivot and multipliers from
// the column's owner warp to the others. The arithmetic is the reference's unblocked
// right-looking LU (sgetrf_batched_kernel.cpp:106-150) element for element, so the factors are
// bit-identical to the other batched kernels and to the oracle.
#include <cuda_runtime.h>

#include "internal.h"
#include "lu_core.cuh"

namespace opsblas {

template <int R, int NW, bool PIVOT>
__global__ void __launch_bounds__(NW * 32, NW == 8 ? 2 : (NW == 4 ? 3 : 8))
getrf_reg_kernel(float* const* __restrict__ Aarray, int n, int lda, int* __restrict__ piv, int* __restrict__ info)
{
    constexpr int CW = RegShape<R, NW>::CW;
    __shared__ RegTeamSmem S;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long m = blockIdx.x;
    float* A = Aarray[m];
    float a[R][CW];
    int pos[R];
    reg_load<R, NW>(a, A, lda, n, warp, lane);
#pragma unroll
    for (int t = 0; t < R; t++) pos[t] = lane + 32 * t;
    int* pm = PIVOT ? piv + m * n : nullptr;
    if (PIVOT)
        for (int i = threadIdx.x; i < n; i += NW * 32) pm[i] = 0;
    __syncthreads();
    const int inf = reg_getrf_core<R, NW, PIVOT>(a, pos, n, S, pm, warp, lane, -1);
    reg_store<R, NW>(a, pos, A, lda, n, warp, lane);
    if (threadIdx.x == 0 && info != nullptr) info[m] = inf;
}

// Shapes (rows per lane R, warps NW) that are instantiated; R * 32 >= n is required.
bool reg_shape_valid(int n, int rows, int warps)
{
    if (n <= 32 || n > 32 * rows) return false;
    return (rows == 2 && (warps == 2 || warps == 4 || warps == 8)) || (rows == 3 && (warps == 4 || warps == 8)) ||
           (rows == 4 && warps == 8);
}

// Built-in choice (the plain batched path, and the grouped launch without a tuning table): the
// fastest shapes measured per size bucket on B200 -- 2 warps up to 64 rows, 4 warps up to 96,
// 8 warps for 4 rows per lane (ops-blas_b200/grouped_tuning.txt).
void reg_default_shape(int n, int& rows, int& warps)
{
    rows = (n + 31) / 32;
    warps = rows == 2 ? 2 : (rows == 3 ? 4 : 8);
}

bool getrf_reg_supported(int n) { return n > 32 && n <= 128; }

template <int R, int NW>
static void launch_shape(cudaStream_t st, float* const* Aarray, int n, int lda, int* piv, int* info, int batch)
{
    if (piv)
        getrf_reg_kernel<R, NW, true><<<(unsigned)batch, NW * 32, 0, st>>>(Aarray, n, lda, piv, info);
    else
        getrf_reg_kernel<R, NW, false><<<(unsigned)batch, NW * 32, 0, st>>>(Aarray, n, lda, nullptr, info);
}

cudaError_t getrf_reg_launch(cudaStream_t st, float* const* Aarray, int n, int lda, int* piv, int* info, int batch,
                             int rows, int warps)
{
    if (!reg_shape_valid(n, rows, warps)) reg_default_shape(n, rows, warps);
    if (rows == 2 && warps == 2) launch_shape<2, 2>(st, Aarray, n, lda, piv, info, batch);
    else if (rows == 2 && warps == 4) launch_shape<2, 4>(st, Aarray, n, lda, piv, info, batch);
    else if (rows == 2) launch_shape<2, 8>(st, Aarray, n, lda, piv, info, batch);
    else if (rows == 3 && warps == 4) launch_shape<3, 4>(st, Aarray, n, lda, piv, info, batch);
    else if (rows == 3) launch_shape<3, 8>(st, Aarray, n, lda, piv, info, batch);
    else launch_shape<4, 8>(st, Aarray, n, lda, piv, info, batch);
    return cudaGetLastError();
}

}  // namespace opsblas
