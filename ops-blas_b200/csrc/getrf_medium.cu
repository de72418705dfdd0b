// aclblasSgetrfBatched for 32 < n <= 128: one CTA per matrix, matrix resident in shared memory,
// blocked right-looking LU that keeps the reference's per-element arithmetic.
//
// The blocked algorithm (panel by one warp, U12 forward substitution, register-tiled A22 update
// in the reference's per-element order, logical-to-physical row map) is med_getrf_core in
// lu_core.cuh; this kernel loads the matrix, runs it with the whole CTA and stores the result.
#include <cuda_runtime.h>

#include "internal.h"
#include "lu_core.cuh"

namespace opsblas {

constexpr int kMedThreads = 128;  // 4 warps
constexpr int kMedPB = 16;        // panel width

template <bool PIVOT>
__global__ void __launch_bounds__(kMedThreads)
getrf_medium_kernel(float* const* __restrict__ Aarray, int n, int lda, int* __restrict__ piv, int* __restrict__ info)
{
    extern __shared__ __align__(16) float smem[];
    const MedLayout L(n, kMedPB);
    const MedSmem S(smem, L, n, kMedPB);
    const int ld = L.ld;

    const long long m = blockIdx.x;
    float* A = Aarray[m];
    int* pm = PIVOT ? piv + m * n : nullptr;
    const int tid = threadIdx.x;

    for (int e = tid; e < n * n; e += kMedThreads) {
        const int i = e % n, j = e / n;
        S.sa[i + j * ld] = A[i + (long long)j * lda];
    }
    for (int i = tid; i < n; i += kMedThreads) S.rmap[i] = i;
    if (PIVOT)
        for (int i = tid; i < n; i += kMedThreads) pm[i] = 0;
    if (tid == 0) S.sc[0] = 0;
    __syncthreads();

    const int inf = med_getrf_core<PIVOT, kMedThreads, kMedPB>(S, n, ld, L.ls_ld, pm, tid, -1);

    // store: logical row i of the result is physical row rmap[i]
    for (int e = tid; e < n * n; e += kMedThreads) {
        const int i = e % n, j = e / n;
        A[i + (long long)j * lda] = S.sa[S.rmap[i] + j * ld];
    }
    if (tid == 0 && info != nullptr) info[m] = inf;
}

bool getrf_medium_supported(int n) { return n > 32 && n <= kMedMaxN; }

cudaError_t getrf_medium_launch(cudaStream_t st, float* const* Aarray, int n, int lda, int* piv, int* info,
                                int batch)
{
    const MedLayout L(n, kMedPB);
    static bool configured = false;
    if (!configured) {
        const MedLayout big(kMedMaxN, kMedPB);
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
