// aclblasSgetrsBatched, n <= 32, trans N: instantiations of getrs_small.cuh.
#include "getrs_small.cuh"

namespace opsblas {

void getrs_small_dispatch_n(int n, cudaStream_t st, const float* const* Aarray, int lda, const int* ipiv,
                           float* const* Barray, int ldb, int nrhs, int batch)
{
    switch (n) {
#define OPSBLAS_GETRS_CASE(NN)                                                                                      \
    case NN:                                                                                                        \
        launch_getrs_n<NN, false>(st, Aarray, lda, ipiv, Barray, ldb, nrhs, batch);                                 \
        break;
        OPSBLAS_FOR_N_1_32(OPSBLAS_GETRS_CASE)
#undef OPSBLAS_GETRS_CASE
        default:
            break;
    }
}

}  // namespace opsblas
