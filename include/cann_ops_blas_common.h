/*
 * Shared enumerations of the aclblas C API, B200 build.
 *
 * Names and integer values are those of the reference API so that a caller compiled against
 * hicann/ops-blas links against this library unchanged:
 *   aclblasStatus_t       include/cann_ops_blas_common.h:18-31
 *   aclblasOperation_t    include/cann_ops_blas_common.h:55-59
 *   aclblasComputeType_t  include/cann_ops_blas_common.h:81-93
 *   aclblasGemmAlgo_t     include/cann_ops_blas_common.h:97-107
 * The header is plain C (the reference's is C++-only) so that C, Go (cgo) and ctypes callers
 * can use it as well.
 */
#ifndef OPSBLAS_B200_COMMON_H
#define OPSBLAS_B200_COMMON_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum aclblasStatus {
    ACLBLAS_STATUS_SUCCESS = 0,
    ACLBLAS_STATUS_NOT_INITIALIZED = 1,
    ACLBLAS_STATUS_ALLOC_FAILED = 2,
    ACLBLAS_STATUS_INVALID_VALUE = 3,
    ACLBLAS_STATUS_MAPPING_ERROR = 4,
    ACLBLAS_STATUS_EXECUTION_FAILED = 5,
    ACLBLAS_STATUS_INTERNAL_ERROR = 6,
    ACLBLAS_STATUS_NOT_SUPPORTED = 7,
    ACLBLAS_STATUS_ARCH_MISMATCH = 8,
    ACLBLAS_STATUS_HANDLE_IS_NULLPTR = 9,
    ACLBLAS_STATUS_INVALID_ENUM = 10,
    ACLBLAS_STATUS_UNKNOWN = 11
} aclblasStatus_t;

#ifndef ACLBLAS_OPERATION_DECLARED
#define ACLBLAS_OPERATION_DECLARED
typedef enum aclblasOperation {
    ACLBLAS_OP_N = 111,
    ACLBLAS_OP_T = 112,
    ACLBLAS_OP_C = 113
} aclblasOperation_t;
#endif

/* Single-precision complex, real part first (include/cann_ops_blas_common.h:67-71); the layout
 * of cuComplex / std::complex<float>. */
typedef struct aclblasComplex {
    float real;
    float imag;
} aclblasComplex;

typedef enum aclblasComputeType {
    ACLBLAS_COMPUTE_16F = 0,
    ACLBLAS_COMPUTE_16F_PEDANTIC = 1,
    ACLBLAS_COMPUTE_32F = 2,
    ACLBLAS_COMPUTE_32F_PEDANTIC = 3,
    ACLBLAS_COMPUTE_32F_FAST_16F = 4,
    ACLBLAS_COMPUTE_32F_FAST_16BF = 5,
    ACLBLAS_COMPUTE_32F_FAST_TF32 = 6,
    ACLBLAS_COMPUTE_64F = 7,
    ACLBLAS_COMPUTE_64F_PEDANTIC = 8,
    ACLBLAS_COMPUTE_32I = 9,
    ACLBLAS_COMPUTE_32I_PEDANTIC = 10
} aclblasComputeType_t;

typedef enum aclblasGemmAlgo {
    ACLBLAS_GEMM_DEFAULT = 0,
    ACLBLAS_GEMM_ALGO0 = 1,
    ACLBLAS_GEMM_ALGO1 = 2,
    ACLBLAS_GEMM_ALGO2 = 3,
    ACLBLAS_GEMM_ALGO3 = 4,
    ACLBLAS_GEMM_ALGO4 = 5,
    ACLBLAS_GEMM_ALGO5 = 6,
    ACLBLAS_GEMM_ALGO6 = 7,
    ACLBLAS_GEMM_ALGO7 = 8
} aclblasGemmAlgo_t;

/* Host-side LAPACK-style info of the QR entry points (include/cann_ops_blas_common.h:122-132
 * of the reference): 0, or -k when the k-th argument (handle and info not counted) is invalid. */
typedef enum aclblasLapackInfo {
    ACLBLAS_LAPACK_INFO_OK = 0,
    ACLBLAS_LAPACK_INFO_ARG_1 = -1,
    ACLBLAS_LAPACK_INFO_ARG_2 = -2,
    ACLBLAS_LAPACK_INFO_ARG_3 = -3,
    ACLBLAS_LAPACK_INFO_ARG_4 = -4,
    ACLBLAS_LAPACK_INFO_ARG_5 = -5,
    ACLBLAS_LAPACK_INFO_ARG_6 = -6,
    ACLBLAS_LAPACK_INFO_ARG_7 = -7,
    ACLBLAS_LAPACK_INFO_ARG_8 = -8
} aclblasLapackInfo_t;

#ifdef __cplusplus
}
#endif

#endif /* OPSBLAS_B200_COMMON_H */
