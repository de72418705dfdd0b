/*
 * Minimal stand-in for the two CANN runtime types that the aclblas C API names.
 *
 * The reference API (include/cann_ops_blas.h:13 in hicann/ops-blas) includes the CANN
 * runtime header <acl/acl.h> for `aclrtStream` and `aclDataType`. On a B200 the stream is
 * a CUDA stream: `aclrtStream` is an opaque pointer that this library casts to
 * `cudaStream_t` (NULL selects the legacy default stream, as in CANN and CUDA).
 *
 * The integer values of `aclDataType` below follow the CANN runtime's public enumeration as
 * far as it can be known without a CANN installation; only the five members that
 * aclblasGemmBatchedEx accepts are used by this library. A caller that compiles against the
 * real CANN header passes the same integers for ACL_FLOAT, ACL_FLOAT16 and ACL_BF16; the
 * FP8 values are the ones most likely to differ and are rejected with
 * ACLBLAS_STATUS_NOT_SUPPORTED when unknown.
 */
#ifndef OPSBLAS_B200_ACL_COMPAT_H
#define OPSBLAS_B200_ACL_COMPAT_H

#ifdef __cplusplus
extern "C" {
#endif

typedef void* aclrtStream;
typedef int aclError;

typedef enum {
    ACL_DT_UNDEFINED = -1,
    ACL_FLOAT = 0,
    ACL_FLOAT16 = 1,
    ACL_INT8 = 2,
    ACL_INT32 = 3,
    ACL_UINT8 = 4,
    ACL_INT16 = 6,
    ACL_UINT16 = 7,
    ACL_UINT32 = 8,
    ACL_INT64 = 9,
    ACL_UINT64 = 10,
    ACL_DOUBLE = 11,
    ACL_BOOL = 12,
    ACL_COMPLEX64 = 16,
    ACL_COMPLEX128 = 17,
    ACL_BF16 = 27,
    ACL_FLOAT8_E5M2 = 35,
    ACL_FLOAT8_E4M3FN = 36
} aclDataType;

#ifdef __cplusplus
}
#endif

#endif /* OPSBLAS_B200_ACL_COMPAT_H */
