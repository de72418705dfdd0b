// Internal declarations shared by the translation units of libopsblas_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "cann_ops_blas.h"

// Library version reported by aclblasGetVersion: MAJOR*10000 + MINOR*100 + PATCH.
#define OPSBLAS_B200_VERSION 10000

// Opaque handle behind aclblasHandle_t. Mirrors the reference's {stream, workspace,
// workspace_size, owner} (blas/common/helper/aclblas_handle_internal.h:47-58) and adds the
// device the handle was created on.
enum class WorkspaceOwner { Library, User };

struct _aclblas_handle {
    cudaStream_t stream = nullptr;
    void* workspace = nullptr;
    size_t workspace_size = 0;
    WorkspaceOwner owner = WorkspaceOwner::Library;
    size_t library_workspace_size = 0;
    int device = 0;
    // Device status word (4 bytes of device memory owned by the handle): kernels launched through
    // this handle OR in a kStatus* bit when a bounded wait of theirs gives up.
    unsigned* dstatus = nullptr;
    // Device memory for the tcgen05 GEMM's per-CTA TMA tensor maps (kTensorMapSlotBytes): each
    // persistent CTA rewrites its maps' base address there when it moves to another matrix.
    void* tmslots = nullptr;
};

namespace opsblas {

constexpr size_t kDefaultWorkspaceBytes = 32u * 1024u * 1024u;
constexpr size_t kTensorMapSlotBytes = 512u * 3u * 128u;  // up to 512 CTAs x (A, B, C) x 128-byte map

// Logging through the aclblasLoggerConfigure / aclblasSetLoggerCallback configuration.
void log_error(const char* api, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
void log_info(const char* api, const char* fmt, ...) __attribute__((format(printf, 2, 3)));

// Bits of the handle's device status word (aclblasGetDeviceStatus).
constexpr unsigned kStatusBulkCopyTimeout = 1u << 0;  // getrf: a bulk copy of a matrix did not land
constexpr unsigned kStatusTmemLuTimeout = 1u << 1;    // TMEM LU: the trailing-update MMAs did not complete
constexpr unsigned kStatusTcGemmTimeout = 1u << 2;    // tcgen05 GEMM: the MMAs of a tile did not complete

// Polls of a bounded device wait: `def`, unless a test has set an override
// (opsblas_test_set_wait_limit) to make the waits give up.
unsigned wait_limit(unsigned def);

// Number of SMs of the current device (cached per device).
int sm_count();

// Raises a kernel's dynamic shared-memory limit to at least `bytes` on the current device. The
// attribute is per device, so the set-up is remembered per (device, kernel) under a lock; the
// result of cudaFuncSetAttribute is returned (a cached success afterwards). The record does not
// survive a cudaDeviceReset of that device: the library must not be used across one.
cudaError_t ensure_smem_limit(const void* func, int bytes);

template <typename K>
inline cudaError_t ensure_smem_limit(K* kernel, int bytes)
{
    return ensure_smem_limit(reinterpret_cast<const void*>(kernel), bytes);
}

// Maps the error of a kernel launch to a status and logs it. SUCCESS when err == cudaSuccess.
aclblasStatus_t launch_status(const char* api, cudaError_t err);

inline int max1(int n) { return n > 1 ? n : 1; }

// Validation-free launchers shared by the entry points (getrs.cu, gemm_batched_ex.cu).
// getrs_launch skips every matrix whose Barray entry is NULL (the refinement's correction solves
// pass NULL for converged matrices).
cudaError_t getrs_launch(cudaStream_t st, bool trans, int n, int nrhs, const float* const* Aarray, int lda,
                         const int* devIpiv, float* const* Barray, int ldb, int batchCount);
// getrs_blk.cu: trans N, n > 32, blocked substitution with the right-hand sides in shared memory.
bool getrs_blk_supported(int n);
cudaError_t getrs_blk_launch(cudaStream_t st, int n, int nrhs, const float* const* Aarray, int lda, const int* ipiv,
                             float* const* Barray, int ldb, int batch);
// getrs_trhs.cu: trans T / C, n > 32, one thread per right-hand side (reference order).
bool getrs_trhs_supported(int n);
cudaError_t getrs_trhs_launch(cudaStream_t st, int n, int nrhs, const float* const* Aarray, int lda, const int* ipiv,
                              float* const* Barray, int ldb, int batch);
bool getrs_nrhs_preferred(int n, int nrhs, int batch);
cudaError_t getrs_nrhs_launch(cudaStream_t st, int n, int nrhs, const float* const* Aarray, int lda, const int* ipiv,
                              float* const* Barray, int ldb, int batch);
// Element types of the batched GEMMs' operands in global memory.
enum class GemmElem { F32, F16, BF16, E4M3, E5M2 };

// Operand kinds of the tcgen05 GEMM: native FP16 / BF16 / FP8 (E4M3, E5M2), and FP32 operands
// rounded to TF32 (optionally split into TF32 high and low parts) or converted to BF16.
enum class TcIn { F16, BF16, E4M3, E5M2, F32_TF32, F32_BF16 };

// C = alpha * op(A) * op(B) + beta * C, FP32 operands; round: 0 none, 1 TF32, 2 BF16.
cudaError_t gemm_f32_launch(cudaStream_t st, bool transA, bool transB, int m, int n, int k, float alpha,
                            const float* const* A, int lda, const float* const* B, int ldb, float beta,
                            float* const* C, int ldc, int batch, int round);

// gemm_tc.cu: C = alpha * op(A) * op(B) + beta * C on the tcgen05 tensor cores, FP32 accumulation.
// *_off are element offsets added to every matrix pointer; status: the handle's status word.
// Typed form: A / B of kinds ta / tb (both FP8, or equal), C of type tc (F32 for FP32 operands,
// F16 for FP16 and FP8, BF16 for BF16).
// tmslots: the handle's tensor-map slots (native FP16 / BF16 / FP8 operands then arrive by TMA),
// or nullptr (copies by cp.async).
cudaError_t gemm_tc_typed_launch(cudaStream_t st, TcIn ta, TcIn tb, GemmElem tc, bool split, bool transA,
                                 bool transB, int m, int n, int k, float alpha, const void* const* A, long long a_off,
                                 int lda, const void* const* B, long long b_off, int ldb, float beta, void* const* C,
                                 long long c_off, int ldc, int batch, unsigned* status, void* tmslots);
// FP32 operands rounded to TF32; split = 1 adds the low-part products for about FP32 accuracy.
cudaError_t gemm_tc_launch(cudaStream_t st, bool transA, bool transB, int m, int n, int k, float alpha,
                           const float* const* A, long long a_off, int lda, const float* const* B, long long b_off,
                           int ldb, float beta, float* const* C, long long c_off, int ldc, int batch, int split,
                           unsigned* status, void* tmslots);

// Trailing update of the blocked mixed-precision LU: for every matrix b, the m x m block of C[b] at
// element offset c_off (column-major, leading dimension ldc) becomes
// C(r, c) - sum_k Aop[b][k + 32 r] * Bop[b][k + 32 c] with split-TF32 tensor-core products; Aop
// and Bop hold 32 K-contiguous values per row or column (leading dimension 32), each given as its
// TF32 high plane followed, lo_rows rows further, by its low plane.
cudaError_t gemm_tc_lu_update(cudaStream_t st, int m, const float* const* Aop, const float* const* Bop,
                              float* const* C, long long c_off, int ldc, int batch, int lo_rows, unsigned* status,
                              void* tmslots);

// refine.cu: out[i] = base + i * stride (floats), i < count.
__global__ void init_ptr_array_kernel(float** out, float* base, long long stride, int count);

// getrf_blocked_tc.cu: 256 < n <= 1024, blocked mixed-precision LU (FP32 panels, split-TF32
// tensor-core trailing update): reads A (lda), writes the factors to LU (ldlu; LU must not overlap
// A); scratch: getrf_blocked_tc_scratch_bytes(n, batch) bytes of device memory (256-byte aligned).
bool getrf_blocked_tc_supported(int n);
size_t getrf_blocked_tc_scratch_bytes(int n, int batch);
cudaError_t getrf_blocked_tc_launch(cudaStream_t st, const float* const* Aarray, int lda, float* const* LUarray, int n,
                                    int ldlu, int* piv, int* info, int batch, void* scratch, unsigned* status,
                                    void* tmslots);

// getrf_blocked_tc.cu: 128 < n <= 1024, the plain FP32 blocked LU on a by-rows copy made in place
// (bit-identical to the reference's unblocked order); piv and info may be nullptr (no-pivot mode:
// piv == nullptr); stat: batch ints of device scratch (the matrices' stop codes).
bool getrf_rows_supported(int n, int batch);
// aclblasSgetrfBatched with the blocked path's stop codes in `stat` (batch ints of device memory
// that the caller does not use otherwise; nullptr: the blocked path is not taken).
aclblasStatus_t getrf_batched_impl(aclblasHandle_t handle, int n, float* const Aarray[], int lda, int* PivotArray,
                                   int* infoArray, int batchSize, int* stat);
cudaError_t getrf_rows_launch(cudaStream_t st, float* const* Aarray, int n, int lda, int* piv, int* info, int* stat,
                              int batch);

// getrf_tmem.cu: 32 < n <= 256, mixed-precision LU with the matrix resident in TMEM.
bool getrf_tmem_supported(int n);
// Reads A (lda), writes the factors to LU (ldlu); A may equal LU. prec 1: TF32 split update,
// 2: BF16 split update.
cudaError_t getrf_tmem_launch(cudaStream_t st, const float* const* Aarray, int lda, float* const* LUarray, int n,
                              int ldlu, int* piv, int* info, int batch, int prec, unsigned* status);

// getrf_large.cu: 32 < n <= 640, matrix in global memory, the reference's operation order.
bool getrf_large_supported(int n);
cudaError_t getrf_large_launch(cudaStream_t st, float* const* Aarray, int n, int lda, int* piv, int* info, int batch);

// getrf_reg.cu: 32 < n <= 128, matrix in registers; shape = rows per lane x warps per matrix.
bool getrf_reg_supported(int n);
bool reg_shape_valid(int n, int rows, int warps);
void reg_default_shape(int n, int& rows, int& warps);
cudaError_t getrf_reg_launch(cudaStream_t st, float* const* Aarray, int n, int lda, int* piv, int* info, int batch,
                             int rows, int warps);

}  // namespace opsblas
