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
};

namespace opsblas {

constexpr size_t kDefaultWorkspaceBytes = 32u * 1024u * 1024u;

// Logging through the aclblasLoggerConfigure / aclblasSetLoggerCallback configuration.
void log_error(const char* api, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
void log_info(const char* api, const char* fmt, ...) __attribute__((format(printf, 2, 3)));

// Number of SMs of the current device (cached per device).
int sm_count();

// Maps the error of a kernel launch to a status and logs it. SUCCESS when err == cudaSuccess.
aclblasStatus_t launch_status(const char* api, cudaError_t err);

inline int max1(int n) { return n > 1 ? n : 1; }

}  // namespace opsblas
