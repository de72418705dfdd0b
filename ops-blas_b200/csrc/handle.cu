// Handle, stream, workspace, version and logger entry points of the aclblas C API.
//
// Semantics follow blas/common/helper/aclblas_auxiliary.cpp:24-148 and
// blas/common/helper/aclblas_logger_manager.cpp:19-48 of the reference, over CUDA.
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <map>
#include <mutex>
#include <new>
#include <utility>

#include "internal.h"

namespace opsblas {
namespace {

struct LoggerState {
    std::mutex mu;
    bool on = false;
    bool to_stdout = false;
    bool to_stderr = false;
    const char* file = nullptr;
    aclblasLogCallback callback = nullptr;
};

LoggerState& logger()
{
    static LoggerState s;
    return s;
}

void emit(const char* level, const char* api, const char* fmt, va_list ap)
{
    LoggerState& L = logger();
    std::lock_guard<std::mutex> g(L.mu);
    if (!L.on && L.callback == nullptr) return;
    char body[768];
    std::vsnprintf(body, sizeof(body), fmt, ap);
    char line[1024];
    std::snprintf(line, sizeof(line), "[opsblas_b200][%s] %s: %s", level, api, body);
    if (L.callback) L.callback(line);
    if (!L.on) return;
    if (L.to_stdout) std::fprintf(stdout, "%s\n", line);
    if (L.to_stderr) std::fprintf(stderr, "%s\n", line);
    if (L.file) {
        if (FILE* f = std::fopen(L.file, "a")) {
            std::fprintf(f, "%s\n", line);
            std::fclose(f);
        }
    }
}

}  // namespace

void log_error(const char* api, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    emit("E", api, fmt, ap);
    va_end(ap);
}

void log_info(const char* api, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    emit("I", api, fmt, ap);
    va_end(ap);
}

int sm_count()
{
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cache[dev] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        cache[dev] = v;
    }
    return cache[dev];
}

static std::atomic<unsigned> g_wait_limit_override{0xffffffffu};

unsigned wait_limit(unsigned def)
{
    const unsigned v = g_wait_limit_override.load(std::memory_order_relaxed);
    return v == 0xffffffffu ? def : v;
}

cudaError_t ensure_smem_limit(const void* func, int bytes)
{
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, int> done;  // (device, kernel) -> limit set there
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    std::lock_guard<std::mutex> lock(mu);
    auto it = done.find({dev, func});
    if (it != done.end() && it->second >= bytes) return cudaSuccess;
    err = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (err == cudaSuccess) done[{dev, func}] = bytes;
    return err;
}

aclblasStatus_t launch_status(const char* api, cudaError_t err)
{
    if (err == cudaSuccess) return ACLBLAS_STATUS_SUCCESS;
    log_error(api, "kernel launch failed: %s", cudaGetErrorString(err));
    if (err == cudaErrorNoKernelImageForDevice || err == cudaErrorInvalidDeviceFunction)
        return ACLBLAS_STATUS_ARCH_MISMATCH;
    return ACLBLAS_STATUS_EXECUTION_FAILED;
}

}  // namespace opsblas

using opsblas::log_error;

static aclblasStatus_t sync_stream(_aclblas_handle* h)
{
    return cudaStreamSynchronize(h->stream) == cudaSuccess ? ACLBLAS_STATUS_SUCCESS : ACLBLAS_STATUS_EXECUTION_FAILED;
}

static aclblasStatus_t alloc_library_workspace(_aclblas_handle* h, size_t bytes)
{
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return ACLBLAS_STATUS_ALLOC_FAILED;
    }
    h->workspace = p;
    h->workspace_size = bytes;
    h->library_workspace_size = bytes;
    h->owner = WorkspaceOwner::Library;
    return ACLBLAS_STATUS_SUCCESS;
}

static void free_library_workspace(_aclblas_handle* h)
{
    if (h->owner == WorkspaceOwner::Library && h->workspace != nullptr) {
        cudaFree(h->workspace);
        h->workspace = nullptr;
        h->workspace_size = 0;
    }
}

extern "C" {

aclblasStatus_t aclblasCreate(aclblasHandle_t* handle)
{
    if (handle == nullptr) return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    if (*handle != nullptr) return ACLBLAS_STATUS_INVALID_VALUE;
    auto* h = new (std::nothrow) _aclblas_handle();
    if (h == nullptr) return ACLBLAS_STATUS_ALLOC_FAILED;
    if (cudaGetDevice(&h->device) != cudaSuccess) {
        cudaGetLastError();
        delete h;
        log_error("aclblasCreate", "no CUDA device is available");
        return ACLBLAS_STATUS_NOT_INITIALIZED;
    }
    aclblasStatus_t st = alloc_library_workspace(h, opsblas::kDefaultWorkspaceBytes);
    if (st != ACLBLAS_STATUS_SUCCESS) {
        delete h;
        log_error("aclblasCreate", "cannot allocate the %zu-byte default workspace", opsblas::kDefaultWorkspaceBytes);
        return st;
    }
    if (cudaMalloc(&h->dstatus, sizeof(unsigned)) != cudaSuccess ||
        cudaMemset(h->dstatus, 0, sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&h->tmslots, opsblas::kTensorMapSlotBytes) != cudaSuccess) {
        cudaGetLastError();
        if (h->dstatus) cudaFree(h->dstatus);
        if (h->tmslots) cudaFree(h->tmslots);
        free_library_workspace(h);
        delete h;
        log_error("aclblasCreate", "cannot allocate the device status word and tensor-map slots");
        return ACLBLAS_STATUS_ALLOC_FAILED;
    }
    *handle = h;
    return ACLBLAS_STATUS_SUCCESS;
}

aclblasStatus_t aclblasDestroy(aclblasHandle_t handle)
{
    if (handle == nullptr) return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    if (sync_stream(handle) != ACLBLAS_STATUS_SUCCESS) {
        log_error("aclblasDestroy", "stream synchronization failed before handle destruction");
        return ACLBLAS_STATUS_EXECUTION_FAILED;
    }
    free_library_workspace(handle);
    if (handle->dstatus) cudaFree(handle->dstatus);
    if (handle->tmslots) cudaFree(handle->tmslots);
    delete handle;
    return ACLBLAS_STATUS_SUCCESS;
}

aclblasStatus_t aclblasGetDeviceStatus(aclblasHandle_t handle, unsigned int* flags)
{
    static const char* kApi = "aclblasGetDeviceStatus";
    if (handle == nullptr) return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    if (flags == nullptr) {
        log_error(kApi, "flags must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    unsigned v = 0;
    cudaError_t err = cudaMemcpyAsync(&v, handle->dstatus, sizeof(v), cudaMemcpyDeviceToHost, handle->stream);
    if (err == cudaSuccess) err = cudaMemsetAsync(handle->dstatus, 0, sizeof(unsigned), handle->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(handle->stream);
    if (err != cudaSuccess) {
        log_error(kApi, "reading the device status failed: %s", cudaGetErrorString(err));
        return ACLBLAS_STATUS_EXECUTION_FAILED;
    }
    *flags = v;
    if (v != 0) {
        log_error(kApi, "a kernel gave up a bounded wait (flags 0x%x); its results are incomplete", v);
        return ACLBLAS_STATUS_EXECUTION_FAILED;
    }
    return ACLBLAS_STATUS_SUCCESS;
}

// Test hook for the failure path (not part of the API): every bounded device wait launched after
// this call polls at most `polls` times (0 = gives up at once); 0xffffffff restores the defaults.
__attribute__((visibility("default"))) void opsblas_test_set_wait_limit(unsigned int polls)
{
    opsblas::g_wait_limit_override.store(polls, std::memory_order_relaxed);
}

aclblasStatus_t aclblasSetStream(aclblasHandle_t handle, aclrtStream stream)
{
    if (handle == nullptr) return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    aclblasStatus_t st = sync_stream(handle);
    if (st != ACLBLAS_STATUS_SUCCESS) return st;
    handle->stream = static_cast<cudaStream_t>(stream);
    // Switching streams reverts to the library workspace (aclblas_auxiliary.cpp:86-89).
    if (handle->owner == WorkspaceOwner::Library && handle->workspace != nullptr) return ACLBLAS_STATUS_SUCCESS;
    size_t bytes = handle->library_workspace_size ? handle->library_workspace_size : opsblas::kDefaultWorkspaceBytes;
    handle->workspace = nullptr;
    handle->workspace_size = 0;
    return alloc_library_workspace(handle, bytes);
}

aclblasStatus_t aclblasGetStream(aclblasHandle_t handle, aclrtStream* stream)
{
    if (handle == nullptr) return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    if (stream == nullptr) return ACLBLAS_STATUS_INVALID_VALUE;
    *stream = static_cast<aclrtStream>(handle->stream);
    return ACLBLAS_STATUS_SUCCESS;
}

aclblasStatus_t aclblasSetWorkspace(aclblasHandle_t handle, void* workspace, size_t workspaceSize)
{
    if (handle == nullptr) return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    if (workspace == nullptr || workspaceSize == 0) return ACLBLAS_STATUS_INVALID_VALUE;
    if (handle->owner == WorkspaceOwner::User && workspaceSize <= handle->workspace_size) return ACLBLAS_STATUS_SUCCESS;
    aclblasStatus_t st = sync_stream(handle);
    if (st != ACLBLAS_STATUS_SUCCESS) return st;
    if (handle->owner == WorkspaceOwner::Library && handle->workspace != nullptr) {
        handle->library_workspace_size = handle->workspace_size;
        free_library_workspace(handle);
    }
    handle->workspace = workspace;
    handle->workspace_size = workspaceSize;
    handle->owner = WorkspaceOwner::User;
    return ACLBLAS_STATUS_SUCCESS;
}

aclblasStatus_t aclblasGetVersion(aclblasHandle_t handle, int* version)
{
    (void)handle;
    if (version == nullptr) return ACLBLAS_STATUS_INVALID_VALUE;
    *version = OPSBLAS_B200_VERSION;
    return ACLBLAS_STATUS_SUCCESS;
}

aclblasStatus_t aclblasLoggerConfigure(int logIsOn, int logToStdOut, int logToStdErr, const char* logFile)
{
    auto& L = opsblas::logger();
    std::lock_guard<std::mutex> g(L.mu);
    L.on = logIsOn != 0;
    L.to_stdout = logToStdOut != 0;
    L.to_stderr = logToStdErr != 0;
    L.file = logFile;
    return ACLBLAS_STATUS_SUCCESS;
}

aclblasStatus_t aclblasSetLoggerCallback(aclblasLogCallback userCallback)
{
    auto& L = opsblas::logger();
    std::lock_guard<std::mutex> g(L.mu);
    L.callback = userCallback;
    return ACLBLAS_STATUS_SUCCESS;
}

aclblasStatus_t aclblasGetLoggerCallback(aclblasLogCallback* userCallback)
{
    if (userCallback == nullptr) return ACLBLAS_STATUS_INVALID_VALUE;
    auto& L = opsblas::logger();
    std::lock_guard<std::mutex> g(L.mu);
    *userCallback = L.callback;
    return ACLBLAS_STATUS_SUCCESS;
}

}  // extern "C"
