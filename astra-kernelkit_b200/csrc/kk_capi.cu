// Error state and version of the C ABI (include/kk.h).
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

#include <map>
#include <mutex>
#include <utility>

#include "kk_common.cuh"

static thread_local char g_last_error[512] = "";

int kk_fail(int status, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return status;
}

int kk_check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return kk_fail(KK_ERR_CUDA, "%s: launch failed: %s", what, cudaGetErrorString(e));
    return KK_OK;
}

extern "C" const char* kk_last_error(void) { return g_last_error; }

extern "C" int kk_abi_version(void) { return KK_ABI_VERSION; }

// Opt-in to more than 48 KB of dynamic shared memory: a per-device
// function attribute, so it is set once per (kernel, device) pair, from any
// thread, before the first launch that needs it.
int kk_allow_smem(const void* kernel, size_t bytes, const char* who) {
    if (bytes <= 48 * 1024) return KK_OK;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return kk_fail(KK_ERR_CUDA, "%s: %s", who, cudaGetErrorString(e));
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> done;
    std::lock_guard<std::mutex> lock(mu);
    size_t& have = done[std::make_pair(kernel, dev)];
    if (have >= bytes) return KK_OK;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess)
        return kk_fail(KK_ERR_CUDA, "%s: %zu bytes of shared memory: %s", who, bytes, cudaGetErrorString(e));
    have = bytes;
    return KK_OK;
}

// Streaming multiprocessors of the current device (cached per device).
int kk_sm_count() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 148;
    static std::mutex mu;
    static std::map<int, int> seen;
    std::lock_guard<std::mutex> lock(mu);
    auto it = seen.find(dev);
    if (it != seen.end()) return it->second;
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    seen[dev] = n;
    return n;
}
