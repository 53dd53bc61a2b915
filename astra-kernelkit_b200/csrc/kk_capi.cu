// Error state and version of the C ABI (include/kk.h).
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

#include <map>
#include <mutex>
#include <utility>

#include "kk_common.cuh"
#include "kk_async.cuh"

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

// cuTensorMapEncodeTiled, looked up once through the runtime's driver
// entry point, so the library needs no link-time libcuda.
typedef CUresult (*kk_encode_tiled_fn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                       const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                       CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int kk_encode_tile_map(CUtensorMap* map, CUtensorMapDataType type, int rank, void* base, const uint64_t* dims,
                       const uint64_t* strides_bytes, const uint32_t* box, const char* who) {
    static std::once_flag once;
    static kk_encode_tiled_fn fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (kk_encode_tiled_fn)p;
    });
    if (!fn) return kk_fail(KK_ERR_CUDA, "%s: cuTensorMapEncodeTiled is not available", who);
    cuuint64_t d[5], s[4];
    cuuint32_t b[5], e[5];
    for (int k = 0; k < rank; ++k) {
        d[k] = dims[k];
        b[k] = box[k];
        e[k] = 1;
        if (k + 1 < rank) s[k] = strides_bytes[k];
    }
    const CUresult r = fn(map, type, (cuuint32_t)rank, base, d, s, b, e, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return kk_fail(KK_ERR_CUDA, "%s: cuTensorMapEncodeTiled failed (%d)", who, (int)r);
    return KK_OK;
}
