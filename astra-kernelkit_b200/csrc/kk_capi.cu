// Error state and version of the C ABI (include/kk.h).
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

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
