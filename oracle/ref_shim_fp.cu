// Host shim that launches the reference's own ray-driven cone-beam kernel
// (kernelkit/cuda/cone_fp.cu, rendered from its Jinja2 template by
// oracle/build_ref.py and force-included into this translation unit).
//
// Test infrastructure only: it turns the reference into a checker on the
// GPU. It replays the reference's host-side behaviour:
//   * the volume goes into a 3D CUDA array read through a texture object
//     with border addressing and linear filtering (kernelkit/kernel.py:22-32,
//     47-96);
//   * the 12 per-angle parameter arrays go to __constant__ memory
//     (kernels/cone_fp.py:341-363), in groups of at most KKREF_MAX_PROJS
//     angles because of the compiled constant-array size;
//   * the launch loop groups consecutive angles by dominant ray axis and
//     launches one grid per 16-slice slab (kernels/cone_fp.py:206-262).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#ifndef KKREF_MAX_PROJS
#define KKREF_MAX_PROJS 1024
#endif
#ifndef KKREF_SLICES
#define KKREF_SLICES 16
#endif
#ifndef KKREF_PIX
#define KKREF_PIX 32
#endif

static int kkref_fp_err(cudaError_t e) { return e == cudaSuccess ? 0 : (int)e; }
#define KKREF_CHECK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { rc = (int)e_; goto done; } } while (0)

// vol: device float32 vol[nx][ny][nz] (z fastest).
// params: host (n, 12) float32 rows = src.xyz, corner.xyz, u*pw.xyz, v*ph.xyz.
// axes: host (n,) dominant axis per angle. out_scale: host (3, 3).
// proj: device (n, rows, cols) float32, overwritten.
// ms: kernel-only milliseconds (the launches, not the texture copy).
extern "C" int kkref_cone_fp(const float* vol, int nx, int ny, int nz,
                             const float* params, const int* axes, int n,
                             int rows, int cols, const float* out_scale,
                             float* proj, float* ms, void* stream_ptr) {
    cudaStream_t stream = (cudaStream_t)stream_ptr;
    int rc = 0;
    cudaArray_t arr = nullptr;
    cudaTextureObject_t tex = 0;
    unsigned long long* d_ptrs = nullptr;
    unsigned long long* h_ptrs = nullptr;
    float* h_soa = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float total_ms = 0.f;
    {
        cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
        KKREF_CHECK(cudaMalloc3DArray(&arr, &ch, make_cudaExtent(nz, ny, nx)));
        cudaMemcpy3DParms cp;
        memset(&cp, 0, sizeof(cp));
        cp.srcPtr = make_cudaPitchedPtr((void*)vol, (size_t)nz * sizeof(float), nz, ny);
        cp.dstArray = arr;
        cp.extent = make_cudaExtent(nz, ny, nx);
        cp.kind = cudaMemcpyDeviceToDevice;
        KKREF_CHECK(cudaMemcpy3DAsync(&cp, stream));
        cudaResourceDesc rd;
        memset(&rd, 0, sizeof(rd));
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = arr;
        cudaTextureDesc td;
        memset(&td, 0, sizeof(td));
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 0;
        KKREF_CHECK(cudaCreateTextureObject(&tex, &rd, &td, nullptr));

        h_ptrs = (unsigned long long*)malloc(sizeof(unsigned long long) * n);
        for (int i = 0; i < n; ++i)
            h_ptrs[i] = (unsigned long long)(proj + (size_t)i * rows * cols);
        KKREF_CHECK(cudaMalloc(&d_ptrs, sizeof(unsigned long long) * n));
        KKREF_CHECK(cudaMemcpyAsync(d_ptrs, h_ptrs, sizeof(unsigned long long) * n,
                                    cudaMemcpyHostToDevice, stream));
        KKREF_CHECK(cudaMemsetAsync(proj, 0, sizeof(float) * (size_t)n * rows * cols, stream));
        h_soa = (float*)malloc(sizeof(float) * 12 * KKREF_MAX_PROJS);
        KKREF_CHECK(cudaEventCreate(&e0));
        KKREF_CHECK(cudaEventCreate(&e1));
        const int vshape[3] = {nx, ny, nz};
        for (int g0 = 0; g0 < n; g0 += KKREF_MAX_PROJS) {
            int cnt = n - g0 < KKREF_MAX_PROJS ? n - g0 : KKREF_MAX_PROJS;
            for (int k = 0; k < 12; ++k)
                for (int i = 0; i < cnt; ++i)
                    h_soa[k * KKREF_MAX_PROJS + i] = params[(size_t)(g0 + i) * 12 + k];
            float* syms[12];
            KKREF_CHECK(cudaGetSymbolAddress((void**)&syms[0], srcsX));
            KKREF_CHECK(cudaGetSymbolAddress((void**)&syms[1], srcsY));
            KKREF_CHECK(cudaGetSymbolAddress((void**)&syms[2], srcsZ));
            KKREF_CHECK(cudaGetSymbolAddress((void**)&syms[3], detsSX));
            KKREF_CHECK(cudaGetSymbolAddress((void**)&syms[4], detsSY));
            KKREF_CHECK(cudaGetSymbolAddress((void**)&syms[5], detsSZ));
            KKREF_CHECK(cudaGetSymbolAddress((void**)&syms[6], detsUX));
            KKREF_CHECK(cudaGetSymbolAddress((void**)&syms[7], detsUY));
            KKREF_CHECK(cudaGetSymbolAddress((void**)&syms[8], detsUZ));
            KKREF_CHECK(cudaGetSymbolAddress((void**)&syms[9], detsVX));
            KKREF_CHECK(cudaGetSymbolAddress((void**)&syms[10], detsVY));
            KKREF_CHECK(cudaGetSymbolAddress((void**)&syms[11], detsVZ));
            for (int k = 0; k < 12; ++k)
                KKREF_CHECK(cudaMemcpyAsync(syms[k], h_soa + k * KKREF_MAX_PROJS,
                                            sizeof(float) * cnt, cudaMemcpyHostToDevice, stream));
            KKREF_CHECK(cudaStreamSynchronize(stream));
            KKREF_CHECK(cudaEventRecord(e0, stream));
            int start = 0;
            for (int i = 1; i <= cnt; ++i) {
                if (i < cnt && axes[g0 + i] == axes[g0 + start]) continue;
                int ax = axes[g0 + start];
                for (int sl = 0; sl < vshape[ax]; sl += KKREF_SLICES) {
                    dim3 grid((cols + KKREF_PIX - 1) / KKREF_PIX,
                              (rows + KKREF_PIX - 1) / KKREF_PIX, i - start);
                    dim3 block(KKREF_PIX);
                    float** pp = (float**)(d_ptrs + g0);
                    const float* os = out_scale + 3 * ax;
                    if (ax == 0)
                        cone_fp<DIR_X><<<grid, block, 0, stream>>>(tex, pp, sl, start, nx, ny, nz, cnt,
                                                                   rows, cols, cnt, rows, cols, os[0], os[1], os[2]);
                    else if (ax == 1)
                        cone_fp<DIR_Y><<<grid, block, 0, stream>>>(tex, pp, sl, start, nx, ny, nz, cnt,
                                                                   rows, cols, cnt, rows, cols, os[0], os[1], os[2]);
                    else
                        cone_fp<DIR_Z><<<grid, block, 0, stream>>>(tex, pp, sl, start, nx, ny, nz, cnt,
                                                                   rows, cols, cnt, rows, cols, os[0], os[1], os[2]);
                    KKREF_CHECK(cudaGetLastError());
                }
                start = i;
            }
            KKREF_CHECK(cudaEventRecord(e1, stream));
            KKREF_CHECK(cudaEventSynchronize(e1));
            float t = 0.f;
            KKREF_CHECK(cudaEventElapsedTime(&t, e0, e1));
            total_ms += t;
        }
    }
done:
    if (ms) *ms = total_ms;
    cudaStreamSynchronize(stream);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (tex) cudaDestroyTextureObject(tex);
    if (arr) cudaFreeArray(arr);
    if (d_ptrs) cudaFree(d_ptrs);
    free(h_ptrs);
    free(h_soa);
    (void)kkref_fp_err;
    return rc;
}
