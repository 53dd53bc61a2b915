// Host shim that launches the reference's own voxel-driven cone-beam
// backprojection kernel (kernelkit/cuda/cone_bp.cu rendered with
// texture='tex2DLayered' by oracle/build_ref.py and force-included here).
//
// Test infrastructure only. Replays the reference's host side:
//   * projections go into a 2D-layered CUDA array read through a texture
//     object with border addressing and linear filtering
//     (projector.py:529-534, kernel.py:91-96);
//   * per-angle Params (3 float4) go to __constant__ memory
//     (kernels/cone_bp.py:168-190), at most KKREF_MAX_PROJS angles per
//     group; larger scans are processed group by group, each group adding
//     into the volume as an additive call would;
//   * the volume is zero-filled (projector.py:586-588) and one grid is
//     launched per 32 angles (kernels/cone_bp.py:293-302).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#ifndef KKREF_MAX_PROJS
#define KKREF_MAX_PROJS 1024
#endif
#ifndef KKREF_BP_PROJS_BLOCK
#define KKREF_BP_PROJS_BLOCK 32
#endif

#define KKREF_CHECK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { rc = (int)e_; goto done; } } while (0)

// proj: device float32 (n, rows, cols). h_params: host (n, 12) float32 laid
// out as the reference's Params (numU.xyzw, numV.xyzw, den.xyzw).
// vol: device float32 vol[nx][ny][nz], overwritten.
extern "C" int kkref_cone_bp(const float* proj, int n, int rows, int cols,
                             const float* h_params, float* vol, int nx, int ny,
                             int nz, float vox_vol, float* ms, void* stream_ptr) {
    cudaStream_t stream = (cudaStream_t)stream_ptr;
    int rc = 0;
    cudaArray_t arr = nullptr;
    cudaTextureObject_t tex = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float total_ms = 0.f;
    {
        KKREF_CHECK(cudaMemsetAsync(vol, 0, sizeof(float) * (size_t)nx * ny * nz, stream));
        KKREF_CHECK(cudaEventCreate(&e0));
        KKREF_CHECK(cudaEventCreate(&e1));
        Params* d_params = nullptr;
        KKREF_CHECK(cudaGetSymbolAddress((void**)&d_params, params));
        for (int g0 = 0; g0 < n; g0 += KKREF_MAX_PROJS) {
            int cnt = n - g0 < KKREF_MAX_PROJS ? n - g0 : KKREF_MAX_PROJS;
            cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
            KKREF_CHECK(cudaMalloc3DArray(&arr, &ch, make_cudaExtent(cols, rows, cnt), cudaArrayLayered));
            cudaMemcpy3DParms cp;
            memset(&cp, 0, sizeof(cp));
            cp.srcPtr = make_cudaPitchedPtr((void*)(proj + (size_t)g0 * rows * cols),
                                            (size_t)cols * sizeof(float), cols, rows);
            cp.dstArray = arr;
            cp.extent = make_cudaExtent(cols, rows, cnt);
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
            KKREF_CHECK(cudaMemcpyAsync(d_params, h_params + (size_t)g0 * 12, sizeof(float) * 12 * cnt,
                                        cudaMemcpyHostToDevice, stream));
            KKREF_CHECK(cudaStreamSynchronize(stream));
            // voxels_per_block = (6, 32, 16); blocks = ceil(shape / vpb)
            int b0 = (nx + 5) / 6, b1 = (ny + 31) / 32, b2 = (nz + 15) / 16;
            KKREF_CHECK(cudaEventRecord(e0, stream));
            for (int start = 0; start < cnt; start += KKREF_BP_PROJS_BLOCK) {
                cone_bp<<<dim3(b2 * b1, b0), dim3(16, 32), 0, stream>>>(tex, vol, start, cnt, nx, ny, nz,
                                                                       vox_vol);
                KKREF_CHECK(cudaGetLastError());
            }
            KKREF_CHECK(cudaEventRecord(e1, stream));
            KKREF_CHECK(cudaEventSynchronize(e1));
            float t = 0.f;
            KKREF_CHECK(cudaEventElapsedTime(&t, e0, e1));
            total_ms += t;
            cudaDestroyTextureObject(tex);
            tex = 0;
            cudaFreeArray(arr);
            arr = nullptr;
        }
    }
done:
    if (ms) *ms = total_ms;
    cudaStreamSynchronize(stream);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (tex) cudaDestroyTextureObject(tex);
    if (arr) cudaFreeArray(arr);
    return rc;
}
