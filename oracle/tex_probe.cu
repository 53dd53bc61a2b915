// Measures the linear filtering of the GPU texture unit (test
// infrastructure): samples float32 CUDA arrays through texture objects with
// border addressing and linear filtering, the configuration the reference
// kernels use (kernelkit/kernel.py:22-32), at caller-chosen coordinates.
// The tests compare the results with the weight-quantisation models of
// oracle/cone.py to decide which one the hardware follows.
#include <cuda_runtime.h>
#include <string.h>

#define KKP_CHECK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { rc = (int)e_; goto done; } } while (0)

__global__ void kkp_fetch_layered(cudaTextureObject_t t, const float* xs, const float* ys, int layer,
                                  float* out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = tex2DLayered<float>(t, xs[i], ys[i], layer);
}

__global__ void kkp_fetch_3d(cudaTextureObject_t t, const float* xs, const float* ys, const float* zs,
                             float* out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = tex3D<float>(t, xs[i], ys[i], zs[i]);
}

static cudaTextureObject_t kkp_make_tex(cudaArray_t arr) {
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
    cudaTextureObject_t t = 0;
    if (cudaCreateTextureObject(&t, &rd, &td, nullptr) != cudaSuccess) return 0;
    return t;
}

// data: device float32 (depth, h, w); xs/ys/zs/out: device, n samples.
// layered != 0: a 2D-layered array with `depth` layers sampled at layer
// `layer` (zs ignored); otherwise a 3D array.
extern "C" int kkp_probe(const float* data, int w, int h, int depth, int layered, int layer,
                         const float* xs, const float* ys, const float* zs, float* out, int n) {
    int rc = 0;
    cudaArray_t arr = nullptr;
    cudaTextureObject_t t = 0;
    {
        cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
        KKP_CHECK(cudaMalloc3DArray(&arr, &ch, make_cudaExtent(w, h, depth), layered ? cudaArrayLayered : 0));
        cudaMemcpy3DParms cp;
        memset(&cp, 0, sizeof(cp));
        cp.srcPtr = make_cudaPitchedPtr((void*)data, (size_t)w * sizeof(float), w, h);
        cp.dstArray = arr;
        cp.extent = make_cudaExtent(w, h, depth);
        cp.kind = cudaMemcpyDeviceToDevice;
        KKP_CHECK(cudaMemcpy3D(&cp));
        t = kkp_make_tex(arr);
        if (!t) { rc = -1; goto done; }
        if (layered)
            kkp_fetch_layered<<<(n + 255) / 256, 256>>>(t, xs, ys, layer, out, n);
        else
            kkp_fetch_3d<<<(n + 255) / 256, 256>>>(t, xs, ys, zs, out, n);
        KKP_CHECK(cudaGetLastError());
        KKP_CHECK(cudaDeviceSynchronize());
    }
done:
    if (t) cudaDestroyTextureObject(t);
    if (arr) cudaFreeArray(arr);
    return rc;
}
