// Texture-unit throughput probe: bilinear fetches per clock per SM of a
// 2D-layered float32 texture, the same with float16 texels, and trilinear
// fetches of a 3D float32 texture sampled at slice centres. These are the
// rates that bound the cone-beam projectors' texture paths (the peak used
// by bench.py's texture roofline).
//
// Hardware characterisation, not part of the library. Build and run on
// the GPU:
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -o tex_rate tex_rate.cu && ./tex_rate
// All coordinates stay inside the 256^3 arrays (border addressing anyway).
#include <cuda_runtime.h>

#include <cstdio>

__global__ void k2d(cudaTextureObject_t t, float* out, int iters, float step) {
    float y = 10.3f + 0.01f * (threadIdx.x & 31) + 0.37f * (blockIdx.x % 97);
    float z = 20.1f + 0.65f * (threadIdx.x & 31);
    float acc = 0.f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int s = 0; s < 16; ++s) {
            acc += tex2DLayered<float>(t, z, y, s + (blockIdx.x & 15) * 16);
            y += step;
            z += step * 0.7f;
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

__global__ void k3d(cudaTextureObject_t t, float* out, int iters, float step) {
    float y = 10.3f + 0.01f * (threadIdx.x & 31) + 0.37f * (blockIdx.x % 97);
    float z = 20.1f + 0.65f * (threadIdx.x & 31);
    float acc = 0.f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int s = 0; s < 16; ++s) {
            acc += tex3D<float>(t, z, y, s + (blockIdx.x & 15) * 16 + 0.5f);
            y += step;
            z += step * 0.7f;
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

static cudaTextureObject_t make_tex(cudaArray_t a) {
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = a;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    cudaTextureObject_t t = 0;
    cudaCreateTextureObject(&t, &rd, &td, nullptr);
    return t;
}

int main() {
    const int N = 256;
    int dev = 0, sms = 0, khz = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev);
    const cudaChannelFormatDesc f32 = cudaCreateChannelDesc<float>(), f16 = cudaCreateChannelDescHalf();
    cudaArray_t a2, ah, a3;
    cudaMalloc3DArray(&a2, &f32, make_cudaExtent(N, N, N), cudaArrayLayered);
    cudaMalloc3DArray(&ah, &f16, make_cudaExtent(N, N, N), cudaArrayLayered);
    cudaMalloc3DArray(&a3, &f32, make_cudaExtent(N, N, N), 0);
    const cudaTextureObject_t t2 = make_tex(a2), th = make_tex(ah), t3 = make_tex(a3);
    const int blocks = sms * 8, threads = 256, iters = 64;
    float* out = nullptr;
    cudaMalloc(&out, sizeof(float) * blocks * threads);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const double n = (double)blocks * threads * iters * 16;
    const double hz = khz * 1e3;
    for (int rep = 0; rep < 2; ++rep) {  // the second repetition is warm
        const char* names[3] = {"tex2DLayered float32", "tex2DLayered float16", "tex3D float32 (slice centre)"};
        for (int k = 0; k < 3; ++k) {
            float ms = 0.f;
            cudaEventRecord(e0);
            if (k == 0) k2d<<<blocks, threads>>>(t2, out, iters, 0.013f);
            if (k == 1) k2d<<<blocks, threads>>>(th, out, iters, 0.013f);
            if (k == 2) k3d<<<blocks, threads>>>(t3, out, iters, 0.013f);
            cudaEventRecord(e1);
            cudaEventSynchronize(e1);
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep == 1)
                printf("%-30s %.3f ms  %.1f G fetches/s  %.2f /clk/SM at %.0f MHz\n", names[k], ms, n / ms / 1e6,
                       n / (ms * 1e-3) / sms / hz, hz / 1e6);
        }
    }
    printf("status: %s\n", cudaGetErrorString(cudaGetLastError()));
    return 0;
}
