// FDK pre-processing kernels: cone-beam cosine pre-weighting and detector
// row filtering, both in float64 as the reference evaluates them
// (processing.py:96-126, 149-188), plus the SIRT reciprocal helper.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <stdint.h>

#include "kk_common.cuh"

namespace kk {

constexpr int PW_BLOCK = 256;
constexpr int FILT_BLOCK = 256;
constexpr int FILT_MAX_COLS = 8192;  // 24 cols + 64 bytes of shared memory per block

// p *= |d - s| / |pixel - s|; pixel = corner + col * u_pw + row * v_ph.
// Evaluated with the operation order of processing.py:182-186 and of
// numpy's norm (((dx*dx + dy*dy) + dz*dz), then sqrt), no fused
// operations, then rounded once to float32 as the in-place float32
// multiply of the reference does.
__global__ void __launch_bounds__(PW_BLOCK)
    preweight_kernel(float* data, const uint64_t* table, int64_t sa, int64_t sr, int64_t sc, int rows, int cols,
                     const double* __restrict__ geom) {
    const int a = blockIdx.y;
    const int64_t pix = (int64_t)blockIdx.x * PW_BLOCK + threadIdx.x;
    if (pix >= (int64_t)rows * cols) return;
    const int r = (int)(pix / cols), c = (int)(pix % cols);
    const double* g = geom + 13 * (int64_t)a;
    double sq = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double p = __dadd_rn(__dadd_rn(g[k], __dmul_rn((double)c, g[3 + k])), __dmul_rn((double)r, g[6 + k]));
        const double d = __dsub_rn(p, g[9 + k]);
        sq = k == 0 ? __dmul_rn(d, d) : __dadd_rn(sq, __dmul_rn(d, d));
    }
    const double w = __ddiv_rn(g[12], __dsqrt_rn(sq));
    float* e = (table ? (float*)table[a] : data + (int64_t)a * sa) + (int64_t)r * sr + (int64_t)c * sc;
    *e = __double2float_rn(__dmul_rn((double)*e, w));
}

// out[i] = sum_j p[j] * h[(i - j) mod P] for one detector row (j ascending,
// one float64 fma per term). The row is staged in shared memory as float64,
// together with hx[m] = h[(m - cols) mod P], so that term (i, j) reads
// hx[i - j + cols] without a wrap test. Each thread produces four
// consecutive outputs i0..i0+3; their filter taps at step j are
// hx[i0 + cols - j + q], so going from j to j + 1 shifts the four taps by
// one and a single new tap is read (a sliding window in registers). hx is
// stored as four interleaved sub-arrays (index m at [m % 4][m / 4]) so the
// lanes of a warp, whose windows start four taps apart, read consecutive
// doubles of one sub-array: no bank conflicts.
__global__ void __launch_bounds__(FILT_BLOCK)
    filter_rows_kernel(float* data, const uint64_t* table, int64_t sa, int64_t sr, int64_t sc, int rows, int cols,
                       const double* __restrict__ h, int P) {
    extern __shared__ double sm[];
    double* row = sm;
    const int HN = 2 * cols + 8;
    const int HQ = (HN + 3) / 4;
    double* H = sm + cols;
    const int line = blockIdx.x;
    const int a = line / rows, r = line % rows;
    float* base = (table ? (float*)table[a] : data + (int64_t)a * sa) + (int64_t)r * sr;
    for (int j = threadIdx.x; j < cols; j += blockDim.x) row[j] = (double)base[(int64_t)j * sc];
    for (int m = threadIdx.x; m < HN; m += blockDim.x) H[(m & 3) * HQ + (m >> 2)] = __ldg(h + (m - cols + P) % P);
    __syncthreads();
    for (int i0 = 4 * threadIdx.x; i0 < cols; i0 += 4 * blockDim.x) {
        const int b = i0 + cols;
        double h0 = H[(b & 3) * HQ + (b >> 2)];
        double h1 = H[((b + 1) & 3) * HQ + ((b + 1) >> 2)];
        double h2 = H[((b + 2) & 3) * HQ + ((b + 2) >> 2)];
        double h3 = H[((b + 3) & 3) * HQ + ((b + 3) >> 2)];
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll 4
        for (int j = 0; j < cols; ++j) {
            const double x = row[j];
            a0 = fma(x, h0, a0);
            a1 = fma(x, h1, a1);
            a2 = fma(x, h2, a2);
            a3 = fma(x, h3, a3);
            const int n = b - j - 1;  // >= i0 >= 0
            h3 = h2;
            h2 = h1;
            h1 = h0;
            h0 = H[(n & 3) * HQ + (n >> 2)];
        }
        const double acc[4] = {a0, a1, a2, a3};
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (i0 + q < cols) base[(int64_t)(i0 + q) * sc] = __double2float_rn(acc[q]);
    }
}

// x = clip(mask * (x - scale * g)) elementwise (the SIRT update of
// algo.py:356-362 once the backprojection g is complete, e.g. summed over
// the ranks of an angle-sharded solve).
__global__ void sirt_update_kernel(float* x, const float* __restrict__ g, const float* __restrict__ scale,
                                   const float* __restrict__ mask, float vmin, float vmax, int has_min, int has_max,
                                   int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float v = __fsub_rn(x[i], __fmul_rn(g[i], scale[i]));
        if (mask) v = __fmul_rn(v, mask[i]);
        if (has_min) v = fmaxf(v, vmin);
        if (has_max) v = fminf(v, vmax);
        x[i] = v;
    }
}

__global__ void reciprocal_kernel(float* x, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = __fdiv_rn(1.f, x[i]);
        x[i] = (v == __int_as_float(0x7f800000)) ? 0.f : v;
    }
}

}  // namespace kk

using namespace kk;

static int check_f32_projections(const kk_projections* p, const char* who) {
    if (!p || (!p->data && !p->table)) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: projections are NULL", who);
    if (p->dtype != KK_F32) return kk_fail(KK_ERR_UNSUPPORTED, "%s: float32 projections only", who);
    if (p->table && p->table_axis != 0)
        return kk_fail(KK_ERR_UNSUPPORTED, "%s: a pointer table is supported along the angle axis only", who);
    if (p->n_angles <= 0 || p->rows <= 0 || p->cols <= 0 || p->n_angles > 65535 || p->rows > (1 << 20) ||
        p->cols > (1 << 20))
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: bad projection shape", who);
    return KK_OK;
}

extern "C" int kk_preweight(const kk_projections* proj, const double* geom, void* stream) {
    int rc = check_f32_projections(proj, "kk_preweight");
    if (rc) return rc;
    if (!geom) return kk_fail(KK_ERR_INVALID_ARGUMENT, "kk_preweight: geometry is NULL");
    const int64_t npix = proj->rows * proj->cols;
    dim3 grid((unsigned)((npix + PW_BLOCK - 1) / PW_BLOCK), (unsigned)proj->n_angles);
    preweight_kernel<<<grid, PW_BLOCK, 0, (cudaStream_t)stream>>>(
        (float*)proj->data, proj->table, proj->stride[0], proj->stride[1], proj->stride[2], (int)proj->rows,
        (int)proj->cols, geom);
    return kk_check_launch("kk_preweight");
}

extern "C" int kk_filter_rows(const kk_projections* proj, const double* h, int64_t P, void* stream) {
    int rc = check_f32_projections(proj, "kk_filter_rows");
    if (rc) return rc;
    if (!h) return kk_fail(KK_ERR_INVALID_ARGUMENT, "kk_filter_rows: filter is NULL");
    if (proj->cols > FILT_MAX_COLS)
        return kk_fail(KK_ERR_UNSUPPORTED, "kk_filter_rows: at most %d columns", FILT_MAX_COLS);
    if (P < 2 * proj->cols)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "kk_filter_rows: padded length %lld shorter than 2*cols",
                       (long long)P);
    const int64_t lines = proj->n_angles * proj->rows;
    if (lines > 0x7fffffff) return kk_fail(KK_ERR_UNSUPPORTED, "kk_filter_rows: too many rows");
    // the row and the four interleaved copies of hx (2 cols + 8 taps)
    const int64_t hq = (2 * proj->cols + 8 + 3) / 4;
    const size_t smem = sizeof(double) * (size_t)(proj->cols + 4 * hq);
    rc = kk_allow_smem((const void*)filter_rows_kernel, smem, "kk_filter_rows");
    if (rc) return rc;
    const int threads = (int)std::min<int64_t>(FILT_BLOCK, ((proj->cols + 3) / 4 + 31) / 32 * 32);
    filter_rows_kernel<<<(unsigned)lines, threads, smem, (cudaStream_t)stream>>>(
        (float*)proj->data, proj->table, proj->stride[0], proj->stride[1], proj->stride[2], (int)proj->rows,
        (int)proj->cols, h, (int)P);
    return kk_check_launch("kk_filter_rows");
}

extern "C" int kk_reciprocal(float* data, int64_t n, void* stream) {
    if (!data || n < 0) return kk_fail(KK_ERR_INVALID_ARGUMENT, "kk_reciprocal: bad arguments");
    if (n == 0) return KK_OK;
    const int64_t blocks = std::min<int64_t>((n + 255) / 256, (int64_t)kk_sm_count() * 16);
    reciprocal_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(data, n);
    return kk_check_launch("kk_reciprocal");
}

extern "C" int kk_sirt_update(float* x, const float* g, const float* scale, const float* mask, float min_value,
                              float max_value, int32_t has_min, int32_t has_max, int64_t n, void* stream) {
    if (!x || !g || !scale || n < 0) return kk_fail(KK_ERR_INVALID_ARGUMENT, "kk_sirt_update: bad arguments");
    if (n == 0) return KK_OK;
    const int64_t blocks = std::min<int64_t>((n + 255) / 256, (int64_t)kk_sm_count() * 16);
    sirt_update_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(x, g, scale, mask, min_value, max_value,
                                                                         has_min, has_max, n);
    return kk_check_launch("kk_sirt_update");
}
