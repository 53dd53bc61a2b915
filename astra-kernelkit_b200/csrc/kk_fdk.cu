// FDK pre-processing kernels: cone-beam cosine pre-weighting and detector
// row filtering, both in float64 as the reference evaluates them
// (processing.py:96-126, 149-188), plus the SIRT reciprocal helper.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <stdint.h>

#include "kk_cone.cuh"

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

// ---------------------------------------------------------------------------
// fused FDK pre-processing: pre-weighting, zero padding, FFT filtering and
// the store into the backprojector's layered texture in one pass
// ---------------------------------------------------------------------------
// One block filters two detector rows at once: row a is the real part and
// row b the imaginary part of one complex signal z of length P (rows
// zero-padded from cols). The filter's response H is real and even, so
// IFFT(H . FFT(z)) = (h * a) + i (h * b): the real and imaginary parts of
// the filtered signal are the two filtered rows. The reference filters
// each row with a float64 FFT in the same way (processing.py:111-126).
//
// The transform runs in shared memory in float64: decimation-in-frequency
// radix-4 stages (and one radix-2 stage when log2 P is odd) leave the
// spectrum in bit-reversed order, the multiplication by H uses H in
// bit-reversed order, and the inverse stages (conjugate twiddles, in
// reverse order) take bit-reversed input back to natural order, so no
// permutation pass is needed. Shared-memory index i is stored at i + i / 8
// to spread the strided accesses of the short stages over the banks.
//
// The plan (kk_fdk_plan, 3 P doubles) holds what the kernel reads, laid
// out for coalesced loads: H[bitrev(i)] for i < P, then per radix-4 stage
// of length len (P, P/4, ... down to 4) and j < len / 4 the twiddle W^j
// (W = exp(-2 pi i / len)) as two doubles; W^2j and W^3j are formed from
// it in registers (the kernel is bound by its loads and stores, not by
// float64 arithmetic).
constexpr int FFT_THREADS = 256;
constexpr int FFT_MAX_P = 8192;

__global__ void fdk_plan_kernel(double* plan, const double* __restrict__ H, int P, int log2P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P) plan[i] = H[__brev((unsigned)i) >> (32 - log2P)];
    // twiddle records of every stage
    int off = P;
    for (int len = P; len >= 4; len >>= 2) {
        const int q = len >> 2;
        if (i < q) {
            double s1, c1;
            sincospi(-2.0 * (double)i / (double)len, &s1, &c1);
            plan[off + 2 * i] = c1;
            plan[off + 2 * i + 1] = s1;
        }
        off += 2 * q;
    }
}

__device__ __forceinline__ int fpad(int i) { return i + (i >> 3); }

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 w) {
    return make_double2(fma(a.x, w.x, -a.y * w.y), fma(a.x, w.y, a.y * w.x));
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 w) {  // a * conj(w)
    return make_double2(fma(a.x, w.x, a.y * w.y), fma(a.y, w.x, -a.x * w.y));
}

// The pre-weighted float32 value of one pixel, as kk_preweight stores it
// (p *= |d - s| / |pixel - s| in float64, rounded once to float32).
__device__ __forceinline__ double fdk_load(const float* row, int64_t sc, int c, int r, const double* g) {
    const float p = row[(int64_t)c * sc];
    if (!g) return (double)p;
    double sq = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double q = __dadd_rn(__dadd_rn(g[k], __dmul_rn((double)c, g[3 + k])), __dmul_rn((double)r, g[6 + k]));
        const double d = __dsub_rn(q, g[9 + k]);
        sq = k == 0 ? __dmul_rn(d, d) : __dadd_rn(sq, __dmul_rn(d, d));
    }
    const double w = __ddiv_rn(g[12], __dsqrt_rn(sq));
    return (double)__double2float_rn(__dmul_rn((double)p, w));
}

__global__ void __launch_bounds__(FFT_THREADS)
    fdk_filter_kernel(const float* src, const uint64_t* src_table, int64_t sa, int64_t sr, int64_t sc, int n_lines,
                      int rows, int cols, const double* __restrict__ geom, const double* __restrict__ plan,
                      int P, int log2P, float* dst, const uint64_t* dst_table,
                      int64_t da, int64_t dr, int64_t dc, cudaSurfaceObject_t surf, int layer0) {
    extern __shared__ double2 fz[];
    const int tid = threadIdx.x;
    const int line0 = 2 * blockIdx.x;
    const bool two = line0 + 1 < n_lines;
    const int a0 = line0 / rows, r0 = line0 % rows;
    // a block with a single row (odd row count) repeats it as the second
    // one, which is never stored
    const int a1 = two ? (line0 + 1) / rows : a0, r1 = two ? (line0 + 1) % rows : r0;
    const float* row0 = (src_table ? (const float*)src_table[a0] : src + (int64_t)a0 * sa) + (int64_t)r0 * sr;
    const float* row1 = (src_table ? (const float*)src_table[a1] : src + (int64_t)a1 * sa) + (int64_t)r1 * sr;
    const double* g0 = geom ? geom + 13 * (int64_t)a0 : nullptr;
    const double* g1 = geom ? geom + 13 * (int64_t)a1 : nullptr;
    auto load = [&](int j) -> double2 {
        if (j >= cols) return make_double2(0.0, 0.0);
        return make_double2(fdk_load(row0, sc, j, r0, g0), two ? fdk_load(row1, sc, j, r1, g1) : 0.0);
    };
    const double2* tw = reinterpret_cast<const double2*>(plan + P);  // stage records
    const int q0 = P >> 2;
    // forward stage of length P fused with the load: inputs j + 2 P/4 and
    // j + 3 P/4 are zero padding (P >= 2 cols)
    for (int j = tid; j < q0; j += FFT_THREADS) {
        const double2 a = load(j), b = load(j + q0);
        const double2 w1 = __ldg(&tw[j]), w2 = cmul(w1, w1), w3 = cmul(w2, w1);
        const double2 t3 = make_double2(b.y, -b.x);  // b * (-i)
        fz[fpad(j)] = cadd(a, b);
        fz[fpad(j + q0)] = cmul(csub(a, b), w2);
        fz[fpad(j + 2 * q0)] = cmul(cadd(a, t3), w1);
        fz[fpad(j + 3 * q0)] = cmul(csub(a, t3), w3);
    }
    tw += q0;
    __syncthreads();
    // the middle forward stages: radix-4 decimation in frequency
    const int lastlen = (log2P & 1) ? 2 : 4;
    int len = P >> 2, lq = log2P - 4;  // lq = log2(len / 4)
    for (; len > lastlen; tw += (len >> 2), len >>= 2, lq -= 2) {
        const int q = len >> 2;
        for (int t = tid; t < (P >> 2); t += FFT_THREADS) {
            const int j = t & (q - 1), base = ((t >> lq) * len) + j;
            const double2 a = fz[fpad(base)], b = fz[fpad(base + q)], c = fz[fpad(base + 2 * q)],
                          d = fz[fpad(base + 3 * q)];
            const double2 w1 = __ldg(&tw[j]), w2 = cmul(w1, w1), w3 = cmul(w2, w1);
            const double2 t0 = cadd(a, c), t1 = csub(a, c), t2 = cadd(b, d);
            const double2 bd = csub(b, d);
            const double2 t3 = make_double2(bd.y, -bd.x);  // (b - d) * (-i)
            fz[fpad(base)] = cadd(t0, t2);
            fz[fpad(base + q)] = cmul(csub(t0, t2), w2);
            fz[fpad(base + 2 * q)] = cmul(cadd(t1, t3), w1);
            fz[fpad(base + 3 * q)] = cmul(csub(t1, t3), w3);
        }
        __syncthreads();
    }
    // the last forward stage, the product with H (plan order: bit-reversed,
    // as the spectrum) and the first inverse stage, on the same groups of
    // consecutive elements (its twiddles are 1)
    if (lastlen == 2) {
        for (int t = tid; t < (P >> 1); t += FFT_THREADS) {
            const double2 u = fz[fpad(2 * t)], v = fz[fpad(2 * t + 1)];
            const double h0 = __ldg(&plan[2 * t]), h1 = __ldg(&plan[2 * t + 1]);
            const double2 p0 = cadd(u, v), p1 = csub(u, v);
            const double2 f0 = make_double2(p0.x * h0, p0.y * h0), f1 = make_double2(p1.x * h1, p1.y * h1);
            fz[fpad(2 * t)] = cadd(f0, f1);
            fz[fpad(2 * t + 1)] = csub(f0, f1);
        }
    } else {
        for (int t = tid; t < (P >> 2); t += FFT_THREADS) {
            const int base = 4 * t;
            const double2 a = fz[fpad(base)], b = fz[fpad(base + 1)], c = fz[fpad(base + 2)], d = fz[fpad(base + 3)];
            const double2 t0 = cadd(a, c), t1 = csub(a, c), t2 = cadd(b, d);
            const double2 bd = csub(b, d);
            const double2 t3 = make_double2(bd.y, -bd.x);
            double2 y[4] = {cadd(t0, t2), csub(t0, t2), cadd(t1, t3), csub(t1, t3)};
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const double h = __ldg(&plan[base + m]);
                y[m] = make_double2(y[m].x * h, y[m].y * h);
            }
            // inverse of the stage: y0, y2, y1, y3 sit at base, +1, +2, +3
            const double2 s0 = cadd(y[0], y[1]), s2 = csub(y[0], y[1]), s1 = cadd(y[2], y[3]);
            const double2 dd = csub(y[2], y[3]);
            const double2 s3 = make_double2(-dd.y, dd.x);  // (y1 - y3) * i
            fz[fpad(base)] = cadd(s0, s1);
            fz[fpad(base + 1)] = cadd(s2, s3);
            fz[fpad(base + 2)] = csub(s0, s1);
            fz[fpad(base + 3)] = csub(s2, s3);
        }
        tw += 1;  // the length-4 stage's record (its twiddle is 1)
    }
    __syncthreads();
    // the middle inverse stages: conjugate twiddles, reverse order,
    // unnormalised (the result is P times the filtered signal)
    if (lastlen == 4) tw -= 1;
    for (len = lastlen * 4, lq = (lastlen == 4 ? 2 : 1); len <= (P >> 2); len <<= 2, lq += 2) {
        const int q = len >> 2;
        tw -= q;
        for (int t = tid; t < (P >> 2); t += FFT_THREADS) {
            const int j = t & (q - 1), base = ((t >> lq) * len) + j;
            const double2 w1 = __ldg(&tw[j]), w2 = cmul(w1, w1), w3 = cmul(w2, w1);
            const double2 y0 = fz[fpad(base)];
            const double2 y2 = cmulc(fz[fpad(base + q)], w2);
            const double2 y1 = cmulc(fz[fpad(base + 2 * q)], w1);
            const double2 y3 = cmulc(fz[fpad(base + 3 * q)], w3);
            const double2 t0 = cadd(y0, y2), t2 = csub(y0, y2), t1 = cadd(y1, y3);
            const double2 dd = csub(y1, y3);
            const double2 t3 = make_double2(-dd.y, dd.x);  // (y1 - y3) * i
            fz[fpad(base)] = cadd(t0, t1);
            fz[fpad(base + q)] = cadd(t2, t3);
            fz[fpad(base + 2 * q)] = csub(t0, t1);
            fz[fpad(base + 3 * q)] = csub(t2, t3);
        }
        __syncthreads();
    }
    // the inverse stage of length P fused with the store of the first cols
    // values (outputs j and j + P/4; the other two lie beyond P/2 >= cols),
    // scaled by 1 / P (exact: P is a power of two)
    tw -= q0;
    const double inv = 1.0 / (double)P;
    float* out0 = dst ? (dst_table ? (float*)dst_table[a0] : dst + (int64_t)a0 * da) + (int64_t)r0 * dr : nullptr;
    float* out1 = dst ? (dst_table ? (float*)dst_table[a1] : dst + (int64_t)a1 * da) + (int64_t)r1 * dr : nullptr;
    auto store = [&](int j, double2 v) {
        const float f0 = __double2float_rn(v.x * inv);
        if (out0) out0[(int64_t)j * dc] = f0;
        if (surf) surf2DLayeredwrite(f0, surf, j * (int)sizeof(float), r0, layer0 + a0);
        if (two) {
            const float f1 = __double2float_rn(v.y * inv);
            if (out1) out1[(int64_t)j * dc] = f1;
            if (surf) surf2DLayeredwrite(f1, surf, j * (int)sizeof(float), r1, layer0 + a1);
        }
    };
    for (int j = tid; j < q0 && j < cols; j += FFT_THREADS) {
        const double2 w1 = __ldg(&tw[j]), w2 = cmul(w1, w1), w3 = cmul(w2, w1);
        const double2 y0 = fz[fpad(j)];
        const double2 y2 = cmulc(fz[fpad(j + q0)], w2);
        const double2 y1 = cmulc(fz[fpad(j + 2 * q0)], w1);
        const double2 y3 = cmulc(fz[fpad(j + 3 * q0)], w3);
        const double2 t0 = cadd(y0, y2), t2 = csub(y0, y2), t1 = cadd(y1, y3);
        const double2 dd = csub(y1, y3);
        const double2 t3 = make_double2(-dd.y, dd.x);
        store(j, cadd(t0, t1));
        if (j + q0 < cols) store(j + q0, cadd(t2, t3));
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

static int fft_length(int64_t P, const char* who, int* log2P) {
    if (P < 64 || P > FFT_MAX_P || (P & (P - 1)))
        return kk_fail(KK_ERR_UNSUPPORTED, "%s: padded length %lld must be a power of two in [64, %d]", who,
                       (long long)P, FFT_MAX_P);
    *log2P = 0;
    while ((1LL << *log2P) < P) ++*log2P;
    return KK_OK;
}

extern "C" int64_t kk_fdk_plan_size(int64_t P) { return 3 * P; }

extern "C" int kk_fdk_plan(double* plan, const double* H, int64_t P, void* stream) {
    const char* who = "kk_fdk_plan";
    int log2P = 0;
    int rc = fft_length(P, who, &log2P);
    if (rc) return rc;
    if (!plan || !H) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: NULL argument", who);
    fdk_plan_kernel<<<(unsigned)((P + 255) / 256), 256, 0, (cudaStream_t)stream>>>(plan, H, (int)P, log2P);
    return kk_check_launch(who);
}

extern "C" int kk_fdk_filter(const kk_projections* src, const double* geom, const double* plan, int64_t P,
                             const kk_projections* dst, kk_layered* tex, int64_t layer0, void* stream) {
    const char* who = "kk_fdk_filter";
    int rc = check_f32_projections(src, who);
    if (rc) return rc;
    if (!plan) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: plan is NULL", who);
    int log2P = 0;
    rc = fft_length(P, who, &log2P);
    if (rc) return rc;
    if (P < 2 * src->cols)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: padded length %lld shorter than 2*cols", who, (long long)P);
    if (dst) {
        rc = check_f32_projections(dst, who);
        if (rc) return rc;
        if (dst->n_angles != src->n_angles || dst->rows != src->rows || dst->cols != src->cols)
            return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: destination shape differs from the source", who);
    }
    if (tex) {
        if (!tex->surf) return kk_fail(KK_ERR_UNSUPPORTED, "%s: texture has no surface", who);
        if (tex->dtype != KK_F32 || tex->height != src->rows || tex->width != src->cols || layer0 < 0 ||
            layer0 + src->n_angles > tex->layers)
            return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: texture layers [%lld, %lld) do not fit", who,
                           (long long)layer0, (long long)(layer0 + src->n_angles));
    }
    const int64_t lines = src->n_angles * src->rows;
    if (lines > 0x7ffffffe) return kk_fail(KK_ERR_UNSUPPORTED, "%s: too many rows", who);
    const size_t smem = sizeof(double2) * (size_t)(P + P / 8);
    rc = kk_allow_smem((const void*)fdk_filter_kernel, smem, who);
    if (rc) return rc;
    fdk_filter_kernel<<<(unsigned)((lines + 1) / 2), FFT_THREADS, smem, (cudaStream_t)stream>>>(
        (const float*)src->data, src->table, src->stride[0], src->stride[1], src->stride[2], (int)lines,
        (int)src->rows, (int)src->cols, geom, plan, (int)P, log2P, dst ? (float*)dst->data : nullptr,
        dst ? dst->table : nullptr, dst ? dst->stride[0] : 0, dst ? dst->stride[1] : 0, dst ? dst->stride[2] : 0,
        tex ? tex->surf : 0, (int)layer0);
    return kk_check_launch(who);
}
