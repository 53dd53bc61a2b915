// Exact adjoint of the ray-driven forward projection (kk_fp.cu), as a
// voxel-driven gather: no atomics, every voxel sums its own terms.
//
// The forward projection adds, for ray (a, r, c) and every slice s along
// the ray's dominant axis A, the bilinear sample of slice s at in-slice
// coordinates (y_s, z_s), times corr * outputScale. Its transpose gives
// voxel (s, j, k) the sum, over the rays whose slice-s sample touches it, of
// proj[a, r, c] * corr * outputScale * (that sample's weight on the voxel).
// To be the exact transpose of the forward projector (not of an idealised
// one), each candidate ray is set up by the same ray_setup(), its slice-s
// coordinates are rebuilt by the same slab-restart-and-increment sequence
// in the same float32 operations, and its weights come from the same weight
// rule (texture-compatible 1/256 weights or exact ones).
//
// Candidates: the footprint of voxel (j, k) in slice s is the square of
// sample positions y in [j - 1/2, j + 3/2), z in [k - 1/2, k + 3/2); its
// four corners are projected onto the detector and every pixel whose
// centre falls inside their bounding box (widened by 0.05 pixel) is tested
// exactly. Ray set-ups are computed once per chunk of angles into a
// caller-provided work buffer, so any volume size fits by chunking.
#include "kk_cone.cuh"

#include <climits>

namespace kk {

struct FptArgs {
    float* vol;
    int64_t vs[3];
    int vn[3];
    int m0, m1, m2;  // world axes from slowest to fastest in memory
    int rank[3];     // memory rank of each world axis: 0 fastest .. 2 slowest
    const float* proj;
    const uint64_t* table;
    int64_t ps[3];
    int rows, cols;
    const kk_fp_angle* angles;
    float os[9];
    int slab;
    int rec0, nrec;  // records of this chunk
    int accumulate;  // add to the volume (later chunks, or additive)
    float4* ray_ab;  // (a1, b1, a2, b2) per ray of the chunk
    float* ray_pc;   // projection value * corr * outputScale per ray
    int tiled[3];    // the tile pass handles shared records along axis A
};

constexpr int FPT_TILE_2 = 32;
constexpr int FPT_TILE_1 = 8;

__device__ __forceinline__ void cross3(const float* a, const float* b, float* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

__device__ __forceinline__ float dot3(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// Component k of the point whose coordinate along axis A is t, along D1
// is d1 and along D2 is d2 (selects, not an indexed array, so nothing goes
// to local memory).
__device__ __forceinline__ float place(int k, int A, int D1, float t, float d1, float d2) {
    return k == A ? t : (k == D1 ? d1 : d2);
}

// Ray set-up of every (record, column, row) of the chunk, rows fastest: a
// warp of the gather (consecutive voxels along the fastest volume axis,
// which for circular scans map to consecutive detector rows) then reads
// neighbouring entries. The projection value is folded in here, times the
// ray's corr * outputScale.
__global__ void fpt_rays_kernel(const FptArgs L) {
    const int64_t per = (int64_t)L.rows * L.cols;
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= per * L.nrec) return;
    const int k = (int)(id / per);
    const int cr = (int)(id - (int64_t)k * per);
    const int c = cr / L.rows, r = cr - c * L.rows;
    const kk_fp_angle* P = L.angles + L.rec0 + k;
    float src[3], cor[3], u[3], v[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        src[q] = __ldg(&P->src[q]);
        cor[q] = __ldg(&P->corner[q]);
        u[q] = __ldg(&P->u[q]);
        v[q] = __ldg(&P->v[q]);
    }
    const int A = __ldg(&P->axis);
    const int D1 = A == 1 ? 0 : 1, D2 = A == 2 ? 0 : 2;
    const RaySetup R = ray_setup(src, cor, u, v, A, D1, D2, r, c, L.os[3 * A], L.os[3 * A + 1]);
    const int a = __ldg(&P->index);
    const float* plane = L.table ? (const float*)L.table[a] : L.proj + (int64_t)a * L.ps[0];
    const float p = __ldg(plane + (int64_t)r * L.ps[1] + (int64_t)c * L.ps[2]);
    L.ray_ab[id] = make_float4(R.a1, R.b1, R.a2, R.b2);
    L.ray_pc[id] = p * (R.corr * L.os[3 * A + 2]);
}

// A ray's in-slice coordinate at slice off + nst: the slab-start value v0
// followed by nst rounded adds of the slope, exactly as the forward
// projector computes it. With texture-compatible weights the split only
// sees floor(256 v - 127.5); each rounded add errs by at most half an ulp
// (2^-24 relative), so the sequence ends within eps of fma(nst, a, v0), and
// when no boundary of floor() lies within eps of that direct value (for
// |v| < 2^13, q = 256 v - 127.5 and q - floor(q) are exact in float32) it
// splits exactly as the sequence would and is returned instead.
template <bool TEX8>
__device__ __forceinline__ float slice_coord(float v0, float a, int nst) {
    if (TEX8) {
        const float fn = (float)nst;
        const float vd = fmaf(fn, a, v0);
        const float eps = (fn + 1.f) * 1.2e-7f * (fabsf(vd) + fabsf(a) * fn + 1.f);
        const float q = 256.f * vd - 127.5f;
        const float f = q - floorf(q);
        const float e = 256.f * 1.01f * eps + 1e-6f;
        if (fabsf(vd) < 8192.f && f > e && f < 1.f - e) return vd;
    }
    float v = v0;
    for (int q = 0; q < nst; ++q) v = __fadd_rn(v, a);
    return v;
}

// Candidate pixel box on the detector of the sample-position rectangle
// y in [y0, y1), z in [z0, z1) (centred coordinates along D1, D2) of slice
// position t of record P: the corners are projected centrally from the
// source; pixel c is a candidate when its centre c + 1/2 lies in the
// projected range widened by 0.05 pixel. False when a corner does not
// project (behind the source), then every pixel is a candidate.
__device__ __forceinline__ bool footprint_box(const FptArgs& L, const kk_fp_angle* P, int A, int D1, float t, float y0,
                                              float y1, float z0, float z1, int& c0, int& c1, int& rlo, int& rhi) {
    float src[3], cor[3], u[3], v[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        src[q] = __ldg(&P->src[q]);
        cor[q] = __ldg(&P->corner[q]);
        u[q] = __ldg(&P->u[q]);
        v[q] = __ldg(&P->v[q]);
    }
    // detector coordinates (pixel units, centre of pixel c at c + 1/2)
    float nrm[3], e1[3], e2[3], tmp[3];
    cross3(u, v, nrm);
    cross3(v, nrm, tmp);
    const float ue = dot3(u, tmp);
    cross3(nrm, u, e2);
    const float ve = dot3(v, e2);
    // the candidate box only needs a few correct digits (it is widened by
    // 0.05 pixel), so the fast reciprocal and division suffice
    const float iue = __frcp_rn(ue), ive = __frcp_rn(ve);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        e1[q] = tmp[q] * iue;
        e2[q] = e2[q] * ive;
    }
    float cs_[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) cs_[q] = cor[q] - src[q];
    const float num = dot3(cs_, nrm);
    float amin = 1e30f, amax = -1e30f, bmin = 1e30f, bmax = -1e30f;
    bool ok = true;
#pragma unroll
    for (int corner = 0; corner < 4; ++corner) {
        const float d1 = (corner & 1) ? y1 : y0;
        const float d2 = (corner & 2) ? z1 : z0;
        float d[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) d[q] = place(q, A, D1, t, d1, d2) - src[q];
        const float den = dot3(d, nrm);
        const float lam = __fdividef(num, den);
        ok = ok && isfinite(lam) && lam > 0.f;
        float qc[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) qc[q] = src[q] + lam * d[q] - cor[q];
        const float al = dot3(qc, e1), be = dot3(qc, e2);
        amin = fminf(amin, al);
        amax = fmaxf(amax, al);
        bmin = fminf(bmin, be);
        bmax = fmaxf(bmax, be);
    }
    c0 = 0;
    c1 = L.cols - 1;
    rlo = 0;
    rhi = L.rows - 1;
    if (ok && isfinite(amin) && isfinite(amax) && isfinite(bmin) && isfinite(bmax)) {
        c0 = max(c0, (int)ceilf(fmaxf(amin - 0.55f, -1.f)));
        c1 = min(c1, (int)floorf(fminf(amax - 0.45f, (float)L.cols)));
        rlo = max(rlo, (int)ceilf(fmaxf(bmin - 0.55f, -1.f)));
        rhi = min(rhi, (int)floorf(fminf(bmax - 0.45f, (float)L.rows)));
        return true;
    }
    return false;
}

// circular scans: the detector's v has no component along A and D1, so
// every row of a column has bit for bit the same D1 coordinate sequence
// (as in the forward projector's shared path)
__device__ __forceinline__ bool shared_record(const kk_fp_angle* P, int A, int D1) {
    const float vA = A == 0 ? __ldg(&P->v[0]) : (A == 1 ? __ldg(&P->v[1]) : __ldg(&P->v[2]));
    const float vD1 = D1 == 0 ? __ldg(&P->v[0]) : __ldg(&P->v[1]);
    return vA == 0.f && vD1 == 0.f;
}

// Contribution of record k of the chunk to voxel (w0, w1, w2): every pixel
// of the voxel's candidate box is tested exactly.
template <bool TEX8>
__device__ float gather_record(const FptArgs& L, int k, int w0, int w1, int w2) {
    const int64_t per = (int64_t)L.rows * L.cols;
    const kk_fp_angle* P = L.angles + L.rec0 + k;
    const int A = __ldg(&P->axis);
    const int D1 = A == 1 ? 0 : 1, D2 = A == 2 ? 0 : 2;
    const int s = A == 0 ? w0 : (A == 1 ? w1 : w2);
    const int jv = D1 == 0 ? w0 : w1;
    const int kv = D2 == 0 ? w0 : w2;
    const int nS = A == 0 ? L.vn[0] : (A == 1 ? L.vn[1] : L.vn[2]);
    const int n1 = D1 == 0 ? L.vn[0] : L.vn[1];
    const int n2 = D2 == 0 ? L.vn[0] : L.vn[2];
    const float half1 = 0.5f * (float)n1, half2 = 0.5f * (float)n2;
    const int rA = A == 0 ? L.rank[0] : (A == 1 ? L.rank[1] : L.rank[2]);
    const int r1 = D1 == 0 ? L.rank[0] : L.rank[1];
    const int r2 = D2 == 0 ? L.rank[0] : L.rank[2];
    const int rule = 2 - rA;
    const bool a_fast = r1 < r2;
    const float t = (float)s - 0.5f * (float)nS + 0.5f;
    int c0, c1, rlo, rhi;
    footprint_box(L, P, A, D1, t, (float)jv - 0.5f - half1, (float)jv + 1.5f - half1, (float)kv - 0.5f - half2,
                  (float)kv + 1.5f - half2, c0, c1, rlo, rhi);
    const int off = (s / L.slab) * L.slab;
    const float t1 = __fadd_rn(__fsub_rn((float)off, 0.5f * (float)nS), 0.5f);
    const bool shared = shared_record(P, A, D1);
    const int nst = s - off;
    float acc = 0.f;
    for (int c = c0; c <= c1; ++c) {
        // shared case: one D1 coordinate for the whole column
        Split syc;
        bool col = false;
        if (shared && rlo <= rhi) {
            const float4 ab = __ldg(&L.ray_ab[(int64_t)k * per + (int64_t)c * L.rows + rlo]);
            syc = split_coord<TEX8>(slice_coord<TEX8>(__fadd_rn(fmaf(ab.x, t1, ab.y), half1), ab.x, nst));
            if ((unsigned)(jv - syc.i) > 1u) continue;
            col = true;
        }
        for (int r = rlo; r <= rhi; ++r) {
            const int64_t id = (int64_t)k * per + (int64_t)c * L.rows + r;
            const float4 ab = __ldg(&L.ray_ab[id]);
            // the forward projector's coordinates for slice s
            const Split sy =
                col ? syc : split_coord<TEX8>(slice_coord<TEX8>(__fadd_rn(fmaf(ab.x, t1, ab.y), half1), ab.x, nst));
            const Split sz = split_coord<TEX8>(slice_coord<TEX8>(__fadd_rn(fmaf(ab.z, t1, ab.w), half2), ab.z, nst));
            const int di = jv - sy.i, dj = kv - sz.i;
            if ((unsigned)di > 1u || (unsigned)dj > 1u) continue;
            const W4 wt = weights4<TEX8>(sy.w, sz.w, rule, a_fast);
            float wgt = di == 0 ? (dj == 0 ? wt.w00 : wt.w01) : (dj == 0 ? wt.w10 : wt.w11);
            if (TEX8) wgt *= 1.f / 256.f;
            acc = fmaf(__ldg(&L.ray_pc[id]), wgt, acc);
        }
    }
    return acc;
}

// General path: one thread per voxel, every record of the chunk (except
// those a tile pass handles, when L.tiled says so).
template <bool TEX8>
__global__ void __launch_bounds__(FPT_TILE_2* FPT_TILE_1) fpt_gather_kernel(const FptArgs L) {
    // nothing to do when the tile passes handle every record of the chunk
    int todo = 0;
    for (int k = threadIdx.y * FPT_TILE_2 + threadIdx.x; k < L.nrec; k += FPT_TILE_2 * FPT_TILE_1) {
        const kk_fp_angle* P = L.angles + L.rec0 + k;
        const int A = __ldg(&P->axis);
        if (!(L.tiled[A] && shared_record(P, A, A == 1 ? 0 : 1))) todo = 1;
    }
    if (!__syncthreads_or(todo)) return;
    const int i2 = blockIdx.x * FPT_TILE_2 + threadIdx.x;
    const int i1 = blockIdx.y * FPT_TILE_1 + threadIdx.y;
    const int i0 = blockIdx.z;
    if (i2 >= L.vn[L.m2] || i1 >= L.vn[L.m1]) return;
    // world indices of the voxel
    const int w0 = L.m0 == 0 ? i0 : (L.m1 == 0 ? i1 : i2);
    const int w1 = L.m0 == 1 ? i0 : (L.m1 == 1 ? i1 : i2);
    const int w2 = L.m0 == 2 ? i0 : (L.m1 == 2 ? i1 : i2);
    float acc = 0.f;
    for (int k = 0; k < L.nrec; ++k) {
        const kk_fp_angle* P = L.angles + L.rec0 + k;
        const int A = __ldg(&P->axis);
        if (L.tiled[A] && shared_record(P, A, A == 1 ? 0 : 1)) continue;
        acc += gather_record<TEX8>(L, k, w0, w1, w2);
    }
    float* out = L.vol + (int64_t)w0 * L.vs[0] + (int64_t)w1 * L.vs[1] + (int64_t)w2 * L.vs[2];
    *out = L.accumulate ? *out + acc : acc;
}

// ---------------------------------------------------------------------------
// tile pass for circular scans
// ---------------------------------------------------------------------------
// One block owns a FPT_TJ x FPT_TK tile of texels (along D1, D2) of one
// slice of the records whose dominant axis is A and whose rows share their
// D1 coordinate. Per record it (1) finds the candidate columns and rows of
// the tile's footprint, (2) computes every candidate column's D1 split and
// every candidate ray's D2 split with the forward projector's own
// slab-restart sequence, and stores the ray's four contributions
// p * corr * outputScale * weight (one per texel of its bilinear
// footprint) in shared memory, with per-(column, texel row) tables of the
// rays that touch each row, then (3) every texel sums the contributions of
// the rays that touch it. Each ray is set up once per tile instead of once
// per voxel it might touch, and each texel reads only its own ~9 terms.
// Records whose footprint exceeds the tables take the per-voxel path.
constexpr int FPT_TJ = 16, FPT_TK = 32;    // texels of a tile along D1, D2
constexpr int FPT_MAXC = 40, FPT_MAXR = 72;  // candidate columns, rows
constexpr int FPT_THREADS = 256;
constexpr size_t FPT_SMEM = (size_t)FPT_MAXC * FPT_MAXR * (sizeof(float4) + sizeof(int)) +
                            (size_t)FPT_MAXC * (FPT_TK + 1) * 2 * sizeof(int) + (size_t)FPT_MAXC * 2 * sizeof(int) +
                            (size_t)(FPT_TJ + 1) * 2 * sizeof(int);

template <bool TEX8>
__global__ void __launch_bounds__(FPT_THREADS) fpt_tile_kernel(const FptArgs L, int A) {
    extern __shared__ __align__(16) unsigned char fpt_sm[];
    float4* contrib = reinterpret_cast<float4*>(fpt_sm);
    int* ri2 = reinterpret_cast<int*>(contrib + FPT_MAXC * FPT_MAXR);
    int* rlo = ri2 + FPT_MAXC * FPT_MAXR;
    int* rhi = rlo + FPT_MAXC * (FPT_TK + 1);
    int* ci1 = rhi + FPT_MAXC * (FPT_TK + 1);
    float* cS = reinterpret_cast<float*>(ci1 + FPT_MAXC);
    int* clo = reinterpret_cast<int*>(cS + FPT_MAXC);
    int* chi = clo + (FPT_TJ + 1);
    // candidate box per record of the current group: first column, columns,
    // first row, rows (columns <= 0: the record does not touch the tile, or
    // is not this pass'; columns > FPT_MAXC or rows > FPT_MAXR: per voxel)
    __shared__ int4 s_box[FPT_THREADS];

    const int D1 = A == 1 ? 0 : 1, D2 = A == 2 ? 0 : 2;
    const int nS = L.vn[A], n1 = L.vn[D1], n2 = L.vn[D2];
    // slices fastest: the blocks in flight cover few tiles at many slices,
    // which read nearly the same rays, so the ray set-ups are re-read from
    // L2 instead of DRAM
    const int ktiles = (n2 + FPT_TK - 1) / FPT_TK;
    const int s = blockIdx.x % nS, tile = blockIdx.x / nS;
    const int j0 = (tile / ktiles) * FPT_TJ, k0 = (tile % ktiles) * FPT_TK;
    const int tid = threadIdx.x;
    const float half1 = 0.5f * (float)n1, half2 = 0.5f * (float)n2;
    const int rule = 2 - L.rank[A];
    const bool a_fast = L.rank[D1] < L.rank[D2];
    const int off = (s / L.slab) * L.slab;
    const float t1 = __fadd_rn(__fsub_rn((float)off, 0.5f * (float)nS), 0.5f);
    const int nst = s - off;
    const float t = (float)s - 0.5f * (float)nS + 0.5f;
    const int64_t per = (int64_t)L.rows * L.cols;
    // this thread's texels: (j0 + tt / FPT_TK, k0 + tt % FPT_TK), tt = tid, tid + 256
    int tj[2], tk[2];
    float acc[2] = {0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int tt = tid + q * FPT_THREADS;
        tj[q] = j0 + tt / FPT_TK;
        tk[q] = k0 + tt % FPT_TK;
    }
    auto world = [&](int q, int& w0, int& w1, int& w2) {
        const int j = min(tj[q], n1 - 1), kk = min(tk[q], n2 - 1);
        w0 = A == 0 ? s : (D1 == 0 ? j : kk);
        w1 = A == 1 ? s : (D1 == 1 ? j : kk);
        w2 = A == 2 ? s : (D2 == 2 ? kk : j);
    };
    for (int g0 = 0; g0 < L.nrec; g0 += FPT_THREADS) {
        // the candidate boxes of up to 256 records at once, one per thread
        const int gn = min(FPT_THREADS, L.nrec - g0);
        __syncthreads();  // the previous group's boxes are no longer read
        if (tid < gn) {
            const kk_fp_angle* P = L.angles + L.rec0 + g0 + tid;
            int4 bx = make_int4(0, 0, 0, 0);
            if (__ldg(&P->axis) == A && shared_record(P, A, D1)) {
                int c0, c1, rl, rh;
                footprint_box(L, P, A, D1, t, (float)j0 - 0.5f - half1, (float)(j0 + FPT_TJ) + 0.5f - half1,
                              (float)k0 - 0.5f - half2, (float)(k0 + FPT_TK) + 0.5f - half2, c0, c1, rl, rh);
                bx = make_int4(c0, c1 >= c0 && rh >= rl ? c1 - c0 + 1 : 0, rl, rh - rl + 1);
            }
            s_box[tid] = bx;
        }
        __syncthreads();
        for (int kq = 0; kq < gn; ++kq) {
            const int k = g0 + kq;
            const int4 bx = s_box[kq];
            const int c0 = bx.x, nc = bx.y, r0 = bx.z, nr = bx.w;
            if (nc <= 0) continue;  // uniform
            if (nc > FPT_MAXC || nr > FPT_MAXR) {  // beyond the tables: per voxel
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    int w0, w1, w2;
                    world(q, w0, w1, w2);
                    acc[q] += gather_record<TEX8>(L, k, w0, w1, w2);
                }
                continue;
            }
            for (int i = tid; i < nc * (FPT_TK + 1); i += FPT_THREADS) {
                rlo[i] = 1;
                rhi[i] = 0;
            }
            if (tid < FPT_TJ + 1) {
                clo[tid] = 1;
                chi[tid] = 0;
            }
            // (1) the D1 split of every candidate column
            for (int c = tid; c < nc; c += FPT_THREADS) {
                const float4 ab = __ldg(&L.ray_ab[(int64_t)k * per + (int64_t)(c0 + c) * L.rows + r0]);
                const Split sy =
                    split_coord<TEX8>(slice_coord<TEX8>(__fadd_rn(fmaf(ab.x, t1, ab.y), half1), ab.x, nst));
                ci1[c] = sy.i;
                cS[c] = sy.w;
            }
            __syncthreads();
            // the columns of each texel row: the D1 split is monotone in
            // the column, so each row's columns are a range, whose ends are
            // where the split changes (tables are empty where none)
            for (int c = tid; c < nc; c += FPT_THREADS) {
                const int v = ci1[c] - (j0 - 1);
                if (v < 0 || v > FPT_TJ) continue;
                if (c == 0 || ci1[c - 1] != ci1[c]) clo[v] = c;
                if (c == nc - 1 || ci1[c + 1] != ci1[c]) chi[v] = c;
            }
            // (2) every candidate ray: its D2 split and its four contributions
            for (int i = tid; i < nc * nr; i += FPT_THREADS) {
                const int c = i / nr;
                const int64_t id = (int64_t)k * per + (int64_t)(c0 + c) * L.rows + (r0 + i - c * nr);
                const float4 ab = __ldg(&L.ray_ab[id]);
                const Split sz =
                    split_coord<TEX8>(slice_coord<TEX8>(__fadd_rn(fmaf(ab.z, t1, ab.w), half2), ab.z, nst));
                const W4 wt = weights4<TEX8>(cS[c], sz.w, rule, a_fast);
                const float pc = __ldg(&L.ray_pc[id]) * (TEX8 ? 1.f / 256.f : 1.f);
                contrib[i] = make_float4(pc * wt.w00, pc * wt.w01, pc * wt.w10, pc * wt.w11);
                ri2[i] = sz.i;
            }
            __syncthreads();
            // the rows of each (column, texel row): ranges again, ends where
            // the D2 split changes along the column
            for (int i = tid; i < nc * nr; i += FPT_THREADS) {
                const int c = i / nr, r = i - c * nr;
                const int v = ri2[i] - (k0 - 1);
                if (v < 0 || v > FPT_TK) continue;
                if (r == 0 || ri2[i - 1] != ri2[i]) rlo[c * (FPT_TK + 1) + v] = r;
                if (r == nr - 1 || ri2[i + 1] != ri2[i]) rhi[c * (FPT_TK + 1) + v] = r;
            }
            __syncthreads();
            // (3) every texel sums the rays that touch it (each candidate is
            // checked, so a split that is not monotone only costs time)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int j = tj[q], kk = tk[q];
                float sum = 0.f;
#pragma unroll
                for (int di = 0; di < 2; ++di) {
                    const int vj = j - di;  // the ray's D1 texel: j (di = 0) or j - 1 (di = 1)
                    const int cv = vj - (j0 - 1);
                    for (int c = clo[cv]; c <= chi[cv]; ++c) {
                        if (ci1[c] != vj) continue;
#pragma unroll
                        for (int dj = 0; dj < 2; ++dj) {
                            const int vk = kk - dj;
                            const int rv = c * (FPT_TK + 1) + vk - (k0 - 1);
                            for (int r = rlo[rv]; r <= rhi[rv]; ++r) {
                                const int i = c * nr + r;
                                if (ri2[i] != vk) continue;
                                sum += reinterpret_cast<const float*>(&contrib[i])[di * 2 + dj];
                            }
                        }
                    }
                }
                acc[q] += sum;
            }
            __syncthreads();  // the tables are rebuilt for the next record
        }
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        if (tj[q] >= n1 || tk[q] >= n2) continue;
        int w0, w1, w2;
        world(q, w0, w1, w2);
        float* out = L.vol + (int64_t)w0 * L.vs[0] + (int64_t)w1 * L.vs[1] + (int64_t)w2 * L.vs[2];
        *out = L.accumulate ? *out + acc[q] : acc[q];
    }
}

}  // namespace kk

// ===========================================================================
// host side
// ===========================================================================
using namespace kk;

extern "C" int kk_cone_fp_adjoint(const kk_projections* proj, const kk_volume* vol, const kk_fp_angle* angles,
                                  const float* out_scale, int32_t interp, int32_t slab, int32_t additive,
                                  float* work, int64_t work_floats, void* stream) {
    const char* who = "kk_cone_fp_adjoint";
    int rc = check_volume(vol, who);
    if (rc) return rc;
    rc = check_projections(proj, who);
    if (rc) return rc;
    if (!angles || !out_scale) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: angles or out_scale is NULL", who);
    if (interp != KK_INTERP_TEX8 && interp != KK_INTERP_EXACT)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: unknown interpolation mode %d", who, interp);
    if (vol->dtype != KK_F32 || proj->dtype != KK_F32)
        return kk_fail(KK_ERR_UNSUPPORTED, "%s: float32 volume and projections only", who);
    if (proj->table && proj->table_axis != 0)
        return kk_fail(KK_ERR_UNSUPPORTED, "%s: pointer table along the angle axis only", who);
    const int64_t per = proj->rows * proj->cols;
    if (!work || ((uintptr_t)work & 15) != 0)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: work must be a 16-byte aligned device buffer", who);
    const int64_t chunk = work_floats / (5 * per);
    if (chunk < 1)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: work holds %lld floats, at least 5 * rows * cols = %lld needed",
                       who, (long long)work_floats, (long long)(5 * per));
    FptArgs L = {};
    L.vol = (float*)vol->data;
    for (int k = 0; k < 3; ++k) {
        L.vs[k] = vol->stride[k];
        L.vn[k] = (int)vol->shape[k];
        L.ps[k] = proj->stride[k];
    }
    for (int k = 0; k < 3; ++k) {
        L.rank[k] = 0;
        for (int j = 0; j < 3; ++j)
            if (j != k && (vol->stride[j] < vol->stride[k] || (vol->stride[j] == vol->stride[k] && j > k))) ++L.rank[k];
    }
    for (int k = 0; k < 3; ++k) {
        if (L.rank[k] == 2) L.m0 = k;
        if (L.rank[k] == 1) L.m1 = k;
        if (L.rank[k] == 0) L.m2 = k;
    }
    if ((L.vn[L.m1] + FPT_TILE_1 - 1) / FPT_TILE_1 > MAX_GRID_Y || L.vn[L.m0] > MAX_GRID_Y)
        return kk_fail(KK_ERR_UNSUPPORTED, "%s: volume too large for one launch", who);
    L.proj = (const float*)proj->data;
    L.table = proj->table;
    L.rows = (int)proj->rows;
    L.cols = (int)proj->cols;
    L.angles = angles;
    for (int k = 0; k < 9; ++k) L.os[k] = out_scale[k];
    L.slab = slab > 0 ? slab : FP_SLAB;
    const int n = (int)proj->n_angles;
    const int ck = (int)std::min<int64_t>(chunk, n);
    L.ray_ab = (float4*)work;
    L.ray_pc = work + 4 * (int64_t)ck * per;
    const cudaStream_t st = (cudaStream_t)stream;
    const dim3 block(FPT_TILE_2, FPT_TILE_1);
    const dim3 grid((L.vn[L.m2] + FPT_TILE_2 - 1) / FPT_TILE_2, (L.vn[L.m1] + FPT_TILE_1 - 1) / FPT_TILE_1, L.vn[L.m0]);
    const bool tex8 = interp == KK_INTERP_TEX8;
    // the tile passes: one per ray axis A, over that axis' slices
    for (int A = 0; A < 3; ++A) {
        const int D1 = A == 1 ? 0 : 1, D2 = A == 2 ? 0 : 2;
        L.tiled[A] = ((L.vn[D2] + FPT_TK - 1) / FPT_TK) * (int64_t)((L.vn[D1] + FPT_TJ - 1) / FPT_TJ) * L.vn[A] <
                     0x7fffffffLL;
    }
    const void* tk = tex8 ? (const void*)fpt_tile_kernel<true> : (const void*)fpt_tile_kernel<false>;
    rc = kk_allow_smem(tk, FPT_SMEM, who);
    if (rc) return rc;
    for (int r0 = 0; r0 < n; r0 += ck) {
        L.rec0 = r0;
        L.nrec = std::min(ck, n - r0);
        const int first = (r0 > 0 || additive) ? 1 : 0;
        const int64_t rays = (int64_t)L.nrec * per;
        fpt_rays_kernel<<<(unsigned)((rays + 255) / 256), 256, 0, st>>>(L);
        // every voxel is written by the first tile pass (even where no ray
        // of its axis touches it), the later passes and the per-voxel
        // gather of the remaining records add
        bool written = false;
        for (int A = 0; A < 3; ++A) {
            if (!L.tiled[A]) continue;
            const int D1 = A == 1 ? 0 : 1, D2 = A == 2 ? 0 : 2;
            const unsigned tg = (unsigned)(((L.vn[D2] + FPT_TK - 1) / FPT_TK) *
                                           (int64_t)((L.vn[D1] + FPT_TJ - 1) / FPT_TJ) * L.vn[A]);
            L.accumulate = written ? 1 : first;
            if (tex8)
                fpt_tile_kernel<true><<<tg, FPT_THREADS, FPT_SMEM, st>>>(L, A);
            else
                fpt_tile_kernel<false><<<tg, FPT_THREADS, FPT_SMEM, st>>>(L, A);
            written = true;
        }
        L.accumulate = written ? 1 : first;
        if (tex8)
            fpt_gather_kernel<true><<<grid, block, 0, st>>>(L);
        else
            fpt_gather_kernel<false><<<grid, block, 0, st>>>(L);
    }
    return kk_check_launch(who);
}
