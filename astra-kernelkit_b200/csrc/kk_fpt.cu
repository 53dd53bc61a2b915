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

template <bool TEX8>
__global__ void __launch_bounds__(FPT_TILE_2* FPT_TILE_1) fpt_gather_kernel(const FptArgs L) {
    const int i2 = blockIdx.x * FPT_TILE_2 + threadIdx.x;
    const int i1 = blockIdx.y * FPT_TILE_1 + threadIdx.y;
    const int i0 = blockIdx.z;
    if (i2 >= L.vn[L.m2] || i1 >= L.vn[L.m1]) return;
    // world indices of the voxel
    const int w0 = L.m0 == 0 ? i0 : (L.m1 == 0 ? i1 : i2);
    const int w1 = L.m0 == 1 ? i0 : (L.m1 == 1 ? i1 : i2);
    const int w2 = L.m0 == 2 ? i0 : (L.m1 == 2 ? i1 : i2);
    const int64_t per = (int64_t)L.rows * L.cols;
    float acc = 0.f;
    for (int k = 0; k < L.nrec; ++k) {
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

        // detector coordinates (pixel units, centre of pixel c at c + 1/2)
        // of the footprint's corners, by central projection from the source
        float nrm[3], e1[3], e2[3], tmp[3];
        cross3(u, v, nrm);
        cross3(v, nrm, tmp);
        const float ue = dot3(u, tmp);
        cross3(nrm, u, e2);
        const float ve = dot3(v, e2);
        // the candidate box only needs a few correct digits (it is widened
        // by 0.05 pixel), so the fast reciprocal and division suffice
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
        const float t = (float)s - 0.5f * (float)nS + 0.5f;
        float amin = 1e30f, amax = -1e30f, bmin = 1e30f, bmax = -1e30f;
        bool ok = true;
#pragma unroll
        for (int corner = 0; corner < 4; ++corner) {
            const float d1 = (float)jv - 0.5f - half1 + ((corner & 1) ? 2.f : 0.f);
            const float d2 = (float)kv - 0.5f - half2 + ((corner & 2) ? 2.f : 0.f);
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
        int c0 = 0, c1 = L.cols - 1, rlo = 0, rhi = L.rows - 1;
        if (ok && isfinite(amin) && isfinite(amax) && isfinite(bmin) && isfinite(bmax)) {
            // pixel c is a candidate when c + 1/2 lies in [amin, amax]
            c0 = max(c0, (int)ceilf(fmaxf(amin - 0.55f, -1.f)));
            c1 = min(c1, (int)floorf(fminf(amax - 0.45f, (float)L.cols)));
            rlo = max(rlo, (int)ceilf(fmaxf(bmin - 0.55f, -1.f)));
            rhi = min(rhi, (int)floorf(fminf(bmax - 0.45f, (float)L.rows)));
        }
        const int off = (s / L.slab) * L.slab;
        const float t1 = __fadd_rn(__fsub_rn((float)off, 0.5f * (float)nS), 0.5f);
        // circular scans: the detector's v has no component along A and D1,
        // so every row of a column has bit for bit the same D1 coordinate
        // sequence (as in the forward projector's shared path); a column
        // whose D1 sample misses the voxel is then skipped whole
        const float vA = A == 0 ? v[0] : (A == 1 ? v[1] : v[2]);
        const float vD1 = D1 == 0 ? v[0] : v[1];
        const bool shared = vA == 0.f && vD1 == 0.f;
        const int nst = s - off;
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
                    col ? syc
                        : split_coord<TEX8>(slice_coord<TEX8>(__fadd_rn(fmaf(ab.x, t1, ab.y), half1), ab.x, nst));
                const Split sz =
                    split_coord<TEX8>(slice_coord<TEX8>(__fadd_rn(fmaf(ab.z, t1, ab.w), half2), ab.z, nst));
                const int di = jv - sy.i, dj = kv - sz.i;
                if ((unsigned)di > 1u || (unsigned)dj > 1u) continue;
                const W4 wt = weights4<TEX8>(sy.w, sz.w, rule, a_fast);
                float wgt = di == 0 ? (dj == 0 ? wt.w00 : wt.w01) : (dj == 0 ? wt.w10 : wt.w11);
                if (TEX8) wgt *= 1.f / 256.f;
                acc = fmaf(__ldg(&L.ray_pc[id]), wgt, acc);
            }
        }
    }
    float* out = L.vol + (int64_t)w0 * L.vs[0] + (int64_t)w1 * L.vs[1] + (int64_t)w2 * L.vs[2];
    *out = L.accumulate ? *out + acc : acc;
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
    for (int r0 = 0; r0 < n; r0 += ck) {
        L.rec0 = r0;
        L.nrec = std::min(ck, n - r0);
        L.accumulate = (r0 > 0 || additive) ? 1 : 0;
        const int64_t rays = (int64_t)L.nrec * per;
        fpt_rays_kernel<<<(unsigned)((rays + 255) / 256), 256, 0, st>>>(L);
        if (interp == KK_INTERP_TEX8)
            fpt_gather_kernel<true><<<grid, block, 0, st>>>(L);
        else
            fpt_gather_kernel<false><<<grid, block, 0, st>>>(L);
    }
    return kk_check_launch(who);
}
