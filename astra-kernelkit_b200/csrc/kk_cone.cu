// Cone-beam forward projection (ray-driven) and backprojection
// (voxel-driven) for sm_100a, behind the C ABI of include/kk.h.
//
// Arithmetic contract. The reference samples through the texture unit,
// whose interpolation weights live on a 1/256 grid, so a one-ulp change
// of a sample coordinate can move a sample by a whole weight step. To
// agree with it sample for sample, both kernels evaluate every coordinate
// with the same float32 operations, in the same order and with the same
// fused multiply-adds as the reference kernels compiled with CUDA's
// default contraction (cuda/cone_fp.cu:141-193, cuda/cone_bp.cu:84-151):
// explicit __f*_rn intrinsics where the reference rounds separately,
// fmaf() where its compiler fuses. Sums keep the reference's grouping
// too: 16-slice slabs per ray (kernels/cone_fp.py:209) and 32-angle
// chunks per voxel (kernels/cone_bp.py:297).
#include <cuda_runtime.h>
#include <stdint.h>

#include "kk_common.cuh"

namespace kk {

constexpr int FP_SLAB = 16;       // default slices per coordinate restart
constexpr int FP_TILE_R = 32;     // rays per block along detector rows (lanes)
constexpr int FP_TILE_C = 8;      // rays per block along detector columns
constexpr int BP_GROUP = 6;       // voxels per thread along the slowest axis
constexpr int BP_CHUNK = 32;      // angles per accumulation chunk
constexpr int BP_TILE_2 = 32;     // voxels per block along the fastest axis
constexpr int BP_TILE_1 = 8;      // voxels per block along the middle axis
constexpr int MAX_GRID_Y = 65535;

enum FpEpilogue { FP_STORE = 0, FP_RESIDUAL = 1 };
enum BpEpilogue { BP_STORE = 0, BP_UPDATE = 1 };

struct FpArgs {
    const void* vol;
    int64_t vs[3];
    int vn[3];
    void* out;
    const uint64_t* table;
    int64_t ps[3];
    int rows, cols;
    int angle0;  // first angle of this launch
    int slab;    // slices per coordinate restart
    const kk_fp_angle* angles;
    float os[9];
    const float* res_y;
    const float* res_w;
    int additive;
    int rank[3];  // memory rank of each world axis: 0 fastest .. 2 slowest
};

struct BpArgs {
    const void* proj;
    const uint64_t* table;
    int64_t ps[3];
    int n_angles, rows, cols;
    void* vol;
    int64_t vs[3];
    int vn[3];
    int m0, m1, m2;  // world axes from slowest to fastest in memory
    const kk_bp_angle* angles;
    float scale;
    int additive;
    const float* upd_scale;
    const float* upd_mask;
    float vmin, vmax;
    int has_min, has_max;
};

__device__ __forceinline__ float pick3(const float* v, int k) {
    return k == 0 ? v[0] : (k == 1 ? v[1] : v[2]);
}

// ---------------------------------------------------------------------------
// forward projection: one thread per ray, whole ray in 16-slice slabs
// ---------------------------------------------------------------------------
template <typename TV, typename TP, bool TEX8, int EPI>
__global__ void __launch_bounds__(FP_TILE_R* FP_TILE_C)
    cone_fp_kernel(const FpArgs L) {
    const int a = L.angle0 + blockIdx.y;
    const int r = blockIdx.x % ((L.rows + FP_TILE_R - 1) / FP_TILE_R) * FP_TILE_R + threadIdx.x;
    const int c = blockIdx.x / ((L.rows + FP_TILE_R - 1) / FP_TILE_R) * FP_TILE_C + threadIdx.y;
    if (r >= L.rows || c >= L.cols) return;

    const kk_fp_angle* P = L.angles + a;
    float src[3], cor[3], u[3], v[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        src[k] = __ldg(&P->src[k]);
        cor[k] = __ldg(&P->corner[k]);
        u[k] = __ldg(&P->u[k]);
        v[k] = __ldg(&P->v[k]);
    }
    const int A = __ldg(&P->axis);
    const int D1 = A == 1 ? 0 : 1;
    const int D2 = A == 2 ? 0 : 2;
    // texture weight rule of the reference's 3D texture: set by the memory
    // rank of the slice axis (slowest: rule 0, middle: 1, fastest: 2)
    const int rule = 2 - L.rank[A];
    const bool a_fast = L.rank[D1] < L.rank[D2];

    // pixel centre: (corner + u/2) + v/2, then + c u + r v (fused as the
    // reference's compiler fuses them)
    float det[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float ds = __fadd_rn(__fadd_rn(cor[k], __fmul_rn(0.5f, u[k])), __fmul_rn(0.5f, v[k]));
        det[k] = fmaf((float)r, v[k], fmaf((float)c, u[k], ds));
    }
    const float sA = pick3(src, A), s1 = pick3(src, D1), s2 = pick3(src, D2);
    const float sdd = __fsub_rn(sA, pick3(det, A));
    const float a1 = __fdiv_rn(__fsub_rn(s1, pick3(det, D1)), sdd);
    const float a2 = __fdiv_rn(__fsub_rn(s2, pick3(det, D2)), sdd);
    const float b1 = fmaf(-a1, sA, s1);
    const float b2 = fmaf(-a2, sA, s2);

    const float sc1 = L.os[3 * A + 0], sc2 = L.os[3 * A + 1], oscale = L.os[3 * A + 2];
    const float corr = __fsqrt_rn(
        __fadd_rn(fmaf(__fmul_rn(a1, a1), sc1, __fmul_rn(__fmul_rn(a2, a2), sc2)), 1.f));

    const int nS = L.vn[A], n1 = L.vn[D1], n2 = L.vn[D2];
    const int64_t sS = L.vs[A], st1 = L.vs[D1], st2 = L.vs[D2];
    const TV* vol = (const TV*)L.vol;
    const float half1 = 0.5f * (float)n1, half2 = 0.5f * (float)n2;

    // output element
    TP* outp;
    {
        const int64_t off = (int64_t)r * L.ps[1] + (int64_t)c * L.ps[2];
        if (L.table)
            outp = (TP*)L.table[a] + off;
        else
            outp = (TP*)L.out + (int64_t)a * L.ps[0] + off;
    }
    float acc = L.additive ? ld_rw(outp) : 0.f;

    for (int off = 0; off < nS; off += L.slab) {
        const float t1 = __fadd_rn(__fsub_rn((float)off, 0.5f * (float)nS), 0.5f);
        float y = __fadd_rn(fmaf(a1, t1, b1), half1);
        float z = __fadd_rn(fmaf(a2, t1, b2), half2);
        const int end = min(off + L.slab, nS);
        float val = 0.f;
        for (int sl = off; sl < end; ++sl) {
            val = __fadd_rn(val, bilinear<TEX8>(vol + (int64_t)sl * sS, st1, st2, n1, n2, y, z, rule, a_fast));
            y = __fadd_rn(y, a1);
            z = __fadd_rn(z, a2);
        }
        val = __fmul_rn(val, corr);
        acc = fmaf(val, oscale, acc);
    }

    if (EPI == FP_RESIDUAL) {
        const int64_t e = (int64_t)a * L.ps[0] + (int64_t)r * L.ps[1] + (int64_t)c * L.ps[2];
        acc = __fmul_rn(__fsub_rn(acc, __ldg(L.res_y + e)), __ldg(L.res_w + e));
    }
    st(outp, acc);
}

// ---------------------------------------------------------------------------
// backprojection: one thread per (fast, middle) voxel column and a group of
// BP_GROUP voxels along the slowest memory axis
// ---------------------------------------------------------------------------
template <typename TP, typename TV, bool TEX8, int EPI>
__global__ void __launch_bounds__(BP_TILE_2* BP_TILE_1) cone_bp_kernel(const BpArgs L) {
    __shared__ kk_bp_angle sp[BP_CHUNK];
    const int i2 = blockIdx.x * BP_TILE_2 + threadIdx.x;
    const int i1 = blockIdx.y * BP_TILE_1 + threadIdx.y;
    const int g0 = blockIdx.z * BP_GROUP;
    const int n0 = L.vn[L.m0], n1 = L.vn[L.m1], n2 = L.vn[L.m2];
    const bool active = i2 < n2 && i1 < n1;
    const int cnt = min(BP_GROUP, n0 - g0);

    // centre of the group's first voxel, world axes
    float f[3];
    f[L.m0] = __fadd_rn(__fsub_rn((float)g0, 0.5f * (float)n0), 0.5f);
    f[L.m1] = __fadd_rn(__fsub_rn((float)i1, 0.5f * (float)n1), 0.5f);
    f[L.m2] = __fadd_rn(__fsub_rn((float)i2, 0.5f * (float)n2), 0.5f);
    const float X = f[0], Y = f[1], Z = f[2];
    const int m0 = L.m0;

    TV* vol = (TV*)L.vol;
    const int64_t vbase = (int64_t)g0 * L.vs[L.m0] + (int64_t)i1 * L.vs[L.m1] + (int64_t)i2 * L.vs[L.m2];
    const int64_t vstep = L.vs[L.m0];

    float acc[BP_GROUP], vacc[BP_GROUP];
#pragma unroll
    for (int i = 0; i < BP_GROUP; ++i) {
        acc[i] = 0.f;
        vacc[i] = (EPI == BP_STORE && L.additive && active && i < cnt) ? ld_rw(vol + vbase + i * vstep) : 0.f;
    }

    const int tid = threadIdx.y * BP_TILE_2 + threadIdx.x;
    for (int j0 = 0; j0 < L.n_angles; j0 += BP_CHUNK) {
        const int nj = min(BP_CHUNK, L.n_angles - j0);
        __syncthreads();
        for (int k = tid; k < nj * 12; k += BP_TILE_2 * BP_TILE_1)
            ((float*)sp)[k] = __ldg((const float*)(L.angles + j0) + k);
        __syncthreads();
        if (!active) continue;
        for (int jj = 0; jj < nj; ++jj) {
            const kk_bp_angle& q = sp[jj];
            const int j = j0 + jj;
            const TP* plane = L.table ? (const TP*)L.table[j] : (const TP*)L.proj + (int64_t)j * L.ps[0];
            float nu = fmaf(Z, q.num_u[2], fmaf(Y, q.num_u[1], fmaf(X, q.num_u[0], q.num_u[3])));
            float nv = fmaf(Z, q.num_v[2], fmaf(Y, q.num_v[1], fmaf(X, q.num_v[0], q.num_v[3])));
            float dn = fmaf(Z, q.den[2], fmaf(Y, q.den[1], fmaf(X, q.den[0], q.den[3])));
            const float du = q.num_u[m0], dv = q.num_v[m0], dd = q.den[m0];
#pragma unroll
            for (int i = 0; i < BP_GROUP; ++i) {
                if (i < cnt) {
                    const float rr = __fdividef(1.f, dn);
                    const float U = __fmul_rn(nu, rr);
                    const float V = __fmul_rn(nv, rr);
                    const float val = bilinear<TEX8>(plane, L.ps[1], L.ps[2], L.rows, L.cols, V, U);
                    acc[i] = fmaf(__fmul_rn(rr, rr), val, acc[i]);
                }
                nu = __fadd_rn(nu, du);
                nv = __fadd_rn(nv, dv);
                dn = __fadd_rn(dn, dd);
            }
        }
#pragma unroll
        for (int i = 0; i < BP_GROUP; ++i) {
            vacc[i] = fmaf(acc[i], L.scale, vacc[i]);
            acc[i] = 0.f;
        }
    }
    if (!active) return;
#pragma unroll
    for (int i = 0; i < BP_GROUP; ++i) {
        if (i >= cnt) break;
        TV* p = vol + vbase + i * vstep;
        if (EPI == BP_UPDATE) {
            const int64_t e = vbase + i * vstep;
            float x = ld_rw(p);
            x = __fsub_rn(x, __fmul_rn(vacc[i], __ldg(L.upd_scale + e)));
            if (L.upd_mask) x = __fmul_rn(x, __ldg(L.upd_mask + e));
            if (L.has_min) x = fmaxf(x, L.vmin);
            if (L.has_max) x = fminf(x, L.vmax);
            st(p, x);
        } else {
            st(p, vacc[i]);
        }
    }
}

}  // namespace kk

// ===========================================================================
// host side
// ===========================================================================
using namespace kk;

static int check_volume(const kk_volume* v, const char* who) {
    if (!v || !v->data) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: volume is NULL", who);
    for (int k = 0; k < 3; ++k) {
        if (v->shape[k] <= 0 || v->shape[k] >= (int64_t)COORD_LIMIT)
            return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: volume shape[%d]=%lld out of range", who, k,
                           (long long)v->shape[k]);
        if (v->stride[k] <= 0)
            return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: volume stride[%d] must be positive", who, k);
    }
    if (v->dtype < KK_F32 || v->dtype > KK_F16)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: unknown volume dtype %d", who, v->dtype);
    return KK_OK;
}

static int check_projections(const kk_projections* p, const char* who) {
    if (!p) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: projections descriptor is NULL", who);
    if (!p->data && !p->table) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: projections are NULL", who);
    if (p->table && p->table_axis != 0)
        return kk_fail(KK_ERR_UNSUPPORTED, "%s: a pointer table is supported along the angle axis only", who);
    if (p->n_angles <= 0 || p->rows <= 0 || p->cols <= 0 || p->rows >= (int64_t)COORD_LIMIT ||
        p->cols >= (int64_t)COORD_LIMIT || p->n_angles > (1 << 24))
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: bad projection shape (%lld, %lld, %lld)", who,
                       (long long)p->n_angles, (long long)p->rows, (long long)p->cols);
    for (int k = 0; k < 3; ++k)
        if (p->stride[k] <= 0 && !(p->table && k == 0))
            return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: projection stride[%d] must be positive", who, k);
    if (p->dtype < KK_F32 || p->dtype > KK_F16)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: unknown projection dtype %d", who, p->dtype);
    return KK_OK;
}

template <typename TV, typename TP, int EPI>
static void launch_fp_typed(const FpArgs& base, int n_angles, bool tex8, cudaStream_t s) {
    const int tiles = ((base.rows + FP_TILE_R - 1) / FP_TILE_R) * ((base.cols + FP_TILE_C - 1) / FP_TILE_C);
    for (int a0 = 0; a0 < n_angles; a0 += MAX_GRID_Y) {
        FpArgs L = base;
        L.angle0 = a0;
        dim3 grid(tiles, min(MAX_GRID_Y, n_angles - a0));
        dim3 block(FP_TILE_R, FP_TILE_C);
        if (tex8)
            cone_fp_kernel<TV, TP, true, EPI><<<grid, block, 0, s>>>(L);
        else
            cone_fp_kernel<TV, TP, false, EPI><<<grid, block, 0, s>>>(L);
    }
}

template <int EPI>
static int launch_fp(const FpArgs& L, int n_angles, int vdt, int pdt, bool tex8, cudaStream_t s) {
#define KK_FP_CASE(VD, PD, TV, TP)                                   \
    if (vdt == VD && pdt == PD) {                                    \
        launch_fp_typed<TV, TP, EPI>(L, n_angles, tex8, s);          \
        return kk_check_launch("kk_cone_fp");                         \
    }
    KK_FP_CASE(KK_F32, KK_F32, float, float)
    if (EPI == FP_STORE) {
        KK_FP_CASE(KK_BF16, KK_F32, __nv_bfloat16, float)
        KK_FP_CASE(KK_F16, KK_F32, __half, float)
        KK_FP_CASE(KK_BF16, KK_F16, __nv_bfloat16, __half)
        KK_FP_CASE(KK_F16, KK_F16, __half, __half)
        KK_FP_CASE(KK_BF16, KK_BF16, __nv_bfloat16, __nv_bfloat16)
        KK_FP_CASE(KK_F32, KK_F16, float, __half)
        KK_FP_CASE(KK_F32, KK_BF16, float, __nv_bfloat16)
    }
#undef KK_FP_CASE
    return kk_fail(KK_ERR_UNSUPPORTED, "kk_cone_fp: dtype combination volume=%d projections=%d", vdt, pdt);
}

static int fill_fp_args(FpArgs& L, const kk_volume* vol, const kk_projections* proj, const kk_fp_angle* angles,
                        const float* out_scale, int32_t interp, int32_t slab, const char* who) {
    int rc = check_volume(vol, who);
    if (rc) return rc;
    rc = check_projections(proj, who);
    if (rc) return rc;
    if (!angles) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: angle parameters are NULL", who);
    if (!out_scale) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: out_scale is NULL", who);
    if (interp != KK_INTERP_TEX8 && interp != KK_INTERP_EXACT)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: unknown interpolation mode %d", who, interp);
    L = FpArgs{};
    L.vol = vol->data;
    for (int k = 0; k < 3; ++k) {
        L.vs[k] = vol->stride[k];
        L.vn[k] = (int)vol->shape[k];
        L.ps[k] = proj->stride[k];
    }
    L.out = proj->data;
    L.table = proj->table;
    L.rows = (int)proj->rows;
    L.cols = (int)proj->cols;
    L.angles = angles;
    for (int k = 0; k < 9; ++k) L.os[k] = out_scale[k];
    L.slab = slab > 0 ? slab : FP_SLAB;
    for (int k = 0; k < 3; ++k) {
        L.rank[k] = 0;
        for (int j = 0; j < 3; ++j)
            if (j != k && (vol->stride[j] < vol->stride[k] || (vol->stride[j] == vol->stride[k] && j > k)))
                ++L.rank[k];
    }
    return KK_OK;
}

extern "C" int kk_cone_fp(const kk_volume* vol, const kk_projections* proj, const kk_fp_angle* angles,
                          const float* out_scale, int32_t interp, int32_t slab, int32_t additive, void* stream) {
    FpArgs L;
    int rc = fill_fp_args(L, vol, proj, angles, out_scale, interp, slab, "kk_cone_fp");
    if (rc) return rc;
    L.additive = additive ? 1 : 0;
    return launch_fp<FP_STORE>(L, (int)proj->n_angles, vol->dtype, proj->dtype, interp == KK_INTERP_TEX8,
                               (cudaStream_t)stream);
}

extern "C" int kk_cone_fp_residual(const kk_volume* vol, const kk_projections* out, const kk_fp_angle* angles,
                                   const float* out_scale, const kk_fp_residual* residual, int32_t interp,
                                   int32_t slab, void* stream) {
    FpArgs L;
    int rc = fill_fp_args(L, vol, out, angles, out_scale, interp, slab, "kk_cone_fp_residual");
    if (rc) return rc;
    if (!residual || !residual->y || !residual->weight)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "kk_cone_fp_residual: residual operands are NULL");
    if (out->table)
        return kk_fail(KK_ERR_UNSUPPORTED, "kk_cone_fp_residual: strided projections only");
    if (out->dtype != KK_F32 || vol->dtype != KK_F32)
        return kk_fail(KK_ERR_UNSUPPORTED, "kk_cone_fp_residual: float32 volume and projections only");
    L.res_y = residual->y;
    L.res_w = residual->weight;
    return launch_fp<FP_RESIDUAL>(L, (int)out->n_angles, vol->dtype, out->dtype, interp == KK_INTERP_TEX8,
                                  (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------

template <typename TP, typename TV, int EPI>
static void launch_bp_typed(const BpArgs& L, bool tex8, cudaStream_t s) {
    dim3 block(BP_TILE_2, BP_TILE_1);
    dim3 grid((L.vn[L.m2] + BP_TILE_2 - 1) / BP_TILE_2, (L.vn[L.m1] + BP_TILE_1 - 1) / BP_TILE_1,
              (L.vn[L.m0] + BP_GROUP - 1) / BP_GROUP);
    if (tex8)
        cone_bp_kernel<TP, TV, true, EPI><<<grid, block, 0, s>>>(L);
    else
        cone_bp_kernel<TP, TV, false, EPI><<<grid, block, 0, s>>>(L);
}

template <int EPI>
static int launch_bp(const BpArgs& L, int pdt, int vdt, bool tex8, cudaStream_t s) {
#define KK_BP_CASE(PD, VD, TP, TV)                          \
    if (pdt == PD && vdt == VD) {                           \
        launch_bp_typed<TP, TV, EPI>(L, tex8, s);           \
        return kk_check_launch("kk_cone_bp");                \
    }
    KK_BP_CASE(KK_F32, KK_F32, float, float)
    if (EPI == BP_STORE) {
        KK_BP_CASE(KK_F16, KK_F32, __half, float)
        KK_BP_CASE(KK_BF16, KK_F32, __nv_bfloat16, float)
        KK_BP_CASE(KK_F16, KK_BF16, __half, __nv_bfloat16)
        KK_BP_CASE(KK_F16, KK_F16, __half, __half)
        KK_BP_CASE(KK_BF16, KK_BF16, __nv_bfloat16, __nv_bfloat16)
        KK_BP_CASE(KK_F32, KK_BF16, float, __nv_bfloat16)
        KK_BP_CASE(KK_F32, KK_F16, float, __half)
    }
#undef KK_BP_CASE
    return kk_fail(KK_ERR_UNSUPPORTED, "kk_cone_bp: dtype combination projections=%d volume=%d", pdt, vdt);
}

static int fill_bp_args(BpArgs& L, const kk_projections* proj, const kk_volume* vol, const kk_bp_angle* angles,
                        float out_scale, int32_t interp, const char* who) {
    int rc = check_volume(vol, who);
    if (rc) return rc;
    rc = check_projections(proj, who);
    if (rc) return rc;
    if (!angles) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: angle parameters are NULL", who);
    if (interp != KK_INTERP_TEX8 && interp != KK_INTERP_EXACT)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: unknown interpolation mode %d", who, interp);
    L = BpArgs{};
    L.proj = proj->data;
    L.table = proj->table;
    for (int k = 0; k < 3; ++k) {
        L.ps[k] = proj->stride[k];
        L.vs[k] = vol->stride[k];
        L.vn[k] = (int)vol->shape[k];
    }
    L.n_angles = (int)proj->n_angles;
    L.rows = (int)proj->rows;
    L.cols = (int)proj->cols;
    L.vol = vol->data;
    L.angles = angles;
    L.scale = out_scale;
    // memory order of the world axes: the largest stride is the slowest
    // axis, the one the reference's threads step along (cone_bp.cu:148-151)
    int ord[3] = {0, 1, 2};
    for (int i = 0; i < 3; ++i)
        for (int j = i + 1; j < 3; ++j)
            if (vol->stride[ord[j]] > vol->stride[ord[i]]) {
                int t = ord[i];
                ord[i] = ord[j];
                ord[j] = t;
            }
    L.m0 = ord[0];
    L.m1 = ord[1];
    L.m2 = ord[2];
    if ((vol->shape[L.m1] + BP_TILE_1 - 1) / BP_TILE_1 > MAX_GRID_Y ||
        (vol->shape[L.m0] + BP_GROUP - 1) / BP_GROUP > MAX_GRID_Y)
        return kk_fail(KK_ERR_UNSUPPORTED, "%s: volume too large for one launch", who);
    return KK_OK;
}

extern "C" int kk_cone_bp(const kk_projections* proj, const kk_volume* vol, const kk_bp_angle* angles,
                          float out_scale, int32_t interp, int32_t additive, void* stream) {
    BpArgs L;
    int rc = fill_bp_args(L, proj, vol, angles, out_scale, interp, "kk_cone_bp");
    if (rc) return rc;
    L.additive = additive ? 1 : 0;
    return launch_bp<BP_STORE>(L, proj->dtype, vol->dtype, interp == KK_INTERP_TEX8, (cudaStream_t)stream);
}

extern "C" int kk_cone_bp_update(const kk_projections* proj, const kk_volume* vol, const kk_bp_angle* angles,
                                 float out_scale, const kk_bp_update* update, int32_t interp, void* stream) {
    BpArgs L;
    int rc = fill_bp_args(L, proj, vol, angles, out_scale, interp, "kk_cone_bp_update");
    if (rc) return rc;
    if (!update || !update->scale)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "kk_cone_bp_update: update scale is NULL");
    if (proj->dtype != KK_F32 || vol->dtype != KK_F32)
        return kk_fail(KK_ERR_UNSUPPORTED, "kk_cone_bp_update: float32 volume and projections only");
    L.upd_scale = update->scale;
    L.upd_mask = update->mask;
    L.vmin = update->min_value;
    L.vmax = update->max_value;
    L.has_min = update->has_min;
    L.has_max = update->has_max;
    return launch_bp<BP_UPDATE>(L, proj->dtype, vol->dtype, interp == KK_INTERP_TEX8, (cudaStream_t)stream);
}
