// Definitions shared by the cone-beam forward projection (kk_fp.cu,
// ray-driven) and backprojection (kk_bp.cu, voxel-driven) for sm_100a,
// behind the C ABI of include/kk.h.
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
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kk_common.cuh"

namespace kk {

constexpr int FP_SLAB = 16;       // default slices per coordinate restart
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
    int n_angles;
    int col_tiles;  // column tiles per angle
    int slab;       // slices per coordinate restart
    const kk_fp_angle* angles;
    float os[9];
    const void* res_y;  // elements of the projections' type
    const void* res_w;
    int additive;
    int rank[3];  // memory rank of each world axis: 0 fastest .. 2 slowest
    cudaTextureObject_t vtex;  // layered texture of the volume, or 0
    int off32;    // every element offset of the volume fits in 31 bits
    // slices [s_begin, s_end) of every ray's own slice axis are traced in
    // this launch (a multiple of the slab); the epilogue (residual, storage
    // rounding) only in the launch whose final_pass is set
    int s_begin, s_end;
    int final_pass;
    // 16-bit projections traced in several launches: the float32 running
    // sums of this launch's records (record-major, rows x cols each) pass
    // between launches here instead of through the output
    float* sums;
    int load_sums;   // start from sums (later launches)
    int store_sums;  // leave the sums there (all but the last launch)
    // vol is the interior of a copy with two zero texels before and after
    // every axis (the border rule as memory)
    int padded;
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
    const void* upd_scale;  // elements of the volume's type
    const void* upd_mask;
    float vmin, vmax;
    int has_min, has_max;
    cudaTextureObject_t tex;  // layered texture of the projections (FETCH_TEX)
    int j_begin, j_end;       // angles of this launch (one accumulation chunk)
    int load_mode;            // running sum starts from 0 (LOAD_ZERO), vol, work
    int store_mode;           // partial sum goes to vol (STORE_VOL) or work
    float* work;              // float32 running sums between launches
    int fresh;                // running sums were written by other blocks of
                              // this launch: load them past the L1 cache
    int tile_z, tile_y;       // super-column shape in blocks (0: 8 x 64)
};

enum BpLoad { LOAD_ZERO = 0, LOAD_VOL = 1, LOAD_WORK = 2 };
enum BpStore { STORE_VOL = 0, STORE_WORK = 1, STORE_FINAL = 2 };

enum BpFetch { FETCH_GLOBAL = 0, FETCH_TEX = 1 };

}  // namespace kk

// 2D-layered CUDA array with a linear-filtering, border-addressed texture
struct kk_layered {
    cudaArray_t array;
    cudaTextureObject_t tex;
    cudaSurfaceObject_t surf;  // float32 arrays: writable by kernels (FDK filter)
    int64_t layers, height, width;
    int32_t dtype;
};

namespace kk {

__device__ __forceinline__ float pick3(const float* v, int k) {
    return k == 0 ? v[0] : (k == 1 ? v[1] : v[2]);
}

// Ray of the forward projection through detector pixel (r, c): in-slice
// coordinates D1 = a1 A + b1 and D2 = a2 A + b2 along the dominant axis A,
// and the path-length correction. Shared by the projector and its exact
// adjoint, which must see the same bits.
struct RaySetup {
    float a1, a2, b1, b2, corr;
};

// Per-ray slopes/offsets with the reference's float32 operation sequence
// (cuda/cone_fp.cu:150-170, 197).
__device__ __forceinline__ RaySetup ray_setup(const float* src, const float* cor, const float* u, const float* v,
                                              int A, int D1, int D2, int r, int c, float sc1, float sc2) {
    float det[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float ds = __fadd_rn(__fadd_rn(cor[k], __fmul_rn(0.5f, u[k])), __fmul_rn(0.5f, v[k]));
        det[k] = fmaf((float)r, v[k], fmaf((float)c, u[k], ds));
    }
    RaySetup R;
    const float sA = pick3(src, A), s1 = pick3(src, D1), s2 = pick3(src, D2);
    const float sdd = __fsub_rn(sA, pick3(det, A));
    R.a1 = __fdiv_rn(__fsub_rn(s1, pick3(det, D1)), sdd);
    R.a2 = __fdiv_rn(__fsub_rn(s2, pick3(det, D2)), sdd);
    R.b1 = fmaf(-R.a1, sA, s1);
    R.b2 = fmaf(-R.a2, sA, s2);
    R.corr = __fsqrt_rn(__fadd_rn(fmaf(__fmul_rn(R.a1, R.a1), sc1, __fmul_rn(__fmul_rn(R.a2, R.a2), sc2)), 1.f));
    return R;
}
}  // namespace kk

// argument checks shared by the host entry points
inline int check_volume(const kk_volume* v, const char* who) {
    if (!v || !v->data) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: volume is NULL", who);
    for (int k = 0; k < 3; ++k) {
        if (v->shape[k] <= 0 || v->shape[k] >= (int64_t)kk::COORD_LIMIT)
            return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: volume shape[%d]=%lld out of range", who, k,
                           (long long)v->shape[k]);
        if (v->stride[k] <= 0)
            return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: volume stride[%d] must be positive", who, k);
    }
    if (v->dtype < KK_F32 || v->dtype > KK_F16)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: unknown volume dtype %d", who, v->dtype);
    return KK_OK;
}

inline int check_projections(const kk_projections* p, const char* who) {
    if (!p) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: projections descriptor is NULL", who);
    if (!p->data && !p->table) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: projections are NULL", who);
    if (p->table && p->table_axis != 0)
        return kk_fail(KK_ERR_UNSUPPORTED, "%s: a pointer table is supported along the angle axis only", who);
    if (p->n_angles <= 0 || p->rows <= 0 || p->cols <= 0 || p->rows >= (int64_t)kk::COORD_LIMIT ||
        p->cols >= (int64_t)kk::COORD_LIMIT || p->n_angles > (1 << 24))
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: bad projection shape (%lld, %lld, %lld)", who,
                       (long long)p->n_angles, (long long)p->rows, (long long)p->cols);
    for (int k = 0; k < 3; ++k)
        if (p->stride[k] <= 0 && !(p->table && k == 0))
            return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: projection stride[%d] must be positive", who, k);
    if (p->dtype < KK_F32 || p->dtype > KK_F16)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: unknown projection dtype %d", who, p->dtype);
    return KK_OK;
}
