// Cone-beam backprojection (voxel-driven) for sm_100a: kernel, layered
// projection textures and the kk_cone_bp* entry points of include/kk.h.
#include <algorithm>
#include <mutex>

#ifndef KK_BP_LANES
#define KK_BP_LANES 1  // 2 x 2 quads of lanes (0: lanes along the fastest axis)
#endif
#ifndef KK_BP_WZ
#define KK_BP_WZ 16  // voxels per warp along the fastest axis
#endif

#include "kk_cone.cuh"

namespace kk {

// ---------------------------------------------------------------------------
// backprojection: one thread per (fast, middle) voxel column and a group of
// BP_GROUP voxels along the slowest memory axis
// ---------------------------------------------------------------------------
template <typename TP, typename TV, bool TEX8, int EPI, int FETCH>
__device__ __forceinline__ void bp_block(const BpArgs& L, int bx, int by, int bz) {
    // One launch covers the angles [j_begin, j_end): one 32-angle chunk,
    // as one launch of the reference does (kernels/cone_bp.py:297-302), so
    // the chunk's projections stay in L2 while every voxel reads them; the
    // running sum vol += acc * scale is carried between launches in the
    // volume (float32) or in the float32 work buffer.
    __shared__ kk_bp_angle sp[BP_CHUNK];
#if KK_BP_LANES == 0
    const int i2 = bx * BP_TILE_2 + threadIdx.x;
    const int i1 = by * BP_TILE_1 + threadIdx.y;
#else
    // warps cover KK_BP_WZ (fastest axis) x 32 / KK_BP_WZ (middle axis)
    // voxels, and every quad of lanes a 2 x 2 square of them
    const int lane = threadIdx.x, w = threadIdx.y;
    constexpr int WZ = KK_BP_WZ, WY = 32 / WZ;
    const int zl = (lane & 1) | (((lane >> 2) * 2) % WZ);
    const int yl = ((lane >> 1) & 1) | ((((lane >> 2) * 2) / WZ) * 2);
    const int i2 = bx * BP_TILE_2 + (w % (BP_TILE_2 / WZ)) * WZ + zl;
    const int i1 = by * BP_TILE_1 + (w / (BP_TILE_2 / WZ)) * WY + yl;
#endif
    const int g0 = bz * BP_GROUP;
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
    // the work buffer is dense in the volume's memory order
    const int64_t wbase = ((int64_t)g0 * n1 + i1) * n2 + i2;
    const int64_t wstep = (int64_t)n1 * n2;

    float acc[BP_GROUP], vacc[BP_GROUP];
#pragma unroll
    for (int i = 0; i < BP_GROUP; ++i) {
        acc[i] = 0.f;
        vacc[i] = 0.f;
        if (active && i < cnt) {
            if (L.load_mode == LOAD_VOL)
                vacc[i] = L.fresh ? ld_cv(vol + vbase + i * vstep) : ld_cs(vol + vbase + i * vstep);
            else if (L.load_mode == LOAD_WORK)
                vacc[i] = L.fresh ? __ldcv(L.work + wbase + i * wstep) : ld_cs(L.work + wbase + i * wstep);
        }
    }

    const int tid = threadIdx.y * BP_TILE_2 + threadIdx.x;
    for (int j0 = L.j_begin; j0 < L.j_end; j0 += BP_CHUNK) {
        const int nj = min(BP_CHUNK, L.j_end - j0);
        __syncthreads();
        for (int k = tid; k < nj * 12; k += BP_TILE_2 * BP_TILE_1)
            ((float*)sp)[k] = __ldg((const float*)(L.angles + j0) + k);
        __syncthreads();
        if (!active) continue;
        for (int jj = 0; jj < nj; ++jj) {
            const kk_bp_angle& q = sp[jj];
            const int j = j0 + jj;
            const TP* plane = FETCH == FETCH_TEX ? nullptr
                              : (L.table ? (const TP*)L.table[j] : (const TP*)L.proj + (int64_t)j * L.ps[0]);
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
                    float val;
                    if (FETCH == FETCH_TEX)  // the hardware filter the reference samples with
                        val = tex2DLayered<float>(L.tex, U, V, j);
                    else
                        val = bilinear<TEX8>(plane, L.ps[1], L.ps[2], L.rows, L.cols, V, U);
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
        if (L.store_mode == STORE_WORK) {
            st_cs(L.work + wbase + i * wstep, vacc[i]);
        } else if (EPI == BP_UPDATE) {
            const int64_t e = vbase + i * vstep;
            float x = L.fresh ? ld_cv(p) : ld_cs(p);
            x = __fsub_rn(x, __fmul_rn(vacc[i], ld((const TV*)L.upd_scale + e)));
            if (L.upd_mask) x = __fmul_rn(x, ld((const TV*)L.upd_mask + e));
            if (L.has_min) x = fmaxf(x, L.vmin);
            if (L.has_max) x = fminf(x, L.vmax);
            st_cs(p, x);
        } else {
            st_cs(p, vacc[i]);
        }
    }
}

// Blocks run in super-columns: TZ x TY blocks of the two faster axes (up
// to 256 x 512 voxels) swept along the slowest axis, so the blocks in
// flight at any time cover a compact region of the volume whose footprint
// on each projection is small, and the chunk's projections are re-read
// from L2 rather than DRAM (headline BP 97.7 -> 92.6 ms against the plain
// x-fastest order, whose in-flight slab covers most of every projection).
// TZ, TY are the largest powers of two up to KK_BP_TILE_Z and KK_BP_TILE_Y
// dividing the grid's extents nx, ny, so the map from the linear block
// index is a bijection of the nx x ny x nz grid. With four chunks per
// launch (below) the smaller 4 x 32 super-columns keep the four chunks'
// projection footprints in L2 (headline BP: 8 x 64 with one chunk 92.8
// ms; 4 x 32 with 2 / 4 / 6 chunks 91.1 / 90.5 / 90.6 ms; 8 x 64 with 2
// chunks 96.1 ms; 8 x 32 with 4 chunks 94.9 ms; identical output).
#ifndef KK_BP_TILE_Z
#define KK_BP_TILE_Z 4  // super-column extent in blocks along the fastest axis
#endif
#ifndef KK_BP_TILE_Y
#define KK_BP_TILE_Y 32  // and along the middle axis
#endif
__device__ __forceinline__ void bp_tile_order(int lin, int nx, int ny, int nz, int& bx, int& by, int& bz,
                                              int tz_max = KK_BP_TILE_Z, int ty_max = KK_BP_TILE_Y) {
    const int TZ = min(tz_max, nx & -nx), TY = min(ty_max, ny & -ny);
    const int per_x = TZ * TY, col_blocks = per_x * nz;
    const int col = lin / col_blocks, r = lin - col * col_blocks;
    bz = r / per_x;
    const int q = r - bz * per_x;
    const int scx = nx / TZ;
    bx = (col % scx) * TZ + q % TZ;
    by = (col / scx) * TY + q / TZ;
}

template <typename TP, typename TV, bool TEX8, int EPI, int FETCH>
__global__ void __launch_bounds__(BP_TILE_2* BP_TILE_1) cone_bp_kernel(const BpArgs L) {
    int bx, by, bz;
    bp_tile_order(blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z), gridDim.x, gridDim.y,
                  gridDim.z, bx, by, bz, L.tile_z > 0 ? L.tile_z : KK_BP_TILE_Z,
                  L.tile_y > 0 ? L.tile_y : KK_BP_TILE_Y);
    bp_block<TP, TV, TEX8, EPI, FETCH>(L, bx, by, bz);
}

// Many problems in one launch (one 32-angle chunk of each): argument
// blocks in the kernel's parameter space, as for the batched forward
// projection; tiles[i] = (x tiles, y tiles) of problem i's grid.
struct BpBatch {
    int n;
    int block_start[KK_MAX_BATCH + 1];
    int tiles[KK_MAX_BATCH][2];
    BpArgs p[KK_MAX_BATCH];
};

template <int EPI>
__global__ void __launch_bounds__(BP_TILE_2* BP_TILE_1) cone_bp_batched_kernel(const __grid_constant__ BpBatch B) {
    __shared__ BpArgs Ls;
    const int b = blockIdx.x;
    int i = 0;
    while (i + 1 < B.n && B.block_start[i + 1] <= b) ++i;
    static_assert(sizeof(BpArgs) % 4 == 0 && sizeof(BpArgs) <= 4 * BP_TILE_2 * BP_TILE_1, "argument copy");
    const int tid = threadIdx.y * BP_TILE_2 + threadIdx.x;
    const int* src = reinterpret_cast<const int*>(&B.p[i]);
    for (int k = tid; k < (int)(sizeof(BpArgs) / 4); k += BP_TILE_2 * BP_TILE_1) reinterpret_cast<int*>(&Ls)[k] = src[k];
    __syncthreads();
    const int t = b - B.block_start[i];
    const int tx = B.tiles[i][0], ty = B.tiles[i][1];
    const int tz = (B.block_start[i + 1] - B.block_start[i]) / (tx * ty);
    int bx, by, bz;
    // one chunk per launch here: the one-chunk super-column default
    bp_tile_order(t, tx, ty, tz, bx, by, bz, Ls.tile_z > 0 ? Ls.tile_z : 8, Ls.tile_y > 0 ? Ls.tile_y : 64);
    bp_block<float, float, true, EPI, FETCH_TEX>(Ls, bx, by, bz);
}

// ---------------------------------------------------------------------------
// persistent batched backprojection
// ---------------------------------------------------------------------------
// One grid of resident blocks works through every (chunk group, problem,
// tile) item of a batch, a group being BP_PERSIST_GROUP consecutive
// 32-angle chunks that one item backprojects with its running sum in
// registers (each chunk still added on its own, as in the other paths): a
// block claims the next item from a counter in global memory, items
// ordered by group index first, so every group of a tile is claimed after
// the tile's previous group. An item of group c > 0 starts from the
// running sums its tile's group c - 1 left behind: it waits until the
// tile's counter says c groups are done (spinning with a clock64()
// budget; a wait that runs out records a timeout, raises the abort flag
// and skips the item, and every block stops claiming), runs the same
// block code as the one-launch-per-chunk path, then publishes c + 1. The
// item that is waited on was claimed earlier by a running block, which
// itself only waits on still earlier items, so the waits always end.
constexpr int BP_MAX_CHUNKS = 64;  // 2048 angles, the layered-texture limit
constexpr int BP_PERSIST_GROUP = 4;  // 32-angle chunks per item

struct BpSched {
    int n;       // problems
    int chunks;  // largest chunk-group count
    int items;
    int skip_item;  // tests of the bounded wait: this item is never run
    long long budget;
    int cstart[BP_MAX_CHUNKS + 1];  // first item of each group index
    int nchunks[KK_MAX_BATCH];      // chunk groups per problem
    int tiles[KK_MAX_BATCH];
    int grid[KK_MAX_BATCH][3];
    int tile_base[KK_MAX_BATCH];  // first counter of each problem
    BpArgs p[KK_MAX_BATCH];
};

static __device__ unsigned int g_bp_timeouts;

__global__ void __launch_bounds__(BP_TILE_2* BP_TILE_1) cone_bp_persistent_kernel(const __grid_constant__ BpSched S,
                                                                                  int* sync) {
    __shared__ BpArgs Ls;
    __shared__ int s_item, s_go;
    const int tid = threadIdx.y * BP_TILE_2 + threadIdx.x;
    volatile int* abort_flag = sync + 1;
    for (;;) {
        if (tid == 0) s_item = *abort_flag ? S.items : atomicAdd(sync, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= S.items) return;
        int c = 0;
        while (c + 1 < S.chunks && S.cstart[c + 1] <= item) ++c;
        int t = item - S.cstart[c], p = 0;
        for (; p + 1 < S.n; ++p) {
            if (S.nchunks[p] <= c) continue;
            if (t < S.tiles[p]) break;
            t -= S.tiles[p];
        }
        const int* src = reinterpret_cast<const int*>(&S.p[p]);
        for (int k = tid; k < (int)(sizeof(BpArgs) / 4); k += BP_TILE_2 * BP_TILE_1)
            reinterpret_cast<int*>(&Ls)[k] = src[k];
        volatile int* done = sync + 2 + S.tile_base[p] + t;
        __syncthreads();
        if (tid == 0) {
            bool ok = item != S.skip_item;
            if (ok && c > 0 && *done < c) {
                const long long t0 = clock64();
                while (*done < c) {
                    if (*abort_flag || clock64() - t0 > S.budget) {
                        ok = false;
                        if (!*abort_flag) atomicAdd(&g_bp_timeouts, 1u);
                        *abort_flag = 1;
                        break;
                    }
                    __nanosleep(256);
                }
            }
            __threadfence();  // the previous chunk's sums before ours
            Ls.j_begin = c * BP_CHUNK * BP_PERSIST_GROUP;
            Ls.j_end = min(Ls.n_angles, Ls.j_begin + BP_CHUNK * BP_PERSIST_GROUP);
            const bool update = Ls.upd_scale != nullptr;
            const bool need_work = S.nchunks[p] > 1 && update;  // float32 volumes
            const int first_load = (Ls.additive && !update) ? LOAD_VOL : LOAD_ZERO;
            Ls.load_mode = c == 0 ? first_load : (need_work ? LOAD_WORK : LOAD_VOL);
            Ls.store_mode = c == S.nchunks[p] - 1 ? STORE_FINAL : (need_work ? STORE_WORK : STORE_VOL);
            Ls.fresh = 1;
            s_go = ok;
        }
        __syncthreads();
        if (s_go) {
            int bx, by, bz;
            bp_tile_order(t, S.grid[p][0], S.grid[p][1], S.grid[p][2], bx, by, bz,
                          Ls.tile_z > 0 ? Ls.tile_z : KK_BP_TILE_Z, Ls.tile_y > 0 ? Ls.tile_y : KK_BP_TILE_Y);
            if (Ls.upd_scale)
                bp_block<float, float, true, BP_UPDATE, FETCH_TEX>(Ls, bx, by, bz);
            else
                bp_block<float, float, true, BP_STORE, FETCH_TEX>(Ls, bx, by, bz);
            __syncthreads();
            if (tid == 0) {
                __threadfence();  // our sums before the count
                atomicExch((int*)done, c + 1);
            }
        }
        __syncthreads();  // s_item and Ls are rewritten next round
    }
}

}  // namespace kk

// ===========================================================================
// host side
// ===========================================================================
using namespace kk;

// ---------------------------------------------------------------------------

static dim3 bp_grid(const BpArgs& L) {
    return dim3((L.vn[L.m2] + BP_TILE_2 - 1) / BP_TILE_2, (L.vn[L.m1] + BP_TILE_1 - 1) / BP_TILE_1,
                (L.vn[L.m0] + BP_GROUP - 1) / BP_GROUP);
}

template <typename TP, typename TV, int EPI>
static void launch_bp_typed(const BpArgs& L, bool tex8, cudaStream_t s) {
    dim3 block(BP_TILE_2, BP_TILE_1);
    if (tex8)
        cone_bp_kernel<TP, TV, true, EPI, FETCH_GLOBAL><<<bp_grid(L), block, 0, s>>>(L);
    else
        cone_bp_kernel<TP, TV, false, EPI, FETCH_GLOBAL><<<bp_grid(L), block, 0, s>>>(L);
}

// Launch `one` once per KK_BP_CHUNKS_PER_LAUNCH 32-angle chunks (each
// chunk's sum is still added to the running sum on its own, in chunk
// order, inside the launch: the reference's grouping). The running sum
// lives in the volume when it is float32 and the result is a plain sum;
// otherwise in the float32 work buffer (when given). Without a buffer in
// those cases a single launch covers every angle (same arithmetic, more L2
// traffic). Fewer launches save the running sum's round trip through
// memory between chunks.
#ifndef KK_BP_CHUNKS_PER_LAUNCH
#define KK_BP_CHUNKS_PER_LAUNCH 4
#endif
constexpr int BP_LAUNCH_ANGLES = BP_CHUNK * KK_BP_CHUNKS_PER_LAUNCH;

template <typename Fn>
static void bp_chunks(BpArgs L, bool vol_f32, bool additive, bool update, Fn one) {
    const int n = L.n_angles;
    const int chunks = (n + BP_LAUNCH_ANGLES - 1) / BP_LAUNCH_ANGLES;
    const bool need_work = chunks > 1 && (!vol_f32 || update);
    const int first_load = (additive && !update) ? LOAD_VOL : LOAD_ZERO;
    if (need_work && !L.work) {
        L.j_begin = 0;
        L.j_end = n;
        L.load_mode = first_load;
        L.store_mode = STORE_FINAL;
        one(L);
        return;
    }
    for (int c = 0; c < chunks; ++c) {
        L.j_begin = c * BP_LAUNCH_ANGLES;
        L.j_end = min(n, L.j_begin + BP_LAUNCH_ANGLES);
        L.load_mode = c == 0 ? first_load : (need_work ? LOAD_WORK : LOAD_VOL);
        L.store_mode = c == chunks - 1 ? STORE_FINAL : (need_work ? STORE_WORK : STORE_VOL);
        one(L);
    }
}

template <int EPI>
static int launch_bp(const BpArgs& L, int pdt, int vdt, bool tex8, bool additive, cudaStream_t s) {
#define KK_BP_CASE(PD, VD, TP, TV)                                                                  \
    if (pdt == PD && vdt == VD) {                                                                   \
        bp_chunks(L, VD == KK_F32, additive, EPI == BP_UPDATE,                                      \
                  [&](const BpArgs& c) { launch_bp_typed<TP, TV, EPI>(c, tex8, s); });             \
        return kk_check_launch("kk_cone_bp");                                                      \
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
                          float out_scale, int32_t interp, int32_t additive, float* work, void* stream) {
    BpArgs L;
    int rc = fill_bp_args(L, proj, vol, angles, out_scale, interp, "kk_cone_bp");
    if (rc) return rc;
    L.work = work;
    return launch_bp<BP_STORE>(L, proj->dtype, vol->dtype, interp == KK_INTERP_TEX8, additive != 0,
                               (cudaStream_t)stream);
}

extern "C" int kk_cone_bp_update(const kk_projections* proj, const kk_volume* vol, const kk_bp_angle* angles,
                                 float out_scale, const kk_bp_update* update, int32_t interp, float* work,
                                 void* stream) {
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
    L.work = work;
    return launch_bp<BP_UPDATE>(L, proj->dtype, vol->dtype, interp == KK_INTERP_TEX8, false, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// layered texture of the projections (reference: the 2D-layered CUDA array
// BackProjector samples with, projector.py:529-542 and kernel.py:91-96)
// ---------------------------------------------------------------------------

extern "C" int32_t kk_bp_launches(int64_t n_angles) {
    return n_angles < 1 ? 0 : (int32_t)((n_angles + BP_LAUNCH_ANGLES - 1) / BP_LAUNCH_ANGLES);
}

extern "C" int kk_layered_create(int64_t layers, int64_t height, int64_t width, int32_t dtype, kk_layered** out) {
    if (!out) return kk_fail(KK_ERR_INVALID_ARGUMENT, "kk_layered_create: out is NULL");
    *out = nullptr;
    if (layers <= 0 || height <= 0 || width <= 0 || layers > 2048 || height >= (int64_t)COORD_LIMIT ||
        width >= (int64_t)COORD_LIMIT)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "kk_layered_create: bad extent (%lld, %lld, %lld)",
                       (long long)layers, (long long)height, (long long)width);
    if (dtype != KK_F32 && dtype != KK_F16)
        return kk_fail(KK_ERR_UNSUPPORTED, "kk_layered_create: float32 or float16 texels only");
    cudaChannelFormatDesc ch = dtype == KK_F32 ? cudaCreateChannelDesc<float>() : cudaCreateChannelDescHalf();
    kk_layered* t = new kk_layered();
    t->surf = 0;
    t->tex = 0;
    t->layers = layers;
    t->height = height;
    t->width = width;
    t->dtype = dtype;
    cudaError_t e = cudaMalloc3DArray(&t->array, &ch, make_cudaExtent(width, height, layers),
                                      cudaArrayLayered | cudaArraySurfaceLoadStore);
    if (e != cudaSuccess) {
        delete t;
        return kk_fail(KK_ERR_CUDA, "kk_layered_create: %s", cudaGetErrorString(e));
    }
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = t->array;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    e = cudaCreateTextureObject(&t->tex, &rd, &td, nullptr);
    if (e == cudaSuccess) e = cudaCreateSurfaceObject(&t->surf, &rd);
    if (e != cudaSuccess) {
        if (t->tex) cudaDestroyTextureObject(t->tex);
        cudaFreeArray(t->array);
        delete t;
        return kk_fail(KK_ERR_CUDA, "kk_layered_create: %s", cudaGetErrorString(e));
    }
    *out = t;
    return KK_OK;
}

extern "C" int kk_layered_destroy(kk_layered* t) {
    if (!t) return KK_OK;
    if (t->surf) cudaDestroySurfaceObject(t->surf);
    cudaDestroyTextureObject(t->tex);
    cudaFreeArray(t->array);
    delete t;
    return KK_OK;
}

extern "C" int kk_layered_copy(kk_layered* t, const kk_projections* src, void* stream) {
    if (!t || !src) return kk_fail(KK_ERR_INVALID_ARGUMENT, "kk_layered_copy: NULL argument");
    if (src->table || !src->data)
        return kk_fail(KK_ERR_UNSUPPORTED, "kk_layered_copy: strided projections only");
    if (src->n_angles != t->layers || src->rows != t->height || src->cols != t->width || src->dtype != t->dtype)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "kk_layered_copy: shape or dtype differs from the texture");
    const size_t es = t->dtype == KK_F32 ? 4 : 2;
    if (src->stride[2] != 1 || src->stride[0] != src->rows * src->stride[1])
        return kk_fail(KK_ERR_UNSUPPORTED, "kk_layered_copy: rows must be contiguous and angles dense");
    cudaMemcpy3DParms cp = {};
    cp.srcPtr = make_cudaPitchedPtr(src->data, (size_t)src->stride[1] * es, (size_t)src->cols, (size_t)src->rows);
    cp.dstArray = t->array;
    cp.extent = make_cudaExtent(t->width, t->height, t->layers);
    cp.kind = cudaMemcpyDeviceToDevice;
    cudaError_t e = cudaMemcpy3DAsync(&cp, (cudaStream_t)stream);
    if (e != cudaSuccess) return kk_fail(KK_ERR_CUDA, "kk_layered_copy: %s", cudaGetErrorString(e));
    return KK_OK;
}

static int layered_args(BpArgs& L, const kk_layered* t, const kk_volume* vol, const kk_bp_angle* angles,
                        float out_scale, const char* who) {
    if (!t) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: texture is NULL", who);
    kk_projections p = {};
    p.data = (void*)1;  // texels come from the texture; the descriptor carries the extent
    p.n_angles = t->layers;
    p.rows = t->height;
    p.cols = t->width;
    p.stride[0] = t->height * t->width;
    p.stride[1] = t->width;
    p.stride[2] = 1;
    p.dtype = KK_F32;
    int rc = fill_bp_args(L, &p, vol, angles, out_scale, KK_INTERP_TEX8, who);
    if (rc) return rc;
    L.proj = nullptr;
    L.tex = t->tex;
    return KK_OK;
}

extern "C" int kk_cone_bp_layered(const kk_layered* t, const kk_volume* vol, const kk_bp_angle* angles,
                                  float out_scale, int32_t additive, float* work, void* stream) {
    BpArgs L;
    int rc = layered_args(L, t, vol, angles, out_scale, "kk_cone_bp_layered");
    if (rc) return rc;
    L.work = work;
    const dim3 block(BP_TILE_2, BP_TILE_1);
    const cudaStream_t s = (cudaStream_t)stream;
    const int vdt = vol->dtype;
    bp_chunks(L, vdt == KK_F32, additive != 0, false, [&](const BpArgs& c) {
        if (vdt == KK_F32)
            cone_bp_kernel<float, float, true, BP_STORE, FETCH_TEX><<<bp_grid(c), block, 0, s>>>(c);
        else if (vdt == KK_BF16)
            cone_bp_kernel<float, __nv_bfloat16, true, BP_STORE, FETCH_TEX><<<bp_grid(c), block, 0, s>>>(c);
        else
            cone_bp_kernel<float, __half, true, BP_STORE, FETCH_TEX><<<bp_grid(c), block, 0, s>>>(c);
    });
    return kk_check_launch("kk_cone_bp_layered");
}

extern "C" int kk_cone_bp_layered_update(const kk_layered* t, const kk_volume* vol, const kk_bp_angle* angles,
                                         float out_scale, const kk_bp_update* update, float* work, void* stream) {
    const char* who = "kk_cone_bp_layered_update";
    if (!update || !update->scale) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: update scale is NULL", who);
    if (!vol) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: volume is NULL", who);
    BpArgs L;
    int rc = layered_args(L, t, vol, angles, out_scale, who);
    if (rc) return rc;
    L.upd_scale = update->scale;
    L.upd_mask = update->mask;
    L.vmin = update->min_value;
    L.vmax = update->max_value;
    L.has_min = update->has_min;
    L.has_max = update->has_max;
    L.work = work;
    const cudaStream_t s = (cudaStream_t)stream;
    const int vdt = vol->dtype;
    bp_chunks(L, vdt == KK_F32, false, true, [&](const BpArgs& c) {
        const dim3 block(BP_TILE_2, BP_TILE_1);
        if (vdt == KK_F32)
            cone_bp_kernel<float, float, true, BP_UPDATE, FETCH_TEX><<<bp_grid(c), block, 0, s>>>(c);
        else if (vdt == KK_BF16)
            cone_bp_kernel<float, __nv_bfloat16, true, BP_UPDATE, FETCH_TEX><<<bp_grid(c), block, 0, s>>>(c);
        else
            cone_bp_kernel<float, __half, true, BP_UPDATE, FETCH_TEX><<<bp_grid(c), block, 0, s>>>(c);
    });
    return kk_check_launch(who);
}

// ---------------------------------------------------------------------------
// allocation-free backprojection
// ---------------------------------------------------------------------------
// kk_cone_bp needs a float32 running-sum buffer (`work`) whenever the volume
// is stored in 16 bits and there are more than 32 angles. Some callers can
// not provide one: they cannot call cudaMalloc at all, for instance a host
// application whose device memory is owned by a pooled allocator of its
// own, or a program that binds only this library's C entry points and not
// the CUDA runtime. kk_cone_bp_static serves them with a fixed buffer that
// lives in the library itself. The buffer is a file-scope device array of
// KK_STATIC_SCRATCH_VOXELS floats (32 MiB), so every GPU that loads the
// library holds it until the process exits; volumes with more voxels are
// rejected. Host code cannot use the array's name as a device address, so
// the address is looked up once per device with cudaGetSymbolAddress.
#define KK_STATIC_SCRATCH_VOXELS (1 << 23)
static __device__ __align__(256) float g_bp_scratch[KK_STATIC_SCRATCH_VOXELS];

#define KK_STATIC_MAX_DEVICES 64
static float* g_bp_scratch_ptr[KK_STATIC_MAX_DEVICES];
static std::mutex g_bp_scratch_mutex;

// Device address of g_bp_scratch on the current device, looked up on the
// first call per device (with that device current).
static int bp_scratch_address(float** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return kk_fail(KK_ERR_CUDA, "kk_cone_bp_static: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= KK_STATIC_MAX_DEVICES)
        return kk_fail(KK_ERR_UNSUPPORTED, "kk_cone_bp_static: device %d beyond %d", dev, KK_STATIC_MAX_DEVICES);
    std::lock_guard<std::mutex> lock(g_bp_scratch_mutex);
    if (!g_bp_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_bp_scratch);
        if (e != cudaSuccess || !p)
            return kk_fail(KK_ERR_CUDA, "kk_cone_bp_static: cudaGetSymbolAddress failed: %s",
                           cudaGetErrorString(e));
        g_bp_scratch_ptr[dev] = (float*)p;
    }
    *out = g_bp_scratch_ptr[dev];
    return KK_OK;
}

extern "C" int kk_cone_bp_static(const kk_projections* proj, const kk_volume* vol, const kk_bp_angle* angles,
                                 float out_scale, int32_t interp, int32_t additive, void* stream) {
    // only a 16-bit volume keeps its running sums in the buffer: a float32
    // volume carries them itself, so its size is not limited
    if (vol && vol->dtype != KK_F32 && vol->shape[0] > 0 && vol->shape[1] > 0 && vol->shape[2] > 0 &&
        vol->shape[0] * vol->shape[1] * vol->shape[2] > (int64_t)KK_STATIC_SCRATCH_VOXELS)
        return kk_fail(KK_ERR_INVALID_ARGUMENT,
                       "kk_cone_bp_static: %lld 16-bit voxels exceed the built-in buffer of %d voxels; "
                       "use kk_cone_bp with a caller-provided work buffer",
                       (long long)(vol->shape[0] * vol->shape[1] * vol->shape[2]), KK_STATIC_SCRATCH_VOXELS);
    float* scratch = nullptr;
    int rc = bp_scratch_address(&scratch);
    if (rc) return rc;
    // every chunk after the first reads back what the previous chunk of the
    // same call wrote, and the first chunk starts from zero or the volume,
    // so the buffer's previous contents never matter
    return kk_cone_bp(proj, vol, angles, out_scale, interp, additive, scratch, stream);
}

static int batched_args(const kk_bp_problem* pr, int32_t n, BpArgs* args, int* chunks, int* max_chunks,
                        const char* who) {
    if (!pr || n < 1 || n > KK_MAX_BATCH)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: need 1..%d problems, got %d", who, KK_MAX_BATCH, n);
    *max_chunks = 0;
    for (int i = 0; i < n; ++i) {
        const kk_bp_problem& q = pr[i];
        if (q.vol.dtype != KK_F32) return kk_fail(KK_ERR_UNSUPPORTED, "%s: problem %d: float32 volume only", who, i);
        int rc = layered_args(args[i], q.tex, &q.vol, q.angles, q.out_scale, who);
        if (rc) return rc;
        BpArgs& L = args[i];
        const bool update = q.update.scale != nullptr;
        L.upd_scale = q.update.scale;
        L.upd_mask = q.update.mask;
        L.vmin = q.update.min_value;
        L.vmax = q.update.max_value;
        L.has_min = q.update.has_min;
        L.has_max = q.update.has_max;
        L.work = q.work;
        L.tile_z = q.tile_z;
        L.tile_y = q.tile_y;
        if (q.tile_z < 0 || q.tile_y < 0 || (q.tile_z & (q.tile_z - 1)) || (q.tile_y & (q.tile_y - 1)))
            return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: problem %d: tile shape %d x %d is not a power of two", who,
                           i, q.tile_z, q.tile_y);
        chunks[i] = (L.n_angles + BP_CHUNK - 1) / BP_CHUNK;
        if (update && chunks[i] > 1 && !q.work)
            return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: problem %d: an update over %d angles needs work", who, i,
                           L.n_angles);
        *max_chunks = max(*max_chunks, chunks[i]);
    }
    return KK_OK;
}

extern "C" int64_t kk_bp_batch_sync_elems(const kk_bp_problem* pr, int32_t n) {
    if (!pr || n < 1 || n > KK_MAX_BATCH) return -1;
    int64_t total = 2;
    for (int i = 0; i < n; ++i) {
        BpArgs L;
        if (layered_args(L, pr[i].tex, &pr[i].vol, pr[i].angles, pr[i].out_scale, "kk_bp_batch_sync_elems"))
            return -1;
        const dim3 g = bp_grid(L);
        total += (int64_t)g.x * g.y * g.z;
    }
    return total;
}

extern "C" int kk_cone_bp_layered_batched_ex(const kk_bp_problem* pr, int32_t n, const kk_bp_batch_options* opts,
                                             void* stream) {
    const char* who = "kk_cone_bp_layered_batched_ex";
    if (!opts) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: options are NULL", who);
    if (!opts->persistent) return kk_cone_bp_layered_batched(pr, n, stream);
    BpArgs args[KK_MAX_BATCH];
    int chunks[KK_MAX_BATCH];
    int max_chunks = 0;
    int rc = batched_args(pr, n, args, chunks, &max_chunks, who);
    if (rc) return rc;
    if (max_chunks > BP_MAX_CHUNKS) return kk_fail(KK_ERR_UNSUPPORTED, "%s: more than %d chunks", who, BP_MAX_CHUNKS);
    static BpSched S;  // host staging, copied into the launch parameters
    static std::mutex S_mutex;
    std::lock_guard<std::mutex> lock(S_mutex);
    // items of BP_PERSIST_GROUP chunks
    for (int i = 0; i < n; ++i) chunks[i] = (chunks[i] + BP_PERSIST_GROUP - 1) / BP_PERSIST_GROUP;
    max_chunks = (max_chunks + BP_PERSIST_GROUP - 1) / BP_PERSIST_GROUP;
    S.n = n;
    S.chunks = max_chunks;
    S.skip_item = opts->test_skip_item;
    S.budget = opts->wait_budget_cycles > 0 ? opts->wait_budget_cycles : (1LL << 31);
    int64_t counters = 0;
    for (int i = 0; i < n; ++i) {
        const dim3 g = bp_grid(args[i]);
        S.grid[i][0] = (int)g.x;
        S.grid[i][1] = (int)g.y;
        S.grid[i][2] = (int)g.z;
        S.tiles[i] = (int)(g.x * g.y * g.z);
        S.nchunks[i] = chunks[i];
        S.tile_base[i] = (int)counters;
        S.p[i] = args[i];
        counters += S.tiles[i];
    }
    int64_t items = 0;
    for (int c = 0; c < max_chunks; ++c) {
        S.cstart[c] = (int)items;
        for (int i = 0; i < n; ++i)
            if (chunks[i] > c) items += S.tiles[i];
    }
    S.cstart[max_chunks] = (int)items;
    if (items >= 0x7fffffff) return kk_fail(KK_ERR_UNSUPPORTED, "%s: too many items", who);
    S.items = (int)items;
    if (!opts->sync || opts->sync_elems < 2 + counters)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: sync buffer needs %lld ints", who, (long long)(2 + counters));
    const cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(opts->sync, 0, sizeof(int32_t) * (size_t)(2 + counters), st);
    if (e != cudaSuccess) return kk_fail(KK_ERR_CUDA, "%s: %s", who, cudaGetErrorString(e));
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cone_bp_persistent_kernel, BP_TILE_2 * BP_TILE_1, 0);
    if (e != cudaSuccess || per_sm < 1) per_sm = 1;
    const int64_t grid = std::min<int64_t>(items, (int64_t)per_sm * kk_sm_count());
    if (grid > 0) {
        const dim3 block(BP_TILE_2, BP_TILE_1);
        cone_bp_persistent_kernel<<<(unsigned)grid, block, 0, st>>>(S, opts->sync);
    }
    return kk_check_launch(who);
}

int kk_bp_take_timeouts(unsigned int* n) {
    unsigned int zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(n, g_bp_timeouts, sizeof(*n));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_bp_timeouts, &zero, sizeof(zero));
    return e == cudaSuccess ? KK_OK : kk_fail(KK_ERR_CUDA, "kk_wait_timeouts: %s", cudaGetErrorString(e));
}

extern "C" int kk_cone_bp_layered_batched(const kk_bp_problem* pr, int32_t n, void* stream) {
    const char* who = "kk_cone_bp_layered_batched";
    BpArgs args[KK_MAX_BATCH];
    int chunks[KK_MAX_BATCH];
    int max_chunks = 0;
    int rc = batched_args(pr, n, args, chunks, &max_chunks, who);
    if (rc) return rc;
    const cudaStream_t st = (cudaStream_t)stream;
    for (int c = 0; c < max_chunks; ++c) {
        for (int kind = 0; kind < 2; ++kind) {  // plain, then update problems
            BpBatch B;
            B.n = 0;
            int64_t total = 0;
            for (int i = 0; i < n; ++i) {
                const bool update = pr[i].update.scale != nullptr;
                if (update != (kind == 1) || c >= chunks[i]) continue;
                BpArgs L = args[i];
                // as bp_chunks() for a float32 volume
                const bool need_work = chunks[i] > 1 && update;
                const int first_load = (pr[i].additive && !update) ? LOAD_VOL : LOAD_ZERO;
                L.j_begin = c * BP_CHUNK;
                L.j_end = min(L.n_angles, L.j_begin + BP_CHUNK);
                L.load_mode = c == 0 ? first_load : (need_work ? LOAD_WORK : LOAD_VOL);
                L.store_mode = c == chunks[i] - 1 ? STORE_FINAL : (need_work ? STORE_WORK : STORE_VOL);
                const dim3 g = bp_grid(L);
                B.p[B.n] = L;
                B.tiles[B.n][0] = (int)g.x;
                B.tiles[B.n][1] = (int)g.y;
                B.block_start[B.n] = (int)total;
                total += (int64_t)g.x * g.y * g.z;
                ++B.n;
                if (total >= 0x7fffffffLL) return kk_fail(KK_ERR_UNSUPPORTED, "%s: too many blocks for one launch", who);
            }
            if (B.n == 0) continue;
            B.block_start[B.n] = (int)total;
            const dim3 block(BP_TILE_2, BP_TILE_1);
            if (kind == 0)
                cone_bp_batched_kernel<BP_STORE><<<(unsigned)total, block, 0, st>>>(B);
            else
                cone_bp_batched_kernel<BP_UPDATE><<<(unsigned)total, block, 0, st>>>(B);
            const int rc = kk_check_launch(who);
            if (rc) return rc;
        }
    }
    return KK_OK;
}
