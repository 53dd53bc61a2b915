/*
 * kk.h - C ABI of the B200 cone-beam projection library (libkk.so).
 *
 * Drop-in boundary for the cone-beam hot path of ASTRA KernelKit. Every
 * entry point takes plain device pointers, sizes and strides plus a CUDA
 * stream (as void*), launches asynchronously on that stream, allocates no
 * device memory, performs no host<->device copies and never synchronises,
 * so calls may be captured in CUDA graphs. Each returns a kk_status;
 * kk_last_error() describes the most recent failure of the calling thread.
 *
 * Coordinates follow the reference: volumes are indexed by world axes
 * (x, y, z) with caller-given element strides (default layout vol[x][y][z],
 * z fastest); projections by (angle, row, col) with caller-given strides or
 * a per-index pointer table (list-of-arrays / pitched data).
 */
#ifndef KK_H
#define KK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KK_ABI_VERSION 1

#if defined(__GNUC__)
#define KK_API __attribute__((visibility("default")))
#else
#define KK_API
#endif

typedef enum {
    KK_OK = 0,
    KK_ERR_INVALID_ARGUMENT = 1,
    KK_ERR_UNSUPPORTED = 2,
    KK_ERR_CUDA = 3,
    KK_ERR_TIMEOUT = 4
} kk_status;

typedef enum { KK_F32 = 0, KK_BF16 = 1, KK_F16 = 2 } kk_dtype;

/* Interpolation weights. KK_INTERP_TEX8 reproduces the hardware texture
 * filter the reference samples with (weights on a 1/256 grid) and is the
 * reference-compatible default; KK_INTERP_EXACT uses exact float32
 * weights. */
typedef enum { KK_INTERP_TEX8 = 0, KK_INTERP_EXACT = 1 } kk_interp;

/* Per-angle forward-projection parameters (device array, one per angle),
 * in the normalised unit-voxel frame of the volume (reference:
 * kernels/cone_fp.py:302-339 geoms2params, plus the dominant ray axis of
 * kernels/cone_fp.py:264-285 _geom_axes). */
typedef struct {
    float src[3];      /* source position */
    float corner[3];   /* detector corner (outer edge of pixel (0, 0)) */
    float u[3];        /* column step: u * pixel_width */
    float v[3];        /* row step: v * pixel_height */
    int32_t axis;      /* dominant ray axis 0/1/2 (world x/y/z) */
    int32_t index;     /* projection (angle) this record writes; records
                          may come in any order, e.g. interleaved by axis
                          so every SM mixes texture and ALU work */
    int32_t flags;     /* KK_FP_* bits below, 0 by default */
    int32_t pad;
} kk_fp_angle;

/* kk_fp_angle.flags: trace this record on the CUDA cores even when
 * kk_cone_fp_layered has a texture for its rays (same result), so that a
 * caller can balance the texture unit and the arithmetic pipes. */
#define KK_FP_NO_TEXTURE 1

/* Per-angle backprojection parameters: the reference's Params struct
 * (cuda/cone_bp.cu:27-33; kernels/cone_bp.py:304-421), each float4 stored
 * as (x, y, z, w) = coefficients of world X, Y, Z and the constant. */
typedef struct {
    float num_u[4];
    float num_v[4];
    float den[4];
} kk_bp_angle;

typedef struct {
    void* data;          /* device pointer to voxel (0, 0, 0) */
    int64_t shape[3];    /* voxel counts along world x, y, z */
    int64_t stride[3];   /* element strides along world x, y, z */
    int32_t dtype;       /* kk_dtype */
} kk_volume;

typedef struct {
    void* data;              /* device pointer to pixel (0, 0, 0); unused
                                when table != NULL */
    const uint64_t* table;   /* optional device array of base addresses
                                indexed along table_axis */
    int32_t table_axis;      /* 0 angle, 1 row, 2 col */
    int64_t n_angles, rows, cols;
    int64_t stride[3];       /* element strides for angle, row, col (the
                                table axis' stride is ignored) */
    int32_t dtype;           /* kk_dtype */
} kk_projections;

/* Optional fused epilogue of the forward projection (SIRT residual step,
 * reference algo.py:339-344): out = (A x - y) * weight, elementwise in the
 * layout of `out`. y and weight have out's element type and strides. */
typedef struct {
    const void* y;
    const void* weight;
} kk_fp_residual;

/* Optional fused epilogue of the backprojection (SIRT update, reference
 * algo.py:356-362): x = clip(mask * (x - scale * A^T r)), in place on the
 * volume passed to kk_cone_bp_update. scale/mask have the volume's element
 * type and strides; mask may be NULL. */
typedef struct {
    const void* scale;
    const void* mask;
    float min_value;
    float max_value;
    int32_t has_min;
    int32_t has_max;
} kk_bp_update;

/* Opaque 2D-layered texture (see kk_layered_create below). */
typedef struct kk_layered kk_layered;

/* ---- forward projection -------------------------------------------- */

/* Ray-driven cone-beam forward projection (replaces the reference's
 * RayDrivenConeFP.__call__, kernels/cone_fp.py:102-262, and its kernel
 * cuda/cone_fp.cu:73-207). proj = A vol (additive=0) or proj += A vol.
 * out_scale: host array of 9 floats, per dominant axis (scale1, scale2,
 * outputScale) as kernels/cone_fp.py:287-300. slab: slices per coordinate
 * restart, the reference's slices_per_block (16 by default; <= 0 selects
 * 16). */
KK_API int kk_cone_fp(const kk_volume* vol, const kk_projections* proj,
                      const kk_fp_angle* angles, const float* out_scale,
                      int32_t interp, int32_t slab, int32_t additive,
                      void* stream);

/* Forward projection with the SIRT residual epilogue (kk_fp_residual).
 * out may be residual->y or residual->weight (computed in place; such a
 * call runs as one launch, see kk_fp_set_span). */
KK_API int kk_cone_fp_residual(const kk_volume* vol, const kk_projections* out,
                               const kk_fp_angle* angles,
                               const float* out_scale,
                               const kk_fp_residual* residual, int32_t interp,
                               int32_t slab, void* stream);

/* Forward projection where rays stepping along the volume's slowest
 * memory axis sample vtex, a kk_layered copy of the volume with one layer
 * per slice of that axis (filled by the caller with kk_layered_copy):
 * the texture unit then filters exactly as the reference's 3D texture
 * does for those rays. Other rays use the device-memory path on vol.
 * residual may be NULL (plain projection) or the SIRT epilogue. */
KK_API int kk_cone_fp_layered(const kk_layered* vtex, const kk_volume* vol,
                              const kk_projections* proj,
                              const kk_fp_angle* angles,
                              const float* out_scale,
                              const kk_fp_residual* residual, int32_t slab,
                              int32_t additive, void* stream);

/* Options of kk_cone_fp_ex. A zero-initialised struct selects the
 * defaults: texture-compatible weights, 16-slice slabs, overwrite,
 * automatic slice spans, direct loads, no volume texture, no epilogue. */
typedef struct {
    int32_t interp;     /* kk_interp */
    int32_t slab;       /* slices per coordinate restart; <= 0 selects 16 */
    int32_t additive;   /* 0: proj = A vol, 1: proj += A vol */
    int32_t span;       /* launch split (no counterpart in the reference,
                           whose FP is one launch): with float32 projections
                           a projection is traced in launches of `span`
                           slices of every ray's own slice axis (rounded up
                           to the slab; the running float32 sums are carried
                           in the projections, so the result is bit for bit
                           that of one launch) and each launch reads a band
                           of the volume that stays in L2. 0: by the
                           longest axis (one launch up to 256 slices, 192-
                           slice spans up to 640, 128 beyond), -1: one
                           launch */
    int32_t flags;      /* KK_FP_OPT_* bits */
    const kk_layered* vtex;          /* NULL, or a layered copy of the
                                        volume as for kk_cone_fp_layered */
    const kk_fp_residual* residual;  /* NULL, or the SIRT epilogue as for
                                        kk_cone_fp_residual */
    float* sums;          /* 16-bit projections: float32 device buffer for
                             the running sums between span launches (the
                             records are traced in chunks of sums_elems /
                             (rows * cols) angles); NULL (or too small for
                             one angle): one launch, as the sums cannot
                             pass through a 16-bit output unrounded.
                             Unused for float32 projections */
    int64_t sums_elems;   /* elements of sums */
    void* padded;         /* NULL, or a device buffer of padded_elems
                             elements of the volume's type, at least
                             (n0 + 4)(n1 + 4)(n2 + 4) (no counterpart in the
                             reference). With texture-compatible weights
                             (and without KK_FP_OPT_TILES) the volume is
                             copied into it at the start of the call with
                             two zero texels before and after every axis,
                             and the rays are traced from that copy: the
                             CUDA-core rays of circular scans then sample
                             slabs that cross the volume's boundary with
                             the paired, test-free loads of the interior
                             (the zeros are the border), not the per-ray
                             checked loop. Same results bit for bit. */
    int64_t padded_elems; /* elements of padded */
} kk_fp_options;

/* kk_fp_options.flags: rays traced on the CUDA cores sample shared-memory
 * tiles of each slice staged by the tensor-copy unit instead of loading
 * the volume directly (same results bit for bit). Off by default: at the
 * measured shapes the per-slice pipeline costs more instructions than the
 * loads it replaces. */
#define KK_FP_OPT_TILES 1

/* The forward projection with every option per call: kk_cone_fp,
 * kk_cone_fp_residual and kk_cone_fp_layered are this entry point with
 * the calling thread's kk_fp_set_span. With KK_FP_OPT_TILES, float32
 * volumes with float32 projections and texture-compatible weights trace
 * the rays that step along a non-unit-stride axis, whose detector rows
 * share their in-slice coordinate (circular orbits), from shared-memory
 * tiles of each slice staged by the tensor-copy unit (needs the volume's
 * unit-stride axis, 16-byte aligned base and strides); other rays and
 * other storage use direct loads or the texture. */
KK_API int kk_cone_fp_ex(const kk_volume* vol, const kk_projections* proj,
                         const kk_fp_angle* angles, const float* out_scale,
                         const kk_fp_options* opts, void* stream);

/* Launch split of kk_cone_fp, kk_cone_fp_residual and kk_cone_fp_layered,
 * as kk_fp_options.span, for the calling thread (each thread starts with
 * 0 = automatic, as kk_fp_options.span; -1 selects one launch). */
KK_API int kk_fp_set_span(int32_t slices);

/* Number of kernel launches kk_cone_fp* makes for a volume whose longest
 * axis has max_slices voxels, with this slab and projection dtype, at the
 * calling thread's span (kk_fp_launches) or a given span (_ex: per chunk
 * of angles, for any projection dtype given a running-sum buffer). */
KK_API int32_t kk_fp_launches(int32_t max_slices, int32_t slab,
                              int32_t proj_dtype);
KK_API int32_t kk_fp_launches_ex(int32_t max_slices, int32_t slab,
                                 int32_t proj_dtype, int32_t span);

/* Number of waits inside the library's kernels on the current device that
 * gave up since the previous call (and resets it): the shared-memory tile
 * pipeline of the forward projection and the persistent batched
 * backprojection bound every wait (on a copy, a slot or a previous chunk)
 * and a kernel whose wait runs out stops and leaves its outputs unwritten
 * instead of hanging. 0 in normal operation. Synchronous. */
KK_API int kk_wait_timeouts(int32_t* count);

/* Exact adjoint (transpose) of kk_cone_fp for the same records,
 * out_scale, interp and slab: vol = A^T proj (additive=0) or vol += A^T
 * proj, bit for bit the weights kk_cone_fp applies (same ray set-up, same
 * slab-restart coordinate sequence, same weight rule). A voxel-driven
 * gather: every voxel sums the rays whose samples touch it, no atomics.
 * work: 16-byte aligned float32 device scratch; the rays' set-up (5 floats
 * per ray) is computed per chunk of angles that fits in work_floats, which
 * must hold at least 5 * rows * cols. float32 volume and projections.
 * The reference has no adjoint of its forward projector (its autograd
 * backward is the unmatched backprojector, torch_support.py:29-33). */
KK_API int kk_cone_fp_adjoint(const kk_projections* proj, const kk_volume* vol,
                              const kk_fp_angle* angles, const float* out_scale,
                              int32_t interp, int32_t slab, int32_t additive,
                              float* work, int64_t work_floats, void* stream);

/* ---- backprojection ------------------------------------------------- */

/* Voxel-driven cone-beam backprojection (replaces VoxelDrivenConeBP.__call__,
 * kernels/cone_bp.py:192-302, kernel cuda/cone_bp.cu:35-159).
 * vol = A^T proj * out_scale (additive=0) or vol += ...; out_scale is the
 * voxel volume (kernels/cone_bp.py:294). Angles are processed in launches
 * of 32, as the reference does, so each chunk's projections stay in L2;
 * the running sum is kept in the volume when it is float32, otherwise in
 * work: an optional float32 buffer with one element per voxel (dense, in
 * the volume's memory order). With work NULL in that case one launch
 * covers all angles (same result, more memory traffic). */
KK_API int kk_cone_bp(const kk_projections* proj, const kk_volume* vol,
                      const kk_bp_angle* angles, float out_scale,
                      int32_t interp, int32_t additive, float* work,
                      void* stream);

/* kk_cone_bp for callers that cannot allocate device memory (for example
 * an application whose device memory belongs to its own pooled allocator,
 * or a program that links this library but not the CUDA runtime): the
 * float32 running sums of a 16-bit volume come from a buffer built into
 * the library, of 2^23 voxels (32 MiB, held on every GPU that loads the
 * library until the process exits). 16-bit volumes with more voxels are
 * rejected with KK_ERR_INVALID_ARGUMENT; a float32 volume holds its own
 * running sums and may have any size. Nothing is allocated. The first call
 * on a device looks up the buffer's device address and keeps it, so make
 * that call before capturing a stream, and do not call cudaDeviceReset on
 * that device while the library is in use (the kept address would go
 * stale). All calls share the buffer: calls that may run at the same time
 * on the GPU (different streams) race and must not overlap. No
 * counterpart in the reference. */
KK_API int kk_cone_bp_static(const kk_projections* proj, const kk_volume* vol,
                             const kk_bp_angle* angles, float out_scale,
                             int32_t interp, int32_t additive, void* stream);

/* Kernel launches of kk_cone_bp / kk_cone_bp_layered / kk_cone_bp_update
 * for n_angles angles when the running sum has a home (a float32 volume
 * or a work buffer): one per four 32-angle chunks, each chunk still added
 * to the running sum on its own (no counterpart in the reference, which
 * launches once per chunk). */
KK_API int32_t kk_bp_launches(int64_t n_angles);

/* Backprojection fused with the SIRT update epilogue (kk_bp_update); work
 * as for kk_cone_bp (the update needs it whenever there are more than 32
 * angles, to keep one launch per chunk group). */
KK_API int kk_cone_bp_update(const kk_projections* proj, const kk_volume* vol,
                             const kk_bp_angle* angles, float out_scale,
                             const kk_bp_update* update, int32_t interp,
                             float* work, void* stream);

/* ---- layered projection texture ---------------------------------------- */

/* A 2D-layered CUDA array of the projections (one layer per angle) with a
 * border-addressed, linearly filtered texture object: the texture the
 * reference's BackProjector samples (projector.py:529-542, kernel.py:
 * 91-96). Created once per scan (this is the only allocating entry
 * point), refilled from device projections with kk_layered_copy, and
 * sampled by kk_cone_bp_layered*, whose interpolation is then the texture
 * unit's own. float32 or float16 texels; at most 2048 layers. */
KK_API int kk_layered_create(int64_t layers, int64_t height, int64_t width,
                             int32_t dtype, kk_layered** out);
KK_API int kk_layered_copy(kk_layered* tex, const kk_projections* src,
                           void* stream);
KK_API int kk_layered_destroy(kk_layered* tex);

/* kk_cone_bp / kk_cone_bp_update sampling the layered texture. */
KK_API int kk_cone_bp_layered(const kk_layered* tex, const kk_volume* vol,
                              const kk_bp_angle* angles, float out_scale,
                              int32_t additive, float* work, void* stream);
KK_API int kk_cone_bp_layered_update(const kk_layered* tex,
                                     const kk_volume* vol,
                                     const kk_bp_angle* angles,
                                     float out_scale,
                                     const kk_bp_update* update, float* work,
                                     void* stream);

/* ---- batches of independent problems ------------------------------------ */

/* Many volumes and scans of different sizes in one launch: the argument
 * blocks of up to KK_MAX_BATCH problems travel in the kernel parameters
 * (nothing is allocated), and each thread block finds its own problem.
 * The reference runs one problem per call; it has no counterpart. */
#define KK_MAX_BATCH 64

typedef struct {
    kk_volume vol;              /* float32 */
    kk_projections proj;        /* float32 output */
    const kk_fp_angle* angles;  /* this problem's records (device) */
    float out_scale[9];         /* as kk_cone_fp */
    const kk_layered* vtex;     /* layered copy of the volume for rays along
                                   its slowest axis (as kk_cone_fp_layered),
                                   or NULL */
    kk_fp_residual residual;    /* y and weight NULL: plain projection */
    int32_t additive;
    int32_t span;               /* slices per launch, as kk_fp_options.span
                                   (0: automatic, -1: one launch) */
} kk_fp_problem;

/* kk_cone_fp / kk_cone_fp_layered / kk_cone_fp_residual for n problems
 * (1 <= n <= KK_MAX_BATCH): launch k traces slice span k of every problem
 * that has one, plain and residual problems launched apart. Results equal
 * the one-problem calls. */
KK_API int kk_cone_fp_batched(const kk_fp_problem* problems, int32_t n,
                              int32_t interp, int32_t slab, void* stream);

typedef struct {
    const kk_layered* tex;      /* the projections (kk_layered_copy) */
    kk_volume vol;              /* float32 */
    const kk_bp_angle* angles;
    float out_scale;            /* as kk_cone_bp */
    kk_bp_update update;        /* update.scale NULL: plain backprojection */
    float* work;                /* float32 running sums, one per voxel;
                                   required for an update over more than
                                   32 angles */
    int32_t additive;
    int32_t tile_z, tile_y;     /* block order: super-columns of tile_z x
                                   tile_y thread blocks of the two faster
                                   volume axes (powers of two; 0: 8 x 64),
                                   a shape the autotuner may choose */
} kk_bp_problem;

/* kk_cone_bp_layered / kk_cone_bp_layered_update for n problems: one
 * launch per 32-angle chunk index, covering that chunk of every problem
 * that has it (plain and update problems launched apart). Results equal
 * the one-problem calls. */
KK_API int kk_cone_bp_layered_batched(const kk_bp_problem* problems, int32_t n,
                                      void* stream);

typedef struct {
    int32_t persistent;         /* 0: as kk_cone_bp_layered_batched */
    int32_t* sync;              /* device ints for the persistent launch's
                                   work counter, abort flag and per-tile
                                   chunk counters: kk_bp_batch_sync_elems;
                                   zeroed by the call (on the stream) */
    int64_t sync_elems;
    int64_t wait_budget_cycles; /* bound of a wait on the previous chunk
                                   of a tile, in SM clocks (0: 2^31, about
                                   a second) */
    int32_t test_skip_item;     /* -1; for tests of the bounded wait: the
                                   item with this index is never run, so
                                   the tile's next chunk waits out the
                                   budget, the launch aborts and
                                   kk_wait_timeouts reports it */
} kk_bp_batch_options;

/* The batched backprojection as ONE persistent launch (no counterpart in
 * the reference): resident thread blocks claim (chunk group, problem,
 * tile) items, group index first, from a counter, a group being four
 * consecutive 32-angle chunks; an item of group c of a tile waits
 * (bounded) for the tile's group c - 1, then adds its chunks' angles to
 * the running sums one chunk at a time with the same block code, so
 * results equal kk_cone_bp_layered_batched bit for bit. Float32
 * volumes. */
KK_API int kk_cone_bp_layered_batched_ex(const kk_bp_problem* problems,
                                         int32_t n,
                                         const kk_bp_batch_options* opts,
                                         void* stream);
KK_API int64_t kk_bp_batch_sync_elems(const kk_bp_problem* problems,
                                      int32_t n);

/* ---- FDK pre-processing ---------------------------------------------- */

/* Cone-beam cosine pre-weighting (replaces processing.preweight,
 * processing.py:149-188): p *= |d - s| / |pixel - s| in float64, pixel at
 * the pixel corner. geom: device array of 13 doubles per angle: corner[3],
 * u*pw[3], v*ph[3], source[3], central ray length. */
KK_API int kk_preweight(const kk_projections* proj, const double* geom,
                 void* stream);

/* Row filtering (replaces processing.filter, processing.py:96-126): every
 * detector row p (length cols) becomes sum_j p[j] h[(i - j) mod P] in
 * float64, h the real impulse response (length P) of the reference's
 * frequency-domain filter. */
KK_API int kk_filter_rows(const kk_projections* proj, const double* h, int64_t P,
                   void* stream);

/* FDK pre-processing in one pass (replaces processing.preweight,
 * processing.py:149-188, followed by processing.filter, processing.py:
 * 96-126, and the copy into the backprojector's texture): every detector
 * row of src is pre-weighted as kk_preweight does (geom as there; NULL
 * skips the weighting), zero-padded to P values, filtered with the
 * frequency response the plan holds by a float64 FFT (forward, product,
 * inverse, as the reference does with cuFFT), and its first cols values
 * are stored as float32 into dst (NULL: not stored; dst may be src
 * itself) and into layers [layer0, layer0 + n_angles) of tex (NULL: not
 * stored; a float32 kk_layered of the same rows and cols). P is a power of
 * two in [64, 8192], at least 2 cols; float32 data. */
KK_API int kk_fdk_filter(const kk_projections* src, const double* geom,
                         const double* plan, int64_t P,
                         const kk_projections* dst, kk_layered* tex,
                         int64_t layer0, void* stream);

/* The plan kk_fdk_filter reads for padded length P: kk_fdk_plan_size(P)
 * doubles of device memory (caller-owned), filled on the stream from the
 * filter's frequency response H (P doubles on the device, real and even,
 * as processing.py:44-93 builds it): H in bit-reversed order, then for
 * every radix-4 stage of length len = P, P/4, ... (down to 4) the twiddles
 * exp(-2 pi i j / len), j < len / 4, as (re, im) pairs. */
KK_API int64_t kk_fdk_plan_size(int64_t P);
KK_API int kk_fdk_plan(double* plan, const double* H, int64_t P,
                       void* stream);

/* ---- elementwise helpers -------------------------------------------- */

/* x = clip(mask * (x - scale * g)) over n dense float32 elements: the
 * SIRT update (algo.py:356-362) applied after the backprojection g is
 * complete, as in an angle-sharded solve where g is summed over ranks
 * first. mask may be NULL; clipping per has_min / has_max. */
KK_API int kk_sirt_update(float* x, const float* g, const float* scale,
                          const float* mask, float min_value, float max_value,
                          int32_t has_min, int32_t has_max, int64_t n,
                          void* stream);

/* x = 1 / x with +inf mapped to 0 (SIRT scaling, algo.py:320-333). */
KK_API int kk_reciprocal(float* data, int64_t n, void* stream);

/* ---- status ------------------------------------------------------- */

KK_API const char* kk_last_error(void);
KK_API int kk_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* KK_H */
