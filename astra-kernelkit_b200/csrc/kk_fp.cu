// Cone-beam forward projection (ray-driven) for sm_100a: kernel and the
// kk_cone_fp* entry points of include/kk.h.
#include "kk_async.cuh"
#include "kk_cone.cuh"
#include <algorithm>
#include <climits>
#include <type_traits>

namespace kk {

// ---------------------------------------------------------------------------
// forward projection
// ---------------------------------------------------------------------------
// Block = one angle, FP_COLS detector columns (one per warp) x FP_ROWS_T
// rows; lane l of warp w traces rows r0 + l + 32 k (k < FP_RPT) of column
// c0 + w, so a warp's loads for one slice cover consecutive rows, i.e.
// consecutive positions along the fastest volume axis in the usual layout.
// Blocks are ordered (row tile, angle, column tile) with the row tile
// slowest: for circular scans about z the rows of a tile see one z-slab of
// the volume, which then stays in L2 while every angle projects it.
//
// Three code paths, chosen per block: the ray's second in-slice axis D2 is
// the unit-stride axis (FAST) and, in addition, the detector's v vector has
// no component along the ray axis and D1 (SHARED): then every row of a
// column sees the same D1 coordinate sequence, bit for bit, and the D1
// split is done once per slice for the thread's rows. Otherwise a generic
// per-ray path with arbitrary strides is used.
#ifndef KK_FP_COLS
// 4 columns (128-thread blocks, twice the blocks per SM at the same
// registers): 155.5 -> 152.9 ms at the 512^3 x 720 x 768^2 scan, whose
// SMs then mix texture and CUDA-core blocks more finely; 16: 181 ms
#define KK_FP_COLS 4
#endif
#ifndef KK_FP_RPT
#define KK_FP_RPT 2
#endif
#ifndef KK_FP_MINBLOCKS
#define KK_FP_MINBLOCKS (48 / KK_FP_COLS)  // 40 registers
#endif
#ifndef KK_FP_PAD_MINBLOCKS
#define KK_FP_PAD_MINBLOCKS (40 / KK_FP_COLS)  // the padded-copy kernel: 48 registers, no spills
#endif
#ifndef KK_FP_PAD_TEX_UNROLL
#define KK_FP_PAD_TEX_UNROLL 8  // its texture loop (4 in the 40-register kernel)
#endif
#ifndef KK_FP_TEX_UNROLL
#define KK_FP_TEX_UNROLL 4  // slices per unrolled step of the texture loop
#endif
#ifndef KK_FP_UNROLL
#define KK_FP_UNROLL 4  // slices per unrolled step of the unchecked loops
#endif
constexpr int FP_RPT = KK_FP_RPT;       // rays per thread
constexpr int FP_UNROLL = KK_FP_UNROLL;
constexpr int FP_TEX_UNROLL = KK_FP_TEX_UNROLL;
constexpr int FP_PAD_TEX_UNROLL = KK_FP_PAD_TEX_UNROLL;
constexpr int FP_COLS = KK_FP_COLS;     // columns per block (one per warp)
constexpr int FP_ROWS_T = 32 * FP_RPT;  // rows per block

// Bilinear sample times weight_unit() on a plane whose D2 axis has unit
// stride, in the unified form of the texture rules: with F, S the weights
// along the fast (D2) and slow (D1) axes and y = F S / 256,
//   256 v = 256 t00 + S (t01 - t00) + x1 (t11 - t01) + x0 (t10 - t00)
// with t[fast][slow], and (x1, x0) = (h, F - h) for rule 0, (h, F - d) for
// rule 1 (h, d = y rounded half up / half down). Added into acc.
// CHECKED: border texels read zero and the coordinate is clamped;
// otherwise the caller guarantees all four texels lie inside the volume.
template <bool TEX8, bool CHECKED, int RULE, typename T>
__device__ __forceinline__ float fast_sample(float acc, const T* __restrict__ row0, const T* __restrict__ row1,
                                             bool y0ok, bool y1ok, int n2, float S, float zc) {
    const Split b = CHECKED ? split_coord<TEX8>(zc) : split_unclamped<TEX8>(zc);
    float t00, t10, t01, t11;
    if (CHECKED) {
        const bool z0ok = (unsigned)b.i < (unsigned)n2;
        const bool z1ok = (unsigned)(b.i + 1) < (unsigned)n2;
        t00 = (y0ok && z0ok) ? ld(row0 + b.i) : 0.f;      // fast 0, slow 0
        t10 = (y0ok && z1ok) ? ld(row0 + b.i + 1) : 0.f;  // fast 1, slow 0
        t01 = (y1ok && z0ok) ? ld(row1 + b.i) : 0.f;      // fast 0, slow 1
        t11 = (y1ok && z1ok) ? ld(row1 + b.i + 1) : 0.f;
    } else {
        t00 = ld(row0 + b.i);
        t10 = ld(row0 + b.i + 1);
        t01 = ld(row1 + b.i);
        t11 = ld(row1 + b.i + 1);
    }
    const float F = b.w;
    float x1, x0;
    if (TEX8) {
        const float yy = F * S * (1.f / 256.f);  // exact
        x1 = __fadd_rd(yy + 0.5f, 12582912.f) - 12582912.f;  // round half up
        if (RULE == 1) {
            const float d = -(__fadd_rd(0.5f - yy, 12582912.f) - 12582912.f);  // round half down
            x0 = F - d;
        } else {
            x0 = F - x1;
        }
    } else {
        x1 = F * S;
        x0 = F - x1;
    }
    acc = fmaf(weight_unit<TEX8>(), t00, acc);
    acc = fmaf(S, t01 - t00, acc);
    acc = fmaf(x1, t11 - t01, acc);
    acc = fmaf(x0, t10 - t00, acc);
    return acc;
}

// Whether the samples of a ray between coordinates c0 and c1 (first and
// last slice of a slab) can touch a texel of an axis of n texels: the
// complement of span_class's "every sample reads only border zeros".
__device__ __forceinline__ bool span_touches(float c0, float c1, int n) {
    return fmaxf(c0, c1) >= -0.53f && fminf(c0, c1) <= (float)n + 0.53f;
}

// Slab classification of a ray from its coordinates at the first and last
// slice of the slab (coordinates move linearly; the float32 increments
// drift by far less than the margins). 2 = both texels of every sample
// inside the array, 0 = every sample reads only border zeros, 1 = mixed.
__device__ __forceinline__ int span_class(float c0, float c1, int n) {
    const float lo = fminf(c0, c1), hi = fmaxf(c0, c1);
    // texel i = floor(x - 1/2) on the 1/256 grid: i >= 0 iff x >= 0.498,
    // i + 1 <= n - 1 iff x < n - 0.502; both out iff x < -0.502 or
    // x >= n + 0.498
    if (lo >= 0.53f && hi <= (float)n - 0.53f) return 2;
    if (hi < -0.53f || lo > (float)n + 0.53f) return 0;
    return 1;
}

template <typename TV, typename TP, bool TEX8, int EPI, int PATH, int RULE, bool AF = false, bool SUMS = false,
          bool PAD = false>
__device__ __forceinline__ void fp_trace(const FpArgs& L, const kk_fp_angle* P, int rec, int a, int A, int D1, int D2,
                                         int rule, bool a_fast, int r0, int c, int lane) {
    float src[3], cor[3], u[3], v[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        src[k] = __ldg(&P->src[k]);
        cor[k] = __ldg(&P->corner[k]);
        u[k] = __ldg(&P->u[k]);
        v[k] = __ldg(&P->v[k]);
    }
    const float sc1 = L.os[3 * A + 0], sc2 = L.os[3 * A + 1], oscale = L.os[3 * A + 2];
    const int nS = L.vn[A], n1 = L.vn[D1], n2 = L.vn[D2];
    const int64_t sS = L.vs[A], st1 = L.vs[D1], st2 = L.vs[D2];
    const TV* vol = (const TV*)L.vol;
    const float half1 = 0.5f * (float)n1, half2 = 0.5f * (float)n2;
    const float unit_inv = 1.f / weight_unit<TEX8>();

    // output element of ray k (row r0 + lane + 32 k)
    auto out_ptr = [&](int k) -> TP* {
        const int64_t off = (int64_t)(r0 + lane + 32 * k) * L.ps[1] + (int64_t)c * L.ps[2];
        return L.table ? (TP*)L.table[a] + off : (TP*)L.out + (int64_t)a * L.ps[0] + off;
    };
    // running float32 sum of ray k between launches (16-bit outputs)
    auto sum_ptr = [&](int k) -> float* {
        return L.sums + ((int64_t)rec * L.rows + (r0 + lane + 32 * k)) * L.cols + c;
    };
    RaySetup R[FP_RPT];
    float acc[FP_RPT];
#pragma unroll
    for (int k = 0; k < FP_RPT; ++k) {
        const int r = r0 + lane + 32 * k;
        const bool valid = r < L.rows;
        R[k] = ray_setup(src, cor, u, v, A, D1, D2, valid ? r : 0, c, sc1, sc2);
        acc[k] = !valid ? 0.f : (SUMS && L.load_sums) ? *sum_ptr(k) : L.additive ? ld_rw(out_ptr(k)) : 0.f;
    }

    const int s_end = min(nS, L.s_end);
    for (int off = L.s_begin; off < s_end; off += L.slab) {
        const float t1 = __fadd_rn(__fsub_rn((float)off, 0.5f * (float)nS), 0.5f);
        const int end = min(off + L.slab, nS);
        const float span = (float)(end - 1 - off);
        float yc[FP_RPT], zc[FP_RPT], val[FP_RPT];
        int cls = 2, any = 0;
#pragma unroll
        for (int k = 0; k < FP_RPT; ++k) {
            yc[k] = __fadd_rn(fmaf(R[k].a1, t1, R[k].b1), half1);
            zc[k] = __fadd_rn(fmaf(R[k].a2, t1, R[k].b2), half2);
            val[k] = 0.f;
            if (PATH == 3) {
                // the texture unit handles borders: only slabs that miss
                // the volume need a test
                any |= span_touches(yc[k], fmaf(R[k].a1, span, yc[k]), n1) &&
                       span_touches(zc[k], fmaf(R[k].a2, span, zc[k]), n2);
            } else if (PATH != 0) {
                const int cy = span_class(yc[k], fmaf(R[k].a1, span, yc[k]), n1);
                const int cz = span_class(zc[k], fmaf(R[k].a2, span, zc[k]), n2);
                const int ck = min(cy, cz);
                cls = min(cls, ck);
                any |= ck;
            }
        }
        // warp-uniform choice: skip, unchecked or checked loop
        const bool all_in = PATH != 0 && PATH != 3 && __all_sync(0xffffffffu, cls == 2);
        const bool all_out = PATH != 0 && !__any_sync(0xffffffffu, any != 0);
        if (all_out) continue;  // every sample is zero; the slab adds +0
        if (PATH == 3 && FP_RPT == 2) {
            // the texture unit filters: layer = slice, u = the faster and
            // v = the slower in-slice axis; each fetch equals the
            // reference's 3D-texture sample for these rays. Scalar
            // coordinate registers feed the fetches directly (paired FP32
            // chains here cost issue slots that the CUDA-core rays of the
            // same launch need: 169 -> 165 ms on the 512^3 x 720 scan).
            float ya = yc[0], za = zc[0], yb = yc[1], zb = zc[1], va = 0.f, vb = 0.f;
            const float a1a = R[0].a1, a2a = R[0].a2, a1b = R[1].a1, a2b = R[1].a2;
#pragma unroll(PAD ? FP_PAD_TEX_UNROLL : FP_TEX_UNROLL)
            for (int sl = off; sl < end; ++sl) {
                const float s0 = AF ? tex2DLayered<float>(L.vtex, ya, za, sl) : tex2DLayered<float>(L.vtex, za, ya, sl);
                const float s1 = AF ? tex2DLayered<float>(L.vtex, yb, zb, sl) : tex2DLayered<float>(L.vtex, zb, yb, sl);
                va = __fadd_rn(va, s0);
                vb = __fadd_rn(vb, s1);
                ya = __fadd_rn(ya, a1a);
                za = __fadd_rn(za, a2a);
                yb = __fadd_rn(yb, a1b);
                zb = __fadd_rn(zb, a2b);
            }
            val[0] = va;
            val[1] = vb;
        } else if (PATH == 3) {
            for (int sl = off; sl < end; ++sl) {
#pragma unroll
                for (int k = 0; k < FP_RPT; ++k) {
                    const float uc = AF ? yc[k] : zc[k];
                    const float vc = AF ? zc[k] : yc[k];
                    val[k] = __fadd_rn(val[k], tex2DLayered<float>(L.vtex, uc, vc, sl));
                    yc[k] = __fadd_rn(yc[k], R[k].a1);
                    zc[k] = __fadd_rn(zc[k], R[k].a2);
                }
            }
        } else if (PATH == 0) {
            for (int sl = off; sl < end; ++sl) {
                const TV* plane = vol + (int64_t)sl * sS;
#pragma unroll
                for (int k = 0; k < FP_RPT; ++k) {
                    val[k] = fmaf(weight_unit<TEX8>(),
                                  bilinear<TEX8>(plane, st1, st2, n1, n2, yc[k], zc[k], rule, a_fast), val[k]);
                    yc[k] = __fadd_rn(yc[k], R[k].a1);
                    zc[k] = __fadd_rn(zc[k], R[k].a2);
                }
            }
        } else if (TEX8 && PATH == 2 && FP_RPT == 2 && (PAD || (all_in && L.off32))) {
            // Both rays of the thread share the D1 coordinate (and so its
            // split and the two D1 rows); their D2 samples run in paired
            // instructions. Element offsets fit 32 bits (checked on the
            // host); the split's 0x4B4000 bias is folded into the row
            // offset. Same operations, order and rounding as fast_sample.
            // CLAMP (mixed slabs of a volume with two zero texels around
            // it): the coordinates that feed the split are clamped to
            // [-1.5, n + 1.5 - 1/256], which changes no coordinate whose
            // texels can be non-zero and keeps every texel index in
            // [-2, n + 1], so the loads need no test: texels outside the
            // volume read the padding's zeros, as the border does.
            auto shared_loop = [&](auto clamp_tag) {
                constexpr bool CLAMP = decltype(clamp_tag)::value;
                float2 z2 = f2(zc[0], zc[1]), v2 = f2(0.f);
                const float2 a2 = f2(R[0].a2, R[FP_RPT - 1].a2);
                float y = yc[0];
                const float a1 = R[0].a1;
                const float yhi = (float)n1 + 1.49609375f, zhi = (float)n2 + 1.49609375f;
                const TV* vol1 = vol + st1;
                const int st1i = (int)st1, sSi = (int)sS;
                int soff = off * sSi - 0x4B4000;
#pragma unroll FP_UNROLL
                for (int sl = off; sl < end; ++sl, soff += sSi) {
                    const float ys = CLAMP ? fminf(fmaxf(y, -1.5f), yhi) : y;
                    const int yb = __float_as_int(__fadd_rd(__fmaf_rd(ys, 256.f, -127.5f), 12582912.f));
                    const int rowoff = ((yb >> 8) - 0x4B4000) * st1i + soff;
                    const float S = __int_as_float((yb & 255) | 0x4B000000) - 8388608.f;
                    const float S256 = S * (1.f / 256.f);
                    const float2 zs =
                        CLAMP ? f2(fminf(fmaxf(z2.x, -1.5f), zhi), fminf(fmaxf(z2.y, -1.5f), zhi)) : z2;
                    const float2 m = add2_rd(fma2_rd(zs, f2(256.f), f2(-127.5f)), f2(12582912.f));
                    const int b0 = __float_as_int(m.x), b1 = __float_as_int(m.y);
                    const int o0 = (b0 >> 8) + rowoff, o1 = (b1 >> 8) + rowoff;
                    const float2 t00 = f2(ld(vol + o0), ld(vol + o1));
                    const float2 t10 = f2(ld(vol + o0 + 1), ld(vol + o1 + 1));
                    const float2 t01 = f2(ld(vol1 + o0), ld(vol1 + o1));
                    const float2 t11 = f2(ld(vol1 + o0 + 1), ld(vol1 + o1 + 1));
                    // Fr = 2^23 + F, F the fast weight (0..255)
                    const float2 Fr =
                        f2(__int_as_float((b0 & 255) | 0x4B000000), __int_as_float((b1 & 255) | 0x4B000000));
                    const float2 F = add2(Fr, f2(-8388608.f));
                    // x1 = floor(F S / 256 + 1/2), all steps exact
                    const float2 x1 = add2(add2_rd(fma2(F, f2(S256), f2(0.5f)), f2(12582912.f)), f2(-12582912.f));
                    float2 x0;
                    if (RULE == 1)  // F + floor(1/2 - F S / 256); Fr - 2.5 * 2^23 = F - 1.5 * 2^23
                        x0 = add2(add2_rd(fma2(F, f2(-S256), f2(0.5f)), f2(12582912.f)), add2(Fr, f2(-20971520.f)));
                    else
                        x0 = sub2(F, x1);
                    v2 = fma2(f2(256.f), t00, v2);
                    v2 = fma2(f2(S), sub2(t01, t00), v2);
                    v2 = fma2(x1, sub2(t11, t01), v2);
                    v2 = fma2(x0, sub2(t10, t00), v2);
                    z2 = add2(z2, a2);
                    y = __fadd_rn(y, a1);
                }
                val[0] = v2.x;
                val[FP_RPT - 1] = v2.y;
            };
            if (all_in)
                shared_loop(std::false_type{});
            else if constexpr (PAD)
                shared_loop(std::true_type{});
        } else if (all_in) {
#pragma unroll FP_UNROLL
            for (int sl = off; sl < end; ++sl) {
                const TV* plane = vol + (int64_t)sl * sS;
                if (PATH == 2) {
                    const Split ay = split_unclamped<TEX8>(yc[0]);
                    const TV* row0 = plane + (int64_t)ay.i * st1;
#pragma unroll
                    for (int k = 0; k < FP_RPT; ++k) {
                        val[k] = fast_sample<TEX8, false, RULE>(val[k], row0, row0 + st1, true, true, n2, ay.w, zc[k]);
                        zc[k] = __fadd_rn(zc[k], R[k].a2);
                    }
                    const float ynext = __fadd_rn(yc[0], R[0].a1);
#pragma unroll
                    for (int k = 0; k < FP_RPT; ++k) yc[k] = ynext;
                } else {
#pragma unroll
                    for (int k = 0; k < FP_RPT; ++k) {
                        const Split ay = split_unclamped<TEX8>(yc[k]);
                        const TV* row0 = plane + (int64_t)ay.i * st1;
                        val[k] = fast_sample<TEX8, false, RULE>(val[k], row0, row0 + st1, true, true, n2, ay.w, zc[k]);
                        yc[k] = __fadd_rn(yc[k], R[k].a1);
                        zc[k] = __fadd_rn(zc[k], R[k].a2);
                    }
                }
            }
        } else {
            for (int sl = off; sl < end; ++sl) {
                const TV* plane = vol + (int64_t)sl * sS;
#pragma unroll
                for (int k = 0; k < FP_RPT; ++k) {
                    const Split ay = split_coord<TEX8>(yc[k]);
                    const TV* row0 = plane + (int64_t)ay.i * st1;
                    const bool y0ok = (unsigned)ay.i < (unsigned)n1;
                    const bool y1ok = (unsigned)(ay.i + 1) < (unsigned)n1;
                    val[k] = fast_sample<TEX8, true, RULE>(val[k], row0, row0 + st1, y0ok, y1ok, n2, ay.w, zc[k]);
                    yc[k] = __fadd_rn(yc[k], R[k].a1);
                    zc[k] = __fadd_rn(zc[k], R[k].a2);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < FP_RPT; ++k) {
            // texture samples are plain values; the others carry weight_unit
            const float sum = PATH == 3 ? val[k] : __fmul_rn(val[k], unit_inv);
            acc[k] = fmaf(__fmul_rn(sum, R[k].corr), oscale, acc[k]);
        }
    }

#pragma unroll
    for (int k = 0; k < FP_RPT; ++k) {
        if (r0 + lane + 32 * k >= L.rows) continue;
        if (SUMS && L.store_sums) {
            *sum_ptr(k) = acc[k];
            continue;
        }
        float out = acc[k];
        if (EPI == FP_RESIDUAL && L.final_pass) {
            const int r = r0 + lane + 32 * k;
            const int64_t e = (int64_t)a * L.ps[0] + (int64_t)r * L.ps[1] + (int64_t)c * L.ps[2];
            out = __fmul_rn(__fsub_rn(out, ld((const TP*)L.res_y + e)), ld((const TP*)L.res_w + e));
        }
        st(out_ptr(k), out);
    }
}

// PAD: the instance for a zero-padded volume copy (FpArgs.padded, offsets
// in 32 bits), whose shared-D1 rays trace mixed slabs with the clamped
// paired loop; a separate kernel with its own register budget keeps the
// other kernels' allocation as it was.
template <typename TV, typename TP, bool TEX8, int EPI, bool SUMS = false, bool PAD = false>
__device__ __forceinline__ void fp_block(const FpArgs& L, int t) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ct = t % L.col_tiles;
    t /= L.col_tiles;
    const int rec = t % L.n_angles;
    const int rt = t / L.n_angles;
    const int c = ct * FP_COLS + warp;
    if (c >= L.cols) return;  // whole warp; the kernel has no block barrier

    const kk_fp_angle* P = L.angles + rec;
    const int a = __ldg(&P->index);  // projection written by this record
    const int A = __ldg(&P->axis);
    const int D1 = A == 1 ? 0 : 1;
    const int D2 = A == 2 ? 0 : 2;
    // texture weight rule of the reference's 3D texture: set by the memory
    // rank of the slice axis (slowest: rule 0, middle: 1, fastest: 2)
    const int rule = 2 - L.rank[A];
    const bool a_fast = L.rank[D1] < L.rank[D2];
    const bool fast = L.vs[D2] == 1 && rule < 2;
    const bool shared = fast && __ldg(&P->v[A]) == 0.f && __ldg(&P->v[D1]) == 0.f;
    const int r0 = rt * FP_ROWS_T;
    // records flagged KK_FP_NO_TEXTURE run on the CUDA cores even when the
    // layered texture is given, so both units share the work
    const bool use_tex = L.vtex && L.rank[A] == 2 && !(__ldg(&P->flags) & KK_FP_NO_TEXTURE);
    if (use_tex && a_fast)
        fp_trace<TV, TP, TEX8, EPI, 3, 0, true, SUMS, PAD>(L, P, rec, a, A, D1, D2, rule, a_fast, r0, c, lane);
    else if (use_tex)
        fp_trace<TV, TP, TEX8, EPI, 3, 0, false, SUMS, PAD>(L, P, rec, a, A, D1, D2, rule, a_fast, r0, c, lane);
    else if (shared && rule == 1)
        fp_trace<TV, TP, TEX8, EPI, 2, 1, false, SUMS, PAD>(L, P, rec, a, A, D1, D2, rule, a_fast, r0, c, lane);
    else if (shared)
        fp_trace<TV, TP, TEX8, EPI, 2, 0, false, SUMS, PAD>(L, P, rec, a, A, D1, D2, rule, a_fast, r0, c, lane);
    else if (fast && rule == 1)
        fp_trace<TV, TP, TEX8, EPI, 1, 1, false, SUMS>(L, P, rec, a, A, D1, D2, rule, a_fast, r0, c, lane);
    else if (fast)
        fp_trace<TV, TP, TEX8, EPI, 1, 0, false, SUMS>(L, P, rec, a, A, D1, D2, rule, a_fast, r0, c, lane);
    else
        fp_trace<TV, TP, TEX8, EPI, 0, 0, false, SUMS>(L, P, rec, a, A, D1, D2, rule, a_fast, r0, c, lane);
}

template <typename TV, typename TP, bool TEX8, int EPI, bool SUMS = false>
__global__ void __launch_bounds__(32 * FP_COLS, KK_FP_MINBLOCKS) cone_fp_kernel(const FpArgs L) {
    fp_block<TV, TP, TEX8, EPI, SUMS>(L, blockIdx.x);
}

// cone_fp_kernel on a zero-padded volume copy (texture-compatible weights)
template <typename TV, typename TP, int EPI>
__global__ void __launch_bounds__(32 * FP_COLS, KK_FP_PAD_MINBLOCKS) cone_fp_pad_kernel(const FpArgs L) {
    fp_block<TV, TP, true, EPI, false, true>(L, blockIdx.x);
}

// ---------------------------------------------------------------------------
// forward projection with shared-memory volume tiles
// ---------------------------------------------------------------------------
// Rays traced on the CUDA cores whose detector rows share the D1 coordinate
// (circular scans: the PATH 2 blocks above) sample a tile of each slice
// staged in shared memory by the tensor-copy unit, instead of four global
// loads per sample. A block's 8 x 64 rays touch, in every slice, a small
// window of the volume: BRICK_D1 texels along D1 (8 columns) by BRICK_D2
// along D2 (64 rows). A ninth, producer warp computes that window exactly
// and copies it with one TMA tile load per slice into a ring of
// BRICK_STAGES slots; the eight column warps wait for a slot, sample it
// with 32-bit shared-memory addressing and release it. Out-of-volume
// texels of a tile are zero-filled by the copy, which is the border rule
// of the texture path, so every sample has the value the global-memory
// code computes, with the same operations: results are bit-identical.
//
// The window: along D1 every column's coordinate sequence is replicated
// bit for bit by a producer lane (exact), along D2 the block's four corner
// rays bound the others (the D2 coordinate is monotonic in row and column
// for a planar detector), widened by a texel each side. Each warp checks
// its own rays against the window before it samples a tile (per slab for
// D2, per slice for D1); a slice it cannot prove inside (or a window that
// does not fit a slot) is sampled from global memory with the bounds-
// checked code instead, so the tile path can never read outside a slot.
constexpr int BRICK_D1 = 10;  // texels of a tile along D1 (one per column, with margins)
constexpr int BRICK_D2 = 72;  // texels along D2: 288 bytes, a multiple of 16
#ifndef KK_FP_BRICK_STAGES
#define KK_FP_BRICK_STAGES 8
#endif
constexpr int BRICK_STAGES = KK_FP_BRICK_STAGES;
constexpr int BRICK_TILE_BYTES = BRICK_D1 * BRICK_D2 * 4;
constexpr int BRICK_STAGE_FLOATS = (BRICK_TILE_BYTES + 127) / 128 * 32;  // 128-byte aligned slots
constexpr int BRICK_WARPS = FP_COLS + 1;                                   // + the producer
#ifndef KK_FP_BRICK_MINBLOCKS
#define KK_FP_BRICK_MINBLOCKS 5
#endif

enum BrickMode { BRICK_TILE = 0, BRICK_ZERO = 1, BRICK_GLOBAL = 2 };

struct BrickHdr {
    int mode;
    int d1lo, d2lo;    // tile origin (texels) along D1 and D2
    float zlo, zhi;    // the slab's D2 coordinate range of the corner rays
    int pad[3];
};

constexpr size_t BRICK_SMEM = (size_t)BRICK_STAGES * BRICK_STAGE_FLOATS * 4 + BRICK_STAGES * sizeof(BrickHdr) +
                              2 * BRICK_STAGES * sizeof(uint64_t) + 16;

struct FpBrick {
    FpArgs L;
    CUtensorMap map[2];  // slice axis = slowest memory axis [0] or middle axis [1]
    int ok[3];           // rays along world axis A may use tiles
};

// timed-out waits since the last kk_wait_timeouts() (0 unless a copy or a
// barrier failed)
static __device__ unsigned int g_fp_timeouts;

// The block's dynamic shared memory: BRICK_STAGES tile slots, their
// headers, the full / empty barrier arrays and an abort flag. Indexed
// through the array itself so that tile reads are 32-bit shared loads.
extern __shared__ __align__(128) float brick_sm[];

__device__ __forceinline__ BrickHdr* brick_hdr() {
    return reinterpret_cast<BrickHdr*>(brick_sm + BRICK_STAGES * BRICK_STAGE_FLOATS);
}
__device__ __forceinline__ uint32_t brick_full(int st) {
    return smem_addr(brick_hdr() + BRICK_STAGES) + 8 * st;
}
__device__ __forceinline__ uint32_t brick_empty(int st) {
    return smem_addr(brick_hdr() + BRICK_STAGES) + 8 * (BRICK_STAGES + st);
}
__device__ __forceinline__ volatile int* brick_abort() {
    return reinterpret_cast<volatile int*>(reinterpret_cast<uint64_t*>(brick_hdr() + BRICK_STAGES) +
                                           2 * BRICK_STAGES);
}

__device__ __forceinline__ void brick_timeout() {
    *brick_abort() = 1;
    atomicAdd(&g_fp_timeouts, 1u);
}

// Producer warp: per slice, the tile window and one tensor copy.
__device__ __forceinline__ void brick_producer(const FpBrick& B, const kk_fp_angle* P, int A, int D1, int D2, int r0,
                                               int c0, int nw) {
    const FpArgs& L = B.L;
    const int lane = threadIdx.x & 31;
    float src[3], cor[3], u[3], v[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        src[k] = __ldg(&P->src[k]);
        cor[k] = __ldg(&P->corner[k]);
        u[k] = __ldg(&P->u[k]);
        v[k] = __ldg(&P->v[k]);
    }
    // lanes 0..7: D1 of column c0 + lane (shared by its rows); lanes 8..15
    // and 16..23: D2 of the block's first and last row of column c0 + lane % 8
    const int col = lane & 7;
    const bool cvalid = col < nw;
    const int r_last = min(r0 + FP_ROWS_T - 1, L.rows - 1);
    const RaySetup R = ray_setup(src, cor, u, v, A, D1, D2, lane < 16 ? r0 : r_last, c0 + (cvalid ? col : 0),
                                 L.os[3 * A + 0], L.os[3 * A + 1]);
    const bool xl = lane < 8 && cvalid;
    const bool zl = lane >= 8 && lane < 24 && cvalid;
    const int nS = L.vn[A], n1 = L.vn[D1], n2 = L.vn[D2];
    const float half1 = 0.5f * (float)n1, half2 = 0.5f * (float)n2;
    const bool slow = L.rank[A] == 2;
    const CUtensorMap* map = &B.map[slow ? 0 : 1];
    const int s_end = min(nS, L.s_end);
    int k = 0;
    bool alive = true;
    for (int off = L.s_begin; off < s_end && alive; off += L.slab) {
        const float t1 = __fadd_rn(__fsub_rn((float)off, 0.5f * (float)nS), 0.5f);
        const int end = min(off + L.slab, nS);
        float y = __fadd_rn(fmaf(R.a1, t1, R.b1), half1);
        const float zs = __fadd_rn(fmaf(R.a2, t1, R.b2), half2);
        const float ze = fmaf(R.a2, (float)(end - 1 - off), zs);
        // NaN-propagating extremes: a NaN corner makes the window unusable
        float lo = zl ? (zs < ze ? zs : ze) : COORD_LIMIT, hi = zl ? (zs < ze ? ze : zs) : -COORD_LIMIT;
#pragma unroll
        for (int d = 16; d >= 1; d >>= 1) {
            const float ol = __shfl_xor_sync(0xffffffffu, lo, d), oh = __shfl_xor_sync(0xffffffffu, hi, d);
            lo = (ol < lo || ol != ol) ? ol : lo;
            hi = (oh > hi || oh != oh) ? oh : hi;
        }
        const bool finite = lo >= -COORD_LIMIT && hi <= COORD_LIMIT;
        int zlo_i = 0, zhi_i = 0;
        if (finite) {
            zlo_i = (int)floorf(lo - 0.5f) - 1;  // texel of the lowest sample, one more below
            zhi_i = (int)floorf(hi - 0.5f) + 2;  // its right neighbour, one more above
        }
        const int z0 = zlo_i & ~3;  // 16-byte aligned start of the copy
        const bool zfit = finite && zhi_i - z0 < BRICK_D2;
        const bool zout = finite && (zhi_i < 0 || zlo_i > n2 - 1);
        for (int sl = off; sl < end; ++sl, ++k) {
            int xi = INT_MAX, xa = INT_MIN;
            if (xl) {
                xi = split_coord<true>(y).i;
                xa = xi;
            }
            y = __fadd_rn(y, R.a1);
            const int x_lo = __reduce_min_sync(0xffffffffu, xi);
            const int x_hi = __reduce_max_sync(0xffffffffu, xa) + 1;
            const bool xout = x_hi < 0 || x_lo > n1 - 1;
            const int mode = (finite && (zout || xout)) ? BRICK_ZERO
                             : (zfit && x_hi - x_lo < BRICK_D1) ? BRICK_TILE
                                                                 : BRICK_GLOBAL;
            const int st = k % BRICK_STAGES;
            if (k >= BRICK_STAGES) {
                bool ok = true;
                if (lane == 0) ok = mbar_wait(brick_empty(st), ((k / BRICK_STAGES) - 1) & 1) && !*brick_abort();
                ok = __shfl_sync(0xffffffffu, ok, 0);
                if (!ok) {
                    if (lane == 0 && !*brick_abort()) brick_timeout();
                    alive = false;
                    break;
                }
            }
            if (lane == 0) {
                BrickHdr h;
                h.mode = mode;
                h.d1lo = x_lo;
                h.d2lo = z0;
                h.zlo = lo;
                h.zhi = hi;
                brick_hdr()[st] = h;
                if (mode == BRICK_TILE) {
                    mbar_arrive_expect_tx(brick_full(st), BRICK_TILE_BYTES);
                    tma_load_3d(smem_addr(brick_sm + st * BRICK_STAGE_FLOATS), map, z0, slow ? x_lo : sl,
                                slow ? sl : x_lo, brick_full(st));
                } else {
                    mbar_arrive(brick_full(st));
                }
            }
            __syncwarp();
        }
    }
    if (!alive && lane == 0) {
        // let the copies already issued land before the block's shared
        // memory goes away (bounded as well)
        for (int j = max(0, k - BRICK_STAGES); j < k; ++j)
            if (!mbar_wait(brick_full(j % BRICK_STAGES), (j / BRICK_STAGES) & 1)) break;
    }
}

// Bounds-checked samples of slice sl from global memory for the two rays
// of a thread (a window the warp cannot prove its rays inside): the same
// operations as the tile path, so the same values.
template <int RULE>
__device__ __noinline__ float2 brick_global_sample(const FpArgs& L, int A, int D1, int D2, int sl, float y,
                                                   float2 z2, float2 v2) {
    const Split ay = split_coord<true>(y);
    const int n1 = L.vn[D1], n2 = L.vn[D2];
    const int64_t st1 = L.vs[D1];
    const float* row0 = (const float*)L.vol + (int64_t)sl * L.vs[A] + (int64_t)ay.i * st1;
    const bool y0ok = (unsigned)ay.i < (unsigned)n1;
    const bool y1ok = (unsigned)(ay.i + 1) < (unsigned)n1;
    v2.x = fast_sample<true, true, RULE>(v2.x, row0, row0 + st1, y0ok, y1ok, n2, ay.w, z2.x);
    v2.y = fast_sample<true, true, RULE>(v2.y, row0, row0 + st1, y0ok, y1ok, n2, ay.w, z2.y);
    return v2;
}

// Column warp: the rays of column c, rows r0 + lane and r0 + lane + 32.
template <int EPI, int RULE>
__device__ __forceinline__ void brick_consumer(const FpBrick& B, const kk_fp_angle* P, int a, int A, int D1, int D2,
                                               int r0, int c, int lane) {
    static_assert(FP_RPT == 2, "two rays per thread");
    const FpArgs& L = B.L;
    float src[3], cor[3], u[3], v[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        src[k] = __ldg(&P->src[k]);
        cor[k] = __ldg(&P->corner[k]);
        u[k] = __ldg(&P->u[k]);
        v[k] = __ldg(&P->v[k]);
    }
    const float sc1 = L.os[3 * A + 0], sc2 = L.os[3 * A + 1];
    const int nS = L.vn[A];
    auto out_ptr = [&](int k) -> float* {
        const int64_t off = (int64_t)(r0 + lane + 32 * k) * L.ps[1] + (int64_t)c * L.ps[2];
        return L.table ? (float*)L.table[a] + off : (float*)L.out + (int64_t)a * L.ps[0] + off;
    };
    RaySetup R[2];
    float acc[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const bool valid = r0 + lane + 32 * k < L.rows;
        // rows past the detector trace its last row (inside the window)
        R[k] = ray_setup(src, cor, u, v, A, D1, D2, min(r0 + lane + 32 * k, L.rows - 1), c, sc1, sc2);
        // the running sum starts from the stored value, as in fp_trace
        acc[k] = (L.additive && valid) ? ld_rw(out_ptr(k)) : 0.f;
    }
    const float a1 = R[0].a1;
    const float2 a2 = f2(R[0].a2, R[1].a2);
    const int s_end = min(nS, L.s_end);
    int k = 0;
    bool alive = true;
    for (int off = L.s_begin; off < s_end; off += L.slab) {
        const float t1 = __fadd_rn(__fsub_rn((float)off, 0.5f * (float)nS), 0.5f);
        const int end = min(off + L.slab, nS);
        float y = __fadd_rn(fmaf(R[0].a1, t1, R[0].b1), 0.5f * (float)L.vn[D1]);
        const float half2 = 0.5f * (float)L.vn[D2];
        float2 z2 = f2(__fadd_rn(fmaf(R[0].a2, t1, R[0].b2), half2), __fadd_rn(fmaf(R[1].a2, t1, R[1].b2), half2));
        float2 v2 = f2(0.f);
        bool slab_ok = false;
        for (int sl = off; sl < end; ++sl, ++k) {
            const int st = k % BRICK_STAGES;
            if (!mbar_wait(brick_full(st), (k / BRICK_STAGES) & 1)) {
                if (lane == 0) brick_timeout();
                alive = false;
                break;
            }
            const BrickHdr* h = brick_hdr() + st;
            const int mode = h->mode;
            if (sl == off) {
                // every sample of this slab's rays lies within the window's
                // D2 range (false for NaN coordinates)
                const float span = (float)(end - 1 - off);
                const float ze0 = fmaf(a2.x, span, z2.x), ze1 = fmaf(a2.y, span, z2.y);
                const float lo = h->zlo - 0.5f, hi = h->zhi + 0.5f;
                const bool ok = z2.x >= lo && ze0 >= lo && z2.y >= lo && ze1 >= lo && z2.x <= hi && ze0 <= hi &&
                                z2.y <= hi && ze1 <= hi;
                slab_ok = __all_sync(0xffffffffu, ok);
            }
            const Split ay = split_coord<true>(y);  // shared by the column
            const int xi = ay.i - h->d1lo;
            const bool inside = slab_ok && (unsigned)xi <= (unsigned)(BRICK_D1 - 2) && mode != BRICK_GLOBAL;
            if (inside && mode == BRICK_TILE) {
                const float S = ay.w;
                const float S256 = S * (1.f / 256.f);
                const int rbase = st * BRICK_STAGE_FLOATS + xi * BRICK_D2 - 0x4B4000 - h->d2lo;
                const float2 mm = add2_rd(fma2_rd(z2, f2(256.f), f2(-127.5f)), f2(12582912.f));
                const int b0 = __float_as_int(mm.x), b1 = __float_as_int(mm.y);
                const int o0 = rbase + (b0 >> 8), o1 = rbase + (b1 >> 8);
                const float2 t00 = f2(brick_sm[o0], brick_sm[o1]);
                const float2 t10 = f2(brick_sm[o0 + 1], brick_sm[o1 + 1]);
                const float2 t01 = f2(brick_sm[o0 + BRICK_D2], brick_sm[o1 + BRICK_D2]);
                const float2 t11 = f2(brick_sm[o0 + BRICK_D2 + 1], brick_sm[o1 + BRICK_D2 + 1]);
                const float2 Fr = f2(__int_as_float((b0 & 255) | 0x4B000000), __int_as_float((b1 & 255) | 0x4B000000));
                const float2 F = add2(Fr, f2(-8388608.f));
                const float2 x1 = add2(add2_rd(fma2(F, f2(S256), f2(0.5f)), f2(12582912.f)), f2(-12582912.f));
                float2 x0;
                if (RULE == 1)
                    x0 = add2(add2_rd(fma2(F, f2(-S256), f2(0.5f)), f2(12582912.f)), add2(Fr, f2(-20971520.f)));
                else
                    x0 = sub2(F, x1);
                v2 = fma2(f2(256.f), t00, v2);
                v2 = fma2(f2(S), sub2(t01, t00), v2);
                v2 = fma2(x1, sub2(t11, t01), v2);
                v2 = fma2(x0, sub2(t10, t00), v2);
            } else if (!inside) {
                v2 = brick_global_sample<RULE>(L, A, D1, D2, sl, y, z2, v2);
            }  // else: every texel of the window is outside the volume
            z2 = add2(z2, a2);
            y = __fadd_rn(y, a1);
            __syncwarp();
            if (lane == 0) mbar_arrive(brick_empty(st));
        }
        if (!alive) break;
        const float oscale = L.os[3 * A + 2];
        acc[0] = fmaf(__fmul_rn(__fmul_rn(v2.x, 1.f / 256.f), R[0].corr), oscale, acc[0]);
        acc[1] = fmaf(__fmul_rn(__fmul_rn(v2.y, 1.f / 256.f), R[1].corr), oscale, acc[1]);
    }
    if (!alive) return;  // reported through kk_wait_timeouts; outputs untouched
#pragma unroll
    for (int kk2 = 0; kk2 < 2; ++kk2) {
        const int r = r0 + lane + 32 * kk2;
        if (r >= L.rows) continue;
        float out = acc[kk2];
        if (EPI == FP_RESIDUAL && L.final_pass) {
            const int64_t e = (int64_t)a * L.ps[0] + (int64_t)r * L.ps[1] + (int64_t)c * L.ps[2];
            out = __fmul_rn(__fsub_rn(out, ld((const float*)L.res_y + e)), ld((const float*)L.res_w + e));
        }
        st(out_ptr(kk2), out);
    }
}

// One launch of float32 volume and projections in which blocks whose rays
// qualify use the tiles; all other blocks run the code of cone_fp_kernel
// (the producer warp idles there).
template <int EPI>
__global__ void __launch_bounds__(32 * BRICK_WARPS, KK_FP_BRICK_MINBLOCKS)
    cone_fp_brick_kernel(const __grid_constant__ FpBrick B) {
    const FpArgs& L = B.L;
    int t = blockIdx.x;
    const int ct = t % L.col_tiles;
    t /= L.col_tiles;
    const int rec = t % L.n_angles;
    const int rt = t / L.n_angles;
    const kk_fp_angle* P = L.angles + rec;
    const int A = __ldg(&P->axis);
    const int D1 = A == 1 ? 0 : 1;
    const int D2 = A == 2 ? 0 : 2;
    const int rule = 2 - L.rank[A];
    const bool use_tex = L.vtex && L.rank[A] == 2 && !(__ldg(&P->flags) & KK_FP_NO_TEXTURE);
    const bool shared = __ldg(&P->v[A]) == 0.f && __ldg(&P->v[D1]) == 0.f;
    if (use_tex || !shared || !B.ok[A] || rule > 1) {
        if (threadIdx.x < 32 * FP_COLS) fp_block<float, float, true, EPI>(L, blockIdx.x);
        return;
    }
    // a wait of an earlier block gave up: the pipeline is broken, stop
    // quickly instead of letting every block wait out its budget
    if (*(volatile unsigned int*)&g_fp_timeouts) return;
    const int c0 = ct * FP_COLS, r0 = rt * FP_ROWS_T;
    const int nw = min(FP_COLS, L.cols - c0);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < BRICK_STAGES; ++s) {
            mbar_init(brick_full(s), 1);
            mbar_init(brick_empty(s), nw);
        }
        *brick_abort() = 0;
        mbar_fence_init();
    }
    __syncthreads();
    if (warp == FP_COLS) {
        brick_producer(B, P, A, D1, D2, r0, c0, nw);
    } else if (warp < nw) {
        const int a = __ldg(&P->index);
        if (rule == 1)
            brick_consumer<EPI, 1>(B, P, a, A, D1, D2, r0, c0 + warp, lane);
        else
            brick_consumer<EPI, 0>(B, P, a, A, D1, D2, r0, c0 + warp, lane);
    }
}

// Many problems in one launch: the argument blocks of up to KK_MAX_BATCH
// projections travel in the kernel's parameter space (no device memory),
// each block finds its problem from the prefix block counts and copies that
// problem's arguments to shared memory before tracing.
struct FpBatch {
    int n;
    int block_start[KK_MAX_BATCH + 1];
    FpArgs p[KK_MAX_BATCH];
};

template <bool TEX8, int EPI>
__global__ void __launch_bounds__(32 * FP_COLS, 32 / FP_COLS) cone_fp_batched_kernel(const __grid_constant__ FpBatch B) {
    __shared__ FpArgs Ls;
    const int b = blockIdx.x;
    int i = 0;
    while (i + 1 < B.n && B.block_start[i + 1] <= b) ++i;
    static_assert(sizeof(FpArgs) % 4 == 0 && sizeof(FpArgs) <= 4 * 32 * FP_COLS, "argument copy");
    const int* src = reinterpret_cast<const int*>(&B.p[i]);
    for (int k = threadIdx.x; k < (int)(sizeof(FpArgs) / 4); k += blockDim.x) reinterpret_cast<int*>(&Ls)[k] = src[k];
    __syncthreads();
    fp_block<float, float, TEX8, EPI>(Ls, b - B.block_start[i]);
}


}  // namespace kk

// ===========================================================================
// host side
// ===========================================================================
using namespace kk;

// A projection with float32 output is traced in several launches of a
// span of slices of every ray's own slice axis (kk_fp_set_span sets
// another span, or one launch). Each launch then reads a band of the
// volume across the rays' slice axes, whose slab per row tile stays in L2
// (at 512^3 / 720 angles / 768^2: DRAM reads down, FP 183.0 -> 168.4 ms
// with two launches; 64-slice spans lose to the per-launch ray set-up).
// The running float32 sums are carried in the projections between
// launches: same operations and rounding as one launch. The automatic
// span follows the longest axis, as measured with the padded-copy kernel:
// one launch up to 256 slices (256^3 / 360 / 384^2: 9.7 ms, 10.4 ms with
// 128 or 192), 192 up to 640 (512^3: 155.4 ms; 158.3 / 158.8 / 180.6 at
// 128 / 256 / one launch), 128 beyond (1024^3 / 1440 / 1536^2: 2744 ms;
// 2888 / 3059 / 3600 at 192 / 256 / one launch).
static int fp_auto_span(int nmax) { return nmax <= 256 ? 256 : nmax <= 640 ? 192 : 128; }
// span of the legacy entry points (kk_fp_set_span), per calling thread:
// 0 = automatic (fp_auto_span), < 0 = one launch, > 0 = slices
static thread_local int g_fp_span = 0;

static int fp_span(int nmax, int slab, int setting) {
    const int span = setting == 0 ? fp_auto_span(nmax) : setting;
    if (span < 0 || span >= nmax) return 0;
    return (span + slab - 1) / slab * slab;
}

// Tensor maps of the volume for the shared-memory tile path: float32, the
// unit-stride axis is the tiles' D2, the other strides multiples of 16
// bytes and a 16-byte aligned base. False: the path is not available
// (the kernel then traces with direct loads).
static bool brick_prepare(FpBrick& B, const FpArgs& L) {
    int ax_of_rank[3];
    for (int k = 0; k < 3; ++k) ax_of_rank[L.rank[k]] = k;
    const int r0 = ax_of_rank[0], r1 = ax_of_rank[1], r2 = ax_of_rank[2];
    if (L.vs[r0] != 1 || (L.vs[r1] * 4) % 16 != 0 || (L.vs[r2] * 4) % 16 != 0 || ((uintptr_t)L.vol & 15) != 0 ||
        L.vs[r2] * 4 >= ((int64_t)1 << 40))
        return false;
    bool any = false;
    for (int A = 0; A < 3; ++A) {
        const int D2 = A == 2 ? 0 : 2;
        B.ok[A] = A != r0 && D2 == r0;
        any = any || B.ok[A];
    }
    if (!any) return false;
    const uint64_t dims[3] = {(uint64_t)L.vn[r0], (uint64_t)L.vn[r1], (uint64_t)L.vn[r2]};
    const uint64_t strides[2] = {(uint64_t)L.vs[r1] * 4, (uint64_t)L.vs[r2] * 4};
    const uint32_t box_slow[3] = {BRICK_D2, BRICK_D1, 1};  // slices along the slowest axis
    const uint32_t box_mid[3] = {BRICK_D2, 1, BRICK_D1};   // slices along the middle axis
    if (kk_encode_tile_map(&B.map[0], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)L.vol, dims, strides, box_slow,
                           "kk_cone_fp") != KK_OK ||
        kk_encode_tile_map(&B.map[1], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)L.vol, dims, strides, box_mid,
                           "kk_cone_fp") != KK_OK)
        return false;
    return true;
}

struct FpLaunch {
    int span_setting;    // as kk_fp_options.span
    bool tiles;          // shared-memory tiles where the rays qualify
    float* sums;         // float32 running sums for 16-bit outputs, or NULL
    int64_t sums_elems;  // its size in elements
};

// 16-bit projections with a float32 running-sum buffer: the records are
// traced in chunks that fit the buffer, each chunk in span launches whose
// sums pass through the buffer (the output is written once, by the last
// launch of the chunk, with the epilogue), so the result is that of one
// launch bit for bit. The residual may then be computed in place too.
template <typename TV, typename TP, int EPI>
static bool launch_fp_sums(const FpArgs& base, bool tex8, cudaStream_t s, const FpLaunch& opt) {
    const int64_t per = (int64_t)base.rows * base.cols;
    const int nmax = max(base.vn[0], max(base.vn[1], base.vn[2]));
    const int span = fp_span(nmax, base.slab, opt.span_setting);
    if (!opt.sums || opt.sums_elems < per || !span) return false;
    const int passes = (nmax + span - 1) / span;
    const int chunk = (int)std::min<int64_t>((int64_t)base.n_angles, opt.sums_elems / per);
    FpArgs L = base;
    L.col_tiles = (L.cols + FP_COLS - 1) / FP_COLS;
    const int row_tiles = (L.rows + FP_ROWS_T - 1) / FP_ROWS_T;
    L.sums = opt.sums;
    for (int c0 = 0; c0 < base.n_angles; c0 += chunk) {
        L.angles = base.angles + c0;
        L.n_angles = min(chunk, base.n_angles - c0);
        const int64_t blocks = (int64_t)row_tiles * L.n_angles * L.col_tiles;
        for (int p = 0; p < passes; ++p) {
            L.s_begin = p * span;
            L.s_end = (p + 1) * span;
            L.load_sums = p > 0;
            L.store_sums = p < passes - 1;
            L.final_pass = p == passes - 1;
            if (tex8)
                cone_fp_kernel<TV, TP, true, EPI, true><<<(unsigned)blocks, 32 * FP_COLS, 0, s>>>(L);
            else
                cone_fp_kernel<TV, TP, false, EPI, true><<<(unsigned)blocks, 32 * FP_COLS, 0, s>>>(L);
        }
    }
    return true;
}

template <typename TV, typename TP, int EPI>
static void launch_fp_typed(const FpArgs& base, bool tex8, cudaStream_t s, const FpLaunch& opt) {
    if (!std::is_same<TP, float>::value && launch_fp_sums<TV, TP, EPI>(base, tex8, s, opt)) return;
    FpArgs L = base;
    L.col_tiles = (L.cols + FP_COLS - 1) / FP_COLS;
    const int row_tiles = (L.rows + FP_ROWS_T - 1) / FP_ROWS_T;
    const int64_t blocks = (int64_t)row_tiles * L.n_angles * L.col_tiles;  // < 2^31: checked by the caller
    const int nmax = max(L.vn[0], max(L.vn[1], L.vn[2]));
    // intermediate sums must stay float32: spans only for float32 output;
    // and a residual computed in place (out is y or the weight) needs its
    // operand intact until the last launch: one launch then
    const bool in_place = EPI == FP_RESIDUAL && (L.res_y == L.out || L.res_w == L.out);
    const int span = std::is_same<TP, float>::value && !in_place ? fp_span(nmax, L.slab, opt.span_setting) : 0;
    const int passes = span ? (nmax + span - 1) / span : 1;
    // float32 volume and projections with texture-compatible weights may
    // use the shared-memory tiles
    FpBrick Bl;
    const bool brick = std::is_same<TV, float>::value && std::is_same<TP, float>::value && tex8 && opt.tiles &&
                       brick_prepare(Bl, L);
    for (int p = 0; p < passes; ++p) {
        if (span) {
            L.s_begin = p * span;
            L.s_end = (p + 1) * span;
            L.additive = p == 0 ? base.additive : 1;
            L.final_pass = p == passes - 1;
        }
        if (brick) {
            Bl.L = L;
            cone_fp_brick_kernel<EPI><<<(unsigned)blocks, 32 * BRICK_WARPS, BRICK_SMEM, s>>>(Bl);
        } else if (tex8 && L.padded) {
            cone_fp_pad_kernel<TV, TP, EPI><<<(unsigned)blocks, 32 * FP_COLS, 0, s>>>(L);
        } else if (tex8) {
            cone_fp_kernel<TV, TP, true, EPI><<<(unsigned)blocks, 32 * FP_COLS, 0, s>>>(L);
        } else {
            cone_fp_kernel<TV, TP, false, EPI><<<(unsigned)blocks, 32 * FP_COLS, 0, s>>>(L);
        }
    }
}

template <int EPI>
static int launch_fp(const FpArgs& L, int vdt, int pdt, bool tex8, cudaStream_t s, const FpLaunch& opt) {
#define KK_FP_CASE(VD, PD, TV, TP)                                   \
    if (vdt == VD && pdt == PD) {                                    \
        launch_fp_typed<TV, TP, EPI>(L, tex8, s, opt);               \
        return kk_check_launch("kk_cone_fp");                         \
    }
    KK_FP_CASE(KK_F32, KK_F32, float, float)
    // 16-bit storage (volume in bf16 or f16, projections in f16)
    KK_FP_CASE(KK_BF16, KK_F16, __nv_bfloat16, __half)
    KK_FP_CASE(KK_F16, KK_F16, __half, __half)
    if (EPI == FP_STORE) {
        KK_FP_CASE(KK_BF16, KK_F32, __nv_bfloat16, float)
        KK_FP_CASE(KK_F16, KK_F32, __half, float)
        KK_FP_CASE(KK_BF16, KK_BF16, __nv_bfloat16, __nv_bfloat16)
        KK_FP_CASE(KK_F32, KK_F16, float, __half)
        KK_FP_CASE(KK_F32, KK_BF16, float, __nv_bfloat16)
    }
#undef KK_FP_CASE
    return kk_fail(KK_ERR_UNSUPPORTED, "kk_cone_fp: dtype combination volume=%d projections=%d", vdt, pdt);
}

// The zero-padded copy: dst holds the volume with two zero texels before
// and after every axis, in C order over the memory ranks (extents n[r] + 4,
// rank 0 fastest); src has the volume's own strides (per rank). Block =
// blockDim.y padded rows (rank 1) of one padded plane (rank 2, block y);
// threads stride along the padded rank-0 row, so both sides stream.
template <typename T>
__global__ void fp_pad_kernel(const T* __restrict__ src, T* __restrict__ dst, int n0, int n1, int n2, int64_t s0,
                              int64_t s1, int64_t s2) {
    const int m0 = n0 + 4, m1 = n1 + 4;
    const int r = blockIdx.x * blockDim.y + threadIdx.y;
    if (r >= m1) return;
    const int i1 = r - 2, i2 = (int)blockIdx.y - 2;
    T* row = dst + ((int64_t)blockIdx.y * m1 + r) * m0;
    const bool row_in = (unsigned)i1 < (unsigned)n1 && (unsigned)i2 < (unsigned)n2;
    for (int p = threadIdx.x; p < m0; p += blockDim.x) {
        const int i0 = p - 2;
        row[p] = row_in && (unsigned)i0 < (unsigned)n0 ? src[i0 * s0 + i1 * s1 + i2 * s2] : T(0);
    }
}

// Copy the volume into the caller's buffer with a zero border of two
// texels per side (kk_fp_options.padded) and trace from its interior. The
// paired loops need every offset from the interior, within
// [-interior, total - interior), in 32 bits: larger volumes keep tracing
// the volume itself.
static int fp_pad_volume(FpArgs& L, const kk_volume* vol, const kk_fp_options* opts, cudaStream_t s,
                         const char* who) {
    int64_t n[3], st[3];
    for (int k = 0; k < 3; ++k) {
        n[L.rank[k]] = vol->shape[k];
        st[L.rank[k]] = vol->stride[k];
    }
    const int64_t pst[3] = {1, n[0] + 4, (n[0] + 4) * (n[1] + 4)};
    const int64_t total = pst[2] * (n[2] + 4);
    if (opts->padded_elems < total)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: the padded copy needs %lld elements", who, (long long)total);
    if (total >= ((int64_t)1 << 31) - 0x4B4000 - 2) return KK_OK;
    const dim3 block(128, 4), grid((unsigned)((n[1] + 4 + 3) / 4), (unsigned)(n[2] + 4));
    const int es = vol->dtype == KK_F32 ? 4 : 2;
    if (es == 4)
        fp_pad_kernel<float><<<grid, block, 0, s>>>((const float*)vol->data, (float*)opts->padded, (int)n[0],
                                                   (int)n[1], (int)n[2], st[0], st[1], st[2]);
    else
        fp_pad_kernel<unsigned short><<<grid, block, 0, s>>>((const unsigned short*)vol->data,
                                                           (unsigned short*)opts->padded, (int)n[0], (int)n[1],
                                                           (int)n[2], st[0], st[1], st[2]);
    const int64_t interior = 2 * (pst[0] + pst[1] + pst[2]);
    L.vol = (const char*)opts->padded + interior * es;
    for (int k = 0; k < 3; ++k) L.vs[k] = pst[L.rank[k]];
    L.off32 = 1;
    L.padded = 1;
    return KK_OK;
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
    L.s_begin = 0;
    L.s_end = 1 << 30;
    L.final_pass = 1;
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
    L.n_angles = (int)proj->n_angles;
    L.angles = angles;
    for (int k = 0; k < 9; ++k) L.os[k] = out_scale[k];
    L.slab = slab > 0 ? slab : FP_SLAB;
    if ((int64_t)((L.rows + FP_ROWS_T - 1) / FP_ROWS_T) * L.n_angles * ((L.cols + FP_COLS - 1) / FP_COLS) >=
        0x7fffffffLL)
        return kk_fail(KK_ERR_UNSUPPORTED, "%s: too many projection tiles for one launch", who);
    int64_t last = 0;
    for (int k = 0; k < 3; ++k) last += (vol->shape[k] - 1) * vol->stride[k];
    L.off32 = last + 2 < ((int64_t)1 << 31) - 0x4B4000 && vol->stride[0] < (1 << 30) && vol->stride[1] < (1 << 30) &&
              vol->stride[2] < (1 << 30);
    for (int k = 0; k < 3; ++k) {
        L.rank[k] = 0;
        for (int j = 0; j < 3; ++j)
            if (j != k && (vol->stride[j] < vol->stride[k] || (vol->stride[j] == vol->stride[k] && j > k)))
                ++L.rank[k];
    }
    return KK_OK;
}

// The residual epilogue reads y and weight at the element it writes, so
// out may be y or weight itself (same base and layout: computed in place,
// in one launch) but must not overlap either at an offset, where a thread
// would read an element another thread has already overwritten.
static int check_residual_aliasing(const kk_projections* out, const kk_fp_residual* res, const char* who) {
    const size_t es = out->dtype == KK_F32 ? 4 : 2;
    int64_t last = 0;
    const int64_t n[3] = {out->n_angles, out->rows, out->cols};
    for (int k = 0; k < 3; ++k) last += (n[k] - 1) * out->stride[k];
    const uintptr_t lo = (uintptr_t)out->data, hi = lo + (uintptr_t)((last + 1) * (int64_t)es);
    const void* ops[2] = {res->y, res->weight};
    for (int i = 0; i < 2; ++i) {
        const uintptr_t b = (uintptr_t)ops[i], e = b + (hi - lo);  // same layout as out
        if (b == lo || e <= lo || b >= hi) continue;
        return kk_fail(KK_ERR_INVALID_ARGUMENT,
                       "%s: the output overlaps residual %s at an offset (in place is allowed only on the same "
                       "elements)", who, i == 0 ? "y" : "weight");
    }
    return KK_OK;
}

extern "C" int kk_cone_fp_ex(const kk_volume* vol, const kk_projections* proj, const kk_fp_angle* angles,
                             const float* out_scale, const kk_fp_options* opts, void* stream) {
    const char* who = "kk_cone_fp_ex";
    if (!opts) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: options are NULL", who);
    if (opts->span < -1) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: span %d", who, opts->span);
    FpArgs L;
    int rc = fill_fp_args(L, vol, proj, angles, out_scale, opts->interp, opts->slab, who);
    if (rc) return rc;
    const bool tex8 = opts->interp == KK_INTERP_TEX8;
    if (opts->vtex) {
        const kk_layered* vtex = opts->vtex;
        if (!tex8) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: a volume texture needs texture interpolation", who);
        // the texture holds the volume with one layer per slice of the
        // slowest axis, rows along the middle axis and columns along the
        // fastest
        int ax_of_rank[3];
        for (int k = 0; k < 3; ++k) ax_of_rank[L.rank[k]] = k;
        if (vtex->layers != vol->shape[ax_of_rank[2]] || vtex->height != vol->shape[ax_of_rank[1]] ||
            vtex->width != vol->shape[ax_of_rank[0]])
            return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: texture extent differs from the volume", who);
        if ((vol->dtype == KK_F32) != (vtex->dtype == KK_F32))
            return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: texture and volume storage differ", who);
        L.vtex = vtex->tex;
    }
    if (opts->padded && tex8 && !(opts->flags & KK_FP_OPT_TILES)) {
        rc = fp_pad_volume(L, vol, opts, (cudaStream_t)stream, who);
        if (rc) return rc;
    }
    L.additive = opts->additive ? 1 : 0;
    if (opts->sums_elems < 0 || (opts->sums_elems > 0 && !opts->sums))
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: bad running-sum buffer", who);
    const FpLaunch lo = {opts->span, (opts->flags & KK_FP_OPT_TILES) != 0, opts->sums, opts->sums_elems};
    if (opts->residual) {
        const kk_fp_residual* res = opts->residual;
        if (!res->y || !res->weight) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: residual operands are NULL", who);
        if (proj->table) return kk_fail(KK_ERR_UNSUPPORTED, "%s: residual epilogue needs strided data", who);
        rc = check_residual_aliasing(proj, res, who);
        if (rc) return rc;
        L.res_y = res->y;
        L.res_w = res->weight;
        return launch_fp<FP_RESIDUAL>(L, vol->dtype, proj->dtype, tex8, (cudaStream_t)stream, lo);
    }
    return launch_fp<FP_STORE>(L, vol->dtype, proj->dtype, tex8, (cudaStream_t)stream, lo);
}

extern "C" int kk_fp_set_span(int32_t slices) {
    if (slices < -1) return kk_fail(KK_ERR_INVALID_ARGUMENT, "kk_fp_set_span: %d slices", slices);
    g_fp_span = slices;
    return KK_OK;
}

extern "C" int32_t kk_fp_launches(int32_t max_slices, int32_t slab, int32_t proj_dtype) {
    if (max_slices < 1) return 1;
    const int sl = slab > 0 ? slab : FP_SLAB;
    const int span = proj_dtype == KK_F32 ? fp_span(max_slices, sl, g_fp_span) : 0;
    return span ? (max_slices + span - 1) / span : 1;
}

extern "C" int32_t kk_fp_launches_ex(int32_t max_slices, int32_t slab, int32_t proj_dtype, int32_t span) {
    // launches per chunk of records; 16-bit outputs split only with a
    // running-sum buffer
    if (max_slices < 1) return 1;
    const int sl = slab > 0 ? slab : FP_SLAB;
    const int sp = fp_span(max_slices, sl, span);
    (void)proj_dtype;
    return sp ? (max_slices + sp - 1) / sp : 1;
}

extern "C" int kk_wait_timeouts(int32_t* count) {
    if (!count) return kk_fail(KK_ERR_INVALID_ARGUMENT, "kk_wait_timeouts: count is NULL");
    unsigned int n = 0, zero = 0, nbp = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&n, g_fp_timeouts, sizeof(n));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_fp_timeouts, &zero, sizeof(zero));
    if (e != cudaSuccess) return kk_fail(KK_ERR_CUDA, "kk_wait_timeouts: %s", cudaGetErrorString(e));
    const int rc = kk_bp_take_timeouts(&nbp);
    if (rc) return rc;
    *count = (int32_t)(n + nbp);
    return KK_OK;
}

// legacy entry points: kk_cone_fp_ex with the calling thread's span
extern "C" int kk_cone_fp(const kk_volume* vol, const kk_projections* proj, const kk_fp_angle* angles,
                          const float* out_scale, int32_t interp, int32_t slab, int32_t additive, void* stream) {
    kk_fp_options o = {};
    o.interp = interp;
    o.slab = slab;
    o.additive = additive;
    o.span = g_fp_span;
    return kk_cone_fp_ex(vol, proj, angles, out_scale, &o, stream);
}

extern "C" int kk_cone_fp_residual(const kk_volume* vol, const kk_projections* out, const kk_fp_angle* angles,
                                   const float* out_scale, const kk_fp_residual* residual, int32_t interp,
                                   int32_t slab, void* stream) {
    if (!residual || !residual->y || !residual->weight)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "kk_cone_fp_residual: residual operands are NULL");
    if (out && out->table) return kk_fail(KK_ERR_UNSUPPORTED, "kk_cone_fp_residual: strided projections only");
    kk_fp_options o = {};
    o.interp = interp;
    o.slab = slab;
    o.span = g_fp_span;
    o.residual = residual;
    return kk_cone_fp_ex(vol, out, angles, out_scale, &o, stream);
}

extern "C" int kk_cone_fp_layered(const kk_layered* vtex, const kk_volume* vol, const kk_projections* proj,
                                  const kk_fp_angle* angles, const float* out_scale,
                                  const kk_fp_residual* residual, int32_t slab, int32_t additive, void* stream) {
    if (!vtex) return kk_fail(KK_ERR_INVALID_ARGUMENT, "kk_cone_fp_layered: texture is NULL");
    if (residual && (!residual->y || !residual->weight))
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "kk_cone_fp_layered: residual operands are NULL");
    kk_fp_options o = {};
    o.interp = KK_INTERP_TEX8;
    o.slab = slab;
    o.additive = residual ? 0 : additive;
    o.span = g_fp_span;
    o.vtex = vtex;
    o.residual = residual;
    return kk_cone_fp_ex(vol, proj, angles, out_scale, &o, stream);
}

extern "C" int kk_cone_fp_batched(const kk_fp_problem* pr, int32_t n, int32_t interp, int32_t slab, void* stream) {
    const char* who = "kk_cone_fp_batched";
    if (!pr || n < 1 || n > KK_MAX_BATCH)
        return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: need 1..%d problems, got %d", who, KK_MAX_BATCH, n);
    const cudaStream_t st = (cudaStream_t)stream;
    // every problem's arguments, its slice span and launch count
    FpArgs args[KK_MAX_BATCH];
    int spans[KK_MAX_BATCH], passes[KK_MAX_BATCH];
    int max_passes = 1;
    for (int i = 0; i < n; ++i) {
        const kk_fp_problem& q = pr[i];
        FpArgs& L = args[i];
        int rc = fill_fp_args(L, &q.vol, &q.proj, q.angles, q.out_scale, interp, slab, who);
        if (rc) return rc;
        if (q.vol.dtype != KK_F32 || q.proj.dtype != KK_F32)
            return kk_fail(KK_ERR_UNSUPPORTED, "%s: problem %d: float32 volume and projections only", who, i);
        if (q.span < -1) return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: problem %d: span %d", who, i, q.span);
        if (q.vtex) {
            int ax_of_rank[3];
            for (int k = 0; k < 3; ++k) ax_of_rank[L.rank[k]] = k;
            if (interp != KK_INTERP_TEX8 || q.vtex->dtype != KK_F32 || q.vtex->layers != q.vol.shape[ax_of_rank[2]] ||
                q.vtex->height != q.vol.shape[ax_of_rank[1]] || q.vtex->width != q.vol.shape[ax_of_rank[0]])
                return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: problem %d: texture does not match the volume", who, i);
            L.vtex = q.vtex->tex;
        }
        const bool res = q.residual.y || q.residual.weight;
        if (res) {
            if (!q.residual.y || !q.residual.weight || q.proj.table)
                return kk_fail(KK_ERR_INVALID_ARGUMENT, "%s: problem %d: residual needs y, weight, strided data",
                               who, i);
            L.res_y = q.residual.y;
            L.res_w = q.residual.weight;
        }
        L.additive = q.additive ? 1 : 0;
        L.col_tiles = (L.cols + FP_COLS - 1) / FP_COLS;
        // a residual computed in place needs its operand intact: one launch
        const bool in_place = res && (L.res_y == L.out || L.res_w == L.out);
        const int nmax = max(L.vn[0], max(L.vn[1], L.vn[2]));
        spans[i] = in_place ? 0 : fp_span(nmax, L.slab, q.span);
        passes[i] = spans[i] ? (nmax + spans[i] - 1) / spans[i] : 1;
        max_passes = max(max_passes, passes[i]);
    }
    // launch p traces span p of every problem that has one; plain and
    // residual problems are launched apart
    for (int p = 0; p < max_passes; ++p) {
        for (int kind = 0; kind < 2; ++kind) {
            FpBatch B;  // about 14 KB, copied into the launch's parameters
            B.n = 0;
            int64_t total = 0;
            for (int i = 0; i < n; ++i) {
                if ((args[i].res_y != nullptr) != (kind == 1) || p >= passes[i]) continue;
                FpArgs L = args[i];
                if (spans[i]) {
                    L.s_begin = p * spans[i];
                    L.s_end = (p + 1) * spans[i];
                    L.additive = p == 0 ? args[i].additive : 1;
                    L.final_pass = p == passes[i] - 1;
                }
                const int64_t blocks = (int64_t)((L.rows + FP_ROWS_T - 1) / FP_ROWS_T) * L.n_angles * L.col_tiles;
                B.p[B.n] = L;
                B.block_start[B.n] = (int)total;
                total += blocks;
                ++B.n;
                if (total >= 0x7fffffffLL)
                    return kk_fail(KK_ERR_UNSUPPORTED, "%s: too many blocks for one launch", who);
            }
            if (B.n == 0) continue;
            B.block_start[B.n] = (int)total;
            const bool tex8 = interp == KK_INTERP_TEX8;
            if (kind == 0) {
                if (tex8)
                    cone_fp_batched_kernel<true, FP_STORE><<<(unsigned)total, 32 * FP_COLS, 0, st>>>(B);
                else
                    cone_fp_batched_kernel<false, FP_STORE><<<(unsigned)total, 32 * FP_COLS, 0, st>>>(B);
            } else {
                if (tex8)
                    cone_fp_batched_kernel<true, FP_RESIDUAL><<<(unsigned)total, 32 * FP_COLS, 0, st>>>(B);
                else
                    cone_fp_batched_kernel<false, FP_RESIDUAL><<<(unsigned)total, 32 * FP_COLS, 0, st>>>(B);
            }
            const int rc = kk_check_launch(who);
            if (rc) return rc;
        }
    }
    return KK_OK;
}
