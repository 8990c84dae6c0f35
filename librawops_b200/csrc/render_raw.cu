// Fused RAW render kernels: demosaic (bilinear v1 or menon_base v1) + the
// per-pixel stage program, one CTA per output tile, whole viewport per launch.
//
// Reference path replaced: Renderer::render_tiles -> Node::render_level chain
// -> RawUnpackNode::render (RawEngine.cpp:299-344) / detail::render_menon_base
// (MenonDemosaic.cpp:89-218), then one full-tile pass per point node.  Here the
// sensor tile plus its halo is staged once in shared memory, every stage runs
// on chip, and only the final float32 RGB leaves the SM.
//
// Both demosaics are pure functions of the pixel position (the reference's
// tiling/blocking never changes a value), so one launch over the viewport with
// the CTA grid as the tile grid gives the reference's result for any tile size.
#include "re_program.cuh"
#include "re_batch.cuh"

namespace re {

// ------------------------------------------------------------- bilinear v1

constexpr int BL_TW = 64, BL_TH = 16, BL_THREADS = 256;
constexpr int BL_SW = BL_TW + 2, BL_SH = BL_TH + 2;
// a batched bilinear tile's curve tables follow its sample tile in shared memory
constexpr size_t BL_CURVE_OFFSET = (sizeof(float) * BL_SW * BL_SH + 15) / 16 * 16;

// Colour of quad position k = 2*j + i for the four Bayer layouts (RGGB, BGGR, GRBG, GBRG).
__host__ __device__ constexpr int pat(int l, int k) {
    return l == 0   ? (k == 0 ? 0 : k == 3 ? 2 : 1)
           : l == 1 ? (k == 0 ? 2 : k == 3 ? 0 : 1)
           : l == 2 ? (k == 1 ? 0 : k == 2 ? 2 : 1)
                    : (k == 1 ? 2 : k == 2 ? 0 : 1);
}

// Interior tiles of RawEngine.cpp:299-344: every 3x3 neighbourhood is present,
// so each colour's neighbours and their row-major order are fixed by the
// quad position -- four edge neighbours (N, W, E, S) or four diagonals at R/B
// sites, a horizontal or vertical pair at G sites -- and the division by the
// count (4 or 2, a power of two) is an exact multiply.  A thread renders one
// 2x2 quad from its 4x4 neighbourhood, read as eight 8-byte shared-memory
// loads; a warp covers one quad row of the tile.
template <int L>
__device__ __forceinline__ void bilinear_fast(const float (*tile)[BL_SW], int x0, int y0, int ox, int oy, int ow,
                                              int oh, int stage_end, const DevProgram& P, float* __restrict__ out,
                                              size_t out_stride, uint32_t& err, const SmemCurve* sc, int sc_stage) {
    // The tile's row span inside the viewport and 16-byte aligned (the same
    // for the whole block): adjacent lanes pair up per row and the pair's four
    // pixels (48 bytes) leave as three aligned 16-byte stores.
    const bool wide = x0 >= ox && x0 + BL_TW <= ox + ow && ((x0 - ox) & 3) == 0 && (out_stride & 3) == 0 &&
                      (reinterpret_cast<uintptr_t>(out) & 15) == 0;
    for (int q = threadIdx.x; q < (BL_TW / 2) * (BL_TH / 2); q += BL_THREADS) {
        const int qx = q % (BL_TW / 2), qy = q / (BL_TW / 2);
        float n[4][4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float2 a = *reinterpret_cast<const float2*>(&tile[2 * qy + j][2 * qx]);
            const float2 b = *reinterpret_cast<const float2*>(&tile[2 * qy + j][2 * qx + 2]);
            n[j][0] = a.x;
            n[j][1] = a.y;
            n[j][2] = b.x;
            n[j][3] = b.y;
        }
        float R[4], G[4], B[4];
        bool keep[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int i = k & 1, j = k >> 1;
            const int x = x0 + 2 * qx + i, y = y0 + 2 * qy + j;
            const int own = pat(L, k);
            const float c = n[1 + j][1 + i];
            const float nn = n[j][1 + i], ss = n[2 + j][1 + i], ww = n[1 + j][i], ee = n[1 + j][2 + i];
            float rgb[3];
            rgb[own] = c;
            if (own == 1) {
                const int row_colour = pat(L, (j << 1) | (i ^ 1));       // colour of the W/E neighbours
                rgb[row_colour] = __fmul_rn(__fadd_rn(ww, ee), 0.5f);
                rgb[2 - row_colour] = __fmul_rn(__fadd_rn(nn, ss), 0.5f);
            } else {
                const float edge = __fadd_rn(__fadd_rn(__fadd_rn(nn, ww), ee), ss);
                const float diag =
                    __fadd_rn(__fadd_rn(__fadd_rn(n[j][i], n[j][2 + i]), n[2 + j][i]), n[2 + j][2 + i]);
                rgb[1] = __fmul_rn(edge, 0.25f);
                rgb[2 - own] = __fmul_rn(diag, 0.25f);
            }
            keep[k] = x >= ox && y >= oy && x < ox + ow && y < oy + oh;
            // pixels outside the viewport enter the stages as zeros (never written)
            R[k] = keep[k] ? rgb[0] : 0.0f;
            G[k] = keep[k] ? rgb[1] : 0.0f;
            B[k] = keep[k] ? rgb[2] : 0.0f;
        }
        apply_stages_n<4, 6>(P, 0, stage_end, R, G, B, err, sc, sc_stage);
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int y = y0 + 2 * qy + j;
            const int a = 2 * j, b = 2 * j + 1;   // the row's two pixels
            if (wide) {
                const float p0 = __shfl_down_sync(0xffffffffu, R[a], 1);
                const float p1 = __shfl_down_sync(0xffffffffu, G[a], 1);
                if (y < oy || y >= oy + oh) continue;
                float* o = out + (size_t)(y - oy) * out_stride + (size_t)(x0 - ox) * 3 + 6 * qx;
                if ((qx & 1) == 0) {
                    reinterpret_cast<float4*>(o)[0] = make_float4(R[a], G[a], B[a], R[b]);
                    reinterpret_cast<float4*>(o)[1] = make_float4(G[b], B[b], p0, p1);
                } else {
                    *reinterpret_cast<float4*>(o + 2) = make_float4(B[a], R[b], G[b], B[b]);
                }
                continue;
            }
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int k = 2 * j + i;
                if (!keep[k]) continue;
                float* o = out + (size_t)(y - oy) * out_stride + (size_t)(x0 + 2 * qx + i - ox) * 3;
                o[0] = R[k];
                o[1] = G[k];
                o[2] = B[k];
            }
        }
    }
}

// RawEngine.cpp:299-344.  The normalized samples of the tile and its one-pixel
// halo are computed once into shared memory (positions outside the active area
// are never read: the reference skips them and counts only present neighbours).
// Tiles are anchored at even sensor coordinates; interior tiles take the quad
// path, tiles meeting the active-area edge the general neighbour scan.
__device__ __forceinline__ void bilinear_cta(float (*tile)[BL_SW], const DevRaw& raw, int x0, int y0,
                                             int ox, int oy, int ow, int oh, int layout, int stage_end,
                                             const DevProgram& P, float* __restrict__ out, size_t out_stride,
                                             uint32_t& err, SmemCurve* sc) {
    // interior: the halo's even-aligned quads lie inside the active area
    const bool interior = x0 - 2 >= raw.ax && y0 - 2 >= raw.ay && x0 + BL_TW + 2 <= raw.ax + raw.aw &&
                          y0 + BL_TH + 2 <= raw.ay + raw.ah;
    if (interior) {
        load_quads<BL_SW / 2 + 1, BL_SH / 2 + 1, BL_SW, BL_SH, 1, BL_THREADS>(&tile[0][0], raw, x0 - 2, y0 - 2,
                                                                              nullptr);
    } else {
        for (int i = threadIdx.x; i < BL_SW * BL_SH; i += BL_THREADS) {
            const int sx = i % BL_SW, sy = i / BL_SW;
            const int x = x0 - 1 + sx, y = y0 - 1 + sy;
            float v = 0.0f;
            if (x >= raw.ax && x < raw.ax + raw.aw && y >= raw.ay && y < raw.ay + raw.ah)
                v = normalize_sample(raw, x, y);
            tile[sy][sx] = v;
        }
    }
    const int sc_stage = interior ? stage_curve_smem(*sc, P, 0, stage_end) : -1;
    __syncthreads();
    if (interior) {
        switch (layout) {
        case 0: bilinear_fast<0>(tile, x0, y0, ox, oy, ow, oh, stage_end, P, out, out_stride, err, sc, sc_stage); break;
        case 1: bilinear_fast<1>(tile, x0, y0, ox, oy, ow, oh, stage_end, P, out, out_stride, err, sc, sc_stage); break;
        case 2: bilinear_fast<2>(tile, x0, y0, ox, oy, ow, oh, stage_end, P, out, out_stride, err, sc, sc_stage); break;
        default: bilinear_fast<3>(tile, x0, y0, ox, oy, ow, oh, stage_end, P, out, out_stride, err, sc, sc_stage); break;
        }
        return;
    }
    for (int i = threadIdx.x; i < BL_TW * BL_TH; i += BL_THREADS) {
        const int tx = i % BL_TW, ty = i / BL_TW;
        const int x = x0 + tx, y = y0 + ty;
        if (x < ox || y < oy || x >= ox + ow || y >= oy + oh) continue;
        const int own = color_of(raw, x, y);
        float rgb[3];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            if (own == ch) {
                rgb[ch] = tile[ty + 1][tx + 1];
                continue;
            }
            float sum = 0.0f;
            int count = 0;
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy) {
                const int yy = y + dy;
                if (yy < raw.ay || yy >= raw.ay + raw.ah) continue;
#pragma unroll
                for (int dx = -1; dx <= 1; ++dx) {
                    const int xx = x + dx;
                    if (xx < raw.ax || xx >= raw.ax + raw.aw) continue;
                    if (color_of(raw, xx, yy) != ch) continue;
                    sum = __fadd_rn(sum, tile[ty + 1 + dy][tx + 1 + dx]);
                    ++count;
                }
            }
            rgb[ch] = count ? __fdiv_rn(sum, (float)count) : 0.0f;
        }
        apply_stages(P, 0, stage_end, rgb[0], rgb[1], rgb[2], err);
        float* o = out + (size_t)(y - oy) * out_stride + (size_t)(x - ox) * 3;
        o[0] = rgb[0];
        o[1] = rgb[1];
        o[2] = rgb[2];
    }
}

// Six CTAs per SM (40 registers, no spills): the tile's load, barrier and
// stores overlap across more CTAs than at four (24 MP demosaic 0.146 -> 0.116 ms).
__global__ void __launch_bounds__(BL_THREADS, 6)
bilinear_kernel(const __grid_constant__ DevRaw raw, int ox, int oy, int ow, int oh, int layout, int stage_end,
                const __grid_constant__ DevProgram P, float* __restrict__ out,
                size_t out_stride, uint32_t* status) {
    __shared__ __align__(16) float tile[BL_SH][BL_SW];
    __shared__ SmemCurve curve;
    const int x0 = (ox & ~1) + blockIdx.x * BL_TW, y0 = (oy & ~1) + blockIdx.y * BL_TH;
    uint32_t err = 0;
    bilinear_cta(tile, raw, x0, y0, ox, oy, ow, oh, layout, stage_end, P, out, out_stride, err, &curve);
    report(status, err);
}

// ------------------------------------------------------------- menon_base v1

// Output tile and the virtual extents of each on-chip plane (MenonDemosaic.cpp:96-105):
// raw r=6, directional chroma r=4, forward gradients [-4,+2]x[-4,+4] (and its
// transpose), green/direction r=2, red/blue r=1.  A plane entry at a virtual
// position outside the active area holds the plane's value at the mirrored
// position (MenonDemosaic.cpp:67-72), so every mirrored read is a plain
// shared-memory read; gradients are zero outside (MenonDemosaic.cpp:126-129).
constexpr int MN_TW = 32, MN_TH = 16, MN_THREADS = 256;
constexpr int RAW_W = MN_TW + 12, RAW_H = MN_TH + 12;   // origin (-6,-6)
constexpr int CH_W = MN_TW + 8, CH_H = MN_TH + 8;       // origin (-4,-4)
constexpr int DH_W = MN_TW + 6, DH_H = MN_TH + 8;       // origin (-4,-4), x to +2
constexpr int DV_W = MN_TW + 8, DV_H = MN_TH + 6;       // origin (-4,-4), y to +2
constexpr int GR_W = MN_TW + 4, GR_H = MN_TH + 4;       // origin (-2,-2)
constexpr int CO_W = MN_TW + 2, CO_H = MN_TH + 2;       // origin (-1,-1)

template <typename T>
struct MenonSmemT {
    T ch[CH_H][CH_W];
    T cv[CH_H][CH_W];
    T dh[DH_H][DH_W];
    T dv[DV_H][DV_W];
    T green[GR_H][GR_W];
    T red[CO_H][CO_W];
    T blue[CO_H][CO_W];
    float raw[RAW_H][RAW_W];
    uint8_t horiz[GR_H][GR_W];
    unsigned smax_bits;          // max |sample| of the loaded footprint (float bits)
};
using MenonSmem = MenonSmemT<double>;

struct MenonCtx {
    int x0, y0;                  // tile origin (sensor coordinates)
    int xe, ye;                  // end of this tile's output pixels (exclusive)
    int ax, ay, aw, ah;
    // A plane of radius r is needed only at virtual positions within r of the
    // tile's output pixels; positions of a partial tile further out are skipped,
    // which keeps every mirrored read inside its shared-memory plane.
    __device__ __forceinline__ bool needed(int x, int y, int rx, int ry) const {
        return x < xe + rx && y < ye + ry;
    }
    __device__ __forceinline__ int mx(int x) const { return mirror_coord(x, ax, aw); }
    __device__ __forceinline__ int my(int y) const { return mirror_coord(y, ay, ah); }
    __device__ __forceinline__ bool inside(int x, int y) const {
        return x >= ax && x < ax + aw && y >= ay && y < ay + ah;
    }
};

// Correctly rounded binary64 / binary32 operations (no contraction).
__device__ __forceinline__ double r_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double r_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double r_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float r_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float r_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float r_mul(float a, float b) { return __fmul_rn(a, b); }

__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
template <typename T>
__device__ __forceinline__ T half_sum(T a, T b) { return r_mul(T(0.5), r_add(a, b)); }

// Whether a binary32 decision lies inside the error band.
__device__ __forceinline__ bool near_tie(float h, float v, float band_abs) {
    const float band = __fmaf_rn(9.0f * 5.9604644775390625e-8f, __fadd_rn(h, v), band_abs);
    return fabsf(__fsub_rn(v, h)) <= band;
}
__device__ __forceinline__ bool near_tie(double, double, float) { return false; }

// MenonDemosaic.cpp:112-115 directional five-tap green estimate along one axis.
template <typename T>
__device__ __forceinline__ T five_tap(T m2, T m1, T own, T p1, T p2) {
    return r_sub(r_add(r_mul(T(0.5), r_add(m1, p1)), r_mul(T(0.5), own)), r_mul(T(0.25), r_add(m2, p2)));
}

template <typename R, typename Sm>
__device__ __forceinline__ R raw_at(const Sm& S, const MenonCtx& c, int x, int y) {
    return (R)S.raw[y - (c.y0 - 6)][x - (c.x0 - 6)];
}

template <typename R, typename Sm>
__device__ __forceinline__ R green_h(const Sm& S, const MenonCtx& c, int x, int y) {
    return five_tap(raw_at<R>(S, c, x - 2, y), raw_at<R>(S, c, x - 1, y), raw_at<R>(S, c, x, y),
                    raw_at<R>(S, c, x + 1, y), raw_at<R>(S, c, x + 2, y));
}
template <typename R, typename Sm>
__device__ __forceinline__ R green_v(const Sm& S, const MenonCtx& c, int x, int y) {
    return five_tap(raw_at<R>(S, c, x, y - 2), raw_at<R>(S, c, x, y - 1), raw_at<R>(S, c, x, y),
                    raw_at<R>(S, c, x, y + 1), raw_at<R>(S, c, x, y + 2));
}

// MenonDemosaic.cpp:148-150 pair mean of a mirrored plane.
template <int W, int OX, int OY, typename T>
__device__ __forceinline__ T pair_mean(const T (*p)[W], const MenonCtx& c, int x, int y, int dx, int dy) {
    return r_mul(T(0.5), r_add(p[y - dy - (c.y0 + OY)][x - dx - (c.x0 + OX)],
                               p[y + dy - (c.y0 + OY)][x + dx - (c.x0 + OX)]));
}

// The reference's classifier in binary64 at the site (x, y) of the general
// path: chroma at virtual positions is the chroma of the mirrored position
// (zero at green sites), gradients are zero at virtual positions outside the
// active area (MenonDemosaic.cpp:107-147).
__device__ __forceinline__ bool generic_exact_horizontal(const MenonSmemT<float>& S, const DevRaw& raw,
                                                         const MenonCtx& c, int x, int y) {
    auto chroma = [&](int xv, int yv, bool horizontal_axis) {
        const int mxp = c.mx(xv), myp = c.my(yv);
        if (color_of(raw, mxp, myp) == 1) return 0.0;
        const double g = horizontal_axis ? green_h<double>(S, c, mxp, myp) : green_v<double>(S, c, mxp, myp);
        return dsub(raw_at<double>(S, c, mxp, myp), g);
    };
    auto dh = [&](int xv, int yv) {
        return c.inside(xv, yv) ? fabs(dsub(chroma(xv, yv, true), chroma(xv + 2, yv, true))) : 0.0;
    };
    auto dv = [&](int xv, int yv) {
        return c.inside(xv, yv) ? fabs(dsub(chroma(xv, yv, false), chroma(xv, yv + 2, false))) : 0.0;
    };
    double h = 0.0, v = 0.0;
    h = dadd(h, dh(x, y + 2));                     v = dadd(v, dv(x + 2, y));
    h = dadd(h, dh(x - 2, y + 2));                 v = dadd(v, dv(x + 2, y - 2));
    h = dadd(h, dh(x - 1, y + 1));                 v = dadd(v, dv(x + 1, y - 1));
    h = dadd(h, __dmul_rn(3.0, dh(x, y)));         v = dadd(v, __dmul_rn(3.0, dv(x, y)));
    h = dadd(h, __dmul_rn(3.0, dh(x - 2, y)));     v = dadd(v, __dmul_rn(3.0, dv(x, y - 2)));
    h = dadd(h, dh(x - 1, y - 1));                 v = dadd(v, dv(x - 1, y - 1));
    h = dadd(h, dh(x, y - 2));                     v = dadd(v, dv(x - 2, y));
    h = dadd(h, dh(x - 2, y - 2));                 v = dadd(v, dv(x - 2, y - 2));
    return v >= h;
}

// The general (mirrored) path.  T = double: the reference's binary64
// arithmetic; T = float: the same operations in binary32 with exact decisions
// (the band test and binary64 recheck of the fast path), so that an interior
// pixel gets the same float whichever path its tile takes.
template <typename T>
__device__ __forceinline__ void menon_tile(MenonSmemT<T>& S, const DevRaw& raw, const MenonCtx& c,
                                           unsigned long long* ties) {
    constexpr bool F32 = sizeof(T) == 4;
    const int t = threadIdx.x;
    if (t == 0) S.smax_bits = 0;
    // 1. normalized raw over r=6 at mirrored positions (MenonDemosaic.cpp:106).
    float local_max = 0.0f;
    for (int i = t; i < RAW_W * RAW_H; i += MN_THREADS) {
        const int sx = i % RAW_W, sy = i / RAW_W;
        if (!c.needed(c.x0 - 6 + sx, c.y0 - 6 + sy, 6, 6)) continue;
        const float v = normalize_sample(raw, c.mx(c.x0 - 6 + sx), c.my(c.y0 - 6 + sy));
        local_max = fmaxf(local_max, fabsf(v));
        S.raw[sy][sx] = v;
    }
    if constexpr (F32) {
        for (int o = 16; o; o >>= 1) local_max = fmaxf(local_max, __shfl_xor_sync(0xffffffffu, local_max, o));
        __syncthreads();
        if ((t & 31) == 0) atomicMax(&S.smax_bits, __float_as_uint(local_max));
    }
    __syncthreads();
    // 2. directional chroma (MenonDemosaic.cpp:107-119), evaluated at the
    //    mirrored position; green sites keep zero chroma.
    for (int i = t; i < CH_W * CH_H; i += MN_THREADS) {
        const int sx = i % CH_W, sy = i / CH_W;
        if (!c.needed(c.x0 - 4 + sx, c.y0 - 4 + sy, 4, 4)) continue;
        const int x = c.mx(c.x0 - 4 + sx), y = c.my(c.y0 - 4 + sy);
        T h = 0, v = 0;
        if (color_of(raw, x, y) != 1) {
            const T own = raw_at<T>(S, c, x, y);
            h = r_sub(own, green_h<T>(S, c, x, y));
            v = r_sub(own, green_v<T>(S, c, x, y));
        }
        S.ch[sy][sx] = h;
        S.cv[sy][sx] = v;
    }
    __syncthreads();
    // 3. forward chroma gradients, zero outside the active area (MenonDemosaic.cpp:120-129).
    for (int i = t; i < DH_W * DH_H; i += MN_THREADS) {
        const int sx = i % DH_W, sy = i / DH_W;
        const int x = c.x0 - 4 + sx, y = c.y0 - 4 + sy;
        if (!c.needed(x, y, 2, 4)) continue;
        T d = 0;
        if (c.inside(x, y)) d = fabs(r_sub(S.ch[sy][sx], S.ch[sy][sx + 2]));
        S.dh[sy][sx] = d;
    }
    for (int i = t; i < DV_W * DV_H; i += MN_THREADS) {
        const int sx = i % DV_W, sy = i / DV_W;
        const int x = c.x0 - 4 + sx, y = c.y0 - 4 + sy;
        if (!c.needed(x, y, 4, 2)) continue;
        T d = 0;
        if (c.inside(x, y)) d = fabs(r_sub(S.cv[sy][sx], S.cv[sy + 2][sx]));
        S.dv[sy][sx] = d;
    }
    __syncthreads();
    // 4. classifier and green (MenonDemosaic.cpp:130-147): terms in the
    //    reference's order, horizontal wins ties (v >= h).
    const float band_abs = F32 ? 640.0f * 5.9604644775390625e-8f * __uint_as_float(S.smax_bits) : 0.0f;
    unsigned long long local_ties = 0;
    for (int i = t; i < GR_W * GR_H; i += MN_THREADS) {
        const int sx = i % GR_W, sy = i / GR_W;
        if (!c.needed(c.x0 - 2 + sx, c.y0 - 2 + sy, 2, 2)) continue;
        const int x = c.mx(c.x0 - 2 + sx), y = c.my(c.y0 - 2 + sy);
        if (color_of(raw, x, y) == 1) {
            S.horiz[sy][sx] = 1;
            S.green[sy][sx] = raw_at<T>(S, c, x, y);
            continue;
        }
        // dh index of (x+a, y+b): [y+b-(y0-4)][x+a-(x0-4)]
        const int hx = x - (c.x0 - 4), hy = y - (c.y0 - 4);
        const T (*dh)[DH_W] = S.dh;
        const T (*dv)[DV_W] = S.dv;
        const T three = T(3);
        T h = 0, v = 0;
        h = r_add(h, dh[hy + 2][hx + 0]);
        v = r_add(v, dv[hy + 0][hx + 2]);
        h = r_add(h, dh[hy + 2][hx - 2]);
        v = r_add(v, dv[hy - 2][hx + 2]);
        h = r_add(h, dh[hy + 1][hx - 1]);
        v = r_add(v, dv[hy - 1][hx + 1]);
        h = r_add(h, r_mul(three, dh[hy + 0][hx + 0]));
        v = r_add(v, r_mul(three, dv[hy + 0][hx + 0]));
        h = r_add(h, r_mul(three, dh[hy + 0][hx - 2]));
        v = r_add(v, r_mul(three, dv[hy - 2][hx + 0]));
        h = r_add(h, dh[hy - 1][hx - 1]);
        v = r_add(v, dv[hy - 1][hx - 1]);
        h = r_add(h, dh[hy - 2][hx + 0]);
        v = r_add(v, dv[hy + 0][hx - 2]);
        h = r_add(h, dh[hy - 2][hx - 2]);
        v = r_add(v, dv[hy - 2][hx - 2]);
        bool horizontal = v >= h;
        if constexpr (F32) {
            if (near_tie(h, v, band_abs)) {
                horizontal = generic_exact_horizontal(S, raw, c, x, y);
                if (ties && sx >= 2 && sx < GR_W - 2 && sy >= 2 && sy < GR_H - 2) ++local_ties;
            }
        } else {
            if (ties && v == h && sx >= 2 && sx < GR_W - 2 && sy >= 2 && sy < GR_H - 2) ++local_ties;
        }
        S.horiz[sy][sx] = horizontal;
        S.green[sy][sx] = horizontal ? green_h<T>(S, c, x, y) : green_v<T>(S, c, x, y);
    }
    if (ties && local_ties) atomicAdd(ties, local_ties);
    __syncthreads();
    // 5. red and blue at every colour-support site (MenonDemosaic.cpp:151-161).
    for (int i = t; i < CO_W * CO_H; i += MN_THREADS) {
        const int sx = i % CO_W, sy = i / CO_W;
        if (!c.needed(c.x0 - 1 + sx, c.y0 - 1 + sy, 1, 1)) continue;
        const int x = c.mx(c.x0 - 1 + sx), y = c.my(c.y0 - 1 + sy);
        const int own = color_of(raw, x, y);
        T rr = 0, bb = 0;
        if (own == 0) rr = raw_at<T>(S, c, x, y);
        if (own == 2) bb = raw_at<T>(S, c, x, y);
        if (own == 1) {
            const bool red_h = color_of(raw, x + 1, y) == 0;
            const int dx = red_h ? 1 : 0, dy = red_h ? 0 : 1;
            const T g = S.green[y - (c.y0 - 2)][x - (c.x0 - 2)];
            const T rm = r_mul(T(0.5), r_add(raw_at<T>(S, c, x - dx, y - dy), raw_at<T>(S, c, x + dx, y + dy)));
            const T bm = r_mul(T(0.5), r_add(raw_at<T>(S, c, x - dy, y - dx), raw_at<T>(S, c, x + dy, y + dx)));
            const T gr = pair_mean<GR_W, -2, -2>(S.green, c, x, y, dx, dy);
            const T gb = pair_mean<GR_W, -2, -2>(S.green, c, x, y, dy, dx);
            rr = r_sub(r_add(g, rm), gr);
            bb = r_sub(r_add(g, bm), gb);
        }
        S.red[sy][sx] = rr;
        S.blue[sy][sx] = bb;
    }
    __syncthreads();
}

// Final opposite colour at R/B sites, float cast, stage program
// (MenonDemosaic.cpp:162-173) for the general path.
template <typename T>
__device__ __forceinline__ void menon_tile_out(MenonSmemT<T>& S, const DevRaw& raw, const MenonCtx& c, int ox, int oy,
                                               int ow, int oh, int stage_end, const DevProgram& P,
                                               float* __restrict__ out, size_t out_stride, uint32_t& err,
                                               uint8_t* dirs) {
    for (int i = threadIdx.x; i < MN_TW * MN_TH; i += MN_THREADS) {
        const int tx = i % MN_TW, ty = i / MN_TW;
        const int x = c.x0 + tx, y = c.y0 + ty;
        if (x < ox || y < oy || x >= ox + ow || y >= oy + oh) continue;
        const int own = color_of(raw, x, y);
        const bool horizontal = S.horiz[ty + 2][tx + 2];
        const int dx = horizontal ? 1 : 0, dy = horizontal ? 0 : 1;
        T rr = S.red[ty + 1][tx + 1], bb = S.blue[ty + 1][tx + 1];
        if (own == 2)
            rr = r_sub(r_add(bb, pair_mean<CO_W, -1, -1>(S.red, c, x, y, dx, dy)),
                       pair_mean<CO_W, -1, -1>(S.blue, c, x, y, dx, dy));
        if (own == 0)
            bb = r_sub(r_add(rr, pair_mean<CO_W, -1, -1>(S.blue, c, x, y, dx, dy)),
                       pair_mean<CO_W, -1, -1>(S.red, c, x, y, dx, dy));
        float r = (float)rr, g = (float)S.green[ty + 2][tx + 2], b = (float)bb;
        apply_stages(P, 0, stage_end, r, g, b, err);
        float* o = out + (size_t)(y - oy) * out_stride + (size_t)(x - ox) * 3;
        o[0] = r;
        o[1] = g;
        o[2] = b;
        if (dirs) dirs[(size_t)(y - oy) * ow + (x - ox)] = horizontal;
    }
}

// ------------------------------------------------- menon fast interior path
//
// Tiles whose r=6 raw footprint lies inside the active area need no mirroring
// and no zero extension, and with an even tile origin the CFA colour of each
// position k = 2*j + i of a 2x2 quad is a compile-time constant (template L =
// the Bayer layout seen from the quad's top-left).  Every plane is stored by
// quad position: one dense row-major plane of quads per position, so the
// neighbour (dx, dy) of a sample is a compile-time position and quad offset,
// consecutive threads touch consecutive elements (no shared-memory bank
// conflicts), and chroma, gradients and directions are kept only at the two
// non-green positions A (first row, column ax(L)) and B (second row, column
// 1 - ax(L)), red and blue only at the two green positions.
//
// T = double: the reference's arithmetic, in binary64, in the reference's
// order (bit-exact outputs).  T = float: the same steps in binary32 (outputs
// within a few ulp of the reference's float cast) with the direction decision
// made exactly.  The binary32 classifier sums h and v are within
//   300 u smax + 8 u h      (u = 2^-24, smax = max |sample| of the tile's
// footprint: every five-tap green, chroma, gradient and weighted sum rounds at
// most once per operation on values bounded by small multiples of smax), so a
// site with |v - h| <= 640 u smax + 9 u (h + v) is re-decided by the
// reference's classifier in binary64 (a second pass over a list of such
// sites); every other site's binary32 decision equals the reference's.

constexpr int RQW = (MN_TW + 12) / 2, RQH = (MN_TH + 12) / 2;  // raw planes: quads of the r=6 region, origin (-6,-6)
constexpr int RQN = RQW * RQH;
constexpr int QW = (MN_TW + 8) / 2, QH = (MN_TH + 8) / 2;      // chroma planes: quads of the r=4 region, origin (-4,-4)
constexpr int QN = QW * QH;
constexpr int GQW = QW - 2, GQH = QH - 2;                      // green, direction, red, blue: r=2 region, origin (-2,-2)
constexpr int GQN = GQW * GQH;
constexpr int MN_WARPS = MN_THREADS / 32;
static_assert(MN_TW == 32 && MN_TH == 2 * MN_WARPS,
              "epilogue mapping: warp w renders rows w and w + MN_TH/2, each lane two pixels of one row");

// Column of the first row's non-green position (A); B sits in the second row
// at the other column.  Green positions: G0 = (1 - ax, 0), G1 = (ax, 1).
__host__ __device__ constexpr int ng_col(int l) { return l < 2 ? 0 : 1; }
__host__ __device__ constexpr int floor_half(int v) { return v >= 0 ? v / 2 : -((1 - v) / 2); }
// Quad position of the sample (dx, dy) away from position (i, j) of a quad.
__host__ __device__ constexpr int pos_at(int i, int j, int dx, int dy) { return ((j + dy) & 1) * 2 + ((i + dx) & 1); }
// Its quad, as an offset on a grid of W quads per row.
__host__ __device__ constexpr int quad_at(int i, int j, int dx, int dy, int W) {
    return floor_half(j + dy) * W + floor_half(i + dx);
}

enum { GH_A, GH_B, GV_A, GV_B, CH_A, CH_B, CV_A, CV_B, DH_A, DH_B, DV_A, DV_B, NG_PLANES };

template <typename T>
struct FastSmemT {
    float raw[4][RQN];           // normalized samples by quad position, r = 6 (binary32 values, widened on use)
    T ng[NG_PLANES][QN];         // chroma stage at A and B, r = 4; later red/blue
    T green[2][GQN];             // interpolated green at A and B, r = 2
    uint8_t horiz[2][GQN];       // direction at A and B, r = 2
    unsigned smax_bits;          // max |sample| of the footprint (float bits)
    unsigned rechecks;           // entries of `recheck`
    uint16_t recheck[2 * GQN];   // near-tie sites: quad of the r=2 region * 2 + (site B)
    SmemCurve curve;             // the program's master curve when small (stage_curve_smem)
};
using FastSmem = FastSmemT<double>;
constexpr int FAST_RB_PLANES = 3;   // ng planes holding red and blue at G0, G1 (4 * GQN values)
static_assert(4 * GQN <= FAST_RB_PLANES * QN, "red/blue must fit in the dead chroma planes");

// Raw sample (DX, DY) away from position (I, J) of raw quad rq.
template <typename T, int I, int J, int DX, int DY>
__device__ __forceinline__ T raw_q(const float (*raw)[RQN], int rq) {
    return (T)raw[pos_at(I, J, DX, DY)][rq + quad_at(I, J, DX, DY, RQW)];
}

// MenonDemosaic.cpp:112-115 five-tap directional green at position (I, J)
// along (DX, DY).
template <typename T, int I, int J, int DX, int DY>
__device__ __forceinline__ T five_q(const float (*raw)[RQN], int rq) {
    return five_tap<T>(raw_q<T, I, J, -2 * DX, -2 * DY>(raw, rq), raw_q<T, I, J, -DX, -DY>(raw, rq),
                       (T)raw[2 * J + I][rq], raw_q<T, I, J, DX, DY>(raw, rq), raw_q<T, I, J, 2 * DX, 2 * DY>(raw, rq));
}

// Interpolated green at the non-green sample (DX, DY) away from position
// (I, J) of r=2 quad k (plane 0 holds A, plane 1 B: a non-green position's
// row picks its plane).
template <int I, int J, int DX, int DY, typename T>
__device__ __forceinline__ T green_q(const T (*green)[GQN], int k) {
    return green[pos_at(I, J, DX, DY) >> 1][k + quad_at(I, J, DX, DY, GQW)];
}

// The reference's classifier at non-green position (I, J) of raw quad rq, in
// binary64 from the binary32 samples, terms in its order
// (MenonDemosaic.cpp:120-147): chroma C = s - five-tap green, gradients
// |C(p) - C(p + 2 along the axis)|, horizontal iff v >= h.
template <int I, int J>
__device__ __forceinline__ bool exact_horizontal_q(const float (*raw)[RQN], int rq) {
    auto at = [&](int dx, int dy) -> double {
        return (double)raw[pos_at(I, J, dx, dy)][rq + quad_at(I, J, dx, dy, RQW)];
    };
    auto five_d = [&](int x, int y, int dx, int dy) {
        return dsub(dadd(__dmul_rn(0.5, dadd(at(x - dx, y - dy), at(x + dx, y + dy))), __dmul_rn(0.5, at(x, y))),
                    __dmul_rn(0.25, dadd(at(x - 2 * dx, y - 2 * dy), at(x + 2 * dx, y + 2 * dy))));
    };
    auto dh = [&](int x, int y) {
        return fabs(dsub(dsub(at(x, y), five_d(x, y, 1, 0)), dsub(at(x + 2, y), five_d(x + 2, y, 1, 0))));
    };
    auto dv = [&](int x, int y) {
        return fabs(dsub(dsub(at(x, y), five_d(x, y, 0, 1)), dsub(at(x, y + 2), five_d(x, y + 2, 0, 1))));
    };
    double h = 0.0, v = 0.0;
    h = dadd(h, dh(0, 2));                    v = dadd(v, dv(2, 0));
    h = dadd(h, dh(-2, 2));                   v = dadd(v, dv(2, -2));
    h = dadd(h, dh(-1, 1));                   v = dadd(v, dv(1, -1));
    h = dadd(h, __dmul_rn(3.0, dh(0, 0)));    v = dadd(v, __dmul_rn(3.0, dv(0, 0)));
    h = dadd(h, __dmul_rn(3.0, dh(-2, 0)));   v = dadd(v, __dmul_rn(3.0, dv(0, -2)));
    h = dadd(h, dh(-1, -1));                  v = dadd(v, dv(-1, -1));
    h = dadd(h, dh(0, -2));                   v = dadd(v, dv(-2, 0));
    h = dadd(h, dh(-2, -2));                  v = dadd(v, dv(-2, -2));
    return v >= h;
}

// MenonDemosaic.cpp:151-161 red and blue at green position (I, J) of raw quad
// rq / r=2 quad k: the row's non-green neighbours carry that colour along the
// row, the other colour comes from the column.
template <int L, int I, int J, typename T>
__device__ __forceinline__ void rb_at_green(const FastSmemT<T>& S, int rq, int k, T& rr, T& bb) {
    constexpr bool red_h = pat(L, (J << 1) | (I ^ 1)) == 0;
    constexpr int rx = red_h ? 1 : 0, ry = red_h ? 0 : 1;   // red axis
    constexpr int bx = 1 - rx, by = 1 - ry;                 // blue axis
    const T g = (T)S.raw[2 * J + I][rq];
    rr = r_sub(r_add(g, half_sum(raw_q<T, I, J, -rx, -ry>(S.raw, rq), raw_q<T, I, J, rx, ry>(S.raw, rq))),
               half_sum(green_q<I, J, -rx, -ry>(S.green, k), green_q<I, J, rx, ry>(S.green, k)));
    bb = r_sub(r_add(g, half_sum(raw_q<T, I, J, -bx, -by>(S.raw, rq), raw_q<T, I, J, bx, by>(S.raw, rq))),
               half_sum(green_q<I, J, -bx, -by>(S.green, k), green_q<I, J, bx, by>(S.green, k)));
}

// Row J of output quad (r=2 quad k, raw quad rq): both pixels' RGB after the
// opposite colour at the R/B site (MenonDemosaic.cpp:162-173), and their
// directions.  rb = red at G0, G1 then blue at G0, G1 (GQN each).
template <int L, int J, typename T>
__device__ __forceinline__ void fast_row(const FastSmemT<T>& S, const T* rb, int rq, int k, T (&rr)[2], T (&gg)[2],
                                         T (&bb)[2], bool (&hz)[2]) {
    constexpr int AX = ng_col(L);
    constexpr int NI = J == 0 ? AX : 1 - AX;   // column of this row's non-green position
    constexpr int GI = 1 - NI;
    constexpr int own = pat(L, 2 * J + NI);     // 0 red or 2 blue
    // green position of this row
    rr[GI] = rb[J * GQN + k];
    bb[GI] = rb[(2 + J) * GQN + k];
    gg[GI] = (T)S.raw[2 * J + GI][rq];
    hz[GI] = true;
    // non-green position: its neighbours along the direction are green
    // positions, of this row's kind along the row and of the other row's kind
    // along the column
    const bool h = S.horiz[J][k];
    const T* red = rb + (h ? J : 1 - J) * GQN;
    const T* blue = red + 2 * GQN;
    const int om = k + (h ? quad_at(NI, J, -1, 0, GQW) : quad_at(NI, J, 0, -1, GQW));
    const int op = k + (h ? quad_at(NI, J, 1, 0, GQW) : quad_at(NI, J, 0, 1, GQW));
    const T s = (T)S.raw[2 * J + NI][rq];
    if (own == 2) {
        bb[NI] = s;
        rr[NI] = r_sub(r_add(s, half_sum(red[om], red[op])), half_sum(blue[om], blue[op]));
    } else {
        rr[NI] = s;
        bb[NI] = r_sub(r_add(s, half_sum(blue[om], blue[op])), half_sum(red[om], red[op]));
    }
    gg[NI] = S.green[J][k];
    hz[NI] = h;
}

template <int L, typename T>
__device__ __forceinline__ void menon_fast(FastSmemT<T>& S, const DevRaw& raw, int x0, int y0, int ox, int oy,
                                           int ow, int oh, int stage_end, const DevProgram& P,
                                           float* __restrict__ out, size_t out_stride, uint32_t& err,
                                           unsigned long long* ties, uint8_t* dirs) {
    constexpr bool F32 = sizeof(T) == 4;
    constexpr int AX = ng_col(L), BX = 1 - AX;
    const int t = threadIdx.x;
    if (t == 0) {
        S.smax_bits = 0;
        S.rechecks = 0;
    }
    // 1. normalized raw (RawEngine.cpp:89-97), r = 6 around the tile, by quad position
    float local_max = 0.0f;
    load_quad_planes<RQW, RQH, MN_THREADS>(S.raw, raw, x0 - 6, y0 - 6, &local_max);
    const int sc_stage = stage_curve_smem(S.curve, P, 0, stage_end);
    if constexpr (F32) {
        for (int o = 16; o; o >>= 1) local_max = fmaxf(local_max, __shfl_xor_sync(0xffffffffu, local_max, o));
        __syncthreads();   // smax_bits and rechecks are zeroed
        if ((t & 31) == 0) atomicMax(&S.smax_bits, __float_as_uint(local_max));
    }
    __syncthreads();
    // 2. directional green and chroma at A and B of every quad of the r=4
    //    region (MenonDemosaic.cpp:107-119)
#pragma unroll 2
    for (int q = t; q < QN; q += MN_THREADS) {
        const int qx = q % QW, qy = q / QW;
        const int rq = (qy + 1) * RQW + qx + 1;
        const T sa = (T)S.raw[AX][rq], sb = (T)S.raw[2 + BX][rq];
        const T ha = five_q<T, AX, 0, 1, 0>(S.raw, rq), va = five_q<T, AX, 0, 0, 1>(S.raw, rq);
        const T hb = five_q<T, BX, 1, 1, 0>(S.raw, rq), vb = five_q<T, BX, 1, 0, 1>(S.raw, rq);
        S.ng[GH_A][q] = ha;
        S.ng[GV_A][q] = va;
        S.ng[CH_A][q] = r_sub(sa, ha);
        S.ng[CV_A][q] = r_sub(sa, va);
        S.ng[GH_B][q] = hb;
        S.ng[GV_B][q] = vb;
        S.ng[CH_B][q] = r_sub(sb, hb);
        S.ng[CV_B][q] = r_sub(sb, vb);
    }
    __syncthreads();
    // 3. forward chroma gradients (MenonDemosaic.cpp:120-125): the same-position
    //    neighbour two pixels right is the next quad, two pixels down the next row
#pragma unroll 2
    for (int q = t; q < QN; q += MN_THREADS) {
        const int qx = q % QW, qy = q / QW;
        if (qx < QW - 1) {
            S.ng[DH_A][q] = fabs(r_sub(S.ng[CH_A][q], S.ng[CH_A][q + 1]));
            S.ng[DH_B][q] = fabs(r_sub(S.ng[CH_B][q], S.ng[CH_B][q + 1]));
        }
        if (qy < QH - 1) {
            S.ng[DV_A][q] = fabs(r_sub(S.ng[CV_A][q], S.ng[CV_A][q + QW]));
            S.ng[DV_B][q] = fabs(r_sub(S.ng[CV_B][q], S.ng[CV_B][q + QW]));
        }
    }
    __syncthreads();
    // 4. classifier and green (MenonDemosaic.cpp:130-147) for the quads of the r=2
    //    region, terms in the reference's order; (-1,+-1) offsets land on the other position
    const float band_abs = F32 ? 640.0f * 5.9604644775390625e-8f * __uint_as_float(S.smax_bits) : 0.0f;
#pragma unroll 2
    for (int k = t; k < GQN; k += MN_THREADS) {
        const int qx = k % GQW + 1, qy = k / GQW + 1;
        const int q = qy * QW + qx;
        const T* dhA = S.ng[DH_A];
        const T* dhB = S.ng[DH_B];
        const T* dvA = S.ng[DV_A];
        const T* dvB = S.ng[DV_B];
        const T three = T(3);
        // A site: B quads at column offsets -(1-AX) / +AX
        T h = 0, v = 0;
        h = r_add(h, dhA[q + QW]);               v = r_add(v, dvA[q + 1]);
        h = r_add(h, dhA[q + QW - 1]);           v = r_add(v, dvA[q - QW + 1]);
        h = r_add(h, dhB[q - BX]);               v = r_add(v, dvB[q - QW + AX]);
        h = r_add(h, r_mul(three, dhA[q]));      v = r_add(v, r_mul(three, dvA[q]));
        h = r_add(h, r_mul(three, dhA[q - 1]));  v = r_add(v, r_mul(three, dvA[q - QW]));
        h = r_add(h, dhB[q - QW - BX]);          v = r_add(v, dvB[q - QW - BX]);
        h = r_add(h, dhA[q - QW]);               v = r_add(v, dvA[q - 1]);
        h = r_add(h, dhA[q - QW - 1]);           v = r_add(v, dvA[q - QW - 1]);
        const bool hzA = v >= h;
        if (F32 && near_tie(h, v, band_abs)) S.recheck[atomicAdd(&S.rechecks, 1u)] = (uint16_t)(2 * k);
        // B site: A quads at column offsets -AX / +(1-AX)
        h = 0;
        v = 0;
        h = r_add(h, dhB[q + QW]);               v = r_add(v, dvB[q + 1]);
        h = r_add(h, dhB[q + QW - 1]);           v = r_add(v, dvB[q - QW + 1]);
        h = r_add(h, dhA[q + QW - AX]);          v = r_add(v, dvA[q + BX]);
        h = r_add(h, r_mul(three, dhB[q]));      v = r_add(v, r_mul(three, dvB[q]));
        h = r_add(h, r_mul(three, dhB[q - 1]));  v = r_add(v, r_mul(three, dvB[q - QW]));
        h = r_add(h, dhA[q - AX]);               v = r_add(v, dvA[q - AX]);
        h = r_add(h, dhB[q - QW]);               v = r_add(v, dvB[q - 1]);
        h = r_add(h, dhB[q - QW - 1]);           v = r_add(v, dvB[q - QW - 1]);
        const bool hzB = v >= h;
        if (F32 && near_tie(h, v, band_abs)) S.recheck[atomicAdd(&S.rechecks, 1u)] = (uint16_t)(2 * k + 1);
        S.horiz[0][k] = hzA;
        S.horiz[1][k] = hzB;
        S.green[0][k] = hzA ? S.ng[GH_A][q] : S.ng[GV_A][q];
        S.green[1][k] = hzB ? S.ng[GH_B][q] : S.ng[GV_B][q];
    }
    __syncthreads();
    if constexpr (F32) {
        // the near-tie sites, re-decided by the reference's binary64 classifier
        const unsigned n = S.rechecks;
        if (n) {
            // Rechecks are also made for halo sites that a neighbouring tile
            // renders; only the sites of this tile's own output are counted, so
            // every output site is counted once per render.
            const int cx0 = max(x0, ox), cx1 = min(x0 + MN_TW, ox + ow);
            const int cy0 = max(y0, oy), cy1 = min(y0 + MN_TH, oy + oh);
            unsigned own = 0;
            for (unsigned e = t; e < n; e += MN_THREADS) {
                const int code = S.recheck[e];
                const int k = code >> 1, site = code & 1;
                const int qx = k % GQW, qy = k / GQW;
                const int rq = (qy + 2) * RQW + qx + 2;
                const int q = (qy + 1) * QW + qx + 1;
                const bool hz = site ? exact_horizontal_q<BX, 1>(S.raw, rq) : exact_horizontal_q<AX, 0>(S.raw, rq);
                S.horiz[site][k] = hz;
                S.green[site][k] = hz ? S.ng[site ? GH_B : GH_A][q] : S.ng[site ? GV_B : GV_A][q];
                const int px = x0 + 2 * qx - 2 + (site ? BX : AX), py = y0 + 2 * qy - 2 + site;
                own += px >= cx0 && px < cx1 && py >= cy0 && py < cy1;
            }
            if (ties && own) atomicAdd(ties, (unsigned long long)own);
            __syncthreads();
        }
    }
    // 5. red and blue at the green positions of the r=1 ring (MenonDemosaic.cpp:151-161);
    //    the chroma planes are dead.  rb: red at G0, G1, then blue at G0, G1.
    T* rb = S.ng[0];
#pragma unroll 2
    for (int k = t; k < GQN; k += MN_THREADS) {
        const int qx = k % GQW, qy = k / GQW;
        const int rq = (qy + 2) * RQW + qx + 2;
        // relative pixel of the quad's top-left: (2 qx - 2, 2 qy - 2)
        const int px0 = 2 * qx - 2 + BX, py0 = 2 * qy - 2;   // G0
        const int px1 = 2 * qx - 2 + AX, py1 = 2 * qy - 1;   // G1
        if (px0 >= -1 && px0 <= MN_TW && py0 >= -1 && py0 <= MN_TH) {
            T rr, bb;
            rb_at_green<L, BX, 0>(S, rq, k, rr, bb);
            rb[k] = rr;
            rb[2 * GQN + k] = bb;
        }
        if (px1 >= -1 && px1 <= MN_TW && py1 >= -1 && py1 <= MN_TH) {
            T rr, bb;
            rb_at_green<L, AX, 1>(S, rq, k, rr, bb);
            rb[GQN + k] = rr;
            rb[3 * GQN + k] = bb;
        }
    }
    __syncthreads();
    // 6. opposite colour at R/B sites and float cast (MenonDemosaic.cpp:162-173),
    //    then the fused stages.  Warp w renders rows w and w + MN_TH/2 (the same
    //    quad row parity, so the row's layout is warp-uniform), a lane two
    //    adjacent pixels of one row.
    {
        const int w = t >> 5, lane = t & 31;
        const int row = w + (MN_TH / 2) * (lane >> 4);
        const int qx = lane & 15, qy = row >> 1;
        const int k = (qy + 1) * GQW + qx + 1;
        const int rq = (qy + 3) * RQW + qx + 3;
        T rr[2], gg[2], bb[2];
        bool hz[2];
        if (w & 1) fast_row<L, 1>(S, rb, rq, k, rr, gg, bb, hz);
        else fast_row<L, 0>(S, rb, rq, k, rr, gg, bb, hz);
        const int y = y0 + row;
        float R[2], G[2], B[2];
        bool keep[2];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int x = x0 + 2 * qx + i;
            keep[i] = x >= ox && y >= oy && x < ox + ow && y < oy + oh;
            // pixels outside the viewport enter the stages as zeros (never written)
            R[i] = keep[i] ? (float)rr[i] : 0.0f;
            G[i] = keep[i] ? (float)gg[i] : 0.0f;
            B[i] = keep[i] ? (float)bb[i] : 0.0f;
        }
        apply_stages_n<2>(P, 0, stage_end, R, G, B, err, &S.curve, sc_stage);
        // The tile's row span inside the viewport and 16-byte aligned (the
        // same for every thread of the block): adjacent lanes pair up, and the
        // pair's four pixels (48 bytes) leave as three aligned 16-byte stores --
        // the even lane's own first four floats plus its last two and the odd
        // lane's first two, the odd lane's last four.  Otherwise single floats.
        const bool wide = x0 >= ox && x0 + MN_TW <= ox + ow && ((x0 - ox) & 3) == 0 && (out_stride & 3) == 0 &&
                          (reinterpret_cast<uintptr_t>(out) & 15) == 0;
        if (wide) {
            const float p0 = __shfl_down_sync(0xffffffffu, R[0], 1);
            const float p1 = __shfl_down_sync(0xffffffffu, G[0], 1);
            if (y >= oy && y < oy + oh) {
                float* o = out + (size_t)(y - oy) * out_stride + (size_t)(x0 - ox) * 3 + 6 * qx;
                if ((qx & 1) == 0) {
                    reinterpret_cast<float4*>(o)[0] = make_float4(R[0], G[0], B[0], R[1]);
                    reinterpret_cast<float4*>(o)[1] = make_float4(G[1], B[1], p0, p1);
                } else {
                    *reinterpret_cast<float4*>(o + 2) = make_float4(B[0], R[1], G[1], B[1]);
                }
            }
        } else {
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                if (!keep[i]) continue;
                const int x = x0 + 2 * qx + i;
                float* o = out + (size_t)(y - oy) * out_stride + (size_t)(x - ox) * 3;
                o[0] = R[i];
                o[1] = G[i];
                o[2] = B[i];
            }
        }
        if (dirs) {
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int x = x0 + 2 * qx + i;
                if (keep[i]) dirs[(size_t)(y - oy) * ow + (x - ox)] = hz[i];
            }
        }
    }
}

union MenonShared {
    MenonSmemT<double> generic;
    MenonSmemT<float> generic32;
    FastSmemT<double> fast;
    FastSmemT<float> fast32;
};


// One CTA per MN_TW x MN_TH tile of the viewport, tiles anchored at an even
// sensor coordinate.  Interior tiles take the fast quad path; tiles whose
// footprint meets the active-area edge take the general mirrored path.
// Writes float32 RGB after stages [0, stage_end) (row stride in floats).
__device__ __forceinline__ void menon_cta(unsigned char* smem_raw, const DevRaw& raw, int x0, int y0, int ox,
                                          int oy, int ow, int oh, int layout, int stage_end, const DevProgram& P,
                                          float* __restrict__ out, size_t out_stride, unsigned long long* ties,
                                          uint32_t& err, bool exact, uint8_t* dirs) {
    // binary64 mode with tie counting takes the general path, which counts exact ties
    const bool interior = !(exact && ties) && x0 - 6 >= raw.ax && y0 - 6 >= raw.ay &&
                          x0 + MN_TW + 6 <= raw.ax + raw.aw && y0 + MN_TH + 6 <= raw.ay + raw.ah;
    if (interior && exact) {
        FastSmemT<double>& F = reinterpret_cast<MenonShared*>(smem_raw)->fast;
        switch (layout) {
        case 0: menon_fast<0>(F, raw, x0, y0, ox, oy, ow, oh, stage_end, P, out, out_stride, err, ties, dirs); break;
        case 1: menon_fast<1>(F, raw, x0, y0, ox, oy, ow, oh, stage_end, P, out, out_stride, err, ties, dirs); break;
        case 2: menon_fast<2>(F, raw, x0, y0, ox, oy, ow, oh, stage_end, P, out, out_stride, err, ties, dirs); break;
        default: menon_fast<3>(F, raw, x0, y0, ox, oy, ow, oh, stage_end, P, out, out_stride, err, ties, dirs); break;
        }
        return;
    }
    if (interior) {
        FastSmemT<float>& F = reinterpret_cast<MenonShared*>(smem_raw)->fast32;
        switch (layout) {
        case 0: menon_fast<0>(F, raw, x0, y0, ox, oy, ow, oh, stage_end, P, out, out_stride, err, ties, dirs); break;
        case 1: menon_fast<1>(F, raw, x0, y0, ox, oy, ow, oh, stage_end, P, out, out_stride, err, ties, dirs); break;
        case 2: menon_fast<2>(F, raw, x0, y0, ox, oy, ow, oh, stage_end, P, out, out_stride, err, ties, dirs); break;
        default: menon_fast<3>(F, raw, x0, y0, ox, oy, ow, oh, stage_end, P, out, out_stride, err, ties, dirs); break;
        }
        return;
    }
    MenonCtx c;
    c.x0 = x0;
    c.y0 = y0;
    c.xe = min(c.x0 + MN_TW, ox + ow);
    c.ye = min(c.y0 + MN_TH, oy + oh);
    c.ax = raw.ax; c.ay = raw.ay; c.aw = raw.aw; c.ah = raw.ah;
    if (exact) {
        MenonSmemT<double>& S = reinterpret_cast<MenonShared*>(smem_raw)->generic;
        menon_tile(S, raw, c, ties);
        menon_tile_out(S, raw, c, ox, oy, ow, oh, stage_end, P, out, out_stride, err, dirs);
    } else {
        MenonSmemT<float>& S = reinterpret_cast<MenonShared*>(smem_raw)->generic32;
        menon_tile(S, raw, c, ties);
        menon_tile_out(S, raw, c, ox, oy, ow, oh, stage_end, P, out, out_stride, err, dirs);
    }
}

__global__ void __launch_bounds__(MN_THREADS, 4)
menon_kernel(const __grid_constant__ DevRaw raw, int ox, int oy, int ow, int oh, int layout, int stage_end,
             const __grid_constant__ DevProgram P, float* __restrict__ out, size_t out_stride,
             uint32_t* status, unsigned long long* ties, int exact, uint8_t* dirs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int x0 = (ox & ~1) + blockIdx.x * MN_TW;
    const int y0 = (oy & ~1) + blockIdx.y * MN_TH;
    uint32_t err = 0;
    menon_cta(smem_raw, raw, x0, y0, ox, oy, ow, oh, layout, stage_end, P, out, out_stride, ties, err, exact != 0,
              dirs);
    report(status, err);
}

// ------------------------------------------------------------ mip reduction

// RawEngine.cpp:585-600: each reduced pixel averages its native footprint
// (clipped at the native region's edge, actual count) in double, row-major
// footprint order; then the stages after the anchor run on the reduced pixel.
__device__ __forceinline__ void reduce_pixel(const float* __restrict__ native, int nw, int nh, size_t native_stride,
                                             int scale, int x, int y, int stage_begin, int stage_end,
                                             const DevProgram& P, float* __restrict__ out, size_t out_stride,
                                             uint32_t& err) {
    double s0 = 0, s1 = 0, s2 = 0;
    int count = 0;
    const int y1 = min((y + 1) * scale, nh), x1 = min((x + 1) * scale, nw);
    for (int sy = y * scale; sy < y1; ++sy)
        for (int sx = x * scale; sx < x1; ++sx) {
            const float* p = native + (size_t)sy * native_stride + (size_t)sx * 3;
            s0 = __dadd_rn(s0, (double)p[0]);
            s1 = __dadd_rn(s1, (double)p[1]);
            s2 = __dadd_rn(s2, (double)p[2]);
            ++count;
        }
    const double n = (double)count;
    float r = (float)__ddiv_rn(s0, n), g = (float)__ddiv_rn(s1, n), b = (float)__ddiv_rn(s2, n);
    apply_stages(P, stage_begin, stage_end, r, g, b, err);
    float* o = out + (size_t)y * out_stride + (size_t)x * 3;
    o[0] = r;
    o[1] = g;
    o[2] = b;
}

__global__ void mip_reduce_kernel(const float* __restrict__ native, int nw, int nh,
                                  size_t native_stride, int scale, int ow, int oh, int stage_begin,
                                  int stage_end, const __grid_constant__ DevProgram P,
                                  float* __restrict__ out, size_t out_stride, uint32_t* status) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= ow || y >= oh) return;
    uint32_t err = 0;
    reduce_pixel(native, nw, nh, native_stride, scale, x, y, stage_begin, stage_end, P, out, out_stride, err);
    report(status, err);
}

// ----------------------------------------------------------- batched render

// Phase 1 of a batched render.  Dispatch 0: a grid sized to the SMs takes
// tiles from an atomic queue until it is empty; 1: one CTA per tile; 2: a grid
// sized to the SMs takes tiles blockIdx.x, +gridDim.x, ..., prefetching the
// next tile's record into shared memory (cp.async) while the current tile
// renders.  Each tile runs exactly the per-tile code of the single-request
// kernels, so a batched request's pixels equal its single render bit for bit.
template <int POLICY>
__device__ __forceinline__ void batch_tile(unsigned char* smem_raw, const BatchParams& A, const BatchUnit& T,
                                           uint32_t& err) {
    const int image = T.image, program = T.program, x0 = T.x0, y0 = T.y0, ox = T.ox, oy = T.oy, ow = T.ow,
              oh = T.oh, layout = T.layout, stage_end = T.stage_end, menon = T.menon;
    float* out = T.out;
    const size_t out_stride = (size_t)T.out_stride;
    const DevRaw& raw = A.images[image];
    const DevProgram& P = A.programs[program];
    if (menon)
        menon_cta(smem_raw, raw, x0, y0, ox, oy, ow, oh, layout, stage_end, P, out, out_stride, nullptr, err,
                  POLICY == 1, nullptr);
    else
        bilinear_cta(reinterpret_cast<float(*)[BL_SW]>(smem_raw), raw, x0, y0, ox, oy, ow, oh, layout, stage_end, P,
                     out, out_stride, err, reinterpret_cast<SmemCurve*>(smem_raw + BL_CURVE_OFFSET));
}

__device__ __forceinline__ void prefetch_unit(BatchUnit* dst, const BatchUnit* src) {
    if (threadIdx.x < 4) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(reinterpret_cast<char*>(dst) + 16 * threadIdx.x);
        const char* g = reinterpret_cast<const char*>(src) + 16 * threadIdx.x;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(g) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <int POLICY>
__global__ void __launch_bounds__(MN_THREADS, 4) batch_render_kernel(const __grid_constant__ BatchParams A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(16) BatchUnit s_rec[2];
    __shared__ uint32_t s_unit;
    uint32_t err = 0;
    if (A.dispatch == 1) {
        if (blockIdx.x < A.units) batch_tile<POLICY>(smem_raw, A, A.units_rec[blockIdx.x], err);
    } else if (A.dispatch == 0) {
        for (;;) {
            if (threadIdx.x == 0) s_unit = atomicAdd(A.queue, 1u);
            __syncthreads();
            const uint32_t u = s_unit;
            __syncthreads();
            if (u >= A.units) break;
            batch_tile<POLICY>(smem_raw, A, A.units_rec[u], err);
            __syncthreads();
        }
    } else {
        uint32_t u = blockIdx.x;
        if (u < A.units) prefetch_unit(&s_rec[0], &A.units_rec[u]);
        for (uint32_t i = 0; u < A.units; ++i) {
            asm volatile("cp.async.wait_all;\n" ::: "memory");
            __syncthreads();
            const uint32_t next = u + gridDim.x;
            if (next < A.units) prefetch_unit(&s_rec[(i + 1) & 1], &A.units_rec[next]);
            batch_tile<POLICY>(smem_raw, A, s_rec[i & 1], err);
            __syncthreads();
            u = next;
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
    }
    report(A.status, err);
}

// Phase 2: one CTA of RD_TW x RD_TH threads per block of reduced pixels.
__global__ void __launch_bounds__(RD_TW * RD_TH) batch_reduce_kernel(const __grid_constant__ BatchParams A) {
    const uint32_t u = blockIdx.x;
    if (u >= A.runits) return;
    const ReduceTask& T = A.rtasks[A.runit_task[u]];
    const int local = (int)(u - T.unit_begin);
    const int x = (local % T.tiles_x) * RD_TW + (int)threadIdx.x % RD_TW;
    const int y = (local / T.tiles_x) * RD_TH + (int)threadIdx.x / RD_TW;
    if (x >= T.ow || y >= T.oh) return;
    uint32_t err = 0;
    reduce_pixel(T.native, T.nw, T.nh, T.native_stride, T.scale, x, y, T.stage_begin, T.stage_end,
                 A.programs[T.program], T.out, T.out_stride, err);
    report(A.status, err);
}

static_assert(BL_THREADS == MN_THREADS, "batched tiles share one block size");
static_assert(BATCH_MENON_TW == MN_TW && BATCH_MENON_TH == MN_TH && BATCH_BILINEAR_TW == BL_TW &&
                  BATCH_BILINEAR_TH == BL_TH,
              "batch planner tile sizes");
static_assert(sizeof(MenonShared) >= BL_CURVE_OFFSET + sizeof(SmemCurve),
              "bilinear tiles and their curve tables fit the batch's shared memory");

static_assert(sizeof(BatchParams) <= 32000, "batch launch parameters exceed the 32 KB kernel parameter limit");

// Phase 1 of one launch group (grid CTAs), or phase 2 when reduce is set.
cudaError_t launch_batch_group(const BatchParams& A, uint32_t grid, bool reduce, cudaStream_t stream) {
    if (!reduce) {
        const size_t smem = sizeof(MenonShared);
        auto kernel = A.menon_policy == 2 ? batch_render_kernel<2> : batch_render_kernel<1>;
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        if (A.units && grid) kernel<<<grid, MN_THREADS, smem, stream>>>(A);
    } else if (A.runits) {
        batch_reduce_kernel<<<A.runits, RD_TW * RD_TH, 0, stream>>>(A);
    }
    return cudaGetLastError();
}

// ----------------------------------------------------------- raster sources

// RasterSourceNode::render_level (RawEngine.cpp:346-406) followed by the stage
// program: mip 0 copies the pixel, mip 1/2 average the clipped scale x scale
// footprint in double (row-major, per channel) with the actual count.
__global__ void raster_render_kernel(const float* __restrict__ in, size_t in_stride, int width, int height,
                                     int ox, int oy, int ow, int oh, int scale, int stage_end,
                                     const __grid_constant__ DevProgram P, float* __restrict__ out,
                                     size_t out_stride, uint32_t* status) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= ow || y >= oh) return;
    float r, g, b;
    if (scale == 1) {
        const float* p = in + (size_t)(oy + y) * in_stride + (size_t)(ox + x) * 3;
        r = p[0]; g = p[1]; b = p[2];
    } else {
        const int sy0 = (oy + y) * scale, sx0 = (ox + x) * scale;
        const int sy1 = min(sy0 + scale, height), sx1 = min(sx0 + scale, width);
        double s0 = 0, s1 = 0, s2 = 0;
        for (int sy = sy0; sy < sy1; ++sy)
            for (int sx = sx0; sx < sx1; ++sx) {
                const float* p = in + (size_t)sy * in_stride + (size_t)sx * 3;
                s0 = __dadd_rn(s0, (double)p[0]);
                s1 = __dadd_rn(s1, (double)p[1]);
                s2 = __dadd_rn(s2, (double)p[2]);
            }
        const double n = (double)((sx1 - sx0) * (sy1 - sy0));
        r = (float)__ddiv_rn(s0, n);
        g = (float)__ddiv_rn(s1, n);
        b = (float)__ddiv_rn(s2, n);
    }
    uint32_t err = 0;
    apply_stages(P, 0, stage_end, r, g, b, err);
    float* o = out + (size_t)y * out_stride + (size_t)x * 3;
    o[0] = r;
    o[1] = g;
    o[2] = b;
    report(status, err);
}

cudaError_t launch_raster(const float* in, size_t in_stride, int width, int height, int ox, int oy, int ow, int oh,
                          int mip, const DevProgram& P, float* out, size_t out_stride, uint32_t* status,
                          cudaStream_t stream) {
    if (ow <= 0 || oh <= 0) return cudaSuccess;
    dim3 block(32, 8);
    dim3 grid((ow + 31) / 32, (oh + 7) / 8);
    raster_render_kernel<<<grid, block, 0, stream>>>(in, in_stride, width, height, ox, oy, ow, oh, 1 << mip,
                                                     (int)P.count, P, out, out_stride, status);
    return cudaGetLastError();
}

// ------------------------------------------------------------------- launch

size_t menon_smem_bytes() { return sizeof(MenonShared); }

// Bayer layout seen from an even sensor coordinate (the fast path's template).
int quad_layout(const DevRaw& raw) {
    int e[4];
    for (int k = 0; k < 4; ++k) {
        const int i = k & 1, j = k >> 1;
        e[k] = raw.site_color[((j + (int)raw.phase_y) & 1) * 2 + ((i + (int)raw.phase_x) & 1)];
    }
    for (int l = 0; l < 4; ++l)
        if (pat(l, 0) == e[0] && pat(l, 1) == e[1] && pat(l, 2) == e[2] && pat(l, 3) == e[3]) return l;
    return 0;
}

// demosaic: 0 bilinear, 1 Menon in binary64 (bit-exact), 2 Menon in binary32
// with exact directions.  dirs (optional, device, ow x oh) receives the Menon
// direction of every viewport pixel (1 = horizontal; green sites 1).
cudaError_t launch_demosaic(uint32_t demosaic, const DevRaw& raw, int ox, int oy, int ow, int oh,
                            int stage_end, const DevProgram& P, float* out, size_t out_stride,
                            uint32_t* status, unsigned long long* ties, cudaStream_t stream,
                            uint32_t* launches, uint8_t* dirs) {
    if (ow <= 0 || oh <= 0) return cudaSuccess;
    // Menon with a singleton active-area axis is bilinear (RawEngine.cpp:303).
    if (demosaic >= 1 && raw.aw > 1 && raw.ah > 1) {
        const size_t smem = sizeof(MenonShared);
        cudaError_t e = cudaFuncSetAttribute(menon_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        const int gx0 = ox & ~1, gy0 = oy & ~1;
        dim3 grid((ox + ow - gx0 + MN_TW - 1) / MN_TW, (oy + oh - gy0 + MN_TH - 1) / MN_TH);
        menon_kernel<<<grid, MN_THREADS, smem, stream>>>(raw, ox, oy, ow, oh, quad_layout(raw), stage_end, P, out,
                                                         out_stride, status, ties, demosaic == 1 ? 1 : 0, dirs);
    } else {
        const int gx0 = ox & ~1, gy0 = oy & ~1;
        dim3 grid((ox + ow - gx0 + BL_TW - 1) / BL_TW, (oy + oh - gy0 + BL_TH - 1) / BL_TH);
        bilinear_kernel<<<grid, BL_THREADS, 0, stream>>>(raw, ox, oy, ow, oh, quad_layout(raw), stage_end, P, out,
                                                         out_stride, status);
    }
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t launch_mip_reduce(const float* native, int nw, int nh, size_t native_stride, int mip,
                              int ow, int oh, int stage_begin, int stage_end, const DevProgram& P,
                              float* out, size_t out_stride, uint32_t* status, cudaStream_t stream,
                              uint32_t* launches) {
    if (ow <= 0 || oh <= 0) return cudaSuccess;
    dim3 block(32, 8);
    dim3 grid((ow + 31) / 32, (oh + 7) / 8);
    mip_reduce_kernel<<<grid, block, 0, stream>>>(native, nw, nh, native_stride, 1 << mip, ow, oh,
                                                  stage_begin, stage_end, P, out, out_stride, status);
    if (launches) ++*launches;
    return cudaGetLastError();
}

}  // namespace re
