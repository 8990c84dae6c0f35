// Local-contrast stencils of the render path: Sharpen, Clarity, Texture and
// Convolution (SpatialOps.cpp:319-701), bit-exact with the reference.
//
// Every stencil reads a caller window of the node's input (the output
// rectangle grown by the stencil's halo and clipped to the image, the
// reference's `needed` region) and writes the output rectangle.  A CTA owns a
// 16 x 16 output tile: it stages the tile plus its halo from the window in
// shared memory (RGB or working Y, as binary64), flags any
// non-finite staged sample, and each thread evaluates one output pixel with
// the reference's binary64 operations in the reference's order:
//   Sharpen      per channel, the ordered sum over the clipped square of
//                (neighbour - centre), detail = -(sum / count),
//                out = centre + amount * detail;
//   Clarity      the same over working Y, applied to all three channels with
//                the midtone weight (4 Y)(1 - Y) for 0 < Y < 1;
//   Texture      2 * scale passes of the true-edge-normalised horizontal then
//                vertical [1, 2, 1] blur of working Y on two shared planes
//                that shrink by one pixel per pass, detail = B^scale -
//                B^(2 scale), the same midtone weighting;
//   Convolution  the flipped kernel over replicate-clamped coordinates,
//                sum = sum + w * x in row-major kernel order.
// The staged tile is every sample the reference checks for finiteness (the
// union of the CTAs' staged regions is the `needed` region), so a non-finite
// input anywhere in it is reported like the reference reports it.  Results
// beyond float32 range are reported after the launch; the first failure kind
// wins as in the reference (input checks run before any output).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <string>
#include <vector>

#include "re_device.cuh"

namespace re {
void set_last_error(const std::string& msg);
}

using namespace re;

namespace {

constexpr int ST_TILE = 16;
constexpr int ST_MAX_HALO = 8;
constexpr int ST_SPAN = ST_TILE + 2 * ST_MAX_HALO;   // 32
constexpr uint32_t KEY_INPUT = (2u << 8) | ST_INVALID;    // non-finite input sample
constexpr uint32_t KEY_OUTPUT = (1u << 8) | ST_INVALID;   // result beyond float32

struct Geo {
    const float* in;
    size_t in_stride;      // floats per row
    int wx, wy, ww, wh;    // window (image coordinates of in[0])
    int ix, iy, iw, ih;    // image bounds at this level
    int ox, oy, ow, oh;    // output rectangle
    float* out;
    size_t out_stride;
    uint32_t* status;
};

__device__ __forceinline__ void flag(uint32_t* status, uint32_t key) { atomicMax(status, key); }

// Stages this CTA's tile grown by (hx, hy), clipped to the window and to the
// output grown by the halo (the reference's `needed` region, which a tile
// reaching past the output's right or bottom edge must not read beyond), as
// RGB values at smem[((y - sy0) * ST_SPAN + (x - sx0)) * 3 + c], widened to
// binary64 once here (exactly) rather than at every tap that reads them.
// TW x TH is the tile, SPAN the staged row pitch in pixels.
template <int TW = ST_TILE, int TH = ST_TILE, int SPAN = ST_SPAN>
__device__ __forceinline__ void stage_rgb(const Geo& G, int hx, int hy, double* smem, int sx0, int sy0) {
    const int x0 = max(G.wx, sx0), x1 = min(min(G.wx + G.ww, sx0 + TW + 2 * hx), G.ox + G.ow + hx);
    const int y0 = max(G.wy, sy0), y1 = min(min(G.wy + G.wh, sy0 + TH + 2 * hy), G.oy + G.oh + hy);
    const int n = (x1 - x0) * 3;   // floats of one staged row; a warp copies a row per step
    bool bad = false;
    for (int y = y0 + (int)(threadIdx.x >> 5); n > 0 && y < y1; y += (int)(blockDim.x >> 5)) {
        const float* src = G.in + (size_t)(y - G.wy) * G.in_stride + (size_t)(x0 - G.wx) * 3;
        double* dst = smem + ((y - sy0) * SPAN + (x0 - sx0)) * 3;
        for (int i = (int)(threadIdx.x & 31u); i < n; i += 32) {
            const float v = src[i];
            bad |= !isfinite(v);
            dst[i] = (double)v;
        }
    }
    if (bad) flag(G.status, KEY_INPUT);
}

// Working Y of SpatialOps.cpp:482-483: (g + wr (r - g)) + wb (b - g).
__device__ __forceinline__ double working_y(float r, float g, float b, double wr, double wb) {
    const double R = r, Gc = g, B = b;
    return __dadd_rn(__dadd_rn(Gc, __dmul_rn(wr, __dsub_rn(R, Gc))), __dmul_rn(wb, __dsub_rn(B, Gc)));
}

// Stages working Y (binary64) of the TILE x TH tile grown by h, clipped like
// stage_rgb, at plane[(y - sy0) * SPAN + (x - sx0)].
template <int TILE = ST_TILE, int SPAN = ST_SPAN, int TH = TILE>
__device__ __forceinline__ void stage_y(const Geo& G, int h, double wr, double wb, double* plane, int sx0, int sy0) {
    const int x0 = max(G.wx, sx0), x1 = min(min(G.wx + G.ww, sx0 + TILE + 2 * h), G.ox + G.ow + h);
    const int y0 = max(G.wy, sy0), y1 = min(min(G.wy + G.wh, sy0 + TH + 2 * h), G.oy + G.oh + h);
    const int w = x1 - x0;   // a warp stages a row per step
    bool bad = false;
    for (int y = y0 + (int)(threadIdx.x >> 5); w > 0 && y < y1; y += (int)(blockDim.x >> 5)) {
        const float* src = G.in + (size_t)(y - G.wy) * G.in_stride + (size_t)(x0 - G.wx) * 3;
        double* dst = plane + (y - sy0) * SPAN + (x0 - sx0);
        for (int i = (int)(threadIdx.x & 31u); i < w; i += 32) {
            const float r = src[3 * i], g = src[3 * i + 1], b = src[3 * i + 2];
            bad |= !(isfinite(r) && isfinite(g) && isfinite(b));
            dst[i] = working_y(r, g, b, wr, wb);
        }
    }
    if (bad) flag(G.status, KEY_INPUT);
}

// Stores one output channel value from binary64, flagging results beyond
// float32 (SpatialOps.cpp checks |mapped| <= FLT_MAX before the cast).
__device__ __forceinline__ float to_output(const Geo& G, double mapped) {
    if (!(fabs(mapped) <= (double)FLT_MAX)) {
        flag(G.status, KEY_OUTPUT);
        return 0.0f;
    }
    return __double2float_rn(mapped);
}

// Output pixel of this thread, or false when it lies outside the output.
__device__ __forceinline__ bool my_pixel(const Geo& G, int& x, int& y) {
    x = G.ox + blockIdx.x * ST_TILE + (threadIdx.x % ST_TILE);
    y = G.oy + blockIdx.y * ST_TILE + (threadIdx.x / ST_TILE);
    return x < G.ox + G.ow && y < G.oy + G.oh;
}

// ---------------------------------------------------------------- sharpen

// Sharpen renders 16 x 64 output tiles: each thread owns four vertically
// adjacent pixels, so every staged sample it loads serves each of its pixels
// whose square holds it (radius <= 3: the staged tile is 22 x 70).
constexpr int SH_MAX_RADIUS = 3, SH_PX = 4, SH_TW = ST_TILE, SH_TH = ST_TILE * SH_PX;
constexpr int SH_SPAN = SH_TW + 2 * SH_MAX_RADIUS, SH_ROWS = SH_TH + 2 * SH_MAX_RADIUS;

// Sharpen's output for channel value `center` and its window sum
// (SpatialOps.cpp:688-696).
__device__ __forceinline__ float sharpen_out(const Geo& G, double center, double sum, double count, double amount) {
    const float cf = (float)center;   // exact: the value came from a float
    const double detail = -__ddiv_rn(sum, count);
    if (detail == 0.0) return cf;
    const double offset = __dmul_rn(amount, detail);
    return offset == 0.0 ? cf : to_output(G, __dadd_rn(center, offset));
}

// SpatialOps.cpp:667-697, radius R.  Each pixel's sum runs over its clipped
// square in row-major order (rows ascending, then columns), as in the
// reference.  Where no square of the thread's four pixels is clipped, the
// thread walks their rows once, holding a row's 2R+1 samples in registers, and
// adds them to every pixel whose square holds that row (compile-time row and
// pixel ranges); elsewhere each pixel sums its own clipped square.
// Six CTAs per SM (40 registers): 6 % faster than five at 48 for r 2.
template <int R>
__global__ void __launch_bounds__(ST_TILE* ST_TILE, 6) sharpen_kernel(Geo G, double amount) {
    __shared__ double tile[SH_SPAN * SH_ROWS * 3];
    const int tx0 = G.ox + blockIdx.x * SH_TW, ty0 = G.oy + blockIdx.y * SH_TH;
    const int sx0 = tx0 - R, sy0 = ty0 - R;
    stage_rgb<SH_TW, SH_TH, SH_SPAN>(G, R, R, tile, sx0, sy0);
    __syncthreads();
    const int x = tx0 + (int)(threadIdx.x % ST_TILE);
    const int y0 = ty0 + SH_PX * (int)(threadIdx.x / ST_TILE);
    const int rows = min(SH_PX, G.oy + G.oh - y0);   // this thread's pixels y0 .. y0 + rows - 1
    if (x >= G.ox + G.ow || rows <= 0) return;
    float* o = G.out + (size_t)(y0 - G.oy) * G.out_stride + (size_t)(x - G.ox) * 3;
    const bool whole = rows == SH_PX && x - R >= G.ix && x + R < G.ix + G.iw && y0 - R >= G.iy &&
                       y0 + SH_PX - 1 + R < G.iy + G.ih;
    if (whole) {
        constexpr int K = 2 * R + 1;
        const double count = (double)(K * K);
        for (int c = 0; c < 3; ++c) {
            double center[SH_PX], sum[SH_PX];
#pragma unroll
            for (int p = 0; p < SH_PX; ++p) {
                center[p] = tile[((y0 + p - sy0) * SH_SPAN + (x - sx0)) * 3 + c];
                sum[p] = 0.0;
            }
#pragma unroll
            for (int j = 0; j < SH_PX + 2 * R; ++j) {   // row y0 - R + j
                const double* row = tile + ((y0 - R + j - sy0) * SH_SPAN + (x - R - sx0)) * 3 + c;
                double v[K];
#pragma unroll
                for (int k = 0; k < K; ++k) v[k] = row[3 * k];
#pragma unroll
                for (int p = 0; p < SH_PX; ++p) {
                    if (j < p || j > p + 2 * R) continue;
#pragma unroll
                    for (int k = 0; k < K; ++k) sum[p] = __dadd_rn(sum[p], __dsub_rn(v[k], center[p]));
                }
            }
#pragma unroll
            for (int p = 0; p < SH_PX; ++p)
                o[(size_t)p * G.out_stride + c] = sharpen_out(G, center[p], sum[p], count, amount);
        }
        return;
    }
    const int left = max(G.ix, x - R), right = min(G.ix + G.iw - 1, x + R);
    for (int p = 0; p < rows; ++p) {
        const int y = y0 + p;
        const int top = max(G.iy, y - R), bottom = min(G.iy + G.ih - 1, y + R);
        const double count = (double)((right - left + 1) * (bottom - top + 1));
        for (int c = 0; c < 3; ++c) {
            const double center = tile[((y - sy0) * SH_SPAN + (x - sx0)) * 3 + c];
            double sum = 0.0;
            for (int yy = top; yy <= bottom; ++yy)
                for (int xx = left; xx <= right; ++xx)
                    sum = __dadd_rn(sum, __dsub_rn(tile[((yy - sy0) * SH_SPAN + (xx - sx0)) * 3 + c], center));
            o[(size_t)p * G.out_stride + c] = sharpen_out(G, center, sum, count, amount);
        }
    }
}

// ---------------------------------------------------------------- clarity

// SpatialOps.cpp:465-494 (per-pixel midtone offset shared by Clarity and Texture).
__device__ __forceinline__ void apply_offset(const Geo& G, int x, int y, double center, double detail, double amount) {
    const float* src = G.in + (size_t)(y - G.wy) * G.in_stride + (size_t)(x - G.wx) * 3;
    float* o = G.out + (size_t)(y - G.oy) * G.out_stride + (size_t)(x - G.ox) * 3;
    double offset = 0.0;
    if (center > 0.0 && center < 1.0 && detail != 0.0) {
        const double weight = __dmul_rn(__dmul_rn(4.0, center), __dsub_rn(1.0, center));
        const double strength = __dmul_rn(amount, weight);
        offset = __dmul_rn(strength, detail);
    }
    for (int c = 0; c < 3; ++c) o[c] = offset == 0.0 ? src[c] : to_output(G, __dadd_rn((double)src[c], offset));
}

// Clarity renders 16 x 64 output tiles like sharpen: four vertically adjacent
// pixels per thread (radius <= 8: the staged plane is 32 x 80).
constexpr int CL_MAX_RADIUS = 8, CL_SPAN = ST_TILE + 2 * CL_MAX_RADIUS, CL_ROWS = SH_TH + 2 * CL_MAX_RADIUS;

// SpatialOps.cpp:437-495, radius R.  A pixel with 0 < Y < 1 sums its clipped
// square of (neighbour - centre) in row-major order.  Where no square of the
// thread's four pixels is clipped, the thread walks their rows once with a
// row's 2R+1 values in registers and adds them to every pixel whose square
// holds the row (each pixel's sum keeps its own row-major order); elsewhere
// each pixel sums its own clipped square.
// Five CTAs per SM (48 registers): 3 % faster than four at 60 for r 8.
template <int R>
__global__ void __launch_bounds__(ST_TILE* ST_TILE, 5) clarity_kernel(Geo G, double amount, double wr, double wb) {
    __shared__ double plane[CL_SPAN * CL_ROWS];
    const int tx0 = G.ox + blockIdx.x * SH_TW, ty0 = G.oy + blockIdx.y * SH_TH;
    const int sx0 = tx0 - R, sy0 = ty0 - R;
    stage_y<SH_TW, CL_SPAN, SH_TH>(G, R, wr, wb, plane, sx0, sy0);
    __syncthreads();
    const int x = tx0 + (int)(threadIdx.x % ST_TILE);
    const int y0 = ty0 + SH_PX * (int)(threadIdx.x / ST_TILE);
    const int rows = min(SH_PX, G.oy + G.oh - y0);
    if (x >= G.ox + G.ow || rows <= 0) return;
    double center[SH_PX], detail[SH_PX];
#pragma unroll
    for (int p = 0; p < SH_PX; ++p) {
        center[p] = p < rows ? plane[(y0 + p - sy0) * CL_SPAN + (x - sx0)] : 0.0;
        detail[p] = 0.0;
    }
    const bool whole = rows == SH_PX && x - R >= G.ix && x + R < G.ix + G.iw && y0 - R >= G.iy &&
                       y0 + SH_PX - 1 + R < G.iy + G.ih;
    if (whole) {
        constexpr int K = 2 * R + 1;
        double sum[SH_PX];
#pragma unroll
        for (int p = 0; p < SH_PX; ++p) sum[p] = 0.0;
#pragma unroll
        for (int j = 0; j < SH_PX + 2 * R; ++j) {   // row y0 - R + j
            const double* row = plane + (y0 - R + j - sy0) * CL_SPAN + (x - R - sx0);
            double v[K];
#pragma unroll
            for (int k = 0; k < K; ++k) v[k] = row[k];
#pragma unroll
            for (int p = 0; p < SH_PX; ++p) {
                if (j < p || j > p + 2 * R) continue;
#pragma unroll
                for (int k = 0; k < K; ++k) sum[p] = __dadd_rn(sum[p], __dsub_rn(v[k], center[p]));
            }
        }
#pragma unroll
        for (int p = 0; p < SH_PX; ++p)
            if (center[p] > 0.0 && center[p] < 1.0) detail[p] = -__ddiv_rn(sum[p], (double)(K * K));
    } else {
        const int left = max(G.ix, x - R), right = min(G.ix + G.iw - 1, x + R);
        for (int p = 0; p < rows; ++p) {
            if (!(center[p] > 0.0 && center[p] < 1.0)) continue;
            const int y = y0 + p;
            const int top = max(G.iy, y - R), bottom = min(G.iy + G.ih - 1, y + R);
            double sum = 0.0;
            for (int yy = top; yy <= bottom; ++yy)
                for (int xx = left; xx <= right; ++xx)
                    sum = __dadd_rn(sum, __dsub_rn(plane[(yy - sy0) * CL_SPAN + (xx - sx0)], center[p]));
            detail[p] = -__ddiv_rn(sum, (double)((right - left + 1) * (bottom - top + 1)));
        }
    }
#pragma unroll
    for (int p = 0; p < SH_PX; ++p)
        if (p < rows) apply_offset(G, x, y0 + p, center[p], detail[p], amount);
}

// ---------------------------------------------------------------- texture

// Texture renders 32 x 32 output tiles (its halo of 2 * scale, up to 8, costs
// less against a larger tile); each thread owns four pixels of one column.
constexpr int TX_TILE = 32, TX_SPAN = TX_TILE + 2 * ST_MAX_HALO;   // 48
constexpr int TX_THREADS = 256, TX_ROWS = TX_THREADS / 32, TX_PX = TX_TILE / TX_ROWS;

// One axis pass of SpatialOps.cpp:557-587 over the image rectangle
// [x0, x1) x [y0, y1) (smem coordinates relative to sx0, sy0), its cells dealt
// to the threads in row-major order.  The division by the weight is exact
// scaling for weights 2
// and 4 (the correctly rounded product by 1/2 or 1/4 is the correctly rounded
// quotient); weight 3 divides.
__device__ __forceinline__ void texture_axis(const Geo& G, const double* src, double* dst, int x0, int x1, int y0,
                                             int y1, bool vertical, int sx0, int sy0) {
    const int lower = vertical ? G.iy : G.ix, upper = vertical ? G.iy + G.ih : G.ix + G.iw;
    const int step = vertical ? TX_SPAN : 1;
    const int w = x1 - x0, n = w > 0 && y1 > y0 ? w * (y1 - y0) : 0;
    // element i of the rectangle is row i / w, found as the truncated product
    // (i + 1/2) * (1 / w): exact here, since the product's fractional part
    // stays at least 1/(2w) >= 1/96 away from an integer while its rounding
    // error is below n * 2^-23 < 1/3000
    const float inv_w = 1.0f / (float)max(w, 1);
    for (int i = (int)threadIdx.x; i < n; i += TX_THREADS) {
        {
            const int r = __float2int_rz(((float)i + 0.5f) * inv_w);
            const int y = y0 + r, x = x0 + (i - r * w);
            const int k = (y - sy0) * TX_SPAN + (x - sx0), coord = vertical ? y : x;
            const double center = src[k];
            double sum = 0.0;
            unsigned weight = 2;
            if (coord > lower) {
                sum = __dadd_rn(sum, __dsub_rn(src[k - step], center));
                ++weight;
            }
            if (coord + 1 < upper) {
                sum = __dadd_rn(sum, __dsub_rn(src[k + step], center));
                ++weight;
            }
            const double delta = weight == 4 ? __dmul_rn(sum, 0.25)
                                 : weight == 2 ? __dmul_rn(sum, 0.5)
                                               : __ddiv_rn(sum, 3.0);
            dst[k] = delta == 0.0 ? center : __dadd_rn(center, delta);
        }
    }
}

// SpatialOps.cpp:536-620
__global__ void __launch_bounds__(TX_THREADS) texture_kernel(Geo G, double amount, int scale, double wr, double wb) {
    __shared__ double plane[TX_SPAN * TX_SPAN], temp[TX_SPAN * TX_SPAN];
    const int halo = 2 * scale;
    const int tx0 = G.ox + blockIdx.x * TX_TILE, ty0 = G.oy + blockIdx.y * TX_TILE;
    const int tx1 = min(G.ox + G.ow, tx0 + TX_TILE), ty1 = min(G.oy + G.oh, ty0 + TX_TILE);
    const int sx0 = tx0 - halo, sy0 = ty0 - halo;
    stage_y<TX_TILE, TX_SPAN>(G, halo, wr, wb, plane, sx0, sy0);
    __syncthreads();
    // this thread's pixels: column x, rows y0p + TX_ROWS * k
    const int x = tx0 + (int)(threadIdx.x & 31u), y0p = ty0 + (int)(threadIdx.x >> 5);
    double center[TX_PX], fine[TX_PX];
#pragma unroll
    for (int k = 0; k < TX_PX; ++k) {
        const int y = y0p + TX_ROWS * k;
        center[k] = x < tx1 && y < ty1 ? plane[(y - sy0) * TX_SPAN + (x - sx0)] : 0.0;
        fine[k] = 0.0;
    }
    for (int pass = 1; pass <= halo; ++pass) {
        const int r = halo - pass;
        // valid = the tile grown by r; the horizontal pass also covers one row above and below
        const int vx0 = max(G.ix, tx0 - r), vx1 = min(G.ix + G.iw, tx1 + r);
        const int vy0 = max(G.iy, ty0 - r), vy1 = min(G.iy + G.ih, ty1 + r);
        texture_axis(G, plane, temp, vx0, vx1, max(G.iy, vy0 - 1), min(G.iy + G.ih, vy1 + 1), false, sx0, sy0);
        __syncthreads();
        texture_axis(G, temp, plane, vx0, vx1, vy0, vy1, true, sx0, sy0);
        __syncthreads();
        if (pass == scale) {
#pragma unroll
            for (int k = 0; k < TX_PX; ++k) {
                const int y = y0p + TX_ROWS * k;
                if (x < tx1 && y < ty1) fine[k] = plane[(y - sy0) * TX_SPAN + (x - sx0)];
            }
        }
    }
#pragma unroll
    for (int k = 0; k < TX_PX; ++k) {
        const int y = y0p + TX_ROWS * k;
        if (x >= tx1 || y >= ty1) continue;
        const double detail = __dsub_rn(fine[k], plane[(y - sy0) * TX_SPAN + (x - sx0)]);
        apply_offset(G, x, y, center[k], detail, amount);
    }
}

// ------------------------------------------------------------ convolution

constexpr int CONV_MAX = 17;

struct ConvKernel {
    int w, h;
    double k[CONV_MAX * CONV_MAX];
};

// SpatialOps.cpp:354-383
__global__ void __launch_bounds__(ST_TILE* ST_TILE) convolution_kernel(Geo G, const __grid_constant__ ConvKernel K) {
    __shared__ double tile[ST_SPAN * ST_SPAN * 3];
    __shared__ double coef[CONV_MAX * CONV_MAX];
    const int kw = K.w, kh = K.h, hx = kw / 2, hy = kh / 2;
    for (int i = threadIdx.x; i < kw * kh; i += blockDim.x) coef[i] = K.k[i];
    const int sx0 = G.ox + blockIdx.x * ST_TILE - hx, sy0 = G.oy + blockIdx.y * ST_TILE - hy;
    stage_rgb(G, hx, hy, tile, sx0, sy0);
    __syncthreads();
    int x, y;
    if (!my_pixel(G, x, y)) return;
    const int right = G.ix + G.iw - 1, bottom = G.iy + G.ih - 1;
    double sum[3] = {0.0, 0.0, 0.0};
    for (int ky = 0; ky < kh; ++ky) {
        const int yy = min(max(y + hy - ky, G.iy), bottom);
        for (int kx = 0; kx < kw; ++kx) {
            const int xx = min(max(x + hx - kx, G.ix), right);
            const double* s = tile + ((yy - sy0) * ST_SPAN + (xx - sx0)) * 3;
            const double wgt = coef[ky * kw + kx];
#pragma unroll
            for (int c = 0; c < 3; ++c) sum[c] = __dadd_rn(sum[c], __dmul_rn(wgt, s[c]));
        }
    }
    float* o = G.out + (size_t)(y - G.oy) * G.out_stride + (size_t)(x - G.ox) * 3;
    for (int c = 0; c < 3; ++c) o[c] = to_output(G, sum[c]);
}

// SpatialOps.cpp:354-383 for a square KS x KS kernel (3 or 5), on 16 x 64
// output tiles with four vertically adjacent pixels per thread.  Pixel p's
// sum runs over kernel rows ky ascending (image rows descending) and columns
// kx ascending, as in the reference.  Where no tap of the thread's pixels is
// clamped, the thread walks the image rows once from the bottom, holding a
// row's KS samples in registers, and adds w * x to every pixel whose kernel
// reaches that row (the coefficients are compile-time kernel-parameter
// operands); elsewhere each pixel runs the clamped loop.
// Five CTAs per SM (48 registers, a few spilled bytes): 5x5 on 6000x4000
// 0.66 -> 0.51 ms against three CTAs at 72 registers.
template <int KS>
__global__ void __launch_bounds__(ST_TILE* ST_TILE, 5) convolution_square_kernel(Geo G,
                                                                              const __grid_constant__ ConvKernel K) {
    constexpr int H = KS / 2;
    static_assert(H <= SH_MAX_RADIUS, "the staged tile holds a halo of at most 3");
    __shared__ double tile[SH_SPAN * SH_ROWS * 3];
    const int tx0 = G.ox + blockIdx.x * SH_TW, ty0 = G.oy + blockIdx.y * SH_TH;
    const int sx0 = tx0 - H, sy0 = ty0 - H;
    stage_rgb<SH_TW, SH_TH, SH_SPAN>(G, H, H, tile, sx0, sy0);
    __syncthreads();
    const int x = tx0 + (int)(threadIdx.x % ST_TILE);
    const int y0 = ty0 + SH_PX * (int)(threadIdx.x / ST_TILE);
    const int rows = min(SH_PX, G.oy + G.oh - y0);
    if (x >= G.ox + G.ow || rows <= 0) return;
    float* o = G.out + (size_t)(y0 - G.oy) * G.out_stride + (size_t)(x - G.ox) * 3;
    const int right = G.ix + G.iw - 1, bottom = G.iy + G.ih - 1;
    const bool whole = rows == SH_PX && x - H >= G.ix && x + H <= right && y0 - H >= G.iy &&
                       y0 + SH_PX - 1 + H <= bottom;
    if (whole) {
        double sum[SH_PX][3];
#pragma unroll
        for (int p = 0; p < SH_PX; ++p) sum[p][0] = sum[p][1] = sum[p][2] = 0.0;
#pragma unroll
        for (int j = 0; j < SH_PX + 2 * H; ++j) {   // image row y0 + SH_PX - 1 + H - j
            const double* row = tile + ((y0 + SH_PX - 1 + H - j - sy0) * SH_SPAN + (x + H - sx0)) * 3;
            double v[KS][3];
#pragma unroll
            for (int kx = 0; kx < KS; ++kx)
#pragma unroll
                for (int c = 0; c < 3; ++c) v[kx][c] = row[c - 3 * kx];   // column x + H - kx
#pragma unroll
            for (int p = 0; p < SH_PX; ++p) {
                const int ky = j + p - (SH_PX - 1);
                if (ky < 0 || ky >= KS) continue;
#pragma unroll
                for (int kx = 0; kx < KS; ++kx) {
                    const double wgt = K.k[ky * KS + kx];
#pragma unroll
                    for (int c = 0; c < 3; ++c) sum[p][c] = __dadd_rn(sum[p][c], __dmul_rn(wgt, v[kx][c]));
                }
            }
        }
#pragma unroll
        for (int p = 0; p < SH_PX; ++p)
#pragma unroll
            for (int c = 0; c < 3; ++c) o[(size_t)p * G.out_stride + c] = to_output(G, sum[p][c]);
        return;
    }
    for (int p = 0; p < rows; ++p) {
        const int y = y0 + p;
        double sum[3] = {0.0, 0.0, 0.0};
        for (int ky = 0; ky < KS; ++ky) {
            const int yy = min(max(y + H - ky, G.iy), bottom);
            for (int kx = 0; kx < KS; ++kx) {
                const int xx = min(max(x + H - kx, G.ix), right);
                const double* t = tile + ((yy - sy0) * SH_SPAN + (xx - sx0)) * 3;
                const double wgt = K.k[ky * KS + kx];
#pragma unroll
                for (int c = 0; c < 3; ++c) sum[c] = __dadd_rn(sum[c], __dmul_rn(wgt, t[c]));
            }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) o[(size_t)p * G.out_stride + c] = to_output(G, sum[c]);
    }
}

// Input check and copy of the output rectangle (zero amount, identity kernel).
__global__ void check_copy_kernel(Geo G) {
    const size_t n = (size_t)G.ow * G.oh * 3;
    bool bad = false;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % 3);
        const size_t p = i / 3;
        const int x = G.ox + (int)(p % G.ow), y = G.oy + (int)(p / G.ow);
        const float v = G.in[(size_t)(y - G.wy) * G.in_stride + (size_t)(x - G.wx) * 3 + c];
        bad |= !isfinite(v);
        G.out[(size_t)(y - G.oy) * G.out_stride + (size_t)(x - G.ox) * 3 + c] = v;
    }
    if (bad) flag(G.status, KEY_INPUT);
}

// ------------------------------------------------------------------ host

struct Op {
    const char* name;
    const char* input_message;
    const char* output_message;
};
constexpr Op kSharpen{"sharpen", "sharpen requires finite complete RGB halo",
                      "sharpen output exceeds finite float32 range"};
constexpr Op kClarity{"clarity", "clarity requires finite complete input halo",
                      "clarity output exceeds finite float32 range"};
constexpr Op kTexture{"texture", "texture requires finite complete input halo",
                      "texture output exceeds finite float32 range"};
constexpr Op kConvolution{"convolution", "convolution requires finite input samples",
                          "convolution output exceeds finite float32 range"};

re_status st_fail(re_status s, const std::string& msg) {
    set_last_error(msg);
    return s;
}

bool inside(re_rect outer, re_rect r) {
    return r.x >= outer.x && r.y >= outer.y && (uint64_t)r.x + r.width <= (uint64_t)outer.x + outer.width &&
           (uint64_t)r.y + r.height <= (uint64_t)outer.y + outer.height;
}

re_rect grown(re_rect r, re_rect image, uint32_t hx, uint32_t hy) {
    const int64_t left = std::max<int64_t>(image.x, (int64_t)r.x - hx), top = std::max<int64_t>(image.y, (int64_t)r.y - hy);
    const uint64_t right = std::min<uint64_t>((uint64_t)image.x + image.width, (uint64_t)r.x + r.width + hx);
    const uint64_t bottom = std::min<uint64_t>((uint64_t)image.y + image.height, (uint64_t)r.y + r.height + hy);
    return {(uint32_t)left, (uint32_t)top, (uint32_t)(right - left), (uint32_t)(bottom - top)};
}

// Validates the geometry, fills G, launches `launch(G, halo_x, halo_y)`
// (or the check-and-copy kernel for halo (0, 0) when `copy` is set),
// waits, and maps the status word to the reference's message.
template <class F>
re_status run_stencil(const Op& op, const float* in, size_t in_stride, re_rect window, re_rect image, re_rect output,
                      uint32_t hx, uint32_t hy, bool copy, float* out, size_t out_stride, void* stream_, F&& launch) {
    if (!in || !out) return st_fail(RE_INVALID_ARGUMENT, std::string(op.name) + ": null image");
    const uint64_t limit = 1ull << 30;   // int coordinates with room for the halo
    if (!image.width || !image.height || (uint64_t)image.x + image.width > limit ||
        (uint64_t)image.y + image.height > limit)
        return st_fail(RE_INVALID_ARGUMENT, "spatial operation requires nonempty addressable bounds");
    if (!output.width || !output.height)
        return st_fail(RE_INVALID_ARGUMENT, "spatial operation requires nonempty addressable bounds");
    if (!inside(image, output)) return st_fail(RE_OUT_OF_RANGE, "spatial viewport is outside image bounds");
    if ((output.height + ST_TILE - 1) / ST_TILE > 65535)
        return st_fail(RE_LENGTH_ERROR, std::string(op.name) + ": output taller than 1048560 rows");
    const re_rect needed = grown(output, image, hx, hy);
    if (!inside(image, window) || !inside(window, needed))
        return st_fail(RE_INVALID_ARGUMENT, std::string(op.name) + ": input window does not cover the output halo");
    if (in_stride < (size_t)window.width * 3 || out_stride < (size_t)output.width * 3)
        return st_fail(RE_INVALID_ARGUMENT, std::string(op.name) + ": row stride too small");
    cudaStream_t s = (cudaStream_t)stream_;
    void* scratch = nullptr;
    cudaError_t e = scratch_alloc(&scratch, 256, s);
    if (e != cudaSuccess) return st_fail(RE_CUDA_ERROR, std::string(op.name) + ": " + cudaGetErrorString(e));
    Geo G;
    G.in = in;
    G.in_stride = in_stride;
    G.wx = (int)window.x;
    G.wy = (int)window.y;
    G.ww = (int)window.width;
    G.wh = (int)window.height;
    G.ix = (int)image.x;
    G.iy = (int)image.y;
    G.iw = (int)image.width;
    G.ih = (int)image.height;
    G.ox = (int)output.x;
    G.oy = (int)output.y;
    G.ow = (int)output.width;
    G.oh = (int)output.height;
    G.out = out;
    G.out_stride = out_stride;
    G.status = static_cast<uint32_t*>(scratch);
    e = cudaMemsetAsync(scratch, 0, 4, s);
    if (e == cudaSuccess) {
        if (copy) {
            const size_t n = (size_t)output.width * output.height * 3;
            check_copy_kernel<<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 16), 256, 0, s>>>(G);
        } else {
            launch(G, dim3((output.width + ST_TILE - 1) / ST_TILE, (output.height + ST_TILE - 1) / ST_TILE));
        }
        e = cudaGetLastError();
    }
    uint32_t key = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&key, scratch, 4, cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(scratch, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return st_fail(RE_CUDA_ERROR, std::string(op.name) + ": " + cudaGetErrorString(e));
    if (key == KEY_INPUT) return st_fail(RE_INVALID_ARGUMENT, op.input_message);
    if (key == KEY_OUTPUT) return st_fail(RE_INVALID_ARGUMENT, op.output_message);
    if (key) return st_fail(RE_INVALID_ARGUMENT, std::string(op.name) + ": device status " + std::to_string(key));
    return RE_OK;
}

void y_weights(uint32_t space, double& wr, double& wb) {
    if (space == 0) {
        wr = 0.28807112822929337;
        wb = 0.00008565396060525903;
    } else {
        wr = 0.26270021201126703;
        wb = 0.059301716469861945;
    }
}

}  // namespace

extern "C" {

re_status re_sharpen_window(const float* in, size_t in_stride, re_rect window, re_rect image, re_rect output,
                            double amount, uint32_t radius, float* out, size_t out_stride, void* stream) {
    if (!std::isfinite(amount) || amount < 0 || amount > 2 || radius < 1 || radius > 3)
        return st_fail(RE_INVALID_ARGUMENT, "sharpen requires finite amount 0..2 and radius 1..3");
    const uint32_t h = amount == 0 ? 0 : radius;
    return run_stencil(kSharpen, in, in_stride, window, image, output, h, h, amount == 0, out, out_stride, stream,
                       [&](const Geo& G, dim3 grid) {
                           const dim3 tiles((G.ow + SH_TW - 1) / SH_TW, (G.oh + SH_TH - 1) / SH_TH);
                           (void)grid;
                           auto kernel = radius == 1 ? sharpen_kernel<1> : radius == 2 ? sharpen_kernel<2> : sharpen_kernel<3>;
                           kernel<<<tiles, ST_TILE * ST_TILE, 0, (cudaStream_t)stream>>>(G, amount);
                       });
}

re_status re_clarity_window(const float* in, size_t in_stride, re_rect window, re_rect image, re_rect output,
                            double amount, uint32_t radius, uint32_t working_space, float* out, size_t out_stride,
                            void* stream) {
    if (!std::isfinite(amount) || std::abs(amount) > 1 || radius < 1 || radius > 8)
        return st_fail(RE_INVALID_ARGUMENT, "clarity requires finite amount [-1,1] and radius 1..8");
    if (working_space > 1) return st_fail(RE_INVALID_ARGUMENT, "clarity requires scene-linear working RGB");
    double wr, wb;
    y_weights(working_space, wr, wb);
    const uint32_t h = amount == 0 ? 0 : radius;
    return run_stencil(kClarity, in, in_stride, window, image, output, h, h, amount == 0, out, out_stride, stream,
                       [&](const Geo& G, dim3 grid) {
                           const dim3 tiles((G.ow + SH_TW - 1) / SH_TW, (G.oh + SH_TH - 1) / SH_TH);
                           (void)grid;
                           void (*const kernels[])(Geo, double, double, double) = {
                               clarity_kernel<1>, clarity_kernel<2>, clarity_kernel<3>, clarity_kernel<4>,
                               clarity_kernel<5>, clarity_kernel<6>, clarity_kernel<7>, clarity_kernel<8>};
                           kernels[radius - 1]<<<tiles, ST_TILE * ST_TILE, 0, (cudaStream_t)stream>>>(G, amount, wr, wb);
                       });
}

re_status re_texture_window(const float* in, size_t in_stride, re_rect window, re_rect image, re_rect output,
                            double amount, uint32_t scale, uint32_t working_space, float* out, size_t out_stride,
                            void* stream) {
    if (!std::isfinite(amount) || std::abs(amount) > 1 || scale < 1 || scale > 4)
        return st_fail(RE_INVALID_ARGUMENT, "texture requires finite amount [-1,1] and scale 1..4");
    if (working_space > 1) return st_fail(RE_INVALID_ARGUMENT, "texture requires scene-linear working RGB");
    double wr, wb;
    y_weights(working_space, wr, wb);
    const uint32_t h = amount == 0 ? 0 : 2 * scale;
    return run_stencil(kTexture, in, in_stride, window, image, output, h, h, amount == 0, out, out_stride, stream,
                       [&](const Geo& G, dim3 grid) {
                           const dim3 tiles((G.ow + TX_TILE - 1) / TX_TILE, (G.oh + TX_TILE - 1) / TX_TILE);
                           (void)grid;
                           texture_kernel<<<tiles, TX_THREADS, 0, (cudaStream_t)stream>>>(G, amount, (int)scale, wr, wb);
                       });
}

re_status re_convolution_window(const float* in, size_t in_stride, re_rect window, re_rect image, re_rect output,
                                uint32_t kernel_width, uint32_t kernel_height, const double* coefficients,
                                float* out, size_t out_stride, void* stream) {
    if (!kernel_width || !kernel_height || kernel_width > 17 || kernel_height > 17 || kernel_width % 2 != 1 ||
        kernel_height % 2 != 1 || !coefficients)
        return st_fail(RE_INVALID_ARGUMENT, "convolution kernel needs odd dimensions 1..17 and matching coefficients");
    const size_t taps = (size_t)kernel_width * kernel_height;
    bool identity = true;
    for (size_t i = 0; i < taps; ++i) {
        if (!std::isfinite(coefficients[i]) || std::abs(coefficients[i]) > 65536)
            return st_fail(RE_INVALID_ARGUMENT, "convolution coefficients must be finite with magnitude <=65536");
        if (coefficients[i] != (i == taps / 2 ? 1.0 : 0.0)) identity = false;
    }
    ConvKernel K{};
    K.w = (int)kernel_width;
    K.h = (int)kernel_height;
    std::copy(coefficients, coefficients + taps, K.k);
    return run_stencil(kConvolution, in, in_stride, window, image, output, identity ? 0 : kernel_width / 2,
                       identity ? 0 : kernel_height / 2, identity, out, out_stride, stream,
                       [&](const Geo& G, dim3 grid) {
                           const dim3 tiles((G.ow + SH_TW - 1) / SH_TW, (G.oh + SH_TH - 1) / SH_TH);
                           if (K.w == K.h && K.w == 3)
                               convolution_square_kernel<3><<<tiles, ST_TILE * ST_TILE, 0, (cudaStream_t)stream>>>(G, K);
                           else if (K.w == K.h && K.w == 5)
                               convolution_square_kernel<5><<<tiles, ST_TILE * ST_TILE, 0, (cudaStream_t)stream>>>(G, K);
                           else
                               convolution_kernel<<<grid, ST_TILE * ST_TILE, 0, (cudaStream_t)stream>>>(G, K);
                       });
}

}  // extern "C"
