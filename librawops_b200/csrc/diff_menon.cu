// Differentiable Menon demosaic with directions frozen from the forward pass
// (MenonDemosaic.cpp:97-173).
//
// Forward, over a whole normalized sensor plane with mirrored borders
// (MenonDemosaic.cpp:60-71), in binary64 in the reference's order:
//   directional greens gh, gv and chroma ch, cv at non-green sites;
//   forward gradients dh = |ch - ch(x+2)|, dv = |cv - cv(y+2)|;
//   the classifier (eight weighted gradient terms, zero outside the frame)
//   picks horizontal where v >= h; green = gh or gv (the sample at green
//   sites); red and blue at green sites = (green + mean(raw)) - mean(green)
//   along the neighbouring colour's axis; the opposite colour at red and blue
//   sites = (own + mean(other)) - mean(own) along the chosen direction.
// The direction map is returned.  With it held fixed every step is linear in
// the samples, so the backward is the exact transpose, taken in three
// gathers: each output site collects from the sites whose (mirrored) taps
// land on it, so no atomics are needed, and mirror folds at the borders fall
// out of comparing tap indices.  Planes live in binary64 scratch from the
// library's pool; the direction map (one byte per site) is the caller's.
#include <cmath>
#include <string>

#include "re_device.cuh"

namespace re {
void set_last_error(const std::string& msg);
}  // namespace re

using namespace re;

namespace {

constexpr int MT = 256;

__device__ __forceinline__ int colour_at(uint32_t quad, int x, int y) {
    return (int)((quad >> (2 * (((y & 1) << 1) | (x & 1)))) & 3u);
}

// MenonDemosaic.cpp:60-66
__device__ __forceinline__ int mirror(int i, int n) {
    if (n == 1) return 0;
    const int period = 2 * (n - 1);
    int f = i % period;
    if (f < 0) f += period;
    return f < n ? f : period - f;
}

struct MenonGeom {
    int w, h;
    uint32_t quad;
    size_t n;   // w * h
};

__device__ __forceinline__ size_t idx(const MenonGeom& g, int x, int y) { return (size_t)y * g.w + x; }

// ------------------------------------------------------------------ forward

// gh, gv, ch, cv (MenonDemosaic.cpp:107-121).
__global__ void __launch_bounds__(MT) menon_f1(const float* __restrict__ s, size_t ss, MenonGeom g,
                                               double* __restrict__ GH, double* __restrict__ GV,
                                               double* __restrict__ CH, double* __restrict__ CV) {
    const size_t i = blockIdx.x * (size_t)MT + threadIdx.x;
    if (i >= g.n) return;
    const int x = (int)(i % g.w), y = (int)(i / g.w);
    const double own = s[(size_t)y * ss + x];
    if (colour_at(g.quad, x, y) == 1) {
        GH[i] = GV[i] = own;
        CH[i] = CV[i] = 0.0;
        return;
    }
    auto S = [&](int xx, int yy) { return (double)s[(size_t)mirror(yy, g.h) * ss + mirror(xx, g.w)]; };
    const double hh = __dsub_rn(__dadd_rn(__dmul_rn(0.5, __dadd_rn(S(x - 1, y), S(x + 1, y))), __dmul_rn(0.5, own)),
                                __dmul_rn(0.25, __dadd_rn(S(x - 2, y), S(x + 2, y))));
    const double vv = __dsub_rn(__dadd_rn(__dmul_rn(0.5, __dadd_rn(S(x, y - 1), S(x, y + 1))), __dmul_rn(0.5, own)),
                                __dmul_rn(0.25, __dadd_rn(S(x, y - 2), S(x, y + 2))));
    GH[i] = hh;
    GV[i] = vv;
    CH[i] = __dsub_rn(own, hh);
    CV[i] = __dsub_rn(own, vv);
}

// dh, dv (MenonDemosaic.cpp:122-127).
__global__ void __launch_bounds__(MT) menon_f2(MenonGeom g, const double* __restrict__ CH,
                                               const double* __restrict__ CV, double* __restrict__ DH,
                                               double* __restrict__ DV) {
    const size_t i = blockIdx.x * (size_t)MT + threadIdx.x;
    if (i >= g.n) return;
    const int x = (int)(i % g.w), y = (int)(i / g.w);
    DH[i] = fabs(__dsub_rn(CH[i], CH[idx(g, mirror(x + 2, g.w), y)]));
    DV[i] = fabs(__dsub_rn(CV[i], CV[idx(g, x, mirror(y + 2, g.h))]));
}

// Classifier and green (MenonDemosaic.cpp:128-147); gradients are zero outside the frame.
__global__ void __launch_bounds__(MT) menon_f3(const float* __restrict__ s, size_t ss, MenonGeom g,
                                               const double* __restrict__ GH, const double* __restrict__ GV,
                                               const double* __restrict__ DH, const double* __restrict__ DV,
                                               double* __restrict__ GREEN, uint8_t* __restrict__ dirs) {
    const size_t i = blockIdx.x * (size_t)MT + threadIdx.x;
    if (i >= g.n) return;
    const int x = (int)(i % g.w), y = (int)(i / g.w);
    if (colour_at(g.quad, x, y) == 1) {
        dirs[i] = 1;
        GREEN[i] = (double)s[(size_t)y * ss + x];
        return;
    }
    constexpr int tx[8] = {0, -2, -1, 0, -2, -1, 0, -2}, ty[8] = {2, 2, 1, 0, 0, -1, -2, -2};
    constexpr double tw[8] = {1, 1, 1, 3, 3, 1, 1, 1};
    double hs = 0, vs = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int hx = x + tx[k], hy = y + ty[k], vx = x + ty[k], vy = y + tx[k];
        const double gh = (hx >= 0 && hx < g.w && hy >= 0 && hy < g.h) ? DH[idx(g, hx, hy)] : 0.0;
        const double gv = (vx >= 0 && vx < g.w && vy >= 0 && vy < g.h) ? DV[idx(g, vx, vy)] : 0.0;
        hs = __dadd_rn(hs, __dmul_rn(tw[k], gh));
        vs = __dadd_rn(vs, __dmul_rn(tw[k], gv));
    }
    const bool horizontal = vs >= hs;
    dirs[i] = horizontal ? 1 : 0;
    GREEN[i] = horizontal ? GH[i] : GV[i];
}

__device__ __forceinline__ double mean_along(const double* p, const MenonGeom& g, int x, int y, bool horiz) {
    const double a = horiz ? p[idx(g, mirror(x - 1, g.w), y)] : p[idx(g, x, mirror(y - 1, g.h))];
    const double b = horiz ? p[idx(g, mirror(x + 1, g.w), y)] : p[idx(g, x, mirror(y + 1, g.h))];
    return __dmul_rn(0.5, __dadd_rn(a, b));
}
__device__ __forceinline__ double mean_raw(const float* s, size_t ss, const MenonGeom& g, int x, int y, bool horiz) {
    const double a = horiz ? s[(size_t)y * ss + mirror(x - 1, g.w)] : s[(size_t)mirror(y - 1, g.h) * ss + x];
    const double b = horiz ? s[(size_t)y * ss + mirror(x + 1, g.w)] : s[(size_t)mirror(y + 1, g.h) * ss + x];
    return __dmul_rn(0.5, __dadd_rn(a, b));
}

// Red and blue at every site (MenonDemosaic.cpp:151-161).
__global__ void __launch_bounds__(MT) menon_f4(const float* __restrict__ s, size_t ss, MenonGeom g,
                                               const double* __restrict__ GREEN, double* __restrict__ RED,
                                               double* __restrict__ BLUE) {
    const size_t i = blockIdx.x * (size_t)MT + threadIdx.x;
    if (i >= g.n) return;
    const int x = (int)(i % g.w), y = (int)(i / g.w);
    const int own = colour_at(g.quad, x, y);
    const double v = s[(size_t)y * ss + x];
    double r = 0.0, b = 0.0;
    if (own == 0) r = v;
    if (own == 2) b = v;
    if (own == 1) {
        const bool red_h = colour_at(g.quad, x + 1, y) == 0;
        r = __dsub_rn(__dadd_rn(GREEN[i], mean_raw(s, ss, g, x, y, red_h)), mean_along(GREEN, g, x, y, red_h));
        b = __dsub_rn(__dadd_rn(GREEN[i], mean_raw(s, ss, g, x, y, !red_h)), mean_along(GREEN, g, x, y, !red_h));
    }
    RED[i] = r;
    BLUE[i] = b;
}

// Output pixels (MenonDemosaic.cpp:162-172).
__global__ void __launch_bounds__(MT) menon_f5(MenonGeom g, const double* __restrict__ GREEN,
                                               const double* __restrict__ RED, const double* __restrict__ BLUE,
                                               const uint8_t* __restrict__ dirs, float* __restrict__ rgb) {
    const size_t i = blockIdx.x * (size_t)MT + threadIdx.x;
    if (i >= g.n) return;
    const int x = (int)(i % g.w), y = (int)(i / g.w);
    const int own = colour_at(g.quad, x, y);
    const bool horiz = dirs[i] != 0;
    double rr = RED[i], bb = BLUE[i];
    if (own == 2) rr = __dsub_rn(__dadd_rn(bb, mean_along(RED, g, x, y, horiz)), mean_along(BLUE, g, x, y, horiz));
    if (own == 0) bb = __dsub_rn(__dadd_rn(rr, mean_along(BLUE, g, x, y, horiz)), mean_along(RED, g, x, y, horiz));
    rgb[i * 3 + 0] = (float)rr;
    rgb[i * 3 + 1] = (float)GREEN[i];
    rgb[i * 3 + 2] = (float)bb;
}

// ------------------------------------------------------------------ backward

// How many of site (x, y)'s two mirrored taps along `horiz` land on (tx, ty).
__device__ __forceinline__ int taps_on(const MenonGeom& g, int x, int y, bool horiz, int tx, int ty) {
    if (horiz) {
        if (y != ty) return 0;
        return (mirror(x - 1, g.w) == tx) + (mirror(x + 1, g.w) == tx);
    }
    if (x != tx) return 0;
    return (mirror(y - 1, g.h) == ty) + (mirror(y + 1, g.h) == ty);
}

// Candidate sites whose radius-1 taps can reach (x, y): itself and its four neighbours.
constexpr int NB1 = 5;
__device__ __forceinline__ bool candidate1(const MenonGeom& g, int x, int y, int k, int& cx, int& cy) {
    constexpr int ox[NB1] = {0, -1, 1, 0, 0}, oy[NB1] = {0, 0, 0, -1, 1};
    cx = x + ox[k];
    cy = y + oy[k];
    return cx >= 0 && cx < g.w && cy >= 0 && cy < g.h;
}

// Final step transposed: dred, dblue, dgreen from the output gradient.
__global__ void __launch_bounds__(MT) menon_b1(MenonGeom g, const float* __restrict__ dout,
                                               const uint8_t* __restrict__ dirs, double* __restrict__ DRED,
                                               double* __restrict__ DBLUE, double* __restrict__ DGREEN) {
    const size_t i = blockIdx.x * (size_t)MT + threadIdx.x;
    if (i >= g.n) return;
    const int x = (int)(i % g.w), y = (int)(i / g.w);
    const int own = colour_at(g.quad, x, y);
    const double dR = dout[i * 3], dG = dout[i * 3 + 1], dB = dout[i * 3 + 2];
    double dr = (own != 2 ? dR : 0.0) + (own == 0 ? dB : 0.0);
    double db = (own != 0 ? dB : 0.0) + (own == 2 ? dR : 0.0);
    for (int k = 0; k < NB1; ++k) {
        int cx, cy;
        if (!candidate1(g, x, y, k, cx, cy)) continue;
        const int oc = colour_at(g.quad, cx, cy);
        if (oc == 1) continue;
        const size_t j = idx(g, cx, cy);
        const double dd = oc == 2 ? (double)dout[j * 3] : -(double)dout[j * 3 + 2];
        const int n = taps_on(g, cx, cy, dirs[j] != 0, x, y);
        if (n) {
            dr += 0.5 * n * dd;
            db -= 0.5 * n * dd;
        }
    }
    DRED[i] = dr;
    DBLUE[i] = db;
    DGREEN[i] = dG;
}

// Red and blue at green sites transposed: the sample gradient so far and dgreen.
__global__ void __launch_bounds__(MT) menon_b2(MenonGeom g, const double* __restrict__ DRED,
                                               const double* __restrict__ DBLUE, double* __restrict__ DGREEN,
                                               double* __restrict__ DS) {
    const size_t i = blockIdx.x * (size_t)MT + threadIdx.x;
    if (i >= g.n) return;
    const int x = (int)(i % g.w), y = (int)(i / g.w);
    const int own = colour_at(g.quad, x, y);
    double ds = (own == 0 ? DRED[i] : 0.0) + (own == 2 ? DBLUE[i] : 0.0);
    double dg = DGREEN[i] + (own == 1 ? DRED[i] + DBLUE[i] : 0.0);
    for (int k = 0; k < NB1; ++k) {
        int cx, cy;
        if (!candidate1(g, x, y, k, cx, cy)) continue;
        if (colour_at(g.quad, cx, cy) != 1) continue;
        const size_t j = idx(g, cx, cy);
        const bool red_h = colour_at(g.quad, cx + 1, cy) == 0;
        const double t = 0.5 * taps_on(g, cx, cy, red_h, x, y) * DRED[j] +
                         0.5 * taps_on(g, cx, cy, !red_h, x, y) * DBLUE[j];
        ds += t;
        dg -= t;
    }
    DS[i] = ds;
    DGREEN[i] = dg;   // each thread rewrites only its own entry after reading others' DRED/DBLUE
}

// Green transposed: green sites take dgreen; gh/gv taps (0.5 own, 0.5 at +-1,
// -0.25 at +-2, mirrored) gather from the non-green sites within 2.
__global__ void __launch_bounds__(MT) menon_b3(MenonGeom g, const double* __restrict__ DGREEN,
                                               const double* __restrict__ DS, const uint8_t* __restrict__ dirs,
                                               float* __restrict__ dp, size_t dps) {
    const size_t i = blockIdx.x * (size_t)MT + threadIdx.x;
    if (i >= g.n) return;
    const int x = (int)(i % g.w), y = (int)(i / g.w);
    double ds = DS[i] + (colour_at(g.quad, x, y) == 1 ? DGREEN[i] : 0.0);
    for (int axis = 0; axis < 2; ++axis) {
        for (int o = -2; o <= 2; ++o) {
            const int cx = axis == 0 ? x + o : x, cy = axis == 0 ? y : y + o;
            if (cx < 0 || cx >= g.w || cy < 0 || cy >= g.h) continue;
            if (colour_at(g.quad, cx, cy) == 1) continue;
            const size_t j = idx(g, cx, cy);
            if ((dirs[j] != 0) != (axis == 0)) continue;
            const double gj = DGREEN[j];
            double wsum = o == 0 ? 0.5 : 0.0;
            for (int t = -2; t <= 2; ++t) {
                if (!t) continue;
                const int m = axis == 0 ? mirror(cx + t, g.w) : mirror(cy + t, g.h);
                if (m == (axis == 0 ? x : y)) wsum += (t == 1 || t == -1) ? 0.5 : -0.25;
            }
            ds += wsum * gj;
        }
    }
    dp[(size_t)y * dps + x] = (float)ds;
}

struct Pool {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~Pool() {
        if (p) cudaFreeAsync(p, s);
    }
};

re_status fail(re_status st, const char* msg) {
    set_last_error(msg);
    return st;
}

#define DM_CUDA(call)                                                              \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_));    \
            return RE_CUDA_ERROR;                                                  \
        }                                                                          \
    } while (0)

}  // namespace

extern "C" {

re_status re_diff_menon_forward(const float* plane, size_t plane_stride, uint32_t w, uint32_t h, uint32_t quad,
                                float* rgb, uint8_t* directions, void* stream_) {
    if (!plane || !rgb || !directions || !w || !h || plane_stride < w)
        return fail(RE_INVALID_ARGUMENT, "bad demosaic arguments");
    cudaStream_t s = (cudaStream_t)stream_;
    const MenonGeom g{(int)w, (int)h, quad, (size_t)w * h};
    Pool sc;
    sc.s = s;
    DM_CUDA(scratch_alloc(&sc.p, 9 * g.n * sizeof(double), s));
    double* base = (double*)sc.p;
    double *GH = base, *GV = GH + g.n, *CH = GV + g.n, *CV = CH + g.n, *DH = CV + g.n, *DV = DH + g.n;
    double *GREEN = DV + g.n, *RED = GREEN + g.n, *BLUE = RED + g.n;
    const unsigned blocks = (unsigned)((g.n + MT - 1) / MT);
    menon_f1<<<blocks, MT, 0, s>>>(plane, plane_stride, g, GH, GV, CH, CV);
    menon_f2<<<blocks, MT, 0, s>>>(g, CH, CV, DH, DV);
    menon_f3<<<blocks, MT, 0, s>>>(plane, plane_stride, g, GH, GV, DH, DV, GREEN, directions);
    menon_f4<<<blocks, MT, 0, s>>>(plane, plane_stride, g, GREEN, RED, BLUE);
    menon_f5<<<blocks, MT, 0, s>>>(g, GREEN, RED, BLUE, directions, rgb);
    DM_CUDA(cudaGetLastError());
    return RE_OK;
}

re_status re_diff_menon_backward(const float* drgb, uint32_t w, uint32_t h, uint32_t quad, const uint8_t* directions,
                                 float* dplane, size_t dplane_stride, void* stream_) {
    if (!drgb || !dplane || !directions || !w || !h || dplane_stride < w)
        return fail(RE_INVALID_ARGUMENT, "bad demosaic arguments");
    cudaStream_t s = (cudaStream_t)stream_;
    const MenonGeom g{(int)w, (int)h, quad, (size_t)w * h};
    Pool sc;
    sc.s = s;
    DM_CUDA(scratch_alloc(&sc.p, 4 * g.n * sizeof(double), s));
    double* base = (double*)sc.p;
    double *DRED = base, *DBLUE = DRED + g.n, *DGREEN = DBLUE + g.n, *DS = DGREEN + g.n;
    const unsigned blocks = (unsigned)((g.n + MT - 1) / MT);
    menon_b1<<<blocks, MT, 0, s>>>(g, drgb, directions, DRED, DBLUE, DGREEN);
    menon_b2<<<blocks, MT, 0, s>>>(g, DRED, DBLUE, DGREEN, DS);
    menon_b3<<<blocks, MT, 0, s>>>(g, DGREEN, DS, directions, dplane, dplane_stride);
    DM_CUDA(cudaGetLastError());
    return RE_OK;
}

}  // extern "C"
