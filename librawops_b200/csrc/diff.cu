// Differentiable render: forward kernels and their hand-written adjoints.
//
// The forward model restates the render path's arithmetic with the recipe as
// parameters (the reference computes no gradients):
//   bilinear demosaic of the normalized sensor plane (RawEngine.cpp:299-344)
//   -> white balance (RawEngine.cpp:417-431) -> exposure multiplier
//   (RawEngine.cpp:488-500) -> 3x3 matrix (RawEngine.cpp:539-545) -> the master
//   curve of ExtendedCurvesNode, shape-preserving cubic (ToneOps.cpp:795-844)
//   -> detail boost v + k (v - GF(v)) with the self-guided working-Y guided
//   filter (SpatialOps.cpp:168-287).
// Images are contiguous float32 (h, w, 3); the sensor plane is (h, w) over the
// active area with the CFA quad's colours given relative to its origin.
//
// Adjoints.  Demosaic: the transpose of the averaging stencil as a gather
// (each site collects dout/count from the 3x3 pixels that averaged it).  Point
// stages: each pixel's forward is recomputed; parameter gradients are reduced
// per block in double (curve gradients per segment in shared memory) and
// added to a caller-zeroed double vector.  Guided filter: the box adjoint is a
// box sum of g/N (windows are symmetric), and every mean the backward needs is
// recomputed from the input instead of being saved by the forward.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "re_device.cuh"

namespace re {
void set_last_error(const std::string& msg);
}  // namespace re

using namespace re;

namespace {

#define DF_CUDA(call)                                                                                    \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) {                                                                         \
            set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_));                          \
            return RE_CUDA_ERROR;                                                                        \
        }                                                                                                \
    } while (0)

re_status df_fail(re_status s, const char* msg) {
    set_last_error(msg);
    return s;
}

// ------------------------------------------------------------------ demosaic

__device__ __forceinline__ int quad_colour(uint32_t quad, int x, int y) {
    return (int)((quad >> (2 * (((y & 1) << 1) | (x & 1)))) & 3u);
}

__global__ void bilinear_fwd_kernel(const float* __restrict__ s, size_t ss, int w, int h, uint32_t quad,
                                    float* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int own = quad_colour(quad, x, y);
    float sum[3] = {0, 0, 0};
    int cnt[3] = {0, 0, 0};
    for (int dy = -1; dy <= 1; ++dy) {
        const int yy = y + dy;
        if (yy < 0 || yy >= h) continue;
        for (int dx = -1; dx <= 1; ++dx) {
            const int xx = x + dx;
            if (xx < 0 || xx >= w) continue;
            const int c = quad_colour(quad, xx, yy);
            sum[c] += s[(size_t)yy * ss + xx];
            ++cnt[c];
        }
    }
    float* o = out + ((size_t)y * w + x) * 3;
    for (int c = 0; c < 3; ++c)
        o[c] = c == own ? s[(size_t)y * ss + x] : (cnt[c] ? sum[c] / (float)cnt[c] : 0.0f);
}

__device__ __forceinline__ int colour_count(uint32_t quad, int x, int y, int w, int h, int c) {
    int n = 0;
    for (int dy = -1; dy <= 1; ++dy) {
        const int yy = y + dy;
        if (yy < 0 || yy >= h) continue;
        for (int dx = -1; dx <= 1; ++dx) {
            const int xx = x + dx;
            if (xx >= 0 && xx < w && quad_colour(quad, xx, yy) == c) ++n;
        }
    }
    return n;
}

__global__ void bilinear_bwd_kernel(const float* __restrict__ dout, int w, int h, uint32_t quad,
                                    float* __restrict__ ds, size_t dss) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int c = quad_colour(quad, x, y);
    float g = dout[((size_t)y * w + x) * 3 + c];
    for (int dy = -1; dy <= 1; ++dy) {
        const int yy = y + dy;
        if (yy < 0 || yy >= h) continue;
        for (int dx = -1; dx <= 1; ++dx) {
            const int xx = x + dx;
            if (xx < 0 || xx >= w || (dx == 0 && dy == 0)) continue;
            if (quad_colour(quad, xx, yy) == c) continue;   // that pixel's channel c is its own sample
            g += dout[((size_t)yy * w + xx) * 3 + c] / (float)colour_count(quad, xx, yy, w, h, c);
        }
    }
    ds[(size_t)y * dss + x] = g;
}

// ------------------------------------------------------------- point stages

constexpr int PT_THREADS = 256, MAX_KNOTS = 256;

struct PointParams {
    const float* scalars;          // device: wb[3], e, m[9], s_first, s_last
    int n;                         // knots (0: no curve)
    const float *kx, *ky, *c0, *c1;
};

// The point-stage constants, read once per block from device memory.
struct PointScalars {
    float wb[3], e, m[9], s_first, s_last;
};
static_assert(sizeof(PointScalars) == 15 * sizeof(float), "scalar block layout");

struct CurveSmem {
    float kx[MAX_KNOTS], ky[MAX_KNOTS], c0[MAX_KNOTS], c1[MAX_KNOTS];
};

__device__ __forceinline__ void load_scalars(PointScalars& K, const PointParams& P) {
    if (threadIdx.x < 15) reinterpret_cast<float*>(&K)[threadIdx.x] = P.scalars[threadIdx.x];
}

__device__ __forceinline__ void load_curve(CurveSmem& C, const PointParams& P) {
    for (int i = threadIdx.x; i < P.n; i += blockDim.x) {
        C.kx[i] = P.kx[i];
        C.ky[i] = P.ky[i];
        if (i + 1 < P.n) {
            C.c0[i] = P.c0[i];
            C.c1[i] = P.c1[i];
        }
    }
}

// Segment of v: largest i with kx[i] <= v, clamped to [0, n-2].
__device__ __forceinline__ int segment(const CurveSmem& C, int n, float v) {
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (C.kx[mid] <= v) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ float curve_eval(const CurveSmem& C, const PointScalars& K, int n, float v,
                                            float* dvdx) {
    if (v < C.kx[0]) {
        *dvdx = K.s_first;
        return C.ky[0] + (v - C.kx[0]) * K.s_first;
    }
    if (v > C.kx[n - 1]) {
        *dvdx = K.s_last;
        return C.ky[n - 1] + (v - C.kx[n - 1]) * K.s_last;
    }
    const int i = segment(C, n, v);
    const float h = C.kx[i + 1] - C.kx[i];
    const float t = (v - C.kx[i]) / h, u = 1.0f - t;
    const float y0 = C.ky[i], a = C.c0[i], b = C.c1[i], y1 = C.ky[i + 1];
    *dvdx = 3.0f * (u * u * (a - y0) + 2.0f * u * t * (b - a) + t * t * (y1 - b)) / h;
    return u * u * u * y0 + 3.0f * u * u * t * a + 3.0f * u * t * t * b + t * t * t * y1;
}

__global__ void __launch_bounds__(PT_THREADS) point_fwd_kernel(const float* __restrict__ x, size_t count,
                                                               const PointParams P, float* __restrict__ y) {
    __shared__ CurveSmem C;
    __shared__ PointScalars K;
    load_curve(C, P);
    load_scalars(K, P);
    __syncthreads();
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        float z[3];
        for (int c = 0; c < 3; ++c) z[c] = x[i * 3 + c] * K.wb[c] * K.e;
        for (int r = 0; r < 3; ++r) {
            float v = K.m[3 * r] * z[0] + K.m[3 * r + 1] * z[1] + K.m[3 * r + 2] * z[2];
            if (P.n) {
                float d;
                v = curve_eval(C, K, P.n, v, &d);
            }
            y[i * 3 + r] = v;
        }
    }
}

// grads layout: [wb 3 | e 1 | m 9 | ky n | c0 n-1 | c1 n-1 | s_first | s_last]
struct CurveGradSmem {
    double ky[MAX_KNOTS], c0[MAX_KNOTS], c1[MAX_KNOTS], s[2];
};

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(PT_THREADS) point_bwd_kernel(const float* __restrict__ x,
                                                               const float* __restrict__ dy, size_t count,
                                                               const PointParams P, float* __restrict__ dx,
                                                               double* __restrict__ grads) {
    __shared__ CurveSmem C;
    __shared__ CurveGradSmem G;
    __shared__ double red[PT_THREADS / 32][13];
    __shared__ PointScalars K;
    load_curve(C, P);
    load_scalars(K, P);
    for (int i = threadIdx.x; i < MAX_KNOTS; i += blockDim.x) G.ky[i] = G.c0[i] = G.c1[i] = 0.0;
    if (threadIdx.x < 2) G.s[threadIdx.x] = 0.0;
    __syncthreads();
    double acc[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int n = P.n;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        float xs[3], t1[3], z[3], g[3];
        for (int c = 0; c < 3; ++c) {
            xs[c] = x[i * 3 + c];
            t1[c] = xs[c] * K.wb[c];
            z[c] = t1[c] * K.e;
        }
        for (int r = 0; r < 3; ++r) {
            const float v = K.m[3 * r] * z[0] + K.m[3 * r + 1] * z[1] + K.m[3 * r + 2] * z[2];
            const float go = dy[i * 3 + r];
            float d = 1.0f;
            if (n) {
                // this sample's contributions to the curve gradients: key -1
                // (left extrapolation: ky[0], s_first), -2 (right: ky[n-1],
                // s_last) or the segment k (ky[k], ky[k+1], c0[k], c1[k])
                int key;
                double w0, w1, w2 = 0.0, w3 = 0.0;
                if (v < C.kx[0]) {
                    d = K.s_first;
                    key = -1;
                    w0 = (double)go;
                    w1 = (double)go * (double)(v - C.kx[0]);
                } else if (v > C.kx[n - 1]) {
                    d = K.s_last;
                    key = -2;
                    w0 = (double)go;
                    w1 = (double)go * (double)(v - C.kx[n - 1]);
                } else {
                    const int k = segment(C, n, v);
                    const float h = C.kx[k + 1] - C.kx[k];
                    const float t = (v - C.kx[k]) / h, u = 1.0f - t;
                    const float y0 = C.ky[k], a = C.c0[k], b = C.c1[k], y1 = C.ky[k + 1];
                    d = 3.0f * (u * u * (a - y0) + 2.0f * u * t * (b - a) + t * t * (y1 - b)) / h;
                    key = k;
                    w0 = (double)(go * u * u * u);
                    w1 = (double)(go * t * t * t);
                    w2 = (double)(go * 3.0f * u * u * t);
                    w3 = (double)(go * 3.0f * u * t * t);
                }
                // Lanes of a warp mostly share a few keys: each group of equal
                // keys sums its contributions by shuffles and its first lane
                // adds them to shared memory, instead of one atomic per lane.
                const unsigned group = __match_any_sync(__activemask(), key);
                double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                for (unsigned m = group; m; m &= m - 1) {
                    const int src = __ffs(m) - 1;
                    s0 += __shfl_sync(group, w0, src);
                    s1 += __shfl_sync(group, w1, src);
                    s2 += __shfl_sync(group, w2, src);
                    s3 += __shfl_sync(group, w3, src);
                }
                if ((threadIdx.x & 31) == __ffs(group) - 1) {
                    if (key == -1) {
                        atomicAdd(&G.ky[0], s0);
                        atomicAdd(&G.s[0], s1);
                    } else if (key == -2) {
                        atomicAdd(&G.ky[n - 1], s0);
                        atomicAdd(&G.s[1], s1);
                    } else {
                        atomicAdd(&G.ky[key], s0);
                        atomicAdd(&G.ky[key + 1], s1);
                        atomicAdd(&G.c0[key], s2);
                        atomicAdd(&G.c1[key], s3);
                    }
                }
            }
            g[r] = go * d;
            for (int c = 0; c < 3; ++c) acc[4 + 3 * r + c] += (double)g[r] * (double)z[c];
        }
        float dz[3];
        for (int c = 0; c < 3; ++c) dz[c] = K.m[c] * g[0] + K.m[3 + c] * g[1] + K.m[6 + c] * g[2];
        for (int c = 0; c < 3; ++c) {
            acc[3] += (double)dz[c] * (double)t1[c];
            const float dt1 = dz[c] * K.e;
            acc[c] += (double)dt1 * (double)xs[c];
            dx[i * 3 + c] = dt1 * K.wb[c];
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < 13; ++k) {
        const double v = warp_sum(acc[k]);
        if (lane == 0) red[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < 13) {
        double v = 0;
        for (int wi = 0; wi < PT_THREADS / 32; ++wi) v += red[wi][threadIdx.x];
        atomicAdd(&grads[threadIdx.x], v);
    }
    if (n) {
        double* gk = grads + 13;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            if (G.ky[i] != 0.0) atomicAdd(&gk[i], G.ky[i]);
            if (i + 1 < n) {
                if (G.c0[i] != 0.0) atomicAdd(&gk[n + i], G.c0[i]);
                if (G.c1[i] != 0.0) atomicAdd(&gk[2 * n - 1 + i], G.c1[i]);
            }
        }
        if (threadIdx.x < 2 && G.s[threadIdx.x] != 0.0) atomicAdd(&gk[3 * n - 2 + threadIdx.x], G.s[threadIdx.x]);
    }
}

// ------------------------------------------------------------ guided filter

struct GfGeom {
    int w, h, r;
    size_t plane;   // elements per plane (w * h)
};

__device__ __forceinline__ double count_at(const GfGeom& g, int x, int y) {
    const int nx = min(x + g.r, g.w - 1) - max(x - g.r, 0) + 1;
    const int ny = min(y + g.r, g.h - 1) - max(y - g.r, 0) + 1;
    return (double)(nx * ny);
}

constexpr int BOX_CHUNK = 64;

// out[p][y][x] = sum of in[p][y][x-r..x+r] clipped.  One CTA per (plane, row,
// segment of BOX_SEG columns): the segment and its halo are staged in shared
// memory with coalesced loads; each thread then slides a window over
// BOX_RUN consecutive outputs (one full window sum, then one entering and one
// leaving sample per step).  Entry i of the staged row sits at i + i / BOX_RUN,
// so the threads' stride-BOX_RUN reads fall in distinct banks.
constexpr int BOX_THREADS = 256, BOX_RUN = 8, BOX_SEG = BOX_THREADS * BOX_RUN, BOX_MAX_R = 64;
constexpr int BOX_STAGE = BOX_SEG + 2 * BOX_MAX_R;
__device__ __forceinline__ int box_slot(int i) { return i + i / BOX_RUN; }
__global__ void __launch_bounds__(BOX_THREADS) box_rows_kernel(const double* __restrict__ in, double* __restrict__ out,
                                                               GfGeom g, int planes) {
    __shared__ double seg[BOX_STAGE + BOX_STAGE / BOX_RUN + 1];
    const int x0 = blockIdx.x * BOX_SEG, y = blockIdx.y, p = blockIdx.z;
    const double* row = in + p * g.plane + (size_t)y * g.w;
    const int n = BOX_SEG + 2 * g.r;
    for (int i = threadIdx.x; i < n; i += BOX_THREADS) {
        const int x = x0 - g.r + i;
        seg[box_slot(i)] = (x >= 0 && x < g.w) ? row[x] : 0.0;
    }
    __syncthreads();
    const int i0 = (int)threadIdx.x * BOX_RUN;   // first output of this thread, relative to x0
    if (x0 + i0 >= g.w) return;
    double s = 0;
    for (int j = 0; j <= 2 * g.r; ++j) s += seg[box_slot(i0 + j)];
    double* o = out + p * g.plane + (size_t)y * g.w + x0 + i0;
    o[0] = s;
#pragma unroll
    for (int k = 1; k < BOX_RUN; ++k) {
        if (x0 + i0 + k >= g.w) break;
        s += seg[box_slot(i0 + k + 2 * g.r)];
        s -= seg[box_slot(i0 + k - 1)];
        o[k] = s;
    }
}

// out[p][y][x] = sum of in[p][y-r..y+r][x] clipped; one thread per (plane,
// column, chunk of rows), a sliding sum down the chunk.  The rows entering and
// leaving the window are fetched BOX_STEP at a time before any is added, so a
// thread keeps that many loads in flight; the additions run in the order of a
// row-by-row slide.
constexpr int BOX_STEP = 8;
__global__ void box_cols_kernel(const double* __restrict__ in, double* __restrict__ out, GfGeom g, int planes) {
    const int chunks = (g.h + BOX_CHUNK - 1) / BOX_CHUNK;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int chunk = blockIdx.y;
    const int p = blockIdx.z;
    if (x >= g.w || chunk >= chunks || p >= planes) return;
    const double* col = in + p * g.plane + x;
    double* ocol = out + p * g.plane + x;
    const int y0 = chunk * BOX_CHUNK, y1 = min(y0 + BOX_CHUNK, g.h);
    double s = 0;
    for (int j = max(0, y0 - g.r); j <= min(g.h - 1, y0 + g.r); ++j) s += col[(size_t)j * g.w];
    for (int y = y0; y < y1; y += BOX_STEP) {
        double add[BOX_STEP], sub[BOX_STEP];
#pragma unroll
        for (int k = 0; k < BOX_STEP; ++k) {
            const int a = y + k + 1 + g.r, b = y + k - g.r;
            add[k] = (y + k < y1 && a < g.h) ? col[(size_t)a * g.w] : 0.0;
            sub[k] = (y + k < y1 && b >= 0) ? col[(size_t)b * g.w] : 0.0;
        }
#pragma unroll
        for (int k = 0; k < BOX_STEP; ++k) {
            if (y + k >= y1) break;
            ocol[(size_t)(y + k) * g.w] = s;
            if (y + k + 1 + g.r < g.h) s += add[k];
            if (y + k - g.r >= 0) s -= sub[k];
        }
    }
}

struct YW {
    double wr, wb;
};

__device__ __forceinline__ double guide_of(const float* p, YW w) {
    const double r = p[0], g = p[1], b = p[2];
    return (g + w.wr * (r - g)) + w.wb * (b - g);
}

// planes: I, I^2, p0, p1, p2, I p0, I p1, I p2
__global__ void gf_prep_kernel(const float* __restrict__ p, GfGeom g, YW w, double* __restrict__ P8) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= g.plane) return;
    const float* px = p + i * 3;
    const double I = guide_of(px, w);
    P8[i] = I;
    P8[g.plane + i] = I * I;
    for (int c = 0; c < 3; ++c) {
        P8[(2 + c) * g.plane + i] = px[c];
        P8[(5 + c) * g.plane + i] = I * px[c];
    }
}

struct Moments {
    double mI, mII, mp[3], mIp[3], var, cov[3], a[3], b[3];
};

__device__ __forceinline__ Moments moments_at(const double* __restrict__ S8, const GfGeom& g, size_t i, double n,
                                              double eps) {
    Moments M;
    M.mI = S8[i] / n;
    M.mII = S8[g.plane + i] / n;
    M.var = M.mII - M.mI * M.mI;
    for (int c = 0; c < 3; ++c) {
        M.mp[c] = S8[(2 + c) * g.plane + i] / n;
        M.mIp[c] = S8[(5 + c) * g.plane + i] / n;
        M.cov[c] = M.mIp[c] - M.mI * M.mp[c];
        M.a[c] = M.cov[c] / (M.var + eps);
        M.b[c] = M.mp[c] - M.a[c] * M.mI;
    }
    return M;
}

// planes a0, a1, a2, b0, b1, b2
__global__ void gf_coef_kernel(const double* __restrict__ S8, GfGeom g, double eps, double* __restrict__ AB) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= g.plane) return;
    const int x = (int)(i % g.w), y = (int)(i / g.w);
    const Moments M = moments_at(S8, g, i, count_at(g, x, y), eps);
    for (int c = 0; c < 3; ++c) {
        AB[c * g.plane + i] = M.a[c];
        AB[(3 + c) * g.plane + i] = M.b[c];
    }
}

__global__ void gf_out_kernel(const float* __restrict__ p, const double* __restrict__ SAB, GfGeom g, YW w,
                              const float* __restrict__ kp, float* __restrict__ out) {
    const float k = *kp;
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= g.plane) return;
    const int x = (int)(i % g.w), y = (int)(i / g.w);
    const double n = count_at(g, x, y);
    const float* px = p + i * 3;
    const double I = guide_of(px, w);
    for (int c = 0; c < 3; ++c) {
        const double q = SAB[c * g.plane + i] / n * I + SAB[(3 + c) * g.plane + i] / n;
        out[i * 3 + c] = (float)(px[c] + (double)k * (px[c] - q));
    }
}

// Backward step 1: planes dq I / N and dq / N; dk partial sums.
__global__ void gf_bwd1_kernel(const float* __restrict__ p, const float* __restrict__ dout,
                               const double* __restrict__ SAB, GfGeom g, YW w, const float* __restrict__ kp,
                               double* __restrict__ G6, double* __restrict__ dk) {
    __shared__ double red[8];
    const float k = *kp;
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    double part = 0;
    if (i < g.plane) {
        const int x = (int)(i % g.w), y = (int)(i / g.w);
        const double n = count_at(g, x, y);
        const float* px = p + i * 3;
        const double I = guide_of(px, w);
        for (int c = 0; c < 3; ++c) {
            const double q = SAB[c * g.plane + i] / n * I + SAB[(3 + c) * g.plane + i] / n;
            const double d = dout[i * 3 + c];
            part += (px[c] - q) * d;
            const double dq = -(double)k * d;
            G6[c * g.plane + i] = dq * I / n;
            G6[(3 + c) * g.plane + i] = dq / n;
        }
    }
    part = warp_sum(part);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int j = 0; j < (int)(blockDim.x >> 5); ++j) s += red[j];
        atomicAdd(dk, s);
    }
}

// Backward step 2: from the box sums of step 1 (da, db) to the adjoints of
// the eight moment means, divided by N for the next box adjoint.  epsilon
// enters every centre only through var + eps, so its adjoint is the sum over
// centres of the variance adjoint; each CTA adds its part to *deps.
__device__ __forceinline__ double gf_bwd2_centre(const double* __restrict__ S8, const double* __restrict__ DAB,
                                                 const GfGeom& g, double eps, size_t i, double* __restrict__ H8) {
    const int x = (int)(i % g.w), y = (int)(i / g.w);
    const double n = count_at(g, x, y);
    const Moments M = moments_at(S8, g, i, n, eps);
    const double inv = 1.0 / (M.var + eps);
    double dmI = 0, dvar = 0;
    for (int c = 0; c < 3; ++c) {
        const double da = DAB[c * g.plane + i], db = DAB[(3 + c) * g.plane + i];
        double dmp = db;
        const double dA = da - db * M.mI;
        dmI -= db * M.a[c];
        const double dcov = dA * inv;
        dvar -= dA * M.cov[c] * inv * inv;
        dmI -= dcov * M.mp[c];
        dmp -= dcov * M.mI;
        H8[(2 + c) * g.plane + i] = dmp / n;
        H8[(5 + c) * g.plane + i] = dcov / n;
    }
    dmI -= 2.0 * M.mI * dvar;
    H8[i] = dmI / n;
    H8[g.plane + i] = dvar / n;
    return dvar;
}

__global__ void gf_bwd2_kernel(const double* __restrict__ S8, const double* __restrict__ DAB, GfGeom g, double eps,
                               double* __restrict__ H8, double* __restrict__ deps) {
    __shared__ double red[8];
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    double part = i < g.plane ? gf_bwd2_centre(S8, DAB, g, eps, i, H8) : 0.0;
    part = warp_sum(part);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int j = 0; j < (int)(blockDim.x >> 5); ++j) s += red[j];
        atomicAdd(deps, s);
    }
}

__global__ void gf_bwd3_kernel(const float* __restrict__ p, const float* __restrict__ dout,
                               const double* __restrict__ SAB, const double* __restrict__ B8, GfGeom g, YW w,
                               const float* __restrict__ kp, float* __restrict__ dp) {
    const float k = *kp;
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= g.plane) return;
    const int x = (int)(i % g.w), y = (int)(i / g.w);
    const double n = count_at(g, x, y);
    const float* px = p + i * 3;
    const double I = guide_of(px, w);
    double dI = B8[i] + 2.0 * I * B8[g.plane + i];
    double d[3];
    for (int c = 0; c < 3; ++c) {
        const double go = dout[i * 3 + c];
        const double ma = SAB[c * g.plane + i] / n;
        dI += ma * (-(double)k * go);
        const double bip = B8[(5 + c) * g.plane + i];
        dI += px[c] * bip;
        d[c] = (1.0 + (double)k) * go + B8[(2 + c) * g.plane + i] + I * bip;
    }
    const double wg = 1.0 - w.wr - w.wb;
    dp[i * 3 + 0] = (float)(d[0] + dI * w.wr);
    dp[i * 3 + 1] = (float)(d[1] + dI * wg);
    dp[i * 3 + 2] = (float)(d[2] + dI * w.wb);
}

YW weights(uint32_t space) {
    return space == 0 ? YW{0.28807112822929337, 0.00008565396060525903}
                      : YW{0.26270021201126703, 0.059301716469861945};
}

void box(const double* in, double* tmp, double* out, const GfGeom& g, int planes, cudaStream_t s) {
    box_rows_kernel<<<dim3((g.w + BOX_SEG - 1) / BOX_SEG, g.h, planes), BOX_THREADS, 0, s>>>(in, tmp, g, planes);
    dim3 grid((g.w + 127) / 128, (g.h + BOX_CHUNK - 1) / BOX_CHUNK, planes);
    box_cols_kernel<<<grid, 128, 0, s>>>(tmp, out, g, planes);
}

struct DScratch {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~DScratch() {
        if (p) cudaFreeAsync(p, s);
    }
};

re_status gf_check(uint32_t w, uint32_t h, uint32_t radius, double eps, uint32_t space) {
    if (!w || !h) return df_fail(RE_INVALID_ARGUMENT, "detail boost needs a nonempty image");
    if (h > 65535) return df_fail(RE_LENGTH_ERROR, "detail boost supports at most 65535 rows");
    if (radius > 64 || !(eps >= 0x1p-24) || !(eps <= 65536.0))
        return df_fail(RE_INVALID_ARGUMENT, "detail boost needs radius 0..64 and finite epsilon [2^-24,65536]");
    if (space > 1) return df_fail(RE_INVALID_ARGUMENT, "detail boost needs a scene-linear working space");
    return RE_OK;
}

// Forward passes shared by forward and backward: S8 = box moments, SAB = box(a, b).
void gf_forward_planes(const float* p, const GfGeom& g, YW w, double eps, double* S8, double* T8, double* AB,
                       double* SAB, cudaStream_t s) {
    const unsigned blocks = (unsigned)((g.plane + 255) / 256);
    gf_prep_kernel<<<blocks, 256, 0, s>>>(p, g, w, AB);          // AB holds the 8 prepared planes here
    box(AB, T8, S8, g, 8, s);
    gf_coef_kernel<<<blocks, 256, 0, s>>>(S8, g, eps, AB);
    box(AB, T8, SAB, g, 6, s);
}

}  // namespace

extern "C" {

re_status re_diff_bilinear_forward(const float* s, size_t s_stride, uint32_t w, uint32_t h, uint32_t quad,
                                   float* rgb, void* stream) {
    if (!s || !rgb || !w || !h || s_stride < w) return df_fail(RE_INVALID_ARGUMENT, "bad demosaic arguments");
    dim3 block(32, 8), grid((w + 31) / 32, (h + 7) / 8);
    bilinear_fwd_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(s, s_stride, (int)w, (int)h, quad, rgb);
    DF_CUDA(cudaGetLastError());
    return RE_OK;
}

re_status re_diff_bilinear_backward(const float* drgb, uint32_t w, uint32_t h, uint32_t quad, float* ds,
                                    size_t ds_stride, void* stream) {
    if (!drgb || !ds || !w || !h || ds_stride < w) return df_fail(RE_INVALID_ARGUMENT, "bad demosaic arguments");
    dim3 block(32, 8), grid((w + 31) / 32, (h + 7) / 8);
    bilinear_bwd_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(drgb, (int)w, (int)h, quad, ds, ds_stride);
    DF_CUDA(cudaGetLastError());
    return RE_OK;
}

static re_status point_params(const re_diff_point_params* in, PointParams& P) {
    if (!in || !in->scalars) return df_fail(RE_INVALID_ARGUMENT, "null point parameters");
    if (in->knots == 1 || in->knots > MAX_KNOTS) return df_fail(RE_INVALID_ARGUMENT, "curve needs 2..256 knots");
    if (in->knots && (!in->kx || !in->ky || !in->c0 || !in->c1))
        return df_fail(RE_INVALID_ARGUMENT, "curve arrays are null");
    P.scalars = in->scalars;
    P.n = (int)in->knots;
    P.kx = in->kx;
    P.ky = in->ky;
    P.c0 = in->c0;
    P.c1 = in->c1;
    return RE_OK;
}

static unsigned point_blocks(size_t count) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (unsigned)std::max<size_t>(1, std::min<size_t>((count + PT_THREADS - 1) / PT_THREADS, (size_t)sms * 4));
}

re_status re_diff_point_forward(const float* x, size_t count, const re_diff_point_params* params, float* y,
                                void* stream) {
    PointParams P;
    re_status st = point_params(params, P);
    if (st) return st;
    if (!count) return RE_OK;
    if (!x || !y) return df_fail(RE_INVALID_ARGUMENT, "null image");
    point_fwd_kernel<<<point_blocks(count), PT_THREADS, 0, (cudaStream_t)stream>>>(x, count, P, y);
    DF_CUDA(cudaGetLastError());
    return RE_OK;
}

re_status re_diff_point_backward(const float* x, const float* dy, size_t count, const re_diff_point_params* params,
                                 float* dx, double* grads, void* stream) {
    PointParams P;
    re_status st = point_params(params, P);
    if (st) return st;
    if (!count) return RE_OK;
    if (!x || !dy || !dx || !grads) return df_fail(RE_INVALID_ARGUMENT, "null image or gradient");
    point_bwd_kernel<<<point_blocks(count), PT_THREADS, 0, (cudaStream_t)stream>>>(x, dy, count, P, dx, grads);
    DF_CUDA(cudaGetLastError());
    return RE_OK;
}

size_t re_diff_point_grad_count(uint32_t knots) { return 13 + (knots ? 3 * (size_t)knots : 0); }

re_status re_diff_detail_forward(const float* p, uint32_t w, uint32_t h, uint32_t radius, double eps,
                                 const float* strength, uint32_t space, float* out, void* stream_) {
    re_status st = gf_check(w, h, radius, eps, space);
    if (st) return st;
    if (!p || !out || !strength) return df_fail(RE_INVALID_ARGUMENT, "null image or strength");
    cudaStream_t s = (cudaStream_t)stream_;
    const GfGeom g{(int)w, (int)h, (int)radius, (size_t)w * h};
    DScratch sc;
    sc.s = s;
    DF_CUDA(scratch_alloc(&sc.p, (8 + 8 + 8 + 6) * g.plane * sizeof(double), s));
    double* S8 = (double*)sc.p;
    double* T8 = S8 + 8 * g.plane;
    double* AB = T8 + 8 * g.plane;
    double* SAB = AB + 8 * g.plane;
    const YW yw = weights(space);
    gf_forward_planes(p, g, yw, eps, S8, T8, AB, SAB, s);
    gf_out_kernel<<<(unsigned)((g.plane + 255) / 256), 256, 0, s>>>(p, SAB, g, yw, strength, out);
    DF_CUDA(cudaGetLastError());
    return RE_OK;
}

re_status re_diff_detail_backward(const float* p, const float* dout, uint32_t w, uint32_t h, uint32_t radius,
                                  double eps, const float* strength, uint32_t space, float* dp, double* dstrength,
                                  double* depsilon, void* stream_) {
    re_status st = gf_check(w, h, radius, eps, space);
    if (st) return st;
    if (!p || !dout || !dp || !dstrength || !depsilon || !strength)
        return df_fail(RE_INVALID_ARGUMENT, "null image, strength or gradient");
    cudaStream_t s = (cudaStream_t)stream_;
    const GfGeom g{(int)w, (int)h, (int)radius, (size_t)w * h};
    DScratch sc;
    sc.s = s;
    DF_CUDA(scratch_alloc(&sc.p, (8 + 8 + 8 + 6 + 8) * g.plane * sizeof(double), s));
    double* S8 = (double*)sc.p;
    double* T8 = S8 + 8 * g.plane;
    double* W8 = T8 + 8 * g.plane;      // prepared planes, then a/b, then step-1 and step-2 planes
    double* SAB = W8 + 8 * g.plane;
    double* B8 = SAB + 6 * g.plane;     // box sums of the adjoint planes
    const YW yw = weights(space);
    const unsigned blocks = (unsigned)((g.plane + 255) / 256);
    gf_forward_planes(p, g, yw, eps, S8, T8, W8, SAB, s);       // the means, recomputed
    gf_bwd1_kernel<<<blocks, 256, 0, s>>>(p, dout, SAB, g, yw, strength, W8, dstrength);
    box(W8, T8, B8, g, 6, s);                                   // da, db
    gf_bwd2_kernel<<<blocks, 256, 0, s>>>(S8, B8, g, eps, W8, depsilon);
    box(W8, T8, B8, g, 8, s);
    gf_bwd3_kernel<<<blocks, 256, 0, s>>>(p, dout, SAB, B8, g, yw, strength, dp);
    DF_CUDA(cudaGetLastError());
    return RE_OK;
}

}  // extern "C"
