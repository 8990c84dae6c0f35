// Spatial stages: the working-Y guided filter (SpatialOps.cpp:159-317) and
// box local statistics (SpatialOps.cpp:52-157).
//
// Guided filter.  The reference evaluates, per coefficient centre k, centred
// moments over its clipped (2r+1)^2 window and then, per output pixel x,
// p(x) + mean_k[(p_k - p_x) + meanP_delta(k) + a(k)(Y_x - Y_k - meanY_delta(k))]
// in binary64 (O(r^2) per pixel).  Expanding the sum gives the classical form
//     q(x) = mean_{k in W(x)} a(k) * Y(x) + mean_{k in W(x)} b(k),
//     a(k) = cov(Y, p)/(var(Y) + eps),  b(k) = mean(p) - a(k) mean(Y),
// with clipped windows and actual counts, which box filters evaluate in O(1)
// per pixel independent of r.  The first box filter accumulates the eight
// moments (Y, R, G, B, Y^2, YR, YG, YB) in binary64 (so E[Y^2]-E[Y]^2 keeps
// ~1e-16 relative precision against eps >= 2^-24); a and b stay binary64 through
// the second box filter, since a*Y and b can cancel when eps is small.  Output equals p(x) exactly when
// the correction is zero (constants, signed zeros), as in SpatialOps.cpp:278.
//
// Local statistics.  Per channel, the finite count, mean and population
// variance over the clipped window.  Each CTA shifts its samples by one of its
// own values before summing (x - s, (x - s)^2 in binary64), so windows far
// from zero (the reference's 1e20 offset test) keep their precision; the
// reference's Welford/merge order is not reproduced, the result agrees within
// float32 rounding of the outputs.
#include <cfloat>
#include <cmath>
#include <string>

#include "re_device.cuh"

namespace re {
void set_last_error(const std::string& msg);
}

using namespace re;

namespace {

constexpr int GF_CHUNK = 32;  // pixels per thread along the sliding direction

// Working-Y weights of SpatialOps.cpp:191-192.
struct YWeights {
    double wr, wb;
};

__device__ __forceinline__ double working_y(double r, double g, double b, const YWeights& w) {
    return __dadd_rn(__dadd_rn(g, __dmul_rn(w.wr, __dsub_rn(r, g))), __dmul_rn(w.wb, __dsub_rn(b, g)));
}

__device__ __forceinline__ void moments(const float* p, const YWeights& w, double m[8]) {
    const double r = p[0], g = p[1], b = p[2];
    const double y = working_y(r, g, b, w);
    m[0] = y; m[1] = r; m[2] = g; m[3] = b;
    m[4] = y * y; m[5] = y * r; m[6] = y * g; m[7] = y * b;
}

// Horizontal box sums of the eight moments: one thread slides along GF_CHUNK
// pixels of a row.  H: (height, width, 8) doubles.
__global__ void gf_hbox_moments(const float* __restrict__ in, size_t in_stride, int width, int height, int r,
                                YWeights w, double* __restrict__ H, uint32_t* status) {
    const int row = blockIdx.y;
    const int x0 = (blockIdx.x * blockDim.x + threadIdx.x) * GF_CHUNK;
    if (x0 >= width || row >= height) return;
    const float* src = in + (size_t)row * in_stride;
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0}, m[8];
    bool bad = false;
    const int lo0 = max(0, x0 - r), hi0 = min(width - 1, x0 + r);
    for (int j = lo0; j <= hi0; ++j) {
        const float* p = src + (size_t)j * 3;
        bad |= !(isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]));
        moments(p, w, m);
#pragma unroll
        for (int q = 0; q < 8; ++q) s[q] += m[q];
    }
    const int x1 = min(width, x0 + GF_CHUNK);
    for (int x = x0; x < x1; ++x) {
        if (x > x0) {
            const int enter = x + r, leave = x - r - 1;
            if (enter < width) {
                const float* p = src + (size_t)enter * 3;
                bad |= !(isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]));
                moments(p, w, m);
#pragma unroll
                for (int q = 0; q < 8; ++q) s[q] += m[q];
            }
            if (leave >= 0) {
                moments(src + (size_t)leave * 3, w, m);
#pragma unroll
                for (int q = 0; q < 8; ++q) s[q] -= m[q];
            }
        }
        double* h = H + ((size_t)row * width + x) * 8;
#pragma unroll
        for (int q = 0; q < 8; ++q) h[q] = s[q];
    }
    if (bad && status) atomicMax(status, (uint32_t)((401u << 8) | ST_INVALID));
}

// Vertical box sums of H, then the per-centre regression a, b (float AB: 6 per px).
__global__ void gf_vbox_coefficients(const double* __restrict__ H, int width, int height, int r, double eps,
                                     double* __restrict__ AB, uint32_t* status) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y0 = blockIdx.y * GF_CHUNK;
    if (x >= width || y0 >= height) return;
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int lo0 = max(0, y0 - r), hi0 = min(height - 1, y0 + r);
    for (int j = lo0; j <= hi0; ++j) {
        const double* h = H + ((size_t)j * width + x) * 8;
#pragma unroll
        for (int q = 0; q < 8; ++q) s[q] += h[q];
    }
    const int wx = min(width - 1, x + r) - max(0, x - r) + 1;
    const int y1 = min(height, y0 + GF_CHUNK);
    bool overflow = false;
    for (int y = y0; y < y1; ++y) {
        if (y > y0) {
            const int enter = y + r, leave = y - r - 1;
            if (enter < height) {
                const double* h = H + ((size_t)enter * width + x) * 8;
#pragma unroll
                for (int q = 0; q < 8; ++q) s[q] += h[q];
            }
            if (leave >= 0) {
                const double* h = H + ((size_t)leave * width + x) * 8;
#pragma unroll
                for (int q = 0; q < 8; ++q) s[q] -= h[q];
            }
        }
        const int wy = min(height - 1, y + r) - max(0, y - r) + 1;
        const double n = (double)wx * (double)wy;
        const double my = s[0] / n;
        double var = s[4] / n - my * my;
        if (var < 0) var = 0;
        const double inv = 1.0 / (var + eps);
        double* ab = AB + ((size_t)y * width + x) * 6;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double mp = s[1 + c] / n;
            const double cov = s[5 + c] / n - my * mp;
            const double a = cov * inv;
            const double b = mp - a * my;
            overflow |= !(isfinite(a) && isfinite(b));
            ab[c] = a;
            ab[3 + c] = b;
        }
    }
    if (overflow && status) atomicMax(status, (uint32_t)((400u << 8) | ST_OVERFLOW));
}

// Horizontal box sums of AB.
__global__ void gf_hbox_ab(const double* __restrict__ AB, int width, int height, int r, double* __restrict__ H2) {
    const int row = blockIdx.y;
    const int x0 = (blockIdx.x * blockDim.x + threadIdx.x) * GF_CHUNK;
    if (x0 >= width || row >= height) return;
    const double* src = AB + (size_t)row * width * 6;
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int j = max(0, x0 - r); j <= min(width - 1, x0 + r); ++j)
#pragma unroll
        for (int q = 0; q < 6; ++q) s[q] += src[(size_t)j * 6 + q];
    const int x1 = min(width, x0 + GF_CHUNK);
    for (int x = x0; x < x1; ++x) {
        if (x > x0) {
            const int enter = x + r, leave = x - r - 1;
            if (enter < width)
#pragma unroll
                for (int q = 0; q < 6; ++q) s[q] += src[(size_t)enter * 6 + q];
            if (leave >= 0)
#pragma unroll
                for (int q = 0; q < 6; ++q) s[q] -= src[(size_t)leave * 6 + q];
        }
        double* h = H2 + ((size_t)row * width + x) * 6;
#pragma unroll
        for (int q = 0; q < 6; ++q) h[q] = s[q];
    }
}

// Vertical box sums of H2 and the output q = mean(a) Y + mean(b).
__global__ void gf_vbox_output(const double* __restrict__ H2, const float* __restrict__ in, size_t in_stride,
                               int width, int height, int r, YWeights w, float* __restrict__ out,
                               size_t out_stride, uint32_t* status) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y0 = blockIdx.y * GF_CHUNK;
    if (x >= width || y0 >= height) return;
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int j = max(0, y0 - r); j <= min(height - 1, y0 + r); ++j)
#pragma unroll
        for (int q = 0; q < 6; ++q) s[q] += H2[((size_t)j * width + x) * 6 + q];
    const int wx = min(width - 1, x + r) - max(0, x - r) + 1;
    const int y1 = min(height, y0 + GF_CHUNK);
    bool overflow = false;
    for (int y = y0; y < y1; ++y) {
        if (y > y0) {
            const int enter = y + r, leave = y - r - 1;
            if (enter < height)
#pragma unroll
                for (int q = 0; q < 6; ++q) s[q] += H2[((size_t)enter * width + x) * 6 + q];
            if (leave >= 0)
#pragma unroll
                for (int q = 0; q < 6; ++q) s[q] -= H2[((size_t)leave * width + x) * 6 + q];
        }
        const int wy = min(height - 1, y + r) - max(0, y - r) + 1;
        const double n = (double)wx * (double)wy;
        const float* p = in + (size_t)y * in_stride + (size_t)x * 3;
        const double Y = working_y(p[0], p[1], p[2], w);
        float* o = out + (size_t)y * out_stride + (size_t)x * 3;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double q = (s[c] / n) * Y + s[3 + c] / n;
            const double delta = q - (double)p[c];
            if (delta == 0) {
                o[c] = p[c];
                continue;
            }
            if (!isfinite(q) || fabs(q) > (double)FLT_MAX) overflow = true;
            o[c] = (float)q;
        }
    }
    if (overflow && status) atomicMax(status, (uint32_t)((400u << 8) | ST_OVERFLOW));
}

// ----------------------------------------------------------- local statistics

constexpr int LS_TW = 32, LS_TH = 16, LS_THREADS = 256, LS_MAX_R = 32;

struct LsSmem {
    double s1[LS_TH + 2 * LS_MAX_R][LS_TW];
    double s2[LS_TH + 2 * LS_MAX_R][LS_TW];
    int n[LS_TH + 2 * LS_MAX_R][LS_TW];
};

// T = float (re_local_statistics) or double (re_local_statistics_f64, the
// reference's LocalStatisticsTile precision).
template <typename T>
__global__ void __launch_bounds__(LS_THREADS)
local_stats_kernel(const float* __restrict__ in, size_t in_stride, int width, int height, int r,
                   T* __restrict__ mean_out, T* __restrict__ var_out, uint32_t* __restrict__ count_out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    LsSmem& S = *reinterpret_cast<LsSmem*>(smem_raw);
    const int x0 = blockIdx.x * LS_TW, y0 = blockIdx.y * LS_TH;
    const int rows_lo = max(0, y0 - r), rows_hi = min(height - 1, y0 + LS_TH - 1 + r);
    const int nrows = rows_hi - rows_lo + 1;
    for (int c = 0; c < 3; ++c) {
        // the CTA's shift: its first in-image sample of this channel (0 if not finite)
        float sh = in[(size_t)y0 * in_stride + (size_t)x0 * 3 + c];
        const double shift = isfinite(sh) ? (double)sh : 0.0;
        // horizontal window moments for every needed row and output column
        for (int i = threadIdx.x; i < nrows * LS_TW; i += LS_THREADS) {
            const int tx = i % LS_TW, ty = i / LS_TW;
            const int x = x0 + tx, y = rows_lo + ty;
            double a = 0, b = 0;
            int n = 0;
            if (x < width) {
                const float* row = in + (size_t)y * in_stride;
                for (int j = max(0, x - r); j <= min(width - 1, x + r); ++j) {
                    const float v = row[(size_t)j * 3 + c];
                    if (!isfinite(v)) continue;
                    const double d = (double)v - shift;
                    a += d;
                    b += d * d;
                    ++n;
                }
            }
            S.s1[ty][tx] = a;
            S.s2[ty][tx] = b;
            S.n[ty][tx] = n;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < LS_TW * LS_TH; i += LS_THREADS) {
            const int tx = i % LS_TW, ty = i / LS_TW;
            const int x = x0 + tx, y = y0 + ty;
            if (x >= width || y >= height) continue;
            double a = 0, b = 0;
            int n = 0;
            for (int j = max(0, y - r); j <= min(height - 1, y + r); ++j) {
                a += S.s1[j - rows_lo][tx];
                b += S.s2[j - rows_lo][tx];
                n += S.n[j - rows_lo][tx];
            }
            const size_t o = (size_t)y * width * 3 + (size_t)x * 3 + c;
            if (count_out) count_out[o] = (uint32_t)n;
            if (n == 0) {
                mean_out[o] = NAN;
                var_out[o] = NAN;
                continue;
            }
            const double mean = a / n;
            double var = (b - a * mean) / n;
            if (var < 0) var = 0;
            mean_out[o] = (T)(shift + mean);
            var_out[o] = (T)var;
        }
        __syncthreads();
    }
}

struct Scratch {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~Scratch() {
        if (p) cudaFreeAsync(p, s);
    }
};

#define SP_CUDA(call)                                                         \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) {                                              \
            set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
            return RE_CUDA_ERROR;                                             \
        }                                                                     \
    } while (0)

template <typename T>
re_status local_statistics(const float* in, size_t in_stride, uint32_t width, uint32_t height, uint32_t radius,
                           T* mean_out, T* var_out, uint32_t* count_out, void* stream_) {
    if (radius > LS_MAX_R) {
        set_last_error("local statistics radius must be in 0..32");
        return RE_INVALID_ARGUMENT;
    }
    if (!width || !height || !in || !mean_out || !var_out || in_stride < (size_t)width * 3) {
        set_last_error("spatial operation requires nonempty addressable bounds");
        return RE_INVALID_ARGUMENT;
    }
    cudaStream_t stream = (cudaStream_t)stream_;
    SP_CUDA(cudaFuncSetAttribute(local_stats_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(LsSmem)));
    dim3 grid((width + LS_TW - 1) / LS_TW, (height + LS_TH - 1) / LS_TH);
    local_stats_kernel<T><<<grid, LS_THREADS, sizeof(LsSmem), stream>>>(in, in_stride, (int)width, (int)height,
                                                                         (int)radius, mean_out, var_out, count_out);
    SP_CUDA(cudaGetLastError());
    SP_CUDA(cudaStreamSynchronize(stream));
    return RE_OK;
}

}  // namespace

extern "C" {

// SpatialOps.cpp:159-163 settings (radius extended to 64), 168-287 output.
re_status re_guided_filter(const float* in, size_t in_stride, float* out, size_t out_stride, uint32_t width,
                           uint32_t height, uint32_t radius, double epsilon, uint32_t space, void* stream_) {
    if (radius > 64 || !std::isfinite(epsilon) || epsilon < 0x1p-24 || epsilon > 65536.0) {
        set_last_error("guided filter requires radius 0..64 and finite epsilon [2^-24,65536]");
        return RE_INVALID_ARGUMENT;
    }
    if (space > 1) {
        set_last_error("guided filter requires scene-linear working RGB");
        return RE_INVALID_ARGUMENT;
    }
    if (!width || !height || !in || !out || in_stride < (size_t)width * 3 || out_stride < (size_t)width * 3) {
        set_last_error("guided filter requires nonempty addressable bounds");
        return RE_INVALID_ARGUMENT;
    }
    cudaStream_t stream = (cudaStream_t)stream_;
    const YWeights w = space == 0 ? YWeights{0.28807112822929337, 0.00008565396060525903}
                                  : YWeights{0.26270021201126703, 0.059301716469861945};
    const size_t px = (size_t)width * height;
    Scratch sc;
    sc.s = stream;
    SP_CUDA(cudaMallocAsync(&sc.p, 256 + px * 8 * sizeof(double) + 2 * px * 6 * sizeof(double), stream));
    uint32_t* status = (uint32_t*)sc.p;
    double* H = (double*)((char*)sc.p + 256);
    double* AB = H + px * 8;
    double* H2 = AB + px * 6;
    SP_CUDA(cudaMemsetAsync(status, 0, 4, stream));
    const int r = (int)radius;
    const int chunks = ((int)width + GF_CHUNK - 1) / GF_CHUNK;
    gf_hbox_moments<<<dim3((chunks + 63) / 64, height), 64, 0, stream>>>(in, in_stride, width, height, r, w, H,
                                                                         status);
    gf_vbox_coefficients<<<dim3((width + 127) / 128, (height + GF_CHUNK - 1) / GF_CHUNK), 128, 0, stream>>>(
        H, width, height, r, epsilon, AB, status);
    gf_hbox_ab<<<dim3((chunks + 63) / 64, height), 64, 0, stream>>>(AB, width, height, r, H2);
    gf_vbox_output<<<dim3((width + 127) / 128, (height + GF_CHUNK - 1) / GF_CHUNK), 128, 0, stream>>>(
        H2, in, in_stride, width, height, r, w, out, out_stride, status);
    SP_CUDA(cudaGetLastError());
    uint32_t key = 0;
    SP_CUDA(cudaMemcpyAsync(&key, status, 4, cudaMemcpyDeviceToHost, stream));
    SP_CUDA(cudaStreamSynchronize(stream));
    if (key & ST_INVALID) {
        set_last_error("guided filter requires finite complete input halo");
        return RE_INVALID_ARGUMENT;
    }
    if (key & ST_OVERFLOW) {
        set_last_error("guided filter float32 output overflow");
        return RE_OVERFLOW_ERROR;
    }
    return RE_OK;
}

// SpatialOps.cpp:74-121 (radius extended to 32).
re_status re_local_statistics(const float* in, size_t in_stride, uint32_t width, uint32_t height, uint32_t radius,
                              float* mean_out, float* var_out, uint32_t* count_out, void* stream) {
    return local_statistics<float>(in, in_stride, width, height, radius, mean_out, var_out, count_out, stream);
}

re_status re_local_statistics_f64(const float* in, size_t in_stride, uint32_t width, uint32_t height,
                                  uint32_t radius, double* mean_out, double* var_out, uint32_t* count_out,
                                  void* stream) {
    return local_statistics<double>(in, in_stride, width, height, radius, mean_out, var_out, count_out, stream);
}

}  // extern "C"
