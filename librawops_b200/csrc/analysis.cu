// RGB histogram of a rendered image (ImageAnalysis.cpp:9-69), one pass over
// device memory.
//
// Per channel: `bins` equal bins over [lower, upper] (half-open except the
// last, which includes upper), underflow / overflow / non-finite tallies, and
// the minimum and maximum of all finite samples.  A sample's bin is the
// reference's binary64 expression min(bins - 1, uint32((double(s) - lower) /
// span * bins)), divided before multiplying, evaluated with the same IEEE
// operations in the same order.
//
// The reference walks tiles in row-major tile order and keeps the FIRST
// sample that compares lower (higher) than the running extremum, so among
// samples that compare equal -- only +0 and -0 differ in bits -- the earliest
// in that traversal wins.  Each extremum here is one 64-bit key combined with
// atomicMin / atomicMax:
//     bits 63..32  the sample's order code (-0 coded as +0),
//     bits 31..1   its traversal index (for the maximum: 2^31 - 1 - index),
//     bit 0        the sample's sign bit,
// so the order of keys is the order of values, then of traversal, and the
// winning key still carries the sign of its zero.  Traversal indices saturate
// at 2^31 - 1 (viewports beyond 2^31 pixels break signed-zero ties among the
// later pixels by position instead).
//
// Layout and work split: the image is interleaved float32 RGB rows; rows are
// dealt to CTAs and a row's pixels to its threads (a warp reads 384
// contiguous bytes), counts into per-CTA shared-memory bins when 3 * bins
// fit (bins <= 4096), else straight into the global 64-bit counters, and keeps
// its tallies and extremum keys in registers; each CTA reduces those and
// issues one atomic per counter.  The bound is HBM: 12 bytes per pixel read,
// O(bins) written.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "re_device.cuh"

namespace re {
void set_last_error(const std::string& msg);
}

using namespace re;

namespace {

constexpr int HIST_THREADS = 256;
constexpr uint32_t HIST_SMEM_BINS = 4096;   // per channel; 48 KiB of uint32 counters for three channels

struct HistParams {
    const float* rgb;
    size_t stride;          // floats per row
    uint32_t width, height;
    uint32_t tile;          // traversal tile size (>= max(width, height) for one tile)
    uint64_t first_index;   // traversal index of the region's first pixel
    uint32_t bins;
    double lower, upper, span, scale;   // scale = bins / span (rounded)
    unsigned long long* counts;    // [3][bins]
    unsigned long long* tallies;   // under[3], over[3], nonfinite[3]
    unsigned long long* extrema;   // min key[3], max key[3]
};

__device__ __forceinline__ uint32_t order_code(float v) {
    const uint32_t u = __float_as_uint(v == 0.0f ? 0.0f : v);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ uint64_t traversal(const HistParams& P, uint32_t x, uint32_t y) {
    const uint32_t T = P.tile;
    const uint32_t y0 = y / T * T, x0 = x / T * T;
    const uint32_t th = min(T, P.height - y0), tw = min(T, P.width - x0);
    return P.first_index + (uint64_t)y0 * P.width + (uint64_t)x0 * th + (uint64_t)(y - y0) * tw + (x - x0);
}

// The reference's bin min(bins - 1, uint32((double(s) - lower) / span * bins)).
// The quotient-then-product is first approximated by one product with
// bins / span (both forms are within 4 ulp of the exact value, ~3e-11 for
// 65536 bins); when that lies more than 2^-30 from an integer both floor to
// the same bin, otherwise the reference's division is evaluated exactly.
__device__ __forceinline__ uint32_t bin_of(const HistParams& P, double d) {
    const double x = __dsub_rn(d, P.lower);
    const double a = __dmul_rn(x, P.scale);
    const double f = floor(a);
    double t = a;
    // (also taken when bins / span overflowed, so a is infinite or NaN)
    if (!(a - f >= 0x1p-30 && f + 1.0 - a >= 0x1p-30)) t = __dmul_rn(__ddiv_rn(x, P.span), (double)P.bins);
    return min(P.bins - 1, __double2uint_rz(t));
}

__device__ __forceinline__ unsigned long long warp_min(unsigned long long v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ unsigned long long warp_max(unsigned long long v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ uint32_t warp_add(uint32_t v) {
    return __reduce_add_sync(0xffffffffu, v);
}

template <bool SHARED>
__global__ void __launch_bounds__(HIST_THREADS) histogram_kernel(HistParams P) {
    extern __shared__ uint32_t sbins[];   // [3][bins] when SHARED
    __shared__ unsigned long long s_min[3][HIST_THREADS / 32], s_max[3][HIST_THREADS / 32];
    __shared__ uint32_t s_tally[9][HIST_THREADS / 32];
    if (SHARED) {
        for (uint32_t i = threadIdx.x; i < 3 * P.bins; i += HIST_THREADS) sbins[i] = 0;
        __syncthreads();
    }
    // Each thread's extrema as (order code, position, sign); the 64-bit keys
    // (order code, traversal index, sign) are formed only where two samples
    // share a code and at the end, so the common path carries no index
    // arithmetic (a divergent branch costs the whole warp).  Sentinels: no
    // finite sample has order code 0xffffffff or 0.
    uint32_t mn_code[3] = {~0u, ~0u, ~0u}, mx_code[3] = {0u, 0u, 0u};
    uint32_t mn_x[3], mn_y[3], mn_s[3], mx_x[3], mx_y[3], mx_s[3];
    auto min_key = [&](uint32_t code, uint32_t x, uint32_t y, uint32_t sign) {
        const uint64_t idx = min(traversal(P, x, y), (uint64_t)0x7fffffffu);
        return ((unsigned long long)code << 32) | (idx << 1) | sign;
    };
    auto max_key = [&](uint32_t code, uint32_t x, uint32_t y, uint32_t sign) {
        const uint64_t idx = min(traversal(P, x, y), (uint64_t)0x7fffffffu);
        return ((unsigned long long)code << 32) | ((0x7fffffffull - idx) << 1) | sign;
    };
    uint32_t tally[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    // rows are dealt to CTAs, a row's pixels to the CTA's threads (coalesced)
    for (uint32_t y = blockIdx.x; y < P.height; y += gridDim.x) {
        const float* row = P.rgb + (size_t)y * P.stride;
        for (uint32_t x = threadIdx.x; x < P.width; x += HIST_THREADS) {
            const float v[3] = {__ldcs(row + (size_t)x * 3), __ldcs(row + (size_t)x * 3 + 1),
                                __ldcs(row + (size_t)x * 3 + 2)};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float s = v[c];
                if (!isfinite(s)) {
                    ++tally[6 + c];
                    continue;
                }
                // the traversal index only decides between equal codes
                const uint32_t code = order_code(s);
                const uint32_t sign = __float_as_uint(s) >> 31;
                if (code < mn_code[c] ||
                    (code == mn_code[c] && min_key(code, x, y, sign) < min_key(code, mn_x[c], mn_y[c], mn_s[c]))) {
                    mn_code[c] = code;
                    mn_x[c] = x;
                    mn_y[c] = y;
                    mn_s[c] = sign;
                }
                if (code > mx_code[c] ||
                    (code == mx_code[c] && max_key(code, x, y, sign) > max_key(code, mx_x[c], mx_y[c], mx_s[c]))) {
                    mx_code[c] = code;
                    mx_x[c] = x;
                    mx_y[c] = y;
                    mx_s[c] = sign;
                }
                const double d = (double)s;
                if (d < P.lower) {
                    ++tally[c];
                    continue;
                }
                if (d > P.upper) {
                    ++tally[3 + c];
                    continue;
                }
                const uint32_t bin = bin_of(P, d);
                if (SHARED)
                    atomicAdd(&sbins[c * P.bins + bin], 1u);
                else
                    atomicAdd(&P.counts[(size_t)c * P.bins + bin], 1ull);
            }
        }
    }
    unsigned long long kmin[3], kmax[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        kmin[c] = mn_code[c] == ~0u ? ~0ull : min_key(mn_code[c], mn_x[c], mn_y[c], mn_s[c]);
        kmax[c] = mx_code[c] == 0u ? 0ull : max_key(mx_code[c], mx_x[c], mx_y[c], mx_s[c]);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const unsigned long long a = warp_min(kmin[c]), b = warp_max(kmax[c]);
        if (!lane) {
            s_min[c][warp] = a;
            s_max[c][warp] = b;
        }
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const uint32_t t = warp_add(tally[k]);
        if (!lane) s_tally[k][warp] = t;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        const int c = threadIdx.x;
        unsigned long long a = ~0ull, b = 0;
        for (int w = 0; w < HIST_THREADS / 32; ++w) {
            a = min(a, s_min[c][w]);
            b = max(b, s_max[c][w]);
        }
        if (a != ~0ull) atomicMin(&P.extrema[c], a);
        if (b) atomicMax(&P.extrema[3 + c], b);
    } else if (threadIdx.x >= 32 && threadIdx.x < 41) {
        const int k = threadIdx.x - 32;
        unsigned long long t = 0;
        for (int w = 0; w < HIST_THREADS / 32; ++w) t += s_tally[k][w];
        if (t) atomicAdd(&P.tallies[k], t);
    }
    if (SHARED) {
        for (uint32_t i = threadIdx.x; i < 3 * P.bins; i += HIST_THREADS)
            if (sbins[i]) atomicAdd(&P.counts[i], (unsigned long long)sbins[i]);
    }
}

re_status hist_fail(re_status s, const char* msg) {
    set_last_error(msg);
    return s;
}

}  // namespace

extern "C" {

re_status re_histogram_reset(uint32_t bins, uint64_t* counts, uint64_t* tallies, uint64_t* extrema, void* stream_) {
    if (!bins || bins > 65536) return hist_fail(RE_INVALID_ARGUMENT, "histogram requires 1..65536 bins and a finite positive range");
    if (!counts || !tallies || !extrema) return hist_fail(RE_INVALID_ARGUMENT, "null histogram counters");
    cudaStream_t s = (cudaStream_t)stream_;
    cudaError_t e = cudaMemsetAsync(counts, 0, (size_t)3 * bins * sizeof(uint64_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(tallies, 0, 9 * sizeof(uint64_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(extrema, 0xff, 3 * sizeof(uint64_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(extrema + 3, 0, 3 * sizeof(uint64_t), s);
    if (e != cudaSuccess) {
        set_last_error(std::string("histogram reset: ") + cudaGetErrorString(e));
        return RE_CUDA_ERROR;
    }
    return RE_OK;
}

re_status re_histogram_rgb(const float* rgb, size_t row_stride, uint32_t width, uint32_t height, uint32_t tile_size,
                           uint64_t first_index, uint32_t bins, double lower, double upper, uint64_t* counts,
                           uint64_t* tallies, uint64_t* extrema, void* stream_) {
    const double span = upper - lower;
    if (bins == 0 || bins > 65536 || !std::isfinite(lower) || !std::isfinite(upper) || !(span > 0.0) ||
        !std::isfinite(span))
        return hist_fail(RE_INVALID_ARGUMENT, "histogram requires 1..65536 bins and a finite positive range");
    if (!counts || !tallies || !extrema) return hist_fail(RE_INVALID_ARGUMENT, "null histogram counters");
    if (!width || !height) return RE_OK;
    if (!rgb || row_stride < (size_t)width * 3) return hist_fail(RE_INVALID_ARGUMENT, "invalid histogram image");
    HistParams P;
    P.rgb = rgb;
    P.stride = row_stride;
    P.width = width;
    P.height = height;
    P.tile = tile_size ? tile_size : 0xffffffffu;
    P.first_index = first_index;
    P.bins = bins;
    P.lower = lower;
    P.upper = upper;
    P.span = span;
    P.scale = (double)bins / span;
    P.counts = reinterpret_cast<unsigned long long*>(counts);
    P.tallies = reinterpret_cast<unsigned long long*>(tallies);
    P.extrema = reinterpret_cast<unsigned long long*>(extrema);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(height, (uint64_t)sms * 8));
    cudaStream_t s = (cudaStream_t)stream_;
    if (bins <= HIST_SMEM_BINS) {
        const size_t smem = (size_t)3 * bins * sizeof(uint32_t);
        cudaError_t a = cudaFuncSetAttribute(histogram_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)(3 * HIST_SMEM_BINS * sizeof(uint32_t)));
        if (a != cudaSuccess) {
            set_last_error(std::string("histogram: ") + cudaGetErrorString(a));
            return RE_CUDA_ERROR;
        }
        histogram_kernel<true><<<grid, HIST_THREADS, smem, s>>>(P);
    }
    else
        histogram_kernel<false><<<grid, HIST_THREADS, 0, s>>>(P);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_error(std::string("histogram: ") + cudaGetErrorString(e));
        return RE_CUDA_ERROR;
    }
    return RE_OK;
}

int re_histogram_extremum(uint64_t key, int is_max, float* value) {
    if (is_max ? key == 0 : key == ~0ull) return 0;
    const uint32_t code = (uint32_t)(key >> 32);
    uint32_t bits = (code & 0x80000000u) ? (code & 0x7fffffffu) : ~code;
    if (bits == 0 && (key & 1u)) bits = 0x80000000u;   // the winning sample was -0
    if (value) std::memcpy(value, &bits, sizeof(float));
    return 1;
}

}  // extern "C"
