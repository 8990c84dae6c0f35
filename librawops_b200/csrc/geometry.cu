// Geometry stages: CubicResizeNode and RotateNode (GeometryOps.cpp of the
// reference), with their mip-1/2 footprint averaging.
//
// Both are bit-exact restatements: the reference evaluates them in binary64
// with a frozen operation order and rounds once to float32; the kernels use
// explicitly rounded double ops in that order.  The cubic resize is split into
// a horizontal pass (one double per source row, output column and channel --
// exactly the value the reference's `horizontal(row, c)` returns) and a
// vertical pass that accumulates the rows in the reference's tap order, so the
// separable form changes no bit.  Axis tables (Catmull-Rom taps with the
// reference's clamping, normalization and guards, GeometryOps.cpp:362-389) are
// planned on the host in binary64 and uploaded per call.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <string>
#include <vector>

#include "re_device.cuh"

namespace re {
cudaError_t launch_mip_reduce(const float* native, int nw, int nh, size_t native_stride, int mip,
                              int ow, int oh, int stage_begin, int stage_end, const DevProgram& P,
                              float* out, size_t out_stride, uint32_t* status, cudaStream_t stream,
                              uint32_t* launches);
void set_last_error(const std::string& msg);
}  // namespace re

using namespace re;

namespace {

constexpr int MAX_TAPS = 18;

struct Axis {
    uint32_t center, count;
    uint32_t index[MAX_TAPS];
    double weight[MAX_TAPS];
};

// GeometryOps.cpp:362-389
re_status cubic_axis(uint32_t input, uint32_t output, uint32_t index, Axis& a) {
    a = Axis{};
    if (input == output) {
        a.center = index;
        a.count = 1;
        a.index[0] = index;
        a.weight[0] = 1;
        return RE_OK;
    }
    const double z = std::clamp(((double(index) + .5) * double(input) / double(output)) - .5, 0.,
                                double(input - 1));
    const double scale = std::max(1., double(input) / double(output));
    a.center = (uint32_t)std::floor(z);
    const int64_t first = (int64_t)std::floor(z - 2 * scale);
    const int64_t last = (int64_t)std::ceil(z + 2 * scale);
    double total = 0;
    for (int64_t i = first; i <= last; ++i) {
        const double distance = std::abs((double(i) - z) / scale);
        double value = 0;
        if (distance < 1) value = ((1.5 * distance - 2.5) * distance) * distance + 1;
        else if (distance < 2) value = (-.5 * (distance - 1)) * ((distance - 2) * (distance - 2));
        const double weight = value / scale;
        if (weight == 0) continue;
        if (a.count == MAX_TAPS) {
            set_last_error("cubic resize axis tap cap exceeded");
            return RE_INVALID_ARGUMENT;
        }
        a.index[a.count] = (uint32_t)std::clamp<int64_t>(i, 0, int64_t(input) - 1);
        a.weight[a.count] = weight;
        ++a.count;
        total = total + weight;
    }
    if (!std::isfinite(total) || total <= .5) {
        set_last_error("cubic resize normalization guard failed");
        return RE_INVALID_ARGUMENT;
    }
    for (uint32_t i = 0; i < a.count; ++i) {
        a.weight[i] = a.weight[i] / total;
        if (!std::isfinite(a.weight[i]) || std::abs(a.weight[i]) > 4) {
            set_last_error("cubic resize axis weight guard failed");
            return RE_INVALID_ARGUMENT;
        }
    }
    return RE_OK;
}

__device__ __forceinline__ float finite_float(double v, uint32_t& err) {
    if (!isfinite(v) || fabs(v) > (double)FLT_MAX) {
        err = max(err, (uint32_t)((200u << 8) | ST_INVALID));
        return 0.0f;
    }
    return (float)v;
}

// Horizontal pass: H[r][x][c] for source rows [row0, row0+rows) and native
// output columns [0, nw), GeometryOps.cpp:453-465.
__global__ void cubic_h_kernel(const float* __restrict__ src, size_t src_stride, int src_x0, int src_y0,
                               const Axis* __restrict__ ax, int nw, int row0, int rows, double* __restrict__ H,
                               uint32_t* status) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= nw || r >= rows) return;
    const Axis& a = ax[x];
    const float* row = src + (size_t)(row0 + r - src_y0) * src_stride - (ptrdiff_t)src_x0 * 3;
    uint32_t err = 0;
    double* h = H + ((size_t)r * nw + x) * 3;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float b = row[(size_t)a.center * 3 + c];
        if (!isfinite(b)) err = ST_INVALID | (201u << 8);
        const double base = (double)b;
        double v = base;
        for (uint32_t i = 0; i < a.count; ++i) {
            const float s = row[(size_t)a.index[i] * 3 + c];
            if (!isfinite(s)) err = ST_INVALID | (201u << 8);
            const double delta = __dmul_rn(a.weight[i], __dsub_rn((double)s, base));
            if (delta != 0) v = __dadd_rn(v, delta);
        }
        h[c] = v;
    }
    if (err && status) atomicMax(status, err);
}

// Vertical pass, GeometryOps.cpp:466-479 (row reuse only caches equal values).
__global__ void cubic_v_kernel(const double* __restrict__ H, const Axis* __restrict__ ay, int nw, int nh,
                               int row0, float* __restrict__ out, size_t out_stride, uint32_t* status) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= nw || y >= nh) return;
    const Axis& a = ay[y];
    uint32_t err = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double base = H[((size_t)(a.center - row0) * nw + x) * 3 + c];
        double v = base;
        for (uint32_t i = 0; i < a.count; ++i) {
            const double rv = H[((size_t)(a.index[i] - row0) * nw + x) * 3 + c];
            const double delta = __dmul_rn(a.weight[i], __dsub_rn(rv, base));
            if (delta != 0) v = __dadd_rn(v, delta);
        }
        out[(size_t)y * out_stride + (size_t)x * 3 + c] = finite_float(v, err);
    }
    if (err && status) atomicMax(status, err);
}

// GeometryOps.cpp:29-34
__device__ __forceinline__ double blend(double a, double b, double t) {
    if (t == 0) return a;
    if (t == 1) return b;
    if (a == b) return a;
    return __dadd_rn(a, __dmul_rn(t, __dsub_rn(b, a)));
}

struct RotateParams {
    double cx, cy, cosine, sine;
    int width, height;
};

// GeometryOps.cpp:68-76 taps and 129-141 sampling, one native output pixel per thread.
__global__ void rotate_kernel(const float* __restrict__ src, size_t src_stride, int src_x0, int src_y0,
                              RotateParams p, int nx0, int ny0, int nw, int nh, float* __restrict__ out,
                              size_t out_stride, uint32_t* status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= nw || j >= nh) return;
    const double dx = __dsub_rn((double)(nx0 + i), p.cx), dy = __dsub_rn((double)(ny0 + j), p.cy);
    double sx = __dadd_rn(__dadd_rn(p.cx, __dmul_rn(p.cosine, dx)), __dmul_rn(p.sine, dy));
    double sy = __dadd_rn(__dsub_rn(p.cy, __dmul_rn(p.sine, dx)), __dmul_rn(p.cosine, dy));
    const double mx = (double)p.width - 1, my = (double)p.height - 1;
    sx = sx < 0. ? 0. : (mx < sx ? mx : sx);
    sy = sy < 0. ? 0. : (my < sy ? my : sy);
    const uint32_t x0 = (uint32_t)floor(sx), y0 = (uint32_t)floor(sy);
    const double fx = __dsub_rn(sx, (double)x0), fy = __dsub_rn(sy, (double)y0);
    const uint32_t x1 = fx == 0 ? x0 : min(x0 + 1, (uint32_t)p.width - 1);
    const uint32_t y1 = fy == 0 ? y0 : min(y0 + 1, (uint32_t)p.height - 1);
    const float* base = src - (ptrdiff_t)src_y0 * (ptrdiff_t)src_stride - (ptrdiff_t)src_x0 * 3;
    uint32_t err = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float a00 = base[(size_t)y0 * src_stride + (size_t)x0 * 3 + c];
        const float a10 = base[(size_t)y0 * src_stride + (size_t)x1 * 3 + c];
        const float a01 = base[(size_t)y1 * src_stride + (size_t)x0 * 3 + c];
        const float a11 = base[(size_t)y1 * src_stride + (size_t)x1 * 3 + c];
        if (!(isfinite(a00) && isfinite(a10) && isfinite(a01) && isfinite(a11))) err = ST_INVALID | (201u << 8);
        const double upper = blend((double)a00, (double)a10, fx);
        const double lower = blend((double)a01, (double)a11, fx);
        out[(size_t)j * out_stride + (size_t)i * 3 + c] = finite_float(blend(upper, lower, fy), err);
    }
    if (err && status) atomicMax(status, err);
}

// GeometryOps.cpp:68-76 taps and 99-111 support scan, on the host (relative to the rotation bounds).
re_status rotate_support_host(const RotateParams& p, re_rect out, re_rect& support) {
    uint32_t left = (uint32_t)p.width, top = (uint32_t)p.height, right = 0, bottom = 0;
    for (uint64_t y = out.y; y < (uint64_t)out.y + out.height; ++y)
        for (uint64_t x = out.x; x < (uint64_t)out.x + out.width; ++x) {
            const double dx = double(x) - p.cx, dy = double(y) - p.cy;
            const double sx = std::clamp((p.cx + p.cosine * dx) + p.sine * dy, 0., double(p.width) - 1);
            const double sy = std::clamp((p.cy - p.sine * dx) + p.cosine * dy, 0., double(p.height) - 1);
            const uint32_t ix = (uint32_t)std::floor(sx), iy = (uint32_t)std::floor(sy);
            const double fx = sx - ix, fy = sy - iy;
            const uint32_t x1 = fx == 0 ? ix : std::min(ix + 1, (uint32_t)p.width - 1);
            const uint32_t y1 = fy == 0 ? iy : std::min(iy + 1, (uint32_t)p.height - 1);
            left = std::min(left, ix);
            top = std::min(top, iy);
            right = std::max(right, x1);
            bottom = std::max(bottom, y1);
        }
    support = {left, top, right - left + 1, bottom - top + 1};
    return RE_OK;
}

// native footprint of a reduced request over a canvas (GeometryOps.cpp:86-98, 399-410)
bool native_region(uint32_t cw, uint32_t ch, re_rect out, uint32_t mip, re_rect& native) {
    const uint32_t scale = 1u << mip;
    const uint32_t ew = cw / scale + (cw % scale != 0), eh = ch / scale + (ch % scale != 0);
    if ((uint64_t)out.x + out.width > ew || (uint64_t)out.y + out.height > eh) return false;
    const uint64_t l = std::min<uint64_t>((uint64_t)out.x * scale, cw), t = std::min<uint64_t>((uint64_t)out.y * scale, ch);
    const uint64_t r = std::min<uint64_t>(((uint64_t)out.x + out.width) * scale, cw);
    const uint64_t b = std::min<uint64_t>(((uint64_t)out.y + out.height) * scale, ch);
    native = {(uint32_t)l, (uint32_t)t, (uint32_t)(r - l), (uint32_t)(b - t)};
    return true;
}

struct Scratch {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~Scratch() {
        if (p) cudaFreeAsync(p, s);
    }
};

re_status finish(cudaStream_t stream, uint32_t* status_dev) {
    uint32_t key = 0;
    cudaError_t e = cudaMemcpyAsync(&key, status_dev, 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        set_last_error(std::string("geometry: ") + cudaGetErrorString(e));
        return RE_CUDA_ERROR;
    }
    if (key) {
        set_last_error("geometry requires finite input within float32 range");
        return RE_INVALID_ARGUMENT;
    }
    return RE_OK;
}

#define GEO_CUDA(call)                                                        \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) {                                              \
            set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
            return RE_CUDA_ERROR;                                             \
        }                                                                     \
    } while (0)

}  // namespace

extern "C" {
re_status re_cubic_resize_window(const float* in, size_t in_stride, re_rect window, uint32_t in_w, uint32_t in_h,
                                 uint32_t out_w, uint32_t out_h, re_rect output, uint32_t mip, float* out,
                                 size_t out_stride, void* stream_);
re_status re_rotate_window(const float* in, size_t in_stride, re_rect window, uint32_t width, uint32_t height,
                           double angle, re_rect output, uint32_t mip, float* out, size_t out_stride, void* stream_);

re_status re_rotation_support(uint32_t width, uint32_t height, double angle, re_rect native_output, re_rect* support) {
    RotateParams p{};
    re_status s = re_rotation_coefficients(angle, &p.cosine, &p.sine);
    if (s) return s;
    p.cx = (double(width) - 1) / 2;
    p.cy = (double(height) - 1) / 2;
    p.width = (int)width;
    p.height = (int)height;
    if (!native_output.width || !native_output.height) {
        *support = {0, 0, 0, 0};
        return RE_OK;
    }
    return rotate_support_host(p, native_output, *support);
}

re_status re_cubic_axis(uint32_t input, uint32_t output, uint32_t index, uint32_t* center, uint32_t tap_index[18],
                        double tap_weight[18], uint32_t* count) {
    if (!input || !output) {
        set_last_error("cubic resize requires positive input and canvas extents");
        return RE_INVALID_ARGUMENT;
    }
    Axis a;
    re_status s = cubic_axis(input, output, index, a);
    if (s) return s;
    *center = a.center;
    *count = a.count;
    for (uint32_t i = 0; i < a.count; ++i) {
        tap_index[i] = a.index[i];
        tap_weight[i] = a.weight[i];
    }
    return RE_OK;
}

// GeometryOps.cpp:346-352 validation, 431-513 render.
re_status re_cubic_resize(const float* in, size_t in_stride, uint32_t in_w, uint32_t in_h, uint32_t out_w,
                          uint32_t out_h, re_rect output, uint32_t mip, float* out, size_t out_stride, void* stream) {
    return re_cubic_resize_window(in, in_stride, {0, 0, in_w, in_h}, in_w, in_h, out_w, out_h, output, mip, out,
                                  out_stride, stream);
}

re_status re_cubic_resize_window(const float* in, size_t in_stride, re_rect window, uint32_t in_w, uint32_t in_h,
                                 uint32_t out_w, uint32_t out_h, re_rect output, uint32_t mip, float* out,
                                 size_t out_stride, void* stream_) {
    if (!in_w || !in_h || !out_w || !out_h) {
        set_last_error("cubic resize requires positive input and canvas extents");
        return RE_INVALID_ARGUMENT;
    }
    if ((uint64_t)out_w * 4 < in_w || (uint64_t)out_h * 4 < in_h) {
        set_last_error("cubic resize native shrink exceeds fourfold per axis");
        return RE_INVALID_ARGUMENT;
    }
    if (mip > 2) {
        set_last_error("cubic resize does not support render level");
        return RE_INVALID_ARGUMENT;
    }
    re_rect native;
    if (!native_region(out_w, out_h, output, mip, native)) {
        set_last_error("cubic resize output rectangle is outside image");
        return RE_OUT_OF_RANGE;
    }
    if (!output.width || !output.height) return RE_OK;
    if (!in || !out || in_stride < (size_t)window.width * 3 || out_stride < (size_t)output.width * 3 ||
        (uint64_t)window.x + window.width > in_w || (uint64_t)window.y + window.height > in_h) {
        set_last_error("invalid cubic resize buffers");
        return RE_INVALID_ARGUMENT;
    }
    std::vector<Axis> xs(native.width), ys(native.height);
    uint32_t row_lo = in_h, row_hi = 0;
    for (uint32_t i = 0; i < native.width; ++i) {
        re_status s = cubic_axis(in_w, out_w, native.x + i, xs[i]);
        if (s) return s;
    }
    for (uint32_t j = 0; j < native.height; ++j) {
        re_status s = cubic_axis(in_h, out_h, native.y + j, ys[j]);
        if (s) return s;
        row_lo = std::min(row_lo, ys[j].center);
        row_hi = std::max(row_hi, ys[j].center);
        for (uint32_t k = 0; k < ys[j].count; ++k) {
            row_lo = std::min(row_lo, ys[j].index[k]);
            row_hi = std::max(row_hi, ys[j].index[k]);
        }
    }
    const uint32_t rows = row_hi - row_lo + 1;
    uint32_t col_lo = in_w, col_hi = 0;
    for (const Axis& a : xs) {
        col_lo = std::min(col_lo, a.center);
        col_hi = std::max(col_hi, a.center);
        for (uint32_t k = 0; k < a.count; ++k) {
            col_lo = std::min(col_lo, a.index[k]);
            col_hi = std::max(col_hi, a.index[k]);
        }
    }
    if (col_lo < window.x || col_hi >= window.x + window.width || row_lo < window.y ||
        row_hi >= window.y + window.height) {
        set_last_error("cubic resize input window does not cover the taps' support");
        return RE_INVALID_ARGUMENT;
    }
    cudaStream_t stream = (cudaStream_t)stream_;
    const size_t axes_bytes = (xs.size() + ys.size()) * sizeof(Axis);
    const size_t h_bytes = (size_t)rows * native.width * 3 * sizeof(double);
    const size_t nat_bytes = mip ? (size_t)native.width * native.height * 3 * sizeof(float) : 0;
    Scratch sc;
    sc.s = stream;
    GEO_CUDA(scratch_alloc(&sc.p, 256 + axes_bytes + h_bytes + nat_bytes, stream));
    char* base = (char*)sc.p;
    uint32_t* status = (uint32_t*)base;
    Axis* dax = (Axis*)(base + 256);
    Axis* day = dax + xs.size();
    double* H = (double*)(base + 256 + axes_bytes);
    float* nat = (float*)(base + 256 + axes_bytes + h_bytes);
    GEO_CUDA(cudaMemsetAsync(status, 0, 4, stream));
    GEO_CUDA(cudaMemcpyAsync(dax, xs.data(), xs.size() * sizeof(Axis), cudaMemcpyHostToDevice, stream));
    GEO_CUDA(cudaMemcpyAsync(day, ys.data(), ys.size() * sizeof(Axis), cudaMemcpyHostToDevice, stream));
    dim3 b(32, 8);
    cubic_h_kernel<<<dim3((native.width + 31) / 32, (rows + 7) / 8), b, 0, stream>>>(
        in, in_stride, (int)window.x, (int)window.y, dax, (int)native.width, (int)row_lo, (int)rows, H, status);
    float* target = mip ? nat : out;
    const size_t tstride = mip ? (size_t)native.width * 3 : out_stride;
    cubic_v_kernel<<<dim3((native.width + 31) / 32, (native.height + 7) / 8), b, 0, stream>>>(
        H, day, (int)native.width, (int)native.height, (int)row_lo, target, tstride, status);
    GEO_CUDA(cudaGetLastError());
    if (mip) {
        DevProgram P{};
        GEO_CUDA(launch_mip_reduce(nat, (int)native.width, (int)native.height, tstride, (int)mip, (int)output.width,
                                   (int)output.height, 0, 0, P, out, out_stride, status, stream, nullptr));
    }
    return finish(stream, status);
}

// GeometryOps.cpp:42-67
re_status re_rotation_coefficients(double a, double* cosine, double* sine) {
    if (!std::isfinite(a) || a < -180 || a > 180) {
        set_last_error("rotation angle_degrees must be finite in [-180,180]");
        return RE_INVALID_ARGUMENT;
    }
    if (a == 0) { *cosine = 1; *sine = 0; }
    else if (a == 90) { *cosine = 0; *sine = 1; }
    else if (a == -90) { *cosine = 0; *sine = -1; }
    else if (std::abs(a) == 180) { *cosine = -1; *sine = 0; }
    else {
        const double theta = (a / 180) * 0x1.921fb54442d18p+1;
        *cosine = std::cos(theta);
        *sine = std::sin(theta);
        if (!std::isfinite(*cosine) || !std::isfinite(*sine) || std::abs(*cosine) > 1 || std::abs(*sine) > 1) {
            set_last_error("rotation math runtime returned invalid coefficients");
            return RE_INVALID_ARGUMENT;
        }
    }
    return RE_OK;
}

re_status re_rotate(const float* in, size_t in_stride, uint32_t width, uint32_t height, double angle,
                    re_rect output, uint32_t mip, float* out, size_t out_stride, void* stream) {
    return re_rotate_window(in, in_stride, {0, 0, width, height}, width, height, angle, output, mip, out, out_stride,
                            stream);
}

re_status re_rotate_window(const float* in, size_t in_stride, re_rect window, uint32_t width, uint32_t height,
                           double angle, re_rect output, uint32_t mip, float* out, size_t out_stride,
                           void* stream_) {
    if (!width || !height) {
        set_last_error("rotation requires input and nonempty image bounds");
        return RE_INVALID_ARGUMENT;
    }
    RotateParams p{};
    re_status s = re_rotation_coefficients(angle, &p.cosine, &p.sine);
    if (s) return s;
    if (mip > 2) {
        set_last_error("rotation does not support render level");
        return RE_INVALID_ARGUMENT;
    }
    p.cx = (double(width) - 1) / 2;
    p.cy = (double(height) - 1) / 2;
    p.width = (int)width;
    p.height = (int)height;
    re_rect native;
    if (!native_region(width, height, output, mip, native)) {
        set_last_error("rotation output rectangle is outside image");
        return RE_OUT_OF_RANGE;
    }
    if (!output.width || !output.height) return RE_OK;
    if (!in || !out || in_stride < (size_t)window.width * 3 || out_stride < (size_t)output.width * 3 ||
        (uint64_t)window.x + window.width > width || (uint64_t)window.y + window.height > height) {
        set_last_error("invalid rotation buffers");
        return RE_INVALID_ARGUMENT;
    }
    if (window.x || window.y || window.width != width || window.height != height) {
        // the taps of every native output pixel must lie inside the window (GeometryOps.cpp:99-111)
        re_rect support;
        re_status ss = rotate_support_host(p, native, support);
        if (ss) return ss;
        if (support.x < window.x || support.y < window.y ||
            (uint64_t)support.x + support.width > (uint64_t)window.x + window.width ||
            (uint64_t)support.y + support.height > (uint64_t)window.y + window.height) {
            set_last_error("rotation input window does not cover the taps' support");
            return RE_INVALID_ARGUMENT;
        }
    }
    cudaStream_t stream = (cudaStream_t)stream_;
    const size_t nat_bytes = mip ? (size_t)native.width * native.height * 3 * sizeof(float) : 0;
    Scratch sc;
    sc.s = stream;
    GEO_CUDA(scratch_alloc(&sc.p, 256 + nat_bytes, stream));
    uint32_t* status = (uint32_t*)sc.p;
    float* nat = (float*)((char*)sc.p + 256);
    GEO_CUDA(cudaMemsetAsync(status, 0, 4, stream));
    float* target = mip ? nat : out;
    const size_t tstride = mip ? (size_t)native.width * 3 : out_stride;
    dim3 b(32, 8);
    rotate_kernel<<<dim3((native.width + 31) / 32, (native.height + 7) / 8), b, 0, stream>>>(
        in, in_stride, (int)window.x, (int)window.y, p, (int)native.x, (int)native.y, (int)native.width, (int)native.height, target, tstride,
        status);
    GEO_CUDA(cudaGetLastError());
    if (mip) {
        DevProgram P{};
        GEO_CUDA(launch_mip_reduce(nat, (int)native.width, (int)native.height, tstride, (int)mip, (int)output.width,
                                   (int)output.height, 0, 0, P, out, out_stride, status, stream, nullptr));
    }
    return finish(stream, status);
}

}  // extern "C"
