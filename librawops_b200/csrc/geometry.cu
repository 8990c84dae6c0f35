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
#include "re_geometry.cuh"

namespace re {
cudaError_t launch_mip_reduce(const float* native, int nw, int nh, size_t native_stride, int mip,
                              int ow, int oh, int stage_begin, int stage_end, const DevProgram& P,
                              float* out, size_t out_stride, uint32_t* status, cudaStream_t stream,
                              uint32_t* launches);
void set_last_error(const std::string& msg);
}  // namespace re

extern "C" re_status re_rotation_coefficients(double a, double* cosine, double* sine);

using namespace re;

namespace {

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
        if (a.count == GEO_MAX_TAPS) {
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

// Horizontal sum of one source row at one native output column, all three
// channels (GeometryOps.cpp:453-465).  `row` points at the source row's
// input-bound column 0.
__device__ __forceinline__ void cubic_h_pixel(const float* row, const Axis& a, double* h, uint32_t& err) {
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
}

// Vertical pass at one native output pixel (GeometryOps.cpp:466-479; the
// reference's row reuse only caches equal values).
__device__ __forceinline__ void cubic_v_pixel(const double* H, const Axis& a, int nw, int row0, int x, float* o,
                                              uint32_t& err) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double base = H[((size_t)(a.center - row0) * nw + x) * 3 + c];
        double v = base;
        for (uint32_t i = 0; i < a.count; ++i) {
            const double rv = H[((size_t)(a.index[i] - row0) * nw + x) * 3 + c];
            const double delta = __dmul_rn(a.weight[i], __dsub_rn(rv, base));
            if (delta != 0) v = __dadd_rn(v, delta);
        }
        o[c] = finite_float(v, err);
    }
}

// GeometryOps.cpp:29-34
__device__ __forceinline__ double blend(double a, double b, double t) {
    if (t == 0) return a;
    if (t == 1) return b;
    if (a == b) return a;
    return __dadd_rn(a, __dmul_rn(t, __dsub_rn(b, a)));
}

// GeometryOps.cpp:68-76 taps and 129-141 sampling at native output (x, y).
// `base` points at input-bound pixel (0, 0) of the source.
__device__ __forceinline__ void rotate_pixel(const float* base, size_t src_stride, const RotateParams& p, int x, int y,
                                             float* o, uint32_t& err) {
    const double dx = __dsub_rn((double)x, p.cx), dy = __dsub_rn((double)y, p.cy);
    double sx = __dadd_rn(__dadd_rn(p.cx, __dmul_rn(p.cosine, dx)), __dmul_rn(p.sine, dy));
    double sy = __dadd_rn(__dsub_rn(p.cy, __dmul_rn(p.sine, dx)), __dmul_rn(p.cosine, dy));
    const double mx = (double)p.width - 1, my = (double)p.height - 1;
    sx = sx < 0. ? 0. : (mx < sx ? mx : sx);
    sy = sy < 0. ? 0. : (my < sy ? my : sy);
    const uint32_t x0 = (uint32_t)floor(sx), y0 = (uint32_t)floor(sy);
    const double fx = __dsub_rn(sx, (double)x0), fy = __dsub_rn(sy, (double)y0);
    const uint32_t x1 = fx == 0 ? x0 : min(x0 + 1, (uint32_t)p.width - 1);
    const uint32_t y1 = fy == 0 ? y0 : min(y0 + 1, (uint32_t)p.height - 1);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float a00 = base[(size_t)y0 * src_stride + (size_t)x0 * 3 + c];
        const float a10 = base[(size_t)y0 * src_stride + (size_t)x1 * 3 + c];
        const float a01 = base[(size_t)y1 * src_stride + (size_t)x0 * 3 + c];
        const float a11 = base[(size_t)y1 * src_stride + (size_t)x1 * 3 + c];
        if (!(isfinite(a00) && isfinite(a10) && isfinite(a01) && isfinite(a11))) err = ST_INVALID | (201u << 8);
        const double upper = blend((double)a00, (double)a10, fx);
        const double lower = blend((double)a01, (double)a11, fx);
        o[c] = finite_float(blend(upper, lower, fy), err);
    }
}

// Source pixel (0, 0) of a request's input bounds, addressed through its support buffer.
__device__ __forceinline__ const float* source_origin(const GeoRequest& R) {
    return R.src - (ptrdiff_t)R.src_y0 * (ptrdiff_t)R.src_stride - (ptrdiff_t)R.src_x0 * 3;
}

// Pass 1 of one 32 x 8 block: cubic horizontal sums (rows of H) or the rotation.
__device__ __forceinline__ void geo_pass1(const GeoRequest& R, int bx, int by, uint32_t& err) {
    const int x = bx * GEO_BW + (int)threadIdx.x % GEO_BW, r = by * GEO_BH + (int)threadIdx.x / GEO_BW;
    if (R.kind == 1) {
        if (x >= R.nw || r >= R.rows) return;
        const float* row = source_origin(R) + (size_t)(R.row0 + r) * R.src_stride;
        cubic_h_pixel(row, R.ax[x], R.H + ((size_t)r * R.nw + x) * 3, err);
    } else {
        if (x >= R.nw || r >= R.nh) return;
        rotate_pixel(source_origin(R), R.src_stride, R.rot, R.nx0 + x, R.ny0 + r,
                     R.out + (size_t)r * R.out_stride + (size_t)x * 3, err);
    }
}

// Pass 2 of one block: the cubic vertical pass.
__device__ __forceinline__ void geo_pass2(const GeoRequest& R, int bx, int by, uint32_t& err) {
    const int x = bx * GEO_BW + (int)threadIdx.x % GEO_BW, y = by * GEO_BH + (int)threadIdx.x / GEO_BW;
    if (x >= R.nw || y >= R.nh) return;
    cubic_v_pixel(R.H, R.ay[y], R.nw, R.row0, x, R.out + (size_t)y * R.out_stride + (size_t)x * 3, err);
}

__global__ void __launch_bounds__(GEO_BW* GEO_BH) geo_batch_kernel(const GeoRequest* __restrict__ requests,
                                                                    const GeoBlock* __restrict__ blocks, uint32_t n,
                                                                    int pass, uint32_t* status) {
    if (blockIdx.x >= n) return;
    const GeoBlock b = blocks[blockIdx.x];
    uint32_t err = 0;
    if (pass == 1)
        geo_pass1(requests[b.request], b.bx, b.by, err);
    else
        geo_pass2(requests[b.request], b.bx, b.by, err);
    if (err && status) atomicMax(status, err);
}

// One request, blocks laid out as a 2-D grid.
__global__ void __launch_bounds__(GEO_BW* GEO_BH) geo_single_kernel(const __grid_constant__ GeoRequest R, int pass,
                                                                     uint32_t* status) {
    uint32_t err = 0;
    if (pass == 1)
        geo_pass1(R, blockIdx.x, blockIdx.y, err);
    else
        geo_pass2(R, blockIdx.x, blockIdx.y, err);
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

re_status geo_fail(re_status s, const char* msg) {
    set_last_error(msg);
    return s;
}

re_status finish(cudaStream_t stream, uint32_t* status_dev) {
    uint32_t key = 0;
    cudaError_t e = cudaMemcpyAsync(&key, status_dev, 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        set_last_error(std::string("geometry: ") + cudaGetErrorString(e));
        return RE_CUDA_ERROR;
    }
    if (key) return geo_fail(RE_INVALID_ARGUMENT, "geometry requires finite input within float32 range");
    return RE_OK;
}

struct Scratch {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~Scratch() {
        if (p) cudaFreeAsync(p, s);
    }
};

#define GEO_CUDA(call)                                                        \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) {                                              \
            set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
            return RE_CUDA_ERROR;                                             \
        }                                                                     \
    } while (0)

// Checks a caller's input window against a plan's support.
re_status check_window(const GeoPlan& g, re_rect window, const char* msg) {
    if (g.support.x < window.x || g.support.y < window.y ||
        (uint64_t)g.support.x + g.support.width > (uint64_t)window.x + window.width ||
        (uint64_t)g.support.y + g.support.height > (uint64_t)window.y + window.height)
        return geo_fail(RE_INVALID_ARGUMENT, msg);
    return RE_OK;
}

// Runs a planned request on `stream` (single-request form): device axis
// tables, H and the native scratch of a reduced request in one block.
re_status run_single(const GeoPlan& g, const float* in, size_t in_stride, re_rect window, uint32_t mip, re_rect output,
                     float* out, size_t out_stride, cudaStream_t stream) {
    const size_t axes_bytes = (g.xs.size() + g.ys.size()) * sizeof(Axis);
    const size_t h_bytes = (size_t)g.rows * g.native.width * 3 * sizeof(double);
    const size_t nat_bytes = mip ? (size_t)g.native.width * g.native.height * 3 * sizeof(float) : 0;
    Scratch sc;
    sc.s = stream;
    const size_t a0 = 256, h0 = a0 + ((axes_bytes + 255) & ~(size_t)255), n0 = h0 + ((h_bytes + 255) & ~(size_t)255);
    GEO_CUDA(scratch_alloc(&sc.p, n0 + nat_bytes, stream));
    char* base = (char*)sc.p;
    uint32_t* status = (uint32_t*)base;
    GEO_CUDA(cudaMemsetAsync(status, 0, 4, stream));
    GeoRequest R{};
    R.kind = g.kind;
    R.nx0 = (int)g.native.x;
    R.ny0 = (int)g.native.y;
    R.nw = (int)g.native.width;
    R.nh = (int)g.native.height;
    R.src_x0 = (int)window.x;
    R.src_y0 = (int)window.y;
    R.row0 = (int)g.row0;
    R.rows = (int)g.rows;
    R.rot = g.rot;
    R.src = in;
    R.src_stride = in_stride;
    if (g.kind == 1) {
        Axis* dax = (Axis*)(base + a0);
        GEO_CUDA(cudaMemcpyAsync(dax, g.xs.data(), g.xs.size() * sizeof(Axis), cudaMemcpyHostToDevice, stream));
        GEO_CUDA(cudaMemcpyAsync(dax + g.xs.size(), g.ys.data(), g.ys.size() * sizeof(Axis), cudaMemcpyHostToDevice,
                                 stream));
        R.ax = dax;
        R.ay = dax + g.xs.size();
        R.H = (double*)(base + h0);
    }
    float* nat = (float*)(base + n0);
    R.out = mip ? nat : out;
    R.out_stride = mip ? (uint64_t)g.native.width * 3 : out_stride;
    GEO_CUDA(launch_geometry_single(R, status, stream));
    if (mip) {
        DevProgram P{};
        GEO_CUDA(launch_mip_reduce(nat, (int)g.native.width, (int)g.native.height, (size_t)R.out_stride, (int)mip,
                                   (int)output.width, (int)output.height, 0, 0, P, out, out_stride, status, stream,
                                   nullptr));
    }
    return finish(stream, status);
}

}  // namespace

namespace re {

re_status plan_cubic(uint32_t in_w, uint32_t in_h, uint32_t out_w, uint32_t out_h, re_rect output, uint32_t mip,
                     GeoPlan& g) {
    g = GeoPlan{};
    g.kind = 1;
    if (!in_w || !in_h || !out_w || !out_h)
        return geo_fail(RE_INVALID_ARGUMENT, "cubic resize requires positive input and canvas extents");
    if ((uint64_t)out_w * 4 < in_w || (uint64_t)out_h * 4 < in_h)
        return geo_fail(RE_INVALID_ARGUMENT, "cubic resize native shrink exceeds fourfold per axis");
    if (mip > 2) return geo_fail(RE_INVALID_ARGUMENT, "cubic resize does not support render level");
    if (!native_region(out_w, out_h, output, mip, g.native))
        return geo_fail(RE_OUT_OF_RANGE, "cubic resize output rectangle is outside image");
    if (!output.width || !output.height) return RE_OK;
    g.xs.resize(g.native.width);
    g.ys.resize(g.native.height);
    uint32_t row_lo = in_h, row_hi = 0, col_lo = in_w, col_hi = 0;
    for (uint32_t i = 0; i < g.native.width; ++i) {
        re_status s = cubic_axis(in_w, out_w, g.native.x + i, g.xs[i]);
        if (s) return s;
        const Axis& a = g.xs[i];
        col_lo = std::min(col_lo, a.center);
        col_hi = std::max(col_hi, a.center);
        for (uint32_t k = 0; k < a.count; ++k) {
            col_lo = std::min(col_lo, a.index[k]);
            col_hi = std::max(col_hi, a.index[k]);
        }
    }
    for (uint32_t j = 0; j < g.native.height; ++j) {
        re_status s = cubic_axis(in_h, out_h, g.native.y + j, g.ys[j]);
        if (s) return s;
        const Axis& a = g.ys[j];
        row_lo = std::min(row_lo, a.center);
        row_hi = std::max(row_hi, a.center);
        for (uint32_t k = 0; k < a.count; ++k) {
            row_lo = std::min(row_lo, a.index[k]);
            row_hi = std::max(row_hi, a.index[k]);
        }
    }
    g.row0 = row_lo;
    g.rows = row_hi - row_lo + 1;
    g.support = {col_lo, row_lo, col_hi - col_lo + 1, g.rows};
    return RE_OK;
}

re_status plan_rotate(uint32_t width, uint32_t height, double angle, re_rect output, uint32_t mip, GeoPlan& g,
                      bool exact_support) {
    g = GeoPlan{};
    g.kind = 2;
    if (!width || !height) return geo_fail(RE_INVALID_ARGUMENT, "rotation requires input and nonempty image bounds");
    re_status s = re_rotation_coefficients(angle, &g.rot.cosine, &g.rot.sine);
    if (s) return s;
    if (mip > 2) return geo_fail(RE_INVALID_ARGUMENT, "rotation does not support render level");
    g.rot.cx = (double(width) - 1) / 2;
    g.rot.cy = (double(height) - 1) / 2;
    g.rot.width = (int)width;
    g.rot.height = (int)height;
    if (!native_region(width, height, output, mip, g.native))
        return geo_fail(RE_OUT_OF_RANGE, "rotation output rectangle is outside image");
    if (!output.width || !output.height) return RE_OK;
    if (exact_support) return rotate_support_host(g.rot, g.native, g.support);
    // The source coordinates are an affine function of the output pixel,
    // evaluated with a few roundings (relative error ~1e-16), so over the
    // native rectangle they lie within a hair of the range spanned at its four
    // corners: floor() moves by at most one and the second tap adds one more.
    // Two pixels of margin on each side (clipped to the image) therefore cover
    // every tap.
    double lo_x = 1e300, hi_x = -1e300, lo_y = 1e300, hi_y = -1e300;
    for (int k = 0; k < 4; ++k) {
        const double x = double(g.native.x) + ((k & 1) ? g.native.width - 1 : 0);
        const double y = double(g.native.y) + ((k & 2) ? g.native.height - 1 : 0);
        const double dx = x - g.rot.cx, dy = y - g.rot.cy;
        const double sx = (g.rot.cx + g.rot.cosine * dx) + g.rot.sine * dy;
        const double sy = (g.rot.cy - g.rot.sine * dx) + g.rot.cosine * dy;
        lo_x = std::min(lo_x, sx);
        hi_x = std::max(hi_x, sx);
        lo_y = std::min(lo_y, sy);
        hi_y = std::max(hi_y, sy);
    }
    auto clampi = [](double v, uint32_t n) {
        return (uint32_t)std::clamp<double>(std::floor(v), 0.0, double(n) - 1);
    };
    const uint32_t x0 = clampi(lo_x - 2, width), x1 = clampi(hi_x + 2, width);
    const uint32_t y0 = clampi(lo_y - 2, height), y1 = clampi(hi_y + 2, height);
    g.support = {x0, y0, x1 - x0 + 1, y1 - y0 + 1};
    return RE_OK;
}

cudaError_t launch_geometry_batch(const GeoRequest* requests, const GeoBlock* pass1, uint32_t n1,
                                  const GeoBlock* pass2, uint32_t n2, uint32_t* status, cudaStream_t stream) {
    if (n1) geo_batch_kernel<<<n1, GEO_BW * GEO_BH, 0, stream>>>(requests, pass1, n1, 1, status);
    if (n2) geo_batch_kernel<<<n2, GEO_BW * GEO_BH, 0, stream>>>(requests, pass2, n2, 2, status);
    return cudaGetLastError();
}

cudaError_t launch_geometry_single(const GeoRequest& R, uint32_t* status, cudaStream_t stream) {
    if (R.nw <= 0 || R.nh <= 0) return cudaSuccess;
    const unsigned bx = (unsigned)((R.nw + GEO_BW - 1) / GEO_BW);
    if (R.kind == 1) {
        geo_single_kernel<<<dim3(bx, (R.rows + GEO_BH - 1) / GEO_BH), GEO_BW * GEO_BH, 0, stream>>>(R, 1, status);
        geo_single_kernel<<<dim3(bx, (R.nh + GEO_BH - 1) / GEO_BH), GEO_BW * GEO_BH, 0, stream>>>(R, 2, status);
    } else {
        geo_single_kernel<<<dim3(bx, (R.nh + GEO_BH - 1) / GEO_BH), GEO_BW * GEO_BH, 0, stream>>>(R, 1, status);
    }
    return cudaGetLastError();
}

}  // namespace re

extern "C" {

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
    if (!input || !output) return geo_fail(RE_INVALID_ARGUMENT, "cubic resize requires positive input and canvas extents");
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
re_status re_cubic_resize_window(const float* in, size_t in_stride, re_rect window, uint32_t in_w, uint32_t in_h,
                                 uint32_t out_w, uint32_t out_h, re_rect output, uint32_t mip, float* out,
                                 size_t out_stride, void* stream) {
    GeoPlan g;
    re_status s = plan_cubic(in_w, in_h, out_w, out_h, output, mip, g);
    if (s) return s;
    if (!output.width || !output.height) return RE_OK;
    if (!in || !out || in_stride < (size_t)window.width * 3 || out_stride < (size_t)output.width * 3 ||
        (uint64_t)window.x + window.width > in_w || (uint64_t)window.y + window.height > in_h)
        return geo_fail(RE_INVALID_ARGUMENT, "invalid cubic resize buffers");
    s = check_window(g, window, "cubic resize input window does not cover the taps' support");
    if (s) return s;
    return run_single(g, in, in_stride, window, mip, output, out, out_stride, (cudaStream_t)stream);
}

re_status re_cubic_resize(const float* in, size_t in_stride, uint32_t in_w, uint32_t in_h, uint32_t out_w,
                          uint32_t out_h, re_rect output, uint32_t mip, float* out, size_t out_stride, void* stream) {
    return re_cubic_resize_window(in, in_stride, {0, 0, in_w, in_h}, in_w, in_h, out_w, out_h, output, mip, out,
                                  out_stride, stream);
}

// GeometryOps.cpp:42-67
re_status re_rotation_coefficients(double a, double* cosine, double* sine) {
    if (!std::isfinite(a) || a < -180 || a > 180)
        return geo_fail(RE_INVALID_ARGUMENT, "rotation angle_degrees must be finite in [-180,180]");
    if (a == 0) { *cosine = 1; *sine = 0; }
    else if (a == 90) { *cosine = 0; *sine = 1; }
    else if (a == -90) { *cosine = 0; *sine = -1; }
    else if (std::abs(a) == 180) { *cosine = -1; *sine = 0; }
    else {
        const double theta = (a / 180) * 0x1.921fb54442d18p+1;
        *cosine = std::cos(theta);
        *sine = std::sin(theta);
        if (!std::isfinite(*cosine) || !std::isfinite(*sine) || std::abs(*cosine) > 1 || std::abs(*sine) > 1)
            return geo_fail(RE_INVALID_ARGUMENT, "rotation math runtime returned invalid coefficients");
    }
    return RE_OK;
}

re_status re_rotate_window(const float* in, size_t in_stride, re_rect window, uint32_t width, uint32_t height,
                           double angle, re_rect output, uint32_t mip, float* out, size_t out_stride, void* stream) {
    GeoPlan g;
    // a caller's window must cover the exact support (GeometryOps.cpp:99-111)
    const bool whole = !window.x && !window.y && window.width == width && window.height == height;
    re_status s = plan_rotate(width, height, angle, output, mip, g, !whole);
    if (s) return s;
    if (!output.width || !output.height) return RE_OK;
    if (!in || !out || in_stride < (size_t)window.width * 3 || out_stride < (size_t)output.width * 3 ||
        (uint64_t)window.x + window.width > width || (uint64_t)window.y + window.height > height)
        return geo_fail(RE_INVALID_ARGUMENT, "invalid rotation buffers");
    if (!whole) {
        s = check_window(g, window, "rotation input window does not cover the taps' support");
        if (s) return s;
    }
    return run_single(g, in, in_stride, window, mip, output, out, out_stride, (cudaStream_t)stream);
}

re_status re_rotate(const float* in, size_t in_stride, uint32_t width, uint32_t height, double angle,
                    re_rect output, uint32_t mip, float* out, size_t out_stride, void* stream) {
    return re_rotate_window(in, in_stride, {0, 0, width, height}, width, height, angle, output, mip, out, out_stride,
                            stream);
}

}  // extern "C"
