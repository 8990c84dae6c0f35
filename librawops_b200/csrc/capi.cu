// C ABI of the B200 render path: validation and host-side planning with the
// reference's exact rules and exception classes, then fused launches.
//
// Host planning code here (metadata normalization, level bounds, colour
// matrices composed in binary64, curve preparation) follows the reference
// lines cited at each function so that every integer decision and every
// matrix coefficient equals the reference's.
#include <algorithm>
#include <array>
#include <cmath>
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "re_device.cuh"

namespace re {
size_t menon_smem_bytes();
cudaError_t launch_demosaic(uint32_t demosaic, const DevRaw& raw, int ox, int oy, int ow, int oh,
                            int stage_end, const DevProgram& P, float* out, size_t out_stride,
                            uint32_t* status, unsigned long long* ties, cudaStream_t stream,
                            uint32_t* launches, uint8_t* dirs = nullptr);
cudaError_t launch_mip_reduce(const float* native, int nw, int nh, size_t native_stride, int mip,
                              int ow, int oh, int stage_begin, int stage_end, const DevProgram& P,
                              float* out, size_t out_stride, uint32_t* status, cudaStream_t stream,
                              uint32_t* launches);
cudaError_t launch_raster(const float* in, size_t in_stride, int width, int height, int ox, int oy, int ow, int oh,
                          int mip, const DevProgram& P, float* out, size_t out_stride, uint32_t* status,
                          cudaStream_t stream);
}  // namespace re

using namespace re;

namespace {

thread_local std::string g_error;

re_status fail(re_status s, const std::string& msg) {
    g_error = msg;
    return s;
}

re_status cuda_fail(cudaError_t e, const char* where) {
    return fail(RE_CUDA_ERROR, std::string(where) + ": " + cudaGetErrorString(e));
}

}  // namespace

namespace re {
void set_last_error(const std::string& msg) { g_error = msg; }

namespace {
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_mutex;
cudaMemPool_t g_pools[kMaxPoolDevices] = {};

cudaError_t pool_for_current_device(cudaMemPool_t* out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxPoolDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (!g_pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        e = cudaMemPoolCreate(&pool, &props);
        if (e != cudaSuccess) return e;
        uint64_t keep = ~0ull;
        e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return e;
        }
        g_pools[dev] = pool;
    }
    *out = g_pools[dev];
    return cudaSuccess;
}
}  // namespace

cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t stream) {
    cudaMemPool_t pool = nullptr;
    cudaError_t e = pool_for_current_device(&pool);
    if (e != cudaSuccess) return e;
    return cudaMallocFromPoolAsync(p, bytes, pool, stream);
}
}  // namespace re

extern "C" re_status re_release_scratch(void) {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    for (cudaMemPool_t pool : g_pools)
        if (pool) {
            const cudaError_t e = cudaMemPoolTrimTo(pool, 0);
            if (e != cudaSuccess) return cuda_fail(e, "release scratch");
        }
    return RE_OK;
}

namespace {

#define RE_CUDA(call)                                       \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

bool inside(re_rect area, re_rect r) {
    return r.x >= area.x && r.y >= area.y &&
           (uint64_t)r.x + r.width <= (uint64_t)area.x + area.width &&
           (uint64_t)r.y + r.height <= (uint64_t)area.y + area.height;
}

const int k_pattern_colors[4][4] = {{0, 1, 1, 2}, {2, 1, 1, 0}, {1, 0, 2, 1}, {1, 2, 0, 1}};

// ------------------------------------------------------------- colour maths
// RawEngine.cpp:116-219, restated in binary64 in the reference's order.
using M3 = std::array<double, 9>;

M3 mul(const M3& a, const M3& b) {
    M3 o{};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            for (int k = 0; k < 3; ++k) o[r * 3 + c] += a[r * 3 + k] * b[k * 3 + c];
    return o;
}
std::array<double, 3> mulv(const M3& a, const std::array<double, 3>& v) {
    return {a[0] * v[0] + a[1] * v[1] + a[2] * v[2], a[3] * v[0] + a[4] * v[1] + a[5] * v[2],
            a[6] * v[0] + a[7] * v[1] + a[8] * v[2]};
}
bool inv(const M3& m, M3& o) {
    const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                       m[2] * (m[3] * m[7] - m[4] * m[6]);
    if (!std::isfinite(det) || std::abs(det) < 1e-12) return false;
    const double d = 1.0 / det;
    o = {(m[4] * m[8] - m[5] * m[7]) * d, (m[2] * m[7] - m[1] * m[8]) * d,
         (m[1] * m[5] - m[2] * m[4]) * d, (m[5] * m[6] - m[3] * m[8]) * d,
         (m[0] * m[8] - m[2] * m[6]) * d, (m[2] * m[3] - m[0] * m[5]) * d,
         (m[3] * m[7] - m[4] * m[6]) * d, (m[1] * m[6] - m[0] * m[7]) * d,
         (m[0] * m[4] - m[1] * m[3]) * d};
    return true;
}
std::array<double, 3> white(double x, double y) { return {x / y, 1.0, (1.0 - x - y) / y}; }
M3 rgb_to_xyz(const std::array<double, 6>& xy, double wx, double wy) {
    M3 basis{};
    for (int c = 0; c < 3; ++c) {
        const double x = xy[2 * c], y = xy[2 * c + 1];
        basis[c] = x / y;
        basis[3 + c] = 1.0;
        basis[6 + c] = (1.0 - x - y) / y;
    }
    M3 bi;
    inv(basis, bi);
    const auto s = mulv(bi, white(wx, wy));
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) basis[r * 3 + c] *= s[c];
    return basis;
}
// ICC ROMM, ITU-R BT.2020 and sRGB chromaticities (the reference's constants).
const std::array<double, 6> kProPhoto{0.7347, 0.2653, 0.1596, 0.8404, 0.0366, 0.0001};
const std::array<double, 6> kRec2020{0.708, 0.292, 0.170, 0.797, 0.131, 0.046};
const std::array<double, 6> kSrgb{0.640, 0.330, 0.300, 0.600, 0.150, 0.060};
M3 d50_to_d65() {
    const M3 bradford{0.8951, 0.2664, -0.1614, -0.7502, 1.7135, 0.0367, 0.0389, -0.0685, 1.0296};
    const auto d50 = mulv(bradford, white(0.3457, 0.3585));
    const auto d65 = mulv(bradford, white(0.3127, 0.3290));
    const M3 scale{d65[0] / d50[0], 0, 0, 0, d65[1] / d50[1], 0, 0, 0, d65[2] / d50[2]};
    M3 bi;
    inv(bradford, bi);
    return mul(bi, mul(scale, bradford));
}
bool xyz_d50_to_working(uint32_t target, M3& out) {
    M3 t;
    if (target == 0) return inv(rgb_to_xyz(kProPhoto, 0.3457, 0.3585), out);
    if (target == 1) {
        inv(rgb_to_xyz(kRec2020, 0.3127, 0.3290), t);
        out = mul(t, d50_to_d65());
        return true;
    }
    return false;
}

// ------------------------------------------------------------------ handles
}  // namespace

struct re_image {
    re_raw_metadata meta;
    const uint16_t* dev = nullptr;
    bool owned = false;
    DevRaw raw{};
};

struct re_curve_set {
    DevCurveSet* dev = nullptr;
    DevCurveSet host;
};

namespace {

DevRaw make_dev_raw(const re_raw_metadata& m, const uint16_t* dev) {
    DevRaw r{};
    r.samples = dev;
    r.stride = m.row_stride_samples;
    r.ax = (int32_t)m.active_area.x;
    r.ay = (int32_t)m.active_area.y;
    r.aw = (int32_t)m.active_area.width;
    r.ah = (int32_t)m.active_area.height;
    r.phase_x = m.cfa_phase_x;
    r.phase_y = m.cfa_phase_y;
    r.rcp_exact = 0;
    for (int s = 0; s < 4; ++s) {
        r.site_color[s] = k_pattern_colors[m.pattern][s];
        r.black[s] = (float)m.black_levels[s];
        r.span[s] = (float)((int)m.white_levels[s] - (int)m.black_levels[s]);
        // Exhaustive check of the reciprocal quotient against IEEE division for
        // every numerator a 16-bit code can produce at this site.
        const float d = r.span[s], rc = 1.0f / d;
        bool exact = true;
        for (int code = 0; code <= 65535 && exact; ++code) {
            const float n = (float)code - r.black[s];
            const float q0 = n * rc;
            const float res = std::fma(-q0, d, n);
            const float q = std::fma(res, rc, q0);
            const float want = n / d;
            exact = std::memcmp(&q, &want, sizeof(float)) == 0;
        }
        r.rcp[s] = rc;
        if (exact) r.rcp_exact |= 1u << s;
    }
    return r;
}

re_status status_from_key(uint32_t key) {
    if (!key) return RE_OK;
    const uint32_t kind = key & 0xFFu;
    if (kind & ST_GUARD) return fail(RE_DOMAIN_ERROR, "internal bounds guard tripped");
    if (kind & ST_TIMEOUT) return fail(RE_TIMEOUT, "bounded device wait expired");
    if (kind & ST_DOMAIN) return fail(RE_DOMAIN_ERROR, "non-finite value at output boundary");
    if (kind & ST_INVALID)
        return fail(RE_INVALID_ARGUMENT, "extended curves need finite samples within float32 range");
    if (kind & ST_OVERFLOW) return fail(RE_OVERFLOW_ERROR, "guided filter nonfinite intermediate");
    return fail(RE_DOMAIN_ERROR, "device status");
}

re_status build_program(const re_render_desc* d, DevProgram& P) {
    if (!d) return fail(RE_INVALID_ARGUMENT, "render description is null");
    if (d->demosaic > 2) return fail(RE_INVALID_ARGUMENT, "unsupported RAW demosaic algorithm or processing version");
    if (d->count > RE_MAX_STAGES) return fail(RE_LENGTH_ERROR, "too many fused stages");
    if (d->anchor < -1 || d->anchor >= (int32_t)d->count)
        return fail(RE_INVALID_ARGUMENT, "mip anchor is not a stage of this chain");
    std::memset(&P, 0, sizeof(P));
    P.count = d->count;
    P.anchor = d->anchor;
    for (uint32_t i = 0; i < d->count; ++i) {
        const re_stage& s = d->stages[i];
        if (s.kind < RE_STAGE_GAIN3 || s.kind > RE_STAGE_CURVES)
            return fail(RE_INVALID_ARGUMENT, "unknown stage kind");
        if (s.kind == RE_STAGE_CURVES && (s.arg > 3 || !d->curves[s.arg]))
            return fail(RE_INVALID_ARGUMENT, "curves stage without a curve set");
        P.st[i] = s;
        if (s.kind == RE_STAGE_CURVES) {
            // the master curve's lookup scalars and the channel identities travel
            // with the stage (kernel parameters), so the device reads only tables
            const DevCurveSet& h = d->curves[s.arg]->host;
            float* f = P.st[i].f;
            f[0] = h.c[0].identity ? 1.0f : 0.0f;
            f[1] = (float)h.c[0].n;
            f[2] = (float)h.c[0].ncells;
            f[3] = h.c[0].key_grid ? 1.0f : 0.0f;
            std::memcpy(&f[4], &h.c[0].grid_p, sizeof(float));
            std::memcpy(&f[5], &h.c[0].grid_q, sizeof(float));
            for (int c = 0; c < 3; ++c) f[6 + c] = h.c[c + 1].identity ? 1.0f : 0.0f;
        }
    }
    for (int k = 0; k < 4; ++k) P.curves[k] = d->curves[k] ? d->curves[k]->dev : nullptr;
    return RE_OK;
}

struct DeviceScratch {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~DeviceScratch() {
        if (p) cudaFreeAsync(p, s);
    }
};

}  // namespace

extern "C" {

const char* re_last_error(void) { return g_error.c_str(); }
int re_version(void) { return 100; }
int re_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// RawEngine.cpp:223-250
re_status re_raw_metadata_normalize(re_raw_metadata* m, size_t count) {
    if (!m) return fail(RE_INVALID_ARGUMENT, "metadata is null");
    if (!m->width || !m->height || m->pattern > 3 || m->cfa_phase_x > 1 || m->cfa_phase_y > 1)
        return fail(RE_INVALID_ARGUMENT, "invalid RAW dimensions, Bayer pattern, or CFA phase");
    if (m->row_stride_samples == 0) m->row_stride_samples = m->width;
    if (m->row_stride_samples < m->width)
        return fail(RE_INVALID_ARGUMENT, "RAW row stride is smaller than width");
    re_rect& a = m->active_area;
    if (!a.x && !a.y && !a.width && !a.height) a = {0, 0, m->width, m->height};
    if (!a.width || !a.height || (uint64_t)a.x + a.width > m->width ||
        (uint64_t)a.y + a.height > m->height)
        return fail(RE_INVALID_ARGUMENT, "RAW active area is outside the sensor");
    for (int s = 0; s < 4; ++s)
        if (m->white_levels[s] <= m->black_levels[s])
            return fail(RE_INVALID_ARGUMENT, "RAW white level must exceed black level at every site");
    if ((uint64_t)m->row_stride_samples * m->height != count)
        return fail(RE_INVALID_ARGUMENT, "Bayer sample count does not match stride and height");
    return RE_OK;
}

int re_site_index(const re_raw_metadata* m, uint32_t x, uint32_t y) {
    return (int)((((y & 1u) + m->cfa_phase_y) & 1u) * 2u + (((x & 1u) + m->cfa_phase_x) & 1u));
}
int re_cfa_color(const re_raw_metadata* m, uint32_t x, uint32_t y) {
    return k_pattern_colors[m->pattern & 3][re_site_index(m, x, y)];
}

re_status re_image_create(re_raw_metadata* meta, const uint16_t* samples, size_t count, re_image** out) {
    if (!out || !samples) return fail(RE_INVALID_ARGUMENT, "null image arguments");
    re_status s = re_raw_metadata_normalize(meta, count);
    if (s) return s;
    uint16_t* dev = nullptr;
    RE_CUDA(cudaMalloc(&dev, count * sizeof(uint16_t)));
    cudaError_t e = cudaMemcpy(dev, samples, count * sizeof(uint16_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(dev);
        return cuda_fail(e, "upload RAW samples");
    }
    auto* img = new (std::nothrow) re_image;
    if (!img) {
        cudaFree(dev);
        return fail(RE_LENGTH_ERROR, "out of host memory");
    }
    img->meta = *meta;
    img->dev = dev;
    img->owned = true;
    img->raw = make_dev_raw(*meta, dev);
    *out = img;
    return RE_OK;
}

re_status re_image_wrap_device(re_raw_metadata* meta, const uint16_t* device_samples, size_t count,
                               re_image** out) {
    if (!out || !device_samples) return fail(RE_INVALID_ARGUMENT, "null image arguments");
    re_status s = re_raw_metadata_normalize(meta, count);
    if (s) return s;
    auto* img = new (std::nothrow) re_image;
    if (!img) return fail(RE_LENGTH_ERROR, "out of host memory");
    img->meta = *meta;
    img->dev = device_samples;
    img->owned = false;
    img->raw = make_dev_raw(*meta, device_samples);
    *out = img;
    return RE_OK;
}

re_status re_image_destroy(re_image* img) {
    if (!img) return RE_OK;
    if (img->owned && img->dev) cudaFree(const_cast<uint16_t*>(img->dev));
    delete img;
    return RE_OK;
}

re_status re_image_metadata(const re_image* img, re_raw_metadata* out) {
    if (!img || !out) return fail(RE_INVALID_ARGUMENT, "null image");
    *out = img->meta;
    return RE_OK;
}

// RawEngine.cpp:31-43
re_status re_request_bounds(re_rect s, uint32_t mip, uint32_t quality, re_rect* out) {
    if (mip == 0 && (quality == 0 || quality == 1)) {
        *out = s;
        return RE_OK;
    }
    if (mip >= 1 && mip <= 2 && quality == 0) {
        const uint32_t scale = 1u << mip;
        *out = {0, 0, s.width / scale + (s.width % scale != 0), s.height / scale + (s.height % scale != 0)};
        return RE_OK;
    }
    return fail(RE_INVALID_ARGUMENT, "render level is not implemented for these source bounds");
}

// RawEngine.cpp:49-64, 290-297
re_status re_raw_input_region(const re_raw_metadata* m, uint32_t demosaic, re_rect output, re_rect* region) {
    const re_rect a = m->active_area;
    if (!inside(a, output)) return fail(RE_OUT_OF_RANGE, "viewport is outside the active RAW area");
    const uint32_t radius = demosaic >= 1 && a.width > 1 && a.height > 1 ? 6u : 1u;
    const int64_t left = std::max<int64_t>(a.x, (int64_t)output.x - radius);
    const int64_t top = std::max<int64_t>(a.y, (int64_t)output.y - radius);
    const uint64_t right = std::min<uint64_t>((uint64_t)a.x + a.width, (uint64_t)output.x + output.width + radius);
    const uint64_t bottom = std::min<uint64_t>((uint64_t)a.y + a.height, (uint64_t)output.y + output.height + radius);
    *region = {(uint32_t)left, (uint32_t)top, (uint32_t)(right - left), (uint32_t)(bottom - top)};
    return RE_OK;
}

// RawEngine.cpp:563-578
re_status re_mip_native_region(re_rect area, uint32_t mip, re_rect output, re_rect* native) {
    re_rect reduced;
    re_status s = re_request_bounds(area, mip, 0, &reduced);
    if (s) return s;
    if (!inside(reduced, output)) return fail(RE_OUT_OF_RANGE, "viewport is outside the active RAW area");
    const uint64_t scale = 1u << mip;
    const uint64_t left = std::min<uint64_t>((uint64_t)output.x * scale, area.width);
    const uint64_t top = std::min<uint64_t>((uint64_t)output.y * scale, area.height);
    const uint64_t right = std::min<uint64_t>(((uint64_t)output.x + output.width) * scale, area.width);
    const uint64_t bottom = std::min<uint64_t>(((uint64_t)output.y + output.height) * scale, area.height);
    *native = {(uint32_t)(area.x + left), (uint32_t)(area.y + top), (uint32_t)(right - left), (uint32_t)(bottom - top)};
    return RE_OK;
}

// RawEngine.cpp:1399-1411
re_status re_plan_tiles(re_rect vp, uint32_t tile, re_rect* tiles, size_t capacity, size_t* count) {
    if (!tile) return fail(RE_INVALID_ARGUMENT, "callback and tile size are required");
    size_t n = 0;
    const uint64_t right = (uint64_t)vp.x + vp.width, bottom = (uint64_t)vp.y + vp.height;
    for (uint64_t y = vp.y; y < bottom; y += tile)
        for (uint64_t x = vp.x; x < right; x += tile) {
            if (tiles && n < capacity)
                tiles[n] = {(uint32_t)x, (uint32_t)y, (uint32_t)std::min<uint64_t>(tile, right - x),
                            (uint32_t)std::min<uint64_t>(tile, bottom - y)};
            ++n;
        }
    if (count) *count = n;
    return RE_OK;
}

// RawEngine.cpp:502-530
re_status re_camera_to_working_matrix(const double cam[9], uint32_t target, float out[9]) {
    M3 c, ci, w;
    for (int i = 0; i < 9; ++i) {
        if (!std::isfinite(cam[i])) return fail(RE_INVALID_ARGUMENT, "camera-to-XYZ matrix must be finite");
        c[i] = cam[i];
    }
    if (!inv(c, ci)) return fail(RE_INVALID_ARGUMENT, "color matrix is singular");
    if (!xyz_d50_to_working(target, w)) return fail(RE_INVALID_ARGUMENT, "unknown working space");
    const M3 composed = mul(w, c);
    for (int i = 0; i < 9; ++i) {
        if (!std::isfinite(composed[i]) || std::abs(composed[i]) > FLT_MAX)
            return fail(RE_INVALID_ARGUMENT, "composed color matrix exceeds float32 range");
        out[i] = (float)composed[i];
    }
    return RE_OK;
}

// RawEngine.cpp:198-214
re_status re_working_to_srgb_matrix(uint32_t source, float out[9]) {
    M3 si;
    inv(rgb_to_xyz(kSrgb, 0.3127, 0.3290), si);
    M3 m;
    if (source == 0) m = mul(si, mul(d50_to_d65(), rgb_to_xyz(kProPhoto, 0.3457, 0.3585)));
    else if (source == 1) m = mul(si, rgb_to_xyz(kRec2020, 0.3127, 0.3290));
    else return fail(RE_INVALID_ARGUMENT, "unknown working space");
    for (int i = 0; i < 9; ++i) out[i] = (float)m[i];
    return RE_OK;
}

// RawEngine.cpp:216-219
re_status re_working_to_working_matrix(uint32_t source, uint32_t target, float out[9]) {
    M3 s, t, si;
    if (!xyz_d50_to_working(source, s) || !xyz_d50_to_working(target, t))
        return fail(RE_INVALID_ARGUMENT, "unknown working space");
    inv(s, si);
    const M3 m = mul(t, si);
    for (int i = 0; i < 9; ++i) out[i] = (float)m[i];
    return RE_OK;
}

// RawEngine.cpp:465-468
re_status re_exposure_multiplier(float stops, float* out) {
    if (!std::isfinite(stops) || stops < -32.0f || stops > 32.0f)
        return fail(RE_INVALID_ARGUMENT, "exposure stops must be finite and in [-32, 32]");
    *out = std::exp2(stops);
    return RE_OK;
}

// ToneOps.cpp:17-31, 117-122, 795-816: validate, slopes, shape-preserving
// tangents and Bezier controls in binary64, then per-segment float32 tables.
re_status re_curve_set_create(uint32_t interpolation, const uint32_t counts[4], const double* knots,
                              re_curve_set** out) {
    if (!out || !counts || !knots) return fail(RE_INVALID_ARGUMENT, "null curve arguments");
    if (interpolation > 1) return fail(RE_INVALID_ARGUMENT, "extended curves interpolation is unsupported");
    auto* cs = new (std::nothrow) re_curve_set;
    if (!cs) return fail(RE_LENGTH_ERROR, "out of host memory");
    std::memset(&cs->host, 0, sizeof(cs->host));
    const double* k = knots;
    for (int c = 0; c < 4; ++c) {
        const uint32_t n = counts[c];
        DevCurve& d = cs->host.c[c];
        if (n < 2 || n > 256) {
            delete cs;
            return fail(RE_INVALID_ARGUMENT, "curve knot count exceeds selected operation bounds");
        }
        std::vector<double> x(n), y(n), slope(n - 1), tangent(n);
        for (uint32_t i = 0; i < n; ++i) {
            x[i] = k[2 * i];
            y[i] = k[2 * i + 1];
            if (!std::isfinite(x[i]) || !std::isfinite(y[i]) || std::abs(x[i]) > 65536 || std::abs(y[i]) > 65536) {
                delete cs;
                return fail(RE_INVALID_ARGUMENT, "curve coordinates must be finite with magnitude <=65536");
            }
            if (i) {
                if (!(x[i] > x[i - 1])) {
                    delete cs;
                    return fail(RE_INVALID_ARGUMENT, "curve x coordinates must increase strictly");
                }
                const double s = (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
                if (!std::isfinite(s) || std::abs(s) > 65536) {
                    delete cs;
                    return fail(RE_INVALID_ARGUMENT, "curve slope must be finite with magnitude <=65536");
                }
                slope[i - 1] = s;
            }
        }
        k += 2 * n;
        d.n = n;
        d.cubic = interpolation;
        d.identity = 1;
        for (uint32_t i = 0; i < n; ++i)
            if (x[i] != y[i]) d.identity = 0;
        tangent[0] = slope[0];
        for (uint32_t i = 1; i + 1 < n; ++i) {
            const double a = slope[i - 1], b = slope[i];
            tangent[i] = (a == 0 || b == 0 || std::signbit(a) != std::signbit(b))
                             ? 0
                             : std::copysign(std::min(std::abs(a), std::abs(b)), a);
        }
        tangent[n - 1] = slope[n - 2];
        for (uint32_t i = 0; i < n; ++i) {
            const float rn = (float)x[i];
            float ru = rn;
            if ((double)ru < x[i]) ru = std::nextafter(ru, INFINITY);
            d.xf[i] = ru;
            d.xn[i] = rn;
            d.xeq[i] = (double)rn == x[i] ? rn : NAN;
            d.y[i] = (float)y[i];
        }
        for (uint32_t i = 0; i + 1 < n; ++i) {
            const double h = x[i + 1] - x[i];
            const double p0 = y[i] + (h * tangent[i]) / 3, p1 = y[i + 1] - (h * tangent[i + 1]) / 3;
            d.slope[i] = (float)slope[i];
            d.inv_h[i] = (float)(1.0 / h);
            d.coef[i] = make_float4((float)y[i], (float)(3 * (p0 - y[i])), (float)(3 * (y[i] - 2 * p0 + p1)),
                                    (float)(y[i + 1] - y[i] + 3 * (p0 - p1)));
            // cell-lookup records in s = v - x_i: cubic segments with the power
            // basis of t = s/h rescaled in binary64, linear ones (and the
            // extrapolations) as y_i + s*slope like ToneOps.cpp:826
            d.anchor[i] = d.xn[i];
            if (interpolation) {
                const double r = 1.0 / h;
                d.e[0][i] = (float)y[i];
                d.e[1][i] = (float)(3 * (p0 - y[i]) * r);
                d.e[2][i] = (float)(3 * (y[i] - 2 * p0 + p1) * r * r);
                d.e[3][i] = (float)((y[i + 1] - y[i] + 3 * (p0 - p1)) * r * r * r);
            } else {
                d.e[0][i] = d.y[i];
                d.e[1][i] = d.slope[i];
                d.e[2][i] = 0.0f;
                d.e[3][i] = 0.0f;
            }
        }
        auto linear_rec = [&](uint32_t r, uint32_t knot, float s) {
            d.anchor[r] = d.xn[knot];
            d.e[0][r] = d.y[knot];
            d.e[1][r] = s;
            d.e[2][r] = 0.0f;
            d.e[3][r] = 0.0f;
        };
        linear_rec(n - 1, n - 1, d.slope[n - 2]);
        linear_rec(n, 0, d.slope[0]);
        // Segment lookup grids, in one record format: a cell holds the one knot
        // its samples can meet (+inf if none) with the records below and at or
        // above it.  Two grids are tried and the one with fewer cells kept; a
        // curve that fits neither in 4096 cells keeps the binary search.
        //  * key grid: cells uniform in curve_key, so they narrow toward zero
        //    like a tone curve's knots.  The widest cells that put no two knots
        //    in one cell win; the base is the highest that leaves knot 0 alone
        //    in cell 0 (lower samples land there too), and the last knot's cell
        //    is the last (higher samples land there).
        //  * uniform grid over [x0, x_last], cells a quarter of the narrowest
        //    segment: a float sample's computed cell is within one of its true
        //    cell, so the samples reaching cell c lie in cells c-1..c+1, a span
        //    holding at most one knot (x0 for cell 0, x_last for the last).
        std::vector<CurveCell> key_cells, uniform_cells;
        int32_t key_base = 0;
        uint32_t key_shift = 0;
        for (int shift = 30; shift >= 0 && key_cells.empty(); --shift) {
            const int64_t base = (int64_t)curve_key(d.xf[1]) - (int64_t(1) << shift);
            if (base < INT32_MIN) continue;
            auto cell_of = [&](uint32_t i) { return ((int64_t)curve_key(d.xf[i]) - base) >> shift; };
            bool ok = true;
            for (uint32_t i = 1; i < n && ok; ++i)
                ok = cell_of(i) > (i > 1 ? cell_of(i - 1) : 0) && cell_of(i) < CURVE_CELLS;
            if (!ok) continue;
            key_cells.assign((size_t)cell_of(n - 1) + 1, CurveCell{});
            key_cells[0] = CurveCell{d.xf[0], (uint16_t)n, 0};   // below knot 0: left extrapolation
            int64_t prev = 0;
            for (uint32_t i = 1; i < n; ++i) {
                const int64_t c = cell_of(i);
                for (int64_t e = prev + 1; e < c; ++e) key_cells[e] = CurveCell{INFINITY, (uint16_t)(i - 1), (uint16_t)(i - 1)};
                key_cells[c] = CurveCell{d.xf[i], (uint16_t)(i - 1), (uint16_t)i};   // above the last knot: record n-1
                prev = c;
            }
            key_base = (int32_t)base;
            key_shift = (uint32_t)shift;
        }
        const double span = x[n - 1] - x[0];
        double min_h = INFINITY;
        for (uint32_t i = 0; i + 1 < n; ++i) min_h = std::min(min_h, x[i + 1] - x[i]);
        const double cells = std::ceil(span / (0.25 * min_h));
        double dx = 0.0;
        if (cells >= 1 && cells <= CURVE_CELLS) {
            const uint32_t nc = (uint32_t)cells;
            dx = span / nc;
            uniform_cells.resize(nc);
            for (uint32_t c = 0; c < nc; ++c) {
                const double lo = x[0] + (double(c) - 1.0) * dx, hi = x[0] + (double(c) + 2.0) * dx;
                int knot = -1, inside = 0;
                for (uint32_t i = 0; i < n; ++i)
                    if ((double)d.xf[i] >= lo && (double)d.xf[i] < hi) {
                        knot = (int)i;
                        ++inside;
                    }
                if (inside > 1) {
                    uniform_cells.clear();
                    break;
                }
                if (inside) {
                    uniform_cells[c] = CurveCell{d.xf[knot], (uint16_t)(knot ? knot - 1 : (int)n), (uint16_t)knot};
                } else {
                    uint32_t seg = 0;
                    while (seg + 2 < n && (double)d.xf[seg + 1] <= lo) ++seg;
                    uniform_cells[c] = CurveCell{INFINITY, (uint16_t)seg, (uint16_t)seg};
                }
            }
        }
        d.ncells = 0;
        const bool use_key = !key_cells.empty() && (uniform_cells.empty() || key_cells.size() <= uniform_cells.size());
        if (use_key) {
            d.key_grid = 1;
            d.grid_p = (uint32_t)key_base;
            d.grid_q = key_shift;
            d.ncells = (uint32_t)key_cells.size();
            std::copy(key_cells.begin(), key_cells.end(), d.cell);
        } else if (!uniform_cells.empty()) {
            d.key_grid = 0;
            const float x0c = d.xn[0], inv_dx = (float)(1.0 / dx);
            std::memcpy(&d.grid_p, &x0c, sizeof x0c);
            std::memcpy(&d.grid_q, &inv_dx, sizeof inv_dx);
            d.ncells = (uint32_t)uniform_cells.size();
            std::copy(uniform_cells.begin(), uniform_cells.end(), d.cell);
        }
    }
    cudaError_t e = cudaMalloc(&cs->dev, sizeof(DevCurveSet));
    if (e == cudaSuccess) e = cudaMemcpy(cs->dev, &cs->host, sizeof(DevCurveSet), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        if (cs->dev) cudaFree(cs->dev);
        delete cs;
        return cuda_fail(e, "upload curve set");
    }
    *out = cs;
    return RE_OK;
}

re_status re_curve_set_destroy(re_curve_set* cs) {
    if (!cs) return RE_OK;
    if (cs->dev) cudaFree(cs->dev);
    delete cs;
    return RE_OK;
}

re_status re_status_from_device(uint32_t word) { return status_from_key(word); }

// Level/viewport validation of Renderer::render_image (RawEngine.cpp:1426-1431)
// and the mapping of a reduced request onto its native footprint.
static re_status plan_render(const re_image* img, const DevProgram& P, re_rect viewport, uint32_t mip,
                             uint32_t quality, re_rect* native) {
    const re_rect area = img->meta.active_area;
    re_rect level;
    re_status s = re_request_bounds(area, mip, quality, &level);
    if (s) return s;
    if (!inside(level, viewport)) return fail(RE_OUT_OF_RANGE, "viewport is outside the active RAW area");
    if (mip == 0) {
        *native = viewport;
        return RE_OK;
    }
    if (P.anchor < 0) return fail(RE_INVALID_ARGUMENT, "node does not support this render level");
    return re_mip_native_region(area, mip, viewport, native);
}

size_t re_render_scratch_bytes(const re_image* img, const re_render_desc* desc, re_rect viewport, uint32_t mip) {
    if (!img || !desc || mip == 0) return 0;
    DevProgram P;
    if (build_program(desc, P)) return 0;
    re_rect native;
    if (plan_render(img, P, viewport, mip, 0, &native)) return 0;
    return (size_t)native.width * native.height * 3 * sizeof(float);
}

static re_status enqueue_render(const re_image* img, const DevProgram& P, uint32_t demosaic, re_rect viewport,
                                uint32_t mip, re_rect native, float* out, size_t out_stride, uint32_t* status,
                                unsigned long long* ties, void* scratch, cudaStream_t stream, uint32_t* launches) {
    if (mip == 0) {
        RE_CUDA(launch_demosaic(demosaic, img->raw, (int)viewport.x, (int)viewport.y, (int)viewport.width,
                                (int)viewport.height, (int)P.count, P, out, out_stride, status, ties, stream,
                                launches));
        return RE_OK;
    }
    float* nat = static_cast<float*>(scratch);
    const size_t nstride = (size_t)native.width * 3;
    RE_CUDA(launch_demosaic(demosaic, img->raw, (int)native.x, (int)native.y, (int)native.width,
                            (int)native.height, P.anchor + 1, P, nat, nstride, status, ties, stream, launches));
    RE_CUDA(launch_mip_reduce(nat, (int)native.width, (int)native.height, nstride, (int)mip, (int)viewport.width,
                              (int)viewport.height, P.anchor + 1, (int)P.count, P, out, out_stride, status, stream,
                              launches));
    return RE_OK;
}

}  // extern "C"

namespace re {
// Planning shared with entry points defined in other translation units.
re_status render_plan(const re_image* img, const re_render_desc* desc, re_rect viewport, uint32_t mip,
                      uint32_t quality, DevProgram& P, re_rect& native, const DevRaw** raw) {
    re_status s = build_program(desc, P);
    if (s) return s;
    s = plan_render(img, P, viewport, mip, quality, &native);
    if (s) return s;
    *raw = &img->raw;
    return RE_OK;
}
re_status status_key_to_error(uint32_t key) { return status_from_key(key); }
re_status stage_program(const re_render_desc* desc, DevProgram& P) { return build_program(desc, P); }

// An image that owns an already uploaded device plane (metadata normalized by the caller).
re_status image_adopt_device(re_raw_metadata* meta, uint16_t* device_samples, size_t count, re_image** out) {
    re_status s = re_raw_metadata_normalize(meta, count);
    if (s) return s;
    auto* img = new (std::nothrow) re_image;
    if (!img) return fail(RE_LENGTH_ERROR, "out of host memory");
    img->meta = *meta;
    img->dev = device_samples;
    img->owned = true;
    img->raw = make_dev_raw(*meta, device_samples);
    *out = img;
    return RE_OK;
}
}  // namespace re

extern "C" {

re_status re_render_raw_async(const re_image* img, const re_render_desc* desc, re_rect viewport, uint32_t mip,
                              uint32_t quality, float* out, size_t out_stride, uint32_t* device_status,
                              void* scratch, void* stream) {
    if (!img || !out) return fail(RE_INVALID_ARGUMENT, "null render arguments");
    DevProgram P;
    re_status s = build_program(desc, P);
    if (s) return s;
    re_rect native;
    s = plan_render(img, P, viewport, mip, quality, &native);
    if (s) return s;
    if (out_stride < (size_t)viewport.width * 3) return fail(RE_INVALID_ARGUMENT, "output row stride too small");
    if (mip && !scratch) return fail(RE_INVALID_ARGUMENT, "reduced render needs scratch");
    return enqueue_render(img, P, desc->demosaic, viewport, mip, native, out, out_stride, device_status, nullptr,
                          scratch, (cudaStream_t)stream, nullptr);
}

re_status re_render_raw(const re_image* img, const re_render_desc* desc, re_rect viewport, uint32_t mip,
                        uint32_t quality, float* out, size_t out_stride, int out_on_device, void* stream_,
                        re_render_stats* stats) {
    if (!img || (!out && viewport.width && viewport.height)) return fail(RE_INVALID_ARGUMENT, "null render arguments");
    DevProgram P;
    re_status s = build_program(desc, P);
    if (s) return s;
    re_rect native;
    s = plan_render(img, P, viewport, mip, quality, &native);
    if (s) return s;
    if (out_stride < (size_t)viewport.width * 3) return fail(RE_INVALID_ARGUMENT, "output row stride too small");
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (!viewport.width || !viewport.height) return RE_OK;
    cudaStream_t stream = (cudaStream_t)stream_;
    // one scratch block: [status word | tie counter | (host) output | (mip) native]
    const size_t out_bytes = out_on_device ? 0 : (size_t)viewport.width * viewport.height * 3 * sizeof(float);
    const size_t native_bytes = mip ? (size_t)native.width * native.height * 3 * sizeof(float) : 0;
    const size_t head = 256;
    DeviceScratch scratch;
    scratch.s = stream;
    RE_CUDA(scratch_alloc(&scratch.p, head + out_bytes + native_bytes, stream));
    char* base = static_cast<char*>(scratch.p);
    uint32_t* status = reinterpret_cast<uint32_t*>(base);
    unsigned long long* ties = reinterpret_cast<unsigned long long*>(base + 8);
    float* dev_out = out_on_device ? out : reinterpret_cast<float*>(base + head);
    const size_t dev_stride = out_on_device ? out_stride : (size_t)viewport.width * 3;
    void* nat = mip ? base + head + out_bytes : nullptr;
    RE_CUDA(cudaMemsetAsync(base, 0, head, stream));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (stats) {
        RE_CUDA(cudaEventCreate(&e0));
        RE_CUDA(cudaEventCreate(&e1));
        RE_CUDA(cudaEventRecord(e0, stream));
    }
    uint32_t launches = 0;
    s = enqueue_render(img, P, desc->demosaic, viewport, mip, native, dev_out, dev_stride, status,
                       stats ? ties : nullptr, nat, stream, &launches);
    if (s) return s;
    if (stats) RE_CUDA(cudaEventRecord(e1, stream));
    uint64_t head_host[2] = {0, 0};
    RE_CUDA(cudaMemcpyAsync(head_host, base, 16, cudaMemcpyDeviceToHost, stream));
    if (!out_on_device)
        RE_CUDA(cudaMemcpy2DAsync(out, out_stride * sizeof(float), dev_out, dev_stride * sizeof(float),
                                  (size_t)viewport.width * 3 * sizeof(float), viewport.height,
                                  cudaMemcpyDeviceToHost, stream));
    RE_CUDA(cudaStreamSynchronize(stream));
    if (stats) {
        cudaEventElapsedTime(&stats->device_ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        stats->pixels = (uint64_t)viewport.width * viewport.height;
        stats->native_pixels = (uint64_t)native.width * native.height;
        stats->menon_decisions = desc->demosaic >= 1 ? stats->native_pixels / 2 : 0;
        stats->menon_near_ties = head_host[1];
        stats->launches = launches;
    }
    return status_from_key((uint32_t)head_host[0]);
}

// The direction map of a Menon render (viewport pixels, 1 = horizontal).
re_status re_menon_directions(const re_image* img, uint32_t demosaic, re_rect viewport, uint8_t* out,
                              uint64_t* near_ties, void* stream_) {
    if (!img || (!out && viewport.width && viewport.height)) return fail(RE_INVALID_ARGUMENT, "null arguments");
    if (demosaic < 1 || demosaic > 2) return fail(RE_INVALID_ARGUMENT, "directions exist for the Menon policies only");
    if (!inside(img->meta.active_area, viewport)) return fail(RE_OUT_OF_RANGE, "viewport is outside the active RAW area");
    if (near_ties) *near_ties = 0;
    if (!viewport.width || !viewport.height) return RE_OK;
    if (img->raw.aw <= 1 || img->raw.ah <= 1) return fail(RE_INVALID_ARGUMENT, "a singleton active axis is bilinear");
    cudaStream_t stream = (cudaStream_t)stream_;
    DevProgram P;
    std::memset(&P, 0, sizeof(P));
    P.anchor = -1;
    const size_t rgb = (size_t)viewport.width * viewport.height * 3 * sizeof(float);
    DeviceScratch scratch;
    scratch.s = stream;
    RE_CUDA(scratch_alloc(&scratch.p, 256 + rgb, stream));
    char* base = static_cast<char*>(scratch.p);
    RE_CUDA(cudaMemsetAsync(base, 0, 256, stream));
    RE_CUDA(launch_demosaic(demosaic, img->raw, (int)viewport.x, (int)viewport.y, (int)viewport.width,
                            (int)viewport.height, 0, P, reinterpret_cast<float*>(base + 256), (size_t)viewport.width * 3,
                            reinterpret_cast<uint32_t*>(base), reinterpret_cast<unsigned long long*>(base + 8), stream,
                            nullptr, out));
    uint64_t ties = 0;
    RE_CUDA(cudaMemcpyAsync(&ties, base + 8, 8, cudaMemcpyDeviceToHost, stream));
    RE_CUDA(cudaStreamSynchronize(stream));
    if (near_ties) *near_ties = ties;
    return RE_OK;
}

// RasterSourceNode::render_level (RawEngine.cpp:346-406) + fused stages.
re_status re_render_raster(const float* in, size_t in_stride, uint32_t width, uint32_t height,
                           const re_render_desc* desc, re_rect viewport, uint32_t mip, uint32_t quality, float* out,
                           size_t out_stride, void* stream_) {
    DevProgram P;
    re_status s = build_program(desc, P);
    if (s) return s;
    if (!width || !height) return fail(RE_INVALID_ARGUMENT, "invalid scene-linear raster metadata");
    re_rect level;
    s = re_request_bounds({0, 0, width, height}, mip, quality, &level);
    if (s) return fail(RE_INVALID_ARGUMENT, "raster source does not support this render level");
    if (!inside(level, viewport)) return fail(RE_OUT_OF_RANGE, "viewport is outside the active RAW area");
    if (!viewport.width || !viewport.height) return RE_OK;
    if (!in || !out || in_stride < (size_t)width * 3 || out_stride < (size_t)viewport.width * 3)
        return fail(RE_INVALID_ARGUMENT, "invalid raster buffers");
    cudaStream_t stream = (cudaStream_t)stream_;
    DeviceScratch scratch;
    scratch.s = stream;
    RE_CUDA(scratch_alloc(&scratch.p, 256, stream));
    uint32_t* status = static_cast<uint32_t*>(scratch.p);
    RE_CUDA(cudaMemsetAsync(status, 0, 4, stream));
    RE_CUDA(launch_raster(in, in_stride, (int)width, (int)height, (int)viewport.x, (int)viewport.y,
                          (int)viewport.width, (int)viewport.height, (int)mip, P, out, out_stride, status, stream));
    uint32_t key = 0;
    RE_CUDA(cudaMemcpyAsync(&key, status, 4, cudaMemcpyDeviceToHost, stream));
    RE_CUDA(cudaStreamSynchronize(stream));
    return status_from_key(key);
}

// Renderer::render_tiles (RawEngine.cpp:1390-1412): tile loop in the
// reference's order, one fused render per tile, callback per tile.
re_status re_render_tiles(const re_image* img, const re_render_desc* desc, re_rect viewport, uint32_t tile_size,
                          uint32_t mip, uint32_t quality, re_tile_callback callback, void* user, void* stream) {
    if (!img) return fail(RE_INVALID_ARGUMENT, "null image");
    DevProgram P;
    re_status s = build_program(desc, P);
    if (s) return s;
    re_rect native;
    s = plan_render(img, P, viewport, mip, quality, &native);
    if (s) return s;
    if (!callback || !tile_size) return fail(RE_INVALID_ARGUMENT, "callback and tile size are required");
    std::vector<float> host((size_t)std::min<uint64_t>(tile_size, viewport.width) *
                            std::min<uint64_t>(tile_size, viewport.height) * 3);
    const uint64_t right = (uint64_t)viewport.x + viewport.width, bottom = (uint64_t)viewport.y + viewport.height;
    for (uint64_t y = viewport.y; y < bottom; y += tile_size)
        for (uint64_t x = viewport.x; x < right; x += tile_size) {
            const re_rect r{(uint32_t)x, (uint32_t)y, (uint32_t)std::min<uint64_t>(tile_size, right - x),
                            (uint32_t)std::min<uint64_t>(tile_size, bottom - y)};
            s = re_render_raw(img, desc, r, mip, quality, host.data(), (size_t)r.width * 3, 0, stream, nullptr);
            if (s) return s;
            if (callback(&r, host.data(), user)) return fail(RE_CANCELLED, "render cancelled");
        }
    return RE_OK;
}

}  // extern "C"
