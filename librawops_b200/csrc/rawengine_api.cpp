// Drop-in C++ surface (include/rawengine/*.hpp) over the C ABI.
//
// Node constructors validate exactly what the reference's constructors
// validate (RawEngine.cpp, SpatialOps.cpp, ToneOps.cpp, GeometryOps.cpp of
// tylermcm/librawops) and throw the same exception classes.  Rendering goes
// through `Executor::eval`, which walks a node chain from the requested node
// downward and turns it into device work:
//   * point nodes (white balance, exposure, matrices, tone, curves, clip,
//     sRGB) become stages of one fused launch, together with the RAW demosaic
//     or raster source below them (CameraToWorking is the mip anchor);
//   * guided filter, cubic resize and rotate render their input footprint
//     into device memory, run their own kernels, and feed any point stages
//     above them through the raster kernel;
//   * any other Node (a caller's subclass) is pulled through its own
//     render_level, validated like the reference validates upstream tiles,
//     and uploaded.
// Results do not depend on the render tile size, so Renderer::render_image
// renders a whole viewport in one pass while render_tiles keeps the
// reference's per-tile loop and callback order.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <limits>
#include <list>
#include <map>
#include <mutex>
#include <queue>
#include <thread>

#include <cuda_runtime.h>

#include "rawengine/EditOps.hpp"
#include "rawengine/ImageAnalysis.hpp"
#include "rawengine/Operators.hpp"
#include "rawengine_b200.h"

namespace re {
// The library's stream-ordered scratch pool (capi.cu).
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t stream);
}  // namespace re

namespace rawengine {

// ------------------------------------------------------------- errors

namespace {

[[noreturn]] void throw_status(re_status s) {
    const std::string msg = re_last_error();
    switch (s) {
    case RE_OUT_OF_RANGE: throw std::out_of_range(msg);
    case RE_DOMAIN_ERROR: throw std::domain_error(msg);
    case RE_LENGTH_ERROR: throw std::length_error(msg);
    case RE_OVERFLOW_ERROR: throw std::overflow_error(msg);
    case RE_CANCELLED: throw RenderCancelled();
    case RE_INVALID_ARGUMENT: throw std::invalid_argument(msg);
    default: throw std::runtime_error(msg);
    }
}

void check(re_status s) {
    if (s != RE_OK) throw_status(s);
}

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

re_rect to_re(Rect r) { return {r.x, r.y, r.width, r.height}; }

bool level_native(RenderLevel l) { return l.mip == 0 && l.quality == RenderQuality::Final; }
bool level_any_native(RenderLevel l) {
    return l.mip == 0 && (l.quality == RenderQuality::Final || l.quality == RenderQuality::Preview);
}
bool level_reduced(RenderLevel l) { return l.mip >= 1 && l.mip <= 2 && l.quality == RenderQuality::Preview; }

bool addressable(Rect r) {
    return (uint64_t)r.x + r.width <= (1ull << 32) && (uint64_t)r.y + r.height <= (1ull << 32);
}
bool contains(Rect area, Rect r) {
    return r.x >= area.x && r.y >= area.y && (uint64_t)r.x + r.width <= (uint64_t)area.x + area.width &&
           (uint64_t)r.y + r.height <= (uint64_t)area.y + area.height;
}
bool same(Rect a, Rect b) { return a.x == b.x && a.y == b.y && a.width == b.width && a.height == b.height; }

// RawEngine.cpp:31-43
Rect request_bounds(Rect s, RenderLevel level) {
    re_rect out;
    check(re_request_bounds(to_re(s), level.mip, (uint32_t)level.quality, &out));
    return {out.x, out.y, out.width, out.height};
}

// Scene-linear working descriptor check used by the spatial/curve/geometry nodes.
bool scene_linear(const ImageDescriptor& d) {
    return d == ImageDescriptor::scene_linear(WorkingSpace::LinearProPhotoD50) ||
           d == ImageDescriptor::scene_linear(WorkingSpace::LinearRec2020D65);
}

uint32_t space_code(const ImageDescriptor& d) {
    return d == ImageDescriptor::scene_linear(WorkingSpace::LinearRec2020D65) ? 1u : 0u;
}

// Per-thread stream used by the executor (TileScheduler workers each get their own).
cudaStream_t thread_stream() {
    thread_local cudaStream_t stream = [] {
        cudaStream_t s = nullptr;
        check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
        return s;
    }();
    return stream;
}

}  // namespace

// ------------------------------------------------------------- sources

struct DeviceRaw {
    std::once_flag once;
    re_image* handle = nullptr;
    ~DeviceRaw() {
        if (handle) re_image_destroy(handle);
    }
};

struct DeviceRaster {
    std::once_flag once;
    float* data = nullptr;
    size_t stride = 0;  // floats
    ~DeviceRaster() {
        if (data) cudaFree(data);
    }
};

namespace {
re_raw_metadata to_re(const RawMetadata& m) {
    re_raw_metadata r{};
    r.width = m.width;
    r.height = m.height;
    r.row_stride_samples = m.row_stride_samples;
    r.pattern = (uint32_t)m.pattern;
    r.cfa_phase_x = m.cfa_phase_x;
    r.cfa_phase_y = m.cfa_phase_y;
    r.active_area = to_re(m.active_area);
    for (int i = 0; i < 4; ++i) {
        r.black_levels[i] = m.black_levels[i];
        r.white_levels[i] = m.white_levels[i];
    }
    return r;
}
}  // namespace

// RawEngine.cpp:223-250 (validation and normalization of the metadata)
RawImage::RawImage(RawMetadata metadata, std::vector<std::uint16_t> samples)
    : metadata_(metadata),
      bayer_(std::make_shared<const std::vector<std::uint16_t>>(std::move(samples))),
      device_(std::make_shared<DeviceRaw>()) {
    if ((int)metadata_.pattern < 0 || (int)metadata_.pattern > 3)
        throw std::invalid_argument("invalid RAW dimensions, Bayer pattern, or CFA phase");
    re_raw_metadata m = to_re(metadata_);
    check(re_raw_metadata_normalize(&m, bayer_->size()));
    metadata_.row_stride_samples = m.row_stride_samples;
    metadata_.active_area = {m.active_area.x, m.active_area.y, m.active_area.width, m.active_area.height};
}

RawImage::RawImage(std::uint32_t width, std::uint32_t height, std::vector<std::uint16_t> samples,
                   BayerPattern pattern, std::uint16_t black, std::uint16_t white)
    : RawImage(
          [&] {
              RawMetadata m;
              m.width = width;
              m.height = height;
              m.pattern = pattern;
              m.black_levels.fill(black);
              m.white_levels.fill(white);
              return m;
          }(),
          std::move(samples)) {}

const DeviceRaw& RawImage::device() const {
    std::call_once(device_->once, [&] {
        re_raw_metadata m = to_re(metadata_);
        check(re_image_create(&m, bayer_->data(), bayer_->size(), &device_->handle));
    });
    if (!device_->handle) throw std::runtime_error("RAW image upload failed");
    return *device_;
}

// RawEngine.cpp:258-274
RasterImage::RasterImage(RasterMetadata metadata, std::vector<float> pixels)
    : metadata_(metadata), pixels_(std::make_shared<const std::vector<float>>(std::move(pixels))),
      device_(std::make_shared<DeviceRaster>()) {
    if (!metadata_.width || !metadata_.height ||
        (metadata_.working_space != WorkingSpace::LinearProPhotoD50 &&
         metadata_.working_space != WorkingSpace::LinearRec2020D65))
        throw std::invalid_argument("invalid scene-linear raster metadata");
    if (!metadata_.row_stride_pixels) metadata_.row_stride_pixels = metadata_.width;
    if (metadata_.row_stride_pixels < metadata_.width ||
        pixels_->size() != (size_t)metadata_.row_stride_pixels * metadata_.height * 3)
        throw std::invalid_argument("raster float count does not match stride and height");
    for (float v : *pixels_)
        if (!std::isfinite(v)) throw std::invalid_argument("scene-linear raster pixels must be finite");
}

const DeviceRaster& RasterImage::device() const {
    std::call_once(device_->once, [&] {
        const size_t bytes = pixels_->size() * sizeof(float);
        check_cuda(cudaMalloc(&device_->data, bytes), "raster upload");
        check_cuda(cudaMemcpy(device_->data, pixels_->data(), bytes, cudaMemcpyHostToDevice), "raster upload");
        device_->stride = (size_t)metadata_.row_stride_pixels * 3;
    });
    if (!device_->data) throw std::runtime_error("raster upload failed");
    return *device_;
}

// RawEngine.cpp:276-280
void validate_raw_demosaic(const RawDemosaicIdentity& identity) {
    if ((identity.algorithm != "rawengine.bilinear" && identity.algorithm != "rawengine.menon_base") ||
        identity.processing_version != 1)
        throw std::invalid_argument("unsupported RAW demosaic algorithm or processing version");
}

RawUnpackNode::RawUnpackNode(RawImage image) : RawUnpackNode(std::move(image), RawDemosaicIdentity{}) {}
RawUnpackNode::RawUnpackNode(RawImage image, RawDemosaicIdentity demosaic)
    : image_(std::move(image)), demosaic_(std::move(demosaic)) {
    validate_raw_demosaic(demosaic_);
}
bool RawUnpackNode::menon() const noexcept { return demosaic_.algorithm == "rawengine.menon_base"; }

// RawEngine.cpp:290-297
Rect RawUnpackNode::input_region(Rect output, Rect source_bounds) const {
    if (!same(source_bounds, image_.metadata().active_area))
        throw std::invalid_argument("RAW source bounds differ from active area");
    re_raw_metadata m = to_re(image_.metadata());
    re_rect out;
    check(re_raw_input_region(&m, menon() ? 1u : 0u, to_re(output), &out));
    return {out.x, out.y, out.width, out.height};
}

RasterSourceNode::RasterSourceNode(RasterImage image) : image_(std::move(image)) {}
bool RasterSourceNode::supports_level(RenderLevel level) const noexcept {
    return level_any_native(level) || level_reduced(level);
}
Rect RasterSourceNode::input_region_level(Rect output, Rect, RenderLevel level) const {
    if (!supports_level(level)) throw std::invalid_argument("raster source has no mapping for this render level");
    return output;
}

// ------------------------------------------------------------ point nodes

// RawEngine.cpp:408-415
WhiteBalanceNode::WhiteBalanceNode(std::shared_ptr<const Node> input, float red, float green, float blue)
    : PointNode(std::move(input)), gains_{red, green, blue} {
    if (!input_) throw std::invalid_argument("white balance input is null");
    if (input_->output_descriptor() != ImageDescriptor::camera_linear())
        throw std::invalid_argument("white balance requires camera-linear RGB input");
    for (float g : gains_)
        if (!std::isfinite(g) || g <= 0.0f || g > 65536.0f)
            throw std::invalid_argument("white balance gains must be finite and in (0, 65536]");
}

// RawEngine.cpp:465-486
ExposureNode::ExposureNode(std::shared_ptr<const Node> input, float stops)
    : PointNode(std::move(input)), multiplier_(std::exp2(stops)) {
    if (!input_ || !std::isfinite(stops) || stops < -32.0f || stops > 32.0f)
        throw std::invalid_argument("exposure stops must be finite and in [-32, 32]");
    descriptor_ = input_->output_descriptor();
    if (descriptor_ != ImageDescriptor::camera_linear() && !scene_linear(descriptor_))
        throw std::invalid_argument("exposure requires linear RGB input");
}
bool ExposureNode::supports_level(RenderLevel level) const noexcept {
    if (level_native(level)) return true;
    return level_reduced(level) && descriptor_.domain == PixelDomain::SceneLinearRGB && input_->supports_level(level);
}
Rect ExposureNode::input_region_level(Rect output, Rect, RenderLevel level) const {
    if (!supports_level(level)) throw std::invalid_argument("exposure has no mapping for this render level");
    return output;
}

// RawEngine.cpp:502-578
CameraToWorkingNode::CameraToWorkingNode(std::shared_ptr<const Node> input, CameraColorTransform transform,
                                         Rect native_input_bounds)
    : PointNode(std::move(input)), descriptor_(ImageDescriptor::scene_linear(transform.target)),
      native_input_bounds_(native_input_bounds) {
    if (!input_ || input_->output_descriptor() != ImageDescriptor::camera_linear())
        throw std::invalid_argument("color transform requires camera-linear RGB input");
    const auto b = native_input_bounds_;
    if ((b.width == 0) != (b.height == 0) || (!b.width && (b.x || b.y)) || !addressable(b))
        throw std::invalid_argument("invalid camera preview input bounds");
    for (double v : transform.camera_to_xyz_d50)
        if (!std::isfinite(v)) throw std::invalid_argument("camera-to-XYZ matrix must be finite");
    check(re_camera_to_working_matrix(transform.camera_to_xyz_d50.data(), (uint32_t)transform.target,
                                      matrix_.data()));
}
bool CameraToWorkingNode::supports_level(RenderLevel level) const noexcept {
    if (level_native(level)) return input_->supports_level(level);
    return level_reduced(level) && native_input_bounds_.width && native_input_bounds_.height &&
           input_->supports_level({});
}
RenderLevel CameraToWorkingNode::input_level(RenderLevel level) const {
    if (!supports_level(level)) throw std::invalid_argument("camera calibration has no mapping for this level");
    return {};
}
Rect CameraToWorkingNode::input_region_level(Rect output, Rect input_bounds, RenderLevel level) const {
    if (!supports_level(level)) throw std::invalid_argument("camera calibration has no mapping for this level");
    if (!level.mip) return output;
    if (!same(input_bounds, native_input_bounds_))
        throw std::invalid_argument("camera preview input bounds differ from construction");
    re_rect native;
    check(re_mip_native_region(to_re(native_input_bounds_), level.mip, to_re(output), &native));
    return {native.x, native.y, native.width, native.height};
}

// RawEngine.cpp:603-623
WorkingSpaceConvertNode::WorkingSpaceConvertNode(std::shared_ptr<const Node> input, WorkingSpace target)
    : PointNode(std::move(input)), descriptor_(ImageDescriptor::scene_linear(target)) {
    if (!input_) throw std::invalid_argument("working-space conversion input is null");
    const auto d = input_->output_descriptor();
    if (!scene_linear(d)) throw std::invalid_argument("working-space conversion requires declared scene-linear RGB");
    if (target != WorkingSpace::LinearProPhotoD50 && target != WorkingSpace::LinearRec2020D65)
        throw std::invalid_argument("unknown working space");
    const uint32_t source = space_code(d);
    identity_ = source == (uint32_t)target;
    if (!identity_) check(re_working_to_working_matrix(source, (uint32_t)target, matrix_.data()));
}
bool WorkingSpaceConvertNode::supports_level(RenderLevel level) const noexcept {
    if (level_native(level)) return true;
    return level_reduced(level) && input_->supports_level(level);
}
Rect WorkingSpaceConvertNode::input_region_level(Rect output, Rect, RenderLevel level) const {
    if (!supports_level(level))
        throw std::invalid_argument("working-space conversion has no mapping for this render level");
    return output;
}

// RawEngine.cpp:658-672
WorkingToSrgbNode::WorkingToSrgbNode(std::shared_ptr<const Node> input) : PointNode(std::move(input)) {
    if (!input_) throw std::invalid_argument("working-to-sRGB input is null");
    const auto d = input_->output_descriptor();
    if (!scene_linear(d)) throw std::invalid_argument("sRGB conversion requires declared scene-linear working RGB");
    check(re_working_to_srgb_matrix(space_code(d), matrix_.data()));
}
bool WorkingToSrgbNode::supports_level(RenderLevel level) const noexcept {
    if (level_native(level)) return true;
    return level_reduced(level) && input_->supports_level(level);
}
Rect WorkingToSrgbNode::input_region_level(Rect output, Rect, RenderLevel level) const {
    if (!supports_level(level)) throw std::invalid_argument("sRGB preview stage has no mapping for this render level");
    return output;
}

// RawEngine.cpp:705-736
ToneCurveNode::ToneCurveNode(std::shared_ptr<const Node> input, float shoulder, float gamma)
    : PointNode(std::move(input)), shoulder_(shoulder), inverse_gamma_(1.0f / gamma) {
    if (!input_ || !std::isfinite(shoulder) || shoulder <= 0.0f || !std::isfinite(gamma) || gamma <= 0.0f ||
        !std::isfinite(inverse_gamma_))
        throw std::invalid_argument("tone shoulder and gamma must be finite and positive");
    const auto source = input_->output_descriptor();
    if (source != ImageDescriptor::camera_linear() && !scene_linear(source) &&
        source != ImageDescriptor::linear_srgb())
        throw std::invalid_argument("tone curve requires linear RGB input");
    if (source == ImageDescriptor::linear_srgb()) {
        descriptor_ = ImageDescriptor::display_linear_srgb();
    } else {
        descriptor_ = ImageDescriptor::tone_mapped();
        descriptor_.primaries = source.primaries;
        descriptor_.white_point = source.white_point;
    }
}
bool ToneCurveNode::supports_level(RenderLevel level) const noexcept {
    if (level_native(level)) return true;
    return level_reduced(level) && input_->output_descriptor() == ImageDescriptor::linear_srgb() &&
           input_->supports_level(level);
}
Rect ToneCurveNode::input_region_level(Rect output, Rect, RenderLevel level) const {
    if (!supports_level(level)) throw std::invalid_argument("sRGB preview stage has no mapping for this render level");
    return output;
}

// RawEngine.cpp:1215-1221
OutputClipNode::OutputClipNode(std::shared_ptr<const Node> input) : PointNode(std::move(input)) {
    if (!input_ || input_->output_descriptor().domain != PixelDomain::ToneMappedUnmanagedRGB)
        throw std::invalid_argument("output clip requires tone-mapped RGB input");
    descriptor_ = input_->output_descriptor();
    descriptor_.domain = PixelDomain::BoundedUnmanagedRGB;
}

// RawEngine.cpp:1235-1252
SrgbEncodeNode::SrgbEncodeNode(std::shared_ptr<const Node> input) : PointNode(std::move(input)) {
    if (!input_) throw std::invalid_argument("sRGB encode input is null");
    if (input_->output_descriptor() != ImageDescriptor::display_linear_srgb())
        throw std::invalid_argument("sRGB encode requires display-linear sRGB input");
}
bool SrgbEncodeNode::supports_level(RenderLevel level) const noexcept {
    if (level_native(level)) return true;
    return level_reduced(level) && input_->supports_level(level);
}
Rect SrgbEncodeNode::input_region_level(Rect output, Rect, RenderLevel level) const {
    if (!supports_level(level)) throw std::invalid_argument("sRGB preview stage has no mapping for this render level");
    return output;
}

// ------------------------------------------------------------------ curves

struct CurveTables {
    re_curve_set* set = nullptr;
    ~CurveTables() {
        if (set) re_curve_set_destroy(set);
    }
};

// ToneOps.cpp:17-31, 117-122
void validate_extended_curves_settings(const ExtendedCurvesSettings& s) {
    if (s.interpolation != CurveInterpolation::Linear && s.interpolation != CurveInterpolation::ShapePreservingCubic)
        throw std::invalid_argument("extended curves interpolation is unsupported");
    auto one = [](const CurveKnots& c) {
        if (c.knots.size() < 2 || c.knots.size() > 256)
            throw std::invalid_argument("curve knot count exceeds selected operation bounds");
        for (size_t i = 0; i < c.knots.size(); ++i) {
            const auto& p = c.knots[i];
            if (!std::isfinite(p.x) || !std::isfinite(p.y) || std::abs(p.x) > 65536 || std::abs(p.y) > 65536)
                throw std::invalid_argument("curve coordinates must be finite with magnitude <=65536");
            if (i) {
                const auto& q = c.knots[i - 1];
                if (!(p.x > q.x)) throw std::invalid_argument("curve x coordinates must increase strictly");
                const double slope = (p.y - q.y) / (p.x - q.x);
                if (!std::isfinite(slope) || std::abs(slope) > 65536)
                    throw std::invalid_argument("curve slope must be finite with magnitude <=65536");
            }
        }
    };
    one(s.master);
    for (const auto& c : s.channels) one(c);
}

// ToneOps.cpp:795-816, 817-820
ExtendedCurvesNode::ExtendedCurvesNode(std::shared_ptr<const Node> input, ExtendedCurvesSettings settings)
    : PointNode(std::move(input)), settings_(std::move(settings)), tables_(std::make_shared<CurveTables>()) {
    validate_extended_curves_settings(settings_);
    if (!input_ || !scene_linear(input_->output_descriptor()))
        throw std::invalid_argument("extended curves/levels require scene-linear working RGB");
    uint32_t counts[4];
    std::vector<double> knots;
    const CurveKnots* all[4] = {&settings_.master, &settings_.channels[0], &settings_.channels[1],
                                &settings_.channels[2]};
    for (int k = 0; k < 4; ++k) {
        counts[k] = (uint32_t)all[k]->knots.size();
        for (const auto& p : all[k]->knots) {
            knots.push_back(p.x);
            knots.push_back(p.y);
        }
    }
    check(re_curve_set_create(settings_.interpolation == CurveInterpolation::ShapePreservingCubic ? 1u : 0u, counts,
                              knots.data(), &tables_->set));
}
bool ExtendedCurvesNode::supports_level(RenderLevel level) const noexcept {
    return (level_any_native(level) || level_reduced(level)) && input_->supports_level(level);
}
Rect ExtendedCurvesNode::input_region_level(Rect r, Rect, RenderLevel level) const {
    if (!supports_level(level)) throw std::invalid_argument("extended curves do not support this render level");
    return r;
}

// -------------------------------------------------------------- SpatialOps

namespace {
// SpatialOps.cpp:14-41
void bounded_rect(Rect r) {
    if (!r.width || !r.height || !addressable(r))
        throw std::invalid_argument("spatial operation requires nonempty addressable bounds");
}
Rect spatial_expanded(Rect r, Rect image, uint32_t rx, uint32_t ry) {
    bounded_rect(r);
    bounded_rect(image);
    if (!contains(image, r)) throw std::out_of_range("spatial viewport is outside image bounds");
    const int64_t left = std::max<int64_t>(image.x, (int64_t)r.x - rx);
    const int64_t top = std::max<int64_t>(image.y, (int64_t)r.y - ry);
    const uint64_t right = std::min<uint64_t>((uint64_t)image.x + image.width, (uint64_t)r.x + r.width + rx);
    const uint64_t bottom = std::min<uint64_t>((uint64_t)image.y + image.height, (uint64_t)r.y + r.height + ry);
    return {(uint32_t)left, (uint32_t)top, (uint32_t)(right - left), (uint32_t)(bottom - top)};
}
Rect level_bounds(Rect native, RenderLevel level) {
    bounded_rect(native);
    if (level_any_native(level)) return native;
    if (!level_reduced(level)) throw std::invalid_argument("unsupported spatial render level");
    const uint32_t s = 1u << level.mip;
    return {0, 0, native.width / s + (native.width % s != 0), native.height / s + (native.height % s != 0)};
}
}  // namespace

void validate_working_y_guided_filter_settings(const WorkingYGuidedFilterSettings& s) {
    if (s.radius > 8 || !std::isfinite(s.epsilon) || s.epsilon < 0x1p-24 || s.epsilon > 65536.0)
        throw std::invalid_argument("guided filter requires radius 0..8 and finite epsilon [2^-24,65536]");
}
Rect working_y_guided_filter_region(Rect output, Rect image_bounds, std::uint32_t radius) {
    if (radius > 8) throw std::invalid_argument("guided filter radius must be 0..8");
    return spatial_expanded(output, image_bounds, 2 * radius, 2 * radius);
}
Rect local_statistics_region(Rect output, Rect image_bounds, std::uint32_t radius) {
    if (radius > 8) throw std::invalid_argument("local statistics radius must be in 0..8");
    return spatial_expanded(output, image_bounds, radius, radius);
}

WorkingYGuidedFilterNode::WorkingYGuidedFilterNode(std::shared_ptr<const Node> input, Rect native_bounds,
                                                   WorkingYGuidedFilterSettings settings)
    : input_(std::move(input)), native_bounds_(native_bounds), settings_(settings) {
    bounded_rect(native_bounds_);
    validate_working_y_guided_filter_settings(settings_);
    if (!input_) throw std::invalid_argument("guided filter requires input");
    descriptor_ = input_->output_descriptor();
    if (!scene_linear(descriptor_)) throw std::invalid_argument("guided filter requires scene-linear working RGB");
}
bool WorkingYGuidedFilterNode::supports_level(RenderLevel level) const noexcept {
    return (level_any_native(level) || level_reduced(level)) && input_->supports_level(level);
}
Rect WorkingYGuidedFilterNode::input_region(Rect output, Rect source_bounds) const {
    return input_region_level(output, source_bounds, {});
}
Rect WorkingYGuidedFilterNode::input_region_level(Rect output, Rect source_bounds, RenderLevel level) const {
    const Rect image = level_bounds(native_bounds_, level);
    if (!same(source_bounds, image) || !supports_level(level))
        throw std::invalid_argument("guided filter source bounds or level differ");
    return working_y_guided_filter_region(output, image, settings_.radius);
}

// ------------------------------------------------------------- stencils

// SpatialOps.cpp:319-327, 386-390, 496-500, 621-624
void validate_convolution_kernel(const ConvolutionKernel& k) {
    if (!k.width || !k.height || k.width > 17 || k.height > 17 || k.width % 2 != 1 || k.height % 2 != 1 ||
        k.coefficients.size() != (size_t)k.width * k.height)
        throw std::invalid_argument("convolution kernel needs odd dimensions 1..17 and matching coefficients");
    for (double v : k.coefficients)
        if (!std::isfinite(v) || std::abs(v) > 65536)
            throw std::invalid_argument("convolution coefficients must be finite with magnitude <=65536");
}
void validate_clarity_settings(const ClaritySettings& s) {
    if (!std::isfinite(s.amount) || std::abs(s.amount) > 1 || s.radius < 1 || s.radius > 8)
        throw std::invalid_argument("clarity requires finite amount [-1,1] and radius 1..8");
}
void validate_texture_settings(const TextureSettings& s) {
    if (!std::isfinite(s.amount) || std::abs(s.amount) > 1 || s.scale < 1 || s.scale > 4)
        throw std::invalid_argument("texture requires finite amount [-1,1] and scale 1..4");
}
void validate_sharpen_settings(const SharpenSettings& s) {
    if (!std::isfinite(s.amount) || s.amount < 0 || s.amount > 2 || s.radius < 1 || s.radius > 3)
        throw std::invalid_argument("sharpen requires finite amount 0..2 and radius 1..3");
}

StencilNode::StencilNode(std::shared_ptr<const Node> input, Rect native_bounds, const char* name)
    : input_(std::move(input)), native_bounds_(native_bounds), name_(name) {
    bounded_rect(native_bounds_);
    const std::string n(name);
    if (!input_)
        throw std::invalid_argument(n == "clarity" || n == "texture" ? n + " requires input"
                                                                     : n + " requires scene-linear working RGB");
    if (!scene_linear(input_->output_descriptor()))
        throw std::invalid_argument(n + " requires scene-linear working RGB");
    space_ = space_code(input_->output_descriptor());
}
bool StencilNode::supports_level(RenderLevel level) const noexcept {
    return (level_any_native(level) || level_reduced(level)) && input_->supports_level(level);
}
Rect StencilNode::input_region(Rect output, Rect source_bounds) const {
    return input_region_level(output, source_bounds, {});
}
Rect StencilNode::input_region_level(Rect output, Rect source_bounds, RenderLevel level) const {
    const Rect image = level_bounds(native_bounds_, level);
    if (!same(source_bounds, image) || !supports_level(level))
        throw std::invalid_argument(std::string(name_) + (std::string(name_) == "sharpen"
                                                               ? " source bounds or render level differ"
                                                               : " source bounds or level differ"));
    return spatial_expanded(output, image, halo_x(), halo_y());
}

ClarityNode::ClarityNode(std::shared_ptr<const Node> input, Rect native_bounds, ClaritySettings settings)
    : StencilNode((validate_clarity_settings(settings), std::move(input)), native_bounds, "clarity"),
      settings_(settings) {}
TextureNode::TextureNode(std::shared_ptr<const Node> input, Rect native_bounds, TextureSettings settings)
    : StencilNode((validate_texture_settings(settings), std::move(input)), native_bounds, "texture"),
      settings_(settings) {}
SharpenNode::SharpenNode(std::shared_ptr<const Node> input, Rect native_bounds, SharpenSettings settings)
    : StencilNode((validate_sharpen_settings(settings), std::move(input)), native_bounds, "sharpen"),
      settings_(settings) {}
ConvolutionNode::ConvolutionNode(std::shared_ptr<const Node> input, Rect native_bounds, ConvolutionKernel kernel)
    : StencilNode((validate_convolution_kernel(kernel), std::move(input)), native_bounds, "convolution"),
      kernel_(std::move(kernel)) {
    identity_ = true;
    const size_t center = kernel_.coefficients.size() / 2;
    for (size_t i = 0; i < kernel_.coefficients.size(); ++i)
        if (kernel_.coefficients[i] != (i == center ? 1.0 : 0.0)) identity_ = false;
}

// ------------------------------------------------------------- GeometryOps

void validate_rotate_settings(const RotateSettings& s) {
    if (!std::isfinite(s.angle_degrees) || s.angle_degrees < -180 || s.angle_degrees > 180)
        throw std::invalid_argument("rotation angle_degrees must be finite in [-180,180]");
}

// GeometryOps.cpp:46-67
RotateNode::RotateNode(std::shared_ptr<const Node> input, Rect bounds, RotateSettings settings)
    : input_(std::move(input)), input_bounds_(bounds), settings_(settings) {
    if (!addressable(bounds)) throw std::invalid_argument("rotation rectangle exceeds uint32 coordinates");
    validate_rotate_settings(settings_);
    if (!input_ || !bounds.width || !bounds.height)
        throw std::invalid_argument("rotation requires input and nonempty image bounds");
    descriptor_ = input_->output_descriptor();
    if (!scene_linear(descriptor_)) throw std::invalid_argument("rotation requires scene-linear working RGB");
    cx_ = (double(bounds.width) - 1) / 2;
    cy_ = (double(bounds.height) - 1) / 2;
    check(re_rotation_coefficients(settings_.angle_degrees, &cosine_, &sine_));
}
bool RotateNode::supports_level(RenderLevel level) const noexcept {
    if (level_native(level)) return input_->supports_level(level);
    return level_reduced(level) && input_->supports_level({}) && input_->supports_level(level);
}
RenderLevel RotateNode::input_level(RenderLevel level) const {
    if (!supports_level(level)) throw std::invalid_argument("rotation has no mapping for render level");
    return {};
}
// GeometryOps.cpp:86-98
Rect RotateNode::native_output_region(Rect output, RenderLevel level) const {
    if (!supports_level(level)) throw std::invalid_argument("rotation does not support render level");
    const uint32_t s = 1u << level.mip;
    const Rect extent{0, 0, input_bounds_.width / s + (input_bounds_.width % s != 0),
                      input_bounds_.height / s + (input_bounds_.height % s != 0)};
    if (!addressable(output)) throw std::invalid_argument("rotation rectangle exceeds uint32 coordinates");
    if (!contains(extent, output)) throw std::out_of_range("rotation output rectangle is outside image");
    const uint64_t l = std::min<uint64_t>((uint64_t)output.x * s, input_bounds_.width);
    const uint64_t t = std::min<uint64_t>((uint64_t)output.y * s, input_bounds_.height);
    const uint64_t r = std::min<uint64_t>(((uint64_t)output.x + output.width) * s, input_bounds_.width);
    const uint64_t b = std::min<uint64_t>(((uint64_t)output.y + output.height) * s, input_bounds_.height);
    return {(uint32_t)l, (uint32_t)t, (uint32_t)(r - l), (uint32_t)(b - t)};
}
// GeometryOps.cpp:99-111 (in input coordinates)
Rect RotateNode::support(Rect output) const {
    if (!output.width || !output.height) return {input_bounds_.x, input_bounds_.y, 0, 0};
    re_rect s;
    check(re_rotation_support(input_bounds_.width, input_bounds_.height, settings_.angle_degrees, to_re(output), &s));
    return {input_bounds_.x + s.x, input_bounds_.y + s.y, s.width, s.height};
}
Rect RotateNode::input_region(Rect output, Rect bounds) const { return input_region_level(output, bounds, {}); }
Rect RotateNode::input_region_level(Rect output, Rect bounds, RenderLevel level) const {
    if (!same(bounds, input_bounds_)) throw std::invalid_argument("rotation input bounds differ from construction");
    return support(native_output_region(output, level));
}

// GeometryOps.cpp:346-352
void validate_cubic_resize_settings(const CubicResizeSettings& settings, Rect bounds) {
    if (!addressable(bounds)) throw std::invalid_argument("rotation rectangle exceeds uint32 coordinates");
    if (!bounds.width || !bounds.height || !settings.width || !settings.height)
        throw std::invalid_argument("cubic resize requires positive input and canvas extents");
    if ((uint64_t)settings.width * 4 < bounds.width || (uint64_t)settings.height * 4 < bounds.height)
        throw std::invalid_argument("cubic resize native shrink exceeds fourfold per axis");
}
CubicResizeNode::CubicResizeNode(std::shared_ptr<const Node> input, Rect bounds, CubicResizeSettings settings)
    : input_(std::move(input)), input_bounds_(bounds), settings_(settings) {
    validate_cubic_resize_settings(settings_, bounds);
    if (!input_) throw std::invalid_argument("cubic resize requires input");
    descriptor_ = input_->output_descriptor();
    if (!scene_linear(descriptor_)) throw std::invalid_argument("cubic resize requires scene-linear working RGB");
}
bool CubicResizeNode::supports_level(RenderLevel level) const noexcept {
    if (level_native(level)) return input_->supports_level(level);
    return level_reduced(level) && input_->supports_level({}) && input_->supports_level(level);
}
RenderLevel CubicResizeNode::input_level(RenderLevel level) const {
    if (!supports_level(level)) throw std::invalid_argument("cubic resize has no mapping for render level");
    return {};
}
// GeometryOps.cpp:399-410
Rect CubicResizeNode::native_output_region(Rect output, RenderLevel level) const {
    if (!supports_level(level)) throw std::invalid_argument("cubic resize does not support render level");
    const uint32_t s = 1u << level.mip;
    const Rect extent{0, 0, settings_.width / s + (settings_.width % s != 0),
                      settings_.height / s + (settings_.height % s != 0)};
    if (!addressable(output)) throw std::invalid_argument("rotation rectangle exceeds uint32 coordinates");
    if (!contains(extent, output)) throw std::out_of_range("rotation output rectangle is outside image");
    const uint64_t l = std::min<uint64_t>((uint64_t)output.x * s, settings_.width);
    const uint64_t t = std::min<uint64_t>((uint64_t)output.y * s, settings_.height);
    const uint64_t r = std::min<uint64_t>(((uint64_t)output.x + output.width) * s, settings_.width);
    const uint64_t b = std::min<uint64_t>(((uint64_t)output.y + output.height) * s, settings_.height);
    return {(uint32_t)l, (uint32_t)t, (uint32_t)(r - l), (uint32_t)(b - t)};
}
// GeometryOps.cpp:411-425
Rect CubicResizeNode::support(Rect output) const {
    if (!output.width || !output.height) return {input_bounds_.x, input_bounds_.y, 0, 0};
    auto extent = [](uint32_t input, uint32_t canvas, uint32_t start, uint32_t length) {
        uint32_t first = input, last = 0;
        for (uint64_t i = start; i < (uint64_t)start + length; ++i) {
            uint32_t center, idx[18], count;
            double w[18];
            check(re_cubic_axis(input, canvas, (uint32_t)i, &center, idx, w, &count));
            for (uint32_t j = 0; j < count; ++j) {
                first = std::min(first, idx[j]);
                last = std::max(last, idx[j]);
            }
        }
        return std::pair<uint32_t, uint32_t>{first, last - first + 1};
    };
    const auto x = extent(input_bounds_.width, settings_.width, output.x, output.width);
    const auto y = extent(input_bounds_.height, settings_.height, output.y, output.height);
    return {input_bounds_.x + x.first, input_bounds_.y + y.first, x.second, y.second};
}
Rect CubicResizeNode::input_region(Rect output, Rect bounds) const { return input_region_level(output, bounds, {}); }
Rect CubicResizeNode::input_region_level(Rect output, Rect bounds, RenderLevel level) const {
    if (!same(bounds, input_bounds_)) throw std::invalid_argument("cubic resize input bounds differ from construction");
    return support(native_output_region(output, level));
}

// ----------------------------------------------------------------- executor

namespace {

struct DevImage {
    float* data = nullptr;
    size_t stride = 0;  // floats per row
    Rect bounds;
    cudaStream_t stream = nullptr;
    std::shared_ptr<const float> shared;   // a cached tile read in place (not freed here)
    DevImage(Rect r, cudaStream_t s) : stride((size_t)r.width * 3), bounds(r), stream(s) {
        if (r.width && r.height)
            check_cuda(re::scratch_alloc((void**)&data, (size_t)r.width * r.height * 3 * sizeof(float), s),
                       "device tile");
    }
    // A read-only view of a contiguous device tile; the executor never writes
    // into an image it evaluated, so a cached tile can be used without a copy.
    DevImage(Rect r, cudaStream_t s, std::shared_ptr<const float> tile)
        : data(const_cast<float*>(tile.get())), stride((size_t)r.width * 3), bounds(r), stream(s),
          shared(std::move(tile)) {}
    ~DevImage() {
        if (data && !shared) cudaFreeAsync(data, stream);
    }
    DevImage(const DevImage&) = delete;
    DevImage& operator=(const DevImage&) = delete;
};
using DevPtr = std::unique_ptr<DevImage>;

// Point stages of a chain (top-down order collected, applied bottom-up).
struct StageList {
    re_render_desc desc{};
    std::vector<std::shared_ptr<CurveTables>> keep;
    int anchor_node = -1;  // index (bottom-up) of a CameraToWorking anchor
};

void add_stage(StageList& sl, const PointNode* n, bool reduced_anchor_allowed, RenderLevel level) {
    re_stage st{};
    if (auto* p = dynamic_cast<const WhiteBalanceNode*>(n)) {
        st.kind = RE_STAGE_GAIN3;
        for (int i = 0; i < 3; ++i) st.f[i] = p->gains()[i];
    } else if (auto* p = dynamic_cast<const ExposureNode*>(n)) {
        st.kind = RE_STAGE_SCALE;
        st.f[0] = p->multiplier();
    } else if (auto* p = dynamic_cast<const CameraToWorkingNode*>(n)) {
        st.kind = RE_STAGE_MATRIX;
        std::copy(p->matrix().begin(), p->matrix().end(), st.f);
        if (level.mip && reduced_anchor_allowed) sl.desc.anchor = (int32_t)sl.desc.count;
    } else if (auto* p = dynamic_cast<const WorkingSpaceConvertNode*>(n)) {
        if (p->identity()) return;
        st.kind = RE_STAGE_MATRIX;
        std::copy(p->matrix().begin(), p->matrix().end(), st.f);
    } else if (auto* p = dynamic_cast<const WorkingToSrgbNode*>(n)) {
        st.kind = RE_STAGE_MATRIX;
        std::copy(p->matrix().begin(), p->matrix().end(), st.f);
    } else if (auto* p = dynamic_cast<const ToneCurveNode*>(n)) {
        st.kind = RE_STAGE_TONE;
        st.f[0] = p->shoulder();
        st.f[1] = p->inverse_gamma();
    } else if (dynamic_cast<const OutputClipNode*>(n)) {
        st.kind = RE_STAGE_CLIP;
    } else if (dynamic_cast<const SrgbEncodeNode*>(n)) {
        st.kind = RE_STAGE_SRGB;
    } else if (auto* p = dynamic_cast<const ExtendedCurvesNode*>(n)) {
        uint32_t slot = 0;
        while (slot < 4 && sl.desc.curves[slot]) ++slot;
        if (slot == 4) throw std::length_error("more than four curve nodes in one fused chain");
        st.kind = RE_STAGE_CURVES;
        st.arg = slot;
        sl.desc.curves[slot] = p->tables().set;
    } else {
        throw std::logic_error("unknown point node");
    }
    if (sl.desc.count == RE_MAX_STAGES) throw std::length_error("too many fused stages");
    sl.desc.stages[sl.desc.count++] = st;
}

struct Executor {
    cudaStream_t s;
    const CancellationToken* cancel;

    void check_cancel() const {
        if (cancel && cancel->is_cancelled()) throw RenderCancelled();
    }

    // Renders `node` over `r` at `level` into device memory.
    DevPtr eval(const Node& node, Rect r, RenderLevel level) {
        check_cancel();
        if (!node.supports_level(level)) throw std::invalid_argument("node does not support this render level");
        // collect point nodes down to the first non-point node
        std::vector<const PointNode*> chain;
        const Node* cur = &node;
        while (auto* p = dynamic_cast<const PointNode*>(cur)) {
            chain.push_back(p);
            cur = p->input().get();
        }
        std::reverse(chain.begin(), chain.end());  // bottom-up
        // the level below a CameraToWorking anchor is native
        int anchor = -1;
        for (int i = (int)chain.size() - 1; i >= 0; --i)
            if (level.mip && dynamic_cast<const CameraToWorkingNode*>(chain[i])) {
                anchor = i;
                break;
            }
        if (auto* raw = dynamic_cast<const RawUnpackNode*>(cur)) return eval_raw(*raw, chain, anchor, r, level);
        if (auto* ras = dynamic_cast<const RasterSourceNode*>(cur); ras && anchor < 0)
            return eval_raster(*ras, chain, r, level);
        // a non-point bottom: render it, then the stages (an anchor reduces there)
        Rect bottom_rect = r;
        RenderLevel bottom_level = level;
        if (anchor >= 0) {
            auto* ctw = static_cast<const CameraToWorkingNode*>(chain[anchor]);
            bottom_rect = ctw->input_region_level(r, ctw->native_bounds(), level);
            bottom_level = {};
        }
        DevPtr base = eval_bottom(*cur, bottom_rect, bottom_level);
        if (chain.empty()) return base;
        if (anchor < 0) return stages_over(std::move(base), chain, 0, (int)chain.size(), 0);
        DevPtr native = stages_over(std::move(base), chain, 0, anchor + 1, 0);
        // reduce over the native footprint, then the stages above the anchor
        return stages_over(std::move(native), chain, anchor + 1, (int)chain.size(), level.mip, r);
    }

    // Stages [begin, end) of `chain` over a device image; mip > 0 averages the
    // image's footprints into `reduced` (zero-based in the image) first.
    DevPtr stages_over(DevPtr in, const std::vector<const PointNode*>& chain, int begin, int end, uint32_t mip,
                       Rect reduced = {}) {
        StageList sl;
        sl.desc.anchor = -1;
        for (int i = begin; i < end; ++i) add_stage(sl, chain[i], false, {});
        const Rect out_rect = mip ? reduced : in->bounds;
        auto out = std::make_unique<DevImage>(out_rect, s);
        const re_rect vp = mip ? re_rect{0, 0, reduced.width, reduced.height}
                               : re_rect{0, 0, in->bounds.width, in->bounds.height};
        if (vp.width && vp.height)
            check(re_render_raster(in->data, in->stride, in->bounds.width, in->bounds.height, &sl.desc, vp, mip,
                                   mip ? 0u : 1u, out->data, out->stride, s));
        return out;
    }

    DevPtr eval_raw(const RawUnpackNode& raw, const std::vector<const PointNode*>& chain, int anchor, Rect r,
                    RenderLevel level) {
        StageList sl;
        sl.desc.demosaic = raw.menon() ? 1u : 0u;
        sl.desc.anchor = -1;
        for (int i = 0; i < (int)chain.size(); ++i) add_stage(sl, chain[i], i == anchor, level);
        if (level.mip && sl.desc.anchor < 0) throw std::invalid_argument("node does not support this render level");
        auto out = std::make_unique<DevImage>(r, s);
        if (!r.width || !r.height) return out;
        const DeviceRaw& dev = raw.image().device();
        check(re_render_raw(dev.handle, &sl.desc, to_re(r), level.mip, (uint32_t)level.quality, out->data,
                            out->stride, 1, s, nullptr));
        return out;
    }

    DevPtr eval_raster(const RasterSourceNode& src, const std::vector<const PointNode*>& chain, Rect r,
                       RenderLevel level) {
        StageList sl;
        sl.desc.anchor = -1;
        for (auto* p : chain) add_stage(sl, p, false, {});
        auto out = std::make_unique<DevImage>(r, s);
        const auto& img = src.image();
        const Rect bounds = request_bounds({0, 0, img.width(), img.height()}, level);
        if (!contains(bounds, r)) throw std::out_of_range("viewport is outside the active RAW area");
        if (!r.width || !r.height) return out;
        const DeviceRaster& dev = img.device();
        check(re_render_raster(dev.data, dev.stride, img.width(), img.height(), &sl.desc, to_re(r), level.mip,
                               (uint32_t)level.quality, out->data, out->stride, s));
        return out;
    }

    DevPtr eval_bottom(const Node& node, Rect r, RenderLevel level) {
        if (auto* gf = dynamic_cast<const WorkingYGuidedFilterNode*>(&node)) return eval_gf(*gf, r, level);
        if (auto* cr = dynamic_cast<const CubicResizeNode*>(&node)) return eval_cubic(*cr, r, level);
        if (auto* ro = dynamic_cast<const RotateNode*>(&node)) return eval_rotate(*ro, r, level);
        if (auto* st = dynamic_cast<const StencilNode*>(&node)) return eval_stencil(*st, r, level);
        if (auto* cn = dynamic_cast<const CachedNode*>(&node)) return eval_cached(*cn, r, level);
        if (dynamic_cast<const DeviceNode*>(&node)) return eval(node, r, level);
        return upload(node, r, level);
    }

    // A node of another library: its own render_level, validated like the
    // reference validates upstream tiles (RawEngine.cpp:66-72), then uploaded.
    DevPtr upload(const Node& node, Rect r, RenderLevel level) {
        const Tile t = node.render_level(r, level);
        if (!same(t.bounds, r) || t.descriptor != node.output_descriptor() ||
            t.rgb.size() != (size_t)r.width * r.height * 3)
            throw std::domain_error("upstream node returned an invalid tile");
        auto out = std::make_unique<DevImage>(r, s);
        if (!t.rgb.empty())
            check_cuda(cudaMemcpyAsync(out->data, t.rgb.data(), t.rgb.size() * sizeof(float), cudaMemcpyHostToDevice,
                                       s),
                       "upload tile");
        check_cuda(cudaStreamSynchronize(s), "upload tile");
        return out;
    }

    // SpatialOps.cpp:312-317: render the 2r-expanded input, filter, crop.
    DevPtr eval_gf(const WorkingYGuidedFilterNode& gf, Rect r, RenderLevel level) {
        const Rect image = level_bounds(gf.native_bounds(), level);
        const Rect needed = gf.input_region_level(r, image, level);
        DevPtr in = eval(*gf.input_node(), needed, level);
        auto filtered = std::make_unique<DevImage>(needed, s);
        check(re_guided_filter(in->data, in->stride, filtered->data, filtered->stride, needed.width, needed.height,
                               gf.settings().radius, gf.settings().epsilon,
                               space_code(gf.output_descriptor()), s));
        auto out = std::make_unique<DevImage>(r, s);
        check_cuda(cudaMemcpy2DAsync(out->data, out->stride * sizeof(float),
                                     filtered->data + (size_t)(r.y - needed.y) * filtered->stride +
                                         (size_t)(r.x - needed.x) * 3,
                                     filtered->stride * sizeof(float), (size_t)r.width * 3 * sizeof(float), r.height,
                                     cudaMemcpyDeviceToDevice, s),
                   "crop");
        return out;
    }

    // GeometryOps.cpp:483-513: native support of the request, then the resize.
    DevPtr eval_cubic(const CubicResizeNode& cr, Rect r, RenderLevel level) {
        const Rect native = cr.native_output_region(r, level);
        auto out = std::make_unique<DevImage>(r, s);
        if (!native.width || !native.height) return out;
        const Rect support = cr.support(native);
        DevPtr in = eval(*cr.input_node(), support, {});
        const Rect ib = cr.input_bounds();
        const re_rect window{support.x - ib.x, support.y - ib.y, support.width, support.height};
        check(re_cubic_resize_window(in->data, in->stride, window, ib.width, ib.height, cr.settings().width,
                                     cr.settings().height, to_re(r), level.mip, out->data, out->stride, s));
        return out;
    }

    // A cached node: the cache's device tile for exactly this rectangle and
    // level, read in place (rendered through the input on a miss).
    DevPtr eval_cached(const CachedNode& cn, Rect r, RenderLevel level) {
        check_cancel();
        if (!r.width || !r.height) return std::make_unique<DevImage>(r, s);
        DeviceTile t = cn.cache()->render_device(*cn.input_node(), cn.signature(), r, level);
        return std::make_unique<DevImage>(r, s, std::move(t.rgb));
    }

    // SpatialOps.cpp:343-383, 410-495, 509-620, 637-697: render the input over
    // the node's `needed` region, then one stencil launch.
    DevPtr eval_stencil(const StencilNode& st, Rect r, RenderLevel level) {
        const Rect image = level_bounds(st.native_bounds(), level);
        const Rect needed = st.input_region_level(r, image, level);
        DevPtr in = eval(*st.input_node(), needed, level);
        auto out = std::make_unique<DevImage>(r, s);
        const re_rect w = to_re(needed), im = to_re(image), o = to_re(r);
        const uint32_t space = st.working_space();
        if (auto* p = dynamic_cast<const SharpenNode*>(&st))
            check(re_sharpen_window(in->data, in->stride, w, im, o, p->settings().amount, p->settings().radius,
                                    out->data, out->stride, s));
        else if (auto* p = dynamic_cast<const ClarityNode*>(&st))
            check(re_clarity_window(in->data, in->stride, w, im, o, p->settings().amount, p->settings().radius,
                                    space, out->data, out->stride, s));
        else if (auto* p = dynamic_cast<const TextureNode*>(&st))
            check(re_texture_window(in->data, in->stride, w, im, o, p->settings().amount, p->settings().scale,
                                    space, out->data, out->stride, s));
        else if (auto* p = dynamic_cast<const ConvolutionNode*>(&st))
            check(re_convolution_window(in->data, in->stride, w, im, o, p->kernel().width, p->kernel().height,
                                        p->kernel().coefficients.data(), out->data, out->stride, s));
        else
            throw std::logic_error("unknown stencil node");
        return out;
    }

    // GeometryOps.cpp:145-174
    DevPtr eval_rotate(const RotateNode& ro, Rect r, RenderLevel level) {
        const Rect native = ro.native_output_region(r, level);
        auto out = std::make_unique<DevImage>(r, s);
        if (!native.width || !native.height) return out;
        const Rect support = ro.support(native);
        DevPtr in = eval(*ro.input_node(), support, {});
        const Rect ib = ro.input_bounds();
        const re_rect window{support.x - ib.x, support.y - ib.y, support.width, support.height};
        check(re_rotate_window(in->data, in->stride, window, ib.width, ib.height, ro.angle(), to_re(r), level.mip,
                               out->data, out->stride, s));
        return out;
    }
};

Tile download(const DevImage& img, ImageDescriptor descriptor, cudaStream_t s) {
    Tile t{img.bounds, std::vector<float>((size_t)img.bounds.width * img.bounds.height * 3), descriptor};
    if (!t.rgb.empty())
        check_cuda(cudaMemcpy2DAsync(t.rgb.data(), (size_t)img.bounds.width * 3 * sizeof(float), img.data,
                                     img.stride * sizeof(float), (size_t)img.bounds.width * 3 * sizeof(float),
                                     img.bounds.height, cudaMemcpyDeviceToHost, s),
                   "download");
    check_cuda(cudaStreamSynchronize(s), "download");
    return t;
}

}  // namespace

Tile DeviceNode::render(Rect bounds) const { return render_level(bounds, {}); }

Tile DeviceNode::render_level(Rect bounds, RenderLevel level) const {
    cudaStream_t s = thread_stream();
    Executor ex{s, nullptr};
    DevPtr img = ex.eval(*this, bounds, level);
    return download(*img, output_descriptor(), s);
}

// ------------------------------------------------------------------ graphs

// RawEngine.cpp:1306-1333 (the ICC display output needs the LittleCMS backend,
// which this library does not include: IccDisplay is rejected as unsupported)
ImageGraph::ImageGraph(RawImage image, GraphRecipe recipe)
    : raw_image_(std::move(image)), source_bounds_(raw_image_->metadata().active_area), recipe_(recipe) {
    auto node = std::make_shared<RawUnpackNode>(*raw_image_);
    auto wb = std::make_shared<WhiteBalanceNode>(node, recipe.red_gain, recipe.green_gain, recipe.blue_gain);
    std::shared_ptr<const Node> linear = std::make_shared<ExposureNode>(wb, recipe.exposure_stops);
    if (recipe.camera_color)
        linear = std::make_shared<CameraToWorkingNode>(linear, *recipe.camera_color, source_bounds_);
    if (recipe.output_mode == OutputMode::SrgbPreview) linear = std::make_shared<WorkingToSrgbNode>(linear);
    else if (recipe.output_mode != OutputMode::LegacyBounded)
        throw std::invalid_argument("ICC display output is not available in this library");
    auto tone = std::make_shared<ToneCurveNode>(linear, recipe.tone_shoulder, recipe.tone_gamma);
    output_ = recipe.output_mode == OutputMode::SrgbPreview
                  ? std::static_pointer_cast<const Node>(std::make_shared<SrgbEncodeNode>(tone))
                  : std::static_pointer_cast<const Node>(std::make_shared<OutputClipNode>(tone));
}

ImageGraph::ImageGraph(RasterImage image, GraphRecipe recipe)
    : ImageGraph(std::make_shared<RasterSourceNode>(image), Rect{0, 0, image.width(), image.height()}, recipe) {}

// RawEngine.cpp:1341-1376
ImageGraph::ImageGraph(std::shared_ptr<const Node> source, Rect bounds, GraphRecipe recipe)
    : source_bounds_(bounds), recipe_(recipe) {
    if (!source || !bounds.width || !bounds.height || !addressable(bounds))
        throw std::invalid_argument("scene-linear source and valid bounds are required");
    if (!scene_linear(source->output_descriptor()))
        throw std::invalid_argument("graph source must output a supported scene-linear space");
    if (recipe.red_gain != 1.0f || recipe.green_gain != 1.0f || recipe.blue_gain != 1.0f || recipe.camera_color)
        throw std::invalid_argument("raster input does not accept RAW calibration controls");
    std::shared_ptr<const Node> linear = std::make_shared<ExposureNode>(source, recipe.exposure_stops);
    if (recipe.output_mode == OutputMode::SrgbPreview) linear = std::make_shared<WorkingToSrgbNode>(linear);
    else if (recipe.output_mode != OutputMode::LegacyBounded)
        throw std::invalid_argument("ICC display output is not available in this library");
    auto tone = std::make_shared<ToneCurveNode>(linear, recipe.tone_shoulder, recipe.tone_gamma);
    output_ = recipe.output_mode == OutputMode::SrgbPreview
                  ? std::static_pointer_cast<const Node>(std::make_shared<SrgbEncodeNode>(tone))
                  : std::static_pointer_cast<const Node>(std::make_shared<OutputClipNode>(tone));
}

const RawImage& ImageGraph::image() const {
    if (!raw_image_) throw std::logic_error("graph has a raster source, not a RAW source");
    return *raw_image_;
}

// ---------------------------------------------------------------- renderer

namespace {
void validate_request(const Node& output, Rect source_bounds, const RenderRequest& request,
                      const CancellationToken* cancellation) {
    const Rect bounds = request_bounds(source_bounds, request.level);
    if (!contains(bounds, request.viewport)) throw std::out_of_range("viewport is outside the active RAW area");
    if (!output.supports_level(request.level)) throw std::invalid_argument("node does not support this render level");
    if (cancellation && cancellation->is_cancelled()) throw RenderCancelled();
}
}  // namespace

// RawEngine.cpp:1390-1412
void Renderer::render_tiles(const Node& output, Rect source_bounds, RenderRequest request,
                            const TileCallback& callback, const CancellationToken* cancellation) const {
    validate_request(output, source_bounds, request, nullptr);
    if (!callback || !request.tile_size) throw std::invalid_argument("callback and tile size are required");
    if (cancellation && cancellation->is_cancelled()) throw RenderCancelled();
    const uint64_t right = (uint64_t)request.viewport.x + request.viewport.width;
    const uint64_t bottom = (uint64_t)request.viewport.y + request.viewport.height;
    for (uint64_t y = request.viewport.y; y < bottom; y += request.tile_size)
        for (uint64_t x = request.viewport.x; x < right; x += request.tile_size) {
            if (cancellation && cancellation->is_cancelled()) throw RenderCancelled();
            const Rect r{(uint32_t)x, (uint32_t)y, (uint32_t)std::min<uint64_t>(request.tile_size, right - x),
                         (uint32_t)std::min<uint64_t>(request.tile_size, bottom - y)};
            callback(output.render_level(r, request.level));
        }
}

void Renderer::render_tiles(const ImageGraph& graph, RenderRequest request, const TileCallback& callback,
                            const CancellationToken* cancellation) const {
    render_tiles(graph.output(), graph.source_bounds(), request, callback, cancellation);
}
void Renderer::render_tiles(const ImageGraph& graph, Rect viewport, const TileCallback& callback,
                            std::uint32_t tile_size, const CancellationToken* cancellation) const {
    render_tiles(graph.output(), graph.source_bounds(), RenderRequest{viewport, tile_size, {}}, callback,
                 cancellation);
}
void Renderer::render_tiles(const Node& output, Rect source_bounds, Rect viewport, const TileCallback& callback,
                            std::uint32_t tile_size, const CancellationToken* cancellation) const {
    render_tiles(output, source_bounds, RenderRequest{viewport, tile_size, {}}, callback, cancellation);
}

// RawEngine.cpp:1426-1447: nodes of this library render the whole viewport in
// one pass (results do not depend on the tile size); other nodes keep the
// reference's tile loop.
Tile Renderer::render_image(const Node& output, Rect source_bounds, RenderRequest request,
                            const CancellationToken* cancellation) const {
    validate_request(output, source_bounds, request, cancellation);
    if (!request.tile_size) throw std::invalid_argument("callback and tile size are required");
    if (dynamic_cast<const DeviceNode*>(&output)) {
        cudaStream_t s = thread_stream();
        Executor ex{s, cancellation};
        DevPtr img = ex.eval(output, request.viewport, request.level);
        return download(*img, output.output_descriptor(), s);
    }
    Tile image{request.viewport, std::vector<float>((size_t)request.viewport.width * request.viewport.height * 3),
               output.output_descriptor()};
    render_tiles(output, source_bounds, request, [&](const Tile& tile) {
        if (tile.descriptor != image.descriptor || tile.rgb.size() != (size_t)tile.bounds.width * tile.bounds.height * 3)
            throw std::domain_error("upstream node returned an invalid tile");
        for (uint32_t row = 0; row < tile.bounds.height; ++row)
            std::memcpy(image.rgb.data() + ((size_t)(tile.bounds.y - request.viewport.y + row) * request.viewport.width +
                                            tile.bounds.x - request.viewport.x) * 3,
                        tile.rgb.data() + (size_t)row * tile.bounds.width * 3, (size_t)tile.bounds.width * 3 * sizeof(float));
    }, cancellation);
    return image;
}

Tile Renderer::render_image(const ImageGraph& graph, RenderRequest request,
                            const CancellationToken* cancellation) const {
    return render_image(graph.output(), graph.source_bounds(), request, cancellation);
}
Tile Renderer::render_image(const ImageGraph& graph, Rect viewport, std::uint32_t tile_size,
                            const CancellationToken* cancellation) const {
    return render_image(graph.output(), graph.source_bounds(), RenderRequest{viewport, tile_size, {}}, cancellation);
}
Tile Renderer::render_image(const Node& node, Rect source_bounds, Rect viewport, std::uint32_t tile_size,
                            const CancellationToken* cancellation) const {
    return render_image(node, source_bounds, RenderRequest{viewport, tile_size, {}}, cancellation);
}
std::vector<float> Renderer::render_roi(const ImageGraph& graph, Rect viewport, std::uint32_t tile_size,
                                        const CancellationToken* cancellation) const {
    return std::move(render_image(graph, viewport, tile_size, cancellation).rgb);
}

// ------------------------------------------------------- spatial functions

// SpatialOps.cpp:168-287 on a caller tile covering the 2r-expanded output.
Tile working_y_guided_filter_rgb(const Tile& input, Rect output, Rect image,
                                 const WorkingYGuidedFilterSettings& settings) {
    validate_working_y_guided_filter_settings(settings);
    if (!scene_linear(input.descriptor)) throw std::invalid_argument("guided filter requires scene-linear working RGB");
    const Rect needed = working_y_guided_filter_region(output, image, settings.radius);
    if (!same(input.bounds, needed) || input.rgb.size() != (size_t)needed.width * needed.height * 3)
        throw std::invalid_argument("spatial input tile bounds, storage or descriptor differ");
    for (float v : input.rgb)
        if (!std::isfinite(v)) throw std::invalid_argument("guided filter requires finite complete input halo");
    if (settings.radius == 0) return input;
    cudaStream_t s = thread_stream();
    DevImage in(needed, s), filtered(needed, s);
    check_cuda(cudaMemcpyAsync(in.data, input.rgb.data(), input.rgb.size() * sizeof(float), cudaMemcpyHostToDevice, s),
               "upload");
    check(re_guided_filter(in.data, in.stride, filtered.data, filtered.stride, needed.width, needed.height,
                           settings.radius, settings.epsilon, space_code(input.descriptor), s));
    Tile t = download(filtered, input.descriptor, s);
    Tile out{output, std::vector<float>((size_t)output.width * output.height * 3), input.descriptor};
    for (uint32_t row = 0; row < output.height; ++row)
        std::memcpy(out.rgb.data() + (size_t)row * output.width * 3,
                    t.rgb.data() + ((size_t)(output.y - needed.y + row) * needed.width + (output.x - needed.x)) * 3,
                    (size_t)output.width * 3 * sizeof(float));
    return out;
}

// SpatialOps.cpp:79-121 on a caller tile covering the r-expanded output.
LocalStatisticsTile local_statistics_rgb(const Tile& input, Rect output, Rect image, std::uint32_t radius) {
    const Rect needed = local_statistics_region(output, image, radius);
    if (!same(input.bounds, needed) || input.rgb.size() != (size_t)needed.width * needed.height * 3)
        throw std::invalid_argument("spatial input tile bounds, storage or descriptor differ");
    cudaStream_t s = thread_stream();
    const size_t n_needed = (size_t)needed.width * needed.height * 3;
    DevImage in(needed, s);
    void* scratch = nullptr;
    check_cuda(re::scratch_alloc(&scratch, n_needed * (2 * sizeof(double) + sizeof(uint32_t)), s), "statistics");
    double* mean = (double*)scratch;
    double* var = mean + n_needed;
    uint32_t* count = (uint32_t*)(var + n_needed);
    check_cuda(cudaMemcpyAsync(in.data, input.rgb.data(), input.rgb.size() * sizeof(float), cudaMemcpyHostToDevice, s),
               "upload");
    re_status st = re_local_statistics_f64(in.data, in.stride, needed.width, needed.height, radius, mean, var, count,
                                           s);
    std::vector<double> m(n_needed), v(n_needed);
    std::vector<uint32_t> c(n_needed);
    if (st == RE_OK) {
        cudaMemcpyAsync(m.data(), mean, n_needed * sizeof(double), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(v.data(), var, n_needed * sizeof(double), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(c.data(), count, n_needed * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    }
    cudaFreeAsync(scratch, s);
    check_cuda(cudaStreamSynchronize(s), "local statistics");
    check(st);
    LocalStatisticsTile out{output, input.descriptor, radius, {}, {}, {}};
    const size_t n = (size_t)output.width * output.height * 3;
    out.mean.resize(n);
    out.variance.resize(n);
    out.finite_count.resize(n);
    for (uint32_t row = 0; row < output.height; ++row)
        for (uint32_t col = 0; col < output.width; ++col)
            for (int k = 0; k < 3; ++k) {
                const size_t src = ((size_t)(output.y - needed.y + row) * needed.width + (output.x - needed.x + col)) * 3 + k;
                const size_t dst = ((size_t)row * output.width + col) * 3 + k;
                out.mean[dst] = m[src];
                out.variance[dst] = v[src];
                out.finite_count[dst] = c[src];
            }
    return out;
}

// SpatialOps.cpp:123-149
void analyze_local_rgb(const Node& output, Rect native_bounds, const RenderRequest& request,
                       const LocalStatisticsCallback& callback, std::uint32_t radius,
                       const CancellationToken* cancellation) {
    const Rect image = level_bounds(native_bounds, request.level);
    (void)local_statistics_region(request.viewport, image, radius);
    if (!callback || !request.tile_size || !output.supports_level(request.level))
        throw std::invalid_argument("local analysis needs a callback, positive tile size and supported level");
    auto check_c = [&] {
        if (cancellation && cancellation->is_cancelled()) throw RenderCancelled();
    };
    check_c();
    const uint64_t right = (uint64_t)request.viewport.x + request.viewport.width;
    const uint64_t bottom = (uint64_t)request.viewport.y + request.viewport.height;
    for (uint64_t y = request.viewport.y; y < bottom; y += request.tile_size)
        for (uint64_t x = request.viewport.x; x < right; x += request.tile_size) {
            check_c();
            const Rect rect{(uint32_t)x, (uint32_t)y, (uint32_t)std::min<uint64_t>(request.tile_size, right - x),
                            (uint32_t)std::min<uint64_t>(request.tile_size, bottom - y)};
            const Rect needed = local_statistics_region(rect, image, radius);
            const Tile input = output.render_level(needed, request.level);
            check_c();
            callback(local_statistics_rgb(input, rect, image, radius));
            check_c();
        }
}
void analyze_local_rgb(const ImageGraph& graph, const RenderRequest& request, const LocalStatisticsCallback& callback,
                       std::uint32_t radius, const CancellationToken* cancellation) {
    analyze_local_rgb(graph.output(), graph.source_bounds(), request, callback, radius, cancellation);
}

// ---------------------------------------------------------- ImageAnalysis

namespace {

// Device counters of one histogram: counts[3 * bins], tallies[9], extrema[6].
struct HistogramCounters {
    uint64_t* base = nullptr;
    uint32_t bins;
    cudaStream_t s;
    HistogramCounters(uint32_t b, cudaStream_t stream) : bins(b), s(stream) {
        check_cuda(re::scratch_alloc((void**)&base, ((size_t)3 * bins + 15) * sizeof(uint64_t), s), "histogram");
        check(re_histogram_reset(bins, counts(), tallies(), extrema(), s));
    }
    ~HistogramCounters() {
        if (base) cudaFreeAsync(base, s);
    }
    uint64_t* counts() const { return base; }
    uint64_t* tallies() const { return base + (size_t)3 * bins; }
    uint64_t* extrema() const { return base + (size_t)3 * bins + 9; }
};

// Rows of device scratch per band: whole tile rows, about 24 MiB, so that a
// band written by the render is still in L2 when the histogram reads it.
constexpr uint64_t kHistogramBandBytes = 24ull << 20;

}  // namespace

// ImageAnalysis.cpp:9-69
RgbHistogram histogram_rgb(const Node& output, Rect source_bounds, const RenderRequest& request,
                           const HistogramOptions& options, const CancellationToken* cancellation) {
    const double span = options.upper - options.lower;
    if (options.bins == 0 || options.bins > 65536 || !std::isfinite(options.lower) || !std::isfinite(options.upper) ||
        !(span > 0.0) || !std::isfinite(span))
        throw std::invalid_argument("histogram requires 1..65536 bins and a finite positive range");
    auto check_cancelled = [&] {
        if (cancellation && cancellation->is_cancelled()) throw RenderCancelled();
    };
    check_cancelled();
    RgbHistogram result;
    result.request = request;
    result.options = options;
    result.descriptor = output.output_descriptor();
    if (result.descriptor.format != PixelFormat::RGBFloat32)
        throw std::invalid_argument("histogram requires RGBFloat32 output");
    const Rect vp = request.viewport;
    const uint64_t right = (uint64_t)vp.x + vp.width, bottom = (uint64_t)vp.y + vp.height;
    if (!vp.width || !vp.height || right > (1ull << 32) || bottom > (1ull << 32))
        throw std::invalid_argument("histogram requires a nonempty addressable viewport");
    validate_request(output, source_bounds, request, nullptr);
    if (!request.tile_size) throw std::invalid_argument("callback and tile size are required");
    const uint32_t T = request.tile_size;
    cudaStream_t s = thread_stream();
    HistogramCounters hc(options.bins, s);
    auto count = [&](const float* rgb, size_t stride, uint32_t w, uint32_t h, uint32_t tile, uint64_t first) {
        check(re_histogram_rgb(rgb, stride, w, h, tile, first, options.bins, options.lower, options.upper,
                               hc.counts(), hc.tallies(), hc.extrema(), s));
    };
    if (dynamic_cast<const DeviceNode*>(&output)) {
        const uint64_t row_bytes = (uint64_t)vp.width * 3 * sizeof(float);
        const uint64_t band = std::max<uint64_t>(T, kHistogramBandBytes / row_bytes / T * T);
        Executor ex{s, cancellation};
        for (uint64_t y = vp.y; y < bottom; y += band) {
            check_cancelled();
            const Rect r{vp.x, (uint32_t)y, vp.width, (uint32_t)std::min<uint64_t>(band, bottom - y)};
            DevPtr img = ex.eval(output, r, request.level);
            count(img->data, img->stride, r.width, r.height, T, (y - vp.y) * vp.width);
        }
    } else {
        // The reference's tile stream with its checks on each delivered tile.
        uint64_t next_x = vp.x, next_y = vp.y, first = 0;
        Renderer{}.render_tiles(output, source_bounds, request, [&](const Tile& tile) {
            check_cancelled();
            const Rect expected{(uint32_t)next_x, (uint32_t)next_y,
                                (uint32_t)std::min<uint64_t>(T, right - next_x),
                                (uint32_t)std::min<uint64_t>(T, bottom - next_y)};
            const uint64_t pixels = (uint64_t)expected.width * expected.height;
            if (!same(tile.bounds, expected) || tile.rgb.size() % 3 != 0 || tile.rgb.size() / 3 != pixels ||
                tile.descriptor != result.descriptor)
                throw std::invalid_argument("histogram received inconsistent tile bounds, storage or descriptor");
            DevImage dev(expected, s);
            check_cuda(cudaMemcpyAsync(dev.data, tile.rgb.data(), tile.rgb.size() * sizeof(float),
                                       cudaMemcpyHostToDevice, s),
                       "histogram tile");
            count(dev.data, dev.stride, expected.width, expected.height, 0, first);
            first += pixels;
            next_x += expected.width;
            if (next_x == right) {
                next_x = vp.x;
                next_y += expected.height;
            }
            check_cancelled();
        }, cancellation);
    }
    std::vector<uint64_t> host((size_t)3 * options.bins + 15);
    check_cuda(cudaMemcpyAsync(host.data(), hc.base, host.size() * sizeof(uint64_t), cudaMemcpyDeviceToHost, s),
               "histogram");
    check_cuda(cudaStreamSynchronize(s), "histogram");
    check_cancelled();
    const uint64_t* tallies = host.data() + (size_t)3 * options.bins;
    const uint64_t* keys = tallies + 9;
    for (int c = 0; c < 3; ++c) {
        ChannelHistogram& ch = result.channels[c];
        ch.counts.assign(host.begin() + (size_t)c * options.bins, host.begin() + (size_t)(c + 1) * options.bins);
        ch.underflow = tallies[c];
        ch.overflow = tallies[3 + c];
        ch.nonfinite = tallies[6 + c];
        float v = 0;
        if (re_histogram_extremum(keys[c], 0, &v)) ch.minimum = v;
        if (re_histogram_extremum(keys[3 + c], 1, &v)) ch.maximum = v;
    }
    result.pixel_count = (uint64_t)vp.width * vp.height;
    return result;
}

RgbHistogram histogram_rgb(const ImageGraph& graph, const RenderRequest& request, const HistogramOptions& options,
                           const CancellationToken* cancellation) {
    return histogram_rgb(graph.output(), graph.source_bounds(), request, options, cancellation);
}

// ----------------------------------------------------------- TileScheduler

namespace {

// A request whose chain is a RAW source under point nodes only, lowered to the
// fused render the executor would launch for it (Executor::eval_raw): the
// device image and the render description.  Returns false for any other chain
// (spatial, geometry, raster or caller nodes), and for chains the executor
// must reject, so that the error comes from the executor as it would for a
// direct render.
struct RawLowering {
    const re_image* image = nullptr;
    re_render_desc desc{};
    // a cubic resize or rotation between the RAW chain and later point stages
    uint32_t geometry = 0, canvas_width = 0, canvas_height = 0;
    double angle = 0;
    re_render_desc post{};
};

bool lower_raw_chain(const Node& node, RenderLevel level, RawLowering& out) {
    if (!node.supports_level(level)) return false;
    std::vector<const PointNode*> chain;
    const Node* cur = &node;
    while (auto* p = dynamic_cast<const PointNode*>(cur)) {
        chain.push_back(p);
        cur = p->input().get();
    }
    auto* raw = dynamic_cast<const RawUnpackNode*>(cur);
    if (!raw) return false;
    std::reverse(chain.begin(), chain.end());
    int anchor = -1;
    for (int i = (int)chain.size() - 1; i >= 0 && level.mip; --i)
        if (dynamic_cast<const CameraToWorkingNode*>(chain[i])) {
            anchor = i;
            break;
        }
    StageList sl;
    sl.desc.demosaic = raw->menon() ? 1u : 0u;
    sl.desc.anchor = -1;
    try {
        for (int i = 0; i < (int)chain.size(); ++i) add_stage(sl, chain[i], i == anchor, level);
        if (level.mip && sl.desc.anchor < 0) return false;
        out.image = raw->image().device().handle;
    } catch (...) {
        return false;
    }
    out.desc = sl.desc;
    return true;
}

// A request whose chain is point nodes over one CubicResizeNode or RotateNode
// over a RAW point chain (whose extent is the geometry's input bounds),
// lowered to a geometry item: the RAW chain at native resolution, the
// geometry, the point stages after it.
bool lower_geometry_chain(const Node& node, RenderLevel level, RawLowering& out) {
    if (!node.supports_level(level)) return false;
    std::vector<const PointNode*> chain;
    const Node* cur = &node;
    while (auto* p = dynamic_cast<const PointNode*>(cur)) {
        chain.push_back(p);
        cur = p->input().get();
    }
    std::reverse(chain.begin(), chain.end());
    const Node* input = nullptr;
    Rect bounds;
    if (auto* cr = dynamic_cast<const CubicResizeNode*>(cur)) {
        out.geometry = 1;
        out.canvas_width = cr->settings().width;
        out.canvas_height = cr->settings().height;
        input = cr->input_node();
        bounds = cr->input_bounds();
    } else if (auto* ro = dynamic_cast<const RotateNode*>(cur)) {
        out.geometry = 2;
        out.angle = ro->angle();
        input = ro->input_node();
        bounds = ro->input_bounds();
    } else {
        return false;
    }
    if (!input || !cur->supports_level(level) || !lower_raw_chain(*input, {}, out)) return false;
    const Node* src = input;
    while (auto* p = dynamic_cast<const PointNode*>(src)) src = p->input().get();
    auto* raw = dynamic_cast<const RawUnpackNode*>(src);
    if (!raw || !same(raw->image().metadata().active_area, bounds)) return false;
    StageList post;
    post.desc.anchor = -1;
    try {
        for (const PointNode* p : chain) add_stage(post, p, false, {});
    } catch (...) {
        return false;
    }
    out.post = post.desc;
    return true;
}

// Canonical bytes of a render description, so that requests with equal
// recipes share one device program inside a batch.
std::string desc_key(const re_render_desc& d) {
    std::string k;
    auto put = [&](const void* p, size_t n) { k.append(static_cast<const char*>(p), n); };
    put(&d.demosaic, sizeof d.demosaic);
    put(&d.anchor, sizeof d.anchor);
    put(&d.count, sizeof d.count);
    for (uint32_t i = 0; i < d.count && i < RE_MAX_STAGES; ++i) {
        put(&d.stages[i].kind, sizeof(uint32_t));
        put(&d.stages[i].arg, sizeof(uint32_t));
        put(d.stages[i].f, sizeof d.stages[i].f);
    }
    put(d.curves, sizeof d.curves);
    return k;
}

// Device memory handed out in DeviceTiles: freed stream-ordered on the legacy
// default stream once the last tile that points into it is released.
std::shared_ptr<float> device_block(size_t bytes, cudaStream_t s) {
    float* p = nullptr;
    if (bytes) check_cuda(re::scratch_alloc((void**)&p, bytes, s), "scheduler output");
    return std::shared_ptr<float>(p, [](float* q) {
        if (q) cudaFreeAsync(q, nullptr);
    });
}

}  // namespace

Tile DeviceTile::to_host() const {
    Tile t{bounds, std::vector<float>((size_t)bounds.width * bounds.height * 3), descriptor};
    if (!t.rgb.empty())
        check_cuda(cudaMemcpy(t.rgb.data(), rgb.get(), t.rgb.size() * sizeof(float), cudaMemcpyDeviceToHost),
                   "device tile download");
    return t;
}

// --------------------------------------------------------------- TileCache

struct TileCache::Impl {
    struct Key {
        std::array<std::uint8_t, 32> signature{};
        std::array<std::uint32_t, 4> bounds{};
        std::uint32_t mip = 0;
        RenderQuality quality = RenderQuality::Final;
        auto operator<=>(const Key&) const = default;
    };
    struct Entry {
        DeviceTile tile;
        std::list<Key>::iterator recency;
        std::size_t charged = 0;
    };
    std::size_t max_bytes = 0, used = 0, hits = 0, misses = 0;
    std::uint64_t generation = 0;
    std::map<Key, Entry> entries;
    std::list<Key> recency;
    mutable std::mutex mu;
};

TileCache::TileCache(std::size_t max_bytes) : impl_(std::make_unique<Impl>()) { impl_->max_bytes = max_bytes; }
TileCache::~TileCache() = default;

namespace {
// One tile of `node` in device memory: device nodes through the executor,
// other nodes through their own render_level, validated as the reference
// validates cache tiles (EditGraph.cpp:46-52), then uploaded.
DeviceTile render_to_device(const Node& node, Rect bounds, RenderLevel level) {
    cudaStream_t s = thread_stream();
    const size_t row = (size_t)bounds.width * 3;
    DeviceTile d{bounds, nullptr, node.output_descriptor()};
    auto block = device_block(row * bounds.height * sizeof(float), s);
    if (dynamic_cast<const DeviceNode*>(&node)) {
        Executor ex{s, nullptr};
        DevPtr img = ex.eval(node, bounds, level);
        if (bounds.width && bounds.height)
            check_cuda(cudaMemcpy2DAsync(block.get(), row * sizeof(float), img->data, img->stride * sizeof(float),
                                         row * sizeof(float), bounds.height, cudaMemcpyDeviceToDevice, s),
                       "cache tile");
    } else {
        const Tile t = node.render_level(bounds, level);
        const uint64_t pixels = (uint64_t)bounds.width * bounds.height;
        if (!same(t.bounds, bounds) || t.descriptor != node.output_descriptor() || t.rgb.size() != pixels * 3)
            throw std::domain_error("node returned an invalid cache tile");
        if (!t.rgb.empty())
            check_cuda(cudaMemcpyAsync(block.get(), t.rgb.data(), t.rgb.size() * sizeof(float),
                                       cudaMemcpyHostToDevice, s),
                       "cache tile");
    }
    check_cuda(cudaStreamSynchronize(s), "cache tile");
    d.rgb = block;
    return d;
}
}  // namespace

// EditGraph.cpp:23-80
DeviceTile TileCache::render_device(const Node& node, std::array<std::uint8_t, 32> signature, Rect bounds,
                                    RenderLevel level) {
    if (level.mip > 31 || (level.quality != RenderQuality::Preview && level.quality != RenderQuality::Final))
        throw std::invalid_argument("invalid cache render level");
    if (!node.supports_level(level)) throw std::invalid_argument("node does not support this cache render level");
    Impl& m = *impl_;
    const Impl::Key key{signature, {bounds.x, bounds.y, bounds.width, bounds.height}, level.mip, level.quality};
    std::uint64_t generation;
    {
        std::lock_guard<std::mutex> lock(m.mu);
        if (auto found = m.entries.find(key); found != m.entries.end()) {
            ++m.hits;
            m.recency.splice(m.recency.begin(), m.recency, found->second.recency);
            return found->second.tile;
        }
        ++m.misses;
        generation = m.generation;
    }
    DeviceTile tile = render_to_device(node, bounds, level);
    constexpr std::size_t entry_charge = 256;
    const std::size_t floats = (std::size_t)bounds.width * bounds.height * 3;
    if (!floats || floats > (m.max_bytes - std::min(m.max_bytes, entry_charge)) / sizeof(float)) return tile;
    const std::size_t charge = entry_charge + floats * sizeof(float);
    std::lock_guard<std::mutex> lock(m.mu);
    if (generation != m.generation) return tile;
    if (auto found = m.entries.find(key); found != m.entries.end()) {
        ++m.hits;
        m.recency.splice(m.recency.begin(), m.recency, found->second.recency);
        return found->second.tile;
    }
    while (m.used > m.max_bytes - charge) {
        const auto oldest = std::prev(m.recency.end());
        m.used -= m.entries.at(*oldest).charged;
        m.entries.erase(*oldest);
        m.recency.erase(oldest);
    }
    m.recency.push_front(key);
    m.entries.emplace(key, Impl::Entry{tile, m.recency.begin(), charge});
    m.used += charge;
    return tile;
}

Tile TileCache::render(const Node& node, std::array<std::uint8_t, 32> signature, Rect bounds, RenderLevel level) {
    return render_device(node, signature, bounds, level).to_host();
}

TileCache::Stats TileCache::stats() const {
    std::lock_guard<std::mutex> lock(impl_->mu);
    return {impl_->entries.size(), impl_->used, impl_->hits, impl_->misses};
}

void TileCache::clear() {
    std::lock_guard<std::mutex> lock(impl_->mu);
    ++impl_->generation;
    impl_->entries.clear();
    impl_->recency.clear();
    impl_->used = 0;
    impl_->hits = 0;
    impl_->misses = 0;
}

CachedNode::CachedNode(std::shared_ptr<const Node> input, std::shared_ptr<TileCache> cache,
                       std::array<std::uint8_t, 32> signature)
    : input_(std::move(input)), cache_(std::move(cache)), signature_(signature) {
    if (!input_ || !cache_) throw std::invalid_argument("cached node requires an input and a cache");
}

// Pending requests sit in one ordered map keyed by (descending priority,
// arrival), with a count per supersession group for the budget rule.  Lanes
// take WAVES: everything pending (up to a request and byte limit) in key order.
// Taken requests stay listed as in flight until their futures resolve, so that
// a newer request of their group can cancel them.
struct TileScheduler::Impl {
    struct Request {
        std::shared_ptr<const Node> node;
        Rect source_bounds;
        RenderRequest request;
        std::shared_ptr<CancellationToken> token;
        std::string group;
        bool device = false;
        std::promise<Tile> host_result;
        std::promise<DeviceTile> device_result;

        bool cancelled() const { return token && token->is_cancelled(); }
        void fail(std::exception_ptr e) {
            if (device) device_result.set_exception(e);
            else host_result.set_exception(e);
        }
        uint64_t bytes() const { return (uint64_t)request.viewport.width * request.viewport.height * 12; }
    };
    using RequestPtr = std::shared_ptr<Request>;
    using Order = std::pair<int, uint64_t>;

    static constexpr size_t kWaveRequests = 8192;
    static constexpr uint64_t kWaveBytes = 3ull << 30;   // device outputs of one wave

    struct Lane {
        cudaStream_t stream = nullptr;   // batched renders and their copies
        re_batch* batch = nullptr;
        float* staging = nullptr;        // pinned host copy of a wave's host tiles
        size_t staging_floats = 0;
        std::thread thread;
    };

    Impl(size_t lanes, size_t budget) : budget_(budget) {
        if (!lanes || lanes > 64 || !budget)
            throw std::invalid_argument("scheduler needs 1-64 workers and a pending budget");
        if (cudaGetDevice(&device_) != cudaSuccess) device_ = 0;   // lanes then report the error per request
        copy_threads_ = std::max<size_t>(1, std::min<size_t>(8, std::thread::hardware_concurrency() / lanes));
        lanes_.resize(lanes);
        try {
            for (Lane& lane : lanes_) lane.thread = std::thread([this, &lane] { run_lane(lane); });
        } catch (...) {
            close();   // joins the lanes that did start
            throw;
        }
    }

    ~Impl() { close(); }

    // Fails every pending request with RenderCancelled, lets each lane finish
    // the wave it holds, and joins the lanes.
    void close() {
        std::vector<RequestPtr> dropped;
        {
            std::lock_guard<std::mutex> lock(mu_);
            closing_ = true;
            for (auto& entry : pending_) dropped.push_back(std::move(entry.second));
            pending_.clear();
            pending_in_group_.clear();
        }
        for (auto& r : dropped) r->fail(std::make_exception_ptr(RenderCancelled()));
        wake_.notify_all();
        for (Lane& lane : lanes_)
            if (lane.thread.joinable()) lane.thread.join();
    }

    // Adds a request (the budget and supersession rules of TileScheduler.cpp:122-160).
    void add(RequestPtr r, RenderPriority priority) {
        std::vector<RequestPtr> superseded;
        {
            std::lock_guard<std::mutex> lock(mu_);
            const size_t replaceable = r->group.empty() ? 0 : count_in_group(r->group);
            if (pending_.size() - replaceable >= budget_)
                throw std::length_error("scheduler pending request budget is full");
            if (!r->group.empty()) {
                for (auto it = pending_.begin(); it != pending_.end();) {
                    if (it->second->group == r->group) {
                        if (it->second->token) it->second->token->cancel();
                        superseded.push_back(std::move(it->second));
                        it = pending_.erase(it);
                    } else {
                        ++it;
                    }
                }
                for (const RequestPtr& f : in_flight_)
                    if (f->group == r->group && f->token) f->token->cancel();
                pending_in_group_[r->group] = 1;
            }
            pending_.emplace(Order{-(int)priority, next_arrival_++}, std::move(r));
        }
        for (auto& s : superseded) s->fail(std::make_exception_ptr(RenderCancelled()));
        wake_.notify_one();
    }

    Stats stats() const {
        std::lock_guard<std::mutex> lock(mu_);
        return stats_;
    }

private:
    size_t count_in_group(const std::string& g) const {
        auto it = pending_in_group_.find(g);
        return it == pending_in_group_.end() ? 0 : it->second;
    }

    // Blocks until requests are pending (or the scheduler closes: empty wave).
    std::vector<RequestPtr> take_wave() {
        std::unique_lock<std::mutex> lock(mu_);
        wake_.wait(lock, [&] { return closing_ || !pending_.empty(); });
        std::vector<RequestPtr> wave;
        uint64_t bytes = 0;
        while (!pending_.empty() && wave.size() < kWaveRequests) {
            const RequestPtr& next = pending_.begin()->second;
            if (!wave.empty() && bytes + next->bytes() > kWaveBytes) break;
            bytes += next->bytes();
            if (!next->group.empty()) --pending_in_group_[next->group];
            in_flight_.push_back(next);
            wave.push_back(next);
            pending_.erase(pending_.begin());
        }
        if (!wave.empty()) ++stats_.waves;
        return wave;
    }

    void retire(const std::vector<RequestPtr>& wave) {
        std::lock_guard<std::mutex> lock(mu_);
        for (const RequestPtr& r : wave) {
            auto it = std::find(in_flight_.begin(), in_flight_.end(), r);
            if (it != in_flight_.end()) in_flight_.erase(it);
        }
    }

    void run_lane(Lane& lane) {
        cudaSetDevice(device_);
        if (cudaStreamCreateWithFlags(&lane.stream, cudaStreamNonBlocking) != cudaSuccess) lane.stream = nullptr;
        if (re_batch_create(&lane.batch) != RE_OK) lane.batch = nullptr;
        for (;;) {
            std::vector<RequestPtr> wave = take_wave();
            if (wave.empty()) break;
            render_wave(lane, wave);
            retire(wave);
        }
        if (lane.batch) re_batch_destroy(lane.batch);
        if (lane.staging) cudaFreeHost(lane.staging);
        if (lane.stream) cudaStreamDestroy(lane.stream);
    }

    // One request through its node on this thread's executor stream, exactly
    // as Renderer::render_image would render it.
    void render_one(Request& r) {
        try {
            if (r.cancelled()) throw RenderCancelled();
            if (!r.device) {
                Tile t = Renderer().render_image(*r.node, r.source_bounds, r.request, r.token.get());
                if (r.cancelled()) throw RenderCancelled();
                r.host_result.set_value(std::move(t));
                return;
            }
            validate_request(*r.node, r.source_bounds, r.request, r.token.get());
            cudaStream_t s = thread_stream();
            DeviceTile d{r.request.viewport, nullptr, r.node->output_descriptor()};
            const Rect vp = r.request.viewport;
            const size_t row = (size_t)vp.width * 3;
            auto block = device_block(row * vp.height * sizeof(float), s);
            if (dynamic_cast<const DeviceNode*>(r.node.get())) {
                Executor ex{s, r.token.get()};
                DevPtr img = ex.eval(*r.node, vp, r.request.level);
                if (vp.width && vp.height)
                    check_cuda(cudaMemcpy2DAsync(block.get(), row * sizeof(float), img->data,
                                                 img->stride * sizeof(float), row * sizeof(float), vp.height,
                                                 cudaMemcpyDeviceToDevice, s),
                               "device tile");
            } else {
                Tile t = Renderer().render_image(*r.node, r.source_bounds, r.request, r.token.get());
                if (!t.rgb.empty())
                    check_cuda(cudaMemcpyAsync(block.get(), t.rgb.data(), t.rgb.size() * sizeof(float),
                                               cudaMemcpyHostToDevice, s),
                               "device tile");
            }
            check_cuda(cudaStreamSynchronize(s), "device tile");
            if (r.cancelled()) throw RenderCancelled();
            d.rgb = block;
            r.device_result.set_value(std::move(d));
        } catch (...) {
            r.fail(std::current_exception());
        }
    }

    void add_time(double Stats::*field, std::chrono::steady_clock::time_point& since) {
        const auto now = std::chrono::steady_clock::now();
        std::lock_guard<std::mutex> lock(mu_);
        stats_.*field += std::chrono::duration<double>(now - since).count();
        since = now;
    }

    void render_wave(Lane& lane, const std::vector<RequestPtr>& wave) {
        auto mark = std::chrono::steady_clock::now();
        // 1. split: cancelled requests fail now; RAW point chains join the batch
        std::vector<Request*> batched, by_node;
        std::vector<RawLowering> lowered;
        lowered.reserve(wave.size());
        for (const RequestPtr& r : wave) {
            if (r->cancelled()) {
                r->fail(std::make_exception_ptr(RenderCancelled()));
                continue;
            }
            RawLowering L;
            const Rect vp = r->request.viewport;
            const bool batchable = lane.batch && lane.stream && vp.width && vp.height &&
                                   dynamic_cast<const DeviceNode*>(r->node.get()) &&
                                   (lower_raw_chain(*r->node, r->request.level, L) ||
                                    lower_geometry_chain(*r->node, r->request.level, (L = RawLowering{})));
            if (batchable) {
                lowered.push_back(L);
                batched.push_back(r.get());
            } else {
                by_node.push_back(r.get());
            }
        }
        add_time(&Stats::lower_s, mark);
        // 2. one output block for the batch; requests with equal recipes share a program
        bool launched = false;
        std::shared_ptr<float> block;
        std::vector<size_t> offset(batched.size());
        std::map<std::string, const re_render_desc*> programs;
        if (!batched.empty()) {
            size_t floats = 0;
            for (size_t i = 0; i < batched.size(); ++i) {
                offset[i] = floats;
                const Rect vp = batched[i]->request.viewport;
                floats += ((size_t)vp.width * vp.height * 3 + 63) & ~(size_t)63;
            }
            std::vector<re_batch_item> items(batched.size());
            try {
                block = device_block(floats * sizeof(float), lane.stream);
                for (size_t i = 0; i < batched.size(); ++i) {
                    const Request& r = *batched[i];
                    const RawLowering& L = lowered[i];
                    const re_render_desc*& shared = programs[desc_key(L.desc)];
                    if (!shared) shared = &L.desc;
                    re_batch_item& it = items[i];
                    it = re_batch_item{};
                    it.image = L.image;
                    it.desc = shared;
                    it.viewport = to_re(r.request.viewport);
                    it.mip = r.request.level.mip;
                    it.quality = (uint32_t)r.request.level.quality;
                    it.out = block.get() + offset[i];
                    it.out_row_stride = (size_t)r.request.viewport.width * 3;
                    if (L.geometry) {
                        it.geometry = L.geometry;
                        it.canvas_width = L.canvas_width;
                        it.canvas_height = L.canvas_height;
                        it.angle_degrees = L.angle;
                        const re_render_desc*& post = programs["post" + desc_key(L.post)];
                        if (!post) post = &L.post;
                        it.post = post;
                    }
                }
                re_batch_options opt{};
                opt.dispatch = 2;
                opt.ctas_per_sm = 4;
                opt.order = 1;
                opt.use_graph = 0;
                launched = re_batch_plan(lane.batch, items.data(), items.size(), &opt) == RE_OK &&
                           re_batch_launch(lane.batch, lane.stream) == RE_OK;
                if (!launched) note_fallback(std::string("batch plan/launch: ") + re_last_error());
            } catch (const std::exception& e) {
                launched = false;
                note_fallback(std::string("batch outputs: ") + e.what());
            }
        }
        add_time(&Stats::plan_s, mark);
        // 3. the other requests render through their nodes while the batch runs
        //    (statistics are updated before any future of the wave resolves)
        count(0, by_node.size(), by_node.size());
        for (Request* r : by_node) render_one(*r);
        // 4. deliver the batch; if it failed as a whole, each request renders
        //    alone so that it gets its own error, as a direct render reports it
        if (launched && re_batch_status(lane.batch, lane.stream) != RE_OK) {
            launched = false;
            note_fallback(std::string("batch status: ") + re_last_error());
        }
        add_time(&Stats::device_s, mark);
        if (!launched) {
            count(0, batched.size(), 0);
            for (Request* r : batched) render_one(*r);
        } else {
            count(batched.size(), 0, 0);
            deliver(lane, batched, block, offset);
        }
        add_time(&Stats::deliver_s, mark);
    }

    void count(size_t batched, size_t node, size_t unbatchable) {
        std::lock_guard<std::mutex> lock(mu_);
        stats_.batched_requests += batched;
        stats_.node_requests += node;
        stats_.unbatchable_requests += unbatchable;
    }

    void note_fallback(const std::string& why) {
        std::lock_guard<std::mutex> lock(mu_);
        ++stats_.batch_fallbacks;
        stats_.last_fallback = why;
    }

    void deliver(Lane& lane, const std::vector<Request*>& batched, const std::shared_ptr<float>& block,
                 const std::vector<size_t>& offset) {
        // Host tiles: one copy of the wave's output block into the lane's
        // pinned staging buffer, then every tile's vector is constructed from
        // its slice (no zero fill; each page is touched once), spread over a
        // few host threads when the wave is large.
        std::vector<Tile> host(batched.size());
        std::vector<size_t> wanted;
        size_t end = 0;
        for (size_t i = 0; i < batched.size(); ++i)
            if (!batched[i]->device) {
                wanted.push_back(i);
                const Rect vp = batched[i]->request.viewport;
                end = std::max(end, offset[i] + (size_t)vp.width * vp.height * 3);
            }
        bool copied = true;
        if (!wanted.empty()) {
            if (lane.staging_floats < end) {
                if (lane.staging) cudaFreeHost(lane.staging);
                lane.staging = nullptr;
                lane.staging_floats = 0;
                copied = cudaHostAlloc((void**)&lane.staging, end * sizeof(float), cudaHostAllocDefault) ==
                         cudaSuccess;
                if (copied) lane.staging_floats = end;
            }
            copied = copied && cudaMemcpyAsync(lane.staging, block.get(), end * sizeof(float),
                                               cudaMemcpyDeviceToHost, lane.stream) == cudaSuccess &&
                     cudaStreamSynchronize(lane.stream) == cudaSuccess;
        }
        if (copied && !wanted.empty()) {
            auto build = [&](size_t from, size_t to) {
                for (size_t k = from; k < to; ++k) {
                    const size_t i = wanted[k];
                    const Request& r = *batched[i];
                    const float* src = lane.staging + offset[i];
                    const size_t n = (size_t)r.request.viewport.width * r.request.viewport.height * 3;
                    host[i] = Tile{r.request.viewport, std::vector<float>(src, src + n), r.node->output_descriptor()};
                }
            };
            const size_t parts = end * sizeof(float) < (size_t(32) << 20) ? 1 : copy_threads_;
            std::vector<std::thread> helpers;
            const size_t per = (wanted.size() + parts - 1) / parts;
            for (size_t p = 1; p < parts && p * per < wanted.size(); ++p)
                helpers.emplace_back(build, p * per, std::min(wanted.size(), (p + 1) * per));
            build(0, std::min(wanted.size(), per));
            for (auto& h : helpers) h.join();
        }
        for (size_t i = 0; i < batched.size(); ++i) {
            Request& r = *batched[i];
            if (!copied) {
                r.fail(std::make_exception_ptr(std::runtime_error("scheduler result download failed")));
            } else if (r.cancelled()) {
                r.fail(std::make_exception_ptr(RenderCancelled()));
            } else if (r.device) {
                // the tile shares the wave's block (aliasing pointer)
                r.device_result.set_value(DeviceTile{r.request.viewport,
                                                     std::shared_ptr<const float>(block, block.get() + offset[i]),
                                                     r.node->output_descriptor()});
            } else {
                r.host_result.set_value(std::move(host[i]));
            }
        }
    }

    const size_t budget_;
    size_t copy_threads_ = 1;
    int device_ = 0;
    mutable std::mutex mu_;
    std::condition_variable wake_;
    std::map<Order, RequestPtr> pending_;
    std::map<std::string, size_t> pending_in_group_;
    std::vector<RequestPtr> in_flight_;
    std::vector<Lane> lanes_;
    uint64_t next_arrival_ = 0;
    bool closing_ = false;
    Stats stats_;
};

TileScheduler::TileScheduler(std::size_t workers, std::size_t max_pending)
    : impl_(std::make_unique<Impl>(workers, max_pending)) {}
TileScheduler::~TileScheduler() = default;

TileScheduler::Stats TileScheduler::stats() const { return impl_->stats(); }

namespace {
// TileScheduler.cpp:205-236: the argument checks of a scheduled request.
void validate_scheduled(const std::shared_ptr<const Node>& output, Rect source_bounds, const RenderRequest& request,
                        RenderPriority priority) {
    const Rect vp = request.viewport;
    const bool native = level_any_native(request.level);
    const bool reduced = level_reduced(request.level);
    const uint32_t scale = reduced ? 1u << request.level.mip : 1u;
    const Rect bounds = reduced ? Rect{0, 0, source_bounds.width / scale + (source_bounds.width % scale != 0),
                                       source_bounds.height / scale + (source_bounds.height % scale != 0)}
                                : source_bounds;
    if (!output || !request.tile_size || (!native && !reduced) || !output->supports_level(request.level) ||
        !source_bounds.width || !source_bounds.height || (int)priority < 0 || (int)priority > 2 ||
        !addressable(source_bounds) || !contains(bounds, vp))
        throw std::invalid_argument("invalid scheduled render request");
}
}  // namespace

std::future<Tile> TileScheduler::submit(std::shared_ptr<const Node> output, Rect source_bounds, RenderRequest request,
                                        RenderPriority priority, std::shared_ptr<CancellationToken> cancellation) {
    validate_scheduled(output, source_bounds, request, priority);
    auto r = std::make_shared<Impl::Request>();
    *r = Impl::Request{std::move(output), source_bounds, request, std::move(cancellation), {}, false, {}, {}};
    auto f = r->host_result.get_future();
    impl_->add(std::move(r), priority);
    return f;
}
std::future<Tile> TileScheduler::submit(std::shared_ptr<const Node> output, Rect source_bounds, Rect viewport,
                                        RenderPriority priority, std::uint32_t tile_size,
                                        std::shared_ptr<CancellationToken> cancellation) {
    return submit(std::move(output), source_bounds, RenderRequest{viewport, tile_size, {}}, priority,
                  std::move(cancellation));
}
std::future<Tile> TileScheduler::submit_latest(std::string group, std::shared_ptr<const Node> output,
                                               Rect source_bounds, RenderRequest request, RenderPriority priority,
                                               std::shared_ptr<CancellationToken> cancellation) {
    if (group.empty()) throw std::invalid_argument("latest request group is empty");
    validate_scheduled(output, source_bounds, request, priority);
    if (!cancellation) cancellation = std::make_shared<CancellationToken>();
    auto r = std::make_shared<Impl::Request>();
    *r = Impl::Request{std::move(output), source_bounds, request, std::move(cancellation), std::move(group), false,
                       {}, {}};
    auto f = r->host_result.get_future();
    impl_->add(std::move(r), priority);
    return f;
}
std::future<Tile> TileScheduler::submit_latest(std::string group, std::shared_ptr<const Node> output,
                                               Rect source_bounds, Rect viewport, RenderPriority priority,
                                               std::uint32_t tile_size,
                                               std::shared_ptr<CancellationToken> cancellation) {
    return submit_latest(std::move(group), std::move(output), source_bounds, RenderRequest{viewport, tile_size, {}},
                         priority, std::move(cancellation));
}
std::future<DeviceTile> TileScheduler::submit_device(std::shared_ptr<const Node> output, Rect source_bounds,
                                                     RenderRequest request, RenderPriority priority,
                                                     std::shared_ptr<CancellationToken> cancellation) {
    validate_scheduled(output, source_bounds, request, priority);
    auto r = std::make_shared<Impl::Request>();
    *r = Impl::Request{std::move(output), source_bounds, request, std::move(cancellation), {}, true, {}, {}};
    auto f = r->device_result.get_future();
    impl_->add(std::move(r), priority);
    return f;
}
std::future<DeviceTile> TileScheduler::submit_latest_device(std::string group, std::shared_ptr<const Node> output,
                                                            Rect source_bounds, RenderRequest request,
                                                            RenderPriority priority,
                                                            std::shared_ptr<CancellationToken> cancellation) {
    if (group.empty()) throw std::invalid_argument("latest request group is empty");
    validate_scheduled(output, source_bounds, request, priority);
    if (!cancellation) cancellation = std::make_shared<CancellationToken>();
    auto r = std::make_shared<Impl::Request>();
    *r = Impl::Request{std::move(output), source_bounds, request, std::move(cancellation), std::move(group), true,
                       {}, {}};
    auto f = r->device_result.get_future();
    impl_->add(std::move(r), priority);
    return f;
}

}  // namespace rawengine
