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
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <queue>
#include <thread>

#include <cuda_runtime.h>

#include "rawengine/Operators.hpp"
#include "rawengine_b200.h"

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
    DevImage(Rect r, cudaStream_t s) : stride((size_t)r.width * 3), bounds(r), stream(s) {
        if (r.width && r.height)
            check_cuda(cudaMallocAsync((void**)&data, (size_t)r.width * r.height * 3 * sizeof(float), s),
                       "device tile");
    }
    ~DevImage() {
        if (data) cudaFreeAsync(data, stream);
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
// which is outside this build: IccDisplay is rejected as unsupported)
ImageGraph::ImageGraph(RawImage image, GraphRecipe recipe)
    : raw_image_(std::move(image)), source_bounds_(raw_image_->metadata().active_area), recipe_(recipe) {
    auto node = std::make_shared<RawUnpackNode>(*raw_image_);
    auto wb = std::make_shared<WhiteBalanceNode>(node, recipe.red_gain, recipe.green_gain, recipe.blue_gain);
    std::shared_ptr<const Node> linear = std::make_shared<ExposureNode>(wb, recipe.exposure_stops);
    if (recipe.camera_color)
        linear = std::make_shared<CameraToWorkingNode>(linear, *recipe.camera_color, source_bounds_);
    if (recipe.output_mode == OutputMode::SrgbPreview) linear = std::make_shared<WorkingToSrgbNode>(linear);
    else if (recipe.output_mode != OutputMode::LegacyBounded)
        throw std::invalid_argument("ICC display output is not available in this build");
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
        throw std::invalid_argument("ICC display output is not available in this build");
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
    check_cuda(cudaMallocAsync(&scratch, n_needed * (2 * sizeof(double) + sizeof(uint32_t)), s), "statistics");
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

// ----------------------------------------------------------- TileScheduler

// The queue semantics of TileScheduler.cpp:19-304: priority then FIFO, a
// pending budget (length_error) in which queued requests of the caller's
// supersession group do not count, a new group request cancelling the group's
// running request and failing its queued ones, destruction failing pending
// requests and waiting for running ones.  Queued jobs live in one ordered map
// keyed by (descending priority, arrival), with a per-group count; each worker
// thread renders on its own CUDA stream, so requests on different workers
// overlap on the device.
struct TileScheduler::Impl {
    struct Job {
        std::shared_ptr<const Node> output;
        Rect source_bounds;
        RenderRequest request;
        std::shared_ptr<CancellationToken> cancellation;
        std::string group;
        std::promise<Tile> result;
    };
    using Key = std::pair<int, uint64_t>;  // (-priority, arrival)

    Impl(size_t workers, size_t budget) : budget(budget) {
        if (!workers || workers > 64 || !budget)
            throw std::invalid_argument("scheduler needs 1-64 workers and a pending budget");
        try {
            for (size_t i = 0; i < workers; ++i) threads.emplace_back([this] { work(); });
        } catch (...) {
            shutdown();
            throw;
        }
    }
    ~Impl() { shutdown(); }

    void shutdown() {
        {
            std::lock_guard<std::mutex> lock(mutex);
            stopping = true;
            for (auto& [key, job] : queued) job->result.set_exception(std::make_exception_ptr(RenderCancelled()));
            queued.clear();
            group_count.clear();
            latest.clear();
        }
        ready.notify_all();
        for (auto& t : threads)
            if (t.joinable()) t.join();
    }

    std::shared_ptr<Job> take() {
        std::unique_lock<std::mutex> lock(mutex);
        ready.wait(lock, [&] { return stopping || !queued.empty(); });
        if (queued.empty()) return nullptr;
        auto job = std::move(queued.begin()->second);
        queued.erase(queued.begin());
        if (!job->group.empty()) --group_count[job->group];
        return job;
    }

    void work() {
        while (auto job = take()) {
            std::optional<Tile> tile;
            std::exception_ptr failure;
            try {
                if (job->cancellation && job->cancellation->is_cancelled()) throw RenderCancelled();
                tile = Renderer().render_image(*job->output, job->source_bounds, job->request, job->cancellation.get());
            } catch (...) {
                failure = std::current_exception();
            }
            std::lock_guard<std::mutex> lock(mutex);
            if (!failure && job->cancellation && job->cancellation->is_cancelled())
                failure = std::make_exception_ptr(RenderCancelled());
            if (failure) job->result.set_exception(failure);
            else job->result.set_value(std::move(*tile));
            if (!job->group.empty()) {
                auto it = latest.find(job->group);
                if (it != latest.end() && it->second.lock() == job->cancellation) latest.erase(it);
            }
        }
    }

    void enqueue(std::shared_ptr<Job> job, RenderPriority priority) {
        {
            std::lock_guard<std::mutex> lock(mutex);
            const size_t replaced = job->group.empty() ? 0 : group_count[job->group];
            if (queued.size() - replaced >= budget) throw std::length_error("scheduler pending request budget is full");
            if (!job->group.empty()) {
                if (auto it = latest.find(job->group); it != latest.end())
                    if (auto running = it->second.lock()) running->cancel();
                for (auto it = queued.begin(); it != queued.end();) {
                    if (it->second->group != job->group) {
                        ++it;
                        continue;
                    }
                    it->second->cancellation->cancel();
                    it->second->result.set_exception(std::make_exception_ptr(RenderCancelled()));
                    it = queued.erase(it);
                }
                group_count[job->group] = 1;
                latest[job->group] = job->cancellation;
            }
            queued.emplace(Key{-(int)priority, arrivals++}, std::move(job));
        }
        ready.notify_one();
    }

    const size_t budget;
    std::mutex mutex;
    std::condition_variable ready;
    std::map<Key, std::shared_ptr<Job>> queued;
    std::map<std::string, size_t> group_count;
    std::map<std::string, std::weak_ptr<CancellationToken>> latest;
    std::vector<std::thread> threads;
    uint64_t arrivals = 0;
    bool stopping = false;
};

TileScheduler::TileScheduler(std::size_t workers, std::size_t max_pending)
    : impl_(std::make_unique<Impl>(workers, max_pending)) {}
TileScheduler::~TileScheduler() = default;

std::future<Tile> TileScheduler::submit(std::shared_ptr<const Node> output, Rect source_bounds, RenderRequest request,
                                        RenderPriority priority, std::shared_ptr<CancellationToken> cancellation) {
    return submit_request({}, std::move(output), source_bounds, request, priority, std::move(cancellation));
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
    if (!cancellation) cancellation = std::make_shared<CancellationToken>();
    return submit_request(std::move(group), std::move(output), source_bounds, request, priority,
                          std::move(cancellation));
}
std::future<Tile> TileScheduler::submit_latest(std::string group, std::shared_ptr<const Node> output,
                                               Rect source_bounds, Rect viewport, RenderPriority priority,
                                               std::uint32_t tile_size,
                                               std::shared_ptr<CancellationToken> cancellation) {
    return submit_latest(std::move(group), std::move(output), source_bounds, RenderRequest{viewport, tile_size, {}},
                         priority, std::move(cancellation));
}

// TileScheduler.cpp:205-236
std::future<Tile> TileScheduler::submit_request(std::string group, std::shared_ptr<const Node> output,
                                                Rect source_bounds, RenderRequest request, RenderPriority priority,
                                                std::shared_ptr<CancellationToken> cancellation) {
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
    auto job = std::make_shared<Impl::Job>();
    job->output = std::move(output);
    job->source_bounds = source_bounds;
    job->request = request;
    job->cancellation = std::move(cancellation);
    job->group = std::move(group);
    auto result = job->result.get_future();
    impl_->enqueue(std::move(job), priority);
    return result;
}

}  // namespace rawengine
