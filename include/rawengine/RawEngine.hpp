// Drop-in C++ surface of RawEngine's render path, executed on a B200.
//
// The names, signatures, argument meaning and exception behaviour follow the
// reference's public header (RawEngine.hpp, GeometryOps.hpp, SpatialOps.hpp,
// ToneOps.hpp and TileScheduler.hpp of tylermcm/librawops) for the nodes on
// the tiled-render hot path, so that code written against those headers
// compiles and behaves the same.  Rendering is done by the sm_100a kernels
// behind include/rawengine_b200.h: a chain of point nodes over a RAW source is
// one fused launch per render; spatial and geometry nodes render their input
// footprint into device memory and run their own kernels.  Nodes outside this
// library (user subclasses of Node) are pulled through their own render_level
// and uploaded.
#pragma once

#include <array>
#include <atomic>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <future>
#include <memory>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#if defined(__GNUC__)
#define RAWENGINE_API __attribute__((visibility("default")))
#else
#define RAWENGINE_API
#endif

namespace rawengine {

enum class BayerPattern { RGGB, BGGR, GRBG, GBRG };
enum class WorkingSpace { LinearProPhotoD50, LinearRec2020D65 };

struct Rect {
    std::uint32_t x = 0, y = 0, width = 0, height = 0;
};

enum class RenderQuality : std::uint8_t { Preview = 0, Final = 1 };

// Mip 1/2 request coordinates are zero-based within the reduced extent.
struct RenderLevel {
    std::uint32_t mip = 0;
    RenderQuality quality = RenderQuality::Final;
};

struct RenderRequest {
    Rect viewport;
    std::uint32_t tile_size = 256;
    RenderLevel level;
    RenderRequest() = default;
    explicit constexpr RenderRequest(Rect requested_viewport, std::uint32_t requested_tile_size = 256,
                                     RenderLevel requested_level = {}) noexcept
        : viewport(requested_viewport), tile_size(requested_tile_size), level(requested_level) {}
};

struct RawMetadata {
    std::uint32_t width = 0, height = 0;
    std::uint32_t row_stride_samples = 0;  // 0 = tightly packed
    BayerPattern pattern = BayerPattern::RGGB;
    std::uint8_t cfa_phase_x = 0, cfa_phase_y = 0;
    Rect active_area;                       // all zero = full sensor
    std::array<std::uint16_t, 4> black_levels{0, 0, 0, 0};
    std::array<std::uint16_t, 4> white_levels{65535, 65535, 65535, 65535};
};

struct DeviceRaw;  // device copy of a RawImage (created lazily, shared by copies)

// Decoded uint16 Bayer samples; validated and normalized on construction.
// Copies share the immutable samples and their device copy.
class RAWENGINE_API RawImage {
public:
    RawImage(RawMetadata metadata, std::vector<std::uint16_t> samples);
    RawImage(std::uint32_t width, std::uint32_t height, std::vector<std::uint16_t> samples,
             BayerPattern pattern = BayerPattern::RGGB, std::uint16_t black_level = 0,
             std::uint16_t white_level = 65535);
    const RawMetadata& metadata() const noexcept { return metadata_; }
    const std::vector<std::uint16_t>& samples() const noexcept { return *bayer_; }
    std::uint32_t width() const noexcept { return metadata_.width; }
    std::uint32_t height() const noexcept { return metadata_.height; }
    const DeviceRaw& device() const;  // uploads on first use (thread-safe)
private:
    RawMetadata metadata_;
    std::shared_ptr<const std::vector<std::uint16_t>> bayer_;
    std::shared_ptr<DeviceRaw> device_;
};

struct RasterMetadata {
    std::uint32_t width = 0, height = 0;
    std::uint32_t row_stride_pixels = 0;
    WorkingSpace working_space = WorkingSpace::LinearProPhotoD50;
};

struct DeviceRaster;

class RAWENGINE_API RasterImage {
public:
    RasterImage(RasterMetadata metadata, std::vector<float> pixels);
    const RasterMetadata& metadata() const noexcept { return metadata_; }
    const std::vector<float>& pixels() const noexcept { return *pixels_; }
    std::uint32_t width() const noexcept { return metadata_.width; }
    std::uint32_t height() const noexcept { return metadata_.height; }
    const DeviceRaster& device() const;
private:
    RasterMetadata metadata_;
    std::shared_ptr<const std::vector<float>> pixels_;
    std::shared_ptr<DeviceRaster> device_;
};

struct CameraColorTransform {
    std::array<double, 9> camera_to_xyz_d50{};
    WorkingSpace target = WorkingSpace::LinearProPhotoD50;
};

enum class OutputMode { LegacyBounded, SrgbPreview, IccDisplay };

struct GraphRecipe {
    float red_gain = 1.0f, green_gain = 1.0f, blue_gain = 1.0f;
    float exposure_stops = 0.0f;
    float tone_shoulder = 0.25f;
    float tone_gamma = 1.0f;
    std::optional<CameraColorTransform> camera_color;
    OutputMode output_mode = OutputMode::LegacyBounded;
};

enum class PixelFormat { RGBFloat32 };
enum class PixelDomain { CameraLinearRGB, SceneLinearRGB, ToneMappedUnmanagedRGB, BoundedUnmanagedRGB,
                         DisplayLinearRGB, DisplayEncodedRGB };
enum class ColorPrimaries { CameraNative, ProPhoto, Rec2020, SRGB, ICCProfile };
enum class WhitePoint { Unspecified, D50, D65 };
enum class TransferFunction { Linear, CustomTone, SRGB, ICCProfile };
enum class ReferenceState { CameraReferred, SceneReferred, DisplayReferred, Unspecified };
enum class AlphaMode { None };

struct ImageDescriptor {
    PixelFormat format = PixelFormat::RGBFloat32;
    PixelDomain domain = PixelDomain::CameraLinearRGB;
    ColorPrimaries primaries = ColorPrimaries::CameraNative;
    WhitePoint white_point = WhitePoint::Unspecified;
    TransferFunction transfer = TransferFunction::Linear;
    ReferenceState reference = ReferenceState::CameraReferred;
    AlphaMode alpha = AlphaMode::None;
    std::array<std::uint8_t, 32> profile_sha256{};

    static constexpr ImageDescriptor camera_linear() noexcept { return {}; }
    static constexpr ImageDescriptor scene_linear(WorkingSpace s) noexcept {
        return {PixelFormat::RGBFloat32, PixelDomain::SceneLinearRGB,
                s == WorkingSpace::LinearProPhotoD50 ? ColorPrimaries::ProPhoto : ColorPrimaries::Rec2020,
                s == WorkingSpace::LinearProPhotoD50 ? WhitePoint::D50 : WhitePoint::D65,
                TransferFunction::Linear, ReferenceState::SceneReferred, AlphaMode::None, {}};
    }
    static constexpr ImageDescriptor linear_srgb() noexcept {
        return {PixelFormat::RGBFloat32, PixelDomain::SceneLinearRGB, ColorPrimaries::SRGB, WhitePoint::D65,
                TransferFunction::Linear, ReferenceState::SceneReferred, AlphaMode::None, {}};
    }
    static constexpr ImageDescriptor tone_mapped() noexcept {
        return {PixelFormat::RGBFloat32, PixelDomain::ToneMappedUnmanagedRGB, ColorPrimaries::CameraNative,
                WhitePoint::Unspecified, TransferFunction::CustomTone, ReferenceState::Unspecified,
                AlphaMode::None, {}};
    }
    static constexpr ImageDescriptor bounded_output() noexcept {
        return {PixelFormat::RGBFloat32, PixelDomain::BoundedUnmanagedRGB, ColorPrimaries::CameraNative,
                WhitePoint::Unspecified, TransferFunction::CustomTone, ReferenceState::Unspecified,
                AlphaMode::None, {}};
    }
    static constexpr ImageDescriptor srgb_output() noexcept {
        return {PixelFormat::RGBFloat32, PixelDomain::DisplayEncodedRGB, ColorPrimaries::SRGB, WhitePoint::D65,
                TransferFunction::SRGB, ReferenceState::DisplayReferred, AlphaMode::None, {}};
    }
    static constexpr ImageDescriptor display_linear_srgb() noexcept {
        return {PixelFormat::RGBFloat32, PixelDomain::DisplayLinearRGB, ColorPrimaries::SRGB, WhitePoint::D65,
                TransferFunction::Linear, ReferenceState::DisplayReferred, AlphaMode::None, {}};
    }
    bool operator==(const ImageDescriptor&) const = default;
};

struct Tile {
    Rect bounds;
    std::vector<float> rgb;  // interleaved float32 RGB, row-major
    ImageDescriptor descriptor = ImageDescriptor::camera_linear();
};

// The ICC profile and conversion policy an encoded-raster source node reports
// (RawEngine.hpp:212-219 of the reference).  No node of this library has one;
// the type exists so that nodes written against the reference's Node
// interface compile unchanged.
struct IccProfileIdentity {
    std::array<std::uint8_t, 32> profile_sha256{};
    std::string intent = "relative_colorimetric";
    bool black_point_compensation = false;
    std::string engine = "lcms2-core";
    std::string engine_version = "2.19.1";
    bool operator==(const IccProfileIdentity&) const = default;
};

struct RawDemosaicIdentity {
    std::string algorithm = "rawengine.bilinear";
    std::uint32_t processing_version = 1;
    bool operator==(const RawDemosaicIdentity&) const = default;
};
RAWENGINE_API void validate_raw_demosaic(const RawDemosaicIdentity& identity);

class RAWENGINE_API Node {
public:
    virtual ~Node() = default;
    virtual Tile render(Rect bounds) const = 0;
    virtual Tile render_level(Rect bounds, RenderLevel level) const {
        if (level.mip == 0 && level.quality == RenderQuality::Final) return render(bounds);
        throw std::invalid_argument("node does not support this render level");
    }
    virtual bool supports_level(RenderLevel level) const noexcept {
        return level.mip == 0 && level.quality == RenderQuality::Final;
    }
    virtual ImageDescriptor output_descriptor() const noexcept = 0;
    virtual const Node* input_node() const noexcept { return nullptr; }
    virtual RenderLevel input_level(RenderLevel output_level) const { return output_level; }
    virtual Rect input_region(Rect output, Rect source_bounds) const {
        (void)source_bounds;
        return output;
    }
    virtual Rect input_region_level(Rect output, Rect source_bounds, RenderLevel level) const {
        if (level.mip == 0 && level.quality == RenderQuality::Final) return input_region(output, source_bounds);
        throw std::invalid_argument("node has no mapping for this render level");
    }
    // Identity hooks of the reference's Node (RawEngine.hpp:263-268).  The
    // device executor does not consult them; they return no identity unless a
    // subclass overrides them.
    virtual std::optional<IccProfileIdentity> input_icc_identity() const { return std::nullopt; }
    virtual std::optional<std::array<std::uint8_t, 32>> source_fingerprint() const { return std::nullopt; }
    virtual std::optional<Rect> source_bounds() const { return std::nullopt; }
    virtual std::optional<RawDemosaicIdentity> raw_demosaic_identity() const { return std::nullopt; }
};

// Base of the nodes this library renders on the GPU (render/render_level go
// through the device executor; see Renderer).
class RAWENGINE_API DeviceNode : public Node {
public:
    Tile render(Rect bounds) const override;
    Tile render_level(Rect bounds, RenderLevel level) const override;
};

class RAWENGINE_API RawUnpackNode final : public DeviceNode {
public:
    explicit RawUnpackNode(RawImage image);
    RawUnpackNode(RawImage image, RawDemosaicIdentity demosaic);
    Rect input_region(Rect output, Rect source_bounds) const override;
    ImageDescriptor output_descriptor() const noexcept override { return ImageDescriptor::camera_linear(); }
    std::optional<Rect> source_bounds() const override { return image_.metadata().active_area; }
    std::optional<RawDemosaicIdentity> raw_demosaic_identity() const override { return demosaic_; }
    const RawImage& image() const noexcept { return image_; }
    bool menon() const noexcept;
private:
    RawImage image_;
    RawDemosaicIdentity demosaic_;
};

class RAWENGINE_API RasterSourceNode final : public DeviceNode {
public:
    explicit RasterSourceNode(RasterImage image);
    bool supports_level(RenderLevel level) const noexcept override;
    Rect input_region_level(Rect output, Rect, RenderLevel level) const override;
    ImageDescriptor output_descriptor() const noexcept override {
        return ImageDescriptor::scene_linear(image_.metadata().working_space);
    }
    std::optional<Rect> source_bounds() const override { return Rect{0, 0, image_.width(), image_.height()}; }
    const RasterImage& image() const noexcept { return image_; }
private:
    RasterImage image_;
};

// Point nodes: one fused stage each.
class RAWENGINE_API PointNode : public DeviceNode {
public:
    const Node* input_node() const noexcept override { return input_.get(); }
    const std::shared_ptr<const Node>& input() const noexcept { return input_; }
protected:
    explicit PointNode(std::shared_ptr<const Node> input) : input_(std::move(input)) {}
    std::shared_ptr<const Node> input_;
};

class RAWENGINE_API WhiteBalanceNode final : public PointNode {
public:
    WhiteBalanceNode(std::shared_ptr<const Node> input, float red, float green, float blue);
    ImageDescriptor output_descriptor() const noexcept override { return ImageDescriptor::camera_linear(); }
    const float* gains() const noexcept { return gains_; }
private:
    float gains_[3];
};

class RAWENGINE_API ExposureNode final : public PointNode {
public:
    ExposureNode(std::shared_ptr<const Node> input, float stops);
    bool supports_level(RenderLevel level) const noexcept override;
    Rect input_region_level(Rect output, Rect, RenderLevel level) const override;
    ImageDescriptor output_descriptor() const noexcept override { return descriptor_; }
    float multiplier() const noexcept { return multiplier_; }
private:
    float multiplier_;
    ImageDescriptor descriptor_;
};

class RAWENGINE_API CameraToWorkingNode final : public PointNode {
public:
    CameraToWorkingNode(std::shared_ptr<const Node> input, CameraColorTransform transform,
                        Rect native_input_bounds = {});
    bool supports_level(RenderLevel level) const noexcept override;
    RenderLevel input_level(RenderLevel level) const override;
    Rect input_region_level(Rect output, Rect input_bounds, RenderLevel level) const override;
    ImageDescriptor output_descriptor() const noexcept override { return descriptor_; }
    const std::array<float, 9>& matrix() const noexcept { return matrix_; }
    Rect native_bounds() const noexcept { return native_input_bounds_; }
private:
    std::array<float, 9> matrix_{};
    ImageDescriptor descriptor_;
    Rect native_input_bounds_;
};

class RAWENGINE_API WorkingSpaceConvertNode final : public PointNode {
public:
    WorkingSpaceConvertNode(std::shared_ptr<const Node> input, WorkingSpace target);
    bool supports_level(RenderLevel level) const noexcept override;
    Rect input_region_level(Rect output, Rect, RenderLevel level) const override;
    ImageDescriptor output_descriptor() const noexcept override { return descriptor_; }
    const std::array<float, 9>& matrix() const noexcept { return matrix_; }
    bool identity() const noexcept { return identity_; }
private:
    std::array<float, 9> matrix_{};
    ImageDescriptor descriptor_;
    bool identity_ = false;
};

class RAWENGINE_API WorkingToSrgbNode final : public PointNode {
public:
    explicit WorkingToSrgbNode(std::shared_ptr<const Node> input);
    bool supports_level(RenderLevel level) const noexcept override;
    Rect input_region_level(Rect output, Rect, RenderLevel level) const override;
    ImageDescriptor output_descriptor() const noexcept override { return ImageDescriptor::linear_srgb(); }
    const std::array<float, 9>& matrix() const noexcept { return matrix_; }
private:
    std::array<float, 9> matrix_{};
};

class RAWENGINE_API ToneCurveNode final : public PointNode {
public:
    ToneCurveNode(std::shared_ptr<const Node> input, float shoulder, float gamma);
    bool supports_level(RenderLevel level) const noexcept override;
    Rect input_region_level(Rect output, Rect, RenderLevel level) const override;
    ImageDescriptor output_descriptor() const noexcept override { return descriptor_; }
    float shoulder() const noexcept { return shoulder_; }
    float inverse_gamma() const noexcept { return inverse_gamma_; }
private:
    float shoulder_, inverse_gamma_;
    ImageDescriptor descriptor_;
};

class RAWENGINE_API OutputClipNode final : public PointNode {
public:
    explicit OutputClipNode(std::shared_ptr<const Node> input);
    ImageDescriptor output_descriptor() const noexcept override { return descriptor_; }
private:
    ImageDescriptor descriptor_;
};

class RAWENGINE_API SrgbEncodeNode final : public PointNode {
public:
    explicit SrgbEncodeNode(std::shared_ptr<const Node> input);
    bool supports_level(RenderLevel level) const noexcept override;
    Rect input_region_level(Rect output, Rect, RenderLevel level) const override;
    ImageDescriptor output_descriptor() const noexcept override { return ImageDescriptor::srgb_output(); }
};

class ImageGraph;
class ExecutableEditGraph;

class RAWENGINE_API ImageGraph final {
public:
    ImageGraph(RawImage image, GraphRecipe recipe = {});
    ImageGraph(RasterImage image, GraphRecipe recipe = {});
    ImageGraph(std::shared_ptr<const Node> scene_linear_source, Rect source_bounds, GraphRecipe recipe = {});
    const RawImage& image() const;
    Rect source_bounds() const noexcept { return source_bounds_; }
    const GraphRecipe& recipe() const noexcept { return recipe_; }
    const Node& output() const noexcept { return *output_; }
    std::shared_ptr<const Node> output_node() const noexcept { return output_; }
private:
    std::optional<RawImage> raw_image_;
    Rect source_bounds_;
    GraphRecipe recipe_;
    std::shared_ptr<const Node> output_;
};

class RAWENGINE_API RenderCancelled final : public std::runtime_error {
public:
    RenderCancelled() : std::runtime_error("render cancelled") {}
};

class RAWENGINE_API CancellationToken final {
public:
    void cancel() noexcept { cancelled_.store(true, std::memory_order_relaxed); }
    bool is_cancelled() const noexcept { return cancelled_.load(std::memory_order_relaxed); }
private:
    std::atomic<bool> cancelled_{false};
};

class RAWENGINE_API Renderer final {
public:
    using TileCallback = std::function<void(const Tile&)>;
    void render_tiles(const ImageGraph& graph, RenderRequest request, const TileCallback& callback,
                      const CancellationToken* cancellation = nullptr) const;
    void render_tiles(const Node& output, Rect source_bounds, RenderRequest request, const TileCallback& callback,
                      const CancellationToken* cancellation = nullptr) const;
    void render_tiles(const ImageGraph& graph, Rect viewport, const TileCallback& callback,
                      std::uint32_t tile_size = 256, const CancellationToken* cancellation = nullptr) const;
    void render_tiles(const Node& output, Rect source_bounds, Rect viewport, const TileCallback& callback,
                      std::uint32_t tile_size = 256, const CancellationToken* cancellation = nullptr) const;
    Tile render_image(const ImageGraph& graph, RenderRequest request,
                      const CancellationToken* cancellation = nullptr) const;
    Tile render_image(const Node& output, Rect source_bounds, RenderRequest request,
                      const CancellationToken* cancellation = nullptr) const;
    Tile render_image(const ImageGraph& graph, Rect viewport, std::uint32_t tile_size = 256,
                      const CancellationToken* cancellation = nullptr) const;
    Tile render_image(const Node& output, Rect source_bounds, Rect viewport, std::uint32_t tile_size = 256,
                      const CancellationToken* cancellation = nullptr) const;
    std::vector<float> render_roi(const ImageGraph& graph, Rect viewport, std::uint32_t tile_size = 256,
                                  const CancellationToken* cancellation = nullptr) const;
};

}  // namespace rawengine
