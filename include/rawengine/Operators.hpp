// Drop-in spatial, tone and geometry operators of RawEngine's render path
// (the reference's SpatialOps.hpp, ToneOps.hpp and GeometryOps.hpp entries
// that the tiled render reaches), executed on the B200 kernels.
#pragma once

#include "RawEngine.hpp"

namespace rawengine {

// ----------------------------------------------------------------- ToneOps

struct CurvePoint { double x = 0, y = 0; };
enum class CurveInterpolation { Linear, ShapePreservingCubic };
struct CurveKnots { std::vector<CurvePoint> knots{{0, 0}, {1, 1}}; };
struct ExtendedCurvesSettings {
    CurveKnots master;
    std::array<CurveKnots, 3> channels;
    CurveInterpolation interpolation = CurveInterpolation::Linear;
};
RAWENGINE_API void validate_extended_curves_settings(const ExtendedCurvesSettings& settings);

struct CurveTables;  // device curve set

// Master then per-channel curve (ToneOps.cpp:795-844); scene-linear working input.
class RAWENGINE_API ExtendedCurvesNode final : public PointNode {
public:
    ExtendedCurvesNode(std::shared_ptr<const Node> input, ExtendedCurvesSettings settings = {});
    bool supports_level(RenderLevel level) const noexcept override;
    Rect input_region_level(Rect output, Rect bounds, RenderLevel level) const override;
    ImageDescriptor output_descriptor() const noexcept override { return input_->output_descriptor(); }
    const CurveTables& tables() const noexcept { return *tables_; }
private:
    ExtendedCurvesSettings settings_;
    std::shared_ptr<CurveTables> tables_;
};

// -------------------------------------------------------------- SpatialOps

struct LocalStatisticsTile {
    Rect bounds;
    ImageDescriptor descriptor;
    std::uint32_t radius = 3;
    std::vector<double> mean, variance;       // interleaved RGB; population variance
    std::vector<std::uint32_t> finite_count;  // non-finite samples excluded per channel
};

RAWENGINE_API Rect local_statistics_region(Rect output, Rect image_bounds, std::uint32_t radius);
RAWENGINE_API LocalStatisticsTile local_statistics_rgb(const Tile& input, Rect output, Rect image_bounds,
                                                       std::uint32_t radius = 3);
using LocalStatisticsCallback = std::function<void(const LocalStatisticsTile&)>;
RAWENGINE_API void analyze_local_rgb(const Node& output, Rect native_bounds, const RenderRequest& request,
                                     const LocalStatisticsCallback& callback, std::uint32_t radius = 3,
                                     const CancellationToken* cancellation = nullptr);
RAWENGINE_API void analyze_local_rgb(const ImageGraph& graph, const RenderRequest& request,
                                     const LocalStatisticsCallback& callback, std::uint32_t radius = 3,
                                     const CancellationToken* cancellation = nullptr);

struct WorkingYGuidedFilterSettings {
    std::uint32_t radius = 3;   // 0..8 (the reference's contract)
    double epsilon = 0x1p-12;   // finite [2^-24, 65536]
};
RAWENGINE_API void validate_working_y_guided_filter_settings(const WorkingYGuidedFilterSettings& settings);
RAWENGINE_API Rect working_y_guided_filter_region(Rect output, Rect image_bounds, std::uint32_t radius);
RAWENGINE_API Tile working_y_guided_filter_rgb(const Tile& input, Rect output, Rect image_bounds,
                                               const WorkingYGuidedFilterSettings& settings = {});

class RAWENGINE_API WorkingYGuidedFilterNode final : public DeviceNode {
public:
    WorkingYGuidedFilterNode(std::shared_ptr<const Node> input, Rect native_bounds,
                             WorkingYGuidedFilterSettings settings = {});
    bool supports_level(RenderLevel level) const noexcept override;
    Rect input_region(Rect output, Rect source_bounds) const override;
    Rect input_region_level(Rect output, Rect source_bounds, RenderLevel level) const override;
    const Node* input_node() const noexcept override { return input_.get(); }
    ImageDescriptor output_descriptor() const noexcept override { return descriptor_; }
    const WorkingYGuidedFilterSettings& settings() const noexcept { return settings_; }
    Rect native_bounds() const noexcept { return native_bounds_; }
private:
    std::shared_ptr<const Node> input_;
    Rect native_bounds_;
    WorkingYGuidedFilterSettings settings_;
    ImageDescriptor descriptor_;
};

// Local-contrast stencils (SpatialOps.hpp:36-170): settings and validators
// with the reference's names and ranges, and nodes rendered on the device.
struct ConvolutionKernel {
    std::uint32_t width = 1, height = 1;       // odd, each 1..17
    std::vector<double> coefficients{1.0};     // row-major, finite, |c| <= 65536
};
RAWENGINE_API void validate_convolution_kernel(const ConvolutionKernel& kernel);

struct ClaritySettings {
    double amount = 0.0;          // finite [-1, 1]
    std::uint32_t radius = 3;     // 1..8, requested-level pixels
};
RAWENGINE_API void validate_clarity_settings(const ClaritySettings& settings);

struct TextureSettings {
    double amount = 0.0;          // finite [-1, 1]
    std::uint32_t scale = 2;      // 1..4 unit blur passes; support is 2 * scale pixels
};
RAWENGINE_API void validate_texture_settings(const TextureSettings& settings);

struct SharpenSettings {
    double amount = 0.0;          // finite 0..2; exact zero passes the input through
    std::uint32_t radius = 1;     // 1..3, requested-level pixels
};
RAWENGINE_API void validate_sharpen_settings(const SharpenSettings& settings);

// Base of the four stencil nodes: a scene-linear working-RGB input rendered
// over the output grown by halo_x() x halo_y() (clipped to the level's image
// bounds), then one stencil launch.  Levels: mip 0 Final or Preview, mip 1/2
// Preview, when the input supports them.
class RAWENGINE_API StencilNode : public DeviceNode {
public:
    bool supports_level(RenderLevel level) const noexcept override;
    Rect input_region(Rect output, Rect source_bounds) const override;
    Rect input_region_level(Rect output, Rect source_bounds, RenderLevel level) const override;
    const Node* input_node() const noexcept override { return input_.get(); }
    ImageDescriptor output_descriptor() const noexcept override { return input_->output_descriptor(); }
    Rect native_bounds() const noexcept { return native_bounds_; }
    virtual std::uint32_t halo_x() const noexcept = 0;
    virtual std::uint32_t halo_y() const noexcept = 0;
    std::uint32_t working_space() const noexcept { return space_; }
protected:
    StencilNode(std::shared_ptr<const Node> input, Rect native_bounds, const char* name);
    std::shared_ptr<const Node> input_;
    Rect native_bounds_;
    std::uint32_t space_ = 0;
    const char* name_;
};

class RAWENGINE_API ClarityNode final : public StencilNode {
public:
    ClarityNode(std::shared_ptr<const Node> input, Rect native_bounds, ClaritySettings settings = {});
    std::uint32_t halo_x() const noexcept override { return settings_.amount == 0 ? 0 : settings_.radius; }
    std::uint32_t halo_y() const noexcept override { return halo_x(); }
    const ClaritySettings& settings() const noexcept { return settings_; }
private:
    ClaritySettings settings_;
};

class RAWENGINE_API TextureNode final : public StencilNode {
public:
    TextureNode(std::shared_ptr<const Node> input, Rect native_bounds, TextureSettings settings = {});
    std::uint32_t halo_x() const noexcept override { return settings_.amount == 0 ? 0 : 2 * settings_.scale; }
    std::uint32_t halo_y() const noexcept override { return halo_x(); }
    const TextureSettings& settings() const noexcept { return settings_; }
private:
    TextureSettings settings_;
};

class RAWENGINE_API SharpenNode final : public StencilNode {
public:
    SharpenNode(std::shared_ptr<const Node> input, Rect native_bounds, SharpenSettings settings = {});
    std::uint32_t halo_x() const noexcept override { return settings_.amount == 0 ? 0 : settings_.radius; }
    std::uint32_t halo_y() const noexcept override { return halo_x(); }
    const SharpenSettings& settings() const noexcept { return settings_; }
private:
    SharpenSettings settings_;
};

// Flipped on both axes (a convolution), binary64 accumulation, replicate
// boundary, no normalisation or clipping.
class RAWENGINE_API ConvolutionNode final : public StencilNode {
public:
    ConvolutionNode(std::shared_ptr<const Node> input, Rect native_bounds, ConvolutionKernel kernel);
    std::uint32_t halo_x() const noexcept override { return identity_ ? 0 : kernel_.width / 2; }
    std::uint32_t halo_y() const noexcept override { return identity_ ? 0 : kernel_.height / 2; }
    const ConvolutionKernel& kernel() const noexcept { return kernel_; }
private:
    ConvolutionKernel kernel_;
    bool identity_ = false;
};

// ------------------------------------------------------------- GeometryOps

struct RAWENGINE_API RotateSettings {
    double angle_degrees = 0;
};
RAWENGINE_API void validate_rotate_settings(const RotateSettings& settings);

class RAWENGINE_API RotateNode final : public DeviceNode {
public:
    RotateNode(std::shared_ptr<const Node> input, Rect input_bounds, RotateSettings settings = {});
    bool supports_level(RenderLevel level) const noexcept override;
    RenderLevel input_level(RenderLevel level) const override;
    Rect input_region(Rect output, Rect input_bounds) const override;
    Rect input_region_level(Rect output, Rect input_bounds, RenderLevel level) const override;
    const Node* input_node() const noexcept override { return input_.get(); }
    ImageDescriptor output_descriptor() const noexcept override { return descriptor_; }
    Rect output_bounds() const noexcept { return {0, 0, input_bounds_.width, input_bounds_.height}; }
    Rect native_output_region(Rect output, RenderLevel level) const;
    Rect support(Rect native_output) const;
    Rect input_bounds() const noexcept { return input_bounds_; }
    double angle() const noexcept { return settings_.angle_degrees; }
private:
    std::shared_ptr<const Node> input_;
    Rect input_bounds_;
    RotateSettings settings_;
    ImageDescriptor descriptor_;
    double cx_, cy_, cosine_, sine_;
};

struct RAWENGINE_API CubicResizeSettings {
    std::uint32_t width = 0, height = 0;
};
RAWENGINE_API void validate_cubic_resize_settings(const CubicResizeSettings& settings, Rect native_input_bounds);

class RAWENGINE_API CubicResizeNode final : public DeviceNode {
public:
    CubicResizeNode(std::shared_ptr<const Node> input, Rect input_bounds, CubicResizeSettings settings);
    bool supports_level(RenderLevel level) const noexcept override;
    RenderLevel input_level(RenderLevel level) const override;
    Rect input_region(Rect output, Rect input_bounds) const override;
    Rect input_region_level(Rect output, Rect input_bounds, RenderLevel level) const override;
    const Node* input_node() const noexcept override { return input_.get(); }
    ImageDescriptor output_descriptor() const noexcept override { return descriptor_; }
    Rect output_bounds() const noexcept { return {0, 0, settings_.width, settings_.height}; }
    Rect native_output_region(Rect output, RenderLevel level) const;
    Rect support(Rect native_output) const;
    Rect input_bounds() const noexcept { return input_bounds_; }
    const CubicResizeSettings& settings() const noexcept { return settings_; }
private:
    std::shared_ptr<const Node> input_;
    Rect input_bounds_;
    CubicResizeSettings settings_;
    ImageDescriptor descriptor_;
};

// ----------------------------------------------------------- TileScheduler

enum class RenderPriority { Background = 0, Normal = 1, Interactive = 2 };

// A render result left in device memory (no counterpart in the reference,
// whose results are host tiles): bounds.height rows of bounds.width * 3
// interleaved float32 RGB values, contiguous, on the device that was current
// when the scheduler was created.  The memory stays valid while any copy of
// the DeviceTile (or of its rgb pointer) lives.
struct DeviceTile {
    Rect bounds;
    std::shared_ptr<const float> rgb;
    ImageDescriptor descriptor = ImageDescriptor::camera_linear();
    RAWENGINE_API Tile to_host() const;   // copies the pixels into a host Tile
};

// Queued requests are taken in priority order, FIFO within a priority, and
// rendered in waves: a dispatch lane takes every pending request it can hold
// at once, renders the requests whose chains are a RAW source under point
// nodes as ONE batched device render (a persistent kernel over all of their
// tiles), renders any other request through its node, and resolves the
// futures.  `workers` is the number of lanes (1..64); each lane has its own
// CUDA stream, so waves of different lanes overlap.  Throws length_error when
// the pending budget is full; cancellation is checked before a wave is
// rendered and again before its result is delivered.
class RAWENGINE_API TileScheduler final {
public:
    TileScheduler(std::size_t workers, std::size_t max_pending);
    ~TileScheduler();
    TileScheduler(const TileScheduler&) = delete;
    TileScheduler& operator=(const TileScheduler&) = delete;
    std::future<Tile> submit(std::shared_ptr<const Node> output, Rect source_bounds, RenderRequest request,
                             RenderPriority priority = RenderPriority::Normal,
                             std::shared_ptr<CancellationToken> cancellation = nullptr);
    std::future<Tile> submit(std::shared_ptr<const Node> output, Rect source_bounds, Rect viewport,
                             RenderPriority priority = RenderPriority::Normal, std::uint32_t tile_size = 256,
                             std::shared_ptr<CancellationToken> cancellation = nullptr);
    std::future<Tile> submit_latest(std::string group, std::shared_ptr<const Node> output, Rect source_bounds,
                                    RenderRequest request, RenderPriority priority = RenderPriority::Interactive,
                                    std::shared_ptr<CancellationToken> cancellation = nullptr);
    std::future<Tile> submit_latest(std::string group, std::shared_ptr<const Node> output, Rect source_bounds,
                                    Rect viewport, RenderPriority priority = RenderPriority::Interactive,
                                    std::uint32_t tile_size = 256,
                                    std::shared_ptr<CancellationToken> cancellation = nullptr);
    // The same request with the result left in device memory (no
    // counterpart in the reference): no device-to-host copy is made.
    std::future<DeviceTile> submit_device(std::shared_ptr<const Node> output, Rect source_bounds,
                                          RenderRequest request, RenderPriority priority = RenderPriority::Normal,
                                          std::shared_ptr<CancellationToken> cancellation = nullptr);
    std::future<DeviceTile> submit_latest_device(std::string group, std::shared_ptr<const Node> output,
                                                 Rect source_bounds, RenderRequest request,
                                                 RenderPriority priority = RenderPriority::Interactive,
                                                 std::shared_ptr<CancellationToken> cancellation = nullptr);
    struct Stats {
        std::uint64_t waves = 0;            // waves rendered
        std::uint64_t batched_requests = 0; // requests rendered inside a batched device render
        std::uint64_t node_requests = 0;    // requests rendered through their node
        std::uint64_t unbatchable_requests = 0;  // node requests whose chain is not a RAW point chain
        std::uint64_t batch_fallbacks = 0;  // waves whose batched render failed and were re-rendered per request
        std::string last_fallback;          // the error text of the last such failure
        // host seconds spent by the lanes: lowering chains to batch items,
        // planning the batches, waiting for the batched renders, delivering tiles
        double lower_s = 0, plan_s = 0, device_s = 0, deliver_s = 0;
    };
    Stats stats() const;
private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

}  // namespace rawengine
