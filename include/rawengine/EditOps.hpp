// Drop-in subset of the reference's EditGraph.hpp: the saved-graph operation
// record (EditValue, EditDomain, EditOperation, EditGraph.hpp:20-65), the
// factory that turns one operation into a node (EditGraph.cpp:1655-1733) for
// the operations of the render path, and the tile cache (EditGraph.hpp:
// 106-144).  The manifest, its JSON codec and the graph compiler around the
// factory are not part of this library.
#pragma once

#include "Operators.hpp"
#include "RawEngine.hpp"

#include <array>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <variant>
#include <vector>

namespace rawengine {

struct EditValue {
    using Array = std::vector<EditValue>;
    using Object = std::map<std::string, EditValue>;
    std::variant<std::nullptr_t, bool, std::int64_t, double, std::string, Array, Object> data = nullptr;
    bool operator==(const EditValue&) const = default;
};

enum class EditDomain {
    CameraLinear, SceneLinearProPhotoD50, SceneLinearRec2020D65, SceneLinearSrgb, ToneMappedUnmanaged,
    DisplayLinearSrgb, DisplayEncodedSrgb, DisplayEncodedIcc, UnmanagedBounded, Coverage,
    PremultipliedSceneLinearProPhotoD50, PremultipliedSceneLinearRec2020D65
};

struct EditOperation {
    std::string id;
    std::string type_id;   // e.g. rawengine.exposure
    std::uint32_t schema_version = 1;
    std::uint32_t processing_version = 1;
    bool enabled = true;
    EditDomain input_domain = EditDomain::SceneLinearProPhotoD50;
    EditDomain output_domain = EditDomain::SceneLinearProPhotoD50;
    EditValue::Object parameters;
    std::map<std::string, std::string> inputs;
    std::map<std::string, std::string> masks;
    std::string blend_mode = "normal";
    double opacity = 1.0;
    EditValue::Object extra_fields;
    bool operator==(const EditOperation&) const = default;
};

// The node of one saved operation over `input`, with the reference's
// parameter parsing, validation and exception messages.  Operation types:
//   rawengine.white_balance       red_gain, green_gain, blue_gain
//   rawengine.exposure            stops
//   rawengine.camera_to_working   matrix[9]; target from output_domain
//   rawengine.working_space_convert   target from output_domain
//   rawengine.working_to_srgb, rawengine.output_clip, rawengine.srgb_encode
//   rawengine.tone_curve          shoulder, gamma
//   rawengine.curves_extended     master/red/green/blue [[x, y]...], interpolation
//   rawengine.guided_filter_working_y   radius, epsilon
//   rawengine.sharpen             amount, radius
//   rawengine.clarity             amount, radius
//   rawengine.texture             amount, scale
//   rawengine.convolution         width, height, coefficients, border "replicate"
//   rawengine.cubic_resize        width, height
//   rawengine.rotate              angle_degrees
//   rawengine.legacy.fixed_chain  recipe {gains, exposure_stops, tone_shoulder,
//                                 tone_gamma, output_mode, [camera_to_xyz_d50,
//                                 camera_target]}; output_mode legacy_bounded or
//                                 srgb_preview
// Spatial and geometry operations take `source_bounds` as their native
// bounds.  A disabled operation returns `input`.  Any other type (the
// reference's colour-grading, mask, LUT and ICC operations) throws
// std::invalid_argument naming the type.
RAWENGINE_API std::shared_ptr<const Node> build_operation(const EditOperation& op, std::shared_ptr<const Node> input,
                                                          WorkingSpace working_space, Rect source_bounds);

// Process-local LRU cache of rendered tiles (EditGraph.hpp:106-144), held in
// DEVICE memory: a hit costs no render and, through render_device, no copy,
// so demosaiced tiles stay warm on the GPU across recipe edits.  Keys are
// (signature, bounds, mip, quality); the byte budget charges 256 bytes per
// entry plus the tile's float32 pixels (device bytes); tiles larger than the
// budget render normally without entering the cache.  Thread-safe; clear()
// drops every entry, resets the statistics and keeps renders that were in
// flight from entering.
class RAWENGINE_API TileCache final {
public:
    struct Stats {
        std::size_t entries = 0, used_bytes = 0, hits = 0, misses = 0;
    };
    explicit TileCache(std::size_t max_bytes);
    ~TileCache();
    TileCache(const TileCache&) = delete;
    TileCache& operator=(const TileCache&) = delete;
    // `node` renders `bounds` in the coordinates of `level`; distinct levels
    // never share an entry.
    Tile render(const Node& node, std::array<std::uint8_t, 32> signature, Rect bounds, RenderLevel level = {});
    // The same lookup with the tile left in device memory (no counterpart in
    // the reference): a hit returns the cached device tile itself.
    DeviceTile render_device(const Node& node, std::array<std::uint8_t, 32> signature, Rect bounds,
                             RenderLevel level = {});
    Stats stats() const;
    void clear();
private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

// A node whose renders go through a TileCache under a fixed signature (no
// counterpart in the reference, whose edit graph inserts such lookups
// itself): put it over the part of a chain that does not change between
// edits -- typically the RAW source -- and the stages above it re-render from
// the cached device tiles.  The signature must identify the input's content
// and recipe; the caller owns that contract.
class RAWENGINE_API CachedNode final : public DeviceNode {
public:
    CachedNode(std::shared_ptr<const Node> input, std::shared_ptr<TileCache> cache,
               std::array<std::uint8_t, 32> signature);
    bool supports_level(RenderLevel level) const noexcept override { return input_->supports_level(level); }
    RenderLevel input_level(RenderLevel level) const override { return level; }
    Rect input_region(Rect output, Rect) const override { return output; }
    Rect input_region_level(Rect output, Rect, RenderLevel level) const override {
        if (!supports_level(level)) throw std::invalid_argument("node has no mapping for this render level");
        return output;
    }
    const Node* input_node() const noexcept override { return input_.get(); }
    ImageDescriptor output_descriptor() const noexcept override { return input_->output_descriptor(); }
    std::optional<Rect> source_bounds() const override { return input_->source_bounds(); }
    const std::shared_ptr<TileCache>& cache() const noexcept { return cache_; }
    const std::array<std::uint8_t, 32>& signature() const noexcept { return signature_; }
private:
    std::shared_ptr<const Node> input_;
    std::shared_ptr<TileCache> cache_;
    std::array<std::uint8_t, 32> signature_;
};

// The edit domain of a node's output descriptor (EditGraph.cpp:1540-1560).
RAWENGINE_API EditDomain descriptor_domain(const ImageDescriptor& descriptor);

}  // namespace rawengine
