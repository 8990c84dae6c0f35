// Drop-in subset of the reference's EditGraph.hpp: the saved-graph operation
// record (EditValue, EditDomain, EditOperation, EditGraph.hpp:20-65) and the
// factory that turns one operation into a node (EditGraph.cpp:1655-1733) for
// the operations of the render path.  The manifest, its JSON codec and the
// graph compiler around the factory are not part of this library.
#pragma once

#include "Operators.hpp"
#include "RawEngine.hpp"

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

// The edit domain of a node's output descriptor (EditGraph.cpp:1540-1560).
RAWENGINE_API EditDomain descriptor_domain(const ImageDescriptor& descriptor);

}  // namespace rawengine
