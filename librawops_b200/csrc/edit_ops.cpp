// Saved-graph operation factory (include/rawengine/EditOps.hpp): one saved
// operation record -> the device node that renders it.
//
// Parameter parsing follows the reference's EditGraph.cpp field by field
// (which keys are required, which numeric forms are accepted, the range
// checks and their exception messages), since a saved graph that the
// reference accepts or rejects must be accepted or rejected here too; the
// nodes it builds are this library's device nodes.
#include "rawengine/EditOps.hpp"

#include <cmath>
#include <limits>
#include <stdexcept>

namespace rawengine {

namespace {

// EditGraph.cpp:431-466
EditValue::Object object(const EditValue& v) {
    if (auto* r = std::get_if<EditValue::Object>(&v.data)) return *r;
    throw std::invalid_argument("edit JSON object expected");
}
EditValue::Array array(const EditValue& v) {
    if (auto* r = std::get_if<EditValue::Array>(&v.data)) return *r;
    throw std::invalid_argument("edit JSON array expected");
}
std::string string(const EditValue& v) {
    if (auto* r = std::get_if<std::string>(&v.data)) return *r;
    throw std::invalid_argument("edit string expected");
}
double number(const EditValue& v) {
    if (auto* r = std::get_if<double>(&v.data)) return *r;
    if (auto* r = std::get_if<std::int64_t>(&v.data)) return (double)*r;
    throw std::invalid_argument("edit number expected");
}
std::uint32_t positive_u32(const EditValue& v) {
    const auto* i = std::get_if<std::int64_t>(&v.data);
    if (!i || *i <= 0 || *i > (std::int64_t)std::numeric_limits<std::uint32_t>::max())
        throw std::invalid_argument("positive edit version expected");
    return (std::uint32_t)*i;
}
EditValue take(EditValue::Object& o, const char* key) {
    auto found = o.find(key);
    if (found == o.end()) throw std::invalid_argument(std::string("missing edit field: ") + key);
    EditValue v = std::move(found->second);
    o.erase(found);
    return v;
}

// EditGraph.cpp:1576-1611
WorkingSpace working_from_domain(EditDomain d) {
    if (d == EditDomain::SceneLinearProPhotoD50) return WorkingSpace::LinearProPhotoD50;
    if (d == EditDomain::SceneLinearRec2020D65) return WorkingSpace::LinearRec2020D65;
    throw std::invalid_argument("operation target is not a supported working space");
}
float scalar(const EditValue::Object& p, const char* key) {
    const auto found = p.find(key);
    if (found == p.end()) throw std::invalid_argument("missing operation scalar");
    const double v = number(found->second);
    if (!std::isfinite(v) || std::abs(v) > std::numeric_limits<float>::max())
        throw std::invalid_argument("operation scalar exceeds float32 range");
    return (float)v;
}
CameraColorTransform camera_transform(const EditValue::Object& p, WorkingSpace target, const char* key) {
    const auto found = p.find(key);
    if (found == p.end()) throw std::invalid_argument("missing camera color matrix");
    const auto values = array(found->second);
    if (values.size() != 9) throw std::invalid_argument("camera matrix needs nine values");
    CameraColorTransform t;
    t.target = target;
    for (size_t i = 0; i < 9; ++i) t.camera_to_xyz_d50[i] = number(values[i]);
    return t;
}
const char* working_name(WorkingSpace s) {
    return s == WorkingSpace::LinearProPhotoD50 ? "linear_prophoto_d50" : "linear_rec2020_d65";
}

// EditGraph.cpp:683-743, 860-878
ConvolutionKernel convolution_kernel(const EditValue::Object& p) {
    if (p.size() != 4 || !p.contains("width") || !p.contains("height") || !p.contains("coefficients") ||
        !p.contains("border") || string(p.at("border")) != "replicate")
        throw std::invalid_argument("convolution needs width, height, coefficients and replicate border");
    ConvolutionKernel k{positive_u32(p.at("width")), positive_u32(p.at("height")), {}};
    const auto values = array(p.at("coefficients"));
    if (values.size() > 289) throw std::invalid_argument("convolution kernel exceeds 289 coefficients");
    for (const auto& v : values) k.coefficients.push_back(number(v));
    validate_convolution_kernel(k);
    return k;
}
SharpenSettings sharpen_settings(const EditValue::Object& p) {
    if (p.size() != 2 || !p.contains("amount") || !p.contains("radius"))
        throw std::invalid_argument("sharpen needs amount and radius only");
    SharpenSettings s{number(p.at("amount")), positive_u32(p.at("radius"))};
    validate_sharpen_settings(s);
    return s;
}
ClaritySettings clarity_settings(const EditValue::Object& p) {
    if (p.size() != 2 || !p.contains("amount") || !p.contains("radius"))
        throw std::invalid_argument("clarity needs amount and radius only");
    ClaritySettings s{number(p.at("amount")), positive_u32(p.at("radius"))};
    validate_clarity_settings(s);
    return s;
}
TextureSettings texture_settings(const EditValue::Object& p) {
    if (p.size() != 2 || !p.contains("amount") || !p.contains("scale"))
        throw std::invalid_argument("texture needs amount and scale only");
    TextureSettings s{number(p.at("amount")), positive_u32(p.at("scale"))};
    validate_texture_settings(s);
    return s;
}
WorkingYGuidedFilterSettings guided_filter_settings(const EditValue::Object& p) {
    if (p.size() != 2 || !p.contains("radius") || !p.contains("epsilon"))
        throw std::invalid_argument("guided filter needs radius and epsilon only");
    const double r = number(p.at("radius"));
    if (!std::isfinite(r) || r < 0 || r > 8 || std::floor(r) != r)
        throw std::invalid_argument("guided filter radius must be integral 0..8");
    WorkingYGuidedFilterSettings s{(std::uint32_t)r, number(p.at("epsilon"))};
    validate_working_y_guided_filter_settings(s);
    return s;
}
CubicResizeSettings cubic_resize_settings(const EditValue::Object& p) {
    if (p.size() != 2 || !p.contains("width") || !p.contains("height"))
        throw std::invalid_argument("cubic resize requires width and height only");
    return {positive_u32(p.at("width")), positive_u32(p.at("height"))};
}
ExtendedCurvesSettings extended_curves_settings(const EditValue::Object& p) {
    if (p.size() != 5 || !p.contains("master") || !p.contains("red") || !p.contains("green") ||
        !p.contains("blue") || !p.contains("interpolation"))
        throw std::invalid_argument(
            "extended curves need master/red/green/blue knots and interpolation only");
    ExtendedCurvesSettings s;
    unsigned c = 0;
    for (const char* name : {"master", "red", "green", "blue"}) {
        const auto points = array(p.at(name));
        if (points.size() < 2 || points.size() > 256) throw std::invalid_argument("extended curve needs 2..256 knots");
        auto& knots = c == 0 ? s.master.knots : s.channels[c - 1].knots;
        ++c;
        knots.clear();
        for (const auto& point : points) {
            const auto pair = array(point);
            if (pair.size() != 2) throw std::invalid_argument("extended curve knot needs x and y");
            knots.push_back({number(pair[0]), number(pair[1])});
        }
    }
    const auto token = string(p.at("interpolation"));
    if (token == "linear")
        s.interpolation = CurveInterpolation::Linear;
    else if (token == "shape_preserving_cubic")
        s.interpolation = CurveInterpolation::ShapePreservingCubic;
    else
        throw std::invalid_argument("unsupported extended curve interpolation");
    validate_extended_curves_settings(s);
    return s;
}

// EditGraph.cpp:1613-1653
std::shared_ptr<const Node> build_legacy_chain(const EditOperation& op, std::shared_ptr<const Node> source,
                                               WorkingSpace working_space) {
    const auto found = op.parameters.find("recipe");
    if (found == op.parameters.end()) throw std::invalid_argument("missing edit field: recipe");
    auto fields = object(found->second);
    const float red = scalar(fields, "red_gain"), green = scalar(fields, "green_gain");
    const float blue = scalar(fields, "blue_gain"), exposure = scalar(fields, "exposure_stops");
    const float shoulder = scalar(fields, "tone_shoulder"), gamma = scalar(fields, "tone_gamma");
    const std::string mode = string(take(fields, "output_mode"));
    std::shared_ptr<const Node> linear = source;
    if (descriptor_domain(source->output_descriptor()) == EditDomain::CameraLinear) {
        linear = std::make_shared<WhiteBalanceNode>(linear, red, green, blue);
        linear = std::make_shared<ExposureNode>(linear, exposure);
        if (fields.contains("camera_to_xyz_d50")) {
            if (string(take(fields, "camera_target")) != working_name(working_space))
                throw std::invalid_argument("legacy camera target disagrees with working space");
            linear = std::make_shared<CameraToWorkingNode>(
                linear, camera_transform(fields, working_space, "camera_to_xyz_d50"));
            fields.erase("camera_to_xyz_d50");
        }
    } else {
        if (red != 1.0f || green != 1.0f || blue != 1.0f || fields.contains("camera_to_xyz_d50") ||
            fields.contains("camera_target"))
            throw std::invalid_argument("legacy raster recipe contains RAW controls");
        linear = std::make_shared<ExposureNode>(linear, exposure);
    }
    if (mode == "icc_display") throw std::invalid_argument("ICC display output is not available in this library");
    if (mode == "srgb_preview")
        linear = std::make_shared<WorkingToSrgbNode>(linear);
    else if (mode != "legacy_bounded")
        throw std::invalid_argument("unknown legacy output mode");
    if (fields.size() != 6) throw std::invalid_argument("legacy recipe contains unrecognized fields");
    auto tone = std::make_shared<ToneCurveNode>(linear, shoulder, gamma);
    if (mode == "srgb_preview") return std::make_shared<SrgbEncodeNode>(tone);
    return std::make_shared<OutputClipNode>(tone);
}

}  // namespace

// EditGraph.cpp:1540-1560
EditDomain descriptor_domain(const ImageDescriptor& d) {
    if (d == ImageDescriptor::camera_linear()) return EditDomain::CameraLinear;
    if (d == ImageDescriptor::scene_linear(WorkingSpace::LinearProPhotoD50)) return EditDomain::SceneLinearProPhotoD50;
    if (d == ImageDescriptor::scene_linear(WorkingSpace::LinearRec2020D65)) return EditDomain::SceneLinearRec2020D65;
    if (d == ImageDescriptor::linear_srgb()) return EditDomain::SceneLinearSrgb;
    if (d.domain == PixelDomain::ToneMappedUnmanagedRGB && d.transfer == TransferFunction::CustomTone)
        return EditDomain::ToneMappedUnmanaged;
    if (d == ImageDescriptor::display_linear_srgb()) return EditDomain::DisplayLinearSrgb;
    if (d == ImageDescriptor::srgb_output()) return EditDomain::DisplayEncodedSrgb;
    if (d.domain == PixelDomain::DisplayEncodedRGB && d.primaries == ColorPrimaries::ICCProfile &&
        d.transfer == TransferFunction::ICCProfile)
        return EditDomain::DisplayEncodedIcc;
    if (d.domain == PixelDomain::BoundedUnmanagedRGB && d.transfer == TransferFunction::CustomTone)
        return EditDomain::UnmanagedBounded;
    throw std::invalid_argument("runtime node has an unsupported edit color domain");
}

// EditGraph.cpp:1655-1733, the render-path operation types.
std::shared_ptr<const Node> build_operation(const EditOperation& op, std::shared_ptr<const Node> input,
                                            WorkingSpace working_space, Rect source_bounds) {
    if (!input) throw std::invalid_argument("operation requires an input node");
    if (!op.masks.empty() || op.blend_mode != "normal" || op.opacity != 1.0 || !op.extra_fields.empty())
        throw std::invalid_argument("operation uses an unsupported input, mask, blend or extension");
    if (!op.enabled) return input;
    const auto& p = op.parameters;
    const std::string& t = op.type_id;
    if (t == "rawengine.curves_extended") return std::make_shared<ExtendedCurvesNode>(input, extended_curves_settings(p));
    if (t == "rawengine.sharpen") return std::make_shared<SharpenNode>(input, source_bounds, sharpen_settings(p));
    if (t == "rawengine.white_balance")
        return std::make_shared<WhiteBalanceNode>(input, scalar(p, "red_gain"), scalar(p, "green_gain"),
                                                  scalar(p, "blue_gain"));
    if (t == "rawengine.exposure") return std::make_shared<ExposureNode>(input, scalar(p, "stops"));
    if (t == "rawengine.camera_to_working")
        return std::make_shared<CameraToWorkingNode>(
            input, camera_transform(p, working_from_domain(op.output_domain), "matrix"), source_bounds);
    if (t == "rawengine.working_space_convert")
        return std::make_shared<WorkingSpaceConvertNode>(input, working_from_domain(op.output_domain));
    if (t == "rawengine.working_to_srgb") return std::make_shared<WorkingToSrgbNode>(input);
    if (t == "rawengine.tone_curve")
        return std::make_shared<ToneCurveNode>(input, scalar(p, "shoulder"), scalar(p, "gamma"));
    if (t == "rawengine.convolution")
        return std::make_shared<ConvolutionNode>(input, source_bounds, convolution_kernel(p));
    if (t == "rawengine.clarity") return std::make_shared<ClarityNode>(input, source_bounds, clarity_settings(p));
    if (t == "rawengine.guided_filter_working_y")
        return std::make_shared<WorkingYGuidedFilterNode>(input, source_bounds, guided_filter_settings(p));
    if (t == "rawengine.texture") return std::make_shared<TextureNode>(input, source_bounds, texture_settings(p));
    if (t == "rawengine.cubic_resize")
        return std::make_shared<CubicResizeNode>(input, source_bounds, cubic_resize_settings(p));
    if (t == "rawengine.rotate") {
        const auto found = p.find("angle_degrees");
        if (found == p.end()) throw std::invalid_argument("missing edit field: angle_degrees");
        return std::make_shared<RotateNode>(input, source_bounds, RotateSettings{number(found->second)});
    }
    if (t == "rawengine.output_clip") return std::make_shared<OutputClipNode>(input);
    if (t == "rawengine.srgb_encode") return std::make_shared<SrgbEncodeNode>(input);
    if (t == "rawengine.legacy.fixed_chain") return build_legacy_chain(op, input, working_space);
    throw std::invalid_argument("operation is not supported by this library: " + t);
}

}  // namespace rawengine
