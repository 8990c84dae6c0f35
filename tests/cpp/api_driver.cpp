// Test driver for the drop-in C++ surface (include/rawengine/*.hpp).
//
//   api_driver validate            host-only checks (no device work)
//   api_driver render <dir>        renders the scenarios of <dir>/params.txt
//
// `render` reads the RAW and raster inputs written by the pytest side, renders
// each scenario through the rawengine:: classes, writes <dir>/<name>.bin and
// prints "OUT <name> <x> <y> <w> <h> <type>" lines; the pytest side compares
// them with the oracle.  Behavioural checks (exceptions, descriptors, tile
// assembly, scheduler order) are asserted here and reported as "CHECK <name>".
// The checks mirror the reference's own core, spatial, geometry and scheduler
// tests (tests/core_tests.cpp, spatial_ops_tests.cpp, rotate_tests.cpp,
// cubic_resize_tests.cpp of tylermcm/librawops) on this path.
#include <rawengine/EditOps.hpp>
#include <rawengine/GeometryOps.hpp>
#include <rawengine/ImageAnalysis.hpp>
#include <rawengine/RawEngine.hpp>
#include <rawengine/SpatialOps.hpp>
#include <rawengine/TileScheduler.hpp>
#include <rawengine/ToneOps.hpp>

#include <chrono>
#include <limits>
#include <numeric>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>

using namespace rawengine;

namespace {

int failures = 0;

void check(bool ok, const std::string& name) {
    std::cout << (ok ? "CHECK " : "FAIL ") << name << std::endl;
    if (!ok) ++failures;
}

template <class E, class F>
void expect_throw(F&& f, const std::string& name) {
    try {
        f();
    } catch (const E&) {
        check(true, name);
        return;
    } catch (const std::exception& e) {
        std::cout << "  (threw " << e.what() << ")" << std::endl;
    }
    check(false, name);
}

std::map<std::string, std::vector<double>> read_params(const std::string& path) {
    std::map<std::string, std::vector<double>> out;
    std::ifstream in(path);
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ss(line);
        std::string key;
        if (!(ss >> key)) continue;
        double v;
        while (ss >> v) out[key].push_back(v);
    }
    return out;
}

template <class T>
std::vector<T> read_file(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    in.seekg(0, std::ios::end);
    const size_t bytes = (size_t)in.tellg();
    in.seekg(0);
    std::vector<T> v(bytes / sizeof(T));
    in.read(reinterpret_cast<char*>(v.data()), (std::streamsize)bytes);
    return v;
}

template <class T>
void emit(const std::string& dir, const std::string& name, Rect r, const std::vector<T>& data, const char* type) {
    std::ofstream out(dir + "/" + name + ".bin", std::ios::binary);
    out.write(reinterpret_cast<const char*>(data.data()), (std::streamsize)(data.size() * sizeof(T)));
    std::cout << "OUT " << name << " " << r.x << " " << r.y << " " << r.width << " " << r.height << " " << type
              << std::endl;
}

Rect rect_of(const std::vector<double>& v, size_t at = 0) {
    return {(uint32_t)v[at], (uint32_t)v[at + 1], (uint32_t)v[at + 2], (uint32_t)v[at + 3]};
}

bool bit_equal(const std::vector<float>& a, const std::vector<float>& b) {
    return a.size() == b.size() && std::memcmp(a.data(), b.data(), a.size() * sizeof(float)) == 0;
}

// A node of another library: constant camera-linear RGB.
class ConstantCameraNode final : public Node {
public:
    explicit ConstantCameraNode(std::array<float, 3> px) : px_(px) {}
    ImageDescriptor output_descriptor() const noexcept override { return ImageDescriptor::camera_linear(); }
    Tile render(Rect b) const override {
        Tile t{b, std::vector<float>((size_t)b.width * b.height * 3)};
        for (size_t i = 0; i < t.rgb.size(); i += 3) std::copy(px_.begin(), px_.end(), t.rgb.begin() + i);
        return t;
    }
    // The reference's identity hooks, overridden as a reference user would.
    std::optional<IccProfileIdentity> input_icc_identity() const override { return std::nullopt; }
    std::optional<std::array<std::uint8_t, 32>> source_fingerprint() const override {
        std::array<std::uint8_t, 32> f{};
        f[0] = 0x5a;
        return f;
    }
private:
    std::array<float, 3> px_;
};

// A node that returns a tile with the wrong descriptor.
class WrongDescriptorNode final : public Node {
public:
    ImageDescriptor output_descriptor() const noexcept override { return ImageDescriptor::camera_linear(); }
    Tile render(Rect b) const override {
        return {b, std::vector<float>((size_t)b.width * b.height * 3), ImageDescriptor::tone_mapped()};
    }
};

// Scene-linear node whose render blocks until released, recording the order
// in which requests reach it (scheduler tests).
struct Gate {
    std::mutex m;
    std::condition_variable cv;
    bool open = false;
    int entered = 0;
    std::vector<int> order;
};
class GatedNode final : public Node {
public:
    GatedNode(Gate* g, int id) : g_(g), id_(id) {}
    ImageDescriptor output_descriptor() const noexcept override {
        return ImageDescriptor::scene_linear(WorkingSpace::LinearProPhotoD50);
    }
    Tile render(Rect b) const override {
        std::unique_lock<std::mutex> lock(g_->m);
        ++g_->entered;
        g_->order.push_back(id_);
        g_->cv.notify_all();
        g_->cv.wait_for(lock, std::chrono::seconds(20), [&] { return g_->open; });
        return {b, std::vector<float>((size_t)b.width * b.height * 3, (float)id_), output_descriptor()};
    }
private:
    Gate* g_;
    int id_;
};

RawImage make_raw(const std::map<std::string, std::vector<double>>& P, const std::string& dir) {
    const auto& m = P.at("raw_meta");
    RawMetadata md;
    md.width = (uint32_t)m[0];
    md.height = (uint32_t)m[1];
    md.row_stride_samples = (uint32_t)m[2];
    md.pattern = (BayerPattern)(int)m[3];
    md.cfa_phase_x = (uint8_t)m[4];
    md.cfa_phase_y = (uint8_t)m[5];
    md.active_area = rect_of(m, 6);
    for (int i = 0; i < 4; ++i) {
        md.black_levels[i] = (uint16_t)m[10 + i];
        md.white_levels[i] = (uint16_t)m[14 + i];
    }
    return RawImage(md, read_file<uint16_t>(dir + "/raw.u16"));
}

CameraColorTransform camera(const std::map<std::string, std::vector<double>>& P, WorkingSpace target) {
    CameraColorTransform t;
    const auto& c = P.at("camera");
    std::copy(c.begin(), c.begin() + 9, t.camera_to_xyz_d50.begin());
    t.target = target;
    return t;
}

// ------------------------------------------------------------------ render

// ------------------------------------------------------------- histogram

// The reference's analysis probe (image_analysis_tests.cpp:20-41): a caller
// Node whose tiles are R = (x % 9) / 4 - 0.5, G = (y % 9) / 4 - 0.5, B = NaN,
// with optional faults in the delivered tile.
class HistogramProbe final : public Node {
public:
    enum class Fault { None, Bounds, Storage, Descriptor };
    Fault fault = Fault::None;
    CancellationToken* cancellation = nullptr;
    mutable unsigned calls = 0;
    mutable std::uint64_t largest_tile = 0;
    ImageDescriptor output_descriptor() const noexcept override { return ImageDescriptor::camera_linear(); }
    Tile render(Rect r) const override {
        ++calls;
        largest_tile = std::max<std::uint64_t>(largest_tile, std::uint64_t(r.width) * r.height);
        Tile tile{r, {}, output_descriptor()};
        for (std::uint32_t y = r.y; y < r.y + r.height; ++y)
            for (std::uint32_t x = r.x; x < r.x + r.width; ++x) {
                tile.rgb.push_back(float(x % 9) * 0.25f - 0.5f);
                tile.rgb.push_back(float(y % 9) * 0.25f - 0.5f);
                tile.rgb.push_back(std::numeric_limits<float>::quiet_NaN());
            }
        if (fault == Fault::Bounds) ++tile.bounds.x;
        if (fault == Fault::Storage) tile.rgb.pop_back();
        if (fault == Fault::Descriptor) tile.descriptor = ImageDescriptor::srgb_output();
        if (cancellation) cancellation->cancel();
        return tile;
    }
};

bool same_histogram(const RgbHistogram& a, const RgbHistogram& b) {
    for (int c = 0; c < 3; ++c) {
        const auto &x = a.channels[c], &y = b.channels[c];
        if (x.counts != y.counts || x.underflow != y.underflow || x.overflow != y.overflow ||
            x.nonfinite != y.nonfinite || x.minimum != y.minimum || x.maximum != y.maximum)
            return false;
    }
    return a.pixel_count == b.pixel_count;
}

// Histogram of a rendered device image counted sample by sample on the host,
// for comparing the device path of a DeviceNode chain.
RgbHistogram host_histogram(const Tile& t, const HistogramOptions& o) {
    RgbHistogram h;
    for (auto& c : h.channels) c.counts.assign(o.bins, 0);
    const double span = o.upper - o.lower;
    for (size_t i = 0; i < t.rgb.size(); ++i) {
        const float s = t.rgb[i];
        auto& c = h.channels[i % 3];
        if (!std::isfinite(s)) {
            ++c.nonfinite;
            continue;
        }
        if (!c.minimum || s < *c.minimum) c.minimum = s;
        if (!c.maximum || s > *c.maximum) c.maximum = s;
        if (s < o.lower) {
            ++c.underflow;
            continue;
        }
        if (s > o.upper) {
            ++c.overflow;
            continue;
        }
        ++c.counts[std::min<std::uint32_t>(o.bins - 1, (std::uint32_t)((double(s) - o.lower) / span * o.bins))];
    }
    h.pixel_count = t.rgb.size() / 3;
    return h;
}

void histogram_checks(const std::shared_ptr<const Node>& graph_node, Rect area) {
    {   // edge bins, clipped tiles over a nonzero viewport, tile partitions
        HistogramProbe node;
        const Rect bounds{7, 5, 31, 23};
        const RenderRequest request{{9, 7, 19, 13}, 4};
        const auto result = histogram_rgb(node, bounds, request, {4, 0, 1});
        check(result.pixel_count == 247 && node.largest_tile <= 16 && node.calls == 20, "histogram_streams_tiles");
        check(result.descriptor == node.output_descriptor(), "histogram_descriptor");
        bool bins_ok = true;
        for (unsigned c = 0; c < 2; ++c) {
            std::array<std::uint64_t, 4> expected{};
            std::uint64_t below = 0, above = 0;
            for (unsigned y = 7; y < 20; ++y)
                for (unsigned x = 9; x < 28; ++x) {
                    const auto site = (c == 0 ? x : y) % 9;
                    if (site < 2) ++below;
                    else if (site > 6) ++above;
                    else ++expected[site == 6 ? 3 : site - 2];
                }
            const auto& ch = result.channels[c];
            bins_ok &= std::equal(expected.begin(), expected.end(), ch.counts.begin()) && ch.underflow == below &&
                       ch.overflow == above && ch.nonfinite == 0 && ch.minimum == -0.5f && ch.maximum == 1.5f;
        }
        check(bins_ok, "histogram_bin_edges_and_outliers");
        check(result.channels[2].nonfinite == 247 && !result.channels[2].minimum && !result.channels[2].maximum,
              "histogram_all_nonfinite_channel");
        bool partitions = true;
        for (unsigned size : {1u, 3u, 7u, 256u})
            partitions &= same_histogram(histogram_rgb(node, bounds, RenderRequest{request.viewport, size}, {4, 0, 1}),
                                         result);
        check(partitions, "histogram_tile_partitions");
    }
    {   // non-finite samples and extreme ranges
        class Values final : public Node {
        public:
            ImageDescriptor output_descriptor() const noexcept override { return ImageDescriptor::linear_srgb(); }
            Tile render(Rect r) const override {
                const float inf = std::numeric_limits<float>::infinity();
                return {r, {-inf, 0, -2, inf, 1, 2, std::numeric_limits<float>::quiet_NaN(), 0.5f, 0},
                        output_descriptor()};
            }
        } node;
        auto result = histogram_rgb(node, {0, 0, 3, 1}, RenderRequest{{0, 0, 3, 1}}, {1, 0, 1});
        check(result.channels[0].nonfinite == 3 && !result.channels[0].minimum, "histogram_infinities_nonfinite");
        check(result.channels[1].counts[0] == 3 && result.channels[2].underflow == 1 &&
                  result.channels[2].overflow == 1,
              "histogram_single_bin_endpoints");
        result = histogram_rgb(node, {0, 0, 3, 1}, RenderRequest{{0, 0, 3, 1}}, {65536, -1e300, 1e300});
        check(result.channels[1].counts[32768] == 3, "histogram_wide_range");
        result = histogram_rgb(node, {0, 0, 3, 1}, RenderRequest{{0, 0, 3, 1}},
                               {2, 0, std::numeric_limits<double>::denorm_min()});
        check(result.channels[1].counts[0] == 1 && result.channels[1].overflow == 2, "histogram_tiny_range");
    }
    {   // invalid arguments and cancellation
        HistogramProbe node;
        const Rect bounds{0, 0, 9, 9};
        const RenderRequest request{bounds, 3};
        const double nan = std::numeric_limits<double>::quiet_NaN(), inf = std::numeric_limits<double>::infinity();
        int i = 0;
        for (const auto options : {HistogramOptions{0, 0, 1}, {65537, 0, 1}, {4, 1, 1}, {4, 2, 1}, {4, nan, 1},
                                   {4, 0, inf}, {4, -1e308, 1e308}})
            expect_throw<std::invalid_argument>([&] { histogram_rgb(node, bounds, request, options); },
                                                "histogram_rejects_options_" + std::to_string(i++));
        check(node.calls == 0, "histogram_invalid_options_render_nothing");
        expect_throw<std::invalid_argument>([&] { histogram_rgb(node, bounds, RenderRequest{{0, 0, 0, 1}}); },
                                            "histogram_rejects_empty");
        expect_throw<std::invalid_argument>([&] { histogram_rgb(node, bounds, RenderRequest{bounds, 0}); },
                                            "histogram_rejects_zero_tile");
        expect_throw<std::invalid_argument>(
            [&] { histogram_rgb(node, bounds, RenderRequest{{0, 0, 4, 4}, 3, {1, RenderQuality::Preview}}); },
            "histogram_rejects_level");
        expect_throw<std::out_of_range>([&] { histogram_rgb(node, bounds, RenderRequest{{8, 8, 2, 2}}); },
                                        "histogram_rejects_outside");
        expect_throw<std::invalid_argument>(
            [&] { histogram_rgb(node, {0xffffffffu, 0, 2, 1}, RenderRequest{{0xffffffffu, 0, 2, 1}}); },
            "histogram_rejects_unaddressable");
        for (auto fault : {HistogramProbe::Fault::Bounds, HistogramProbe::Fault::Storage,
                           HistogramProbe::Fault::Descriptor}) {
            node.fault = fault;
            expect_throw<std::invalid_argument>([&] { histogram_rgb(node, bounds, request); },
                                                "histogram_rejects_fault_" + std::to_string((int)fault));
        }
        node.fault = HistogramProbe::Fault::None;
        CancellationToken token;
        token.cancel();
        const auto before = node.calls;
        expect_throw<RenderCancelled>([&] { histogram_rgb(node, bounds, request, {}, &token); },
                                      "histogram_precancelled");
        check(node.calls == before, "histogram_precancelled_renders_nothing");
        CancellationToken last_tile;
        node.cancellation = &last_tile;
        expect_throw<RenderCancelled>([&] { histogram_rgb(node, bounds, RenderRequest{bounds}, {}, &last_tile); },
                                      "histogram_cancelled_in_tile");
        check(node.calls == before + 1, "histogram_cancelled_after_one_tile");
    }
    {   // ImageGraph overload
        RawImage image(5, 3, std::vector<std::uint16_t>(15, 32768));
        ImageGraph graph(image, GraphRecipe{});
        const auto h = histogram_rgb(graph, RenderRequest{{0, 0, 5, 3}, 2});
        bool covered = h.pixel_count == 15 && h.descriptor == graph.output().output_descriptor();
        for (const auto& c : h.channels)
            covered &= std::accumulate(c.counts.begin(), c.counts.end(), std::uint64_t{}) + c.underflow + c.overflow +
                           c.nonfinite == 15;
        check(covered, "histogram_image_graph_overload");
    }
    {   // a device chain: counted on the device in bands, equal to counting its rendered image
        const HistogramOptions o{1024, -0.1, 1.1};
        bool ok = true;
        for (std::uint32_t tile : {5u, 64u, 4096u}) {
            const RenderRequest req{area, tile};
            const Tile img = Renderer{}.render_image(*graph_node, area, req);
            ok &= same_histogram(histogram_rgb(*graph_node, area, req, o), host_histogram(img, o));
        }
        check(ok, "histogram_device_chain_equals_rendered_image");
    }
}

// --------------------------------------------------------------- stencils

// Sharpen, Clarity, Texture and Convolution over the working chain: outputs
// at mip 0 over stencil_vp and over the whole mip 1 level (compared with the
// reference on the pytest side), tile independence, pass-through cases and
// the nodes' validation.
void stencil_checks(const std::string& dir, const std::map<std::string, std::vector<double>>& P,
                    const std::shared_ptr<const Node>& working, Rect area) {
    Renderer renderer;
    const auto& sp = P.at("sharpen");
    const auto& cl = P.at("clarity");
    const auto& tx = P.at("texture");
    const auto& cv = P.at("convolution");
    ConvolutionKernel k;
    k.width = (uint32_t)cv[0];
    k.height = (uint32_t)cv[1];
    k.coefficients.assign(cv.begin() + 2, cv.end());
    const std::vector<std::pair<std::string, std::shared_ptr<const Node>>> nodes = {
        {"sharpen", std::make_shared<SharpenNode>(working, area, SharpenSettings{sp[0], (uint32_t)sp[1]})},
        {"clarity", std::make_shared<ClarityNode>(working, area, ClaritySettings{cl[0], (uint32_t)cl[1]})},
        {"texture", std::make_shared<TextureNode>(working, area, TextureSettings{tx[0], (uint32_t)tx[1]})},
        {"convolution", std::make_shared<ConvolutionNode>(working, area, k)}};
    const Rect vp = rect_of(P.at("stencil_vp"));
    const RenderLevel mip1{1, RenderQuality::Preview};
    const Rect level1{0, 0, (area.width + 1) / 2, (area.height + 1) / 2};
    for (const auto& [name, node] : nodes) {
        const Tile t = renderer.render_image(*node, area, RenderRequest{vp, 4096});
        emit(dir, "stencil_" + name, t.bounds, t.rgb, "f32");
        const Tile m = renderer.render_image(*node, area, RenderRequest{level1, 4096, mip1});
        emit(dir, "stencil_" + name + "_mip1", m.bounds, m.rgb, "f32");
        std::vector<float> tiled(t.rgb.size());
        renderer.render_tiles(*node, area, RenderRequest{vp, 13}, [&](const Tile& tile) {
            for (uint32_t row = 0; row < tile.bounds.height; ++row)
                std::memcpy(tiled.data() + ((size_t)(tile.bounds.y - vp.y + row) * vp.width + tile.bounds.x - vp.x) * 3,
                            tile.rgb.data() + (size_t)row * tile.bounds.width * 3,
                            (size_t)tile.bounds.width * 3 * sizeof(float));
        });
        check(bit_equal(tiled, t.rgb), "stencil_tiles_equal_whole_" + name);
        check(node->output_descriptor() == working->output_descriptor(), "stencil_descriptor_" + name);
        expect_throw<std::invalid_argument>(
            [&] { (void)node->input_region_level(vp, Rect{0, 0, area.width, area.height}, {}); },
            "stencil_rejects_other_bounds_" + name);
        expect_throw<std::out_of_range>(
            [&] { (void)node->input_region(Rect{area.x + area.width - 2, area.y, 5, 5}, area); },
            "stencil_rejects_outside_" + name);
        check(node->supports_level(mip1) && node->supports_level({}) && !node->supports_level({1, RenderQuality::Final}) &&
                  node->supports_level({0, RenderQuality::Preview}) == working->supports_level({0, RenderQuality::Preview}),
              "stencil_levels_" + name);
    }
    // pass-through: zero amounts and an identity kernel return the input pixels
    const Tile in = renderer.render_image(*working, area, RenderRequest{vp, 4096});
    ConvolutionKernel ident{3, 3, {0, 0, 0, 0, 1, 0, 0, 0, 0}};
    const std::vector<std::shared_ptr<const Node>> passes = {
        std::make_shared<SharpenNode>(working, area, SharpenSettings{0.0, 3}),
        std::make_shared<ClarityNode>(working, area, ClaritySettings{0.0, 8}),
        std::make_shared<TextureNode>(working, area, TextureSettings{0.0, 4}),
        std::make_shared<ConvolutionNode>(working, area, ident)};
    bool same_pixels = true;
    for (const auto& n : passes) {
        same_pixels &= bit_equal(renderer.render_image(*n, area, RenderRequest{vp, 4096}).rgb, in.rgb);
        const Rect r = n->input_region(vp, area);
        same_pixels &= r.x == vp.x && r.y == vp.y && r.width == vp.width && r.height == vp.height;
    }
    check(same_pixels, "stencil_pass_through");
    // settings and input validation
    expect_throw<std::invalid_argument>([&] { SharpenNode(working, area, SharpenSettings{2.5, 1}); },
                                        "sharpen_rejects_amount");
    expect_throw<std::invalid_argument>([&] { SharpenNode(working, area, SharpenSettings{1.0, 4}); },
                                        "sharpen_rejects_radius");
    expect_throw<std::invalid_argument>([&] { ClarityNode(working, area, ClaritySettings{-1.5, 3}); },
                                        "clarity_rejects_amount");
    expect_throw<std::invalid_argument>([&] { ClarityNode(working, area, ClaritySettings{0.5, 9}); },
                                        "clarity_rejects_radius");
    expect_throw<std::invalid_argument>([&] { TextureNode(working, area, TextureSettings{0.5, 5}); },
                                        "texture_rejects_scale");
    expect_throw<std::invalid_argument>([&] { ConvolutionNode(working, area, ConvolutionKernel{2, 3, {1, 1, 1, 1, 1, 1}}); },
                                        "convolution_rejects_even");
    expect_throw<std::invalid_argument>([&] { ConvolutionNode(working, area, ConvolutionKernel{3, 1, {1, 1e6, 1}}); },
                                        "convolution_rejects_coefficient");
    expect_throw<std::invalid_argument>([&] { ClarityNode(nullptr, area, ClaritySettings{0.5, 3}); },
                                        "clarity_requires_input");
    expect_throw<std::invalid_argument>(
        [&] { SharpenNode(std::make_shared<SrgbEncodeNode>(std::make_shared<WorkingToSrgbNode>(working)), area,
                          SharpenSettings{1.0, 1}); },
        "sharpen_requires_working_rgb");
    expect_throw<std::invalid_argument>([&] { TextureNode(working, Rect{0, 0, 0, 4}, TextureSettings{0.5, 1}); },
                                        "texture_rejects_empty_bounds");
}

// ------------------------------------------------------ operation factory

EditValue num(double v) { return EditValue{v}; }
EditValue integer(std::int64_t v) { return EditValue{v}; }
EditValue str(const char* v) { return EditValue{std::string(v)}; }
EditValue list(std::initializer_list<double> v) {
    EditValue::Array a;
    for (double x : v) a.push_back(num(x));
    return EditValue{a};
}
EditOperation operation(const char* type, EditValue::Object params,
                        EditDomain out = EditDomain::SceneLinearProPhotoD50) {
    EditOperation op;
    op.id = std::string("op-") + type;
    op.type_id = type;
    op.parameters = std::move(params);
    op.output_domain = out;
    op.inputs = {{"image", "source"}};
    return op;
}
EditValue knots(const std::vector<CurvePoint>& k) {
    EditValue::Array a;
    for (const auto& p : k) a.push_back(EditValue{EditValue::Array{num(p.x), num(p.y)}});
    return EditValue{a};
}

// Chains built by build_operation render exactly as the same chains built
// from the node constructors (EditGraph.cpp:1655-1733).
void factory_checks(const std::map<std::string, std::vector<double>>& P, const RawImage& raw, Rect area) {
    Renderer renderer;
    const auto cam = camera(P, WorkingSpace::LinearProPhotoD50);
    EditValue::Array m;
    for (double v : cam.camera_to_xyz_d50) m.push_back(num(v));
    auto same_render = [&](const Node& a, const Node& b, Rect bounds, RenderRequest req) {
        return bit_equal(renderer.render_image(a, bounds, req).rgb, renderer.render_image(b, bounds, req).rgb) &&
               a.output_descriptor() == b.output_descriptor();
    };
    auto menon = std::make_shared<RawUnpackNode>(raw, RawDemosaicIdentity{"rawengine.menon_base", 1});
    const WorkingSpace pp = WorkingSpace::LinearProPhotoD50;
    // point chain: WB -> camera-to-working -> curves -> sRGB
    std::shared_ptr<const Node> f = build_operation(
        operation("rawengine.white_balance", {{"red_gain", num(1.9)}, {"green_gain", integer(1)}, {"blue_gain", num(1.4)}}),
        menon, pp, area);
    f = build_operation(operation("rawengine.exposure", {{"stops", num(0.25)}}), f, pp, area);
    f = build_operation(operation("rawengine.camera_to_working", {{"matrix", EditValue{m}}}), f, pp, area);
    const std::vector<CurvePoint> curve{{0, 0}, {0.3, 0.4}, {0.7, 0.75}, {1, 1}};
    f = build_operation(operation("rawengine.curves_extended",
                                  {{"master", knots(curve)}, {"red", knots({{0, 0}, {1, 1}})},
                                   {"green", knots({{0, 0}, {0.5, 0.55}, {1, 1}})}, {"blue", knots({{0, 0}, {1, 1}})},
                                   {"interpolation", str("shape_preserving_cubic")}}),
                        f, pp, area);
    std::shared_ptr<const Node> d = std::make_shared<WhiteBalanceNode>(menon, 1.9f, 1.0f, 1.4f);
    d = std::make_shared<ExposureNode>(d, 0.25f);
    d = std::make_shared<CameraToWorkingNode>(d, cam, area);
    ExtendedCurvesSettings cs;
    cs.master.knots = curve;
    cs.channels[1].knots = {{0, 0}, {0.5, 0.55}, {1, 1}};
    cs.interpolation = CurveInterpolation::ShapePreservingCubic;
    d = std::make_shared<ExtendedCurvesNode>(d, cs);
    const Rect vp{area.x + 5, area.y + 4, 60, 45};
    const RenderLevel mip1{1, RenderQuality::Preview};
    check(same_render(*f, *d, area, RenderRequest{vp, 32}) &&
              same_render(*f, *d, area, RenderRequest{{0, 0, 30, 20}, 32, mip1}),
          "factory_point_chain");
    const auto working_f = f, working_d = d;
    auto srgb_f = build_operation(operation("rawengine.srgb_encode", {}),
                                  build_operation(operation("rawengine.tone_curve", {{"shoulder", num(0.3)}, {"gamma", num(2.2)}}),
                                                  build_operation(operation("rawengine.working_to_srgb", {}), f, pp, area),
                                                  pp, area),
                                  pp, area);
    auto srgb_d = std::make_shared<SrgbEncodeNode>(
        std::make_shared<ToneCurveNode>(std::make_shared<WorkingToSrgbNode>(d), 0.3f, 2.2f));
    check(same_render(*srgb_f, *srgb_d, area, RenderRequest{vp, 32}), "factory_srgb_chain");
    // spatial, stencil and geometry operations over the working image
    struct Case {
        const char* name;
        std::shared_ptr<const Node> f, d;
    };
    const Rect image{0, 0, area.width, area.height};
    ConvolutionKernel k{3, 3, {0.0, -0.25, 0.0, -0.25, 2.0, -0.25, 0.0, -0.25, 0.0}};
    EditValue::Array kc;
    for (double v : k.coefficients) kc.push_back(num(v));
    const uint32_t cw = (area.width + 1) / 2, ch = (area.height + 2) / 3;
    std::vector<Case> cases = {
        {"guided_filter",
         build_operation(operation("rawengine.guided_filter_working_y", {{"radius", integer(3)}, {"epsilon", num(0.001)}}),
                         working_f, pp, area),
         std::make_shared<WorkingYGuidedFilterNode>(working_d, area, WorkingYGuidedFilterSettings{3, 0.001})},
        {"sharpen", build_operation(operation("rawengine.sharpen", {{"amount", num(0.8)}, {"radius", integer(2)}}),
                                    working_f, pp, area),
         std::make_shared<SharpenNode>(working_d, area, SharpenSettings{0.8, 2})},
        {"clarity", build_operation(operation("rawengine.clarity", {{"amount", num(-0.4)}, {"radius", integer(4)}}),
                                    working_f, pp, area),
         std::make_shared<ClarityNode>(working_d, area, ClaritySettings{-0.4, 4})},
        {"texture", build_operation(operation("rawengine.texture", {{"amount", num(0.5)}, {"scale", integer(2)}}),
                                    working_f, pp, area),
         std::make_shared<TextureNode>(working_d, area, TextureSettings{0.5, 2})},
        {"convolution",
         build_operation(operation("rawengine.convolution", {{"width", integer(3)}, {"height", integer(3)},
                                                             {"coefficients", EditValue{kc}}, {"border", str("replicate")}}),
                         working_f, pp, area),
         std::make_shared<ConvolutionNode>(working_d, area, k)},
        {"working_space_convert",
         build_operation(operation("rawengine.working_space_convert", {}, EditDomain::SceneLinearRec2020D65), working_f, pp,
                         area),
         std::make_shared<WorkingSpaceConvertNode>(working_d, WorkingSpace::LinearRec2020D65)},
        {"tone_output_clip",
         build_operation(operation("rawengine.output_clip", {}),
                         build_operation(operation("rawengine.tone_curve", {{"shoulder", num(0.2)}, {"gamma", num(1.8)}}),
                                         working_f, pp, area),
                         pp, area),
         std::make_shared<OutputClipNode>(std::make_shared<ToneCurveNode>(working_d, 0.2f, 1.8f))},
    };
    for (const auto& c : cases)
        check(same_render(*c.f, *c.d, area, RenderRequest{vp, 32}), std::string("factory_") + c.name);
    auto cubic_f = build_operation(operation("rawengine.cubic_resize", {{"width", integer(cw)}, {"height", integer(ch)}}),
                                   working_f, pp, area);
    auto cubic_d = std::make_shared<CubicResizeNode>(working_d, area, CubicResizeSettings{cw, ch});
    check(same_render(*cubic_f, *cubic_d, Rect{0, 0, cw, ch}, RenderRequest{{0, 0, cw, ch}, 32}), "factory_cubic");
    auto rot_f = build_operation(operation("rawengine.rotate", {{"angle_degrees", num(-23.5)}}), working_f, pp, area);
    auto rot_d = std::make_shared<RotateNode>(working_d, area, RotateSettings{-23.5});
    check(same_render(*rot_f, *rot_d, image, RenderRequest{{3, 2, 40, 30}, 32}), "factory_rotate");
    // the legacy fixed chain, both output modes
    auto bil = std::make_shared<RawUnpackNode>(raw);
    for (const char* mode : {"legacy_bounded", "srgb_preview"}) {
        EditValue::Object recipe{{"red_gain", num(1.7)},      {"green_gain", num(1.0)},  {"blue_gain", num(1.3)},
                                 {"exposure_stops", num(0.4)}, {"tone_shoulder", num(0.25)}, {"tone_gamma", num(2.0)},
                                 {"output_mode", str(mode)}};
        const bool srgb = std::string(mode) == "srgb_preview";
        if (srgb) {
            recipe.emplace("camera_to_xyz_d50", EditValue{m});
            recipe.emplace("camera_target", str("linear_prophoto_d50"));
        }
        auto lf = build_operation(operation("rawengine.legacy.fixed_chain", {{"recipe", EditValue{recipe}}}), bil, pp, area);
        std::shared_ptr<const Node> ld = std::make_shared<ExposureNode>(std::make_shared<WhiteBalanceNode>(bil, 1.7f, 1.0f, 1.3f), 0.4f);
        if (srgb) ld = std::make_shared<WorkingToSrgbNode>(std::make_shared<CameraToWorkingNode>(ld, cam));
        auto tone = std::make_shared<ToneCurveNode>(ld, 0.25f, 2.0f);
        ld = srgb ? std::static_pointer_cast<const Node>(std::make_shared<SrgbEncodeNode>(tone))
                  : std::static_pointer_cast<const Node>(std::make_shared<OutputClipNode>(tone));
        check(same_render(*lf, *ld, area, RenderRequest{vp, 32}), std::string("factory_legacy_") + mode);
    }
    // a disabled operation is its input
    auto off = operation("rawengine.exposure", {{"stops", num(3.0)}});
    off.enabled = false;
    check(build_operation(off, working_f, pp, area) == working_f, "factory_disabled_passes_input");
}

// Factory rejections (host only).
void factory_validation(const std::shared_ptr<const Node>& working, Rect area) {
    const WorkingSpace pp = WorkingSpace::LinearProPhotoD50;
    auto rejects = [&](const EditOperation& op, const std::string& name) {
        expect_throw<std::invalid_argument>([&] { (void)build_operation(op, working, pp, area); }, name);
    };
    rejects(operation("rawengine.vibrance", {{"amount", num(0.2)}}), "factory_rejects_unsupported_type");
    rejects(operation("rawengine.exposure", {}), "factory_rejects_missing_scalar");
    rejects(operation("rawengine.exposure", {{"stops", num(1e300)}}), "factory_rejects_float32_range");
    rejects(operation("rawengine.sharpen", {{"amount", num(0.5)}}), "factory_rejects_sharpen_fields");
    rejects(operation("rawengine.sharpen", {{"amount", num(0.5)}, {"radius", num(2.0)}}), "factory_rejects_float_radius");
    rejects(operation("rawengine.clarity", {{"amount", num(2.0)}, {"radius", integer(2)}}), "factory_rejects_clarity_amount");
    rejects(operation("rawengine.guided_filter_working_y", {{"radius", num(2.5)}, {"epsilon", num(0.01)}}),
            "factory_rejects_fractional_gf_radius");
    rejects(operation("rawengine.convolution", {{"width", integer(1)}, {"height", integer(1)}, {"coefficients", list({1})},
                                                {"border", str("zero")}}),
            "factory_rejects_border");
    rejects(operation("rawengine.curves_extended", {{"master", knots({{0, 0}, {1, 1}})}, {"red", knots({{0, 0}, {1, 1}})},
                                                    {"green", knots({{0, 0}, {1, 1}})}, {"blue", knots({{0, 0}, {1, 1}})},
                                                    {"interpolation", str("spline")}}),
            "factory_rejects_interpolation");
    rejects(operation("rawengine.camera_to_working", {{"matrix", list({1, 0, 0})}}), "factory_rejects_matrix_size");
    rejects(operation("rawengine.working_space_convert", {}, EditDomain::DisplayEncodedSrgb), "factory_rejects_target");
    auto masked = operation("rawengine.exposure", {{"stops", num(1.0)}});
    masked.masks = {{"mask", "brush"}};
    rejects(masked, "factory_rejects_masks");
    auto blended = operation("rawengine.exposure", {{"stops", num(1.0)}});
    blended.opacity = 0.5;
    rejects(blended, "factory_rejects_opacity");
    EditValue::Object recipe{{"red_gain", num(1)},       {"green_gain", num(1)},    {"blue_gain", num(1)},
                             {"exposure_stops", num(0)}, {"tone_shoulder", num(0.2)}, {"tone_gamma", num(2)},
                             {"output_mode", str("legacy_bounded")}, {"unknown", num(1)}};
    rejects(operation("rawengine.legacy.fixed_chain", {{"recipe", EditValue{recipe}}}), "factory_rejects_legacy_field");
    check(descriptor_domain(working->output_descriptor()) == EditDomain::SceneLinearProPhotoD50,
          "factory_descriptor_domain");
}

// ----------------------------------------------------------- tile cache

// A caller Node that counts its renders (a constant per-position image).
class CountingNode final : public Node {
public:
    mutable unsigned calls = 0;
    bool broken = false;
    ImageDescriptor output_descriptor() const noexcept override {
        return ImageDescriptor::scene_linear(WorkingSpace::LinearProPhotoD50);
    }
    Tile render(Rect r) const override {
        ++calls;
        Tile t{r, std::vector<float>((size_t)r.width * r.height * 3), output_descriptor()};
        for (size_t i = 0; i < t.rgb.size(); ++i) t.rgb[i] = 0.001f * (float)((r.x + r.y + i) % 997);
        if (broken) t.rgb.pop_back();
        return t;
    }
};

// TileCache (EditGraph.cpp:23-80 rules) and CachedNode over a device chain.
void cache_checks(const RawImage& raw, Rect area, const std::map<std::string, std::vector<double>>& P) {
    std::array<std::uint8_t, 32> sig{};
    sig[0] = 7;
    {
        CountingNode node;
        TileCache cache(64 * 1024);
        const Rect r{3, 4, 20, 10};   // 2400 bytes + 256
        const Tile a = cache.render(node, sig, r);
        const Tile b = cache.render(node, sig, r);
        auto st = cache.stats();
        check(node.calls == 1 && bit_equal(a.rgb, b.rgb) && st.hits == 1 && st.misses == 1 && st.entries == 1 &&
                  st.used_bytes == 256 + 2400,
              "cache_hit_after_miss");
        const DeviceTile d = cache.render_device(node, sig, r);
        check(node.calls == 1 && bit_equal(d.to_host().rgb, a.rgb), "cache_device_hit");
        auto other = sig;
        other[1] = 1;
        (void)cache.render(node, other, r);
        (void)cache.render(node, sig, Rect{3, 4, 20, 11});
        check(node.calls == 3 && cache.stats().entries == 3, "cache_keys_signature_and_bounds");
        expect_throw<std::invalid_argument>([&] { (void)cache.render(node, sig, r, {32, RenderQuality::Preview}); },
                                            "cache_rejects_level");
        expect_throw<std::invalid_argument>([&] { (void)cache.render(node, sig, r, {1, RenderQuality::Preview}); },
                                            "cache_rejects_unsupported_level");
        node.broken = true;
        expect_throw<std::domain_error>([&] { (void)cache.render(node, sig, Rect{0, 0, 3, 3}); },
                                        "cache_rejects_invalid_tile");
        node.broken = false;
        cache.clear();
        st = cache.stats();
        check(st.entries == 0 && st.used_bytes == 0 && st.hits == 0 && st.misses == 0, "cache_clear");
    }
    {   // LRU eviction within the budget; oversized tiles are not cached
        CountingNode node;
        TileCache cache(2 * (256 + 1200) + 100);   // room for two 10x10 tiles
        const Rect a{0, 0, 10, 10}, b{10, 0, 10, 10}, c{20, 0, 10, 10};
        (void)cache.render(node, sig, a);
        (void)cache.render(node, sig, b);
        (void)cache.render(node, sig, a);   // a most recent
        (void)cache.render(node, sig, c);   // evicts b
        const unsigned before = node.calls;
        (void)cache.render(node, sig, a);
        (void)cache.render(node, sig, c);
        const bool kept = node.calls == before;
        (void)cache.render(node, sig, b);
        check(kept && node.calls == before + 1 && cache.stats().entries == 2, "cache_lru_eviction");
        (void)cache.render(node, sig, Rect{0, 0, 40, 40});
        (void)cache.render(node, sig, Rect{0, 0, 40, 40});
        check(node.calls == before + 3 && cache.stats().used_bytes <= 2 * (256 + 1200) + 100, "cache_oversized_uncached");
    }
    {   // CachedNode: a RAW source kept warm across recipe edits
        auto cache = std::make_shared<TileCache>(std::size_t(256) << 20);
        for (int menon = 0; menon <= 1; ++menon) {
            auto src = std::make_shared<RawUnpackNode>(
                raw, menon ? RawDemosaicIdentity{"rawengine.menon_base", 1} : RawDemosaicIdentity{});
            std::array<std::uint8_t, 32> s2 = sig;
            s2[2] = (std::uint8_t)menon;
            auto cached = std::make_shared<CachedNode>(src, cache, s2);
            const auto cam = camera(P, WorkingSpace::LinearProPhotoD50);
            bool same = true;
            for (float gain : {1.7f, 2.1f}) {
                auto chain_of = [&](std::shared_ptr<const Node> in) {
                    std::shared_ptr<const Node> n = std::make_shared<WhiteBalanceNode>(in, gain, 1.0f, 1.4f);
                    n = std::make_shared<CameraToWorkingNode>(n, cam, area);
                    n = std::make_shared<WorkingToSrgbNode>(n);
                    return std::make_shared<SrgbEncodeNode>(std::make_shared<ToneCurveNode>(n, 0.3f, 2.0f));
                };
                auto plain = chain_of(src), warm = chain_of(cached);
                Renderer renderer;
                const Rect vp{area.x + 3, area.y + 5, 70, 50};
                same &= bit_equal(renderer.render_image(*plain, area, RenderRequest{vp, 4096}).rgb,
                                  renderer.render_image(*warm, area, RenderRequest{vp, 4096}).rgb);
                const RenderRequest m1{{0, 0, 40, 30}, 4096, {1, RenderQuality::Preview}};
                same &= bit_equal(renderer.render_image(*plain, area, m1).rgb, renderer.render_image(*warm, area, m1).rgb);
            }
            check(same, std::string("cached_node_equals_direct_") + (menon ? "menon" : "bilinear"));
        }
        const auto st = cache->stats();
        check(st.hits == 4 && st.misses == 4, "cached_node_reused_across_edits");
    }
}

int run_render(const std::string& dir) {
    const auto P = read_params(dir + "/params.txt");
    const RawImage raw = make_raw(P, dir);
    const Rect area = raw.metadata().active_area;
    Renderer renderer;

    // 1. ImageGraph legacy bounded output, bilinear, whole active area.
    GraphRecipe legacy;
    {
        const auto& g = P.at("legacy");
        legacy.red_gain = (float)g[0];
        legacy.green_gain = (float)g[1];
        legacy.blue_gain = (float)g[2];
        legacy.exposure_stops = (float)g[3];
        legacy.tone_shoulder = (float)g[4];
        legacy.tone_gamma = (float)g[5];
    }
    ImageGraph graph(raw, legacy);
    check(graph.output().output_descriptor() == ImageDescriptor::bounded_output(), "legacy_descriptor");
    const Tile full = renderer.render_image(graph, area, 16);
    check(full.descriptor == ImageDescriptor::bounded_output(), "legacy_tile_descriptor");
    emit(dir, "legacy", full.bounds, full.rgb, "f32");

    // 2. render_tiles in row-major order, tiles bit-equal to the whole render.
    {
        const Rect vp{area.x + 3, area.y + 2, area.width - 5, area.height - 4};
        std::vector<Rect> order;
        bool same = true;
        renderer.render_tiles(graph, vp, [&](const Tile& t) {
            order.push_back(t.bounds);
            for (uint32_t row = 0; row < t.bounds.height; ++row)
                same &= std::memcmp(t.rgb.data() + (size_t)row * t.bounds.width * 3,
                                    full.rgb.data() + ((size_t)(t.bounds.y - area.y + row) * area.width +
                                                       (t.bounds.x - area.x)) * 3,
                                    (size_t)t.bounds.width * 3 * sizeof(float)) == 0;
        }, 7);
        bool row_major = !order.empty() && order.front().x == vp.x && order.front().y == vp.y;
        for (size_t i = 1; i < order.size(); ++i)
            row_major &= order[i].y > order[i - 1].y || (order[i].y == order[i - 1].y && order[i].x > order[i - 1].x);
        check(same, "render_tiles_equal_whole");
        check(row_major, "render_tiles_row_major");
        const auto roi = renderer.render_roi(graph, vp, 5);
        const Tile img = renderer.render_image(graph, vp, 1000);
        check(bit_equal(roi, img.rgb), "render_roi_equal_image");
    }

    // 3/4. Menon sRGB chain at mip 1 (Preview) and native.
    auto menon = std::make_shared<RawUnpackNode>(raw, RawDemosaicIdentity{"rawengine.menon_base", 1});
    const auto& s = P.at("srgb");
    auto wb = std::make_shared<WhiteBalanceNode>(menon, (float)s[0], (float)s[1], (float)s[2]);
    auto ex = std::make_shared<ExposureNode>(wb, (float)s[3]);
    auto ctw = std::make_shared<CameraToWorkingNode>(ex, camera(P, WorkingSpace::LinearProPhotoD50), area);
    auto to_srgb = std::make_shared<WorkingToSrgbNode>(ctw);
    auto tone = std::make_shared<ToneCurveNode>(to_srgb, (float)s[4], (float)s[5]);
    auto enc = std::make_shared<SrgbEncodeNode>(tone);
    check(enc->supports_level({1, RenderQuality::Preview}), "srgb_supports_mip1");
    check(!enc->supports_level({1, RenderQuality::Final}), "srgb_rejects_mip1_final");
    {
        const Rect reduced{0, 0, (area.width + 1) / 2, (area.height + 1) / 2};
        const Tile t = renderer.render_image(*enc, area, RenderRequest{reduced, 9, {1, RenderQuality::Preview}});
        check(t.descriptor == ImageDescriptor::srgb_output(), "srgb_descriptor");
        emit(dir, "srgb_mip1", t.bounds, t.rgb, "f32");
        const Rect vp = rect_of(P.at("srgb_native_vp"));
        const Tile n = renderer.render_image(*enc, area, vp, 64);
        emit(dir, "srgb_native", n.bounds, n.rgb, "f32");
        // the node's own render equals the renderer's result
        check(bit_equal(enc->render(vp).rgb, n.rgb), "node_render_equal_renderer");
    }

    // 5. Guided filter over a working-space chain, then extended curves.
    {
        const auto& gp = P.at("gf");
        auto ctw2 = std::make_shared<CameraToWorkingNode>(wb, camera(P, WorkingSpace::LinearProPhotoD50), area);
        auto gf = std::make_shared<WorkingYGuidedFilterNode>(
            ctw2, area, WorkingYGuidedFilterSettings{(uint32_t)gp[0], gp[1]});
        ExtendedCurvesSettings cs;
        cs.interpolation = CurveInterpolation::ShapePreservingCubic;
        const auto& k = P.at("curve_master");
        cs.master.knots.clear();
        for (size_t i = 0; i + 1 < k.size(); i += 2) cs.master.knots.push_back({k[i], k[i + 1]});
        auto curves = std::make_shared<ExtendedCurvesNode>(gf, cs);
        const Rect vp = rect_of(P.at("gf_vp"));
        const Tile t = renderer.render_image(*curves, area, vp, 32);
        emit(dir, "gf_curves", t.bounds, t.rgb, "f32");
        // the guided filter alone, through working_y_guided_filter_rgb on a host tile
        const Rect needed = working_y_guided_filter_region(vp, area, (uint32_t)gp[0]);
        const Tile in = ctw2->render(needed);
        const Tile host = working_y_guided_filter_rgb(in, vp, area, {(uint32_t)gp[0], gp[1]});
        const Tile node = gf->render(vp);
        check(bit_equal(host.rgb, node.rgb), "gf_function_equal_node");
        emit(dir, "gf_only", node.bounds, node.rgb, "f32");
        // local statistics of the working image, tile by tile
        const Rect lvp = rect_of(P.at("ls_vp"));
        const uint32_t radius = (uint32_t)P.at("ls_radius")[0];
        std::vector<double> mean((size_t)lvp.width * lvp.height * 3), var(mean.size());
        std::vector<uint32_t> count(mean.size());
        analyze_local_rgb(*ctw2, area, RenderRequest{lvp, 11, {}}, [&](const LocalStatisticsTile& t) {
            for (uint32_t row = 0; row < t.bounds.height; ++row)
                for (uint32_t col = 0; col < t.bounds.width * 3; ++col) {
                    const size_t d = (size_t)(t.bounds.y - lvp.y + row) * lvp.width * 3 + (t.bounds.x - lvp.x) * 3 + col;
                    const size_t s2 = (size_t)row * t.bounds.width * 3 + col;
                    mean[d] = t.mean[s2];
                    var[d] = t.variance[s2];
                    count[d] = t.finite_count[s2];
                }
        }, radius);
        emit(dir, "ls_mean", lvp, mean, "f64");
        emit(dir, "ls_var", lvp, var, "f64");
        emit(dir, "ls_count", lvp, count, "u32");
    }

    // 6/7. Cubic resize and rotation of a Rec.2020 working image.
    {
        auto bil_wb = std::make_shared<WhiteBalanceNode>(std::make_shared<RawUnpackNode>(raw), (float)s[0],
                                                         (float)s[1], (float)s[2]);
        auto rec = std::make_shared<CameraToWorkingNode>(bil_wb, camera(P, WorkingSpace::LinearRec2020D65), area);
        const auto& cp = P.at("cubic");
        auto cubic = std::make_shared<CubicResizeNode>(rec, area, CubicResizeSettings{(uint32_t)cp[0], (uint32_t)cp[1]});
        const Rect cvp = rect_of(P.at("cubic_vp"));
        const Tile c = renderer.render_image(*cubic, cubic->output_bounds(), cvp, 16);
        emit(dir, "cubic", c.bounds, c.rgb, "f32");
        const Rect cvp1 = rect_of(P.at("cubic_vp_mip1"));
        const Tile c1 = renderer.render_image(*cubic, cubic->output_bounds(),
                                              RenderRequest{cvp1, 16, {1, RenderQuality::Preview}});
        emit(dir, "cubic_mip1", c1.bounds, c1.rgb, "f32");
        auto rot = std::make_shared<RotateNode>(rec, area, RotateSettings{P.at("rotate_angle")[0]});
        const Rect rvp = rect_of(P.at("rotate_vp"));
        const Tile r = renderer.render_image(*rot, rot->output_bounds(), rvp, 16);
        emit(dir, "rotate", r.bounds, r.rgb, "f32");
        const Rect rvp2 = rect_of(P.at("rotate_vp_mip2"));
        const Tile r2 = renderer.render_image(*rot, rot->output_bounds(),
                                              RenderRequest{rvp2, 16, {2, RenderQuality::Preview}});
        emit(dir, "rotate_mip2", r2.bounds, r2.rgb, "f32");
        const Tile rec_full = rec->render(area);
        emit(dir, "rec2020_native", rec_full.bounds, rec_full.rgb, "f32");
    }

    // 8. Raster graph, sRGB preview, mip 2 and native.
    {
        const auto& rm = P.at("raster_meta");
        RasterMetadata md;
        md.width = (uint32_t)rm[0];
        md.height = (uint32_t)rm[1];
        md.working_space = (WorkingSpace)(int)rm[2];
        RasterImage img(md, read_file<float>(dir + "/raster.f32"));
        GraphRecipe rr;
        rr.exposure_stops = (float)P.at("raster_recipe")[0];
        rr.tone_gamma = (float)P.at("raster_recipe")[1];
        rr.output_mode = OutputMode::SrgbPreview;
        ImageGraph rg(img, rr);
        const Rect red{0, 0, (md.width + 3) / 4, (md.height + 3) / 4};
        const Tile t = renderer.render_image(rg, RenderRequest{red, 8, {2, RenderQuality::Preview}});
        emit(dir, "raster_mip2", t.bounds, t.rgb, "f32");
        const Tile n = renderer.render_image(rg, Rect{0, 0, md.width, md.height}, 13);
        emit(dir, "raster_native", n.bounds, n.rgb, "f32");
        GraphRecipe bad;
        bad.red_gain = 2.0f;
        expect_throw<std::invalid_argument>([&] { ImageGraph x(img, bad); }, "raster_rejects_raw_controls");
    }

    // 9. Nodes of another library, uploaded into the device chain.
    {
        auto c = std::make_shared<ConstantCameraNode>(std::array<float, 3>{0.25f, 0.5f, 0.75f});
        auto g = std::make_shared<WhiteBalanceNode>(c, 2.0f, 1.0f, 0.5f);
        const Tile t = g->render({0, 0, 3, 2});
        bool ok = t.rgb.size() == 18;
        for (size_t i = 0; ok && i < t.rgb.size(); i += 3)
            ok = t.rgb[i] == 0.25f * 2.0f && t.rgb[i + 1] == 0.5f && t.rgb[i + 2] == 0.75f * 0.5f;
        check(ok, "foreign_node_uploaded");
        const Node& base = *c;
        check(!base.input_icc_identity() && base.source_fingerprint() && (*base.source_fingerprint())[0] == 0x5a &&
                  !WhiteBalanceNode(c, 1.0f, 1.0f, 1.0f).source_fingerprint(),
              "node_identity_hooks");
        auto w = std::make_shared<WhiteBalanceNode>(std::make_shared<WrongDescriptorNode>(), 1.0f, 1.0f, 1.0f);
        expect_throw<std::domain_error>([&] { w->render({0, 0, 2, 2}); }, "foreign_wrong_descriptor_domain_error");
    }

    // 10. Errors and cancellation.
    {
        expect_throw<std::out_of_range>([&] { renderer.render_image(graph, Rect{0, 0, area.width + area.x + 1, 1}); },
                                        "viewport_out_of_range");
        expect_throw<std::invalid_argument>(
            [&] { renderer.render_image(graph, RenderRequest{{0, 0, 2, 2}, 16, {1, RenderQuality::Preview}}); },
            "legacy_graph_rejects_mip1");
        expect_throw<std::out_of_range>([&] { (void)RawUnpackNode(raw).render({0, 0, 1, 1}); },
                                        "inactive_area_out_of_range");
        CancellationToken cancelled;
        cancelled.cancel();
        expect_throw<RenderCancelled>([&] { renderer.render_image(graph, area, 16, &cancelled); },
                                      "pre_cancelled_render");
        CancellationToken mid;
        int tiles = 0;
        expect_throw<RenderCancelled>([&] {
            renderer.render_tiles(graph, area, [&](const Tile&) {
                if (++tiles == 2) mid.cancel();
            }, 8, &mid);
        }, "cancel_between_tiles");
        check(tiles == 2, "cancel_stops_after_current_tile");
    }

    // 11. TileScheduler: priority order, FIFO, pending budget, supersession,
    // destruction.
    {
        const Rect b{0, 0, 4, 4};
        auto open = [](Gate& g) {
            {
                std::lock_guard<std::mutex> lock(g.m);
                g.open = true;
            }
            g.cv.notify_all();
        };
        auto wait_entered = [](Gate& g, int n) {
            std::unique_lock<std::mutex> lock(g.m);
            return g.cv.wait_for(lock, std::chrono::seconds(10), [&] { return g.entered >= n; });
        };
        auto node = [](Gate& g, int id) { return std::make_shared<GatedNode>(&g, id); };
        {
            Gate gate;
            TileScheduler sched(1, 2);
            auto busy = sched.submit(node(gate, 0), b, b, RenderPriority::Normal, 4);
            check(wait_entered(gate, 1), "scheduler_started");
            auto low = sched.submit(node(gate, 1), b, b, RenderPriority::Background, 4);
            auto high = sched.submit(node(gate, 2), b, b, RenderPriority::Interactive, 4);
            expect_throw<std::length_error>([&] { sched.submit(node(gate, 3), b, b, RenderPriority::Normal, 4); },
                                            "scheduler_pending_budget");
            open(gate);
            const Tile t0 = busy.get(), t2 = high.get(), t1 = low.get();
            check(t0.rgb[0] == 0.0f && t2.rgb[0] == 2.0f && t1.rgb[0] == 1.0f, "scheduler_results");
            check(gate.order == std::vector<int>({0, 2, 1}), "scheduler_priority_order");
        }
        {
            Gate gate;
            TileScheduler sched(1, 3);
            auto busy = sched.submit(node(gate, 10), b, b, RenderPriority::Interactive, 4);
            check(wait_entered(gate, 1), "scheduler_started_2");
            auto a = sched.submit(node(gate, 11), b, b, RenderPriority::Normal, 4);
            auto c = sched.submit(node(gate, 12), b, b, RenderPriority::Normal, 4);
            auto v1 = sched.submit_latest("view", node(gate, 13), b, b, RenderPriority::Normal, 4);
            // the budget counts the queued request this one replaces
            auto v2 = sched.submit_latest("view", node(gate, 14), b, b, RenderPriority::Normal, 4);
            open(gate);
            expect_throw<RenderCancelled>([&] { v1.get(); }, "superseded_queued_cancelled");
            (void)busy.get();
            (void)a.get();
            (void)c.get();
            check(v2.get().rgb[0] == 14.0f, "latest_request_renders");
            check(gate.order == std::vector<int>({10, 11, 12, 14}), "scheduler_fifo_within_priority");
        }
        {
            Gate gate;
            TileScheduler sched(1, 2);
            auto first = sched.submit_latest("run", node(gate, 20), b, b, RenderPriority::Interactive, 4);
            check(wait_entered(gate, 1), "scheduler_started_3");
            auto second = sched.submit_latest("run", node(gate, 21), b, b, RenderPriority::Interactive, 4);
            open(gate);
            expect_throw<RenderCancelled>([&] { first.get(); }, "superseded_running_cancelled");
            check(second.get().rgb[0] == 21.0f, "superseding_request_renders");
        }
        {
            Gate gate;
            auto sched = std::make_unique<TileScheduler>(1, 2);
            auto busy = sched->submit(node(gate, 30), b, b, RenderPriority::Normal, 4);
            check(wait_entered(gate, 1), "scheduler_started_4");
            auto queued = sched->submit(node(gate, 31), b, b, RenderPriority::Normal, 4);
            std::thread closer([&] { sched.reset(); });
            std::this_thread::sleep_for(std::chrono::milliseconds(300));
            open(gate);
            closer.join();
            expect_throw<RenderCancelled>([&] { queued.get(); }, "destruction_cancels_pending");
            check(busy.get().rgb[0] == 30.0f, "destruction_waits_for_running");
        }
        // device renders through the scheduler equal direct renders
        {
            TileScheduler sched(2, 8);
            auto out = graph.output_node();
            auto f1 = sched.submit(out, area, area, RenderPriority::Normal, 64);
            auto f2 = sched.submit(enc, area, RenderRequest{{0, 0, 8, 6}, 4, {1, RenderQuality::Preview}});
            check(bit_equal(f1.get().rgb, full.rgb), "scheduled_equals_direct");
            check(bit_equal(f2.get().rgb,
                            renderer.render_image(*enc, area, RenderRequest{{0, 0, 8, 6}, 4, {1, RenderQuality::Preview}})
                                .rgb),
                  "scheduled_mip1_equals_direct");
            expect_throw<std::invalid_argument>(
                [&] { sched.submit(out, area, Rect{0, 0, 1, 1}, RenderPriority::Normal, 0); },
                "scheduler_rejects_zero_tile");
        }
    }
    stencil_checks(dir, P, ctw, area);
    factory_checks(P, raw, area);
    cache_checks(raw, area, P);
    histogram_checks(graph.output_node(), area);
    return failures ? 1 : 0;
}

// ---------------------------------------------------------------- validate

void region(const std::string& name, Rect r) {
    std::cout << "REGION " << name << " " << r.x << " " << r.y << " " << r.width << " " << r.height << std::endl;
}

int run_validate() {
    RawMetadata md;
    md.width = 40;
    md.height = 30;
    md.active_area = {4, 2, 32, 26};
    const RawImage raw(md, std::vector<uint16_t>(40 * 30, 1000));
    auto bil = std::make_shared<RawUnpackNode>(raw);
    auto menon = std::make_shared<RawUnpackNode>(raw, RawDemosaicIdentity{"rawengine.menon_base", 1});
    const Rect area = md.active_area;

    // metadata and demosaic identity
    {
        RawMetadata bad = md;
        bad.row_stride_samples = 39;
        expect_throw<std::invalid_argument>([&] { (void)RawImage(bad, std::vector<uint16_t>(39 * 30)); },
                                            "stride_below_width");
        expect_throw<std::invalid_argument>([&] { (void)RawImage(md, std::vector<uint16_t>(10)); }, "sample_count");
        RawMetadata outside = md;
        outside.active_area = {30, 0, 20, 10};
        expect_throw<std::invalid_argument>([&] { (void)RawImage(outside, std::vector<uint16_t>(40 * 30)); },
                                            "active_area_outside");
        expect_throw<std::invalid_argument>(
            [&] { (void)RawUnpackNode(raw, RawDemosaicIdentity{"rawengine.menon_base", 2}); }, "menon_version_2");
        expect_throw<std::invalid_argument>([&] { (void)RawUnpackNode(raw, RawDemosaicIdentity{"ahd", 1}); },
                                            "unknown_demosaic");
        RawMetadata packed;
        packed.width = 6;
        packed.height = 4;
        const RawImage p(packed, std::vector<uint16_t>(24));
        check(p.metadata().row_stride_samples == 6 && p.metadata().active_area.width == 6 &&
                  p.metadata().active_area.height == 4,
              "metadata_normalized");
    }
    // regions (compared with the oracle on the pytest side)
    region("bilinear_input", bil->input_region({4, 2, 5, 5}, area));
    region("menon_input", menon->input_region({10, 9, 7, 6}, area));
    region("menon_input_edge", menon->input_region({33, 25, 3, 3}, area));
    expect_throw<std::invalid_argument>([&] { bil->input_region({4, 2, 5, 5}, {0, 0, 40, 30}); },
                                        "raw_region_bounds_differ");
    // point node validation and descriptors
    {
        expect_throw<std::invalid_argument>([&] { (void)WhiteBalanceNode(bil, 0.0f, 1.0f, 1.0f); }, "wb_zero_gain");
        expect_throw<std::invalid_argument>([&] { (void)WhiteBalanceNode(bil, 1.0f, 70000.0f, 1.0f); }, "wb_large_gain");
        expect_throw<std::invalid_argument>([&] { (void)ExposureNode(bil, 33.0f); }, "exposure_range");
        auto tone = std::make_shared<ToneCurveNode>(bil, 0.25f, 1.0f);
        check(tone->output_descriptor() == ImageDescriptor::tone_mapped(), "tone_on_camera_descriptor");
        expect_throw<std::invalid_argument>([&] { (void)ExposureNode(tone, 1.0f); }, "exposure_rejects_tone_mapped");
        expect_throw<std::invalid_argument>([&] { (void)ToneCurveNode(bil, 0.25f, 0.0f); }, "tone_zero_gamma");
        auto clip = std::make_shared<OutputClipNode>(tone);
        check(clip->output_descriptor() == ImageDescriptor::bounded_output(), "clip_descriptor");
        expect_throw<std::invalid_argument>([&] { (void)OutputClipNode(bil); }, "clip_requires_tone_mapped");
        expect_throw<std::invalid_argument>([&] { (void)SrgbEncodeNode(tone); }, "encode_requires_display_linear");
        CameraColorTransform singular{{1, 0, 0, 1, 0, 0, 0, 0, 1}, WorkingSpace::LinearProPhotoD50};
        expect_throw<std::invalid_argument>([&] { (void)CameraToWorkingNode(bil, singular); }, "singular_camera_matrix");
        CameraColorTransform id{{1, 0, 0, 0, 1, 0, 0, 0, 1}, WorkingSpace::LinearRec2020D65};
        auto ctw = std::make_shared<CameraToWorkingNode>(bil, id, area);
        check(ctw->output_descriptor() == ImageDescriptor::scene_linear(WorkingSpace::LinearRec2020D65),
              "ctw_descriptor");
        expect_throw<std::invalid_argument>([&] { (void)CameraToWorkingNode(ctw, id); }, "ctw_requires_camera_linear");
        expect_throw<std::invalid_argument>([&] { (void)CameraToWorkingNode(bil, id, Rect{1, 1, 0, 0}); },
                                            "ctw_bad_preview_bounds");
        region("ctw_mip1", ctw->input_region_level({3, 2, 6, 5}, area, {1, RenderQuality::Preview}));
        region("ctw_mip2_edge", ctw->input_region_level({6, 4, 2, 3}, area, {2, RenderQuality::Preview}));
        check(!bil->supports_level({1, RenderQuality::Preview}) && ctw->supports_level({1, RenderQuality::Preview}) &&
                  !ctw->supports_level({3, RenderQuality::Preview}) && !ctw->supports_level({1, RenderQuality::Final}),
              "ctw_levels");
        auto srgb = std::make_shared<WorkingToSrgbNode>(ctw);
        check(srgb->output_descriptor() == ImageDescriptor::linear_srgb(), "working_to_srgb_descriptor");
        auto dl = std::make_shared<ToneCurveNode>(srgb, 0.25f, 2.2f);
        check(dl->output_descriptor() == ImageDescriptor::display_linear_srgb(), "tone_on_srgb_descriptor");
        check(std::make_shared<SrgbEncodeNode>(dl)->output_descriptor() == ImageDescriptor::srgb_output(),
              "encode_descriptor");
        auto conv = std::make_shared<WorkingSpaceConvertNode>(ctw, WorkingSpace::LinearRec2020D65);
        check(conv->identity(), "convert_identity");
        expect_throw<std::invalid_argument>([&] { (void)WorkingSpaceConvertNode(bil, WorkingSpace::LinearProPhotoD50); },
                                            "convert_requires_scene_linear");
        // spatial and geometry regions
        region("gf_region", working_y_guided_filter_region({10, 8, 6, 5}, area, 3));
        region("gf_region_edge", working_y_guided_filter_region({4, 2, 3, 3}, area, 2));
        region("ls_region", local_statistics_region({10, 8, 6, 5}, area, 4));
        expect_throw<std::invalid_argument>([&] { local_statistics_region({10, 8, 6, 5}, area, 9); }, "ls_radius_9");
        expect_throw<std::out_of_range>([&] { local_statistics_region({0, 0, 6, 5}, area, 1); }, "ls_outside");
        expect_throw<std::invalid_argument>(
            [&] { (void)WorkingYGuidedFilterNode(ctw, area, WorkingYGuidedFilterSettings{9, 0.01}); }, "gf_radius_9");
        expect_throw<std::invalid_argument>(
            [&] { (void)WorkingYGuidedFilterNode(ctw, area, WorkingYGuidedFilterSettings{2, 0.0}); }, "gf_epsilon_0");
        expect_throw<std::invalid_argument>([&] { (void)WorkingYGuidedFilterNode(bil, area); }, "gf_requires_scene_linear");
        auto gf = std::make_shared<WorkingYGuidedFilterNode>(ctw, area, WorkingYGuidedFilterSettings{2, 0.01});
        region("gf_node_mip1", gf->input_region_level({2, 3, 4, 4}, Rect{0, 0, 16, 13}, {1, RenderQuality::Preview}));
        auto cubic = std::make_shared<CubicResizeNode>(ctw, area, CubicResizeSettings{20, 17});
        region("cubic_support", cubic->input_region({3, 4, 6, 5}, area));
        region("cubic_support_mip1", cubic->input_region_level({1, 2, 4, 3}, area, {1, RenderQuality::Preview}));
        expect_throw<std::invalid_argument>([&] { (void)CubicResizeNode(ctw, area, CubicResizeSettings{7, 17}); },
                                            "cubic_shrink_over_4");
        auto rot = std::make_shared<RotateNode>(ctw, area, RotateSettings{23.5});
        region("rotate_support", rot->input_region({5, 6, 7, 4}, area));
        region("rotate_support_mip2", rot->input_region_level({1, 1, 3, 2}, area, {2, RenderQuality::Preview}));
        expect_throw<std::invalid_argument>([&] { (void)RotateNode(ctw, area, RotateSettings{190}); }, "rotate_angle");
        expect_throw<std::out_of_range>([&] { rot->input_region({30, 0, 5, 5}, area); }, "rotate_outside");
    }
    // graphs
    {
        GraphRecipe icc;
        icc.output_mode = OutputMode::IccDisplay;
        expect_throw<std::invalid_argument>([&] { (void)ImageGraph(raw, icc); }, "icc_output_unavailable");
        GraphRecipe preview;
        preview.output_mode = OutputMode::SrgbPreview;
        preview.camera_color = CameraColorTransform{{0.6, 0.3, 0.1, 0.25, 0.7, 0.05, 0.02, 0.1, 0.8},
                                                    WorkingSpace::LinearProPhotoD50};
        ImageGraph g(raw, preview);
        check(g.output().output_descriptor() == ImageDescriptor::srgb_output() &&
                  g.output().supports_level({1, RenderQuality::Preview}) &&
                  g.output().supports_level({2, RenderQuality::Preview}),
              "preview_graph_levels");
        ImageGraph legacy(raw);
        check(!legacy.output().supports_level({1, RenderQuality::Preview}), "legacy_graph_native_only");
        expect_throw<std::logic_error>(
            [&] {
                ImageGraph r(std::make_shared<CameraToWorkingNode>(
                                 bil, CameraColorTransform{{1, 0, 0, 0, 1, 0, 0, 0, 1}, WorkingSpace::LinearProPhotoD50}),
                             area);
                (void)r.image();
            },
            "node_graph_has_no_raw_image");
    }
    factory_validation(std::make_shared<CameraToWorkingNode>(
                           bil, CameraColorTransform{{1, 0, 0, 0, 1, 0, 0, 0, 1}, WorkingSpace::LinearProPhotoD50}, area),
                       area);
    // scheduler argument checks (no work is queued)
    {
        expect_throw<std::invalid_argument>([&] { (void)TileScheduler(0, 4); }, "scheduler_zero_workers");
        expect_throw<std::invalid_argument>([&] { (void)TileScheduler(65, 4); }, "scheduler_65_workers");
        expect_throw<std::invalid_argument>([&] { (void)TileScheduler(1, 0); }, "scheduler_zero_budget");
        TileScheduler sched(1, 1);
        expect_throw<std::invalid_argument>([&] { sched.submit(bil, area, Rect{0, 0, 2, 2}); },
                                            "scheduler_viewport_outside");
        expect_throw<std::invalid_argument>([&] { sched.submit(nullptr, area, area); }, "scheduler_null_node");
        expect_throw<std::invalid_argument>([&] { sched.submit_latest("", bil, area, area); },
                                            "scheduler_empty_group");
        expect_throw<std::invalid_argument>(
            [&] { sched.submit(bil, area, RenderRequest{{0, 0, 2, 2}, 16, {1, RenderQuality::Preview}}); },
            "scheduler_unsupported_level");
    }
    return failures ? 1 : 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::cerr << "usage: api_driver validate | render <dir>\n";
        return 2;
    }
    const std::string mode = argv[1];
    try {
        if (mode == "render" && argc == 3) return run_render(argv[2]);
        if (mode == "validate") return run_validate();
    } catch (const std::exception& e) {
        std::cout << "FAIL uncaught " << e.what() << std::endl;
        return 1;
    }
    std::cerr << "unknown mode\n";
    return 2;
}
