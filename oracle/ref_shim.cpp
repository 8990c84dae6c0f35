// Test-infrastructure shim over the UNMODIFIED reference library (oracle/_ref).
//
// It is compiled by `make -C oracle ref` against the reference headers where
// they lie and linked with oracle/_ref/libRawEngine.so.  Only tests/, the
// smoke check and bench.py's CPU baseline load it, and only as the checker or
// as the timed CPU reference; the product never does.
//
// Every entry point builds a chain of the reference's own nodes from a flat
// op list and renders it through the reference's own public API
// (Renderer::render_image, TileScheduler::submit, local_statistics_rgb,
// working_y_guided_filter_rgb, Node::input_region_level), so results are the
// reference's results.  Exceptions become status codes with a message.
#include "RawEngine.hpp"
#include "SpatialOps.hpp"
#include "ToneOps.hpp"
#include "GeometryOps.hpp"
#include "TileScheduler.hpp"
#include "ImageAnalysis.hpp"

#include <cstdint>
#include <cstring>
#include <future>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

using namespace rawengine;

namespace {

enum Op : std::int32_t {
    OP_WB = 1, OP_EXPOSURE = 2, OP_CAMERA_TO_WORKING = 3, OP_WORKING_TO_SRGB = 4,
    OP_TONE = 5, OP_OUTPUT_CLIP = 6, OP_SRGB_ENCODE = 7, OP_DISPLAY_TAG = 8,
    OP_CURVES_EXT = 9, OP_GUIDED_FILTER = 10, OP_CUBIC_RESIZE = 11, OP_ROTATE = 12,
    OP_WORKING_SPACE_CONVERT = 13,
    OP_SHARPEN = 14,
    OP_CLARITY = 15,
    OP_TEXTURE = 16,
    OP_CONVOLUTION = 17,
};

// The reference's own tests retag linear sRGB as display-linear sRGB with an
// adapter node (tests/core_tests.cpp:88-103 builds such nodes) so that an
// explicit SrgbEncodeNode can follow a curve chain without the shoulder tone.
class DisplayTagNode final : public Node {
public:
    explicit DisplayTagNode(std::shared_ptr<const Node> input) : input_(std::move(input)) {
        if (input_->output_descriptor() != ImageDescriptor::linear_srgb())
            throw std::invalid_argument("display tag requires linear sRGB");
    }
    Tile render(Rect r) const override { return render_level(r, {}); }
    Tile render_level(Rect r, RenderLevel level) const override {
        auto tile = input_->render_level(r, level);
        tile.descriptor = output_descriptor();
        return tile;
    }
    bool supports_level(RenderLevel level) const noexcept override { return input_->supports_level(level); }
    Rect input_region_level(Rect output, Rect, RenderLevel) const override { return output; }
    const Node* input_node() const noexcept override { return input_.get(); }
    ImageDescriptor output_descriptor() const noexcept override {
        return ImageDescriptor::display_linear_srgb();
    }
private:
    std::shared_ptr<const Node> input_;
};

thread_local std::string last_error;

int fail(int code, const char* what) {
    last_error = what ? what : "";
    return code;
}

template <class F> int guarded(F&& body) {
    try {
        body();
        last_error.clear();
        return 0;
    } catch (const RenderCancelled& e) { return fail(6, e.what()); }
    catch (const std::invalid_argument& e) { return fail(1, e.what()); }
    catch (const std::out_of_range& e) { return fail(2, e.what()); }
    catch (const std::domain_error& e) { return fail(3, e.what()); }
    catch (const std::length_error& e) { return fail(4, e.what()); }
    catch (const std::overflow_error& e) { return fail(5, e.what()); }
    catch (const std::logic_error& e) { return fail(9, e.what()); }
    catch (const std::exception& e) { return fail(10, e.what()); }
}

RawMetadata metadata_from(const std::uint32_t* m, const std::uint16_t* levels) {
    RawMetadata meta;
    meta.width = m[0]; meta.height = m[1]; meta.row_stride_samples = m[2];
    meta.pattern = static_cast<BayerPattern>(m[3]);
    meta.cfa_phase_x = static_cast<std::uint8_t>(m[4]);
    meta.cfa_phase_y = static_cast<std::uint8_t>(m[5]);
    meta.active_area = {m[6], m[7], m[8], m[9]};
    for (int i = 0; i < 4; ++i) {
        meta.black_levels[i] = levels[i];
        meta.white_levels[i] = levels[4 + i];
    }
    return meta;
}

CurveKnots read_knots(const double*& p) {
    CurveKnots curve;
    const auto n = static_cast<std::size_t>(*p++);
    curve.knots.resize(n);
    for (auto& k : curve.knots) { k.x = *p++; k.y = *p++; }
    return curve;
}

// Appends the op list to `node`; `bounds` tracks the current source bounds the
// way ExecutableEditGraph passes them to its op factory (EditGraph.cpp:1655-1730).
std::shared_ptr<const Node> build_chain(std::shared_ptr<const Node> node, Rect& bounds,
                                        const std::int32_t* ops, int nops, const double* p,
                                        std::shared_ptr<const Node>* before_last = nullptr,
                                        Rect* bounds_before_last = nullptr) {
    for (int i = 0; i < nops; ++i) {
        if (before_last) *before_last = node;
        if (bounds_before_last) *bounds_before_last = bounds;
        switch (ops[i]) {
        case OP_WB:
            node = std::make_shared<WhiteBalanceNode>(node, float(p[0]), float(p[1]), float(p[2]));
            p += 3; break;
        case OP_EXPOSURE:
            node = std::make_shared<ExposureNode>(node, float(p[0])); p += 1; break;
        case OP_CAMERA_TO_WORKING: {
            CameraColorTransform t;
            for (int k = 0; k < 9; ++k) t.camera_to_xyz_d50[k] = p[k];
            t.target = static_cast<WorkingSpace>(int(p[9]));
            node = std::make_shared<CameraToWorkingNode>(node, t, bounds);
            p += 10; break;
        }
        case OP_WORKING_TO_SRGB: node = std::make_shared<WorkingToSrgbNode>(node); break;
        case OP_TONE:
            node = std::make_shared<ToneCurveNode>(node, float(p[0]), float(p[1])); p += 2; break;
        case OP_OUTPUT_CLIP: node = std::make_shared<OutputClipNode>(node); break;
        case OP_SRGB_ENCODE: node = std::make_shared<SrgbEncodeNode>(node); break;
        case OP_DISPLAY_TAG: node = std::make_shared<DisplayTagNode>(node); break;
        case OP_CURVES_EXT: {
            ExtendedCurvesSettings s;
            s.interpolation = p[0] != 0 ? CurveInterpolation::ShapePreservingCubic
                                        : CurveInterpolation::Linear;
            ++p;
            s.master = read_knots(p);
            for (auto& c : s.channels) c = read_knots(p);
            node = std::make_shared<ExtendedCurvesNode>(node, s);
            break;
        }
        case OP_GUIDED_FILTER: {
            WorkingYGuidedFilterSettings s;
            s.radius = static_cast<std::uint32_t>(p[0]); s.epsilon = p[1];
            node = std::make_shared<WorkingYGuidedFilterNode>(node, bounds, s);
            p += 2; break;
        }
        case OP_CUBIC_RESIZE: {
            CubicResizeSettings s{static_cast<std::uint32_t>(p[0]), static_cast<std::uint32_t>(p[1])};
            node = std::make_shared<CubicResizeNode>(node, bounds, s);
            bounds = {0, 0, s.width, s.height};
            p += 2; break;
        }
        case OP_ROTATE: {
            node = std::make_shared<RotateNode>(node, bounds, RotateSettings{p[0]});
            bounds = {0, 0, bounds.width, bounds.height};
            p += 1; break;
        }
        case OP_WORKING_SPACE_CONVERT:
            node = std::make_shared<WorkingSpaceConvertNode>(node, static_cast<WorkingSpace>(int(p[0])));
            p += 1; break;
        case OP_SHARPEN:
            node = std::make_shared<SharpenNode>(node, bounds, SharpenSettings{p[0], std::uint32_t(p[1])});
            p += 2; break;
        case OP_CLARITY:
            node = std::make_shared<ClarityNode>(node, bounds, ClaritySettings{p[0], std::uint32_t(p[1])});
            p += 2; break;
        case OP_TEXTURE:
            node = std::make_shared<TextureNode>(node, bounds, TextureSettings{p[0], std::uint32_t(p[1])});
            p += 2; break;
        case OP_CONVOLUTION: {
            ConvolutionKernel k;
            k.width = std::uint32_t(p[0]);
            k.height = std::uint32_t(p[1]);
            k.coefficients.assign(p + 2, p + 2 + std::size_t(k.width) * k.height);
            node = std::make_shared<ConvolutionNode>(node, bounds, k);
            p += 2 + std::size_t(k.width) * k.height; break;
        }
        default: throw std::invalid_argument("shim: unknown op");
        }
    }
    return node;
}

void copy_out(const Tile& tile, float* out) {
    if (!tile.rgb.empty()) std::memcpy(out, tile.rgb.data(), tile.rgb.size() * sizeof(float));
}

std::shared_ptr<const Node> raw_source(const std::uint32_t* meta, const std::uint16_t* levels,
                                       const std::uint16_t* samples, std::size_t count,
                                       int demosaic, Rect& bounds) {
    RawImage image(metadata_from(meta, levels), std::vector<std::uint16_t>(samples, samples + count));
    bounds = image.metadata().active_area;
    RawDemosaicIdentity id;
    if (demosaic == 1) id = {"rawengine.menon_base", 1};
    return std::make_shared<RawUnpackNode>(image, id);
}

} // namespace

extern "C" {

const char* refshim_last_error(void) { return last_error.c_str(); }

// Renders a RAW chain through Renderer::render_image (RawEngine.cpp:1426-1447).
// meta: width,height,stride,pattern,phase_x,phase_y,active x,y,w,h; levels: black[4],white[4].
// demosaic: 0 bilinear v1, 1 menon_base v1.  out receives viewport.w*h*3 floats.
// out_bounds (4 words) receives the final node's source bounds.
int refshim_render_raw(const std::uint32_t* meta, const std::uint16_t* levels,
                       const std::uint16_t* samples, std::size_t count, int demosaic,
                       const std::int32_t* ops, int nops, const double* params,
                       const std::uint32_t* viewport, std::uint32_t tile_size,
                       std::uint32_t mip, std::uint32_t quality, float* out,
                       std::uint32_t* out_bounds) {
    return guarded([&] {
        Rect bounds;
        auto node = build_chain(raw_source(meta, levels, samples, count, demosaic, bounds),
                                bounds, ops, nops, params);
        if (out_bounds) { out_bounds[0] = bounds.x; out_bounds[1] = bounds.y; out_bounds[2] = bounds.width; out_bounds[3] = bounds.height; }
        if (!out) return;
        RenderRequest req{{viewport[0], viewport[1], viewport[2], viewport[3]}, tile_size,
                          {mip, static_cast<RenderQuality>(quality)}};
        copy_out(Renderer{}.render_image(*node, bounds, req), out);
    });
}

// Same chain, one TileScheduler request per render tile (TileScheduler.cpp:170-236),
// `workers` threads: the reference's own way to use every host core.
int refshim_render_raw_scheduled(const std::uint32_t* meta, const std::uint16_t* levels,
                                 const std::uint16_t* samples, std::size_t count, int demosaic,
                                 const std::int32_t* ops, int nops, const double* params,
                                 const std::uint32_t* viewport, std::uint32_t tile_size,
                                 std::uint32_t mip, std::uint32_t quality, float* out,
                                 std::uint32_t workers) {
    return guarded([&] {
        Rect bounds;
        auto node = build_chain(raw_source(meta, levels, samples, count, demosaic, bounds),
                                bounds, ops, nops, params);
        const Rect vp{viewport[0], viewport[1], viewport[2], viewport[3]};
        TileScheduler scheduler(workers, 1u << 20);
        std::vector<std::future<Tile>> futures;
        for (std::uint64_t y = vp.y; y < std::uint64_t(vp.y) + vp.height; y += tile_size)
            for (std::uint64_t x = vp.x; x < std::uint64_t(vp.x) + vp.width; x += tile_size) {
                const Rect r{std::uint32_t(x), std::uint32_t(y),
                             std::uint32_t(std::min<std::uint64_t>(tile_size, vp.x + std::uint64_t(vp.width) - x)),
                             std::uint32_t(std::min<std::uint64_t>(tile_size, vp.y + std::uint64_t(vp.height) - y))};
                futures.push_back(scheduler.submit(node, bounds,
                    RenderRequest{r, tile_size, {mip, static_cast<RenderQuality>(quality)}}));
            }
        for (auto& f : futures) {
            const auto t = f.get();
            for (std::uint32_t row = 0; row < t.bounds.height; ++row)
                std::memcpy(out + ((std::size_t(t.bounds.y - vp.y + row) * vp.width) + (t.bounds.x - vp.x)) * 3,
                            t.rgb.data() + std::size_t(row) * t.bounds.width * 3,
                            std::size_t(t.bounds.width) * 3 * sizeof(float));
        }
    });
}

// Raster (scene-linear float32 RGB) source chain (RawEngine.cpp:346-406).
int refshim_render_raster(std::uint32_t width, std::uint32_t height, std::uint32_t stride,
                          int space, const float* pixels, std::size_t count,
                          const std::int32_t* ops, int nops, const double* params,
                          const std::uint32_t* viewport, std::uint32_t tile_size,
                          std::uint32_t mip, std::uint32_t quality, float* out,
                          std::uint32_t* out_bounds) {
    return guarded([&] {
        RasterMetadata m{width, height, stride, static_cast<WorkingSpace>(space)};
        RasterImage image(m, std::vector<float>(pixels, pixels + count));
        Rect bounds{0, 0, width, height};
        auto node = build_chain(std::make_shared<RasterSourceNode>(image), bounds, ops, nops, params);
        if (out_bounds) { out_bounds[0] = bounds.x; out_bounds[1] = bounds.y; out_bounds[2] = bounds.width; out_bounds[3] = bounds.height; }
        if (!out) return;
        RenderRequest req{{viewport[0], viewport[1], viewport[2], viewport[3]}, tile_size,
                          {mip, static_cast<RenderQuality>(quality)}};
        copy_out(Renderer{}.render_image(*node, bounds, req), out);
    });
}

// histogram_rgb (ImageAnalysis.cpp:9-69) of a raster-source chain: counts
// (3 * bins), tallies (underflow[3], overflow[3], nonfinite[3]), extrema
// (min[3], max[3]) with present[6] flags.
int refshim_histogram_raster(std::uint32_t width, std::uint32_t height, int space, const float* pixels,
                             std::size_t count, const std::int32_t* ops, int nops, const double* params,
                             const std::uint32_t* viewport, std::uint32_t tile_size, std::uint32_t mip,
                             std::uint32_t quality, std::uint32_t bins, double lower, double upper,
                             std::uint64_t* counts, std::uint64_t* tallies, float* extrema,
                             std::uint8_t* present) {
    return guarded([&] {
        RasterMetadata m{width, height, 0, static_cast<WorkingSpace>(space)};
        RasterImage image(m, std::vector<float>(pixels, pixels + count));
        Rect bounds{0, 0, width, height};
        auto node = build_chain(std::make_shared<RasterSourceNode>(image), bounds, ops, nops, params);
        RenderRequest req{{viewport[0], viewport[1], viewport[2], viewport[3]}, tile_size,
                          {mip, static_cast<RenderQuality>(quality)}};
        const auto h = histogram_rgb(*node, bounds, req, HistogramOptions{bins, lower, upper});
        for (int c = 0; c < 3; ++c) {
            const auto& ch = h.channels[c];
            std::memcpy(counts + std::size_t(c) * bins, ch.counts.data(), bins * sizeof(std::uint64_t));
            tallies[c] = ch.underflow;
            tallies[3 + c] = ch.overflow;
            tallies[6 + c] = ch.nonfinite;
            present[c] = ch.minimum.has_value();
            present[3 + c] = ch.maximum.has_value();
            extrema[c] = ch.minimum.value_or(0.0f);
            extrema[3 + c] = ch.maximum.value_or(0.0f);
        }
    });
}

// Sharpen (kind 0: amount, radius), Clarity (1: amount, radius), Texture (2:
// amount, scale) or Convolution (3: width, height, coefficients...) over a
// raster source (SpatialOps.cpp:319-701), rendered through render_image.
int refshim_stencil_raster(int kind, std::uint32_t width, std::uint32_t height, int space, const float* pixels,
                           std::size_t count, const double* params, const std::uint32_t* viewport,
                           std::uint32_t tile_size, std::uint32_t mip, std::uint32_t quality, float* out) {
    return guarded([&] {
        RasterMetadata m{width, height, 0, static_cast<WorkingSpace>(space)};
        RasterImage image(m, std::vector<float>(pixels, pixels + count));
        const Rect bounds{0, 0, width, height};
        std::shared_ptr<const Node> src = std::make_shared<RasterSourceNode>(image), node;
        const auto u = [](double v) { return static_cast<std::uint32_t>(v); };
        switch (kind) {
        case 0: node = std::make_shared<SharpenNode>(src, bounds, SharpenSettings{params[0], u(params[1])}); break;
        case 1: node = std::make_shared<ClarityNode>(src, bounds, ClaritySettings{params[0], u(params[1])}); break;
        case 2: node = std::make_shared<TextureNode>(src, bounds, TextureSettings{params[0], u(params[1])}); break;
        case 3: {
            ConvolutionKernel k;
            k.width = u(params[0]);
            k.height = u(params[1]);
            k.coefficients.assign(params + 2, params + 2 + std::size_t(k.width) * k.height);
            node = std::make_shared<ConvolutionNode>(src, bounds, k);
            break;
        }
        default: throw std::invalid_argument("shim: unknown stencil");
        }
        RenderRequest req{{viewport[0], viewport[1], viewport[2], viewport[3]}, tile_size,
                          {mip, static_cast<RenderQuality>(quality)}};
        copy_out(Renderer{}.render_image(*node, bounds, req), out);
    });
}

// RawImage::fingerprint / RasterImage::fingerprint (SourceFingerprint.cpp:65-101).
int refshim_fingerprint_raw(const std::uint32_t* meta, const std::uint16_t* levels, const std::uint16_t* samples,
                            std::size_t count, std::uint8_t* digest) {
    return guarded([&] {
        RawImage image(metadata_from(meta, levels), std::vector<std::uint16_t>(samples, samples + count));
        const auto d = fingerprint_raw_source(image);
        std::memcpy(digest, d.data(), d.size());
    });
}
int refshim_fingerprint_raster(std::uint32_t width, std::uint32_t height, int space, const float* pixels,
                               std::size_t count, std::uint8_t* digest) {
    return guarded([&] {
        RasterImage image(RasterMetadata{width, height, 0, static_cast<WorkingSpace>(space)},
                          std::vector<float>(pixels, pixels + count));
        const auto d = fingerprint_raster_source(image);
        std::memcpy(digest, d.data(), d.size());
    });
}

// input_region_level of the LAST op (or of the RAW source when nops == 0):
// the reference's halo/support planner (RawEngine.cpp:290-297, SpatialOps.cpp:302-310,
// GeometryOps.cpp:112-118, 426-430).
int refshim_raw_input_region(const std::uint32_t* meta, const std::uint16_t* levels,
                             const std::uint16_t* samples, std::size_t count, int demosaic,
                             const std::int32_t* ops, int nops, const double* params,
                             const std::uint32_t* output, std::uint32_t mip, std::uint32_t quality,
                             std::uint32_t* region) {
    return guarded([&] {
        Rect bounds;
        auto source = raw_source(meta, levels, samples, count, demosaic, bounds);
        std::shared_ptr<const Node> before = source;
        Rect before_bounds = bounds;
        auto node = build_chain(source, bounds, ops, nops, params, &before, &before_bounds);
        const Rect o{output[0], output[1], output[2], output[3]};
        const Rect r = node->input_region_level(o, nops ? before_bounds : bounds,
                                                {mip, static_cast<RenderQuality>(quality)});
        region[0] = r.x; region[1] = r.y; region[2] = r.width; region[3] = r.height;
    });
}

// Raster-source variant of the planner query (GF / cubic / rotate supports).
int refshim_raster_input_region(std::uint32_t width, std::uint32_t height, int space,
                                const std::int32_t* ops, int nops, const double* params,
                                const std::uint32_t* output, std::uint32_t mip,
                                std::uint32_t quality, std::uint32_t* region) {
    return guarded([&] {
        RasterMetadata m{width, height, 0, static_cast<WorkingSpace>(space)};
        RasterImage image(m, std::vector<float>(std::size_t(width) * height * 3, 0.0f));
        Rect bounds{0, 0, width, height};
        std::shared_ptr<const Node> before;
        Rect before_bounds;
        auto node = build_chain(std::make_shared<RasterSourceNode>(image), bounds, ops, nops,
                                params, &before, &before_bounds);
        const Rect o{output[0], output[1], output[2], output[3]};
        const Rect r = node->input_region_level(o, before_bounds,
                                                {mip, static_cast<RenderQuality>(quality)});
        region[0] = r.x; region[1] = r.y; region[2] = r.width; region[3] = r.height;
    });
}

// local_statistics_rgb (SpatialOps.cpp:79-121) on a tile covering `needed`.
int refshim_local_statistics(const float* rgb, const std::uint32_t* needed,
                             const std::uint32_t* output, const std::uint32_t* image,
                             std::uint32_t radius, int space, double* mean, double* variance,
                             std::uint32_t* finite_count) {
    return guarded([&] {
        const Rect n{needed[0], needed[1], needed[2], needed[3]};
        Tile t{n, std::vector<float>(rgb, rgb + std::size_t(n.width) * n.height * 3),
               ImageDescriptor::scene_linear(static_cast<WorkingSpace>(space))};
        const auto r = local_statistics_rgb(t, {output[0], output[1], output[2], output[3]},
                                            {image[0], image[1], image[2], image[3]}, radius);
        std::memcpy(mean, r.mean.data(), r.mean.size() * sizeof(double));
        std::memcpy(variance, r.variance.data(), r.variance.size() * sizeof(double));
        std::memcpy(finite_count, r.finite_count.data(), r.finite_count.size() * sizeof(std::uint32_t));
    });
}

// working_y_guided_filter_rgb (SpatialOps.cpp:168-287) on a tile covering `needed`.
int refshim_guided_filter(const float* rgb, const std::uint32_t* needed,
                          const std::uint32_t* output, const std::uint32_t* image,
                          std::uint32_t radius, double epsilon, int space, float* out) {
    return guarded([&] {
        const Rect n{needed[0], needed[1], needed[2], needed[3]};
        Tile t{n, std::vector<float>(rgb, rgb + std::size_t(n.width) * n.height * 3),
               ImageDescriptor::scene_linear(static_cast<WorkingSpace>(space))};
        const auto r = working_y_guided_filter_rgb(t, {output[0], output[1], output[2], output[3]},
                                                   {image[0], image[1], image[2], image[3]},
                                                   WorkingYGuidedFilterSettings{radius, epsilon});
        copy_out(r, out);
    });
}

} // extern "C"

namespace {

// A reference render session for timing: the RawImage, the node chain and a
// TileScheduler with `workers` threads are built once by
// refshim_session_create; refshim_session_render then only submits one
// TileScheduler request per render tile of the viewport (the reference
// renderer's row-major cut, RawEngine.cpp:1399-1411), waits for them and
// copies each tile into `out` -- the work a caller of the reference repeats
// per frame.
struct RefSession {
    std::shared_ptr<const Node> node;
    Rect bounds;
    std::unique_ptr<TileScheduler> scheduler;
};

} // namespace

extern "C" {


void* refshim_session_create(const std::uint32_t* meta, const std::uint16_t* levels,
                             const std::uint16_t* samples, std::size_t count, int demosaic,
                             const std::int32_t* ops, int nops, const double* params,
                             std::uint32_t workers) {
    RefSession* out = nullptr;
    const int st = guarded([&] {
        auto s = std::make_unique<RefSession>();
        s->node = build_chain(raw_source(meta, levels, samples, count, demosaic, s->bounds), s->bounds, ops,
                              nops, params);
        s->scheduler = std::make_unique<TileScheduler>(workers, 1u << 20);
        out = s.release();
    });
    return st ? nullptr : out;
}

int refshim_session_render(void* session, const std::uint32_t* viewport, std::uint32_t tile_size,
                           std::uint32_t mip, std::uint32_t quality, float* out) {
    return guarded([&] {
        auto* s = static_cast<RefSession*>(session);
        const Rect vp{viewport[0], viewport[1], viewport[2], viewport[3]};
        std::vector<std::future<Tile>> futures;
        for (std::uint64_t y = vp.y; y < std::uint64_t(vp.y) + vp.height; y += tile_size)
            for (std::uint64_t x = vp.x; x < std::uint64_t(vp.x) + vp.width; x += tile_size) {
                const Rect r{std::uint32_t(x), std::uint32_t(y),
                             std::uint32_t(std::min<std::uint64_t>(tile_size, vp.x + std::uint64_t(vp.width) - x)),
                             std::uint32_t(std::min<std::uint64_t>(tile_size, vp.y + std::uint64_t(vp.height) - y))};
                futures.push_back(s->scheduler->submit(
                    s->node, s->bounds, RenderRequest{r, tile_size, {mip, static_cast<RenderQuality>(quality)}}));
            }
        for (auto& f : futures) {
            const auto t = f.get();
            for (std::uint32_t row = 0; row < t.bounds.height; ++row)
                std::memcpy(out + ((std::size_t(t.bounds.y - vp.y + row) * vp.width) + (t.bounds.x - vp.x)) * 3,
                            t.rgb.data() + std::size_t(row) * t.bounds.width * 3,
                            std::size_t(t.bounds.width) * 3 * sizeof(float));
        }
    });
}

void refshim_session_destroy(void* session) { delete static_cast<RefSession*>(session); }

} // extern "C"
