// TileScheduler over a mixed batch of render requests, through the drop-in
// C++ surface (include/rawengine/*.hpp).
//
//   scheduler_driver <spec.txt> [lanes]
//
// The spec lists RAW images, recipes and tile requests (written by the pytest
// side or bench.py from the mixed-batch workload: several RAW sizes, Bayer
// patterns and phases, bilinear and Menon sources, mip 0 Final and mip 1/2
// Preview, tiles of 128..1024 with edge remainders).  Each image's samples are
// synthesized here from its seed.  The driver renders every request
//   (1) once through Renderer::render_image, one request at a time (the
//       reference scheduler's unit of work: one render per request);
//   (2) through TileScheduler::submit (host tiles), all submitted at once;
//   (3) through TileScheduler::submit_device (device tiles);
// checks that (2) and (3) equal (1) bit for bit, and prints one JSON line
// with the wall times (steady clock, after one untimed warm-up pass of each).
//
// Spec lines:
//   image w h stride pattern phase_x phase_y ax ay aw ah b0 b1 b2 b3 white demosaic seed
//   recipe wb_r wb_g wb_b stops m0..m8 shoulder gamma nknots x0 y0 ... (nknots 0: tone chain)
//   tile image recipe x y w h mip quality geometry canvas_w canvas_h angle
// (geometry 1: a cubic resize to the canvas, 2: a rotation by angle degrees,
// between the camera-to-working stage and the rest of the recipe)
#include <rawengine/GeometryOps.hpp>
#include <rawengine/RawEngine.hpp>
#include <rawengine/TileScheduler.hpp>
#include <rawengine/ToneOps.hpp>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <future>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

using namespace rawengine;

namespace {

struct ImageSpec {
    RawMetadata meta;
    int demosaic = 0;
    uint64_t seed = 0;
};
struct RecipeSpec {
    float wb[3];
    float stops;
    std::array<double, 9> cam;
    float shoulder, gamma;
    std::vector<CurvePoint> knots;
};
struct TileSpec {
    int image, recipe;
    Rect viewport;
    RenderLevel level;
    int geometry = 0;
    uint32_t canvas_w = 0, canvas_h = 0;
    double angle = 0;
};

// Deterministic sensor samples: a smooth gradient, a few soft blobs and
// hash noise between the image's black and white levels.
std::vector<uint16_t> synthesize(const RawMetadata& m, uint64_t seed) {
    std::vector<uint16_t> s((size_t)m.row_stride_samples * m.height);
    const double span = (double)m.white_levels[0] - m.black_levels[0];
    for (uint32_t y = 0; y < m.height; ++y)
        for (uint32_t x = 0; x < m.row_stride_samples; ++x) {
            uint64_t h = seed * 0x9e3779b97f4a7c15ull ^ ((uint64_t)y << 32 | x);
            h ^= h >> 33;
            h *= 0xff51afd7ed558ccdull;
            h ^= h >> 33;
            const double gx = (double)x / m.width, gy = (double)y / m.height;
            double v = 0.08 + 0.5 * gx * (1.0 - 0.4 * gy);
            const double dx = gx - 0.3 - 0.1 * (seed % 5), dy = gy - 0.5;
            v += 0.4 * std::exp(-(dx * dx + dy * dy) * 30.0);
            v += 0.02 * ((double)(h & 0xffff) / 65535.0 - 0.5);
            if (((x / 37) + (y / 53)) % 7 == 0) v *= 0.3;
            const double code = m.black_levels[0] + v * span;
            s[(size_t)y * m.row_stride_samples + x] = (uint16_t)std::min(65535.0, std::max(0.0, code));
        }
    return s;
}

std::shared_ptr<const Node> chain(const std::shared_ptr<const Node>& src, const RecipeSpec& r, Rect bounds,
                                  const TileSpec& geo) {
    std::shared_ptr<const Node> n = std::make_shared<WhiteBalanceNode>(src, r.wb[0], r.wb[1], r.wb[2]);
    CameraColorTransform t;
    t.camera_to_xyz_d50 = r.cam;
    auto geometry = [&](std::shared_ptr<const Node> in) -> std::shared_ptr<const Node> {
        if (geo.geometry == 1)
            return std::make_shared<CubicResizeNode>(in, bounds, CubicResizeSettings{geo.canvas_w, geo.canvas_h});
        if (geo.geometry == 2) return std::make_shared<RotateNode>(in, bounds, RotateSettings{geo.angle});
        return in;
    };
    if (r.knots.empty()) {
        n = std::make_shared<ExposureNode>(n, r.stops);
        n = geometry(std::make_shared<CameraToWorkingNode>(n, t, bounds));
    } else {
        n = geometry(std::make_shared<CameraToWorkingNode>(n, t, bounds));
        n = std::make_shared<ExposureNode>(n, r.stops);
        ExtendedCurvesSettings cs;
        cs.master.knots = r.knots;
        cs.interpolation = CurveInterpolation::ShapePreservingCubic;
        n = std::make_shared<ExtendedCurvesNode>(n, cs);
    }
    n = std::make_shared<WorkingToSrgbNode>(n);
    n = std::make_shared<ToneCurveNode>(n, r.shoulder, r.gamma);
    return std::make_shared<SrgbEncodeNode>(n);
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::cerr << "usage: scheduler_driver <spec.txt> [lanes]\n";
        return 2;
    }
    const size_t lanes = argc > 2 ? (size_t)std::stoul(argv[2]) : 2;
    std::vector<ImageSpec> images;
    std::vector<RecipeSpec> recipes;
    std::vector<TileSpec> tiles;
    {
        std::ifstream in(argv[1]);
        std::string line;
        while (std::getline(in, line)) {
            std::istringstream ss(line);
            std::string kind;
            ss >> kind;
            if (kind == "image") {
                ImageSpec s;
                uint32_t pattern, px, py, b[4], white;
                ss >> s.meta.width >> s.meta.height >> s.meta.row_stride_samples >> pattern >> px >> py >>
                    s.meta.active_area.x >> s.meta.active_area.y >> s.meta.active_area.width >>
                    s.meta.active_area.height >> b[0] >> b[1] >> b[2] >> b[3] >> white >> s.demosaic >> s.seed;
                s.meta.pattern = (BayerPattern)pattern;
                s.meta.cfa_phase_x = (uint8_t)px;
                s.meta.cfa_phase_y = (uint8_t)py;
                for (int i = 0; i < 4; ++i) {
                    s.meta.black_levels[i] = (uint16_t)b[i];
                    s.meta.white_levels[i] = (uint16_t)white;
                }
                images.push_back(s);
            } else if (kind == "recipe") {
                RecipeSpec r;
                size_t n = 0;
                ss >> r.wb[0] >> r.wb[1] >> r.wb[2] >> r.stops;
                for (double& v : r.cam) ss >> v;
                ss >> r.shoulder >> r.gamma >> n;
                r.knots.resize(n);
                for (auto& k : r.knots) ss >> k.x >> k.y;
                recipes.push_back(r);
            } else if (kind == "tile") {
                TileSpec t;
                uint32_t mip, quality;
                ss >> t.image >> t.recipe >> t.viewport.x >> t.viewport.y >> t.viewport.width >> t.viewport.height >>
                    mip >> quality >> t.geometry >> t.canvas_w >> t.canvas_h >> t.angle;
                t.level = RenderLevel{mip, (RenderQuality)quality};
                tiles.push_back(t);
            }
        }
    }
    // nodes: one chain per (image, recipe) pair used
    std::vector<RawImage> raws;
    std::vector<std::shared_ptr<const Node>> sources;
    for (const ImageSpec& s : images) {
        raws.emplace_back(s.meta, synthesize(s.meta, s.seed));
        RawDemosaicIdentity id;
        if (s.demosaic) id = {"rawengine.menon_base", 1};
        sources.push_back(std::make_shared<RawUnpackNode>(raws.back(), id));
    }
    using ChainKey = std::tuple<int, int, int, uint32_t, uint32_t, double>;
    auto key_of = [](const TileSpec& t) {
        return ChainKey{t.image, t.recipe, t.geometry, t.canvas_w, t.canvas_h, t.angle};
    };
    std::map<ChainKey, std::shared_ptr<const Node>> chains;
    for (const TileSpec& t : tiles) {
        auto& c = chains[key_of(t)];
        if (!c) c = chain(sources[t.image], recipes[t.recipe], raws[t.image].metadata().active_area, t);
    }
    auto node_of = [&](const TileSpec& t) { return chains.at(key_of(t)); };
    auto bounds_of = [&](const TileSpec& t) {
        const Rect a = raws[t.image].metadata().active_area;
        if (t.geometry == 1) return Rect{0, 0, t.canvas_w, t.canvas_h};
        if (t.geometry == 2) return Rect{0, 0, a.width, a.height};
        return a;
    };
    uint64_t out_px = 0;
    for (const TileSpec& t : tiles) out_px += (uint64_t)t.viewport.width * t.viewport.height;

    Renderer renderer;
    auto direct_pass = [&](std::vector<Tile>* keep) {
        for (const TileSpec& t : tiles) {
            Tile r = renderer.render_image(*node_of(t), bounds_of(t), RenderRequest{t.viewport, 256, t.level});
            if (keep) keep->push_back(std::move(r));
        }
    };
    TileScheduler scheduler(lanes, tiles.size() + 16);
    auto host_pass = [&](std::vector<Tile>* keep) {
        std::vector<std::future<Tile>> f;
        f.reserve(tiles.size());
        for (const TileSpec& t : tiles)
            f.push_back(scheduler.submit(node_of(t), bounds_of(t), RenderRequest{t.viewport, 256, t.level}));
        for (auto& x : f) {
            Tile r = x.get();
            if (keep) keep->push_back(std::move(r));
        }
    };
    auto device_pass = [&](std::vector<DeviceTile>* keep) {
        std::vector<std::future<DeviceTile>> f;
        f.reserve(tiles.size());
        for (const TileSpec& t : tiles)
            f.push_back(scheduler.submit_device(node_of(t), bounds_of(t), RenderRequest{t.viewport, 256, t.level}));
        for (auto& x : f) {
            DeviceTile r = x.get();
            if (keep) keep->push_back(std::move(r));
        }
    };

    // reference results and bit-equality (this pass also warms every path up)
    std::vector<Tile> want, got_host;
    std::vector<DeviceTile> got_dev;
    direct_pass(&want);
    host_pass(&got_host);
    device_pass(&got_dev);
    size_t mismatches = 0;
    for (size_t i = 0; i < tiles.size(); ++i) {
        const Tile d = got_dev[i].to_host();
        const bool ok = want[i].rgb.size() == got_host[i].rgb.size() && want[i].rgb.size() == d.rgb.size() &&
                        std::memcmp(want[i].rgb.data(), got_host[i].rgb.data(), want[i].rgb.size() * 4) == 0 &&
                        std::memcmp(want[i].rgb.data(), d.rgb.data(), want[i].rgb.size() * 4) == 0 &&
                        want[i].descriptor == got_host[i].descriptor && want[i].descriptor == d.descriptor;
        mismatches += !ok;
    }
    want.clear();
    got_host.clear();
    got_dev.clear();
    const auto before = scheduler.stats();

    auto t0 = std::chrono::steady_clock::now();
    direct_pass(nullptr);
    const double direct_s = seconds_since(t0);
    t0 = std::chrono::steady_clock::now();
    host_pass(nullptr);
    const double host_s = seconds_since(t0);
    t0 = std::chrono::steady_clock::now();
    device_pass(nullptr);
    const double device_s = seconds_since(t0);
    const auto after = scheduler.stats();

    std::printf("{\"requests\": %zu, \"images\": %zu, \"lanes\": %zu, \"output_mpix\": %.3f, \"mismatches\": %zu, "
                "\"per_request_s\": %.5f, \"scheduler_host_s\": %.5f, \"scheduler_device_s\": %.5f, "
                "\"waves\": %llu, \"batched_requests\": %llu, \"node_requests\": %llu, \"unbatchable_requests\": %llu, \"batch_fallbacks\": %llu, "
                "\"last_fallback\": \"%s\", \"lane_lower_s\": %.4f, \"lane_plan_s\": %.4f, "
                "\"lane_device_s\": %.4f, \"lane_deliver_s\": %.4f}\n",
                tiles.size(), images.size(), lanes, out_px / 1e6, mismatches, direct_s, host_s, device_s,
                (unsigned long long)(after.waves - before.waves),
                (unsigned long long)(after.batched_requests - before.batched_requests),
                (unsigned long long)(after.node_requests - before.node_requests),
                (unsigned long long)(after.unbatchable_requests - before.unbatchable_requests),
                (unsigned long long)after.batch_fallbacks, after.last_fallback.c_str(), after.lower_s - before.lower_s,
                after.plan_s - before.plan_s, after.device_s - before.device_s, after.deliver_s - before.deliver_s);
    return mismatches ? 1 : 0;
}
