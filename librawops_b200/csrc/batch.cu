// Host side of the batched render (include/rawengine_b200.h, re_batch_*).
//
// A plan turns N render requests into one queue of CTA tiles: each request is
// validated exactly as re_render_raw_async validates it, its native region
// (the viewport, or the native footprint of a reduced request) is cut into the
// same even-anchored CTA tiles as the single-request kernels, and the tiles of
// all requests are laid end to end.  Reduced requests get a slice of one
// scratch arena for their native pixels and a second table of reduction
// blocks.  The images and programs of a launch group travel as kernel
// parameters; the tile records, the reduction tables and the mip scratch live in
// one device arena owned by the batch.  A launch is a memset of the queue heads
// and status word plus two kernel launches per group (one group unless the
// batch holds more than 24 distinct programs or 32 images, or both Menon
// policies, each of which has its own kernel), optionally
// replayed from a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "re_batch.cuh"
#include "re_geometry.cuh"

namespace re {
cudaError_t launch_demosaic(uint32_t demosaic, const DevRaw& raw, int ox, int oy, int ow, int oh,
                            int stage_end, const DevProgram& P, float* out, size_t out_stride,
                            uint32_t* status, unsigned long long* ties, cudaStream_t stream,
                            uint32_t* launches, uint8_t* dirs = nullptr);
cudaError_t launch_mip_reduce(const float* native, int nw, int nh, size_t native_stride, int mip,
                              int ow, int oh, int stage_begin, int stage_end, const DevProgram& P,
                              float* out, size_t out_stride, uint32_t* status, cudaStream_t stream,
                              uint32_t* launches);
cudaError_t launch_batch_group(const BatchParams& A, uint32_t grid, bool reduce, cudaStream_t stream);
int quad_layout(const DevRaw& raw);
void set_last_error(const std::string& msg);
re_status render_plan(const re_image* img, const re_render_desc* desc, re_rect viewport, uint32_t mip,
                      uint32_t quality, DevProgram& P, re_rect& native, const DevRaw** raw);
re_status status_key_to_error(uint32_t key);
re_status stage_program(const re_render_desc* desc, DevProgram& P);
}  // namespace re

using namespace re;

// Shape of a batch for the autotuner's cache: request count and tile count
// (log2 buckets), Menon and reduced shares (tenths), device.
using BatchShape = std::tuple<int, int, int, int, int>;

// One request as the single-request path launches it (the per-request form).
struct PerRequest {
    DevRaw raw;
    DevProgram program;
    uint32_t demosaic, mip;
    re_rect viewport, native;
    float* out;
    size_t out_stride;
    float* scratch;
};

struct LaunchGroup {
    BatchParams params;
    uint32_t grid;
};

// One geometry request as the per-request form launches it: its support was
// rendered by the RAW request listed with the others; then the geometry
// passes, then (reduce) the footprint average and the later stages.
struct GeoSingle {
    GeoRequest request;
    bool reduce;
    DevProgram post;
    uint32_t mip;
    re_rect viewport;
    float* out;
    size_t out_stride;
};

struct re_batch {
    BatchShape shape{};
    std::vector<re_batch_item> items;      // RAW requests, geometry supports included
    std::vector<re_batch_item> given;      // the caller's requests
    std::vector<PerRequest> singles;       // the requests as given
    std::vector<PerRequest> directs;       // the merged renders
    bool direct = false;                   // dispatch 3: plain launches of the merged renders
    std::vector<LaunchGroup> groups;
    re_batch_options opt{};
    re_batch_info info{};
    char* dev = nullptr;
    size_t cap = 0;
    uint32_t* head = nullptr;            // [status, queue of each group]
    uint32_t head_words = 0;
    uint32_t units = 0, runits = 0;
    cudaStream_t capture = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool planned = false;
    // geometry requests: tables and scratch in their own device block
    char* geo = nullptr;
    size_t geo_cap = 0;
    const GeoRequest* geo_requests = nullptr;
    const GeoBlock* geo_pass1 = nullptr;
    const GeoBlock* geo_pass2 = nullptr;
    uint32_t geo_n1 = 0, geo_n2 = 0;
    std::vector<LaunchGroup> geo_groups;   // footprint averages and later stages (reduce launches)
    std::vector<GeoSingle> geo_singles;
};

namespace {

re_status fail(re_status s, const std::string& msg) {
    set_last_error(msg);
    return s;
}

#define BT_CUDA(call)                                                                        \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) return fail(RE_CUDA_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

std::mutex g_tuned_mutex;
std::map<BatchShape, re_batch_options> g_tuned;

int log2_bucket(uint64_t v) {
    int b = 0;
    while (v > 1) {
        v >>= 1;
        ++b;
    }
    return b;
}

re_batch_options default_options() {
    re_batch_options o{};
    o.dispatch = 2;
    o.ctas_per_sm = 4;
    o.order = 1;
    o.use_graph = 1;
    return o;
}

void release_graph(re_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

// One plain launch sequence per render (demosaic, then the mip reduction).
re_status launch_singles(re_batch* b, const std::vector<PerRequest>& list, cudaStream_t stream) {
    uint32_t* status = b->head;
    if (!list.empty()) BT_CUDA(cudaMemsetAsync(b->head, 0, b->head_words * sizeof(uint32_t), stream));
    for (const PerRequest& q : list) {
        const DevProgram& P = q.program;
        if (!q.mip) {
            BT_CUDA(launch_demosaic(q.demosaic, q.raw, (int)q.viewport.x, (int)q.viewport.y, (int)q.viewport.width,
                                    (int)q.viewport.height, (int)P.count, P, q.out, q.out_stride, status, nullptr,
                                    stream, nullptr));
            continue;
        }
        const size_t nstride = (size_t)q.native.width * 3;
        BT_CUDA(launch_demosaic(q.demosaic, q.raw, (int)q.native.x, (int)q.native.y, (int)q.native.width,
                                (int)q.native.height, P.anchor + 1, P, q.scratch, nstride, status, nullptr, stream,
                                nullptr));
        BT_CUDA(launch_mip_reduce(q.scratch, (int)q.native.width, (int)q.native.height, nstride, (int)q.mip,
                                  (int)q.viewport.width, (int)q.viewport.height, P.anchor + 1, (int)P.count, P,
                                  q.out, q.out_stride, status, stream, nullptr));
    }
    return RE_OK;
}

// The geometry passes of every geometry request, then their footprint
// averages and later stages (after the RAW renders of their supports).
re_status enqueue_geometry(re_batch* b, cudaStream_t stream) {
    if (b->geo_n1 || b->geo_n2)
        BT_CUDA(launch_geometry_batch(b->geo_requests, b->geo_pass1, b->geo_n1, b->geo_pass2, b->geo_n2, b->head,
                                      stream));
    for (const LaunchGroup& g : b->geo_groups) BT_CUDA(launch_batch_group(g.params, 0, true, stream));
    return RE_OK;
}

re_status enqueue(re_batch* b, cudaStream_t stream) {
    if (b->direct) {
        re_status s = launch_singles(b, b->directs, stream);
        return s ? s : enqueue_geometry(b, stream);
    }
    BT_CUDA(cudaMemsetAsync(b->head, 0, b->head_words * sizeof(uint32_t), stream));
    for (const LaunchGroup& g : b->groups) BT_CUDA(launch_batch_group(g.params, g.grid, false, stream));
    re_status s = enqueue_geometry(b, stream);
    if (s) return s;
    for (const LaunchGroup& g : b->groups) BT_CUDA(launch_batch_group(g.params, 0, true, stream));
    return RE_OK;
}

// The per-request form of the geometry requests (after launch_singles).
re_status launch_geo_singles(re_batch* b, cudaStream_t stream) {
    for (const GeoSingle& q : b->geo_singles) {
        BT_CUDA(launch_geometry_single(q.request, b->head, stream));
        if (q.reduce)
            BT_CUDA(launch_mip_reduce(q.request.out, q.request.nw, q.request.nh, (size_t)q.request.out_stride,
                                      (int)q.mip, (int)q.viewport.width, (int)q.viewport.height, 0,
                                      (int)q.post.count, q.post, q.out, q.out_stride, b->head, stream, nullptr));
    }
    return RE_OK;
}

// Requests of one image, description, level and output row stride whose
// viewports tile a rectangle and whose outputs sit where one render of that
// rectangle would write them (the merged rows fit in the row stride) merge
// into that one render (results do not depend
// on how a viewport is cut, so the pixels are the same): first along rows,
// then along columns.
std::vector<re_batch_item> merge_items(std::vector<re_batch_item> v) {
    auto same = [](const re_batch_item& a, const re_batch_item& b) {
        return a.image == b.image && a.desc == b.desc && a.mip == b.mip && a.quality == b.quality &&
               a.out_row_stride == b.out_row_stride;
    };
    auto key = [](const re_batch_item& a) {
        return std::make_tuple((uintptr_t)a.image, (uintptr_t)a.desc, a.mip, a.quality, a.out_row_stride);
    };
    for (int pass = 0; pass < 2; ++pass) {
        const bool rows = pass == 0;
        std::sort(v.begin(), v.end(), [&](const re_batch_item& a, const re_batch_item& b) {
            const auto ka = key(a), kb = key(b);
            if (ka != kb) return ka < kb;
            if (rows) return std::make_tuple(a.viewport.y, a.viewport.height, a.viewport.x) <
                             std::make_tuple(b.viewport.y, b.viewport.height, b.viewport.x);
            return std::make_tuple(a.viewport.x, a.viewport.width, a.viewport.y) <
                   std::make_tuple(b.viewport.x, b.viewport.width, b.viewport.y);
        });
        std::vector<re_batch_item> out;
        for (const re_batch_item& it : v) {
            if (!out.empty()) {
                re_batch_item& a = out.back();
                const bool adjacent =
                    same(a, it) &&
                    (rows ? (a.viewport.y == it.viewport.y && a.viewport.height == it.viewport.height &&
                             (uint64_t)a.viewport.x + a.viewport.width == it.viewport.x &&
                             it.out == a.out + (size_t)a.viewport.width * 3 &&
                             ((size_t)a.viewport.width + it.viewport.width) * 3 <= a.out_row_stride)
                          : (a.viewport.x == it.viewport.x && a.viewport.width == it.viewport.width &&
                             (uint64_t)a.viewport.y + a.viewport.height == it.viewport.y &&
                             it.out == a.out + (size_t)a.viewport.height * a.out_row_stride));
                if (adjacent) {
                    if (rows) a.viewport.width += it.viewport.width;
                    else a.viewport.height += it.viewport.height;
                    continue;
                }
            }
            out.push_back(it);
        }
        v = std::move(out);
    }
    return v;
}

// Plans the geometry requests of a batch (GeometryOps.cpp:42-174, 346-513):
// each one's input support becomes a RAW request (appended to `supports`)
// rendered into the batch's geometry block, the geometry passes of all of
// them run as two launches over a block table, and the requests that reduce
// to mip 1/2 or have later stages get reduction tasks in their own launch
// groups.  Status pointers of those groups are set once the batch head exists.
re_status plan_geometry(re_batch* b, const std::vector<re_batch_item>& items, std::vector<re_batch_item>& supports,
                        re_batch_info& info) {
    struct G {
        size_t item;
        GeoPlan plan;
        re_rect area;
        DevProgram post;
        bool reduce;
        size_t o_axes, o_support, o_h, o_native;
    };
    std::vector<G> gs;
    b->geo_singles.clear();
    b->geo_groups.clear();
    b->geo_n1 = b->geo_n2 = 0;
    size_t tables = 0, data = 0;
    auto take = [](size_t& off, size_t bytes) {
        const size_t at = off;
        off = align256(off + bytes);
        return at;
    };
    for (size_t i = 0; i < items.size(); ++i) {
        const re_batch_item& it = items[i];
        if (!it.image || !it.desc) return fail(RE_INVALID_ARGUMENT, "null render arguments");
        if (it.geometry > 2) return fail(RE_INVALID_ARGUMENT, "unknown batch geometry");
        const bool native_level = it.mip == 0 && it.quality == 1;
        const bool reduced = (it.mip == 1 || it.mip == 2) && it.quality == 0;
        if (!native_level && !reduced) return fail(RE_INVALID_ARGUMENT, "node does not support this render level");
        re_raw_metadata meta{};
        re_status s = re_image_metadata(it.image, &meta);
        if (s) return s;
        G g{};
        g.item = i;
        g.area = meta.active_area;
        s = it.geometry == 1 ? plan_cubic(g.area.width, g.area.height, it.canvas_width, it.canvas_height, it.viewport,
                                          it.mip, g.plan)
                             : plan_rotate(g.area.width, g.area.height, it.angle_degrees, it.viewport, it.mip, g.plan,
                                           false);
        if (s) return s;
        DevProgram pre;
        if ((s = stage_program(it.desc, pre))) return s;
        std::memset(&g.post, 0, sizeof(g.post));
        g.post.anchor = -1;
        if (it.post && (s = stage_program(it.post, g.post))) return s;
        g.post.anchor = -1;
        if (!it.viewport.width || !it.viewport.height) continue;
        if (!it.out) return fail(RE_INVALID_ARGUMENT, "null render arguments");
        if (it.out_row_stride < (size_t)it.viewport.width * 3)
            return fail(RE_INVALID_ARGUMENT, "output row stride too small");
        g.reduce = it.mip != 0 || g.post.count != 0;
        const re_rect& sp = g.plan.support;
        g.o_axes = take(tables, (g.plan.xs.size() + g.plan.ys.size()) * sizeof(Axis));
        g.o_support = take(data, (size_t)sp.width * sp.height * 3 * sizeof(float));
        g.o_h = take(data, (size_t)g.plan.rows * g.plan.native.width * 3 * sizeof(double));
        g.o_native = take(data, g.reduce ? (size_t)g.plan.native.width * g.plan.native.height * 3 * sizeof(float) : 0);
        info.output_pixels += (uint64_t)it.viewport.width * it.viewport.height;
        info.reduced_requests += it.mip ? 1 : 0;
        gs.push_back(std::move(g));
    }
    info.geometry_requests = (uint32_t)gs.size();
    if (gs.empty()) return RE_OK;
    // block tables and reduction groups (host), then one device block:
    // [requests | pass 1 | pass 2 | groups' tasks | axes] [supports, H, natives]
    std::vector<GeoRequest> reqs(gs.size());
    std::vector<GeoBlock> pass1, pass2;
    struct RGroup {
        std::map<const re_render_desc*, int> programs;
        std::vector<DevProgram> program_list;
        std::vector<ReduceTask> tasks;
        std::vector<uint32_t> unit_task;
    };
    std::vector<RGroup> rgroups;
    for (size_t k = 0; k < gs.size(); ++k) {
        const G& g = gs[k];
        const re_batch_item& it = items[g.item];
        GeoRequest& R = reqs[k];
        R = GeoRequest{};
        R.kind = g.plan.kind;
        R.nx0 = (int)g.plan.native.x;
        R.ny0 = (int)g.plan.native.y;
        R.nw = (int)g.plan.native.width;
        R.nh = (int)g.plan.native.height;
        R.src_x0 = (int)g.plan.support.x;
        R.src_y0 = (int)g.plan.support.y;
        R.row0 = (int)g.plan.row0;
        R.rows = (int)g.plan.rows;
        R.rot = g.plan.rot;
        R.src_stride = (uint64_t)g.plan.support.width * 3;
        R.out_stride = g.reduce ? (uint64_t)R.nw * 3 : (uint64_t)it.out_row_stride;
        const uint32_t bx = (uint32_t)((R.nw + GEO_BW - 1) / GEO_BW);
        const uint32_t by1 = (uint32_t)(((R.kind == 1 ? R.rows : R.nh) + GEO_BH - 1) / GEO_BH);
        if (bx > 65535 || by1 > 65535 || (uint32_t)((R.nh + GEO_BH - 1) / GEO_BH) > 65535)
            return fail(RE_LENGTH_ERROR, "geometry request too large for one batch");
        for (uint32_t y = 0; y < by1; ++y)
            for (uint32_t x = 0; x < bx; ++x) pass1.push_back({(uint32_t)k, (uint16_t)x, (uint16_t)y});
        if (R.kind == 1)
            for (uint32_t y = 0; y < (uint32_t)((R.nh + GEO_BH - 1) / GEO_BH); ++y)
                for (uint32_t x = 0; x < bx; ++x) pass2.push_back({(uint32_t)k, (uint16_t)x, (uint16_t)y});
        if (g.reduce) {
            if (rgroups.empty() || (!rgroups.back().programs.count(it.post) &&
                                    rgroups.back().programs.size() == (size_t)BATCH_PROGRAMS))
                rgroups.emplace_back();
            RGroup& rg = rgroups.back();
            if (!rg.programs.count(it.post)) {
                rg.programs.emplace(it.post, (int)rg.program_list.size());
                rg.program_list.push_back(g.post);
            }
            ReduceTask q{};
            q.program = rg.programs.at(it.post);
            q.scale = 1 << it.mip;
            q.stage_begin = 0;
            q.stage_end = (int)g.post.count;
            q.nw = R.nw;
            q.nh = R.nh;
            q.ow = (int)it.viewport.width;
            q.oh = (int)it.viewport.height;
            q.tiles_x = (q.ow + RD_TW - 1) / RD_TW;
            q.unit_begin = (uint32_t)rg.unit_task.size();
            q.native_stride = (uint64_t)R.nw * 3;
            q.out = it.out;
            q.out_stride = it.out_row_stride;
            const uint32_t blocks = (uint32_t)q.tiles_x * (uint32_t)((q.oh + RD_TH - 1) / RD_TH);
            rg.unit_task.insert(rg.unit_task.end(), blocks, (uint32_t)rg.tasks.size());
            rg.tasks.push_back(q);   // native pointer filled below
        }
    }
    const size_t o_req = take(tables, reqs.size() * sizeof(GeoRequest));
    const size_t o_p1 = take(tables, pass1.size() * sizeof(GeoBlock));
    const size_t o_p2 = take(tables, pass2.size() * sizeof(GeoBlock));
    std::vector<std::pair<size_t, size_t>> o_rg(rgroups.size());
    for (size_t r = 0; r < rgroups.size(); ++r) {
        o_rg[r].first = take(tables, rgroups[r].tasks.size() * sizeof(ReduceTask));
        o_rg[r].second = take(tables, rgroups[r].unit_task.size() * sizeof(uint32_t));
    }
    const size_t total = tables + data;
    if (total > b->geo_cap) {
        release_graph(b);
        if (b->geo) BT_CUDA(cudaFree(b->geo));
        b->geo = nullptr;
        b->geo_cap = 0;
        BT_CUDA(cudaMalloc(&b->geo, total));
        b->geo_cap = total;
    }
    char* base = b->geo;
    char* dbase = base + tables;
    std::vector<char> host(tables);
    // fill device pointers, supports, reduction tasks
    size_t rgi = 0, rti = 0;
    for (size_t k = 0; k < gs.size(); ++k) {
        const G& g = gs[k];
        const re_batch_item& it = items[g.item];
        GeoRequest& R = reqs[k];
        R.src = reinterpret_cast<const float*>(dbase + g.o_support);
        if (R.kind == 1) {
            Axis* ax = reinterpret_cast<Axis*>(base + g.o_axes);
            R.ax = ax;
            R.ay = ax + g.plan.xs.size();
            std::memcpy(host.data() + g.o_axes, g.plan.xs.data(), g.plan.xs.size() * sizeof(Axis));
            std::memcpy(host.data() + g.o_axes + g.plan.xs.size() * sizeof(Axis), g.plan.ys.data(),
                        g.plan.ys.size() * sizeof(Axis));
            R.H = reinterpret_cast<double*>(dbase + g.o_h);
        }
        R.out = g.reduce ? reinterpret_cast<float*>(dbase + g.o_native) : it.out;
        re_batch_item sup{};
        sup.image = it.image;
        sup.desc = it.desc;
        sup.viewport = {g.area.x + g.plan.support.x, g.area.y + g.plan.support.y, g.plan.support.width,
                        g.plan.support.height};
        sup.mip = 0;
        sup.quality = 1;
        sup.out = reinterpret_cast<float*>(dbase + g.o_support);
        sup.out_row_stride = (size_t)g.plan.support.width * 3;
        supports.push_back(sup);
        GeoSingle q{};
        q.request = R;
        q.reduce = g.reduce;
        q.post = g.post;
        q.mip = it.mip;
        q.viewport = it.viewport;
        q.out = it.out;
        q.out_stride = it.out_row_stride;
        b->geo_singles.push_back(q);
        if (g.reduce) {
            while (rti == rgroups[rgi].tasks.size()) {
                ++rgi;
                rti = 0;
            }
            rgroups[rgi].tasks[rti++].native = R.out;
        }
    }
    std::memcpy(host.data() + o_req, reqs.data(), reqs.size() * sizeof(GeoRequest));
    std::memcpy(host.data() + o_p1, pass1.data(), pass1.size() * sizeof(GeoBlock));
    std::memcpy(host.data() + o_p2, pass2.data(), pass2.size() * sizeof(GeoBlock));
    for (size_t r = 0; r < rgroups.size(); ++r) {
        std::memcpy(host.data() + o_rg[r].first, rgroups[r].tasks.data(), rgroups[r].tasks.size() * sizeof(ReduceTask));
        std::memcpy(host.data() + o_rg[r].second, rgroups[r].unit_task.data(),
                    rgroups[r].unit_task.size() * sizeof(uint32_t));
        LaunchGroup lg{};
        BatchParams& A = lg.params;
        std::memset(&A, 0, sizeof(A));
        for (size_t i = 0; i < rgroups[r].program_list.size(); ++i) A.programs[i] = rgroups[r].program_list[i];
        A.rtasks = reinterpret_cast<const ReduceTask*>(base + o_rg[r].first);
        A.runit_task = reinterpret_cast<const uint32_t*>(base + o_rg[r].second);
        A.runits = (uint32_t)rgroups[r].unit_task.size();
        A.menon_policy = 1;
        b->geo_groups.push_back(lg);
    }
    BT_CUDA(cudaMemcpy(base, host.data(), tables, cudaMemcpyHostToDevice));
    b->geo_requests = reinterpret_cast<const GeoRequest*>(base + o_req);
    b->geo_pass1 = reinterpret_cast<const GeoBlock*>(base + o_p1);
    b->geo_pass2 = reinterpret_cast<const GeoBlock*>(base + o_p2);
    b->geo_n1 = (uint32_t)pass1.size();
    b->geo_n2 = (uint32_t)pass2.size();
    return RE_OK;
}

}  // namespace

extern "C" {

re_status re_batch_create(re_batch** out) {
    if (!out) return fail(RE_INVALID_ARGUMENT, "null batch handle");
    *out = new re_batch();
    return RE_OK;
}

re_status re_batch_destroy(re_batch* b) {
    if (!b) return RE_OK;
    release_graph(b);
    if (b->capture) cudaStreamDestroy(b->capture);
    if (b->dev) cudaFree(b->dev);
    if (b->geo) cudaFree(b->geo);
    delete b;
    return RE_OK;
}

re_status re_batch_plan(re_batch* b, const re_batch_item* items, size_t count, const re_batch_options* options) {
    if (!b || (count && !items)) return fail(RE_INVALID_ARGUMENT, "null batch arguments");
    if (count > (1u << 24)) return fail(RE_LENGTH_ERROR, "too many batch requests");
    b->planned = false;
    std::vector<re_batch_item> given(items, items + count), copy, geometry;
    for (const re_batch_item& it : given) (it.geometry ? geometry : copy).push_back(it);
    const size_t n_plain = copy.size();
    // 1. validate and describe every request
    struct Req {
        size_t item;
        const DevRaw* raw;
        const re_render_desc* desc;
        DevProgram program;
        re_rect native;
        int menon, layout, stage_end, mip;
        uint32_t tiles_x, tiles;
    };
    re_batch_info info{};
    // 0. geometry requests: their supports join the RAW requests
    {
        std::vector<re_batch_item> supports;
        re_status s = plan_geometry(b, geometry, supports, info);
        if (s) return s;
        copy.insert(copy.end(), supports.begin(), supports.end());
    }
    auto describe = [&](const re_batch_item& it, size_t index, Req& r) -> re_status {
        if (!it.image || !it.desc) return fail(RE_INVALID_ARGUMENT, "null render arguments");
        r = Req{};
        re_status s = render_plan(it.image, it.desc, it.viewport, it.mip, it.quality, r.program, r.native, &r.raw);
        if (s) return s;
        if (!it.viewport.width || !it.viewport.height) return RE_OK;
        if (!it.out) return fail(RE_INVALID_ARGUMENT, "null render arguments");
        if (it.out_row_stride < (size_t)it.viewport.width * 3)
            return fail(RE_INVALID_ARGUMENT, "output row stride too small");
        r.item = index;
        r.desc = it.desc;
        r.mip = (int)it.mip;
        r.menon = it.desc->demosaic >= 1 && r.raw->aw > 1 && r.raw->ah > 1 ? (int)it.desc->demosaic : 0;
        r.layout = quad_layout(*r.raw);
        r.stage_end = it.mip ? r.program.anchor + 1 : (int)r.program.count;
        const int tw = r.menon ? BATCH_MENON_TW : BATCH_BILINEAR_TW;
        const int th = r.menon ? BATCH_MENON_TH : BATCH_BILINEAR_TH;
        const int gx0 = (int)r.native.x & ~1, gy0 = (int)r.native.y & ~1;
        r.tiles_x = (uint32_t)(((int)(r.native.x + r.native.width) - gx0 + tw - 1) / tw);
        const uint32_t tiles_y = (uint32_t)(((int)(r.native.y + r.native.height) - gy0 + th - 1) / th);
        r.tiles = r.tiles_x * tiles_y;
        return RE_OK;
    };
    // the requests as given (validated; the per-request form renders these)
    std::vector<Req> orig;
    std::vector<re_batch_item> valid;
    for (size_t i = 0; i < copy.size(); ++i) {
        Req r;
        re_status s = describe(copy[i], i, r);
        if (s) return s;
        if (!copy[i].viewport.width || !copy[i].viewport.height) continue;
        orig.push_back(r);
        valid.push_back(copy[i]);
        info.native_pixels += (uint64_t)r.native.width * r.native.height;
        if (i < n_plain) {   // a support's pixels are intermediate, not output
            info.output_pixels += (uint64_t)copy[i].viewport.width * copy[i].viewport.height;
            info.reduced_requests += copy[i].mip ? 1 : 0;
            ++info.requests;
        }
    }
    info.requests += info.geometry_requests;
    // the renders the batch performs: adjacent requests merged
    const std::vector<re_batch_item> merged = merge_items(valid);
    std::vector<Req> reqs(merged.size());
    for (size_t i = 0; i < merged.size(); ++i) {
        re_status s = describe(merged[i], i, reqs[i]);
        if (s) return s;
    }
    info.tasks = (uint32_t)reqs.size();
    uint64_t tiles = 0, menon_tiles = 0;
    for (const Req& r : reqs) {
        tiles += r.tiles;
        menon_tiles += r.menon ? r.tiles : 0;
    }
    if (tiles >= (1ull << 31)) return fail(RE_LENGTH_ERROR, "batch tile queue exceeds 2^31 tiles");
    // 2. options: caller's, else the tuned choice for this shape, else defaults
    int device = 0;
    BT_CUDA(cudaGetDevice(&device));
    const BatchShape shape{(int)log2_bucket(reqs.size()), log2_bucket(tiles),
                           (int)(tiles ? 10 * menon_tiles / tiles : 0),
                           (int)(reqs.empty() ? 0 : 10 * info.reduced_requests / reqs.size()), device};
    re_batch_options opt = default_options();
    if (options) {
        opt = *options;
    } else {
        std::lock_guard<std::mutex> lock(g_tuned_mutex);
        auto t = g_tuned.find(shape);
        if (t != g_tuned.end()) opt = t->second;
    }
    if (opt.dispatch > 3 || opt.ctas_per_sm > 4 || opt.order > 1)
        return fail(RE_INVALID_ARGUMENT, "invalid batch options");
    if (!opt.ctas_per_sm) opt.ctas_per_sm = 4;
    // 3. queue order, then launch groups of at most BATCH_PROGRAMS programs and
    //    BATCH_IMAGES images (programs are shared by requests with one description)
    std::vector<size_t> order(reqs.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    if (opt.order == 1)
        std::stable_partition(order.begin(), order.end(), [&](size_t i) { return reqs[i].menon != 0; });
    struct GroupPlan {
        std::vector<size_t> reqs;
        std::map<const DevRaw*, int> images;
        std::map<const re_render_desc*, int> programs;
        int policy = 0;          // Menon policy of the group (0: bilinear requests only so far)
    };
    std::vector<GroupPlan> gplans(1);
    for (size_t k : order) {
        GroupPlan* g = &gplans.back();
        const bool new_image = !g->images.count(reqs[k].raw);
        const bool new_program = !g->programs.count(reqs[k].desc);
        const int policy = reqs[k].menon;
        if ((new_image && g->images.size() == BATCH_IMAGES) ||
            (new_program && g->programs.size() == BATCH_PROGRAMS) || (policy && g->policy && policy != g->policy)) {
            gplans.emplace_back();
            g = &gplans.back();
        }
        if (policy) g->policy = policy;
        if (!g->images.count(reqs[k].raw)) g->images.emplace(reqs[k].raw, (int)g->images.size());
        if (!g->programs.count(reqs[k].desc)) g->programs.emplace(reqs[k].desc, (int)g->programs.size());
        g->reqs.push_back(k);
    }
    if (gplans.back().reqs.empty()) gplans.pop_back();
    // 4. host tables of every group
    size_t scratch_bytes = 0;
    std::vector<size_t> scratch_off(reqs.size(), 0), orig_scratch_off(orig.size(), 0);
    for (size_t k = 0; k < reqs.size(); ++k)
        if (reqs[k].mip) {
            scratch_off[k] = scratch_bytes;
            scratch_bytes += align256((size_t)reqs[k].native.width * reqs[k].native.height * 3 * sizeof(float));
        }
    for (size_t k = 0; k < orig.size(); ++k)
        if (orig[k].mip) {
            orig_scratch_off[k] = scratch_bytes;
            scratch_bytes += align256((size_t)orig[k].native.width * orig[k].native.height * 3 * sizeof(float));
        }
    struct GroupTables {
        std::vector<BatchUnit> units;
        std::vector<size_t> unit_req;      // request of each unit (for scratch pointers)
        std::vector<ReduceTask> rtasks;
        std::vector<uint32_t> runit_task;
        std::vector<size_t> rtask_req;
    };
    std::vector<GroupTables> tabs(gplans.size());
    for (size_t gi = 0; gi < gplans.size(); ++gi) {
        GroupTables& T = tabs[gi];
        for (size_t k : gplans[gi].reqs) {
            const Req& r = reqs[k];
            const re_batch_item& it = merged[r.item];
            BatchUnit t{};
            t.image = gplans[gi].images.at(r.raw);
            t.program = gplans[gi].programs.at(r.desc);
            t.ox = (int)r.native.x;
            t.oy = (int)r.native.y;
            t.ow = (int)r.native.width;
            t.oh = (int)r.native.height;
            t.menon = r.menon;
            t.layout = r.layout;
            t.stage_end = r.stage_end;
            t.out = it.out;   // reduced requests: replaced by their scratch slice
            t.out_stride = it.mip ? (uint64_t)r.native.width * 3 : it.out_row_stride;
            const int tw = r.menon ? BATCH_MENON_TW : BATCH_BILINEAR_TW;
            const int th = r.menon ? BATCH_MENON_TH : BATCH_BILINEAR_TH;
            const int gx0 = t.ox & ~1, gy0 = t.oy & ~1;
            for (uint32_t u = 0; u < r.tiles; ++u) {
                t.x0 = gx0 + (int)(u % r.tiles_x) * tw;
                t.y0 = gy0 + (int)(u / r.tiles_x) * th;
                T.units.push_back(t);
                T.unit_req.push_back(k);
            }
            if (r.mip) {
                ReduceTask q{};
                q.program = t.program;
                q.scale = 1 << r.mip;
                q.stage_begin = r.program.anchor + 1;
                q.stage_end = (int)r.program.count;
                q.nw = (int)r.native.width;
                q.nh = (int)r.native.height;
                q.ow = (int)it.viewport.width;
                q.oh = (int)it.viewport.height;
                q.tiles_x = (q.ow + RD_TW - 1) / RD_TW;
                q.unit_begin = (uint32_t)T.runit_task.size();
                q.native_stride = (uint64_t)r.native.width * 3;
                q.out = it.out;
                q.out_stride = it.out_row_stride;
                const uint32_t blocks = (uint32_t)q.tiles_x * (uint32_t)((q.oh + RD_TH - 1) / RD_TH);
                T.runit_task.insert(T.runit_task.end(), blocks, (uint32_t)T.rtasks.size());
                T.rtasks.push_back(q);
                T.rtask_req.push_back(k);
            }
        }
    }
    // 5. one device arena: head | per group: tile records, reduce tasks, reduce map | scratch
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off = align256(off + bytes);
        return at;
    };
    const uint32_t head_words = 1 + (uint32_t)gplans.size();
    const size_t o_head = take(head_words * sizeof(uint32_t));
    struct GroupOffsets {
        size_t unit, rtask, runit;
    };
    std::vector<GroupOffsets> go(gplans.size());
    for (size_t gi = 0; gi < gplans.size(); ++gi) {
        go[gi].unit = take(tabs[gi].units.size() * sizeof(BatchUnit));
        go[gi].rtask = take(tabs[gi].rtasks.size() * sizeof(ReduceTask));
        go[gi].runit = take(tabs[gi].runit_task.size() * sizeof(uint32_t));
    }
    const size_t o_scratch = take(scratch_bytes);
    if (off > b->cap) {
        release_graph(b);
        if (b->dev) BT_CUDA(cudaFree(b->dev));
        b->dev = nullptr;
        b->cap = 0;
        BT_CUDA(cudaMalloc(&b->dev, off));
        b->cap = off;
    }
    char* base = b->dev;
    auto scratch_of = [&](size_t k) { return reinterpret_cast<float*>(base + o_scratch + scratch_off[k]); };
    auto orig_scratch_of = [&](size_t k) { return reinterpret_cast<float*>(base + o_scratch + orig_scratch_off[k]); };
    auto put = [&](size_t at, const void* src, size_t bytes) -> cudaError_t {
        return bytes ? cudaMemcpy(base + at, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
    };
    int sms = 0;
    BT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    b->head = reinterpret_cast<uint32_t*>(base + o_head);
    b->head_words = head_words;
    std::vector<LaunchGroup> groups(gplans.size());
    uint32_t grid_total = 0;
    for (size_t gi = 0; gi < gplans.size(); ++gi) {
        GroupTables& T = tabs[gi];
        for (size_t t = 0; t < T.units.size(); ++t)
            if (reqs[T.unit_req[t]].mip) T.units[t].out = scratch_of(T.unit_req[t]);
        for (size_t t = 0; t < T.rtasks.size(); ++t) T.rtasks[t].native = scratch_of(T.rtask_req[t]);
        BT_CUDA(put(go[gi].unit, T.units.data(), T.units.size() * sizeof(BatchUnit)));
        BT_CUDA(put(go[gi].rtask, T.rtasks.data(), T.rtasks.size() * sizeof(ReduceTask)));
        BT_CUDA(put(go[gi].runit, T.runit_task.data(), T.runit_task.size() * sizeof(uint32_t)));
        BatchParams& A = groups[gi].params;
        std::memset(&A, 0, sizeof(A));
        for (const auto& [raw, idx] : gplans[gi].images) A.images[idx] = *raw;
        for (size_t k : gplans[gi].reqs) A.programs[gplans[gi].programs.at(reqs[k].desc)] = reqs[k].program;
        A.units_rec = reinterpret_cast<const BatchUnit*>(base + go[gi].unit);
        A.rtasks = reinterpret_cast<const ReduceTask*>(base + go[gi].rtask);
        A.runit_task = reinterpret_cast<const uint32_t*>(base + go[gi].runit);
        A.units = (uint32_t)T.units.size();
        A.runits = (uint32_t)T.runit_task.size();
        A.dispatch = opt.dispatch;
        A.menon_policy = gplans[gi].policy ? (uint32_t)gplans[gi].policy : 1u;
        A.status = b->head;
        A.queue = b->head + 1 + gi;
        groups[gi].grid = A.dispatch != 1 ? (uint32_t)std::min<uint64_t>(A.units, (uint64_t)sms * opt.ctas_per_sm)
                                          : A.units;
        grid_total += groups[gi].grid;
    }
    b->groups = std::move(groups);
    for (LaunchGroup& g : b->geo_groups) {
        g.params.status = b->head;
        g.params.queue = b->head;
        g.params.dispatch = opt.dispatch;
    }
    b->units = (uint32_t)tiles;
    b->runits = 0;
    for (const GroupTables& T : tabs) b->runits += (uint32_t)T.runit_task.size();
    for (const LaunchGroup& g : b->geo_groups) b->runits += g.params.runits;
    b->items = std::move(copy);
    b->given = std::move(given);
    b->opt = opt;
    info.tiles = b->units;
    info.reduce_blocks = b->runits;
    info.grid = grid_total;
    info.raw_bytes = 2 * info.native_pixels;
    info.output_bytes = 12 * info.output_pixels;
    info.options = opt;
    b->info = info;
    b->shape = shape;
    // 7. the requests as single-request launches (re_batch_launch_per_request),
    //    and the merged renders as plain launches (dispatch 3)
    auto single = [&](const Req& r, const re_batch_item& it, float* scratch) {
        PerRequest q{};
        q.raw = *r.raw;
        q.program = r.program;
        q.demosaic = it.desc->demosaic;
        q.mip = it.mip;
        q.viewport = it.viewport;
        q.native = r.native;
        q.out = it.out;
        q.out_stride = it.out_row_stride;
        q.scratch = scratch;
        return q;
    };
    b->singles.clear();
    for (size_t k = 0; k < orig.size(); ++k)
        b->singles.push_back(single(orig[k], b->items[orig[k].item], orig[k].mip ? orig_scratch_of(k) : nullptr));
    b->directs.clear();
    for (size_t k = 0; k < reqs.size(); ++k)
        b->directs.push_back(single(reqs[k], merged[reqs[k].item], reqs[k].mip ? scratch_of(k) : nullptr));
    b->direct = opt.dispatch == 3;
    // 6. CUDA graph of the launch sequence
    release_graph(b);
    if (opt.use_graph && !b->groups.empty()) {
        if (!b->capture) BT_CUDA(cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking));
        BT_CUDA(cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal));
        re_status s = enqueue(b, b->capture);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->capture, &g);
        if (s) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        BT_CUDA(e);
        b->graph = g;
        BT_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
    }
    b->planned = true;
    return RE_OK;
}

re_status re_batch_launch_per_request(re_batch* b, void* stream_) {
    if (!b || !b->planned) return fail(RE_INVALID_ARGUMENT, "batch is not planned");
    re_status s = launch_singles(b, b->singles, (cudaStream_t)stream_);
    return s ? s : launch_geo_singles(b, (cudaStream_t)stream_);
}

re_status re_batch_launch(re_batch* b, void* stream_) {
    if (!b || !b->planned) return fail(RE_INVALID_ARGUMENT, "batch is not planned");
    cudaStream_t stream = (cudaStream_t)stream_;
    if (b->groups.empty()) return RE_OK;
    if (b->exec) {
        BT_CUDA(cudaGraphLaunch(b->exec, stream));
        return RE_OK;
    }
    return enqueue(b, stream);
}

re_status re_batch_status(re_batch* b, void* stream_) {
    if (!b || !b->planned) return fail(RE_INVALID_ARGUMENT, "batch is not planned");
    if (b->groups.empty()) return RE_OK;
    BT_CUDA(cudaStreamSynchronize((cudaStream_t)stream_));
    uint32_t word = 0;
    BT_CUDA(cudaMemcpy(&word, b->head, sizeof(word), cudaMemcpyDeviceToHost));
    return status_key_to_error(word);
}

re_status re_batch_info_get(const re_batch* b, re_batch_info* info) {
    if (!b || !info) return fail(RE_INVALID_ARGUMENT, "null batch arguments");
    *info = b->info;
    return RE_OK;
}

re_status re_batch_autotune(re_batch* b, uint32_t reps, void* stream_, re_batch_options* best) {
    if (!b || !b->planned) return fail(RE_INVALID_ARGUMENT, "batch is not planned");
    if (!reps) reps = 5;
    cudaStream_t stream = (cudaStream_t)stream_;
    const std::vector<re_batch_item> items = b->given;
    const uint32_t graph = b->opt.use_graph;
    std::vector<re_batch_options> cands;
    for (uint32_t order = 0; order <= 1; ++order) {
        for (uint32_t c = 2; c <= 4; ++c) {
            cands.push_back({0, c, order, graph});
            cands.push_back({2, c, order, graph});
        }
        cands.push_back({1, 4, order, graph});
    }
    cands.push_back({3, 4, 0, graph});
    cudaEvent_t e0, e1;
    BT_CUDA(cudaEventCreate(&e0));
    BT_CUDA(cudaEventCreate(&e1));
    float best_ms = 0;
    re_batch_options pick = b->opt;
    re_status st = RE_OK;
    for (const re_batch_options& o : cands) {
        if ((st = re_batch_plan(b, items.data(), items.size(), &o))) break;
        if ((st = re_batch_launch(b, stream))) break;   // warm-up
        cudaEventRecord(e0, stream);
        for (uint32_t r = 0; r < reps && !st; ++r) st = re_batch_launch(b, stream);
        cudaEventRecord(e1, stream);
        if (st) break;
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            st = fail(RE_CUDA_ERROR, "autotune timing failed");
            break;
        }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (best_ms == 0 || ms < best_ms) {
            best_ms = ms;
            pick = o;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    if ((st = re_batch_plan(b, items.data(), items.size(), &pick))) return st;
    {
        std::lock_guard<std::mutex> lock(g_tuned_mutex);
        g_tuned[b->shape] = pick;
    }
    if (best) *best = pick;
    return RE_OK;
}

}  // extern "C"
