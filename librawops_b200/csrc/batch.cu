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

struct re_batch {
    BatchShape shape{};
    std::vector<re_batch_item> items;
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

re_status enqueue(re_batch* b, cudaStream_t stream) {
    if (b->direct) return launch_singles(b, b->directs, stream);
    BT_CUDA(cudaMemsetAsync(b->head, 0, b->head_words * sizeof(uint32_t), stream));
    for (const LaunchGroup& g : b->groups) BT_CUDA(launch_batch_group(g.params, g.grid, false, stream));
    for (const LaunchGroup& g : b->groups) BT_CUDA(launch_batch_group(g.params, 0, true, stream));
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
    delete b;
    return RE_OK;
}

re_status re_batch_plan(re_batch* b, const re_batch_item* items, size_t count, const re_batch_options* options) {
    if (!b || (count && !items)) return fail(RE_INVALID_ARGUMENT, "null batch arguments");
    if (count > (1u << 24)) return fail(RE_LENGTH_ERROR, "too many batch requests");
    b->planned = false;
    std::vector<re_batch_item> copy(items, items + count);
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
    for (size_t i = 0; i < count; ++i) {
        Req r;
        re_status s = describe(copy[i], i, r);
        if (s) return s;
        if (!copy[i].viewport.width || !copy[i].viewport.height) continue;
        orig.push_back(r);
        valid.push_back(copy[i]);
        info.native_pixels += (uint64_t)r.native.width * r.native.height;
        info.output_pixels += (uint64_t)copy[i].viewport.width * copy[i].viewport.height;
        info.reduced_requests += copy[i].mip ? 1 : 0;
    }
    info.requests = (uint32_t)orig.size();
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
    b->units = (uint32_t)tiles;
    b->runits = 0;
    for (const GroupTables& T : tabs) b->runits += (uint32_t)T.runit_task.size();
    b->items = std::move(copy);
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
    return launch_singles(b, b->singles, (cudaStream_t)stream_);
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
    const std::vector<re_batch_item> items = b->items;
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
