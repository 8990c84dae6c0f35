// Device-side layout of a batched render: many render requests (tiles of
// several images, recipes and mip levels) drained by one persistent kernel.
//
// Phase 1 renders every request's native region (the viewport at mip 0, the
// native footprint at mip 1/2) in CTA tiles -- the same tiles and per-tile
// code as the single-request kernels -- taking tiles from one queue of tile
// records (the tiles of one request are contiguous).  Phase 2 averages the
// footprints of the reduced requests and runs their stages after the mip
// anchor.
#pragma once

#include <cstdint>

#include "re_device.cuh"

namespace re {

// One CTA tile of the queue (64 bytes, so that a tile's record is one aligned
// line that cp.async can prefetch while the previous tile renders).
struct BatchUnit {
    int32_t image, program;
    int32_t x0, y0;              // CTA tile origin (even sensor coordinates)
    int32_t ox, oy, ow, oh;      // rendered native region of the request
    int32_t menon, layout, stage_end, pad;
    float* out;                  // final output, or the native scratch of a reduced request
    uint64_t out_stride;         // floats
};
static_assert(sizeof(BatchUnit) == 64, "tile record size");

struct ReduceTask {
    int32_t program, scale, stage_begin, stage_end;
    int32_t nw, nh, ow, oh;
    int32_t tiles_x;
    uint32_t unit_begin;
    const float* native;
    uint64_t native_stride;
    float* out;
    uint64_t out_stride;
};

// Kernel parameters of one launch group: the images and render programs of
// its requests ride in the kernel's parameter space (read through the constant
// cache like the single-request kernels' grid constants), the task tables in
// global memory.  A batch with more distinct programs or images than one group
// holds is split into several groups, launched back to back.
constexpr int BATCH_PROGRAMS = 24, BATCH_IMAGES = 32;

struct BatchParams {
    DevRaw images[BATCH_IMAGES];
    DevProgram programs[BATCH_PROGRAMS];
    const BatchUnit* units_rec;
    const ReduceTask* rtasks;
    const uint32_t* runit_task;
    uint32_t units, runits;
    uint32_t dispatch;           // 0 persistent queue, 1 one CTA per tile, 2 persistent strided + prefetch
    uint32_t menon_policy;       // the group's Menon policy (1 binary64, 2 binary32); its kernel has only that path
    uint32_t* queue;             // next unit of this group (persistent queue)
    uint32_t* status;
};

constexpr int RD_TW = 32, RD_TH = 8;   // reduced pixels per phase-2 unit (one per thread)
// CTA tile of the Menon and bilinear kernels (asserted against their definitions).
constexpr int BATCH_MENON_TW = 32, BATCH_MENON_TH = 16, BATCH_BILINEAR_TW = 64, BATCH_BILINEAR_TH = 16;

}  // namespace re
