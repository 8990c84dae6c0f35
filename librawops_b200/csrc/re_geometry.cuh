// Geometry stages shared by the single-request entry points (geometry.cu)
// and the batched render (batch.cu): Catmull-Rom axis tables, rotation
// constants, the per-request plan, and the batched task records.
#pragma once

#include <cstdint>
#include <vector>

#include "re_device.cuh"

namespace re {

constexpr int GEO_MAX_TAPS = 18;

// One output column (or row) of a cubic resize: the taps of GeometryOps.cpp:362-389.
struct Axis {
    uint32_t center, count;
    uint32_t index[GEO_MAX_TAPS];
    double weight[GEO_MAX_TAPS];
};

struct RotateParams {
    double cx, cy, cosine, sine;
    int width, height;
};

// Host plan of one geometry request: the native output region of the canvas
// (the requested level's footprint), the input support it reads (relative
// to the geometry's input bounds) and, for a cubic resize, its axis tables
// and the source rows of the horizontal pass.
struct GeoPlan {
    int kind = 0;                 // 1 cubic resize, 2 rotation
    re_rect native{}, support{};
    std::vector<Axis> xs, ys;
    uint32_t row0 = 0, rows = 0;
    RotateParams rot{};
};

// kind 1: input in_w x in_h resized to a cw x ch canvas; kind 2: rotation of
// a width x height image by angle degrees.  `output` is in level coordinates.
// Validates like the single-request entry points (same messages).  A cubic
// plan's support is exact; a rotation's is exact (the reference's scan of
// every output pixel) when exact_support is set, else a cover of it from the
// native rectangle's corners with two pixels of margin (O(1) planning).
re_status plan_cubic(uint32_t in_w, uint32_t in_h, uint32_t cw, uint32_t ch, re_rect output, uint32_t mip,
                     GeoPlan& plan);
re_status plan_rotate(uint32_t width, uint32_t height, double angle, re_rect output, uint32_t mip, GeoPlan& plan,
                      bool exact_support);

// One geometry request of a batch, device side.  `src` holds the support
// region (src_x0, src_y0 its origin in input-bound coordinates); the result
// of the native region goes to out (the request's output at mip 0 without
// later stages, else a native scratch that the reduction reads).
struct GeoRequest {
    int32_t kind, nx0, ny0, nw, nh;
    int32_t src_x0, src_y0, row0, rows, pad;
    RotateParams rot;
    const float* src;
    uint64_t src_stride;
    const Axis* ax;
    const Axis* ay;
    double* H;                    // cubic: rows x nw x 3 horizontal sums
    float* out;
    uint64_t out_stride;
};

// A 32 x 8 block of one request's pass: request index, block column, row.
struct GeoBlock {
    uint32_t request;
    uint16_t bx, by;
};
constexpr int GEO_BW = 32, GEO_BH = 8;

// Pass 1: every cubic request's horizontal sums and every rotation; pass 2:
// every cubic request's vertical pass.  Either table may be empty.
cudaError_t launch_geometry_batch(const GeoRequest* requests, const GeoBlock* pass1, uint32_t n1,
                                  const GeoBlock* pass2, uint32_t n2, uint32_t* status, cudaStream_t stream);
// The same passes for one request, as the single-request entry points run them.
cudaError_t launch_geometry_single(const GeoRequest& request, uint32_t* status, cudaStream_t stream);

}  // namespace re
