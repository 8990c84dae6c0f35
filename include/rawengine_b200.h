/* rawengine_b200 -- C ABI of the B200 tiled-render hot path of RawEngine.
 *
 * Plain C: fixed-width integers, pointers and sizes; no C++ or torch types.
 * Every function returns an re_status; on failure re_last_error() holds a
 * thread-local message.  Status codes map one-to-one onto the exception types
 * the reference throws on the same condition (RawEngine.hpp, SpatialOps.hpp,
 * GeometryOps.hpp, TileScheduler.hpp of tylermcm/librawops):
 *   RE_INVALID_ARGUMENT <-> std::invalid_argument, RE_OUT_OF_RANGE <-> std::out_of_range,
 *   RE_DOMAIN_ERROR <-> std::domain_error, RE_LENGTH_ERROR <-> std::length_error,
 *   RE_OVERFLOW_ERROR <-> std::overflow_error, RE_CANCELLED <-> RenderCancelled.
 *
 * Each entry point names the reference interface it replaces.  Images are
 * device-resident once created; outputs may be host or device memory.
 * Calls are reentrant: state is per handle, streams are caller-supplied
 * (cudaStream_t passed as void*, NULL = the legacy default stream).
 */
#ifndef RAWENGINE_B200_H
#define RAWENGINE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define RE_API __attribute__((visibility("default")))
#else
#define RE_API
#endif

typedef enum re_status {
    RE_OK = 0,
    RE_INVALID_ARGUMENT = 1,
    RE_OUT_OF_RANGE = 2,
    RE_DOMAIN_ERROR = 3,
    RE_LENGTH_ERROR = 4,
    RE_OVERFLOW_ERROR = 5,
    RE_CANCELLED = 6,
    RE_CUDA_ERROR = 7,
    RE_TIMEOUT = 8,
} re_status;

/* Rect (RawEngine.hpp:29-31). */
typedef struct re_rect { uint32_t x, y, width, height; } re_rect;

/* RawMetadata (RawEngine.hpp:57-65).  pattern: 0 RGGB, 1 BGGR, 2 GRBG, 3 GBRG. */
typedef struct re_raw_metadata {
    uint32_t width, height, row_stride_samples;
    uint32_t pattern;
    uint32_t cfa_phase_x, cfa_phase_y;
    re_rect active_area;
    uint16_t black_levels[4];
    uint16_t white_levels[4];
} re_raw_metadata;

/* ------------------------------------------------------------------ errors */

/* Thread-local text of the last failure on this thread. */
RE_API const char* re_last_error(void);
/* Library version (major*10000 + minor*100 + patch). */
RE_API int re_version(void);
/* CUDA device count visible to the library (0 without a GPU; never fails). */
RE_API int re_device_count(void);

/* ------------------------------------------------------------ RAW sources */

typedef struct re_image re_image;

/* RawImage::RawImage(RawMetadata, std::vector<uint16_t>) (RawEngine.cpp:223-250):
 * validates and normalizes `meta` in place (stride 0 -> width, empty active area
 * -> full sensor), then uploads the samples to the current device.  `samples`
 * is HOST memory of `count` uint16 values (count == stride * height). */
RE_API re_status re_image_create(re_raw_metadata* meta, const uint16_t* samples, size_t count,
                                 re_image** out);
/* Same, but `device_samples` is already device memory; it is NOT copied and must
 * outlive the handle. */
RE_API re_status re_image_wrap_device(re_raw_metadata* meta, const uint16_t* device_samples,
                                      size_t count, re_image** out);
RE_API re_status re_image_destroy(re_image* image);

/* Source ingest (SourceFingerprint.cpp:65-101): the canonical content
 * fingerprint, SHA-256 of the reference's byte stream (version tag, metadata
 * little-endian, the active area's samples row by row), into digest[32].
 * re_fingerprint_raw normalizes *meta like re_image_create.  The raster form
 * hashes width, height, working space (0 ProPhoto D50, 1 Rec.2020 D65) and
 * the bits of every float (row stride in pixels, 0 = width). */
RE_API re_status re_fingerprint_raw(re_raw_metadata* meta, const uint16_t* samples, size_t count,
                                    uint8_t digest[32]);
RE_API re_status re_fingerprint_raster(uint32_t width, uint32_t height, size_t row_stride_pixels,
                                       uint32_t working_space, const float* pixels, uint8_t digest[32]);
/* re_image_create whose upload runs while the fingerprint is computed: the
 * plane goes to the device in chunks through pinned staging buffers, each
 * chunk hashed on the host while its copy is in flight.  No counterpart in
 * the reference (its sources stay in host memory). */
RE_API re_status re_image_create_fingerprinted(re_raw_metadata* meta, const uint16_t* samples, size_t count,
                                               re_image** out, uint8_t digest[32]);
RE_API re_status re_image_metadata(const re_image* image, re_raw_metadata* out);

/* Metadata normalization/validation only (no device work): RawEngine.cpp:223-250. */
RE_API re_status re_raw_metadata_normalize(re_raw_metadata* meta, size_t count);
/* RawEngine.cpp:74-87: photosite index and CFA colour (R=0, G=1, B=2). */
RE_API int re_site_index(const re_raw_metadata* meta, uint32_t x, uint32_t y);
RE_API int re_cfa_color(const re_raw_metadata* meta, uint32_t x, uint32_t y);

/* ------------------------------------------------------ host-side planning */

/* RawEngine.cpp:31-43 request_bounds: extent of a render level. */
RE_API re_status re_request_bounds(re_rect source_bounds, uint32_t mip, uint32_t quality,
                                   re_rect* out);
/* RawEngine.cpp:290-297 RawUnpackNode::input_region: the clipped demosaic halo
 * (1 for bilinear, 6 for Menon unless an active-area axis is a singleton). */
RE_API re_status re_raw_input_region(const re_raw_metadata* meta, uint32_t demosaic,
                                     re_rect output, re_rect* region);
/* RawEngine.cpp:563-578 CameraToWorkingNode::input_region_level: native
 * footprint of a reduced (mip 1/2) request. */
RE_API re_status re_mip_native_region(re_rect native_bounds, uint32_t mip, re_rect output,
                                      re_rect* native);
/* RawEngine.cpp:1399-1411 render_tiles tile order: writes up to `capacity`
 * tiles and returns the total count in *count. */
RE_API re_status re_plan_tiles(re_rect viewport, uint32_t tile_size, re_rect* tiles,
                               size_t capacity, size_t* count);

/* RawEngine.cpp:116-219, 502-530: camera->XYZ(D50) composed with XYZ->working
 * space in double, cast to float32.  target: 0 LinearProPhotoD50, 1 LinearRec2020D65. */
RE_API re_status re_camera_to_working_matrix(const double camera_to_xyz_d50[9], uint32_t target,
                                             float out[9]);
/* RawEngine.cpp:198-214, 658-672 WorkingToSrgbNode matrix. */
RE_API re_status re_working_to_srgb_matrix(uint32_t source, float out[9]);
/* RawEngine.cpp:216-219, 603-623 WorkingSpaceConvertNode matrix. */
RE_API re_status re_working_to_working_matrix(uint32_t source, uint32_t target, float out[9]);
/* RawEngine.cpp:465-468 ExposureNode multiplier (exp2 of stops, stops in [-32,32]). */
RE_API re_status re_exposure_multiplier(float stops, float* out);

/* ------------------------------------------------------- point programs */

/* The per-pixel stages of a render chain, fused into the demosaic kernel.
 * Each kind restates one reference node's pixel arithmetic:
 *   RE_STAGE_GAIN3   WhiteBalanceNode::render        RawEngine.cpp:417-431  f[0..2] gains
 *   RE_STAGE_SCALE   ExposureNode::render_level      RawEngine.cpp:488-500  f[0] multiplier
 *   RE_STAGE_MATRIX  CameraToWorking / WorkingToSrgb / WorkingSpaceConvert
 *                    RawEngine.cpp:539-545, 646-652, 694-700             f[0..8] row-major
 *   RE_STAGE_TONE    ToneCurveNode::render_level     RawEngine.cpp:738-758  f[0] shoulder, f[1] 1/gamma
 *   RE_STAGE_CLIP    OutputClipNode::render          RawEngine.cpp:1223-1233
 *   RE_STAGE_SRGB    SrgbEncodeNode::render_level    RawEngine.cpp:1254-1277
 *   RE_STAGE_CURVES  ExtendedCurvesNode::render_level ToneOps.cpp:833-844   arg = curve set
 */
typedef enum re_stage_kind {
    RE_STAGE_GAIN3 = 1,
    RE_STAGE_SCALE = 2,
    RE_STAGE_MATRIX = 3,
    RE_STAGE_TONE = 4,
    RE_STAGE_CLIP = 5,
    RE_STAGE_SRGB = 6,
    RE_STAGE_CURVES = 7,
} re_stage_kind;

#define RE_MAX_STAGES 16

typedef struct re_stage {
    uint32_t kind;
    uint32_t arg;
    float f[12];
} re_stage;

typedef struct re_curve_set re_curve_set;

/* ExtendedCurvesSettings (ToneOps.hpp:19-25) -> a device curve set.
 * knots: x0,y0,x1,y1,... for the master, R, G, B curves concatenated;
 * counts[4] knot counts (2..256 each); interpolation 0 Linear, 1
 * ShapePreservingCubic.  Validation follows ToneOps.cpp:17-31, 117-122. */
RE_API re_status re_curve_set_create(uint32_t interpolation, const uint32_t counts[4],
                                     const double* knots, re_curve_set** out);
RE_API re_status re_curve_set_destroy(re_curve_set* curves);

/* A render description: demosaic policy (RawEngine.cpp:276-280) -- 0
 * rawengine.bilinear v1; 1 rawengine.menon_base v1 in binary64, bit-exact; 2
 * rawengine.menon_base v1 computed in binary32 with every direction decision
 * equal to the reference's (decisions inside the binary32 error band are
 * recomputed in binary64) and demosaic outputs within a few ulp of the
 * reference's (steep curves after it can magnify that past 1e-5) -- then
 * `count` stages.  Stages
 * [0, anchor] run at native resolution; when a reduced level is requested the
 * result is averaged over each output pixel's native footprint after stage
 * `anchor` (the CameraToWorking mip anchor, RawEngine.cpp:580-601), and stages
 * after the anchor run on the reduced pixels.  anchor = -1: no reduced levels. */
typedef struct re_render_desc {
    uint32_t demosaic;
    int32_t anchor;
    uint32_t count;
    re_stage stages[RE_MAX_STAGES];
    const re_curve_set* curves[4];
} re_render_desc;

/* Statistics of one render (Menon near-tie and guard counters). */
typedef struct re_render_stats {
    uint64_t pixels;             /* output pixels written */
    uint64_t native_pixels;      /* demosaiced native pixels */
    uint64_t menon_decisions;    /* directional decisions evaluated */
    uint64_t menon_near_ties;    /* decisions within the exact-recheck band */
    uint32_t launches;           /* kernels launched */
    float device_ms;             /* device time of the render (CUDA events) */
} re_render_stats;

/* Renderer::render_image(node, source_bounds, RenderRequest) for a RAW chain
 * (RawEngine.cpp:1426-1447) fused into one pass per render: demosaic + stages
 * (+ mip reduction).  `viewport` is in level coordinates (the active-area
 * origin at mip 0, zero-based at mip 1/2; RawEngine.hpp:35-40).  quality: 0
 * Preview, 1 Final.  `out` receives viewport.height rows of
 * `out_row_stride` floats (>= 3*viewport.width); out_on_device selects device
 * vs host memory (host output is copied back inside this call).  stats may be
 * NULL.  The call returns after the render completed on `stream`. */
RE_API re_status re_render_raw(const re_image* image, const re_render_desc* desc,
                               re_rect viewport, uint32_t mip, uint32_t quality, float* out,
                               size_t out_row_stride, int out_on_device, void* stream,
                               re_render_stats* stats);

/* The Menon direction of every pixel of a viewport (1 horizontal, 0
 * vertical; green sites 1), as demosaic policy `demosaic` (1 or 2) decides
 * it, into DEVICE memory `out` (viewport.width x viewport.height bytes).
 * *near_ties (host, may be NULL) receives the number of exact ties v == h
 * (policy 1) or of decisions taken by the binary64 recheck (policy 2).
 * Returns after completion on `stream`. */
RE_API re_status re_menon_directions(const re_image* image, uint32_t demosaic, re_rect viewport, uint8_t* out,
                                     uint64_t* near_ties, void* stream);

/* Asynchronous device-only form: enqueues the render on `stream` and returns.
 * Non-finite/overflow guards are OR-ed into *device_status (a device word the
 * caller zeroes and later reads; re_status_from_device maps it).  No host sync.
 * `scratch` must be device memory of at least re_render_scratch_bytes() bytes
 * when mip > 0 (NULL otherwise). */
RE_API re_status re_render_raw_async(const re_image* image, const re_render_desc* desc,
                                     re_rect viewport, uint32_t mip, uint32_t quality, float* out,
                                     size_t out_row_stride, uint32_t* device_status,
                                     void* scratch, void* stream);
RE_API size_t re_render_scratch_bytes(const re_image* image, const re_render_desc* desc,
                                      re_rect viewport, uint32_t mip);
RE_API re_status re_status_from_device(uint32_t device_status_word);

/* Per-call device scratch of the synchronous entry points (the native
 * footprint of a reduced render, geometry and filter intermediates, the
 * differentiable planes) comes from a stream-ordered memory pool that the
 * library creates on each device and that keeps freed blocks mapped, so
 * repeated calls of the same size do not map and unmap device memory.  No
 * counterpart in the reference (its scratch is host memory).  This returns
 * the pool's idle blocks to the driver; blocks in use are unaffected. */
RE_API re_status re_release_scratch(void);

/* Reduced-level (mip 1 or 2, Preview) RAW render that allocates no memory.
 * No counterpart in the reference: it exists for callers that cannot allocate
 * device memory while rendering -- a plug-in inside a host application whose
 * device memory is budgeted up front, or a real-time preview thread that must
 * not take allocator locks or risk running out of memory mid-frame.  Output
 * goes to caller DEVICE memory (`out`, row stride in floats); the native
 * footprint is staged in a fixed device array of
 * re_render_raw_reduced_noalloc_max_native_pixels() pixels (12 MiB, held on
 * every GPU that loads the library until exit).  Larger footprints return
 * RE_LENGTH_ERROR.  All calls share that array: calls that overlap on the GPU
 * race, so order them on one stream or serialize them.  The first call on a
 * device looks up the array's address with that device current; make it
 * before any stream capture.  Returns after the render completed on `stream`. */
RE_API re_status re_render_raw_reduced_noalloc(const re_image* image, const re_render_desc* desc,
                                               re_rect viewport, uint32_t mip, float* out,
                                               size_t out_row_stride, void* stream);
RE_API size_t re_render_raw_reduced_noalloc_max_native_pixels(void);

/* Renderer::render_tiles (RawEngine.cpp:1390-1412): the reference's per-tile
 * loop, one fused launch per tile, each tile copied to the host callback in
 * tile order.  The callback may return nonzero to cancel (RE_CANCELLED). */
typedef int (*re_tile_callback)(const re_rect* bounds, const float* rgb, void* user);
RE_API re_status re_render_tiles(const re_image* image, const re_render_desc* desc,
                                 re_rect viewport, uint32_t tile_size, uint32_t mip,
                                 uint32_t quality, re_tile_callback callback, void* user,
                                 void* stream);

/* ------------------------------------------------------------ batched render */

/* Many render requests -- tiles of several images, recipes, viewports and mip
 * levels, as TileScheduler and Renderer::render_tiles issue them
 * (TileScheduler.cpp:19-304, RawEngine.cpp:1390-1412) -- rendered by one
 * persistent kernel that drains a device queue of CTA tiles, plus one launch
 * that reduces the mip 1/2 footprints.  Every request's pixels equal
 * re_render_raw's for the same request bit for bit.  Outputs are DEVICE
 * memory.  No counterpart in the reference: its scheduler renders request by
 * request. */
typedef struct re_batch_item {
    const re_image* image;
    const re_render_desc* desc;
    re_rect viewport;           /* level coordinates, as re_render_raw */
    uint32_t mip, quality;
    float* out;                 /* device memory */
    size_t out_row_stride;      /* floats, >= 3 * viewport.width */
    /* Geometry requests (CubicResizeNode / RotateNode over a RAW chain,
     * GeometryOps.cpp:42-174, 346-513): `desc` renders the RAW source's point
     * stages at native resolution (its anchor is ignored) over the active
     * area, whose extent is the geometry's input; the geometry maps it to its
     * canvas (cubic: canvas_width x canvas_height; rotation: the input's
     * extent) at level `mip` (1/2 with quality Preview: native then the
     * footprint average); then the stages of `post` (point stages only, may
     * be NULL) run at the level.  viewport is in canvas level coordinates.
     * geometry 0 = a plain RAW request (the fields below are ignored). */
    uint32_t geometry;          /* 0 none, 1 cubic resize, 2 rotation */
    uint32_t canvas_width, canvas_height;
    double angle_degrees;
    const re_render_desc* post;
} re_batch_item;

typedef struct re_batch_options {
    uint32_t dispatch;          /* 0: persistent grid draining an atomic tile queue; 1: one CTA per
                                   tile; 2: persistent grid taking every grid-th tile, prefetching
                                   the next tile's record while the current one renders; 3: one
                                   plain render launch per merged render (see re_batch_plan) */
    uint32_t ctas_per_sm;       /* persistent grid = SMs x this (1..4); 0 = 4 */
    uint32_t order;             /* 0: requests in submission order; 1: Menon requests first */
    uint32_t use_graph;         /* nonzero: launches replayed from a CUDA graph */
} re_batch_options;

typedef struct re_batch_info {
    uint32_t requests, reduced_requests;
    uint32_t tasks;             /* renders after merging adjacent requests */
    uint32_t tiles;             /* phase-1 CTA tiles (queue length) */
    uint32_t reduce_blocks;     /* phase-2 blocks */
    uint32_t grid;              /* phase-1 CTAs launched */
    uint64_t native_pixels, output_pixels;
    uint64_t raw_bytes, output_bytes;    /* algorithmic: 2 B per native pixel, 12 B per output pixel */
    re_batch_options options;
    uint32_t geometry_requests;          /* requests with a cubic resize or rotation */
} re_batch_info;

typedef struct re_batch re_batch;

RE_API re_status re_batch_create(re_batch** out);
RE_API re_status re_batch_destroy(re_batch* batch);
/* Validates every item like re_render_raw_async (geometry items like
 * re_cubic_resize_window / re_rotate_window), merges requests of one
 * image, description, level and row stride whose viewports tile a rectangle
 * and whose outputs lie where one render of it would write (the pixels are the
 * same either way), lays out the tile queue and the reduction blocks, uploads
 * them and sizes the mip scratch (held by the batch).  options may be NULL (defaults, or the autotuned choice cached for
 * a batch of the same shape). */
RE_API re_status re_batch_plan(re_batch* batch, const re_batch_item* items, size_t count,
                               const re_batch_options* options);
/* Enqueues the planned batch on `stream` (no host synchronization). */
RE_API re_status re_batch_launch(re_batch* batch, void* stream);
/* The same planned requests launched one by one with the single-request
 * kernels (demosaic, then the mip reduction for reduced requests): the
 * per-tile form the batch replaces, for comparison.  Same outputs. */
RE_API re_status re_batch_launch_per_request(re_batch* batch, void* stream);
/* Waits for `stream` and maps the batch's device status word (non-finite or
 * out-of-range values at the output boundary, as re_render_raw). */
RE_API re_status re_batch_status(re_batch* batch, void* stream);
RE_API re_status re_batch_info_get(const re_batch* batch, re_batch_info* info);
/* Times the dispatch choices (queue or strided persistent grids of 2..4
 * CTAs/SM, one CTA per tile, either request order; plain launches per merged
 * render) over `reps` launches of the planned batch and re-plans
 * with the fastest; the choice is cached for batches of the same shape. */
RE_API re_status re_batch_autotune(re_batch* batch, uint32_t reps, void* stream, re_batch_options* best);

/* ------------------------------------------------------- differentiable render */

/* Forward kernels of the render path with the recipe as parameters, and their
 * hand-written adjoints (vector-Jacobian products), for fitting recipes by
 * gradient descent.  No counterpart in the reference, which has no gradients;
 * the forward arithmetic restates RawEngine.cpp:299-344 (bilinear) or
 * MenonDemosaic.cpp:97-173 (Menon), RawEngine.cpp:417-431/488-500/539-545
 * (WB, exposure, 3x3), ToneOps.cpp:795-844 (the
 * master curve, shape-preserving cubic) and SpatialOps.cpp:168-287 (the
 * working-Y guided filter, used as a detail boost v + k (v - GF(v))).  All
 * buffers are DEVICE memory; images are contiguous float32 (h, w, 3); the
 * sensor plane is (h, w) over the active area; `quad` packs the colours of the
 * 2x2 CFA cell at the plane's origin, 2 bits each, index (y&1)*2+(x&1).
 * Calls enqueue on `stream` and return. */
RE_API re_status re_diff_bilinear_forward(const float* plane, size_t plane_row_stride, uint32_t width,
                                          uint32_t height, uint32_t quad, float* rgb, void* stream);
RE_API re_status re_diff_bilinear_backward(const float* drgb, uint32_t width, uint32_t height, uint32_t quad,
                                           float* dplane, size_t dplane_row_stride, void* stream);
/* Menon demosaic (MenonDemosaic.cpp:97-173, mirrored borders, binary64) of
 * the normalized plane, with the direction of every site written to
 * `directions` (device, width x height bytes, 1 = horizontal; green sites
 * 1).  The backward is the transpose of the demosaic with those directions
 * held fixed (the directions' own derivative is zero almost everywhere). */
RE_API re_status re_diff_menon_forward(const float* plane, size_t plane_row_stride, uint32_t width, uint32_t height,
                                       uint32_t quad, float* rgb, uint8_t* directions, void* stream);
RE_API re_status re_diff_menon_backward(const float* drgb, uint32_t width, uint32_t height, uint32_t quad,
                                        const uint8_t* directions, float* dplane, size_t dplane_row_stride,
                                        void* stream);

/* WB gains, exposure multiplier, row-major 3x3, then the master curve: knots
 * kx/ky (n of each), Bezier controls c0/c1 (n-1 of each) and the end slopes
 * used for linear extrapolation.  All device memory, so that parameters that
 * live on the device (an optimizer's) need no host round trip: `scalars` holds
 * wb[3], exposure, matrix[9], slope_first, slope_last (15 floats); knots = 0:
 * no curve. */
typedef struct re_diff_point_params {
    const float* scalars;
    uint32_t knots;
    const float* kx;
    const float* ky;
    const float* c0;
    const float* c1;
} re_diff_point_params;
RE_API re_status re_diff_point_forward(const float* x, size_t pixels, const re_diff_point_params* params,
                                       float* y, void* stream);
/* Adds the parameter gradients to `grads` (double, caller-zeroed, length
 * re_diff_point_grad_count(knots)): wb[3], exposure, matrix[9], ky[n],
 * c0[n-1], c1[n-1], slope_first, slope_last. */
RE_API re_status re_diff_point_backward(const float* x, const float* dy, size_t pixels,
                                        const re_diff_point_params* params, float* dx, double* grads,
                                        void* stream);
RE_API size_t re_diff_point_grad_count(uint32_t knots);

/* Detail boost out = p + strength (p - GF(p)), GF the self-guided working-Y
 * guided filter (radius 0..64, epsilon [2^-24, 65536], clipped windows with
 * actual counts; at most 65535 rows).  `strength` is one device float.  The
 * backward recomputes every box mean from p and adds d loss / d strength to
 * *dstrength and d loss / d epsilon to *depsilon (doubles, device). */
RE_API re_status re_diff_detail_forward(const float* p, uint32_t width, uint32_t height, uint32_t radius,
                                        double epsilon, const float* strength, uint32_t working_space, float* out,
                                        void* stream);
RE_API re_status re_diff_detail_backward(const float* p, const float* dout, uint32_t width, uint32_t height,
                                         uint32_t radius, double epsilon, const float* strength,
                                         uint32_t working_space, float* dp, double* dstrength, double* depsilon,
                                         void* stream);

/* ------------------------------------------------------------- raster I/O */

/* RasterSourceNode::render_level (RawEngine.cpp:346-406) followed by the
 * stages of `desc` (its demosaic and anchor are ignored): `in` is a device
 * float32 RGB image (width x height, row stride in floats); mip 1/2 Preview
 * average each output pixel's clipped footprint in double with the actual
 * count.  `out` is device memory.  Returns after completion on `stream`. */
RE_API re_status re_render_raster(const float* in, size_t in_row_stride, uint32_t width, uint32_t height,
                                  const re_render_desc* desc, re_rect viewport, uint32_t mip,
                                  uint32_t quality, float* out, size_t out_row_stride, void* stream);

/* float32 interleaved RGB device buffers for spatial/geometry stages. */

/* working_y_guided_filter_rgb (SpatialOps.cpp:168-287) over a whole image:
 * `in` is a device image of width*height RGB pixels (row stride in floats),
 * `out` a device buffer of the same shape.  working_space selects the Y weights
 * (0 ProPhoto, 1 Rec2020, SpatialOps.cpp:191-192).  Radius 0..64, epsilon in
 * [2^-24, 65536].  Windows clip at the image edge with actual counts.  `out`
 * must not overlap `in`.  Returns after the filter completed on `stream`. */
RE_API re_status re_guided_filter(const float* in, size_t in_row_stride, float* out,
                                  size_t out_row_stride, uint32_t width, uint32_t height,
                                  uint32_t radius, double epsilon, uint32_t working_space,
                                  void* stream);
/* The same filter, enqueued on `stream` without a host synchronization:
 * non-finite input and float32 overflow are OR-ed into *device_status (a
 * device word the caller zeroes and maps with re_status_from_device), and
 * `scratch` is device memory of re_guided_filter_scratch_bytes(width, height,
 * radius) bytes (the kernel's per-CTA rings of row sums).  `out` must not
 * overlap `in`. */
RE_API re_status re_guided_filter_async(const float* in, size_t in_row_stride, float* out,
                                        size_t out_row_stride, uint32_t width, uint32_t height,
                                        uint32_t radius, double epsilon, uint32_t working_space,
                                        uint32_t* device_status, void* scratch, void* stream);
RE_API size_t re_guided_filter_scratch_bytes(uint32_t width, uint32_t height, uint32_t radius);
/* local_statistics_rgb (SpatialOps.cpp:79-121) over a whole image: per channel
 * box mean and population variance over the clipped (2r+1)^2 window, excluding
 * non-finite samples (count_out gets the finite count; mean/variance NaN when
 * it is 0).  Outputs are float32 interleaved RGB; count_out may be NULL.
 * Enqueued on `stream`; returns without waiting for it. */
RE_API re_status re_local_statistics(const float* in, size_t in_row_stride, uint32_t width,
                                     uint32_t height, uint32_t radius, float* mean_out,
                                     float* variance_out, uint32_t* count_out, void* stream);
/* The same with binary64 mean/variance, the precision of the reference's
 * LocalStatisticsTile (SpatialOps.hpp:7-13). */
RE_API re_status re_local_statistics_f64(const float* in, size_t in_row_stride, uint32_t width,
                                         uint32_t height, uint32_t radius, double* mean_out,
                                         double* variance_out, uint32_t* count_out, void* stream);

/* CubicResizeNode (GeometryOps.cpp:346-513): scale-aware Catmull-Rom from an
 * in_w x in_h device image to the `output` rect of an out_w x out_h canvas at
 * `mip` (0..2, footprint-averaged like the reference). */
RE_API re_status re_cubic_resize(const float* in, size_t in_row_stride, uint32_t in_w,
                                 uint32_t in_h, uint32_t out_w, uint32_t out_h, re_rect output,
                                 uint32_t mip, float* out, size_t out_row_stride, void* stream);
/* RotateNode (GeometryOps.cpp:42-174): fixed-canvas clockwise rotation about
 * the pixel-centre pivot, clamped bilinear taps, mip 0..2 footprint average. */
RE_API re_status re_rotate(const float* in, size_t in_row_stride, uint32_t width, uint32_t height,
                           double angle_degrees, re_rect output, uint32_t mip, float* out,
                           size_t out_row_stride, void* stream);
/* The same two operators on an input WINDOW: `in` holds only the input
 * columns [window.x, window.x + window.width) and rows [window.y, ...) of the
 * full in_w x in_h (width x height) image -- the support a tile needs, as the
 * reference's nodes request it (GeometryOps.cpp:99-118, 411-430).  The window
 * must cover the taps of every requested output pixel (checked on the host). */
RE_API re_status re_cubic_resize_window(const float* in, size_t in_row_stride, re_rect window, uint32_t in_w,
                                        uint32_t in_h, uint32_t out_w, uint32_t out_h, re_rect output,
                                        uint32_t mip, float* out, size_t out_row_stride, void* stream);
RE_API re_status re_rotate_window(const float* in, size_t in_row_stride, re_rect window, uint32_t width,
                                  uint32_t height, double angle_degrees, re_rect output, uint32_t mip,
                                  float* out, size_t out_row_stride, void* stream);
/* GeometryOps.cpp:99-111 support of a native output rectangle (relative to the
 * rotation's own bounds). */
RE_API re_status re_rotation_support(uint32_t width, uint32_t height, double angle_degrees,
                                     re_rect native_output, re_rect* support);
/* GeometryOps.cpp:362-389 one Catmull-Rom axis (host): returns taps in *count. */
RE_API re_status re_cubic_axis(uint32_t input, uint32_t output, uint32_t index, uint32_t* center,
                               uint32_t tap_index[18], double tap_weight[18], uint32_t* count);
/* GeometryOps.cpp:46-67 rotation constants (host). */
RE_API re_status re_rotation_coefficients(double angle_degrees, double* cosine, double* sine);

/* ----------------------------------------------------- local-contrast stencils */

/* SharpenNode, ClarityNode, TextureNode and ConvolutionNode::render_level
 * (SpatialOps.cpp:319-701) on device float32 RGB, bit-exact: `in` holds the
 * image rectangle `window` (row stride in floats), which must cover `output`
 * grown by the stencil's halo and clipped to `image` (the level's image
 * bounds; the reference's `needed` region): radius for Sharpen and Clarity,
 * 2 * scale for Texture, kernel_width/2 x kernel_height/2 for Convolution,
 * none for a zero amount or an identity kernel.  `out` receives the output
 * rectangle.  A non-finite sample of the needed region or a result beyond
 * float32 returns RE_INVALID_ARGUMENT with the reference's message.  Working
 * space 0 = linear ProPhoto D50, 1 = linear Rec.2020 D65.  Returns after
 * completion on `stream`. */
RE_API re_status re_sharpen_window(const float* in, size_t in_row_stride, re_rect window, re_rect image,
                                   re_rect output, double amount, uint32_t radius, float* out,
                                   size_t out_row_stride, void* stream);
RE_API re_status re_clarity_window(const float* in, size_t in_row_stride, re_rect window, re_rect image,
                                   re_rect output, double amount, uint32_t radius, uint32_t working_space,
                                   float* out, size_t out_row_stride, void* stream);
RE_API re_status re_texture_window(const float* in, size_t in_row_stride, re_rect window, re_rect image,
                                   re_rect output, double amount, uint32_t scale, uint32_t working_space,
                                   float* out, size_t out_row_stride, void* stream);
/* coefficients: host, row-major kernel_height x kernel_width (flipped on both
 * axes when applied, as a convolution). */
RE_API re_status re_convolution_window(const float* in, size_t in_row_stride, re_rect window, re_rect image,
                                       re_rect output, uint32_t kernel_width, uint32_t kernel_height,
                                       const double* coefficients, float* out, size_t out_row_stride,
                                       void* stream);

/* ------------------------------------------------------------------ analysis */

/* histogram_rgb (ImageAnalysis.cpp:9-69) over a DEVICE float32 RGB image:
 * per channel `bins` equal bins over [lower, upper] (the last includes upper;
 * bin = min(bins-1, uint32((double(s) - lower) / (upper - lower) * bins))),
 * under/overflow and non-finite tallies, and the extrema of all finite
 * samples.  Accumulates into DEVICE counters, so an image may be passed in
 * pieces: counts (3 * bins, R then G then B), tallies (underflow[3],
 * overflow[3], nonfinite[3]) and extrema (min key[3], max key[3]), all
 * uint64.  re_histogram_reset clears them.  The pieces' pixels are numbered
 * in the reference's tile traversal (tiles of tile_size, row-major, pixels
 * row-major in a tile; tile_size 0 = one tile) starting at first_index, and
 * among equal extrema (+0 and -0) the earliest in that order wins, as in the
 * reference.  re_histogram_extremum decodes a key (host): returns 0 when the
 * channel had no finite sample.  Enqueued on `stream`; no host sync. */
RE_API re_status re_histogram_reset(uint32_t bins, uint64_t* counts, uint64_t* tallies, uint64_t* extrema,
                                    void* stream);
RE_API re_status re_histogram_rgb(const float* rgb, size_t row_stride, uint32_t width, uint32_t height,
                                  uint32_t tile_size, uint64_t first_index, uint32_t bins, double lower,
                                  double upper, uint64_t* counts, uint64_t* tallies, uint64_t* extrema,
                                  void* stream);
RE_API int re_histogram_extremum(uint64_t key, int is_max, float* value);

#ifdef __cplusplus
}
#endif
#endif
