/* CPU restatement of RawEngine's tiled-render hot path -- TEST INFRASTRUCTURE.
 *
 * This is the oracle: only tests/, the smoke check and bench.py's CPU
 * baseline call it, and only as the checker (or the timed CPU port).  The
 * product never links it.  Each function names the reference file:line whose
 * algorithm it restates; the arithmetic order is kept where the reference
 * freezes it, so that results are bit-identical to the reference on the same
 * inputs (this is pinned by tests against the reference's own golden vectors
 * and against the reference library built in oracle/_ref).
 *
 * Conventions: rectangles are {x, y, width, height}; RGB is interleaved
 * float32, row-major; status 0 = ok, otherwise an OR_* code below.
 */
#ifndef RAWENGINE_ORACLE_H
#define RAWENGINE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    OR_OK = 0,
    OR_INVALID_ARGUMENT = 1,
    OR_OUT_OF_RANGE = 2,
    OR_DOMAIN_ERROR = 3,
    OR_LENGTH_ERROR = 4,
    OR_OVERFLOW_ERROR = 5,
};

typedef struct or_rect { uint32_t x, y, width, height; } or_rect;

typedef struct or_raw_metadata {
    uint32_t width, height, row_stride_samples;
    uint32_t pattern;            /* 0 RGGB, 1 BGGR, 2 GRBG, 3 GBRG */
    uint32_t cfa_phase_x, cfa_phase_y;
    or_rect active_area;
    uint16_t black_levels[4], white_levels[4];
} or_raw_metadata;

/* RawEngine.cpp:223-250: normalize stride/active area in place and validate. */
int or_raw_normalize(or_raw_metadata* m, size_t sample_count);
/* RawEngine.cpp:74-87 */
int or_site_index(const or_raw_metadata* m, uint32_t x, uint32_t y);
int or_cfa_color(const or_raw_metadata* m, uint32_t x, uint32_t y);
/* RawEngine.cpp:89-97 */
float or_sample(const or_raw_metadata* m, const uint16_t* samples, uint32_t x, uint32_t y);

/* RawEngine.cpp:299-344 bilinear v1 over rect r (inside the active area). */
int or_bilinear(const or_raw_metadata* m, const uint16_t* samples, or_rect r, float* out);
/* MenonDemosaic.cpp:89-218 menon_base v1 over rect r; directions (1 = horizontal)
 * are written per output pixel when `horizontal` is non-null. */
int or_menon(const or_raw_metadata* m, const uint16_t* samples, or_rect r, float* out,
             uint8_t* horizontal);
/* RawEngine.cpp:290-297 source halo of the RAW source node. */
int or_raw_input_region(const or_raw_metadata* m, int menon, or_rect output, or_rect* region);

/* RawEngine.cpp:408-431 */
void or_white_balance(float* rgb, size_t pixels, float r, float g, float b);
/* RawEngine.cpp:465-500 (multiplier = exp2f(stops)) */
float or_exposure_multiplier(float stops);
void or_scale(float* rgb, size_t count, float multiplier);
/* RawEngine.cpp:116-219, 502-530: camera->XYZ(D50) composed with XYZ->working,
 * in double, then cast to float.  target: 0 ProPhoto D50, 1 Rec2020 D65. */
int or_camera_to_working_matrix(const double camera_to_xyz[9], int target, float out[9]);
/* RawEngine.cpp:198-214, 658-672 */
int or_working_to_srgb_matrix(int source, float out[9]);
/* RawEngine.cpp:216-219, 603-623 */
int or_working_to_working_matrix(int source, int target, float out[9]);
/* RawEngine.cpp:539-545: the float 3x3 product in the reference's order. */
void or_matrix3(float* rgb, size_t pixels, const float m[9]);
/* RawEngine.cpp:705-758 */
void or_tone_curve(float* rgb, size_t count, float shoulder, float gamma);
/* RawEngine.cpp:1215-1233; returns OR_DOMAIN_ERROR on non-finite input. */
int or_output_clip(float* rgb, size_t count);
/* RawEngine.cpp:1254-1277; returns OR_DOMAIN_ERROR on non-finite input. */
int or_srgb_encode(float* rgb, size_t count);

/* ToneOps.cpp:795-844 extended curves.  knots: x0,y0,x1,y1,... counts[4] =
 * master, R, G, B; interpolation 0 linear, 1 shape-preserving cubic. */
typedef struct or_curves {
    int interpolation;
    uint32_t count[4];
    double knots[4][512];          /* up to 256 (x, y) pairs per curve */
    double slopes[4][256];
    double controls[4][256][2];
    int identity[4];
} or_curves;
int or_curves_prepare(or_curves* c);
int or_curves_apply(const or_curves* c, float* rgb, size_t count);
double or_curve_map(const or_curves* c, unsigned curve, double value);

/* RawEngine.cpp:31-43 */
int or_request_bounds(or_rect source_bounds, uint32_t mip, uint32_t quality, or_rect* out);
/* RawEngine.cpp:563-578 (RAW anchor) */
int or_mip_native_region(or_rect native_bounds, uint32_t mip, or_rect output, or_rect* native);
/* RawEngine.cpp:580-601: reduce a native tile (covering `mapped`) to `output`. */
void or_mip_reduce(const float* native, or_rect mapped, uint32_t mip, or_rect output, float* out);

/* SpatialOps.cpp:164-167, 168-287: guided filter of the tile `in` covering
 * `needed` (= the 2r-expanded output) into `out` (output rect). */
int or_guided_filter(const float* in, or_rect needed, or_rect output, or_rect image,
                     uint32_t radius, double epsilon, int prophoto, float* out);
int or_guided_filter_region(or_rect output, or_rect image, uint32_t radius, or_rect* needed);
/* SpatialOps.cpp:74-121 */
int or_local_statistics(const float* in, or_rect needed, or_rect output, or_rect image,
                        uint32_t radius, double* mean, double* variance, uint32_t* count);
int or_local_statistics_region(or_rect output, or_rect image, uint32_t radius, or_rect* needed);

/* GeometryOps.cpp:362-389: one Catmull-Rom axis.  Returns tap count (<=18)
 * or a negative OR_* code. */
int or_cubic_axis(uint32_t input, uint32_t output, uint32_t index, uint32_t* center,
                  uint32_t* tap_index, double* tap_weight);
/* GeometryOps.cpp:411-425 */
int or_cubic_support(uint32_t in_w, uint32_t in_h, uint32_t out_w, uint32_t out_h,
                     or_rect output, or_rect* support);
/* GeometryOps.cpp:431-482: `src` is the full (in_w x in_h) input. */
int or_cubic_resize(const float* src, uint32_t in_w, uint32_t in_h, uint32_t out_w,
                    uint32_t out_h, or_rect output, float* out);

/* GeometryOps.cpp:46-76 rotation constants and taps. */
typedef struct or_rotation { double cx, cy, cosine, sine; uint32_t width, height; } or_rotation;
int or_rotation_prepare(double angle_degrees, uint32_t width, uint32_t height, or_rotation* r);
int or_rotate_support(const or_rotation* r, or_rect output, or_rect* support);
/* GeometryOps.cpp:119-143: `src` is the full (width x height) input. */
int or_rotate(const or_rotation* r, const float* src, or_rect output, float* out);

/* RawEngine.cpp:1399-1411 tile enumeration: fills up to `capacity` rects,
 * returns the number of tiles. */
size_t or_plan_tiles(or_rect viewport, uint32_t tile_size, or_rect* tiles, size_t capacity);

#ifdef __cplusplus
}
#endif
#endif
