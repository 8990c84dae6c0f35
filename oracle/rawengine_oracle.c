/* CPU restatement of RawEngine's tiled-render hot path -- TEST INFRASTRUCTURE.
 *
 * The oracle: used only by tests/, the smoke check and bench.py's CPU baseline,
 * as the checker.  Each function cites the reference (tylermcm/librawops) file
 * and lines whose algorithm it restates.  Floating-point expressions keep the
 * reference's evaluation order and are compiled with -ffp-contract=off, as the
 * reference's CMakeLists.txt:13 does for its numeric translation units, so the
 * results are bit-identical to the reference on the same inputs.  That claim
 * is pinned by tests/test_oracle_pin.py against the reference's own frozen
 * Menon fixtures and against the reference library built in oracle/_ref.
 */
#include "rawengine_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- metadata */

static int rect_inside(or_rect area, or_rect r) {
    return r.x >= area.x && r.y >= area.y &&
           (uint64_t)r.x + r.width <= (uint64_t)area.x + area.width &&
           (uint64_t)r.y + r.height <= (uint64_t)area.y + area.height;
}

/* RawEngine.cpp:223-250 */
int or_raw_normalize(or_raw_metadata* m, size_t sample_count) {
    if (!m->width || !m->height || m->pattern > 3 || m->cfa_phase_x > 1 || m->cfa_phase_y > 1)
        return OR_INVALID_ARGUMENT;
    if (m->row_stride_samples == 0) m->row_stride_samples = m->width;
    if (m->row_stride_samples < m->width) return OR_INVALID_ARGUMENT;
    or_rect* a = &m->active_area;
    if (!a->x && !a->y && !a->width && !a->height) {
        a->width = m->width;
        a->height = m->height;
    }
    if (!a->width || !a->height || (uint64_t)a->x + a->width > m->width ||
        (uint64_t)a->y + a->height > m->height)
        return OR_INVALID_ARGUMENT;
    for (int s = 0; s < 4; ++s)
        if (m->white_levels[s] <= m->black_levels[s]) return OR_INVALID_ARGUMENT;
    if ((uint64_t)m->row_stride_samples * m->height != sample_count) return OR_INVALID_ARGUMENT;
    return OR_OK;
}

/* RawEngine.cpp:74-77 */
int or_site_index(const or_raw_metadata* m, uint32_t x, uint32_t y) {
    return (int)((((y & 1u) + m->cfa_phase_y) & 1u) * 2u + (((x & 1u) + m->cfa_phase_x) & 1u));
}

/* RawEngine.cpp:79-87: the 2x2 top-left cell of each Bayer pattern (R=0 G=1 B=2). */
static const int k_pattern_colors[4][4] = {
    {0, 1, 1, 2}, /* RGGB */
    {2, 1, 1, 0}, /* BGGR */
    {1, 0, 2, 1}, /* GRBG */
    {1, 2, 0, 1}, /* GBRG */
};

int or_cfa_color(const or_raw_metadata* m, uint32_t x, uint32_t y) {
    return k_pattern_colors[m->pattern][or_site_index(m, x, y)];
}

/* RawEngine.cpp:89-97: float subtraction of the black level, float division
 * by the integer white-black span. */
float or_sample(const or_raw_metadata* m, const uint16_t* samples, uint32_t x, uint32_t y) {
    const int s = or_site_index(m, x, y);
    const uint16_t raw = samples[(size_t)y * m->row_stride_samples + x];
    const float numerator = (float)raw - (float)m->black_levels[s];
    const float span = (float)((int)m->white_levels[s] - (int)m->black_levels[s]);
    return numerator / span;
}

/* --------------------------------------------------------------- bilinear */

/* RawEngine.cpp:299-344 */
int or_bilinear(const or_raw_metadata* m, const uint16_t* samples, or_rect r, float* out) {
    const or_rect a = m->active_area;
    if (!rect_inside(a, r)) return OR_OUT_OF_RANGE;
    for (uint32_t row = 0; row < r.height; ++row) {
        const uint32_t y = r.y + row;
        for (uint32_t col = 0; col < r.width; ++col) {
            const uint32_t x = r.x + col;
            float* px = out + ((size_t)row * r.width + col) * 3;
            const int own = or_cfa_color(m, x, y);
            for (int ch = 0; ch < 3; ++ch) {
                if (own == ch) {
                    px[ch] = or_sample(m, samples, x, y);
                    continue;
                }
                float sum = 0.0f;
                int count = 0;
                for (int dy = -1; dy <= 1; ++dy) {
                    const int64_t yy = (int64_t)y + dy;
                    if (yy < a.y || yy >= (int64_t)a.y + a.height) continue;
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int64_t xx = (int64_t)x + dx;
                        if (xx < a.x || xx >= (int64_t)a.x + a.width) continue;
                        if (or_cfa_color(m, (uint32_t)xx, (uint32_t)yy) != ch) continue;
                        sum += or_sample(m, samples, (uint32_t)xx, (uint32_t)yy);
                        ++count;
                    }
                }
                px[ch] = count ? sum / (float)count : 0.0f;
            }
        }
    }
    return OR_OK;
}

/* ------------------------------------------------------------------ Menon */

/* A bounded double plane.  Reads outside its rectangle set `bad`, mirroring
 * the reference's logic_error on an undeclared support (MenonDemosaic.cpp:34-45). */
typedef struct plane {
    or_rect b;
    double* v;
} plane;

static int g_plane_bad;

static int plane_init(plane* p, or_rect b) {
    p->b = b;
    p->v = (double*)calloc((size_t)b.width * b.height + 1, sizeof(double));
    return p->v ? 0 : -1;
}

static double* plane_at(const plane* p, int64_t x, int64_t y) {
    if (x < p->b.x || y < p->b.y || x >= (int64_t)p->b.x + p->b.width ||
        y >= (int64_t)p->b.y + p->b.height) {
        g_plane_bad = 1;
        return p->v + (size_t)p->b.width * p->b.height; /* spare slot */
    }
    return p->v + (size_t)(y - p->b.y) * p->b.width + (size_t)(x - p->b.x);
}

/* MenonDemosaic.cpp:23-32: clip a halo'd rectangle to the active area. */
static or_rect support_rect(or_rect r, or_rect a, unsigned left, unsigned top, unsigned right,
                            unsigned bottom) {
    int64_t x0 = (int64_t)r.x - left, y0 = (int64_t)r.y - top;
    int64_t x1 = (int64_t)r.x + r.width + right, y1 = (int64_t)r.y + r.height + bottom;
    if (x0 < a.x) x0 = a.x;
    if (y0 < a.y) y0 = a.y;
    if (x1 > (int64_t)a.x + a.width) x1 = (int64_t)a.x + a.width;
    if (y1 > (int64_t)a.y + a.height) y1 = (int64_t)a.y + a.height;
    or_rect out = {(uint32_t)x0, (uint32_t)y0, (uint32_t)(x1 - x0), (uint32_t)(y1 - y0)};
    return out;
}

/* MenonDemosaic.cpp:60-66: whole-sample mirror about the active-area edges. */
static int64_t mirror_coord(int64_t v, int64_t origin, int64_t size) {
    if (size == 1) return origin;
    const int64_t period = 2 * (size - 1);
    int64_t folded = (v - origin) % period;
    if (folded < 0) folded += period;
    return origin + (folded < size ? folded : period - folded);
}

typedef struct sensor {
    const or_raw_metadata* m;
    or_rect a;
} sensor;

static int sensor_contains(const sensor* s, int64_t x, int64_t y) {
    return x >= s->a.x && y >= s->a.y && x < (int64_t)s->a.x + s->a.width &&
           y < (int64_t)s->a.y + s->a.height;
}

/* MenonDemosaic.cpp:67-72 */
static double sensor_get(const sensor* s, const plane* p, int64_t x, int64_t y) {
    if (!sensor_contains(s, x, y)) {
        x = mirror_coord(x, s->a.x, s->a.width);
        y = mirror_coord(y, s->a.y, s->a.height);
    }
    return *plane_at(p, x, y);
}

/* MenonDemosaic.cpp:73-80 (colour of any integer position, by parity). */
static int sensor_color(const sensor* s, int64_t x, int64_t y) {
    const unsigned site = ((((unsigned)(y & 1)) + s->m->cfa_phase_y) & 1u) * 2u +
                          ((((unsigned)(x & 1)) + s->m->cfa_phase_x) & 1u);
    return k_pattern_colors[s->m->pattern][site];
}

/* MenonDemosaic.cpp:148-150 */
static double pair_mean(const sensor* s, const plane* p, int64_t x, int64_t y, int dx, int dy) {
    return 0.5 * (sensor_get(s, p, x - dx, y - dy) + sensor_get(s, p, x + dx, y + dy));
}

/* Classifier terms, MenonDemosaic.cpp:130-132 (x, y, weight). */
static const int k_terms[8][3] = {{0, 2, 1}, {-2, 2, 1}, {-1, 1, 1}, {0, 0, 3},
                                  {-2, 0, 3}, {-1, -1, 1}, {0, -2, 1}, {-2, -2, 1}};

/* MenonDemosaic.cpp:89-174, one block.  Output pixels of block `r` are written
 * into `out` laid out over `request`. */
static int menon_block(const sensor* s, const uint16_t* samples, or_rect r, or_rect request,
                       float* out, uint8_t* dir) {
    const or_rect a = s->a;
    plane raw, gh, gv, ch, cv, green, horiz, dh, dv, red, blue;
    const or_rect raw_b = support_rect(r, a, 6, 6, 6, 6);
    const or_rect dir_b = support_rect(r, a, 4, 4, 4, 4);
    const or_rect green_b = support_rect(r, a, 2, 2, 2, 2);
    const or_rect dh_b = support_rect(green_b, a, 2, 2, 0, 2);
    const or_rect dv_b = support_rect(green_b, a, 2, 2, 2, 0);
    const or_rect col_b = support_rect(r, a, 1, 1, 1, 1);
    plane* all[] = {&raw, &gh, &gv, &ch, &cv, &green, &horiz, &dh, &dv, &red, &blue};
    const or_rect bounds[] = {raw_b, dir_b, dir_b, dir_b, dir_b, green_b, green_b, dh_b, dv_b,
                              col_b, col_b};
    int status = OR_OK;
    for (int i = 0; i < 11; ++i) all[i]->v = NULL;
    for (int i = 0; i < 11; ++i)
        if (plane_init(all[i], bounds[i])) { status = OR_LENGTH_ERROR; goto done; }

    /* raw: float samples held as double (MenonDemosaic.cpp:106) */
    for (int64_t y = raw_b.y; y < (int64_t)raw_b.y + raw_b.height; ++y)
        for (int64_t x = raw_b.x; x < (int64_t)raw_b.x + raw_b.width; ++x)
            *plane_at(&raw, x, y) = (double)or_sample(s->m, samples, (uint32_t)x, (uint32_t)y);

    /* directional green and chroma (MenonDemosaic.cpp:107-119) */
    for (int64_t y = dir_b.y; y < (int64_t)dir_b.y + dir_b.height; ++y)
        for (int64_t x = dir_b.x; x < (int64_t)dir_b.x + dir_b.width; ++x) {
            const double own = *plane_at(&raw, x, y);
            if (sensor_color(s, x, y) == 1) {
                *plane_at(&gh, x, y) = own;
                *plane_at(&gv, x, y) = own;
                continue;
            }
            const double h = 0.5 * (sensor_get(s, &raw, x - 1, y) + sensor_get(s, &raw, x + 1, y)) +
                             0.5 * own -
                             0.25 * (sensor_get(s, &raw, x - 2, y) + sensor_get(s, &raw, x + 2, y));
            const double v = 0.5 * (sensor_get(s, &raw, x, y - 1) + sensor_get(s, &raw, x, y + 1)) +
                             0.5 * own -
                             0.25 * (sensor_get(s, &raw, x, y - 2) + sensor_get(s, &raw, x, y + 2));
            *plane_at(&gh, x, y) = h;
            *plane_at(&gv, x, y) = v;
            *plane_at(&ch, x, y) = own - h;
            *plane_at(&cv, x, y) = own - v;
        }

    /* forward chroma gradients (MenonDemosaic.cpp:120-125) */
    for (int64_t y = dh_b.y; y < (int64_t)dh_b.y + dh_b.height; ++y)
        for (int64_t x = dh_b.x; x < (int64_t)dh_b.x + dh_b.width; ++x)
            *plane_at(&dh, x, y) = fabs(*plane_at(&ch, x, y) - sensor_get(s, &ch, x + 2, y));
    for (int64_t y = dv_b.y; y < (int64_t)dv_b.y + dv_b.height; ++y)
        for (int64_t x = dv_b.x; x < (int64_t)dv_b.x + dv_b.width; ++x)
            *plane_at(&dv, x, y) = fabs(*plane_at(&cv, x, y) - sensor_get(s, &cv, x, y + 2));

    /* direction classifier with zero-extended gradients (MenonDemosaic.cpp:126-147) */
    for (int64_t y = green_b.y; y < (int64_t)green_b.y + green_b.height; ++y)
        for (int64_t x = green_b.x; x < (int64_t)green_b.x + green_b.width; ++x) {
            if (sensor_color(s, x, y) == 1) {
                *plane_at(&horiz, x, y) = 1.0;
                *plane_at(&green, x, y) = *plane_at(&raw, x, y);
                continue;
            }
            double h = 0, v = 0;
            for (int t = 0; t < 8; ++t) {
                const double w = (double)k_terms[t][2];
                const int64_t hx = x + k_terms[t][0], hy = y + k_terms[t][1];
                const int64_t vx = x + k_terms[t][1], vy = y + k_terms[t][0];
                h += w * (sensor_contains(s, hx, hy) ? *plane_at(&dh, hx, hy) : 0.0);
                v += w * (sensor_contains(s, vx, vy) ? *plane_at(&dv, vx, vy) : 0.0);
            }
            const int horizontal = v >= h;
            *plane_at(&horiz, x, y) = horizontal ? 1.0 : 0.0;
            *plane_at(&green, x, y) = horizontal ? *plane_at(&gh, x, y) : *plane_at(&gv, x, y);
        }

    /* red/blue at every colour-support site (MenonDemosaic.cpp:151-161) */
    for (int64_t y = col_b.y; y < (int64_t)col_b.y + col_b.height; ++y)
        for (int64_t x = col_b.x; x < (int64_t)col_b.x + col_b.width; ++x) {
            const int own = sensor_color(s, x, y);
            if (own == 0) *plane_at(&red, x, y) = *plane_at(&raw, x, y);
            if (own == 2) *plane_at(&blue, x, y) = *plane_at(&raw, x, y);
            if (own == 1) {
                const int red_h = sensor_color(s, x + 1, y) == 0;
                const int dx = red_h ? 1 : 0, dy = red_h ? 0 : 1;
                const double g = *plane_at(&green, x, y);
                *plane_at(&red, x, y) = g + pair_mean(s, &raw, x, y, dx, dy) -
                                        pair_mean(s, &green, x, y, dx, dy);
                *plane_at(&blue, x, y) = g + pair_mean(s, &raw, x, y, dy, dx) -
                                         pair_mean(s, &green, x, y, dy, dx);
            }
        }

    /* final opposite colour at R/B sites and float cast (MenonDemosaic.cpp:162-173) */
    for (int64_t y = r.y; y < (int64_t)r.y + r.height; ++y)
        for (int64_t x = r.x; x < (int64_t)r.x + r.width; ++x) {
            const int own = sensor_color(s, x, y);
            const int horizontal = *plane_at(&horiz, x, y) != 0.0;
            const int dx = horizontal ? 1 : 0, dy = horizontal ? 0 : 1;
            double rr = *plane_at(&red, x, y), bb = *plane_at(&blue, x, y);
            if (own == 2)
                rr = bb + pair_mean(s, &red, x, y, dx, dy) - pair_mean(s, &blue, x, y, dx, dy);
            if (own == 0)
                bb = rr + pair_mean(s, &blue, x, y, dx, dy) - pair_mean(s, &red, x, y, dx, dy);
            const size_t i = (size_t)(y - request.y) * request.width + (size_t)(x - request.x);
            out[i * 3 + 0] = (float)rr;
            out[i * 3 + 1] = (float)*plane_at(&green, x, y);
            out[i * 3 + 2] = (float)bb;
            if (dir) dir[i] = (uint8_t)horizontal;
        }
done:
    for (int i = 0; i < 11; ++i) free(all[i]->v);
    return status;
}

/* MenonDemosaic.cpp:177-218 and the singleton-axis bilinear route of
 * RawEngine.cpp:299-304.  Blocks of 256 keep the planes bounded; results do
 * not depend on the blocking. */
int or_menon(const or_raw_metadata* m, const uint16_t* samples, or_rect r, float* out,
             uint8_t* horizontal) {
    if (!rect_inside(m->active_area, r)) return OR_OUT_OF_RANGE;
    if (m->active_area.width <= 1 || m->active_area.height <= 1) {
        if (horizontal) memset(horizontal, 1, (size_t)r.width * r.height);
        return or_bilinear(m, samples, r, out);
    }
    sensor s = {m, m->active_area};
    g_plane_bad = 0;
    const uint32_t block = 256;
    for (uint64_t by = r.y; by < (uint64_t)r.y + r.height; by += block)
        for (uint64_t bx = r.x; bx < (uint64_t)r.x + r.width; bx += block) {
            or_rect b = {(uint32_t)bx, (uint32_t)by,
                         (uint32_t)((uint64_t)r.x + r.width - bx < block ? (uint64_t)r.x + r.width - bx : block),
                         (uint32_t)((uint64_t)r.y + r.height - by < block ? (uint64_t)r.y + r.height - by : block)};
            const int st = menon_block(&s, samples, b, r, out, horizontal);
            if (st) return st;
        }
    return g_plane_bad ? OR_DOMAIN_ERROR : OR_OK;
}

/* RawEngine.cpp:49-64 */
static int expand_rect(or_rect output, or_rect bounds, uint32_t radius, or_rect* out) {
    if (!rect_inside(bounds, output)) return OR_OUT_OF_RANGE;
    *out = support_rect(output, bounds, radius, radius, radius, radius);
    return OR_OK;
}

/* RawEngine.cpp:290-297 */
int or_raw_input_region(const or_raw_metadata* m, int menon, or_rect output, or_rect* region) {
    const or_rect a = m->active_area;
    const uint32_t radius = menon && a.width > 1 && a.height > 1 ? 6u : 1u;
    return expand_rect(output, a, radius, region);
}

/* ------------------------------------------------------------ point stages */

/* RawEngine.cpp:417-431 */
void or_white_balance(float* rgb, size_t pixels, float r, float g, float b) {
    for (size_t i = 0; i < pixels; ++i) {
        rgb[i * 3 + 0] *= r;
        rgb[i * 3 + 1] *= g;
        rgb[i * 3 + 2] *= b;
    }
}

/* RawEngine.cpp:465-466 */
float or_exposure_multiplier(float stops) { return exp2f(stops); }

/* RawEngine.cpp:488-500 */
void or_scale(float* rgb, size_t count, float multiplier) {
    for (size_t i = 0; i < count; ++i) rgb[i] *= multiplier;
}

typedef double mat3[9];

/* RawEngine.cpp:118-125 */
static void mat_mul(const double* a, const double* b, double* out) {
    double t[9] = {0};
    for (int row = 0; row < 3; ++row)
        for (int col = 0; col < 3; ++col)
            for (int k = 0; k < 3; ++k) t[row * 3 + col] += a[row * 3 + k] * b[k * 3 + col];
    memcpy(out, t, sizeof(t));
}

/* RawEngine.cpp:127-131 */
static void mat_vec(const double* a, const double* v, double* out) {
    const double t0 = a[0] * v[0] + a[1] * v[1] + a[2] * v[2];
    const double t1 = a[3] * v[0] + a[4] * v[1] + a[5] * v[2];
    const double t2 = a[6] * v[0] + a[7] * v[1] + a[8] * v[2];
    out[0] = t0; out[1] = t1; out[2] = t2;
}

/* RawEngine.cpp:133-150 (cofactor inverse, singular below |det| 1e-12) */
static int mat_inverse(const double* m, double* out) {
    const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                       m[2] * (m[3] * m[7] - m[4] * m[6]);
    if (!isfinite(det) || fabs(det) < 1e-12) return OR_INVALID_ARGUMENT;
    const double d = 1.0 / det;
    double t[9] = {(m[4] * m[8] - m[5] * m[7]) * d, (m[2] * m[7] - m[1] * m[8]) * d,
                   (m[1] * m[5] - m[2] * m[4]) * d, (m[5] * m[6] - m[3] * m[8]) * d,
                   (m[0] * m[8] - m[2] * m[6]) * d, (m[2] * m[3] - m[0] * m[5]) * d,
                   (m[3] * m[7] - m[4] * m[6]) * d, (m[1] * m[6] - m[0] * m[7]) * d,
                   (m[0] * m[4] - m[1] * m[3]) * d};
    memcpy(out, t, sizeof(t));
    return OR_OK;
}

/* RawEngine.cpp:152-154 */
static void xyz_white(double x, double y, double* out) {
    out[0] = x / y; out[1] = 1.0; out[2] = (1.0 - x - y) / y;
}

/* RawEngine.cpp:156-169: primaries (x,y) of R,G,B and white (wx,wy). */
static void rgb_to_xyz(const double xy[6], double wx, double wy, double* out) {
    double basis[9], inv[9], white[3], scales[3];
    for (int col = 0; col < 3; ++col) {
        const double x = xy[2 * col], y = xy[2 * col + 1];
        basis[col] = x / y;
        basis[3 + col] = 1.0;
        basis[6 + col] = (1.0 - x - y) / y;
    }
    mat_inverse(basis, inv);
    xyz_white(wx, wy, white);
    mat_vec(inv, white, scales);
    for (int row = 0; row < 3; ++row)
        for (int col = 0; col < 3; ++col) basis[row * 3 + col] *= scales[col];
    memcpy(out, basis, sizeof(basis));
}

/* Chromaticities: ICC ROMM (ProPhoto), ITU-R BT.2020, sRGB (RawEngine.cpp:188-211). */
static const double k_prophoto[6] = {0.7347, 0.2653, 0.1596, 0.8404, 0.0366, 0.0001};
static const double k_rec2020[6] = {0.708, 0.292, 0.170, 0.797, 0.131, 0.046};
static const double k_srgb[6] = {0.640, 0.330, 0.300, 0.600, 0.150, 0.060};

/* RawEngine.cpp:171-181 Bradford D50 -> D65 */
static void d50_to_d65(double* out) {
    static const double bradford[9] = {0.8951, 0.2664, -0.1614, -0.7502, 1.7135,
                                       0.0367, 0.0389, -0.0685, 1.0296};
    double w50[3], w65[3], d50[3], d65[3], inv[9], t[9];
    xyz_white(0.3457, 0.3585, w50);
    xyz_white(0.3127, 0.3290, w65);
    mat_vec(bradford, w50, d50);
    mat_vec(bradford, w65, d65);
    const double scale[9] = {d65[0] / d50[0], 0, 0, 0, d65[1] / d50[1], 0, 0, 0, d65[2] / d50[2]};
    mat_inverse(bradford, inv);
    mat_mul(scale, bradford, t);
    mat_mul(inv, t, out);
}

/* RawEngine.cpp:183-196 */
static int xyz_d50_to_working(int target, double* out) {
    double m[9], d[9];
    if (target == 0) {
        rgb_to_xyz(k_prophoto, 0.3457, 0.3585, m);
        return mat_inverse(m, out);
    }
    if (target == 1) {
        rgb_to_xyz(k_rec2020, 0.3127, 0.3290, m);
        double inv[9];
        mat_inverse(m, inv);
        d50_to_d65(d);
        mat_mul(inv, d, out);
        return OR_OK;
    }
    return OR_INVALID_ARGUMENT;
}

static int to_float_matrix(const double* d, float* out) {
    for (int i = 0; i < 9; ++i) {
        if (!isfinite(d[i]) || fabs(d[i]) > FLT_MAX) return OR_INVALID_ARGUMENT;
        out[i] = (float)d[i];
    }
    return OR_OK;
}

/* RawEngine.cpp:502-530 */
int or_camera_to_working_matrix(const double camera_to_xyz[9], int target, float out[9]) {
    double inv[9], w[9], composed[9];
    for (int i = 0; i < 9; ++i)
        if (!isfinite(camera_to_xyz[i])) return OR_INVALID_ARGUMENT;
    if (mat_inverse(camera_to_xyz, inv)) return OR_INVALID_ARGUMENT;
    if (xyz_d50_to_working(target, w)) return OR_INVALID_ARGUMENT;
    mat_mul(w, camera_to_xyz, composed);
    return to_float_matrix(composed, out);
}

/* RawEngine.cpp:198-214 */
int or_working_to_srgb_matrix(int source, float out[9]) {
    double srgb[9], inv[9], src[9], d[9], t[9], r[9];
    rgb_to_xyz(k_srgb, 0.3127, 0.3290, srgb);
    mat_inverse(srgb, inv);
    if (source == 0) {
        rgb_to_xyz(k_prophoto, 0.3457, 0.3585, src);
        d50_to_d65(d);
        mat_mul(d, src, t);
        mat_mul(inv, t, r);
    } else if (source == 1) {
        rgb_to_xyz(k_rec2020, 0.3127, 0.3290, src);
        mat_mul(inv, src, r);
    } else {
        return OR_INVALID_ARGUMENT;
    }
    for (int i = 0; i < 9; ++i) out[i] = (float)r[i];
    return OR_OK;
}

/* RawEngine.cpp:216-219 */
int or_working_to_working_matrix(int source, int target, float out[9]) {
    double s[9], t[9], inv[9], r[9];
    if (xyz_d50_to_working(source, s) || xyz_d50_to_working(target, t)) return OR_INVALID_ARGUMENT;
    mat_inverse(s, inv);
    mat_mul(t, inv, r);
    for (int i = 0; i < 9; ++i) out[i] = (float)r[i];
    return OR_OK;
}

/* RawEngine.cpp:539-545 */
void or_matrix3(float* rgb, size_t pixels, const float m[9]) {
    for (size_t i = 0; i < pixels; ++i) {
        float* p = rgb + i * 3;
        const float r = p[0], g = p[1], b = p[2];
        p[0] = m[0] * r + m[1] * g + m[2] * b;
        p[1] = m[3] * r + m[4] * g + m[5] * b;
        p[2] = m[6] * r + m[7] * g + m[8] * b;
    }
}

/* RawEngine.cpp:705-758 */
void or_tone_curve(float* rgb, size_t count, float shoulder, float gamma) {
    const float inverse_gamma = 1.0f / gamma;
    for (size_t i = 0; i < count; ++i) {
        const float linear = rgb[i];
        const float magnitude = fabsf(linear);
        const float compressed = magnitude / (magnitude + shoulder);
        const float mapped = inverse_gamma == 1.0f ? compressed : powf(compressed, inverse_gamma);
        rgb[i] = copysignf(mapped, linear);
    }
}

/* RawEngine.cpp:1223-1233 */
int or_output_clip(float* rgb, size_t count) {
    for (size_t i = 0; i < count; ++i) {
        if (!isfinite(rgb[i])) return OR_DOMAIN_ERROR;
        rgb[i] = rgb[i] < 0.0f ? 0.0f : (rgb[i] > 1.0f ? 1.0f : rgb[i]);
    }
    return OR_OK;
}

/* RawEngine.cpp:1254-1277 */
int or_srgb_encode(float* rgb, size_t count) {
    for (size_t i = 0; i < count; ++i)
        if (!isfinite(rgb[i])) return OR_DOMAIN_ERROR;
    for (size_t i = 0; i < count; ++i) {
        const float v = rgb[i];
        const float linear = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
        rgb[i] = linear <= 0.0031308f ? 12.92f * linear
                                      : 1.055f * powf(linear, 1.0f / 2.4f) - 0.055f;
    }
    return OR_OK;
}

/* ---------------------------------------------------------- extended curves */

/* ToneOps.cpp:17-31 */
static int validate_curve(const double* k, uint32_t n) {
    if (n < 2 || n > 256) return OR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < n; ++i) {
        const double x = k[2 * i], y = k[2 * i + 1];
        if (!isfinite(x) || !isfinite(y) || fabs(x) > 65536 || fabs(y) > 65536) return OR_INVALID_ARGUMENT;
        if (i) {
            const double px = k[2 * i - 2], py = k[2 * i - 1];
            if (!(x > px)) return OR_INVALID_ARGUMENT;
            const double slope = (y - py) / (x - px);
            if (!isfinite(slope) || fabs(slope) > 65536) return OR_INVALID_ARGUMENT;
        }
    }
    return OR_OK;
}

/* ToneOps.cpp:795-816: slopes, shape-preserving tangents, Bezier controls. */
int or_curves_prepare(or_curves* c) {
    if (c->interpolation != 0 && c->interpolation != 1) return OR_INVALID_ARGUMENT;
    for (int k = 0; k < 4; ++k) {
        const double* kn = c->knots[k];
        const uint32_t n = c->count[k];
        if (validate_curve(kn, n)) return OR_INVALID_ARGUMENT;
        c->identity[k] = 1;
        for (uint32_t i = 0; i < n; ++i)
            if (kn[2 * i] != kn[2 * i + 1]) c->identity[k] = 0;
        for (uint32_t i = 1; i < n; ++i)
            c->slopes[k][i - 1] = (kn[2 * i + 1] - kn[2 * i - 1]) / (kn[2 * i] - kn[2 * i - 2]);
        if (c->interpolation == 0) continue;
        double tangent[256];
        tangent[0] = c->slopes[k][0];
        for (uint32_t i = 1; i + 1 < n; ++i) {
            const double a = c->slopes[k][i - 1], b = c->slopes[k][i];
            tangent[i] = (a == 0 || b == 0 || signbit(a) != signbit(b))
                             ? 0
                             : copysign(fmin(fabs(a), fabs(b)), a);
        }
        tangent[n - 1] = c->slopes[k][n - 2];
        for (uint32_t i = 0; i + 1 < n; ++i) {
            const double h = kn[2 * i + 2] - kn[2 * i];
            c->controls[k][i][0] = kn[2 * i + 1] + (h * tangent[i]) / 3;
            c->controls[k][i][1] = kn[2 * i + 3] - (h * tangent[i + 1]) / 3;
        }
    }
    return OR_OK;
}

/* ToneOps.cpp:787-791 */
static double cubic_blend(double a, double b, double t) {
    if (a == b || t == 0) return a;
    if (t == 1) return b;
    return t <= .5 ? a + t * (b - a) : b + (1 - t) * (a - b);
}

/* ToneOps.cpp:821-832 */
double or_curve_map(const or_curves* c, unsigned k, double value) {
    if (c->identity[k]) return value;
    const double* kn = c->knots[k];
    const uint32_t n = c->count[k];
    uint32_t next = 0; /* upper_bound: first knot with x > value */
    while (next < n && !(value < kn[2 * next])) ++next;
    const uint32_t left = next == 0 ? 0 : next - 1;
    const uint32_t i = left < n - 2 ? left : n - 2;
    if (value == kn[2 * left]) return kn[2 * left + 1];
    if (c->interpolation == 0 || value < kn[0] || value > kn[2 * (n - 1)])
        return c->slopes[k][i] == 0 ? kn[2 * left + 1]
                                    : kn[2 * left + 1] + (value - kn[2 * left]) * c->slopes[k][i];
    const double t = (value - kn[2 * i]) / (kn[2 * i + 2] - kn[2 * i]);
    const double c0 = c->controls[k][i][0], c1 = c->controls[k][i][1];
    const double a = cubic_blend(kn[2 * i + 1], c0, t), b = cubic_blend(c0, c1, t),
                 d = cubic_blend(c1, kn[2 * i + 3], t);
    return cubic_blend(cubic_blend(a, b, t), cubic_blend(b, d, t), t);
}

/* ToneOps.cpp:165-184 (finite input) and 833-844 (master then channel, one cast). */
int or_curves_apply(const or_curves* c, float* rgb, size_t count) {
    for (size_t i = 0; i < count; ++i)
        if (!isfinite(rgb[i])) return OR_INVALID_ARGUMENT;
    for (size_t i = 0; i < count; ++i) {
        const unsigned ch = (unsigned)(i % 3) + 1;
        if (c->identity[0] && c->identity[ch]) continue;
        const double master = or_curve_map(c, 0, (double)rgb[i]);
        if (!isfinite(master)) return OR_INVALID_ARGUMENT;
        const double mapped = or_curve_map(c, ch, master);
        if (!isfinite(mapped) || fabs(mapped) > FLT_MAX) return OR_INVALID_ARGUMENT;
        const float rounded = (float)mapped;
        if (!isfinite(rounded)) return OR_INVALID_ARGUMENT;
        rgb[i] = rounded;
    }
    return OR_OK;
}

/* -------------------------------------------------------------- mip levels */

/* RawEngine.cpp:31-43 */
int or_request_bounds(or_rect s, uint32_t mip, uint32_t quality, or_rect* out) {
    if (mip == 0 && (quality == 0 || quality == 1)) {
        *out = s;
        return OR_OK;
    }
    if (mip >= 1 && mip <= 2 && quality == 0) {
        const uint32_t scale = 1u << mip;
        or_rect r = {0, 0, s.width / scale + (s.width % scale != 0),
                     s.height / scale + (s.height % scale != 0)};
        *out = r;
        return OR_OK;
    }
    return OR_INVALID_ARGUMENT;
}

/* RawEngine.cpp:563-578 */
int or_mip_native_region(or_rect area, uint32_t mip, or_rect output, or_rect* native) {
    or_rect reduced;
    if (or_request_bounds(area, mip, 0, &reduced)) return OR_INVALID_ARGUMENT;
    if (!rect_inside(reduced, output)) return OR_OUT_OF_RANGE;
    const uint64_t scale = 1u << mip;
    uint64_t left = (uint64_t)output.x * scale, top = (uint64_t)output.y * scale;
    uint64_t right = ((uint64_t)output.x + output.width) * scale;
    uint64_t bottom = ((uint64_t)output.y + output.height) * scale;
    if (left > area.width) left = area.width;
    if (top > area.height) top = area.height;
    if (right > area.width) right = area.width;
    if (bottom > area.height) bottom = area.height;
    or_rect r = {(uint32_t)(area.x + left), (uint32_t)(area.y + top), (uint32_t)(right - left),
                 (uint32_t)(bottom - top)};
    *native = r;
    return OR_OK;
}

/* RawEngine.cpp:585-600: double sums in row-major footprint order, actual counts. */
void or_mip_reduce(const float* native, or_rect mapped, uint32_t mip, or_rect output, float* out) {
    const uint32_t scale = 1u << mip;
    for (uint32_t y = 0; y < output.height; ++y)
        for (uint32_t x = 0; x < output.width; ++x) {
            double sums[3] = {0, 0, 0};
            uint32_t count = 0;
            const uint64_t y1 = (uint64_t)(y + 1) * scale < mapped.height ? (uint64_t)(y + 1) * scale : mapped.height;
            const uint64_t x1 = (uint64_t)(x + 1) * scale < mapped.width ? (uint64_t)(x + 1) * scale : mapped.width;
            for (uint64_t sy = (uint64_t)y * scale; sy < y1; ++sy)
                for (uint64_t sx = (uint64_t)x * scale; sx < x1; ++sx) {
                    const float* p = native + ((size_t)sy * mapped.width + sx) * 3;
                    for (int c = 0; c < 3; ++c) sums[c] += p[c];
                    ++count;
                }
            float* o = out + ((size_t)y * output.width + x) * 3;
            for (int c = 0; c < 3; ++c) o[c] = (float)(sums[c] / count);
        }
}

/* ---------------------------------------------------------- guided filter */

/* SpatialOps.cpp:14-41 */
static int bounded_rect(or_rect r) {
    return r.width && r.height && (uint64_t)r.x + r.width <= (1ull << 32) &&
           (uint64_t)r.y + r.height <= (1ull << 32);
}

static int spatial_expanded(or_rect r, or_rect image, uint32_t rx, uint32_t ry, or_rect* out) {
    if (!bounded_rect(r) || !bounded_rect(image)) return OR_INVALID_ARGUMENT;
    if (!rect_inside(image, r)) return OR_OUT_OF_RANGE;
    *out = support_rect(r, image, rx, ry, rx, ry);
    return OR_OK;
}

/* SpatialOps.cpp:164-167 */
int or_guided_filter_region(or_rect output, or_rect image, uint32_t radius, or_rect* needed) {
    if (radius > 8) return OR_INVALID_ARGUMENT;
    return spatial_expanded(output, image, 2 * radius, 2 * radius, needed);
}

typedef struct gf_coefficient {
    double mean_y_delta, mean_p_delta[3], slope[3];
} gf_coefficient;

/* SpatialOps.cpp:217-223: working-Y of an RGB delta. */
static double y_delta(const double d[3], double wr, double wb) {
    const double dr = d[0] - d[1], db = d[2] - d[1];
    const double first = d[1] + wr * dr;
    return first + wb * db;
}

/* SpatialOps.cpp:168-287.  Radius up to 8 is the reference's contract; the
 * restatement accepts any radius (for out-of-contract configurations the
 * caller checks radius itself). */
int or_guided_filter(const float* in, or_rect needed, or_rect output, or_rect image,
                     uint32_t radius, double eps, int prophoto, float* out) {
    if (!isfinite(eps) || eps < 0x1p-24 || eps > 65536.0) return OR_INVALID_ARGUMENT;
    or_rect centers, want;
    int st = spatial_expanded(output, image, radius, radius, &centers);
    if (st) return st;
    st = spatial_expanded(output, image, 2 * radius, 2 * radius, &want);
    if (st) return st;
    if (want.x != needed.x || want.y != needed.y || want.width != needed.width ||
        want.height != needed.height)
        return OR_INVALID_ARGUMENT;
    for (size_t i = 0; i < (size_t)needed.width * needed.height * 3; ++i)
        if (!isfinite(in[i])) return OR_INVALID_ARGUMENT;
    if (radius == 0) {
        memcpy(out, in, (size_t)needed.width * needed.height * 3 * sizeof(float));
        return OR_OK;
    }
    const double wr = prophoto ? 0.28807112822929337 : 0.26270021201126703;
    const double wb = prophoto ? 0.00008565396060525903 : 0.059301716469861945;
    gf_coefficient* table =
        (gf_coefficient*)malloc(sizeof(gf_coefficient) * (size_t)centers.width * centers.height);
    if (!table) return OR_LENGTH_ERROR;
#define GF_AT(px_, py_) (in + (((size_t)((py_) - needed.y) * needed.width + (size_t)((px_) - needed.x)) * 3))
    st = OR_OK;
    for (uint64_t ky = centers.y; ky < (uint64_t)centers.y + centers.height && !st; ++ky)
        for (uint64_t kx = centers.x; kx < (uint64_t)centers.x + centers.width; ++kx) {
            or_rect one = {(uint32_t)kx, (uint32_t)ky, 1, 1}, w;
            spatial_expanded(one, image, radius, radius, &w);
            const double count = (double)((uint64_t)w.width * w.height);
            const float* k = GF_AT(kx, ky);
            double sg = 0, sp[3] = {0, 0, 0};
            for (uint64_t y = w.y; y < (uint64_t)w.y + w.height; ++y)
                for (uint64_t x = w.x; x < (uint64_t)w.x + w.width; ++x) {
                    const float* p = GF_AT(x, y);
                    const double d[3] = {(double)p[0] - (double)k[0], (double)p[1] - (double)k[1],
                                         (double)p[2] - (double)k[2]};
                    sg += y_delta(d, wr, wb);
                    for (int c = 0; c < 3; ++c) sp[c] += d[c];
                }
            gf_coefficient co;
            co.mean_y_delta = sg / count;
            if (!isfinite(co.mean_y_delta)) { st = OR_OVERFLOW_ERROR; break; }
            for (int c = 0; c < 3; ++c) {
                co.mean_p_delta[c] = sp[c] / count;
                if (!isfinite(co.mean_p_delta[c])) st = OR_OVERFLOW_ERROR;
            }
            double vv = 0, cov[3] = {0, 0, 0};
            for (uint64_t y = w.y; y < (uint64_t)w.y + w.height; ++y)
                for (uint64_t x = w.x; x < (uint64_t)w.x + w.width; ++x) {
                    const float* p = GF_AT(x, y);
                    const double d[3] = {(double)p[0] - (double)k[0], (double)p[1] - (double)k[1],
                                         (double)p[2] - (double)k[2]};
                    const double dy = y_delta(d, wr, wb) - co.mean_y_delta;
                    vv += dy * dy;
                    for (int c = 0; c < 3; ++c) {
                        const double dp = d[c] - co.mean_p_delta[c];
                        cov[c] += dy * dp;
                    }
                }
            const double variance = vv / count, denominator = variance + eps;
            if (!isfinite(variance) || !isfinite(denominator) || variance < 0 || denominator < eps) {
                st = OR_OVERFLOW_ERROR;
                break;
            }
            for (int c = 0; c < 3; ++c) {
                co.slope[c] = (cov[c] / count) / denominator;
                if (!isfinite(co.slope[c])) st = OR_OVERFLOW_ERROR;
            }
            table[(size_t)(ky - centers.y) * centers.width + (size_t)(kx - centers.x)] = co;
        }
    for (uint64_t y = output.y; y < (uint64_t)output.y + output.height && !st; ++y)
        for (uint64_t x = output.x; x < (uint64_t)output.x + output.width; ++x) {
            or_rect one = {(uint32_t)x, (uint32_t)y, 1, 1}, w;
            spatial_expanded(one, image, radius, radius, &w);
            const double count = (double)((uint64_t)w.width * w.height);
            const float* p = GF_AT(x, y);
            double correction[3] = {0, 0, 0};
            for (uint64_t ky = w.y; ky < (uint64_t)w.y + w.height; ++ky)
                for (uint64_t kx = w.x; kx < (uint64_t)w.x + w.width; ++kx) {
                    const gf_coefficient* co =
                        &table[(size_t)(ky - centers.y) * centers.width + (size_t)(kx - centers.x)];
                    const float* k = GF_AT(kx, ky);
                    const double d[3] = {(double)k[0] - (double)p[0], (double)k[1] - (double)p[1],
                                         (double)k[2] - (double)p[2]};
                    const double rev[3] = {(double)p[0] - (double)k[0], (double)p[1] - (double)k[1],
                                           (double)p[2] - (double)k[2]};
                    const double guide = y_delta(rev, wr, wb) - co->mean_y_delta;
                    for (int c = 0; c < 3; ++c) {
                        double term = d[c] + co->mean_p_delta[c];
                        if (co->slope[c] != 0) term += co->slope[c] * guide;
                        correction[c] += term;
                    }
                }
            float* o = out + ((size_t)(y - output.y) * output.width + (size_t)(x - output.x)) * 3;
            for (int c = 0; c < 3; ++c) {
                const double delta = correction[c] / count;
                if (!isfinite(delta)) { st = OR_OVERFLOW_ERROR; break; }
                if (delta == 0) { o[c] = p[c]; continue; }
                const double value = (double)p[c] + delta;
                if (!isfinite(value) || value < -(double)FLT_MAX || value > (double)FLT_MAX) {
                    st = OR_OVERFLOW_ERROR;
                    break;
                }
                o[c] = (float)value;
                if (!isfinite(o[c])) { st = OR_OVERFLOW_ERROR; break; }
            }
        }
#undef GF_AT
    free(table);
    return st;
}

/* ------------------------------------------------------- local statistics */

/* SpatialOps.cpp:52-71 */
typedef struct moment {
    uint32_t count;
    double mean, m2;
} moment;

static void moment_add(moment* m, float value) {
    if (!isfinite(value)) return;
    ++m->count;
    const double delta = (double)value - m->mean;
    m->mean += delta / m->count;
    m->m2 += delta * ((double)value - m->mean);
}

static void moment_merge(moment* a, const moment* b) {
    if (!b->count) return;
    if (!a->count) { *a = *b; return; }
    const uint32_t total = a->count + b->count;
    const double delta = b->mean - a->mean;
    a->m2 += b->m2 + delta * delta * ((double)a->count * b->count / total);
    a->mean += delta * ((double)b->count / total);
    a->count = total;
}

/* SpatialOps.cpp:74-77 */
int or_local_statistics_region(or_rect output, or_rect image, uint32_t radius, or_rect* needed) {
    if (radius > 8) return OR_INVALID_ARGUMENT;
    return spatial_expanded(output, image, radius, radius, needed);
}

/* SpatialOps.cpp:79-121 (radius checked by the caller for out-of-contract use) */
int or_local_statistics(const float* in, or_rect needed, or_rect output, or_rect image,
                        uint32_t radius, double* mean, double* variance, uint32_t* count) {
    or_rect want;
    int st = spatial_expanded(output, image, radius, radius, &want);
    if (st) return st;
    if (want.x != needed.x || want.y != needed.y || want.width != needed.width ||
        want.height != needed.height)
        return OR_INVALID_ARGUMENT;
    moment* h = (moment*)calloc((size_t)output.width * needed.height * 3, sizeof(moment));
    if (!h) return OR_LENGTH_ERROR;
    for (uint32_t row = 0; row < needed.height; ++row)
        for (uint32_t col = 0; col < output.width; ++col) {
            const uint64_t x = (uint64_t)output.x + col;
            const int64_t left = (int64_t)x - radius < (int64_t)image.x ? (int64_t)image.x : (int64_t)x - radius;
            const uint64_t last = (uint64_t)image.x + image.width - 1;
            const uint64_t right = x + radius < last ? x + radius : last;
            moment* t = h + ((size_t)row * output.width + col) * 3;
            for (uint64_t xx = (uint64_t)left; xx <= right; ++xx) {
                const float* p = in + ((size_t)row * needed.width + (size_t)(xx - needed.x)) * 3;
                for (int c = 0; c < 3; ++c) moment_add(&t[c], p[c]);
            }
        }
    for (uint32_t row = 0; row < output.height; ++row) {
        const uint64_t y = (uint64_t)output.y + row;
        const int64_t top = (int64_t)y - radius < (int64_t)image.y ? (int64_t)image.y : (int64_t)y - radius;
        const uint64_t last = (uint64_t)image.y + image.height - 1;
        const uint64_t bottom = y + radius < last ? y + radius : last;
        for (uint32_t col = 0; col < output.width; ++col) {
            moment total[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            for (uint64_t yy = (uint64_t)top; yy <= bottom; ++yy) {
                const moment* s = h + ((size_t)(yy - needed.y) * output.width + col) * 3;
                for (int c = 0; c < 3; ++c) moment_merge(&total[c], &s[c]);
            }
            const size_t t = ((size_t)row * output.width + col) * 3;
            for (int c = 0; c < 3; ++c) {
                count[t + c] = total[c].count;
                mean[t + c] = total[c].count ? total[c].mean : NAN;
                variance[t + c] = total[c].count ? fmax(0.0, total[c].m2 / total[c].count) : NAN;
            }
        }
    }
    free(h);
    return OR_OK;
}

/* --------------------------------------------------------------- geometry */

/* GeometryOps.cpp:362-389 */
int or_cubic_axis(uint32_t input, uint32_t output, uint32_t index, uint32_t* center,
                  uint32_t* tap_index, double* tap_weight) {
    if (input == output) {
        *center = index;
        tap_index[0] = index;
        tap_weight[0] = 1;
        return 1;
    }
    double z = (((double)index + .5) * (double)input / (double)output) - .5;
    if (z < 0.) z = 0.;
    if (z > (double)(input - 1)) z = (double)(input - 1);
    const double ratio = (double)input / (double)output;
    const double scale = ratio > 1. ? ratio : 1.;
    *center = (uint32_t)floor(z);
    const int64_t first = (int64_t)floor(z - 2 * scale);
    const int64_t last = (int64_t)ceil(z + 2 * scale);
    double total = 0;
    int count = 0;
    for (int64_t i = first; i <= last; ++i) {
        const double distance = fabs(((double)i - z) / scale);
        double value = 0;
        if (distance < 1) value = ((1.5 * distance - 2.5) * distance) * distance + 1;
        else if (distance < 2) value = (-.5 * (distance - 1)) * ((distance - 2) * (distance - 2));
        const double weight = value / scale;
        if (weight == 0) continue;
        if (count == 18) return -OR_INVALID_ARGUMENT;
        const int64_t clamped = i < 0 ? 0 : (i > (int64_t)input - 1 ? (int64_t)input - 1 : i);
        tap_index[count] = (uint32_t)clamped;
        tap_weight[count] = weight;
        ++count;
        total = total + weight;
    }
    if (!isfinite(total) || total <= .5) return -OR_INVALID_ARGUMENT;
    for (int i = 0; i < count; ++i) {
        tap_weight[i] = tap_weight[i] / total;
        if (!isfinite(tap_weight[i]) || fabs(tap_weight[i]) > 4) return -OR_INVALID_ARGUMENT;
    }
    return count;
}

/* GeometryOps.cpp:411-425 */
int or_cubic_support(uint32_t in_w, uint32_t in_h, uint32_t out_w, uint32_t out_h,
                     or_rect output, or_rect* support) {
    uint32_t idx[18];
    double w[18];
    uint32_t center;
    uint32_t lo[2] = {in_w, in_h}, hi[2] = {0, 0};
    const uint32_t ins[2] = {in_w, in_h}, outs[2] = {out_w, out_h};
    const uint32_t starts[2] = {output.x, output.y}, lens[2] = {output.width, output.height};
    for (int a = 0; a < 2; ++a)
        for (uint64_t i = starts[a]; i < (uint64_t)starts[a] + lens[a]; ++i) {
            const int n = or_cubic_axis(ins[a], outs[a], (uint32_t)i, &center, idx, w);
            if (n < 0) return -n;
            for (int j = 0; j < n; ++j) {
                if (idx[j] < lo[a]) lo[a] = idx[j];
                if (idx[j] > hi[a]) hi[a] = idx[j];
            }
        }
    or_rect r = {lo[0], lo[1], hi[0] - lo[0] + 1, hi[1] - lo[1] + 1};
    *support = r;
    return OR_OK;
}

/* GeometryOps.cpp:446-481: horizontal double pass, then vertical, ordered
 * delta accumulation around the centre tap, one float32 rounding. */
int or_cubic_resize(const float* src, uint32_t in_w, uint32_t in_h, uint32_t out_w,
                    uint32_t out_h, or_rect output, float* out) {
    uint32_t xi[18], yi[18], xc, yc;
    double xw[18], yw[18];
    for (uint32_t y = 0; y < output.height; ++y)
        for (uint32_t x = 0; x < output.width; ++x) {
            const int nx = or_cubic_axis(in_w, out_w, output.x + x, &xc, xi, xw);
            const int ny = or_cubic_axis(in_h, out_h, output.y + y, &yc, yi, yw);
            if (nx < 0) return -nx;
            if (ny < 0) return -ny;
            for (int c = 0; c < 3; ++c) {
#define CR_AT(col, row) ((double)src[((size_t)(row) * in_w + (col)) * 3 + c])
#define CR_ROW(row, result)                                             \
    do {                                                                \
        const double base_ = CR_AT(xc, row);                            \
        double v_ = base_;                                              \
        for (int i_ = 0; i_ < nx; ++i_) {                               \
            const double delta_ = xw[i_] * (CR_AT(xi[i_], row) - base_); \
            if (delta_ != 0) v_ = v_ + delta_;                          \
        }                                                               \
        (result) = v_;                                                  \
    } while (0)
                double base;
                CR_ROW(yc, base);
                double v = base, previous_value = base;
                uint32_t previous_row = yc;
                for (int i = 0; i < ny; ++i) {
                    const uint32_t row = yi[i];
                    double row_value;
                    if (row == yc) row_value = base;
                    else if (row == previous_row) row_value = previous_value;
                    else CR_ROW(row, row_value);
                    previous_row = row;
                    previous_value = row_value;
                    const double delta = yw[i] * (row_value - base);
                    if (delta != 0) v = v + delta;
                }
#undef CR_ROW
#undef CR_AT
                if (!isfinite(v) || fabs(v) > FLT_MAX) return OR_INVALID_ARGUMENT;
                out[((size_t)y * output.width + x) * 3 + c] = (float)v;
            }
        }
    return OR_OK;
}

/* GeometryOps.cpp:46-67 */
int or_rotation_prepare(double a, uint32_t width, uint32_t height, or_rotation* r) {
    if (!isfinite(a) || a < -180 || a > 180 || !width || !height) return OR_INVALID_ARGUMENT;
    r->width = width;
    r->height = height;
    r->cx = ((double)width - 1) / 2;
    r->cy = ((double)height - 1) / 2;
    if (a == 0) { r->cosine = 1; r->sine = 0; }
    else if (a == 90) { r->cosine = 0; r->sine = 1; }
    else if (a == -90) { r->cosine = 0; r->sine = -1; }
    else if (fabs(a) == 180) { r->cosine = -1; r->sine = 0; }
    else {
        const double theta = (a / 180) * 0x1.921fb54442d18p+1;
        r->cosine = cos(theta);
        r->sine = sin(theta);
    }
    return OR_OK;
}

typedef struct rot_taps { uint32_t x0, y0, x1, y1; double fx, fy; } rot_taps;

/* GeometryOps.cpp:68-76 */
static rot_taps rotation_taps(const or_rotation* r, uint32_t x, uint32_t y) {
    const double dx = (double)x - r->cx, dy = (double)y - r->cy;
    double sx = (r->cx + r->cosine * dx) + r->sine * dy;
    double sy = (r->cy - r->sine * dx) + r->cosine * dy;
    const double mx = (double)r->width - 1, my = (double)r->height - 1;
    sx = sx < 0. ? 0. : (sx > mx ? mx : sx);
    sy = sy < 0. ? 0. : (sy > my ? my : sy);
    rot_taps t;
    t.x0 = (uint32_t)floor(sx);
    t.y0 = (uint32_t)floor(sy);
    t.fx = sx - t.x0;
    t.fy = sy - t.y0;
    t.x1 = t.fx == 0 ? t.x0 : (t.x0 + 1 < r->width - 1 ? t.x0 + 1 : r->width - 1);
    t.y1 = t.fy == 0 ? t.y0 : (t.y0 + 1 < r->height - 1 ? t.y0 + 1 : r->height - 1);
    return t;
}

/* GeometryOps.cpp:99-111 (support relative to the rotation's own bounds) */
int or_rotate_support(const or_rotation* r, or_rect output, or_rect* support) {
    uint32_t left = r->width, top = r->height, right = 0, bottom = 0;
    for (uint64_t y = output.y; y < (uint64_t)output.y + output.height; ++y)
        for (uint64_t x = output.x; x < (uint64_t)output.x + output.width; ++x) {
            const rot_taps t = rotation_taps(r, (uint32_t)x, (uint32_t)y);
            if (t.x0 < left) left = t.x0;
            if (t.y0 < top) top = t.y0;
            if (t.x1 > right) right = t.x1;
            if (t.y1 > bottom) bottom = t.y1;
        }
    or_rect s = {left, top, right - left + 1, bottom - top + 1};
    *support = s;
    return OR_OK;
}

/* GeometryOps.cpp:29-34 */
static double rot_blend(double a, double b, double t) {
    if (t == 0) return a;
    if (t == 1) return b;
    if (a == b) return a;
    return a + t * (b - a);
}

/* GeometryOps.cpp:129-141 */
int or_rotate(const or_rotation* r, const float* src, or_rect output, float* out) {
    for (uint32_t y = 0; y < output.height; ++y)
        for (uint32_t x = 0; x < output.width; ++x) {
            const rot_taps t = rotation_taps(r, output.x + x, output.y + y);
            for (int c = 0; c < 3; ++c) {
#define RT_AT(xx, yy) ((double)src[((size_t)(yy) * r->width + (xx)) * 3 + c])
                const double upper = rot_blend(RT_AT(t.x0, t.y0), RT_AT(t.x1, t.y0), t.fx);
                const double lower = rot_blend(RT_AT(t.x0, t.y1), RT_AT(t.x1, t.y1), t.fx);
#undef RT_AT
                const double v = rot_blend(upper, lower, t.fy);
                if (!isfinite(v) || fabs(v) > FLT_MAX) return OR_INVALID_ARGUMENT;
                out[((size_t)y * output.width + x) * 3 + c] = (float)v;
            }
        }
    return OR_OK;
}

/* ------------------------------------------------------------ tile planner */

/* RawEngine.cpp:1399-1411 */
size_t or_plan_tiles(or_rect vp, uint32_t tile, or_rect* tiles, size_t capacity) {
    size_t n = 0;
    if (!tile) return 0;
    const uint64_t right = (uint64_t)vp.x + vp.width, bottom = (uint64_t)vp.y + vp.height;
    for (uint64_t y = vp.y; y < bottom; y += tile)
        for (uint64_t x = vp.x; x < right; x += tile) {
            if (n < capacity) {
                or_rect r = {(uint32_t)x, (uint32_t)y,
                             (uint32_t)(right - x < tile ? right - x : tile),
                             (uint32_t)(bottom - y < tile ? bottom - y : tile)};
                tiles[n] = r;
            }
            ++n;
        }
    return n;
}
