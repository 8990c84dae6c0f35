// Device-side data layout shared by the render kernels.
//
// HBM layout: a RAW image is its uint16 sensor plane exactly as the caller
// supplied it (row stride in samples, active area inside it); renders write
// interleaved float32 RGB rows (3 floats per pixel, caller row stride).  All
// per-image constants the kernels need travel by value in DevRaw; the per-pixel
// stage program travels by value in DevProgram (kernel parameter space), so a
// launch reads nothing but the sensor samples and writes nothing but pixels.
#pragma once

#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

#include "rawengine_b200.h"

namespace re {

// Device status word: zero = ok.  A failure stores key = (priority << 8) | kind
// with atomicMax, so the highest-priority failure survives: internal guards
// and timeouts (priority 511) first, then the earliest failing chain stage
// (priority 255 - stage index).  The low byte is the failure kind.
enum : uint32_t {
    ST_DOMAIN = 1u << 0,     // non-finite at an output boundary (domain_error)
    ST_INVALID = 1u << 1,    // non-finite curve input / float32 overflow (invalid_argument)
    ST_OVERFLOW = 1u << 2,   // guided filter intermediate overflow (overflow_error)
    ST_GUARD = 1u << 3,      // internal bounds guard tripped (logic error)
    ST_TIMEOUT = 1u << 4,    // bounded wait expired
};

struct DevRaw {
    const uint16_t* samples;
    uint32_t stride;          // samples per row
    int32_t ax, ay, aw, ah;   // active area (sensor coordinates)
    uint32_t phase_x, phase_y;
    int32_t site_color[4];    // colour of each photosite index (pattern applied)
    float black[4];           // per-site black level as float
    float span[4];            // per-site (white - black) as float
    float rcp[4];             // 1/span, used only where rcp_exact says it is exact
    uint32_t rcp_exact;       // bit s: the reciprocal form equals IEEE division for every code
};

// Photosite index of RawEngine.cpp:74-77 for any integer position.
__host__ __device__ __forceinline__ int site_of(const DevRaw& r, int x, int y) {
    return (int)((((unsigned)(y & 1) + r.phase_y) & 1u) * 2u + (((unsigned)(x & 1) + r.phase_x) & 1u));
}

__host__ __device__ __forceinline__ int color_of(const DevRaw& r, int x, int y) {
    return r.site_color[site_of(r, x, y)];
}

// RawEngine.cpp:89-97: (float(raw) - black) / (white - black), IEEE division.
// The numerator is an integer in [-65535, 65535]; for a site whose span passed
// the host's exhaustive check (every numerator gives the same float as IEEE
// division) the quotient is formed as q = n*rcp refined by one fused residual
// step, which is three instructions instead of the division sequence.
__device__ __forceinline__ float normalize_code(const DevRaw& r, int s, float code) {
    const float n = __fsub_rn(code, r.black[s]);
    if ((r.rcp_exact >> s) & 1u) {
        const float q0 = __fmul_rn(n, r.rcp[s]);
        const float res = __fmaf_rn(-q0, r.span[s], n);
        return __fmaf_rn(res, r.rcp[s], q0);
    }
    return __fdiv_rn(n, r.span[s]);
}

__device__ __forceinline__ float normalize_sample(const DevRaw& r, int x, int y) {
    const int s = site_of(r, x, y);
    return normalize_code(r, s, (float)__ldg(r.samples + (size_t)y * r.stride + x));
}

// Normalization constants of the four positions of a 2x2 quad whose top-left
// sample sits at an even sensor coordinate (the photosite of position k =
// 2*j + i is then fixed by the CFA phase alone).
struct QuadNorm {
    float black[4], span[4], rcp[4];
    unsigned exact;              // bit k: the reciprocal form is exact at position k
};

__device__ __forceinline__ QuadNorm quad_norm(const DevRaw& r) {
    QuadNorm q;
    q.exact = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int s = (int)(((((unsigned)(k >> 1)) + r.phase_y) & 1u) * 2u + ((((unsigned)(k & 1)) + r.phase_x) & 1u));
        q.black[k] = r.black[s];
        q.span[k] = r.span[s];
        q.rcp[k] = r.rcp[s];
        q.exact |= ((r.rcp_exact >> s) & 1u) << k;
    }
    return q;
}

// normalize_code for quad position k (same arithmetic).
__device__ __forceinline__ float quad_normalize(const QuadNorm& q, int k, float code) {
    const float n = __fsub_rn(code, q.black[k]);
    if ((q.exact >> k) & 1u) {
        const float q0 = __fmul_rn(n, q.rcp[k]);
        const float res = __fmaf_rn(-q0, q.span[k], n);
        return __fmaf_rn(res, q.rcp[k], q0);
    }
    return __fdiv_rn(n, q.span[k]);
}

// The four sample codes of the 2x2 quad at the even sensor position (gx, gy);
// two samples of a quad row are read as one 32-bit word when `words` (rows
// 4-byte aligned).
__device__ __forceinline__ void quad_codes(const DevRaw& raw, bool words, int gx, int gy, unsigned (&c)[4]) {
    const uint16_t* r0 = raw.samples + (size_t)gy * raw.stride + gx;
    const uint16_t* r1 = r0 + raw.stride;
    if (words) {
        const unsigned w0 = __ldg(reinterpret_cast<const unsigned*>(r0));
        const unsigned w1 = __ldg(reinterpret_cast<const unsigned*>(r1));
        c[0] = w0 & 0xFFFFu; c[1] = w0 >> 16; c[2] = w1 & 0xFFFFu; c[3] = w1 >> 16;
    } else {
        c[0] = __ldg(r0); c[1] = __ldg(r0 + 1); c[2] = __ldg(r1); c[3] = __ldg(r1 + 1);
    }
}

__device__ __forceinline__ bool quad_words(const DevRaw& raw) {
    return ((raw.stride & 1u) == 0) && ((reinterpret_cast<uintptr_t>(raw.samples) & 3u) == 0);
}

// Normalized samples of QX x QY quads from the even sensor position (gx0, gy0)
// into a row-major plane of PW x PH entries whose origin is OFF samples right
// of and below (gx0, gy0); quad positions outside the plane are skipped.  The
// caller guarantees every sample of the quads lies inside the sensor buffer.
template <int QX, int QY, int PW, int PH, int OFF, int THREADS, typename T>
__device__ __forceinline__ void load_quads(T* plane, const DevRaw& raw, int gx0, int gy0, float* vmax) {
    const QuadNorm N = quad_norm(raw);
    const bool words = quad_words(raw);
    float m = 0.0f;
    for (int q = threadIdx.x; q < QX * QY; q += THREADS) {
        const int qx = q % QX, qy = q / QX;
        unsigned c[4];
        quad_codes(raw, words, gx0 + 2 * qx, gy0 + 2 * qy, c);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int px = 2 * qx + (k & 1) - OFF, py = 2 * qy + (k >> 1) - OFF;
            if (OFF != 0 && (px < 0 || px >= PW || py < 0 || py >= PH)) continue;
            const float v = quad_normalize(N, k, (float)c[k]);
            m = fmaxf(m, fabsf(v));
            plane[py * PW + px] = (T)v;
        }
    }
    if (vmax) *vmax = m;
}

// The same samples by quad position: planes[k][q] holds position k = 2*j + i
// of quad q (row-major over the QX x QY quads).
template <int QX, int QY, int THREADS, typename T>
__device__ __forceinline__ void load_quad_planes(T (*planes)[QX * QY], const DevRaw& raw, int gx0, int gy0,
                                                 float* vmax) {
    const QuadNorm N = quad_norm(raw);
    const bool words = quad_words(raw);
    float m = 0.0f;
    for (int q = threadIdx.x; q < QX * QY; q += THREADS) {
        const int qx = q % QX, qy = q / QX;
        unsigned c[4];
        quad_codes(raw, words, gx0 + 2 * qx, gy0 + 2 * qy, c);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float v = quad_normalize(N, k, (float)c[k]);
            m = fmaxf(m, fabsf(v));
            planes[k][q] = (T)v;
        }
    }
    if (vmax) *vmax = m;
}

// MenonDemosaic.cpp:60-66 whole-sample mirror about [origin, origin+size).
__host__ __device__ __forceinline__ int mirror_coord(int v, int origin, int size) {
    if (v >= origin && v < origin + size) return v;
    if (size == 1) return origin;
    const int period = 2 * (size - 1);
    int folded = (v - origin) % period;
    if (folded < 0) folded += period;
    return origin + (folded < size ? folded : period - folded);
}

// ---------------------------------------------------------------- curves

// A cell of the lookup grid: the knot (RU-rounded) that falls in the cell,
// +inf if none, and the records of the samples below and at or above it.
constexpr int CURVE_RECS = 288;   // 258 records, padded to whole cache lines

struct __align__(8) CurveCell {
    float next;
    uint16_t below, above;
};
constexpr int CURVE_CELLS = 4096;

// Order-preserving integer key of a float: its bit pattern with the magnitude
// bits of negative values inverted (-0 is folded to +0 first, so the two zeros
// share a key as they compare equal).  Uniform within each binade, a key step
// doubles in width from one binade to the next.
__host__ __device__ inline int32_t curve_key(float v) {
#ifdef __CUDA_ARCH__
    const int32_t i = __float_as_int(__fadd_rn(v, 0.0f));
#else
    const float z = v + 0.0f;
    int32_t i;
    std::memcpy(&i, &z, sizeof i);
#endif
    return i < 0 ? i ^ 0x7FFFFFFF : i;
}

// One ExtendedCurves curve prepared for float32 evaluation (ToneOps.cpp:795-832).
// Knot x are rounded UP to float so that `v < xf` equals the reference's
// double comparison `v < x` for every float v; xeq holds x only when x is a
// float (else NaN) so that `v == xeq` equals the double equality test.
struct DevCurve {
    uint32_t n;               // knots
    uint32_t identity;        // every knot has x == y
    uint32_t cubic;           // ShapePreservingCubic
    uint32_t pad;
    float xf[256];
    float xeq[256];
    float xn[256];            // x rounded to nearest (arithmetic anchor)
    float y[256];
    float slope[256];         // segment slopes (linear segments and extrapolation)
    float4 coef[256];         // power-basis cubic per segment: c0 + t(c1 + t(c2 + t c3))
    float inv_h[256];         // 1 / (x[i+1] - x[i])
    // O(1) segment lookup (0 cells: none, the binary search over xf).  Key
    // grid: cell c holds the keys [p + c 2^q, p + (c+1) 2^q) (p, q as int32 and
    // uint32), lower keys fall in cell 0 and higher ones in the last.  Uniform
    // grid: a sample's cell is (v - p) * q (p, q the bits of floats) truncated
    // and clamped.  One comparison with the cell's knot finds the record.
    // Record r (0..n-2 the segments, n-1 the right and n the left linear
    // extrapolation) is p(s) = e0 + s(e1 + s(e2 + s e3)), s = v - anchor[r];
    // each field is its own 128-byte aligned array, so a warp's gather of one
    // field over a short curve touches a single cache line.
    uint32_t ncells;
    uint32_t key_grid;
    uint32_t grid_p, grid_q;
    alignas(128) float anchor[CURVE_RECS];
    alignas(128) float e[4][CURVE_RECS];
    CurveCell cell[CURVE_CELLS];
};

struct DevCurveSet {
    DevCurve c[4];            // master, R, G, B
};


// --------------------------------------------------------------- program

struct DevProgram {
    uint32_t count;
    int32_t anchor;
    re_stage st[RE_MAX_STAGES];
    const DevCurveSet* curves[4];
};

constexpr uint32_t KEY_GUARD = (511u << 8) | ST_GUARD;
constexpr uint32_t KEY_TIMEOUT = (511u << 8) | ST_TIMEOUT;

// Per-call device scratch, stream-ordered, from a memory pool the library
// owns on each device (capi.cu).  The pool keeps freed blocks mapped (its
// release threshold is unlimited), so steady-state calls neither map nor
// unmap device memory; re_release_scratch() returns the idle blocks.  Free
// with cudaFreeAsync on a stream ordered after the last use.
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t stream);

}  // namespace re
