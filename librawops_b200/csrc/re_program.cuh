// Per-pixel stage program: the point nodes of a render chain, fused into the
// epilogue of whichever kernel produced the pixel.
//
// Bit-exactness: WhiteBalance, Exposure and the 3x3 matrices use explicitly
// rounded float ops in the reference's evaluation order (no contraction), so
// they reproduce the reference's float32 results exactly.  ToneCurve and
// SrgbEncode take their power through exp2(e*log2(x)) on the hardware
// approximations (a few 1e-7 from the host libm's powf); ExtendedCurves are
// evaluated in float32 from host-prepared per-segment polynomials instead of
// the reference's binary64 de Casteljau blend -- both stay far inside the
// 1e-5 full-scale tolerance of the float outputs.
#pragma once

#include "re_device.cuh"

namespace re {

template <class Curve>
__device__ __forceinline__ float curve_map(const Curve* __restrict__ c, float v) {
    if (c->identity) return v;
    const int n = (int)c->n;
    int lo = 0, hi = n;  // upper_bound over the RU-rounded knots
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (v < c->xf[mid]) hi = mid; else lo = mid + 1;
    }
    const int left = lo == 0 ? 0 : lo - 1;
    const int seg = left < n - 2 ? left : n - 2;
    if (v == c->xeq[left]) return c->y[left];
    const float xl = c->xf[n - 1];
    const bool above = v > xl || (v == xl && isnan(c->xeq[n - 1]));
    if (!c->cubic || v < c->xf[0] || above) {
        const float s = c->slope[seg];
        const float yl = c->y[left];
        return s == 0.0f ? yl : yl + (v - c->xn[left]) * s;
    }
    const float t = (v - c->xn[seg]) * c->inv_h[seg];
    const float4 k = c->coef[seg];
    return k.x + t * (k.y + t * (k.z + t * k.w));
}

// The lookup-grid cell of sample v (DevCurve: key grid or uniform grid).
__device__ __forceinline__ unsigned curve_cell(float v, unsigned ncells, bool key_grid, uint32_t p, uint32_t q) {
    if (key_grid) {
        const int32_t k = curve_key(v);
        return k < (int32_t)p ? 0u : min(((unsigned)k - p) >> q, ncells - 1u);
    }
    const int c = __float2int_rz((v - __uint_as_float(p)) * __uint_as_float(q));
    return (unsigned)min(max(c, 0), (int)ncells - 1);
}

// Cell lookup (DevCurve::ncells > 0) of M samples at once: the sample's cell
// gives the one knot it can meet and the records either side of it, one
// comparison with that knot (RU-rounded, so the float comparison equals the
// reference's double one) picks the record, and one power-basis polynomial
// evaluates it.  Extrapolation and linear curves are records of the same
// form.  The loads of all M samples are issued before any of them is used.
template <int M>
__device__ __forceinline__ void curve_lookup_n(const DevCurve* __restrict__ c, unsigned ncells, bool key_grid,
                                               uint32_t p, uint32_t q, float* v) {
    int rec[M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
        const uint2 e = __ldg(reinterpret_cast<const uint2*>(&c->cell[curve_cell(v[i], ncells, key_grid, p, q)]));
        rec[i] = (int)(v[i] >= __uint_as_float(e.x) ? e.y >> 16 : e.y & 0xFFFFu);
    }
    float s[M], e0[M], e1[M], e2[M], e3[M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
        s[i] = __ldg(&c->anchor[rec[i]]);
        e0[i] = __ldg(&c->e[0][rec[i]]);
        e1[i] = __ldg(&c->e[1][rec[i]]);
        e2[i] = __ldg(&c->e[2][rec[i]]);
        e3[i] = __ldg(&c->e[3][rec[i]]);
    }
#pragma unroll
    for (int i = 0; i < M; ++i) {
        const float d = v[i] - s[i];
        v[i] = e0[i] + d * (e1[i] + d * (e2[i] + d * e3[i]));
    }
}

__device__ __forceinline__ float curve_cells(const DevCurve* __restrict__ c, float v) {
    float x[1] = {v};
    curve_lookup_n<1>(c, c->ncells, c->key_grid != 0, c->grid_p, c->grid_q, x);
    return x[0];
}

__device__ __forceinline__ float curve_apply(const DevCurve* __restrict__ c, float v) {
    if (c->identity) return v;
    return c->ncells ? curve_cells(c, v) : curve_map(c, v);
}

// x^e for x in [0, 1] through the hardware log2/exp2 approximations: a few
// 1e-7 relative, inside the float tolerance of the tone and sRGB stages.
__device__ __forceinline__ float unit_pow(float x, float e) {
    return x > 0.0f ? exp2f(e * __log2f(x)) : (e == 0.0f ? 1.0f : 0.0f);
}

// Error key of a failing stage: the earliest stage in chain order wins when
// keys are combined with atomicMax (the reference throws at the first node
// whose tile holds an invalid value; point nodes are pixel-independent, so
// that node is the minimum over pixels of each pixel's first failing stage).
__device__ __forceinline__ uint32_t stage_key(int s, uint32_t kind) {
    return ((uint32_t)(255 - s) << 8) | kind;
}

// Applies stages [begin, end) of P to one pixel; `err` keeps the max key.
__device__ __forceinline__ void apply_stages(const DevProgram& P, int begin, int end, float& r,
                                             float& g, float& b, uint32_t& err) {
    float v[3] = {r, g, b};
    for (int s = begin; s < end; ++s) {
        const re_stage& st = P.st[s];
        switch (st.kind) {
        case RE_STAGE_GAIN3:
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c] = __fmul_rn(v[c], st.f[c]);
            break;
        case RE_STAGE_SCALE:
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c] = __fmul_rn(v[c], st.f[0]);
            break;
        case RE_STAGE_MATRIX: {
            const float* m = st.f;
            const float nr = __fadd_rn(__fadd_rn(__fmul_rn(m[0], v[0]), __fmul_rn(m[1], v[1])), __fmul_rn(m[2], v[2]));
            const float ng = __fadd_rn(__fadd_rn(__fmul_rn(m[3], v[0]), __fmul_rn(m[4], v[1])), __fmul_rn(m[5], v[2]));
            const float nb = __fadd_rn(__fadd_rn(__fmul_rn(m[6], v[0]), __fmul_rn(m[7], v[1])), __fmul_rn(m[8], v[2]));
            v[0] = nr; v[1] = ng; v[2] = nb;
            break;
        }
        case RE_STAGE_TONE: {
            const float shoulder = st.f[0], inv_gamma = st.f[1];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float lin = v[c];
                const float mag = fabsf(lin);
                const float comp = __fdiv_rn(mag, __fadd_rn(mag, shoulder));
                const float mapped = inv_gamma == 1.0f ? comp : unit_pow(comp, inv_gamma);
                v[c] = copysignf(mapped, lin);
            }
            break;
        }
        case RE_STAGE_CLIP: {
            if (!(isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]))) err = max(err, stage_key(s, ST_DOMAIN));
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c] = fminf(fmaxf(v[c], 0.0f), 1.0f);
            break;
        }
        case RE_STAGE_SRGB: {
            if (!(isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]))) err = max(err, stage_key(s, ST_DOMAIN));
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float lin = fminf(fmaxf(v[c], 0.0f), 1.0f);
                v[c] = lin <= 0.0031308f
                           ? __fmul_rn(12.92f, lin)
                           : __fsub_rn(__fmul_rn(1.055f, unit_pow(lin, 1.0f / 2.4f)), 0.055f);
            }
            break;
        }
        case RE_STAGE_CURVES: {
            bool bad = !(isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]));
            const DevCurveSet* cs = P.curves[st.arg];
            const bool master_id = cs->c[0].identity;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const DevCurve* ch = &cs->c[c + 1];
                const float master = master_id ? v[c] : curve_apply(&cs->c[0], v[c]);
                const float mapped = curve_apply(ch, master);
                if (!isfinite(master) || !isfinite(mapped)) bad = true;
                v[c] = mapped;
            }
            if (bad) {
                err = max(err, stage_key(s, ST_INVALID));
            }
            break;
        }
        default:
            break;
        }
    }
    r = v[0];
    g = v[1];
    b = v[2];
}

// A small curve's lookup tables staged in shared memory by the CTA that
// evaluates the program: the cells' knots and record pairs and the records'
// fields as separate 32-bit arrays, so every gather is one conflict-free
// shared-memory access instead of a load through L1.
constexpr int SM_CURVE_CELLS = 64, SM_CURVE_RECS = 32;
struct SmemCurve {
    float next[SM_CURVE_CELLS];
    uint32_t recs[SM_CURVE_CELLS];
    float anchor[SM_CURVE_RECS];
    float e[4][SM_CURVE_RECS];
};

// curve_lookup_n on the staged tables (same cells, records and arithmetic).
template <int M>
__device__ __forceinline__ void curve_lookup_smem(const SmemCurve& t, unsigned ncells, bool key_grid, uint32_t p,
                                                  uint32_t q, float* v) {
    int rec[M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
        const unsigned cell = curve_cell(v[i], ncells, key_grid, p, q);
        const uint32_t pair = t.recs[cell];
        rec[i] = (int)(v[i] >= t.next[cell] ? pair >> 16 : pair & 0xFFFFu);
    }
#pragma unroll
    for (int i = 0; i < M; ++i) {
        const int k = rec[i];
        const float d = v[i] - t.anchor[k];
        v[i] = t.e[0][k] + d * (t.e[1][k] + d * (t.e[2][k] + d * t.e[3][k]));
    }
}

// Stages the master curve of the first curves stage in [begin, end) when its
// tables fit SmemCurve; every thread of the CTA calls this (the CTA's threads
// must synchronize before the tables are read).  Returns that stage's index,
// or -1 when nothing was staged.
__device__ __forceinline__ int stage_curve_smem(SmemCurve& t, const DevProgram& P, int begin, int end) {
    for (int s = begin; s < end; ++s) {
        const re_stage& st = P.st[s];
        if (st.kind != RE_STAGE_CURVES) continue;
        const unsigned n = (unsigned)st.f[1], ncells = (unsigned)st.f[2];
        if (st.f[0] != 0.0f || ncells == 0 || ncells > SM_CURVE_CELLS || n + 1 > SM_CURVE_RECS) return -1;
        const DevCurve* c = &P.curves[st.arg]->c[0];
        for (unsigned i = threadIdx.x; i < ncells; i += blockDim.x) {
            const uint2 e = __ldg(reinterpret_cast<const uint2*>(&c->cell[i]));
            t.next[i] = __uint_as_float(e.x);
            t.recs[i] = e.y;
        }
        for (unsigned i = threadIdx.x; i <= n; i += blockDim.x) {
            t.anchor[i] = __ldg(&c->anchor[i]);
            t.e[0][i] = __ldg(&c->e[0][i]);
            t.e[1][i] = __ldg(&c->e[1][i]);
            t.e[2][i] = __ldg(&c->e[2][i]);
            t.e[3][i] = __ldg(&c->e[3][i]);
        }
        return s;
    }
    return -1;
}

// The master curve with its lookup scalars from the stage's parameters
// (f[0] identity, f[1] knots, f[2] cells, f[3] key grid, f[4] and f[5] the
// bits of the grid's p and q; build_program fills them).
struct MasterCurve {
    const DevCurve* c;
    unsigned ncells;
    bool key_grid;
    uint32_t p, q;
    bool identity;
    __device__ __forceinline__ void load(const DevCurve* curve, const float* f) {
        c = curve;
        identity = f[0] != 0.0f;
        ncells = (unsigned)f[2];
        key_grid = f[3] != 0.0f;
        p = __float_as_uint(f[4]);
        q = __float_as_uint(f[5]);
    }
    // maps v[0..M) in place
    template <int M>
    __device__ __forceinline__ void eval_n(float* v) const {
        if (identity) return;
        if (!ncells) {
#pragma unroll
            for (int i = 0; i < M; ++i) v[i] = curve_map(c, v[i]);
            return;
        }
        curve_lookup_n<M>(c, ncells, key_grid, p, q, v);
    }
    // the same from tables staged by stage_curve_smem
    template <int M>
    __device__ __forceinline__ void eval_n(const SmemCurve& t, float* v) const {
        curve_lookup_smem<M>(t, ncells, key_grid, p, q, v);
    }
};

// One stage (kind KIND, index s of the program) over N pixels held by one
// thread.  Per pixel the operations and their order are exactly
// apply_stages'.  CHUNK: master-curve lookups kept in flight together (more
// hides the table loads' latency, fewer keeps registers free).
template <int KIND, int N, int CHUNK>
__device__ __forceinline__ void stage_n(const DevProgram& P, int s, float (&r)[N], float (&g)[N], float (&b)[N],
                                        uint32_t& err, const SmemCurve* sc, int sc_stage) {
    const re_stage& st = P.st[s];
    if constexpr (KIND == RE_STAGE_GAIN3) {
        const float k0 = st.f[0], k1 = st.f[1], k2 = st.f[2];
#pragma unroll
        for (int i = 0; i < N; ++i) {
            r[i] = __fmul_rn(r[i], k0);
            g[i] = __fmul_rn(g[i], k1);
            b[i] = __fmul_rn(b[i], k2);
        }
    } else if constexpr (KIND == RE_STAGE_SCALE) {
        const float k = st.f[0];
#pragma unroll
        for (int i = 0; i < N; ++i) {
            r[i] = __fmul_rn(r[i], k);
            g[i] = __fmul_rn(g[i], k);
            b[i] = __fmul_rn(b[i], k);
        }
    } else if constexpr (KIND == RE_STAGE_MATRIX) {
        const float m0 = st.f[0], m1 = st.f[1], m2 = st.f[2], m3 = st.f[3], m4 = st.f[4], m5 = st.f[5],
                    m6 = st.f[6], m7 = st.f[7], m8 = st.f[8];
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const float nr = __fadd_rn(__fadd_rn(__fmul_rn(m0, r[i]), __fmul_rn(m1, g[i])), __fmul_rn(m2, b[i]));
            const float ng = __fadd_rn(__fadd_rn(__fmul_rn(m3, r[i]), __fmul_rn(m4, g[i])), __fmul_rn(m5, b[i]));
            const float nb = __fadd_rn(__fadd_rn(__fmul_rn(m6, r[i]), __fmul_rn(m7, g[i])), __fmul_rn(m8, b[i]));
            r[i] = nr;
            g[i] = ng;
            b[i] = nb;
        }
    } else if constexpr (KIND == RE_STAGE_TONE) {
        const float shoulder = st.f[0], inv_gamma = st.f[1];
        const bool linear = inv_gamma == 1.0f;
        auto tone = [&](float lin) {
            const float mag = fabsf(lin);
            const float comp = __fdiv_rn(mag, __fadd_rn(mag, shoulder));
            return copysignf(linear ? comp : unit_pow(comp, inv_gamma), lin);
        };
#pragma unroll
        for (int i = 0; i < N; ++i) {
            r[i] = tone(r[i]);
            g[i] = tone(g[i]);
            b[i] = tone(b[i]);
        }
    } else if constexpr (KIND == RE_STAGE_CLIP) {
        bool bad = false;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            bad |= !(isfinite(r[i]) && isfinite(g[i]) && isfinite(b[i]));
            r[i] = fminf(fmaxf(r[i], 0.0f), 1.0f);
            g[i] = fminf(fmaxf(g[i], 0.0f), 1.0f);
            b[i] = fminf(fmaxf(b[i], 0.0f), 1.0f);
        }
        if (bad) err = max(err, stage_key(s, ST_DOMAIN));
    } else if constexpr (KIND == RE_STAGE_SRGB) {
        bool bad = false;
        auto enc = [](float v) {
            const float lin = fminf(fmaxf(v, 0.0f), 1.0f);
            return lin <= 0.0031308f ? __fmul_rn(12.92f, lin)
                                     : __fsub_rn(__fmul_rn(1.055f, unit_pow(lin, 1.0f / 2.4f)), 0.055f);
        };
#pragma unroll
        for (int i = 0; i < N; ++i) {
            bad |= !(isfinite(r[i]) && isfinite(g[i]) && isfinite(b[i]));
            r[i] = enc(r[i]);
            g[i] = enc(g[i]);
            b[i] = enc(b[i]);
        }
        if (bad) err = max(err, stage_key(s, ST_DOMAIN));
    } else if constexpr (KIND == RE_STAGE_CURVES) {
        const DevCurveSet* cs = P.curves[st.arg];
        MasterCurve m;
        m.load(&cs->c[0], st.f);
        const bool id_r = st.f[6] != 0.0f, id_g = st.f[7] != 0.0f, id_b = st.f[8] != 0.0f;
        bool bad = false;
        // master curve over the 3N channel values, CHUNK lookups in flight
        float mv[3 * N];
#pragma unroll
        for (int i = 0; i < N; ++i) {
            bad |= !(isfinite(r[i]) && isfinite(g[i]) && isfinite(b[i]));
            mv[3 * i] = r[i];
            mv[3 * i + 1] = g[i];
            mv[3 * i + 2] = b[i];
        }
        static_assert((3 * N) % CHUNK == 0, "channel values split into whole chunks");
        if (s == sc_stage) {
#pragma unroll
            for (int j = 0; j < 3 * N; j += CHUNK) m.eval_n<CHUNK>(*sc, mv + j);
        } else {
#pragma unroll
            for (int j = 0; j < 3 * N; j += CHUNK) m.eval_n<CHUNK>(mv + j);
        }
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const float mr = mv[3 * i], mg = mv[3 * i + 1], mb = mv[3 * i + 2];
            bad |= !(isfinite(mr) && isfinite(mg) && isfinite(mb));
            r[i] = id_r ? mr : curve_apply(&cs->c[1], mr);
            g[i] = id_g ? mg : curve_apply(&cs->c[2], mg);
            b[i] = id_b ? mb : curve_apply(&cs->c[3], mb);
            bad |= !(isfinite(r[i]) && isfinite(g[i]) && isfinite(b[i]));
        }
        if (bad) err = max(err, stage_key(s, ST_INVALID));
    }
}

// Kinds of stages [begin, end) against a fixed sequence.
template <int... KINDS>
__device__ __forceinline__ bool chain_is(const DevProgram& P, int begin, int end) {
    if (end - begin != (int)sizeof...(KINDS)) return false;
    int s = begin;
    return ((P.st[s++].kind == KINDS) && ...);
}

template <int N, int CHUNK, int... KINDS>
__device__ __forceinline__ void chain_n(const DevProgram& P, int begin, float (&r)[N], float (&g)[N],
                                        float (&b)[N], uint32_t& err, const SmemCurve* sc, int sc_stage) {
    int s = begin;
    (stage_n<KINDS, N, CHUNK>(P, s++, r, g, b, err, sc, sc_stage), ...);
}

template <int... KINDS>
struct Chain {};

template <int N, int CHUNK, int... KINDS>
__device__ __forceinline__ bool try_chain(Chain<KINDS...>, const DevProgram& P, int begin, int end, float (&r)[N],
                                          float (&g)[N], float (&b)[N], uint32_t& err, const SmemCurve* sc,
                                          int sc_stage) {
    if (!chain_is<KINDS...>(P, begin, end)) return false;
    chain_n<N, CHUNK, KINDS...>(P, begin, r, g, b, err, sc, sc_stage);
    return true;
}

// The stage program over N pixels held by one thread: the stage loop is
// outside, so each stage's constants are read once and its arithmetic runs
// over N independent pixels.  Two chains of the reference renderer's usual
// node order run as straight-line code, which the compiler schedules across
// stages: white balance, camera matrix, curves, output matrix, sRGB encode
// (a finished sRGB render), and white balance, camera matrix (scene-linear
// output).  Any other program goes through the per-stage dispatch (each more
// specialised chain multiplies the code of every render kernel).  Either way
// each pixel sees apply_stages' operations.
// sc / sc_stage: the master curve of stage sc_stage staged in shared memory
// by stage_curve_smem (nullptr / -1: none).
template <int N, int CHUNK = 3>
__device__ __forceinline__ void apply_stages_n(const DevProgram& P, int begin, int end, float (&r)[N],
                                               float (&g)[N], float (&b)[N], uint32_t& err,
                                               const SmemCurve* sc = nullptr, int sc_stage = -1) {
    constexpr int G = RE_STAGE_GAIN3, M = RE_STAGE_MATRIX, C = RE_STAGE_CURVES, S = RE_STAGE_SRGB;
    if (try_chain<N, CHUNK>(Chain<G, M, C, M, S>{}, P, begin, end, r, g, b, err, sc, sc_stage) ||
        try_chain<N, CHUNK>(Chain<G, M>{}, P, begin, end, r, g, b, err, sc, sc_stage))
        return;
    for (int s = begin; s < end; ++s) {
        switch (P.st[s].kind) {
        case RE_STAGE_GAIN3: stage_n<RE_STAGE_GAIN3, N, CHUNK>(P, s, r, g, b, err, sc, sc_stage); break;
        case RE_STAGE_SCALE: stage_n<RE_STAGE_SCALE, N, CHUNK>(P, s, r, g, b, err, sc, sc_stage); break;
        case RE_STAGE_MATRIX: stage_n<RE_STAGE_MATRIX, N, CHUNK>(P, s, r, g, b, err, sc, sc_stage); break;
        case RE_STAGE_TONE: stage_n<RE_STAGE_TONE, N, CHUNK>(P, s, r, g, b, err, sc, sc_stage); break;
        case RE_STAGE_CLIP: stage_n<RE_STAGE_CLIP, N, CHUNK>(P, s, r, g, b, err, sc, sc_stage); break;
        case RE_STAGE_SRGB: stage_n<RE_STAGE_SRGB, N, CHUNK>(P, s, r, g, b, err, sc, sc_stage); break;
        case RE_STAGE_CURVES: stage_n<RE_STAGE_CURVES, N, CHUNK>(P, s, r, g, b, err, sc, sc_stage); break;
        default: break;
        }
    }
}

__device__ __forceinline__ void report(uint32_t* status, uint32_t err) {
    if (err && status) atomicMax(status, err);
}

}  // namespace re
