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

// Three samples through one shared-memory curve at once: a fixed-length,
// branch-free upper_bound (binary lifting over the RU-rounded knots) so that
// the three searches interleave instead of chaining their loads.
__device__ __forceinline__ void curve_map3(const SmemCurve* __restrict__ c, float v[3]) {
    if (c->identity) return;
    const int n = (int)c->n;
    int lo[3] = {0, 0, 0};
    for (int step = (int)c->pad; step > 0; step >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int cand = lo[k] + step;
            if (cand <= n && v[k] >= c->xf[cand - 1]) lo[k] = cand;
        }
    }
    const float xl = c->xf[n - 1], x0 = c->xf[0];
    const bool tail_nan = isnan(c->xeq[n - 1]);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int left = lo[k] == 0 ? 0 : lo[k] - 1;
        const int seg = left < n - 2 ? left : n - 2;
        const float x = v[k];
        float r;
        if (x == c->xeq[left]) {
            r = c->y[left];
        } else if (!c->cubic || x < x0 || x > xl || (x == xl && tail_nan)) {
            const float s = c->slope[seg];
            const float yl = c->y[left];
            r = s == 0.0f ? yl : yl + (x - c->xn[left]) * s;
        } else {
            const float t = (x - c->xn[seg]) * c->inv_h[seg];
            const float4 kf = c->coef[seg];
            r = kf.x + t * (kf.y + t * (kf.z + t * kf.w));
        }
        v[k] = r;
    }
}

// Loads curve set 0 of P into shared memory when every curve fits; returns it
// (or null, in which case curves are read from global memory).  All threads
// of the block must call it; it ends with a barrier.
__device__ __forceinline__ const SmemCurveSet* load_curves(const DevProgram& P, SmemCurveSet* sc) {
    const DevCurveSet* g = P.curves[0];
    bool fits = g != nullptr;
    if (fits)
        for (int k = 0; k < 4; ++k) fits &= g->c[k].n <= (uint32_t)SC_MAX;
    if (!fits) return nullptr;
    for (int k = 0; k < 4; ++k) {
        const DevCurve& src = g->c[k];
        SmemCurve& dst = sc->c[k];
        const int n = (int)src.n;
        if (threadIdx.x == 0) {
            dst.n = src.n;
            dst.identity = src.identity;
            dst.cubic = src.cubic;
            uint32_t p2 = 1;                    // largest power of two <= n (search span)
            while (p2 * 2 <= src.n) p2 *= 2;
            dst.pad = p2;
        }
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            dst.xf[i] = src.xf[i];
            dst.xeq[i] = src.xeq[i];
            dst.xn[i] = src.xn[i];
            dst.y[i] = src.y[i];
            dst.slope[i] = src.slope[i];
            dst.inv_h[i] = src.inv_h[i];
            dst.coef[i] = src.coef[i];
        }
    }
    __syncthreads();
    return sc;
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
                                             float& g, float& b, uint32_t& err,
                                             const SmemCurveSet* sc = nullptr) {
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
            if (sc && st.arg == 0) {
                curve_map3(&sc->c[0], v);
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    if (!isfinite(v[c])) bad = true;
                    const SmemCurve* ch = &sc->c[c + 1];
                    if (!ch->identity) {
                        float one[3] = {v[c], v[c], v[c]};
                        curve_map3(ch, one);
                        v[c] = one[0];
                    }
                    if (!isfinite(v[c])) bad = true;
                }
            } else {
                const DevCurveSet* cs = P.curves[st.arg];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const DevCurve* ch = &cs->c[c + 1];
                    if (cs->c[0].identity && ch->identity) continue;
                    const float master = curve_map(&cs->c[0], v[c]);
                    const float mapped = curve_map(ch, master);
                    if (!isfinite(master) || !isfinite(mapped)) bad = true;
                    v[c] = mapped;
                }
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

__device__ __forceinline__ void report(uint32_t* status, uint32_t err) {
    if (err && status) atomicMax(status, err);
}

}  // namespace re
