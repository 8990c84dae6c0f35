// Per-pixel stage program: the point nodes of a render chain, fused into the
// epilogue of whichever kernel produced the pixel.
//
// Bit-exactness: WhiteBalance, Exposure and the 3x3 matrices use explicitly
// rounded float ops in the reference's evaluation order (no contraction), so
// they reproduce the reference's float32 results exactly.  ToneCurve and
// SrgbEncode call powf (a few ulp from the host libm); ExtendedCurves are
// evaluated in float32 from host-prepared per-segment polynomials instead of
// the reference's binary64 de Casteljau blend -- both stay far inside the
// 1e-5 full-scale tolerance of the float outputs.
#pragma once

#include "re_device.cuh"

namespace re {

__device__ __forceinline__ float curve_map(const DevCurve* __restrict__ c, float v) {
    if (c->identity) return v;
    const int n = (int)c->n;
    int lo = 0, hi = n;  // upper_bound over the RU-rounded knots
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (v < __ldg(&c->xf[mid])) hi = mid; else lo = mid + 1;
    }
    const int left = lo == 0 ? 0 : lo - 1;
    const int seg = left < n - 2 ? left : n - 2;
    if (v == __ldg(&c->xeq[left])) return __ldg(&c->y[left]);
    const float xl = __ldg(&c->xf[n - 1]);
    const bool above = v > xl || (v == xl && isnan(__ldg(&c->xeq[n - 1])));
    if (!c->cubic || v < __ldg(&c->xf[0]) || above) {
        const float s = __ldg(&c->slope[seg]);
        const float yl = __ldg(&c->y[left]);
        return s == 0.0f ? yl : yl + (v - __ldg(&c->xn[left])) * s;
    }
    const float t = (v - __ldg(&c->xn[seg])) * __ldg(&c->inv_h[seg]);
    const float4 k = __ldg(&c->coef[seg]);
    return k.x + t * (k.y + t * (k.z + t * k.w));
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
                const float mapped = inv_gamma == 1.0f ? comp : powf(comp, inv_gamma);
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
                           : __fsub_rn(__fmul_rn(1.055f, powf(lin, 1.0f / 2.4f)), 0.055f);
            }
            break;
        }
        case RE_STAGE_CURVES: {
            const DevCurveSet* cs = P.curves[st.arg];
            bool bad = !(isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]));
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const DevCurve* ch = &cs->c[c + 1];
                if (cs->c[0].identity && ch->identity) continue;
                const float master = curve_map(&cs->c[0], v[c]);
                const float mapped = curve_map(ch, master);
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

__device__ __forceinline__ void report(uint32_t* status, uint32_t err) {
    if (err && status) atomicMax(status, err);
}

}  // namespace re
