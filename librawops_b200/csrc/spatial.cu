// Spatial stages: the working-Y guided filter (SpatialOps.cpp:159-317) and box
// local statistics (SpatialOps.cpp:52-157), each ONE streaming kernel.
//
// Guided filter.  The reference evaluates, per coefficient centre k, centred
// moments over its clipped (2r+1)^2 window and then, per output pixel x,
// p(x) + mean_k[(p_k - p_x) + meanP_delta(k) + a(k)(Y_x - Y_k - meanY_delta(k))]
// in binary64 (O(r^2) per pixel).  Expanding the sum gives the classical form
//     q(x) = mean_{k in W(x)} a(k) * Y(x) + mean_{k in W(x)} b(k),
//     a(k) = cov(Y, p)/(var(Y) + eps),  b(k) = mean(p) - a(k) mean(Y),
// with clipped windows and actual counts, which box sums evaluate in O(1) per
// pixel independent of r.  Y is a fixed linear combination of R, G and B, so
// the box sums of Y and Y^2 follow from those of R, G, B, YR, YG and YB: six
// binary64 moments per pixel.  a and b stay binary64 through the second box
// sum, since a*Y and b can cancel when eps is small.  Output equals p(x)
// exactly when the correction is zero (constants, signed zeros), as in
// SpatialOps.cpp:278.
//
// Local statistics.  Per channel, the finite count, mean and population
// variance over the clipped window.  Each task shifts its samples by one of
// its own values before summing (x - s, (x - s)^2 in binary64), so windows far
// from zero (the reference's 1e20 offset test) keep their precision; the
// reference's Welford/merge order is not reproduced, the result agrees within
// float32 rounding of the outputs.
//
// Both kernels stream vertical STRIPS of the image from top to bottom.  A task
// is one strip (the CTA's NT columns of input: TW output columns plus the
// halo) over one band of output rows; tasks are taken band-major by a
// persistent grid, so CTAs that run together share their strips' halo
// columns in L2.  Per block of R rows:
//   A  column owners (one thread per input column) keep the vertical window
//      sums of the moments in registers, adding the entering row and
//      subtracting the leaving one (re-read from the input, an L2 hit, instead
//      of stored), and write the R rows of sums to shared memory;
//   B  row segments (one thread per K consecutive centres of one row) slide
//      the horizontal window over those sums -- two reads per centre and
//      moment after the first window -- giving each centre's box sums;
// and for the guided filter, additionally
//   C  row segments slide the horizontal window over the centres' a and b;
//   D  column owners keep the vertical window sums of C's rows in registers
//      (the leaving row from a ring of 2r+1 rows per CTA in global memory,
//      which stays in L2) and write the output rows.
// Intermediates never reach HBM: DRAM traffic is the input (plus the strips'
// halo columns where L2 misses them) and the output.  Shared-memory planes
// are moment-major and skewed by one element every K, so the K-strided reads
// of a warp's row segments are conflict-free.
#include <cfloat>
#include <cmath>
#include <mutex>
#include <string>

#include "re_device.cuh"

namespace re {
void set_last_error(const std::string& msg);
}

using namespace re;

namespace {

// Working-Y weights of SpatialOps.cpp:191-192.
struct YWeights {
    double wr, wb;
};

__device__ __forceinline__ double working_y(double r, double g, double b, const YWeights& w) {
    return __dadd_rn(__dadd_rn(g, __dmul_rn(w.wr, __dsub_rn(r, g))), __dmul_rn(w.wb, __dsub_rn(b, g)));
}

// Skewed index of element j in a plane whose segments are K long.
template <int K>
__device__ __forceinline__ int sk(int j) {
    return j + j / K;
}

template <int K>
__host__ __device__ constexpr int plane_len(int n) {
    return n + n / K + 1;
}

// Sums of the K-element blocks of `rows` rows of M skewed planes of length
// plen: bs[(i * M + k) * nb + b] = plane (i, k) summed over columns
// [b K, b K + K), which sit contiguously from b (K + 1).
template <int NT, int K, int M, typename V>
__device__ __forceinline__ void block_sums(const V* planes, int plen, int rows, int nb, V* bs) {
    for (int item = threadIdx.x; item < rows * nb; item += NT) {
        const int i = item / nb, b = item % nb;
        const V* row = planes + (size_t)i * M * plen + b * (K + 1);
        V acc[M];
#pragma unroll
        for (int k = 0; k < M; ++k) acc[k] = 0;
#pragma unroll
        for (int j = 0; j < K; ++j)
#pragma unroll
            for (int k = 0; k < M; ++k) acc[k] += row[k * plen + j];
#pragma unroll
        for (int k = 0; k < M; ++k) bs[((size_t)i * M + k) * nb + b] = acc[k];
    }
}

// The window sum over columns [c0, c0 + 2r] (c0 a multiple of K) of one row
// of M skewed planes: the whole blocks from their block sums, the rest
// element by element.
template <int K, int M, typename V>
__device__ __forceinline__ void window_start(const V* row, int plen, const V* bsrow, int nb, int c0, int r, V S[M]) {
    const int b0 = c0 / K, q = (2 * r + 1) / K;
#pragma unroll
    for (int k = 0; k < M; ++k) S[k] = 0;
    for (int b = b0; b < b0 + q; ++b)
#pragma unroll
        for (int k = 0; k < M; ++k) S[k] += bsrow[k * nb + b];
    for (int j = (b0 + q) * K; j <= c0 + 2 * r; ++j)
#pragma unroll
        for (int k = 0; k < M; ++k) S[k] += row[k * plen + j + j / K];
}

// Clipped window extent along one axis of length len.
__device__ __forceinline__ int extent(int c, int r, int len) {
    return min(len - 1, c + r) - max(0, c - r) + 1;
}

struct StripTask {
    int x0, y0, y1;   // first output column; output rows [y0, y1)
};

__device__ __forceinline__ StripTask strip_task(int task, int strips, int tw, int th, int height) {
    const int band = task / strips, strip = task % strips;
    StripTask t;
    t.x0 = strip * tw;
    t.y0 = band * th;
    t.y1 = min(height, t.y0 + th);
    return t;
}

// --------------------------------------------------------------- guided filter

constexpr int GF_MOMENTS = 6;   // R, G, B, YR, YG, YB

struct GfParams {
    const float* in;
    size_t in_stride;
    float* out;
    size_t out_stride;
    int width, height, r;
    int tw, th, strips, tasks;
    double eps;
    YWeights w;
    double* ring;          // per CTA: (2r+1) rows x 6 moments x tw outputs
    uint32_t* status;
};

// One input pixel; zero outside the image or when `use` is false.  `last`
// marks the pixel's last read by the CTA (the row leaving the vertical
// window), loaded evict-first so that it leaves L2 before the rings do.
__device__ __forceinline__ float3 gf_pixel(const GfParams& P, int x, int y, bool use, bool last = false) {
    if (!use || x < 0 || x >= P.width) return make_float3(0.f, 0.f, 0.f);
    const float* p = P.in + (size_t)y * P.in_stride + (size_t)x * 3;
    if (last) return make_float3(__ldcs(p), __ldcs(p + 1), __ldcs(p + 2));
    return make_float3(__ldg(p), __ldg(p + 1), __ldg(p + 2));
}

// The six moments of one pixel; flags non-finite input.
__device__ __forceinline__ void gf_moments(const GfParams& P, float3 v, double m[GF_MOMENTS], bool& bad) {
    bad |= !(isfinite(v.x) && isfinite(v.y) && isfinite(v.z));
    const double r = v.x, g = v.y, b = v.z;
    const double y_ = fma(P.w.wb, b - g, fma(P.w.wr, r - g, g));
    m[0] = r; m[1] = g; m[2] = b;
    m[3] = y_ * r; m[4] = y_ * g; m[5] = y_ * b;
}

// 1/n for a window count 1 <= n <= 2^24: the correctly rounded binary32
// reciprocal refined by two Newton steps in binary64 (relative error below
// 2^-50).
__device__ __forceinline__ double rcp_count(int n) {
    const double x = (double)n;
    double q = (double)__frcp_rn((float)n);
    q = fma(q, fma(-x, q, 1.0), q);
    q = fma(q, fma(-x, q, 1.0), q);
    return q;
}

template <int NT, int R, int K, int MINB>
__global__ void __launch_bounds__(NT, MINB) gf_strip_kernel(const GfParams P) {
    constexpr int C1 = NT;                  // input columns of a strip
    constexpr int C1P = plane_len<K>(C1);
    extern __shared__ __align__(16) double smem_gf[];
    const int r = P.r, tw = P.tw, c2 = tw + 2 * r, c2p = c2 + c2 / K + 1;
    double* Vb = smem_gf;                                   // [R][6][C1P]  phase A sums
    double* ABb = Vb + (size_t)R * GF_MOMENTS * C1P;        // [R][6][c2p]  a (3), b (3) per centre
    double* H2b = Vb;                                       // [R][6][C1P]  phase C sums (aliases Vb)
    double* Bs = ABb + (size_t)R * GF_MOMENTS * c2p;        // [R][6][C1 / K] block sums (V, then a/b)
    constexpr int NBV = C1 / K;
    const int nba = c2 / K;
    const int period = 2 * r + 1;
    double* ring = P.ring + (size_t)blockIdx.x * period * GF_MOMENTS * tw;
    const int tid = threadIdx.x;
    bool bad = false, overflow = false;
    for (int task = blockIdx.x; task < P.tasks; task += gridDim.x) {
        const StripTask T = strip_task(task, P.strips, tw, P.th, P.height);
        const int xa = T.x0 - 2 * r;                        // image column of input column 0
        const int tc0 = max(0, T.y0 - r);                   // first centre row
        const int t_end = T.y1 - 1 + r;                     // last step (emits output row T.y1 - 1)
        const int last_centre = min(P.height - 1, t_end);
        // phase A state: window sums of the column's moments for centre row t
        double V[GF_MOMENTS];
        {
            const int x = xa + tid;
#pragma unroll
            for (int k = 0; k < GF_MOMENTS; ++k) V[k] = 0.0;
            for (int y = max(0, tc0 - r); y <= min(P.height - 1, tc0 + r - 1); ++y) {
                if (x < 0 || x >= P.width) break;
                double m[GF_MOMENTS];
                gf_moments(P, gf_pixel(P, x, y, true), m, bad);
#pragma unroll
                for (int k = 0; k < GF_MOMENTS; ++k) V[k] += m[k];
            }
        }
        // phase D state: window sums of the centres' horizontal a/b sums
        double Q[GF_MOMENTS];
#pragma unroll
        for (int k = 0; k < GF_MOMENTS; ++k) Q[k] = 0.0;
        for (int tb = tc0; tb <= t_end; tb += R) {
            const int rows = min(R, last_centre - tb + 1);   // centre rows in this block (may be <= 0)
            // A: vertical window sums, one column per thread
            if (rows > 0) {
                const int x = xa + tid;
                // every pixel of the block's rows is requested before any is used
                float3 pin[R], pout[R];
#pragma unroll
                for (int i = 0; i < R; ++i) {
                    const int t = tb + i;
                    pin[i] = gf_pixel(P, x, t + r, i < rows && t + r <= P.height - 1);
                    pout[i] = gf_pixel(P, x, t - r - 1, i < rows && t - r - 1 >= max(0, tc0 - r), true);
                }
#pragma unroll
                for (int i = 0; i < R; ++i) {
                    if (i >= rows) break;
                    double m[GF_MOMENTS], l[GF_MOMENTS];
                    gf_moments(P, pin[i], m, bad);
                    gf_moments(P, pout[i], l, bad);
                    double* vrow = Vb + (size_t)i * GF_MOMENTS * C1P + sk<K>(tid);
#pragma unroll
                    for (int k = 0; k < GF_MOMENTS; ++k) {
                        V[k] += m[k] - l[k];
                        vrow[k * C1P] = V[k];
                    }
                }
            }
            __syncthreads();
            block_sums<NT, K, GF_MOMENTS>(Vb, C1P, max(rows, 0), NBV, Bs);
            __syncthreads();
            // B: horizontal window sums per centre, then a and b
            const int segs_b = (c2 + K - 1) / K;
            for (int item = tid; item < max(rows, 0) * segs_b; item += NT) {
                const int i = item / segs_b, c0 = (item % segs_b) * K, c1 = min(c0 + K, c2);
                const int t = tb + i;
                const double* vrow = Vb + (size_t)i * GF_MOMENTS * C1P;
                double* abrow = ABb + (size_t)i * GF_MOMENTS * c2p;
                double S[GF_MOMENTS];
                window_start<K, GF_MOMENTS>(vrow, C1P, Bs + (size_t)i * GF_MOMENTS * NBV, NBV, c0, r, S);
                const int wy = extent(t, r, P.height);
                for (int c = c0; c < c1; ++c) {
                    if (c > c0)
#pragma unroll
                        for (int k = 0; k < GF_MOMENTS; ++k)
                            S[k] += vrow[k * C1P + sk<K>(c + 2 * r)] - vrow[k * C1P + sk<K>(c - 1)];
                    const int xc = T.x0 - r + c;
                    if (xc < 0 || xc >= P.width) {
#pragma unroll
                        for (int k = 0; k < GF_MOMENTS; ++k) abrow[k * c2p + sk<K>(c)] = 0.0;
                        continue;
                    }
                    const double inv_n = rcp_count(extent(xc, r, P.width) * wy);
                    const double sy = fma(P.w.wb, S[2] - S[1], fma(P.w.wr, S[0] - S[1], S[1]));
                    const double syy = fma(P.w.wb, S[5] - S[4], fma(P.w.wr, S[3] - S[4], S[4]));
                    const double my = sy * inv_n;
                    double var = syy * inv_n - my * my;
                    if (var < 0) var = 0;
                    const double inv = 1.0 / (var + P.eps);
#pragma unroll
                    for (int ch = 0; ch < 3; ++ch) {
                        const double mp = S[ch] * inv_n;
                        const double cov = S[3 + ch] * inv_n - my * mp;
                        const double a = cov * inv;
                        const double b = mp - a * my;
                        overflow |= !(isfinite(a) && isfinite(b));
                        abrow[ch * c2p + sk<K>(c)] = a;
                        abrow[(3 + ch) * c2p + sk<K>(c)] = b;
                    }
                }
            }
            __syncthreads();
            block_sums<NT, K, GF_MOMENTS>(ABb, c2p, max(rows, 0), nba, Bs);
            __syncthreads();
            // C: horizontal window sums of a and b per output column
            const int segs_c = (tw + K - 1) / K;
            for (int item = tid; item < max(rows, 0) * segs_c; item += NT) {
                const int i = item / segs_c, o0 = (item % segs_c) * K, o1 = min(o0 + K, tw);
                const double* abrow = ABb + (size_t)i * GF_MOMENTS * c2p;
                double* hrow = H2b + (size_t)i * GF_MOMENTS * C1P;
                double S[GF_MOMENTS];
                window_start<K, GF_MOMENTS>(abrow, c2p, Bs + (size_t)i * GF_MOMENTS * nba, nba, o0, r, S);
                for (int o = o0; o < o1; ++o) {
                    if (o > o0)
#pragma unroll
                        for (int k = 0; k < GF_MOMENTS; ++k)
                            S[k] += abrow[k * c2p + sk<K>(o + 2 * r)] - abrow[k * c2p + sk<K>(o - 1)];
#pragma unroll
                    for (int k = 0; k < GF_MOMENTS; ++k) hrow[k * C1P + sk<K>(o)] = S[k];
                }
            }
            __syncthreads();
            // D: vertical window sums of C's rows, one output column per thread.
            //    The leaving ring rows and the input pixels of up to four steps
            //    are requested before any is used (a step's ring slot is the one
            //    it overwrites, so no more steps than the ring has rows).
            if (tid < tw) {
                const int x = T.x0 + tid;
                const int steps = min(R, t_end - tb + 1);
                const int chunk = period >= 4 ? 4 : 1;
                for (int i0 = 0; i0 < steps; i0 += chunk) {
                    double lv[4][GF_MOMENTS];
                    float3 pv[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int i = i0 + u, t = tb + i;
                        const bool live = u < chunk && i < steps;
                        const bool leave = live && t - period >= tc0;
                        const double* slot = ring + (size_t)(t % period) * GF_MOMENTS * tw + tid;
#pragma unroll
                        for (int k = 0; k < GF_MOMENTS; ++k) lv[u][k] = leave ? slot[(size_t)k * tw] : 0.0;
                        const int yo = t - r;
                        pv[u] = gf_pixel(P, x, yo, live && yo >= T.y0 && yo < T.y1);
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int i = i0 + u, t = tb + i;
                        if (u >= chunk || i >= steps) break;
                        double* slot = ring + (size_t)(t % period) * GF_MOMENTS * tw + tid;
                        if (t <= last_centre) {
                            const double* hrow = H2b + (size_t)i * GF_MOMENTS * C1P + sk<K>(tid);
#pragma unroll
                            for (int k = 0; k < GF_MOMENTS; ++k) {
                                const double h = hrow[k * C1P];
                                Q[k] += h - lv[u][k];
                                slot[(size_t)k * tw] = h;
                            }
                        } else {
#pragma unroll
                            for (int k = 0; k < GF_MOMENTS; ++k) Q[k] -= lv[u][k];
                        }
                        const int yo = t - r;
                        if (yo < T.y0 || yo >= T.y1 || x >= P.width) continue;
                        const float pc[3] = {pv[u].x, pv[u].y, pv[u].z};
                        const double Y = working_y(pc[0], pc[1], pc[2], P.w);
                        const double inv_n = rcp_count(extent(x, r, P.width) * extent(yo, r, P.height));
                        float* o = P.out + (size_t)yo * P.out_stride + (size_t)x * 3;
#pragma unroll
                        for (int ch = 0; ch < 3; ++ch) {
                            const double q = (Q[ch] * inv_n) * Y + Q[3 + ch] * inv_n;
                            const double delta = q - (double)pc[ch];
                            if (delta == 0) {
                                __stcs(o + ch, pc[ch]);   // written once, never re-read: evict first
                                continue;
                            }
                            if (!isfinite(q) || fabs(q) > (double)FLT_MAX) overflow = true;
                            __stcs(o + ch, (float)q);
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
    if (P.status) {
        if (bad) atomicMax(P.status, (uint32_t)((401u << 8) | ST_INVALID));
        if (overflow) atomicMax(P.status, (uint32_t)((400u << 8) | ST_OVERFLOW));
    }
}

// ---------------------------------------------------------- local statistics

constexpr int LS_NT = 256, LS_R = 4, LS_K = 8, LS_MAX_R = 32;

struct LsParams {
    const float* in;
    size_t in_stride;
    int width, height, r;
    int tw, th, strips, tasks;
    void* mean_out;
    void* var_out;
    uint32_t* count_out;
};

// Byte offsets of the local-statistics planes in shared memory (16-byte
// aligned).  The output staging planes are channel-major and skewed like the
// sum planes, so that the row segments' K-strided writes do not conflict.
struct LsSmem {
    size_t v, n, o, c, bv, bn, total;
    int twp;
};
__host__ __device__ inline LsSmem ls_smem_layout(int tw, size_t out_bytes) {
    const size_t c1p = plane_len<LS_K>(LS_NT);
    auto up = [](size_t b) { return (b + 15) & ~(size_t)15; };
    LsSmem L;
    L.twp = plane_len<LS_K>(tw);
    L.v = 0;
    L.n = up(L.v + (size_t)LS_R * 6 * c1p * sizeof(double));
    L.o = up(L.n + (size_t)LS_R * 3 * c1p * sizeof(int));
    L.c = up(L.o + (size_t)LS_R * 6 * L.twp * out_bytes);
    L.bv = up(L.c + (size_t)LS_R * 3 * L.twp * sizeof(uint32_t));
    L.bn = up(L.bv + (size_t)LS_R * 6 * (LS_NT / LS_K) * sizeof(double));
    L.total = up(L.bn + (size_t)LS_R * 3 * (LS_NT / LS_K) * sizeof(int));
    return L;
}

template <typename T>
__global__ void __launch_bounds__(LS_NT, 2) ls_strip_kernel(const LsParams P) {
    constexpr int C1P = plane_len<LS_K>(LS_NT);
    extern __shared__ __align__(16) double smem_ls[];
    const LsSmem L = ls_smem_layout(P.tw, sizeof(T));
    char* base = reinterpret_cast<char*>(smem_ls);
    double* Vb = reinterpret_cast<double*>(base + L.v);       // [R][6][C1P]: s1 x3, s2 x3
    int* Nb = reinterpret_cast<int*>(base + L.n);             // [R][3][C1P]
    T* Ob = reinterpret_cast<T*>(base + L.o);                 // [6][R][twp]: mean x3, var x3
    uint32_t* Cb = reinterpret_cast<uint32_t*>(base + L.c);   // [3][R][twp]
    double* BsV = reinterpret_cast<double*>(base + L.bv);     // [R][6][NB] block sums
    int* BsN = reinterpret_cast<int*>(base + L.bn);           // [R][3][NB]
    constexpr int NB = LS_NT / LS_K;
    const int r = P.r, tw = P.tw, twp = L.twp, tid = threadIdx.x;
    T* mean_out = static_cast<T*>(P.mean_out);
    T* var_out = static_cast<T*>(P.var_out);
    for (int task = blockIdx.x; task < P.tasks; task += gridDim.x) {
        const StripTask Tk = strip_task(task, P.strips, tw, P.th, P.height);
        const int xa = Tk.x0 - r;
        // the task's shift: its first output pixel, per channel (0 if not finite)
        double shift[3];
        {
            const float* p = P.in + (size_t)Tk.y0 * P.in_stride + (size_t)Tk.x0 * 3;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float v = __ldg(p + c);
                shift[c] = isfinite(v) ? (double)v : 0.0;
            }
        }
        const int x = xa + tid;
        const bool in_image = x >= 0 && x < P.width;
        double s1[3] = {0, 0, 0}, s2[3] = {0, 0, 0};
        int n[3] = {0, 0, 0};
        auto load = [&](int y, bool use, bool last = false) -> float3 {
            if (!use || !in_image) return make_float3(NAN, NAN, NAN);
            const float* p = P.in + (size_t)y * P.in_stride + (size_t)x * 3;
            if (last) return make_float3(__ldcs(p), __ldcs(p + 1), __ldcs(p + 2));
            return make_float3(__ldg(p), __ldg(p + 1), __ldg(p + 2));
        };
        // adds (sign +1) or removes (sign -1) one pixel's finite channels
        auto add = [&](float3 v, int sign) {
            const float c3[3] = {v.x, v.y, v.z};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                if (!isfinite(c3[c])) continue;
                const double d = (double)c3[c] - shift[c];
                s1[c] += sign > 0 ? d : -d;
                s2[c] += sign > 0 ? d * d : -(d * d);
                n[c] += sign;
            }
        };
        for (int y = max(0, Tk.y0 - r); y <= min(P.height - 1, Tk.y0 + r - 1); ++y) add(load(y, true), 1);
        for (int tb = Tk.y0; tb < Tk.y1; tb += LS_R) {
            const int rows = min(LS_R, Tk.y1 - tb);
            // A: vertical window sums of the column; every pixel of the block's
            //    rows is requested before any is used
            float3 pin[LS_R], pout[LS_R];
#pragma unroll
            for (int i = 0; i < LS_R; ++i) {
                const int t = tb + i;
                pin[i] = load(t + r, i < rows && t + r <= P.height - 1);
                pout[i] = load(t - r - 1, i < rows && t - r - 1 >= max(0, Tk.y0 - r), true);
            }
#pragma unroll
            for (int i = 0; i < LS_R; ++i) {
                if (i >= rows) break;
                add(pin[i], 1);
                add(pout[i], -1);
                double* vrow = Vb + (size_t)i * 6 * C1P + sk<LS_K>(tid);
                int* nrow = Nb + (size_t)i * 3 * C1P + sk<LS_K>(tid);
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    vrow[c * C1P] = s1[c];
                    vrow[(3 + c) * C1P] = s2[c];
                    nrow[c * C1P] = n[c];
                }
            }
            __syncthreads();
            block_sums<LS_NT, LS_K, 6>(Vb, C1P, rows, NB, BsV);
            block_sums<LS_NT, LS_K, 3>(Nb, C1P, rows, NB, BsN);
            __syncthreads();
            // B: horizontal window sums per output column, mean and variance
            const int segs = (tw + LS_K - 1) / LS_K;
            for (int item = tid; item < rows * segs; item += LS_NT) {
                const int i = item / segs, o0 = (item % segs) * LS_K, o1 = min(o0 + LS_K, tw);
                const double* vrow = Vb + (size_t)i * 6 * C1P;
                const int* nrow = Nb + (size_t)i * 3 * C1P;
                double S[6];
                int N[3];
                window_start<LS_K, 6>(vrow, C1P, BsV + (size_t)i * 6 * NB, NB, o0, r, S);
                window_start<LS_K, 3>(nrow, C1P, BsN + (size_t)i * 3 * NB, NB, o0, r, N);
                for (int o = o0; o < o1; ++o) {
                    if (o > o0) {
                        const int in_j = sk<LS_K>(o + 2 * r), out_j = sk<LS_K>(o - 1);
#pragma unroll
                        for (int k = 0; k < 6; ++k) S[k] += vrow[k * C1P + in_j] - vrow[k * C1P + out_j];
#pragma unroll
                        for (int c = 0; c < 3; ++c) N[c] += nrow[c * C1P + in_j] - nrow[c * C1P + out_j];
                    }
                    const int so = sk<LS_K>(o);
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        Cb[((size_t)c * LS_R + i) * twp + so] = (uint32_t)N[c];
                        T mean = (T)NAN, var = (T)NAN;
                        if (N[c]) {
                            const double inv = rcp_count(N[c]);
                            const double m = S[c] * inv;
                            double v = (S[3 + c] - S[c] * m) * inv;
                            if (v < 0) v = 0;
                            mean = (T)(shift[c] + m);
                            var = (T)v;
                        }
                        Ob[((size_t)c * LS_R + i) * twp + so] = mean;
                        Ob[((size_t)(3 + c) * LS_R + i) * twp + so] = var;
                    }
                }
            }
            __syncthreads();
            // coalesced stores of the block's rows
            const int width_out = min(tw, P.width - Tk.x0);
            for (int e = tid; e < rows * width_out * 3; e += LS_NT) {
                const int i = e / (width_out * 3), rem = e % (width_out * 3);
                const int o = rem / 3, c = rem % 3;
                const size_t at = ((size_t)(tb + i) * P.width + Tk.x0 + o) * 3 + c;
                const int so = sk<LS_K>(o);
                __stcs(mean_out + at, Ob[((size_t)c * LS_R + i) * twp + so]);
                __stcs(var_out + at, Ob[((size_t)(3 + c) * LS_R + i) * twp + so]);
                if (P.count_out) __stcs(P.count_out + at, Cb[((size_t)c * LS_R + i) * twp + so]);
            }
            __syncthreads();
        }
    }
}

#define SP_CUDA(call)                                                         \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) {                                              \
            set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
            return RE_CUDA_ERROR;                                             \
        }                                                                     \
    } while (0)

// Bands of output rows: when the strips leave room, as many equal bands as
// there are resident CTAs per strip, so that each CTA streams one long band
// and pays the vertical halo (`halo` rows above and below) once; bands stay at
// least 2 halo (and 16) rows tall.
int band_height(int height, int strips, int ctas, int halo) {
    const int bands = std::max(1, ctas / strips);
    int th = (height + bands - 1) / bands;
    th = std::max(th, std::max(16, 2 * halo));
    return std::min(th, height);
}

int sm_count() {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

struct GfLaunch {
    GfParams P;
    dim3 grid;
    int threads;
    size_t smem;
    void (*kernel)(GfParams);
};

// MINB CTAs per SM.  Up to r = 32, two CTAs of 256 columns and 4-row blocks
// (each CTA's ring of a/b row sums is at most 400 KB, so the resident rings
// fill most of the 126 MB L2 at r = 32, yet the second CTA per SM still wins:
// 2.08 ms against 2.88 ms for one CTA of 8-row blocks on 6000x4000); one CTA
// of 512 columns above.
template <int NT, int R, int K, int MINB>
GfLaunch gf_plan(GfParams P, int sms) {
    GfLaunch L;
    P.tw = NT - 4 * P.r;
    P.strips = (P.width + P.tw - 1) / P.tw;
    const int ctas = MINB * sms;
    P.th = band_height(P.height, P.strips, ctas, 2 * P.r);
    P.tasks = P.strips * ((P.height + P.th - 1) / P.th);
    const int c2 = P.tw + 2 * P.r;
    L.smem = ((size_t)R * GF_MOMENTS * plane_len<K>(NT) + (size_t)R * GF_MOMENTS * (c2 + c2 / K + 1) +
              (size_t)R * GF_MOMENTS * (NT / K)) * sizeof(double);
    L.grid = dim3(std::min(P.tasks, ctas));
    L.threads = NT;
    L.kernel = gf_strip_kernel<NT, R, K, MINB>;
    L.P = P;
    return L;
}

GfLaunch gf_choose(const GfParams& P, int sms) {
    if (P.r <= 16) return gf_plan<256, 4, 8, 2>(P, sms);
    if (P.r <= 32) return gf_plan<256, 4, 8, 2>(P, sms);
    return gf_plan<512, 4, 16, 1>(P, sms);
}

size_t gf_ring_bytes(const GfLaunch& L) {
    return (size_t)L.grid.x * (2 * L.P.r + 1) * GF_MOMENTS * L.P.tw * sizeof(double);
}

re_status gf_validate(const float* in, size_t in_stride, const float* out, size_t out_stride, uint32_t width,
                      uint32_t height, uint32_t radius, double epsilon, uint32_t space) {
    if (radius > 64 || !std::isfinite(epsilon) || epsilon < 0x1p-24 || epsilon > 65536.0) {
        set_last_error("guided filter requires radius 0..64 and finite epsilon [2^-24,65536]");
        return RE_INVALID_ARGUMENT;
    }
    if (space > 1) {
        set_last_error("guided filter requires scene-linear working RGB");
        return RE_INVALID_ARGUMENT;
    }
    if (!width || !height || !in || !out || in_stride < (size_t)width * 3 || out_stride < (size_t)width * 3) {
        set_last_error("guided filter requires nonempty addressable bounds");
        return RE_INVALID_ARGUMENT;
    }
    const char* ib = reinterpret_cast<const char*>(in);
    const char* ie = reinterpret_cast<const char*>(in + ((size_t)height - 1) * in_stride + (size_t)width * 3);
    const char* ob = reinterpret_cast<const char*>(out);
    const char* oe = reinterpret_cast<const char*>(out + ((size_t)height - 1) * out_stride + (size_t)width * 3);
    if (ob < ie && ib < oe) {
        set_last_error("guided filter output must not overlap its input");
        return RE_INVALID_ARGUMENT;
    }
    return RE_OK;
}

GfParams gf_params(const float* in, size_t in_stride, float* out, size_t out_stride, uint32_t width,
                   uint32_t height, uint32_t radius, double epsilon, uint32_t space) {
    GfParams P{};
    P.in = in;
    P.in_stride = in_stride;
    P.out = out;
    P.out_stride = out_stride;
    P.width = (int)width;
    P.height = (int)height;
    P.r = (int)radius;
    P.eps = epsilon;
    P.w = space == 0 ? YWeights{0.28807112822929337, 0.00008565396060525903}
                     : YWeights{0.26270021201126703, 0.059301716469861945};
    return P;
}

re_status gf_enqueue(GfLaunch L, void* scratch, uint32_t* status, cudaStream_t stream) {
    L.P.ring = static_cast<double*>(scratch);
    L.P.status = status;
    SP_CUDA(cudaFuncSetAttribute(L.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem));
    L.kernel<<<L.grid, L.threads, L.smem, stream>>>(L.P);
    SP_CUDA(cudaGetLastError());
    return RE_OK;
}

template <typename T>
re_status local_statistics(const float* in, size_t in_stride, uint32_t width, uint32_t height, uint32_t radius,
                           T* mean_out, T* var_out, uint32_t* count_out, void* stream_) {
    if (radius > LS_MAX_R) {
        set_last_error("local statistics radius must be in 0..32");
        return RE_INVALID_ARGUMENT;
    }
    if (!width || !height || !in || !mean_out || !var_out || in_stride < (size_t)width * 3) {
        set_last_error("spatial operation requires nonempty addressable bounds");
        return RE_INVALID_ARGUMENT;
    }
    cudaStream_t stream = (cudaStream_t)stream_;
    LsParams P{};
    P.in = in;
    P.in_stride = in_stride;
    P.width = (int)width;
    P.height = (int)height;
    P.r = (int)radius;
    P.tw = LS_NT - 2 * P.r;
    P.strips = (P.width + P.tw - 1) / P.tw;
    const int ctas = 2 * sm_count();
    P.th = band_height(P.height, P.strips, ctas, P.r);
    P.tasks = P.strips * ((P.height + P.th - 1) / P.th);
    P.mean_out = mean_out;
    P.var_out = var_out;
    P.count_out = count_out;
    const size_t smem = ls_smem_layout(P.tw, sizeof(T)).total;
    SP_CUDA(cudaFuncSetAttribute(ls_strip_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ls_strip_kernel<T><<<std::min(P.tasks, ctas), LS_NT, smem, stream>>>(P);
    SP_CUDA(cudaGetLastError());
    return RE_OK;
}

struct Scratch {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~Scratch() {
        if (p) cudaFreeAsync(p, s);
    }
};

}  // namespace

extern "C" {

size_t re_guided_filter_scratch_bytes(uint32_t width, uint32_t height, uint32_t radius) {
    if (!width || !height || radius > 64) return 0;
    GfParams P = gf_params(nullptr, 0, nullptr, 0, width, height, radius, 1.0, 0);
    return 256 + gf_ring_bytes(gf_choose(P, sm_count()));
}

// SpatialOps.cpp:159-163 settings (radius extended to 64), 168-287 output.
re_status re_guided_filter_async(const float* in, size_t in_stride, float* out, size_t out_stride, uint32_t width,
                                 uint32_t height, uint32_t radius, double epsilon, uint32_t space,
                                 uint32_t* device_status, void* scratch, void* stream) {
    re_status s = gf_validate(in, in_stride, out, out_stride, width, height, radius, epsilon, space);
    if (s) return s;
    if (!scratch) {
        set_last_error("guided filter needs scratch of re_guided_filter_scratch_bytes()");
        return RE_INVALID_ARGUMENT;
    }
    const GfLaunch L = gf_choose(gf_params(in, in_stride, out, out_stride, width, height, radius, epsilon, space),
                                 sm_count());
    return gf_enqueue(L, static_cast<char*>(scratch) + 256, device_status, (cudaStream_t)stream);
}

re_status re_guided_filter(const float* in, size_t in_stride, float* out, size_t out_stride, uint32_t width,
                           uint32_t height, uint32_t radius, double epsilon, uint32_t space, void* stream_) {
    re_status s = gf_validate(in, in_stride, out, out_stride, width, height, radius, epsilon, space);
    if (s) return s;
    cudaStream_t stream = (cudaStream_t)stream_;
    const GfLaunch L = gf_choose(gf_params(in, in_stride, out, out_stride, width, height, radius, epsilon, space),
                                 sm_count());
    Scratch sc;
    sc.s = stream;
    SP_CUDA(scratch_alloc(&sc.p, 256 + gf_ring_bytes(L), stream));
    uint32_t* status = (uint32_t*)sc.p;
    SP_CUDA(cudaMemsetAsync(status, 0, 4, stream));
    s = gf_enqueue(L, static_cast<char*>(sc.p) + 256, status, stream);
    if (s) return s;
    uint32_t key = 0;
    SP_CUDA(cudaMemcpyAsync(&key, status, 4, cudaMemcpyDeviceToHost, stream));
    SP_CUDA(cudaStreamSynchronize(stream));
    if (key & ST_INVALID) {
        set_last_error("guided filter requires finite complete input halo");
        return RE_INVALID_ARGUMENT;
    }
    if (key & ST_OVERFLOW) {
        set_last_error("guided filter float32 output overflow");
        return RE_OVERFLOW_ERROR;
    }
    return RE_OK;
}

// SpatialOps.cpp:74-121 (radius extended to 32).
re_status re_local_statistics(const float* in, size_t in_stride, uint32_t width, uint32_t height, uint32_t radius,
                              float* mean_out, float* var_out, uint32_t* count_out, void* stream) {
    return local_statistics<float>(in, in_stride, width, height, radius, mean_out, var_out, count_out, stream);
}

re_status re_local_statistics_f64(const float* in, size_t in_stride, uint32_t width, uint32_t height,
                                  uint32_t radius, double* mean_out, double* var_out, uint32_t* count_out,
                                  void* stream) {
    return local_statistics<double>(in, in_stride, width, height, radius, mean_out, var_out, count_out, stream);
}

}  // extern "C"
