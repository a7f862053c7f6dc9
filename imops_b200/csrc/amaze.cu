// amaze.cu -- AMaZE demosaic for sm_100a, bit-identical to the reference's
// demosaic_algorithms::Amaze (pichromatic/src/demosaic.rs:358-1379).
//
// Why the structure looks like the reference's tile loop: the reference
// demosaics 128x128 tiles stepped by 96 from (-16,-16), restarts every tile
// from zeroed scratch, mirrors a 16-pixel border at the image edge, bounds a
// per-tile "Nyquist" region, and several stages update arrays in place while
// scanning (a site reads its left / upper neighbours' already-updated
// values).  All of that decides output bits, so one CTA owns one reference
// tile and each stage runs over the same index domain; only the iteration
// order within a stage is parallel, except where the reference's scan order
// is observable:
//   * the hcd / vcd refinement (demosaic.rs:700-786) is a chain along each
//     row (hcd, step 2) and each column (vcd, step 2): one thread per chain;
//   * the hvwt smoothing (demosaic.rs:949-958) and pmwt smoothing
//     (demosaic.rs:1109-1118) read the row above already updated: one row
//     per step, with a block barrier between rows.
// Divisions are IEEE (-prec-div) and the file is built with --fmad=false so
// every a*b+c rounds twice, as in the reference's Rust f32 code.
//
// Memory: the per-tile arrays of the reference total ~1.2 MB; the mosaic,
// hcd, vcd and hvwt (the most re-read) live in shared memory (224 KB), the
// others in a per-CTA slot of a global scratch buffer that the persistent
// grid reuses tile after tile, so it stays resident in L2.
#include "amaze.cuh"
#include "color.cuh"

#include <mutex>
#include <vector>

namespace imops {
namespace amaze {

constexpr int TS = 128, TSH = 64, NF = TS * TS, NH = TS * TSH;
constexpr int V1 = 128, V2 = 256, V3 = 384, P1 = 127, P2 = 254, P3 = 381, M1 = 129, M2 = 258, M3 = 387;
constexpr int NTHREADS = 512;
static_assert(NTHREADS % TS == 0 && NTHREADS % TSH == 0, "row mapping of the stage loops");

// global scratch per CTA slot: 8 full arrays, 14 half arrays, 2 byte maps
constexpr size_t SLOT_FLOATS = 8 * (size_t)NF + 14 * (size_t)NH;
constexpr size_t SLOT_BYTES = SLOT_FLOATS * 4 + 2 * (size_t)NH;
constexpr size_t SMEM_BYTES = (3 * (size_t)NF + (size_t)NH) * 4 + 64;

struct Bufs {
    float *mos, *hcd, *vcd, *hvwt;                                  // shared
    float *wv, *wh, *gsq, *vcda, *hcda, *cdd, *dgv, *dgh;           // global, full
    float *dgrb0, *dgrb1, *delp, *delm, *rbint, *q1m, *q1p, *pmwt;  // global, half
    float *rbm, *rbp, *nyqt, *rg, *d2h, *d2v;
    uint8_t *nyq, *nyq2;
};

struct Geo {
    int top, left, rr1, cc1, rrmin, ccmin, rrmax, ccmax;
};

struct Bayer {
    uint8_t c[4];
    __device__ __forceinline__ int at(int r, int q) const { return c[((r & 1) << 1) | (q & 1)]; }
};

// Mosaic sources: the reference's f32 mosaic, or a u16 sensor frame scaled
// on load with the same f32 arithmetic as imops_scale_u16 (so the values,
// and hence the output bits, are identical).
struct SrcF32 {
    const float* p;
    int W;
    __device__ __forceinline__ float operator()(int r, int q) const { return __ldg(p + (size_t)r * W + q); }
};
struct SrcU16 {
    const uint16_t* raw;
    int raw_w, cx, cy, pw, ph;
    float black[16], white[16];
    __device__ __forceinline__ float operator()(int r, int q) const {
        int sy = cy + r, sx = cx + q;
        int site = (sy % ph) * pw + (sx % pw);
        float v = (float)__ldg(raw + (size_t)sy * raw_w + sx);
        return (v - black[site]) / (white[site] - black[site]);
    }
};

template <class Src>
struct Params {
    Src in;
    int W, H;
    Bayer cfa;
    float clip;
    int ntx, ntiles;
    uint8_t* scratch;
};

__device__ __forceinline__ float sqr(float x) { return x * x; }
__device__ __forceinline__ float lim(float x, float lo, float hi) { return fmaxf(lo, fminf(x, hi)); }
__device__ __forceinline__ float ulim(float x, float y, float z) { return y < z ? lim(x, y, z) : lim(x, z, y); }
__device__ __forceinline__ float clampnan(float x, float lo, float hi) {
    if (isnan(x)) return (lo + hi) * 0.5f;
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

__host__ __device__ inline Geo tile_geo(int W, int H, int top, int left) {
    Geo g;
    g.top = top;
    g.left = left;
    int bottom = (top + 128 < H + 16) ? top + 128 : H + 16;
    int right = (left + 128 < W + 16) ? left + 128 : W + 16;
    g.rr1 = bottom - top;
    g.cc1 = right - left;
    g.rrmin = top < 0 ? 16 : 0;
    g.ccmin = left < 0 ? 16 : 0;
    g.rrmax = bottom > H ? H - top : g.rr1;
    g.ccmax = right > W ? W - left : g.cc1;
    return g;
}

// Largest flat index the border fill writes (same ranges as fill()).
static long fill_max_index(int W, int H, int top, int left) {
    Geo g = tile_geo(W, H, top, left);
    long hi = -1;
    auto span = [&](int r0, int r1, int c0, int c1) {
        if (r0 < r1 && c0 < c1) {
            long v = (long)(r1 - 1) * TS + (c1 - 1);
            if (v > hi) hi = v;
        }
    };
    if (g.rrmin > 0) span(0, 16, g.ccmin, g.ccmax);
    span(g.rrmin, g.rrmax, g.ccmin, g.ccmax);
    if (g.rrmax < g.rr1) span(g.rrmax, g.rrmax + 16, g.ccmin, g.ccmax);
    if (g.ccmin > 0) span(g.rrmin, g.rrmax, 0, 16);
    if (g.ccmax < g.cc1) span(g.rrmin, g.rrmax, g.ccmax, g.ccmax + 16);
    if (g.rrmin > 0 && g.ccmin > 0) span(0, 16, 0, 16);
    if (g.rrmax < g.rr1 && g.ccmax < g.cc1) span(g.rrmax, g.rrmax + 16, g.ccmax, g.ccmax + 16);
    if (g.rrmin > 0 && g.ccmax < g.cc1) span(0, 16, g.ccmax, g.ccmax + 16);
    if (g.rrmax < g.rr1 && g.ccmin > 0) span(g.rrmax, g.rrmax + 16, 0, 16);
    return hi;
}

bool size_supported(int W, int H) {
    if (W <= 0 || H <= 0) return false;
    for (int top = -16; top < H; top += 96)
        for (int left = -16; left < W; left += 96)
            if (fill_max_index(W, H, top, left) >= NF) return false;
    return true;
}

template <class P>
__device__ __forceinline__ float get_in(const P& p, int r, int q) {
    r = r < 0 ? 0 : (r > p.H - 1 ? p.H - 1 : r);
    q = q < 0 ? 0 : (q > p.W - 1 ? p.W - 1 : q);
    return p.in(r, q);
}

// One rectangular fill pass: rows [r0,r1) x cols [c0,c1) of the loop space;
// dst(rr,cc) / src(rr,cc) give the flat index and the value.
template <class Dst, class Src>
__device__ __forceinline__ void fill_pass(float* mos, int r0, int r1, int c0, int c1, Dst dst, Src src) {
    const int cc = c0 + (int)(threadIdx.x & (TS - 1));
    if (cc >= c1) return;
    for (int rr = r0 + (int)(threadIdx.x / TS); rr < r1; rr += NTHREADS / TS) mos[dst(rr, cc)] = src(rr, cc);
}

// Tile fill: demosaic.rs:499-610, passes in the reference's order so later
// passes overwrite earlier ones exactly as there.
template <class P>
__device__ void fill(const P& p, const Geo& g, float* mos) {
    const int top = g.top, left = g.left, W = p.W, H = p.H;
    if (g.rrmin == 0 && g.ccmin == 0 && g.rrmax == g.rr1 && g.ccmax == g.cc1) {
        fill_pass(mos, 0, g.rr1, 0, g.cc1, [](int rr, int cc) { return rr * TS + cc; },
                  [&](int rr, int cc) { return get_in(p, rr + top, cc + left); });
        return;
    }
    if (g.rrmin > 0)
        fill_pass(mos, 0, 16, g.ccmin, g.ccmax, [](int rr, int cc) { return rr * TS + cc; },
                  [&](int rr, int cc) { return get_in(p, 32 - rr + top, cc + left); });
    __syncthreads();
    fill_pass(mos, g.rrmin, g.rrmax, g.ccmin, g.ccmax, [](int rr, int cc) { return rr * TS + cc; },
              [&](int rr, int cc) { return get_in(p, rr + top, cc + left); });
    __syncthreads();
    if (g.rrmax < g.rr1)
        fill_pass(mos, 0, 16, g.ccmin, g.ccmax, [&](int rr, int cc) { return (g.rrmax + rr) * TS + cc; },
                  [&](int rr, int cc) { return get_in(p, H - rr - 2, left + cc); });
    __syncthreads();
    if (g.ccmin > 0)
        fill_pass(mos, g.rrmin, g.rrmax, 0, 16, [](int rr, int cc) { return rr * TS + cc; },
                  [&](int rr, int cc) { return get_in(p, rr + top, 32 - cc + left); });
    __syncthreads();
    if (g.ccmax < g.cc1)
        fill_pass(mos, g.rrmin, g.rrmax, 0, 16, [&](int rr, int cc) { return rr * TS + g.ccmax + cc; },
                  [&](int rr, int cc) { return get_in(p, top + rr, W - cc - 2); });
    __syncthreads();
    if (g.rrmin > 0 && g.ccmin > 0)
        fill_pass(mos, 0, 16, 0, 16, [](int rr, int cc) { return rr * TS + cc; },
                  [&](int rr, int cc) { return get_in(p, 32 - rr, 32 - cc); });
    __syncthreads();
    if (g.rrmax < g.rr1 && g.ccmax < g.cc1)
        fill_pass(mos, 0, 16, 0, 16, [&](int rr, int cc) { return (g.rrmax + rr) * TS + g.ccmax + cc; },
                  [&](int rr, int cc) { return get_in(p, H - rr - 2, W - cc - 2); });
    __syncthreads();
    if (g.rrmin > 0 && g.ccmax < g.cc1)
        fill_pass(mos, 0, 16, 0, 16, [&](int rr, int cc) { return rr * TS + g.ccmax + cc; },
                  [&](int rr, int cc) { return get_in(p, 32 - rr, W - cc - 2); });
    __syncthreads();
    if (g.rrmax < g.rr1 && g.ccmin > 0)
        fill_pass(mos, 0, 16, 0, 16, [&](int rr, int cc) { return (g.rrmax + rr) * TS + cc; },
                  [&](int rr, int cc) { return get_in(p, H - rr - 2, 32 - cc); });
}

// Loop helpers: every site of rows [r0,r1) x cols [c0,c1), and the R/B
// sites of those rows (first R/B column = c0 + parity of the row; c0 even).
// Threads map to (row group, column) directly: a tile row has at most 128
// sites and 64 R/B sites, so no integer division is needed.
template <class F>
__device__ __forceinline__ void for_rect(int r0, int r1, int c0, int c1, F f) {
    const int cc = c0 + (int)(threadIdx.x & (TS - 1));
    if (cc >= c1) return;
    for (int rr = r0 + (int)(threadIdx.x / TS); rr < r1; rr += NTHREADS / TS) f(rr, cc);
}

template <class F, class P>
__device__ __forceinline__ void for_rb(const P& p, const Geo& g, int r0, int r1, int c0, int c1, F f) {
    const int k = (int)(threadIdx.x & (TSH - 1));
    for (int rr = r0 + (int)(threadIdx.x / TSH); rr < r1; rr += NTHREADS / TSH) {
        int cc = c0 + (p.cfa.at(g.top + rr, g.left + 2) & 1) + 2 * k;
        if (cc < c1) f(rr, cc);
    }
}

// A subset of the block's threads working one stage: thread t of n.
struct Team {
    int t, n;
};
__device__ __forceinline__ Team whole_block() { return Team{(int)threadIdx.x, NTHREADS}; }
// warps 1.. of the block, while warp 0 runs a wavefront
constexpr int WORKERS = NTHREADS - 32;
__device__ __forceinline__ Team workers() { return Team{(int)threadIdx.x - 32, WORKERS}; }
__device__ __forceinline__ void workers_sync() { asm volatile("bar.sync 1, %0;" ::"r"(WORKERS) : "memory"); }

// R/B sites of rows [r0,r1) x cols [c0,c1) split over a team (c0 even).
template <class F, class P>
__device__ __forceinline__ void for_rb_team(const P& p, const Geo& g, Team tm, int r0, int r1, int c0, int c1,
                                            F f) {
    const int n = (r1 - r0) * TSH;
    for (int k = tm.t; k < n; k += tm.n) {
        int rr = r0 + (k >> 6);
        int cc = c0 + (p.cfa.at(g.top + rr, g.left + 2) & 1) + 2 * (k & (TSH - 1));
        if (cc < c1) f(rr, cc);
    }
}

// The kernel's dynamic shared memory, named at namespace scope so that the
// wavefronts index it directly (shared-memory loads, not generic ones).
extern __shared__ __align__(16) float amaze_smem[];

// Row wavefront of the weight smoothing (demosaic.rs:949-958 for hvwt,
// :1109-1118 for pmwt), run by ONE warp.  At R/B site (r, c) of rows
// [lo, rr1-lo) x cols [lo, cc1-lo):
//     alt = (w(r-1,c-1) + w(r-1,c+1) + w(r+1,c-1) + w(r+1,c+1)) / 4
//     if |0.5 - w(r,c)| < |0.5 - alt|: w(r,c) = alt
// where row r-1 holds already-updated values.  Lane L owns sites k = L and
// L+32 of every row and keeps the updated row in registers; the neighbours
// (r-1, c-+1) are sites k-1/k/k+1 of the previous row, fetched by shuffle.
// Sites outside the updated range keep their stored values.  Division by 4
// is exact, so * 0.25f gives the same bits.  post(r, c, w_new) runs after
// each update.  The array is amaze_smem[woff ...].
template <class P, class Post>
__device__ void wavefront(const P& p, const Geo& g, int woff, int lo, Post post) {
    float* const w = amaze_smem + woff;
    const int lane = threadIdx.x & 31;
    const int rhi = g.rr1 - lo, chi = g.cc1 - lo;
    // Bayer rows alternate the column parity of their R/B sites
    int par = p.cfa.at(g.top + lo, g.left + 2) & 1;
    const int n0 = (chi - lo + 1) >> 1, n1 = (chi - lo) >> 1;
    // row being updated: own value, stored upper neighbours (used where the
    // previous row was not updated) and the lower neighbours (not updated yet)
    float own[2], upl[2], upr[2], lwl[2], lwr[2];
    auto load = [&](int rr, int pr, float* o, float* ul, float* ur, float* dl, float* dr) {
        const int c0 = lo + pr, n = pr ? n1 : n0;
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int i = rr * TS + c0 + 2 * min(lane + 32 * j, n - 1);
            o[j] = w[i >> 1];
            ul[j] = w[(i - M1) >> 1];
            ur[j] = w[(i - P1) >> 1];
            dl[j] = w[(i + P1) >> 1];
            dr[j] = w[(i + M1) >> 1];
        }
    };
    load(lo, par, own, upl, upr, lwl, lwr);
    float prevA = 0.f, prevB = 0.f;  // updated previous row, sites lane / lane+32
    int nprev = 0;
    for (int rr = lo; rr < rhi; rr++) {
        const int n = par ? n1 : n0, c0 = lo + par;
        float nown[2], nul[2], nur[2], ndl[2], ndr[2];
        if (rr + 1 < rhi) load(rr + 1, par ^ 1, nown, nul, nur, ndl, ndr);
        const float aM = __shfl_up_sync(0xffffffffu, prevA, 1), aP = __shfl_down_sync(0xffffffffu, prevA, 1);
        const float bM = __shfl_up_sync(0xffffffffu, prevB, 1), bP = __shfl_down_sync(0xffffffffu, prevB, 1);
        const float a31 = __shfl_sync(0xffffffffu, prevA, 31), b0 = __shfl_sync(0xffffffffu, prevB, 0);
        float nv[2];
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int k = lane + 32 * j;
            const float vm1 = j == 0 ? aM : (lane == 0 ? a31 : bM);  // previous-row site k-1
            const float v0 = j == 0 ? prevA : prevB;                 // site k
            const float vp1 = j == 0 ? (lane == 31 ? b0 : aP) : bP;  // site k+1
            const int kl = par == 0 ? k - 1 : k, kr = par == 0 ? k : k + 1;
            const float ul = (kl >= 0 && kl < nprev) ? (par == 0 ? vm1 : v0) : upl[j];
            const float ur = (kr >= 0 && kr < nprev) ? (par == 0 ? v0 : vp1) : upr[j];
            const float alt = (ul + ur + lwl[j] + lwr[j]) * 0.25f;
            const float v = fabsf(0.5f - own[j]) < fabsf(0.5f - alt) ? alt : own[j];
            nv[j] = v;
            if (k < n) {
                w[(rr * TS + c0 + 2 * k) >> 1] = v;
                post(rr, c0 + 2 * k, rr * TS + c0 + 2 * k, v);
            }
        }
        prevA = nv[0];
        prevB = nv[1];
        nprev = n;
        par ^= 1;
#pragma unroll
        for (int j = 0; j < 2; j++) {
            own[j] = nown[j];
            upl[j] = nul[j];
            upr[j] = nur[j];
            lwl[j] = ndl[j];
            lwr[j] = ndr[j];
        }
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// stages

// demosaic.rs:612-622
__device__ void st_gradients(const Geo& g, const Bufs& b) {
    const float eps = 1e-5f;
    for_rect(2, g.rr1 - 2, 2, g.cc1 - 2, [&](int rr, int cc) {
        int i = rr * TS + cc;
        const float* m = b.mos;
        float dh = fabsf(m[i + 1] - m[i - 1]);
        float dv = fabsf(m[i + V1] - m[i - V1]);
        b.wv[i] = eps + fabsf(m[i + V2] - m[i]) + fabsf(m[i] - m[i - V2]) + dv;
        b.wh[i] = eps + fabsf(m[i + 2] - m[i]) + fabsf(m[i] - m[i - 2]) + dh;
        b.gsq[i] = sqr(dh) + sqr(dv);
    });
}

// demosaic.rs:624-698.  Also writes the zeros the reference's freshly
// allocated arrays hold just outside the computed band (read by the
// refinement at rows/cols 2,3 and rr1-4, rr1-3).
template <class P>
__device__ void st_colour_diff(const P& p, const Geo& g, const Bufs& b) {
    const float eps = 1e-5f, arth = 0.75f;
    const float clip8 = p.clip * 0.8f;
    for_rect(2, g.rr1 - 2, 2, g.cc1 - 2, [&](int rr, int cc) {
        int i = rr * TS + cc;
        bool in_r = rr >= 4 && rr < g.rr1 - 4, in_c = cc >= 4 && cc < g.cc1 - 4;
        if (!(in_r && in_c)) {
            if (in_c) { b.vcd[i] = 0.f; b.vcda[i] = 0.f; }
            if (in_r) { b.hcd[i] = 0.f; b.hcda[i] = 0.f; }
            return;
        }
        const float *m = b.mos, *wv = b.wv, *wh = b.wh;
        float cru = m[i - V1] * (wv[i - V2] + wv[i]) /
                    fmaxf(wv[i - V2] * (eps + m[i]) + wv[i] * (eps + m[i - V2]), 1e-10f);
        float crd = m[i + V1] * (wv[i + V2] + wv[i]) /
                    fmaxf(wv[i + V2] * (eps + m[i]) + wv[i] * (eps + m[i + V2]), 1e-10f);
        float crl = m[i - 1] * (wh[i - 2] + wh[i]) /
                    fmaxf(wh[i - 2] * (eps + m[i]) + wh[i] * (eps + m[i - 2]), 1e-10f);
        float crr = m[i + 1] * (wh[i + 2] + wh[i]) /
                    fmaxf(wh[i + 2] * (eps + m[i]) + wh[i] * (eps + m[i + 2]), 1e-10f);
        float guha = m[i - V1] + (m[i] - m[i - V2]) * 0.5f;
        float gdha = m[i + V1] + (m[i] - m[i + V2]) * 0.5f;
        float glha = m[i - 1] + (m[i] - m[i - 2]) * 0.5f;
        float grha = m[i + 1] + (m[i] - m[i + 2]) * 0.5f;
        float guar = fabsf(1.0f - cru) < arth ? m[i] * cru : guha;
        float gdar = fabsf(1.0f - crd) < arth ? m[i] * crd : gdha;
        float glar = fabsf(1.0f - crl) < arth ? m[i] * crl : glha;
        float grar = fabsf(1.0f - crr) < arth ? m[i] * crr : grha;
        float hwt = wh[i - 1] / fmaxf(wh[i - 1] + wh[i + 1], 1e-10f);
        float vwt = wv[i - V1] / fmaxf(wv[i + V1] + wv[i - V1], 1e-10f);
        float gintvha = vwt * gdha + (1.0f - vwt) * guha;
        float ginthha = hwt * grha + (1.0f - hwt) * glha;
        // the reference toggles a G/non-G switch per column; for a Bayer
        // row that equals the site's own colour test
        bool gsite = (p.cfa.at(g.top + rr, g.left + cc) & 1) != 0;
        float vcdv, hcdv, vcdalt, hcdalt;
        if (gsite) {
            vcdv = m[i] - (vwt * gdar + (1.0f - vwt) * guar);
            hcdv = m[i] - (hwt * grar + (1.0f - hwt) * glar);
            vcdalt = m[i] - gintvha;
            hcdalt = m[i] - ginthha;
        } else {
            vcdv = (vwt * gdar + (1.0f - vwt) * guar) - m[i];
            hcdv = (hwt * grar + (1.0f - hwt) * glar) - m[i];
            vcdalt = gintvha - m[i];
            hcdalt = ginthha - m[i];
        }
        float gu = guar, gd = gdar, gl = glar, gr = grar;
        if (m[i] > clip8 || gintvha > clip8 || ginthha > clip8) {
            vcdv = vcdalt;
            hcdv = hcdalt;
            gu = guha; gd = gdha; gl = glha; gr = grha;
        }
        b.vcd[i] = vcdv;
        b.hcd[i] = hcdv;
        b.vcda[i] = vcdalt;
        b.hcda[i] = hcdalt;
        b.dgv[i] = fminf(sqr(guha - gdha), sqr(gu - gd));
        b.dgh[i] = fminf(sqr(glha - grha), sqr(gl - gr));
    });
}

// Bound a colour difference by the two neighbours along its direction
// (the clamp half of demosaic.rs:724-784).  nb0/nb1: neighbours.
__device__ __forceinline__ float cd_bound(float cd, float m, float nb0, float nb1, bool gsite, float clip) {
    const float eps = 1e-5f;
    if (gsite) {
        float gint = -cd + m;
        if (cd > 0.0f) {
            if (3.0f * cd > (gint + m)) {
                cd = -ulim(gint, nb0, nb1) + m;
            } else {
                float w = 1.0f - 3.0f * cd / (eps + gint + m);
                cd = w * cd + (1.0f - w) * (-ulim(gint, nb0, nb1) + m);
            }
        }
        if (gint > clip) cd = -ulim(gint, nb0, nb1) + m;
    } else {
        float gint = cd + m;
        if (cd < 0.0f) {
            if (3.0f * cd < -(gint + m)) {
                cd = ulim(gint, nb0, nb1) - m;
            } else {
                float w = 1.0f + 3.0f * cd / (eps + gint + m);
                cd = w * cd + (1.0f - w) * (ulim(gint, nb0, nb1) - m);
            }
        }
        if (gint > clip) cd = ulim(gint, nb0, nb1) - m;
    }
    return cd;
}

// demosaic.rs:700-786.  hcd at a site depends on the already-refined hcd two
// columns left, vcd on the refined vcd two rows up; the two are independent,
// so each (row, parity) hcd chain and each (column, parity) vcd chain is one
// thread walking in the reference's order.
template <class P>
__device__ void st_cd_refine(const P& p, const Geo& g, const Bufs& b) {
    const int nr = g.rr1 - 8, nc = g.cc1 - 8;
    const int nh = nr > 0 ? 2 * nr : 0, nv = nc > 0 ? 2 * nc : 0;
    const float* m = b.mos;
    for (int t = threadIdx.x; t < nh + nv; t += blockDim.x) {
        if (t < nh) {
            int rr = 4 + t / 2, cc0 = 4 + (t & 1);
            bool gs = (p.cfa.at(g.top + rr, g.left + cc0) & 1) != 0;
            float* hcd = b.hcd;
            const float* ha = b.hcda;
            for (int cc = cc0; cc < g.cc1 - 4; cc += 2) {
                int i = rr * TS + cc;
                float hv = 3.0f * (sqr(hcd[i - 2]) + sqr(hcd[i]) + sqr(hcd[i + 2])) -
                           sqr(hcd[i - 2] + hcd[i] + hcd[i + 2]);
                float hav = 3.0f * (sqr(ha[i - 2]) + sqr(ha[i]) + sqr(ha[i + 2])) -
                            sqr(ha[i - 2] + ha[i] + ha[i + 2]);
                float v = hav < hv ? ha[i] : hcd[i];
                hcd[i] = cd_bound(v, m[i], m[i - 1], m[i + 1], gs, p.clip);
            }
        } else {
            int tt = t - nh;
            int cc = 4 + tt / 2, rr0 = 4 + (tt & 1);
            bool gs = (p.cfa.at(g.top + rr0, g.left + cc) & 1) != 0;
            float* vcd = b.vcd;
            const float* va = b.vcda;
            for (int rr = rr0; rr < g.rr1 - 4; rr += 2) {
                int i = rr * TS + cc;
                float vv = 3.0f * (sqr(vcd[i - V2]) + sqr(vcd[i]) + sqr(vcd[i + V2])) -
                           sqr(vcd[i - V2] + vcd[i] + vcd[i + V2]);
                float vav = 3.0f * (sqr(va[i - V2]) + sqr(va[i]) + sqr(va[i + V2])) -
                            sqr(va[i - V2] + va[i] + va[i + V2]);
                float v = vav < vv ? va[i] : vcd[i];
                vcd[i] = cd_bound(v, m[i], m[i - V1], m[i + V1], gs, p.clip);
            }
        }
    }
    __syncthreads();
    for_rb(p, g, 4, g.rr1 - 4, 4, g.cc1 - 4, [&](int rr, int cc) {
        int i = rr * TS + cc;
        b.cdd[i] = sqr(b.vcd[i] - b.hcd[i]);
    });
}

// demosaic.rs:788-828
template <class P>
__device__ void st_hv_weight(const P& p, const Geo& g, const Bufs& b) {
    const float epssq = 1e-10f;
    for_rb(p, g, 6, g.rr1 - 6, 6, g.cc1 - 6, [&](int rr, int cc) {
        int i = rr * TS + cc;
        const float *vcd = b.vcd, *hcd = b.hcd, *dv = b.dgv, *dh = b.dgh;
        float uave = vcd[i] + vcd[i - V1] + vcd[i - V2] + vcd[i - V3];
        float dave = vcd[i] + vcd[i + V1] + vcd[i + V2] + vcd[i + V3];
        float lave = hcd[i] + hcd[i - 1] + hcd[i - 2] + hcd[i - 3];
        float rave = hcd[i] + hcd[i + 1] + hcd[i + 2] + hcd[i + 3];
        float vu = sqr(vcd[i] - uave) + sqr(vcd[i - V1] - uave) + sqr(vcd[i - V2] - uave) + sqr(vcd[i - V3] - uave);
        float vd = sqr(vcd[i] - dave) + sqr(vcd[i + V1] - dave) + sqr(vcd[i + V2] - dave) + sqr(vcd[i + V3] - dave);
        float hl = sqr(hcd[i] - lave) + sqr(hcd[i - 1] - lave) + sqr(hcd[i - 2] - lave) + sqr(hcd[i - 3] - lave);
        float hr = sqr(hcd[i] - rave) + sqr(hcd[i + 1] - rave) + sqr(hcd[i + 2] - rave) + sqr(hcd[i + 3] - rave);
        float hwt = b.wh[i - 1] / fmaxf(b.wh[i - 1] + b.wh[i + 1], 1e-10f);
        float vwt = b.wv[i - V1] / fmaxf(b.wv[i + V1] + b.wv[i - V1], 1e-10f);
        float vvar = epssq + vwt * vd + (1.0f - vwt) * vu;
        float hvar = epssq + hwt * hr + (1.0f - hwt) * hl;
        float vu1 = dv[i] + dv[i - V1] + dv[i - V2];
        float vd1 = dv[i] + dv[i + V1] + dv[i + V2];
        float hl1 = dh[i] + dh[i - 1] + dh[i - 2];
        float hr1 = dh[i] + dh[i + 1] + dh[i + 2];
        float vvar1 = epssq + vwt * vd1 + (1.0f - vwt) * vu1;
        float hvar1 = epssq + hwt * hr1 + (1.0f - hwt) * hl1;
        float varwt = hvar / fmaxf(vvar + hvar, 1e-10f);
        float diffwt = hvar1 / fmaxf(vvar1 + hvar1, 1e-10f);
        if ((0.5f - varwt) * (0.5f - diffwt) > 0.0f && fabsf(0.5f - diffwt) < fabsf(0.5f - varwt))
            b.hvwt[i >> 1] = varwt;
        else
            b.hvwt[i >> 1] = diffwt;
    });
}

struct NyqBox {
    int on, r0, r1, c0, c1;
};

// demosaic.rs:830-869: Nyquist test, flags and their bounding box
// (first/last flagged row, min/max flagged column).
template <class P>
__device__ NyqBox st_nyquist_flags(const P& p, const Geo& g, const Bufs& b, int* sh) {
    const float nyqthresh = 0.5f;
    const float go0 = 0.14659727707323927f, go1 = 0.103592713382435f, go2 = 0.0732036125103057f,
                go3 = 0.0365543548389495f;
    const float gg0 = nyqthresh * 0.07384411893421103f, gg1 = nyqthresh * 0.06207511968171489f,
                gg2 = nyqthresh * 0.0521818194747806f, gg3 = nyqthresh * 0.03687419286733595f,
                gg4 = nyqthresh * 0.03099732204057846f, gg5 = nyqthresh * 0.018413194161458882f;
    if (threadIdx.x == 0) {
        sh[0] = 1 << 30;  // min row
        sh[1] = -1;       // max row
        sh[2] = TS + 1;   // min col
        sh[3] = 0;        // max col
    }
    __syncthreads();
    int lr0 = 1 << 30, lr1 = -1, lc0 = TS + 1, lc1 = 0;
    for_rb(p, g, 6, g.rr1 - 6, 6, g.cc1 - 6, [&](int rr, int cc) {
        int i = rr * TS + cc;
        const float *q = b.cdd, *s = b.gsq;
        float t = (go0 * q[i] + go1 * (q[i - M1] + q[i - P1] + q[i + P1] + q[i + M1]) +
                   go2 * (q[i - V2] + q[i - 2] + q[i + 2] + q[i + V2]) +
                   go3 * (q[i - M2] + q[i - P2] + q[i + P2] + q[i + M2])) -
                  (gg0 * s[i] + gg1 * (s[i - V1] + s[i + 1] + s[i - 1] + s[i + V1]) +
                   gg2 * (s[i - M1] + s[i - P1] + s[i + P1] + s[i + M1]) +
                   gg3 * (s[i - V2] + s[i - 2] + s[i + 2] + s[i + V2]) +
                   gg4 * (s[i - V2 - 1] + s[i - V2 + 1] + s[i - TS - 2] + s[i - TS + 2] + s[i + TS - 2] +
                          s[i + TS + 2] + s[i + V2 - 1] + s[i + V2 + 1]) +
                   gg5 * (s[i - M2] + s[i - P2] + s[i + P2] + s[i + M2]));
        uint8_t f = t > 0.0f ? 1 : 0;
        b.nyq[i >> 1] = f;
        if (f) {
            lr0 = min(lr0, rr);
            lr1 = max(lr1, rr);
            lc0 = min(lc0, cc);
            lc1 = max(lc1, cc);
        }
    });
    if (lr1 >= 0) {
        atomicMin(&sh[0], lr0);
        atomicMax(&sh[1], lr1);
        atomicMin(&sh[2], lc0);
        atomicMax(&sh[3], lc1);
    }
    __syncthreads();
    NyqBox box;
    int r0 = sh[1] >= 0 ? sh[0] : 0, r1 = sh[1] >= 0 ? sh[1] : 0, c0 = sh[2], c1 = sh[3];
    box.on = (r0 != r1 && c0 != c1);
    r1 += 1;
    c1 += 1;
    c0 -= c0 & 1;
    box.r0 = max(r0, 8);
    box.r1 = min(r1, g.rr1 - 8);
    box.c0 = max(c0, 8);
    box.c1 = min(c1, g.cc1 - 8);
    __syncthreads();
    return box;
}

// demosaic.rs:873-947: majority vote inside the box, then the area-based
// weight at voted sites.
template <class P>
__device__ void st_nyquist_area(const P& p, const Geo& g, const Bufs& b, const NyqBox& box) {
    const float epssq = 1e-10f;
    for_rb(p, g, box.r0, box.r1, box.c0, box.c1, [&](int rr, int cc) {
        int i = rr * TS + cc;
        const uint8_t* n = b.nyq;
        unsigned s = n[(i - V2) >> 1] + n[(i - M1) >> 1] + n[(i - P1) >> 1] + n[(i - 2) >> 1] + n[(i + 2) >> 1] +
                     n[(i + P1) >> 1] + n[(i + M1) >> 1] + n[(i + V2) >> 1];
        b.nyq2[i >> 1] = s > 4 ? 1 : (s < 4 ? 0 : n[i >> 1]);
    });
    __syncthreads();
    for_rb(p, g, box.r0, box.r1, box.c0, box.c1, [&](int rr, int cc) {
        int i = rr * TS + cc;
        if (!b.nyq2[i >> 1]) return;
        const float* m = b.mos;
        float sumcfa = 0.f, sumh = 0.f, sumv = 0.f, sumsqh = 0.f, sumsqv = 0.f, area = 0.f;
        for (int di = -6; di < 7; di += 2)
            for (int dj = -6; dj < 7; dj += 2) {
                int j = i + di * TS + dj;
                if (b.nyq2[j >> 1]) {
                    float v = m[j];
                    sumcfa += v;
                    sumh += m[j - 1] + m[j + 1];
                    sumv += m[j - V1] + m[j + V1];
                    sumsqh += sqr(v - m[j - 1]) + sqr(v - m[j + 1]);
                    sumsqv += sqr(v - m[j - V1]) + sqr(v - m[j + V1]);
                    area += 1.0f;
                }
            }
        sumh = sumcfa - sumh * 0.5f;
        sumv = sumcfa - sumv * 0.5f;
        area = area * 0.5f;
        float hvar = epssq + fabsf(area * sumsqh - sumh * sumh);
        float vvar = epssq + fabsf(area * sumsqv - sumv * sumv);
        b.hvwt[i >> 1] = hvar / (vvar + hvar);
    });
}

// demosaic.rs:949-958: hvwt smoothing (one warp).
template <class P>
__device__ void wave_hvwt(const P& p, const Geo& g, const Bufs& b) {
    wavefront(p, g, 3 * NF, 8, [](int, int, int, float) {});
}

// demosaic.rs:959-976: green at R/B sites from the smoothed weights.
template <class P>
__device__ void st_green_rb(const P& p, const Geo& g, const Bufs& b, Team tm) {
    for_rb_team(p, g, tm, 8, g.rr1 - 8, 8, g.cc1 - 8, [&](int rr, int cc) {
        int i = rr * TS + cc;
        float wt = b.hvwt[i >> 1];
        float d0 = wt * b.vcd[i] + (1.0f - wt) * b.hcd[i];
        b.dgrb0[i >> 1] = d0;
        float gr = b.mos[i] + d0;
        b.rg[i >> 1] = gr;
        if (b.nyq2[i >> 1]) {
            // neighbours of an R/B site are green sites: rgbgreen == mosaic there
            b.d2h[i >> 1] = sqr(gr - (b.mos[i - 1] + b.mos[i + 1]) * 0.5f);
            b.d2v[i >> 1] = sqr(gr - (b.mos[i - V1] + b.mos[i + V1]) * 0.5f);
        } else {
            b.d2h[i >> 1] = 0.0f;
            b.d2v[i >> 1] = 0.0f;
        }
    });
}

// demosaic.rs:978-998
template <class P>
__device__ void st_nyquist_green(const P& p, const Geo& g, const Bufs& b, const NyqBox& box, Team tm) {
    const float epssq = 1e-10f;
    const float q0 = 0.169917f, q1 = 0.108947f, q2 = 0.069855f, q3 = 0.0287182f;
    for_rb_team(p, g, tm, box.r0, box.r1, box.c0, box.c1, [&](int rr, int cc) {
        int i = rr * TS + cc;
        if (!b.nyq2[i >> 1]) return;
        // dgrb2_h/v are zero wherever the vote map is zero (the reference
        // writes 0 there or never writes them); masking keeps a previous
        // tile's values in the reused scratch out of the sums
        const uint8_t* n2 = b.nyq2;
        auto h = [&](int s) { return n2[s] ? b.d2h[s] : 0.0f; };
        auto v = [&](int s) { return n2[s] ? b.d2v[s] : 0.0f; };
        float gvarh = epssq + (q0 * h(i >> 1) + q1 * (h((i - M1) >> 1) + h((i - P1) >> 1) + h((i + P1) >> 1) + h((i + M1) >> 1)) +
                               q2 * (h((i - V2) >> 1) + h((i - 2) >> 1) + h((i + 2) >> 1) + h((i + V2) >> 1)) +
                               q3 * (h((i - M2) >> 1) + h((i - P2) >> 1) + h((i + P2) >> 1) + h((i + M2) >> 1)));
        float gvarv = epssq + (q0 * v(i >> 1) + q1 * (v((i - M1) >> 1) + v((i - P1) >> 1) + v((i + P1) >> 1) + v((i + M1) >> 1)) +
                               q2 * (v((i - V2) >> 1) + v((i - 2) >> 1) + v((i + 2) >> 1) + v((i + V2) >> 1)) +
                               q3 * (v((i - M2) >> 1) + v((i - P2) >> 1) + v((i + P2) >> 1) + v((i + M2) >> 1)));
        float d0 = (b.hcd[i] * gvarv + b.vcd[i] * gvarh) / (gvarv + gvarh);
        b.dgrb0[i >> 1] = d0;
        b.rg[i >> 1] = b.mos[i] + d0;
    });
}

// demosaic.rs:1000-1019, the dgrbsq1m/p half: squared diagonal differences
// at the green site of each column pair.  (The delm/delp half is a single
// absolute difference at the R/B site of the pair; st_diag_rb recomputes it.)
template <class P>
__device__ void st_diag_setup(const P& p, const Geo& g, const Bufs& b, Team tm) {
    const int n = (g.rr1 - 12) * TSH;
    for (int k = tm.t; k < n; k += tm.n) {
        int rr = 6 + (k >> 6), cc = 6 + 2 * (k & (TSH - 1));
        if (cc >= g.cc1 - 6) continue;
        int i = rr * TS + cc, h = i >> 1;
        const float* m = b.mos;
        bool rb_even = (p.cfa.at(g.top + rr, g.left + 2) & 1) == 0;
        if (rb_even) {
            b.q1p[h] = sqr(m[i + 1] - m[i + 1 - P1]) + sqr(m[i + 1] - m[i + 1 + P1]);
            b.q1m[h] = sqr(m[i + 1] - m[i + 1 + M1]) + sqr(m[i + 1] - m[i + 1 - M1]);
        } else {
            b.q1p[h] = sqr(m[i] - m[i - P1]) + sqr(m[i] - m[i + P1]);
            b.q1m[h] = sqr(m[i] - m[i - M1]) + sqr(m[i] - m[i + M1]);
        }
    }
}

// demosaic.rs:1021-1107, the diagonal weight pmwt (from dgrbsq1m/p).
template <class P>
__device__ void st_diag_weight(const P& p, const Geo& g, const Bufs& b, Team tm) {
    const float epssq = 1e-10f;
    const float ge0 = 0.13719494435797422f, ge1 = 0.05640252782101291f;
    for_rb_team(p, g, tm, 8, g.rr1 - 8, 8, g.cc1 - 8, [&](int rr, int cc) {
        int i = rr * TS + cc, h = i >> 1;
        const float *qm = b.q1m, *qp = b.q1p;
        float varm = epssq + ge0 * (qm[(i - V1) >> 1] + qm[(i - 1) >> 1] + qm[(i + 1) >> 1] + qm[(i + V1) >> 1]) +
                     ge1 * (qm[(i - V2 - 1) >> 1] + qm[(i - V2 + 1) >> 1] + qm[(i - 2 - V1) >> 1] + qm[(i + 2 - V1) >> 1] +
                            qm[(i - 2 + V1) >> 1] + qm[(i + 2 + V1) >> 1] + qm[(i + V2 - 1) >> 1] + qm[(i + V2 + 1) >> 1]);
        float varp = epssq + ge0 * (qp[(i - V1) >> 1] + qp[(i - 1) >> 1] + qp[(i + 1) >> 1] + qp[(i + V1) >> 1]) +
                     ge1 * (qp[(i - V2 - 1) >> 1] + qp[(i - V2 + 1) >> 1] + qp[(i - 2 - V1) >> 1] + qp[(i + 2 - V1) >> 1] +
                            qp[(i - 2 + V1) >> 1] + qp[(i + 2 + V1) >> 1] + qp[(i + V2 - 1) >> 1] + qp[(i + V2 + 1) >> 1]);
        b.pmwt[h] = varm / (varp + varm);
    });
}

// demosaic.rs:1021-1107, the diagonal R+B estimates rbm/rbp.  delm/delp of
// the R/B site j are |m[j+M1] - m[j-M1]| and |m[j-P1] - m[j+P1]| (the
// reference stores them per column pair; the sign inside fabs does not
// change the value).
template <class P>
__device__ void st_diag_rb(const P& p, const Geo& g, const Bufs& b, Team tm) {
    const float eps = 1e-5f, arth = 0.75f;
    for_rb_team(p, g, tm, 8, g.rr1 - 8, 8, g.cc1 - 8, [&](int rr, int cc) {
        int i = rr * TS + cc, h = i >> 1;
        const float* m = b.mos;
        auto dm = [&](int j) { return fabsf(m[j + M1] - m[j - M1]); };
        auto dp = [&](int j) { return fabsf(m[j - P1] - m[j + P1]); };
        float crse = (m[i + M1] * 2.0f) / (eps + m[i] + m[i + M2]);
        float crnw = (m[i - M1] * 2.0f) / (eps + m[i] + m[i - M2]);
        float crne = (m[i - P1] * 2.0f) / (eps + m[i] + m[i - P2]);
        float crsw = (m[i + P1] * 2.0f) / (eps + m[i] + m[i + P2]);
        float rbse = fabsf(1.0f - crse) < arth ? m[i] * crse : m[i + M1] + (m[i] - m[i + M2]) * 0.5f;
        float rbnw = fabsf(1.0f - crnw) < arth ? m[i] * crnw : m[i - M1] + (m[i] - m[i - M2]) * 0.5f;
        float rbne = fabsf(1.0f - crne) < arth ? m[i] * crne : m[i - P1] + (m[i] - m[i - P2]) * 0.5f;
        float rbsw = fabsf(1.0f - crsw) < arth ? m[i] * crsw : m[i + P1] + (m[i] - m[i + P2]) * 0.5f;
        const float dm0 = dm(i), dp0 = dp(i);
        float wtse = eps + dm0 + dm(i + M1) + dm(i + M2);
        float wtnw = eps + dm0 + dm(i - M1) + dm(i - M2);
        float wtne = eps + dp0 + dp(i - P1) + dp(i - P2);
        float wtsw = eps + dp0 + dp(i + P1) + dp(i + P2);
        float rbm = (wtse * rbnw + wtnw * rbse) / (wtse + wtnw);
        float rbp = (wtne * rbsw + wtsw * rbne) / (wtne + wtsw);
        if (rbp < m[i]) {
            if (rbp * 2.0f < m[i]) {
                rbp = ulim(rbp, m[i - P1], m[i + P1]);
            } else {
                float pw = (m[i] - rbp) * 2.0f / (eps + rbp + m[i]);
                rbp = pw * rbp + (1.0f - pw) * ulim(rbp, m[i - P1], m[i + P1]);
            }
        }
        if (rbm < m[i]) {
            if (rbm * 2.0f < m[i]) {
                rbm = ulim(rbm, m[i - M1], m[i + M1]);
            } else {
                float mw = (m[i] - rbm) * 2.0f / (eps + rbm + m[i]);
                rbm = mw * rbm + (1.0f - mw) * ulim(rbm, m[i - M1], m[i + M1]);
            }
        }
        if (rbp > p.clip) rbp = ulim(rbp, m[i - P1], m[i + P1]);
        if (rbm > p.clip) rbm = ulim(rbm, m[i - M1], m[i + M1]);
        b.rbp[h] = rbp;
        b.rbm[h] = rbm;
    });
}

// demosaic.rs:1109-1118: pmwt smoothing (one warp); pmwt lives at the vcd
// region of shared memory (amaze_smem + 2 NF) while it runs.
template <class P>
__device__ void wave_pmwt(const P& p, const Geo& g) {
    wavefront(p, g, 2 * NF, 10, [](int, int, int, float) {});
}

// demosaic.rs:1119-1122: rbint from the final diagonal weight.
template <class P>
__device__ void st_rbint(const P& p, const Geo& g, const Bufs& b) {
    for_rb(p, g, 10, g.rr1 - 10, 10, g.cc1 - 10, [&](int rr, int cc) {
        const int i = rr * TS + cc, h = i >> 1;
        const float pm = b.pmwt[h];
        b.rbint[h] = (b.mos[i] + b.rbm[h] * (1.0f - pm) + b.rbp[h] * pm) * 0.5f;
    });
}

// demosaic.rs:1125-1194
template <class P>
__device__ void st_green_refine(const P& p, const Geo& g, const Bufs& b) {
    const float eps = 1e-5f, arth = 0.75f;
    for_rb(p, g, 12, g.rr1 - 12, 12, g.cc1 - 12, [&](int rr, int cc) {
        int i = rr * TS + cc, h = i >> 1;
        if (!(fabsf(0.5f - b.pmwt[h]) >= fabsf(0.5f - b.hvwt[h]))) return;
        const float *m = b.mos, *rb = b.rbint, *wv = b.wv, *wh = b.wh;
        float cru = m[i - V1] * 2.0f / (eps + rb[h] + rb[h - V1]);
        float crd = m[i + V1] * 2.0f / (eps + rb[h] + rb[h + V1]);
        float crl = m[i - 1] * 2.0f / (eps + rb[h] + rb[h - 1]);
        float crr = m[i + 1] * 2.0f / (eps + rb[h] + rb[h + 1]);
        float gu = fabsf(1.0f - cru) < arth ? rb[h] * cru : m[i - V1] + (rb[h] - rb[h - V1]) * 0.5f;
        float gd = fabsf(1.0f - crd) < arth ? rb[h] * crd : m[i + V1] + (rb[h] - rb[h + V1]) * 0.5f;
        float gl = fabsf(1.0f - crl) < arth ? rb[h] * crl : m[i - 1] + (rb[h] - rb[h - 1]) * 0.5f;
        float gr = fabsf(1.0f - crr) < arth ? rb[h] * crr : m[i + 1] + (rb[h] - rb[h + 1]) * 0.5f;
        float gintv = (wv[i - V1] * gd + wv[i + V1] * gu) / fmaxf(wv[i + V1] + wv[i - V1], 1e-10f);
        float ginth = (wh[i - 1] * gr + wh[i + 1] * gl) / fmaxf(wh[i - 1] + wh[i + 1], 1e-10f);
        if (gintv < rb[h]) {
            if (2.0f * gintv < rb[h]) {
                gintv = ulim(gintv, m[i - V1], m[i + V1]);
            } else {
                float w = 2.0f * (rb[h] - gintv) / (eps + gintv + rb[h]);
                gintv = w * gintv + (1.0f - w) * ulim(gintv, m[i - V1], m[i + V1]);
            }
        }
        if (ginth < rb[h]) {
            if (2.0f * ginth < rb[h]) {
                ginth = ulim(ginth, m[i - 1], m[i + 1]);
            } else {
                float w = 2.0f * (rb[h] - ginth) / (eps + ginth + rb[h]);
                ginth = w * ginth + (1.0f - w) * ulim(ginth, m[i - 1], m[i + 1]);
            }
        }
        if (ginth > p.clip) ginth = ulim(ginth, m[i - 1], m[i + 1]);
        if (gintv > p.clip) gintv = ulim(gintv, m[i - V1], m[i + V1]);
        float gnew = ginth * (1.0f - b.hvwt[h]) + gintv * b.hvwt[h];
        b.rg[h] = gnew;
        b.dgrb0[h] = gnew - m[i];
    });
}

// demosaic.rs:1196-1252
template <class P>
__device__ void st_chroma(const P& p, const Geo& g, const Bufs& b) {
    const float eps = 1e-5f;
    int ex, ey;
    if (p.cfa.at(0, 0) == 1) {
        if (p.cfa.at(0, 1) == 0) { ex = 1; ey = 0; } else { ex = 0; ey = 1; }
    } else {
        if (p.cfa.at(0, 0) == 0) { ex = 0; ey = 0; } else { ex = 1; ey = 1; }
    }
    {
        int r0 = 13 - ey;
        int nrows = r0 < g.rr1 - 12 ? (g.rr1 - 12 - r0 + 1) / 2 : 0;
        int wmax = TSH;
        for (int k = threadIdx.x; k < nrows * wmax; k += blockDim.x) {
            int rr = r0 + 2 * (k / wmax);
            int h0 = (rr * TS + 13 - ex) >> 1, h1 = (rr * TS + g.cc1 - 12) >> 1;
            int h = h0 + k % wmax;
            if (h < h1) {
                b.dgrb1[h] = b.dgrb0[h];
                b.dgrb0[h] = 0.0f;
            }
        }
    }
    __syncthreads();
    for_rb(p, g, 14, g.rr1 - 14, 14, g.cc1 - 14, [&](int rr, int cc) {
        int i = rr * TS + cc;
        int which = 1 - (p.cfa.at(g.top + rr, g.left + cc) / 2);
        float* d = which == 0 ? b.dgrb0 : b.dgrb1;
#define D(o) d[(i + (o)) >> 1]
        float wtnw = 1.0f / (eps + fabsf(D(-M1) - D(M1)) + fabsf(D(-M1) - D(-M3)) + fabsf(D(M1) - D(-M3)));
        float wtne = 1.0f / (eps + fabsf(D(-P1) - D(P1)) + fabsf(D(-P1) - D(-P3)) + fabsf(D(P1) - D(-P3)));
        float wtsw = 1.0f / (eps + fabsf(D(P1) - D(-P1)) + fabsf(D(P1) - D(M3)) + fabsf(D(-P1) - D(P3)));
        float wtse = 1.0f / (eps + fabsf(D(M1) - D(-M1)) + fabsf(D(M1) - D(P3)) + fabsf(D(-M1) - D(M3)));
        float v = (wtnw * (1.325f * D(-M1) - 0.175f * D(-M3) - 0.075f * D(-M1 - 2) - 0.075f * D(-M1 - V2)) +
                   wtne * (1.325f * D(-P1) - 0.175f * D(-P3) - 0.075f * D(-P1 + 2) - 0.075f * D(-P1 + V2)) +
                   wtsw * (1.325f * D(P1) - 0.175f * D(P3) - 0.075f * D(P1 - 2) - 0.075f * D(-M1)) +
                   wtse * (1.325f * D(M1) - 0.175f * D(M3) - 0.075f * D(M1 + 2) - 0.075f * D(M1 + V2))) /
                  (wtnw + wtne + wtsw + wtse);
#undef D
        d[i >> 1] = v;
    });
}

// demosaic.rs:1254-1366; the epilogue receives (row, col, r, g, b).
template <class Epi, class P>
__device__ void st_output(const P& p, const Geo& g, const Bufs& b, const Epi& epi) {
    for_rect(16, g.rr1 - 16, 16, g.cc1 - 16, [&](int rr, int cc) {
        int row = rr + g.top, col = cc + g.left;
        if (!(col >= 0 && col < p.W && row >= 0 && row < p.H)) return;
        int i = rr * TS + cc;
        const float *w = b.hvwt, *d0 = b.dgrb0, *d1 = b.dgrb1;
        bool gsite = (p.cfa.at(row, col) & 1) == 1;
        float gr = gsite ? b.mos[i] : b.rg[i >> 1];
        float r, bl;
        if (gsite) {
            float tmp = 1.0f / fmaxf(w[(i - V1) >> 1] + 2.0f - w[(i + 1) >> 1] - w[(i - 1) >> 1] + w[(i + V1) >> 1], 1e-5f);
            r = clampnan(gr - ((w[(i - V1) >> 1]) * d0[(i - V1) >> 1] + (1.0f - w[(i + 1) >> 1]) * d0[(i + 1) >> 1] +
                               (1.0f - w[(i - 1) >> 1]) * d0[(i - 1) >> 1] + (w[(i + V1) >> 1]) * d0[(i + V1) >> 1]) *
                                  tmp,
                         0.0f, 1.0f);
            bl = clampnan(gr - ((w[(i - V1) >> 1]) * d1[(i - V1) >> 1] + (1.0f - w[(i + 1) >> 1]) * d1[(i + 1) >> 1] +
                                (1.0f - w[(i - 1) >> 1]) * d1[(i - 1) >> 1] + (w[(i + V1) >> 1]) * d1[(i + V1) >> 1]) *
                                   tmp,
                          0.0f, 1.0f);
        } else {
            r = clampnan(gr - d0[i >> 1], 0.0f, 1.0f);
            bl = clampnan(gr - d1[i >> 1], 0.0f, 1.0f);
        }
        epi(row, col, r, clampnan(gr, 0.0f, 1.0f), bl);
    });
}

struct EpiRGB {
    float* rgb;
    int W;
    __device__ __forceinline__ void operator()(int row, int col, float r, float g, float b) const {
        float* o = rgb + ((size_t)row * W + col) * 3;
        o[0] = r;
        o[1] = g;
        o[2] = b;
    }
};

// Colour epilogue: WB / exposure / camera CST on the demosaiced pixel before
// it is stored (the reference runs them as separate passes over the image;
// the arithmetic per pixel is the same).
struct EpiColor {
    float* rgb;
    int W;
    color::Epilogue e;
    __device__ __forceinline__ void operator()(int row, int col, float r, float g, float b) const {
        e.apply(r, g, b);
        float* o = rgb + ((size_t)row * W + col) * 3;
        o[0] = r;
        o[1] = g;
        o[2] = b;
    }
};

template <class Src, class Epi>
__global__ void __launch_bounds__(NTHREADS, 1) amaze_kernel(const __grid_constant__ Params<Src> p, const __grid_constant__ Epi epi) {
    float* smem = amaze_smem;
    __shared__ int box_sh[4];
    Bufs b;
    b.mos = smem;
    b.hcd = smem + NF;
    b.vcd = smem + 2 * NF;
    b.hvwt = smem + 3 * NF;
    float* s = reinterpret_cast<float*>(p.scratch + (size_t)blockIdx.x * SLOT_BYTES);
    b.wv = s; s += NF;
    b.wh = s; s += NF;
    b.gsq = s; s += NF;
    b.vcda = s; s += NF;
    b.hcda = s; s += NF;
    b.cdd = s; s += NF;
    b.dgv = s; s += NF;
    b.dgh = s; s += NF;
    b.dgrb0 = s; s += NH;
    b.dgrb1 = s; s += NH;
    b.delp = s; s += NH;
    b.delm = s; s += NH;
    b.rbint = s; s += NH;
    b.q1m = s; s += NH;
    b.q1p = s; s += NH;
    b.pmwt = s; s += NH;
    b.rbm = s; s += NH;
    b.rbp = s; s += NH;
    b.nyqt = s; s += NH;
    b.rg = s; s += NH;
    b.d2h = s; s += NH;
    b.d2v = s; s += NH;
    b.nyq = reinterpret_cast<uint8_t*>(s);
    b.nyq2 = b.nyq + NH;

    for (int tile = blockIdx.x; tile < p.ntiles; tile += gridDim.x) {
        Geo g = tile_geo(p.W, p.H, -16 + (tile / p.ntx) * 96, -16 + (tile % p.ntx) * 96);
        // arrays whose unwritten entries the reference reads as zero
        for (int k = threadIdx.x; k < NH; k += blockDim.x) {
            b.dgrb1[k] = 0.0f;
            b.nyq2[k] = 0;
        }
        for (int k = threadIdx.x; k < NF; k += blockDim.x) b.mos[k] = 0.0f;
        __syncthreads();
        fill(p, g, b.mos);
        __syncthreads();
        st_gradients(g, b);
        __syncthreads();
        st_colour_diff(p, g, b);
        __syncthreads();
        st_cd_refine(p, g, b);
        __syncthreads();
        st_hv_weight(p, g, b);
        __syncthreads();
        NyqBox box = st_nyquist_flags(p, g, b, box_sh);
        if (box.on) {
            st_nyquist_area(p, g, b, box);
            __syncthreads();
        }
        // hvwt smoothing: one warp walks the rows (the others wait)
        if ((threadIdx.x >> 5) == 0) wave_hvwt(p, g, b);
        __syncthreads();
        st_green_rb(p, g, b, whole_block());
        __syncthreads();
        if (box.on) st_nyquist_green(p, g, b, box, whole_block());
        __syncthreads();
        // hcd / vcd are dead from here: the diagonal stage keeps its arrays
        // in their shared memory
        Bufs d = b;
        d.q1m = b.hcd;
        d.q1p = b.hcd + NH;
        d.pmwt = b.vcd;
        d.rbint = b.vcd + NH;
        st_diag_setup(p, g, d, whole_block());
        __syncthreads();
        st_diag_weight(p, g, d, whole_block());
        __syncthreads();
        d.rbm = b.hcd;  // over dgrbsq1m/p, no longer read
        d.rbp = b.hcd + NH;
        st_diag_rb(p, g, d, whole_block());
        __syncthreads();
        if ((threadIdx.x >> 5) == 0) wave_pmwt(p, g);
        __syncthreads();
        st_rbint(p, g, d);
        __syncthreads();
        st_green_refine(p, g, d);
        __syncthreads();
        st_chroma(p, g, d);
        __syncthreads();
        st_output(p, g, d, epi);
        __syncthreads();
    }
}

// Per-(device, stream) scratch cache for the convenience entry point.
struct ScratchCache {
    std::mutex mu;
    struct Entry {
        int dev;
        cudaStream_t stream;
        void* ptr;
        size_t bytes;
    };
    std::vector<Entry> entries;
};
ScratchCache g_cache;

int get_scratch(cudaStream_t stream, size_t bytes, void** out) {
    if (fault_injected("alloc")) return fail(IMOPS_ERR_OUT_OF_MEMORY, "injected allocation failure (AMaZE scratch)");
    int dev = 0;
    IMOPS_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(g_cache.mu);
    for (auto& e : g_cache.entries) {
        if (e.dev == dev && e.stream == stream) {
            if (e.bytes >= bytes) {
                *out = e.ptr;
                return IMOPS_OK;
            }
            IMOPS_CUDA_TRY(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
            IMOPS_CUDA_TRY(cudaFree(e.ptr), "cudaFree(AMaZE scratch)");
            e.ptr = nullptr;
            e.bytes = 0;
            IMOPS_CUDA_TRY(cudaMalloc(&e.ptr, bytes), "cudaMalloc(AMaZE scratch)");
            e.bytes = bytes;
            *out = e.ptr;
            return IMOPS_OK;
        }
    }
    void* ptr = nullptr;
    IMOPS_CUDA_TRY(cudaMalloc(&ptr, bytes), "cudaMalloc(AMaZE scratch)");
    g_cache.entries.push_back({dev, stream, ptr, bytes});
    *out = ptr;
    return IMOPS_OK;
}

int tiles_of(int W, int H, int* ntx) {
    int nty = 0, nx = 0;
    for (int top = -16; top < H; top += 96) nty++;
    for (int left = -16; left < W; left += 96) nx++;
    *ntx = nx;
    return nty * nx;
}

template <class Src, class Epi>
int launch(const Src& src, int W, int H, const CfaDev& cfa, float clip, const Epi& epi, cudaStream_t stream) {
    if (W <= 0 || H <= 0) return fail(IMOPS_ERR_INVALID_ARGUMENT, "AMaZE: empty image");
    if (!cfa_is_bayer(cfa)) return fail(IMOPS_ERR_UNSUPPORTED_CFA, "AMaZE needs a 2x2 Bayer CFA");
    if (!size_supported(W, H))
        return fail(IMOPS_ERR_UNSUPPORTED_SIZE,
                    "AMaZE: for this image size the reference's 128x128 tile border fill indexes past its tile "
                    "buffer (width or height mod 96 in 1..15)");
    Params<Src> p;
    p.in = src;
    p.W = W;
    p.H = H;
    for (int i = 0; i < 4; i++) p.cfa.c[i] = cfa.col[i];
    p.clip = clip;
    p.ntiles = tiles_of(W, H, &p.ntx);
    int grid = sm_count();
    if (grid > p.ntiles) grid = p.ntiles;
    void* scratch = nullptr;
    int rc = get_scratch(stream, SLOT_BYTES * (size_t)grid, &scratch);
    if (rc) return rc;
    p.scratch = static_cast<uint8_t*>(scratch);
    if (fault_injected("launch")) return fail(IMOPS_ERR_CUDA, "injected launch failure (AMaZE)");
    IMOPS_CUDA_TRY(cudaFuncSetAttribute(amaze_kernel<Src, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)SMEM_BYTES),
                   "cudaFuncSetAttribute(AMaZE)");
    amaze_kernel<Src, Epi><<<grid, NTHREADS, SMEM_BYTES, stream>>>(p, epi);
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), "AMaZE launch");
    return IMOPS_OK;
}

int demosaic_color_f32(const float* mosaic, int W, int H, const CfaDev& cfa, float clip,
                       const color::Epilogue& e, float* rgb, cudaStream_t s) {
    if (!mosaic || !rgb) return fail(IMOPS_ERR_INVALID_ARGUMENT, "AMaZE: NULL buffer");
    return launch(SrcF32{mosaic, W}, W, H, cfa, clip, EpiColor{rgb, W, e}, s);
}

int demosaic_color_u16(const uint16_t* raw, int raw_w, int raw_h, int cx, int cy, int W, int H, const float* black,
                       const float* white, int pw, int ph, const CfaDev& cfa, float clip, const color::Epilogue& e,
                       float* rgb, cudaStream_t s) {
    if (!raw || !rgb) return fail(IMOPS_ERR_INVALID_ARGUMENT, "AMaZE: NULL buffer");
    if (pw <= 0 || ph <= 0 || pw * ph > 16) return fail(IMOPS_ERR_INVALID_ARGUMENT, "AMaZE: level period above 16 cells");
    if (cx < 0 || cy < 0 || cx + W > raw_w || cy + H > raw_h)
        return fail(IMOPS_ERR_INVALID_ARGUMENT, "AMaZE: crop rectangle outside the frame");
    SrcU16 src;
    src.raw = raw;
    src.raw_w = raw_w;
    src.cx = cx;
    src.cy = cy;
    src.pw = pw;
    src.ph = ph;
    for (int i = 0; i < pw * ph; i++) {
        src.black[i] = black[i];
        src.white[i] = white[i];
    }
    return launch(src, W, H, cfa, clip, EpiColor{rgb, W, e}, s);
}

}  // namespace amaze
}  // namespace imops

extern "C" int imops_amaze_size_supported(int w, int h) { return imops::amaze::size_supported(w, h) ? 1 : 0; }

extern "C" int imops_demosaic_amaze(const float* mosaic, int w, int h, const char* cfa, int shift_x, int shift_y,
                                    float clip_pt, float* rgb, imops_stream_t stream) {
    using namespace imops;
    clear_error();
    CfaDev c;
    int rc = parse_cfa(cfa, shift_x, shift_y, &c);
    if (rc) return rc;
    if (!rgb || !mosaic) return fail(IMOPS_ERR_INVALID_ARGUMENT, "AMaZE: NULL buffer");
    amaze::EpiRGB epi{rgb, w};
    return amaze::launch(amaze::SrcF32{mosaic, w}, w, h, c, clip_pt, epi, as_stream(stream));
}

// ---------------------------------------------------------------------------
// No-allocation variant.
//
// Some callers cannot call cudaMalloc: code recording work into a CUDA graph
// (allocation is not a stream operation), host applications whose device
// memory is owned by their own allocator or budget, and latency-critical
// paths where cudaMalloc's implicit device synchronisation is unacceptable.
// imops_demosaic_amaze_noalloc serves them: the same AMaZE kernel, with its
// per-CTA scratch slots taken from the fixed pool below instead of the
// library's cached cudaMalloc buffer.
//
// The pool holds NOALLOC_SLOTS slots of SLOT_BYTES (31,981,568 bytes in all);
// every GPU that loads this library holds it until the process exits.  A call
// runs min(tiles, NOALLOC_SLOTS) persistent CTAs, one slot each, so any image
// size the reference's tiling accepts fits in the pool (large frames are
// slower than with imops_demosaic_amaze, which uses one CTA per SM).
namespace imops {
namespace amaze {

constexpr int NOALLOC_SLOTS = 32;
constexpr size_t NOALLOC_BYTES = (size_t)NOALLOC_SLOTS * SLOT_BYTES;
static_assert(SLOT_BYTES % 256 == 0, "scratch slots must stay 256-byte aligned");

static __device__ __align__(256) uint8_t g_noalloc_scratch[NOALLOC_BYTES];

struct NoallocSetup {
    std::mutex mu;
    void* ptr[128] = {};
};
NoallocSetup g_noalloc;

// Once per device, with that device current: the device address of the pool
// (host code must not pass the symbol itself to a kernel) and the kernel's
// shared-memory opt-in.
int noalloc_pool(void** out) {
    int dev = 0;
    IMOPS_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 128) return fail(IMOPS_ERR_INVALID_ARGUMENT, "AMaZE no-alloc: device index above 127");
    std::lock_guard<std::mutex> lock(g_noalloc.mu);
    if (!g_noalloc.ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(AMaZE no-alloc pool)");
        e = cudaFuncSetAttribute(amaze_kernel<SrcF32, EpiRGB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SMEM_BYTES);
        if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(AMaZE no-alloc)");
        g_noalloc.ptr[dev] = p;
    }
    *out = g_noalloc.ptr[dev];
    return IMOPS_OK;
}

}  // namespace amaze
}  // namespace imops

extern "C" int imops_demosaic_amaze_noalloc(const float* mosaic, int w, int h, const char* cfa, int shift_x,
                                            int shift_y, float clip_pt, float* rgb, imops_stream_t stream) {
    using namespace imops;
    using namespace imops::amaze;
    clear_error();
    CfaDev c;
    int rc = parse_cfa(cfa, shift_x, shift_y, &c);
    if (rc) return rc;
    if (!mosaic || !rgb) return fail(IMOPS_ERR_INVALID_ARGUMENT, "AMaZE no-alloc: NULL buffer");
    if (w <= 0 || h <= 0) return fail(IMOPS_ERR_INVALID_ARGUMENT, "AMaZE no-alloc: empty image");
    if (!cfa_is_bayer(c)) return fail(IMOPS_ERR_UNSUPPORTED_CFA, "AMaZE needs a 2x2 Bayer CFA");
    if (!size_supported(w, h))
        return fail(IMOPS_ERR_UNSUPPORTED_SIZE,
                    "AMaZE: for this image size the reference's 128x128 tile border fill indexes past its tile "
                    "buffer (width or height mod 96 in 1..15)");
    Params<SrcF32> p;
    p.in = SrcF32{mosaic, w};
    p.W = w;
    p.H = h;
    for (int i = 0; i < 4; i++) p.cfa.c[i] = c.col[i];
    p.clip = clip_pt;
    p.ntiles = tiles_of(w, h, &p.ntx);
    int grid = p.ntiles < NOALLOC_SLOTS ? p.ntiles : NOALLOC_SLOTS;
    if ((size_t)grid * SLOT_BYTES > NOALLOC_BYTES)
        return fail(IMOPS_ERR_UNSUPPORTED_SIZE, "AMaZE no-alloc: request exceeds the 31,981,568-byte scratch pool");
    void* pool = nullptr;
    if ((rc = noalloc_pool(&pool))) return rc;
    p.scratch = static_cast<uint8_t*>(pool);
    // nothing in the pool has to start at zero: every tile clears the arrays
    // whose unwritten entries it reads before using them
    amaze_kernel<SrcF32, EpiRGB><<<grid, NTHREADS, SMEM_BYTES, as_stream(stream)>>>(p, EpiRGB{rgb, w});
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), "AMaZE no-alloc launch");
    return IMOPS_OK;
}
