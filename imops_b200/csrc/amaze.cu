// amaze.cu -- AMaZE demosaic for sm_100a, bit-identical to the reference's
// demosaic_algorithms::Amaze (pichromatic/src/demosaic.rs:358-1379).
//
// Why the structure follows the reference's tile loop: the reference
// demosaics 128x128 tiles stepped by 96 from (-16,-16), restarts every tile
// from zeroed scratch, mirrors a 16-pixel border at the image edge, bounds a
// per-tile "Nyquist" region, and several stages update arrays in place while
// scanning (a site reads its left / upper neighbours' already-updated
// values).  All of that decides output bits, so one persistent CTA works one
// reference tile at a time over the same index domain.  Where the scan order
// is observable:
//   * the hcd / vcd refinement (demosaic.rs:700-786) is a chain along each
//     row and column (step 2).  Each chain position picks one of two
//     candidates from the previous position's pick, so a position is a map
//     on two states and the chain a composition of maps: a warp scan for
//     hcd, segment-wise composition for vcd.
//   * the hvwt smoothing (demosaic.rs:949-958) and pmwt smoothing
//     (demosaic.rs:1109-1118) read the row above already updated: one warp
//     walks the rows, the previous row's values in registers.
// Divisions are IEEE (-prec-div) and the file is built with --fmad=false so
// every a*b+c rounds twice, as in the reference's Rust f32 code.
//
// Memory: the reference's per-tile arrays total ~1.2 MB.  Here the H/V stage
// is fused into a column pass and a row pass that keep gradients, colour
// differences and chain states in registers, so every array a later stage
// reads fits four shared-memory regions (224 KB, see Bufs) whose contents
// change as the tile advances.  Nothing goes to global memory but the
// output.
#include "amaze.cuh"
#include "color.cuh"


namespace imops {
namespace amaze {

constexpr int TS = 128, TSH = 64, NF = TS * TS, NH = TS * TSH;
constexpr int V1 = 128, V2 = 256, V3 = 384, P1 = 127, P2 = 254, P3 = 381, M1 = 129, M2 = 258, M3 = 387;
constexpr int NTHREADS = 512;
static_assert(NTHREADS % TS == 0 && NTHREADS % TSH == 0, "row mapping of the stage loops");

constexpr size_t SMEM_BYTES = (3 * (size_t)NF + (size_t)NH) * 4 + 64;

// Shared-memory regions and what they hold over a tile (H0/H1, V0/V1: the
// halves of HCD / VCD, each a half array indexed by flat index >> 1):
//   mos  [NF]  the tile's mosaic
//   HCD  [NF]  column pass: raw candidates | row pass: H0 cddiffsq, H1
//              refined hcd at R/B sites | H0 vcd at R/B sites (after the
//              Nyquist test), replaced in place by dgrb0 | H1 final green
//   VCD  [NF]  alternative candidates, then the refined vcd | V0 dgrbsq1m,
//              V1 dgrbsq1p | V0 pmwt, V1 rbint | V0 dgrb1
//   hvwt [NH]  vvar1, then hvwt
struct Bufs {
    float *mos, *hcd, *vcd, *hvwt;
    float *cdd, *hcd_rb, *vcd_rb, *dgrb0, *dgrb1, *rg;
    float *q1m, *q1p, *pmwt, *rbint;
    unsigned long long *nyqw, *nyq2w;  // per-row bit masks of the R/B sites
};

// Nyquist flags are kept as one 64-bit mask per tile row, bit k for the R/B
// site of column pair k (a Bayer row has one R/B site per pair).
__device__ __forceinline__ bool rbflag(const unsigned long long* w, int i) {
    return (w[i >> 7] >> ((i & (TS - 1)) >> 1)) & 1ull;
}
__device__ __forceinline__ void rbflag_set(unsigned long long* w, int i) {
    atomicOr(&w[i >> 7], 1ull << ((i & (TS - 1)) >> 1));
}

struct Geo {
    int top, left, rr1, cc1, rrmin, ccmin, rrmax, ccmax;
};

struct Bayer {
    uint8_t c[4];
    __device__ __forceinline__ int at(int r, int q) const { return c[((r & 1) << 1) | (q & 1)]; }
};

// The mosaic source: the reference's f32 mosaic (a u16 sensor frame is
// scaled to one first, see demosaic_color_u16).
struct SrcF32 {
    const float* p;
    int W;
    __device__ __forceinline__ float operator()(int r, int q) const { return __ldg(p + (size_t)r * W + q); }
};

template <class Src>
struct Params {
    Src in;
    int W, H;
    Bayer cfa;
    float clip;
    int ntx, ntiles;
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
        // a whole 128 x 128 tile inside the image: every load in flight
        // before the first store
        constexpr int RPT = TS / (NTHREADS / TS);
        const int cc = (int)(threadIdx.x & (TS - 1)), r0 = (int)(threadIdx.x / TS);
        float v[RPT];
#pragma unroll
        for (int i = 0; i < RPT; i++) v[i] = p.in(top + r0 + i * (NTHREADS / TS), left + cc);
#pragma unroll
        for (int i = 0; i < RPT; i++) mos[(r0 + i * (NTHREADS / TS)) * TS + cc] = v[i];
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

// The same sites dense over the block's threads: thread t takes sites t,
// t + NTHREADS, ... in row-major order, so no lane idles at a row's end (the
// inner stages' rows are 96-112 sites of 128, or 50-56 R/B sites of 64); the
// row and column advance without a division.  Bayer rows alternate the
// parity of their R/B columns.
template <class F>
__device__ __forceinline__ void for_rect_dense(int r0, int r1, int c0, int c1, F f) {
    const int w = c1 - c0;
    if (w <= 0 || r1 <= r0) return;
    const int n = (r1 - r0) * w, dq = NTHREADS / w, dr = NTHREADS - dq * w;
    int rr = r0 + (int)threadIdx.x / w, cc = c0 + (int)threadIdx.x % w;
    for (int k = threadIdx.x; k < n; k += NTHREADS) {
        f(rr, cc);
        rr += dq;
        cc += dr;
        if (cc >= c1) {
            cc -= w;
            rr++;
        }
    }
}

template <class F, class P>
__device__ __forceinline__ void for_rb_dense(const P& p, const Geo& g, int r0, int r1, int c0, int c1, F f) {
    const int w = (c1 - c0 + 1) >> 1;  // R/B sites a row (one fewer in rows whose first is at c0 + 1, if odd)
    if (w <= 0 || r1 <= r0) return;
    const int par0 = p.cfa.at(g.top + r0, g.left + 2) & 1;
    const int n = (r1 - r0) * w, dq = NTHREADS / w, dr = NTHREADS - dq * w;
    int rr = r0 + (int)threadIdx.x / w, k = (int)threadIdx.x % w;
    for (int j = threadIdx.x; j < n; j += NTHREADS) {
        const int cc = c0 + (par0 ^ ((rr - r0) & 1)) + 2 * k;
        if (cc < c1) f(rr, cc);
        rr += dq;
        k += dr;
        if (k >= w) {
            k -= w;
            rr++;
        }
    }
}

// The R/B sites of rows [r0, r1) x cols [c0, c1) (c0 even) numbered densely
// in row-major order, for stages whose threads keep per-site values in
// registers across a barrier: site k of the enumeration is row r0 + k / w,
// R/B column k % w of it, the division a multiply-high by ceil(2^32 / w)
// (exact for k < 2^16 and w <= 64).
struct RbDense {
    int r0, c0, c1, w, n, par0;
    unsigned magic;
};

template <class P>
__device__ __forceinline__ RbDense rb_dense(const P& p, const Geo& g, int r0, int r1, int c0, int c1) {
    RbDense d;
    const int w = (c1 - c0 + 1) >> 1;
    d.r0 = r0;
    d.c0 = c0;
    d.c1 = c1;
    d.w = w > 0 ? w : 1;
    d.n = (w > 0 && r1 > r0) ? (r1 - r0) * w : 0;
    d.par0 = p.cfa.at(g.top + r0, g.left + 2) & 1;
    d.magic = 0xFFFFFFFFu / (unsigned)d.w + 1u;
    return d;
}

// Flat index of site k, or false past the end (or the one missing site of
// the rows with fewer).
__device__ __forceinline__ bool rb_dense_site(const RbDense& d, int k, int& i) {
    if (k >= d.n) return false;
    const int q = (int)__umulhi((unsigned)k, d.magic), kk = k - q * d.w;
    const int cc = d.c0 + (d.par0 ^ (q & 1)) + 2 * kk;
    if (cc >= d.c1) return false;
    i = (d.r0 + q) * TS + cc;
    return true;
}

// R/B sites of rows [8, rr1-8) per thread, for stages that keep their
// results in registers across a barrier (two-phase in-place updates).
constexpr int RB_PER_THREAD = (TS - 16) * TSH / NTHREADS + 1;

// A subset of the block's threads working one stage: thread t of n.
struct Team {
    int t, n;
};
__device__ __forceinline__ Team whole_block() { return Team{(int)threadIdx.x, NTHREADS}; }

// The kernel's dynamic shared memory, named at namespace scope so that the
// wavefronts index it directly (shared-memory loads, not generic ones).
extern __shared__ __align__(16) float amaze_smem[];

// Row wavefront of the weight smoothing (demosaic.rs:949-958 for hvwt,
// :1109-1118 for pmwt), run by ONE warp.  At R/B site (r, c) of rows
// [lo, rr1-lo) x cols [lo, cc1-lo):
//     alt = (w(r-1,c-1) + w(r-1,c+1) + w(r+1,c-1) + w(r+1,c+1)) / 4
//     if |0.5 - w(r,c)| < |0.5 - alt|: w(r,c) = alt
// where row r-1 holds already-updated values.  Site k of a row is column
// lo + par + 2k (par: the row's R/B column parity, alternating by row); lane
// L owns sites 2L and 2L+1 of every row.  The upper neighbours of site k are
// sites k-1, k (par 0) or k, k+1 (par 1) of the row above, so a lane needs
// one value of one neighbouring lane a row.  Each lane carries its two sites
// of the row above: the updated value where that row was updated, else the
// stored one (sites past the row's range, and the row before lo); site -1
// (lane 0, par 0) is read from memory.  The lower neighbours and the own
// value are the stored ones, loaded a row ahead.  Division by 4 is exact,
// so * 0.25f gives the same bits.  post(r, c, i, w_new) runs after each
// update.  The array is amaze_smem[woff ...] (R/B half array).
template <class P, class Post>
__device__ void wavefront(const P& p, const Geo& g, int woff, int lo, Post post) {
    float* const w = amaze_smem + woff;
    const int lane = threadIdx.x & 31;
    const int rhi = g.rr1 - lo, chi = g.cc1 - lo;
    // Bayer rows alternate the column parity of their R/B sites
    int par = p.cfa.at(g.top + lo, g.left + 2) & 1;
    const int n0 = (chi - lo + 1) >> 1, n1 = (chi - lo) >> 1;
    const int kA = 2 * lane, kB = 2 * lane + 1;
    // stored value of site k of row r (parity pr); columns past the tile
    // (sites that are never a neighbour) read the last column
    auto at = [&](int r, int pr, int k) { return w[(r * TS + min(lo + pr + 2 * k, TS - 1)) >> 1]; };
    // the row above lo, never updated
    float pA = at(lo - 1, par ^ 1, kA), pB = at(lo - 1, par ^ 1, kB);
    // own and lower neighbours (r+1, c-1), (r+1, c+1) of the row being updated
    auto load = [&](int r, int pr, float& oA, float& oB, float& dlA, float& drA, float& dlB, float& drB) {
        const int cA = min(lo + pr + 2 * kA, TS - 1), cB = min(lo + pr + 2 * kB, TS - 1);
        oA = w[(r * TS + cA) >> 1];
        oB = w[(r * TS + cB) >> 1];
        dlA = w[(r * TS + cA + P1) >> 1];
        drA = w[(r * TS + cA + M1) >> 1];
        dlB = w[(r * TS + cB + P1) >> 1];
        drB = w[(r * TS + cB + M1) >> 1];
    };
    float oA, oB, dlA, drA, dlB, drB;
    load(lo, par, oA, oB, dlA, drA, dlB, drB);
    for (int rr = lo; rr < rhi; rr++) {
        const int n = par ? n1 : n0, c0 = lo + par;
        float noA, noB, ndlA, ndrA, ndlB, ndrB;
        if (rr + 1 < rhi) load(rr + 1, par ^ 1, noA, noB, ndlA, ndrA, ndlB, ndrB);
        float ulA, urA, ulB, urB;
        if (par == 0) {
            // site 2L-1 above: lane L-1's second site; site -1 from memory
            float left = __shfl_up_sync(0xffffffffu, pB, 1);
            if (lane == 0) left = w[((rr - 1) * TS + lo - 1) >> 1];
            ulA = left;
            urA = pA;
            ulB = pA;
            urB = pB;
        } else {
            // site 2L+2 above: lane L+1's first site
            const float right = __shfl_down_sync(0xffffffffu, pA, 1);
            ulA = pA;
            urA = pB;
            ulB = pB;
            urB = right;
        }
        const float altA = (ulA + urA + dlA + drA) * 0.25f;
        const float altB = (ulB + urB + dlB + drB) * 0.25f;
        const float vA = fabsf(0.5f - oA) < fabsf(0.5f - altA) ? altA : oA;
        const float vB = fabsf(0.5f - oB) < fabsf(0.5f - altB) ? altB : oB;
        if (kA < n) {
            const int i = rr * TS + c0 + 2 * kA;
            w[i >> 1] = vA;
            post(rr, c0 + 2 * kA, i, vA);
        }
        if (kB < n) {
            const int i = rr * TS + c0 + 2 * kB;
            w[i >> 1] = vB;
            post(rr, c0 + 2 * kB, i, vB);
        }
        pA = kA < n ? vA : oA;
        pB = kB < n ? vB : oB;
        par ^= 1;
        oA = noA;
        oB = noB;
        dlA = ndlA;
        drA = ndrA;
        dlB = ndlB;
        drB = ndrB;
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// stages

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

// ---------------------------------------------------------------------------
// Per-site arithmetic of demosaic.rs:612-698 by direction.  n[0..4]: mosaic
// at -2..+2 along the direction, w[0..4]: that direction's gradient weight
// (dirwts) at -2..+2.

// dirwts at a site from the mosaic at -2..+2 along the direction
// (demosaic.rs:612-622): eps + |m+2 - m0| + |m0 - m-2| + |m+1 - m-1|.
__device__ __forceinline__ float grad_w(float a, float b, float c, float d, float e) {
    return 1e-5f + fabsf(e - c) + fabsf(c - a) + fabsf(d - b);
}

// The direction's blend weight (vwt / hwt) and Hamilton-Adams estimate
// (gintvha / ginthha).
__device__ __forceinline__ float dir_hha(const float* n, const float* w, float& wt) {
    wt = w[1] / fmaxf(w[3] + w[1], 1e-10f);
    const float lo = n[1] + (n[2] - n[0]) * 0.5f, hi = n[3] + (n[2] - n[4]) * 0.5f;
    return wt * hi + (1.0f - wt) * lo;
}

// Colour difference along a direction (vcd / hcd), its alternative (vcdalt /
// hcdalt), the min squared difference (dgintv / dginth) and the blend weight.
// cross_hha: the other direction's Hamilton-Adams estimate (clip test).
__device__ __forceinline__ void dir_cd(const float* n, const float* w, float cross_hha, bool gsite, float clip8,
                                       float& val, float& alt, float& dg, float& wt) {
    const float eps = 1e-5f, arth = 0.75f;
    const float m0 = n[2];
    const float cr_lo = n[1] * (w[0] + w[2]) / fmaxf(w[0] * (eps + m0) + w[2] * (eps + n[0]), 1e-10f);
    const float cr_hi = n[3] * (w[4] + w[2]) / fmaxf(w[4] * (eps + m0) + w[2] * (eps + n[4]), 1e-10f);
    const float ha_lo = n[1] + (m0 - n[0]) * 0.5f, ha_hi = n[3] + (m0 - n[4]) * 0.5f;
    const float ar_lo = fabsf(1.0f - cr_lo) < arth ? m0 * cr_lo : ha_lo;
    const float ar_hi = fabsf(1.0f - cr_hi) < arth ? m0 * cr_hi : ha_hi;
    wt = w[1] / fmaxf(w[3] + w[1], 1e-10f);
    const float hha = wt * ha_hi + (1.0f - wt) * ha_lo;
    const float est = wt * ar_hi + (1.0f - wt) * ar_lo;
    if (gsite) {
        val = m0 - est;
        alt = m0 - hha;
    } else {
        val = est - m0;
        alt = hha - m0;
    }
    float glo = ar_lo, ghi = ar_hi;
    if (m0 > clip8 || hha > clip8 || cross_hha > clip8) {
        val = alt;
        glo = ha_lo;
        ghi = ha_hi;
    }
    dg = fminf(sqr(ha_lo - ha_hi), sqr(glo - ghi));
}

// The refinement chains of demosaic.rs:700-786 as scans.  At a chain
// position the refined value is cd_bound() of either the alternative or the
// raw colour difference; which one depends on the refined value two sites
// back, itself one of that site's two candidates.  So each position is a map
// on two states {0: alternative, 1: raw}, encoded f(0) | f(1) << 1, and the
// chain is the composition of its maps: associative, hence a parallel scan.
// The first position of a chain reads the zero before the band, which makes
// its map constant.
constexpr int MAP_ID = 2;
__device__ __forceinline__ int map_at(int f, int x) { return (f >> x) & 1; }
// g after f
__device__ __forceinline__ int map_then(int f, int g) { return map_at(g, f & 1) | (map_at(g, (f >> 1) & 1) << 1); }

// 3 * sum of squares - square of sum, in the reference's operation order
__device__ __forceinline__ float var3(float a, float b, float c) {
    return 3.0f * (sqr(a) + sqr(b) + sqr(c)) - sqr(a + b + c);
}

// Transition of one position: hav (variance of the alternatives at -2,0,+2),
// the two candidates of the previous position and the raw values at 0, +2.
__device__ __forceinline__ int chain_map(float hav, float prevA, float prevB, float raw0, float raw2) {
    const int f0 = hav < var3(prevA, raw0, raw2) ? 0 : 1;
    const int f1 = hav < var3(prevB, raw0, raw2) ? 0 : 1;
    return f0 | (f1 << 1);
}

constexpr int VSEG = NTHREADS / TS;  // row segments of the column pass
constexpr int VSEGLEN = 30;          // chain rows per segment
static_assert(VSEG * VSEGLEN >= TS - 8, "column-pass segments must cover the band");

// Column pass: demosaic.rs:612-698 (vertical half), the vcd chains of
// :700-786 and the vertical half of :788-828.  Thread (column c, row segment
// sg) walks rows t = r0-2 .. r1+1 of its column once, unrolled, with the
// mosaic column, the vertical gradients and the colour differences held in
// register windows.  At step t it forms the colour difference of row t and
// the chain step of row u = t-2 (which needs rows u-2 .. u+2).  Outputs:
//   b.vcd  <- alternative candidate of each chain row, then the refined vcd
//   b.hcd  <- raw candidate of each chain row (read back before the barrier)
//   b.hvwt <- vvar1 (the dgintv variance term) at the R/B sites
// Rows 3 and rr1-4 of b.vcd are zeroed: the H/V weight reads them.
template <class P>
__device__ void st_vpass(const P& p, const Geo& g, const Bufs& b, uint8_t* segmap) {
    const float epssq = 1e-10f;
    const float clip8 = p.clip * 0.8f;
    const int c = threadIdx.x & (TS - 1), sg = threadIdx.x / TS;
    const int rhi = g.rr1 - 4;
    const bool col_cd = c >= 4 && c < g.cc1 - 4;
    const bool col_hv = c >= 6 && c < g.cc1 - 6;
    const int r0 = 4 + VSEGLEN * sg, r1 = min(r0 + VSEGLEN, rhi);
    const bool on = col_cd && r0 < r1;
    const float* m = b.mos;
    unsigned run0 = 0, run1 = 0;
    int x00 = 0, x01 = 1, x10 = 0, x11 = 1;
    if (on) {
        auto mrow = [&](int x) { return (x >= 0 && x < g.rr1) ? m[x * TS + c] : 0.0f; };
        // windows, for step t: mosaic rows t-4 .. t+4, dirwts rows t-2 .. t+2,
        // and the last four rows' colour differences and candidates
        float mw[9], wv[5];
#pragma unroll
        for (int j = 0; j < 9; j++) mw[j] = mrow(r0 - 6 + j);
#pragma unroll
        for (int j = 0; j < 5; j++) wv[j] = grad_w(mw[j], mw[j + 1], mw[j + 2], mw[j + 3], mw[j + 4]);
        float rawp[2] = {0.f, 0.f}, altp[4] = {0.f, 0.f, 0.f, 0.f}, dgp[4] = {0.f, 0.f, 0.f, 0.f};
        float vwp[2] = {0.f, 0.f}, Ap[4] = {0.f, 0.f, 0.f, 0.f}, Bp[4] = {0.f, 0.f, 0.f, 0.f};
        const int nk = r1 - r0 + 4;  // steps t = r0-2 .. r1+1
#pragma unroll 2
        for (int k = 0; k < nk; k++) {
            const int t = r0 - 2 + k;
            float raw = 0.f, alt = 0.f, dg = 0.f, vw = 0.f, A = 0.f, B = 0.f;
            if (t >= 4 && t < rhi) {
                const bool gs = (p.cfa.at(g.top + t, g.left + c) & 1) != 0;
                const float* rowp = m + t * TS + c;
                const float h[7] = {rowp[-3], rowp[-2], rowp[-1], mw[4], rowp[1], rowp[2], rowp[3]};
                const float whm = grad_w(h[0], h[1], h[2], h[3], h[4]), whp = grad_w(h[2], h[3], h[4], h[5], h[6]);
                const float nh[5] = {h[1], h[2], h[3], h[4], h[5]};
                const float wh5[5] = {0.0f, whm, 0.0f, whp, 0.0f};
                float hwt;
                const float hha = dir_hha(nh, wh5, hwt);
                const float nv[5] = {mw[2], mw[3], mw[4], mw[5], mw[6]};
                dir_cd(nv, wv, hha, gs, clip8, raw, alt, dg, vw);
                A = cd_bound(alt, mw[4], mw[3], mw[5], gs, p.clip);
                B = cd_bound(raw, mw[4], mw[3], mw[5], gs, p.clip);
            }
            const int u = t - 2;  // chain row of this step
            if (k >= 4) {
                const int ku = k - 4;
                const int f = chain_map(var3(altp[0], altp[2], alt), Ap[0], Bp[0], rawp[0], raw);
                if (u & 1) {
                    x10 = map_at(f, x10);
                    x11 = map_at(f, x11);
                    run0 |= (unsigned)x10 << ku;
                    run1 |= (unsigned)x11 << ku;
                } else {
                    x00 = map_at(f, x00);
                    x01 = map_at(f, x01);
                    run0 |= (unsigned)x00 << ku;
                    run1 |= (unsigned)x01 << ku;
                }
                const int i = u * TS + c;
                b.vcd[i] = Ap[2];
                b.hcd[i] = Bp[2];
                if (col_hv && u >= 6 && u < g.rr1 - 6 && (p.cfa.at(g.top + u, g.left + c) & 1) == 0) {
                    const float vu1 = dgp[2] + dgp[1] + dgp[0];
                    const float vd1 = dgp[2] + dgp[3] + dg;
                    b.hvwt[i >> 1] = epssq + vwp[0] * vd1 + (1.0f - vwp[0]) * vu1;
                }
            }
            // advance the windows by one row
            rawp[0] = rawp[1]; rawp[1] = raw;
            vwp[0] = vwp[1]; vwp[1] = vw;
#pragma unroll
            for (int j = 0; j < 3; j++) {
                altp[j] = altp[j + 1];
                dgp[j] = dgp[j + 1];
                Ap[j] = Ap[j + 1];
                Bp[j] = Bp[j + 1];
            }
            altp[3] = alt; dgp[3] = dg; Ap[3] = A; Bp[3] = B;
#pragma unroll
            for (int j = 0; j < 8; j++) mw[j] = mw[j + 1];
            mw[8] = mrow(t + 5);
#pragma unroll
            for (int j = 0; j < 4; j++) wv[j] = wv[j + 1];
            wv[4] = grad_w(mw[4], mw[5], mw[6], mw[7], mw[8]);
        }
    }
    segmap[(sg * TS + c) * 2] = (uint8_t)(x00 | (x01 << 1));
    segmap[(sg * TS + c) * 2 + 1] = (uint8_t)(x10 | (x11 << 1));
    __syncthreads();
    if (!col_cd) return;
    if (sg == 0) b.vcd[3 * TS + c] = 0.0f;
    if (r0 <= rhi && rhi <= r0 + VSEGLEN) b.vcd[rhi * TS + c] = 0.0f;
    if (!on) return;
    int E0 = MAP_ID, E1 = MAP_ID;
    for (int k = 0; k < sg; k++) {
        E0 = map_then(E0, segmap[(k * TS + c) * 2]);
        E1 = map_then(E1, segmap[(k * TS + c) * 2 + 1]);
    }
    const int e0 = map_at(E0, 0), e1 = map_at(E1, 0);
#pragma unroll
    for (int k = 0; k < VSEGLEN; k++) {
        const int u = r0 + k;
        if (u < r1) {
            const int i = u * TS + c;
            const int st = ((((u & 1) ? e1 : e0) ? run1 : run0) >> k) & 1;
            if (st) b.vcd[i] = b.hcd[i];
        }
    }
}

// Row pass: demosaic.rs:612-698 (horizontal half), the hcd chains of
// :700-786, the H/V weight of :788-828 and cddiffsq (:785).  One warp per
// row r of [4, rr1-4); lane L owns columns c0 = 4+4L .. c0+3 and gets the
// neighbouring columns from lanes L-1 / L+1.  Reads the refined vcd and
// vvar1 the column pass left; writes hvwt over vvar1, and at the R/B sites
// cdd to b.hcd[0 .. NH) and the refined hcd to b.hcd[NH .. 2 NH) (half
// arrays indexed by flat index >> 1).
template <class P>
__device__ void st_hpass(const P& p, const Geo& g, const Bufs& b) {
    const float epssq = 1e-10f;
    const float clip8 = p.clip * 0.8f;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int cend = g.cc1 - 4;
    const int c0 = 4 + 4 * lane;
    float* cdd = b.hcd;
    float* hcd_rb = b.hcd + NH;
    for (int rr = 4 + (int)(threadIdx.x >> 5); rr < g.rr1 - 4; rr += NTHREADS / 32) {
        // mosaic: row rr at columns c0-4 .. c0+7, rows rr-3 .. rr+3 at c0 .. c0+3
        float mr[12], mv[7][4];
        {
            const float4* q = reinterpret_cast<const float4*>(b.mos + rr * TS + c0 - 4);
            const float4 x0 = q[0], x1 = q[1], x2 = q[2];
            const float t[12] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w, x2.x, x2.y, x2.z, x2.w};
#pragma unroll
            for (int k = 0; k < 12; k++) mr[k] = t[k];
#pragma unroll
            for (int d = 0; d < 7; d++) {
                const float4 y = *reinterpret_cast<const float4*>(b.mos + (rr - 3 + d) * TS + c0);
                mv[d][0] = y.x; mv[d][1] = y.y; mv[d][2] = y.z; mv[d][3] = y.w;
            }
        }
        float wh[8];  // wh at columns c0-2 .. c0+5
#pragma unroll
        for (int k = 0; k < 8; k++) wh[k] = grad_w(mr[k], mr[k + 1], mr[k + 2], mr[k + 3], mr[k + 4]);
        float raw[4], alt[4], dg[4], hw[4], vw[4], A[4], B[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            raw[j] = alt[j] = dg[j] = hw[j] = vw[j] = A[j] = B[j] = 0.0f;
            const int c = c0 + j;
            // vertical Hamilton-Adams estimate and weight (clip test, H/V weight)
            const float nv[5] = {mv[1][j], mv[2][j], mv[3][j], mv[4][j], mv[5][j]};
            const float wv5[5] = {0.0f, grad_w(mv[0][j], mv[1][j], mv[2][j], mv[3][j], mv[4][j]), 0.0f,
                                  grad_w(mv[2][j], mv[3][j], mv[4][j], mv[5][j], mv[6][j]), 0.0f};
            const float vha = dir_hha(nv, wv5, vw[j]);
            if (c < cend) {
                const bool gs = (p.cfa.at(g.top + rr, g.left + c) & 1) != 0;
                const float nh[5] = {mr[j + 2], mr[j + 3], mr[j + 4], mr[j + 5], mr[j + 6]};
                const float wh5[5] = {wh[j], wh[j + 1], wh[j + 2], wh[j + 3], wh[j + 4]};
                dir_cd(nh, wh5, vha, gs, clip8, raw[j], alt[j], dg[j], hw[j]);
                A[j] = cd_bound(alt[j], mr[j + 4], mr[j + 3], mr[j + 5], gs, p.clip);
                B[j] = cd_bound(raw[j], mr[j + 4], mr[j + 3], mr[j + 5], gs, p.clip);
            }
        }
        // neighbours: columns c0-2, c0-1 from lane L-1 (zero before the band),
        // c0+4, c0+5 from lane L+1 (zero past it)
        float altL2 = __shfl_up_sync(FULL, alt[2], 1), altL3 = __shfl_up_sync(FULL, alt[3], 1);
        float aL2 = __shfl_up_sync(FULL, A[2], 1), aL3 = __shfl_up_sync(FULL, A[3], 1);
        float bL2 = __shfl_up_sync(FULL, B[2], 1), bL3 = __shfl_up_sync(FULL, B[3], 1);
        if (lane == 0) altL2 = altL3 = aL2 = aL3 = bL2 = bL3 = 0.0f;
        const float altR0 = __shfl_down_sync(FULL, alt[0], 1), altR1 = __shfl_down_sync(FULL, alt[1], 1);
        const float rawR0 = __shfl_down_sync(FULL, raw[0], 1), rawR1 = __shfl_down_sync(FULL, raw[1], 1);
        const float altx[8] = {altL2, altL3, alt[0], alt[1], alt[2], alt[3], altR0, altR1};  // c0-2 .. c0+5
        const float rawx[6] = {raw[0], raw[1], raw[2], raw[3], rawR0, rawR1};                 // c0 .. c0+5
        const float pa[4] = {aL2, aL3, A[0], A[1]}, pb[4] = {bL2, bL3, B[0], B[1]};
        int f[4];
#pragma unroll
        for (int j = 0; j < 4; j++)
            f[j] = c0 + j < cend ? chain_map(var3(altx[j], altx[j + 2], altx[j + 4]), pa[j], pb[j], rawx[j], rawx[j + 2])
                                 : MAP_ID;
        int G0 = map_then(f[0], f[2]), G1 = map_then(f[1], f[3]);
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int u0 = __shfl_up_sync(FULL, G0, d), u1 = __shfl_up_sync(FULL, G1, d);
            if (lane >= d) {
                G0 = map_then(u0, G0);
                G1 = map_then(u1, G1);
            }
        }
        int E0 = __shfl_up_sync(FULL, G0, 1), E1 = __shfl_up_sync(FULL, G1, 1);
        if (lane == 0) E0 = E1 = MAP_ID;
        int st[4];
        st[0] = map_at(f[0], map_at(E0, 0));
        st[1] = map_at(f[1], map_at(E1, 0));
        st[2] = map_at(f[2], st[0]);
        st[3] = map_at(f[3], st[1]);
        float hr[4];
#pragma unroll
        for (int j = 0; j < 4; j++) hr[j] = c0 + j < cend ? (st[j] ? B[j] : A[j]) : 0.0f;
        // refined hcd at c0-3 .. c0+6 and dginth at c0-2 .. c0+5
        float h1 = __shfl_up_sync(FULL, hr[1], 1), h2 = __shfl_up_sync(FULL, hr[2], 1), h3 = __shfl_up_sync(FULL, hr[3], 1);
        if (lane == 0) h1 = h2 = h3 = 0.0f;
        const float hx[10] = {h1, h2, h3, hr[0], hr[1], hr[2], hr[3], __shfl_down_sync(FULL, hr[0], 1),
                              __shfl_down_sync(FULL, hr[1], 1), __shfl_down_sync(FULL, hr[2], 1)};
        const float dx[8] = {__shfl_up_sync(FULL, dg[2], 1), __shfl_up_sync(FULL, dg[3], 1), dg[0], dg[1], dg[2], dg[3],
                             __shfl_down_sync(FULL, dg[0], 1), __shfl_down_sync(FULL, dg[1], 1)};
        const bool row_hv = rr >= 6 && rr < g.rr1 - 6;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int c = c0 + j;
            if (c >= cend || (p.cfa.at(g.top + rr, g.left + c) & 1) != 0) continue;  // R/B sites of the band
            const int i = rr * TS + c;
            cdd[i >> 1] = sqr(b.vcd[i] - hr[j]);
            hcd_rb[i >> 1] = hr[j];
            if (!row_hv || c < 6 || c >= g.cc1 - 6) continue;
            const float* h = hx + j + 3;  // h[0] = hcd at c
            const float lave = h[0] + h[-1] + h[-2] + h[-3];
            const float rave = h[0] + h[1] + h[2] + h[3];
            const float hl = sqr(h[0] - lave) + sqr(h[-1] - lave) + sqr(h[-2] - lave) + sqr(h[-3] - lave);
            const float hrr = sqr(h[0] - rave) + sqr(h[1] - rave) + sqr(h[2] - rave) + sqr(h[3] - rave);
            const float* v = b.vcd + i;
            const float uave = v[0] + v[-V1] + v[-V2] + v[-V3];
            const float dave = v[0] + v[V1] + v[V2] + v[V3];
            const float vu = sqr(v[0] - uave) + sqr(v[-V1] - uave) + sqr(v[-V2] - uave) + sqr(v[-V3] - uave);
            const float vd = sqr(v[0] - dave) + sqr(v[V1] - dave) + sqr(v[V2] - dave) + sqr(v[V3] - dave);
            const float vvar = epssq + vw[j] * vd + (1.0f - vw[j]) * vu;
            const float hvar = epssq + hw[j] * hrr + (1.0f - hw[j]) * hl;
            const float* d = dx + j + 2;  // d[0] = dginth at c
            const float hl1 = d[0] + d[-1] + d[-2];
            const float hr1 = d[0] + d[1] + d[2];
            const float vvar1 = b.hvwt[i >> 1];
            const float hvar1 = epssq + hw[j] * hr1 + (1.0f - hw[j]) * hl1;
            const float varwt = hvar / fmaxf(vvar + hvar, 1e-10f);
            const float diffwt = hvar1 / fmaxf(vvar1 + hvar1, 1e-10f);
            b.hvwt[i >> 1] = ((0.5f - varwt) * (0.5f - diffwt) > 0.0f && fabsf(0.5f - diffwt) < fabsf(0.5f - varwt))
                                 ? varwt : diffwt;
        }
    }
}

struct NyqBox {
    int on, r0, r1, c0, c1;
};

// demosaic.rs:830-869: the Nyquist texture test at the R/B sites of
// [6, rr1-6) x [6, cc1-6), the flags and their bounding box (first / last
// flagged row, min / max flagged column).  Thread (column c, segment sg)
// walks the R/B rows of its column with the squared gradients delhvsqsum
// (demosaic.rs:612-622) of the 5x5 neighbourhood in a register window;
// cddiffsq comes from the row pass (b.hcd[0 .. NH)).
template <class P>
__device__ NyqBox st_nyq_test(const P& p, const Geo& g, const Bufs& b, int* sh) {
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
    if (threadIdx.x < TS) {
        b.nyqw[threadIdx.x] = 0ull;
        b.nyq2w[threadIdx.x] = 0ull;
    }
    __syncthreads();
    constexpr int PER = 15;  // R/B rows per segment: 4 x 15 >= 58
    static_assert(VSEG * PER * 2 >= TS - 12, "Nyquist segments must cover the rows");
    const int c = threadIdx.x & (TS - 1), sg = threadIdx.x / TS;
    int lr0 = 1 << 30, lr1 = -1, lc0 = TS + 1, lc1 = 0;
    const int ufirst = 6 + ((p.cfa.at(g.top + 6, g.left + c) & 1) != 0 ? 1 : 0);
    const int nrb = (g.rr1 - 6 - ufirst + 1) / 2;
    const int n0 = sg * PER, n1 = min(n0 + PER, nrb);
    if (c >= 6 && c < g.cc1 - 6 && n0 < n1) {
        const float* q = b.hcd;  // cddiffsq, half array
        auto gsq = [&](int x, int y) {
            const float* o = b.mos + x * TS + y;
            return sqr(o[1] - o[-1]) + sqr(o[TS] - o[-TS]);
        };
        float w[5][5];  // delhvsqsum at rows u-2 .. u+2, columns c-2 .. c+2
        const int ub = ufirst + 2 * n0;
#pragma unroll
        for (int x = 0; x < 5; x++)
#pragma unroll
            for (int y = 0; y < 5; y++) w[x][y] = gsq(ub - 2 + x, c - 2 + y);
#pragma unroll 1
        for (int n = 0; n < n1 - n0; n++) {
            {
                const int u = ub + 2 * n;
                if (n > 0) {
#pragma unroll
                    for (int y = 0; y < 5; y++) {
                        w[0][y] = w[2][y];
                        w[1][y] = w[3][y];
                        w[2][y] = w[4][y];
                        w[3][y] = gsq(u + 1, c - 2 + y);
                        w[4][y] = gsq(u + 2, c - 2 + y);
                    }
                }
                const int i = u * TS + c;
                auto Q = [&](int o) { return q[(i + o) >> 1]; };
                const float qs = go0 * Q(0) + go1 * (Q(-M1) + Q(-P1) + Q(P1) + Q(M1)) +
                                 go2 * (Q(-V2) + Q(-2) + Q(2) + Q(V2)) + go3 * (Q(-M2) + Q(-P2) + Q(P2) + Q(M2));
                const float gs = gg0 * w[2][2] + gg1 * (w[1][2] + w[2][3] + w[2][1] + w[3][2]) +
                                 gg2 * (w[1][1] + w[1][3] + w[3][1] + w[3][3]) +
                                 gg3 * (w[0][2] + w[2][0] + w[2][4] + w[4][2]) +
                                 gg4 * (w[0][1] + w[0][3] + w[1][0] + w[1][4] + w[3][0] + w[3][4] + w[4][1] + w[4][3]) +
                                 gg5 * (w[0][0] + w[0][4] + w[4][0] + w[4][4]);
                if (qs - gs > 0.0f) {
                    rbflag_set(b.nyqw, i);
                    lr0 = min(lr0, u);
                    lr1 = max(lr1, u);
                    lc0 = min(lc0, c);
                    lc1 = max(lc1, c);
                }
            }
        }
    }
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
        const unsigned long long* n = b.nyqw;
        unsigned s = rbflag(n, i - V2) + rbflag(n, i - M1) + rbflag(n, i - P1) + rbflag(n, i - 2) + rbflag(n, i + 2) +
                     rbflag(n, i + P1) + rbflag(n, i + M1) + rbflag(n, i + V2);
        if (s > 4 || (s == 4 && rbflag(n, i))) rbflag_set(b.nyq2w, i);
    });
    __syncthreads();
    for_rb(p, g, box.r0, box.r1, box.c0, box.c1, [&](int rr, int cc) {
        int i = rr * TS + cc;
        if (!rbflag(b.nyq2w, i)) return;
        const float* m = b.mos;
        float sumcfa = 0.f, sumh = 0.f, sumv = 0.f, sumsqh = 0.f, sumsqv = 0.f, area = 0.f;
        for (int di = -6; di < 7; di += 2)
            for (int dj = -6; dj < 7; dj += 2) {
                int j = i + di * TS + dj;
                if (rbflag(b.nyq2w, j)) {
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

// demosaic.rs:959-976: the colour difference at R/B sites from the smoothed
// weights.  rgbgreen there is mos + dgrb0 (not stored; st_green_refine
// stores the final green).  dgrb2h/v are formed where st_nyquist_green
// reads them.
template <class P>
__device__ void st_green_rb(const P& p, const Geo& g, const Bufs& b) {
    for_rb_dense(p, g, 8, g.rr1 - 8, 8, g.cc1 - 8, [&](int rr, int cc) {
        const int i = rr * TS + cc;
        // dgrb0 replaces vcd in place; the voted Nyquist sites keep vcd for
        // st_nyquist_green, which stores their dgrb0
        if (rbflag(b.nyq2w, i)) return;
        const float wt = b.hvwt[i >> 1];
        b.dgrb0[i >> 1] = wt * b.vcd_rb[i >> 1] + (1.0f - wt) * b.hcd_rb[i >> 1];
    });
}

// demosaic.rs:978-998.  dgrb2h/v of a voted site j are
// (rgbgreen_j - mean of its horizontal / vertical green neighbours)^2 with
// rgbgreen_j = mos_j + the colour difference st_green_rb forms at j, and
// zero at the other sites.  New values are computed by all sites first and stored after a
// barrier, so every site reads the pre-update dgrb0.

template <class P>
__device__ void st_nyquist_green(const P& p, const Geo& g, const Bufs& b, const NyqBox& box) {
    const float epssq = 1e-10f;
    const float q0 = 0.169917f, q1 = 0.108947f, q2 = 0.069855f, q3 = 0.0287182f;
    const float* m = b.mos;
    auto d2 = [&](int j, float& h, float& v) {
        if (!rbflag(b.nyq2w, j)) {
            h = v = 0.0f;
            return;
        }
        // j is voted: its colour difference as st_green_rb forms it (not
        // stored there for voted sites)
        const float wt = b.hvwt[j >> 1];
        const float gr = m[j] + (wt * b.vcd_rb[j >> 1] + (1.0f - wt) * b.hcd_rb[j >> 1]);
        h = sqr(gr - (m[j - 1] + m[j + 1]) * 0.5f);
        v = sqr(gr - (m[j - V1] + m[j + V1]) * 0.5f);
    };
    float nd[RB_PER_THREAD];
    const int n = (box.r1 - box.r0) * TSH;
#pragma unroll
    for (int s = 0; s < RB_PER_THREAD; s++) {
        const int k = (int)threadIdx.x + s * NTHREADS;
        nd[s] = 0.0f;
        if (k >= n) continue;
        const int rr = box.r0 + (k >> 6);
        const int cc = box.c0 + (p.cfa.at(g.top + rr, g.left + 2) & 1) + 2 * (k & (TSH - 1));
        const int i = rr * TS + cc;
        if (cc >= box.c1 || !rbflag(b.nyq2w, i)) continue;
        float h[13], v[13];
        const int off[13] = {0, -M1, -P1, P1, M1, -V2, -2, 2, V2, -M2, -P2, P2, M2};
#pragma unroll
        for (int t = 0; t < 13; t++) d2(i + off[t], h[t], v[t]);
        const float gvarh = epssq + (q0 * h[0] + q1 * (h[1] + h[2] + h[3] + h[4]) + q2 * (h[5] + h[6] + h[7] + h[8]) +
                                     q3 * (h[9] + h[10] + h[11] + h[12]));
        const float gvarv = epssq + (q0 * v[0] + q1 * (v[1] + v[2] + v[3] + v[4]) + q2 * (v[5] + v[6] + v[7] + v[8]) +
                                     q3 * (v[9] + v[10] + v[11] + v[12]));
        nd[s] = (b.hcd_rb[i >> 1] * gvarv + b.vcd_rb[i >> 1] * gvarh) / (gvarv + gvarh);
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < RB_PER_THREAD; s++) {
        const int k = (int)threadIdx.x + s * NTHREADS;
        if (k >= n) continue;
        const int rr = box.r0 + (k >> 6);
        const int cc = box.c0 + (p.cfa.at(g.top + rr, g.left + 2) & 1) + 2 * (k & (TSH - 1));
        const int i = rr * TS + cc;
        if (cc < box.c1 && rbflag(b.nyq2w, i)) b.dgrb0[i >> 1] = nd[s];
    }
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

// demosaic.rs:1021-1107, the diagonal weight pmwt (from dgrbsq1m/p), at
// the R/B sites of [8, rr1-8).  pmwt goes over dgrbsq1m, so every site is
// computed before any is stored.
template <class P>
__device__ void st_diag_weight(const P& p, const Geo& g, const Bufs& b) {
    const float epssq = 1e-10f;
    const float ge0 = 0.13719494435797422f, ge1 = 0.05640252782101291f;
    const float *qm = b.q1m, *qp = b.q1p;
    const int n = (g.rr1 - 16) * TSH;
    float pw[RB_PER_THREAD];
#pragma unroll
    for (int t = 0; t < RB_PER_THREAD; t++) {
        const int k = (int)threadIdx.x + t * NTHREADS;
        const int rr = 8 + (k >> 6);
        const int cc = 8 + (p.cfa.at(g.top + rr, g.left + 2) & 1) + 2 * (k & (TSH - 1));
        pw[t] = 0.0f;
        if (k >= n || cc >= g.cc1 - 8) continue;
        const int i = rr * TS + cc;
        float varm = epssq + ge0 * (qm[(i - V1) >> 1] + qm[(i - 1) >> 1] + qm[(i + 1) >> 1] + qm[(i + V1) >> 1]) +
                     ge1 * (qm[(i - V2 - 1) >> 1] + qm[(i - V2 + 1) >> 1] + qm[(i - 2 - V1) >> 1] + qm[(i + 2 - V1) >> 1] +
                            qm[(i - 2 + V1) >> 1] + qm[(i + 2 + V1) >> 1] + qm[(i + V2 - 1) >> 1] + qm[(i + V2 + 1) >> 1]);
        float varp = epssq + ge0 * (qp[(i - V1) >> 1] + qp[(i - 1) >> 1] + qp[(i + 1) >> 1] + qp[(i + V1) >> 1]) +
                     ge1 * (qp[(i - V2 - 1) >> 1] + qp[(i - V2 + 1) >> 1] + qp[(i - 2 - V1) >> 1] + qp[(i + 2 - V1) >> 1] +
                            qp[(i - 2 + V1) >> 1] + qp[(i + 2 + V1) >> 1] + qp[(i + V2 - 1) >> 1] + qp[(i + V2 + 1) >> 1]);
        pw[t] = varm / (varp + varm);
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < RB_PER_THREAD; t++) {
        const int k = (int)threadIdx.x + t * NTHREADS;
        const int rr = 8 + (k >> 6);
        const int cc = 8 + (p.cfa.at(g.top + rr, g.left + 2) & 1) + 2 * (k & (TSH - 1));
        if (k < n && cc < g.cc1 - 8) b.pmwt[(rr * TS + cc) >> 1] = pw[t];
    }
}

// The refined vcd of the R/B sites of [8, rr1-8), the only ones read after
// the Nyquist test, into a half array (frees the VCD region).
template <class P>
__device__ void st_compact_vcd(const P& p, const Geo& g, const Bufs& b) {
    for_rb_dense(p, g, 8, g.rr1 - 8, 8, g.cc1 - 8, [&](int rr, int cc) {
        const int i = rr * TS + cc;
        b.vcd_rb[i >> 1] = b.vcd[i];
    });
}

// demosaic.rs:1021-1107: the diagonal R+B estimates rbm / rbp at R/B site i.
// delm / delp of the R/B site j are |m[j+M1] - m[j-M1]| and |m[j-P1] - m[j+P1]|
// (the reference stores them per column pair; the sign inside fabs does not
// change the value).
__device__ __forceinline__ void diag_rb(const float* m, int i, float clip, float& rbm_out, float& rbp_out) {
    const float eps = 1e-5f, arth = 0.75f;
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
        if (rbp > clip) rbp = ulim(rbp, m[i - P1], m[i + P1]);
        if (rbm > clip) rbm = ulim(rbm, m[i - M1], m[i + M1]);
    rbm_out = rbm;
    rbp_out = rbp;
}

// rbm / rbp are read only by rbint (demosaic.rs:1119-1122), which needs the
// final pmwt.  Warps 2.. form them for the R/B sites of [10, rr1-10) while
// warps 0 and 1 run the weight wavefronts, keep them in registers, and form
// rbint once the wavefronts are done.
constexpr int RB_WORKERS = NTHREADS - 64;
constexpr int RB_SLOTS = ((TS - 20) * ((TS - 20) / 2) + RB_WORKERS - 1) / RB_WORKERS;

__device__ __forceinline__ bool rb_slot(const RbDense& d, int s, int& i) {
    return rb_dense_site(d, (int)threadIdx.x - 64 + s * RB_WORKERS, i);
}

template <class P>
__device__ void st_rb_early(const P& p, const Geo& g, const Bufs& b, float (&rbm)[RB_SLOTS], float (&rbp)[RB_SLOTS]) {
    const RbDense d = rb_dense(p, g, 10, g.rr1 - 10, 10, g.cc1 - 10);
#pragma unroll
    for (int s = 0; s < RB_SLOTS; s++) {
        int i;
        rbm[s] = rbp[s] = 0.0f;
        if (rb_slot(d, s, i)) diag_rb(b.mos, i, p.clip, rbm[s], rbp[s]);
    }
}

template <class P>
__device__ void st_rbint_late(const P& p, const Geo& g, const Bufs& b, const float (&rbm)[RB_SLOTS],
                              const float (&rbp)[RB_SLOTS]) {
    const RbDense d = rb_dense(p, g, 10, g.rr1 - 10, 10, g.cc1 - 10);
#pragma unroll
    for (int s = 0; s < RB_SLOTS; s++) {
        int i;
        if (!rb_slot(d, s, i)) continue;
        const float pm = b.pmwt[i >> 1];
        b.rbint[i >> 1] = (b.mos[i] + rbm[s] * (1.0f - pm) + rbp[s] * pm) * 0.5f;
    }
}

// demosaic.rs:1109-1118: pmwt smoothing (one warp); pmwt lives in the
// first half of the VCD region (amaze_smem + 2 NF).
template <class P>
__device__ void wave_pmwt(const P& p, const Geo& g) {
    wavefront(p, g, 2 * NF, 10, [](int, int, int, float) {});
}

// demosaic.rs:1125-1194
template <class P>
__device__ void st_green_refine(const P& p, const Geo& g, const Bufs& b) {
    const float eps = 1e-5f, arth = 0.75f;
    for_rb_dense(p, g, 12, g.rr1 - 12, 12, g.cc1 - 12, [&](int rr, int cc) {
        int i = rr * TS + cc, h = i >> 1;
        if (!(fabsf(0.5f - b.pmwt[h]) >= fabsf(0.5f - b.hvwt[h]))) {
            b.rg[h] = b.mos[i] + b.dgrb0[h];  // rgbgreen as st_green_rb / st_nyquist_green left it
            return;
        }
        const float *m = b.mos, *rb = b.rbint;
        // dirwts (demosaic.rs:612-622) of the four neighbours, from the mosaic
        const float wvu = grad_w(m[i - 3 * V1], m[i - V2], m[i - V1], m[i], m[i + V1]);
        const float wvd = grad_w(m[i - V1], m[i], m[i + V1], m[i + V2], m[i + 3 * V1]);
        const float whl = grad_w(m[i - 3], m[i - 2], m[i - 1], m[i], m[i + 1]);
        const float whr = grad_w(m[i - 1], m[i], m[i + 1], m[i + 2], m[i + 3]);
        float cru = m[i - V1] * 2.0f / (eps + rb[h] + rb[h - V1]);
        float crd = m[i + V1] * 2.0f / (eps + rb[h] + rb[h + V1]);
        float crl = m[i - 1] * 2.0f / (eps + rb[h] + rb[h - 1]);
        float crr = m[i + 1] * 2.0f / (eps + rb[h] + rb[h + 1]);
        float gu = fabsf(1.0f - cru) < arth ? rb[h] * cru : m[i - V1] + (rb[h] - rb[h - V1]) * 0.5f;
        float gd = fabsf(1.0f - crd) < arth ? rb[h] * crd : m[i + V1] + (rb[h] - rb[h + V1]) * 0.5f;
        float gl = fabsf(1.0f - crl) < arth ? rb[h] * crl : m[i - 1] + (rb[h] - rb[h - 1]) * 0.5f;
        float gr = fabsf(1.0f - crr) < arth ? rb[h] * crr : m[i + 1] + (rb[h] - rb[h + 1]) * 0.5f;
        float gintv = (wvu * gd + wvd * gu) / fmaxf(wvd + wvu, 1e-10f);
        float ginth = (whl * gr + whr * gl) / fmaxf(whl + whr, 1e-10f);
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
    for_rb_dense(p, g, 14, g.rr1 - 14, 14, g.cc1 - 14, [&](int rr, int cc) {
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
    for_rect_dense(16, g.rr1 - 16, 16, g.cc1 - 16, [&](int rr, int cc) {
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
    // chain segment maps of the column pass, later the Nyquist row masks
    __shared__ __align__(8) unsigned long long rowbits[2 * TS];
    static_assert(VSEG * TS * 2 <= sizeof(unsigned long long) * TS, "segment maps fit the first mask array");
    uint8_t* segmap = reinterpret_cast<uint8_t*>(rowbits);
    Bufs b;
    b.mos = smem;
    b.hcd = smem + NF;
    b.vcd = smem + 2 * NF;
    b.hvwt = smem + 3 * NF;
    b.nyqw = rowbits;
    b.nyq2w = rowbits + TS;
    b.cdd = b.vcd_rb = b.dgrb0 = b.hcd;
    b.hcd_rb = b.rg = b.hcd + NH;
    b.q1m = b.pmwt = b.dgrb1 = b.vcd;
    b.q1p = b.rbint = b.vcd + NH;

    for (int tile = blockIdx.x; tile < p.ntiles; tile += gridDim.x) {
        Geo g = tile_geo(p.W, p.H, -16 + (tile / p.ntx) * 96, -16 + (tile % p.ntx) * 96);
        if (!(g.rrmin == 0 && g.ccmin == 0 && g.rrmax == g.rr1 && g.ccmax == g.cc1)) {
            // edge tiles: the border fill leaves parts of the tile zero
            for (int k = threadIdx.x; k < NF; k += blockDim.x) b.mos[k] = 0.0f;
            __syncthreads();
        }
        fill(p, g, b.mos);
        __syncthreads();
        st_vpass(p, g, b, segmap);
        __syncthreads();
        st_hpass(p, g, b);
        __syncthreads();
        NyqBox box = st_nyq_test(p, g, b, box_sh);
        if (box.on) st_nyquist_area(p, g, b, box);
        st_compact_vcd(p, g, b);
        __syncthreads();
        // the diagonal weight (needs only the mosaic) before the smoothing,
        // so both weight wavefronts run at once, one warp each
        st_diag_setup(p, g, b, whole_block());
        __syncthreads();
        st_diag_weight(p, g, b);
        __syncthreads();
        {
            float rbm[RB_SLOTS], rbp[RB_SLOTS];
            const int warp = threadIdx.x >> 5;
            if (warp == 0) {
                wave_hvwt(p, g, b);
            } else if (warp == 1) {
                wave_pmwt(p, g);
            } else {
                st_rb_early(p, g, b, rbm, rbp);
            }
            __syncthreads();
            if (warp >= 2) st_rbint_late(p, g, b, rbm, rbp);
        }
        st_green_rb(p, g, b);
        __syncthreads();
        if (box.on) st_nyquist_green(p, g, b, box);
        __syncthreads();
        st_green_refine(p, g, b);
        __syncthreads();
        // dgrb1 starts at zero, as the reference's fresh array does
        for (int k = threadIdx.x; k < NH; k += blockDim.x) b.dgrb1[k] = 0.0f;
        __syncthreads();
        st_chroma(p, g, b);
        __syncthreads();
        st_output(p, g, b, epi);
        __syncthreads();
    }
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

// A u16 sensor frame: scaled once into an f32 mosaic by imops_scale_u16
// (the reference's f32 arithmetic, so the values and hence the output bits
// are those of the f32 path), then the f32 path.  Scaling inside the tile
// load instead divided every pixel 1.78 times (the tiles overlap) and was
// 0.14 ms slower at 24 MP than this extra pass over the frame.
StreamCache g_scaled("AMaZE scaled mosaic");

int demosaic_color_u16(const uint16_t* raw, int raw_w, int raw_h, int cx, int cy, int W, int H, const float* black,
                       const float* white, int pw, int ph, const CfaDev& cfa, float clip, const color::Epilogue& e,
                       float* rgb, cudaStream_t s) {
    if (!raw || !rgb) return fail(IMOPS_ERR_INVALID_ARGUMENT, "AMaZE: NULL buffer");
    if (pw <= 0 || ph <= 0 || pw * ph > 16) return fail(IMOPS_ERR_INVALID_ARGUMENT, "AMaZE: level period above 16 cells");
    if (cx < 0 || cy < 0 || W <= 0 || H <= 0 || cx + W > raw_w || cy + H > raw_h)
        return fail(IMOPS_ERR_INVALID_ARGUMENT, "AMaZE: crop rectangle outside the frame");
    void* m = nullptr;
    int rc = g_scaled.get(s, (size_t)W * H * sizeof(float), &m);
    if (rc) return rc;
    if ((rc = imops_scale_u16(raw, raw_w, raw_h, cx, cy, W, H, black, white, pw, ph, static_cast<float*>(m),
                              reinterpret_cast<imops_stream_t>(s))))
        return rc;
    return demosaic_color_f32(static_cast<const float*>(m), W, H, cfa, clip, e, rgb, s);
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
