// markesteijn.cu -- 3-pass directional X-Trans demosaic
// (imops_demosaic_markesteijn3), after Frank Markesteijn's method as
// published in dcraw 9.x.  The reference has no such algorithm (its
// "markesteijn" is the 3x3 same-colour mean, demosaic.rs:108-186); this is
// the library's own design, specified step by step in oracle/xtrans.c and
// checked against it bit for bit:
//   1. green along four directions (H, V and both diagonals) from the nearest
//      greens on each side, bounded by the orthogonal green neighbours;
//   2. red and blue from the mean colour difference of the 3x3 neighbours;
//   3. two refinement passes of the green from the colour difference along
//      the direction, each followed by step 2 again;
//   4. CIELab of every direction's RGB and its squared difference to the two
//      neighbours along the direction;
//   5. a vote over 3x3 windows: directions whose difference is within 8x of
//      the smallest count; the most homogeneous directions are averaged.
// Pixels within 10 of an edge take the reference's 3x3 mean.
//
// One block per 32 x 32 tile of interior pixels runs every step in shared
// memory (see `fused`); a second kernel fills the edge band.  Nothing is
// allocated.  Built with --fmad=false: the same IEEE f32 operations in the
// same order as the oracle, including its cube root (t r^2 with
// r = t^(-1/3) by a division-free Newton iteration).
#include "common.cuh"

namespace imops {
namespace xtrans {

constexpr int BAND = 10;  // output band that takes the 3x3 mean

struct Img {
    const float* m;
    int W, H;
    CfaFixed<6, 6> cfa;
    __device__ __forceinline__ int ci(int v, int n) const { return v < 0 ? 0 : (v >= n ? n - 1 : v); }
    __device__ __forceinline__ size_t at(int r, int c) const { return (size_t)ci(r, H) * W + ci(c, W); }
    __device__ __forceinline__ int col(int r, int c) const { return cfa.at(ci(r, H), ci(c, W)); }
};

__device__ __forceinline__ float clampg(float g, float lo, float hi, int n) {
    if (n == 0) return g;
    g = g < lo ? lo : g;
    return g > hi ? hi : g;
}

// cube root of t > 0 as t r^2, r = t^(-1/3) by Newton's method for the
// reciprocal cube root, r <- r (4 - t r^3) / 3: four steps, no division.
// First guess: the bit pattern of an IEEE float is close to a scaled,
// offset log2, so bits(t^p) ~ p bits(t) + (1 - p) bits(1.0f) (the
// exponent-field trick of Blinn, "Floating-point tricks", IEEE CG&A 17(4),
// 1997); for p = -1/3 the offset (4/3) 0x3F800000 is 0x54AAAAAA.  Its
// error repeats every three binades and lies in [0, +8.17%] for every normal
// t > 0 (so t r^3 < 4, inside Newton's convergence region); four steps then
// give the cube root to 4.6e-7 relative.  The oracle's xt_cbrt is the same
// arithmetic, checked against the exact cube root over 2^-126 .. 2^127.
__device__ __forceinline__ float cbrt_nt(float t) {
    float r = __uint_as_float(0x54AAAAAAu - __float_as_uint(t) / 3u);
#pragma unroll
    for (int it = 0; it < 4; it++) {
        const float r2 = r * r, r3 = r2 * r, q = t * r3;
        r = (r * (4.0f - q)) * (1.0f / 3.0f);
    }
    return (t * r) * r;
}

// CIELab's f, the linear part as one multiply-add of folded constants
__device__ __forceinline__ float lab_f(float t) {
    if (t > 216.0f / 24389.0f) return cbrt_nt(t);
    return 7.787037037037037f * t + 0.13793103448275862f;
}

// the reference's 3x3 same-colour mean (demosaic.rs:108-186), as
// demosaic_simple.cu computes it
__device__ void mean3(const Img& im, int r, int c, float* o) {
    const int y0 = r > 0 ? r - 1 : 0, y1 = r + 1 < im.H - 1 ? r + 1 : im.H - 1;
    const int x0 = c > 0 ? c - 1 : 0, x1 = c + 1 < im.W - 1 ? c + 1 : im.W - 1;
    const int centre = im.cfa.at(r, c);
#pragma unroll
    for (int ch = 0; ch < 3; ch++) {
        if (ch == centre) {
            o[ch] = im.m[(size_t)r * im.W + c];
            continue;
        }
        float s = 0.0f, cnt = 0.0f;
        for (int y = y0; y <= y1; y++)
            for (int x = x0; x <= x1; x++) {
                if (y == r && x == c) continue;
                if (im.cfa.at(y, x) == ch) {
                    s += im.m[(size_t)y * im.W + x];
                    cnt += 1.0f;
                }
            }
        o[ch] = cnt > 0.0f ? s / cnt : 0.0f;
    }
}

// ---- fused tiles ---------------------------------------------------------
// An interior output (at least BAND from every edge) depends on inputs within
// radius 9 only, all inside the image, so a block takes a 32 x 32 tile of
// interior outputs and runs the whole method for it in shared memory on a
// 50 x 50 frame (the tile and a halo of 9): per direction the green
// estimate on the frame less 2, red / blue on radius 6, refinement on 5, red /
// blue on 4, refinement on 3, red / blue and Lab on 2, the difference on 1,
// each stage over the cells the next one reads.  The directions run one
// after another through the same buffers; each thread keeps its two
// outputs' red, green and blue of every direction for the vote, and the four
// difference planes stay in shared memory.  Every cell is the same f32
// arithmetic, in the same order, as the staged specification.
//
// Work a cell does not need is not done: the green stages (step 1 and the
// refinements) return the sample at green cells, so the green planes hold
// the mosaic there from the start and those stages run over per-tile lists
// of the non-green cells; and the red / blue sums take each phase's list of
// red and blue window sites (at most four of each: two or three in the
// X-Trans pattern) instead of testing all nine.
namespace fused {

constexpr int T = 32;              // outputs a tile side
constexpr int S = T + 18;          // frame side (radius 9 each way)
constexpr int N = S * S;
constexpr int DS = T + 2;          // difference planes: radius 1
constexpr int THREADS = 512;
constexpr int OUT = T * T / THREADS;  // outputs a thread
__constant__ int OFF[4] = {1, S, S + 1, S - 1};  // frame step of each direction
// 1/n for the method's counts n (the specification multiplies by these
// instead of dividing), each rounded once to f32; index 0 is unused
__constant__ float RECIP[9] = {1.0f,        1.0f,        1.0f / 2.0f, 1.0f / 3.0f, 1.0f / 4.0f,
                               1.0f / 5.0f, 1.0f / 6.0f, 1.0f / 7.0f, 1.0f / 8.0f};

// Colour facts of a site, by its phase in the 6x6 period (a cell of the
// frame whose neighbourhood lies inside the image, which every cell an
// interior output depends on does):
//   bits 0-1    its colour
//   bits 2-10   red sites of its 3x3 window, row-major (bit 2 + 3(a+1) + b+1)
//   bits 11-19  blue sites of the window
//   bits 20-23  green orthogonal neighbours (0,+1) (0,-1) (+1,0) (-1,0)
//   bits 24+4d  direction d: green at +1, +2, -1, -2 steps
//
// and the red / blue window sites of each phase in row-major order (rbn):
//   bits 0-1    its colour
//   bits 2-4    number of red sites (centre excluded), bits 5-7 blue
//   bits 8+7t   frame offset + 64 of red site t (t < 4), bits 36+7t blue
// `lists` is 0 when a phase has more than four of either (a 6x6 CFA other
// than X-Trans), and the red / blue step then tests the window masks.
struct Masks {
    unsigned long long m[36];
    unsigned long long rbn[36];
    int lists;
};
constexpr int MB_R = 2, MB_B = 11, MB_GO = 20, MB_DIR = 24;

// per-tile lists of the non-green frame cells in [LO, S - LO)^2 for the
// green stages, LO = 2, 4, 6
constexpr int NL0 = (S - 4) * (S - 4), NL1 = (S - 8) * (S - 8), NL2 = (S - 12) * (S - 12);
constexpr int NLCAP = NL0 + NL1 + NL2;

// shared memory: mosaic, two green planes, red, blue, two Lab planes (the
// third is the red plane, overwritten in place), four difference planes,
// the two phase tables, the non-green lists and their lengths, and each
// frame cell's phase: 100 KB, two blocks an SM
constexpr size_t SMEM = (size_t)(7 * N + 4 * DS * DS) * sizeof(float) + 2 * 36 * 8 + NLCAP * 2 + 16 + N;
static_assert((7 * N + 4 * DS * DS) % 2 == 0, "the phase tables are 8-byte aligned");
static_assert(NLCAP % 2 == 0, "the list lengths are 4-byte aligned");

// host: the colour facts of the 36 phases of a 6x6 CFA
inline Masks build_masks(const CfaDev& c) {
    Masks M;
    const int dy[4] = {0, 1, 1, 1}, dx[4] = {1, 0, 1, -1};
    for (int py = 0; py < 6; py++)
        for (int px = 0; px < 6; px++) {
            auto col = [&](int y, int x) { return c.at(py + y, px + x); };
            unsigned long long v = (unsigned long long)col(0, 0);
            for (int a = -1; a <= 1; a++)
                for (int b = -1; b <= 1; b++) {
                    const int k = (a + 1) * 3 + (b + 1);
                    if (col(a, b) == 0) v |= 1ull << (MB_R + k);
                    if (col(a, b) == 2) v |= 1ull << (MB_B + k);
                }
            const int oy[4] = {0, 0, 1, -1}, ox[4] = {1, -1, 0, 0};
            for (int t = 0; t < 4; t++)
                if (col(oy[t], ox[t]) == 1) v |= 1ull << (MB_GO + t);
            for (int d = 0; d < 4; d++) {
                const int st[4] = {1, 2, -1, -2};
                for (int q = 0; q < 4; q++)
                    if (col(st[q] * dy[d], st[q] * dx[d]) == 1) v |= 1ull << (MB_DIR + 4 * d + q);
            }
            M.m[py * 6 + px] = v;
        }
    M.lists = 1;
    for (int py = 0; py < 6; py++)
        for (int px = 0; px < 6; px++) {
            auto col = [&](int y, int x) { return c.at(py + y, px + x); };
            unsigned long long v = (unsigned long long)col(0, 0);
            int nr = 0, nb = 0;
            for (int a = -1; a <= 1; a++)
                for (int b = -1; b <= 1; b++) {
                    if (a == 0 && b == 0) continue;
                    const unsigned long long o = (unsigned long long)(a * S + b + 64);
                    if (col(a, b) == 0 && nr++ < 4) v |= o << (8 + 7 * (nr - 1));
                    if (col(a, b) == 2 && nb++ < 4) v |= o << (36 + 7 * (nb - 1));
                }
            if (nr > 4 || nb > 4) M.lists = 0;
            v |= (unsigned long long)(nr & 7) << 2 | (unsigned long long)(nb & 7) << 5;
            M.rbn[py * 6 + px] = v;
        }
    return M;
}

struct Frame {
    float *m, *ga, *gb, *r, *b, *l1, *l2, *d;
    const uint8_t* ph;                 // phase of each frame cell
    const unsigned long long* masks;   // Masks::m, in shared memory
    const unsigned long long* rbn;     // Masks::rbn, in shared memory
};

// min / max / sum / count of the green orthogonal neighbours, branch-free in
// the neighbour order of the specification
__device__ __forceinline__ void gbounds_f(const Frame& F, int f, unsigned long long M, float& lo, float& hi, float& sum,
                                          int& n) {
    const int nb[4] = {f + 1, f - 1, f + S, f - S};
    n = 0;
    sum = lo = hi = 0.0f;
#pragma unroll
    for (int t = 0; t < 4; t++) {
        const bool ok = (M >> (MB_GO + t)) & 1ull;
        const float v = F.m[nb[t]];
        const bool first = ok && n == 0;
        lo = first ? v : (ok ? (v < lo ? v : lo) : lo);
        hi = first ? v : (ok ? (v > hi ? v : hi) : hi);
        sum = ok ? sum + v : sum;
        n += ok ? 1 : 0;
    }
}

__device__ __forceinline__ float green1_f(const Frame& F, int f, int d, int off) {
    const unsigned long long M = F.masks[F.ph[f]];
    float lo, hi, sum;
    int cnt;
    gbounds_f(F, f, M, lo, hi, sum, cnt);
    const unsigned dm = (unsigned)(M >> (MB_DIR + 4 * d)) & 15u;
    const bool p1 = dm & 1u, p2 = dm & 2u, m1 = dm & 4u, m2 = dm & 8u;
    const int kp = p1 ? 1 : (p2 ? 2 : 0), km = m1 ? 1 : (m2 ? 2 : 0);
    const float vp1 = F.m[f + off], vp2 = F.m[f + 2 * off], vm1 = F.m[f - off], vm2 = F.m[f - 2 * off];
    const float a = p1 ? vp1 : (p2 ? vp2 : 0.0f), b = m1 ? vm1 : (m2 ? vm2 : 0.0f);
    const float both = (a * (float)km + b * (float)kp) * RECIP[kp + km];
    const float mean = sum * RECIP[cnt];
    const float g = (kp && km) ? both : (kp ? a : (km ? b : (cnt ? mean : F.m[f])));
    return (M & 3ull) == 1ull ? F.m[f] : clampg(g, lo, hi, cnt);
}

// red and blue at f from the green plane G: their sums over the window's
// red / blue sites in row-major order.  LISTS: from the phase's site lists
// (each list in the same row-major order as the masks).
template <bool LISTS>
__device__ __forceinline__ void rb_f(const Frame& F, const float* G, int f, float& R, float& B) {
    if constexpr (LISTS) {
        const unsigned long long L = F.rbn[F.ph[f]];
        const int own = (int)(L & 3ull), nr = (int)((L >> 2) & 7ull), nb = (int)((L >> 5) & 7ull);
        float sr = 0.0f, sbl = 0.0f;
#pragma unroll
        for (int t = 0; t < 4; t++)
            if (t < nr) {
                const int j = f + (int)((L >> (8 + 7 * t)) & 127ull) - 64;
                sr = sr + (F.m[j] - G[j]);
            }
#pragma unroll
        for (int t = 0; t < 4; t++)
            if (t < nb) {
                const int j = f + (int)((L >> (36 + 7 * t)) & 127ull) - 64;
                sbl = sbl + (F.m[j] - G[j]);
            }
        const float g = G[f];
        R = own == 0 ? F.m[f] : (nr ? g + sr * RECIP[nr] : g);
        B = own == 2 ? F.m[f] : (nb ? g + sbl * RECIP[nb] : g);
        return;
    }
    const unsigned long long M = F.masks[F.ph[f]];
    const unsigned mr = (unsigned)(M >> MB_R) & 511u, mb = (unsigned)(M >> MB_B) & 511u;
    float sr = 0.0f, sbl = 0.0f;
#pragma unroll
    for (int a = -1; a <= 1; a++)
#pragma unroll
        for (int b = -1; b <= 1; b++) {
            const int k = (a + 1) * 3 + (b + 1), j = f + a * S + b;
            const float e = F.m[j] - G[j];
            sr = ((mr >> k) & 1u) ? sr + e : sr;
            sbl = ((mb >> k) & 1u) ? sbl + e : sbl;
        }
    const int nr = __popc(mr), nb = __popc(mb);
    const int own = (int)(M & 3ull);
    const float g = G[f];
    const float qr = sr * RECIP[nr], qb = sbl * RECIP[nb];
    R = own == 0 ? F.m[f] : (nr ? g + qr : g);
    B = own == 2 ? F.m[f] : (nb ? g + qb : g);
}

__device__ __forceinline__ float refine_f(const Frame& F, const float* G, int f, int off) {
    const unsigned long long M = F.masks[F.ph[f]];
    const int ch = (int)(M & 3ull);
    const float* C = ch == 0 ? F.r : F.b;
    const float k = ((C[f + off] - G[f + off]) + (C[f - off] - G[f - off])) * 0.5f;
    float lo, hi, sum;
    int cnt;
    gbounds_f(F, f, M, lo, hi, sum, cnt);
    return ch == 1 ? F.m[f] : clampg(F.m[f] - k, lo, hi, cnt);
}

// the cells [LO, S - LO)^2 of the frame, spread over the block
template <int LO, class Fn>
__device__ __forceinline__ void over(Fn fn) {
    constexpr int W = S - 2 * LO;
    for (int k = threadIdx.x; k < W * W; k += THREADS) fn((LO + k / W) * S + LO + k % W);
}

// the cells of a list, spread over the block
template <class Fn>
__device__ __forceinline__ void over_list(const uint16_t* list, int n, Fn fn) {
    for (int k = threadIdx.x; k < n; k += THREADS) fn((int)list[k]);
}

template <bool LISTS>
__global__ void __launch_bounds__(THREADS, 2) tile_kernel(const __grid_constant__ Img im, const __grid_constant__ Masks mk,
                                                         float* __restrict__ out) {
    extern __shared__ __align__(16) float fsm[];
    Frame F;
    F.m = fsm;
    F.ga = fsm + N;
    F.gb = fsm + 2 * N;
    F.r = fsm + 3 * N;
    F.b = fsm + 4 * N;
    F.l1 = fsm + 5 * N;
    F.l2 = fsm + 6 * N;
    F.d = fsm + 7 * N;
    unsigned long long* msk = reinterpret_cast<unsigned long long*>(fsm + 7 * N + 4 * DS * DS);
    unsigned long long* rbn = msk + 36;
    uint16_t* ngl = reinterpret_cast<uint16_t*>(rbn + 36);  // non-green lists, LO = 2, 4, 6
    int* nng = reinterpret_cast<int*>(ngl + NLCAP);         // their lengths
    uint8_t* phw = reinterpret_cast<uint8_t*>(nng + 4);
    F.masks = msk;
    F.rbn = rbn;
    F.ph = phw;
    const int oy = BAND + blockIdx.y * T, ox = BAND + blockIdx.x * T;  // first output of the tile
    if (threadIdx.x < 36) {
        msk[threadIdx.x] = mk.m[threadIdx.x];
        rbn[threadIdx.x] = mk.rbn[threadIdx.x];
    }
    // frame: image rows oy-9 .. oy+T+8 (clamped at the far edges of a partial
    // tile, whose cells there feed only outputs outside the interior); the
    // phase of each cell in the period (periodic, unclamped)
    const int py0 = (oy - 9) % 6, px0 = (ox - 9) % 6;
    for (int k = threadIdx.x; k < N; k += THREADS) {
        const int fy = k / S, fx = k % S;
        const int y = im.ci(oy - 9 + fy, im.H), x = im.ci(ox - 9 + fx, im.W);
        F.m[k] = im.m[(size_t)y * im.W + x];
        phw[k] = (uint8_t)(((py0 + fy) % 6) * 6 + (px0 + fx) % 6);
    }
    __syncthreads();
    // green cells: both green planes hold the sample, which the green
    // stages would return there
    for (int k = threadIdx.x; k < N; k += THREADS)
        if ((msk[phw[k]] & 3ull) == 1ull) F.ga[k] = F.gb[k] = F.m[k];
    // the non-green cells of the green stages' regions [LO, S - LO)^2, LO =
    // 2, 4, 6, listed row-major by all warps: each frame row's non-green
    // bits and per region its count, the rows' offsets (a warp scan per
    // region), then each row's entries.  The difference planes, not used
    // before the first direction's last stage, hold the row tables.
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned* rowbal = reinterpret_cast<unsigned*>(F.d);  // [S][2]: columns 0-31, 32-49
    int* rowcnt = reinterpret_cast<int*>(F.d) + 2 * S;    // [3][S]
    int* rowoff = rowcnt + 3 * S;                          // [3][S]
    // the columns [lo, S - lo) among 32 starting at 32 * chunk
    auto regmask = [](int lo, int chunk) -> unsigned {
        const int a = max(lo - 32 * chunk, 0), b = min(S - lo - 32 * chunk, 32);
        if (b <= a) return 0u;
        return (b >= 32 ? 0xffffffffu : ((1u << b) - 1u)) & ~((1u << a) - 1u);
    };
    for (int fy = warp; fy < S; fy += THREADS / 32) {
        const bool g0 = (msk[phw[fy * S + lane]] & 3ull) != 1ull;
        const bool g1 = 32 + lane < S && (msk[phw[fy * S + 32 + lane]] & 3ull) != 1ull;
        const unsigned b0 = __ballot_sync(0xffffffffu, g0), b1 = __ballot_sync(0xffffffffu, g1);
        if (lane == 0) {
            rowbal[2 * fy] = b0;
            rowbal[2 * fy + 1] = b1;
        }
        if (lane < 3) {
            const int lo = 2 + 2 * lane;
            rowcnt[lane * S + fy] =
                (fy >= lo && fy < S - lo) ? __popc(b0 & regmask(lo, 0)) + __popc(b1 & regmask(lo, 1)) : 0;
        }
    }
    __syncthreads();
    if (warp < 3) {
        const int* rc = rowcnt + warp * S;
        const int a = rc[lane], b = 32 + lane < S ? rc[32 + lane] : 0;
        int sa = a, sb = b;  // inclusive scans of rows 0-31 and 32-49
        for (int o = 1; o < 32; o <<= 1) {
            const int ua = __shfl_up_sync(0xffffffffu, sa, o), ub = __shfl_up_sync(0xffffffffu, sb, o);
            if (lane >= o) {
                sa += ua;
                sb += ub;
            }
        }
        const int ta = __shfl_sync(0xffffffffu, sa, 31), tb = __shfl_sync(0xffffffffu, sb, 31);
        rowoff[warp * S + lane] = sa - a;
        if (32 + lane < S) rowoff[warp * S + 32 + lane] = ta + sb - b;
        if (lane == 0) nng[warp] = ta + tb;
    }
    __syncthreads();
    for (int fy = warp; fy < S; fy += THREADS / 32) {
        const unsigned b0 = rowbal[2 * fy], b1 = rowbal[2 * fy + 1], lt = (1u << lane) - 1u;
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const int lo = 2 + 2 * q;
            if (fy < lo || fy >= S - lo) continue;
            const unsigned m0 = b0 & regmask(lo, 0), m1 = b1 & regmask(lo, 1);
            uint16_t* list = ngl + (q == 0 ? 0 : (q == 1 ? NL0 : NL0 + NL1));
            const int base = rowoff[q * S + fy];
            if ((m0 >> lane) & 1u) list[base + __popc(m0 & lt)] = (uint16_t)(fy * S + lane);
            if ((m1 >> lane) & 1u) list[base + __popc(m0) + __popc(m1 & lt)] = (uint16_t)(fy * S + 32 + lane);
        }
    }
    float keep[4][3][OUT];
    __syncthreads();
    const int n0 = nng[0], n1 = nng[1], n2 = nng[2];
    const uint16_t *l0 = ngl, *l1 = ngl + NL0, *l2 = ngl + NL0 + NL1;
#pragma unroll 1
    for (int d = 0; d < 4; d++) {
        const int off = OFF[d];
        over_list(l0, n0, [&](int f) { F.ga[f] = green1_f(F, f, d, off); });
        __syncthreads();
        over<3>([&](int f) { rb_f<LISTS>(F, F.ga, f, F.r[f], F.b[f]); });
        __syncthreads();
        over_list(l1, n1, [&](int f) { F.gb[f] = refine_f(F, F.ga, f, off); });
        __syncthreads();
        over<5>([&](int f) { rb_f<LISTS>(F, F.gb, f, F.r[f], F.b[f]); });
        __syncthreads();
        over_list(l2, n2, [&](int f) { F.ga[f] = refine_f(F, F.gb, f, off); });
        __syncthreads();
        over<7>([&](int f) { rb_f<LISTS>(F, F.ga, f, F.r[f], F.b[f]); });
        __syncthreads();
#pragma unroll
        for (int q = 0; q < OUT; q++) {
            const int o = threadIdx.x + q * THREADS, f = (o / T + 9) * S + o % T + 9;
            keep[d][0][q] = F.r[f];
            keep[d][1][q] = F.ga[f];
            keep[d][2][q] = F.b[f];
        }
        __syncthreads();
        // Lab of this direction's RGB, in place: L over red, a and b into
        // the Lab planes (the green planes keep their green cells)
        over<7>([&](int f) {
            const float r = F.r[f], g = F.ga[f], b = F.b[f];
            const float x = 0.4338873455660398f * r + 0.3762240091374988f * g + 0.18988864529646143f * b;
            const float y = 0.21263900587151027f * r + 0.715168678767756f * g + 0.07219231536073371f * b;
            const float z = 0.017750040070973232f * r + 0.10944762085523847f * g + 0.8728023390737883f * b;
            const float fx = lab_f(x), fy = lab_f(y), fz = lab_f(z);
            F.r[f] = 116.0f * fy - 16.0f;
            F.l1[f] = 500.0f * (fx - fy);
            F.l2[f] = 200.0f * (fy - fz);
        });
        __syncthreads();
        // the next direction's first stage touches none of the planes read
        // here, and its second waits at a barrier after the first
        float* Dd = F.d + d * DS * DS;
        over<8>([&](int f) {
            const float* L[3] = {F.r, F.l1, F.l2};
            float sp = 0.0f, sm = 0.0f;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const float ep = L[k][f] - L[k][f + off], em = L[k][f] - L[k][f - off];
                sp = sp + ep * ep;
                sm = sm + em * em;
            }
            Dd[(f / S - 8) * DS + (f % S - 8)] = sp + sm;
        });
    }
    __syncthreads();
    // vote over the 3x3 window of the four difference planes
#pragma unroll
    for (int q = 0; q < OUT; q++) {
        const int o = threadIdx.x + q * THREADS, ty = o / T, tx = o % T;
        const int y = oy + ty, x = ox + tx;
        if (y >= im.H - BAND || x >= im.W - BAND) continue;
        int hm[4] = {0, 0, 0, 0};
        for (int a = -1; a <= 1; a++)
            for (int b = -1; b <= 1; b++) {
                const int j = (ty + 1 + a) * DS + (tx + 1 + b);
                float mn = F.d[j];
                for (int d = 1; d < 4; d++) mn = F.d[d * DS * DS + j] < mn ? F.d[d * DS * DS + j] : mn;
                const float t = 8.0f * mn;
#pragma unroll
                for (int d = 0; d < 4; d++) hm[d] += F.d[d * DS * DS + j] <= t;
            }
        int hx = hm[0];
#pragma unroll
        for (int d = 1; d < 4; d++) hx = hm[d] > hx ? hm[d] : hx;
        const int thr = hx - hx / 8;
        int cnt = 0;
        float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
#pragma unroll
        for (int d = 0; d < 4; d++) {
            if (hm[d] < thr) continue;
            s0 = s0 + keep[d][0][q];
            s1 = s1 + keep[d][1][q];
            s2 = s2 + keep[d][2][q];
            cnt++;
        }
        const int fc = (ty + 9) * S + tx + 9;
        const int own = (int)(F.masks[F.ph[fc]] & 3ull);
        float* po = out + 3 * ((size_t)y * im.W + x);
        po[0] = own == 0 ? F.m[fc] : s0 * RECIP[cnt];
        po[1] = own == 1 ? F.m[fc] : s1 * RECIP[cnt];
        po[2] = own == 2 ? F.m[fc] : s2 * RECIP[cnt];
    }
}

// the edge band (within BAND of an edge): the reference's 3x3 mean.  Band
// pixels are indexed flat: whole rows at the top and bottom, then BAND
// columns either side of each middle row.
__global__ void band_kernel(const __grid_constant__ Img im, float* __restrict__ out, int top, int bottom, int left,
                            int right, size_t total) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
        int r, c;
        const size_t rows = (size_t)(top + bottom) * im.W;
        if (k < rows) {
            const int rr = (int)(k / im.W);
            r = rr < top ? rr : im.H - bottom + (rr - top);
            c = (int)(k % im.W);
        } else {
            const size_t q = k - rows;
            const int per = left + right;
            r = top + (int)(q / per);
            const int cc = (int)(q % per);
            c = cc < left ? cc : im.W - right + (cc - left);
        }
        float v[3];
        mean3(im, r, c, v);
        float* po = out + 3 * ((size_t)r * im.W + c);
        po[0] = v[0];
        po[1] = v[1];
        po[2] = v[2];
    }
}

}  // namespace fused

}  // namespace xtrans
}  // namespace imops

using namespace imops;

extern "C" int imops_demosaic_markesteijn3(const float* mosaic, int w, int h, const char* cfa, int shift_x,
                                           int shift_y, float* rgb, imops_stream_t stream) {
    clear_error();
    if (!mosaic || !rgb) return fail(IMOPS_ERR_INVALID_ARGUMENT, "markesteijn3: NULL buffer");
    if (w <= 0 || h <= 0) return fail(IMOPS_ERR_INVALID_ARGUMENT, "markesteijn3: empty image");
    CfaDev c;
    int rc = parse_cfa(cfa, shift_x, shift_y, &c);
    if (rc) return rc;
    if (c.pw != 6 || c.ph != 6) return fail(IMOPS_ERR_UNSUPPORTED_CFA, "markesteijn3 needs a 6x6 (X-Trans) CFA");
    cudaStream_t s = as_stream(stream);
    if (fault_injected("launch")) return fail(IMOPS_ERR_CUDA, "injected launch failure (markesteijn3)");
    const xtrans::Img im{mosaic, w, h, CfaFixed<6, 6>::from(c)};
    using xtrans::BAND;
    // interior tiles, then the band (every pixel within BAND of an edge)
    const int iw = w - 2 * BAND, ih = h - 2 * BAND;
    if (iw > 0 && ih > 0) {
        namespace F = xtrans::fused;
        const dim3 grd((iw + F::T - 1) / F::T, (ih + F::T - 1) / F::T);
        const F::Masks mk = F::build_masks(c);
        auto kern = mk.lists ? F::tile_kernel<true> : F::tile_kernel<false>;
        IMOPS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)F::SMEM),
                       "cudaFuncSetAttribute(markesteijn3)");
        kern<<<grd, F::THREADS, F::SMEM, s>>>(im, mk, rgb);
        note_launch();
    }
    const int top = h < BAND ? h : BAND, bottom = h - top < BAND ? h - top : BAND;
    const int mid = h - top - bottom;
    const int left = w < BAND ? w : BAND, right = w - left < BAND ? w - left : BAND;
    const size_t total = (size_t)(top + bottom) * w + (size_t)mid * (left + right);
    if (total) {
        size_t g = (total + 255) / 256, cap = (size_t)sm_count() * 8;
        xtrans::fused::band_kernel<<<(int)(g < cap ? g : cap), 256, 0, s>>>(im, rgb, top, bottom, left, right, total);
        note_launch();
    }
    IMOPS_CUDA_TRY(cudaGetLastError(), "markesteijn3 launch");
    return IMOPS_OK;
}
