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
// One thread per pixel in six stencil kernels over planar per-direction
// buffers in HBM (4 directions x G, R, B, Lab, difference); the stencils
// re-read their neighbours from L1/L2.  Built with --fmad=false: the same
// IEEE f32 operations in the same order as the oracle, including its cube
// root (t r^2 with r = t^(-1/3) by a division-free Newton iteration).
#include "common.cuh"

namespace imops {
namespace xtrans {

constexpr int BAND = 10;  // output band that takes the 3x3 mean
__constant__ int DY[4] = {0, 1, 1, 1};
__constant__ int DX[4] = {1, 0, 1, -1};

struct Img {
    const float* m;
    int W, H;
    CfaFixed<6, 6> cfa;
    __device__ __forceinline__ int ci(int v, int n) const { return v < 0 ? 0 : (v >= n ? n - 1 : v); }
    __device__ __forceinline__ size_t at(int r, int c) const { return (size_t)ci(r, H) * W + ci(c, W); }
    __device__ __forceinline__ int col(int r, int c) const { return cfa.at(ci(r, H), ci(c, W)); }
};

// min / max / sum / count of the orthogonal green neighbours
__device__ __forceinline__ void gbounds(const Img& im, int r, int c, float& lo, float& hi, float& sum, int& n) {
    const int oy[4] = {0, 0, 1, -1}, ox[4] = {1, -1, 0, 0};
    n = 0;
    sum = lo = hi = 0.0f;
#pragma unroll
    for (int t = 0; t < 4; t++) {
        if (im.col(r + oy[t], c + ox[t]) != 1) continue;
        const float v = im.m[im.at(r + oy[t], c + ox[t])];
        if (n == 0) {
            lo = v;
            hi = v;
        } else {
            lo = v < lo ? v : lo;
            hi = v > hi ? v : hi;
        }
        sum = sum + v;
        n++;
    }
}

__device__ __forceinline__ float clampg(float g, float lo, float hi, int n) {
    if (n == 0) return g;
    g = g < lo ? lo : g;
    return g > hi ? hi : g;
}

__global__ void green1_kernel(const __grid_constant__ Img im, float* __restrict__ G) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= im.W || r >= im.H) return;
    const size_t n = (size_t)im.W * im.H, i = (size_t)r * im.W + c;
    if (im.col(r, c) == 1) {
        for (int d = 0; d < 4; d++) G[d * n + i] = im.m[i];
        return;
    }
    float lo, hi, sum;
    int cnt;
    gbounds(im, r, c, lo, hi, sum, cnt);
#pragma unroll
    for (int d = 0; d < 4; d++) {
        // nearest green at distance 1 or 2 on each side, both candidates read
        // (clamped, so in bounds) and chosen by selects, no divergent loop
        const int dy = DY[d], dx = DX[d];
        const bool p1 = im.col(r + dy, c + dx) == 1, p2 = im.col(r + 2 * dy, c + 2 * dx) == 1;
        const bool m1 = im.col(r - dy, c - dx) == 1, m2 = im.col(r - 2 * dy, c - 2 * dx) == 1;
        const float vp1 = im.m[im.at(r + dy, c + dx)], vp2 = im.m[im.at(r + 2 * dy, c + 2 * dx)];
        const float vm1 = im.m[im.at(r - dy, c - dx)], vm2 = im.m[im.at(r - 2 * dy, c - 2 * dx)];
        const int kp = p1 ? 1 : (p2 ? 2 : 0), km = m1 ? 1 : (m2 ? 2 : 0);
        const float a = p1 ? vp1 : (p2 ? vp2 : 0.0f), b = m1 ? vm1 : (m2 ? vm2 : 0.0f);
        float g;
        if (kp && km) g = (a * (float)km + b * (float)kp) / (float)(kp + km);
        else if (kp) g = a;
        else if (km) g = b;
        else g = cnt ? sum / (float)cnt : im.m[i];
        G[d * n + i] = clampg(g, lo, hi, cnt);
    }
}

__global__ void rb_kernel(const __grid_constant__ Img im, const float* __restrict__ G, float* __restrict__ R, float* __restrict__ B) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= im.W || r >= im.H) return;
    const size_t n = (size_t)im.W * im.H, i = (size_t)r * im.W + c;
    const int own = im.col(r, c);
    // window rows / columns (clamped), the red and blue sites as bit masks
    // and the mosaic values, all in registers
    size_t ro[3];
    int co[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        ro[a] = (size_t)im.ci(r + a - 1, im.H) * im.W;
        co[a] = im.ci(c + a - 1, im.W);
    }
    unsigned mr = 0u, mb = 0u;
    float mv[9];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const int cl = im.col(r + a - 1, c + b - 1);
            mr |= (cl == 0 ? 1u : 0u) << (a * 3 + b);
            mb |= (cl == 2 ? 1u : 0u) << (a * 3 + b);
            mv[a * 3 + b] = im.m[ro[a] + co[b]];
        }
    int nr = 0, nb = 0;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        nr += (mr >> k) & 1u;
        nb += (mb >> k) & 1u;
    }
    // every direction reads all nine G values (no divergent loads); the red
    // and blue sums take their sites in row-major order (predicated adds)
#pragma unroll
    for (int d = 0; d < 4; d++) {
        const float* Gd = G + d * n;
        float sr = 0.0f, sb = 0.0f;
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const int k = a * 3 + b;
                const float e = mv[k] - Gd[ro[a] + co[b]];
                sr = ((mr >> k) & 1u) ? sr + e : sr;
                sb = ((mb >> k) & 1u) ? sb + e : sb;
            }
        const float g = Gd[i];
        R[d * n + i] = own == 0 ? im.m[i] : (nr ? g + sr / (float)nr : g);
        B[d * n + i] = own == 2 ? im.m[i] : (nb ? g + sb / (float)nb : g);
    }
}

__global__ void refine_kernel(const __grid_constant__ Img im, const float* __restrict__ G, const float* __restrict__ R,
                              const float* __restrict__ B, float* __restrict__ G2) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= im.W || r >= im.H) return;
    const size_t n = (size_t)im.W * im.H, i = (size_t)r * im.W + c;
    const int ch = im.col(r, c);
    if (ch == 1) {
        for (int d = 0; d < 4; d++) G2[d * n + i] = im.m[i];
        return;
    }
    float lo, hi, sum;
    int cnt;
    gbounds(im, r, c, lo, hi, sum, cnt);
#pragma unroll
    for (int d = 0; d < 4; d++) {
        const float* C = (ch == 0 ? R : B) + d * n;
        const float* Gd = G + d * n;
        const size_t jp = im.at(r + DY[d], c + DX[d]), jm = im.at(r - DY[d], c - DX[d]);
        const float k = ((C[jp] - Gd[jp]) + (C[jm] - Gd[jm])) * 0.5f;
        G2[d * n + i] = clampg(im.m[i] - k, lo, hi, cnt);
    }
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

__global__ void lab_kernel(const float* __restrict__ R, const float* __restrict__ G, const float* __restrict__ B,
                           size_t n, float* __restrict__ L) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        for (int d = 0; d < 4; d++) {
            const float r = R[d * n + i], g = G[d * n + i], b = B[d * n + i];
            // linear sRGB -> XYZ (CSS Color 4) over the D65 white, folded into
            // the X and Z rows
            const float x = 0.4338873455660398f * r + 0.3762240091374988f * g + 0.18988864529646143f * b;
            const float y = 0.21263900587151027f * r + 0.715168678767756f * g + 0.07219231536073371f * b;
            const float z = 0.017750040070973232f * r + 0.10944762085523847f * g + 0.8728023390737883f * b;
            const float fx = lab_f(x), fy = lab_f(y), fz = lab_f(z);
            L[(d * 3 + 0) * n + i] = 116.0f * fy - 16.0f;
            L[(d * 3 + 1) * n + i] = 500.0f * (fx - fy);
            L[(d * 3 + 2) * n + i] = 200.0f * (fy - fz);
        }
}

__global__ void diff_kernel(const __grid_constant__ Img im, const float* __restrict__ L, float* __restrict__ D) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= im.W || r >= im.H) return;
    const size_t n = (size_t)im.W * im.H, i = (size_t)r * im.W + c;
    for (int d = 0; d < 4; d++) {
        const size_t jp = im.at(r + DY[d], c + DX[d]), jm = im.at(r - DY[d], c - DX[d]);
        float sp = 0.0f, sm = 0.0f;
        for (int k = 0; k < 3; k++) {
            const float* Lk = L + (d * 3 + k) * n;
            const float ep = Lk[i] - Lk[jp], em = Lk[i] - Lk[jm];
            sp = sp + ep * ep;
            sm = sm + em * em;
        }
        D[d * n + i] = sp + sm;
    }
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

__global__ void vote_kernel(const __grid_constant__ Img im, const float* __restrict__ R, const float* __restrict__ G,
                            const float* __restrict__ B, const float* __restrict__ D, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= im.W || r >= im.H) return;
    const size_t n = (size_t)im.W * im.H, i = (size_t)r * im.W + c;
    float* o = out + 3 * i;
    if (r < BAND || r >= im.H - BAND || c < BAND || c >= im.W - BAND) {
        float v[3];
        mean3(im, r, c, v);
        o[0] = v[0];
        o[1] = v[1];
        o[2] = v[2];
        return;
    }
    int hm[4] = {0, 0, 0, 0};
    for (int a = -1; a <= 1; a++)
        for (int b = -1; b <= 1; b++) {
            const size_t j = (size_t)(r + a) * im.W + (c + b);
            float mn = D[j];
            for (int d = 1; d < 4; d++) mn = D[d * n + j] < mn ? D[d * n + j] : mn;
            const float t = 8.0f * mn;
#pragma unroll
            for (int d = 0; d < 4; d++) hm[d] += D[d * n + j] <= t;
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
        s0 = s0 + R[d * n + i];
        s1 = s1 + G[d * n + i];
        s2 = s2 + B[d * n + i];
        cnt++;
    }
    const int own = im.cfa.at(r, c);  // the site's own colour keeps its sample
    o[0] = own == 0 ? im.m[i] : s0 / (float)cnt;
    o[1] = own == 1 ? im.m[i] : s1 / (float)cnt;
    o[2] = own == 2 ? im.m[i] : s2 / (float)cnt;
}

// per (device, stream) working planes, grown on demand
StreamCache g_ws("X-Trans planes");

int workspace(cudaStream_t s, size_t bytes, float** out) {
    void* p = nullptr;
    int rc = g_ws.get(s, bytes, &p);
    *out = static_cast<float*>(p);
    return rc;
}

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
    const size_t n = (size_t)w * h;
    float* ws = nullptr;
    if ((rc = xtrans::workspace(s, n * 32 * sizeof(float), &ws))) return rc;
    if (fault_injected("launch")) return fail(IMOPS_ERR_CUDA, "injected launch failure (markesteijn3)");
    float *G = ws, *G2 = ws + 4 * n, *R = ws + 8 * n, *B = ws + 12 * n, *L = ws + 16 * n, *D = ws + 28 * n;
    const xtrans::Img im{mosaic, w, h, CfaFixed<6, 6>::from(c)};
    const dim3 blk(32, 8), grd((w + 31) / 32, (h + 7) / 8);
    xtrans::green1_kernel<<<grd, blk, 0, s>>>(im, G);
    note_launch();
    for (int pass = 0; pass < 3; pass++) {
        if (pass > 0) {
            xtrans::refine_kernel<<<grd, blk, 0, s>>>(im, G, R, B, G2);
            note_launch();
            float* t = G;
            G = G2;
            G2 = t;
        }
        xtrans::rb_kernel<<<grd, blk, 0, s>>>(im, G, R, B);
        note_launch();
    }
    int g1 = (int)((n + 255) / 256);
    const int cap = sm_count() * 8;
    xtrans::lab_kernel<<<g1 < cap ? g1 : cap, 256, 0, s>>>(R, G, B, n, L);
    note_launch();
    xtrans::diff_kernel<<<grd, blk, 0, s>>>(im, L, D);
    note_launch();
    xtrans::vote_kernel<<<grd, blk, 0, s>>>(im, R, G, B, D, rgb);
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), "markesteijn3 launch");
    return IMOPS_OK;
}
