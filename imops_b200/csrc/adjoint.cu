// adjoint.cu -- hand-written adjoints of the colour + film stages for
// parameter fitting (the reference has no gradients; this is new).
//
// Differentiable forward per pixel, from demosaiced camera RGB x (demosaic is
// upstream of every parameter, so its decisions are simply held fixed):
//   y   = 2^ev * (wb (.) x)                     WB + exposure
//   a   = C y                                   camera -> ACEScg matrix (9)
//   w   = max(0, Minv a);  e_l = sum_k w_k A[k][l]     spectral exposure
//   h   = max(0, a_R - thr);  B = G_sigma * h   halation (fixed tap radius)
//   E_l = e_l + s bleed_l B
//   D_l = Dmax_l / (1 + exp(-k_l (log10 max(E_l,1e-6) - x0_l)))
//   T(l)= 2^(-sum_l D_l eps'_l(lambda));  out_c = sum_lambda Cscan[lambda][c] T
// with the baseline preset's tables (film_host.cpp), grain off.
//
// Backward: a per-pixel kernel recomputes the forward, takes the upstream
// gradient (or 2/N (out - target) for an MSE loss), and produces the curve /
// halation-strength / sigma partials, the gradient w.r.t. B (a plane) and
// w.r.t. a (3 planes).  The halation blur is recomputed instead of stored; its
// sigma-derivative uses derivative taps, and the gradient w.r.t. h is the
// exact transpose of the mirror-reflect blur.  Parameter partials are summed
// per block in f64 and reduced by one block in a fixed order (deterministic).
#include <cmath>
#include <mutex>
#include <vector>

#include "film.cuh"

namespace imops {
namespace adj {

using film::HAL_R;
using film::NB81;

constexpr int NPAR = 24;  // wb3 C9 ev1 dmax3 k3 x03 s1 sigma1
constexpr int BLK = 256;

constexpr int NP = NB81 / 2;  // 40 bin pairs + bin 80

struct Const {
    float wb[3], C[9], ev2, ev;
    float dmax[3], k[3], x0[3], s, thr;
    float minv[9];
    float A[3][3];
    float bleed[3];
    float eps[3][NB81];
    float Cs[NB81][3];
    // Q[l][e][c] = -ln2 eps[e][l] Cs[l][c]: dL/dD_e = sum_c go_c sum_l Q[l][e][c] T_l,
    // so the backward needs only the forward's T_l, weighted before go is known
    float Q[NB81][3][3];
    // the forward's tables as pairs of bins (2l, 2l+1) for the packed f32x2
    // FMA, bin 80 alone: ne2 = -eps (the sum is -d), Cs2 per channel.  (The
    // backward keeps scalar bins: reading single lanes of a float2 parameter
    // costs the constant-bank operands, and packed 3x3 accumulators cost
    // occupancy.)
    float2 ne2[3][NP];
    float2 Cs2[3][NP];
    float ne_l[3], Cs_l[3];
};

__device__ __forceinline__ void color_fwd(const Const& c, const float* x, float y[3], float a[3]) {
    for (int i = 0; i < 3; i++) y[i] = c.ev2 * (c.wb[i] * x[i]);
    for (int i = 0; i < 3; i++) a[i] = c.C[3 * i] * y[0] + c.C[3 * i + 1] * y[1] + c.C[3 * i + 2] * y[2];
}

__global__ void prep_kernel(const float* __restrict__ x, size_t n, const __grid_constant__ Const c,
                            float* __restrict__ h) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        float y[3], a[3];
        color_fwd(c, x + 3 * p, y, a);
        h[p] = fmaxf(0.0f, a[0] - c.thr);
    }
}

// Per-pixel forward (and optionally backward).  MODE 0: write out.  MODE 1:
// backward with g_out or target; writes gB (plane) and ga (3 planes) and the
// block partials of dmax, k, x0, s, sigma and the loss.
template <int MODE>
__global__ void __launch_bounds__(BLK) pixel_kernel(const float* __restrict__ x, const float* __restrict__ B,
                                                    const float* __restrict__ Bs, const float* __restrict__ g_out,
                                                    const float* __restrict__ target, float loss_scale, size_t n,
                                                    const __grid_constant__ Const c, float* __restrict__ out,
                                                    float* __restrict__ gB, float* __restrict__ ga,
                                                    double* __restrict__ partial) {
    // partials: dmax0-2 (0..2), k0-2 (3..5), x00-2 (6..8), s (9), sigma (10), loss (11)
    float acc[12];
    for (int i = 0; i < 12; i++) acc[i] = 0.0f;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    // the next pixel's inputs are loaded while this one is scanned, so the
    // global-load latency hides behind the 81-bin loop
    float nx[3] = {0.f, 0.f, 0.f}, nb = 0.f;
    size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (p < n) {
        nx[0] = x[3 * p];
        nx[1] = x[3 * p + 1];
        nx[2] = x[3 * p + 2];
        nb = B[p];
    }
    for (; p < n; p += stride) {
        const float xp[3] = {nx[0], nx[1], nx[2]};
        const float b = nb;
        if (p + stride < n) {
            nx[0] = x[3 * (p + stride)];
            nx[1] = x[3 * (p + stride) + 1];
            nx[2] = x[3 * (p + stride) + 2];
            nb = B[p + stride];
        }
        // the backward's per-pixel inputs, loaded before the scan that hides
        // their latency
        float gin[3] = {0.f, 0.f, 0.f}, bsp = 0.f;
        if (MODE == 1) {
            const float* src = g_out ? g_out : target;
            gin[0] = src[3 * p];
            gin[1] = src[3 * p + 1];
            gin[2] = src[3 * p + 2];
            bsp = Bs[p];
        }
        float y[3], a[3];
        color_fwd(c, xp, y, a);
        float w[3];
        for (int k = 0; k < 3; k++) w[k] = c.minv[3 * k] * a[0] + c.minv[3 * k + 1] * a[1] + c.minv[3 * k + 2] * a[2];
        float E[3], le[3], sg[3], D[3];
        for (int l = 0; l < 3; l++) {
            float e = fmaxf(w[0], 0.0f) * c.A[0][l] + fmaxf(w[1], 0.0f) * c.A[1][l] + fmaxf(w[2], 0.0f) * c.A[2][l];
            E[l] = e + c.s * c.bleed[l] * b;
            le[l] = log10f(fmaxf(E[l], 1e-6f));
            sg[l] = 1.0f / (1.0f + expf(-c.k[l] * (le[l] - c.x0[l])));
            D[l] = c.dmax[l] * sg[l];
        }
        float o0, o1, o2v;
        float M[3][3];
        if (MODE == 0) {
            // forward: bins in pairs on the packed f32x2 FMA
            const float2 d0 = make_float2(D[0], D[0]), d1 = make_float2(D[1], D[1]), d2 = make_float2(D[2], D[2]);
            float2 oo[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
#pragma unroll
            for (int l = 0; l < NP; l++) {
                float2 xd = __fmul2_rn(d0, c.ne2[0][l]);
                xd = __ffma2_rn(d1, c.ne2[1][l], xd);
                xd = __ffma2_rn(d2, c.ne2[2][l], xd);
                const float2 t = make_float2(film::ex2_fast(xd.x), film::ex2_fast(xd.y));
#pragma unroll
                for (int j = 0; j < 3; j++) oo[j] = __ffma2_rn(c.Cs2[j][l], t, oo[j]);
            }
            float xl = D[0] * c.ne_l[0];
            xl = fmaf(D[1], c.ne_l[1], xl);
            xl = fmaf(D[2], c.ne_l[2], xl);
            const float tl = film::ex2_fast(xl);
            o0 = fmaf(c.Cs_l[0], tl, oo[0].x + oo[0].y);
            o1 = fmaf(c.Cs_l[1], tl, oo[1].x + oo[1].y);
            o2v = fmaf(c.Cs_l[2], tl, oo[2].x + oo[2].y);
        } else {
            o0 = o1 = o2v = 0.0f;
#pragma unroll
            for (int e = 0; e < 3; e++)
#pragma unroll
                for (int j = 0; j < 3; j++) M[e][j] = 0.0f;
#pragma unroll
            for (int l = 0; l < NB81; l++) {
                float d = D[0] * c.eps[0][l];
                d = fmaf(D[1], c.eps[1][l], d);
                d = fmaf(D[2], c.eps[2][l], d);
                const float t = film::ex2_fast(-d);
                o0 = fmaf(c.Cs[l][0], t, o0);
                o1 = fmaf(c.Cs[l][1], t, o1);
                o2v = fmaf(c.Cs[l][2], t, o2v);
#pragma unroll
                for (int e = 0; e < 3; e++)
#pragma unroll
                    for (int j = 0; j < 3; j++) M[e][j] = fmaf(c.Q[l][e][j], t, M[e][j]);
            }
        }
        if (MODE == 0) {
            out[3 * p] = o0;
            out[3 * p + 1] = o1;
            out[3 * p + 2] = o2v;
            continue;
        }
        float go[3];
        if (g_out) {
            go[0] = gin[0];
            go[1] = gin[1];
            go[2] = gin[2];
        } else {
            float r0 = o0 - gin[0], r1 = o1 - gin[1], r2 = o2v - gin[2];
            acc[11] += loss_scale * (r0 * r0 + r1 * r1 + r2 * r2);
            go[0] = 2.0f * loss_scale * r0;
            go[1] = 2.0f * loss_scale * r1;
            go[2] = 2.0f * loss_scale * r2;
        }
        // scan backward: dL/dD_e = sum_c M[e][c] go_c (see Const::Q)
        const float gD0 = M[0][0] * go[0] + M[0][1] * go[1] + M[0][2] * go[2];
        const float gD1 = M[1][0] * go[0] + M[1][1] * go[1] + M[1][2] * go[2];
        const float gD2 = M[2][0] * go[0] + M[2][1] * go[1] + M[2][2] * go[2];
        float gD[3] = {gD0, gD1, gD2};
        float gE[3];
        for (int l = 0; l < 3; l++) {
            float ds = sg[l] * (1.0f - sg[l]);
            acc[l] += gD[l] * sg[l];
            acc[3 + l] += gD[l] * c.dmax[l] * ds * (le[l] - c.x0[l]);
            acc[6 + l] += -gD[l] * c.dmax[l] * ds * c.k[l];
            gE[l] = E[l] > 1e-6f ? gD[l] * c.dmax[l] * ds * c.k[l] / (E[l] * 2.302585092994046f) : 0.0f;
        }
        float gb = c.s * (c.bleed[0] * gE[0] + c.bleed[1] * gE[1] + c.bleed[2] * gE[2]);
        acc[9] += (c.bleed[0] * gE[0] + c.bleed[1] * gE[1] + c.bleed[2] * gE[2]) * b;
        acc[10] += gb * bsp;
        gB[p] = gb;
        float gw[3];
        for (int k = 0; k < 3; k++)
            gw[k] = w[k] > 0.0f ? c.A[k][0] * gE[0] + c.A[k][1] * gE[1] + c.A[k][2] * gE[2] : 0.0f;
        for (int j = 0; j < 3; j++) ga[j * n + p] = c.minv[j] * gw[0] + c.minv[3 + j] * gw[1] + c.minv[6 + j] * gw[2];
    }
    if (MODE == 0) return;
    // block reduction in f64
    __shared__ double red[12][BLK / 32];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int i = 0; i < 12; i++) {
        double v = (double)acc[i];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[i][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 12) {
        double v = 0.0;
        for (int k = 0; k < (int)(blockDim.x / 32); k++) v += red[threadIdx.x][k];
        partial[(size_t)blockIdx.x * 12 + threadIdx.x] = v;
    }
}

// Colour backward: ga (+ the halation path through h) -> C, ev, wb partials.
__global__ void __launch_bounds__(BLK) color_back_kernel(const float* __restrict__ x, const float* __restrict__ ga,
                                                         const float* __restrict__ gh, size_t n,
                                                         const __grid_constant__ Const c,
                                                         double* __restrict__ partial) {
    // wb0-2 (0..2), C00..C22 (3..11), ev (12)
    float acc[13];
    for (int i = 0; i < 13; i++) acc[i] = 0.0f;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        float y[3], a[3];
        const float* xp = x + 3 * p;
        color_fwd(c, xp, y, a);
        float g[3] = {ga[p], ga[n + p], ga[2 * n + p]};
        if (a[0] - c.thr > 0.0f) g[0] += gh[p];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) acc[3 + 3 * i + j] += g[i] * y[j];
        float gy[3];
        for (int j = 0; j < 3; j++) gy[j] = c.C[j] * g[0] + c.C[3 + j] * g[1] + c.C[6 + j] * g[2];
        acc[12] += 0.69314718055994531f * (gy[0] * y[0] + gy[1] * y[1] + gy[2] * y[2]);
        for (int j = 0; j < 3; j++) acc[j] += gy[j] * c.ev2 * xp[j];
    }
    __shared__ double red[13][BLK / 32];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int i = 0; i < 13; i++) {
        double v = (double)acc[i];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[i][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 13) {
        double v = 0.0;
        for (int k = 0; k < (int)(blockDim.x / 32); k++) v += red[threadIdx.x][k];
        partial[(size_t)blockIdx.x * 13 + threadIdx.x] = v;
    }
}

// One block: sum the partials in block order and add into grad[25]
// (24 parameters + loss), in the parameter order of ImopsFilmGradParams.
__global__ void finish_kernel(const double* __restrict__ p1, int nb1, const double* __restrict__ p2, int nb2,
                              double* __restrict__ grad) {
    int t = threadIdx.x;
    if (t < 12) {
        double v = 0.0;
        for (int b = 0; b < nb1; b++) v += p1[(size_t)b * 12 + t];
        // p1 order: dmax(0..2) k(3..5) x0(6..8) s(9) sigma(10) loss(11)
        int dst = t < 9 ? 13 + t : (t == 9 ? 22 : (t == 10 ? 23 : 24));
        grad[dst] += v;
    } else if (t >= 32 && t < 32 + 13) {
        int i = t - 32;
        double v = 0.0;
        for (int b = 0; b < nb2; b++) v += p2[(size_t)b * 13 + i];
        // p2 order: wb(0..2) C(3..11) ev(12) -> grad wb(0..2) C(3..11) ev(12)
        grad[i] += v;
    }
}

// Transpose of the mirror-reflect blur pass (blur.rs:70-89) for symmetric
// taps and a line length n > R + 1 (one reflection at most).  The blur reads
// index -j as j; its transpose sends the weight meant for -j to j.  So the
// transpose is the blur itself plus terms at the ends only: at distance
// d (1 <= d <= R) from an end, + w[R - d] * g[end]; at the end itself,
// - sum_{j=1..R} w[R - j] * g[end -+ j].  This kernel adds those terms to
// `out`, which already holds the blur of g.  along_cols: the pass runs down
// the columns (y), else along the rows (x).
__global__ void blurT_edges_kernel(const float* __restrict__ g, float* __restrict__ out, int W, int H,
                                   const float* __restrict__ taps, int R, int along_cols) {
    const int n = along_cols ? H : W;   // length of a line
    const int lines = along_cols ? W : H;
    const size_t step = along_cols ? (size_t)W : 1;   // along a line
    const size_t lstep = along_cols ? 1 : (size_t)W;  // between lines
    const size_t total = (size_t)lines * (2 * R + 2);
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int line = (int)(t % lines), r = (int)(t / lines);
        const int pos = r <= R ? r : n - 1 - (r - R - 1);
        if (r > R && pos <= R) continue;  // the first-end thread of this position adds both ends' terms
        const float* gl = g + line * lstep;
        float d = 0.0f;
        if (pos == 0) {
            float acc = 0.0f;
            for (int j = 1; j <= R; j++) acc = fmaf(taps[R - j], gl[j * step], acc);
            d -= acc;
        } else if (pos <= R) {
            d = fmaf(taps[R - pos], gl[0], d);
        }
        const int q = n - 1 - pos;
        if (q == 0) {
            float acc = 0.0f;
            for (int j = 1; j <= R; j++) acc = fmaf(taps[R - j], gl[(size_t)(n - 1 - j) * step], acc);
            d -= acc;
        } else if (q <= R) {
            d = fmaf(taps[R - q], gl[(size_t)(n - 1) * step], d);
        }
        out[line * lstep + pos * step] += d;
    }
}

// ---- host ---------------------------------------------------------------------

StreamCache g_ws("adjoint workspace");

int workspace(cudaStream_t s, size_t bytes, void** out) { return g_ws.get(s, bytes, out); }

struct Arena {
    char* base;
    size_t off;
    template <class T>
    T* take(size_t count) {
        size_t a = (off + 255) & ~(size_t)255;
        T* p = reinterpret_cast<T*>(base + a);
        off = a + count * sizeof(T);
        return p;
    }
};

// Halation taps and their sigma-derivative for the fixed radius R:
// w_i = g_i / S, g_i = exp(-x_i^2 / (2 s^2)); dw_i/ds = w_i (x_i^2 - sum_j w_j x_j^2) / s^3.
void halation_taps(float sigma, int R, float* t, float* dt) {
    double sum = 0.0, m2 = 0.0;
    std::vector<double> g(2 * R + 1);
    for (int i = 0; i <= 2 * R; i++) {
        double x = i - R;
        g[i] = std::exp(-x * x / (2.0 * sigma * sigma));
        sum += g[i];
    }
    for (int i = 0; i <= 2 * R; i++) {
        double x = i - R;
        m2 += g[i] / sum * x * x;
    }
    double s3 = (double)sigma * sigma * sigma;
    for (int i = 0; i <= 2 * R; i++) {
        double x = i - R, w = g[i] / sum;
        t[i] = (float)w;
        dt[i] = (float)(w * (x * x - m2) / s3);
    }
}

int build_const(const ImopsFilmGradParams& P, const ImopsBaselineFilm& F, Const* c, float* taps, float* dtaps) {
    film::Stock st;
    float pitch;
    ImopsBaselineFilm f2 = F;
    f2.grain_on = 0;
    int rc = film::build_stock(IMOPS_STOCK_BASELINE81, 0, 1, -1.0f, &f2, &st, &pitch);
    if (rc) return rc;
    for (int i = 0; i < 3; i++) c->wb[i] = P.wb[i];
    for (int i = 0; i < 9; i++) c->C[i] = P.matrix[i];
    c->ev = P.ev;
    c->ev2 = std::exp2(P.ev);
    for (int l = 0; l < 3; l++) {
        c->dmax[l] = P.dmax[l];
        c->k[l] = P.k[l];
        c->x0[l] = P.x0[l];
        c->bleed[l] = st.base.bleed[l];
    }
    c->s = P.hal_strength;
    c->thr = F.hal_threshold;
    for (int i = 0; i < 9; i++) c->minv[i] = st.expose.minv[i];
    for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++) c->A[k][l] = st.expose.A[k][l];
    const film::ScanSpec81& S = st.scan81;
    auto q = [&](int e, int j, int i) {
        return (float)(-0.69314718055994531 * (double)S.eps[e][i] * (double)S.C[i][j]);
    };
    for (int e = 0; e < 3; e++)
        for (int i = 0; i < NB81; i++) c->eps[e][i] = S.eps[e][i];
    for (int i = 0; i < NB81; i++)
        for (int e = 0; e < 3; e++) {
            c->Cs[i][e] = S.C[i][e];
            for (int j = 0; j < 3; j++) c->Q[i][e][j] = q(e, j, i);
        }
    for (int l = 0; l < NP; l++)
        for (int e = 0; e < 3; e++) {
            c->ne2[e][l] = make_float2(-S.eps[e][2 * l], -S.eps[e][2 * l + 1]);
            c->Cs2[e][l] = make_float2(S.C[2 * l][e], S.C[2 * l + 1][e]);
        }
    for (int e = 0; e < 3; e++) {
        c->ne_l[e] = -S.eps[e][NB81 - 1];
        c->Cs_l[e] = S.C[NB81 - 1][e];
    }
    if (F.hal_radius < 1 || F.hal_radius > HAL_R) return fail(IMOPS_ERR_INVALID_ARGUMENT, "hal_radius must be 1..64");
    if (!(P.hal_sigma > 0.0f)) return fail(IMOPS_ERR_INVALID_ARGUMENT, "hal_sigma must be > 0");
    halation_taps(P.hal_sigma, F.hal_radius, taps, dtaps);
    return IMOPS_OK;
}

struct Bufs {
    Const c;  // passed to the kernels by value
    float *taps, *dtaps;
    float htaps[2 * HAL_R + 1];  // host copy of the halation taps
    float *h, *t1, *B, *t2, *Bs, *gB, *t3, *gh, *ga;
    double *p1, *p2;
    int nb;
};

int prepare(const float* x, int W, int H, const ImopsFilmGradParams* P, const ImopsBaselineFilm* F, bool backward,
            cudaStream_t s, Bufs* b) {
    if (!x || !P) return fail(IMOPS_ERR_INVALID_ARGUMENT, "param film: NULL argument");
    if (W <= 0 || H <= 0) return fail(IMOPS_ERR_INVALID_DIMENSIONS, "invalid image dimensions");
    ImopsBaselineFilm Fd;
    if (F) Fd = *F;
    else imops_baseline_film_defaults(&Fd);
    if (backward && (W <= Fd.hal_radius + 1 || H <= Fd.hal_radius + 1))
        return fail(IMOPS_ERR_UNSUPPORTED_SIZE, "param film backward: image sides must exceed the halation radius + 1");
    const size_t n = (size_t)W * H;
    b->nb = film::grid_for_n(n);
    size_t bytes = 2 * (2 * HAL_R + 1) * 4 + (backward ? 12 : 3) * n * 4 +
                   (size_t)b->nb * 25 * 8 + 8192;
    void* ws = nullptr;
    int rc = workspace(s, bytes, &ws);
    if (rc) return rc;
    Arena A{static_cast<char*>(ws), 0};
    b->taps = A.take<float>(2 * HAL_R + 1);
    b->dtaps = A.take<float>(2 * HAL_R + 1);
    b->h = A.take<float>(n);
    b->t1 = A.take<float>(n);
    b->B = A.take<float>(n);
    if (backward) {
        b->t2 = A.take<float>(n);
        b->Bs = A.take<float>(n);
        b->gB = A.take<float>(n);
        b->t3 = A.take<float>(n);
        b->gh = A.take<float>(n);
        b->ga = A.take<float>(3 * n);
        b->p1 = A.take<double>((size_t)b->nb * 12);
        b->p2 = A.take<double>((size_t)b->nb * 13);
    }
    std::vector<float> taps(2 * HAL_R + 1), dtaps(2 * HAL_R + 1);
    if ((rc = build_const(*P, Fd, &b->c, taps.data(), dtaps.data()))) return rc;
    for (int i = 0; i < 2 * HAL_R + 1; i++) b->htaps[i] = taps[i];
    IMOPS_CUDA_TRY(cudaMemcpyAsync(b->taps, taps.data(), taps.size() * 4, cudaMemcpyHostToDevice, s), "copy taps");
    IMOPS_CUDA_TRY(cudaMemcpyAsync(b->dtaps, dtaps.data(), dtaps.size() * 4, cudaMemcpyHostToDevice, s), "copy taps");
    const int R = Fd.hal_radius;
    prep_kernel<<<b->nb, BLK, 0, s>>>(x, n, b->c, b->h);
    note_launch();
    if ((rc = film::blur_rows(b->h, b->t1, W, H, taps.data(), R, s))) return rc;
    if ((rc = film::blur_cols(b->t1, b->B, W, H, taps.data(), R, 0, s))) return rc;
    if (backward) {
        // dB/dsigma = cols_G(rows_dG(h)) + cols_dG(rows_G(h))
        if ((rc = film::blur_rows(b->h, b->t2, W, H, dtaps.data(), R, s))) return rc;
        if ((rc = film::blur_cols(b->t2, b->Bs, W, H, taps.data(), R, 0, s))) return rc;
        if ((rc = film::blur_cols(b->t1, b->Bs, W, H, dtaps.data(), R, 1, s))) return rc;
    }
    return IMOPS_OK;
}

}  // namespace adj
}  // namespace imops

using namespace imops;

extern "C" int imops_param_forward(const float* cam_rgb, int w, int h, const ImopsFilmGradParams* params,
                                   const ImopsBaselineFilm* fixed, float* out, imops_stream_t stream) {
    clear_error();
    if (!out) return fail(IMOPS_ERR_INVALID_ARGUMENT, "param forward: NULL output");
    cudaStream_t s = as_stream(stream);
    adj::Bufs b;
    int rc = adj::prepare(cam_rgb, w, h, params, fixed, false, s, &b);
    if (rc) return rc;
    adj::pixel_kernel<0><<<b.nb, adj::BLK, 0, s>>>(cam_rgb, b.B, nullptr, nullptr, nullptr, 0.0f, (size_t)w * h, b.c,
                                                   out, nullptr, nullptr, nullptr);
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), "param forward");
    return IMOPS_OK;
}

extern "C" int imops_param_backward(const float* cam_rgb, const float* g_out, const float* target, float loss_scale,
                                    int w, int h, const ImopsFilmGradParams* params, const ImopsBaselineFilm* fixed,
                                    double* grad, imops_stream_t stream) {
    clear_error();
    if (!grad) return fail(IMOPS_ERR_INVALID_ARGUMENT, "param backward: NULL gradient buffer");
    if (!g_out && !target) return fail(IMOPS_ERR_INVALID_ARGUMENT, "param backward: need g_out or target");
    cudaStream_t s = as_stream(stream);
    adj::Bufs b;
    int rc = adj::prepare(cam_rgb, w, h, params, fixed, true, s, &b);
    if (rc) return rc;
    const size_t n = (size_t)w * h;
    ImopsBaselineFilm Fd;
    if (fixed) Fd = *fixed;
    else imops_baseline_film_defaults(&Fd);
    const int R = Fd.hal_radius;
    adj::pixel_kernel<1><<<b.nb, adj::BLK, 0, s>>>(cam_rgb, b.B, b.Bs, g_out, target, loss_scale, n, b.c, nullptr,
                                                   b.gB, b.ga, b.p1);
    note_launch();
    // gh = rows^T(cols^T(gB)) (the blur is rows then cols): each transposed
    // pass is the tiled blur plus its end terms
    if ((rc = film::blur_cols(b.gB, b.t3, w, h, b.htaps, R, 0, s))) return rc;
    adj::blurT_edges_kernel<<<film::grid_for_n((size_t)w * (2 * R + 2)), adj::BLK, 0, s>>>(b.gB, b.t3, w, h, b.taps,
                                                                                          R, 1);
    note_launch();
    if ((rc = film::blur_rows(b.t3, b.gh, w, h, b.htaps, R, s))) return rc;
    adj::blurT_edges_kernel<<<film::grid_for_n((size_t)h * (2 * R + 2)), adj::BLK, 0, s>>>(b.t3, b.gh, w, h, b.taps,
                                                                                          R, 0);
    note_launch();
    adj::color_back_kernel<<<b.nb, adj::BLK, 0, s>>>(cam_rgb, b.ga, b.gh, n, b.c, b.p2);
    note_launch();
    adj::finish_kernel<<<1, 64, 0, s>>>(b.p1, b.nb, b.p2, b.nb, grad);
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), "param backward");
    return IMOPS_OK;
}
