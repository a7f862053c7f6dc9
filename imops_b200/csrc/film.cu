// film.cu -- spectral film simulation kernels and imops_film_process.
//
// Reference model (film::process, pichromatic/src/film/mod.rs:77-129) as a
// chain of planar kernels:
//   expose (rank-3 spectral collapse) -> local scatter -> support bounce ->
//   capture LUT -> reduce -> DIR -> adjacency -> grain -> 16-bin scan ->
//   [invert].
// Baseline preset (81 bins): expose + halation source -> halation row pass
// -> grain noise -> one fused kernel doing the halation column pass, the
// logistic curves, grain and the 81-bin scan.
//
// Layout: per-layer planes (row-major f32), so every pass is a coalesced
// stream; RGB stays interleaved as in Image.rgb_data.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "film.cuh"

namespace imops {
namespace film {

constexpr int MAXR = 64;  // largest blur radius handled (129 taps)

// The baseline preset's logistic density curve D = dmax / (1 + e^(-k (log10 E
// - x0))) from the hardware base-2 logarithm and exponential (lg2 / ex2
// .approx.ftz, about 2^-22 relative) and a fast reciprocal: log10 E =
// log2 E * log10(2), e^x = 2^(x log2 e).  Within 1e-6 relative of the
// library functions' result; the film's tolerance is 1e-4.
__device__ __forceinline__ float curve_density(float E, float dmax, float k, float x0) {
    float l2;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l2) : "f"(fmaxf(E, 1e-6f)));
    const float le = l2 * 0.30102999566398120f;
    const float t = ex2_fast(-k * (le - x0) * 1.4426950408889634f);
    return __fdividef(dmax, 1.0f + t);
}

struct Taps {
    int R;
    float t[2 * MAXR + 1];
};

// Radius-64 taps as pairs t2[k] = (t[k], t[k-1]), zero outside [0, 128]:
// the radius-64 kernels accumulate two adjacent outputs per packed f32x2 FMA
// (output j takes tap k, output j+1 tap k-1 of the same input sample), each
// output still summing its taps in ascending order.
struct Taps2 {
    float2 t2[2 * MAXR + 2];
};

static Taps2 pair_taps(const Taps& tp) {
    Taps2 p;
    for (int k = 0; k <= 2 * MAXR + 1; k++)
        p.t2[k] = make_float2(k <= 2 * MAXR ? tp.t[k] : 0.0f, k >= 1 ? tp.t[k - 1] : 0.0f);
    return p;
}

__device__ __forceinline__ int reflect(int i, int n) {
    // blur.rs:70-89: mirror without repeating the edge sample
    if (n == 1) return 0;
    int x = i;
    for (;;) {
        if (x < 0) x = -x;
        else if (x >= n) x = 2 * n - 2 - x;
        else return x;
    }
}

// ---------------------------------------------------------------------------
// exposure

// The basis weights of one pixel: w = max(0, Minv * rgb).
__device__ __forceinline__ void basis_weights(const ExposeSpec& X, float r, float g, float b, float (&w)[3]) {
    w[0] = fmaxf(0.0f, X.minv[0] * r + X.minv[1] * g + X.minv[2] * b);
    w[1] = fmaxf(0.0f, X.minv[3] * r + X.minv[4] * g + X.minv[5] * b);
    w[2] = fmaxf(0.0f, X.minv[6] * r + X.minv[7] * g + X.minv[8] * b);
}

// Layer e's absorbed band-mean fluence from the basis weights.
__device__ __forceinline__ float layer_exposure(const ExposeSpec& X, const float (&w)[3], int e) {
    return w[0] * X.A[0][e] + w[1] * X.A[1][e] + w[2] * X.A[2][e];
}

// rgb (interleaved) -> E planes of absorbed band-mean fluence, optional
// halation source plane max(0, R - threshold).
__global__ void expose_kernel(const float* __restrict__ rgb, size_t n, ExposeSpec X, float* __restrict__ planes,
                              float* __restrict__ hal) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        float r = rgb[3 * p], g = rgb[3 * p + 1], b = rgb[3 * p + 2];
        float w[3];
        basis_weights(X, r, g, b, w);
        for (int e = 0; e < X.E; e++) planes[e * n + p] = layer_exposure(X, w, e);
        if (X.hal_src) hal[p] = fmaxf(0.0f, r - X.hal_threshold);
    }
}

// ---------------------------------------------------------------------------
// separable Gaussian blur with mirror reflection (blur.rs:10-89)

constexpr int ROW_TILE = 256;

__global__ void blur_rows_kernel(const float* __restrict__ in, float* __restrict__ out, int W, int H, Taps tp) {
    __shared__ float s[ROW_TILE + 2 * MAXR];
    int y = blockIdx.y;
    int x0 = blockIdx.x * ROW_TILE;
    const float* row = in + (size_t)y * W;
    int span = ROW_TILE + 2 * tp.R;
    for (int j = threadIdx.x; j < span; j += blockDim.x) s[j] = __ldg(row + reflect(x0 - tp.R + j, W));
    __syncthreads();
    int x = x0 + threadIdx.x;
    if (x >= W) return;
    float acc = 0.0f;
    for (int k = 0; k <= 2 * tp.R; k++) acc = fmaf(s[threadIdx.x + k], tp.t[k], acc);
    out[(size_t)y * W + x] = acc;
}

constexpr int COL_TW = 32, COL_TH = 64, COL_RPT = 8;  // 32x8 threads, 8 rows each

// Column pass; epi(index, blurred) writes the result.
template <class Epi>
__global__ void blur_cols_kernel(const float* __restrict__ in, int W, int H, Taps tp, Epi epi) {
    __shared__ float s[(COL_TH + 2 * MAXR) * COL_TW];
    int x0 = blockIdx.x * COL_TW, y0 = blockIdx.y * COL_TH;
    int tx = threadIdx.x, ty = threadIdx.y;
    int x = x0 + tx;
    int span = COL_TH + 2 * tp.R;
    if (x < W)
        for (int j = ty; j < span; j += blockDim.y) s[j * COL_TW + tx] = __ldg(in + (size_t)reflect(y0 - tp.R + j, H) * W + x);
    __syncthreads();
    if (x >= W) return;
    for (int r = 0; r < COL_RPT; r++) {
        int ly = ty * COL_RPT + r, y = y0 + ly;
        if (y >= H) break;
        float acc = 0.0f;
        for (int k = 0; k <= 2 * tp.R; k++) acc = fmaf(s[(ly + k) * COL_TW + tx], tp.t[k], acc);
        epi((size_t)y * W + x, acc);
    }
}

// Radius-64 specialisations (the baseline preset's halation and the adjoint):
// the 129 taps are compile-time indexed parameter-bank operands and each
// thread slides one window of loaded samples over several outputs, so the
// loop is nearly all FMAs.  Every output still sums its taps in ascending
// order: results are bit-identical to the generic kernels.
constexpr int R64 = 64;
constexpr int R64_ROW_OUT = 4;                      // outputs per thread
constexpr int R64_ROW_THREADS = 256;
constexpr int R64_ROW_TILE = R64_ROW_OUT * R64_ROW_THREADS;  // 1024 outputs per block

// Row-pass sources: a plane, or the baseline preset's halation source
// max(0, R - threshold) formed from interleaved RGB as it is read.
struct PlaneSource {
    const float* __restrict__ p;
    __device__ float operator()(size_t i) const { return __ldg(p + i); }
};
struct HalationSource {
    const float* __restrict__ rgb;
    float threshold;
    __device__ float operator()(size_t i) const { return fmaxf(0.0f, __ldg(rgb + 3 * i) - threshold); }
};

template <class Src>
__global__ void __launch_bounds__(R64_ROW_THREADS) blur_rows_r64_kernel(const Src in, float* __restrict__ out, int W,
                                                                       int H, const __grid_constant__ Taps2 tp) {
    static_assert(R64_ROW_OUT % 2 == 0, "outputs go in pairs");
    __shared__ __align__(16) float s[R64_ROW_TILE + 2 * R64];
    const int y = blockIdx.y, x0 = blockIdx.x * R64_ROW_TILE;
    const size_t row = (size_t)y * W;
    for (int j = threadIdx.x; j < R64_ROW_TILE + 2 * R64; j += blockDim.x) s[j] = in(row + reflect(x0 - R64 + j, W));
    __syncthreads();
    const int xb = R64_ROW_OUT * threadIdx.x;
    float2 acc[R64_ROW_OUT / 2];
#pragma unroll
    for (int j = 0; j < R64_ROW_OUT / 2; j++) acc[j] = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int q = 0; q < (R64_ROW_OUT + 2 * R64) / 4; q++) {
        const float4 v4 = *reinterpret_cast<const float4*>(s + xb + 4 * q);
        const float v[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const float2 vv = make_float2(v[u], v[u]);
#pragma unroll
            for (int j = 0; j < R64_ROW_OUT / 2; j++) {
                const int k = 4 * q + u - 2 * j;
                if (k >= 0 && k <= 2 * R64 + 1) acc[j] = __ffma2_rn(vv, tp.t2[k], acc[j]);
            }
        }
    }
    float* o = out + (size_t)y * W;
#pragma unroll
    for (int j = 0; j < R64_ROW_OUT / 2; j++) {
        if (x0 + xb + 2 * j < W) o[x0 + xb + 2 * j] = acc[j].x;
        if (x0 + xb + 2 * j + 1 < W) o[x0 + xb + 2 * j + 1] = acc[j].y;
    }
}

constexpr int R64_COL_TW = 32, R64_COL_GROUPS = 8, R64_COL_OUT = 16;  // 32x8 threads, 16 rows each
constexpr int R64_COL_TH = R64_COL_GROUPS * R64_COL_OUT;              // 128 output rows per block
// the plain column blur: output rows per thread
constexpr int BLUR_COL_OUT = 16;

// Stages rows y0 - 64 .. y0 + TH + 63 of column x into the block's window s
// (mirrored at the image edges).  Blocks whose rows all lie inside
// the image read them directly, the loop unrolled so a thread's 32 loads are
// in flight together; edge blocks mirror each row.
template <int TH>
__device__ __forceinline__ void stage_col_window(float* s, const float* __restrict__ in, int W, int H, int x, int y0,
                                                 int tx, int ty) {
    constexpr int ROWS = TH + 2 * R64;
    if (y0 - R64 >= 0 && y0 + TH + R64 <= H) {
        const float* src = in + (size_t)(y0 - R64) * W + x;
#pragma unroll
        for (int j = ty; j < ROWS; j += R64_COL_GROUPS) s[j * R64_COL_TW + tx] = __ldg(src + (size_t)j * W);
    } else {
        for (int j = ty; j < ROWS; j += R64_COL_GROUPS)
            s[j * R64_COL_TW + tx] = __ldg(in + (size_t)reflect(y0 - R64 + j, H) * W + x);
    }
}

// Streaming radius-64 column pass.  A CTA walks a 32-column strip down a
// segment of SC_CHUNKS chunks of 128 output rows.  Its shared window is a
// ring of three 128-row slabs: chunk j reads slabs j and j+1 while the rows
// of slab j+2 are loaded into registers (issued before the chunk's FMAs, so
// their latency hides behind them) and stored into the slot of slab j-1
// afterwards.  A segment reads (chunks + 2) slabs for its chunks' rows
// (1.5x for four chunks, against 2x for a block that stages the 256 rows of
// one chunk).  Each output sums its taps in ascending order with the pair
// taps (t[k], t[k-1]): the same value as the generic column blur.
constexpr int SC_SLAB = R64_COL_GROUPS * BLUR_COL_OUT;  // 128 rows: one chunk of outputs, one slab of inputs
constexpr int SC_CHUNKS = 4;
constexpr int SC_PER = SC_SLAB / R64_COL_GROUPS;  // slab rows loaded per thread

template <class Epi>
__global__ void __launch_bounds__(R64_COL_TW * R64_COL_GROUPS) blur_cols_r64_stream_kernel(
    const float* __restrict__ in, int W, int H, const __grid_constant__ Taps2 tp, Epi epi) {
    static_assert(SC_SLAB == 2 * R64, "a chunk's 256-row window is two slabs");
    __shared__ float ring[3 * SC_SLAB * R64_COL_TW];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x = blockIdx.x * R64_COL_TW + tx;
    const bool xin = x < W;
    const int ybase = blockIdx.y * SC_CHUNKS * SC_SLAB;
    const int left = (H - ybase + SC_SLAB - 1) / SC_SLAB;
    const int nch = left < SC_CHUNKS ? left : SC_CHUNKS;
    float v[SC_PER];
    // slab s: rows ybase - 64 + 128 s .. + 127 of column x (mirrored at the edges)
    auto load = [&](int sl) {
        const int r0 = ybase - R64 + SC_SLAB * sl;
        if (r0 >= 0 && r0 + SC_SLAB <= H) {
            const float* src = in + (size_t)(r0 + ty) * W + x;
#pragma unroll
            for (int q = 0; q < SC_PER; q++) v[q] = xin ? __ldg(src + (size_t)q * R64_COL_GROUPS * W) : 0.0f;
        } else {
#pragma unroll
            for (int q = 0; q < SC_PER; q++)
                v[q] = xin ? __ldg(in + (size_t)reflect(r0 + ty + q * R64_COL_GROUPS, H) * W + x) : 0.0f;
        }
    };
    auto store = [&](int sl) {
        float* slab = ring + (sl % 3) * SC_SLAB * R64_COL_TW;
#pragma unroll
        for (int q = 0; q < SC_PER; q++) slab[(ty + q * R64_COL_GROUPS) * R64_COL_TW + tx] = v[q];
    };
    load(0);
    store(0);
    load(1);
    store(1);
    __syncthreads();
    const int rb = ty * BLUR_COL_OUT;
    for (int j = 0; j < nch; j++) {
        if (j + 1 < nch) load(j + 2);  // in flight during this chunk
        const float* A = ring + (j % 3) * SC_SLAB * R64_COL_TW;
        const float* B = ring + ((j + 1) % 3) * SC_SLAB * R64_COL_TW;
        float2 acc[BLUR_COL_OUT / 2];
#pragma unroll
        for (int q = 0; q < BLUR_COL_OUT / 2; q++) acc[q] = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int m = 0; m < BLUR_COL_OUT + 2 * R64; m++) {
            const int row = rb + m;
            const float val = row < SC_SLAB ? A[row * R64_COL_TW + tx] : B[(row - SC_SLAB) * R64_COL_TW + tx];
            const float2 vv = make_float2(val, val);
#pragma unroll
            for (int q = 0; q < BLUR_COL_OUT / 2; q++) {
                const int k = m - 2 * q;
                if (k >= 0 && k <= 2 * R64 + 1) acc[q] = __ffma2_rn(vv, tp.t2[k], acc[q]);
            }
        }
        if (xin) {
            const int y0 = ybase + j * SC_SLAB + rb;
#pragma unroll
            for (int q = 0; q < BLUR_COL_OUT / 2; q++) {
                const int yy = y0 + 2 * q;
                if (yy < H) epi((size_t)yy * W + x, acc[q].x);
                if (yy + 1 < H) epi((size_t)(yy + 1) * W + x, acc[q].y);
            }
        }
        if (j + 1 < nch) store(j + 2);  // into the slot of slab j-1, read last in chunk j-1
        __syncthreads();
    }
}

struct EpiStore {
    float* out;
    __device__ __forceinline__ void operator()(size_t i, float v) const { out[i] = v; }
};
// local scatter: p = keep*p + mix*blur(p) (halation.rs:164-181)
struct EpiMix {
    float* plane;
    float keep, mix;
    __device__ __forceinline__ void operator()(size_t i, float v) const { plane[i] = keep * plane[i] + mix * v; }
};
// support bounce: plane_e += gain_e * blur(deep) (halation.rs:80-92)
struct EpiBounce {
    float* planes;
    size_t n;
    int E;
    float gain[MAXE];
    __device__ __forceinline__ void operator()(size_t i, float v) const {
        for (int e = 0; e < E; e++)
            if (gain[e] > 0.0f) planes[e * n + i] += gain[e] * v;
    }
};
// adjacency: d += beta * (d - blur(d)) (diffusion.rs:11-28)
struct EpiAdjacency {
    float* plane;
    float beta;
    __device__ __forceinline__ void operator()(size_t i, float v) const {
        float d = plane[i];
        plane[i] = d + beta * (d - v);
    }
};

struct EpiAdd {
    float* out;
    __device__ __forceinline__ void operator()(size_t i, float v) const { out[i] += v; }
};

int blur_rows(const float* in, float* out, int W, int H, const float* taps, int R, cudaStream_t s) {
    if (R < 0 || R > MAXR) return fail(IMOPS_ERR_INVALID_ARGUMENT, "blur radius above 64");
    Taps tp;
    tp.R = R;
    for (int i = 0; i < 2 * R + 1; i++) tp.t[i] = taps[i];
    if (R == R64) {
        dim3 rg((W + R64_ROW_TILE - 1) / R64_ROW_TILE, H);
        blur_rows_r64_kernel<<<rg, R64_ROW_THREADS, 0, s>>>(PlaneSource{in}, out, W, H, pair_taps(tp));
    } else {
        dim3 rg((W + ROW_TILE - 1) / ROW_TILE, H);
        blur_rows_kernel<<<rg, ROW_TILE, 0, s>>>(in, out, W, H, tp);
    }
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), "blur rows");
    return IMOPS_OK;
}

// The baseline preset's halation row pass straight from interleaved RGB: the
// radius-64 row blur of max(0, R - threshold), the source formed as it is
// read instead of as a plane of its own.
static int blur_rows_halation(const float* rgb, float threshold, float* out, int W, int H, const float* taps,
                              cudaStream_t s) {
    Taps tp;
    tp.R = R64;
    for (int i = 0; i < 2 * R64 + 1; i++) tp.t[i] = taps[i];
    dim3 rg((W + R64_ROW_TILE - 1) / R64_ROW_TILE, H);
    blur_rows_r64_kernel<<<rg, R64_ROW_THREADS, 0, s>>>(HalationSource{rgb, threshold}, out, W, H, pair_taps(tp));
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), "halation row pass");
    return IMOPS_OK;
}

int blur_cols(const float* in, float* out, int W, int H, const float* taps, int R, int add, cudaStream_t s) {
    if (R < 0 || R > MAXR) return fail(IMOPS_ERR_INVALID_ARGUMENT, "blur radius above 64");
    Taps tp;
    tp.R = R;
    for (int i = 0; i < 2 * R + 1; i++) tp.t[i] = taps[i];
    if (R == R64) {
        dim3 cb(R64_COL_TW, R64_COL_GROUPS),
            cg((W + R64_COL_TW - 1) / R64_COL_TW, (H + SC_CHUNKS * SC_SLAB - 1) / (SC_CHUNKS * SC_SLAB));
        const Taps2 t2 = pair_taps(tp);
        if (add) blur_cols_r64_stream_kernel<<<cg, cb, 0, s>>>(in, W, H, t2, EpiAdd{out});
        else blur_cols_r64_stream_kernel<<<cg, cb, 0, s>>>(in, W, H, t2, EpiStore{out});
    } else {
        dim3 cb(COL_TW, COL_TH / COL_RPT), cg((W + COL_TW - 1) / COL_TW, (H + COL_TH - 1) / COL_TH);
        if (add) blur_cols_kernel<<<cg, cb, 0, s>>>(in, W, H, tp, EpiAdd{out});
        else blur_cols_kernel<<<cg, cb, 0, s>>>(in, W, H, tp, EpiStore{out});
    }
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), "blur cols");
    return IMOPS_OK;
}

int taps_for(float sigma, Taps* tp) {
    int r = gaussian_taps(sigma, tp->t, 2 * MAXR + 1);
    if (r < 0) return fail(IMOPS_ERR_UNSUPPORTED_SIZE, "film: blur radius above 64 px (pixel pitch too small)");
    tp->R = r;
    return IMOPS_OK;
}

template <class Epi>
int blur(const float* in, float* tmp, int W, int H, const Taps& tp, Epi epi, cudaStream_t s) {
    dim3 rg((W + ROW_TILE - 1) / ROW_TILE, H);
    blur_rows_kernel<<<rg, ROW_TILE, 0, s>>>(in, tmp, W, H, tp);
    note_launch();
    dim3 cb(COL_TW, COL_TH / COL_RPT), cg((W + COL_TW - 1) / COL_TW, (H + COL_TH - 1) / COL_TH);
    blur_cols_kernel<<<cg, cb, 0, s>>>(tmp, W, H, tp, epi);
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), "film blur launch");
    return IMOPS_OK;
}

// ---------------------------------------------------------------------------
// capture LUT + reduce (capture.rs:61-88, reduction.rs:16-68)

__device__ __forceinline__ float lut_sample(const float* logs, const float* fr, float phi) {
    if (!(phi > 0.0f)) return fr[0];
    float lp = log10f(phi);
    if (lp <= logs[0]) return fr[0];
    if (lp >= logs[LUTN - 1]) return fr[LUTN - 1];
    int lo = 0, hi = LUTN - 1;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (logs[mid] <= lp) lo = mid; else hi = mid;
    }
    float t = (lp - logs[lo]) / (logs[hi] - logs[lo]);
    return fr[lo] * (1.0f - t) + fr[hi] * t;
}

__global__ void lut_reduce_kernel(float* __restrict__ planes, float* __restrict__ mask, size_t n, int E,
                                  const RefSpec* __restrict__ R) {
    __shared__ float logs[MAXE][LUTN], fr[MAXE][LUTN];
    for (int k = threadIdx.x; k < E * LUTN; k += blockDim.x) {
        logs[k / LUTN][k % LUTN] = R->lut_log[k / LUTN][k % LUTN];
        fr[k / LUTN][k % LUTN] = R->lut_frac[k / LUTN][k % LUTN];
    }
    __syncthreads();
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        for (int e = 0; e < E; e++) {
            float phi = planes[e * n + p] * R->eta[e];
            float f = lut_sample(logs[e], fr[e], phi);
            f = fminf(fmaxf(f, 0.0f), 1.0f);
            float ef = R->reversal[e] ? 1.0f - f : f;
            float dmax = R->dmax[e];
            float d = dmax * powf(ef, R->inv_gamma[e]);
            planes[e * n + p] = d;
            mask[e * n + p] = R->has_mask[e] ? R->mask_scale[e] * (1.0f - fminf(fmaxf(d / dmax, 0.0f), 1.0f)) : 0.0f;
        }
}

// DIR inhibition: D_j *= exp(-sum_i m[i][j] * inh_i) (diffusion.rs:39-84)
__global__ void dir_apply_kernel(float* __restrict__ planes, const float* __restrict__ inh, size_t n, int E,
                                 const RefSpec* __restrict__ R) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        for (int j = 0; j < E; j++) {
            float tot = 0.0f;
            bool active = false;
            for (int i = 0; i < E; i++) {
                float w = R->dir[i][j];
                if (w != 0.0f) {
                    active = true;
                    tot += w * inh[i * n + p];
                }
            }
            if (active) planes[j * n + p] *= expf(-tot);
        }
}

// ---------------------------------------------------------------------------
// grain (grain.rs:20-100): SplitMix64 is counter based, so pixel x of row y
// uses draws 12x+1..12x+12 of the row stream and is generated independently.

// The blurred grain fields of LAYERS consecutive RNG layers of one tile in one
// pass: Irwin-Hall noise over the tile plus its halo (grain_noise_at),
// mirrored at the image edge; per layer the row then column passes of blur()
// in shared memory with the same taps and summation order (so each field
// equals blur(noise) bit for bit); the fields written, and each layer's block
// sum of squares (f64) stored in partial[plane][block] for the variance.
// Plane z holds RNG layer layer0 + z.  Radius <= GR_MAXR.
//
// Tiles are 128 x 39: the three layers' noise and one row-blurred layer take
// 96 KB at radius 3, so two blocks (32 warps) share an SM.  Inside the image
// a thread generates a run of GR_RUN consecutive pixels of a row, whose
// layers share all but the last two draws of the next pixel
// (grain_noise_run): 12 GR_RUN + 2 draws a run instead of 14 a pixel.  The
// 45 rows of a tile and its halo at radius 3 are 1530 runs, three for each
// of the 512 threads.
constexpr int GR_TW = 128, GR_TH = 39, GR_MAXR = 16, GR_RUN = 4;
constexpr int GR_THREADS = 512, GR_TY = GR_THREADS / 32;
static_assert(GR_TW == 128, "the blur loops index tile columns with & 127");

// Noise of pixel (y, x) in LAYERS consecutive layers layer0, layer0+1, ...
// (grain.rs:20-45, 53-66).  Layer L of row y is the SplitMix64 stream seeded
// seed*0xD1B54A32D192ED03 + L*golden + y, and pixel x takes its draws
// 12x+1 .. 12x+12, the sum of those 12 uniforms minus 6.  Draw k of layer L
// has the state seed*C + y + (L + 12x + k)*golden, which is draw L + k of
// layer 0's stream: consecutive layers share all but one of their draws.  So
// the layers of pixel x take the LAYERS + 11 draws 12x+layer0+1 .. of one
// stream, each draw mixed once, and layer layer0 + z sums draws z+1 .. z+12
// of them in order (each sum in f32, in the reference's order).
template <int LAYERS>
__device__ __forceinline__ void grain_noise_at(uint64_t seed, int layer0, int y, int x, float (&out)[LAYERS]) {
    const uint64_t golden = 0x9E3779B97F4A7C15ull;
    // state of draw k is s0 + k * golden (mod 2^64): stepped, not multiplied
    uint64_t z0 = seed * 0xD1B54A32D192ED03ull + (uint64_t)layer0 * golden + (uint64_t)y + 12 * (uint64_t)x * golden;
    float acc[LAYERS];
#pragma unroll
    for (int z = 0; z < LAYERS; z++) acc[z] = 0.0f;
#pragma unroll
    for (int k = 1; k <= LAYERS + 11; k++) {
        z0 += golden;
        uint64_t v = (z0 ^ (z0 >> 30)) * 0xBF58476D1CE4E5B9ull;
        v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
        const float u = __ull2float_rn(v ^ (v >> 31)) / 18446744073709551616.0f;
#pragma unroll
        for (int z = 0; z < LAYERS; z++)
            if (k >= z + 1 && k <= z + 12) acc[z] += u;
    }
#pragma unroll
    for (int z = 0; z < LAYERS; z++) out[z] = acc[z] - 6.0f;
}

// The same for RUN consecutive pixels x .. x+RUN-1 of row y: pixel x+i takes
// draws 12i+1 .. 12i+LAYERS+11 counted from pixel x's first, so the run
// mixes its 12 RUN + LAYERS - 1 draws once each; every (pixel, layer) sum adds
// its 12 draws in the order grain_noise_at does, so the values are identical.
template <int LAYERS, int RUN>
__device__ __forceinline__ void grain_noise_run(uint64_t seed, int layer0, int y, int x, float (&out)[RUN][LAYERS]) {
    const uint64_t golden = 0x9E3779B97F4A7C15ull;
    uint64_t z0 = seed * 0xD1B54A32D192ED03ull + (uint64_t)layer0 * golden + (uint64_t)y + 12 * (uint64_t)x * golden;
    float acc[RUN][LAYERS];
#pragma unroll
    for (int i = 0; i < RUN; i++)
#pragma unroll
        for (int z = 0; z < LAYERS; z++) acc[i][z] = 0.0f;
#pragma unroll
    for (int k = 1; k <= 12 * RUN + LAYERS - 1; k++) {
        z0 += golden;
        uint64_t v = (z0 ^ (z0 >> 30)) * 0xBF58476D1CE4E5B9ull;
        v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
        const float u = __ull2float_rn(v ^ (v >> 31)) / 18446744073709551616.0f;
#pragma unroll
        for (int i = 0; i < RUN; i++)
#pragma unroll
            for (int z = 0; z < LAYERS; z++)
                if (k >= 12 * i + z + 1 && k <= 12 * i + z + 12) acc[i][z] += u;
    }
#pragma unroll
    for (int i = 0; i < RUN; i++)
#pragma unroll
        for (int z = 0; z < LAYERS; z++) out[i][z] = acc[i][z] - 6.0f;
}

template <int LAYERS>
__global__ void __launch_bounds__(GR_THREADS, 2) grain_field_kernel(float* __restrict__ noise, int W, int H,
                                                                    uint64_t seed, int layer0, Taps tp,
                                                                    double* __restrict__ partial) {
    extern __shared__ __align__(16) float gsm[];
    __shared__ double red[GR_TY];
    const int R = tp.R;
    const int x0 = blockIdx.x * GR_TW, y0 = blockIdx.y * GR_TH;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    // noise rows are NW samples; stored with a stride of NWP (a multiple of
    // the run, so runs and their float4 stores stay aligned)
    const int NW = GR_TW + 2 * R, NH = GR_TH + 2 * R;
    const int NWP = (NW + GR_RUN - 1) / GR_RUN * GR_RUN;
    float* sn = gsm;                      // noise, tile + halo: LAYERS x NH x NWP
    float* sr = gsm + LAYERS * NH * NWP;  // row-blurred: NH x GR_TW (one layer at a time)
    // blocks whose tile + halo lies inside the image need no mirroring
    const bool inner = x0 - R >= 0 && y0 - R >= 0 && x0 + GR_TW + R <= W && y0 + GR_TH + R <= H;
    if (inner) {
        // runs of GR_RUN pixels over the rows (the last run of a row may
        // reach past NW: those samples are generated and never read);
        // (row, run) of j stepped without a division
        const int RPR = NWP / GR_RUN, nruns = NH * RPR;
        const int dq = GR_THREADS / RPR, dr = GR_THREADS - dq * RPR;
        int r = tid / RPR, q = tid - (tid / RPR) * RPR;
        for (int j = tid; j < nruns; j += GR_THREADS) {
            float v[GR_RUN][LAYERS];
            grain_noise_run<LAYERS, GR_RUN>(seed, layer0, y0 - R + r, x0 - R + q * GR_RUN, v);
#pragma unroll
            for (int z = 0; z < LAYERS; z++) {
                static_assert(GR_RUN == 4, "one float4 store a run and layer");
                *reinterpret_cast<float4*>(sn + (z * NH + r) * NWP + q * GR_RUN) =
                    make_float4(v[0][z], v[1][z], v[2][z], v[3][z]);
            }
            r += dq;
            q += dr;
            if (q >= RPR) {
                q -= RPR;
                r++;
            }
        }
    } else {
        const int dq = GR_THREADS / NW, dr = GR_THREADS - dq * NW;
        int r = tid / NW, c = tid - (tid / NW) * NW;
        for (int idx = tid; idx < NH * NW; idx += GR_THREADS) {
            float v[LAYERS];
            grain_noise_at<LAYERS>(seed, layer0, reflect(y0 - R + r, H), reflect(x0 - R + c, W), v);
#pragma unroll
            for (int z = 0; z < LAYERS; z++) sn[(z * NH + r) * NWP + c] = v[z];
            r += dq;
            c += dr;
            if (c >= NW) {
                c -= NW;
                r++;
            }
        }
    }
    const size_t n = (size_t)W * H;
    for (int z = 0; z < LAYERS; z++) {
        const float* snz = sn + z * NH * NWP;
        __syncthreads();  // the noise is complete; sr is free again
        for (int idx = tid; idx < NH * GR_TW; idx += GR_THREADS) {
            const int r = idx >> 7, c = idx & (GR_TW - 1);
            const float* s = snz + r * NWP + c;
            float acc = 0.0f;
            // radius 3 (a 1 px grain blur, every stock here) unrolled
            if (R == 3) {
#pragma unroll
                for (int k = 0; k <= 6; k++) acc = fmaf(s[k], tp.t[k], acc);
            } else {
                for (int k = 0; k <= 2 * R; k++) acc = fmaf(s[k], tp.t[k], acc);
            }
            sr[idx] = acc;
        }
        __syncthreads();
        double sq = 0.0;
        for (int idx = tid; idx < GR_TH * GR_TW; idx += GR_THREADS) {
            const int r = idx >> 7, c = idx & (GR_TW - 1);
            const int y = y0 + r, x = x0 + c;
            if (y >= H || x >= W) continue;
            const float* s = sr + idx;
            float acc = 0.0f;
            if (R == 3) {
#pragma unroll
                for (int k = 0; k <= 6; k++) acc = fmaf(s[k * GR_TW], tp.t[k], acc);
            } else {
                for (int k = 0; k <= 2 * R; k++) acc = fmaf(s[k * GR_TW], tp.t[k], acc);
            }
            noise[z * n + (size_t)y * W + x] = acc;
            sq += (double)acc * (double)acc;
        }
        for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
        if (threadIdx.x == 0) red[threadIdx.y] = sq;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int w = 0; w < GR_TY; w++) t += red[w];
            partial[(size_t)z * gridDim.x * gridDim.y + blockIdx.y * gridDim.x + blockIdx.x] = t;
        }
    }
}

// sums[layer] = sum of partial[layer][0 .. nb) in a fixed order (one block
// per layer): deterministic run to run.
__global__ void __launch_bounds__(1024) sum_partials_kernel(const double* __restrict__ partial, int nb,
                                                            double* __restrict__ sums) {
    __shared__ double red[1024];
    const double* p = partial + (size_t)blockIdx.x * nb;
    double a = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) a += p[i];
    red[threadIdx.x] = a;
    __syncthreads();
    for (int w = 512; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[blockIdx.x] = red[0];
}

// Blurred grain fields of RNG layers layer0 .. layer0+layers-1 (planes
// noise[z * n]) and their sums of squares sums[z].  partial: scratch of
// grain_partials(W, H, layers) doubles.
size_t grain_partials(int W, int H, int layers) {
    return (size_t)((W + GR_TW - 1) / GR_TW) * ((H + GR_TH - 1) / GR_TH) * layers;
}

int grain_fields(float* noise, int W, int H, uint64_t seed, int layer0, int layers, const Taps& tp, double* partial,
                 double* sums, cudaStream_t s) {
    if (tp.R > GR_MAXR) return fail(IMOPS_ERR_UNSUPPORTED_SIZE, "film: grain blur radius above 16 px");
    dim3 b(32, GR_TY), g((W + GR_TW - 1) / GR_TW, (H + GR_TH - 1) / GR_TH);
    const int NW = GR_TW + 2 * tp.R, NH = GR_TH + 2 * tp.R;
    const int NWP = (NW + GR_RUN - 1) / GR_RUN * GR_RUN;
    // three layers per block (their draws shared) while their noise fits in
    // shared memory; otherwise one block per (tile, layer)
    const size_t smem3 = (size_t)NH * (3 * NWP + GR_TW) * sizeof(float);
    const size_t n = (size_t)W * H, nb = (size_t)g.x * g.y;
    int z = 0;
    if (layers >= 3 && smem3 <= 200 * 1024) {
        IMOPS_CUDA_TRY(cudaFuncSetAttribute(grain_field_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem3),
                       "cudaFuncSetAttribute(grain)");
        for (; z + 3 <= layers; z += 3) {
            grain_field_kernel<3><<<g, b, smem3, s>>>(noise + z * n, W, H, seed, layer0 + z, tp, partial + z * nb);
            note_launch();
        }
    }
    if (z < layers) {
        const size_t smem1 = (size_t)NH * (NWP + GR_TW) * sizeof(float);
        IMOPS_CUDA_TRY(cudaFuncSetAttribute(grain_field_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem1),
                       "cudaFuncSetAttribute(grain)");
        for (; z < layers; z++) {
            grain_field_kernel<1><<<g, b, smem1, s>>>(noise + z * n, W, H, seed, layer0 + z, tp, partial + z * nb);
            note_launch();
        }
    }
    sum_partials_kernel<<<layers, 1024, 0, s>>>(partial, (int)nb, sums);
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), "grain fields");
    return IMOPS_OK;
}

// D <- clamp(D + kappa*taper*sqrt(D(Dmax-D))*n*norm, 0, 1.05 Dmax)
__global__ void grain_apply_kernel(float* __restrict__ plane, const float* __restrict__ noise, size_t n,
                                   const double* __restrict__ sumsq, float kappa, float dmax) {
    double var = *sumsq / (double)n;
    float norm = var > 1e-12 ? (float)(1.0 / sqrt(var)) : 1.0f;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        float d = plane[p];
        float dens = fminf(fmaxf(d, 0.0f), dmax);
        float toe = 0.02f * dmax;
        float taper = fminf(dens / (dens + toe), 1.0f);
        float sd = taper * sqrtf(fmaxf(dens * (dmax - dens), 0.0f));
        d = dens + kappa * sd * noise[p] * norm;
        plane[p] = fminf(fmaxf(d, 0.0f), dmax * 1.05f);
    }
}

// ---------------------------------------------------------------------------
// scan (densitometry.rs:13-73) on the 16-bin grid

__global__ void scan16_kernel(const float* __restrict__ img, const float* __restrict__ mask, size_t n,
                              const ScanSpec16* __restrict__ C, float* __restrict__ rgb) {
    __shared__ ScanSpec16 sc;
    for (int k = threadIdx.x; k < (int)(sizeof(ScanSpec16) / 4); k += blockDim.x)
        reinterpret_cast<float*>(&sc)[k] = reinterpret_cast<const float*>(C)[k];
    __syncthreads();
    const int E = sc.E;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        float di[MAXE], dm[MAXE];
        for (int e = 0; e < E; e++) {
            di[e] = img[e * n + p];
            dm[e] = mask[e * n + p];
        }
        float o0 = 0.f, o1 = 0.f, o2 = 0.f;
#pragma unroll
        for (int l = 0; l < NB16; l++) {
            float d = 0.0f;
            for (int e = 0; e < E; e++) d = fmaf(di[e], sc.eps[e][l], fmaf(dm[e], sc.meps[e][l], d));
            float t = ex2_fast(-d);
            o0 = fmaf(sc.C[l][0], t, o0);
            o1 = fmaf(sc.C[l][1], t, o1);
            o2 = fmaf(sc.C[l][2], t, o2);
        }
        rgb[3 * p] = o0;
        rgb[3 * p + 1] = o1;
        rgb[3 * p + 2] = o2;
    }
}

// invert_negative (invert.rs:36-108); mid/dmin read from device memory.
__global__ void invert_kernel(float* __restrict__ rgb, size_t n, const float* __restrict__ mid_dmin) {
    const float eps = 1e-6f, HEAD = 8.0f, KEEP = 0.55f, FADE = 0.02f, MG = 0.185f;
    const float LR = 0.2722287168f, LG = 0.6740817658f, LB = 0.0536895174f;
    float dmin[3], sh[3], g[3];
    for (int c = 0; c < 3; c++) {
        dmin[c] = fmaxf(mid_dmin[3 + c], eps);
        float mt = fminf(fmaxf(mid_dmin[c] / dmin[c], eps), 1.0f - eps);
        float im = fmaxf(1.0f / mt - 1.0f, 0.0f);
        sh[c] = fmaxf(im * HEAD, eps);
        float i2 = fmaxf(im, 0.0f), s2 = fmaxf(sh[c], 1e-6f);
        float sm = fmaxf(i2 / (1.0f + i2 / s2), eps);
        g[c] = MG / sm;
    }
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        float raw[3];
        for (int c = 0; c < 3; c++) {
            float t = fminf(fmaxf(rgb[3 * p + c] / dmin[c], eps), 1.0f);
            float inv = fmaxf(1.0f / t - 1.0f, 0.0f);
            float i2 = fmaxf(inv, 0.0f), s2 = fmaxf(sh[c], 1e-6f);
            raw[c] = fmaxf(g[c] * (i2 / (1.0f + i2 / s2)), 0.0f);
        }
        float y = fmaxf(LR * raw[0] + LG * raw[1] + LB * raw[2], 0.0f);
        float k = y <= 0.0f ? 0.0f : (y >= FADE ? KEEP : KEEP * (y / FADE));
        for (int c = 0; c < 3; c++) rgb[3 * p + c] = fmaxf(y + k * (raw[c] - y), 0.0f);
    }
}

// mean RGB of a small buffer in f64 (invert.rs:111-125), one block
__global__ void mean_rgb_kernel(const float* __restrict__ rgb, int n, float* __restrict__ out) {
    __shared__ double s[3][256];
    double a[3] = {0, 0, 0};
    for (int p = threadIdx.x; p < n; p += blockDim.x)
        for (int c = 0; c < 3; c++) a[c] += (double)rgb[3 * p + c];
    for (int c = 0; c < 3; c++) s[c][threadIdx.x] = a[c];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int c = 0; c < 3; c++) s[c][threadIdx.x] += s[c][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 3; c++) out[c] = (float)(s[c][0] / (double)n);
}

// ---------------------------------------------------------------------------
// baseline preset: fused halation column pass + logistic curves + grain +
// 81-bin scan.  Each block owns a 32x64 pixel tile and stages the rows of
// the halation row-pass output it needs (64 + 2*64) in shared memory.

// The 81-bin tables as pairs of adjacent bins (2l, 2l+1) for the packed f32x2
// FMA of sm_100 (FFMA2: two lanes per instruction), plus the last bin:
//   ne[e][l]  = -(eps_e(2l), eps_e(2l+1))   (negated: the sum is -d directly)
//   C2[c][l]  = (C(2l)[c], C(2l+1)[c])
// tap2[k] = (taps[k], taps[k-1]) with zero outside [0, 2R] feeds the column
// pass two outputs (rows j, j+1) per instruction; each output still sums its
// taps in ascending order.
constexpr int NP81 = NB81 / 2;  // 40 pairs + bin 80
struct Pairs81 {
    float2 ne[3][NP81];
    float2 C2[3][NP81];
    float ne_last[3], C_last[3];
};

struct Base81 {
    BaselineSpec B;
    ExposeSpec X;
    Pairs81 P;
    float2 tap2[2 * HAL_R + 2];
};

// One thread per 16 consecutive rows of a column: the halation column pass
// (register sliding window, tap pairs as parameter-bank operands, ascending
// tap order as in blur_cols), then per pixel the exposure of the three layers
// from its RGB, the logistic curves, grain and the 81-bin scan with its
// tables as parameter-bank operands; the result replaces the pixel's RGB
// (each pixel is read, a step ahead, and written by the same thread).  Four
// blocks an SM (64 registers a thread): the scan is bound by the MUFU, and
// 32 warps keep more of its exponentials in flight than 24.
__global__ void __launch_bounds__(R64_COL_TW * R64_COL_GROUPS, 4) scan81_fused_kernel(
    const float* __restrict__ hr, const float* __restrict__ noise, const double* __restrict__ sumsq, int W, int H,
    const __grid_constant__ Base81 c, float* __restrict__ rgb) {
    static_assert(HAL_R == R64, "the fused scan's column pass is the radius-64 window");
    static_assert(R64_COL_OUT % 2 == 0, "column outputs go in pairs");
    __shared__ float s[(R64_COL_TH + 2 * HAL_R) * R64_COL_TW];
    const int x0 = blockIdx.x * R64_COL_TW, y0 = blockIdx.y * R64_COL_TH;
    const int tx = threadIdx.x, ty = threadIdx.y, x = x0 + tx;
    if (x < W) stage_col_window<R64_COL_TH>(s, hr, W, H, x, y0, tx, ty);
    __syncthreads();
    if (x >= W) return;
    const size_t n = (size_t)W * H;
    float norm[3] = {1.f, 1.f, 1.f};
    if (c.B.grain_sigma > 0.0f)
        for (int e = 0; e < 3; e++) {
            double var = sumsq[e] / (double)n;
            norm[e] = var > 1e-12 ? (float)(1.0 / sqrt(var)) : 1.0f;
        }
    const int rb = ty * R64_COL_OUT;
    // bs[q] = (output row 2q, output row 2q+1); at window row m the pair takes
    // taps m-2q and m-2q-1
    float2 bs[R64_COL_OUT / 2];
#pragma unroll
    for (int q = 0; q < R64_COL_OUT / 2; q++) bs[q] = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int m = 0; m < R64_COL_OUT + 2 * HAL_R; m++) {
        const float v = s[(rb + m) * R64_COL_TW + tx];
        const float2 vv = make_float2(v, v);
#pragma unroll
        for (int q = 0; q < R64_COL_OUT / 2; q++) {
            const int k = m - 2 * q;
            if (k >= 0 && k <= 2 * HAL_R + 1) bs[q] = __ffma2_rn(vv, c.tap2[k], bs[q]);
        }
    }
    // Two pixels (rows j and j+1 of the column) a step: each table pair is
    // fetched once for both, and the next step's RGB and noise are loaded
    // while this step is scanned, so the global-load latency hides behind
    // the 81-bin loop.  Each pixel's arithmetic is unchanged.
    static_assert(R64_COL_OUT % 2 == 0, "pixels go in pairs");
    const bool grain = c.B.grain_sigma > 0.0f;
    float na[2][3], nz[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    auto fetch = [&](int jj) {  // rows jj, jj+1 (clamped to the image)
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const size_t pp = (size_t)min(y0 + rb + jj + u, H - 1) * W + x;
#pragma unroll
            for (int e = 0; e < 3; e++) {
                na[u][e] = rgb[3 * pp + e];
                if (grain) nz[u][e] = noise[e * n + pp];
            }
        }
    };
    fetch(0);
#pragma unroll 1
    for (int j = 0; j < R64_COL_OUT; j += 2) {
        const int y = y0 + rb + j;
        if (y >= H) break;
        float ca[2][3], cz[2][3];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            float w[3];
            basis_weights(c.X, na[u][0], na[u][1], na[u][2], w);
#pragma unroll
            for (int e = 0; e < 3; e++) {
                ca[u][e] = layer_exposure(c.X, w, e);
                cz[u][e] = nz[u][e];
            }
        }
        if (j + 2 < R64_COL_OUT && y + 2 < H) fetch(j + 2);
        float bsum[2] = {bs[0].x, bs[0].y};
#pragma unroll
        for (int q = 0; q < R64_COL_OUT / 2; q++)
            if (2 * q == j) {
                bsum[0] = bs[q].x;
                bsum[1] = bs[q].y;
            }
        float D[2][3];
#pragma unroll
        for (int u = 0; u < 2; u++)
#pragma unroll
            for (int e = 0; e < 3; e++) {
                const float E = ca[u][e] + c.B.hal_strength * c.B.bleed[e] * bsum[u];
                D[u][e] = curve_density(E, c.B.dmax[e], c.B.k[e], c.B.x0[e]);
                if (grain) D[u][e] += c.B.grain_sigma * cz[u][e] * norm[e];
            }
        float2 d[2][3], o[2][3];
#pragma unroll
        for (int u = 0; u < 2; u++)
#pragma unroll
            for (int e = 0; e < 3; e++) {
                d[u][e] = make_float2(D[u][e], D[u][e]);
                o[u][e] = make_float2(0.f, 0.f);
            }
#pragma unroll
        for (int l = 0; l < NP81; l++) {
            const float2 n0 = c.P.ne[0][l], n1 = c.P.ne[1][l], n2 = c.P.ne[2][l];
            const float2 c0 = c.P.C2[0][l], c1 = c.P.C2[1][l], c2 = c.P.C2[2][l];
#pragma unroll
            for (int u = 0; u < 2; u++) {
                float2 xd = __fmul2_rn(d[u][0], n0);
                xd = __ffma2_rn(d[u][1], n1, xd);
                xd = __ffma2_rn(d[u][2], n2, xd);
                const float2 t = make_float2(ex2_fast(xd.x), ex2_fast(xd.y));
                o[u][0] = __ffma2_rn(c0, t, o[u][0]);
                o[u][1] = __ffma2_rn(c1, t, o[u][1]);
                o[u][2] = __ffma2_rn(c2, t, o[u][2]);
            }
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {
            if (y + u >= H) break;
            float xl = D[u][0] * c.P.ne_last[0];
            xl = fmaf(D[u][1], c.P.ne_last[1], xl);
            xl = fmaf(D[u][2], c.P.ne_last[2], xl);
            const float tl = ex2_fast(xl);
            const size_t p = (size_t)(y + u) * W + x;
            rgb[3 * p] = fmaf(c.P.C_last[0], tl, o[u][0].x + o[u][0].y);
            rgb[3 * p + 1] = fmaf(c.P.C_last[1], tl, o[u][1].x + o[u][1].y);
            rgb[3 * p + 2] = fmaf(c.P.C_last[2], tl, o[u][2].x + o[u][2].y);
        }
    }
}

// ---------------------------------------------------------------------------
// The 81-bin scan on the tensor cores (tcgen05, sm_100a): the same fused
// kernel (halation column pass, logistic curves, grain) with the two spectral
// contractions as BF16 MMAs with FP32 accumulation and a hi/lo split of both
// operands, per tile of 128 pixels (one warpgroup, one TMEM lane a pixel):
//   MMA1  x[128 x 96] = A1[128 x 16] . B1[96 x 16]^T      (A1, B1 in SMEM)
//         A1 row = (Dh, Dl, Dh, Dl) of the three layer densities, B1 row of
//         bin l = (eh, eh, el, el) of -eps(l) (log2 units), so
//         x = (Dh + Dl) . (eh + el) = -d(l) to f32 accuracy;
//   T = 2^x per bin (MUFU), split into bf16 T = Th + Tl, written over x in TMEM;
//   MMA2  rgb[128 x 16] += Th . Ch + Th . Cl + Tl . Ch    (A from TMEM, B in SMEM)
//         over six K-blocks of 16 bins (81 bins padded to 96 with zeros).
// Dropping Tl . Cl and bf16 rounding leave about 2^-17 relative per term.
namespace tc {

constexpr int NBP = 96;                   // bins padded to the MMA's granularity
constexpr uint32_t SBO_K16 = 256;         // K = 16 tiles: two 128-byte K-groups per 8-row group
constexpr uint32_t SBO_K96 = 1536;        // K = 96 tiles: twelve K-groups per 8-row group
constexpr int B1_WORDS = NBP * 16 / 2;    // 96 bins x 16 bf16
constexpr int B2_WORDS = 16 * NBP / 2;    // 16 channel rows (3 used) x 96 bins

// Byte offset of bf16 element (row r, k) in a K-major tile without swizzle:
// core matrices of 8 rows x 16 bytes, K-groups 128 bytes apart (LBO), 8-row
// groups `sbo` apart.
__host__ __device__ __forceinline__ uint32_t cm_off(int r, int k, uint32_t sbo) {
    return (uint32_t)(r >> 3) * sbo + (uint32_t)(k >> 3) * 128u + (uint32_t)(r & 7) * 16u + (uint32_t)(k & 7) * 2u;
}

// B operands, already in their shared-memory layout
struct Tables {
    uint32_t b1[B1_WORDS];
    uint32_t b2h[B2_WORDS];
    uint32_t b2l[B2_WORDS];
};

// dynamic shared memory (bytes)
constexpr uint32_t WIN_BYTES = (R64_COL_TH + 2 * HAL_R) * R64_COL_TW * 4;
constexpr uint32_t OFF_TAB = WIN_BYTES;
constexpr uint32_t OFF_B1 = OFF_TAB, OFF_B2H = OFF_B1 + B1_WORDS * 4, OFF_B2L = OFF_B2H + B2_WORDS * 4;
constexpr uint32_t OFF_A1 = OFF_B2L + B2_WORDS * 4;  // two warpgroups x 128 rows x 16 bf16
constexpr uint32_t OFF_BAR = OFF_A1 + 2 * 4096;      // four mbarriers
constexpr uint32_t OFF_SLOT = OFF_BAR + 32;          // TMEM base address
constexpr uint32_t SMEM_USED = OFF_SLOT + 16;
// Requested per CTA: at most two CTAs an SM, whose 2 x 256 TMEM columns fit
// the SM's 512, so no CTA waits in tcgen05.alloc for another to finish.
constexpr uint32_t SMEM_REQ = 80 * 1024;
static_assert(SMEM_USED <= SMEM_REQ && 3 * SMEM_REQ > 228 * 1024, "two CTAs an SM");

// instruction descriptors: BF16 A and B (K-major), FP32 D, M = 128
constexpr uint32_t idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
constexpr uint32_t IDESC_X = idesc(NBP), IDESC_RGB = idesc(16);

// try_wait suspends the warp until the phase completes or about SUSPEND_NS
// pass; after WAIT_LIMIT tries (about a second) the MMA is declared lost
constexpr int WAIT_LIMIT = 1 << 10;
constexpr uint32_t SUSPEND_NS = 1000000;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, no swizzle, LBO 128 bytes
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t sbo) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);
}

__device__ __forceinline__ void mma_ss(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile("{ .reg .pred p; setp.ne.b32 p, %4, 0; tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p; }"
                 ::"r"(d), "l"(a), "l"(b), "r"(id), "r"(acc));
}
__device__ __forceinline__ void mma_ts(uint32_t d, uint32_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile("{ .reg .pred p; setp.ne.b32 p, %4, 0; tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p; }"
                 ::"r"(d), "r"(a), "l"(b), "r"(id), "r"(acc));
}
__device__ __forceinline__ void commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
// Bounded wait for phase `parity` of an mbarrier: false when it gave up.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
    for (int it = 0; it < WAIT_LIMIT; it++) {
        uint32_t ok;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3; selp.u32 %0, 1, 0, p; }"
            : "=r"(ok) : "r"(bar), "r"(parity), "r"(SUSPEND_NS) : "memory");
        if (ok) return true;
    }
    return false;
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void wg_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }

__device__ __forceinline__ void ld16(uint32_t ta, uint32_t (&v)[16]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                   "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                 : "r"(ta));
}
__device__ __forceinline__ void ld4(uint32_t ta, uint32_t (&v)[4]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]) : "r"(ta));
}
__device__ __forceinline__ void st8(uint32_t ta, const uint32_t (&v)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};"
                 ::"r"(ta), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
                 : "memory");
}
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// bf16x2 of (a, b), round to nearest: a in the low half (the even K index)
__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
    return r;
}
// hi = bf16(a), bf16(b); lo = bf16 of what hi leaves out
__device__ __forceinline__ void split_bf16(float a, float b, uint32_t& hi, uint32_t& lo) {
    hi = pack_bf16(a, b);
    lo = pack_bf16(a - __uint_as_float(hi << 16), b - __uint_as_float(hi & 0xFFFF0000u));
}

}  // namespace tc

struct Base81TC {
    BaselineSpec B;
    ExposeSpec X;
    float2 tap2[2 * HAL_R + 2];
    tc::Tables T;
};

// Lost MMA completions (a bounded wait that gave up), counted across launches.
__device__ unsigned g_tc_timeouts = 0;

__global__ void __launch_bounds__(R64_COL_TW * R64_COL_GROUPS, 2) scan81_tc_kernel(
    const float* __restrict__ hr, const float* __restrict__ noise, const double* __restrict__ sumsq, int W, int H,
    const __grid_constant__ Base81TC c, float* __restrict__ rgb) {
    using namespace tc;
    static_assert(R64_COL_GROUPS == 8, "two warpgroups of four warps");
    extern __shared__ __align__(1024) uint8_t dsm[];
    float* s = reinterpret_cast<float*>(dsm);
    const int x0 = blockIdx.x * R64_COL_TW, y0 = blockIdx.y * R64_COL_TH;
    const int tx = threadIdx.x, ty = threadIdx.y, x = x0 + tx, tid = ty * 32 + tx;
    const int g = ty >> 2;     // warpgroup
    const int row = tid & 127; // this thread's MMA row (TMEM lane)
    const uint32_t sb = smem_u32(dsm);
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(&c.T);
        uint32_t* dst = reinterpret_cast<uint32_t*>(dsm + OFF_TAB);
        for (int i = tid; i < (int)(sizeof(Tables) / 4); i += blockDim.x * blockDim.y) dst[i] = src[i];
    }
    if (x < W) stage_col_window<R64_COL_TH>(s, hr, W, H, x, y0, tx, ty);
    uint32_t* slot = reinterpret_cast<uint32_t*>(dsm + OFF_SLOT);
    if (tid == 0) {
        for (int i = 0; i < 4; i++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sb + OFF_BAR + 8 * i));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (ty == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(sb + OFF_SLOT));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the tables are read by the MMAs
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tm = *slot + (uint32_t)(g * 128);                // this warpgroup's 128 columns
    const uint32_t tl = tm + (((uint32_t)(ty & 3) * 32u) << 16);    // this warp's 32 lanes
    const uint32_t bar_x = sb + OFF_BAR + 16 * g, bar_rgb = bar_x + 8;
    const uint32_t a1 = sb + OFF_A1 + 4096u * g;
    uint8_t* a1p = dsm + OFF_A1 + 4096u * g;

    const size_t n = (size_t)W * H;
    float norm[3] = {1.f, 1.f, 1.f};
    if (c.B.grain_sigma > 0.0f)
        for (int e = 0; e < 3; e++) {
            double var = sumsq[e] / (double)n;
            norm[e] = var > 1e-12 ? (float)(1.0 / sqrt(var)) : 1.0f;
        }
    const int rb = ty * R64_COL_OUT;
    float2 bs[R64_COL_OUT / 2];
#pragma unroll
    for (int q = 0; q < R64_COL_OUT / 2; q++) bs[q] = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int m = 0; m < R64_COL_OUT + 2 * HAL_R; m++) {
        const float v = s[(rb + m) * R64_COL_TW + tx];
        const float2 vv = make_float2(v, v);
#pragma unroll
        for (int q = 0; q < R64_COL_OUT / 2; q++) {
            const int k = m - 2 * q;
            if (k >= 0 && k <= 2 * HAL_R + 1) bs[q] = __ffma2_rn(vv, c.tap2[k], bs[q]);
        }
    }
    const bool grain = c.B.grain_sigma > 0.0f;
    const bool xin = x < W;
    // Per step j (row y0 + rb + j of every warp: 128 pixels a warpgroup) the
    // MMAs of one step overlap the CUDA-core work of its neighbours: MMA2 of
    // step j runs while the densities of step j+1 are formed, MMA1 of step
    // j+1 while step j's pixels are stored.  RGB and noise are loaded a step
    // ahead (each pixel is read and written by the same thread).
    float la[3] = {0.f, 0.f, 0.f}, lz[3] = {0.f, 0.f, 0.f};  // inputs of the next step
    auto load_inputs = [&](int jj) {
        const int yy = y0 + rb + jj;
        if (xin && yy < H && jj < R64_COL_OUT) {
            const size_t p = (size_t)yy * W + x;
#pragma unroll
            for (int e = 0; e < 3; e++) {
                la[e] = rgb[3 * p + e];
                lz[e] = grain ? noise[e * n + p] : 0.0f;
            }
        }
    };
    // densities of step jj into A1 (k 0..11 = Dh0 Dh1 Dh2 Dl0 Dl1 Dl2 Dh0 Dh1
    // Dh2 Dl0 Dl1 Dl2, 12..15 zero), from the inputs loaded for it
    auto write_a1 = [&](int jj) {
        const int yy = y0 + rb + jj;
        float D[3] = {0.0f, 0.0f, 0.0f};
        if (xin && yy < H) {
            float bsum = bs[0].x;
#pragma unroll
            for (int q = 0; q < R64_COL_OUT / 2; q++) {
                if (2 * q == jj) bsum = bs[q].x;
                if (2 * q + 1 == jj) bsum = bs[q].y;
            }
            float w[3];
            basis_weights(c.X, la[0], la[1], la[2], w);
#pragma unroll
            for (int e = 0; e < 3; e++) {
                const float E = layer_exposure(c.X, w, e) + c.B.hal_strength * c.B.bleed[e] * bsum;
                D[e] = curve_density(E, c.B.dmax[e], c.B.k[e], c.B.x0[e]);
                if (grain) D[e] += c.B.grain_sigma * lz[e] * norm[e];
            }
        }
        uint32_t h01, l01, h2, l2;
        split_bf16(D[0], D[1], h01, l01);
        split_bf16(D[2], 0.0f, h2, l2);
        const uint32_t w0 = h01, w1 = (h2 & 0xFFFFu) | (l01 << 16), w2 = (l01 >> 16) | (l2 << 16);
        *reinterpret_cast<uint4*>(a1p + cm_off(row, 0, SBO_K16)) = make_uint4(w0, w1, w2, w0);
        *reinterpret_cast<uint4*>(a1p + cm_off(row, 8, SBO_K16)) = make_uint4(w1, w2, 0u, 0u);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    };
    bool alive = true;
    auto wait_for = [&](uint32_t bar, uint32_t parity) {
        if (alive && !bar_wait(bar, parity)) {
            alive = false;
            atomicAdd(&g_tc_timeouts, 1u);
        }
        fence_after();
    };

    load_inputs(0);
    write_a1(0);
    load_inputs(1);
    wg_sync(1 + g);
    if (row == 0) {
        fence_after();
        mma_ss(tm, sdesc(a1, SBO_K16), sdesc(sb + OFF_B1, SBO_K16), IDESC_X, 0u);
        commit(bar_x);
    }
#pragma unroll 1
    for (int j = 0; j < R64_COL_OUT; j++) {
        const uint32_t parity = (uint32_t)j & 1u;
        wait_for(bar_x, parity);
        // T = 2^x per bin, split to bf16 hi/lo over the same columns: K-block
        // q (bins 16q .. 16q+15) keeps its hi words in columns 16q .. 16q+7
        // and its lo words in 16q+8 .. 16q+15.  Three K-blocks a batch of
        // TMEM loads, one wait each.
#pragma unroll
        for (int h = 0; h < 2; h++) {
            uint32_t v[3][16];
#pragma unroll
            for (int q = 0; q < 3; q++) ld16(tl + 16u * (3 * h + q), v[q]);
            wait_ld();
#pragma unroll
            for (int q = 0; q < 3; q++) {
                uint32_t hw[8], lw[8];
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const int b0 = 16 * (3 * h + q) + 2 * i;
                    const float t0 = b0 < NB81 ? ex2_fast(__uint_as_float(v[q][2 * i])) : 0.0f;
                    const float t1 = b0 + 1 < NB81 ? ex2_fast(__uint_as_float(v[q][2 * i + 1])) : 0.0f;
                    split_bf16(t0, t1, hw[i], lw[i]);
                }
                st8(tl + 16u * (3 * h + q), hw);
                st8(tl + 16u * (3 * h + q) + 8u, lw);
            }
        }
        wait_st();
        fence_before();
        wg_sync(1 + g);
        if (row == 0 && alive) {
            fence_after();
#pragma unroll
            for (int q = 0; q < NBP / 16; q++) {
                const uint64_t bh = sdesc(sb + OFF_B2H + 256u * q, SBO_K96), bl = sdesc(sb + OFF_B2L + 256u * q, SBO_K96);
                mma_ts(tm + NBP, tm + 16u * q, bh, IDESC_RGB, q > 0 ? 1u : 0u);
                mma_ts(tm + NBP, tm + 16u * q, bl, IDESC_RGB, 1u);
                mma_ts(tm + NBP, tm + 16u * q + 8u, bh, IDESC_RGB, 1u);
            }
            commit(bar_rgb);
        }
        // next step's densities while MMA2 runs (A1 is free: MMA1 of this step is done)
        if (j + 1 < R64_COL_OUT) {
            write_a1(j + 1);
            load_inputs(j + 2);
        }
        wait_for(bar_rgb, parity);
        uint32_t o[4];
        ld4(tl + NBP, o);
        wait_ld();
        fence_before();
        wg_sync(1 + g);  // A1 of the next step written; this step's rgb read from TMEM
        if (j + 1 < R64_COL_OUT && row == 0 && alive) {
            fence_after();
            mma_ss(tm, sdesc(a1, SBO_K16), sdesc(sb + OFF_B1, SBO_K16), IDESC_X, 0u);
            commit(bar_x);
        }
        const int y = y0 + rb + j;
        if (xin && y < H) {
            const size_t p = (size_t)y * W + x;
            rgb[3 * p] = __uint_as_float(o[0]);
            rgb[3 * p + 1] = __uint_as_float(o[1]);
            rgb[3 * p + 2] = __uint_as_float(o[2]);
        }
    }
    __syncthreads();
    fence_after();
    if (ty == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(*slot));
}

// Host: bf16 of an f32, round to nearest even (finite values)
static uint16_t host_bf16(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
static float host_bf16_value(uint16_t h) {
    uint32_t u = (uint32_t)h << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// Host: the tensor-core scan's B operands in their shared-memory layout.
static void build_base81_tc(const Stock& st, Base81TC* hp) {
    std::memset(hp, 0, sizeof(*hp));
    hp->B = st.base;
    hp->X = st.expose;
    for (int k = 0; k <= 2 * HAL_R + 1; k++)
        hp->tap2[k] = make_float2(k <= 2 * HAL_R ? st.hal_taps[k] : 0.0f, k >= 1 ? st.hal_taps[k - 1] : 0.0f);
    const ScanSpec81& S = st.scan81;
    auto put = [](uint32_t* words, uint32_t byte_off, uint16_t v) {
        reinterpret_cast<uint16_t*>(words)[byte_off / 2] = v;
    };
    for (int l = 0; l < NB81; l++)
        for (int e = 0; e < 3; e++) {
            const float ne = -S.eps[e][l];
            const uint16_t hi = host_bf16(ne), lo = host_bf16(ne - host_bf16_value(hi));
            // row l of B1 against A1's (Dh, Dl, Dh, Dl): (eh, eh, el, el)
            put(hp->T.b1, tc::cm_off(l, e, tc::SBO_K16), hi);
            put(hp->T.b1, tc::cm_off(l, 3 + e, tc::SBO_K16), hi);
            put(hp->T.b1, tc::cm_off(l, 6 + e, tc::SBO_K16), lo);
            put(hp->T.b1, tc::cm_off(l, 9 + e, tc::SBO_K16), lo);
        }
    for (int ch = 0; ch < 3; ch++)
        for (int l = 0; l < NB81; l++) {
            const float cv = S.C[l][ch];
            const uint16_t hi = host_bf16(cv), lo = host_bf16(cv - host_bf16_value(hi));
            put(hp->T.b2h, tc::cm_off(ch, l, tc::SBO_K96), hi);
            put(hp->T.b2l, tc::cm_off(ch, l, tc::SBO_K96), lo);
        }
}

// Host: the pair tables of the 81-bin scan and halation taps.
static void build_base81(const Stock& st, Base81* hp) {
    hp->B = st.base;
    hp->X = st.expose;
    const ScanSpec81& S = st.scan81;
    for (int e = 0; e < 3; e++) {
        for (int l = 0; l < NP81; l++) hp->P.ne[e][l] = make_float2(-S.eps[e][2 * l], -S.eps[e][2 * l + 1]);
        hp->P.ne_last[e] = -S.eps[e][NB81 - 1];
    }
    for (int ch = 0; ch < 3; ch++) {
        for (int l = 0; l < NP81; l++) hp->P.C2[ch][l] = make_float2(S.C[2 * l][ch], S.C[2 * l + 1][ch]);
        hp->P.C_last[ch] = S.C[NB81 - 1][ch];
    }
    for (int k = 0; k <= 2 * HAL_R + 1; k++)
        hp->tap2[k] = make_float2(k <= 2 * HAL_R ? st.hal_taps[k] : 0.0f, k >= 1 ? st.hal_taps[k - 1] : 0.0f);
}

// ---------------------------------------------------------------------------
// workspace (per device+stream, grows on demand)

StreamCache g_ws("film workspace");

int workspace(cudaStream_t s, size_t bytes, void** out) { return g_ws.get(s, bytes, out); }

int grid_for(size_t n) {
    size_t g = (n + 255) / 256, cap = (size_t)sm_count() * 8;
    return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

int grid_for_n(size_t n) { return grid_for(n); }

// Bump allocator over the workspace.
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

size_t ref_workspace_bytes(size_t n, int E) {
    // planes(E) + mask(E) + inh(E) + tmp(1) + noise(1) + spec copies + sums
    return (size_t)(3 * E + 2) * n * 4 + sizeof(RefSpec) + sizeof(ScanSpec16) + 64 * 1024;
}

// The reference model's stages (film/mod.rs:77-129), each on the stock's E
// planar layers; run_reference chains them, and the imops_film_* entry
// points expose them one by one.
//   expose: ACEScg RGB -> absorbed exposure per layer (exposure/mod.rs:45-137,
//     absorption.rs:24-108)
int stage_expose(const float* rgb, int W, int H, const Stock& st, float* planes, cudaStream_t s) {
    const size_t n = (size_t)W * H;
    expose_kernel<<<grid_for(n), 256, 0, s>>>(rgb, n, st.expose, planes, nullptr);
    note_launch();
    return IMOPS_OK;
}

//   halation: local scatter and the wide bounce of the deepest layer
//     (halation.rs:24-93); tmp, bounce: one plane each
int stage_halation(float* planes, int W, int H, const Stock& st, float* tmp, float* bounce, cudaStream_t s) {
    const RefSpec& R = st.ref;
    const int E = R.E;
    const size_t n = (size_t)W * H;
    Taps tp;
    int rc;
    if (R.sigma_local >= 1e-3f && R.local_mix > 0.0f) {
        if ((rc = taps_for(R.sigma_local, &tp))) return rc;
        for (int e = 0; e < E; e++)
            if ((rc = blur(planes + e * n, tmp, W, H, tp, EpiMix{planes + e * n, 1.0f - R.local_mix, R.local_mix}, s)))
                return rc;
    }
    if (R.sigma_wide >= 1e-3f) {
        if ((rc = taps_for(R.sigma_wide, &tp))) return rc;
        EpiBounce eb;
        eb.planes = planes;
        eb.n = n;
        eb.E = E;
        for (int e = 0; e < MAXE; e++) eb.gain[e] = R.hal_gain[e];
        // the bounce source is the deepest plane before the bounce is added
        IMOPS_CUDA_TRY(cudaMemcpyAsync(bounce, planes + (E - 1) * n, n * 4, cudaMemcpyDeviceToDevice, s), "copy");
        if ((rc = blur(bounce, tmp, W, H, tp, eb, s))) return rc;
    }
    return IMOPS_OK;
}

//   develop: capture LUT + reciprocity + reduction to image-dye and mask
//     densities, DIR inhibition, adjacency (capture.rs:61-88,
//     reduction.rs:16-68, diffusion.rs:11-84); inh: E planes, tmp: one
int stage_develop(float* planes, float* mask, int W, int H, const Stock& st, const RefSpec* dR, float* inh,
                  float* tmp, cudaStream_t s) {
    const RefSpec& R = st.ref;
    const int E = R.E;
    const size_t n = (size_t)W * H;
    const int g = grid_for(n);
    Taps tp;
    int rc;
    lut_reduce_kernel<<<g, 256, 0, s>>>(planes, mask, n, E, dR);
    note_launch();
    if (R.dir_any && R.sigma_dir >= 1e-3f) {
        if ((rc = taps_for(R.sigma_dir, &tp))) return rc;
        for (int i = 0; i < E; i++)
            if ((rc = blur(planes + i * n, tmp, W, H, tp, EpiStore{inh + i * n}, s))) return rc;
        dir_apply_kernel<<<g, 256, 0, s>>>(planes, inh, n, E, dR);
        note_launch();
    }
    if (!(fabsf(R.beta) < 1e-8f || R.sigma_adj < 1e-3f)) {
        if ((rc = taps_for(R.sigma_adj, &tp))) return rc;
        for (int e = 0; e < E; e++)
            if ((rc = blur(planes + e * n, tmp, W, H, tp, EpiAdjacency{planes + e * n, R.beta}, s))) return rc;
    }
    return IMOPS_OK;
}

//   grain: seeded SplitMix64 fields, normalised and scaled per layer
//     (grain.rs:53-100); noise: one plane, partial: grain_partials(W, H, 1)
//     doubles, sums: MAXE doubles
int stage_grain(float* planes, int W, int H, const Stock& st, uint64_t seed, float* noise, double* partial,
                double* sums, cudaStream_t s) {
    const RefSpec& R = st.ref;
    const size_t n = (size_t)W * H;
    Taps tp;
    int rc;
    if ((rc = taps_for(fmaxf(R.sigma_grain, 1.0f), &tp))) return rc;
    IMOPS_CUDA_TRY(cudaMemsetAsync(sums, 0, MAXE * sizeof(double), s), "memset");
    for (int e = 0; e < R.E; e++) {
        if (R.kappa[e] <= 0.0f || R.dmax[e] <= 0.0f) continue;
        if ((rc = grain_fields(noise, W, H, seed, e, 1, tp, partial, sums + e, s))) return rc;
        grain_apply_kernel<<<grid_for(n), 256, 0, s>>>(planes + e * n, noise, n, sums + e, R.kappa[e], R.dmax[e]);
        note_launch();
    }
    return IMOPS_OK;
}

//   scan: densities -> ACEScg RGB of the scanned negative (scan/mod.rs:24-30,
//     densitometry.rs:13-73)
int stage_scan(const float* planes, const float* mask, int W, int H, const ScanSpec16* dC, float* rgb,
               cudaStream_t s) {
    const size_t n = (size_t)W * H;
    scan16_kernel<<<grid_for(n), 256, 0, s>>>(planes, mask, n, dC, rgb);
    note_launch();
    return IMOPS_OK;
}

// expose -> halation -> develop -> grain -> scan for the reference model;
// rgb in, rgb out.
int run_reference(float* rgb, int W, int H, const Stock& st, uint64_t seed, int grain, Arena& A, const RefSpec* dR,
                  const ScanSpec16* dC, cudaStream_t s) {
    const int E = st.ref.E;
    const size_t n = (size_t)W * H;
    float* planes = A.take<float>(E * n);
    float* mask = A.take<float>(E * n);
    float* inh = A.take<float>(E * n);
    float* tmp = A.take<float>(n);
    float* noise = A.take<float>(n);
    double* sums = A.take<double>(MAXE);
    int rc;
    if ((rc = stage_expose(rgb, W, H, st, planes, s))) return rc;
    if ((rc = stage_halation(planes, W, H, st, tmp, noise, s))) return rc;
    if ((rc = stage_develop(planes, mask, W, H, st, dR, inh, tmp, s))) return rc;
    // the inhibition planes are free after develop: they hold the grain's block sums
    if (grain && (rc = stage_grain(planes, W, H, st, seed, noise, reinterpret_cast<double*>(inh), sums, s)))
        return rc;
    if ((rc = stage_scan(planes, mask, W, H, dC, rgb, s))) return rc;
    IMOPS_CUDA_TRY(cudaGetLastError(), "film kernels");
    return IMOPS_OK;
}

// PositiveLinear's reference points (film/mod.rs:136-151): the mean RGB of
// a 32x32 mid-grey patch through the same path (seed 0) into mid_dmin[0..2]
// and the stock's normalised Dmin into mid_dmin[3..5].  Takes
// ref_workspace_bytes(1024, E) + 1024 * 12 bytes of A.
int mid_gray_negative(const Stock& st, int grain, Arena& A, const RefSpec* dR, const ScanSpec16* dC, float* mid_dmin,
                      cudaStream_t s) {
    const size_t nm = 32 * 32;
    float g = relative_to_absolute_y(0.185f, st.ref.box_iso);
    std::vector<float> patch(nm * 3, g);
    float* dpatch = A.take<float>(nm * 3);
    IMOPS_CUDA_TRY(cudaMemcpyAsync(dpatch, patch.data(), nm * 12, cudaMemcpyHostToDevice, s), "copy patch");
    int rc;
    if ((rc = run_reference(dpatch, 32, 32, st, 0, grain, A, dR, dC, s))) return rc;
    mean_rgb_kernel<<<1, 256, 0, s>>>(dpatch, (int)nm, mid_dmin);
    note_launch();
    IMOPS_CUDA_TRY(cudaMemcpyAsync(mid_dmin + 3, st.ref.dmin_norm, 12, cudaMemcpyHostToDevice, s), "copy dmin");
    return IMOPS_OK;
}

int process_reference(float* rgb, int W, int H, const ImopsFilmParams& P, cudaStream_t s) {
    Stock st;
    float pitch = 0;
    int rc = build_stock(P.stock, P.film_format, W, P.shutter_seconds, nullptr, &st, &pitch);
    if (rc) return rc;
    const size_t n = (size_t)W * H;
    const size_t nm = 32 * 32;
    size_t bytes = ref_workspace_bytes(n, st.ref.E) + ref_workspace_bytes(nm, st.ref.E) + nm * 12 + 4096;
    void* ws = nullptr;
    if ((rc = workspace(s, bytes, &ws))) return rc;
    Arena A{static_cast<char*>(ws), 0};
    RefSpec* dR = A.take<RefSpec>(1);
    ScanSpec16* dC = A.take<ScanSpec16>(1);
    float* mid_dmin = A.take<float>(8);
    IMOPS_CUDA_TRY(cudaMemcpyAsync(dR, &st.ref, sizeof(RefSpec), cudaMemcpyHostToDevice, s), "copy spec");
    IMOPS_CUDA_TRY(cudaMemcpyAsync(dC, &st.scan16, sizeof(ScanSpec16), cudaMemcpyHostToDevice, s), "copy spec");
    bool positive = P.output == IMOPS_FILM_POSITIVE_LINEAR && !st.ref.any_reversal;
    if (positive && (rc = mid_gray_negative(st, P.grain, A, dR, dC, mid_dmin, s))) return rc;
    if ((rc = run_reference(rgb, W, H, st, P.seed, P.grain, A, dR, dC, s))) return rc;
    if (positive) {
        invert_kernel<<<grid_for(n), 256, 0, s>>>(rgb, n, mid_dmin);
        note_launch();
    }
    IMOPS_CUDA_TRY(cudaGetLastError(), "film invert");
    return IMOPS_OK;
}

// One sub-stage call: the stock (reference model only), device copies of its
// specs and an arena of `extra` bytes in the film workspace.
struct StageCtx {
    Stock st;
    Arena A;
    RefSpec* dR;
    ScanSpec16* dC;
};

int stage_ctx(const ImopsFilmParams* P, int W, int H, size_t extra, cudaStream_t s, StageCtx* c) {
    if (!P) return fail(IMOPS_ERR_INVALID_ARGUMENT, "film stage: NULL params");
    if (W <= 0 || H <= 0) return fail(IMOPS_ERR_INVALID_DIMENSIONS, "invalid image dimensions");
    float pitch = 0;
    int rc = build_stock(P->stock, P->film_format, W, P->shutter_seconds, nullptr, &c->st, &pitch);
    if (rc) return rc;
    if (c->st.model != MODEL_REFERENCE)
        return fail(IMOPS_ERR_INVALID_STOCK, "film stages: the baseline preset runs only whole (imops_film_process)");
    void* ws = nullptr;
    if ((rc = workspace(s, sizeof(RefSpec) + sizeof(ScanSpec16) + extra + 4096, &ws))) return rc;
    c->A = Arena{static_cast<char*>(ws), 0};
    c->dR = c->A.take<RefSpec>(1);
    c->dC = c->A.take<ScanSpec16>(1);
    IMOPS_CUDA_TRY(cudaMemcpyAsync(c->dR, &c->st.ref, sizeof(RefSpec), cudaMemcpyHostToDevice, s), "copy spec");
    IMOPS_CUDA_TRY(cudaMemcpyAsync(c->dC, &c->st.scan16, sizeof(ScanSpec16), cudaMemcpyHostToDevice, s),
                   "copy spec");
    return IMOPS_OK;
}

}  // namespace film
}  // namespace imops

namespace imops {
namespace film {

// Bytes of the baseline preset's working set for a W x H image: the
// halation row pass, three grain fields, the grain's block sums (and the
// Arena's 256-byte alignment).  The layer exposures and the halation source
// are formed from the RGB where they are read.
size_t baseline_scratch_bytes(int W, int H) {
    const size_t n = (size_t)W * H;
    return (1 + 3) * n * 4 + grain_partials(W, H, 3) * 8 + 4096;
}

int baseline_stock(int W, const ImopsBaselineFilm& P, Stock* st) {
    if (P.scan != IMOPS_SCAN_FP32 && P.scan != IMOPS_SCAN_BF16_TC)
        return fail(IMOPS_ERR_INVALID_ARGUMENT, "film: unknown scan (IMOPS_SCAN_FP32 or IMOPS_SCAN_BF16_TC)");
    float pitch;
    return build_stock(IMOPS_STOCK_BASELINE81, 0, W, -1.0f, &P, st, &pitch);
}

// Baseline preset forward on an ACEScg image in place, with the working set
// in the library's per-(device, stream) workspace.
int baseline_forward_impl(float* rgb, int W, int H, const ImopsBaselineFilm* Pp, cudaStream_t s) {
    ImopsBaselineFilm P;
    if (Pp) P = *Pp;
    else imops_baseline_film_defaults(&P);
    Stock st;
    int rc = baseline_stock(W, P, &st);
    if (rc) return rc;
    void* ws = nullptr;
    if ((rc = workspace(s, baseline_scratch_bytes(W, H), &ws))) return rc;
    return baseline_forward_in(rgb, W, H, P, st, ws, s);
}

// The baseline preset's kernels with the working set at `scratch` (256-byte
// aligned, baseline_scratch_bytes(W, H) long).  Every byte the kernels read
// there is written earlier in the same call.
// A second stream per device for work that does not depend on the image
// (the grain fields), forked from and joined back to the caller's stream with
// events: the grain then runs beside the halation row pass.
struct SideStream {
    bool init = false;
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};
std::mutex g_side_mu;
SideStream g_side[64];

// the current device's side stream, created on first use; call with g_side_mu held
int side_stream(SideStream** out) {
    int dev = 0;
    IMOPS_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) return fail(IMOPS_ERR_INVALID_ARGUMENT, "film: device index above 63");
    SideStream& d = g_side[dev];
    if (!d.init) {
        cudaStream_t st = nullptr;
        cudaEvent_t f = nullptr, j = nullptr;
        cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&j, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            if (st) cudaStreamDestroy(st);
            if (f) cudaEventDestroy(f);
            if (j) cudaEventDestroy(j);
            return cuda_status(e, "film side stream");
        }
        d.side = st;
        d.fork = f;
        d.join = j;
        d.init = true;
    }
    *out = &d;
    return IMOPS_OK;
}

int baseline_forward_in(float* rgb, int W, int H, const ImopsBaselineFilm& P, const Stock& st, void* scratch,
                        cudaStream_t s) {
    int rc;
    const size_t n = (size_t)W * H;
    if (st.expose.E != 3 || !st.expose.hal_src)
        return fail(IMOPS_ERR_INVALID_STOCK, "film: the baseline preset's exposure is three layers with halation");
    Arena A{static_cast<char*>(scratch), 0};
    double* sums = A.take<double>(4);
    float* hr = A.take<float>(n);
    float* noise = A.take<float>(3 * n);
    double* gpart = A.take<double>(grain_partials(W, H, 3));
    Base81 hp;
    build_base81(st, &hp);
    if (P.grain_on && P.grain_sigma != 0.0f) {
        // grain fields on the side stream while the halation row pass runs on
        // s; the scan waits for both.  The lock keeps one call's
        // record / wait pairs of the shared events together.
        Taps tp;
        if ((rc = taps_for(fmaxf(P.grain_blur, 1.0f), &tp))) return rc;
        std::lock_guard<std::mutex> lock(g_side_mu);
        SideStream* ss = nullptr;
        if ((rc = side_stream(&ss))) return rc;
        IMOPS_CUDA_TRY(cudaEventRecord(ss->fork, s), "cudaEventRecord(film fork)");
        IMOPS_CUDA_TRY(cudaStreamWaitEvent(ss->side, ss->fork, 0), "cudaStreamWaitEvent(film fork)");
        if ((rc = grain_fields(noise, W, H, P.seed, 0, 3, tp, gpart, sums, ss->side))) return rc;
        IMOPS_CUDA_TRY(cudaEventRecord(ss->join, ss->side), "cudaEventRecord(film join)");
        if ((rc = blur_rows_halation(rgb, st.expose.hal_threshold, hr, W, H, st.hal_taps, s))) return rc;
        IMOPS_CUDA_TRY(cudaStreamWaitEvent(s, ss->join, 0), "cudaStreamWaitEvent(film join)");
    } else {
        if ((rc = blur_rows_halation(rgb, st.expose.hal_threshold, hr, W, H, st.hal_taps, s))) return rc;
    }
    dim3 cb(R64_COL_TW, R64_COL_GROUPS), cg((W + R64_COL_TW - 1) / R64_COL_TW, (H + R64_COL_TH - 1) / R64_COL_TH);
    if (P.scan == IMOPS_SCAN_BF16_TC) {
        Base81TC tp;
        build_base81_tc(st, &tp);
        IMOPS_CUDA_TRY(cudaFuncSetAttribute(scan81_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)tc::SMEM_REQ),
                       "cudaFuncSetAttribute(tensor-core scan)");
        scan81_tc_kernel<<<cg, cb, tc::SMEM_REQ, s>>>(hr, noise, sums, W, H, tp, rgb);
    } else {
        scan81_fused_kernel<<<cg, cb, 0, s>>>(hr, noise, sums, W, H, hp, rgb);
    }
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), "baseline film kernels");
    return IMOPS_OK;
}

}  // namespace film
}  // namespace imops


using namespace imops;

// ---- the reference model's sub-stages ----------------------------------------

extern "C" int imops_film_layers(const ImopsFilmParams* params, int* layers) {
    clear_error();
    if (!layers) return fail(IMOPS_ERR_INVALID_ARGUMENT, "film_layers: NULL output");
    film::StageCtx c;
    if (!params) return fail(IMOPS_ERR_INVALID_ARGUMENT, "film stage: NULL params");
    float pitch = 0;
    int rc = film::build_stock(params->stock, params->film_format, 1024, params->shutter_seconds, nullptr, &c.st,
                               &pitch);
    if (rc) return rc;
    if (c.st.model != film::MODEL_REFERENCE)
        return fail(IMOPS_ERR_INVALID_STOCK, "film stages: the baseline preset runs only whole (imops_film_process)");
    *layers = c.st.ref.E;
    return IMOPS_OK;
}

extern "C" int imops_film_expose(const float* rgb, int w, int h, const ImopsFilmParams* params, float* planes,
                                 imops_stream_t stream) {
    clear_error();
    cudaStream_t s = as_stream(stream);
    film::StageCtx c;
    int rc = film::stage_ctx(params, w, h, 0, s, &c);
    if (rc) return rc;
    if (!rgb || !planes) return fail(IMOPS_ERR_INVALID_ARGUMENT, "film_expose: NULL buffer");
    if ((rc = film::stage_expose(rgb, w, h, c.st, planes, s))) return rc;
    IMOPS_CUDA_TRY(cudaGetLastError(), "film_expose");
    return IMOPS_OK;
}

extern "C" int imops_film_halation(float* planes, int w, int h, const ImopsFilmParams* params,
                                   imops_stream_t stream) {
    clear_error();
    cudaStream_t s = as_stream(stream);
    const size_t n = (size_t)(w > 0 ? w : 0) * (h > 0 ? h : 0);
    film::StageCtx c;
    int rc = film::stage_ctx(params, w, h, 2 * n * 4 + 512, s, &c);
    if (rc) return rc;
    if (!planes) return fail(IMOPS_ERR_INVALID_ARGUMENT, "film_halation: NULL buffer");
    float* tmp = c.A.take<float>(n);
    float* bounce = c.A.take<float>(n);
    if ((rc = film::stage_halation(planes, w, h, c.st, tmp, bounce, s))) return rc;
    IMOPS_CUDA_TRY(cudaGetLastError(), "film_halation");
    return IMOPS_OK;
}

extern "C" int imops_film_develop(float* planes, float* mask, int w, int h, const ImopsFilmParams* params,
                                  imops_stream_t stream) {
    clear_error();
    cudaStream_t s = as_stream(stream);
    const size_t n = (size_t)(w > 0 ? w : 0) * (h > 0 ? h : 0);
    film::StageCtx c;
    int rc = film::stage_ctx(params, w, h, (size_t)(film::MAXE + 1) * n * 4 + 512, s, &c);
    if (rc) return rc;
    if (!planes || !mask) return fail(IMOPS_ERR_INVALID_ARGUMENT, "film_develop: NULL buffer");
    float* inh = c.A.take<float>((size_t)c.st.ref.E * n);
    float* tmp = c.A.take<float>(n);
    if ((rc = film::stage_develop(planes, mask, w, h, c.st, c.dR, inh, tmp, s))) return rc;
    IMOPS_CUDA_TRY(cudaGetLastError(), "film_develop");
    return IMOPS_OK;
}

extern "C" int imops_film_grain(float* planes, int w, int h, const ImopsFilmParams* params, imops_stream_t stream) {
    clear_error();
    cudaStream_t s = as_stream(stream);
    const size_t n = (size_t)(w > 0 ? w : 0) * (h > 0 ? h : 0);
    const size_t np = w > 0 && h > 0 ? film::grain_partials(w, h, 1) : 0;
    film::StageCtx c;
    int rc = film::stage_ctx(params, w, h, n * 4 + np * 8 + film::MAXE * 8 + 768, s, &c);
    if (rc) return rc;
    if (!planes) return fail(IMOPS_ERR_INVALID_ARGUMENT, "film_grain: NULL buffer");
    if (!params->grain) return IMOPS_OK;
    float* noise = c.A.take<float>(n);
    double* partial = c.A.take<double>(np);
    double* sums = c.A.take<double>(film::MAXE);
    if ((rc = film::stage_grain(planes, w, h, c.st, params->seed, noise, partial, sums, s))) return rc;
    IMOPS_CUDA_TRY(cudaGetLastError(), "film_grain");
    return IMOPS_OK;
}

extern "C" int imops_film_scan(const float* planes, const float* mask, int w, int h, const ImopsFilmParams* params,
                               float* rgb, imops_stream_t stream) {
    clear_error();
    cudaStream_t s = as_stream(stream);
    film::StageCtx c;
    int rc = film::stage_ctx(params, w, h, 0, s, &c);
    if (rc) return rc;
    if (!planes || !mask || !rgb) return fail(IMOPS_ERR_INVALID_ARGUMENT, "film_scan: NULL buffer");
    if ((rc = film::stage_scan(planes, mask, w, h, c.dC, rgb, s))) return rc;
    IMOPS_CUDA_TRY(cudaGetLastError(), "film_scan");
    return IMOPS_OK;
}

extern "C" int imops_film_invert(float* rgb, int w, int h, const ImopsFilmParams* params, imops_stream_t stream) {
    clear_error();
    cudaStream_t s = as_stream(stream);
    // the mid-grey patch's path and its reference points come from the same arena
    const size_t nm = 32 * 32;
    film::StageCtx c;
    int rc = film::stage_ctx(params, w, h, film::ref_workspace_bytes(nm, film::MAXE) + nm * 12 + 1024, s, &c);
    if (rc) return rc;
    if (!rgb) return fail(IMOPS_ERR_INVALID_ARGUMENT, "film_invert: NULL buffer");
    if (!(params->output == IMOPS_FILM_POSITIVE_LINEAR && !c.st.ref.any_reversal)) return IMOPS_OK;
    float* mid_dmin = c.A.take<float>(8);
    if ((rc = film::mid_gray_negative(c.st, params->grain, c.A, c.dR, c.dC, mid_dmin, s))) return rc;
    const size_t n = (size_t)w * h;
    film::invert_kernel<<<film::grid_for(n), 256, 0, s>>>(rgb, n, mid_dmin);
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), "film_invert");
    return IMOPS_OK;
}

extern "C" int imops_film_process(float* rgb, int w, int h, int color_space, const ImopsFilmParams* params,
                                  const ImopsBaselineFilm* baseline, imops_stream_t stream) {
    clear_error();
    if (!params) return fail(IMOPS_ERR_INVALID_ARGUMENT, "film: NULL params");
    if (color_space != IMOPS_CS_ACESCG)
        return fail(IMOPS_ERR_WRONG_COLOR_SPACE, "wrong color space: expected ACEScg");
    if (w <= 0 || h <= 0 || !rgb) return fail(IMOPS_ERR_INVALID_DIMENSIONS, "invalid image dimensions");
    cudaStream_t s = as_stream(stream);
    if (params->stock == IMOPS_STOCK_BASELINE81) {
        // without an explicit preset, the defaults with the module's grain seed
        ImopsBaselineFilm d;
        if (!baseline) {
            imops_baseline_film_defaults(&d);
            d.seed = params->seed;
            d.grain_on = params->grain;
            baseline = &d;
        }
        return film::baseline_forward_impl(rgb, w, h, baseline, s);
    }
    return film::process_reference(rgb, w, h, *params, s);
}

extern "C" int imops_tensor_timeouts(unsigned* count) {
    clear_error();
    if (!count) return fail(IMOPS_ERR_INVALID_ARGUMENT, "imops_tensor_timeouts: NULL output");
    IMOPS_CUDA_TRY(cudaMemcpyFromSymbol(count, film::g_tc_timeouts, sizeof(unsigned)), "read tensor-core timeouts");
    return IMOPS_OK;
}
