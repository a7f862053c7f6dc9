// demosaic_simple.cu -- the reference's 3x3 same-colour mean ("Markesteijn",
// pichromatic/src/demosaic.rs:108-186) and the quad-sampling previews
// (Fast / SuperFast / SuperSuperFast, demosaic.rs:189-356).
//
// The mean is HBM-bound (4 B in, 12 B out per pixel).  Every Bayer CFA is a
// shift of RGGB and every X-Trans sensor's CFA a shift of one 6x6 pattern, so
// for those the kernel aligns each thread's run of pixels with the pattern:
// the colour of every site in a run's window is then a compile-time constant
// (per row phase, and a warp handles one row), the per-colour sums are plain
// adds and the counts constants.  Other CFAs take the per-pixel kernel.  Both
// sum each colour's sites in row-major order and divide once, as the
// reference's f32 code does; built with --fmad=false.
#include "color.cuh"
#include "common.cuh"
#include "demosaic_simple.cuh"

namespace imops {
namespace simple {

// One output pixel: the mean of each colour's sites among the 8 neighbours
// (the window clamped at the image edges), the centre's own colour keeping
// the centre sample.  Cfa: CfaFixed<2, 2> / CfaFixed<6, 6> for Bayer and
// X-Trans, CfaDev for other periods; coordinates here are never negative.
template <class Cfa>
__device__ __forceinline__ void mean_px(const float* __restrict__ in, int W, int H, const Cfa& cfa, int row,
                                        int col, float* o) {
    const int centre = cfa.at(row, col);
    if (row >= 1 && row + 1 < H && col >= 1 && col + 1 < W) {
        // interior: the whole 3x3 window, unrolled and branch-free; each
        // colour's sum takes its sites in row-major order (predicated adds)
        const float* p = in + (size_t)(row - 1) * W + (col - 1);
        float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f, n0 = 0.0f, n1 = 0.0f, n2 = 0.0f;
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) {
                if (a == 1 && b == 1) continue;
                const int k = cfa.at(row + a - 1, col + b - 1);
                const float v = __ldg(p + (size_t)a * W + b);
                s0 = k == 0 ? s0 + v : s0;
                n0 = k == 0 ? n0 + 1.0f : n0;
                s1 = k == 1 ? s1 + v : s1;
                n1 = k == 1 ? n1 + 1.0f : n1;
                s2 = k == 2 ? s2 + v : s2;
                n2 = k == 2 ? n2 + 1.0f : n2;
            }
        const float self = __ldg(in + (size_t)row * W + col);
        o[0] = centre == 0 ? self : (n0 > 0.0f ? s0 / n0 : 0.0f);
        o[1] = centre == 1 ? self : (n1 > 0.0f ? s1 / n1 : 0.0f);
        o[2] = centre == 2 ? self : (n2 > 0.0f ? s2 / n2 : 0.0f);
        return;
    }
    int y0 = row > 0 ? row - 1 : 0, y1 = row + 1 < H - 1 ? row + 1 : H - 1;
    int x0 = col > 0 ? col - 1 : 0, x1 = col + 1 < W - 1 ? col + 1 : W - 1;
    // one row-major pass over the window: each colour's sum takes its sites
    // in the order of the reference's per-colour loops
    float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f, n0 = 0.0f, n1 = 0.0f, n2 = 0.0f;
    for (int ny = y0; ny <= y1; ny++)
        for (int nx = x0; nx <= x1; nx++) {
            if (ny == row && nx == col) continue;
            const int k = cfa.at(ny, nx);
            const float v = __ldg(in + (size_t)ny * W + nx);
            if (k == 0) {
                s0 += v;
                n0 += 1.0f;
            } else if (k == 1) {
                s1 += v;
                n1 += 1.0f;
            } else if (k == 2) {
                s2 += v;
                n2 += 1.0f;
            }
        }
    const float self = __ldg(in + (size_t)row * W + col);
    o[0] = centre == 0 ? self : (n0 > 0.0f ? s0 / n0 : 0.0f);
    o[1] = centre == 1 ? self : (n1 > 0.0f ? s1 / n1 : 0.0f);
    o[2] = centre == 2 ? self : (n2 > 0.0f ? s2 / n2 : 0.0f);
}

// The mean alone.
struct NoEpilogue {
    __device__ __forceinline__ void apply(float&, float&, float&) const {}
};

// One thread per output pixel, for CFAs that are no shift of a canonical
// pattern; epi (NoEpilogue or color::Epilogue) maps each pixel's RGB before
// the store.
template <class Cfa, class Epi>
__global__ void mean3x3_kernel(const float* __restrict__ in, int W, int H, const __grid_constant__ Cfa cfa,
                               const __grid_constant__ Epi epi, float* __restrict__ out) {
    int col = blockIdx.x * blockDim.x + threadIdx.x;
    int row = blockIdx.y * blockDim.y + threadIdx.y;
    if (col >= W || row >= H) return;
    float v[3];
    mean_px(in, W, H, cfa, row, col, v);
    epi.apply(v[0], v[1], v[2]);
    float* o = out + ((size_t)row * W + col) * 3;
    o[0] = v[0];
    o[1] = v[1];
    o[2] = v[2];
}

// Canonical patterns, colour codes as parse_cfa assigns them (R 0, G 1, B 2),
// two bits a cell, packed at compile time.
__host__ __device__ constexpr int colour_code(char ch) { return ch == 'R' ? 0 : ch == 'G' ? 1 : 2; }
__host__ __device__ constexpr unsigned long long pack2(const char* p, int from, int n) {
    unsigned long long v = 0ull;
    for (int i = 0; i < n; i++) v |= (unsigned long long)colour_code(p[from + i]) << (2 * i);
    return v;
}
struct BayerCanon {  // RGGB
    static constexpr int PW = 2, PH = 2;
    static constexpr unsigned long long LO = pack2("RGGB", 0, 4), HI = 0ull;
    __host__ __device__ static constexpr int at(int r, int c) {
        return (int)((r * PW + c < 18 ? LO >> (2 * (r * PW + c)) : HI >> (2 * (r * PW + c - 18))) & 3ull);
    }
};
struct XTransCanon {  // the X-Trans sensors' 6x6 period
    static constexpr int PW = 6, PH = 6;
    static constexpr unsigned long long LO = pack2("GGRGGBGGBGGRBRGRBG", 0, 18);
    static constexpr unsigned long long HI = pack2("GGBGGRGGRGGBRBGBRG", 0, 18);
    __host__ __device__ static constexpr int at(int r, int c) {
        return (int)((r * PW + c < 18 ? LO >> (2 * (r * PW + c)) : HI >> (2 * (r * PW + c - 18))) & 3ull);
    }
};

// Phase-aligned kernel geometry: a warp handles one image row, RUN pixels a
// lane, 32 * RUN pixels a warp; RUN is a multiple of both periods.
constexpr int RUN = 6;
constexpr int WARP_PX = 32 * RUN;              // 192
constexpr int IN_STRIDE = WARP_PX + 4;         // 194 staged columns, padded to a 16-byte multiple
constexpr int OUT_STRIDE = 3 * WARP_PX + 4;    // an RGB row and up to 3 floats of alignment offset
constexpr int MEAN_WARPS = 8;

// The RUN pixels of one lane at canonical row phase RP: window v = rows
// y-1..y+1, columns x0-1..x0+RUN; pixel j sits at canonical column j mod PW.
// Same adds in the same order as mean_px's interior branch, with the colour
// tests and counts folded away.
template <class P, int RP>
__device__ __forceinline__ void run_aligned(const float (&v)[3][RUN + 2], float* o) {
#pragma unroll
    for (int j = 0; j < RUN; j++) {
        float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f, n0 = 0.0f, n1 = 0.0f, n2 = 0.0f;
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) {
                if (a == 1 && b == 1) continue;
                const int k = P::at((RP + a + P::PH - 1) % P::PH, (j + b + P::PW - 1) % P::PW);
                const float x = v[a][j + b];
                if (k == 0) {
                    s0 = s0 + x;
                    n0 = n0 + 1.0f;
                } else if (k == 1) {
                    s1 = s1 + x;
                    n1 = n1 + 1.0f;
                } else {
                    s2 = s2 + x;
                    n2 = n2 + 1.0f;
                }
            }
        const int centre = P::at(RP, j % P::PW);
        const float self = v[1][j + 1];
        o[3 * j + 0] = centre == 0 ? self : (n0 > 0.0f ? s0 / n0 : 0.0f);
        o[3 * j + 1] = centre == 1 ? self : (n1 > 0.0f ? s1 / n1 : 0.0f);
        o[3 * j + 2] = centre == 2 ? self : (n2 > 0.0f ? s2 / n2 : 0.0f);
    }
}

template <class P, int RP>
__device__ __forceinline__ void run_phase(int rp, const float (&v)[3][RUN + 2], float* o) {
    if constexpr (RP < P::PH) {
        if (rp == RP) run_aligned<P, RP>(v, o);
        else run_phase<P, RP + 1>(rp, v, o);
    }
}

// The CFA is P shifted: colour(y, x) = P::at((y - oy) mod PH, (x - ox) mod PW)
// with 0 <= ox < PW, 0 <= oy < PH.  Warp w of block (bx, by) develops row
// y = 8 by + w, pixels x_start + 192 bx .. + 191 with x_start = 0 when
// ox == 0 else ox - PW, so every lane's run starts at canonical column 0.
// The warp stages its three rows in shared memory (coalesced loads), each
// lane computes its run from there -- or, when the run or its window touches
// the image edge, each pixel with mean_px -- into a shared output row that
// the warp then stores coalesced.
template <class P, class Epi>
__global__ void __launch_bounds__(32 * MEAN_WARPS) mean3x3_aligned_kernel(
    const float* __restrict__ in, int W, int H, int ox, int oy, const __grid_constant__ CfaFixed<P::PW, P::PH> cfa,
    const __grid_constant__ Epi epi, float* __restrict__ out) {
    __shared__ __align__(16) float sin_[MEAN_WARPS][3][IN_STRIDE];
    __shared__ __align__(16) float sout[MEAN_WARPS][OUT_STRIDE];
    const int lane = threadIdx.x, w = threadIdx.y;
    const int y = blockIdx.y * MEAN_WARPS + w;
    if (y >= H) return;  // whole warp: only warp-level synchronisation below
    const int xs = ox == 0 ? 0 : ox - P::PW;
    const int xw = xs + blockIdx.x * WARP_PX;  // first pixel of the warp
    // stage rows y-1..y+1, columns xw-1 .. xw+192 (zeros outside the image;
    // only runs whose window lies inside read them).  All 21 loads of a lane
    // are issued before the first store, so a warp keeps them in flight
    // together; warps whose rows lie inside the image skip the per-element
    // tests.
    constexpr int NQ = (WARP_PX + 2 + 31) / 32;
    float t[3][NQ];
    if (y >= 1 && y + 1 < H && xw >= 1 && xw + WARP_PX + 1 <= W) {
        const float* src = in + (size_t)(y - 1) * W + (xw - 1) + lane;
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int q = 0; q < NQ; q++)
                t[a][q] = lane + 32 * q < WARP_PX + 2 ? __ldg(src + (size_t)a * W + 32 * q) : 0.0f;
    } else {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const int yy = y + a - 1;
            const bool yin = yy >= 0 && yy < H;
            const float* src = in + (size_t)(yin ? yy : 0) * W;
#pragma unroll
            for (int q = 0; q < NQ; q++) {
                const int i = lane + 32 * q, x = xw - 1 + i;
                t[a][q] = yin && i < WARP_PX + 2 && x >= 0 && x < W ? __ldg(src + x) : 0.0f;
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int q = 0; q < NQ; q++)
            if (lane + 32 * q < WARP_PX + 2) sin_[w][a][lane + 32 * q] = t[a][q];
    __syncwarp();
    // the warp's pixels inside the image, and the shared output row's offset
    // m: float k of the row goes to address dst0 + (k - K0), and m makes
    // shared and global 16-byte boundaries coincide
    const int p0 = xw > 0 ? xw : 0, p1 = xw + WARP_PX < W ? xw + WARP_PX : W;
    float* dst0 = out + ((size_t)y * W + p0) * 3;
    const int m = ((int)(((uintptr_t)dst0 >> 2) & 3) - 3 * (p0 - xw)) & 3;
    const int x0 = xw + RUN * lane;
    float* o = &sout[w][m + 3 * RUN * lane];
    if (y >= 1 && y + 1 < H && x0 >= 1 && x0 + RUN + 1 <= W) {
        float v[3][RUN + 2];
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int c = 0; c < RUN + 2; c += 2) {
                const float2 t2 = *reinterpret_cast<const float2*>(&sin_[w][a][RUN * lane + c]);
                v[a][c] = t2.x;
                v[a][c + 1] = t2.y;
            }
        const int rp = (y + P::PH - oy) % P::PH;
        float r[3 * RUN];
        run_phase<P, 0>(rp, v, r);
#pragma unroll
        for (int j = 0; j < RUN; j++) epi.apply(r[3 * j], r[3 * j + 1], r[3 * j + 2]);
        if (m & 1) {
#pragma unroll
            for (int c = 0; c < 3 * RUN; c++) o[c] = r[c];
        } else {
#pragma unroll
            for (int c = 0; c < 3 * RUN; c += 2) *reinterpret_cast<float2*>(o + c) = make_float2(r[c], r[c + 1]);
        }
    } else {
        for (int j = 0; j < RUN; j++) {
            const int x = x0 + j;
            if (x >= 0 && x < W) {
                float q[3];
                mean_px(in, W, H, cfa, y, x, q);
                epi.apply(q[0], q[1], q[2]);
                o[3 * j] = q[0];
                o[3 * j + 1] = q[1];
                o[3 * j + 2] = q[2];
            }
        }
    }
    __syncwarp();
    if (p1 <= p0) return;
    // shared floats K0..K1-1 -> dst0: a scalar head up to a 16-byte boundary,
    // float4 chunks, a scalar tail
    const int K0 = m + 3 * (p0 - xw), K1 = m + 3 * (p1 - xw);
    const int c0 = (K0 + 3) >> 2, c1 = K1 >> 2;
    const float* so = sout[w];
    if (c0 >= c1) {
        for (int k = K0 + lane; k < K1; k += 32) dst0[k - K0] = so[k];
        return;
    }
    if (K0 + lane < 4 * c0) dst0[lane] = so[K0 + lane];
    for (int c = c0 + lane; c < c1; c += 32)
        *reinterpret_cast<float4*>(dst0 + (4 * c - K0)) = *reinterpret_cast<const float4*>(so + 4 * c);
    if (4 * c1 + lane < K1) dst0[4 * c1 + lane - K0] = so[4 * c1 + lane];
}

// (ox, oy) with colour(y, x) == P::at((y - oy) mod PH, (x - ox) mod PW) for
// every site of c's period, or false when c is no shift of P.
template <class P>
bool canonical_offset(const CfaDev& c, int* ox, int* oy) {
    if (c.pw != P::PW || c.ph != P::PH) return false;
    for (int dy = 0; dy < P::PH; dy++)
        for (int dx = 0; dx < P::PW; dx++) {
            bool ok = true;
            for (int r = 0; r < P::PH && ok; r++)
                for (int q = 0; q < P::PW && ok; q++)
                    ok = c.col[r * P::PW + q] == P::at((r - dy + P::PH) % P::PH, (q - dx + P::PW) % P::PW);
            if (ok) {
                *ox = dx;
                *oy = dy;
                return true;
            }
        }
    return false;
}

template <class P, class Epi>
void launch_aligned(const float* mosaic, int w, int h, const CfaDev& c, int ox, int oy, const Epi& epi, float* rgb,
                    cudaStream_t s) {
    const int xs = ox == 0 ? 0 : ox - P::PW;
    dim3 block(32, MEAN_WARPS), grid((w - xs + WARP_PX - 1) / WARP_PX, (h + MEAN_WARPS - 1) / MEAN_WARPS);
    mean3x3_aligned_kernel<P, Epi><<<grid, block, 0, s>>>(mosaic, w, h, ox, oy, CfaFixed<P::PW, P::PH>::from(c), epi,
                                                          rgb);
}

template <class Epi>
void launch_mean(const float* mosaic, int w, int h, const CfaDev& c, const Epi& epi, float* rgb, cudaStream_t s) {
    dim3 block(32, 8), grid((w + 31) / 32, (h + 7) / 8);
    int ox, oy;
    if (canonical_offset<BayerCanon>(c, &ox, &oy))
        launch_aligned<BayerCanon>(mosaic, w, h, c, ox, oy, epi, rgb, s);
    else if (canonical_offset<XTransCanon>(c, &ox, &oy))
        launch_aligned<XTransCanon>(mosaic, w, h, c, ox, oy, epi, rgb, s);
    else if (c.pw == 2 && c.ph == 2)
        mean3x3_kernel<<<grid, block, 0, s>>>(mosaic, w, h, CfaFixed<2, 2>::from(c), epi, rgb);
    else if (c.pw == 6 && c.ph == 6)
        mean3x3_kernel<<<grid, block, 0, s>>>(mosaic, w, h, CfaFixed<6, 6>::from(c), epi, rgb);
    else
        mean3x3_kernel<<<grid, block, 0, s>>>(mosaic, w, h, c, epi, rgb);
}

int mean3x3(const float* mosaic, int w, int h, const CfaDev& c, const color::Epilogue* epi, float* rgb,
            cudaStream_t s) {
    if (!mosaic || !rgb) return fail(IMOPS_ERR_INVALID_ARGUMENT, "markesteijn: NULL buffer");
    if (((uintptr_t)mosaic | (uintptr_t)rgb) & 3)
        return fail(IMOPS_ERR_INVALID_ARGUMENT, "markesteijn: buffers must be 4-byte aligned float arrays");
    if (w <= 0 || h <= 0) return fail(IMOPS_ERR_INVALID_ARGUMENT, "markesteijn: empty image");
    if (fault_injected("launch")) return fail(IMOPS_ERR_CUDA, "injected launch failure (markesteijn)");
    if (epi) launch_mean(mosaic, w, h, c, *epi, rgb, s);
    else launch_mean(mosaic, w, h, c, NoEpilogue{}, rgb, s);
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), "markesteijn launch");
    return IMOPS_OK;
}

__global__ void quad_kernel(const float* __restrict__ in, int W, int nw, int nh, int factor, int4 cols,
                            float* __restrict__ out) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= nw || y >= nh) return;
    size_t tl = (size_t)(y * factor) * W + (size_t)(x * factor);
    float v[3] = {0.0f, 0.0f, 0.0f};
    v[cols.x] = in[tl];
    v[cols.y] = in[tl + 1];
    v[cols.z] = in[tl + W];
    v[cols.w] = in[tl + W + 1];
    float* o = out + ((size_t)y * nw + x) * 3;
    o[0] = v[0];
    o[1] = v[1];
    o[2] = v[2];
}

}  // namespace simple
}  // namespace imops

extern "C" int imops_demosaic_markesteijn(const float* mosaic, int w, int h, const char* cfa, int shift_x,
                                          int shift_y, float* rgb, imops_stream_t stream) {
    using namespace imops;
    clear_error();
    CfaDev c;
    int rc = parse_cfa(cfa, shift_x, shift_y, &c);
    if (rc) return rc;
    return simple::mean3x3(mosaic, w, h, c, nullptr, rgb, as_stream(stream));
}

extern "C" int imops_demosaic_quad(const float* mosaic, int w, int h, const char* cfa, int shift_x, int shift_y,
                                   int factor, float* rgb, imops_stream_t stream) {
    using namespace imops;
    clear_error();
    CfaDev c;
    int rc = parse_cfa(cfa, shift_x, shift_y, &c);
    if (rc) return rc;
    if (factor != 2 && factor != 4 && factor != 8)
        return fail(IMOPS_ERR_INVALID_ARGUMENT, "quad demosaic: factor must be 2, 4 or 8");
    if (!mosaic || !rgb) return fail(IMOPS_ERR_INVALID_ARGUMENT, "quad demosaic: NULL buffer");
    int nw = w / factor, nh = h / factor;
    int4 cols = make_int4(c.at(0, 0), c.at(0, 1), c.at(1, 0), c.at(1, 1));
    if (cols.x > 2 || cols.y > 2 || cols.z > 2 || cols.w > 2)
        return fail(IMOPS_ERR_UNSUPPORTED_CFA, "quad demosaic: CFA colour outside R/G/B");
    if (nw <= 0 || nh <= 0) return IMOPS_OK;
    dim3 block(32, 8), grid((nw + 31) / 32, (nh + 7) / 8);
    simple::quad_kernel<<<grid, block, 0, as_stream(stream)>>>(mosaic, w, nw, nh, factor, cols, rgb);
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), "quad demosaic launch");
    return IMOPS_OK;
}
