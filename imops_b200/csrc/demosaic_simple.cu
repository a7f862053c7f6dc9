// demosaic_simple.cu -- the reference's 3x3 same-colour mean ("Markesteijn",
// pichromatic/src/demosaic.rs:108-186) and the quad-sampling previews
// (Fast / SuperFast / SuperSuperFast, demosaic.rs:189-356).
//
// The mean is HBM-bound (4 B in, 12 B out per pixel): one thread per
// output pixel, a 32x8 block so each warp reads 34 consecutive floats of the
// three rows it needs (coalesced, re-read from L1), CFA colours from a
// kernel-parameter period table.  Built with --fmad=false: sums and the
// final division round exactly as the reference's f32 code.
#include "common.cuh"

namespace imops {
namespace simple {

// Cfa: CfaFixed<2, 2> / CfaFixed<6, 6> (modulo by a constant) for Bayer and
// X-Trans, CfaDev for other periods; coordinates here are never negative.
template <class Cfa>
__global__ void mean3x3_kernel(const float* __restrict__ in, int W, int H, const __grid_constant__ Cfa cfa,
                               float* __restrict__ out) {
    int col = blockIdx.x * blockDim.x + threadIdx.x;
    int row = blockIdx.y * blockDim.y + threadIdx.y;
    if (col >= W || row >= H) return;
    int centre = cfa.at(row, col);
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
        float* o = out + ((size_t)row * W + col) * 3;
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
    float v[3];
    v[0] = centre == 0 ? self : (n0 > 0.0f ? s0 / n0 : 0.0f);
    v[1] = centre == 1 ? self : (n1 > 0.0f ? s1 / n1 : 0.0f);
    v[2] = centre == 2 ? self : (n2 > 0.0f ? s2 / n2 : 0.0f);
    float* o = out + ((size_t)row * W + col) * 3;
    o[0] = v[0];
    o[1] = v[1];
    o[2] = v[2];
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
    if (!mosaic || !rgb) return fail(IMOPS_ERR_INVALID_ARGUMENT, "markesteijn: NULL buffer");
    if (w <= 0 || h <= 0) return fail(IMOPS_ERR_INVALID_ARGUMENT, "markesteijn: empty image");
    if (fault_injected("launch")) return fail(IMOPS_ERR_CUDA, "injected launch failure (markesteijn)");
    dim3 block(32, 8), grid((w + 31) / 32, (h + 7) / 8);
    cudaStream_t s = as_stream(stream);
    if (c.pw == 2 && c.ph == 2)
        simple::mean3x3_kernel<<<grid, block, 0, s>>>(mosaic, w, h, CfaFixed<2, 2>::from(c), rgb);
    else if (c.pw == 6 && c.ph == 6)
        simple::mean3x3_kernel<<<grid, block, 0, s>>>(mosaic, w, h, CfaFixed<6, 6>::from(c), rgb);
    else
        simple::mean3x3_kernel<<<grid, block, 0, s>>>(mosaic, w, h, c, rgb);
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), "markesteijn launch");
    return IMOPS_OK;
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
