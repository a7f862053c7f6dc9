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

__global__ void mean3x3_kernel(const float* __restrict__ in, int W, int H, CfaDev cfa, float* __restrict__ out) {
    int col = blockIdx.x * blockDim.x + threadIdx.x;
    int row = blockIdx.y * blockDim.y + threadIdx.y;
    if (col >= W || row >= H) return;
    int y0 = row > 0 ? row - 1 : 0, y1 = row + 1 < H - 1 ? row + 1 : H - 1;
    int x0 = col > 0 ? col - 1 : 0, x1 = col + 1 < W - 1 ? col + 1 : W - 1;
    int centre = cfa.at(row, col);
    float v[3];
    for (int ch = 0; ch < 3; ch++) {
        if (ch == centre) {
            v[ch] = __ldg(in + (size_t)row * W + col);
            continue;
        }
        float sum = 0.0f, cnt = 0.0f;
        for (int ny = y0; ny <= y1; ny++)
            for (int nx = x0; nx <= x1; nx++) {
                if (ny == row && nx == col) continue;
                if (cfa.at(ny, nx) == ch) {
                    sum += __ldg(in + (size_t)ny * W + nx);
                    cnt += 1.0f;
                }
            }
        v[ch] = cnt > 0.0f ? sum / cnt : 0.0f;
    }
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
    simple::mean3x3_kernel<<<grid, block, 0, as_stream(stream)>>>(mosaic, w, h, c, rgb);
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
