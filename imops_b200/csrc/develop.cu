// develop.cu -- the fused forward of the path: demosaic (scaling fused into
// its tile load, WB / exposure / camera CST fused into its output stage),
// then the film simulation.  Same results as the stage entry points run in
// the reference's module order (pipeline.rs:4-13).
#include <mutex>
#include <vector>

#include "amaze.cuh"
#include "color.cuh"
#include "demosaic_simple.cuh"

namespace imops {
namespace develop {

// small per-stream buffer for the Markesteijn path's scaled mosaic
StreamCache g_buf("mosaic buffer");

int mosaic_buffer(cudaStream_t s, size_t bytes, float** out) {
    void* p = nullptr;
    int rc = g_buf.get(s, bytes, &p);
    *out = static_cast<float*>(p);
    return rc;
}

int make_epilogue(const ImopsDevelopParams& P, color::Epilogue* e) {
    *e = color::identity_epilogue();
    for (int i = 0; i < 3; i++) e->wb[i] = P.wb[i];
    if (P.n_gain < 0 || P.n_gain > 2) return fail(IMOPS_ERR_INVALID_ARGUMENT, "develop: n_gain must be 0..2");
    e->n_gain = P.n_gain;
    for (int i = 0; i < P.n_gain; i++) e->gain[i] = color::exp_value(P.ev[i]);
    if (P.target != IMOPS_CS_CAMERA) {
        if (!color::xyz_to_target(P.target, e->tgt))
            return fail(IMOPS_ERR_INVALID_ARGUMENT, "develop: unsupported CST target");
        color::camera_forward_matrix(P.calib_d65, e->fwd);
        e->do_cst = 1;
        e->srgb = P.target == IMOPS_CS_SRGB;
    }
    if (P.film && P.target != IMOPS_CS_ACESCG)
        return fail(IMOPS_ERR_WRONG_COLOR_SPACE, "wrong color space: film expects ACEScg (CST target AcesCg)");
    return IMOPS_OK;
}

int finish(const ImopsDevelopParams& P, float* rgb, int w, int h, cudaStream_t s) {
    if (!P.film) return IMOPS_OK;
    return imops_film_process(rgb, w, h, IMOPS_CS_ACESCG, &P.film_params, &P.baseline, s);
}

}  // namespace develop
}  // namespace imops

using namespace imops;

extern "C" int imops_develop_u16(const uint16_t* raw, int raw_w, int raw_h, int crop_x, int crop_y, int crop_w,
                                 int crop_h, const float* black, const float* white, int period_w, int period_h,
                                 const ImopsDevelopParams* params, float* rgb, imops_stream_t stream) {
    clear_error();
    if (!params || !raw || !rgb || !black || !white) return fail(IMOPS_ERR_INVALID_ARGUMENT, "develop: NULL argument");
    const ImopsDevelopParams& P = *params;
    cudaStream_t s = as_stream(stream);
    color::Epilogue e;
    int rc = develop::make_epilogue(P, &e);
    if (rc) return rc;
    CfaDev cfa;
    if ((rc = parse_cfa(P.cfa, crop_x, crop_y, &cfa))) return rc;
    if (P.demosaic == IMOPS_DEMOSAIC_AMAZE) {
        rc = amaze::demosaic_color_u16(raw, raw_w, raw_h, crop_x, crop_y, crop_w, crop_h, black, white, period_w,
                                       period_h, cfa, P.clip_pt, e, rgb, s);
    } else if (P.demosaic == IMOPS_DEMOSAIC_MARKESTEIJN) {
        float* m = nullptr;
        if ((rc = develop::mosaic_buffer(s, (size_t)crop_w * crop_h * 4, &m))) return rc;
        if ((rc = imops_scale_u16(raw, raw_w, raw_h, crop_x, crop_y, crop_w, crop_h, black, white, period_w,
                                  period_h, m, stream)))
            return rc;
        // the 3x3 mean with the colour epilogue applied before its store
        if ((rc = simple::mean3x3(m, crop_w, crop_h, cfa, &e, rgb, s))) return rc;
    } else {
        return fail(IMOPS_ERR_INVALID_ARGUMENT, "develop: demosaic must be AMaZE or Markesteijn");
    }
    if (rc) return rc;
    return develop::finish(P, rgb, crop_w, crop_h, s);
}

extern "C" int imops_develop_f32(const float* mosaic, int w, int h, int shift_x, int shift_y,
                                 const ImopsDevelopParams* params, float* rgb, imops_stream_t stream) {
    clear_error();
    if (!params || !mosaic || !rgb) return fail(IMOPS_ERR_INVALID_ARGUMENT, "develop: NULL argument");
    const ImopsDevelopParams& P = *params;
    cudaStream_t s = as_stream(stream);
    color::Epilogue e;
    int rc = develop::make_epilogue(P, &e);
    if (rc) return rc;
    CfaDev cfa;
    if ((rc = parse_cfa(P.cfa, shift_x, shift_y, &cfa))) return rc;
    if (P.demosaic == IMOPS_DEMOSAIC_AMAZE) {
        rc = amaze::demosaic_color_f32(mosaic, w, h, cfa, P.clip_pt, e, rgb, s);
    } else if (P.demosaic == IMOPS_DEMOSAIC_MARKESTEIJN) {
        rc = simple::mean3x3(mosaic, w, h, cfa, &e, rgb, s);
    } else {
        return fail(IMOPS_ERR_INVALID_ARGUMENT, "develop: demosaic must be AMaZE or Markesteijn");
    }
    if (rc) return rc;
    return develop::finish(P, rgb, w, h, s);
}
