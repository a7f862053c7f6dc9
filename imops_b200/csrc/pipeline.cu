// pipeline.cu -- the reference's pipeline layer on the GPU: a device-resident
// Image, the PipelineModule set of the hot path (pichromatic-pipeline/src/
// modules.rs), parse_config (config.rs:13-34) and the embedding C-ABI of
// extern_pipeline.rs.
//
// Module semantics follow modules.rs: Demosaic :629-668, CFACoeffs :529-557,
// Exp :295-329, BaselineExposureCompensation :335-373, CST :576-592,
// Film :841-876, LCH :221-261, HighlightReconstruction :265-293,
// SigmoidToneMap :392-415, Gamma :417-453, Contrast :455-489.  Where the
// reference panics (expect / panic!), the call returns NULL / an error code
// and the same message is kept for get_last_error_c.  Modules of the
// reference that are not part of this path (BM3D, ChromaDenoise,
// LumaGuidedChromaDenoise, Vignette) parse with the reference's field rules
// and return IMOPS_ERR_NOT_IMPLEMENTED when run.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "amaze.cuh"
#include "color.cuh"
#include "demosaic_simple.cuh"
#include "config.hpp"
#include "display.cuh"

namespace imops {
namespace pipe {

// ---- device memory and stream ---------------------------------------------

// Each image gets one of a few library-owned streams, round robin, so the
// frames a host submits one after another can overlap on the GPU (one
// frame's compute with the previous frame's download).  Six of them: an
// upload synchronises its image's stream, and with three a host streaming
// frames found the download of the frame three back still queued on it.
//
// Image buffers come from a memory pool of the library's own per device
// (the default pool, shared with the rest of the process, is left as it
// is).  It keeps freed memory (release threshold: never) and reuses it in
// stream order only: a buffer freed on a stream serves the next allocation on
// that stream, so an image reuses the buffers of the image that held its
// stream before it, with no wait on other streams and no growth of the pool
// that depends on timing.
constexpr int POOL_STREAMS = 6;
struct DevState {
    bool init = false;
    cudaStream_t streams[POOL_STREAMS] = {};
    cudaMemPool_t pool = nullptr;
    unsigned next = 0;
    // end of the last queued pipeline run's kernels (see order_compute)
    cudaEvent_t compute_done = nullptr;
    bool has_compute = false;
};
std::mutex g_dev_mu;
DevState g_dev[128];

// The current device's state, created on first use; call with g_dev_mu held.
int dev_state(DevState** out) {
    int dev = 0;
    IMOPS_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 128) return fail(IMOPS_ERR_INVALID_ARGUMENT, "device index above 127");
    DevState& d = g_dev[dev];
    if (!d.init) {
        // all or nothing: a failure leaves no stream or pool behind, and the
        // next call tries again
        cudaStream_t st[POOL_STREAMS] = {};
        cudaMemPool_t pool = nullptr;
        cudaError_t e = cudaSuccess;
        for (int i = 0; i < POOL_STREAMS && e == cudaSuccess; i++)
            e = cudaStreamCreateWithFlags(&st[i], cudaStreamNonBlocking);
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        if (e == cudaSuccess) e = cudaMemPoolCreate(&pool, &props);
        uint64_t keep = UINT64_MAX;
        int off = 0;
        if (e == cudaSuccess) e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e == cudaSuccess) e = cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowOpportunistic, &off);
        if (e == cudaSuccess) e = cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &off);
        cudaEvent_t ev = nullptr;
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            for (int i = 0; i < POOL_STREAMS; i++)
                if (st[i]) cudaStreamDestroy(st[i]);
            if (pool) cudaMemPoolDestroy(pool);
            if (ev) cudaEventDestroy(ev);
            return fail(IMOPS_ERR_CUDA, std::string("image streams / pool: ") + cudaGetErrorString(e));
        }
        for (int i = 0; i < POOL_STREAMS; i++) d.streams[i] = st[i];
        d.pool = pool;
        d.compute_done = ev;
        d.init = true;
    }
    *out = &d;
    return IMOPS_OK;
}

int device_stream(cudaStream_t* out) {
    std::lock_guard<std::mutex> lock(g_dev_mu);
    DevState* d = nullptr;
    int rc = dev_state(&d);
    if (rc) return rc;
    *out = d->streams[d->next++ % POOL_STREAMS];
    return IMOPS_OK;
}

// Pipeline runs on one device execute their kernels in the order they were
// queued: a run first makes its image's stream wait for the end of the run
// queued before it (on whatever stream), and marks its own end.  Images keep
// their own streams, so one frame's download still overlaps the next frame's
// kernels, but the kernels of frames submitted back to back do not share the
// SMs: each frame finishes one frame-time after the one before it instead of
// all finishing late together, which would leave the copy engines idle and
// then bunch their downloads.  Holds its own lock (g_order_mu, not the
// device lock the image buffers take) while the run is queued.
std::mutex g_order_mu;
struct ComputeOrder {
    std::unique_lock<std::mutex> lock;
    DevState* d = nullptr;
    cudaStream_t s = nullptr;
    ~ComputeOrder() {
        if (d) {
            cudaEventRecord(d->compute_done, s);
            d->has_compute = true;
        }
    }
};

int order_compute(cudaStream_t s, ComputeOrder* o) {
    o->lock = std::unique_lock<std::mutex>(g_order_mu);
    DevState* d = nullptr;
    {
        std::lock_guard<std::mutex> dl(g_dev_mu);
        int rc = dev_state(&d);
        if (rc) return rc;
    }
    if (d->has_compute) IMOPS_CUDA_TRY(cudaStreamWaitEvent(s, d->compute_done, 0), "cudaStreamWaitEvent(compute order)");
    o->d = d;
    o->s = s;
    return IMOPS_OK;
}

int image_pool(cudaMemPool_t* out) {
    std::lock_guard<std::mutex> lock(g_dev_mu);
    DevState* d = nullptr;
    int rc = dev_state(&d);
    if (rc) return rc;
    *out = d->pool;
    return IMOPS_OK;
}

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

int buf_alloc(DevBuf& b, size_t bytes, cudaStream_t s) {
    if (b.p && b.bytes >= bytes) return IMOPS_OK;
    if (fault_injected("alloc")) return fail(IMOPS_ERR_OUT_OF_MEMORY, "injected allocation failure (image buffer)");
    if (b.p) {
        cudaFreeAsync(b.p, s);
        b.p = nullptr;
        b.bytes = 0;
    }
    cudaMemPool_t pool = nullptr;
    int rc = image_pool(&pool);
    if (rc) return rc;
    IMOPS_CUDA_TRY(cudaMallocFromPoolAsync(&b.p, bytes, pool, s), "cudaMallocFromPoolAsync(image buffer)");
    b.bytes = bytes;
    return IMOPS_OK;
}

void buf_free(DevBuf& b, cudaStream_t s) {
    if (b.p) cudaFreeAsync(b.p, s);
    b.p = nullptr;
    b.bytes = 0;
}

}  // namespace pipe
}  // namespace imops

// ---- Image -------------------------------------------------------------------

struct ImopsImage {
    int dev = 0;
    cudaStream_t stream = nullptr;
    // raw data: either the u16 sensor frame (full, uncropped) or the f32 mosaic
    int raw_kind = 0;  // 0 none, 1 u16 frame, 2 f32 mosaic
    imops::pipe::DevBuf raw;
    size_t raw_w = 0, raw_h = 0;
    // rgb data
    imops::pipe::DevBuf rgb;
    bool has_rgb = false;
    size_t width = 0, height = 0;  // metadata.width/height (cropped size for raw images)
    int color_space = IMOPS_CS_CAMERA;
    bool has_cs = false;  // color_space == Some(..)
    ImopsImageMeta meta{};
    std::string cfa;
};

struct ImopsPipeline;

namespace imops {
namespace pipe {

using cfg::Value;

// ---- module parameters ------------------------------------------------------

// A Parameter<T> (modules.rs:10-66): a bare value or {value = ..., ...}.
const Value* param_value(const Value& table, const std::string& field) {
    const Value* v = table.get(field);
    if (!v) return nullptr;
    if (v->kind == Value::TABLE) return v->get("value");
    return v;
}

struct ParamError {
    std::string msg;
};

float get_f32(const Value& t, const std::string& mod, const std::string& f) {
    const Value* v = param_value(t, f);
    if (!v) throw ParamError{"Invalid " + mod + " config: missing field `" + f + "`"};
    if (!v->is_number()) throw ParamError{"Invalid " + mod + " config: field `" + f + "` must be a number"};
    return (float)v->number();
}

long long get_int(const Value& t, const std::string& mod, const std::string& f, bool non_negative) {
    const Value* v = param_value(t, f);
    if (!v) throw ParamError{"Invalid " + mod + " config: missing field `" + f + "`"};
    if (v->kind != Value::INT) throw ParamError{"Invalid " + mod + " config: field `" + f + "` must be an integer"};
    if (non_negative && v->i < 0) throw ParamError{"Invalid " + mod + " config: field `" + f + "` must be >= 0"};
    return v->i;
}

std::string get_str(const Value& t, const std::string& mod, const std::string& f) {
    const Value* v = param_value(t, f);
    if (!v) throw ParamError{"Invalid " + mod + " config: missing field `" + f + "`"};
    if (v->kind != Value::STRING) throw ParamError{"Invalid " + mod + " config: field `" + f + "` must be a string"};
    return v->s;
}

// ---- modules ------------------------------------------------------------------

struct Module {
    virtual ~Module() = default;
    virtual int process(ImopsImage& img) = 0;
};

std::string lower(std::string s) {
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

int cs_from_name(const std::string& name, int* cs, bool* known_elsewhere) {
    *known_elsewhere = false;
    if (name == "Srgb") *cs = IMOPS_CS_SRGB;
    else if (name == "LinearSrgb") *cs = IMOPS_CS_LINEAR_SRGB;
    else if (name == "AcesCg") *cs = IMOPS_CS_ACESCG;
    else if (name == "XyzD65") *cs = IMOPS_CS_XYZD65;
    else if (name == "Oklch") *cs = IMOPS_CS_OKLCH;
    else {
        static const char* others[] = {"Lab", "Lch", "Hsl", "Hwb", "Oklab", "DisplayP3", "A98Rgb",
                                       "ProphotoRgb", "Rec2020", "Aces2065_1", "XyzD50"};
        for (const char* o : others)
            if (name == o) *known_elsewhere = true;
        return 0;
    }
    return 1;
}

const char* cs_debug(const ImopsImage& img) {
    if (!img.has_cs) return "None";
    switch (img.color_space) {
        case IMOPS_CS_SRGB: return "Some(Srgb)";
        case IMOPS_CS_LINEAR_SRGB: return "Some(LinearSrgb)";
        case IMOPS_CS_ACESCG: return "Some(AcesCg)";
        case IMOPS_CS_XYZD65: return "Some(XyzD65)";
        case IMOPS_CS_OKLCH: return "Some(Oklch)";
    }
    return "Some(?)";
}

struct Demosaic : Module {
    int algorithm = IMOPS_DEMOSAIC_AMAZE;
    int process(ImopsImage& img) override { return process_fused(img, nullptr, IMOPS_CS_CAMERA); }
    // `fused`: the per-pixel modules run_pixel_pipeline_c folds into the
    // output stage of AMaZE or the 3x3 mean (nullptr: none), and the colour
    // space they leave.  Passed per call, so one pipeline object keeps no
    // per-image state.
    int process_fused(ImopsImage& img, const color::Epilogue* fused, int fused_cs) {
        if (img.raw_kind == 0) return fail(IMOPS_ERR_INVALID_ARGUMENT, "Demosaic: the image has no raw data");
        if (img.cfa.empty()) return fail(IMOPS_ERR_INVALID_ARGUMENT, "A CFA must be set to demosaic raw images");
        const int w = (int)img.width, h = (int)img.height;
        const int cx = img.meta.crop_x, cy = img.meta.crop_y;
        cudaStream_t s = img.stream;
        int rc;
        int ow = w, oh = h;
        if (algorithm >= IMOPS_DEMOSAIC_FAST) {
            int f = algorithm == IMOPS_DEMOSAIC_FAST ? 2 : (algorithm == IMOPS_DEMOSAIC_SUPERFAST ? 4 : 8);
            ow = w / f;
            oh = h / f;
        }
        DevBuf out;
        if ((rc = buf_alloc(out, std::max<size_t>((size_t)ow * oh * 12, 16), s))) return rc;
        float* rgb = static_cast<float*>(out.p);
        DevBuf tmp;
        const float* mosaic = nullptr;
        if (img.raw_kind == 2) {
            mosaic = static_cast<const float*>(img.raw.p);
        } else if (algorithm != IMOPS_DEMOSAIC_AMAZE) {
            if ((rc = buf_alloc(tmp, (size_t)w * h * 4, s))) return rc;
            float bl[1] = {img.meta.black_level}, wh[1] = {img.meta.white_level};
            if ((rc = imops_scale_u16(static_cast<const uint16_t*>(img.raw.p), (int)img.raw_w, (int)img.raw_h, cx, cy,
                                      w, h, bl, wh, 1, 1, static_cast<float*>(tmp.p), s)))
                return rc;
            mosaic = static_cast<const float*>(tmp.p);
        }
        if (algorithm == IMOPS_DEMOSAIC_AMAZE) {
            CfaDev c;
            if ((rc = parse_cfa(img.cfa.c_str(), cx, cy, &c))) return rc;
            const color::Epilogue e = fused ? *fused : color::identity_epilogue();
            if (img.raw_kind == 1) {
                float bl[1] = {img.meta.black_level}, wh[1] = {img.meta.white_level};
                rc = amaze::demosaic_color_u16(static_cast<const uint16_t*>(img.raw.p), (int)img.raw_w,
                                               (int)img.raw_h, cx, cy, w, h, bl, wh, 1, 1, c, 1.0f, e, rgb, s);
            } else {
                rc = amaze::demosaic_color_f32(mosaic, w, h, c, 1.0f, e, rgb, s);
            }
        } else if (algorithm == IMOPS_DEMOSAIC_MARKESTEIJN) {
            CfaDev c;
            rc = parse_cfa(img.cfa.c_str(), cx, cy, &c);
            if (!rc) rc = simple::mean3x3(mosaic, w, h, c, fused, rgb, s);
        } else {
            int f = algorithm == IMOPS_DEMOSAIC_FAST ? 2 : (algorithm == IMOPS_DEMOSAIC_SUPERFAST ? 4 : 8);
            rc = imops_demosaic_quad(mosaic, w, h, img.cfa.c_str(), cx, cy, f, rgb, s);
        }
        buf_free(tmp, s);
        if (rc) {
            buf_free(out, s);
            return rc;
        }
        buf_free(img.rgb, s);
        img.rgb = out;
        img.has_rgb = true;
        img.width = ow;
        img.height = oh;
        img.has_cs = fused_cs != IMOPS_CS_CAMERA;
        img.color_space = fused_cs;
        return IMOPS_OK;
    }
};

int need_rgb(const ImopsImage& img, const char* mod) {
    if (!img.has_rgb) return fail(IMOPS_ERR_INVALID_ARGUMENT, std::string(mod) + ": the image has no RGB data (run Demosaic first)");
    return IMOPS_OK;
}

// A per-pixel module: appends its ops to a chain (display.cuh) and updates
// the image's colour space.  run_pixel_pipeline_c runs each run of
// consecutive per-pixel modules as one chain, one pass over the image; the
// ops are each module's own f32 arithmetic in order, so the result is the
// same as one pass per module.
struct PixelModule : Module {
    // most ops this module appends
    virtual int max_ops() const { return 1; }
    virtual int add_ops(ImopsImage& img, display::Chain& c) = 0;
    int process(ImopsImage& img) override {
        display::Chain c{};
        int rc = add_ops(img, c);
        if (rc) return rc;
        return display::run(static_cast<float*>(img.rgb.p), img.width * img.height, c, img.stream, "pixel modules");
    }
};

struct CFACoeffs : PixelModule {
    int add_ops(ImopsImage& img, display::Chain& c) override {
        int rc = need_rgb(img, "CFACoeffs");
        if (rc) return rc;
        if (!img.meta.has_wb)
            return fail(IMOPS_ERR_INVALID_ARGUMENT, "wb_coeffs needs to be set to perform highlight_reconstruction");
        return display::add_gain(c, img.meta.wb_coeffs[0], img.meta.wb_coeffs[1], img.meta.wb_coeffs[2]);
    }
};

struct Exp : PixelModule {
    float ev = 0.0f;
    int add_ops(ImopsImage& img, display::Chain& c) override {
        int rc = need_rgb(img, "Exp");
        if (rc) return rc;
        float v = color::exp_value(ev);
        return display::add_gain(c, v, v, v);
    }
};

struct BaselineExposureCompensation : PixelModule {
    int max_ops() const override { return 2; }
    int add_ops(ImopsImage& img, display::Chain& c) override {
        int rc = need_rgb(img, "BaselineExposureCompensation");
        if (rc) return rc;
        const ImopsImageMeta& m = img.meta;
        float ev = m.has_baseline_exposure ? m.baseline_exposure : 0.0f;
        if (fabsf(ev) > 1e-6f) {
            float v = color::exp_value(ev);
            if ((rc = display::add_gain(c, v, v, v))) return rc;
        }
        bool ok = m.has_shutter && m.has_f_number && m.has_iso && m.shutter_seconds > 0.0f && m.f_number > 0.0f &&
                  m.iso > 0.0f;
        if (!ok) return IMOPS_OK;
        float g = color::luminance_gain(m.shutter_seconds, m.f_number, m.iso);
        return display::add_gain(c, g, g, g);
    }
};

struct CST : PixelModule {
    std::string target;
    int add_ops(ImopsImage& img, display::Chain& c) override {
        int rc = need_rgb(img, "CST");
        if (rc) return rc;
        std::string name = target;
        name.erase(0, name.find_first_not_of(" \t\r\n"));
        name.erase(name.find_last_not_of(" \t\r\n") + 1);
        int cs;
        bool elsewhere;
        if (!cs_from_name(name, &cs, &elsewhere)) {
            if (elsewhere)
                return fail(IMOPS_ERR_NOT_IMPLEMENTED, "CST to " + name +
                                                           " is not on the GPU path (Srgb, LinearSrgb, AcesCg, "
                                                           "XyzD65, Oklch are)");
            return fail(IMOPS_ERR_CONFIG, "Color space not recognized: " + target);
        }
        if (!img.has_cs) {
            if (!img.meta.has_calibration)
                return fail(IMOPS_ERR_INVALID_ARGUMENT,
                            "A calibration matrix must be set to perform a camera cst transform");
            float fwd[9];
            color::camera_forward_matrix(img.meta.calibration_matrix_d65, fwd);
            rc = display::add_cst(c, IMOPS_CS_CAMERA, cs, fwd);
        } else {
            rc = display::add_cst(c, img.color_space, cs, nullptr);
        }
        if (rc) return rc;
        img.has_cs = true;
        img.color_space = cs;
        return IMOPS_OK;
    }
};

struct HighlightReconstruction : PixelModule {
    int add_ops(ImopsImage& img, display::Chain& c) override {
        int rc = need_rgb(img, "HighlightReconstruction");
        if (rc) return rc;
        if (!img.meta.has_wb)
            return fail(IMOPS_ERR_INVALID_ARGUMENT, "wb_coeffs needs to be set to perform highlight_reconstruction");
        return display::add_highlight(c, img.meta.wb_coeffs[1]);
    }
};

struct Contrast : PixelModule {
    float value = 1.0f;
    int add_ops(ImopsImage& img, display::Chain& c) override {
        int rc = need_rgb(img, "Contrast");
        if (rc) return rc;
        return display::add_contrast(c, value);
    }
};

struct LCH : PixelModule {
    float lc = 1.0f, cc = 1.0f, hc = 1.0f;
    int max_ops() const override { return 3; }
    int add_ops(ImopsImage& img, display::Chain& c) override {
        int rc = need_rgb(img, "LCH");
        if (rc) return rc;
        // Image::lch unwraps metadata.color_space (pixel.rs:60-68)
        if (!img.has_cs) return fail(IMOPS_ERR_INVALID_ARGUMENT, "called `Option::unwrap()` on a `None` value");
        return display::add_lch(c, img.color_space, lc, cc, hc);
    }
};

struct SigmoidToneMap : PixelModule {
    int add_ops(ImopsImage& img, display::Chain& c) override {
        int rc = need_rgb(img, "SigmoidToneMap");
        if (rc) return rc;
        return display::add_sigmoid(c);
    }
};

struct Gamma : PixelModule {
    float gamma = 2.2f;
    int add_ops(ImopsImage& img, display::Chain& c) override {
        int rc = need_rgb(img, "Gamma");
        if (rc) return rc;
        return display::add_gamma(c, gamma);
    }
};

struct Film : Module {
    ImopsFilmParams p{};
    std::string stock_name;
    int process(ImopsImage& img) override {
        int rc = need_rgb(img, "Film");
        if (rc) return rc;
        if (!img.has_cs || img.color_space != IMOPS_CS_ACESCG)
            return fail(IMOPS_ERR_WRONG_COLOR_SPACE,
                        std::string("Film process failed: WrongColorSpace { expected: \"ACEScg\", got: \"") +
                            cs_debug(img) + "\" }");
        ImopsFilmParams q = p;
        q.shutter_seconds = img.meta.has_shutter ? img.meta.shutter_seconds : -1.0f;
        rc = imops_film_process(static_cast<float*>(img.rgb.p), (int)img.width, (int)img.height, IMOPS_CS_ACESCG, &q,
                                nullptr, img.stream);
        if (rc) {
            std::string m = last_error();
            return fail(rc, "Film process failed: " + m);
        }
        return IMOPS_OK;
    }
};

struct OffPath : Module {
    std::string name;
    int process(ImopsImage&) override {
        return fail(IMOPS_ERR_NOT_IMPLEMENTED,
                    "module " + name + " is not part of the GPU path; run it with the reference implementation");
    }
};

// The per-pixel modules directly after an AMaZE Demosaic (CFACoeffs, Exp,
// BaselineExposureCompensation, CST from camera RGB) run inside AMaZE's
// output stage: the same f32 operations per pixel in the same order, one
// pass over the image instead of one per module.  Returns the index of the
// last module folded in (k when none).
size_t plan_fusion(const ImopsImage& img, const std::vector<std::unique_ptr<Module>>& mods, size_t k,
                   color::Epilogue* e, int* out_cs) {
    *e = color::identity_epilogue();
    *out_cs = IMOPS_CS_CAMERA;
    bool wb_used = false;
    size_t last = k;
    for (size_t j = k + 1; j < mods.size(); j++) {
        Module* m = mods[j].get();
        if (auto* c = dynamic_cast<CFACoeffs*>(m)) {
            (void)c;
            if (wb_used || e->n_gain > 0 || !img.meta.has_wb) break;
            for (int i = 0; i < 3; i++) e->wb[i] = img.meta.wb_coeffs[i];
            wb_used = true;
        } else if (auto* x = dynamic_cast<Exp*>(m)) {
            if (e->n_gain >= 4) break;
            e->gain[e->n_gain++] = color::exp_value(x->ev);
        } else if (dynamic_cast<BaselineExposureCompensation*>(m)) {
            const ImopsImageMeta& md = img.meta;
            float ev = md.has_baseline_exposure ? md.baseline_exposure : 0.0f;
            bool g = md.has_shutter && md.has_f_number && md.has_iso && md.shutter_seconds > 0 && md.f_number > 0 &&
                     md.iso > 0;
            int need = (fabsf(ev) > 1e-6f ? 1 : 0) + (g ? 1 : 0);
            if (e->n_gain + need > 4) break;
            if (fabsf(ev) > 1e-6f) e->gain[e->n_gain++] = color::exp_value(ev);
            if (g) e->gain[e->n_gain++] = color::luminance_gain(md.shutter_seconds, md.f_number, md.iso);
        } else if (auto* c = dynamic_cast<CST*>(m)) {
            std::string name = c->target;
            name.erase(0, name.find_first_not_of(" \t\r\n"));
            name.erase(name.find_last_not_of(" \t\r\n") + 1);
            int cs;
            bool elsewhere;
            if (!cs_from_name(name, &cs, &elsewhere) || !img.meta.has_calibration) break;
            color::xyz_to_target(cs, e->tgt);
            color::camera_forward_matrix(img.meta.calibration_matrix_d65, e->fwd);
            e->do_cst = 1;
            e->srgb = cs == IMOPS_CS_SRGB;
            *out_cs = cs;
            last = j;
            break;  // the image now has a colour space; later modules run on their own
        } else {
            break;
        }
        last = j;
    }
    return last;
}

// ---- registry / schema (get_default_modules, modules.rs:897-915) -------------

struct FieldDef {
    const char* name;
    const char* type;  // "float", "integer", "string"
    const char* def_s;
    double def_n;
    const char* desc;
    std::vector<std::string> choices;
};

struct ModDef {
    const char* name;
    const char* desc;
    std::vector<FieldDef> fields;
    bool on_path;
};

const std::vector<ModDef>& registry() {
    static const std::vector<ModDef> r = {
        {"Demosaic", "Demosaic raw image data.",
         {{"algorithm", "string", "amaze", 0, "Demosaicing algorithm to use.",
           {"amaze", "markesteijn", "fast", "superfast", "supersuperfast"}}},
         true},
        {"ChromaDenoise", "Apply chroma-only BM3D denoising.",
         {{"intensity", "float", nullptr, 0.0, "Chroma denoising intensity factor.", {}}}, false},
        {"LumaGuidedChromaDenoise", "Apply luma-guided chroma denoising.",
         {{"epsilon", "float", nullptr, 0.01, "Guided filter edge-preservation epsilon (linear light).", {}},
          {"radius", "integer", nullptr, 4, "Guided filter radius in pixels.", {}}},
         false},
        {"CFACoeffs", "Apply Color Filter Array (CFA) white balance coefficients.", {}, true},
        {"Vignette", "Apply radial vignette correction.",
         {{"strength", "float", nullptr, 1.0, "Correction strength modifier.", {}}}, false},
        {"HighlightReconstruction", "Reconstruct clipped highlight details using white balance coefficients.", {},
         true},
        {"BaselineExposureCompensation",
         "Apply DNG BaselineExposure EV, then convert camera-relative linear values to absolute luminance using "
         "EXIF shutter/f-number/ISO (L = K\xc2\xb7v\xc2\xb7N\xc2\xb2/(t\xc2\xb7S)).",
         {},
         true},
        {"Exp", "Apply manual exposure compensation in EV.",
         {{"ev", "float", nullptr, 0.0, "Exposure compensation value in EV.", {}}}, true},
        {"Contrast", "Adjust image contrast.", {{"c", "float", nullptr, 1.0, "Contrast adjustment factor.", {}}}, true},
        {"CST", "Perform Color Space Transform.",
         {{"target_color_space", "string", "", 0, "Target color space to convert to.",
           {"Srgb", "AcesCg", "Oklch", "XyzD65"}}},
         true},
        {"Film",
         "Physically-based analog film simulation. NegativeLinear exports the densitometric scan; PositiveLinear "
         "inverts with the stock film-base Dmin and mid-gray gain.",
         {{"film_format", "string", "Film35mm", 0, "Film format (sets pixel pitch from frame width).",
           {"Film35mm", "Film6x6", "Film4x5"}},
          {"output", "string", "NegativeLinear", 0,
           "NegativeLinear: densitometric scanned negative. PositiveLinear: mid/Dmin invert from stock film-base + "
           "mid-gray gain.",
           {"NegativeLinear", "PositiveLinear"}},
          {"seed", "integer", nullptr, 1, "RNG seed for grain (deterministic).", {}},
          {"stock", "string", "ColorNeg200", 0, "Film stock identifier.",
           {"BwStub", "ColorNeg200", "Portra400", "Ektar100", "FujiPro400H", "EktachromeE100", "TriX400",
            "Baseline81"}}},
         true},
        {"LCH", "Adjust lightness, chroma, and hue coefficients.",
         {{"cc", "float", nullptr, 1.0, "Chroma (saturation) coefficient multiplier.", {}},
          {"hc", "float", nullptr, 1.0, "Hue coefficient multiplier.", {}},
          {"lc", "float", nullptr, 1.0, "Lightness coefficient multiplier.", {}}},
         true},
        {"SigmoidToneMap", "Sigmoid display tone map with ACES reference gamut compression (ACEScg).", {}, true},
        {"Gamma",
         "Power-law display encode: out = linear^(1/\xce\xb3). Use \xce\xb3=2.2 for sRGB-like, \xce\xb3=2.4 for "
         "BT.1886. Apply after CST to a linear display space.",
         {{"gamma", "float", nullptr, 2.2, "Display gamma (2.2 \xe2\x89\x88 sRGB, 2.4 = BT.1886).", {}}}, true},
        {"BM3D", "Apply BM3D image denoising.", {{"intensity", "float", nullptr, 0.0, "Denoising intensity factor.", {}}},
         false},
    };
    return r;
}

std::unique_ptr<Module> create(const ModDef& d, const Value& table) {
    std::string n = d.name;
    // every field of the module's config struct is required (serde, no defaults)
    for (const FieldDef& f : d.fields) {
        if (std::string(f.type) == "float") (void)get_f32(table, n, f.name);
        else if (std::string(f.type) == "integer") (void)get_int(table, n, f.name, true);
        else (void)get_str(table, n, f.name);
    }
    if (n == "Demosaic") {
        auto m = std::make_unique<Demosaic>();
        std::string a = get_str(table, n, "algorithm");
        const char* names[] = {"amaze", "markesteijn", "fast", "superfast", "supersuperfast"};
        int found = -1;
        for (int i = 0; i < 5; i++)
            if (a == names[i]) found = i;
        if (found < 0) throw ParamError{"Invalid Demosaic config: unknown variant `" + a + "`"};
        m->algorithm = found;
        return m;
    }
    if (n == "CFACoeffs") return std::make_unique<CFACoeffs>();
    if (n == "Exp") {
        auto m = std::make_unique<Exp>();
        m->ev = get_f32(table, n, "ev");
        return m;
    }
    if (n == "BaselineExposureCompensation") return std::make_unique<BaselineExposureCompensation>();
    if (n == "CST") {
        auto m = std::make_unique<CST>();
        m->target = get_str(table, n, "target_color_space");
        return m;
    }
    if (n == "Film") {
        auto m = std::make_unique<Film>();
        std::string st = get_str(table, n, "stock"), fm = get_str(table, n, "film_format"),
                    out = get_str(table, n, "output");
        m->stock_name = st;
        if (st == "BwStub") m->p.stock = IMOPS_STOCK_BWSTUB;
        else if (st == "ColorNeg200") m->p.stock = IMOPS_STOCK_COLORNEG200;
        else if (st == "Portra400") m->p.stock = IMOPS_STOCK_PORTRA400;
        else if (st == "Ektar100") m->p.stock = IMOPS_STOCK_EKTAR100;
        else if (st == "FujiPro400H") m->p.stock = IMOPS_STOCK_FUJIPRO400H;
        else if (st == "EktachromeE100") m->p.stock = IMOPS_STOCK_EKTACHROMEE100;
        else if (st == "TriX400") m->p.stock = IMOPS_STOCK_TRIX400;
        else if (st == "Baseline81") m->p.stock = IMOPS_STOCK_BASELINE81;
        else
            throw ParamError{"Unknown film stock: " + st};
        if (fm == "Film35mm") m->p.film_format = IMOPS_FORMAT_35MM;
        else if (fm == "Film6x6") m->p.film_format = IMOPS_FORMAT_6X6;
        else if (fm == "Film4x5") m->p.film_format = IMOPS_FORMAT_4X5;
        else throw ParamError{"Unknown film format: " + fm};
        if (out == "NegativeLinear") m->p.output = IMOPS_FILM_NEGATIVE_LINEAR;
        else if (out == "PositiveLinear") m->p.output = IMOPS_FILM_POSITIVE_LINEAR;
        else throw ParamError{"Unknown film output: " + out};
        m->p.seed = (uint64_t)get_int(table, n, "seed", true);
        m->p.grain = 1;
        m->p.shutter_seconds = -1.0f;
        return m;
    }
    if (n == "HighlightReconstruction") return std::make_unique<HighlightReconstruction>();
    if (n == "SigmoidToneMap") return std::make_unique<SigmoidToneMap>();
    if (n == "Contrast") {
        auto m = std::make_unique<Contrast>();
        m->value = get_f32(table, n, "c");
        return m;
    }
    if (n == "Gamma") {
        auto m = std::make_unique<Gamma>();
        m->gamma = get_f32(table, n, "gamma");
        return m;
    }
    if (n == "LCH") {
        auto m = std::make_unique<LCH>();
        m->lc = get_f32(table, n, "lc");
        m->cc = get_f32(table, n, "cc");
        m->hc = get_f32(table, n, "hc");
        return m;
    }
    auto m = std::make_unique<OffPath>();
    m->name = n;
    return m;
}

}  // namespace pipe
}  // namespace imops

struct ImopsPipeline {
    std::vector<std::unique_ptr<imops::pipe::Module>> modules;
};

using namespace imops;

namespace {

ImopsImage* new_image(const ImopsImageMeta* meta) {
    auto* img = new ImopsImage();
    if (meta) {
        img->meta = *meta;
        if (meta->cfa) img->cfa = meta->cfa;
        img->meta.cfa = nullptr;
    }
    return img;
}

int attach_stream(ImopsImage* img) {
    int rc = pipe::device_stream(&img->stream);
    if (rc) return rc;
    IMOPS_CUDA_TRY(cudaGetDevice(&img->dev), "cudaGetDevice");
    return IMOPS_OK;
}

}  // namespace

extern "C" ImopsImage* new_raw_image_u16_c(const uint16_t* raw, size_t width, size_t height,
                                           const ImopsImageMeta* meta) {
    clear_error();
    if (!raw || !meta || width == 0 || height == 0) {
        fail(IMOPS_ERR_INVALID_ARGUMENT, "new_raw_image_u16_c: NULL buffer, NULL metadata or empty frame");
        return nullptr;
    }
    int cw = meta->crop_w > 0 ? meta->crop_w : (int)width - meta->crop_x;
    int ch = meta->crop_h > 0 ? meta->crop_h : (int)height - meta->crop_y;
    if (meta->crop_x < 0 || meta->crop_y < 0 || cw <= 0 || ch <= 0 || (size_t)(meta->crop_x + cw) > width ||
        (size_t)(meta->crop_y + ch) > height) {
        fail(IMOPS_ERR_INVALID_ARGUMENT, "new_raw_image_u16_c: crop_area outside the frame");
        return nullptr;
    }
    ImopsImage* img = new_image(meta);
    if (attach_stream(img) || pipe::buf_alloc(img->raw, width * height * 2, img->stream)) {
        delete img;
        return nullptr;
    }
    if (cudaMemcpyAsync(img->raw.p, raw, width * height * 2, cudaMemcpyHostToDevice, img->stream) != cudaSuccess ||
        cudaStreamSynchronize(img->stream) != cudaSuccess) {
        fail(IMOPS_ERR_CUDA, "new_raw_image_u16_c: upload failed");
        pipe::buf_free(img->raw, img->stream);
        delete img;
        return nullptr;
    }
    img->raw_kind = 1;
    img->raw_w = width;
    img->raw_h = height;
    img->width = cw;
    img->height = ch;
    return img;
}

extern "C" ImopsImage* new_raw_image_f32_c(const float* raw_data, size_t width, size_t height,
                                           const ImopsImageMeta* meta) {
    clear_error();
    if (!raw_data || !meta || width == 0 || height == 0) {
        fail(IMOPS_ERR_INVALID_ARGUMENT, "new_raw_image_f32_c: NULL buffer, NULL metadata or empty image");
        return nullptr;
    }
    ImopsImage* img = new_image(meta);
    if (attach_stream(img) || pipe::buf_alloc(img->raw, width * height * 4, img->stream)) {
        delete img;
        return nullptr;
    }
    if (cudaMemcpyAsync(img->raw.p, raw_data, width * height * 4, cudaMemcpyHostToDevice, img->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(img->stream) != cudaSuccess) {
        fail(IMOPS_ERR_CUDA, "new_raw_image_f32_c: upload failed");
        pipe::buf_free(img->raw, img->stream);
        delete img;
        return nullptr;
    }
    img->raw_kind = 2;
    img->raw_w = width;
    img->raw_h = height;
    img->width = width;
    img->height = height;
    return img;
}

extern "C" ImopsImage* new_rgb_image_c(const float* rgb, size_t width, size_t height, int color_space,
                                       const ImopsImageMeta* meta) {
    clear_error();
    if (!rgb || width == 0 || height == 0) {
        fail(IMOPS_ERR_INVALID_ARGUMENT, "new_rgb_image_c: NULL buffer or empty image");
        return nullptr;
    }
    if (color_space < IMOPS_CS_CAMERA || color_space > IMOPS_CS_ACESCG) {
        fail(IMOPS_ERR_INVALID_ARGUMENT, "new_rgb_image_c: unknown colour space");
        return nullptr;
    }
    ImopsImage* img = new_image(meta);
    if (attach_stream(img) || pipe::buf_alloc(img->rgb, width * height * 12, img->stream)) {
        delete img;
        return nullptr;
    }
    if (cudaMemcpyAsync(img->rgb.p, rgb, width * height * 12, cudaMemcpyHostToDevice, img->stream) != cudaSuccess ||
        cudaStreamSynchronize(img->stream) != cudaSuccess) {
        fail(IMOPS_ERR_CUDA, "new_rgb_image_c: upload failed");
        pipe::buf_free(img->rgb, img->stream);
        delete img;
        return nullptr;
    }
    img->has_rgb = true;
    img->width = width;
    img->height = height;
    img->has_cs = color_space != IMOPS_CS_CAMERA;
    img->color_space = color_space;
    return img;
}

extern "C" ImopsPipeline* get_pixel_pipeline_c(const uint8_t* config, size_t config_len) {
    clear_error();
    if (!config) {
        fail(IMOPS_ERR_INVALID_ARGUMENT, "get_pixel_pipeline_c: NULL config");
        return nullptr;
    }
    std::string text(reinterpret_cast<const char*>(config), config_len);
    cfg::Value root;
    std::string e1, e2;
    if (!cfg::parse_toml(text, &root, &e1) && !cfg::parse_json(text, &root, &e2)) {
        fail(IMOPS_ERR_CONFIG, "cant decode config from string: TOML: " + e1 + "; JSON: " + e2);
        return nullptr;
    }
    const cfg::Value* list = root.kind == cfg::Value::TABLE ? root.get("pipeline_modules") : nullptr;
    if (!list || list->kind != cfg::Value::ARRAY) {
        fail(IMOPS_ERR_CONFIG, "cant decode config from string: missing field `pipeline_modules`");
        return nullptr;
    }
    auto* p = new ImopsPipeline();
    try {
        for (const cfg::Value& m : list->a) {
            if (m.kind != cfg::Value::TABLE) throw pipe::ParamError{"cant decode config from string: module is not a table"};
            const cfg::Value* nm = m.get("name");
            if (!nm || nm->kind != cfg::Value::STRING) throw pipe::ParamError{"Module must have a name field"};
            const pipe::ModDef* def = nullptr;
            for (const auto& d : pipe::registry())
                if (pipe::lower(d.name) == pipe::lower(nm->s)) def = &d;
            if (!def) throw pipe::ParamError{"wrong pipeline module name " + nm->s};
            p->modules.push_back(pipe::create(*def, m));
        }
    } catch (const pipe::ParamError& e) {
        delete p;
        fail(IMOPS_ERR_CONFIG, e.msg);
        return nullptr;
    }
    return p;
}

extern "C" ImopsImage* run_pixel_pipeline_c(ImopsImage* image, ImopsPipeline* pipeline) {
    clear_error();
    if (!image || !pipeline) return nullptr;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != image->dev) cudaSetDevice(image->dev);
    pipe::ComputeOrder order;
    if (pipe::order_compute(image->stream, &order)) return nullptr;
    auto& mods = pipeline->modules;
    for (size_t k = 0; k < mods.size(); k++) {
        if (dynamic_cast<pipe::PixelModule*>(mods[k].get())) {
            // a run of per-pixel modules: one pass per display::MAX_OPS ops
            display::Chain c{};
            auto flush = [&]() {
                int rc = display::run(static_cast<float*>(image->rgb.p), image->width * image->height, c,
                                      image->stream, "pixel modules");
                c.n = 0;
                return rc;
            };
            size_t j = k;
            for (; j < mods.size(); j++) {
                auto* q = dynamic_cast<pipe::PixelModule*>(mods[j].get());
                if (!q) break;
                if (c.n + q->max_ops() > display::MAX_OPS && flush() != IMOPS_OK) return nullptr;
                if (int rc = q->add_ops(*image, c)) {
                    // the modules before this one have run, as in the reference
                    std::string msg = last_error();
                    flush();
                    fail(rc, msg);
                    return nullptr;
                }
            }
            if (flush() != IMOPS_OK) return nullptr;
            k = j - 1;
            continue;
        }
        auto* dem = dynamic_cast<pipe::Demosaic*>(mods[k].get());
        size_t fused_until = k;
        color::Epilogue fused = color::identity_epilogue();
        int fused_cs = IMOPS_CS_CAMERA;
        if (dem && (dem->algorithm == IMOPS_DEMOSAIC_AMAZE || dem->algorithm == IMOPS_DEMOSAIC_MARKESTEIJN) &&
            image->raw_kind != 0 && !image->cfa.empty())
            fused_until = pipe::plan_fusion(*image, mods, k, &fused, &fused_cs);
        // nothing folded in: the demosaic keeps its plain output stage
        const int rc = dem ? dem->process_fused(*image, fused_until > k ? &fused : nullptr, fused_cs)
                           : mods[k]->process(*image);
        if (rc != IMOPS_OK) return nullptr;
        k = fused_until;
    }
    // Returns once the work is queued on the image's stream: every call that
    // reads the image's pixels waits for it, so results are as if it had
    // waited here, and frames submitted one after another overlap.  An error
    // raised while the kernels run is reported by that reading call.
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        cuda_status(e, "run_pixel_pipeline_c");
        return nullptr;
    }
    return image;
}

extern "C" int get_image_info_c(const ImopsImage* image, size_t* width, size_t* height, int* color_space) {
    clear_error();
    if (!image) return fail(IMOPS_ERR_INVALID_ARGUMENT, "get_image_info_c: NULL image");
    if (width) *width = image->width;
    if (height) *height = image->height;
    if (color_space) *color_space = image->has_cs ? image->color_space : IMOPS_CS_CAMERA;
    return IMOPS_OK;
}

extern "C" int get_image_rgb_f32_c(ImopsImage* image, float* out, size_t n_floats) {
    clear_error();
    if (!image || !out) return fail(IMOPS_ERR_INVALID_ARGUMENT, "get_image_rgb_f32_c: NULL argument");
    if (!image->has_rgb) return fail(IMOPS_ERR_INVALID_ARGUMENT, "get_image_rgb_f32_c: the image has no RGB data");
    size_t need = image->width * image->height * 3;
    if (n_floats < need) return fail(IMOPS_ERR_INVALID_ARGUMENT, "get_image_rgb_f32_c: output buffer too small");
    IMOPS_CUDA_TRY(cudaMemcpyAsync(out, image->rgb.p, need * 4, cudaMemcpyDeviceToHost, image->stream), "download");
    IMOPS_CUDA_TRY(cudaStreamSynchronize(image->stream), "cudaStreamSynchronize");
    return IMOPS_OK;
}

namespace imops {
namespace pipe {
__global__ void to_u8_kernel(const float* __restrict__ in, size_t n, uint8_t* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float v = in[i];
        // f32::clamp keeps NaN; `as u8` saturates and maps NaN to 0
        if (v < 0.0f) v = 0.0f;
        if (v > 1.0f) v = 1.0f;
        float s = v * 255.0f;
        out[i] = isnan(s) ? 0 : (uint8_t)s;
    }
}
}  // namespace pipe
}  // namespace imops

extern "C" const uint8_t* get_image_rgb_data_c(ImopsImage* image, size_t* out_width, size_t* out_height,
                                               size_t* out_len) {
    clear_error();
    if (!image) return nullptr;
    if (!image->has_rgb) {
        fail(IMOPS_ERR_INVALID_ARGUMENT, "get_image_rgb_data_c: the image has no RGB data");
        return nullptr;
    }
    size_t n = image->width * image->height * 3;
    uint8_t* host = static_cast<uint8_t*>(std::malloc(n ? n : 1));
    if (!host) {
        fail(IMOPS_ERR_OUT_OF_MEMORY, "get_image_rgb_data_c: host allocation failed");
        return nullptr;
    }
    pipe::DevBuf tmp;
    if (pipe::buf_alloc(tmp, n ? n : 1, image->stream)) {
        std::free(host);
        return nullptr;
    }
    pipe::to_u8_kernel<<<color::stream_grid(n, 256), 256, 0, image->stream>>>(static_cast<const float*>(image->rgb.p),
                                                                               n, static_cast<uint8_t*>(tmp.p));
    note_launch();
    cudaError_t e = cudaMemcpyAsync(host, tmp.p, n, cudaMemcpyDeviceToHost, image->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(image->stream);
    pipe::buf_free(tmp, image->stream);
    if (e != cudaSuccess) {
        cuda_status(e, "get_image_rgb_data_c");
        std::free(host);
        return nullptr;
    }
    if (out_width) *out_width = image->width;
    if (out_height) *out_height = image->height;
    if (out_len) *out_len = n;
    return host;
}

namespace {
char* dup_string(const std::string& s) {
    char* p = static_cast<char*>(std::malloc(s.size() + 1));
    if (p) std::memcpy(p, s.c_str(), s.size() + 1);
    return p;
}
}  // namespace

extern "C" char* get_image_metadata_c(const ImopsImage* image) {
    clear_error();
    if (!image) return nullptr;
    using cfg::Value;
    Value root;
    root.kind = Value::TABLE;
    auto num = [](double v, bool integer = false) {
        Value x;
        if (integer) {
            x.kind = Value::INT;
            x.i = (long long)v;
        } else {
            x.kind = Value::FLOAT;
            x.f = v;
        }
        return x;
    };
    auto nul = []() { return Value(); };
    auto arr = [&](const float* a, int n) {
        Value x;
        x.kind = Value::ARRAY;
        for (int i = 0; i < n; i++) x.a.push_back(num(a[i]));
        return x;
    };
    const ImopsImageMeta& m = image->meta;
    Value cfa;
    if (image->cfa.empty()) {
        cfa = nul();
    } else {
        cfa.kind = Value::STRING;
        cfa.s = image->cfa;
    }
    root.t.emplace_back("cfa", cfa);
    root.t.emplace_back("wb_coeffs", m.has_wb ? arr(m.wb_coeffs, 4) : nul());
    root.t.emplace_back("calibration_matrix_d65", m.has_calibration ? arr(m.calibration_matrix_d65, 9) : nul());
    root.t.emplace_back("black_level", num(m.black_level));
    root.t.emplace_back("white_level", num(m.white_level));
    Value cs;
    if (image->has_cs) {
        cs.kind = Value::STRING;
        const char* names[] = {"XyzD65", "LinearSrgb", "Srgb", "AcesCg", "Oklch"};
        cs.s = names[image->color_space];
    }
    root.t.emplace_back("color_space", cs);
    root.t.emplace_back("baseline_exposure", m.has_baseline_exposure ? num(m.baseline_exposure) : nul());
    root.t.emplace_back("shutter_seconds", m.has_shutter ? num(m.shutter_seconds) : nul());
    root.t.emplace_back("f_number", m.has_f_number ? num(m.f_number) : nul());
    root.t.emplace_back("iso", m.has_iso ? num(m.iso) : nul());
    root.t.emplace_back("height", num((double)image->height, true));
    root.t.emplace_back("width", num((double)image->width, true));
    return dup_string(cfg::to_json(root));
}

extern "C" char* get_pipeline_schema_c(void) {
    clear_error();
    using cfg::Value;
    Value root;
    root.kind = Value::ARRAY;
    for (const auto& d : pipe::registry()) {
        Value mod;
        mod.kind = Value::TABLE;
        Value v;
        v.kind = Value::STRING;
        v.s = d.name;
        mod.t.emplace_back("name", v);
        v.s = d.desc;
        mod.t.emplace_back("description", v);
        Value fields;
        fields.kind = Value::ARRAY;
        std::vector<pipe::FieldDef> fs = d.fields;
        std::sort(fs.begin(), fs.end(), [](const pipe::FieldDef& a, const pipe::FieldDef& b) {
            return std::string(a.name) < std::string(b.name);
        });
        for (const auto& f : fs) {
            Value fd;
            fd.kind = Value::TABLE;
            Value s;
            s.kind = Value::STRING;
            s.s = f.name;
            fd.t.emplace_back("name", s);
            s.s = f.type;
            fd.t.emplace_back("field_type", s);
            Value dv;
            if (f.def_s) {
                dv.kind = Value::STRING;
                dv.s = f.def_s;
            } else if (std::string(f.type) == "integer") {
                dv.kind = Value::INT;
                dv.i = (long long)f.def_n;
            } else {
                dv.kind = Value::FLOAT;
                dv.f = (double)(float)f.def_n;
            }
            fd.t.emplace_back("default_value", dv);
            s.s = f.desc;
            fd.t.emplace_back("description", s);
            Value ch;
            if (!f.choices.empty()) {
                ch.kind = Value::ARRAY;
                for (const auto& c : f.choices) {
                    Value x;
                    x.kind = Value::STRING;
                    x.s = c;
                    ch.a.push_back(x);
                }
            }
            fd.t.emplace_back("choices", ch);
            fields.a.push_back(fd);
        }
        mod.t.emplace_back("fields", fields);
        root.a.push_back(mod);
    }
    return dup_string(cfg::to_json(root));
}

extern "C" char* get_last_error_c(void) {
    const char* e = last_error();
    if (!e || !*e) return nullptr;
    return dup_string(e);
}

extern "C" void free_image_c(ImopsImage* image) {
    if (!image) return;
    pipe::buf_free(image->raw, image->stream);
    pipe::buf_free(image->rgb, image->stream);
    delete image;
}

extern "C" void free_pipeline_c(ImopsPipeline* pipeline) { delete pipeline; }

extern "C" void free_rgb_buffer_c(uint8_t* ptr, size_t len) {
    (void)len;
    std::free(ptr);
}

extern "C" void free_string_c(char* ptr) { std::free(ptr); }
