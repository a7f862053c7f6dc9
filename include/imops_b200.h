/*
 * imops_b200.h -- C-ABI of the B200 (sm_100a) raw-development library.
 *
 * Drop-in boundary for the hot path of DavRack/imops (a Rust project): each
 * entry point replaces one stage the reference runs on the CPU and names the
 * reference interface (file:line, paths inside the reference project) whose
 * behaviour it reproduces.  Plain pointers and sizes only.
 *
 * Conventions
 *  - Every call returns an int status (IMOPS_OK == 0).  On failure the
 *    reason is kept in a thread-local string read by imops_last_error(), the
 *    counterpart of get_last_error_c (pichromatic-pipeline/src/extern_pipeline.rs:27-38).
 *  - Stage entry points (imops_*) take DEVICE pointers and run on the
 *    caller's CUDA stream (imops_stream_t is a cudaStream_t; NULL = legacy
 *    default stream).  They allocate nothing unless documented.
 *  - Images are row-major; RGB is interleaved f32 [r,g,b] per pixel, the
 *    reference's Image.rgb_data layout (pichromatic/src/pixel.rs:23-27);
 *    mosaics are one f32 per site, Image.raw_data.
 *  - CFA patterns are strings as CFA::new takes them ("RGGB", 36-char
 *    X-Trans, ...; pichromatic/src/cfa.rs:98-129); shift_x/shift_y apply
 *    CFA::shift (cfa.rs:204-233) for a crop origin.
 */
#ifndef IMOPS_B200_H
#define IMOPS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void *imops_stream_t;

/* Status codes. */
#define IMOPS_OK 0
#define IMOPS_ERR_INVALID_ARGUMENT 1
#define IMOPS_ERR_UNSUPPORTED_CFA 2
#define IMOPS_ERR_UNSUPPORTED_SIZE 3
#define IMOPS_ERR_CUDA 4
#define IMOPS_ERR_OUT_OF_MEMORY 5
#define IMOPS_ERR_WRONG_COLOR_SPACE 6   /* FilmError::WrongColorSpace (film/error.rs:5-13) */
#define IMOPS_ERR_INVALID_DIMENSIONS 7  /* FilmError::InvalidDimensions */
#define IMOPS_ERR_INVALID_STOCK 8       /* FilmError::InvalidStock */
#define IMOPS_ERR_CONFIG 9              /* config::parse_config failures (config.rs:13-34) */
#define IMOPS_ERR_NOT_IMPLEMENTED 10    /* a module that stays on the reference (BM3D, ...) */
#define IMOPS_ERR_TIMEOUT 11            /* a bounded device wait gave up */

/* Colour spaces (subset of the `color` crate's ColorSpaceTag used on the path). */
#define IMOPS_CS_CAMERA (-1)            /* Image.metadata.color_space == None */
#define IMOPS_CS_XYZD65 0
#define IMOPS_CS_LINEAR_SRGB 1
#define IMOPS_CS_SRGB 2
#define IMOPS_CS_ACESCG 3
#define IMOPS_CS_OKLCH 4                /* CSS Color 4 Oklch: L, C, hue in degrees [0, 360) */

/* Demosaic algorithms: DemosaicAlgorithmType (pichromatic-pipeline/src/modules.rs:72-104). */
#define IMOPS_DEMOSAIC_AMAZE 0
#define IMOPS_DEMOSAIC_MARKESTEIJN 1
#define IMOPS_DEMOSAIC_FAST 2
#define IMOPS_DEMOSAIC_SUPERFAST 3
#define IMOPS_DEMOSAIC_SUPERSUPERFAST 4

/* Thread-local message of the last failed call (or "" after a success).
 * Replaces get_last_error_c (extern_pipeline.rs:27-38); the string is owned
 * by the library and valid until the next call on the same thread. */
const char *imops_last_error(void);

/* Library version string. */
const char *imops_version(void);

/* Frees the working sets the stage entry points cache per (device, stream)
 * on the current device (film, adjoint, the scaled mosaics of the u16
 * develop paths), after waiting for the device; the next call allocates
 * again.  No counterpart in the reference (its buffers are Rust Vecs freed
 * with each module).  Call it when no work of this library is in flight on
 * the device from another thread. */
int imops_release_working_sets(void);

/* ---- decode-side normalisation ------------------------------------------
 * Black/white scaling of a u16 sensor frame plus the crop copy.  Replaces
 * RawImage::apply_scaling (rawler 0.7, called at extern_pipeline.rs:263) and
 * demosaic::crop_and_normalize (pichromatic/src/demosaic.rs:61-91):
 * out[y][x] = (raw[cy+y][cx+x] - black[s]) / (white[s] - black[s]),
 * s = ((cy+y) % period_h) * period_w + (cx+x) % period_w (full-frame CFA cell).
 * black/white are HOST arrays of period_w*period_h values. */
int imops_scale_u16(const uint16_t *raw, int raw_w, int raw_h, int crop_x, int crop_y, int crop_w, int crop_h,
                    const float *black, const float *white, int period_w, int period_h, float *out,
                    imops_stream_t stream);

/* ---- demosaic -------------------------------------------------------------
 * AMaZE, bit-identical to demosaic_algorithms::Amaze (demosaic.rs:358-1379)
 * including its 128x128/96-stride tiling.  Requires a 2x2 Bayer CFA;
 * returns IMOPS_ERR_UNSUPPORTED_SIZE for image sizes where the reference's
 * tile fill writes past its tile buffer (the reference panics there).
 * mosaic: w*h f32; rgb: w*h*3 f32. */
int imops_demosaic_amaze(const float *mosaic, int w, int h, const char *cfa, int shift_x, int shift_y, float clip_pt,
                         float *rgb, imops_stream_t stream);

/* Whether imops_demosaic_amaze accepts a w x h image (host-only check). */
int imops_amaze_size_supported(int w, int h);

/* 3x3 same-colour mean, demosaic_algorithms::Markesteijn (demosaic.rs:108-186);
 * any CFA period up to 12x12 (Bayer, X-Trans). */
int imops_demosaic_markesteijn(const float *mosaic, int w, int h, const char *cfa, int shift_x, int shift_y,
                               float *rgb, imops_stream_t stream);

/* 3-pass directional X-Trans demosaic after Markesteijn's method (no
 * counterpart in the reference, whose "markesteijn" is the 3x3 mean above):
 * green along four directions bounded by the orthogonal greens, red / blue
 * from colour differences, two green refinement passes, and a CIELab
 * homogeneity vote between the directions; pixels within 10 of an edge take
 * the 3x3 mean.  6x6 CFAs only (IMOPS_ERR_UNSUPPORTED_CFA otherwise).
 * Allocates nothing: each 32x32 tile runs every step in shared memory. */
int imops_demosaic_markesteijn3(const float *mosaic, int w, int h, const char *cfa, int shift_x, int shift_y,
                                float *rgb, imops_stream_t stream);

/* Quad-sampling previews Fast / SuperFast / SuperSuperFast (demosaic.rs:189-356):
 * factor 2, 4 or 8; rgb holds (w/factor)*(h/factor)*3 floats. */
int imops_demosaic_quad(const float *mosaic, int w, int h, const char *cfa, int shift_x, int shift_y, int factor,
                        float *rgb, imops_stream_t stream);

/* ---- per-pixel colour ------------------------------------------------------ */

/* White balance after demosaic: rgb *= wb[0..3] (cfa_coeffs.rs:4-12). */
int imops_cfa_coeffs(float *rgb, size_t n_pixels, const float wb[4], imops_stream_t stream);

/* Exposure: rgb *= 2^ev (exp.rs:4-11). */
int imops_exp(float *rgb, size_t n_pixels, float ev, imops_stream_t stream);

/* BaselineExposureCompensation (pichromatic-pipeline/src/modules.rs:335-373):
 * 2^baseline_ev when |ev| > 1e-6, then the absolute-luminance gain
 * 12.5*N^2/(t*S) when shutter, f_number and iso are all > 0.  *applied
 * (may be NULL) receives 1 when the gain was applied. */
int imops_baseline_exposure(float *rgb, size_t n_pixels, float baseline_ev, float shutter_seconds, float f_number,
                            float iso, int *applied, imops_stream_t stream);

/* Camera RGB -> XYZ(D65) forward matrix of camera_cst (cst.rs:12-38, 51-95),
 * computed on the host in f32 exactly as the reference does. */
int imops_camera_forward_matrix(const float calib_d65[9], float forward[9]);

/* camera_cst (cst.rs:12-48): xyz = forward * rgb, then XYZ(D65) -> target
 * (IMOPS_CS_*).  calib_d65: the 3x3 row-major calibration matrix. */
int imops_camera_cst(float *rgb, size_t n_pixels, const float calib_d65[9], int target, imops_stream_t stream);

/* ---- display stages and colour-space conversion ---------------------------
 * Each runs in place over interleaved RGB.  The pipeline C-ABI fuses a run of
 * consecutive per-pixel modules into one pass of the same ops.  Conversions
 * involving Oklch restate the `color` crate 0.3.3 ColorSpaceTag::convert:
 * Oklab (Ottosson 2020, linear-sRGB matrices), LCh per CSS Color 4. */

/* cst (cst.rs:6-10): source -> target between IMOPS_CS_XYZD65, _LINEAR_SRGB,
 * _SRGB, _ACESCG and _OKLCH (camera RGB goes through imops_camera_cst). */
int imops_cst(float *rgb, size_t n_pixels, int source, int target, imops_stream_t stream);

/* highlight_reconstruction (highlight_reconstruction.rs:5-13):
 * f = g / wb[1]; g = (1 - f) g + f (r + b) / 2. */
int imops_highlight_reconstruction(float *rgb, size_t n_pixels, const float wb[4], imops_stream_t stream);

/* contrast (contrast.rs:4-8): x = 0.185 (x / 0.185)^value per channel. */
int imops_contrast(float *rgb, size_t n_pixels, float value, imops_stream_t stream);

/* gamma_encode (tone_map.rs:38-49): x <= 0 ? 0 : x^(1 / max(gamma, 1e-6)). */
int imops_gamma(float *rgb, size_t n_pixels, float gamma, imops_stream_t stream);

/* lch (lch.rs:5-18): to Oklch from color_space, (L, C, h) *= (lc, cc, hc),
 * back.  IMOPS_CS_CAMERA is rejected (the reference unwraps None). */
int imops_lch(float *rgb, size_t n_pixels, int color_space, float lc, float cc, float hc, imops_stream_t stream);

/* sigmoid (tone_map.rs:18-33) on ACEScg: ACES reference gamut compression
 * (default RgcParams, :59-69), square_sigmoid per channel, chroma scaled by
 * 1 - Y^5 in Oklch with the hue of the compressed pixel. */
int imops_sigmoid_tone_map(float *rgb, size_t n_pixels, imops_stream_t stream);

/* ---- spectral film simulation ------------------------------------------- */

/* Stocks: StockId (pichromatic/src/film/stock/mod.rs:126-147), plus the
 * library's 81-bin "baseline" preset (not in the reference, see
 * ImopsBaselineFilm). */
#define IMOPS_STOCK_BWSTUB 0
#define IMOPS_STOCK_COLORNEG200 1
#define IMOPS_STOCK_PORTRA400 2
#define IMOPS_STOCK_EKTAR100 3
#define IMOPS_STOCK_FUJIPRO400H 4
#define IMOPS_STOCK_EKTACHROMEE100 5
#define IMOPS_STOCK_TRIX400 6
#define IMOPS_STOCK_BASELINE81 100

/* FilmFormat (film/types.rs:24-49). */
#define IMOPS_FORMAT_35MM 0
#define IMOPS_FORMAT_6X6 1
#define IMOPS_FORMAT_4X5 2

/* FilmOutput (film/mod.rs:45-51). */
#define IMOPS_FILM_NEGATIVE_LINEAR 0
#define IMOPS_FILM_POSITIVE_LINEAR 1

/* FilmParams (film/mod.rs:53-71) plus the image metadata film::process reads. */
typedef struct {
    int stock;              /* IMOPS_STOCK_* */
    int film_format;        /* IMOPS_FORMAT_* */
    uint64_t seed;          /* grain seed */
    int output;             /* IMOPS_FILM_* */
    float shutter_seconds;  /* metadata.shutter_seconds; < 0 when absent (then 1 / box ISO) */
    int grain;              /* 1: grain as the reference (always on); 0: grain off (parity mode) */
} ImopsFilmParams;

/* The "baseline" 81-bin preset (380..780 nm, 5 nm): 3 layers with Gaussian
 * sensitivities (450/550/650 nm), logistic density curves
 * D = dmax / (1 + exp(-k (log10 E - x0))), halation as a Gaussian blur of
 * max(0, R - hal_threshold) (fixed tap radius) added with strength * bleed
 * per layer, and seeded SplitMix64 grain of std grain_sigma.  Operates on
 * relative scene-linear ACEScg.  Field order is part of the ABI. */
typedef struct {
    float dmax[3], k[3], x0[3];
    float hal_strength;     /* 0.15 */
    float hal_sigma;        /* 20 px */
    int hal_radius;         /* 64 (fixed so the output is smooth in sigma) */
    float hal_threshold;    /* 0.8 */
    float grain_sigma;      /* 0.02 (density) */
    float grain_blur;       /* 1 px */
    int grain_on;
    uint64_t seed;
    int scan;               /* IMOPS_SCAN_*: how the 81-bin scan contracts */
} ImopsBaselineFilm;

/* The baseline preset's 81-bin scan (densitometry.rs:13-73 on its grid):
 * FP32: both spectral contractions as packed f32x2 FMAs on the CUDA cores;
 * BF16_TC: both on the tensor cores (tcgen05), BF16 operands split hi + lo
 * (three products per term), FP32 accumulation.  Both are within 1e-4 of
 * the FP64 oracle. */
#define IMOPS_SCAN_FP32 0
#define IMOPS_SCAN_BF16_TC 1

/* Defaults of the baseline preset (the benchmark workload's values). */
void imops_baseline_film_defaults(ImopsBaselineFilm *out);

/* film::process (pichromatic/src/film/mod.rs:77-129) on a device RGB image
 * in place.  color_space must be IMOPS_CS_ACESCG (else
 * IMOPS_ERR_WRONG_COLOR_SPACE, FilmError::WrongColorSpace); w, h > 0 (else
 * IMOPS_ERR_INVALID_DIMENSIONS).  The reference stocks expect absolute
 * luminance (BaselineExposureCompensation); IMOPS_STOCK_BASELINE81 takes the
 * preset in `baseline` and relative ACEScg (baseline == NULL: the defaults,
 * with params->seed as grain seed and params->grain as grain switch).  Uses a
 * library-owned per-stream workspace (allocated on first use). */
int imops_film_process(float *rgb, int w, int h, int color_space, const ImopsFilmParams *params,
                       const ImopsBaselineFilm *baseline, imops_stream_t stream);

/* The baseline preset of imops_film_process (stock IMOPS_STOCK_BASELINE81)
 * without any device allocation.  No counterpart in the reference.  For
 * callers that cannot call cudaMalloc: a host application that gives the GPU
 * a fixed memory budget through its own allocator must not have the library
 * allocate behind its back, and a real-time preview loop cannot take the
 * device-wide synchronisation cudaMalloc and cudaFree may cause.  The
 * preset's working planes (16 bytes a pixel) live in one fixed array of
 * device memory, about 34 MiB, which every GPU that loads the library holds
 * until the process exits; the caller still passes the image.
 *  - Images above imops_film_noalloc_max_pixels() pixels (2,097,152: a
 *    1920 x 1080 preview fits) are rejected with IMOPS_ERR_UNSUPPORTED_SIZE.
 *  - Output equals imops_film_process with the same preset.
 *  - The first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress) and caches it: make that first call on each
 *    device before any stream capture.
 *  - Every call shares the array and it keeps the last call's contents
 *    (each call writes all it reads there): calls that may overlap on the
 *    GPU -- on different streams, or from different threads -- race and
 *    corrupt each other; order them on one stream or with events. */
int imops_film_baseline_noalloc(float *rgb, int w, int h, int color_space, const ImopsBaselineFilm *baseline,
                                imops_stream_t stream);

/* Largest image, in pixels, that imops_film_baseline_noalloc accepts. */
size_t imops_film_noalloc_max_pixels(void);

/* ---- the reference model's film sub-stages -----------------------------------
 * The stages that film::process (film/mod.rs:77-129) chains, one call each,
 * for a host that runs them separately.  imops_film_process is the same
 * chain: expose -> halation -> develop -> grain -> scan -> invert gives its
 * result bit for bit.  Planes are planar f32 (w*h each) of the stock's E
 * emulsion layers (imops_film_layers); rgb is interleaved ACEScg.  The
 * baseline preset runs only whole (IMOPS_ERR_INVALID_STOCK here).  params
 * supply stock, film format (pixel pitch), shutter, seed, grain and output as
 * for imops_film_process.  Each call keeps its scratch in the per-(device,
 * stream) film working set. */

/* E, the stock's emulsion layers (film/stock/mod.rs:152-214). */
int imops_film_layers(const ImopsFilmParams *params, int *layers);

/* Absorbed exposure per layer from absolute-luminance ACEScg
 * (exposure/mod.rs:45-137 with absorption.rs:24-108): rgb -> E planes. */
int imops_film_expose(const float *rgb, int w, int h, const ImopsFilmParams *params, float *planes,
                      imops_stream_t stream);

/* Local scatter and the wide halation bounce, in place (halation.rs:24-93). */
int imops_film_halation(float *planes, int w, int h, const ImopsFilmParams *params, imops_stream_t stream);

/* Development, in place: capture LUT with reciprocity, reduction to image-dye
 * densities (planes) and mask densities (mask, E planes), DIR inhibition and
 * adjacency (capture.rs:61-88, reduction.rs:16-68, diffusion.rs:11-84). */
int imops_film_develop(float *planes, float *mask, int w, int h, const ImopsFilmParams *params,
                       imops_stream_t stream);

/* Seeded grain on the image-dye planes, in place (grain.rs:53-100); nothing
 * when params->grain is 0. */
int imops_film_grain(float *planes, int w, int h, const ImopsFilmParams *params, imops_stream_t stream);

/* Scan of the densities to ACEScg RGB (scan/mod.rs:24-30,
 * densitometry.rs:13-73): planes + mask -> rgb. */
int imops_film_scan(const float *planes, const float *mask, int w, int h, const ImopsFilmParams *params,
                    float *rgb, imops_stream_t stream);

/* PositiveLinear inversion in place (invert.rs:36-108, with the mid-grey
 * negative of film/mod.rs:136-151); nothing for NegativeLinear or a
 * reversal stock. */
int imops_film_invert(float *rgb, int w, int h, const ImopsFilmParams *params, imops_stream_t stream);

/* ---- fused forward -------------------------------------------------------
 * The path Demosaic -> CFACoeffs -> Exp -> CST -> Film (the module chain of
 * run_pixel_pipeline, pichromatic-pipeline/src/pipeline.rs:4-13, with the
 * modules of modules.rs:529-668 and 841-876) as one call: the black/white
 * scaling of the frame, the demosaic with WB / exposure / camera CST fused
 * into its output stage, then the film simulation.  Outputs are the
 * same as calling the stage entry points one after another. */
typedef struct {
    int demosaic;           /* IMOPS_DEMOSAIC_AMAZE or IMOPS_DEMOSAIC_MARKESTEIJN */
    const char *cfa;        /* CFA pattern of the uncropped frame */
    float clip_pt;          /* AMaZE clip point (1.0) */
    float wb[4];            /* metadata.wb_coeffs (CFACoeffs) */
    int n_gain;             /* exposure steps applied after WB, in order (0..2) */
    float ev[2];            /* their EV values: rgb *= 2^ev */
    int target;             /* CST target IMOPS_CS_*, or IMOPS_CS_CAMERA for no CST */
    float calib_d65[9];     /* metadata.calibration_matrix_d65 */
    int film;               /* 1: run the film simulation after the CST (target must be ACEScg) */
    ImopsFilmParams film_params;
    ImopsBaselineFilm baseline; /* used when film_params.stock == IMOPS_STOCK_BASELINE81 */
} ImopsDevelopParams;

/* Forward from a u16 sensor frame: crop (crop_x, crop_y, crop_w, crop_h),
 * per-cell black/white levels over a period_w x period_h CFA period (HOST
 * arrays), output crop_w*crop_h*3 f32 on the device.  The CFA phase is
 * shifted by the crop origin (demosaic::get_cfa, demosaic.rs:93-98). */
int imops_develop_u16(const uint16_t *raw, int raw_w, int raw_h, int crop_x, int crop_y, int crop_w, int crop_h,
                      const float *black, const float *white, int period_w, int period_h,
                      const ImopsDevelopParams *params, float *rgb, imops_stream_t stream);

/* Forward from an already scaled and cropped f32 mosaic (Image.raw_data);
 * shift_x/shift_y: the crop origin used for the CFA phase. */
int imops_develop_f32(const float *mosaic, int w, int h, int shift_x, int shift_y, const ImopsDevelopParams *params,
                      float *rgb, imops_stream_t stream);

/* Number of kernels this library has launched in this process (evidence
 * counter for benchmarks; monotone, thread-safe). */
uint64_t imops_launch_count(void);

/* Tensor-core waits that gave up on the current device since the process
 * started (a bounded wait for an MMA's completion expired; the kernel then
 * skips its remaining MMAs and its output is not valid).  Waits for the
 * device.  0 in normal operation. */
int imops_tensor_timeouts(unsigned *count);

/* ---- adjoints (no counterpart in the reference, which has no gradients) ----
 * Parameters of the differentiable colour + film model, from demosaiced
 * camera RGB x (demosaic decisions held fixed):
 *   y = 2^ev (wb * x);  a = matrix y (ACEScg);  exposure a -> 3 layers;
 *   halation G_sigma * max(0, a_R - threshold) added with hal_strength * bleed;
 *   logistic curves (dmax, k, x0); 81-bin scan -> out (ACEScg negative).
 * Fixed settings (threshold, tap radius) come from an ImopsBaselineFilm;
 * grain is off.  24 parameters, gradient order as the fields below. */
typedef struct {
    float wb[3];
    float matrix[9];        /* camera RGB -> ACEScg, row-major */
    float ev;
    float dmax[3], k[3], x0[3];
    float hal_strength;
    float hal_sigma;
} ImopsFilmGradParams;

/* out (w*h*3) = model(cam_rgb); fixed may be NULL (defaults). */
int imops_param_forward(const float *cam_rgb, int w, int h, const ImopsFilmGradParams *params,
                        const ImopsBaselineFilm *fixed, float *out, imops_stream_t stream);

/* Adds the gradient of a scalar loss w.r.t. the 24 parameters to grad[0..23]
 * and the loss to grad[24] (DEVICE doubles, not cleared: accumulate over a
 * batch).  Either g_out (dL/dout, w*h*3) is given, or target is and the loss
 * is loss_scale * sum((out - target)^2) (e.g. loss_scale = 1/(3 N) for an
 * MSE over N pixels).  Halation is recomputed, not stored.  Requires
 * w, h > hal_radius + 1. */
int imops_param_backward(const float *cam_rgb, const float *g_out, const float *target, float loss_scale, int w,
                         int h, const ImopsFilmGradParams *params, const ImopsBaselineFilm *fixed, double *grad,
                         imops_stream_t stream);

/* ---- pipeline-level C-ABI -------------------------------------------------
 * The embedding interface of pichromatic-pipeline/src/extern_pipeline.rs
 * (get_pixel_pipeline_c :326-341, run_pixel_pipeline_c :343-359,
 * get_image_rgb_data_c :361-397, free_* :399-455, get_last_error_c :27-38)
 * with the same names, ownership and NULL-on-error convention, running the
 * module chain of run_pixel_pipeline (pipeline.rs:4-13) on the GPU.  HOST
 * buffers in and out; images live on the device between modules.
 * Decoding raw files (get_raw_img, rawler) stays on the reference: images
 * are created from the decoded sensor frame or an already scaled mosaic. */
typedef struct ImopsImage ImopsImage;        /* Image (pichromatic/src/pixel.rs:23-27) */
typedef struct ImopsPipeline ImopsPipeline;  /* PipelineConfig (pichromatic-pipeline/src/config.rs:9-11) */

/* The ImageMetadata fields the path reads (pichromatic/src/image.rs:7-50). */
typedef struct {
    const char *cfa;            /* metadata.cfa pattern of the uncropped frame */
    int crop_x, crop_y;         /* metadata.crop_area origin */
    int crop_w, crop_h;         /* crop size (u16 frames; 0 = whole frame) */
    int has_wb;
    float wb_coeffs[4];
    int has_calibration;
    float calibration_matrix_d65[9];
    float black_level, white_level;   /* scaling levels of u16 frames (same for every CFA cell) */
    int has_baseline_exposure;
    float baseline_exposure;
    int has_shutter;
    float shutter_seconds;
    int has_f_number;
    float f_number;
    int has_iso;
    float iso;
} ImopsImageMeta;

/* Image from a decoded u16 sensor frame (what rawler returns before
 * apply_scaling): the Demosaic module scales, crops and demosaics it. */
ImopsImage *new_raw_image_u16_c(const uint16_t *raw, size_t width, size_t height, const ImopsImageMeta *meta);

/* Image from an already scaled and cropped f32 mosaic (Image.raw_data after
 * parse_raw_image, extern_pipeline.rs:239-324); width/height are the cropped
 * size and crop_x/crop_y give the CFA phase. */
ImopsImage *new_raw_image_f32_c(const float *raw_data, size_t width, size_t height, const ImopsImageMeta *meta);

/* Image from interleaved f32 RGB in a colour space (IMOPS_CS_*, or
 * IMOPS_CS_CAMERA for demosaiced camera RGB). */
ImopsImage *new_rgb_image_c(const float *rgb, size_t width, size_t height, int color_space,
                            const ImopsImageMeta *meta);

/* parse_config (config.rs:13-34): TOML, else JSON, list of
 * [[pipeline_modules]] tables matched by case-insensitive name.  NULL on
 * error (get_last_error_c). */
ImopsPipeline *get_pixel_pipeline_c(const uint8_t *config, size_t config_len);

/* Runs every module in order on the image; returns `image`, or NULL on error. */
ImopsImage *run_pixel_pipeline_c(ImopsImage *image, ImopsPipeline *pipeline);

/* RGB as u8 (clamp(0,1)*255 truncated), width*height*3 bytes; free with
 * free_rgb_buffer_c(ptr, len). */
const uint8_t *get_image_rgb_data_c(ImopsImage *image, size_t *out_width, size_t *out_height, size_t *out_len);

/* Copies the f32 RGB (width*height*3 floats) into a host buffer. */
int get_image_rgb_f32_c(ImopsImage *image, float *out, size_t n_floats);

/* Current width, height and colour space (IMOPS_CS_*). */
int get_image_info_c(const ImopsImage *image, size_t *width, size_t *height, int *color_space);

/* Metadata as JSON (free with free_string_c). */
char *get_image_metadata_c(const ImopsImage *image);

/* get_pipeline_schema (modules.rs:917-923) as JSON (free with free_string_c). */
char *get_pipeline_schema_c(void);

/* Last error message of this thread as a new string (free_string_c), or NULL. */
char *get_last_error_c(void);

void free_image_c(ImopsImage *image);
void free_pipeline_c(ImopsPipeline *pipeline);
void free_rgb_buffer_c(uint8_t *ptr, size_t len);
void free_string_c(char *ptr);

#ifdef __cplusplus
}
#endif

#endif /* IMOPS_B200_H */
