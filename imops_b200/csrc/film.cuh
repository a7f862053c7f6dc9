// film.cuh -- device-side description of a film stock for the spectral film
// simulation (pichromatic/src/film/**), built on the host from the stock
// definitions (film_host.cpp) and passed to the kernels by value.
#pragma once

#include "common.cuh"

namespace imops {
namespace film {

constexpr int MAXE = 8;     // emulsion layers (FujiPro400H has 7)
constexpr int NB16 = 16;    // the reference grid, 400..700 nm step 20
constexpr int NB81 = 81;    // the baseline preset grid, 380..780 nm step 5
constexpr int LUTN = 64;    // DevelopableFractionLut entries (capture.rs:37-58)
constexpr int HAL_R = 64;   // fixed halation radius of the baseline preset

enum Model { MODEL_REFERENCE = 0, MODEL_BASELINE = 1 };

// Per-pixel exposure: w = max(0, Minv * rgb) (basis weights), then
// a_e = sum_k w_k * A[k][e].  Exact algebraic collapse of the reference's
// per-pixel spectrum upsample + Beer-Lambert stack walk + band integral
// (exposure/mod.rs:68-81, absorption.rs:24-108), whose layer transmittances
// do not depend on the pixel.
struct ExposeSpec {
    int E;
    float minv[9];
    float A[3][MAXE];
    int hal_src;        // baseline preset: also emit max(0, R - hal_threshold)
    float hal_threshold;
};

// Spectral scan: d(l) = sum_e Dimg_e*eps_e(l) + Dmask_e*meps_e(l);
// T = 2^(-d) * illum(l) (eps pre-scaled by log2(10));
// rgb_c = sum_l C[l][c] * T(l)  (C folds trapezoid weights, CMFs, XYZ->AP1 and
// the 1/peak(Dmin) normalisation; densitometry.rs:13-73).
struct ScanSpec16 {
    int E;
    float eps[MAXE][NB16];
    float meps[MAXE][NB16];
    float C[NB16][3];
};

struct ScanSpec81 {
    float eps[3][NB81];
    float C[NB81][3];
};

// Everything the reference-model pipeline needs after exposure.
struct RefSpec {
    int E;
    // spatial exposure effects (halation.rs:24-93)
    float sigma_local, local_mix, sigma_wide;
    float hal_gain[MAXE];
    // capture LUT + reciprocity (capture.rs:61-88, exposure/mod.rs:97-115)
    float eta[MAXE];
    float lut_log[MAXE][LUTN];
    float lut_frac[MAXE][LUTN];
    // reduce (reduction.rs:16-68)
    float dmax[MAXE], inv_gamma[MAXE], mask_scale[MAXE];
    int reversal[MAXE], has_mask[MAXE];
    // DIR + adjacency (diffusion.rs:11-84)
    float sigma_dir;
    float dir[MAXE][MAXE];
    int dir_any;
    float sigma_adj, beta;
    // grain (grain.rs:53-100)
    float sigma_grain;
    float kappa[MAXE];
    // invert (invert.rs) inputs; mid is measured on the GPU
    float dmin_norm[3];
    float box_iso;
    int any_reversal;
};

// The baseline preset's per-pixel constants.
struct BaselineSpec {
    float dmax[3], k[3], x0[3];
    float hal_strength;
    float bleed[3];
    float grain_sigma;
};

struct Stock {
    int model;
    ExposeSpec expose;
    RefSpec ref;
    ScanSpec16 scan16;
    BaselineSpec base;
    ScanSpec81 scan81;
    float hal_taps[2 * HAL_R + 1];  // baseline preset halation taps
    float grain_blur;               // baseline preset noise blur sigma (px)
};

// 2^x with the hardware approximation (PTX ex2.approx.ftz.f32: relative error
// about 2^-22, subnormal results flushed).  The spectral scans raise 2 to
// minus an optical density; with densities of a few units no result is
// subnormal, and the film's tolerance is 1e-4.
__device__ __forceinline__ float ex2_fast(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Builds the device description of stock `stock_id` for an image of width W
// (pixel pitch = frame width / W, types.rs:45-48) and the given shutter.
// Returns IMOPS_OK or an error code (unknown stock / format).
int build_stock(int stock_id, int film_format, int W, float shutter_seconds, const ImopsBaselineFilm* baseline,
                Stock* out, float* pitch_um);

// Gaussian taps of the reference blur (blur.rs:39-55): radius max(ceil(3 sigma),1),
// exp(-x^2/(2 sigma^2)) in f32, normalised by their f32 sum.  Returns the radius.
int gaussian_taps(float sigma, float* taps, int max_taps);

// Separable-blur launchers shared with the adjoint (film.cu).  taps: 2R+1
// weights (R <= 64), mirror reflection at the edges (blur.rs:70-89).
int blur_rows(const float* in, float* out, int W, int H, const float* taps, int R, cudaStream_t s);
// out = blur_cols(in) (add == 0) or out += blur_cols(in) (add == 1)
int blur_cols(const float* in, float* out, int W, int H, const float* taps, int R, int add, cudaStream_t s);
int grid_for_n(size_t n);

// Relative -> absolute luminance of a value at sunny-16 for a box ISO
// (film/mod.rs:155-166).
float relative_to_absolute_y(float y, float box_iso);

// The baseline 81-bin preset: its working-set size for a W x H image, its
// stock description, and its kernels run with the working set at `scratch`
// (256-byte aligned, at least baseline_scratch_bytes(W, H) bytes).
size_t baseline_scratch_bytes(int W, int H);
int baseline_stock(int W, const ImopsBaselineFilm& P, Stock* st);
int baseline_forward_in(float* rgb, int W, int H, const ImopsBaselineFilm& P, const Stock& st, void* scratch,
                        cudaStream_t s);

}  // namespace film
}  // namespace imops
