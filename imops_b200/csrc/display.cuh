// display.cuh -- the per-pixel display stages after the film scan
// (HighlightReconstruction, Contrast, LCH, SigmoidToneMap, Gamma) and the
// colour-space conversions between XyzD65, LinearSrgb, Srgb, AcesCg and
// Oklch, as one chain of per-pixel ops run in a single pass over the image.
#pragma once

#include "common.cuh"

namespace imops {
namespace display {

enum OpKind : int {
    OP_GAIN = 1,    // rgb *= s[0..2]                         (cfa_coeffs.rs:4-12, exp.rs:4-11)
    OP_HIGHLIGHT,   // g from r, g, b and clip_g = s[0]        (highlight_reconstruction.rs:5-13)
    OP_CONTRAST,    // 0.185 * (x / 0.185)^s[0]                (contrast.rs:4-8)
    OP_GAMMA,       // x <= 0 ? 0 : x^s[0], s[0] = 1/max(g,1e-6) (tone_map.rs:38-49)
    OP_SCALE,       // rgb *= s[0..2] on Oklch components      (lch.rs:14-17)
    OP_CST,         // colour-space conversion, steps in `flags` (cst.rs:6-10)
    OP_SIGMOID,     // sigmoid tone map with gamut compression (tone_map.rs:18-33)
};

// Steps of OP_CST, applied in this order.
enum CstFlag : int {
    CST_DECODE = 1,       // sRGB transfer decode
    CST_FROM_OKLCH = 2,   // Oklch -> linear sRGB
    CST_M0 = 4,           // m[0] mat-vec
    CST_M1 = 8,           // m[1] mat-vec
    CST_TO_OKLCH = 16,    // linear sRGB -> Oklch
    CST_ENCODE = 32,      // sRGB transfer encode
};

struct Op {
    int kind;
    int flags;
    float s[4];
    float m[4][9];  // OP_CST: m[0], m[1]; OP_SIGMOID: AcesCg->XYZ, XYZ->lin sRGB, lin sRGB->XYZ, XYZ->AcesCg
};

constexpr int MAX_OPS = 16;

struct Chain {
    int n;
    Op op[MAX_OPS];
};

// Host-side builders.  Each appends to `c` and returns IMOPS_OK, or an
// error status with the message set (a full chain, an unknown space).
int add_gain(Chain& c, float r, float g, float b);
int add_highlight(Chain& c, float clip_g);
int add_contrast(Chain& c, float value);
int add_gamma(Chain& c, float gamma);
// Conversion from colour space `src` to `dst` (IMOPS_CS_*; src may be
// IMOPS_CS_CAMERA with `camera_fwd` the camera -> XYZ matrix).
int add_cst(Chain& c, int src, int dst, const float* camera_fwd);
// lch (lch.rs:5-18) on an image in colour space `cs`.
int add_lch(Chain& c, int cs, float lc, float cc, float hc);
int add_sigmoid(Chain& c);

// Runs the chain in place over n interleaved RGB pixels on stream s.
int run(float* rgb, size_t n, const Chain& c, cudaStream_t s, const char* what);

}  // namespace display
}  // namespace imops
