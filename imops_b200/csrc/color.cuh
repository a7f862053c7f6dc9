// color.cuh -- host-side colour constants and the per-pixel colour epilogue
// shared by the stage kernels (color.cu) and the fused pipeline.
#pragma once

#include "common.cuh"

namespace imops {
namespace color {

// camera -> XYZ(D65) matrix of camera_cst, pichromatic/src/cst.rs:12-38 and
// pseudo_inverse_matrix cst.rs:51-95, in f32 in the reference's order.
void camera_forward_matrix(const float calib[9], float fwd[9]);

// XYZ(D65) -> target 3x3 (row-major) for IMOPS_CS_{XYZD65,LINEAR_SRGB,SRGB,ACESCG};
// false for other targets.  AcesCg uses the reference's own XYZ->AP1 matrix
// (film/exposure/upsample.rs:34-38); linear sRGB the CSS Color 4 matrix.
bool xyz_to_target(int target, float m[9]);

// 2^ev in f32 as exp.rs:5 computes it (glibc powf, as Rust's f32::powf).
float exp_value(float ev);

// Absolute-luminance gain K*N^2/(t*S) (film/exposure/radiance.rs:19-31), f64 -> f32.
float luminance_gain(float shutter, float f_number, float iso);

// Per-pixel colour after demosaic, applied in the reference's module order:
// WB (cfa_coeffs.rs:4-12), exposure gain(s) (exp.rs:4-11), camera CST
// (cst.rs:39-46).  Each step is its own f32 multiply/mat-vec so the
// rounding matches the separate module passes.
struct Epilogue {
    float wb[3];
    int n_gain;       // 0..4 scalar gains applied one after another
    float gain[4];
    int do_cst;
    float fwd[9];
    float tgt[9];
    int srgb;         // apply the sRGB transfer after the target matrix
    int src_srgb;     // decode an sRGB-encoded input before the first matrix

    __device__ __forceinline__ void apply(float& r, float& g, float& b) const {
        r = r * wb[0];
        g = g * wb[1];
        b = b * wb[2];
        for (int k = 0; k < n_gain; k++) {
            r = r * gain[k];
            g = g * gain[k];
            b = b * gain[k];
        }
        if (do_cst) {
            if (src_srgb) {
                r = srgb_decode(r);
                g = srgb_decode(g);
                b = srgb_decode(b);
            }
            float x = fwd[0] * r + fwd[1] * g + fwd[2] * b;
            float y = fwd[3] * r + fwd[4] * g + fwd[5] * b;
            float z = fwd[6] * r + fwd[7] * g + fwd[8] * b;
            r = tgt[0] * x + tgt[1] * y + tgt[2] * z;
            g = tgt[3] * x + tgt[4] * y + tgt[5] * z;
            b = tgt[6] * x + tgt[7] * y + tgt[8] * z;
            if (srgb) {
                r = srgb_encode(r);
                g = srgb_encode(g);
                b = srgb_encode(b);
            }
        }
    }

    __device__ __forceinline__ static float srgb_decode(float v) {
        float a = fabsf(v);
        float l = a <= 0.04045f ? a / 12.92f : powf((a + 0.055f) / 1.055f, 2.4f);
        return v < 0.0f ? -l : l;
    }

    // sRGB transfer with odd symmetry (IEC 61966-2-1).
    __device__ __forceinline__ static float srgb_encode(float v) {
        float a = fabsf(v);
        float e = a <= 0.0031308f ? 12.92f * a : 1.055f * powf(a, 1.0f / 2.4f) - 0.055f;
        return v < 0.0f ? -e : e;
    }
};

// Colour space -> XYZ(D65) 3x3 for IMOPS_CS_{XYZD65,LINEAR_SRGB,SRGB (after
// decoding),ACESCG}; false otherwise.
bool to_xyz(int space, float m[9]);

// Builds an identity epilogue (no-op).
Epilogue identity_epilogue();

// Applies `e` in place to n interleaved RGB pixels on stream s.
int run_epilogue(float* rgb, size_t n, const Epilogue& e, cudaStream_t s, const char* what);

// Grid size for a grid-stride loop over n items.
int stream_grid(size_t n, int block);

}  // namespace color
}  // namespace imops
