/*
 * color.c -- CPU oracle for the per-pixel colour stages of the path.
 *
 * TEST INFRASTRUCTURE (see oracle_common.h).
 *  - scale:   black/white scaling + crop copy.  The reference delegates the
 *             scaling to rawler 0.7.x RawImage::apply_scaling
 *             (pichromatic-pipeline/src/extern_pipeline.rs:258-267) whose
 *             source is not in the reference tree: restated as
 *             (v - black[site]) / (white[site] - black[site]) with no clamp,
 *             site = full-frame CFA cell.  PARITY UNPINNED for this formula.
 *             The crop copy follows demosaic::crop_and_normalize
 *             (pichromatic/src/demosaic.rs:61-91).
 *  - wb:      cfa_coeffs (pichromatic/src/cfa_coeffs.rs:4-12).
 *  - exp:     exp (pichromatic/src/exp.rs:4-11): value = powf(2, ev).
 *  - baseline exposure: modules.rs:335-373 with
 *             film/exposure/radiance.rs:19-31 (gain in f64, cast to f32).
 *  - camera CST: camera_cst + pseudo_inverse_matrix
 *             (pichromatic/src/cst.rs:12-95), then XYZ(D65) -> target.  The
 *             last step is the `color` crate 0.3.x ColorSpaceTag::convert,
 *             not vendored: restated with the reference's own XYZ->AP1 matrix
 *             (film/exposure/upsample.rs:34-38) for AcesCg and the
 *             CSS Color 4 / IEC 61966-2-1 matrix and transfer for
 *             LinearSrgb / Srgb.  PARITY UNPINNED for that step.
 */
#include "oracle_common.h"

#include <string.h>

int OSYM(oracle_scale_u16)(const uint16_t *raw, int raw_w, int raw_h, int crop_x, int crop_y,
                           int crop_w, int crop_h, const real *black, const real *white, int pw, int ph,
                           real *out)
{
    if (!raw || !out || !black || !white || pw <= 0 || ph <= 0) return ORACLE_ERR_ARG;
    if (crop_x < 0 || crop_y < 0 || crop_w <= 0 || crop_h <= 0 || crop_x + crop_w > raw_w ||
        crop_y + crop_h > raw_h)
        return ORACLE_ERR_ARG;
    for (int y = 0; y < crop_h; y++)
        for (int x = 0; x < crop_w; x++) {
            int sy = crop_y + y, sx = crop_x + x;
            int site = (sy % ph) * pw + (sx % pw);
            real v = (real)raw[(size_t)sy * raw_w + sx];
            out[(size_t)y * crop_w + x] = (v - black[site]) / (white[site] - black[site]);
        }
    return ORACLE_OK;
}

void OSYM(oracle_wb)(real *rgb, size_t n, const real wb[4])
{
    for (size_t i = 0; i < n; i++) {
        rgb[3 * i + 0] = rgb[3 * i + 0] * wb[0];
        rgb[3 * i + 1] = rgb[3 * i + 1] * wb[1];
        rgb[3 * i + 2] = rgb[3 * i + 2] * wb[2];
    }
}

void OSYM(oracle_exp)(real *rgb, size_t n, real ev)
{
#ifdef ORACLE_F32
    real value = powf(2.0f, ev);
#else
    real value = pow(2.0, ev);
#endif
    for (size_t i = 0; i < 3 * n; i++) rgb[i] = rgb[i] * value;
}

/* BaselineExposureCompensation: exposure by baseline_ev when |ev| > 1e-6,
 * then the absolute-luminance gain K*N^2/(t*S) when t, N, S are all > 0.
 * Returns 1 when the gain was applied, 0 when metadata was missing. */
int OSYM(oracle_baseline_exposure)(real *rgb, size_t n, real baseline_ev, real t, real fnum, real iso)
{
    if (RABS(baseline_ev) > K(1e-6)) OSYM(oracle_exp)(rgb, n, baseline_ev);
    if (!(t > 0 && fnum > 0 && iso > 0)) return 0;
    double kv = 12.5 * 1.0;
    double g64 = kv * ((double)fnum * (double)fnum) / ((double)t * (double)iso);
    real gain = (real)(float)g64;
    for (size_t i = 0; i < 3 * n; i++) rgb[i] = rgb[i] * gain;
    return 1;
}

/* pseudo_inverse_matrix for a 3x3 input (cst.rs:51-95). */
static void pinv3(const real m[3][3], real res[3][3])
{
    real work[3][6];
    real tmp[3][3];
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 6; j++) work[i][j] = (j == i + 3) ? K(1.0) : K(0.0);
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) work[i][j] += m[k][i] * m[k][j];
    }
    for (int i = 0; i < 3; i++) {
        real num = work[i][i];
        for (int j = 0; j < 6; j++) work[i][j] /= num;
        for (int k = 0; k < 3; k++) {
            if (k == i) continue;
            num = work[k][i];
            for (int j = 0; j < 6; j++) work[k][j] -= work[i][j] * num;
        }
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            tmp[i][j] = K(0.0);
            for (int k = 0; k < 3; k++) tmp[i][j] += work[j][k + 3] * m[i][k];
        }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) res[i][j] = tmp[j][i];
}

/* camera -> XYZ(D65) matrix of camera_cst (cst.rs:12-38). */
void OSYM(oracle_camera_forward_matrix)(const real calib[9], real fwd[9])
{
    const real xyz[3] = {K(0.95042), K(1.0), K(1.08890)};
    real rgbd65[3], mult[3] = {K(1.0), K(1.0), K(1.0)};
    real x2c[3][3], f[3][3];
    for (int i = 0; i < 3; i++)
        rgbd65[i] = calib[i * 3] * xyz[0] + calib[i * 3 + 1] * xyz[1] + calib[i * 3 + 2] * xyz[2];
    for (int i = 0; i < 3; i++)
        if (rgbd65[i] > K(0.0)) mult[i] = K(1.0) / rgbd65[i];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) x2c[i][j] = calib[i * 3 + j] * mult[i];
    pinv3(x2c, f);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) fwd[i * 3 + j] = f[i][j];
}

/* Target colour spaces (numbering shared with the C-ABI). */
#define CS_XYZD65 0
#define CS_LINEAR_SRGB 1
#define CS_SRGB 2
#define CS_ACESCG 3

/* XYZ(D65) -> target matrix; returns 0 when the target is not a 3x3 map. */
int OSYM(oracle_xyz_to_target_matrix)(int target, real m[9])
{
    static const double xyz_to_lsrgb[9] = {12831.0 / 3959.0,     -329.0 / 214.0,       -1974.0 / 3959.0,
                                           -851781.0 / 878810.0, 1648619.0 / 878810.0, 36519.0 / 878810.0,
                                           705.0 / 12673.0,      -2585.0 / 12673.0,    705.0 / 667.0};
    static const double xyz_to_ap1[9] = {1.6410233797,  -0.3248032942, -0.2364246952,
                                         -0.6636628587, 1.6153315917,  0.0167563477,
                                         0.0117218943,  -0.0082844165, 0.9883948585};
    const double *src = NULL;
    if (target == CS_XYZD65) {
        for (int i = 0; i < 9; i++) m[i] = (i % 4 == 0) ? K(1.0) : K(0.0);
        return 1;
    }
    if (target == CS_LINEAR_SRGB || target == CS_SRGB) src = xyz_to_lsrgb;
    if (target == CS_ACESCG) src = xyz_to_ap1;
    if (!src) return 0;
    for (int i = 0; i < 9; i++) m[i] = (real)(float)src[i];
    return 1;
}

/* sRGB transfer with odd symmetry for negative values (IEC 61966-2-1). */
static real srgb_encode(real v)
{
    real a = RABS(v);
    real e;
#ifdef ORACLE_F32
    e = a <= 0.0031308f ? 12.92f * a : 1.055f * powf(a, 1.0f / 2.4f) - 0.055f;
#else
    e = a <= 0.0031308 ? 12.92 * a : 1.055 * pow(a, 1.0 / 2.4) - 0.055;
#endif
    return v < 0 ? -e : e;
}

int OSYM(oracle_camera_cst)(real *rgb, size_t n, const real calib[9], int target)
{
    real fwd[9], tm[9];
    if (!OSYM(oracle_xyz_to_target_matrix)(target, tm)) return ORACLE_ERR_ARG;
    OSYM(oracle_camera_forward_matrix)(calib, fwd);
    for (size_t p = 0; p < n; p++) {
        real r = rgb[3 * p], g = rgb[3 * p + 1], b = rgb[3 * p + 2];
        real x = fwd[0] * r + fwd[1] * g + fwd[2] * b;
        real y = fwd[3] * r + fwd[4] * g + fwd[5] * b;
        real z = fwd[6] * r + fwd[7] * g + fwd[8] * b;
        real o0 = tm[0] * x + tm[1] * y + tm[2] * z;
        real o1 = tm[3] * x + tm[4] * y + tm[5] * z;
        real o2 = tm[6] * x + tm[7] * y + tm[8] * z;
        if (target == CS_SRGB) {
            o0 = srgb_encode(o0);
            o1 = srgb_encode(o1);
            o2 = srgb_encode(o2);
        }
        rgb[3 * p] = o0;
        rgb[3 * p + 1] = o1;
        rgb[3 * p + 2] = o2;
    }
    return ORACLE_OK;
}
