/*
 * display.c -- CPU oracle for the per-pixel display stages that follow the
 * film scan, and for colour-space conversions to and from Oklch.
 *
 * TEST INFRASTRUCTURE (see oracle_common.h).
 *  - highlight:  highlight_reconstruction
 *                (pichromatic/src/highlight_reconstruction.rs:5-13).
 *  - contrast:   contrast (pichromatic/src/contrast.rs:4-8), MIDDLE_GRAY
 *                0.185 (pichromatic/src/pixel.rs:36).
 *  - gamma:      gamma_encode (pichromatic/src/tone_map.rs:38-49).
 *  - sigmoid:    sigmoid tone map (tone_map.rs:18-33) with square_sigmoid
 *                (:6-16), the ACES reference gamut compression
 *                (gamut_compress_pixel :133-171, compress_value :71-125,
 *                RgcParams::default :59-69) and PixelOps::luminance
 *                (pixel.rs:33-35, 43-47).
 *  - lch:        lch (pichromatic/src/lch.rs:5-18).
 *  - cst:        cst (pichromatic/src/cst.rs:6-10) between XyzD65,
 *                LinearSrgb, Srgb, AcesCg and Oklch.
 *
 * The conversions are the `color` crate 0.3.3 ColorSpaceTag::convert
 * (Cargo.lock), which is not vendored.  They are restated from published
 * definitions and are PARITY UNPINNED:
 *  - Oklab from linear sRGB and back: B. Ottosson, "A perceptual color
 *    space for image processing" (2020), with its linear-sRGB matrices and
 *    a cube root;
 *  - Oklch from Oklab (CSS Color 4): C = hypot(a, b), h = atan2(b, a) in
 *    degrees moved to [0, 360), and a = C cos h, b = C sin h back;
 *  - AcesCg <-> linear sRGB through XYZ(D65), with the AP1 matrices the
 *    reference itself uses (film/exposure/upsample.rs:34-45) and the
 *    CSS Color 4 sRGB matrices, as the camera CST does.
 * Between two matrix spaces the conversion is decode -> to XYZ -> to the
 * target -> encode, exactly as the CUDA library's CST.
 */
#include "oracle_common.h"

#define CS_XYZD65 0
#define CS_LINEAR_SRGB 1
#define CS_SRGB 2
#define CS_ACESCG 3
#define CS_OKLCH 4

typedef struct {
    real m[9];
} M3;

static const double LSRGB_TO_XYZ[9] = {506752.0 / 1228815.0, 87881.0 / 245763.0,  12673.0 / 70218.0,
                                       87098.0 / 409605.0,   175762.0 / 245763.0, 12673.0 / 175545.0,
                                       7918.0 / 409605.0,    87881.0 / 737289.0,  1001167.0 / 1053270.0};
static const double XYZ_TO_LSRGB[9] = {12831.0 / 3959.0,     -329.0 / 214.0,       -1974.0 / 3959.0,
                                       -851781.0 / 878810.0, 1648619.0 / 878810.0, 36519.0 / 878810.0,
                                       705.0 / 12673.0,      -2585.0 / 12673.0,    705.0 / 667.0};
static const double AP1_TO_XYZ[9] = {0.6624541811,  0.1340042065, 0.1561876870, 0.2722287168, 0.6740817658,
                                     0.0536895174,  -0.0055746495, 0.0040607335, 1.0103391003};
static const double XYZ_TO_AP1[9] = {1.6410233797,  -0.3248032942, -0.2364246952, -0.6636628587, 1.6153315917,
                                     0.0167563477,  0.0117218943,  -0.0082844165, 0.9883948585};

/* Ottosson's Oklab: linear sRGB -> LMS, LMS' -> Lab and the inverses. */
static const double OK_M1[9] = {0.4122214708, 0.5363325363, 0.0514459929, 0.2119034982, 0.6806995451,
                                0.1073969566, 0.0883024619, 0.2817188376, 0.6299787005};
static const double OK_M2[9] = {0.2104542553, 0.7936177850, -0.0040720468, 1.9779984951, -2.4285922050,
                                0.4505937099, 0.0259040371, 0.7827717662,  -0.8086757660};
static const double OK_M2I[9] = {1.0, 0.3963377774,  0.2158037573,  1.0, -0.1055613458,
                                 -0.0638541728, 1.0, -0.0894841775, -1.2914855480};
static const double OK_M1I[9] = {4.0767416621,  -3.3077115913, 0.2309699292,  -1.2684380046, 2.6097574011,
                                 -0.3413193965, -0.0041960863, -0.7034186147, 1.7076147010};

static M3 mk(const double *d)
{
    M3 r;
    for (int i = 0; i < 9; i++) r.m[i] = (real)(float)d[i];
    return r;
}

static void mv(const M3 *a, real v[3])
{
    const real *m = a->m;
    real x = m[0] * v[0] + m[1] * v[1] + m[2] * v[2];
    real y = m[3] * v[0] + m[4] * v[1] + m[5] * v[2];
    real z = m[6] * v[0] + m[7] * v[1] + m[8] * v[2];
    v[0] = x;
    v[1] = y;
    v[2] = z;
}

#ifdef ORACLE_F32
#define RPOW powf
#define RCBRT cbrtf
#define RATAN2 atan2f
#define RHYPOT hypotf
#define RSIN sinf
#define RCOS cosf
#else
#define RPOW pow
#define RCBRT cbrt
#define RATAN2 atan2
#define RHYPOT hypot
#define RSIN sin
#define RCOS cos
#endif

static real srgb_dec(real v)
{
    real a = RABS(v);
    real l = a <= K(0.04045) ? a / K(12.92) : RPOW((a + K(0.055)) / K(1.055), K(2.4));
    return v < 0 ? -l : l;
}

static real srgb_enc(real v)
{
    real a = RABS(v);
    real e = a <= K(0.0031308) ? K(12.92) * a : K(1.055) * RPOW(a, K(1.0) / K(2.4)) - K(0.055);
    return v < 0 ? -e : e;
}

/* linear sRGB -> Oklch in place */
static void lin_to_oklch(real v[3])
{
    M3 m1 = mk(OK_M1), m2 = mk(OK_M2);
    mv(&m1, v);
    v[0] = RCBRT(v[0]);
    v[1] = RCBRT(v[1]);
    v[2] = RCBRT(v[2]);
    mv(&m2, v);
    real c = RHYPOT(v[1], v[2]);
    real h = RATAN2(v[2], v[1]) * K(57.29577951308232);
    if (h < 0) h = h + K(360.0);
    v[1] = c;
    v[2] = h;
}

/* Oklch -> linear sRGB in place */
static void oklch_to_lin(real v[3])
{
    M3 m2i = mk(OK_M2I), m1i = mk(OK_M1I);
    real hr = v[2] * K(0.017453292519943295);
    real c = v[1];
    v[1] = c * RCOS(hr);
    v[2] = c * RSIN(hr);
    mv(&m2i, v);
    v[0] = v[0] * v[0] * v[0];
    v[1] = v[1] * v[1] * v[1];
    v[2] = v[2] * v[2] * v[2];
    mv(&m1i, v);
}

static int valid_cs(int cs) { return cs >= CS_XYZD65 && cs <= CS_OKLCH; }

/* One pixel from `src` to `dst` (cst.rs:6-10). */
static void convert(int src, int dst, real v[3])
{
    if (src == dst) return;
    if (src == CS_OKLCH || dst == CS_OKLCH) {
        /* to linear sRGB */
        if (src == CS_OKLCH) oklch_to_lin(v);
        else if (src == CS_SRGB) {
            for (int i = 0; i < 3; i++) v[i] = srgb_dec(v[i]);
        } else if (src == CS_ACESCG) {
            M3 a = mk(AP1_TO_XYZ), b = mk(XYZ_TO_LSRGB);
            mv(&a, v);
            mv(&b, v);
        } else if (src == CS_XYZD65) {
            M3 b = mk(XYZ_TO_LSRGB);
            mv(&b, v);
        }
        /* from linear sRGB */
        if (dst == CS_OKLCH) lin_to_oklch(v);
        else if (dst == CS_SRGB) {
            for (int i = 0; i < 3; i++) v[i] = srgb_enc(v[i]);
        } else if (dst == CS_ACESCG) {
            M3 a = mk(LSRGB_TO_XYZ), b = mk(XYZ_TO_AP1);
            mv(&a, v);
            mv(&b, v);
        } else if (dst == CS_XYZD65) {
            M3 a = mk(LSRGB_TO_XYZ);
            mv(&a, v);
        }
        return;
    }
    /* matrix space -> matrix space through XYZ */
    static const double ID[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    const double *to = src == CS_ACESCG ? AP1_TO_XYZ : (src == CS_XYZD65 ? ID : LSRGB_TO_XYZ);
    const double *from = dst == CS_ACESCG ? XYZ_TO_AP1 : (dst == CS_XYZD65 ? ID : XYZ_TO_LSRGB);
    if (src == CS_SRGB)
        for (int i = 0; i < 3; i++) v[i] = srgb_dec(v[i]);
    M3 a = mk(to), b = mk(from);
    mv(&a, v);
    mv(&b, v);
    if (dst == CS_SRGB)
        for (int i = 0; i < 3; i++) v[i] = srgb_enc(v[i]);
}

int OSYM(oracle_cst_space)(real *rgb, size_t n, int src, int dst)
{
    if (!valid_cs(src) || !valid_cs(dst)) return ORACLE_ERR_ARG;
    for (size_t p = 0; p < n; p++) convert(src, dst, rgb + 3 * p);
    return ORACLE_OK;
}

void OSYM(oracle_highlight)(real *rgb, size_t n, real clip_g)
{
    for (size_t p = 0; p < n; p++) {
        real r = rgb[3 * p], g = rgb[3 * p + 1], b = rgb[3 * p + 2];
        real factor = g / clip_g;
        rgb[3 * p + 1] = ((K(1.0) - factor) * g) + (factor * (r + b) * (K(1.0) / K(2.0)));
    }
}

void OSYM(oracle_contrast)(real *rgb, size_t n, real c)
{
    const real mg = K(0.185);
    for (size_t i = 0; i < 3 * n; i++) rgb[i] = mg * RPOW(rgb[i] / mg, c);
}

void OSYM(oracle_gamma)(real *rgb, size_t n, real gamma)
{
    real inv = K(1.0) / RMAX(gamma, K(1e-6));
    for (size_t i = 0; i < 3 * n; i++) rgb[i] = rgb[i] <= 0 ? K(0.0) : RPOW(rgb[i], inv);
}

int OSYM(oracle_lch)(real *rgb, size_t n, int cs, real lc, real cc, real hc)
{
    if (!valid_cs(cs)) return ORACLE_ERR_ARG;
    for (size_t p = 0; p < n; p++) {
        real *v = rgb + 3 * p;
        convert(cs, CS_OKLCH, v);
        v[0] = v[0] * lc;
        v[1] = v[1] * cc;
        v[2] = v[2] * hc;
        convert(CS_OKLCH, cs, v);
    }
    return ORACLE_OK;
}

real OSYM(oracle_square_sigmoid)(real x)
{
    const real C = K(1.219512);
    if (x <= 0) return K(0.0);
    return K(1.0) / (K(1.0) + (K(1.0) / (C * x)));
}

static real compress_value(real dist, real lim, real thr, real power)
{
    if (dist < thr) return dist;
    real base_inner = (K(1.0) - thr) / (lim - thr);
    if (base_inner <= 0 || RABS(lim - thr) < K(1e-6)) return dist;
    real denom_inner = RPOW(base_inner, -power) - K(1.0);
    if (denom_inner <= 0) return dist;
    real s = (lim - thr) / RPOW(denom_inner, K(1.0) / power);
    real dist_norm = (dist - thr) / s;
    real denominator = RPOW(K(1.0) + RPOW(dist_norm, power), K(1.0) / power);
    return thr + s * (dist_norm / denominator);
}

static void gamut_compress(const real in[3], real out[3])
{
    const real thr[3] = {K(0.815), K(0.803), K(0.88)};
    const real lim[3] = {K(1.147), K(1.264), K(1.312)};
    const real power = K(1.2);
    real ach = RMAX(RMAX(in[0], in[1]), in[2]);
    if (ach == 0) {
        out[0] = out[1] = out[2] = K(0.0);
        return;
    }
    real abs_ach = RABS(ach);
    for (int i = 0; i < 3; i++) {
        real dist = (ach - in[i]) / abs_ach;
        real cd = compress_value(dist, lim[i], thr[i], power);
        out[i] = ach - cd * abs_ach;
    }
}

void OSYM(oracle_sigmoid)(real *rgb, size_t n)
{
    for (size_t q = 0; q < n; q++) {
        real *px = rgb + 3 * q;
        real gc[3], t[3], p[3];
        gamut_compress(px, gc);
        t[0] = gc[0];
        t[1] = gc[1];
        t[2] = gc[2];
        convert(CS_ACESCG, CS_OKLCH, t);
        real h = t[2];
        for (int i = 0; i < 3; i++) p[i] = OSYM(oracle_square_sigmoid)(gc[i]);
        real s = K(0.2722287168) * p[0] + K(0.6740817658) * p[1] + K(0.0536895174) * p[2];
        real m = K(1.0) - RPOW(s, K(5.0));
        convert(CS_ACESCG, CS_OKLCH, p);
        px[0] = p[0];
        px[1] = p[1] * m;
        px[2] = h;
        convert(CS_OKLCH, CS_ACESCG, px);
    }
}
