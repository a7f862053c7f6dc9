// display.cu -- per-pixel display stages and colour-space conversions as a
// chain of ops run in one pass (display.cuh).
//
// Each op is the reference's own f32 arithmetic in its order (built with
// --fmad=false).  A pipeline run of consecutive per-pixel modules becomes one
// launch: 12 B read and 12 B written per pixel for the whole run instead of
// per module.  The chain is a __grid_constant__ parameter, so its matrices
// and constants are read through the constant cache with no global loads.
//
// Oklch follows the `color` crate 0.3.3 ColorSpaceTag::convert, restated
// from its published definitions: Oklab (B. Ottosson, 2020, linear-sRGB
// matrices and a cube root), LCh per CSS Color 4 (hue in degrees in
// [0, 360)), AcesCg <-> linear sRGB through XYZ(D65) with the AP1 matrices
// of film/exposure/upsample.rs:34-45.
#include <cmath>
#include <cstring>
#include <string>

#include "color.cuh"
#include "display.cuh"

namespace imops {
namespace display {

// Ottosson's Oklab: linear sRGB -> LMS, LMS' -> Lab, and the inverses.
__constant__ float OK_M1[9] = {0.4122214708f, 0.5363325363f, 0.0514459929f, 0.2119034982f, 0.6806995451f,
                               0.1073969566f, 0.0883024619f, 0.2817188376f, 0.6299787005f};
__constant__ float OK_M2[9] = {0.2104542553f, 0.7936177850f, -0.0040720468f, 1.9779984951f, -2.4285922050f,
                               0.4505937099f, 0.0259040371f, 0.7827717662f,  -0.8086757660f};
__constant__ float OK_M2I[9] = {1.0f, 0.3963377774f,  0.2158037573f,  1.0f, -0.1055613458f,
                                -0.0638541728f, 1.0f, -0.0894841775f, -1.2914855480f};
__constant__ float OK_M1I[9] = {4.0767416621f,  -3.3077115913f, 0.2309699292f,  -1.2684380046f, 2.6097574011f,
                                -0.3413193965f, -0.0041960863f, -0.7034186147f, 1.7076147010f};

// ---- elementary functions of the chain -------------------------------------
// Powers, cube roots and angles are formed from the hardware base-2
// logarithm and exponential (PTX lg2.approx.ftz / ex2.approx.ftz, about 2^-22
// relative), the hardware sine and cosine on a reduced argument, and a
// polynomial arctangent; against the exact functions each is within a few
// 1e-7 relative over the chain's inputs (the display tests hold the chain to
// 2e-5 of max(1, |x|)).

__device__ __forceinline__ float lg2_hw(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ex2_hw(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// x^y = 2^(y log2 x) for x >= 0 (0^y = 0 for y > 0, x^0 = 1).  The log's
// error (about 1.6e-7 absolute near 1) is multiplied by y, so exponents
// above 64 in magnitude (a gamma near 0) go to the library's powf, as does a
// negative base, where powf defines integer exponents.
__device__ __forceinline__ float pow_fast(float x, float y) {
    if (y == 0.0f) return 1.0f;
    if (x < 0.0f || fabsf(y) > 64.0f) return powf(x, y);
    return ex2_hw(y * lg2_hw(x));
}

// real cube root, sign kept: r = |x|^(-1/3) estimated as 2^(-log2|x| / 3),
// then one step of Newton's method for the reciprocal cube root,
// r <- r (4 - |x| r^3) / 3 (division-free; it squares the estimate's
// relative error), and |x|^(1/3) = |x| r^2.  Zero, subnormal and non-finite
// inputs take the library's cbrtf.
__device__ __forceinline__ float cbrt_fast(float x) {
    const float ax = fabsf(x);
    if (!(ax >= 1.17549435e-38f) || ax == INFINITY) return cbrtf(x);
    float r = ex2_hw(lg2_hw(ax) * (-1.0f / 3.0f));
    const float r3 = (r * r) * r;
    r = (r * fmaf(-ax, r3, 4.0f)) * (1.0f / 3.0f);
    return copysignf((ax * r) * r, x);
}

// atan2(y, x) in radians.  The ratio a = min/max of |x|, |y| is in [0, 1],
// where atan(a) = a P(a^2) with P of degree 8, fitted here for least maximum
// relative error (1.5e-7 in f32); the octant puts it in (-pi, pi].
__device__ __forceinline__ float atan2_fast(float y, float x) {
    const float ax = fabsf(x), ay = fabsf(y);
    const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
    if (isnan(x) || isnan(y) || !(mx < INFINITY)) return atan2f(y, x);
    if (mx == 0.0f) return copysignf(signbit(x) ? 3.14159265358979f : 0.0f, y);
    const float a = __fdividef(mn, mx), t = a * a;
    float p = 0.002849851967766881f;
    p = fmaf(p, t, -0.016068479046225548f);
    p = fmaf(p, t, 0.04269127547740936f);
    p = fmaf(p, t, -0.0750427395105362f);
    p = fmaf(p, t, 0.10640924423933029f);
    p = fmaf(p, t, -0.14203642308712006f);
    p = fmaf(p, t, 0.1999261975288391f);
    p = fmaf(p, t, -0.3333307206630707f);
    p = fmaf(p, t, 1.0f);
    float r = a * p;
    if (ay > ax) r = 1.57079632679490f - r;
    if (signbit(x)) r = 3.14159265358979f - r;
    return copysignf(r, y);
}

// sine and cosine of an angle given in degrees: reduced to [-180, 180)
// degrees, then the hardware approximations (absolute error about 2^-21 on
// [-pi, pi])
__device__ __forceinline__ void sincos_deg(float deg, float* s, float* c) {
    const float turns = rintf(deg * (1.0f / 360.0f));
    const float red = fmaf(-360.0f, turns, deg);
    __sincosf(red * 0.017453292519943295f, s, c);
}

// 3x3 matrix times a column in the reference's operation order (the linear
// conversions match the f32 restatement bit for bit; the file is built
// without automatic contraction)
__device__ __forceinline__ void mv(const float* m, float& r, float& g, float& b) {
    float x = m[0] * r + m[1] * g + m[2] * b;
    float y = m[3] * r + m[4] * g + m[5] * b;
    float z = m[6] * r + m[7] * g + m[8] * b;
    r = x;
    g = y;
    b = z;
}

// the same product as fused multiply-adds, for the Oklch and tone-map paths,
// whose results are held to a tolerance
__device__ __forceinline__ void mv_fma(const float* m, float& r, float& g, float& b) {
    float x = fmaf(m[2], b, fmaf(m[1], g, m[0] * r));
    float y = fmaf(m[5], b, fmaf(m[4], g, m[3] * r));
    float z = fmaf(m[8], b, fmaf(m[7], g, m[6] * r));
    r = x;
    g = y;
    b = z;
}

__device__ __forceinline__ void lin_to_oklch(float& r, float& g, float& b) {
    mv_fma(OK_M1, r, g, b);
    r = cbrt_fast(r);
    g = cbrt_fast(g);
    b = cbrt_fast(b);
    mv_fma(OK_M2, r, g, b);
    float c = sqrtf(g * g + b * b);
    float h = atan2_fast(b, g) * 57.29577951308232f;
    if (h < 0.0f) h = h + 360.0f;
    g = c;
    b = h;
}

__device__ __forceinline__ void oklch_to_lin(float& l, float& c, float& h) {
    float sn, cs;
    sincos_deg(h, &sn, &cs);
    float a = c * cs;
    float bb = c * sn;
    c = a;
    h = bb;
    mv_fma(OK_M2I, l, c, h);
    l = l * l * l;
    c = c * c * c;
    h = h * h * h;
    mv_fma(OK_M1I, l, c, h);
}

__device__ __forceinline__ void cst(const Op& o, float& r, float& g, float& b) {
    const int f = o.flags;
    if (f & CST_DECODE) {
        r = color::Epilogue::srgb_decode(r);
        g = color::Epilogue::srgb_decode(g);
        b = color::Epilogue::srgb_decode(b);
    }
    if (f & CST_FROM_OKLCH) oklch_to_lin(r, g, b);
    if (f & CST_M0) mv(o.m[0], r, g, b);
    if (f & CST_M1) mv(o.m[1], r, g, b);
    if (f & CST_TO_OKLCH) lin_to_oklch(r, g, b);
    if (f & CST_ENCODE) {
        r = color::Epilogue::srgb_encode(r);
        g = color::Epilogue::srgb_encode(g);
        b = color::Epilogue::srgb_encode(b);
    }
}

// compress_value (tone_map.rs:71-125) in the forward direction with the
// default parameters: power 1.2; s_pre = the y = 1 intersect scale, or a
// negative value when the reference returns dist unchanged.
__device__ __forceinline__ float compress(float dist, float thr, float s) {
    if (dist < thr) return dist;
    if (!(s > 0.0f)) return dist;
    const float power = 1.2f, inv_power = 1.0f / 1.2f;
    float dn = __fdividef(dist - thr, s);
    float den = pow_fast(1.0f + pow_fast(dn, power), inv_power);
    return thr + s * __fdividef(dn, den);
}

__device__ __forceinline__ float square_sigmoid(float x) {
    const float C = 1.219512f;
    if (x <= 0.0f) return 0.0f;
    return __fdividef(1.0f, 1.0f + __fdividef(1.0f, C * x));
}

// sigmoid_tone_map (tone_map.rs:18-33) on ACEScg: gamut compression, the
// hue of the compressed pixel in Oklch, the square sigmoid per channel, and
// the sigmoid's Oklch lightness and chroma (chroma scaled by 1 - Y^5) with
// that hue, back to ACEScg.  The conversions are the reference's (ACEScg ->
// XYZ -> linear sRGB -> Oklab) with their matrices multiplied out on the
// host: m[0] = ACEScg -> LMS, m[1] = LMS -> ACEScg; only the Oklch
// components used are formed (the hue of the compressed pixel, the
// lightness and chroma of the sigmoid).
__device__ __forceinline__ void sigmoid(const Op& o, float& r, float& g, float& b) {
    // gamut_compress_pixel (tone_map.rs:133-171); s[0..2] = the per-channel
    // scale of compress_value (thresholds 0.815 / 0.803 / 0.88)
    float gc0, gc1, gc2;
    float ach = fmaxf(fmaxf(r, g), b);
    if (ach == 0.0f) {
        gc0 = gc1 = gc2 = 0.0f;
    } else {
        float aa = fabsf(ach);
        const float ia = __fdividef(1.0f, aa);
        gc0 = ach - compress((ach - r) * ia, 0.815f, o.s[0]) * aa;
        gc1 = ach - compress((ach - g) * ia, 0.803f, o.s[1]) * aa;
        gc2 = ach - compress((ach - b) * ia, 0.88f, o.s[2]) * aa;
    }
    // hue of the compressed pixel: Oklab a, b -> atan2
    float l0 = gc0, l1 = gc1, l2 = gc2;
    mv_fma(o.m[0], l0, l1, l2);
    l0 = cbrt_fast(l0);
    l1 = cbrt_fast(l1);
    l2 = cbrt_fast(l2);
    const float ha = fmaf(OK_M2[5], l2, fmaf(OK_M2[4], l1, OK_M2[3] * l0));
    const float hb = fmaf(OK_M2[8], l2, fmaf(OK_M2[7], l1, OK_M2[6] * l0));
    // the hue enters only through its cosine and sine: (a, b) / |(a, b)|.
    // Where that is 0 / 0 or not finite, the angle itself (atan2 in
    // degrees on [0, 360), as the reference forms it) and its sine and cosine.
    float sn, cs;
    const float n2 = fmaf(ha, ha, hb * hb);
    if (n2 > 0.0f && n2 < INFINITY) {
        const float inv = rsqrtf(n2);
        cs = ha * inv;
        sn = hb * inv;
    } else {
        float h = atan2_fast(hb, ha) * 57.29577951308232f;
        if (h < 0.0f) h = h + 360.0f;
        sincos_deg(h, &sn, &cs);
    }
    float p0 = square_sigmoid(gc0), p1 = square_sigmoid(gc1), p2 = square_sigmoid(gc2);
    float s = 0.2722287168f * p0 + 0.6740817658f * p1 + 0.0536895174f * p2;
    const float s2 = s * s;
    float m = 1.0f - (s2 * s2) * s;
    // lightness and chroma of the sigmoid
    mv_fma(o.m[0], p0, p1, p2);
    p0 = cbrt_fast(p0);
    p1 = cbrt_fast(p1);
    p2 = cbrt_fast(p2);
    mv_fma(OK_M2, p0, p1, p2);
    const float cm = sqrtf(p1 * p1 + p2 * p2) * m;
    // (L, C m, h) -> Oklab -> LMS -> ACEScg
    float L = p0, A = cm * cs, B = cm * sn;
    mv_fma(OK_M2I, L, A, B);
    L = L * L * L;
    A = A * A * A;
    B = B * B * B;
    mv_fma(o.m[1], L, A, B);
    r = L;
    g = A;
    b = B;
}

__device__ __forceinline__ void apply(const Op& o, float& r, float& g, float& b) {
    switch (o.kind) {
        case OP_GAIN:
            r = r * o.s[0];
            g = g * o.s[1];
            b = b * o.s[2];
            break;
        case OP_HIGHLIGHT: {
            float factor = g / o.s[0];
            g = ((1.0f - factor) * g) + (factor * (r + b) * (1.0f / 2.0f));
            break;
        }
        case OP_CONTRAST: {
            const float mg = 0.185f;
            r = mg * pow_fast(r / mg, o.s[0]);
            g = mg * pow_fast(g / mg, o.s[0]);
            b = mg * pow_fast(b / mg, o.s[0]);
            break;
        }
        case OP_GAMMA:
            r = r <= 0.0f ? 0.0f : pow_fast(r, o.s[0]);
            g = g <= 0.0f ? 0.0f : pow_fast(g, o.s[0]);
            b = b <= 0.0f ? 0.0f : pow_fast(b, o.s[0]);
            break;
        case OP_SCALE:
            r = r * o.s[0];
            g = g * o.s[1];
            b = b * o.s[2];
            break;
        case OP_CST:
            cst(o, r, g, b);
            break;
        case OP_SIGMOID:
            sigmoid(o, r, g, b);
            break;
    }
}

__global__ void __launch_bounds__(256) chain_kernel(float* __restrict__ rgb, size_t n, const __grid_constant__ Chain c) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        float* p = rgb + 3 * k;
        float r = p[0], g = p[1], b = p[2];
        for (int i = 0; i < c.n; i++) apply(c.op[i], r, g, b);
        p[0] = r;
        p[1] = g;
        p[2] = b;
    }
}

// ---- host builders ---------------------------------------------------------

static Op* next(Chain& c) {
    if (c.n >= MAX_OPS) {
        fail(IMOPS_ERR_INVALID_ARGUMENT, "display chain: more than 16 per-pixel ops in one pass");
        return nullptr;
    }
    Op* o = &c.op[c.n++];
    std::memset(o, 0, sizeof(Op));
    return o;
}

int add_gain(Chain& c, float r, float g, float b) {
    Op* o = next(c);
    if (!o) return IMOPS_ERR_INVALID_ARGUMENT;
    o->kind = OP_GAIN;
    o->s[0] = r;
    o->s[1] = g;
    o->s[2] = b;
    return IMOPS_OK;
}

int add_highlight(Chain& c, float clip_g) {
    Op* o = next(c);
    if (!o) return IMOPS_ERR_INVALID_ARGUMENT;
    o->kind = OP_HIGHLIGHT;
    o->s[0] = clip_g;
    return IMOPS_OK;
}

int add_contrast(Chain& c, float value) {
    Op* o = next(c);
    if (!o) return IMOPS_ERR_INVALID_ARGUMENT;
    o->kind = OP_CONTRAST;
    o->s[0] = value;
    return IMOPS_OK;
}

int add_gamma(Chain& c, float gamma) {
    Op* o = next(c);
    if (!o) return IMOPS_ERR_INVALID_ARGUMENT;
    o->kind = OP_GAMMA;
    o->s[0] = 1.0f / std::fmax(gamma, 1e-6f);
    return IMOPS_OK;
}

static bool matrix_space(int cs) {
    return cs == IMOPS_CS_XYZD65 || cs == IMOPS_CS_LINEAR_SRGB || cs == IMOPS_CS_SRGB || cs == IMOPS_CS_ACESCG;
}

int add_cst(Chain& c, int src, int dst, const float* camera_fwd) {
    bool src_ok = matrix_space(src) || src == IMOPS_CS_OKLCH || (src == IMOPS_CS_CAMERA && camera_fwd);
    if (!src_ok || !(matrix_space(dst) || dst == IMOPS_CS_OKLCH))
        return fail(IMOPS_ERR_INVALID_ARGUMENT, "cst: unsupported colour space");
    if (src == dst) return IMOPS_OK;
    Op* o = next(c);
    if (!o) return IMOPS_ERR_INVALID_ARGUMENT;
    o->kind = OP_CST;
    int f = 0;
    if (src == IMOPS_CS_CAMERA) {
        // camera_cst (cst.rs:12-48): camera -> XYZ, then XyzD65 -> target
        std::memcpy(o->m[0], camera_fwd, 9 * sizeof(float));
        f |= CST_M0 | CST_M1;
        if (dst == IMOPS_CS_OKLCH) {
            color::xyz_to_target(IMOPS_CS_LINEAR_SRGB, o->m[1]);
            f |= CST_TO_OKLCH;
        } else {
            color::xyz_to_target(dst, o->m[1]);
            if (dst == IMOPS_CS_SRGB) f |= CST_ENCODE;
        }
    } else if (src != IMOPS_CS_OKLCH && dst != IMOPS_CS_OKLCH) {
        // decode -> XYZ -> target -> encode, as the camera CST's second step
        color::to_xyz(src, o->m[0]);
        color::xyz_to_target(dst, o->m[1]);
        f |= CST_M0 | CST_M1;
        if (src == IMOPS_CS_SRGB) f |= CST_DECODE;
        if (dst == IMOPS_CS_SRGB) f |= CST_ENCODE;
    } else if (dst == IMOPS_CS_OKLCH) {
        // to linear sRGB, then Oklch
        if (src == IMOPS_CS_SRGB) f |= CST_DECODE;
        if (src == IMOPS_CS_ACESCG) {
            color::to_xyz(IMOPS_CS_ACESCG, o->m[0]);
            color::xyz_to_target(IMOPS_CS_LINEAR_SRGB, o->m[1]);
            f |= CST_M0 | CST_M1;
        }
        if (src == IMOPS_CS_XYZD65) {
            color::xyz_to_target(IMOPS_CS_LINEAR_SRGB, o->m[0]);
            f |= CST_M0;
        }
        f |= CST_TO_OKLCH;
    } else {
        // Oklch to linear sRGB, then the target
        f |= CST_FROM_OKLCH;
        if (dst == IMOPS_CS_ACESCG) {
            color::to_xyz(IMOPS_CS_LINEAR_SRGB, o->m[0]);
            color::xyz_to_target(IMOPS_CS_ACESCG, o->m[1]);
            f |= CST_M0 | CST_M1;
        }
        if (dst == IMOPS_CS_XYZD65) {
            color::to_xyz(IMOPS_CS_LINEAR_SRGB, o->m[0]);
            f |= CST_M0;
        }
        if (dst == IMOPS_CS_SRGB) f |= CST_ENCODE;
    }
    o->flags = f;
    return IMOPS_OK;
}

int add_lch(Chain& c, int cs, float lc, float cc, float hc) {
    if (!(matrix_space(cs) || cs == IMOPS_CS_OKLCH))
        return fail(IMOPS_ERR_INVALID_ARGUMENT, "lch: the image needs a colour space");
    int rc;
    if ((rc = add_cst(c, cs, IMOPS_CS_OKLCH, nullptr))) return rc;
    Op* o = next(c);
    if (!o) return IMOPS_ERR_INVALID_ARGUMENT;
    o->kind = OP_SCALE;
    o->s[0] = lc;
    o->s[1] = cc;
    o->s[2] = hc;
    return add_cst(c, IMOPS_CS_OKLCH, cs, nullptr);
}

// The y = 1 intersect scale of compress_value (tone_map.rs:90-105) for one
// channel, in f32 as the reference computes it per pixel (it depends on the
// default parameters only); -1 where the reference returns dist unchanged.
static float rgc_scale(float lim, float thr) {
    const float power = 1.2f;
    float base_inner = (1.0f - thr) / (lim - thr);
    if (base_inner <= 0.0f || std::fabs(lim - thr) < 1e-6f) return -1.0f;
    float denom_inner = powf(base_inner, -power) - 1.0f;
    if (denom_inner <= 0.0f) return -1.0f;
    return (lim - thr) / powf(denom_inner, 1.0f / power);
}

// Ottosson's linear sRGB <-> LMS matrices (the device tables OK_M1, OK_M1I)
static const double OK_M1_HOST[9] = {0.4122214708, 0.5363325363, 0.0514459929, 0.2119034982, 0.6806995451,
                                     0.1073969566, 0.0883024619, 0.2817188376, 0.6299787005};
static const double OK_M1I_HOST[9] = {4.0767416621,  -3.3077115913, 0.2309699292,  -1.2684380046, 2.6097574011,
                                      -0.3413193965, -0.0041960863, -0.7034186147, 1.7076147010};

// out = a b (3x3, row-major) in double
static void mat_mul(const float* a, const float* b, double* out) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double acc = 0.0;
            for (int k = 0; k < 3; k++) acc += (double)a[3 * i + k] * (double)b[3 * k + j];
            out[3 * i + j] = acc;
        }
}
static void mat_mul_d(const double* a, const double* b, double* out) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double acc = 0.0;
            for (int k = 0; k < 3; k++) acc += a[3 * i + k] * b[3 * k + j];
            out[3 * i + j] = acc;
        }
}

int add_sigmoid(Chain& c) {
    Op* o = next(c);
    if (!o) return IMOPS_ERR_INVALID_ARGUMENT;
    o->kind = OP_SIGMOID;
    o->s[0] = rgc_scale(1.147f, 0.815f);
    o->s[1] = rgc_scale(1.264f, 0.803f);
    o->s[2] = rgc_scale(1.312f, 0.88f);
    // ACEScg -> XYZ -> linear sRGB -> LMS and back, multiplied out in double
    float a2x[9], x2l[9], l2x[9], x2a[9];
    color::to_xyz(IMOPS_CS_ACESCG, a2x);
    color::xyz_to_target(IMOPS_CS_LINEAR_SRGB, x2l);
    color::to_xyz(IMOPS_CS_LINEAR_SRGB, l2x);
    color::xyz_to_target(IMOPS_CS_ACESCG, x2a);
    double lms_from_lin[9], lin_from_lms[9];
    for (int k = 0; k < 9; k++) {
        lms_from_lin[k] = OK_M1_HOST[k];
        lin_from_lms[k] = OK_M1I_HOST[k];
    }
    double t[9], u[9];
    mat_mul(x2l, a2x, t);              // ACEScg -> linear sRGB
    mat_mul_d(lms_from_lin, t, u);     // -> LMS
    for (int k = 0; k < 9; k++) o->m[0][k] = (float)u[k];
    mat_mul(x2a, l2x, t);              // linear sRGB -> ACEScg
    mat_mul_d(t, lin_from_lms, u);     // LMS -> ... -> ACEScg
    for (int k = 0; k < 9; k++) o->m[1][k] = (float)u[k];
    return IMOPS_OK;
}

int run(float* rgb, size_t n, const Chain& c, cudaStream_t s, const char* what) {
    if (!rgb && n) return fail(IMOPS_ERR_INVALID_ARGUMENT, std::string(what) + ": NULL buffer");
    if (n == 0 || c.n == 0) return IMOPS_OK;
    if (fault_injected("launch")) return fail(IMOPS_ERR_CUDA, std::string("injected launch failure (") + what + ")");
    chain_kernel<<<color::stream_grid(n, 256), 256, 0, s>>>(rgb, n, c);
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), what);
    return IMOPS_OK;
}

}  // namespace display
}  // namespace imops

using namespace imops;

static int run_one(float* rgb, size_t n, const display::Chain& c, int rc, imops_stream_t stream, const char* what) {
    if (rc) return rc;
    return display::run(rgb, n, c, as_stream(stream), what);
}

extern "C" int imops_highlight_reconstruction(float* rgb, size_t n_pixels, const float wb[4], imops_stream_t stream) {
    clear_error();
    if (!wb) return fail(IMOPS_ERR_INVALID_ARGUMENT, "highlight_reconstruction: NULL coefficients");
    display::Chain c{};
    int rc = display::add_highlight(c, wb[1]);
    return run_one(rgb, n_pixels, c, rc, stream, "highlight_reconstruction");
}

extern "C" int imops_contrast(float* rgb, size_t n_pixels, float value, imops_stream_t stream) {
    clear_error();
    display::Chain c{};
    int rc = display::add_contrast(c, value);
    return run_one(rgb, n_pixels, c, rc, stream, "contrast");
}

extern "C" int imops_gamma(float* rgb, size_t n_pixels, float gamma, imops_stream_t stream) {
    clear_error();
    display::Chain c{};
    int rc = display::add_gamma(c, gamma);
    return run_one(rgb, n_pixels, c, rc, stream, "gamma");
}

extern "C" int imops_lch(float* rgb, size_t n_pixels, int color_space, float lc, float cc, float hc,
                         imops_stream_t stream) {
    clear_error();
    display::Chain c{};
    int rc = display::add_lch(c, color_space, lc, cc, hc);
    return run_one(rgb, n_pixels, c, rc, stream, "lch");
}

extern "C" int imops_sigmoid_tone_map(float* rgb, size_t n_pixels, imops_stream_t stream) {
    clear_error();
    display::Chain c{};
    int rc = display::add_sigmoid(c);
    return run_one(rgb, n_pixels, c, rc, stream, "sigmoid_tone_map");
}

extern "C" int imops_cst(float* rgb, size_t n_pixels, int source, int target, imops_stream_t stream) {
    clear_error();
    if (source == IMOPS_CS_CAMERA)
        return fail(IMOPS_ERR_INVALID_ARGUMENT, "cst: camera RGB needs imops_camera_cst (a calibration matrix)");
    display::Chain c{};
    int rc = display::add_cst(c, source, target, nullptr);
    return run_one(rgb, n_pixels, c, rc, stream, "cst");
}
