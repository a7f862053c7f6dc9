/*
 * film.c -- CPU oracle for the spectral film simulation.
 *
 * TEST INFRASTRUCTURE (see oracle_common.h).
 *
 * Part 1 restates the reference's film::process (pichromatic/src/film/mod.rs:77-129)
 * for the stocks ColorNeg200 (film/stock/color_neg_200.rs:38-208) and BwStub
 * (film/stock/bw_stub.rs:18-82), keeping the reference's precision mix:
 * per-pixel spectral work in f64 (exposure/mod.rs:68-81, scan/densitometry.rs:13-73),
 * planes, blurs, development and grain in f32.  With ORACLE_F32 the f32 parts
 * run in f32 (reference order); without it every step runs in f64 (the FP64
 * oracle used for error reporting).
 *
 * Part 2 is the "baseline" preset: the 81-bin (380-780 nm, 5 nm), 3-layer,
 * logistic-curve, red-highlight-halation, seeded-grain stock this library
 * defines for the throughput workload.  The reference has no such stock, so
 * its only oracle is this file; it integrates every pixel over all 81 bins
 * (no rank-3 collapse), which checks the GPU's collapsed exposure.
 */
#include "oracle_common.h"

#include <stdlib.h>
#include <string.h>

#ifdef ORACLE_F32
#define REXP expf
#define RPOW powf
#define RSQRT sqrtf
#define RCEIL ceilf
#else
#define REXP exp
#define RPOW pow
#define RSQRT sqrt
#define RCEIL ceil
#endif

#define NB 16          /* reference grid: 400..700 nm step 20 */
#define MAXL 12

/* ----------------------------------------------------------------------- */
/* constants (film/constants.rs:14-67, upsample.rs:17-45, pixel.rs:33-36)   */

static const double CMF_X[NB] = {0.01431, 0.13438, 0.34828, 0.29080, 0.09564, 0.00490, 0.06327, 0.29040,
                                 0.59450, 0.91630, 1.06220, 0.85445, 0.44790, 0.16490, 0.04677, 0.01136};
static const double CMF_Y[NB] = {0.000396, 0.004000, 0.023000, 0.060000, 0.139020, 0.323000, 0.710000, 0.954000,
                                 0.995000, 0.870000, 0.631000, 0.381000, 0.175000, 0.061000, 0.017000, 0.004100};
static const double CMF_Z[NB] = {0.06785, 0.64560, 1.74706, 1.66920, 0.81295, 0.27200, 0.07825, 0.02030,
                                 0.00390, 0.00165, 0.00080, 0.00019, 0.00002, 0.00000, 0.00000, 0.00000};
static const double XYZ2AP1[3][3] = {{1.6410233797, -0.3248032942, -0.2364246952},
                                     {-0.6636628587, 1.6153315917, 0.0167563477},
                                     {0.0117218943, -0.0082844165, 0.9883948585}};
#define LUM_R K(0.2722287168)
#define LUM_G K(0.6740817658)
#define LUM_B K(0.0536895174)
#define MIDDLE_GRAY K(0.185)

static double grid_nm(int i) { return 400.0 + 20.0 * i; }

static void matvec3(const double m[3][3], const double v[3], double o[3])
{
    for (int i = 0; i < 3; i++) o[i] = m[i][0] * v[0] + m[i][1] * v[1] + m[i][2] * v[2];
}

/* inv3 of upsample.rs:57-79 (cofactor form). */
static void inv3(const double m[3][3], double r[3][3])
{
    double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                 m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    double id = 1.0 / det;
    r[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) * id;
    r[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * id;
    r[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * id;
    r[1][0] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) * id;
    r[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * id;
    r[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * id;
    r[2][0] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) * id;
    r[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * id;
    r[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * id;
}

static double integrate_cmf(const double *s, const double *cmf)
{
    double acc = 0.0;
    for (int i = 0; i < NB - 1; i++) {
        double a = s[i] * cmf[i];
        double b = s[i + 1] * cmf[i + 1];
        acc += 0.5 * (a + b) * 20.0;
    }
    return acc;
}

/* spectrum_to_acescg (upsample.rs:101-112). */
static void spectrum_to_ap1(const double *s, double out[3])
{
    double xyz[3] = {integrate_cmf(s, CMF_X), integrate_cmf(s, CMF_Y), integrate_cmf(s, CMF_Z)};
    matvec3(XYZ2AP1, xyz, out);
}

/* UpsampleBasis (upsample.rs:114-158): three Gaussians 450/550/650, sigma 40. */
typedef struct { double b[3][NB]; double minv[3][3]; } Basis;

static void basis_build(Basis *B)
{
    const double peaks[3] = {450.0, 550.0, 650.0};
    double cols[3][3], m[3][3];
    for (int k = 0; k < 3; k++) {
        for (int i = 0; i < NB; i++) {
            double d = (grid_nm(i) - peaks[k]) / 40.0;
            B->b[k][i] = exp(-0.5 * d * d);
        }
        spectrum_to_ap1(B->b[k], cols[k]);
    }
    for (int r = 0; r < 3; r++)
        for (int k = 0; k < 3; k++) m[r][k] = cols[k][r];
    inv3(m, B->minv);
}

/* upsample_acescg + pixel_fluence_spectrum (upsample.rs:136-170,
 * exposure/mod.rs:124-137). */
static void fluence_spectrum(const Basis *B, const real rgb[3], double out[NB])
{
    double v[3] = {(double)(float)rgb[0], (double)(float)rgb[1], (double)(float)rgb[2]};
#ifndef ORACLE_F32
    v[0] = rgb[0]; v[1] = rgb[1]; v[2] = rgb[2];
#endif
    double w[3];
    matvec3(B->minv, v, w);
    for (int k = 0; k < 3; k++)
        if (w[k] < 0.0) w[k] = 0.0;
    for (int i = 0; i < NB; i++) {
        double s = w[0] * B->b[0][i] + w[1] * B->b[1][i] + w[2] * B->b[2][i];
        double e_rel = 550.0 / grid_nm(i);
        out[i] = s / e_rel;
    }
}

/* ----------------------------------------------------------------------- */
/* stocks                                                                   */

enum { LK_EMULSION, LK_FILTER, LK_OVERCOAT, LK_AH, LK_SUPPORT };

typedef struct {
    int kind;
    float thickness;
    int has_sens;
    double sens[NB];
    double mu_ln, sigma_ln;
    float fraction;
    double eps[NB];
    int has_mask;
    double mask_eps[NB];
    float dmax;
    float gamma;
    double capture_k;
    float recip_p;
    int reversal;
    double lut_log[64], lut_frac[64];
    float kappa;
} OLayer;

typedef struct {
    float box_iso;
    int nl;
    OLayer l[MAXL];
    double refl[NB];
    float psf_local, psf_halation;
    float dev_diff, adj_beta, dir_diff;
    int dir_n;
    float dir[MAXL][MAXL];
    double scanner[NB];
} OStock;

static void gaussian_curve(double peak, double sigma, double amp, double *s)
{
    for (int i = 0; i < NB; i++) {
        double d = (grid_nm(i) - peak) / sigma;
        s[i] = amp * exp(-0.5 * d * d);
    }
}

static void orange_mask(double *s)
{
    for (int i = 0; i < NB; i++) {
        double l = grid_nm(i);
        double bd = (l - 450.0) / 50.0, gd = (l - 520.0) / 60.0;
        double blue = exp(-0.5 * (bd * bd));
        double green = 0.6 * exp(-0.5 * (gd * gd));
        s[i] = 0.35 * blue + 0.25 * green + 0.05;
    }
}

/* E_s[exp(-k s^2 phi)] with 64-node trapezoid over z (capture.rs:91-106). */
static double expected_survival(double mu, double sig, double k, double phi)
{
    const int N = 64;
    const double ZMAX = 8.0;
    double dz = (2.0 * ZMAX) / (double)N;
    double isq = 1.0 / sqrt(2.0 * 3.14159265358979323846);
    double acc = 0.0;
    for (int i = 0; i <= N; i++) {
        double z = -ZMAX + (double)i * dz;
        double tw = (i == 0 || i == N) ? 0.5 : 1.0;
        double pdf = isq * exp(-0.5 * z * z);
        double s = exp(mu + sig * z);
        double g = exp(-k * s * s * phi);
        acc += tw * pdf * g * dz;
    }
    return acc;
}

/* DevelopableFractionLut::build (capture.rs:37-58). */
static void lut_build(OLayer *L)
{
    for (int i = 0; i < 64; i++) {
        double t = (double)i / 63.0;
        double lp = -4.0 + t * (8.0 - -4.0);
        double phi = pow(10.0, lp);
        double f = 1.0 - expected_survival(L->mu_ln, L->sigma_ln, L->capture_k, phi);
        if (f < 0.0) f = 0.0;
        if (f > 1.0) f = 1.0;
        L->lut_log[i] = lp;
        L->lut_frac[i] = f;
    }
}

/* DevelopableFractionLut::sample (capture.rs:61-88). */
static double lut_sample(const OLayer *L, double phi)
{
    if (!(phi > 0.0)) return L->lut_frac[0];
    double lp = log10(phi);
    if (lp <= L->lut_log[0]) return L->lut_frac[0];
    if (lp >= L->lut_log[63]) return L->lut_frac[63];
    int lo = 0, hi = 63;
    while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (L->lut_log[mid] <= lp) lo = mid; else hi = mid;
    }
    double t = (lp - L->lut_log[lo]) / (L->lut_log[hi] - L->lut_log[lo]);
    return L->lut_frac[lo] * (1.0 - t) + L->lut_frac[hi] * t;
}

/* FilmStock::finalize grain kappa (stock/mod.rs:193-211). */
static float layer_kappa(const OLayer *L)
{
    double mean_s = exp(L->mu_ln + 0.5 * L->sigma_ln * L->sigma_ln);
    double r = mean_s * 0.5;
    if (r < 1e-6) r = 1e-6;
    double vol = 1.04719755119659774615421446109316763 * 4.0 * r * r * r; /* FRAC_PI_3 */
    double rho = (double)L->fraction * (double)L->thickness / (vol > 1e-18 ? vol : 1e-18);
    return (float)(1.0 / sqrt(rho));
}

static void finalize(OStock *S)
{
    for (int i = 0; i < S->nl; i++)
        if (S->l[i].kind == LK_EMULSION) {
            lut_build(&S->l[i]);
            S->l[i].kappa = layer_kappa(&S->l[i]);
        }
}

/* A stock as the reference's stock files list it: one row per EmulsionLayer
 * (the film/stock/ files), in stack order.  Curves: 'g' gaussian_curve(a, b, c),
 * 'c' SpectralCurve::constant(a), 'p' panchromatic a + b * max(0, sin(pi t))
 * with t = (lambda - 400) / 300 (bw_stub.rs, trix_400.rs). */
typedef struct {
    int kind;
    float thick;
    char sens;
    double sa, sb, sc;
    double mean_um, sig_ln;
    float frac;
    char eps;
    double ea, eb, ec;
    int mask;
    float dmax, gamma;
    double k;
    float p;
} LayerRow;

typedef struct {
    float box_iso;
    double mask_b, mask_g, mask_0; /* orange mask: mask_b*blue + mask_g*green + mask_0 */
    char refl;
    double ra, rb, rc;
    float psf_local, psf_halation, dev_diff, adj_beta, dir_diff;
    int reversal;
    int nl;
    LayerRow l[MAXL];
    int dir_n;
    float dir[MAXL][MAXL];
} StockRow;

static void row_curve(char kind, double a, double b, double c, double *s)
{
    for (int i = 0; i < NB; i++) {
        if (kind == 'g') {
            double d = (grid_nm(i) - a) / b;
            s[i] = c * exp(-0.5 * d * d);
        } else if (kind == 'c') {
            s[i] = a;
        } else if (kind == 'p') {
            double t = (grid_nm(i) - 400.0) / 300.0;
            double env = sin(3.14159265358979323846 * t);
            if (env < 0.0) env = 0.0;
            s[i] = a + b * env;
        } else {
            s[i] = 0.0;
        }
    }
}

static void build_from_rows(const StockRow *R, OStock *S)
{
    memset(S, 0, sizeof(*S));
    S->box_iso = R->box_iso;
    S->nl = R->nl;
    for (int li = 0; li < R->nl; li++) {
        const LayerRow *r = &R->l[li];
        OLayer *L = &S->l[li];
        L->kind = r->kind;
        L->thickness = r->thick;
        L->has_sens = r->sens != 0;
        row_curve(r->sens, r->sa, r->sb, r->sc, L->sens);
        L->gamma = r->gamma;
        L->capture_k = r->k;
        L->recip_p = r->p;
        L->reversal = R->reversal;
        if (r->kind != LK_EMULSION) continue;
        L->mu_ln = log(r->mean_um);
        L->sigma_ln = r->sig_ln;
        L->fraction = r->frac;
        row_curve(r->eps, r->ea, r->eb, r->ec, L->eps);
        L->has_mask = r->mask;
        if (r->mask)
            for (int i = 0; i < NB; i++) {
                double l = grid_nm(i);
                double bd = (l - 450.0) / 50.0, gd = (l - 520.0) / 60.0;
                double blue = exp(-0.5 * (bd * bd));
                double green = 0.6 * exp(-0.5 * (gd * gd));
                L->mask_eps[i] = R->mask_b * blue + R->mask_g * green + R->mask_0;
            }
        L->dmax = r->dmax;
    }
    row_curve(R->refl, R->ra, R->rb, R->rc, S->refl);
    S->psf_local = R->psf_local;
    S->psf_halation = R->psf_halation;
    S->dev_diff = R->dev_diff;
    S->adj_beta = R->adj_beta;
    S->dir_diff = R->dir_diff;
    S->dir_n = R->dir_n;
    for (int i = 0; i < R->dir_n; i++)
        for (int j = 0; j < R->dir_n; j++) S->dir[i][j] = R->dir[i][j];
    for (int i = 0; i < NB; i++) S->scanner[i] = 1.0;
    finalize(S);
}

#define OVERCOAT_ROW {LK_OVERCOAT, 1.0f, 'c', 0.01, 0, 0, 0, 0, 0.0f, 0, 0, 0, 0, 0, 0.0f, 1.0f, 1.0, 1.0f}
#define ABSORBER_ROW(kind, thick, a, b, c) {kind, thick, 'g', a, b, c, 0, 0, 0.0f, 0, 0, 0, 0, 0, 0.0f, 1.0f, 1.0, 1.0f}
#define EMULSION_ROW(thick, sa, sb, sc, mean, sig, frac, ea, eb, ec, mask, dmax, gamma, k, p) \
    {LK_EMULSION, thick, 'g', sa, sb, sc, mean, sig, frac, 'g', ea, eb, ec, mask, dmax, gamma, k, p}

/* ColorNeg200 (film/stock/color_neg_200.rs:67-208) */
static const StockRow ROW_COLORNEG200 = {
    200.0f, 0.35, 0.25, 0.05, 'g', 680.0, 60.0, 0.08,
    3.0f, 80.0f, 8.0f, 0.35f, 15.0f, 0, 6,
    {
        OVERCOAT_ROW,
        EMULSION_ROW(4.0f, 450.0, 35.0, 1.0, 0.55, 0.3, 0.18f, 450.0, 40.0, 1.0, 1, 2.2f, 0.65f, 4.2, 0.88f),
        ABSORBER_ROW(LK_FILTER, 2.0f, 430.0, 40.0, 1.2),
        EMULSION_ROW(5.0f, 550.0, 40.0, 1.0, 0.6, 0.32, 0.18f, 550.0, 40.0, 1.0, 1, 2.2f, 0.65f, 2.1, 0.9f),
        EMULSION_ROW(6.0f, 650.0, 45.0, 1.0, 0.7, 0.35, 0.18f, 650.0, 45.0, 1.0, 1, 2.2f, 0.65f, 1.35, 0.92f),
        ABSORBER_ROW(LK_AH, 2.0f, 650.0, 80.0, 0.3),
    },
    3,
    {{0.02f, 0.05f, 0.03f}, {0.05f, 0.02f, 0.06f}, {0.03f, 0.06f, 0.02f}},
};
/* Portra400 (film/stock/portra_400.rs:42-245) */
static const StockRow ROW_PORTRA400 = {
    400.0f, 0.32, 0.22, 0.04, 'g', 680.0, 60.0, 0.06,
    3.0f, 70.0f, 7.0f, 0.3f, 16.0f, 0, 9,
    {
        OVERCOAT_ROW,
        EMULSION_ROW(2.5f, 450.0, 35.0, 1.0, 0.85, 0.35, 0.16f, 450.0, 40.0, 1.0, 1, 1.1f, 0.54f, 4.8, 0.85f),
        EMULSION_ROW(2.5f, 450.0, 35.0, 0.8, 0.42, 0.28, 0.2f, 450.0, 40.0, 1.0, 1, 1.1f, 0.54f, 2.2, 0.89f),
        ABSORBER_ROW(LK_FILTER, 2.0f, 430.0, 40.0, 1.3),
        EMULSION_ROW(3.0f, 550.0, 40.0, 1.0, 0.9, 0.35, 0.16f, 550.0, 40.0, 1.0, 1, 1.1f, 0.54f, 2.4, 0.87f),
        EMULSION_ROW(3.0f, 550.0, 40.0, 0.8, 0.45, 0.28, 0.2f, 550.0, 40.0, 1.0, 1, 1.1f, 0.54f, 1.1, 0.91f),
        EMULSION_ROW(3.5f, 650.0, 45.0, 1.0, 0.95, 0.35, 0.16f, 650.0, 45.0, 1.0, 1, 1.1f, 0.54f, 1.5, 0.89f),
        EMULSION_ROW(3.5f, 650.0, 45.0, 0.8, 0.48, 0.28, 0.2f, 650.0, 45.0, 1.0, 1, 1.1f, 0.54f, 0.7, 0.93f),
        ABSORBER_ROW(LK_AH, 2.0f, 650.0, 80.0, 0.3),
    },
    6,
    {{0.02f, 0.01f, 0.04f, 0.02f, 0.03f, 0.01f}, {0.01f, 0.01f, 0.02f, 0.01f, 0.02f, 0.01f}, {0.04f, 0.02f, 0.02f, 0.01f, 0.05f, 0.02f}, {0.02f, 0.01f, 0.01f, 0.01f, 0.02f, 0.01f}, {0.03f, 0.01f, 0.05f, 0.02f, 0.02f, 0.01f}, {0.01f, 0.01f, 0.02f, 0.01f, 0.01f, 0.01f}},
};
/* Ektar100 (film/stock/ektar_100.rs:46-270) */
static const StockRow ROW_EKTAR100 = {
    100.0f, 0.38, 0.26, 0.05, 'g', 680.0, 60.0, 0.05,
    2.5f, 55.0f, 6.0f, 0.55f, 14.0f, 0, 9,
    {
        OVERCOAT_ROW,
        EMULSION_ROW(2.8f, 450.0, 32.0, 1.0, 0.82, 0.32, 0.17f, 450.0, 30.0, 1.25, 1, 1.25f, 0.58f, 4.8, 0.86f),
        EMULSION_ROW(2.5f, 450.0, 32.0, 0.85, 0.38, 0.24, 0.21f, 450.0, 30.0, 1.25, 1, 1.9f, 0.34f, 6.5, 0.9f),
        ABSORBER_ROW(LK_FILTER, 2.0f, 430.0, 38.0, 1.35),
        EMULSION_ROW(3.2f, 545.0, 36.0, 1.0, 0.88, 0.32, 0.17f, 545.0, 30.0, 1.25, 1, 1.25f, 0.58f, 2.6, 0.88f),
        EMULSION_ROW(3.0f, 545.0, 36.0, 0.85, 0.4, 0.24, 0.21f, 545.0, 30.0, 1.25, 1, 1.9f, 0.34f, 3.6, 0.92f),
        EMULSION_ROW(3.6f, 650.0, 40.0, 1.0, 0.92, 0.32, 0.17f, 650.0, 32.0, 1.25, 1, 1.25f, 0.58f, 1.6, 0.9f),
        EMULSION_ROW(3.5f, 650.0, 40.0, 0.85, 0.42, 0.24, 0.21f, 650.0, 32.0, 1.25, 1, 1.9f, 0.34f, 2.4, 0.94f),
        ABSORBER_ROW(LK_AH, 2.0f, 650.0, 80.0, 0.25),
    },
    6,
    {{0.03f, 0.02f, 0.09f, 0.04f, 0.07f, 0.03f}, {0.02f, 0.02f, 0.04f, 0.02f, 0.04f, 0.02f}, {0.09f, 0.04f, 0.03f, 0.02f, 0.1f, 0.04f}, {0.04f, 0.02f, 0.02f, 0.02f, 0.04f, 0.02f}, {0.07f, 0.03f, 0.1f, 0.04f, 0.03f, 0.02f}, {0.03f, 0.02f, 0.04f, 0.02f, 0.02f, 0.02f}},
};
/* FujiPro400H (film/stock/fuji_pro_400h.rs:43-271) */
static const StockRow ROW_FUJIPRO400H = {
    400.0f, 0.28, 0.2, 0.03, 'g', 670.0, 50.0, 0.05,
    2.5f, 65.0f, 6.5f, 0.32f, 14.0f, 0, 10,
    {
        OVERCOAT_ROW,
        EMULSION_ROW(2.5f, 445.0, 35.0, 1.0, 0.82, 0.33, 0.17f, 445.0, 40.0, 1.0, 1, 1.1f, 0.56f, 4.5, 0.86f),
        EMULSION_ROW(2.5f, 445.0, 35.0, 0.8, 0.4, 0.28, 0.19f, 445.0, 40.0, 1.0, 1, 1.1f, 0.56f, 2.1, 0.9f),
        ABSORBER_ROW(LK_FILTER, 2.0f, 430.0, 40.0, 1.3),
        EMULSION_ROW(2.0f, 490.0, 30.0, 0.9, 0.5, 0.3, 0.15f, 650.0, 45.0, 0.6, 1, 0.5f, 0.56f, 2.0, 0.88f),
        EMULSION_ROW(3.0f, 545.0, 40.0, 1.0, 0.88, 0.34, 0.17f, 545.0, 40.0, 1.0, 1, 1.1f, 0.56f, 2.3, 0.87f),
        EMULSION_ROW(3.0f, 545.0, 40.0, 0.8, 0.44, 0.28, 0.19f, 545.0, 40.0, 1.0, 1, 1.1f, 0.56f, 1.1, 0.91f),
        EMULSION_ROW(3.5f, 650.0, 45.0, 1.0, 0.92, 0.34, 0.17f, 650.0, 45.0, 1.0, 1, 1.1f, 0.56f, 1.4, 0.89f),
        EMULSION_ROW(3.5f, 650.0, 45.0, 0.8, 0.46, 0.28, 0.19f, 650.0, 45.0, 1.0, 1, 1.1f, 0.56f, 0.7, 0.93f),
        ABSORBER_ROW(LK_AH, 2.0f, 650.0, 80.0, 0.3),
    },
    7,
    {{0.02f, 0.01f, 0.03f, 0.04f, 0.02f, 0.03f, 0.01f}, {0.01f, 0.01f, 0.02f, 0.02f, 0.01f, 0.02f, 0.01f}, {0.03f, 0.02f, 0.02f, 0.06f, 0.03f, 0.04f, 0.02f}, {0.04f, 0.02f, 0.05f, 0.02f, 0.01f, 0.05f, 0.02f}, {0.02f, 0.01f, 0.02f, 0.01f, 0.01f, 0.02f, 0.01f}, {0.03f, 0.01f, 0.04f, 0.05f, 0.02f, 0.02f, 0.01f}, {0.01f, 0.01f, 0.02f, 0.02f, 0.01f, 0.01f, 0.01f}},
};
/* EktachromeE100 (film/stock/ektachrome_e100.rs:28-157) */
static const StockRow ROW_EKTACHROMEE100 = {
    100.0f, 0.0, 0.0, 0.0, 'g', 660.0, 40.0, 0.02,
    1.5f, 40.0f, 4.0f, 0.4f, 8.0f, 1, 6,
    {
        OVERCOAT_ROW,
        EMULSION_ROW(4.0f, 440.0, 30.0, 1.0, 0.42, 0.25, 0.22f, 440.0, 35.0, 1.0, 0, 3.2f, 1.65f, 3.5, 0.93f),
        ABSORBER_ROW(LK_FILTER, 2.0f, 430.0, 35.0, 1.4),
        EMULSION_ROW(4.0f, 545.0, 35.0, 1.0, 0.45, 0.25, 0.22f, 545.0, 35.0, 1.0, 0, 3.2f, 1.65f, 1.8, 0.94f),
        EMULSION_ROW(5.0f, 650.0, 40.0, 1.0, 0.5, 0.26, 0.22f, 650.0, 40.0, 1.0, 0, 3.2f, 1.65f, 1.1, 0.95f),
        ABSORBER_ROW(LK_AH, 2.0f, 650.0, 80.0, 0.3),
    },
    3,
    {{0.01f, 0.02f, 0.01f}, {0.02f, 0.01f, 0.02f}, {0.01f, 0.02f, 0.01f}},
};
/* BwStub (film/stock/bw_stub.rs:18-82) */
static const StockRow ROW_BWSTUB = {
    100.0f, 0.0, 0.0, 0.0, 'c', 0.0, 0.0, 0.0,
    2.0f, 40.0f, 5.0f, 0.3f, 10.0f, 0, 1,
    {
        {LK_EMULSION, 10.0f, 'p', 0.3, 0.7, 0, 0.7, 0.35, 0.2f, 'c', 1.0, 0, 0, 0, 2.5f, 0.65f, 1.0, 1.0f},
    },
    1,
    {{0.0f}},
};
/* TriX400 (film/stock/trix_400.rs:30-91) */
static const StockRow ROW_TRIX400 = {
    400.0f, 0.0, 0.0, 0.0, 'c', 0.01, 0.0, 0.0,
    3.5f, 50.0f, 6.0f, 0.35f, 12.0f, 0, 2,
    {
        {LK_EMULSION, 6.0f, 'p', 0.35, 0.65, 0, 0.95, 0.38, 0.22f, 'c', 1.0, 0, 0, 0, 1.5f, 0.70f, 2.2, 0.85f},
        {LK_EMULSION, 6.0f, 'p', 0.35, 0.65, 0, 0.45, 0.28, 0.24f, 'c', 1.0, 0, 0, 0, 1.5f, 0.70f, 0.9, 0.89f},
    },
    2,
    {{0.03f, 0.02f}, {0.02f, 0.02f}},
};

/* StockId order (film/stock/mod.rs:126-147). */
static int load_stock(int id, OStock *S)
{
    static const StockRow *const rows[] = {&ROW_BWSTUB, &ROW_COLORNEG200, &ROW_PORTRA400, &ROW_EKTAR100,
                                          &ROW_FUJIPRO400H, &ROW_EKTACHROMEE100, &ROW_TRIX400};
    if (id < 0 || id > 6) return 0;
    build_from_rows(rows[id], S);
    return 1;
}

/* ----------------------------------------------------------------------- */
/* separable Gaussian blur (film/blur.rs:10-89)                              */

static long reflect_index(long i, long n)
{
    if (n == 0) return 0;
    long x = i;
    for (;;) {
        if (x < 0) x = -x;
        else if (x >= n) x = 2 * n - 2 - x;
        else return x;
        if (n == 1) return 0;
    }
}

/* Gaussian taps: radius max(ceil(3 sigma), 1), normalised to sum 1. */
static int blur_kernel(real sigma, real **out)
{
    real r3 = RCEIL(K(3.0) * sigma);
    if (r3 < K(1.0)) r3 = K(1.0);
    int radius = (int)r3;
    real *k = (real *)malloc(sizeof(real) * (2 * radius + 1));
    real inv = K(1.0) / (K(2.0) * sigma * sigma);
    real sum = K(0.0);
    for (int i = 0; i < 2 * radius + 1; i++) {
        real x = (real)i - (real)radius;
        real v = REXP(-x * x * inv);
        k[i] = v;
        sum += v;
    }
    for (int i = 0; i < 2 * radius + 1; i++) k[i] /= sum;
    *out = k;
    return radius;
}

/* Horizontal then vertical 1-D passes with mirror reflection.  `radius_override`
 * >= 0 fixes the tap radius (the baseline preset's halation). */
typedef struct {
    const real *src;
    real *dst;
    int W, H, radius;
    const real *k;
} BlurJob;

static void blur_rows_job(void *p, int worker, long b, long e)
{
    BlurJob *j = (BlurJob *)p;
    (void)worker;
    for (long y = b; y < e; y++)
        for (int x = 0; x < j->W; x++) {
            real acc = K(0.0);
            for (int t = 0; t < 2 * j->radius + 1; t++) {
                long xx = reflect_index((long)x + t - j->radius, j->W);
                acc += j->src[(size_t)y * j->W + xx] * j->k[t];
            }
            j->dst[(size_t)y * j->W + x] = acc;
        }
}

static void blur_cols_job(void *p, int worker, long b, long e)
{
    BlurJob *j = (BlurJob *)p;
    (void)worker;
    for (long y = b; y < e; y++)
        for (int x = 0; x < j->W; x++) {
            real acc = K(0.0);
            for (int t = 0; t < 2 * j->radius + 1; t++) {
                long yy = reflect_index(y + t - j->radius, j->H);
                acc += j->src[(size_t)yy * j->W + x] * j->k[t];
            }
            j->dst[(size_t)y * j->W + x] = acc;
        }
}

static int g_threads = 1; /* worker threads for the film oracle's loops */

/* Horizontal then vertical 1-D passes with mirror reflection. */
static void blur_taps(real *buf, int W, int H, const real *k, int radius)
{
    size_t n = (size_t)W * H;
    real *tmp = (real *)malloc(sizeof(real) * n);
    BlurJob a = {buf, tmp, W, H, radius, k};
    oracle_parallel_for(H, 8, g_threads, blur_rows_job, &a);
    BlurJob c = {tmp, buf, W, H, radius, k};
    oracle_parallel_for(H, 8, g_threads, blur_cols_job, &c);
    free(tmp);
}

void OSYM(oracle_blur)(real *buf, int W, int H, real sigma)
{
    if (sigma < K(1e-3) || W == 0 || H == 0) return;
    real *k;
    int radius = blur_kernel(sigma, &k);
    blur_taps(buf, W, H, k, radius);
    free(k);
}

/* Gaussian taps of the baseline preset's halation: fixed radius, so the
 * output is a smooth function of sigma. */
static void fixed_radius_taps(real sigma, int radius, real *k)
{
    real inv = K(1.0) / (K(2.0) * sigma * sigma);
    real sum = K(0.0);
    for (int i = 0; i < 2 * radius + 1; i++) {
        real x = (real)i - (real)radius;
        real v = REXP(-x * x * inv);
        k[i] = v;
        sum += v;
    }
    for (int i = 0; i < 2 * radius + 1; i++) k[i] /= sum;
}

/* ----------------------------------------------------------------------- */
/* SplitMix64 + Irwin-Hall noise (film/development/grain.rs:20-45, 71-82)   */

static inline uint64_t splitmix_next(uint64_t *s)
{
    *s += 0x9E3779B97F4A7C15ull;
    uint64_t z = *s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline real irwin_hall(uint64_t *s)
{
    real acc = K(0.0);
    for (int i = 0; i < 12; i++) {
#ifdef ORACLE_F32
        acc += (float)splitmix_next(s) / (float)UINT64_MAX;
#else
        acc += (double)splitmix_next(s) / (double)UINT64_MAX;
#endif
    }
    return acc - K(6.0);
}

void OSYM(oracle_grain_noise)(real *noise, int W, int H, uint64_t seed, int layer)
{
    for (int y = 0; y < H; y++) {
        uint64_t s = seed * 0xD1B54A32D192ED03ull + (uint64_t)layer * 0x9E3779B97F4A7C15ull + (uint64_t)y;
        for (int x = 0; x < W; x++) noise[(size_t)y * W + x] = irwin_hall(&s);
    }
}

/* blurred unit-variance noise plane (grain.rs:69-90): returns norm */
static real grain_field(real *noise, int W, int H, uint64_t seed, int layer, real sigma_px)
{
    OSYM(oracle_grain_noise)(noise, W, H, seed, layer);
    OSYM(oracle_blur)(noise, W, H, sigma_px > K(1.0) ? sigma_px : K(1.0));
    size_t n = (size_t)W * H;
    double var = 0.0;
    for (size_t i = 0; i < n; i++) var += (double)noise[i] * (double)noise[i];
    var /= (double)n;
    return var > 1e-12 ? (real)(float)(1.0 / sqrt(var)) : K(1.0);
}

/* ----------------------------------------------------------------------- */
/* film::process for the reference stocks                                    */

typedef struct {
    int E;
    int em_idx[MAXL];
} EmList;

static EmList emulsions(const OStock *S)
{
    EmList e;
    e.E = 0;
    for (int i = 0; i < S->nl; i++)
        if (S->l[i].kind == LK_EMULSION) e.em_idx[e.E++] = i;
    return e;
}

static double curve_eval(const double *s, double lam)
{
    if (lam <= grid_nm(0)) return s[0];
    if (lam >= grid_nm(NB - 1)) return s[NB - 1];
    for (int i = 0; i < NB - 1; i++)
        if (lam >= grid_nm(i) && lam <= grid_nm(i + 1)) {
            double t = (lam - grid_nm(i)) / (grid_nm(i + 1) - grid_nm(i));
            return s[i] * (1.0 - t) + s[i + 1] * t;
        }
    return s[NB - 1];
}

static double curve_integrate(const double *s)
{
    double acc = 0.0;
    for (int i = 0; i < NB - 1; i++) acc += 0.5 * (s[i] + s[i + 1]) * (grid_nm(i + 1) - grid_nm(i));
    return acc;
}

static double curve_peak(const double *s)
{
    double mv = -INFINITY, pk = 550.0;
    for (int i = 0; i < NB; i++)
        if (s[i] > mv) { mv = s[i]; pk = grid_nm(i); }
    return pk;
}

/* Emulsion absorbed band-mean fluence per pixel (exposure/mod.rs:45-81,
 * absorption.rs:24-108) into E planes of `real`. */
static void expose_absorb(const OStock *S, const Basis *B, const real *rgb, size_t n, real **planes)
{
    EmList em = emulsions(S);
    for (size_t p = 0; p < n; p++) {
        double phi[NB];
        fluence_spectrum(B, rgb + 3 * p, phi);
        int e = 0;
        for (int li = 0; li < S->nl; li++) {
            const OLayer *L = &S->l[li];
            double ab[NB];
            memset(ab, 0, sizeof ab);
            if (L->kind == LK_EMULSION) {
                double rho = (double)L->fraction, th = (double)L->thickness;
                for (int i = 0; i < NB; i++) {
                    double sigma = L->sens[i] * 2.0;
                    double od = sigma * rho * th;
                    double tr = exp(-od);
                    double pt = phi[i] * tr;
                    ab[i] = phi[i] - pt;
                    phi[i] = pt;
                }
            } else if (L->kind != LK_SUPPORT && L->has_sens) {
                double th = (double)L->thickness;
                for (int i = 0; i < NB; i++) {
                    double od = L->sens[i] * th;
                    double tr = exp(-od);
                    double pt = phi[i] * tr;
                    ab[i] = phi[i] - pt;
                    phi[i] = pt;
                }
            }
            if (L->kind == LK_EMULSION) {
                double acc = 0.0;
                for (int i = 0; i < NB - 1; i++) acc += 0.5 * (ab[i] + ab[i + 1]) * 20.0;
                planes[e][p] = (real)(float)(acc / 300.0);
#ifndef ORACLE_F32
                planes[e][p] = acc / 300.0;
#endif
                e++;
            }
        }
        (void)em;
    }
}

/* Local scatter + wide support bounce (halation.rs:24-93). */
static void spatial_effects(const OStock *S, real **planes, int E, int W, int H, real pitch)
{
    size_t n = (size_t)W * H;
    real pm = pitch > K(1e-6) ? pitch : K(1e-6);
    real s_loc = (real)S->psf_local / pm;
    if (s_loc < 0) s_loc = 0;
    const real mix = K(0.18);
    if (s_loc >= K(1e-3)) {
        real *tmp = (real *)malloc(sizeof(real) * n);
        for (int e = 0; e < E; e++) {
            memcpy(tmp, planes[e], sizeof(real) * n);
            OSYM(oracle_blur)(tmp, W, H, s_loc);
            real keep = K(1.0) - mix;
            for (size_t p = 0; p < n; p++) planes[e][p] = keep * planes[e][p] + mix * tmp[p];
        }
        free(tmp);
    }
    real s_wide = (real)S->psf_halation / pm;
    if (s_wide < 0) s_wide = 0;
    if (s_wide < K(1e-3)) return;
    const double bands[4] = {450.0, 550.0, 650.0, 700.0};
    real maxr = K(0.0);
    for (int b = 0; b < 4; b++) {
        real r = (real)(float)curve_eval(S->refl, bands[b]);
        maxr = RMAX(maxr, r);
    }
    if (maxr <= K(0.0)) return;
    EmList em = emulsions(S);
    real *bounce = (real *)malloc(sizeof(real) * n);
    memcpy(bounce, planes[E - 1], sizeof(real) * n);
    OSYM(oracle_blur)(bounce, W, H, s_wide);
    const real bw[3] = {K(0.20), K(0.45), K(1.0)};
    for (int e = 0; e < E; e++) {
        const OLayer *L = &S->l[em.em_idx[e]];
        double pk = curve_peak(L->sens);
        real w;
        if (pk <= 450.0) w = bw[0];
        else if (pk <= 550.0) w = bw[0] + (bw[1] - bw[0]) * (real)(float)((pk - 450.0) / 100.0);
        else if (pk <= 650.0) w = bw[1] + (bw[2] - bw[1]) * (real)(float)((pk - 550.0) / 100.0);
        else w = bw[2];
        double norm = curve_integrate(L->sens);
        real r_e;
        if (norm <= 1e-9) {
            r_e = (real)(float)curve_eval(S->refl, 650.0);
        } else {
            double prod[NB];
            for (int i = 0; i < NB; i++) prod[i] = S->refl[i] * L->sens[i];
            r_e = (real)(float)(curve_integrate(prod) / norm);
        }
        real gain = r_e * w;
        if (gain <= K(0.0)) continue;
        for (size_t p = 0; p < n; p++) planes[e][p] += gain * bounce[p];
    }
    free(bounce);
}

static double reciprocity(double t, double p)
{
    if (t <= 1.0 || p >= 0.9999) return 1.0;
    return pow(t > 1.0 ? t : 1.0, p - 1.0);
}

typedef struct { real *img[MAXL]; real *mask[MAXL]; } Dyes;

/* expose -> develop (reduce, DIR, adjacency, grain): exposure/mod.rs:45-122,
 * development/mod.rs:18-48. */
static void expose_develop(const OStock *S, const Basis *B, const real *rgb, int W, int H, real pitch, real shutter,
                           uint64_t seed, int grain_on, Dyes *D)
{
    size_t n = (size_t)W * H;
    EmList em = emulsions(S);
    int E = em.E;
    real *lat[MAXL];
    for (int e = 0; e < E; e++) lat[e] = (real *)calloc(n, sizeof(real));
    expose_absorb(S, B, rgb, n, lat);
    spatial_effects(S, lat, E, W, H, pitch);
    for (int e = 0; e < E; e++) {
        const OLayer *L = &S->l[em.em_idx[e]];
        real eta = (real)(float)reciprocity((double)(float)shutter, (double)L->recip_p);
        for (size_t p = 0; p < n; p++) {
            real prod = lat[e][p] * eta;
            lat[e][p] = (real)(float)lut_sample(L, (double)prod);
#ifndef ORACLE_F32
            lat[e][p] = lut_sample(L, (double)prod);
#endif
        }
    }
    /* reduce (reduction.rs:16-68) */
    for (int e = 0; e < E; e++) {
        const OLayer *L = &S->l[em.em_idx[e]];
        real dmax = (real)L->dmax;
        real gam = RMAX((real)L->gamma, K(1e-6));
        real ig = K(1.0) / gam;
        D->img[e] = (real *)malloc(sizeof(real) * n);
        D->mask[e] = (real *)malloc(sizeof(real) * n);
        for (size_t p = 0; p < n; p++) {
            real f = lat[e][p];
            if (f < K(0.0)) f = K(0.0);
            if (f > K(1.0)) f = K(1.0);
            real ef = L->reversal ? K(1.0) - f : f;
            D->img[e][p] = dmax * RPOW(ef, ig);
        }
        if (L->has_mask) {
            real ms = dmax * K(0.4);
            for (size_t p = 0; p < n; p++) {
                real r = D->img[e][p] / dmax;
                if (r < K(0.0)) r = K(0.0);
                if (r > K(1.0)) r = K(1.0);
                D->mask[e][p] = ms * (K(1.0) - r);
            }
        } else {
            memset(D->mask[e], 0, sizeof(real) * n);
        }
        free(lat[e]);
    }
    real pm = pitch > K(1e-6) ? pitch : K(1e-6);
    /* DIR inhibition (diffusion.rs:39-84) */
    real s_dir = (real)S->dir_diff / pm;
    if (E > 0 && S->dir_n > 0 && s_dir >= K(1e-3)) {
        real *inh[MAXL];
        for (int i = 0; i < E; i++) {
            inh[i] = (real *)malloc(sizeof(real) * n);
            memcpy(inh[i], D->img[i], sizeof(real) * n);
            OSYM(oracle_blur)(inh[i], W, H, s_dir);
        }
        real *tot = (real *)malloc(sizeof(real) * n);
        for (int j = 0; j < E; j++) {
            memset(tot, 0, sizeof(real) * n);
            int active = 0;
            for (int i = 0; i < E; i++) {
                if (i < S->dir_n && j < S->dir_n) {
                    real w = (real)S->dir[i][j];
                    if (RABS(w) > K(1e-6)) {
                        active = 1;
                        for (size_t p = 0; p < n; p++) tot[p] += w * inh[i][p];
                    }
                }
            }
            if (active)
                for (size_t p = 0; p < n; p++) D->img[j][p] *= REXP(-tot[p]);
        }
        free(tot);
        for (int i = 0; i < E; i++) free(inh[i]);
    }
    /* adjacency (diffusion.rs:11-28) */
    real s_adj = (real)S->dev_diff / pm;
    real beta = (real)S->adj_beta;
    if (!(RABS(beta) < K(1e-8) || s_adj < K(1e-3))) {
        real *bl = (real *)malloc(sizeof(real) * n);
        for (int e = 0; e < E; e++) {
            memcpy(bl, D->img[e], sizeof(real) * n);
            OSYM(oracle_blur)(bl, W, H, s_adj);
            for (size_t p = 0; p < n; p++) D->img[e][p] += beta * (D->img[e][p] - bl[p]);
        }
        free(bl);
    }
    /* grain (grain.rs:53-100) */
    if (grain_on) {
        real s_g = K(3.0) / pm;
        real *noise = (real *)malloc(sizeof(real) * n);
        for (int e = 0; e < E; e++) {
            const OLayer *L = &S->l[em.em_idx[e]];
            real dmax = (real)L->dmax;
            real kappa = ((real)L->kappa / pm) * K(0.15);
            if (kappa <= K(0.0) || dmax <= K(0.0)) continue;
            real norm = grain_field(noise, W, H, seed, e, s_g);
            for (size_t p = 0; p < n; p++) {
                real d = D->img[e][p];
                real dens = d < K(0.0) ? K(0.0) : (d > dmax ? dmax : d);
                real toe = K(0.02) * dmax;
                real taper = RMIN(dens / (dens + toe), K(1.0));
                real sd = taper * RSQRT(RMAX(dens * (dmax - dens), K(0.0)));
                d = dens + kappa * sd * noise[p] * norm;
                real hi = dmax * K(1.05);
                if (d < K(0.0)) d = K(0.0);
                if (d > hi) d = hi;
                D->img[e][p] = d;
            }
        }
        free(noise);
    }
}

/* density -> transmittance -> AP1 for one pixel (densitometry.rs:13-73). */
static void scan_pixel(const OStock *S, const real *di, const real *dm, double out[3])
{
    EmList em = emulsions(S);
    double d[NB];
    memset(d, 0, sizeof d);
    for (int e = 0; e < em.E; e++) {
        const OLayer *L = &S->l[em.em_idx[e]];
        double a = (double)di[e], m = (double)dm[e];
        for (int i = 0; i < NB; i++) {
            d[i] += a * L->eps[i];
            if (L->has_mask) d[i] += m * L->mask_eps[i];
        }
    }
    double t[NB];
    for (int i = 0; i < NB; i++) t[i] = pow(10.0, -d[i]) * S->scanner[i];
    spectrum_to_ap1(t, out);
}

static void dmin_rgb(const OStock *S, double out[3])
{
    EmList em = emulsions(S);
    real di[MAXL], dm[MAXL];
    for (int e = 0; e < em.E; e++) {
        const OLayer *L = &S->l[em.em_idx[e]];
        di[e] = K(0.0);
        dm[e] = L->has_mask ? (real)L->dmax * K(0.4) : K(0.0);
    }
    scan_pixel(S, di, dm, out);
}

static void scan_all(const OStock *S, const Dyes *D, int E, size_t n, real *rgb)
{
    double dmn[3];
    dmin_rgb(S, dmn);
    double peak = dmn[0] > dmn[1] ? dmn[0] : dmn[1];
    if (dmn[2] > peak) peak = dmn[2];
    if (peak < 1e-12) peak = 1e-12;
    double scale = 1.0 / peak;
    for (size_t p = 0; p < n; p++) {
        real di[MAXL], dm[MAXL];
        for (int e = 0; e < E; e++) { di[e] = D->img[e][p]; dm[e] = D->mask[e][p]; }
        double o[3];
        scan_pixel(S, di, dm, o);
        for (int c = 0; c < 3; c++) {
            float raw = (float)o[c];
            rgb[3 * p + c] = (real)(float)((double)raw * scale);
#ifndef ORACLE_F32
            rgb[3 * p + c] = o[c] * scale;
#endif
        }
    }
}

static real soft_inv(real inv, real shoulder)
{
    real i = RMAX(inv, K(0.0));
    real s = RMAX(shoulder, K(1e-6));
    return i / (K(1.0) + i / s);
}

/* invert_negative (scan/invert.rs:36-108). */
void OSYM(oracle_invert)(real *buf, size_t n, const real mid[3], const real dmin_in[3])
{
    const real eps = K(1e-6), HEAD = K(8.0), KEEP = K(0.55), FADE = K(0.02);
    real dmin[3], mt[3], im[3], sh[3], sm[3], g[3];
    for (int c = 0; c < 3; c++) {
        dmin[c] = RMAX(dmin_in[c], eps);
        real v = mid[c] / dmin[c];
        if (v < eps) v = eps;
        if (v > K(1.0) - eps) v = K(1.0) - eps;
        mt[c] = v;
        im[c] = RMAX(K(1.0) / mt[c] - K(1.0), K(0.0));
        sh[c] = RMAX(im[c] * HEAD, eps);
    }
    for (int c = 0; c < 3; c++) {
        sm[c] = RMAX(soft_inv(im[c], sh[c]), eps);
        g[c] = MIDDLE_GRAY / sm[c];
    }
    for (size_t p = 0; p < n; p++) {
        real *px = buf + 3 * p;
        real raw[3];
        for (int c = 0; c < 3; c++) {
            real t = px[c] / dmin[c];
            if (t < eps) t = eps;
            if (t > K(1.0)) t = K(1.0);
            real inv = RMAX(K(1.0) / t - K(1.0), K(0.0));
            raw[c] = RMAX(g[c] * soft_inv(inv, sh[c]), K(0.0));
        }
        real y = RMAX(LUM_R * raw[0] + LUM_G * raw[1] + LUM_B * raw[2], K(0.0));
        real k;
        if (y <= K(0.0)) k = K(0.0);
        else if (y >= FADE) k = KEEP;
        else k = KEEP * (y / FADE);
        for (int c = 0; c < 3; c++) px[c] = RMAX(y + k * (raw[c] - y), K(0.0));
    }
}

static void free_dyes(Dyes *D, int E)
{
    for (int e = 0; e < E; e++) { free(D->img[e]); free(D->mask[e]); }
}

/* relative -> absolute luminance at sunny-16 for a box ISO (film/mod.rs:155-166). */
static real rel_to_abs_y(real y, real box_iso)
{
    float s = (float)box_iso > 1.0f ? (float)box_iso : 1.0f;
    float t = 1.0f / s;
    double l = 12.5 * (double)(float)y * (8.0 * 8.0) / ((double)t * (double)s);
    return (real)(float)l;
}

/* film::process.  stock: 0 BwStub, 1 ColorNeg200.  format: 0 35mm, 1 6x6,
 * 2 4x5.  output: 0 NegativeLinear, 1 PositiveLinear.  shutter < 0 means
 * "not in metadata" (1 / box ISO).  grain_on = 0 skips grain (parity mode). */
int OSYM(oracle_film_process)(real *rgb, int W, int H, int stock_id, int format, uint64_t seed, int output,
                              real shutter, int grain_on)
{
    if (W <= 0 || H <= 0 || !rgb) return ORACLE_ERR_ARG;
    OStock S;
    if (!load_stock(stock_id, &S)) return ORACLE_ERR_ARG;
    const float fw[3] = {36.0f, 56.0f, 101.6f};
    if (format < 0 || format > 2) return ORACLE_ERR_ARG;
    real pitch = (real)(fw[format] * 1000.0f / (float)W);
#ifndef ORACLE_F32
    pitch = (double)fw[format] * 1000.0 / (double)W;
#endif
    real sh = shutter >= 0 ? shutter : (real)(1.0f / S.box_iso);
    Basis B;
    basis_build(&B);
    size_t n = (size_t)W * H;
    EmList em = emulsions(&S);
    Dyes D;
    expose_develop(&S, &B, rgb, W, H, pitch, sh, seed, grain_on, &D);
    scan_all(&S, &D, em.E, n, rgb);
    free_dyes(&D, em.E);
    int reversal = 0;
    for (int i = 0; i < S.nl; i++) reversal |= S.l[i].reversal;
    if (!reversal && output == 1) {
        double dmn[3];
        dmin_rgb(&S, dmn);
        double pk = dmn[0] > dmn[1] ? dmn[0] : dmn[1];
        if (dmn[2] > pk) pk = dmn[2];
        if (pk < 1e-12) pk = 1e-12;
        real dmin[3] = {(real)(float)(dmn[0] / pk), (real)(float)(dmn[1] / pk), (real)(float)(dmn[2] / pk)};
        /* mid-gray negative: 32x32 patch through the same path, seed 0 */
        const int NM = 32;
        real g = rel_to_abs_y(MIDDLE_GRAY, (real)S.box_iso);
        real *patch = (real *)malloc(sizeof(real) * NM * NM * 3);
        for (int i = 0; i < NM * NM * 3; i++) patch[i] = g;
        Dyes Dm;
        expose_develop(&S, &B, patch, NM, NM, pitch, sh, 0, grain_on, &Dm);
        scan_all(&S, &Dm, em.E, (size_t)NM * NM, patch);
        free_dyes(&Dm, em.E);
        double acc[3] = {0, 0, 0};
        for (int i = 0; i < NM * NM; i++)
            for (int c = 0; c < 3; c++) acc[c] += (double)patch[3 * i + c];
        real mid[3];
        for (int c = 0; c < 3; c++) mid[c] = (real)(float)(acc[c] / (double)(NM * NM));
        free(patch);
        OSYM(oracle_invert)(rgb, n, mid, dmin);
    }
    return ORACLE_OK;
}

/* Exposed for known-answer tests. */
double OSYM(oracle_lut_sample)(int stock_id, int layer, double phi)
{
    OStock S;
    if (!load_stock(stock_id, &S)) return NAN;
    EmList em = emulsions(&S);
    if (layer < 0 || layer >= em.E) return NAN;
    return lut_sample(&S.l[em.em_idx[layer]], phi);
}

float OSYM(oracle_layer_kappa)(int stock_id, int layer)
{
    OStock S;
    if (!load_stock(stock_id, &S)) return NAN;
    EmList em = emulsions(&S);
    if (layer < 0 || layer >= em.E) return NAN;
    return S.l[em.em_idx[layer]].kappa;
}

/* Normalised film-base RGB (densitometry.rs:109-117). */
void OSYM(oracle_normalized_dmin)(int stock_id, real out[3])
{
    OStock S;
    load_stock(stock_id, &S);
    double d[3];
    dmin_rgb(&S, d);
    double pk = d[0] > d[1] ? d[0] : d[1];
    if (d[2] > pk) pk = d[2];
    if (pk < 1e-12) pk = 1e-12;
    for (int c = 0; c < 3; c++) out[c] = (real)(float)(d[c] / pk);
}

/* Upsample one ACEScg pixel and integrate back to ACEScg (round trip used
 * by upsample.rs:187-224's tests). */
void OSYM(oracle_upsample_roundtrip)(const real rgb[3], double spectrum[NB], double back[3])
{
    Basis B;
    basis_build(&B);
    double v[3] = {(double)rgb[0], (double)rgb[1], (double)rgb[2]}, w[3];
    matvec3(B.minv, v, w);
    for (int k = 0; k < 3; k++)
        if (w[k] < 0.0) w[k] = 0.0;
    for (int i = 0; i < NB; i++) spectrum[i] = w[0] * B.b[0][i] + w[1] * B.b[1][i] + w[2] * B.b[2][i];
    spectrum_to_ap1(spectrum, back);
}

/* ======================================================================= */
/* Part 2: the baseline preset (81 bins, logistic curves, red-highlight     */
/* halation, seeded grain).                                                  */

#define NB81 81

/* CIE 1931 2-degree observer, multi-lobe Gaussian fit of Wyman, Sloan and
 * Shirley, "Simple Analytic Approximations to the CIE XYZ Color Matching
 * Functions", JCGT 2(2), 2013. */
static double lobe(double x, double mu, double s1, double s2)
{
    double t = (x - mu) / (x < mu ? s1 : s2);
    return exp(-0.5 * t * t);
}

void OSYM(oracle_cmf81)(double *xb, double *yb, double *zb)
{
    for (int i = 0; i < NB81; i++) {
        double l = 380.0 + 5.0 * i;
        xb[i] = 1.056 * lobe(l, 599.8, 37.9, 31.0) + 0.362 * lobe(l, 442.0, 16.0, 26.7) -
                0.065 * lobe(l, 501.1, 20.4, 26.2);
        yb[i] = 0.821 * lobe(l, 568.8, 46.9, 40.5) + 0.286 * lobe(l, 530.9, 16.3, 31.1);
        zb[i] = 1.217 * lobe(l, 437.0, 11.8, 36.0) + 0.681 * lobe(l, 459.0, 26.0, 13.8);
    }
}

/* Parameters of the baseline preset; the struct layout is shared with the
 * CUDA library's ImopsBaselineFilm (include/imops_b200.h). */
typedef struct {
    float dmax[3], k[3], x0[3];   /* logistic density curve per layer */
    float hal_strength;           /* 0.15 */
    float hal_sigma;              /* 20 px */
    int hal_radius;               /* fixed tap radius (64) */
    float hal_threshold;          /* 0.8 on ACEScg red */
    float grain_sigma;            /* 0.02 density */
    float grain_blur;             /* 1 px */
    int grain_on;
    uint64_t seed;
} OBaseline;

static const double SENS_PEAK[3] = {450.0, 550.0, 650.0}, SENS_SIG[3] = {35.0, 40.0, 45.0};
static const double DYE_PEAK[3] = {450.0, 550.0, 650.0}, DYE_SIG[3] = {40.0, 40.0, 45.0};
static const double BLEED[3] = {0.20, 0.45, 1.0};

typedef struct {
    double lam[NB81], trap[NB81];
    double xb[NB81], yb[NB81], zb[NB81];
    double basis[3][NB81], minv[3][3];
    double sens[3][NB81], sens_norm[3];
    double dye[3][NB81];
    double white[3];
} B81;

static void b81_build(B81 *b)
{
    OSYM(oracle_cmf81)(b->xb, b->yb, b->zb);
    for (int i = 0; i < NB81; i++) {
        b->lam[i] = 380.0 + 5.0 * i;
        b->trap[i] = (i == 0 || i == NB81 - 1) ? 2.5 : 5.0;
    }
    double cols[3][3];
    for (int k = 0; k < 3; k++) {
        double x = 0, y = 0, z = 0;
        for (int i = 0; i < NB81; i++) {
            double d = (b->lam[i] - SENS_PEAK[k]) / 40.0;
            b->basis[k][i] = exp(-0.5 * d * d);
            x += b->trap[i] * b->basis[k][i] * b->xb[i];
            y += b->trap[i] * b->basis[k][i] * b->yb[i];
            z += b->trap[i] * b->basis[k][i] * b->zb[i];
        }
        double xyz[3] = {x, y, z};
        matvec3(XYZ2AP1, xyz, cols[k]);
    }
    double m[3][3];
    for (int r = 0; r < 3; r++)
        for (int k = 0; k < 3; k++) m[r][k] = cols[k][r];
    inv3(m, b->minv);
    /* flat reference exposure: the upsampled spectrum of ACEScg (1,1,1) */
    double one[3] = {1, 1, 1}, w1[3];
    matvec3(b->minv, one, w1);
    for (int e = 0; e < 3; e++) {
        double nrm = 0;
        for (int i = 0; i < NB81; i++) {
            double d = (b->lam[i] - SENS_PEAK[e]) / SENS_SIG[e];
            b->sens[e][i] = exp(-0.5 * d * d);
            double s1 = 0;
            for (int k = 0; k < 3; k++) s1 += (w1[k] > 0 ? w1[k] : 0) * b->basis[k][i];
            nrm += b->trap[i] * s1 * b->sens[e][i];
        }
        b->sens_norm[e] = nrm;
        for (int i = 0; i < NB81; i++) {
            double d = (b->lam[i] - DYE_PEAK[e]) / DYE_SIG[e];
            b->dye[e][i] = exp(-0.5 * d * d);
        }
    }
    double x = 0, y = 0, z = 0;
    for (int i = 0; i < NB81; i++) {
        x += b->trap[i] * b->xb[i];
        y += b->trap[i] * b->yb[i];
        z += b->trap[i] * b->zb[i];
    }
    double xyz[3] = {x, y, z};
    matvec3(XYZ2AP1, xyz, b->white);
}

/* Forward of the baseline preset on an ACEScg image (relative scene-linear).
 * Output: scanned negative ACEScg normalised so that D = 0 maps to a peak
 * channel of 1.
 *   w   = max(0, Minv rgb)                        basis weights
 *   s   = sum_k w_k basis_k(lambda)                81-bin spectrum
 *   a_e = sum_i trap_i s_i S_e,i / N_e             layer exposure (1 for rgb=1)
 *   h   = max(0, R - threshold);  B = G_sigma * h  halation (fixed radius)
 *   E_e = a_e + strength * bleed_e * B
 *   D_e = Dmax_e / (1 + exp(-k_e (log10 max(E_e,1e-6) - x0_e)))
 *   D_e += grain_sigma * n_e * norm_e              (seeded SplitMix64 noise)
 *   T   = 10^(-sum_e D_e dye_e(lambda));  rgb = AP1(sum_i trap_i cmf_i T_i) / peak(white)
 */
typedef struct {
    const B81 *b;
    const OBaseline *P;
    real *rgb, *a[3], *hal, *noise[3];
    real norm[3];
    double peak;
} BJob;

static void base_expose_job(void *p, int worker, long pb, long pe)
{
    BJob *j = (BJob *)p;
    const B81 *b = j->b;
    (void)worker;
    for (long q = pb; q < pe; q++) {
        size_t p3 = 3 * (size_t)q;
        double v[3] = {(double)j->rgb[p3], (double)j->rgb[p3 + 1], (double)j->rgb[p3 + 2]}, w[3];
        matvec3(b->minv, v, w);
        for (int k = 0; k < 3; k++)
            if (w[k] < 0) w[k] = 0;
        for (int e = 0; e < 3; e++) {
            double acc = 0;
            for (int i = 0; i < NB81; i++) {
                double s = w[0] * b->basis[0][i] + w[1] * b->basis[1][i] + w[2] * b->basis[2][i];
                acc += b->trap[i] * s * b->sens[e][i];
            }
            j->a[e][q] = (real)(acc / b->sens_norm[e]);
        }
        real h = j->rgb[p3] - (real)j->P->hal_threshold;
        j->hal[q] = h > 0 ? h : 0;
    }
}

static void base_scan_job(void *p, int worker, long pb, long pe)
{
    BJob *j = (BJob *)p;
    const B81 *b = j->b;
    const OBaseline *P = j->P;
    (void)worker;
    for (long q = pb; q < pe; q++) {
        double D[3];
        for (int e = 0; e < 3; e++) {
            double E = (double)j->a[e][q] + (double)P->hal_strength * BLEED[e] * (double)j->hal[q];
            double le = log10(E > 1e-6 ? E : 1e-6);
            D[e] = (double)P->dmax[e] / (1.0 + exp(-(double)P->k[e] * (le - (double)P->x0[e])));
            if (P->grain_on) D[e] += (double)P->grain_sigma * (double)j->noise[e][q] * (double)j->norm[e];
        }
        double x = 0, y = 0, z = 0;
        for (int i = 0; i < NB81; i++) {
            double d = D[0] * b->dye[0][i] + D[1] * b->dye[1][i] + D[2] * b->dye[2][i];
            double t = pow(10.0, -d);
            x += b->trap[i] * b->xb[i] * t;
            y += b->trap[i] * b->yb[i] * t;
            z += b->trap[i] * b->zb[i] * t;
        }
        double xyz[3] = {x, y, z}, o[3];
        matvec3(XYZ2AP1, xyz, o);
        for (int c = 0; c < 3; c++) j->rgb[3 * (size_t)q + c] = (real)(o[c] / j->peak);
    }
}

int OSYM(oracle_film_baseline)(real *rgb, int W, int H, const OBaseline *P, int threads)
{
    if (!rgb || !P || W <= 0 || H <= 0) return ORACLE_ERR_ARG;
    g_threads = threads > 0 ? threads : 1;
    B81 b;
    b81_build(&b);
    size_t n = (size_t)W * H;
    BJob j;
    memset(&j, 0, sizeof j);
    j.b = &b;
    j.P = P;
    j.rgb = rgb;
    j.hal = (real *)malloc(sizeof(real) * n);
    for (int e = 0; e < 3; e++) j.a[e] = (real *)malloc(sizeof(real) * n);
    oracle_parallel_for((long)n, 4096, g_threads, base_expose_job, &j);
    int R = P->hal_radius;
    real *taps = (real *)malloc(sizeof(real) * (2 * R + 1));
    fixed_radius_taps((real)P->hal_sigma, R, taps);
    blur_taps(j.hal, W, H, taps, R);
    free(taps);
    if (P->grain_on)
        for (int e = 0; e < 3; e++) {
            j.noise[e] = (real *)malloc(sizeof(real) * n);
            j.norm[e] = grain_field(j.noise[e], W, H, P->seed, e, (real)P->grain_blur);
        }
    double peak = b.white[0] > b.white[1] ? b.white[0] : b.white[1];
    if (b.white[2] > peak) peak = b.white[2];
    j.peak = peak;
    oracle_parallel_for((long)n, 1024, g_threads, base_scan_job, &j);
    for (int e = 0; e < 3; e++) { free(j.a[e]); free(j.noise[e]); }
    free(j.hal);
    g_threads = 1;
    return ORACLE_OK;
}

/* DevelopableFractionLut::build + sample for an explicit crystal
 * distribution and calibration k (capture.rs:37-88), for the reference's
 * own LUT tests (capture.rs:113-186). */
double OSYM(oracle_lut_build_sample)(double mu_ln, double sigma_ln, double k, double phi)
{
    OLayer L;
    memset(&L, 0, sizeof L);
    L.mu_ln = mu_ln;
    L.sigma_ln = sigma_ln;
    L.capture_k = k;
    lut_build(&L);
    return lut_sample(&L, phi);
}

#ifndef ORACLE_F32
/* ======================================================================= */
/* Part 3: FP64 oracle of the library's differentiable colour + film model  */
/* (the reference has no gradients).  Same model as the GPU adjoint:        */
/*   y = 2^ev (wb*x); a = C y; w = max(0, Minv a); e = A^T w;               */
/*   h = max(0, a_R - thr); B = G_sigma * h (fixed radius, mirror);         */
/*   E = e + s bleed B; D = dmax / (1 + exp(-k (log10 max(E,1e-6) - x0)));  */
/*   T = 10^(-sum D dye); out = AP1(sum trap cmf T) / peak.                 */
/* The backward is analytic; the transposed blur is an explicit scatter.    */

typedef struct {
    float wb[3], matrix[9], ev;
    float dmax[3], k[3], x0[3];
    float hal_strength, hal_sigma;
} OGrad;

static void g_taps(double sigma, int R, double *t, double *dt)
{
    double sum = 0, m2 = 0;
    for (int i = 0; i <= 2 * R; i++) {
        double x = i - R;
        t[i] = exp(-x * x / (2 * sigma * sigma));
        sum += t[i];
    }
    for (int i = 0; i <= 2 * R; i++) {
        t[i] /= sum;
        double x = i - R;
        m2 += t[i] * x * x;
    }
    for (int i = 0; i <= 2 * R; i++) {
        double x = i - R;
        dt[i] = t[i] * (x * x - m2) / (sigma * sigma * sigma);
    }
}

/* out = cols(rows(in)) with taps tr (rows) and tc (cols), mirror reflection */
static void conv2(const double *in, double *out, int W, int H, const double *tr, const double *tc, int R)
{
    double *tmp = (double *)malloc(sizeof(double) * (size_t)W * H);
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            double acc = 0;
            for (int k = 0; k <= 2 * R; k++) acc += in[(size_t)y * W + reflect_index((long)x + k - R, W)] * tr[k];
            tmp[(size_t)y * W + x] = acc;
        }
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            double acc = 0;
            for (int k = 0; k <= 2 * R; k++) acc += tmp[(size_t)reflect_index((long)y + k - R, H) * W + x] * tc[k];
            out[(size_t)y * W + x] = acc;
        }
    free(tmp);
}

/* transpose of conv2 (scatter form): out = rows^T(cols^T(in)) */
static void conv2_T(const double *in, double *out, int W, int H, const double *t, int R)
{
    size_t n = (size_t)W * H;
    double *tmp = (double *)calloc(n, sizeof(double));
    memset(out, 0, n * sizeof(double));
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++)
            for (int k = 0; k <= 2 * R; k++)
                tmp[(size_t)reflect_index((long)y + k - R, H) * W + x] += t[k] * in[(size_t)y * W + x];
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++)
            for (int k = 0; k <= 2 * R; k++)
                out[(size_t)y * W + reflect_index((long)x + k - R, W)] += t[k] * tmp[(size_t)y * W + x];
    free(tmp);
}

typedef struct { B81 b; double peak; double ev2; } GCtx;

static void g_color(const OGrad *P, double ev2, const double *x, double y[3], double a[3])
{
    for (int i = 0; i < 3; i++) y[i] = ev2 * ((double)P->wb[i] * x[i]);
    for (int i = 0; i < 3; i++)
        a[i] = (double)P->matrix[3 * i] * y[0] + (double)P->matrix[3 * i + 1] * y[1] + (double)P->matrix[3 * i + 2] * y[2];
}

/* forward for every pixel; optionally returns B (per pixel) */
int oracle_param_forward_f64(const double *x, int W, int H, const OGrad *P, const OBaseline *F, double *out)
{
    size_t n = (size_t)W * H;
    GCtx g;
    b81_build(&g.b);
    double pk = g.b.white[0] > g.b.white[1] ? g.b.white[0] : g.b.white[1];
    if (g.b.white[2] > pk) pk = g.b.white[2];
    double ev2 = exp2((double)P->ev);
    int R = F->hal_radius;
    double *t = malloc(sizeof(double) * (2 * R + 1)), *dt = malloc(sizeof(double) * (2 * R + 1));
    g_taps(P->hal_sigma, R, t, dt);
    double *h = calloc(n + 1, sizeof(double)), *B = calloc(n + 1, sizeof(double));
    for (size_t p = 0; p < n; p++) {
        double y[3], a[3];
        g_color(P, ev2, x + 3 * p, y, a);
        double v = a[0] - (double)F->hal_threshold;
        h[p] = v > 0 ? v : 0;
    }
    conv2(h, B, W, H, t, t, R);
    for (size_t p = 0; p < n; p++) {
        double y[3], a[3], w[3];
        g_color(P, ev2, x + 3 * p, y, a);
        matvec3(g.b.minv, a, w);
        double D[3];
        for (int l = 0; l < 3; l++) {
            double e = 0;
            for (int k = 0; k < 3; k++) {
                double ak = 0;
                for (int i = 0; i < NB81; i++) ak += g.b.trap[i] * g.b.basis[k][i] * g.b.sens[l][i];
                e += (w[k] > 0 ? w[k] : 0) * (ak / g.b.sens_norm[l]);
            }
            double E = e + (double)P->hal_strength * BLEED[l] * B[p];
            double le = log10(E > 1e-6 ? E : 1e-6);
            D[l] = (double)P->dmax[l] / (1.0 + exp(-(double)P->k[l] * (le - (double)P->x0[l])));
        }
        double X = 0, Y = 0, Z = 0;
        for (int i = 0; i < NB81; i++) {
            double d = D[0] * g.b.dye[0][i] + D[1] * g.b.dye[1][i] + D[2] * g.b.dye[2][i];
            double tt = pow(10.0, -d);
            X += g.b.trap[i] * g.b.xb[i] * tt;
            Y += g.b.trap[i] * g.b.yb[i] * tt;
            Z += g.b.trap[i] * g.b.zb[i] * tt;
        }
        double xyz[3] = {X, Y, Z}, o[3];
        matvec3(XYZ2AP1, xyz, o);
        for (int c = 0; c < 3; c++) out[3 * p + c] = o[c] / pk;
    }
    free(t); free(dt); free(h); free(B);
    return ORACLE_OK;
}

/* loss = scale * sum (out - target)^2; grad[0..23] += dloss/dparam, grad[24] += loss */
int oracle_param_grad_f64(const double *x, const double *target, int W, int H, const OGrad *P, const OBaseline *F,
                          double scale, double *grad)
{
    size_t n = (size_t)W * H;
    GCtx g;
    b81_build(&g.b);
    double pk = g.b.white[0] > g.b.white[1] ? g.b.white[0] : g.b.white[1];
    if (g.b.white[2] > pk) pk = g.b.white[2];
    double A[3][3];
    for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++) {
            double ak = 0;
            for (int i = 0; i < NB81; i++) ak += g.b.trap[i] * g.b.basis[k][i] * g.b.sens[l][i];
            A[k][l] = ak / g.b.sens_norm[l];
        }
    double ev2 = exp2((double)P->ev);
    int R = F->hal_radius;
    double *t = malloc(sizeof(double) * (2 * R + 1)), *dt = malloc(sizeof(double) * (2 * R + 1));
    g_taps(P->hal_sigma, R, t, dt);
    double *h = calloc(n + 1, sizeof(double)), *B = calloc(n + 1, sizeof(double)), *Bs = calloc(n + 1, sizeof(double));
    double *Bs2 = malloc(sizeof(double) * n), *gB = malloc(sizeof(double) * n), *gh = malloc(sizeof(double) * n);
    double *ga = malloc(sizeof(double) * 3 * n);
    for (size_t p = 0; p < n; p++) {
        double y[3], a[3];
        g_color(P, ev2, x + 3 * p, y, a);
        double v = a[0] - (double)F->hal_threshold;
        h[p] = v > 0 ? v : 0;
    }
    conv2(h, B, W, H, t, t, R);
    conv2(h, Bs, W, H, dt, t, R);
    conv2(h, Bs2, W, H, t, dt, R);
    for (size_t p = 0; p < n; p++) Bs[p] += Bs2[p];
    double gdmax[3] = {0}, gk[3] = {0}, gx0[3] = {0}, gs = 0, gsig = 0, loss = 0;
    const double LN10 = 2.302585092994045684;
    for (size_t p = 0; p < n; p++) {
        double y[3], a[3], w[3];
        g_color(P, ev2, x + 3 * p, y, a);
        matvec3(g.b.minv, a, w);
        double E[3], le[3], sg[3], D[3];
        for (int l = 0; l < 3; l++) {
            double e = 0;
            for (int k = 0; k < 3; k++) e += (w[k] > 0 ? w[k] : 0) * A[k][l];
            E[l] = e + (double)P->hal_strength * BLEED[l] * B[p];
            le[l] = log10(E[l] > 1e-6 ? E[l] : 1e-6);
            sg[l] = 1.0 / (1.0 + exp(-(double)P->k[l] * (le[l] - (double)P->x0[l])));
            D[l] = (double)P->dmax[l] * sg[l];
        }
        double T[NB81], X = 0, Y = 0, Z = 0;
        for (int i = 0; i < NB81; i++) {
            double d = D[0] * g.b.dye[0][i] + D[1] * g.b.dye[1][i] + D[2] * g.b.dye[2][i];
            T[i] = pow(10.0, -d);
            X += g.b.trap[i] * g.b.xb[i] * T[i];
            Y += g.b.trap[i] * g.b.yb[i] * T[i];
            Z += g.b.trap[i] * g.b.zb[i] * T[i];
        }
        double xyz[3] = {X, Y, Z}, o[3];
        matvec3(XYZ2AP1, xyz, o);
        double go[3];
        for (int c = 0; c < 3; c++) {
            double r = o[c] / pk - target[3 * p + c];
            loss += scale * r * r;
            go[c] = 2 * scale * r / pk;  /* through the /peak */
        }
        /* o = XYZ2AP1 * xyz -> g_xyz = XYZ2AP1^T go */
        double gx = 0, gy = 0, gz = 0;
        for (int c = 0; c < 3; c++) {
            gx += XYZ2AP1[c][0] * go[c];
            gy += XYZ2AP1[c][1] * go[c];
            gz += XYZ2AP1[c][2] * go[c];
        }
        double gD[3] = {0, 0, 0};
        for (int i = 0; i < NB81; i++) {
            double gT = g.b.trap[i] * (g.b.xb[i] * gx + g.b.yb[i] * gy + g.b.zb[i] * gz);
            double gd = -LN10 * T[i] * gT;
            for (int l = 0; l < 3; l++) gD[l] += g.b.dye[l][i] * gd;
        }
        double gE[3];
        for (int l = 0; l < 3; l++) {
            double ds = sg[l] * (1 - sg[l]);
            gdmax[l] += gD[l] * sg[l];
            gk[l] += gD[l] * (double)P->dmax[l] * ds * (le[l] - (double)P->x0[l]);
            gx0[l] += -gD[l] * (double)P->dmax[l] * ds * (double)P->k[l];
            gE[l] = E[l] > 1e-6 ? gD[l] * (double)P->dmax[l] * ds * (double)P->k[l] / (E[l] * LN10) : 0.0;
        }
        double sb = BLEED[0] * gE[0] + BLEED[1] * gE[1] + BLEED[2] * gE[2];
        gs += sb * B[p];
        gB[p] = (double)P->hal_strength * sb;
        gsig += gB[p] * Bs[p];
        double gw[3];
        for (int k = 0; k < 3; k++) gw[k] = w[k] > 0 ? A[k][0] * gE[0] + A[k][1] * gE[1] + A[k][2] * gE[2] : 0;
        for (int j = 0; j < 3; j++)
            ga[3 * p + j] = g.b.minv[0][j] * gw[0] + g.b.minv[1][j] * gw[1] + g.b.minv[2][j] * gw[2];
    }
    conv2_T(gB, gh, W, H, t, R);
    for (size_t p = 0; p < n; p++) {
        double y[3], a[3];
        g_color(P, ev2, x + 3 * p, y, a);
        double gg[3] = {ga[3 * p], ga[3 * p + 1], ga[3 * p + 2]};
        if (a[0] - (double)F->hal_threshold > 0) gg[0] += gh[p];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) grad[3 + 3 * i + j] += gg[i] * y[j];
        double gy3[3];
        for (int j = 0; j < 3; j++)
            gy3[j] = (double)P->matrix[j] * gg[0] + (double)P->matrix[3 + j] * gg[1] + (double)P->matrix[6 + j] * gg[2];
        grad[12] += 0.69314718055994530942 * (gy3[0] * y[0] + gy3[1] * y[1] + gy3[2] * y[2]);
        for (int j = 0; j < 3; j++) grad[j] += gy3[j] * ev2 * x[3 * p + j];
    }
    for (int l = 0; l < 3; l++) {
        grad[13 + l] += gdmax[l];
        grad[16 + l] += gk[l];
        grad[19 + l] += gx0[l];
    }
    grad[22] += gs;
    grad[23] += gsig;
    grad[24] += loss;
    free(t); free(dt); free(h); free(B); free(Bs); free(Bs2); free(gB); free(gh); free(ga);
    return ORACLE_OK;
}
#endif
