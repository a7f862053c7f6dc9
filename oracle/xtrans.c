/*
 * xtrans.c -- CPU oracle for the 3-pass directional X-Trans demosaic
 * (imops_demosaic_markesteijn3) of the CUDA library.
 *
 * TEST INFRASTRUCTURE (see oracle_common.h).  The reference has no such
 * algorithm: its "markesteijn" is the 3x3 same-colour mean
 * (pichromatic/src/demosaic.rs:108-186, restated in demosaic_simple.c).
 * This file is the specification of the library's own method, after Frank
 * Markesteijn's X-Trans demosaic as published in dcraw 9.x: directional
 * green along four lines, bounded by the surrounding greens; red and blue
 * from colour differences; refinement passes; and a vote between the
 * directions by perceptual homogeneity.  PARITY UNPINNED against any
 * external implementation; the GPU kernels are checked bit for bit against
 * this restatement, and its quality by property tests (flat fields, the
 * CFA samples kept, lower error than the 3x3 mean on synthetic scenes).
 *
 * Steps (p = (row, col); s_d the unit step of direction d: H (0,1), V (1,0),
 * D1 (1,1), D2 (1,-1); reads outside the image clamp to the edge; colours
 * from the CFA at the clamped position):
 *  1. green, pass 1: at a green site G_d = m.  Elsewhere the nearest green
 *     on each side along d (distance 1 or 2 on X-Trans), a at k+ and b at
 *     k-, interpolated linearly: (a k- + b k+) / (k+ + k-) (one side only:
 *     its value; none: the mean of the orthogonal greens, else m), clamped
 *     to [min, max] of the orthogonal green neighbours.
 *  2. red / blue: at a site of that colour C_d = m; elsewhere
 *     G_d + the mean of (m - G_d) over the 3x3 sites of that colour
 *     (rows then columns), or G_d if there are none.
 *  Every division by a count n here and in the vote is a product with
 *  XT_RECIP[n], 1/n rounded to the working precision: one multiply on the
 *  GPU instead of an IEEE division, the same value on both sides.
 *  3. green refinement at R/B sites (colour c): the colour difference
 *     K = ((C_d - G_d)(p + s_d) + (C_d - G_d)(p - s_d)) * 0.5 of plane c,
 *     G_d = clamp(m - K, min, max) as in step 1.
 *     Passes: 1, 2, 3, 2, 3, 2 (three green estimates, each followed by
 *     red / blue).
 *  4. perceptual difference: CIELab of each direction's RGB, taking camera
 *     RGB as linear sRGB (CSS Color 4 matrix with the D65 white folded into
 *     its X and Z rows); the cube root as t r^2 with r = t^(-1/3) by Newton's
 *     method for the reciprocal cube root, r <- r (4 - t r^3) / 3, from a
 *     first guess made from the bits (own code, no division, the same IEEE
 *     operations on CPU and GPU).
 *     D_d = |Lab_d(p) - Lab_d(p + s_d)|^2 + |Lab_d(p) - Lab_d(p - s_d)|^2.
 *  5. vote: T(q) = 8 min_d D_d(q); H_d(p) = #{q in 3x3(p): D_d(q) <= T(q)};
 *     the directions with H_d >= Hmax - Hmax / 8 (integer division) are
 *     averaged (sum in direction order, divided by their count); the
 *     site's own colour keeps its sample.
 *  6. pixels within 10 of an edge (the method's dependency radius is 9)
 *     take the 3x3 mean of the reference instead.
 */
#include "oracle_common.h"

#include <stdlib.h>
#include <string.h>

#define XT_BAND 10

static const int XT_DY[4] = {0, 1, 1, 1};
static const int XT_DX[4] = {1, 0, 1, -1};

/* 1/n for the counts of the method (at most 8 sites of a colour in a 3x3
 * window), each rounded once to the working precision; index 0 is unused */
static const real XT_RECIP[9] = {K(1.0),         K(1.0),         K(1.0) / K(2.0), K(1.0) / K(3.0), K(1.0) / K(4.0),
                                 K(1.0) / K(5.0), K(1.0) / K(6.0), K(1.0) / K(7.0), K(1.0) / K(8.0)};

typedef struct {
    const real *m;
    int W, H;
    const OracleCfa *cfa;
} XtImg;

static inline int xt_ci(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }
static inline size_t xt_at(const XtImg *im, int r, int c) { return (size_t)xt_ci(r, im->H) * im->W + xt_ci(c, im->W); }
static inline int xt_col(const XtImg *im, int r, int c) { return ocfa_color(im->cfa, xt_ci(r, im->H), xt_ci(c, im->W)); }

/* min / max / sum / count of the orthogonal green neighbours */
static void xt_gbounds(const XtImg *im, int r, int c, real *lo, real *hi, real *sum, int *n)
{
    static const int oy[4] = {0, 0, 1, -1}, ox[4] = {1, -1, 0, 0};
    *n = 0;
    *sum = K(0.0);
    *lo = K(0.0);
    *hi = K(0.0);
    for (int t = 0; t < 4; t++) {
        if (xt_col(im, r + oy[t], c + ox[t]) != 1) continue;
        real v = im->m[xt_at(im, r + oy[t], c + ox[t])];
        if (*n == 0) {
            *lo = v;
            *hi = v;
        } else {
            *lo = v < *lo ? v : *lo;
            *hi = v > *hi ? v : *hi;
        }
        *sum = *sum + v;
        (*n)++;
    }
}

static inline real xt_clamp(real g, real lo, real hi, int n)
{
    if (n == 0) return g;
    g = g < lo ? lo : g;
    return g > hi ? hi : g;
}

/* step 1 */
static real xt_green1(const XtImg *im, int r, int c, int d)
{
    size_t i = xt_at(im, r, c);
    if (xt_col(im, r, c) == 1) return im->m[i];
    real lo, hi, sum;
    int n;
    xt_gbounds(im, r, c, &lo, &hi, &sum, &n);
    int kp = 0, km = 0;
    real a = K(0.0), b = K(0.0);
    for (int k = 1; k <= 2 && !kp; k++)
        if (xt_col(im, r + k * XT_DY[d], c + k * XT_DX[d]) == 1) {
            kp = k;
            a = im->m[xt_at(im, r + k * XT_DY[d], c + k * XT_DX[d])];
        }
    for (int k = 1; k <= 2 && !km; k++)
        if (xt_col(im, r - k * XT_DY[d], c - k * XT_DX[d]) == 1) {
            km = k;
            b = im->m[xt_at(im, r - k * XT_DY[d], c - k * XT_DX[d])];
        }
    real g;
    if (kp && km) g = (a * (real)km + b * (real)kp) * XT_RECIP[kp + km];
    else if (kp) g = a;
    else if (km) g = b;
    else g = n ? sum * XT_RECIP[n] : im->m[i];
    return xt_clamp(g, lo, hi, n);
}

/* step 2: colour ch (0 red, 2 blue) of direction plane G */
static real xt_rb(const XtImg *im, const real *G, int r, int c, int ch)
{
    size_t i = xt_at(im, r, c);
    if (xt_col(im, r, c) == ch) return im->m[i];
    real s = K(0.0);
    int n = 0;
    for (int a = -1; a <= 1; a++)
        for (int b = -1; b <= 1; b++) {
            if (xt_col(im, r + a, c + b) != ch) continue;
            size_t j = xt_at(im, r + a, c + b);
            s = s + (im->m[j] - G[j]);
            n++;
        }
    return n ? G[i] + s * XT_RECIP[n] : G[i];
}

/* step 3 */
static real xt_refine(const XtImg *im, const real *G, const real *Rp, const real *Bp, int r, int c, int d)
{
    size_t i = xt_at(im, r, c);
    int ch = xt_col(im, r, c);
    if (ch == 1) return im->m[i];
    const real *C = ch == 0 ? Rp : Bp;
    size_t jp = xt_at(im, r + XT_DY[d], c + XT_DX[d]), jm = xt_at(im, r - XT_DY[d], c - XT_DX[d]);
    real k = ((C[jp] - G[jp]) + (C[jm] - G[jm])) * K(0.5);
    real lo, hi, sum;
    int n;
    xt_gbounds(im, r, c, &lo, &hi, &sum, &n);
    return xt_clamp(im->m[i] - k, lo, hi, n);
}

/* step 4: cube root of t > 0 as t * r * r, r = t^(-1/3) by Newton's method
 * for the reciprocal cube root, r <- r (4 - t r^3) / 3, which needs no
 * division.  First guess 0x54AAAAAA - bits(t) / 3: a float's bit pattern is
 * nearly a scaled, offset log2, so bits(t^p) ~ p bits(t) + (1 - p) bits(1.0f)
 * (Blinn, "Floating-point tricks", IEEE CG&A 17(4), 1997), and for p = -1/3
 * the offset (4/3) 0x3F800000 = 0x54AAAAAA.  The guess is 0 .. 8.17% high
 * for every normal t (its error repeats every three binades), inside the
 * iteration's convergence bound (t r^3 < 4). */
static real xt_cbrt(real t)
{
    float tf = (float)t;
    uint32_t u;
    memcpy(&u, &tf, 4);
    u = 0x54AAAAAAu - u / 3u;
    float rf;
    memcpy(&rf, &u, 4);
    real r = (real)rf;
    /* four steps: the cube root to 4.6e-7 relative in f32 */
    for (int it = 0; it < 4; it++) {
        real r2 = r * r, r3 = r2 * r, q = t * r3;
        r = (r * (K(4.0) - q)) * (K(1.0) / K(3.0));
    }
#ifndef ORACLE_F32
    for (int it = 0; it < 2; it++) {
        double r2 = r * r, r3 = r2 * r, q = t * r3;
        r = (r * (4.0 - q)) * (1.0 / 3.0);
    }
#endif
    return (t * r) * r;
}

/* CIELab's f: (24389/27 t + 16) / 116 as one multiply-add of folded
 * constants below the threshold */
static real xt_f(real t)
{
    if (t > K(216.0) / K(24389.0)) return xt_cbrt(t);
    return K(7.787037037037037) * t + K(0.13793103448275862);
}

/* The cube root of step 4 over an array (tests check it against the exact
 * cube root). */
void OSYM(oracle_xt_cbrt)(const real *t, long n, real *out)
{
    for (long i = 0; i < n; i++) out[i] = xt_cbrt(t[i]);
}

static void xt_lab(real r, real g, real b, real lab[3])
{
    /* linear sRGB -> XYZ (CSS Color 4) over the D65 white: the X row divided
     * by 0.9504559270516716 and the Z row by 1.0890577507598784 (in double) */
    real x = K(0.4338873455660398) * r + K(0.3762240091374988) * g + K(0.18988864529646143) * b;
    real y = K(0.21263900587151027) * r + K(0.715168678767756) * g + K(0.07219231536073371) * b;
    real z = K(0.017750040070973232) * r + K(0.10944762085523847) * g + K(0.8728023390737883) * b;
    real fx = xt_f(x), fy = xt_f(y), fz = xt_f(z);
    lab[0] = K(116.0) * fy - K(16.0);
    lab[1] = K(500.0) * (fx - fy);
    lab[2] = K(200.0) * (fy - fz);
}

/* the reference's 3x3 same-colour mean at one pixel (demosaic.rs:108-186) */
static void xt_mean3(const XtImg *im, int r, int c, real out[3])
{
    int y0 = r > 0 ? r - 1 : 0, y1 = r + 1 < im->H - 1 ? r + 1 : im->H - 1;
    int x0 = c > 0 ? c - 1 : 0, x1 = c + 1 < im->W - 1 ? c + 1 : im->W - 1;
    int centre = ocfa_color(im->cfa, r, c);
    for (int ch = 0; ch < 3; ch++) {
        if (ch == centre) {
            out[ch] = im->m[(size_t)r * im->W + c];
            continue;
        }
        real s = K(0.0), n = K(0.0);
        for (int y = y0; y <= y1; y++)
            for (int x = x0; x <= x1; x++) {
                if (y == r && x == c) continue;
                if (ocfa_color(im->cfa, y, x) == ch) {
                    s += im->m[(size_t)y * im->W + x];
                    n += K(1.0);
                }
            }
        out[ch] = n > K(0.0) ? s / n : K(0.0);
    }
}

int OSYM(oracle_markesteijn3)(const real *m, int W, int H, const OracleCfa *cfa, real *out)
{
    if (!m || !out || !cfa || W <= 0 || H <= 0) return ORACLE_ERR_ARG;
    if (cfa->pw != 6 || cfa->ph != 6) return ORACLE_ERR_CFA;
    XtImg im = {m, W, H, cfa};
    size_t n = (size_t)W * H;
    /* planes: G[4], G2[4], R[4], B[4], L[4][3], D[4] */
    real *buf = (real *)malloc(sizeof(real) * n * 32);
    if (!buf) return ORACLE_ERR_ARG;
    real *G = buf, *G2 = buf + 4 * n, *R = buf + 8 * n, *B = buf + 12 * n, *L = buf + 16 * n, *D = buf + 28 * n;
    for (int d = 0; d < 4; d++)
        for (int r = 0; r < H; r++)
            for (int c = 0; c < W; c++) G[d * n + (size_t)r * W + c] = xt_green1(&im, r, c, d);
    for (int pass = 0; pass < 3; pass++) {
        if (pass > 0) {
            for (int d = 0; d < 4; d++)
                for (int r = 0; r < H; r++)
                    for (int c = 0; c < W; c++)
                        G2[d * n + (size_t)r * W + c] = xt_refine(&im, G + d * n, R + d * n, B + d * n, r, c, d);
            real *t = G;
            G = G2;
            G2 = t;
        }
        for (int d = 0; d < 4; d++)
            for (int r = 0; r < H; r++)
                for (int c = 0; c < W; c++) {
                    R[d * n + (size_t)r * W + c] = xt_rb(&im, G + d * n, r, c, 0);
                    B[d * n + (size_t)r * W + c] = xt_rb(&im, G + d * n, r, c, 2);
                }
    }
    for (int d = 0; d < 4; d++)
        for (size_t i = 0; i < n; i++) {
            real lab[3];
            xt_lab(R[d * n + i], G[d * n + i], B[d * n + i], lab);
            for (int k = 0; k < 3; k++) L[(d * 3 + k) * n + i] = lab[k];
        }
    for (int d = 0; d < 4; d++)
        for (int r = 0; r < H; r++)
            for (int c = 0; c < W; c++) {
                size_t i = (size_t)r * W + c, jp = xt_at(&im, r + XT_DY[d], c + XT_DX[d]),
                       jm = xt_at(&im, r - XT_DY[d], c - XT_DX[d]);
                real sp = K(0.0), sm = K(0.0);
                for (int k = 0; k < 3; k++) {
                    const real *Lk = L + (d * 3 + k) * n;
                    real ep = Lk[i] - Lk[jp], em = Lk[i] - Lk[jm];
                    sp = sp + ep * ep;
                    sm = sm + em * em;
                }
                D[d * n + i] = sp + sm;
            }
    for (int r = 0; r < H; r++)
        for (int c = 0; c < W; c++) {
            size_t i = (size_t)r * W + c;
            real *o = out + 3 * i;
            if (r < XT_BAND || r >= H - XT_BAND || c < XT_BAND || c >= W - XT_BAND) {
                xt_mean3(&im, r, c, o);
                continue;
            }
            int hm[4] = {0, 0, 0, 0};
            for (int a = -1; a <= 1; a++)
                for (int b = -1; b <= 1; b++) {
                    size_t j = (size_t)(r + a) * W + (c + b);
                    real mn = D[j];
                    for (int d = 1; d < 4; d++) mn = D[d * n + j] < mn ? D[d * n + j] : mn;
                    real t = K(8.0) * mn;
                    for (int d = 0; d < 4; d++) hm[d] += D[d * n + j] <= t;
                }
            int hx = hm[0];
            for (int d = 1; d < 4; d++) hx = hm[d] > hx ? hm[d] : hx;
            int thr = hx - hx / 8, cnt = 0;  /* a count, not a division of values */
            real s0 = K(0.0), s1 = K(0.0), s2 = K(0.0);
            for (int d = 0; d < 4; d++) {
                if (hm[d] < thr) continue;
                s0 = s0 + R[d * n + i];
                s1 = s1 + G[d * n + i];
                s2 = s2 + B[d * n + i];
                cnt++;
            }
            o[0] = s0 * XT_RECIP[cnt];
            o[1] = s1 * XT_RECIP[cnt];
            o[2] = s2 * XT_RECIP[cnt];
            o[ocfa_color(cfa, r, c)] = m[i];  /* the site's own colour is its sample */
        }
    free(buf);
    return ORACLE_OK;
}
