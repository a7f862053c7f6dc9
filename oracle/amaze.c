/*
 * amaze.c -- CPU oracle for the reference's AMaZE demosaic.
 *
 * TEST INFRASTRUCTURE (see oracle_common.h).  Restates
 * demosaic_algorithms::Amaze::demosaic, pichromatic/src/demosaic.rs:358-1379.
 *
 * The reference works on 128x128 tiles stepped by 96 from (-16,-16); every
 * tile starts from zeroed scratch arrays, fills a mirrored 16-pixel border
 * at the image edge, and several stages update arrays in place while they
 * scan (later sites read values already rewritten by earlier ones).  Those
 * details decide the output bits, so this file keeps the reference's tile
 * geometry, loop bounds, in-place update order and f32 operation order.
 * Each stage is one function whose comment cites the reference lines.
 *
 * Image sizes for which the reference's border fill indexes past its
 * 128x128 tile buffer (a panic in Rust) are reported as ORACLE_ERR_SIZE.
 */
#include "oracle_common.h"

#include <stdlib.h>
#include <string.h>

#define TS 128
#define TSH 64
#define NF (TS * TS)
#define NH (TS * TSH)
/* stencil offsets in the flat 128-wide tile buffer (demosaic.rs:414-422) */
#define V1 128
#define V2 256
#define V3 384
#define P1 127
#define P2 254
#define P3 381
#define M1 129
#define M2 258
#define M3 387

typedef struct {
    /* full-resolution tile arrays */
    real mos[NF];       /* the tile's mosaic values (cfa_buf) */
    real green[NF];     /* green estimate, starts as a copy of mos (rgbgreen) */
    real gradsq[NF];    /* delh^2 + delv^2 (delhvsqsum) */
    real wv[NF];        /* vertical gradient weight (dirwts0) */
    real wh[NF];        /* horizontal gradient weight (dirwts1) */
    real vcd[NF], hcd[NF], vcdalt[NF], hcdalt[NF];
    real cddiffsq[NF], dgintv[NF], dginth[NF];
    /* half arrays: one slot per pair of columns, indexed by flat index >> 1 */
    real hvwt[NH], dgrb0[NH], dgrb1[NH], delp[NH], delm[NH], rbint[NH];
    real dgrb2h[NH], dgrb2v[NH], dgrbsq1m[NH], dgrbsq1p[NH], pmwt[NH];
    real rbm[NH], rbp[NH], nyqutest[NH];
    uint8_t nyq[NH], nyq2[NH];
} Tile;

typedef struct {
    const real *in;
    real *out;          /* interleaved RGB */
    int W, H;
    const OracleCfa *cfa;
    real clip;
    int top, left;
    int rr1, cc1;       /* tile extent */
} Ctx;

static inline real sqr(real x) { return x * x; }
/* lim/ulim/clampnan: demosaic.rs:453-465 */
static inline real lim(real x, real lo, real hi) { return RMAX(lo, RMIN(x, hi)); }
static inline real ulim(real x, real y, real z) { return y < z ? lim(x, y, z) : lim(x, z, y); }
static inline real clampnan(real x, real lo, real hi)
{
    if (isnan(x)) return (lo + hi) * K(0.5);
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

static inline real get_in(const Ctx *c, int r, int q)
{
    if (r < 0) r = 0;
    if (r > c->H - 1) r = c->H - 1;
    if (q < 0) q = 0;
    if (q > c->W - 1) q = c->W - 1;
    return c->in[(size_t)r * c->W + q];
}

static inline int fc(const Ctx *c, int r, int q) { return ocfa_color(c->cfa, r, q); }

/* Store one border/interior value into the two tile arrays the fill writes;
 * an index past the buffer is where the reference would panic. */
static inline int put(Tile *t, long idx, real v)
{
    if (idx < 0 || idx >= NF) return -1;
    t->mos[idx] = v;
    t->green[idx] = v;
    return 0;
}

/* Tile fill with mirrored borders: demosaic.rs:499-610. */
static int fill_tile(Tile *t, Ctx *c)
{
    const int top = c->top, left = c->left, W = c->W, H = c->H;
    const int bottom = (top + 128 < H + 16) ? top + 128 : H + 16;
    const int right = (left + 128 < W + 16) ? left + 128 : W + 16;
    const int rr1 = bottom - top, cc1 = right - left;
    const int rrmin = top < 0 ? 16 : 0, ccmin = left < 0 ? 16 : 0;
    const int rrmax = bottom > H ? H - top : rr1;
    const int ccmax = right > W ? W - left : cc1;
    int bad = 0;
    c->rr1 = rr1;
    c->cc1 = cc1;

    if (rrmin > 0)
        for (int rr = 0; rr < 16; rr++)
            for (int cc = ccmin; cc < ccmax; cc++)
                bad |= put(t, (long)rr * TS + cc, get_in(c, 32 - rr + top, cc + left));
    for (int rr = rrmin; rr < rrmax; rr++)
        for (int cc = ccmin; cc < ccmax; cc++)
            bad |= put(t, (long)rr * TS + cc, get_in(c, rr + top, cc + left));
    if (rrmax < rr1)
        for (int rr = 0; rr < 16; rr++)
            for (int cc = ccmin; cc < ccmax; cc++)
                bad |= put(t, (long)(rrmax + rr) * TS + cc, get_in(c, H - rr - 2, left + cc));
    if (ccmin > 0)
        for (int rr = rrmin; rr < rrmax; rr++)
            for (int cc = 0; cc < 16; cc++)
                bad |= put(t, (long)rr * TS + cc, get_in(c, rr + top, 32 - cc + left));
    if (ccmax < cc1)
        for (int rr = rrmin; rr < rrmax; rr++)
            for (int cc = 0; cc < 16; cc++)
                bad |= put(t, (long)rr * TS + ccmax + cc, get_in(c, top + rr, W - cc - 2));
    if (rrmin > 0 && ccmin > 0)
        for (int rr = 0; rr < 16; rr++)
            for (int cc = 0; cc < 16; cc++)
                bad |= put(t, (long)rr * TS + cc, get_in(c, 32 - rr, 32 - cc));
    if (rrmax < rr1 && ccmax < cc1)
        for (int rr = 0; rr < 16; rr++)
            for (int cc = 0; cc < 16; cc++)
                bad |= put(t, (long)(rrmax + rr) * TS + ccmax + cc, get_in(c, H - rr - 2, W - cc - 2));
    if (rrmin > 0 && ccmax < cc1)
        for (int rr = 0; rr < 16; rr++)
            for (int cc = 0; cc < 16; cc++)
                bad |= put(t, (long)rr * TS + ccmax + cc, get_in(c, 32 - rr, W - cc - 2));
    if (rrmax < rr1 && ccmin > 0)
        for (int rr = 0; rr < 16; rr++)
            for (int cc = 0; cc < 16; cc++)
                bad |= put(t, (long)(rrmax + rr) * TS + cc, get_in(c, H - rr - 2, 32 - cc));
    return bad ? -1 : 0;
}

/* Horizontal/vertical gradients: demosaic.rs:612-622. */
static void st_gradients(Tile *t, const Ctx *c)
{
    const real eps = K(1e-5);
    for (int rr = 2; rr < c->rr1 - 2; rr++)
        for (int cc = 2; cc < c->cc1 - 2; cc++) {
            int i = rr * TS + cc;
            const real *m = t->mos;
            real dh = RABS(m[i + 1] - m[i - 1]);
            real dv = RABS(m[i + V1] - m[i - V1]);
            t->wv[i] = eps + RABS(m[i + V2] - m[i]) + RABS(m[i] - m[i - V2]) + dv;
            t->wh[i] = eps + RABS(m[i + 2] - m[i]) + RABS(m[i] - m[i - 2]) + dh;
            t->gradsq[i] = sqr(dh) + sqr(dv);
        }
}

/* Colour-difference interpolation (Hamilton-Adams + adaptive ratios):
 * demosaic.rs:624-698. */
static void st_colour_diff(Tile *t, const Ctx *c)
{
    const real eps = K(1e-5), arth = K(0.75);
    const real clip8 = c->clip * K(0.8);
    const real *m = t->mos, *wv = t->wv, *wh = t->wh;
    for (int rr = 4; rr < c->rr1 - 4; rr++) {
        int g_site = (fc(c, c->top + rr, c->left + 4) & 1) != 0;
        for (int cc = 4; cc < c->cc1 - 4; cc++) {
            int i = rr * TS + cc;
            real cru = m[i - V1] * (wv[i - V2] + wv[i]) /
                       RMAX(wv[i - V2] * (eps + m[i]) + wv[i] * (eps + m[i - V2]), K(1e-10));
            real crd = m[i + V1] * (wv[i + V2] + wv[i]) /
                       RMAX(wv[i + V2] * (eps + m[i]) + wv[i] * (eps + m[i + V2]), K(1e-10));
            real crl = m[i - 1] * (wh[i - 2] + wh[i]) /
                       RMAX(wh[i - 2] * (eps + m[i]) + wh[i] * (eps + m[i - 2]), K(1e-10));
            real crr = m[i + 1] * (wh[i + 2] + wh[i]) /
                       RMAX(wh[i + 2] * (eps + m[i]) + wh[i] * (eps + m[i + 2]), K(1e-10));
            real guha = m[i - V1] + (m[i] - m[i - V2]) * K(0.5);
            real gdha = m[i + V1] + (m[i] - m[i + V2]) * K(0.5);
            real glha = m[i - 1] + (m[i] - m[i - 2]) * K(0.5);
            real grha = m[i + 1] + (m[i] - m[i + 2]) * K(0.5);
            real guar = RABS(K(1.0) - cru) < arth ? m[i] * cru : guha;
            real gdar = RABS(K(1.0) - crd) < arth ? m[i] * crd : gdha;
            real glar = RABS(K(1.0) - crl) < arth ? m[i] * crl : glha;
            real grar = RABS(K(1.0) - crr) < arth ? m[i] * crr : grha;
            real hwt = wh[i - 1] / RMAX(wh[i - 1] + wh[i + 1], K(1e-10));
            real vwt = wv[i - V1] / RMAX(wv[i + V1] + wv[i - V1], K(1e-10));
            real gintvha = vwt * gdha + (K(1.0) - vwt) * guha;
            real ginthha = hwt * grha + (K(1.0) - hwt) * glha;
            real vcd_v, hcd_v, vcdalt_v, hcdalt_v;
            if (g_site) {
                vcd_v = m[i] - (vwt * gdar + (K(1.0) - vwt) * guar);
                hcd_v = m[i] - (hwt * grar + (K(1.0) - hwt) * glar);
                vcdalt_v = m[i] - gintvha;
                hcdalt_v = m[i] - ginthha;
            } else {
                vcd_v = (vwt * gdar + (K(1.0) - vwt) * guar) - m[i];
                hcd_v = (hwt * grar + (K(1.0) - hwt) * glar) - m[i];
                vcdalt_v = gintvha - m[i];
                hcdalt_v = ginthha - m[i];
            }
            g_site = !g_site;
            real gu = guar, gd = gdar, gl = glar, gr = grar;
            if (m[i] > clip8 || gintvha > clip8 || ginthha > clip8) {
                vcd_v = vcdalt_v;
                hcd_v = hcdalt_v;
                gu = guha; gd = gdha; gl = glha; gr = grha;
            }
            t->vcd[i] = vcd_v;
            t->hcd[i] = hcd_v;
            t->vcdalt[i] = vcdalt_v;
            t->hcdalt[i] = hcdalt_v;
            t->dgintv[i] = RMIN(sqr(guha - gdha), sqr(gu - gd));
            t->dginth[i] = RMIN(sqr(glha - grha), sqr(gl - gr));
        }
    }
}

/* Pick the lower-variance colour difference and bound it by the
 * neighbouring samples; updates hcd/vcd in place in scan order, so each site
 * sees the already-updated value two columns left / two rows up:
 * demosaic.rs:700-786. */
static void st_cd_refine(Tile *t, const Ctx *c)
{
    const real eps = K(1e-5);
    const real *m = t->mos;
    real *hcd = t->hcd, *vcd = t->vcd;
    const real *ha = t->hcdalt, *va = t->vcdalt;
    for (int rr = 4; rr < c->rr1 - 4; rr++)
        for (int cc = 4; cc < c->cc1 - 4; cc++) {
            int i = rr * TS + cc;
            int g_site = (fc(c, c->top + rr, c->left + cc) & 1) != 0;
            real hv = K(3.0) * (sqr(hcd[i - 2]) + sqr(hcd[i]) + sqr(hcd[i + 2])) -
                      sqr(hcd[i - 2] + hcd[i] + hcd[i + 2]);
            real hav = K(3.0) * (sqr(ha[i - 2]) + sqr(ha[i]) + sqr(ha[i + 2])) -
                       sqr(ha[i - 2] + ha[i] + ha[i + 2]);
            real vv = K(3.0) * (sqr(vcd[i - V2]) + sqr(vcd[i]) + sqr(vcd[i + V2])) -
                      sqr(vcd[i - V2] + vcd[i] + vcd[i + V2]);
            real vav = K(3.0) * (sqr(va[i - V2]) + sqr(va[i]) + sqr(va[i + V2])) -
                       sqr(va[i - V2] + va[i] + va[i + V2]);
            if (hav < hv) hcd[i] = ha[i];
            if (vav < vv) vcd[i] = va[i];
            real ginth, gintv;
            if (g_site) {
                ginth = -hcd[i] + m[i];
                gintv = -vcd[i] + m[i];
                if (hcd[i] > K(0.0)) {
                    if (K(3.0) * hcd[i] > (ginth + m[i])) {
                        hcd[i] = -ulim(ginth, m[i - 1], m[i + 1]) + m[i];
                    } else {
                        real w = K(1.0) - K(3.0) * hcd[i] / (eps + ginth + m[i]);
                        hcd[i] = w * hcd[i] + (K(1.0) - w) * (-ulim(ginth, m[i - 1], m[i + 1]) + m[i]);
                    }
                }
                if (vcd[i] > K(0.0)) {
                    if (K(3.0) * vcd[i] > (gintv + m[i])) {
                        vcd[i] = -ulim(gintv, m[i - V1], m[i + V1]) + m[i];
                    } else {
                        real w = K(1.0) - K(3.0) * vcd[i] / (eps + gintv + m[i]);
                        vcd[i] = w * vcd[i] + (K(1.0) - w) * (-ulim(gintv, m[i - V1], m[i + V1]) + m[i]);
                    }
                }
                if (ginth > c->clip) hcd[i] = -ulim(ginth, m[i - 1], m[i + 1]) + m[i];
                if (gintv > c->clip) vcd[i] = -ulim(gintv, m[i - V1], m[i + V1]) + m[i];
            } else {
                ginth = hcd[i] + m[i];
                gintv = vcd[i] + m[i];
                if (hcd[i] < K(0.0)) {
                    if (K(3.0) * hcd[i] < -(ginth + m[i])) {
                        hcd[i] = ulim(ginth, m[i - 1], m[i + 1]) - m[i];
                    } else {
                        real w = K(1.0) + K(3.0) * hcd[i] / (eps + ginth + m[i]);
                        hcd[i] = w * hcd[i] + (K(1.0) - w) * (ulim(ginth, m[i - 1], m[i + 1]) - m[i]);
                    }
                }
                if (vcd[i] < K(0.0)) {
                    if (K(3.0) * vcd[i] < -(gintv + m[i])) {
                        vcd[i] = ulim(gintv, m[i - V1], m[i + V1]) - m[i];
                    } else {
                        real w = K(1.0) + K(3.0) * vcd[i] / (eps + gintv + m[i]);
                        vcd[i] = w * vcd[i] + (K(1.0) - w) * (ulim(gintv, m[i - V1], m[i + V1]) - m[i]);
                    }
                }
                if (ginth > c->clip) hcd[i] = ulim(ginth, m[i - 1], m[i + 1]) - m[i];
                if (gintv > c->clip) vcd[i] = ulim(gintv, m[i - V1], m[i + V1]) - m[i];
                t->cddiffsq[i] = sqr(vcd[i] - hcd[i]);
            }
        }
}

/* First index of the R/B sites of tile row rr at or after column `from`
 * (the reference's `from + (color_at(top+rr, left+2) & 1)`). */
static inline int rb_start(const Ctx *c, int rr, int from)
{
    return from + (fc(c, c->top + rr, c->left + 2) & 1);
}

/* Horizontal/vertical blend weight from colour-difference variances:
 * demosaic.rs:788-828. */
static void st_hv_weight(Tile *t, const Ctx *c)
{
    const real epssq = K(1e-10);
    const real *vcd = t->vcd, *hcd = t->hcd, *wv = t->wv, *wh = t->wh;
    const real *dv = t->dgintv, *dh = t->dginth;
    for (int rr = 6; rr < c->rr1 - 6; rr++)
        for (int cc = rb_start(c, rr, 6); cc < c->cc1 - 6; cc += 2) {
            int i = rr * TS + cc;
            real uave = vcd[i] + vcd[i - V1] + vcd[i - V2] + vcd[i - V3];
            real dave = vcd[i] + vcd[i + V1] + vcd[i + V2] + vcd[i + V3];
            real lave = hcd[i] + hcd[i - 1] + hcd[i - 2] + hcd[i - 3];
            real rave = hcd[i] + hcd[i + 1] + hcd[i + 2] + hcd[i + 3];
            real vu = sqr(vcd[i] - uave) + sqr(vcd[i - V1] - uave) + sqr(vcd[i - V2] - uave) + sqr(vcd[i - V3] - uave);
            real vd = sqr(vcd[i] - dave) + sqr(vcd[i + V1] - dave) + sqr(vcd[i + V2] - dave) + sqr(vcd[i + V3] - dave);
            real hl = sqr(hcd[i] - lave) + sqr(hcd[i - 1] - lave) + sqr(hcd[i - 2] - lave) + sqr(hcd[i - 3] - lave);
            real hr = sqr(hcd[i] - rave) + sqr(hcd[i + 1] - rave) + sqr(hcd[i + 2] - rave) + sqr(hcd[i + 3] - rave);
            real hwt = wh[i - 1] / RMAX(wh[i - 1] + wh[i + 1], K(1e-10));
            real vwt = wv[i - V1] / RMAX(wv[i + V1] + wv[i - V1], K(1e-10));
            real vvar = epssq + vwt * vd + (K(1.0) - vwt) * vu;
            real hvar = epssq + hwt * hr + (K(1.0) - hwt) * hl;
            real vu1 = dv[i] + dv[i - V1] + dv[i - V2];
            real vd1 = dv[i] + dv[i + V1] + dv[i + V2];
            real hl1 = dh[i] + dh[i - 1] + dh[i - 2];
            real hr1 = dh[i] + dh[i + 1] + dh[i + 2];
            real vvar1 = epssq + vwt * vd1 + (K(1.0) - vwt) * vu1;
            real hvar1 = epssq + hwt * hr1 + (K(1.0) - hwt) * hl1;
            real varwt = hvar / RMAX(vvar + hvar, K(1e-10));
            real diffwt = hvar1 / RMAX(vvar1 + hvar1, K(1e-10));
            if ((K(0.5) - varwt) * (K(0.5) - diffwt) > K(0.0) &&
                RABS(K(0.5) - diffwt) < RABS(K(0.5) - varwt))
                t->hvwt[i >> 1] = varwt;
            else
                t->hvwt[i >> 1] = diffwt;
        }
}

/* Nyquist texture test: demosaic.rs:830-849. */
static void st_nyquist_test(Tile *t, const Ctx *c)
{
    const real nyqthresh = K(0.5);
    const real go[4] = {K(0.14659727707323927), K(0.103592713382435), K(0.0732036125103057), K(0.0365543548389495)};
    const real gg[6] = {nyqthresh * K(0.07384411893421103), nyqthresh * K(0.06207511968171489),
                        nyqthresh * K(0.0521818194747806), nyqthresh * K(0.03687419286733595),
                        nyqthresh * K(0.03099732204057846), nyqthresh * K(0.018413194161458882)};
    const real *q = t->cddiffsq, *g = t->gradsq;
    for (int rr = 6; rr < c->rr1 - 6; rr++)
        for (int cc = rb_start(c, rr, 6); cc < c->cc1 - 6; cc += 2) {
            int i = rr * TS + cc;
            t->nyqutest[i >> 1] =
                (go[0] * q[i] + go[1] * (q[i - M1] + q[i - P1] + q[i + P1] + q[i + M1]) +
                 go[2] * (q[i - V2] + q[i - 2] + q[i + 2] + q[i + V2]) +
                 go[3] * (q[i - M2] + q[i - P2] + q[i + P2] + q[i + M2])) -
                (gg[0] * g[i] + gg[1] * (g[i - V1] + g[i + 1] + g[i - 1] + g[i + V1]) +
                 gg[2] * (g[i - M1] + g[i - P1] + g[i + P1] + g[i + M1]) +
                 gg[3] * (g[i - V2] + g[i - 2] + g[i + 2] + g[i + V2]) +
                 gg[4] * (g[i - V2 - 1] + g[i - V2 + 1] + g[i - TS - 2] + g[i - TS + 2] +
                          g[i + TS - 2] + g[i + TS + 2] + g[i + V2 - 1] + g[i + V2 + 1]) +
                 gg[5] * (g[i - M2] + g[i - P2] + g[i + P2] + g[i + M2]));
        }
}

typedef struct { int on, r0, r1, c0, c1; } NyqBox;

/* Nyquist flags, their bounding box, majority vote and area-based
 * H/V weight inside the box: demosaic.rs:851-947. */
static NyqBox st_nyquist(Tile *t, const Ctx *c)
{
    const real epssq = K(1e-10);
    int r0 = 0, r1 = 0, c0 = TS + 1, c1 = 0;
    for (int rr = 6; rr < c->rr1 - 6; rr++)
        for (int cc = rb_start(c, rr, 6); cc < c->cc1 - 6; cc += 2) {
            int i = rr * TS + cc;
            if (t->nyqutest[i >> 1] > K(0.0)) {
                t->nyq[i >> 1] = 1;
                if (r0 == 0) r0 = rr;
                r1 = rr;
                if (cc < c0) c0 = cc;
                if (cc > c1) c1 = cc;
            }
        }
    NyqBox b = {0, 0, 0, 0, 0};
    if (!(r0 != r1 && c0 != c1)) return b;
    r1 += 1;
    c1 += 1;
    c0 -= c0 & 1;
    if (r0 < 8) r0 = 8;
    if (r1 > c->rr1 - 8) r1 = c->rr1 - 8;
    if (c0 < 8) c0 = 8;
    if (c1 > c->cc1 - 8) c1 = c->cc1 - 8;
    b.on = 1; b.r0 = r0; b.r1 = r1; b.c0 = c0; b.c1 = c1;

    memset(t->nyq2 + 4 * TSH, 0, (size_t)(TS - 8 - 4) * TSH);
    for (int rr = r0; rr < r1; rr++)
        for (int i = rr * TS + rb_start(c, rr, c0); i < rr * TS + c1; i += 2) {
            unsigned s = t->nyq[(i - V2) >> 1] + t->nyq[(i - M1) >> 1] + t->nyq[(i - P1) >> 1] +
                         t->nyq[(i - 2) >> 1] + t->nyq[(i + 2) >> 1] + t->nyq[(i + P1) >> 1] +
                         t->nyq[(i + M1) >> 1] + t->nyq[(i + V2) >> 1];
            t->nyq2[i >> 1] = s > 4 ? 1 : (s < 4 ? 0 : t->nyq[i >> 1]);
        }
    const real *m = t->mos;
    for (int rr = r0; rr < r1; rr++)
        for (int i = rr * TS + rb_start(c, rr, c0); i < rr * TS + c1; i += 2) {
            if (!t->nyq2[i >> 1]) continue;
            real sumcfa = 0, sumh = 0, sumv = 0, sumsqh = 0, sumsqv = 0, area = 0;
            for (int di = -6; di < 7; di += 2)
                for (int dj = -6; dj < 7; dj += 2) {
                    int j = i + di * TS + dj;
                    if (t->nyq2[j >> 1]) {
                        real v = m[j];
                        sumcfa += v;
                        sumh += m[j - 1] + m[j + 1];
                        sumv += m[j - V1] + m[j + V1];
                        sumsqh += sqr(v - m[j - 1]) + sqr(v - m[j + 1]);
                        sumsqv += sqr(v - m[j - V1]) + sqr(v - m[j + V1]);
                        area += K(1.0);
                    }
                }
            sumh = sumcfa - sumh * K(0.5);
            sumv = sumcfa - sumv * K(0.5);
            area = area * K(0.5);
            real hvar = epssq + RABS(area * sumsqh - sumh * sumh);
            real vvar = epssq + RABS(area * sumsqv - sumv * sumv);
            t->hvwt[i >> 1] = hvar / (vvar + hvar);
        }
    return b;
}

/* Green at R/B sites; the weight smoothing reads the row above already
 * updated (scan order): demosaic.rs:949-976. */
static void st_green_rb(Tile *t, const Ctx *c)
{
    real *w = t->hvwt, *gr = t->green;
    for (int rr = 8; rr < c->rr1 - 8; rr++)
        for (int i = rr * TS + rb_start(c, rr, 8); i < rr * TS + c->cc1 - 8; i += 2) {
            real alt = (w[(i - M1) >> 1] + w[(i - P1) >> 1] + w[(i + P1) >> 1] + w[(i + M1) >> 1]) / K(4.0);
            if (RABS(K(0.5) - w[i >> 1]) < RABS(K(0.5) - alt)) w[i >> 1] = alt;
            real wt = w[i >> 1];
            t->dgrb0[i >> 1] = wt * t->vcd[i] + (K(1.0) - wt) * t->hcd[i];
            gr[i] = t->mos[i] + t->dgrb0[i >> 1];
            if (t->nyq2[i >> 1]) {
                t->dgrb2h[i >> 1] = sqr(gr[i] - (gr[i - 1] + gr[i + 1]) * K(0.5));
                t->dgrb2v[i >> 1] = sqr(gr[i] - (gr[i - V1] + gr[i + V1]) * K(0.5));
            } else {
                t->dgrb2h[i >> 1] = K(0.0);
                t->dgrb2v[i >> 1] = K(0.0);
            }
        }
}

/* Nyquist-region green refinement: demosaic.rs:978-998. */
static void st_nyquist_green(Tile *t, const Ctx *c, NyqBox b)
{
    const real epssq = K(1e-10);
    const real gq[4] = {K(0.169917), K(0.108947), K(0.069855), K(0.0287182)};
    if (!b.on) return;
    const real *h = t->dgrb2h, *v = t->dgrb2v;
    for (int rr = b.r0; rr < b.r1; rr++)
        for (int i = rr * TS + rb_start(c, rr, b.c0); i < rr * TS + b.c1; i += 2) {
            if (!t->nyq2[i >> 1]) continue;
            real gvarh = epssq + (gq[0] * h[i >> 1] +
                                  gq[1] * (h[(i - M1) >> 1] + h[(i - P1) >> 1] + h[(i + P1) >> 1] + h[(i + M1) >> 1]) +
                                  gq[2] * (h[(i - V2) >> 1] + h[(i - 2) >> 1] + h[(i + 2) >> 1] + h[(i + V2) >> 1]) +
                                  gq[3] * (h[(i - M2) >> 1] + h[(i - P2) >> 1] + h[(i + P2) >> 1] + h[(i + M2) >> 1]));
            real gvarv = epssq + (gq[0] * v[i >> 1] +
                                  gq[1] * (v[(i - M1) >> 1] + v[(i - P1) >> 1] + v[(i + P1) >> 1] + v[(i + M1) >> 1]) +
                                  gq[2] * (v[(i - V2) >> 1] + v[(i - 2) >> 1] + v[(i + 2) >> 1] + v[(i + V2) >> 1]) +
                                  gq[3] * (v[(i - M2) >> 1] + v[(i - P2) >> 1] + v[(i + P2) >> 1] + v[(i + M2) >> 1]));
            t->dgrb0[i >> 1] = (t->hcd[i] * gvarv + t->vcd[i] * gvarh) / (gvarv + gvarh);
            t->green[i] = t->mos[i] + t->dgrb0[i >> 1];
        }
}

/* Diagonal gradients per column pair: demosaic.rs:1000-1019. */
static void st_diag_setup(Tile *t, const Ctx *c)
{
    const real *m = t->mos;
    for (int rr = 6; rr < c->rr1 - 6; rr++) {
        int rb_even = (fc(c, c->top + rr, c->left + 2) & 1) == 0;
        for (int cc = 6; cc < c->cc1 - 6; cc += 2) {
            int i = rr * TS + cc, h = i >> 1;
            if (rb_even) {
                t->delp[h] = RABS(m[i - P1] - m[i + P1]);
                t->delm[h] = RABS(m[i + M1] - m[i - M1]);
                t->dgrbsq1p[h] = sqr(m[i + 1] - m[i + 1 - P1]) + sqr(m[i + 1] - m[i + 1 + P1]);
                t->dgrbsq1m[h] = sqr(m[i + 1] - m[i + 1 + M1]) + sqr(m[i + 1] - m[i + 1 - M1]);
            } else {
                t->dgrbsq1p[h] = sqr(m[i] - m[i - P1]) + sqr(m[i] - m[i + P1]);
                t->dgrbsq1m[h] = sqr(m[i] - m[i - M1]) + sqr(m[i] - m[i + M1]);
                t->delp[h] = RABS(m[i + 1 - P1] - m[i + 1 + P1]);
                t->delm[h] = RABS(m[i + 1 - M1] - m[i + 1 + M1]);
            }
        }
    }
}

/* Diagonal R/B interpolation at R/B sites: demosaic.rs:1021-1107. */
static void st_diag_interp(Tile *t, const Ctx *c)
{
    const real eps = K(1e-5), epssq = K(1e-10), arth = K(0.75);
    const real ge0 = K(0.13719494435797422), ge1 = K(0.05640252782101291);
    const real *m = t->mos, *dm = t->delm, *dp = t->delp, *qm = t->dgrbsq1m, *qp = t->dgrbsq1p;
    for (int rr = 8; rr < c->rr1 - 8; rr++)
        for (int cc = rb_start(c, rr, 8); cc < c->cc1 - 8; cc += 2) {
            int i = rr * TS + cc, h = i >> 1;
            real crse = (m[i + M1] * K(2.0)) / (eps + m[i] + m[i + M2]);
            real crnw = (m[i - M1] * K(2.0)) / (eps + m[i] + m[i - M2]);
            real crne = (m[i - P1] * K(2.0)) / (eps + m[i] + m[i - P2]);
            real crsw = (m[i + P1] * K(2.0)) / (eps + m[i] + m[i + P2]);
            real rbse = RABS(K(1.0) - crse) < arth ? m[i] * crse : m[i + M1] + (m[i] - m[i + M2]) * K(0.5);
            real rbnw = RABS(K(1.0) - crnw) < arth ? m[i] * crnw : m[i - M1] + (m[i] - m[i - M2]) * K(0.5);
            real rbne = RABS(K(1.0) - crne) < arth ? m[i] * crne : m[i - P1] + (m[i] - m[i - P2]) * K(0.5);
            real rbsw = RABS(K(1.0) - crsw) < arth ? m[i] * crsw : m[i + P1] + (m[i] - m[i + P2]) * K(0.5);
            real wtse = eps + dm[h] + dm[(i + M1) >> 1] + dm[(i + M2) >> 1];
            real wtnw = eps + dm[h] + dm[(i - M1) >> 1] + dm[(i - M2) >> 1];
            real wtne = eps + dp[h] + dp[(i - P1) >> 1] + dp[(i - P2) >> 1];
            real wtsw = eps + dp[h] + dp[(i + P1) >> 1] + dp[(i + P2) >> 1];
            t->rbm[h] = (wtse * rbnw + wtnw * rbse) / (wtse + wtnw);
            t->rbp[h] = (wtne * rbsw + wtsw * rbne) / (wtne + wtsw);
            real varm = epssq + ge0 * (qm[(i - V1) >> 1] + qm[(i - 1) >> 1] + qm[(i + 1) >> 1] + qm[(i + V1) >> 1]) +
                        ge1 * (qm[(i - V2 - 1) >> 1] + qm[(i - V2 + 1) >> 1] + qm[(i - 2 - V1) >> 1] + qm[(i + 2 - V1) >> 1] +
                               qm[(i - 2 + V1) >> 1] + qm[(i + 2 + V1) >> 1] + qm[(i + V2 - 1) >> 1] + qm[(i + V2 + 1) >> 1]);
            real varp = epssq + ge0 * (qp[(i - V1) >> 1] + qp[(i - 1) >> 1] + qp[(i + 1) >> 1] + qp[(i + V1) >> 1]) +
                        ge1 * (qp[(i - V2 - 1) >> 1] + qp[(i - V2 + 1) >> 1] + qp[(i - 2 - V1) >> 1] + qp[(i + 2 - V1) >> 1] +
                               qp[(i - 2 + V1) >> 1] + qp[(i + 2 + V1) >> 1] + qp[(i + V2 - 1) >> 1] + qp[(i + V2 + 1) >> 1]);
            t->pmwt[h] = varm / (varp + varm);
            if (t->rbp[h] < m[i]) {
                if (t->rbp[h] * K(2.0) < m[i]) {
                    t->rbp[h] = ulim(t->rbp[h], m[i - P1], m[i + P1]);
                } else {
                    real pw = (m[i] - t->rbp[h]) * K(2.0) / (eps + t->rbp[h] + m[i]);
                    t->rbp[h] = pw * t->rbp[h] + (K(1.0) - pw) * ulim(t->rbp[h], m[i - P1], m[i + P1]);
                }
            }
            if (t->rbm[h] < m[i]) {
                if (t->rbm[h] * K(2.0) < m[i]) {
                    t->rbm[h] = ulim(t->rbm[h], m[i - M1], m[i + M1]);
                } else {
                    real mw = (m[i] - t->rbm[h]) * K(2.0) / (eps + t->rbm[h] + m[i]);
                    t->rbm[h] = mw * t->rbm[h] + (K(1.0) - mw) * ulim(t->rbm[h], m[i - M1], m[i + M1]);
                }
            }
            if (t->rbp[h] > c->clip) t->rbp[h] = ulim(t->rbp[h], m[i - P1], m[i + P1]);
            if (t->rbm[h] > c->clip) t->rbm[h] = ulim(t->rbm[h], m[i - M1], m[i + M1]);
        }
}

/* Diagonal weight smoothing (row above already updated) and the R+B
 * estimate at R/B sites: demosaic.rs:1109-1123. */
static void st_rb_interp(Tile *t, const Ctx *c)
{
    real *pm = t->pmwt;
    for (int rr = 10; rr < c->rr1 - 10; rr++)
        for (int cc = rb_start(c, rr, 10); cc < c->cc1 - 10; cc += 2) {
            int i = rr * TS + cc, h = i >> 1;
            real alt = (pm[(i - M1) >> 1] + pm[(i - P1) >> 1] + pm[(i + P1) >> 1] + pm[(i + M1) >> 1]) / K(4.0);
            if (RABS(K(0.5) - pm[h]) < RABS(K(0.5) - alt)) pm[h] = alt;
            t->rbint[h] = (t->mos[i] + t->rbm[h] * (K(1.0) - pm[h]) + t->rbp[h] * pm[h]) * K(0.5);
        }
}

/* Green refinement where the diagonal estimate is more decisive:
 * demosaic.rs:1125-1194. */
static void st_green_refine(Tile *t, const Ctx *c)
{
    const real eps = K(1e-5), arth = K(0.75);
    const real *m = t->mos, *rb = t->rbint, *wv = t->wv, *wh = t->wh;
    for (int rr = 12; rr < c->rr1 - 12; rr++)
        for (int cc = rb_start(c, rr, 12); cc < c->cc1 - 12; cc += 2) {
            int i = rr * TS + cc, h = i >> 1;
            if (!(RABS(K(0.5) - t->pmwt[h]) >= RABS(K(0.5) - t->hvwt[h]))) continue;
            real cru = m[i - V1] * K(2.0) / (eps + rb[h] + rb[h - V1]);
            real crd = m[i + V1] * K(2.0) / (eps + rb[h] + rb[h + V1]);
            real crl = m[i - 1] * K(2.0) / (eps + rb[h] + rb[h - 1]);
            real crr = m[i + 1] * K(2.0) / (eps + rb[h] + rb[h + 1]);
            real gu = RABS(K(1.0) - cru) < arth ? rb[h] * cru : m[i - V1] + (rb[h] - rb[h - V1]) * K(0.5);
            real gd = RABS(K(1.0) - crd) < arth ? rb[h] * crd : m[i + V1] + (rb[h] - rb[h + V1]) * K(0.5);
            real gl = RABS(K(1.0) - crl) < arth ? rb[h] * crl : m[i - 1] + (rb[h] - rb[h - 1]) * K(0.5);
            real gr = RABS(K(1.0) - crr) < arth ? rb[h] * crr : m[i + 1] + (rb[h] - rb[h + 1]) * K(0.5);
            real gintv = (wv[i - V1] * gd + wv[i + V1] * gu) / RMAX(wv[i + V1] + wv[i - V1], K(1e-10));
            real ginth = (wh[i - 1] * gr + wh[i + 1] * gl) / RMAX(wh[i - 1] + wh[i + 1], K(1e-10));
            if (gintv < rb[h]) {
                if (K(2.0) * gintv < rb[h]) {
                    gintv = ulim(gintv, m[i - V1], m[i + V1]);
                } else {
                    real w = K(2.0) * (rb[h] - gintv) / (eps + gintv + rb[h]);
                    gintv = w * gintv + (K(1.0) - w) * ulim(gintv, m[i - V1], m[i + V1]);
                }
            }
            if (ginth < rb[h]) {
                if (K(2.0) * ginth < rb[h]) {
                    ginth = ulim(ginth, m[i - 1], m[i + 1]);
                } else {
                    real w = K(2.0) * (rb[h] - ginth) / (eps + ginth + rb[h]);
                    ginth = w * ginth + (K(1.0) - w) * ulim(ginth, m[i - 1], m[i + 1]);
                }
            }
            if (ginth > c->clip) ginth = ulim(ginth, m[i - 1], m[i + 1]);
            if (gintv > c->clip) gintv = ulim(gintv, m[i - V1], m[i + V1]);
            t->green[i] = ginth * (K(1.0) - t->hvwt[h]) + gintv * t->hvwt[h];
            t->dgrb0[h] = t->green[i] - m[i];
        }
}

/* Chroma: move the B rows' difference to dgrb1, then interpolate each
 * colour difference at the opposite-colour sites: demosaic.rs:1196-1252. */
static void st_chroma(Tile *t, const Ctx *c)
{
    const real eps = K(1e-5);
    int ex, ey;
    if (fc(c, 0, 0) == 1) {
        if (fc(c, 0, 1) == 0) { ex = 1; ey = 0; } else { ex = 0; ey = 1; }
    } else {
        if (fc(c, 0, 0) == 0) { ex = 0; ey = 0; } else { ex = 1; ey = 1; }
    }
    for (int rr = 13 - ey; rr < c->rr1 - 12; rr += 2)
        for (int h = (rr * TS + 13 - ex) >> 1; h < (rr * TS + c->cc1 - 12) >> 1; h++) {
            t->dgrb1[h] = t->dgrb0[h];
            t->dgrb0[h] = K(0.0);
        }
    for (int rr = 14; rr < c->rr1 - 14; rr++)
        for (int cc = rb_start(c, rr, 14); cc < c->cc1 - 14; cc += 2) {
            int i = rr * TS + cc;
            int which = 1 - (fc(c, c->top + rr, c->left + cc) / 2);
            real *d = which == 0 ? t->dgrb0 : t->dgrb1;
#define D(o) d[(i + (o)) >> 1]
            real wtnw = K(1.0) / (eps + RABS(D(-M1) - D(M1)) + RABS(D(-M1) - D(-M3)) + RABS(D(M1) - D(-M3)));
            real wtne = K(1.0) / (eps + RABS(D(-P1) - D(P1)) + RABS(D(-P1) - D(-P3)) + RABS(D(P1) - D(-P3)));
            real wtsw = K(1.0) / (eps + RABS(D(P1) - D(-P1)) + RABS(D(P1) - D(M3)) + RABS(D(-P1) - D(P3)));
            real wtse = K(1.0) / (eps + RABS(D(M1) - D(-M1)) + RABS(D(M1) - D(P3)) + RABS(D(-M1) - D(M3)));
            real v = (wtnw * (K(1.325) * D(-M1) - K(0.175) * D(-M3) - K(0.075) * D(-M1 - 2) - K(0.075) * D(-M1 - V2)) +
                      wtne * (K(1.325) * D(-P1) - K(0.175) * D(-P3) - K(0.075) * D(-P1 + 2) - K(0.075) * D(-P1 + V2)) +
                      wtsw * (K(1.325) * D(P1) - K(0.175) * D(P3) - K(0.075) * D(P1 - 2) - K(0.075) * D(-M1)) +
                      wtse * (K(1.325) * D(M1) - K(0.175) * D(M3) - K(0.075) * D(M1 + 2) - K(0.075) * D(M1 + V2))) /
                     (wtnw + wtne + wtsw + wtse);
#undef D
            d[i >> 1] = v;
        }
}

static inline void out_px(const Ctx *c, int row, int col, real r, real g, real b)
{
    if (col >= 0 && col < c->W && row >= 0 && row < c->H) {
        real *o = c->out + ((size_t)row * c->W + col) * 3;
        o[0] = r; o[1] = g; o[2] = b;
    }
}

/* Output writes: demosaic.rs:1254-1366. */
static void st_output(Tile *t, const Ctx *c)
{
    const real *w = t->hvwt, *d0 = t->dgrb0, *d1 = t->dgrb1, *gr = t->green;
    for (int rr = 16; rr < c->rr1 - 16; rr++) {
        int row = rr + c->top, col = c->left + 16, i = rr * TS + 16;
        int first_is_g = (fc(c, c->top + rr, c->left + 2) & 1) == 1;
        int end = rr * TS + c->cc1 - 16 - (c->cc1 & 1);
        /* green site: weighted neighbour differences; R/B site: own differences */
#define GSITE()                                                                          \
    do {                                                                                 \
        real tmp = K(1.0) / RMAX(w[(i - V1) >> 1] + K(2.0) - w[(i + 1) >> 1] -            \
                                     w[(i - 1) >> 1] + w[(i + V1) >> 1], K(1e-5));       \
        real r = clampnan(gr[i] - ((w[(i - V1) >> 1]) * d0[(i - V1) >> 1] +              \
                                   (K(1.0) - w[(i + 1) >> 1]) * d0[(i + 1) >> 1] +       \
                                   (K(1.0) - w[(i - 1) >> 1]) * d0[(i - 1) >> 1] +       \
                                   (w[(i + V1) >> 1]) * d0[(i + V1) >> 1]) * tmp,        \
                          K(0.0), K(1.0));                                               \
        real b = clampnan(gr[i] - ((w[(i - V1) >> 1]) * d1[(i - V1) >> 1] +              \
                                   (K(1.0) - w[(i + 1) >> 1]) * d1[(i + 1) >> 1] +       \
                                   (K(1.0) - w[(i - 1) >> 1]) * d1[(i - 1) >> 1] +       \
                                   (w[(i + V1) >> 1]) * d1[(i + V1) >> 1]) * tmp,        \
                          K(0.0), K(1.0));                                               \
        out_px(c, row, col, r, clampnan(gr[i], K(0.0), K(1.0)), b);                      \
    } while (0)
#define RBSITE()                                                                         \
    out_px(c, row, col, clampnan(gr[i] - d0[i >> 1], K(0.0), K(1.0)),                   \
           clampnan(gr[i], K(0.0), K(1.0)), clampnan(gr[i] - d1[i >> 1], K(0.0), K(1.0)))
        if (first_is_g) {
            while (i < end) {
                GSITE(); i++; col++;
                RBSITE(); i++; col++;
            }
            if (c->cc1 & 1) GSITE();
        } else {
            while (i < end) {
                RBSITE(); i++; col++;
                GSITE(); i++; col++;
            }
            if (c->cc1 & 1) RBSITE();
        }
#undef GSITE
#undef RBSITE
    }
}

/* Largest flat tile index the border fill of tile (top,left) writes: the
 * same ranges as fill_tile, evaluated without filling. */
static long fill_max_index(int W, int H, int top, int left)
{
    const int bottom = (top + 128 < H + 16) ? top + 128 : H + 16;
    const int right = (left + 128 < W + 16) ? left + 128 : W + 16;
    const int rr1 = bottom - top, cc1 = right - left;
    const int rrmin = top < 0 ? 16 : 0, ccmin = left < 0 ? 16 : 0;
    const int rrmax = bottom > H ? H - top : rr1;
    const int ccmax = right > W ? W - left : cc1;
    long hi = -1;
#define SPAN(r0, r1, c0, c1)                                            \
    if ((r0) < (r1) && (c0) < (c1)) {                                   \
        long v = (long)((r1) - 1) * TS + ((c1) - 1);                    \
        if (v > hi) hi = v;                                             \
    }
    if (rrmin > 0) SPAN(0, 16, ccmin, ccmax);
    SPAN(rrmin, rrmax, ccmin, ccmax);
    if (rrmax < rr1) SPAN(rrmax, rrmax + 16, ccmin, ccmax);
    if (ccmin > 0) SPAN(rrmin, rrmax, 0, 16);
    if (ccmax < cc1) SPAN(rrmin, rrmax, ccmax, ccmax + 16);
    if (rrmin > 0 && ccmin > 0) SPAN(0, 16, 0, 16);
    if (rrmax < rr1 && ccmax < cc1) SPAN(rrmax, rrmax + 16, ccmax, ccmax + 16);
    if (rrmin > 0 && ccmax < cc1) SPAN(0, 16, ccmax, ccmax + 16);
    if (rrmax < rr1 && ccmin > 0) SPAN(rrmax, rrmax + 16, 0, 16);
#undef SPAN
    return hi;
}

/* Whether the reference's border fill stays inside the 128x128 tile buffer
 * for every tile of a W x H image (the reference panics otherwise). */
int OSYM(oracle_amaze_size_ok)(int W, int H)
{
    for (int top = -16; top < H; top += 96)
        for (int left = -16; left < W; left += 96)
            if (fill_max_index(W, H, top, left) >= NF) return 0;
    return 1;
}

typedef struct {
    const real *in;
    real *out;
    int W, H, ntx;
    const OracleCfa *cfa;
    real clip;
    Tile **scratch;
    int err;
} Job;

static void run_tiles(void *p, int worker, long b, long e)
{
    Job *j = (Job *)p;
    Tile *t = j->scratch[worker];
    for (long k = b; k < e; k++) {
        Ctx c;
        c.in = j->in; c.out = j->out; c.W = j->W; c.H = j->H; c.cfa = j->cfa; c.clip = j->clip;
        c.top = -16 + (int)(k / j->ntx) * 96;
        c.left = -16 + (int)(k % j->ntx) * 96;
        memset(t, 0, sizeof(Tile));
        if (fill_tile(t, &c) != 0) { __atomic_store_n(&j->err, 1, __ATOMIC_RELAXED); continue; }
        st_gradients(t, &c);
        st_colour_diff(t, &c);
        st_cd_refine(t, &c);
        st_hv_weight(t, &c);
        st_nyquist_test(t, &c);
        NyqBox box = st_nyquist(t, &c);
        st_green_rb(t, &c);
        st_nyquist_green(t, &c, box);
        st_diag_setup(t, &c);
        st_diag_interp(t, &c);
        st_rb_interp(t, &c);
        st_green_refine(t, &c);
        st_chroma(t, &c);
        st_output(t, &c);
    }
}

/* Demosaic a W x H mosaic (row-major, values ~[0,1]) into interleaved RGB.
 * cfa: the crop-shifted 2x2 Bayer period.  Tiles write disjoint output
 * pixels, so they run in parallel on `threads` threads. */
int OSYM(oracle_amaze)(const real *in, int W, int H, const OracleCfa *cfa, real clip_pt,
                        real *out, int threads)
{
    if (!in || !out || !cfa || W <= 0 || H <= 0) return ORACLE_ERR_ARG;
    if (cfa->pw != 2 || cfa->ph != 2) return ORACLE_ERR_CFA;
    if (!OSYM(oracle_amaze_size_ok)(W, H)) return ORACLE_ERR_SIZE;
    int nty = 0, ntx = 0;
    for (int top = -16; top < H; top += 96) nty++;
    for (int left = -16; left < W; left += 96) ntx++;
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    Job j = {in, out, W, H, ntx, cfa, clip_pt, NULL, 0};
    j.scratch = (Tile **)calloc((size_t)threads, sizeof(Tile *));
    if (!j.scratch) return ORACLE_ERR_ARG;
    for (int i = 0; i < threads; i++) {
        j.scratch[i] = (Tile *)malloc(sizeof(Tile));
        if (!j.scratch[i]) j.err = 1;
    }
    if (!j.err) oracle_parallel_for((long)nty * ntx, 2, threads, run_tiles, &j);
    for (int i = 0; i < threads; i++) free(j.scratch[i]);
    free(j.scratch);
    return j.err ? ORACLE_ERR_SIZE : ORACLE_OK;
}
