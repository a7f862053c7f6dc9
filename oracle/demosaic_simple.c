/*
 * demosaic_simple.c -- CPU oracle for the reference's non-AMaZE demosaics.
 *
 * TEST INFRASTRUCTURE (see oracle_common.h).
 *  - "Markesteijn": the reference's 3x3 same-colour mean
 *    (pichromatic/src/demosaic.rs:108-186); works for any CFA period.
 *  - Fast / SuperFast / SuperSuperFast: one 2x2 quad sampled every
 *    2 / 4 / 8 pixels (demosaic.rs:189-356).
 */
#include "oracle_common.h"

/* 3x3 same-colour mean: window clamped at the image edge, rows then columns
 * in ascending order, centre skipped; a channel with no neighbour stays 0
 * (demosaic.rs:121-174). */
typedef struct {
    const real *in;
    real *out;
    int W, H;
    const OracleCfa *cfa;
} MJob;

static void mean_rows(void *p, int worker, long rb, long re)
{
    MJob *j = (MJob *)p;
    const real *in = j->in;
    real *out = j->out;
    const int W = j->W, H = j->H;
    const OracleCfa *cfa = j->cfa;
    (void)worker;
    for (int row = (int)rb; row < (int)re; row++) {
        int y0 = row > 0 ? row - 1 : 0;
        int y1 = row + 1 < H - 1 ? row + 1 : H - 1;
        for (int col = 0; col < W; col++) {
            int x0 = col > 0 ? col - 1 : 0;
            int x1 = col + 1 < W - 1 ? col + 1 : W - 1;
            int centre = ocfa_color(cfa, row, col);
            real *o = out + ((size_t)row * W + col) * 3;
            for (int ch = 0; ch < 3; ch++) {
                if (ch == centre) {
                    o[ch] = in[(size_t)row * W + col];
                    continue;
                }
                real sum = K(0.0), cnt = K(0.0);
                for (int ny = y0; ny <= y1; ny++)
                    for (int nx = x0; nx <= x1; nx++) {
                        if (ny == row && nx == col) continue;
                        if (ocfa_color(cfa, ny, nx) == ch) {
                            sum += in[(size_t)ny * W + nx];
                            cnt += K(1.0);
                        }
                    }
                o[ch] = cnt > K(0.0) ? sum / cnt : K(0.0);
            }
        }
    }
}

int OSYM(oracle_mean3x3)(const real *in, int W, int H, const OracleCfa *cfa, real *out, int threads)
{
    if (!in || !out || !cfa || W <= 0 || H <= 0) return ORACLE_ERR_ARG;
    MJob j = {in, out, W, H, cfa};
    oracle_parallel_for(H, 16, threads, mean_rows, &j);
    return ORACLE_OK;
}

/* Subsampled quad demosaic (factor 2, 4 or 8): output (W/f) x (H/f); the
 * quad's four sites are assigned in the order (0,0),(0,1),(1,0),(1,1), so a
 * later site of the same colour wins (demosaic.rs:201-222). */
int OSYM(oracle_quad)(const real *in, int W, int H, const OracleCfa *cfa, int factor, real *out)
{
    if (!in || !out || !cfa || W <= 0 || H <= 0) return ORACLE_ERR_ARG;
    if (factor != 2 && factor != 4 && factor != 8) return ORACLE_ERR_ARG;
    int c00 = ocfa_color(cfa, 0, 0), c01 = ocfa_color(cfa, 0, 1);
    int c10 = ocfa_color(cfa, 1, 0), c11 = ocfa_color(cfa, 1, 1);
    if (c00 > 2 || c01 > 2 || c10 > 2 || c11 > 2) return ORACLE_ERR_CFA;
    int nw = W / factor, nh = H / factor;
    for (int y = 0; y < nh; y++)
        for (int x = 0; x < nw; x++) {
            size_t tl = (size_t)(y * factor) * W + (size_t)(x * factor);
            real v[3] = {K(0.0), K(0.0), K(0.0)};
            v[c00] = in[tl];
            v[c01] = in[tl + 1];
            v[c10] = in[tl + W];
            v[c11] = in[tl + W + 1];
            real *o = out + ((size_t)y * nw + x) * 3;
            o[0] = v[0]; o[1] = v[1]; o[2] = v[2];
        }
    return ORACLE_OK;
}
