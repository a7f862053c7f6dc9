// film_host.cpp -- stock definitions and the per-stock precomputation of the
// film simulation, done once on the host in f64 (the reference's precision
// for spectral quantities) and handed to the kernels as f32 tables.
//
// Stocks follow pichromatic/src/film/stock/{color_neg_200.rs, bw_stub.rs};
// the LUT, kappa and scan constants follow stock/mod.rs:152-214,
// exposure/capture.rs:37-110, film/scan/densitometry.rs:13-117.
#include <cmath>
#include <cstring>
#include <vector>

#include "film.cuh"

namespace imops {
namespace film {

namespace {

constexpr double PI = 3.14159265358979323846264338327950288;
constexpr double FRAC_PI_3 = 1.04719755119659774615421446109316763;
constexpr double LOG2_10 = 3.32192809488736234787031942948939018;

// CIE 1931 2-degree CMFs at 400..700 nm / 20 nm (film/exposure/upsample.rs:17-30)
const double CMF16[3][NB16] = {
    {0.01431, 0.13438, 0.34828, 0.29080, 0.09564, 0.00490, 0.06327, 0.29040, 0.59450, 0.91630, 1.06220, 0.85445,
     0.44790, 0.16490, 0.04677, 0.01136},
    {0.000396, 0.004000, 0.023000, 0.060000, 0.139020, 0.323000, 0.710000, 0.954000, 0.995000, 0.870000, 0.631000,
     0.381000, 0.175000, 0.061000, 0.017000, 0.004100},
    {0.06785, 0.64560, 1.74706, 1.66920, 0.81295, 0.27200, 0.07825, 0.02030, 0.00390, 0.00165, 0.00080, 0.00019,
     0.00002, 0.00000, 0.00000, 0.00000}};
// XYZ(D65) -> ACEScg (upsample.rs:34-38)
const double XYZ2AP1[3][3] = {{1.6410233797, -0.3248032942, -0.2364246952},
                              {-0.6636628587, 1.6153315917, 0.0167563477},
                              {0.0117218943, -0.0082844165, 0.9883948585}};

double lam16(int i) { return 400.0 + 20.0 * i; }

void inv3(const double m[3][3], double r[3][3]) {
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

enum Kind { EMULSION, FILTER, OVERCOAT, ANTIHALATION, SUPPORT };

struct Layer {
    Kind kind;
    float thickness;
    std::vector<double> sens;  // spectral sensitivity / absorption curve (16)
    double mu_ln = 0, sigma_ln = 0;
    float fraction = 0;
    std::vector<double> eps, mask_eps;  // dye and mask absorptivity (16)
    float dmax = 0, gamma = 1;
    double capture_k = 1;
    float recip_p = 1;
    bool reversal = false;
};

struct StockDef {
    float box_iso;
    std::vector<Layer> layers;
    std::vector<double> refl;
    float psf_local, psf_halation;
    float dev_diff, adj_beta, dir_diff;
    std::vector<std::vector<float>> dir;
    std::vector<double> scanner;
};

// A stock as the reference's stock files list it: one row per EmulsionLayer,
// in stack order (film/stock/ files).  Curves: 'g' gaussian_curve(a, b, c),
// 'c' SpectralCurve::constant(a), 'p' panchromatic a + b * max(0, sin(pi t))
// with t = (lambda - 400) / 300 (bw_stub.rs, trix_400.rs).
struct LayerRow {
    Kind kind;
    float thick;
    char sens;
    double sa, sb, sc;
    double mean_um, sig_ln;
    float frac;
    char eps;
    double ea, eb, ec;
    bool mask;
    float dmax, gamma;
    double k;
    float p;
};

struct StockRow {
    float box_iso;
    double mask_b, mask_g, mask_0;  // orange mask: mask_b*blue + mask_g*green + mask_0
    char refl;
    double ra, rb, rc;
    float psf_local, psf_halation, dev_diff, adj_beta, dir_diff;
    bool reversal;
    std::vector<LayerRow> layers;
    std::vector<std::vector<float>> dir;
};

std::vector<double> curve16(char kind, double a, double b, double c) {
    std::vector<double> s(NB16, 0.0);
    for (int i = 0; i < NB16; i++) {
        if (kind == 'g') {
            double d = (lam16(i) - a) / b;
            s[i] = c * std::exp(-0.5 * d * d);
        } else if (kind == 'c') {
            s[i] = a;
        } else if (kind == 'p') {
            double t = (lam16(i) - 400.0) / 300.0;
            double env = std::sin(PI * t);
            if (env < 0.0) env = 0.0;
            s[i] = a + b * env;
        }
    }
    return s;
}

StockDef from_rows(const StockRow& R) {
    StockDef sd;
    sd.box_iso = R.box_iso;
    for (const LayerRow& r : R.layers) {
        Layer l;
        l.kind = r.kind;
        l.thickness = r.thick;
        l.sens = curve16(r.sens, r.sa, r.sb, r.sc);
        l.gamma = r.gamma;
        l.capture_k = r.k;
        l.recip_p = r.p;
        l.reversal = R.reversal;
        if (r.kind == EMULSION) {
            l.mu_ln = std::log(r.mean_um);
            l.sigma_ln = r.sig_ln;
            l.fraction = r.frac;
            l.eps = curve16(r.eps, r.ea, r.eb, r.ec);
            if (r.mask) {
                l.mask_eps.resize(NB16);
                for (int i = 0; i < NB16; i++) {
                    double lm = lam16(i), bd = (lm - 450.0) / 50.0, gd = (lm - 520.0) / 60.0;
                    double blue = std::exp(-0.5 * (bd * bd));
                    double green = 0.6 * std::exp(-0.5 * (gd * gd));
                    l.mask_eps[i] = R.mask_b * blue + R.mask_g * green + R.mask_0;
                }
            }
            l.dmax = r.dmax;
        }
        sd.layers.push_back(l);
    }
    sd.refl = curve16(R.refl, R.ra, R.rb, R.rc);
    sd.psf_local = R.psf_local;
    sd.psf_halation = R.psf_halation;
    sd.dev_diff = R.dev_diff;
    sd.adj_beta = R.adj_beta;
    sd.dir_diff = R.dir_diff;
    sd.dir = R.dir;
    sd.scanner.assign(NB16, 1.0);
    return sd;
}

constexpr LayerRow overcoat_row() { return {OVERCOAT, 1.0f, 'c', 0.01, 0, 0, 0, 0, 0.0f, 0, 0, 0, 0, false, 0.0f, 1.0f, 1.0, 1.0f}; }
constexpr LayerRow absorber_row(Kind k, float thick, double a, double b, double c) {
    return {k, thick, 'g', a, b, c, 0, 0, 0.0f, 0, 0, 0, 0, false, 0.0f, 1.0f, 1.0, 1.0f};
}
constexpr LayerRow emulsion_row(float thick, double sa, double sb, double sc, double mean, double sig, float frac,
                                double ea, double eb, double ec, bool mask, float dmax, float gamma, double k, float p) {
    return {EMULSION, thick, 'g', sa, sb, sc, mean, sig, frac, 'g', ea, eb, ec, mask, dmax, gamma, k, p};
}

// The stocks, in StockId order (film/stock/mod.rs:126-147).
StockRow stock_row(int id) {
    switch (id) {
    case 0:  // BwStub (film/stock/bw_stub.rs:18-82)
        return StockRow{100.0f, 0.0, 0.0, 0.0, 'c', 0.0, 0.0, 0.0,
                        2.0f, 40.0f, 5.0f, 0.3f, 10.0f, false,
                        {LayerRow{EMULSION, 10.0f, 'p', 0.3, 0.7, 0, 0.7, 0.35, 0.2f, 'c', 1.0, 0, 0, false, 2.5f, 0.65f, 1.0, 1.0f}},
                        {{0.0f}}};
    case 1:  // ColorNeg200 (film/stock/color_neg_200.rs:67-208)
        return StockRow{200.0f, 0.35, 0.25, 0.05, 'g', 680.0, 60.0, 0.08,
                        3.0f, 80.0f, 8.0f, 0.35f, 15.0f, false,
                        {overcoat_row(),
                         emulsion_row(4.0f, 450.0, 35.0, 1.0, 0.55, 0.3, 0.18f, 450.0, 40.0, 1.0, true, 2.2f, 0.65f, 4.2, 0.88f),
                         absorber_row(FILTER, 2.0f, 430.0, 40.0, 1.2),
                         emulsion_row(5.0f, 550.0, 40.0, 1.0, 0.6, 0.32, 0.18f, 550.0, 40.0, 1.0, true, 2.2f, 0.65f, 2.1, 0.9f),
                         emulsion_row(6.0f, 650.0, 45.0, 1.0, 0.7, 0.35, 0.18f, 650.0, 45.0, 1.0, true, 2.2f, 0.65f, 1.35, 0.92f),
                         absorber_row(ANTIHALATION, 2.0f, 650.0, 80.0, 0.3)},
                        {{0.02f, 0.05f, 0.03f}, {0.05f, 0.02f, 0.06f}, {0.03f, 0.06f, 0.02f}}};
    case 2:  // Portra400 (film/stock/portra_400.rs:42-245)
        return StockRow{400.0f, 0.32, 0.22, 0.04, 'g', 680.0, 60.0, 0.06,
                        3.0f, 70.0f, 7.0f, 0.3f, 16.0f, false,
                        {overcoat_row(),
                         emulsion_row(2.5f, 450.0, 35.0, 1.0, 0.85, 0.35, 0.16f, 450.0, 40.0, 1.0, true, 1.1f, 0.54f, 4.8, 0.85f),
                         emulsion_row(2.5f, 450.0, 35.0, 0.8, 0.42, 0.28, 0.2f, 450.0, 40.0, 1.0, true, 1.1f, 0.54f, 2.2, 0.89f),
                         absorber_row(FILTER, 2.0f, 430.0, 40.0, 1.3),
                         emulsion_row(3.0f, 550.0, 40.0, 1.0, 0.9, 0.35, 0.16f, 550.0, 40.0, 1.0, true, 1.1f, 0.54f, 2.4, 0.87f),
                         emulsion_row(3.0f, 550.0, 40.0, 0.8, 0.45, 0.28, 0.2f, 550.0, 40.0, 1.0, true, 1.1f, 0.54f, 1.1, 0.91f),
                         emulsion_row(3.5f, 650.0, 45.0, 1.0, 0.95, 0.35, 0.16f, 650.0, 45.0, 1.0, true, 1.1f, 0.54f, 1.5, 0.89f),
                         emulsion_row(3.5f, 650.0, 45.0, 0.8, 0.48, 0.28, 0.2f, 650.0, 45.0, 1.0, true, 1.1f, 0.54f, 0.7, 0.93f),
                         absorber_row(ANTIHALATION, 2.0f, 650.0, 80.0, 0.3)},
                        {{0.02f, 0.01f, 0.04f, 0.02f, 0.03f, 0.01f}, {0.01f, 0.01f, 0.02f, 0.01f, 0.02f, 0.01f}, {0.04f, 0.02f, 0.02f, 0.01f, 0.05f, 0.02f}, {0.02f, 0.01f, 0.01f, 0.01f, 0.02f, 0.01f}, {0.03f, 0.01f, 0.05f, 0.02f, 0.02f, 0.01f}, {0.01f, 0.01f, 0.02f, 0.01f, 0.01f, 0.01f}}};
    case 3:  // Ektar100 (film/stock/ektar_100.rs:46-270)
        return StockRow{100.0f, 0.38, 0.26, 0.05, 'g', 680.0, 60.0, 0.05,
                        2.5f, 55.0f, 6.0f, 0.55f, 14.0f, false,
                        {overcoat_row(),
                         emulsion_row(2.8f, 450.0, 32.0, 1.0, 0.82, 0.32, 0.17f, 450.0, 30.0, 1.25, true, 1.25f, 0.58f, 4.8, 0.86f),
                         emulsion_row(2.5f, 450.0, 32.0, 0.85, 0.38, 0.24, 0.21f, 450.0, 30.0, 1.25, true, 1.9f, 0.34f, 6.5, 0.9f),
                         absorber_row(FILTER, 2.0f, 430.0, 38.0, 1.35),
                         emulsion_row(3.2f, 545.0, 36.0, 1.0, 0.88, 0.32, 0.17f, 545.0, 30.0, 1.25, true, 1.25f, 0.58f, 2.6, 0.88f),
                         emulsion_row(3.0f, 545.0, 36.0, 0.85, 0.4, 0.24, 0.21f, 545.0, 30.0, 1.25, true, 1.9f, 0.34f, 3.6, 0.92f),
                         emulsion_row(3.6f, 650.0, 40.0, 1.0, 0.92, 0.32, 0.17f, 650.0, 32.0, 1.25, true, 1.25f, 0.58f, 1.6, 0.9f),
                         emulsion_row(3.5f, 650.0, 40.0, 0.85, 0.42, 0.24, 0.21f, 650.0, 32.0, 1.25, true, 1.9f, 0.34f, 2.4, 0.94f),
                         absorber_row(ANTIHALATION, 2.0f, 650.0, 80.0, 0.25)},
                        {{0.03f, 0.02f, 0.09f, 0.04f, 0.07f, 0.03f}, {0.02f, 0.02f, 0.04f, 0.02f, 0.04f, 0.02f}, {0.09f, 0.04f, 0.03f, 0.02f, 0.1f, 0.04f}, {0.04f, 0.02f, 0.02f, 0.02f, 0.04f, 0.02f}, {0.07f, 0.03f, 0.1f, 0.04f, 0.03f, 0.02f}, {0.03f, 0.02f, 0.04f, 0.02f, 0.02f, 0.02f}}};
    case 4:  // FujiPro400H (film/stock/fuji_pro_400h.rs:43-271)
        return StockRow{400.0f, 0.28, 0.2, 0.03, 'g', 670.0, 50.0, 0.05,
                        2.5f, 65.0f, 6.5f, 0.32f, 14.0f, false,
                        {overcoat_row(),
                         emulsion_row(2.5f, 445.0, 35.0, 1.0, 0.82, 0.33, 0.17f, 445.0, 40.0, 1.0, true, 1.1f, 0.56f, 4.5, 0.86f),
                         emulsion_row(2.5f, 445.0, 35.0, 0.8, 0.4, 0.28, 0.19f, 445.0, 40.0, 1.0, true, 1.1f, 0.56f, 2.1, 0.9f),
                         absorber_row(FILTER, 2.0f, 430.0, 40.0, 1.3),
                         emulsion_row(2.0f, 490.0, 30.0, 0.9, 0.5, 0.3, 0.15f, 650.0, 45.0, 0.6, true, 0.5f, 0.56f, 2.0, 0.88f),
                         emulsion_row(3.0f, 545.0, 40.0, 1.0, 0.88, 0.34, 0.17f, 545.0, 40.0, 1.0, true, 1.1f, 0.56f, 2.3, 0.87f),
                         emulsion_row(3.0f, 545.0, 40.0, 0.8, 0.44, 0.28, 0.19f, 545.0, 40.0, 1.0, true, 1.1f, 0.56f, 1.1, 0.91f),
                         emulsion_row(3.5f, 650.0, 45.0, 1.0, 0.92, 0.34, 0.17f, 650.0, 45.0, 1.0, true, 1.1f, 0.56f, 1.4, 0.89f),
                         emulsion_row(3.5f, 650.0, 45.0, 0.8, 0.46, 0.28, 0.19f, 650.0, 45.0, 1.0, true, 1.1f, 0.56f, 0.7, 0.93f),
                         absorber_row(ANTIHALATION, 2.0f, 650.0, 80.0, 0.3)},
                        {{0.02f, 0.01f, 0.03f, 0.04f, 0.02f, 0.03f, 0.01f}, {0.01f, 0.01f, 0.02f, 0.02f, 0.01f, 0.02f, 0.01f}, {0.03f, 0.02f, 0.02f, 0.06f, 0.03f, 0.04f, 0.02f}, {0.04f, 0.02f, 0.05f, 0.02f, 0.01f, 0.05f, 0.02f}, {0.02f, 0.01f, 0.02f, 0.01f, 0.01f, 0.02f, 0.01f}, {0.03f, 0.01f, 0.04f, 0.05f, 0.02f, 0.02f, 0.01f}, {0.01f, 0.01f, 0.02f, 0.02f, 0.01f, 0.01f, 0.01f}}};
    case 5:  // EktachromeE100 (film/stock/ektachrome_e100.rs:28-157)
        return StockRow{100.0f, 0.0, 0.0, 0.0, 'g', 660.0, 40.0, 0.02,
                        1.5f, 40.0f, 4.0f, 0.4f, 8.0f, true,
                        {overcoat_row(),
                         emulsion_row(4.0f, 440.0, 30.0, 1.0, 0.42, 0.25, 0.22f, 440.0, 35.0, 1.0, false, 3.2f, 1.65f, 3.5, 0.93f),
                         absorber_row(FILTER, 2.0f, 430.0, 35.0, 1.4),
                         emulsion_row(4.0f, 545.0, 35.0, 1.0, 0.45, 0.25, 0.22f, 545.0, 35.0, 1.0, false, 3.2f, 1.65f, 1.8, 0.94f),
                         emulsion_row(5.0f, 650.0, 40.0, 1.0, 0.5, 0.26, 0.22f, 650.0, 40.0, 1.0, false, 3.2f, 1.65f, 1.1, 0.95f),
                         absorber_row(ANTIHALATION, 2.0f, 650.0, 80.0, 0.3)},
                        {{0.01f, 0.02f, 0.01f}, {0.02f, 0.01f, 0.02f}, {0.01f, 0.02f, 0.01f}}};
    case 6:  // TriX400 (film/stock/trix_400.rs:30-91)
        return StockRow{400.0f, 0.0, 0.0, 0.0, 'c', 0.01, 0.0, 0.0,
                        3.5f, 50.0f, 6.0f, 0.35f, 12.0f, false,
                        {LayerRow{EMULSION, 6.0f, 'p', 0.35, 0.65, 0, 0.95, 0.38, 0.22f, 'c', 1.0, 0, 0, false, 1.5f, 0.70f, 2.2, 0.85f},
                         LayerRow{EMULSION, 6.0f, 'p', 0.35, 0.65, 0, 0.45, 0.28, 0.24f, 'c', 1.0, 0, 0, false, 1.5f, 0.70f, 0.9, 0.89f}},
                        {{0.03f, 0.02f}, {0.02f, 0.02f}}};
    default:
        return StockRow{};
    }
}

double integrate_cmf16(const double* s, const double* cmf) {
    double acc = 0.0;
    for (int i = 0; i < NB16 - 1; i++) acc += 0.5 * (s[i] * cmf[i] + s[i + 1] * cmf[i + 1]) * 20.0;
    return acc;
}

void spectrum_to_ap1_16(const double* s, double out[3]) {
    double xyz[3] = {integrate_cmf16(s, CMF16[0]), integrate_cmf16(s, CMF16[1]), integrate_cmf16(s, CMF16[2])};
    for (int i = 0; i < 3; i++) out[i] = XYZ2AP1[i][0] * xyz[0] + XYZ2AP1[i][1] * xyz[1] + XYZ2AP1[i][2] * xyz[2];
}

// E_s[exp(-k s^2 phi)] (capture.rs:91-106)
double expected_survival(double mu, double sig, double k, double phi) {
    const int N = 64;
    const double ZMAX = 8.0;
    double dz = (2.0 * ZMAX) / (double)N;
    double isq = 1.0 / std::sqrt(2.0 * PI);
    double acc = 0.0;
    for (int i = 0; i <= N; i++) {
        double z = -ZMAX + (double)i * dz;
        double tw = (i == 0 || i == N) ? 0.5 : 1.0;
        double pdf = isq * std::exp(-0.5 * z * z);
        double s = std::exp(mu + sig * z);
        double g = std::exp(-k * s * s * phi);
        acc += tw * pdf * g * dz;
    }
    return acc;
}

double curve_integrate(const std::vector<double>& s) {
    double acc = 0.0;
    for (int i = 0; i < NB16 - 1; i++) acc += 0.5 * (s[i] + s[i + 1]) * 20.0;
    return acc;
}

double curve_eval(const std::vector<double>& s, double lam) {
    if (lam <= lam16(0)) return s[0];
    if (lam >= lam16(NB16 - 1)) return s[NB16 - 1];
    for (int i = 0; i < NB16 - 1; i++)
        if (lam >= lam16(i) && lam <= lam16(i + 1)) {
            double t = (lam - lam16(i)) / (lam16(i + 1) - lam16(i));
            return s[i] * (1.0 - t) + s[i + 1] * t;
        }
    return s[NB16 - 1];
}

double curve_peak(const std::vector<double>& s) {
    double mv = -INFINITY, pk = 550.0;
    for (int i = 0; i < NB16; i++)
        if (s[i] > mv) {
            mv = s[i];
            pk = lam16(i);
        }
    return pk;
}

// Upsample basis (upsample.rs:114-158) -> Minv, and the basis samples.
void basis16(double b[3][NB16], double minv[3][3]) {
    const double peaks[3] = {450.0, 550.0, 650.0};
    double cols[3][3], m[3][3];
    for (int k = 0; k < 3; k++) {
        for (int i = 0; i < NB16; i++) {
            double d = (lam16(i) - peaks[k]) / 40.0;
            b[k][i] = std::exp(-0.5 * d * d);
        }
        spectrum_to_ap1_16(b[k], cols[k]);
    }
    for (int r = 0; r < 3; r++)
        for (int k = 0; k < 3; k++) m[r][k] = cols[k][r];
    inv3(m, minv);
}

int build_reference(const StockDef& sd, int W, float shutter, Stock* st, float* pitch_out, float frame_mm) {
    // pixel pitch: width_mm * 1000 / W in f32 (types.rs:45-48)
    float pitch = frame_mm * 1000.0f / (float)W;
    *pitch_out = pitch;
    float pm = pitch > 1e-6f ? pitch : 1e-6f;
    if (shutter < 0) shutter = 1.0f / sd.box_iso;

    Stock& S = *st;
    std::memset(&S, 0, sizeof(S));
    S.model = MODEL_REFERENCE;
    ExposeSpec& X = S.expose;
    RefSpec& R = S.ref;

    double b[3][NB16], minv[3][3];
    basis16(b, minv);
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) X.minv[r * 3 + c] = (float)minv[r][c];

    // absorbed fraction per emulsion and bin for unit incident fluence:
    // product of the transmittances above times (1 - own transmittance)
    std::vector<int> em;
    std::vector<std::vector<double>> frac;
    std::vector<double> phi(NB16, 1.0);
    for (size_t li = 0; li < sd.layers.size(); li++) {
        const Layer& L = sd.layers[li];
        std::vector<double> ab(NB16, 0.0);
        if (L.kind == EMULSION) {
            for (int i = 0; i < NB16; i++) {
                double od = L.sens[i] * 2.0 * (double)L.fraction * (double)L.thickness;
                double pt = phi[i] * std::exp(-od);
                ab[i] = phi[i] - pt;
                phi[i] = pt;
            }
            em.push_back((int)li);
            frac.push_back(ab);
        } else if (L.kind != SUPPORT && !L.sens.empty()) {
            for (int i = 0; i < NB16; i++) {
                double od = L.sens[i] * (double)L.thickness;
                phi[i] = phi[i] * std::exp(-od);
            }
        }
    }
    const int E = (int)em.size();
    if (E < 1 || E > MAXE) return fail(IMOPS_ERR_INVALID_STOCK, "stock must have 1..8 emulsion layers");
    X.E = E;
    R.E = E;
    // band-mean weights: trapezoid over 20 nm, divided by the 300 nm span
    for (int k = 0; k < 3; k++)
        for (int e = 0; e < E; e++) {
            double acc = 0.0;
            for (int i = 0; i < NB16; i++) {
                double w = (i == 0 || i == NB16 - 1) ? 10.0 : 20.0;
                acc += w * b[k][i] * (lam16(i) / 550.0) * frac[e][i];
            }
            X.A[k][e] = (float)(acc / 300.0);
        }

    // spatial effects
    R.sigma_local = std::fmax(sd.psf_local / pm, 0.0f);
    R.local_mix = 0.18f;
    R.sigma_wide = std::fmax(sd.psf_halation / pm, 0.0f);
    {
        const double bands[4] = {450.0, 550.0, 650.0, 700.0};
        float maxr = 0.0f;
        for (double bl : bands) maxr = std::fmax(maxr, (float)curve_eval(sd.refl, bl));
        if (maxr <= 0.0f) R.sigma_wide = 0.0f;
        const float bw[3] = {0.20f, 0.45f, 1.0f};
        for (int e = 0; e < E; e++) {
            const Layer& L = sd.layers[em[e]];
            double pk = curve_peak(L.sens);
            float w;
            if (pk <= 450.0) w = bw[0];
            else if (pk <= 550.0) w = bw[0] + (bw[1] - bw[0]) * (float)((pk - 450.0) / 100.0);
            else if (pk <= 650.0) w = bw[1] + (bw[2] - bw[1]) * (float)((pk - 550.0) / 100.0);
            else w = bw[2];
            double norm = curve_integrate(L.sens);
            float re;
            if (norm <= 1e-9) {
                re = (float)curve_eval(sd.refl, 650.0);
            } else {
                std::vector<double> prod(NB16);
                for (int i = 0; i < NB16; i++) prod[i] = sd.refl[i] * L.sens[i];
                re = (float)(curve_integrate(prod) / norm);
            }
            float gain = re * w;
            R.hal_gain[e] = gain > 0.0f ? gain : 0.0f;
        }
    }
    // capture LUT + reciprocity + development constants
    R.any_reversal = 0;
    for (int e = 0; e < E; e++) {
        const Layer& L = sd.layers[em[e]];
        double p = (double)L.recip_p, t = (double)shutter;
        double eta = (t <= 1.0 || p >= 0.9999) ? 1.0 : std::pow(t > 1.0 ? t : 1.0, p - 1.0);
        R.eta[e] = (float)eta;
        for (int i = 0; i < LUTN; i++) {
            double tt = (double)i / 63.0;
            double lp = -4.0 + tt * (8.0 - -4.0);
            double ph = std::pow(10.0, lp);
            double f = 1.0 - expected_survival(L.mu_ln, L.sigma_ln, L.capture_k, ph);
            f = f < 0.0 ? 0.0 : (f > 1.0 ? 1.0 : f);
            R.lut_log[e][i] = (float)lp;
            R.lut_frac[e][i] = (float)f;
        }
        R.dmax[e] = L.dmax;
        float gam = L.gamma > 1e-6f ? L.gamma : 1e-6f;
        R.inv_gamma[e] = 1.0f / gam;
        R.has_mask[e] = !L.mask_eps.empty();
        R.mask_scale[e] = L.dmax * 0.4f;
        R.reversal[e] = L.reversal;
        R.any_reversal |= L.reversal;
        double mean_s = std::exp(L.mu_ln + 0.5 * L.sigma_ln * L.sigma_ln);
        double r = mean_s * 0.5;
        if (r < 1e-6) r = 1e-6;
        double vol = FRAC_PI_3 * 4.0 * r * r * r;
        double rho = (double)L.fraction * (double)L.thickness / (vol > 1e-18 ? vol : 1e-18);
        float kappa_ref = (float)(1.0 / std::sqrt(rho));
        R.kappa[e] = (kappa_ref / pm) * 0.15f;
    }
    R.sigma_dir = sd.dir_diff / pm;
    R.dir_any = 0;
    for (int i = 0; i < E; i++)
        for (int j = 0; j < E; j++) {
            float w = (i < (int)sd.dir.size() && j < (int)sd.dir[i].size()) ? sd.dir[i][j] : 0.0f;
            R.dir[i][j] = std::fabs(w) > 1e-6f ? w : 0.0f;
            R.dir_any |= std::fabs(w) > 1e-6f;
        }
    R.sigma_adj = sd.dev_diff / pm;
    R.beta = sd.adj_beta;
    R.sigma_grain = 3.0f / pm;
    R.box_iso = sd.box_iso;

    // scan constants and the film-base (Dmin) normalisation
    ScanSpec16& C = S.scan16;
    C.E = E;
    for (int e = 0; e < E; e++) {
        const Layer& L = sd.layers[em[e]];
        for (int i = 0; i < NB16; i++) {
            C.eps[e][i] = (float)(L.eps[i] * LOG2_10);
            C.meps[e][i] = L.mask_eps.empty() ? 0.0f : (float)(L.mask_eps[i] * LOG2_10);
        }
    }
    double dmin[3];
    {
        double d[NB16] = {0};
        for (int e = 0; e < E; e++) {
            const Layer& L = sd.layers[em[e]];
            double m = L.mask_eps.empty() ? 0.0 : (double)(L.dmax * 0.4f);
            for (int i = 0; i < NB16; i++) d[i] += 0.0 * L.eps[i] + (L.mask_eps.empty() ? 0.0 : m * L.mask_eps[i]);
        }
        double t[NB16];
        for (int i = 0; i < NB16; i++) t[i] = std::pow(10.0, -d[i]) * sd.scanner[i];
        spectrum_to_ap1_16(t, dmin);
    }
    double peak = std::fmax(std::fmax(dmin[0], dmin[1]), dmin[2]);
    if (peak < 1e-12) peak = 1e-12;
    for (int c = 0; c < 3; c++) R.dmin_norm[c] = (float)(dmin[c] / peak);
    for (int i = 0; i < NB16; i++) {
        double w = (i == 0 || i == NB16 - 1) ? 10.0 : 20.0;
        for (int c = 0; c < 3; c++) {
            double acc = 0.0;
            for (int j = 0; j < 3; j++) acc += XYZ2AP1[c][j] * CMF16[j][i];
            C.C[i][c] = (float)(acc * w * sd.scanner[i] / peak);
        }
    }
    return IMOPS_OK;
}

// ---- baseline preset -------------------------------------------------------

// CIE 1931 2-degree observer: multi-lobe Gaussian fit of Wyman, Sloan and
// Shirley, "Simple Analytic Approximations to the CIE XYZ Color Matching
// Functions", JCGT 2(2), 2013.
double lobe(double x, double mu, double s1, double s2) {
    double t = (x - mu) / (x < mu ? s1 : s2);
    return std::exp(-0.5 * t * t);
}

void cmf81(double x[NB81], double y[NB81], double z[NB81]) {
    for (int i = 0; i < NB81; i++) {
        double l = 380.0 + 5.0 * i;
        x[i] = 1.056 * lobe(l, 599.8, 37.9, 31.0) + 0.362 * lobe(l, 442.0, 16.0, 26.7) - 0.065 * lobe(l, 501.1, 20.4, 26.2);
        y[i] = 0.821 * lobe(l, 568.8, 46.9, 40.5) + 0.286 * lobe(l, 530.9, 16.3, 31.1);
        z[i] = 1.217 * lobe(l, 437.0, 11.8, 36.0) + 0.681 * lobe(l, 459.0, 26.0, 13.8);
    }
}

int build_baseline(const ImopsBaselineFilm& P, Stock* st) {
    Stock& S = *st;
    std::memset(&S, 0, sizeof(S));
    S.model = MODEL_BASELINE;
    double xb[NB81], yb[NB81], zb[NB81], lam[NB81], trap[NB81];
    cmf81(xb, yb, zb);
    for (int i = 0; i < NB81; i++) {
        lam[i] = 380.0 + 5.0 * i;
        trap[i] = (i == 0 || i == NB81 - 1) ? 2.5 : 5.0;
    }
    const double speak[3] = {450.0, 550.0, 650.0}, ssig[3] = {35.0, 40.0, 45.0};
    const double dpeak[3] = {450.0, 550.0, 650.0}, dsig[3] = {40.0, 40.0, 45.0};
    double basis[3][NB81], cols[3][3];
    for (int k = 0; k < 3; k++) {
        double X = 0, Y = 0, Z = 0;
        for (int i = 0; i < NB81; i++) {
            double d = (lam[i] - speak[k]) / 40.0;
            basis[k][i] = std::exp(-0.5 * d * d);
            X += trap[i] * basis[k][i] * xb[i];
            Y += trap[i] * basis[k][i] * yb[i];
            Z += trap[i] * basis[k][i] * zb[i];
        }
        for (int c = 0; c < 3; c++) cols[k][c] = XYZ2AP1[c][0] * X + XYZ2AP1[c][1] * Y + XYZ2AP1[c][2] * Z;
    }
    double m[3][3], minv[3][3];
    for (int r = 0; r < 3; r++)
        for (int k = 0; k < 3; k++) m[r][k] = cols[k][r];
    inv3(m, minv);
    ExposeSpec& X = S.expose;
    X.E = 3;
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) X.minv[r * 3 + c] = (float)minv[r][c];
    double w1[3];
    for (int k = 0; k < 3; k++) w1[k] = std::fmax(0.0, minv[k][0] + minv[k][1] + minv[k][2]);
    for (int e = 0; e < 3; e++) {
        double sens[NB81], nrm = 0;
        for (int i = 0; i < NB81; i++) {
            double d = (lam[i] - speak[e]) / ssig[e];
            sens[i] = std::exp(-0.5 * d * d);
            double s1 = w1[0] * basis[0][i] + w1[1] * basis[1][i] + w1[2] * basis[2][i];
            nrm += trap[i] * s1 * sens[i];
        }
        for (int k = 0; k < 3; k++) {
            double acc = 0;
            for (int i = 0; i < NB81; i++) acc += trap[i] * basis[k][i] * sens[i];
            X.A[k][e] = (float)(acc / nrm);
        }
    }
    X.hal_src = 1;
    X.hal_threshold = P.hal_threshold;
    BaselineSpec& B = S.base;
    const float bleed[3] = {0.20f, 0.45f, 1.0f};
    for (int e = 0; e < 3; e++) {
        B.dmax[e] = P.dmax[e];
        B.k[e] = P.k[e];
        B.x0[e] = P.x0[e];
        B.bleed[e] = bleed[e];
    }
    B.hal_strength = P.hal_strength;
    B.grain_sigma = P.grain_on ? P.grain_sigma : 0.0f;
    S.grain_blur = P.grain_blur;
    double white[3];
    {
        double Xw = 0, Yw = 0, Zw = 0;
        for (int i = 0; i < NB81; i++) {
            Xw += trap[i] * xb[i];
            Yw += trap[i] * yb[i];
            Zw += trap[i] * zb[i];
        }
        for (int c = 0; c < 3; c++) white[c] = XYZ2AP1[c][0] * Xw + XYZ2AP1[c][1] * Yw + XYZ2AP1[c][2] * Zw;
    }
    double peak = std::fmax(std::fmax(white[0], white[1]), white[2]);
    for (int i = 0; i < NB81; i++) {
        for (int e = 0; e < 3; e++) {
            double d = (lam[i] - dpeak[e]) / dsig[e];
            S.scan81.eps[e][i] = (float)(std::exp(-0.5 * d * d) * LOG2_10);
        }
        for (int c = 0; c < 3; c++) {
            double acc = XYZ2AP1[c][0] * xb[i] + XYZ2AP1[c][1] * yb[i] + XYZ2AP1[c][2] * zb[i];
            S.scan81.C[i][c] = (float)(acc * trap[i] / peak);
        }
    }
    // halation taps: fixed radius, Gaussian of sigma, normalised in f32
    int R = P.hal_radius;
    if (R < 1 || R > HAL_R) return fail(IMOPS_ERR_INVALID_ARGUMENT, "baseline film: hal_radius must be 1..64");
    float inv = 1.0f / (2.0f * P.hal_sigma * P.hal_sigma), sum = 0.0f;
    for (int i = 0; i < 2 * HAL_R + 1; i++) S.hal_taps[i] = 0.0f;
    for (int i = 0; i < 2 * R + 1; i++) {
        float x = (float)i - (float)R;
        float v = std::exp(-x * x * inv);
        S.hal_taps[HAL_R - R + i] = v;
        sum += v;
    }
    for (int i = 0; i < 2 * HAL_R + 1; i++) S.hal_taps[i] /= sum;
    return IMOPS_OK;
}

}  // namespace

int gaussian_taps(float sigma, float* taps, int max_taps) {
    float r3 = std::ceil(3.0f * sigma);
    if (r3 < 1.0f) r3 = 1.0f;
    int radius = (int)r3;
    if (2 * radius + 1 > max_taps) return -1;
    float inv = 1.0f / (2.0f * sigma * sigma);
    float sum = 0.0f;
    for (int i = 0; i < 2 * radius + 1; i++) {
        float x = (float)i - (float)radius;
        float v = std::exp(-x * x * inv);
        taps[i] = v;
        sum += v;
    }
    for (int i = 0; i < 2 * radius + 1; i++) taps[i] /= sum;
    return radius;
}

float relative_to_absolute_y(float y, float box_iso) {
    float s = box_iso > 1.0f ? box_iso : 1.0f;
    float t = 1.0f / s;
    double l = 12.5 * (double)y * (8.0 * 8.0) / ((double)t * (double)s);
    return (float)l;
}

int build_stock(int stock_id, int film_format, int W, float shutter_seconds, const ImopsBaselineFilm* baseline,
                Stock* out, float* pitch_um) {
    static const float frames[3] = {36.0f, 56.0f, 101.6f};
    if (stock_id == IMOPS_STOCK_BASELINE81) {
        ImopsBaselineFilm d;
        imops_baseline_film_defaults(&d);
        *pitch_um = 0.0f;
        return build_baseline(baseline ? *baseline : d, out);
    }
    if (film_format < 0 || film_format > 2) return fail(IMOPS_ERR_INVALID_ARGUMENT, "unknown film format");
    if (stock_id < IMOPS_STOCK_BWSTUB || stock_id > IMOPS_STOCK_TRIX400)
        return fail(IMOPS_ERR_INVALID_STOCK, "unknown film stock id");
    StockDef sd = from_rows(stock_row(stock_id));
    return build_reference(sd, W, shutter_seconds, out, pitch_um, frames[film_format]);
}

}  // namespace film
}  // namespace imops

extern "C" void imops_baseline_film_defaults(ImopsBaselineFilm* p) {
    if (!p) return;
    const float dmax[3] = {2.0f, 2.1f, 2.2f}, k[3] = {2.3f, 2.5f, 2.7f}, x0[3] = {-0.70f, -0.73f, -0.76f};
    for (int i = 0; i < 3; i++) {
        p->dmax[i] = dmax[i];
        p->k[i] = k[i];
        p->x0[i] = x0[i];
    }
    p->hal_strength = 0.15f;
    p->hal_sigma = 20.0f;
    p->hal_radius = 64;
    p->hal_threshold = 0.8f;
    p->grain_sigma = 0.02f;
    p->grain_blur = 1.0f;
    p->grain_on = 1;
    p->seed = 1;
    p->scan = IMOPS_SCAN_FP32;
}
