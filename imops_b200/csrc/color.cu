// color.cu -- per-pixel colour stages: u16 black/white scaling + crop,
// white balance, exposure, BaselineExposureCompensation and camera CST.
//
// All are HBM-bound streams over interleaved RGB (12 B in + 12 B out per
// pixel, or 2 B in + 4 B out for the scaling); kernels use a grid-stride
// loop sized to a few waves of the SM count and read/write the RGB triple
// as three floats per thread (consecutive threads touch consecutive 12-byte
// records, so each warp instruction is a contiguous 384-byte span).
// Built with --fmad=false: each step is the reference's own f32 arithmetic.
#include "color.cuh"

#include <cmath>

namespace imops {
namespace color {

void camera_forward_matrix(const float calib[9], float fwd[9]) {
    const float xyz[3] = {0.95042f, 1.0f, 1.08890f};
    float rgbd65[3], mult[3] = {1.0f, 1.0f, 1.0f};
    float m[3][3];
    for (int i = 0; i < 3; i++) rgbd65[i] = calib[i * 3] * xyz[0] + calib[i * 3 + 1] * xyz[1] + calib[i * 3 + 2] * xyz[2];
    for (int i = 0; i < 3; i++)
        if (rgbd65[i] > 0.0f) mult[i] = 1.0f / rgbd65[i];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) m[i][j] = calib[i * 3 + j] * mult[i];
    // pseudo-inverse by Gauss-Jordan on [M^T M | I] (cst.rs:51-95)
    float work[3][6], tmp[3][3];
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 6; j++) work[i][j] = (j == i + 3) ? 1.0f : 0.0f;
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) work[i][j] += m[k][i] * m[k][j];
    }
    for (int i = 0; i < 3; i++) {
        float num = work[i][i];
        for (int j = 0; j < 6; j++) work[i][j] /= num;
        for (int k = 0; k < 3; k++) {
            if (k == i) continue;
            num = work[k][i];
            for (int j = 0; j < 6; j++) work[k][j] -= work[i][j] * num;
        }
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            tmp[i][j] = 0.0f;
            for (int k = 0; k < 3; k++) tmp[i][j] += work[j][k + 3] * m[i][k];
        }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) fwd[i * 3 + j] = tmp[j][i];
}

bool xyz_to_target(int target, float m[9]) {
    static const double lsrgb[9] = {12831.0 / 3959.0,     -329.0 / 214.0,       -1974.0 / 3959.0,
                                    -851781.0 / 878810.0, 1648619.0 / 878810.0, 36519.0 / 878810.0,
                                    705.0 / 12673.0,      -2585.0 / 12673.0,    705.0 / 667.0};
    static const double ap1[9] = {1.6410233797, -0.3248032942, -0.2364246952, -0.6636628587, 1.6153315917,
                                  0.0167563477, 0.0117218943,  -0.0082844165, 0.9883948585};
    const double* src = nullptr;
    if (target == IMOPS_CS_XYZD65) {
        for (int i = 0; i < 9; i++) m[i] = (i % 4 == 0) ? 1.0f : 0.0f;
        return true;
    }
    if (target == IMOPS_CS_LINEAR_SRGB || target == IMOPS_CS_SRGB) src = lsrgb;
    if (target == IMOPS_CS_ACESCG) src = ap1;
    if (!src) return false;
    for (int i = 0; i < 9; i++) m[i] = (float)src[i];
    return true;
}

bool to_xyz(int space, float m[9]) {
    static const double lsrgb[9] = {506752.0 / 1228815.0, 87881.0 / 245763.0,  12673.0 / 70218.0,
                                    87098.0 / 409605.0,   175762.0 / 245763.0, 12673.0 / 175545.0,
                                    7918.0 / 409605.0,    87881.0 / 737289.0,  1001167.0 / 1053270.0};
    static const double ap1[9] = {0.6624541811,  0.1340042065, 0.1561876870, 0.2722287168, 0.6740817658,
                                  0.0536895174, -0.0055746495, 0.0040607335, 1.0103391003};
    const double* src = nullptr;
    if (space == IMOPS_CS_XYZD65) {
        for (int i = 0; i < 9; i++) m[i] = (i % 4 == 0) ? 1.0f : 0.0f;
        return true;
    }
    if (space == IMOPS_CS_LINEAR_SRGB || space == IMOPS_CS_SRGB) src = lsrgb;
    if (space == IMOPS_CS_ACESCG) src = ap1;
    if (!src) return false;
    for (int i = 0; i < 9; i++) m[i] = (float)src[i];
    return true;
}

float exp_value(float ev) { return powf(2.0f, ev); }

float luminance_gain(float shutter, float f_number, float iso) {
    double g = 12.5 * 1.0 * ((double)f_number * (double)f_number) / ((double)shutter * (double)iso);
    return (float)g;
}

Epilogue identity_epilogue() {
    Epilogue e;
    e.wb[0] = e.wb[1] = e.wb[2] = 1.0f;
    e.n_gain = 0;
    e.gain[0] = e.gain[1] = e.gain[2] = e.gain[3] = 1.0f;
    e.do_cst = 0;
    for (int i = 0; i < 9; i++) e.fwd[i] = e.tgt[i] = (i % 4 == 0) ? 1.0f : 0.0f;
    e.srgb = 0;
    e.src_srgb = 0;
    return e;
}

struct Levels {
    float v[288];
};

// One thread per column, SCALE_ROWS rows: the CFA site's column is found
// once and its row stepped, the levels are read from shared memory.  A full
// group of rows issues all its loads before the first division, so a thread
// keeps SCALE_ROWS loads in flight.
constexpr int SCALE_ROWS = 16;

__global__ void scale_u16_kernel(const uint16_t* __restrict__ raw, int raw_w, int cx, int cy, int cw, int ch, int pw,
                                 int ph, const __grid_constant__ Levels lv, float* __restrict__ out) {
    __shared__ float sl[288];
    for (int i = threadIdx.x; i < pw * ph; i += blockDim.x) {
        sl[i] = lv.v[i];
        sl[144 + i] = lv.v[144 + i];
    }
    __syncthreads();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y0 = blockIdx.y * SCALE_ROWS;
    if (x >= cw) return;
    const int sx = cx + x, col = sx % pw;
    int rowph = (cy + y0) % ph;
    const uint16_t* src = raw + (size_t)(cy + y0) * raw_w + sx;
    float* dst = out + (size_t)y0 * cw + x;
    const int rows = ch - y0 < SCALE_ROWS ? ch - y0 : SCALE_ROWS;
    if (rows == SCALE_ROWS) {
        float v[SCALE_ROWS];
#pragma unroll
        for (int r = 0; r < SCALE_ROWS; r++) v[r] = (float)__ldg(src + (size_t)r * raw_w);
#pragma unroll
        for (int r = 0; r < SCALE_ROWS; r++) {
            const int site = rowph * pw + col;
            const float bl = sl[site], wh = sl[144 + site];
            dst[(size_t)r * cw] = (v[r] - bl) / (wh - bl);
            rowph = rowph + 1 == ph ? 0 : rowph + 1;
        }
        return;
    }
    for (int r = 0; r < rows; r++) {
        const int site = rowph * pw + col;
        const float v = (float)__ldg(src + (size_t)r * raw_w);
        const float bl = sl[site], wh = sl[144 + site];
        dst[(size_t)r * cw] = (v - bl) / (wh - bl);
        rowph = rowph + 1 == ph ? 0 : rowph + 1;
    }
}

__global__ void epilogue_kernel(float* __restrict__ rgb, size_t n, Epilogue e) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        float* p = rgb + 3 * k;
        float r = p[0], g = p[1], b = p[2];
        e.apply(r, g, b);
        p[0] = r;
        p[1] = g;
        p[2] = b;
    }
}

int stream_grid(size_t n, int block) {
    size_t want = (n + block - 1) / block;
    size_t cap = (size_t)sm_count() * 8;
    if (want > cap) want = cap;
    if (want < 1) want = 1;
    return (int)want;
}

int run_epilogue(float* rgb, size_t n, const Epilogue& e, cudaStream_t s, const char* what) {
    if (!rgb && n) return fail(IMOPS_ERR_INVALID_ARGUMENT, std::string(what) + ": NULL buffer");
    if (n == 0) return IMOPS_OK;
    if (fault_injected("launch")) return fail(IMOPS_ERR_CUDA, std::string("injected launch failure (") + what + ")");
    epilogue_kernel<<<stream_grid(n, 256), 256, 0, s>>>(rgb, n, e);
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), what);
    return IMOPS_OK;
}

}  // namespace color
}  // namespace imops

using namespace imops;

extern "C" int imops_scale_u16(const uint16_t* raw, int raw_w, int raw_h, int crop_x, int crop_y, int crop_w,
                               int crop_h, const float* black, const float* white, int period_w, int period_h,
                               float* out, imops_stream_t stream) {
    clear_error();
    if (!raw || !out || !black || !white) return fail(IMOPS_ERR_INVALID_ARGUMENT, "scale_u16: NULL buffer");
    if (period_w <= 0 || period_h <= 0 || period_w * period_h > 144)
        return fail(IMOPS_ERR_INVALID_ARGUMENT, "scale_u16: CFA period must be 1..144 cells");
    if (crop_x < 0 || crop_y < 0 || crop_w <= 0 || crop_h <= 0 || crop_x + crop_w > raw_w || crop_y + crop_h > raw_h)
        return fail(IMOPS_ERR_INVALID_ARGUMENT, "scale_u16: crop rectangle outside the frame");
    color::Levels lv;
    for (int i = 0; i < period_w * period_h; i++) {
        lv.v[i] = black[i];
        lv.v[144 + i] = white[i];
    }
    dim3 grid((crop_w + 255) / 256, (crop_h + color::SCALE_ROWS - 1) / color::SCALE_ROWS);
    color::scale_u16_kernel<<<grid, 256, 0, as_stream(stream)>>>(raw, raw_w, crop_x, crop_y, crop_w, crop_h,
                                                                  period_w, period_h, lv, out);
    note_launch();
    IMOPS_CUDA_TRY(cudaGetLastError(), "scale_u16 launch");
    return IMOPS_OK;
}

extern "C" int imops_cfa_coeffs(float* rgb, size_t n_pixels, const float wb[4], imops_stream_t stream) {
    clear_error();
    if (!wb) return fail(IMOPS_ERR_INVALID_ARGUMENT, "cfa_coeffs: NULL coefficients");
    color::Epilogue e = color::identity_epilogue();
    e.wb[0] = wb[0];
    e.wb[1] = wb[1];
    e.wb[2] = wb[2];
    return color::run_epilogue(rgb, n_pixels, e, as_stream(stream), "cfa_coeffs");
}

extern "C" int imops_exp(float* rgb, size_t n_pixels, float ev, imops_stream_t stream) {
    clear_error();
    color::Epilogue e = color::identity_epilogue();
    e.n_gain = 1;
    e.gain[0] = color::exp_value(ev);
    return color::run_epilogue(rgb, n_pixels, e, as_stream(stream), "exp");
}

extern "C" int imops_baseline_exposure(float* rgb, size_t n_pixels, float baseline_ev, float shutter_seconds,
                                       float f_number, float iso, int* applied, imops_stream_t stream) {
    clear_error();
    color::Epilogue e = color::identity_epilogue();
    if (fabsf(baseline_ev) > 1e-6f) e.gain[e.n_gain++] = color::exp_value(baseline_ev);
    bool ok = shutter_seconds > 0.0f && f_number > 0.0f && iso > 0.0f;
    if (ok) e.gain[e.n_gain++] = color::luminance_gain(shutter_seconds, f_number, iso);
    if (applied) *applied = ok ? 1 : 0;
    if (e.n_gain == 0) return IMOPS_OK;
    return color::run_epilogue(rgb, n_pixels, e, as_stream(stream), "baseline_exposure");
}

extern "C" int imops_camera_forward_matrix(const float calib_d65[9], float forward[9]) {
    clear_error();
    if (!calib_d65 || !forward) return fail(IMOPS_ERR_INVALID_ARGUMENT, "camera_forward_matrix: NULL matrix");
    color::camera_forward_matrix(calib_d65, forward);
    return IMOPS_OK;
}

extern "C" int imops_camera_cst(float* rgb, size_t n_pixels, const float calib_d65[9], int target,
                                imops_stream_t stream) {
    clear_error();
    if (!calib_d65) return fail(IMOPS_ERR_INVALID_ARGUMENT, "camera_cst: NULL calibration matrix");
    color::Epilogue e = color::identity_epilogue();
    if (!color::xyz_to_target(target, e.tgt))
        return fail(IMOPS_ERR_INVALID_ARGUMENT, "camera_cst: unsupported target colour space");
    color::camera_forward_matrix(calib_d65, e.fwd);
    e.do_cst = 1;
    e.srgb = target == IMOPS_CS_SRGB;
    return color::run_epilogue(rgb, n_pixels, e, as_stream(stream), "camera_cst");
}
