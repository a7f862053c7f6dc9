// film_noalloc.cu -- the baseline 81-bin film preset for callers that cannot
// allocate device memory.
//
// Who needs it: a host application that hands the GPU a fixed memory budget
// through its own allocator (an editor or viewer embedding this library next
// to its own renderer) must not see the library call cudaMalloc behind its
// back, and a real-time preview loop cannot take the implicit device-wide
// synchronisation that cudaMalloc and cudaFree may cause.  imops_film_process
// keeps the preset's working planes in a per-(device, stream) buffer that it
// allocates on first use and grows with the image; this entry point takes
// them from a fixed array in device memory instead, so it allocates nothing,
// and the caller still passes the image.
#include <mutex>

#include "film.cuh"

namespace {

// Largest image: 2 MP (a 1920 x 1080 preview fits).  The preset needs 16
// bytes a pixel (four f32 planes) plus the grain's block sums (three doubles
// a 128 x 39 tile), which for 2 MP stay below 1.5 MiB at any aspect ratio.
constexpr size_t kMaxPixels = (size_t)1 << 21;
constexpr size_t kScratchBytes = 16 * kMaxPixels + ((size_t)2 << 20);

}  // namespace

// The working set of every call on this GPU, shared by all of them.  On the
// host this name is only a stand-in for the device array (its address there
// is not a device address), so kernels get the address that
// cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) unsigned char g_film_noalloc_scratch[kScratchBytes];

namespace {

std::mutex g_mu;
void* g_addr[64] = {};

// The device address of g_film_noalloc_scratch on the current device, looked
// up once per device (with that device current) and cached.
int scratch_address(void** out) {
    int dev = 0;
    IMOPS_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) return imops::fail(IMOPS_ERR_INVALID_ARGUMENT, "film no-alloc: device index above 63");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_film_noalloc_scratch);
        if (e != cudaSuccess) return imops::cuda_status(e, "cudaGetSymbolAddress(film no-alloc scratch)");
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return IMOPS_OK;
}

}  // namespace

extern "C" size_t imops_film_noalloc_max_pixels(void) { return kMaxPixels; }

extern "C" int imops_film_baseline_noalloc(float* rgb, int w, int h, int color_space,
                                           const ImopsBaselineFilm* baseline, imops_stream_t stream) {
    using namespace imops;
    clear_error();
    if (color_space != IMOPS_CS_ACESCG) return fail(IMOPS_ERR_WRONG_COLOR_SPACE, "wrong color space: expected ACEScg");
    if (w <= 0 || h <= 0 || !rgb) return fail(IMOPS_ERR_INVALID_DIMENSIONS, "invalid image dimensions");
    if ((size_t)w * (size_t)h > kMaxPixels)
        return fail(IMOPS_ERR_UNSUPPORTED_SIZE,
                    "film no-alloc: " + std::to_string(w) + "x" + std::to_string(h) + " is above its fixed working " +
                        "set of " + std::to_string(kMaxPixels) + " pixels; use imops_film_process");
    ImopsBaselineFilm P;
    if (baseline) P = *baseline;
    else imops_baseline_film_defaults(&P);
    film::Stock st;
    int rc = film::baseline_stock(w, P, &st);
    if (rc) return rc;
    if (film::baseline_scratch_bytes(w, h) > kScratchBytes)
        return fail(IMOPS_ERR_UNSUPPORTED_SIZE, "film no-alloc: working set above the fixed array");
    void* scratch = nullptr;
    if ((rc = scratch_address(&scratch))) return rc;
    return film::baseline_forward_in(rgb, w, h, P, st, scratch, as_stream(stream));
}
