// common.cu -- error state, CFA parsing and device queries shared by the
// imops_b200 entry points.
#include "common.cuh"

#include <cstdlib>
#include <cstring>
#include <atomic>
#include <mutex>

namespace imops {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }
const char* last_error() { return g_last_error.c_str(); }

int fail(int code, const std::string& msg) {
    set_error(msg);
    return code;
}

int cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return IMOPS_OK;
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    if (e == cudaErrorMemoryAllocation) return fail(IMOPS_ERR_OUT_OF_MEMORY, m);
    return fail(IMOPS_ERR_CUDA, m);
}

int parse_cfa(const char* pattern, int shift_x, int shift_y, CfaDev* out) {
    if (!pattern) return fail(IMOPS_ERR_INVALID_ARGUMENT, "CFA pattern is NULL");
    size_t n = std::strlen(pattern);
    int pw, ph;
    switch (n) {
        case 4: pw = 2; ph = 2; break;
        case 36: pw = 6; ph = 6; break;
        case 16: pw = 2; ph = 8; break;
        case 144: pw = 12; ph = 12; break;
        default:
            return fail(IMOPS_ERR_UNSUPPORTED_CFA, std::string("Unknown CFA size \"") + pattern + "\"");
    }
    uint8_t base[144];
    for (size_t i = 0; i < n; i++) {
        switch (pattern[i]) {
            case 'R': base[i] = 0; break;
            case 'G': base[i] = 1; break;
            case 'B': base[i] = 2; break;
            case 'E': case 'C': base[i] = 3; break;
            case 'M': base[i] = 4; break;
            case 'Y': base[i] = 5; break;
            default:
                return fail(IMOPS_ERR_UNSUPPORTED_CFA, std::string("Unknown CFA color \"") + pattern[i] + "\"");
        }
    }
    out->pw = pw;
    out->ph = ph;
    for (int r = 0; r < ph; r++)
        for (int c = 0; c < pw; c++) {
            int sr = ((r + shift_y) % ph + ph) % ph;
            int sc = ((c + shift_x) % pw + pw) % pw;
            out->col[r * pw + c] = base[sr * pw + sc];
        }
    return IMOPS_OK;
}

bool cfa_is_bayer(const CfaDev& c) {
    if (c.pw != 2 || c.ph != 2) return false;
    int g = 0, r = 0, b = 0;
    for (int i = 0; i < 4; i++) {
        g += c.col[i] == 1;
        r += c.col[i] == 0;
        b += c.col[i] == 2;
    }
    // greens on one diagonal: (0,0)&(1,1) or (0,1)&(1,0)
    bool diag = (c.col[0] == 1 && c.col[3] == 1) || (c.col[1] == 1 && c.col[2] == 1);
    return g == 2 && r == 1 && b == 1 && diag;
}

int sm_count() {
    static std::mutex mu;
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    std::lock_guard<std::mutex> lock(mu);
    if (cached[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cached[dev] = n;
    }
    return cached[dev];
}

namespace {
std::mutex g_caches_mu;
std::vector<StreamCache*>& caches() {
    static std::vector<StreamCache*> v;
    return v;
}
}  // namespace

StreamCache::StreamCache(const char* what) : what_(what) {
    std::lock_guard<std::mutex> lock(g_caches_mu);
    caches().push_back(this);
}

// Buffers are allocated and replaced in stream order (cudaMallocAsync /
// cudaFreeAsync on s): unlike cudaMalloc, neither waits for the work
// already queued on the device, so the first call on a stream, or a larger
// image, does not stall frames in flight on other streams.  Work on other
// streams that uses the buffer is ordered after s with events.
int StreamCache::get(cudaStream_t s, size_t bytes, void** out) {
    if (fault_injected("alloc")) return fail(IMOPS_ERR_OUT_OF_MEMORY, std::string("injected allocation failure (") + what_ + ")");
    int dev = 0;
    IMOPS_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    const std::string m = std::string("cudaMallocAsync(") + what_ + ")";
    std::lock_guard<std::mutex> lock(mu_);
    for (auto& e : v_)
        if (e.dev == dev && e.s == s) {
            if (e.bytes < bytes) {
                IMOPS_CUDA_TRY(cudaFreeAsync(e.p, s), "cudaFreeAsync");
                e.p = nullptr;
                e.bytes = 0;
                IMOPS_CUDA_TRY(cudaMallocAsync(&e.p, bytes, s), m.c_str());
                e.bytes = bytes;
            }
            *out = e.p;
            return IMOPS_OK;
        }
    void* p = nullptr;
    IMOPS_CUDA_TRY(cudaMallocAsync(&p, bytes, s), m.c_str());
    v_.push_back({dev, s, p, bytes});
    *out = p;
    return IMOPS_OK;
}

void StreamCache::release_device(int dev) {
    std::lock_guard<std::mutex> lock(mu_);
    for (size_t k = 0; k < v_.size();) {
        if (v_[k].dev == dev) {
            if (v_[k].p) cudaFree(v_[k].p);
            v_.erase(v_.begin() + k);
        } else {
            k++;
        }
    }
}

int release_working_sets(int dev) {
    IMOPS_CUDA_TRY(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    std::lock_guard<std::mutex> lock(g_caches_mu);
    for (StreamCache* c : caches()) c->release_device(dev);
    return IMOPS_OK;
}

static std::atomic<uint64_t> g_launches{0};

void note_launch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

bool fault_injected(const char* site) {
    const char* v = std::getenv("IMOPS_FAULT_INJECT");
    if (!v || !*v) return false;
    return std::strstr(v, site) != nullptr;
}

}  // namespace imops

extern "C" const char* imops_last_error(void) { return imops::last_error(); }

extern "C" uint64_t imops_launch_count(void) { return imops::g_launches.load(std::memory_order_relaxed); }

extern "C" const char* imops_version(void) { return "imops_b200 0.1.0 (sm_100a)"; }

extern "C" int imops_release_working_sets(void) {
    imops::clear_error();
    int dev = 0;
    IMOPS_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    return imops::release_working_sets(dev);
}
