// common.cuh -- shared helpers of the imops_b200 CUDA library: status codes,
// the thread-local last-error string, CUDA checks and the CFA descriptor
// handed to kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "imops_b200.h"

namespace imops {

// Thread-local last error (the reference keeps one in LAST_ERROR,
// pichromatic-pipeline/src/extern_pipeline.rs:18-38).
void set_error(const std::string& msg);
void clear_error();
const char* last_error();

// Returns `code` after recording `msg`.
int fail(int code, const std::string& msg);

// Converts a CUDA error into IMOPS_ERR_CUDA (or OK).
int cuda_status(cudaError_t e, const char* what);

#define IMOPS_CUDA_TRY(call, what)                                  \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return ::imops::cuda_status(_e, what); \
    } while (0)

// Device-side CFA period (up to 12x12 cells, colour 0=R 1=G 2=B).
struct CfaDev {
    int pw, ph;
    uint8_t col[144];
    __host__ __device__ __forceinline__ int at(int r, int c) const {
        int rr = r % ph;
        if (rr < 0) rr += ph;
        int cc = c % pw;
        if (cc < 0) cc += pw;
        return col[rr * pw + cc];
    }
};

// A CFA whose period is known at compile time, for non-negative
// coordinates, for kernels that look colours up many times per pixel: the
// modulo is by a constant (a multiply-high) instead of a runtime integer
// division, and the colours are 3-bit codes packed into two 64-bit words
// (cells 0..20 and 21..41), read with shifts: no array is indexed at run
// time, so nothing goes through local or parameter-space loads.  Same
// colours as CfaDev::at.
template <int PW, int PH>
struct CfaFixed {
    static_assert(PW * PH <= 42, "at most 42 cells in two 64-bit words");
    unsigned long long lo, hi;
    __device__ __forceinline__ int at(int r, int c) const {
        const int k = (int)(((unsigned)r % PH) * PW + (unsigned)c % PW);
        return (int)((k < 21 ? lo >> (3 * k) : hi >> (3 * (k - 21))) & 7ull);
    }
    static CfaFixed from(const CfaDev& d) {
        CfaFixed f;
        f.lo = f.hi = 0ull;
        for (int i = 0; i < PW * PH; i++) {
            const unsigned long long v = (unsigned long long)(d.col[i] & 7);
            if (i < 21) f.lo |= v << (3 * i);
            else f.hi |= v << (3 * (i - 21));
        }
        return f;
    }
};

// Parses a CFA pattern string the way CFA::new does (cfa.rs:98-129) and
// applies CFA::shift (cfa.rs:204-233).  Returns IMOPS_OK or an error code.
int parse_cfa(const char* pattern, int shift_x, int shift_y, CfaDev* out);

// Whether a CFA is a 2x2 Bayer period with greens on one diagonal.
bool cfa_is_bayer(const CfaDev& c);

// Current stream as a cudaStream_t.
inline cudaStream_t as_stream(imops_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// Number of SMs of the current device (cached per device).
int sm_count();

// Launch evidence counter (imops_launch_count).
void note_launch(int n = 1);

// Host-side fault injection for failure-path tests: when the environment
// variable IMOPS_FAULT_INJECT names `site` ("alloc", "launch"), the call
// reports a failure instead of touching the GPU.
bool fault_injected(const char* site);

// A device buffer per (device, stream), grown on demand: the working sets of
// the film, adjoint, X-Trans and fused-develop paths.  Growing waits for the
// stream, frees the old buffer and allocates the new one.  Every cache
// registers itself, so imops_release_working_sets can free them all.
class StreamCache {
   public:
    explicit StreamCache(const char* what);
    // The buffer of the current device and stream s, at least `bytes` long
    // (fault site "alloc").
    int get(cudaStream_t s, size_t bytes, void** out);
    // Frees every buffer of device `dev`; its work must have finished.
    void release_device(int dev);

   private:
    struct E {
        int dev;
        cudaStream_t s;
        void* p;
        size_t bytes;
    };
    const char* what_;
    std::mutex mu_;
    std::vector<E> v_;
};

// Frees the working sets of every cache on device `dev` (after waiting for it).
int release_working_sets(int dev);

}  // namespace imops
