// Shared internals of the B200 FDTD library: error state, launch counting,
// vector helpers. Device code targets sm_100a only.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/meep_b200.h"

namespace mtb {

// Last error text, one per host thread (mtb_last_error()).
void set_error(const char *fmt, ...);
int fail(int code, const char *fmt, ...);
void count_launch(int64_t n = 1);

#define MTB_CUDA_TRY(expr)                                                    \
    do {                                                                      \
        cudaError_t e_ = (expr);                                              \
        if (e_ != cudaSuccess)                                                \
            return ::mtb::fail(MTB_CUDA_ERROR, "%s failed: %s (%s:%d)", #expr, \
                               cudaGetErrorString(e_), __FILE__, __LINE__);   \
    } while (0)

#define MTB_CHECK_LAUNCH()                                                    \
    do {                                                                      \
        cudaError_t e_ = cudaGetLastError();                                  \
        if (e_ != cudaSuccess)                                                \
            return ::mtb::fail(MTB_CUDA_ERROR, "kernel launch failed: %s (%s:%d)", \
                               cudaGetErrorString(e_), __FILE__, __LINE__);   \
        ::mtb::count_launch();                                                \
    } while (0)

// A device buffer owned by a plan (plan scratch only; fields, coefficients
// and accumulators always belong to the caller).
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    int ensure(size_t n) {
        if (n <= bytes) return MTB_OK;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (n == 0) return MTB_OK;
        cudaError_t e = cudaMalloc(&p, n);
        if (e != cudaSuccess)
            return fail(MTB_CUDA_ERROR, "cudaMalloc(%zu) failed: %s", n, cudaGetErrorString(e));
        bytes = n;
        return MTB_OK;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};

// Pinned host staging buffer.
struct HostBuf {
    void *p = nullptr;
    size_t bytes = 0;
    int ensure(size_t n) {
        if (n <= bytes) return MTB_OK;
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        if (n == 0) return MTB_OK;
        cudaError_t e = cudaMallocHost(&p, n);
        if (e != cudaSuccess)
            return fail(MTB_CUDA_ERROR, "cudaMallocHost(%zu) failed: %s", n, cudaGetErrorString(e));
        bytes = n;
        return MTB_OK;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};

// Opt-in per-launch device timing (event pairs around launches).
// Two pinned host staging buffers used alternately for host -> device
// uploads: a buffer is refilled only after its previous upload completed
// (an event), so back-to-back runs on one stream never wait for the GPU.
struct PinnedPair {
    HostBuf h[2];
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool pending[2] = {false, false};
    int next = 0;
    // a staging buffer of at least `bytes` that may be overwritten now
    int acquire(size_t bytes, void **out) {
        const int b = next;
        if (pending[b]) {
            MTB_CUDA_TRY(cudaEventSynchronize(ev[b]));
            pending[b] = false;
        }
        const int rc = h[b].ensure(bytes);
        if (rc) return rc;
        *out = h[b].p;
        return MTB_OK;
    }
    // the upload from the last acquired buffer has been queued on `st`
    int queued(cudaStream_t st) {
        const int b = next;
        if (!ev[b]) MTB_CUDA_TRY(cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming));
        MTB_CUDA_TRY(cudaEventRecord(ev[b], st));
        pending[b] = true;
        next ^= 1;
        return MTB_OK;
    }
    void release() {
        for (int b = 0; b < 2; ++b) {
            if (ev[b]) {
                cudaEventSynchronize(ev[b]);
                cudaEventDestroy(ev[b]);
            }
            ev[b] = nullptr;
            pending[b] = false;
            h[b].release();
        }
    }
};

struct LaunchTimer {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
    std::vector<int> kind;          // 0 = step kernel, 1 = DFT contraction
    double ms[2] = {0, 0};
    int64_t count[2] = {0, 0};
    int begin(cudaStream_t st, int k);   // record the start event of a launch
    int end(cudaStream_t st);            // record the end event
    int collect();                       // wait and sum; resets the pool cursor
    void release();
};

// ---------------------------------------------------------------- DFT
// Phase tables and the ring contraction shared by the 2D and 3D plans.
struct DftState {
    // host copies
    std::string err;
    int n_regions = 0, n_groups = 0;
    mtb_dft_region *regions_h = nullptr;   // host copy
    int *group_nf = nullptr;               // host
    int *group_mode = nullptr;
    double *group_dt = nullptr;
    double *freqs_h = nullptr;             // concatenated
    int *freq_off = nullptr;               // per group offset into freqs_h
    int total_nf = 0;                      // sum of nf
    // device
    DevBuf regions_d, blk_start_d, blk_region_d, phase_d, ring_d;
    PinnedPair phase_h;
    int64_t slot_elems = 0;
    int slots = 0;                         // ring depth K
    int64_t n_blocks = 0;                  // contraction blocks
    int *blk_start_h = nullptr;

    int init(const mtb_dft_region *regions, int n_regions, const mtb_phase_group *groups,
             int n_groups, int64_t slot_elems, int slots);
    // Fill the phase table for steps [t0, t0+k) and upload it on `st`.
    int upload_phases(int64_t t0, int k, cudaStream_t st);
    // Fold ring slots [0, n) (steps t_first .. t_first+n-1, relative row
    // `row0` of the uploaded table, or of `phase_base` when given) into the
    // accumulators.
    int contract(int row0, int n, cudaStream_t st, LaunchTimer *tm = nullptr,
                 const float *phase_base = nullptr);
    // Transposed contraction: zero ring slots [0, n) and fill them with the
    // adjoint of the samples of the n staged steps (region acc = d J / d acc).
    int expand(int row0, int n, cudaStream_t st);
    void release();
};

}  // namespace mtb
