// Streamed line lists: a Voigt cross-section over a line list held in
// (pinned) host memory as FP64 centres, FP32 intensities S(T) and FP32
// Lorentz half widths gamma(T, P) -- 16 bytes per line, so 5e8 lines are
// 8 GB of host memory.  No counterpart in the reference, whose
// VoigtProfile reads transitions into host chunks and hands each to the
// manager synchronously (VoigtProfile.cpp:56-103, BaseProfile.cpp:49-62).
//
// The list is cut into chunks of consecutive lines.  Chunk k is copied to
// device buffer k % 2 on a copy stream while chunk k - 1 is evaluated on the
// engine's stream; each chunk's step one builds its records from the
// precomputed S and gamma, and its step two adds into the grid points its
// lines reach.  The chunks are evaluated in order on one stream, so the sum
// is deterministic for a given chunk size.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "xs_engine.h"
#include "xsec_b200.h"

namespace {

int st_fail(int code, const std::string& msg) { return xs::set_error(code, msg.c_str()); }

struct Buffers {
    double* nu[2] = {nullptr, nullptr};
    float* s[2] = {nullptr, nullptr};
    float* gl[2] = {nullptr, nullptr};
    cudaEvent_t copied[2] = {nullptr, nullptr}, done[2] = {nullptr, nullptr};
    cudaEvent_t t0 = nullptr, t1 = nullptr, c0 = nullptr, c1 = nullptr;
    cudaStream_t cs = nullptr;
    ~Buffers() {
        for (int b = 0; b < 2; ++b) {
            cudaFree(nu[b]);
            cudaFree(s[b]);
            cudaFree(gl[b]);
            if (copied[b]) cudaEventDestroy(copied[b]);
            if (done[b]) cudaEventDestroy(done[b]);
        }
        for (cudaEvent_t e : {t0, t1, c0, c1})
            if (e) cudaEventDestroy(e);
        if (cs) cudaStreamDestroy(cs);
    }
};

}  // namespace

extern "C" int xs_stream_execute(xs_engine* e, const xs_options* opt, const xs_condition* cond,
                                 const double* h_nu, const float* h_s, const float* h_gamma,
                                 size_t n, const xs_grid* grid, double* out, size_t chunk_lines,
                                 xs_stream_stats* stats) {
    if (!e || !opt || !cond || !grid || !out || (n > 0 && (!h_nu || !h_s || !h_gamma)))
        return st_fail(XS_ERR_INVALID, "xs_stream_execute: NULL argument");
    if (opt->profile != XS_VOIGT || opt->convention != XS_CONV_GPU)
        return st_fail(XS_ERR_UNSUPPORTED, "xs_stream_execute: VOIGT with the GPU convention only");
    if (chunk_lines == 0 || chunk_lines > (size_t(1) << 30))
        return st_fail(XS_ERR_INVALID, "xs_stream_execute: chunk_lines must be 1 .. 2^30");
    if (!grid->freq || grid->npoints_total < 1 || grid->start_idx != 0 ||
        grid->points != grid->npoints_total)
        return st_fail(XS_ERR_INVALID, "xs_stream_execute: give the whole grid (start 0, all points)");
    if (stats) *stats = xs_stream_stats{};
    if (n == 0) return XS_OK;
    // Order inside a chunk is checked on the device (step one's unsorted
    // flag, reported by the final sync); here only across chunk boundaries.
    const size_t cl0 = std::min(chunk_lines, n);
    for (size_t i = cl0; i < n; i += cl0)
        if (h_nu[i] < h_nu[i - 1])
            return st_fail(XS_ERR_UNSORTED, "xs_stream_execute: line centres must be ascending");

    const int dev = xs::engine_device(e);
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
    struct Restore {
        int p, d;
        ~Restore() {
            if (p >= 0 && p != d) cudaSetDevice(p);
        }
    } restore{prev, dev};

    const cudaStream_t es = static_cast<cudaStream_t>(xs::engine_stream(e));
    const size_t cl = std::min(chunk_lines, n);
    Buffers B;
    cudaError_t err = cudaStreamCreateWithFlags(&B.cs, cudaStreamNonBlocking);
    for (int b = 0; b < 2 && err == cudaSuccess; ++b) {
        err = cudaMalloc(&B.nu[b], cl * sizeof(double));
        if (err == cudaSuccess) err = cudaMalloc(&B.s[b], cl * sizeof(float));
        if (err == cudaSuccess) err = cudaMalloc(&B.gl[b], cl * sizeof(float));
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&B.copied[b], cudaEventDisableTiming);
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&B.done[b], cudaEventDisableTiming);
    }
    for (cudaEvent_t* ev : {&B.t0, &B.t1, &B.c0, &B.c1})
        if (err == cudaSuccess) err = cudaEventCreate(ev);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return st_fail(err == cudaErrorMemoryAllocation ? XS_ERR_NOMEM : XS_ERR_CUDA,
                       std::string("xs_stream_execute: ") + cudaGetErrorString(err));
    }
    // reserve the engine's scratch for a full chunk before the pipeline starts
    {
        const size_t need = xs_scratch_bytes_needed(opt, 1, cl);
        const int rc = xs::engine_reserve(e, ((need + 255) & ~size_t(255)) + (size_t(64) << 20));
        if (rc != XS_OK) return rc;
    }

    const double cut = cond->cut > 0.0 ? cond->cut : std::fmin(25.0 * cond->pressure, 100.0);
    // grid bounds on the host for the chunk ranges: the caller's grid is
    // f0 + i df (checked on the device by the engine's grid test)
    double g0 = 0.0;
    err = cudaMemcpy(&g0, grid->freq, sizeof(double), cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return st_fail(XS_ERR_CUDA, cudaGetErrorString(err));
    const double df = opt->dfreq;
    const int N = grid->npoints_total;

    cudaEventRecord(B.t0, es);
    cudaEventRecord(B.c0, B.cs);
    const size_t nchunks = (n + cl - 1) / cl;
    int kernels = 0;
    for (size_t k = 0; k < nchunks; ++k) {
        const int b = int(k & 1);
        const size_t off = k * cl;
        const size_t m = std::min(cl, n - off);
        if (k >= 2) cudaStreamWaitEvent(B.cs, B.done[b], 0);
        err = cudaMemcpyAsync(B.nu[b], h_nu + off, m * sizeof(double), cudaMemcpyHostToDevice, B.cs);
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(B.s[b], h_s + off, m * sizeof(float), cudaMemcpyHostToDevice, B.cs);
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(B.gl[b], h_gamma + off, m * sizeof(float), cudaMemcpyHostToDevice, B.cs);
        if (err == cudaSuccess) err = cudaEventRecord(B.copied[b], B.cs);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(es, B.copied[b], 0);
        if (err != cudaSuccess) return st_fail(XS_ERR_CUDA, cudaGetErrorString(err));
        // grid points this chunk's lines can reach (one point of margin)
        const double lo_f = (h_nu[off] - cut - g0) / df, hi_f = (h_nu[off + m - 1] + cut - g0) / df;
        const long lo = std::max(0L, long(std::floor(lo_f)) - 1);
        const long hi = std::min(long(N), long(std::ceil(hi_f)) + 2);
        if (hi > lo) {
            xs_lines L{};
            L.nu = B.nu[b];
            L.count = m;
            xs_grid G{grid->freq, N, int(lo), int(hi - lo)};
            xs::ExecOverride ov;
            ov.no_timing = true;
            ov.s32 = B.s[b];
            ov.gl32 = B.gl[b];
            const int rc = xs::engine_execute(e, opt, cond, 1, &L, &G, out, 0, &ov);
            if (rc != XS_OK) return rc;
            kernels += ov.kernels;
        }
        err = cudaEventRecord(B.done[b], es);
        if (err != cudaSuccess) return st_fail(XS_ERR_CUDA, cudaGetErrorString(err));
    }
    cudaEventRecord(B.c1, B.cs);
    cudaEventRecord(B.t1, es);
    err = cudaEventSynchronize(B.t1);
    if (err == cudaSuccess) err = cudaEventSynchronize(B.c1);
    if (err != cudaSuccess) return st_fail(XS_ERR_CUDA, cudaGetErrorString(err));
    const int rc = xs_engine_sync(e);
    if (rc != XS_OK) return rc;
    if (stats) {
        float ms = 0.f, cms = 0.f;
        cudaEventElapsedTime(&ms, B.t0, B.t1);
        cudaEventElapsedTime(&cms, B.c0, B.c1);
        stats->total_ms = ms;
        stats->copy_span_ms = cms;
        stats->h2d_bytes = double(n) * (sizeof(double) + 2 * sizeof(float));
        stats->chunks = int(nchunks);
        stats->kernels = kernels;
    }
    return XS_OK;
}
