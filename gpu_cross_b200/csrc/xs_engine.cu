// Host side of the engine and the C ABI declared in include/xsec_b200.h.
//
// An engine owns a stream, a grow-only device scratch area (per-line records
// and windows for every condition of a call) and two device words (an error
// word the kernels OR bits into, and the work counter of the persistent step
// two).  xs_engine_execute computes the per-condition constants on the host
// exactly as the chosen reference backend does, then launches
//   grid check -> step one (k_prep) -> step two (persistent warps)
// on the engine's stream.  Nothing is synchronised until xs_engine_sync,
// which also turns the error word into a status code.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "xs_engine.h"
#include "xs_internal.cuh"
#include "xsec_b200.h"

using namespace xs;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(e == cudaErrorMemoryAllocation ? XS_ERR_NOMEM : XS_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

#define XS_CU(call)                                     \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

// Most slices of a host line list (xs_engine_execute_host).
constexpr int kMaxPieces = 16;

// Restores the caller's current device on scope exit.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace

struct xs_engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 0;
    void* scratch = nullptr;
    size_t scratch_cap = 0;
    unsigned* d_words = nullptr;  // [0] error bits, [1] work counter
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    bool timed = false;
    // host line lists (xs_engine_execute_host): a copy stream and an event
    // per slice, made on first use
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t pev[kMaxPieces + 1] = {};
    // error statement of the last execute: the a-priori bound and, with
    // sampled rows, where their statistics are ([c][4] doubles)
    double bound_rel = 0.0;
    const double* chk_stats = nullptr;
    int chk_rows = 0, chk_ncond = 0;
    std::mutex mu;
};

namespace xs {

int set_error(int code, const char* msg) { return fail(code, msg); }

// Default launch shapes, from measurements on a B200 (the autotuner's table
// takes precedence).  Voigt tiles of 32 P points: wide where a line's window
// spans thousands of points (fewer partial lines per tile, record loads
// shared by more points), narrow on coarse grids, where a 128-point tile
// would hold mostly partial and core lines.  4 warps per block (the mixed
// kernels then fit 28 warps per SM).
void default_shape(int kind, bool mixed, double window_points, int* P, int* warps) {
    if (kind == kVoigt) {
        *P = window_points >= 2048.0 ? 4 : (window_points >= 512.0 ? 2 : 1);
        *warps = 4;
    } else {
        *P = 1;
        *warps = 8;
    }
}

// Launch shapes chosen by xs_engine_autotune, per call signature: profile,
// convention, precision, number of conditions, and the binary magnitudes of
// the grid points and of the lines per grid point inside the window.
struct Shape {
    int P, W, C;
    double ms;
};
std::mutex g_tune_mu;
std::map<std::string, Shape> g_tune;

std::string shape_key(const xs_options& o, const xs_condition* conds, int ncond, long n, int points) {
    double cutmax = 0.0;
    for (int c = 0; c < ncond; ++c) cutmax = std::fmax(cutmax, make_cond(o, conds[c]).cut);
    const double win = 2.0 * cutmax / o.dfreq;
    const double density = double(n) * win / (double(points) + win);
    auto lg = [](double v) { return v < 1.0 ? 0 : int(std::floor(std::log2(v))); };
    char buf[96];
    std::snprintf(buf, sizeof(buf), "p%d.v%d.x%d.c%d.g%d.d%d", o.profile, o.convention, o.precision,
                  ncond < kMaxCond ? ncond : kMaxCond, lg(double(points)), lg(density));
    return buf;
}

// Host copy of the per-condition constants.  GPU convention:
// GpuManager::InitializeConstants (GPUManager.cpp:28-39) and the step-two
// kernels (cross_kernal.cu:667, :938-939).  CPU convention: OpenMPManager
// (OpenMPManager.cpp:65-66, :146-147, :191-192).
CondDev make_cond(const xs_options& o, const xs_condition& c) {
    CondDev d{};
    const double T = c.temperature;
    const double M = o.mean_mass;
    if (o.convention == XS_CONV_GPU) {
        const double planck = 6.6260693e-27, vellgt = 2.99792458e10, boltz = 1.380658e-16;
        const double pi = std::acos(-1.0);
        d.cmcoef = 1.0 / (8.0 * pi * vellgt);
        d.beta = planck * vellgt / (boltz * T);
        d.dpw = std::sqrt(2.0 * kBOLTZ * T * kNA / (M)) / kVELLGT;
    } else {
        d.cmcoef = 1.0 / (8.0 * kPI * kVELLGT);
        d.beta = kPLANCK * kVELLGT / (kBOLTZ * T);
        d.dpw = std::sqrt(2.0 * kLN2 * kBOLTZ * T * kNA / (M)) / kVELLGT;
    }
    d.partition = c.partition;
    d.tratio = o.ref_temp / T;
    d.gamma_scale = c.gamma_scale > 0.0 ? c.gamma_scale : 1.0;
    if (c.cut > 0.0) {
        d.cut = c.cut;
    } else if (o.profile == XS_VOIGT) {
        d.cut = std::fmin(25.0 * c.pressure, 100.0);
    } else if (o.profile == XS_DOPPLER) {
        d.cut = kDOPPLER_CUTOFF;
    } else {
        d.cut = o.half_width * 10.0;
    }
    return d;
}

// A-priori relative error bound of a result against the FP64 path of the
// same convention (see xs_engine_accuracy).
double error_bound(int kind, bool mixed) {
    if (kind == XS_VOIGT && mixed) return 1024.0 * 0x1p-24;
    return 1e-12;
}

// Lines the CPU convention covers: OpenMPManager splits N lines into blocks
// of ceil(float(N)/float(threads)) (OpenMPManager.cpp:186-188); lines beyond
// threads * block are never processed.
long cpu_covered_lines(long n, int threads) {
    if (threads < 1) return n;
    const int nener = int(n);
    const int for_block = int(std::ceil(float(nener) / float(threads)));
    const long covered = long(threads) * long(for_block);
    return covered < n ? covered : n;
}

}  // namespace xs

extern "C" {

const char* xs_last_error(void) { return g_last_error.c_str(); }

const char* xs_version(void) { return "xsec_b200 0.1 (sm_100a)"; }

int xs_device_available(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
        cudaGetLastError();
        return 0;
    }
    for (int d = 0; d < n; ++d) {
        int major = 0;
        if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, d) == cudaSuccess &&
            major == 10)
            return 1;
    }
    return 0;
}

int xs_device_count(int* count) {
    if (!count) return fail(XS_ERR_INVALID, "xs_device_count: count is NULL");
    *count = 0;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return XS_OK;
    }
    *count = n;
    return XS_OK;
}

int xs_engine_create(int device, xs_engine** out) {
    if (!out) return fail(XS_ERR_INVALID, "xs_engine_create: out is NULL");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return fail(XS_ERR_NODEVICE, "xs_engine_create: no such CUDA device");
    }
    int major = 0;
    XS_CU(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    if (major != 10)
        return fail(XS_ERR_NODEVICE, "xs_engine_create: the kernels are built for sm_100a only");
    DeviceGuard g(device);
    auto* e = new xs_engine();
    e->device = device;
    XS_CU(cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, device));
    cudaError_t err = cudaMalloc(&e->d_words, 4 * sizeof(unsigned));
    if (err != cudaSuccess) {
        delete e;
        return cuda_fail(err, "cudaMalloc(engine words)");
    }
    err = cudaMemset(e->d_words, 0, 4 * sizeof(unsigned));
    for (auto& ev : e->ev)
        if (err == cudaSuccess) err = cudaEventCreate(&ev);
    if (err != cudaSuccess) {
        xs_engine_destroy(e);
        return cuda_fail(err, "xs_engine_create");
    }
    *out = e;
    return XS_OK;
}

int xs_engine_destroy(xs_engine* e) {
    if (!e) return XS_OK;
    {
        DeviceGuard g(e->device);
        if (e->stream) cudaStreamSynchronize(e->stream);
        else cudaDeviceSynchronize();
        for (auto& ev : e->ev)
            if (ev) cudaEventDestroy(ev);
        for (auto& ev : e->pev)
            if (ev) cudaEventDestroy(ev);
        if (e->copy_stream) cudaStreamDestroy(e->copy_stream);
        cudaFree(e->scratch);
        cudaFree(e->d_words);
    }
    delete e;
    return XS_OK;
}

int xs_engine_set_stream(xs_engine* e, void* stream) {
    if (!e) return fail(XS_ERR_INVALID, "xs_engine_set_stream: NULL engine");
    std::lock_guard<std::mutex> lk(e->mu);
    e->stream = static_cast<cudaStream_t>(stream);
    return XS_OK;
}

int xs_engine_sync(xs_engine* e) {
    if (!e) return fail(XS_ERR_INVALID, "xs_engine_sync: NULL engine");
    std::lock_guard<std::mutex> lk(e->mu);
    DeviceGuard g(e->device);
    XS_CU(cudaStreamSynchronize(e->stream));
    unsigned w = 0;
    XS_CU(cudaMemcpy(&w, e->d_words, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (w) {
        XS_CU(cudaMemset(e->d_words, 0, sizeof(unsigned)));
        if (w & kErrUnsorted)
            return fail(XS_ERR_UNSORTED, "line centres are not in ascending order (the reference "
                                         "requires nu-sorted input)");
        if (w & kErrGrid)
            return fail(XS_ERR_GRID, "the grid is not ascending with the uniform step dfreq");
        if (w & kErrReach)
            return fail(XS_ERR_UNSUPPORTED, "mixed precision: a line's core lies 3e7 or more grid points "
                                            "from its centre's grid index (grid step too fine for the "
                                            "cut); use FP64");
    }
    return XS_OK;
}

int xs_engine_scratch_bytes(xs_engine* e, size_t* bytes) {
    if (!e || !bytes) return fail(XS_ERR_INVALID, "xs_engine_scratch_bytes: NULL argument");
    *bytes = e->scratch_cap;
    return XS_OK;
}

size_t xs_scratch_bytes_needed(const xs_options* opt, int ncond, size_t n_lines) {
    if (!opt || ncond < 1) return 0;
    const bool mixed = opt->profile == XS_VOIGT && opt->precision == XS_MIXED;
    const int nc = ncond < kMaxCond ? ncond : kMaxCond;
    return plan_scratch(opt->profile, mixed, n_lines, nc, 0).need;
}

int xs_engine_execute(xs_engine* e, const xs_options* opt, const xs_condition* conds, int ncond,
                      const xs_lines* lines, const xs_grid* grid, double* out, size_t out_stride) {
    return xs::engine_execute(e, opt, conds, ncond, lines, grid, out, out_stride, nullptr);
}

int xs_engine_execute_host(xs_engine* e, const xs_options* opt, const xs_condition* conds, int ncond,
                           const xs_lines* host_lines, const xs_lines* dev_lines, const xs_grid* grid,
                           double* out, size_t out_stride, double* host_out, int pieces) {
    if (!e || !host_lines || !dev_lines || !grid)
        return fail(XS_ERR_INVALID, "xs_engine_execute_host: NULL argument");
    if (host_lines->count != dev_lines->count)
        return fail(XS_ERR_INVALID, "xs_engine_execute_host: host and device line counts differ");
    if (!host_lines->nu || !host_lines->energies || !host_lines->aif || !host_lines->gns)
        return fail(XS_ERR_INVALID, "xs_engine_execute_host: host line arrays missing");
    if (opt && opt->profile == XS_VOIGT && (!host_lines->gamma || !host_lines->n))
        return fail(XS_ERR_INVALID, "xs_engine_execute_host: VOIGT needs gamma and n");
    if (pieces < 1 || pieces > kMaxPieces)
        return fail(XS_ERR_INVALID, "xs_engine_execute_host: pieces must be 1..16");
    xs::ExecOverride ov;
    ov.h2d = host_lines;
    ov.h2d_pieces = pieces;
    int rc;
    {
        DeviceGuard g(e->device);
        rc = xs::engine_execute(e, opt, conds, ncond, dev_lines, grid, out, out_stride, &ov);
        if (rc == XS_OK && host_out && ncond > 0 && grid->points > 0) {
            // the chunk's span of every condition's row, rows out_stride apart
            const size_t pitch = sizeof(double) * (ncond > 1 ? out_stride : size_t(grid->start_idx + grid->points));
            const size_t at = size_t(grid->start_idx);
            XS_CU(cudaMemcpy2DAsync(host_out + at, pitch, out + at, pitch, sizeof(double) * size_t(grid->points),
                                    size_t(ncond), cudaMemcpyDeviceToHost, e->stream));
        }
    }
    return rc;
}

double xs_error_bound(int profile, int precision) {
    return error_bound(profile, profile == XS_VOIGT && precision == XS_MIXED);
}

int xs_engine_accuracy(xs_engine* e, xs_accuracy* acc) {
    if (!e || !acc) return fail(XS_ERR_INVALID, "xs_engine_accuracy: NULL argument");
    std::lock_guard<std::mutex> lk(e->mu);
    acc->bound_rel = e->bound_rel;
    acc->sampled_max_rel = -1.0;
    acc->sampled_integrated_rel = -1.0;
    acc->sampled_rows = 0;
    acc->conditions = e->chk_ncond;
    if (e->chk_rows > 0 && e->chk_stats && e->chk_ncond > 0) {
        DeviceGuard g(e->device);
        XS_CU(cudaStreamSynchronize(e->stream));
        std::vector<double> st(size_t(4 * e->chk_ncond));
        XS_CU(cudaMemcpy(st.data(), e->chk_stats, sizeof(double) * st.size(), cudaMemcpyDeviceToHost));
        double mx = 0.0, integ = 0.0;
        for (int c = 0; c < e->chk_ncond; ++c) {
            mx = std::fmax(mx, st[size_t(4 * c)]);
            const double sr = st[size_t(4 * c + 1)], sd = st[size_t(4 * c + 2)];
            if (sr != 0.0) integ = std::fmax(integ, std::fabs(sd) / std::fabs(sr));
        }
        acc->sampled_max_rel = mx;
        acc->sampled_integrated_rel = integ;
        acc->sampled_rows = e->chk_rows;
    }
    return XS_OK;
}

int xs_engine_last_stats(xs_engine* e, double* prep_ms, double* steptwo_ms) {
    if (!e) return fail(XS_ERR_INVALID, "xs_engine_last_stats: NULL engine");
    if (!e->timed) return fail(XS_ERR_STATE, "xs_engine_last_stats: nothing executed yet");
    DeviceGuard g(e->device);
    XS_CU(cudaEventSynchronize(e->ev[2]));
    float a = 0.f, b = 0.f;
    XS_CU(cudaEventElapsedTime(&a, e->ev[0], e->ev[1]));
    XS_CU(cudaEventElapsedTime(&b, e->ev[1], e->ev[2]));
    if (prep_ms) *prep_ms = a;
    if (steptwo_ms) *steptwo_ms = b;
    return XS_OK;
}

}  // extern "C"

namespace xs {

int engine_execute(xs_engine* e, const xs_options* opt, const xs_condition* conds, int ncond,
                   const xs_lines* lines, const xs_grid* grid, double* out, size_t out_stride,
                   const ExecOverride* ov) {
    if (!e || !opt || !conds || !lines || !grid || !out)
        return fail(XS_ERR_INVALID, "xs_engine_execute: NULL argument");
    const int kind = opt->profile;
    if (kind == XS_PSUEDO_VOIGT)
        return fail(XS_ERR_UNSUPPORTED, "PSUEDO_VOIGT is not implemented (nor is it in the reference)");
    if (kind != XS_VOIGT && kind != XS_DOPPLER && kind != XS_GAUSSIAN)
        return fail(XS_ERR_INVALID, "unknown profile");
    if (opt->convention != XS_CONV_GPU && opt->convention != XS_CONV_CPU)
        return fail(XS_ERR_INVALID, "unknown convention");
    if (kind == XS_GAUSSIAN && opt->convention == XS_CONV_CPU)
        return fail(XS_ERR_UNSUPPORTED, "the reference CPU backend has no GAUSSIAN profile");
    if (opt->precision != XS_FP64 && opt->precision != XS_MIXED)
        return fail(XS_ERR_INVALID, "unknown precision");
    if (ncond < 1) return fail(XS_ERR_INVALID, "ncond < 1");
    if (!(opt->dfreq > 0.0)) return fail(XS_ERR_INVALID, "dfreq must be > 0");
    if (!(opt->mean_mass > 0.0) && kind != XS_GAUSSIAN)
        return fail(XS_ERR_INVALID, "mean_mass must be > 0");
    if (kind == XS_GAUSSIAN && !(opt->half_width > 0.0))
        return fail(XS_ERR_INVALID, "half_width must be > 0 for GAUSSIAN");
    if (!grid->freq || grid->npoints_total < 1 || grid->start_idx < 0 || grid->points < 0 ||
        long(grid->start_idx) + long(grid->points) > long(grid->npoints_total))
        return fail(XS_ERR_INVALID, "grid chunk outside the grid");
    if (ncond > 1 && out_stride < size_t(grid->points))
        return fail(XS_ERR_INVALID, "out_stride smaller than the grid chunk");
    const bool streamed = ov && ov->s32;
    if (streamed && (kind != XS_VOIGT || opt->convention != XS_CONV_GPU || !ov->gl32))
        return fail(XS_ERR_UNSUPPORTED, "precomputed intensities: VOIGT, GPU convention, with gamma");
    const int h2d_pieces = (ov && ov->h2d) ? std::max(1, std::min(ov->h2d_pieces, kMaxPieces)) : 0;
    if (h2d_pieces && (streamed || (ov->tc_s != nullptr)))
        return fail(XS_ERR_INVALID, "host lines: not with precomputed intensities or caches");
    const int tc_mode = (ov && ov->tc_s) ? ov->tc_mode : 0;
    if (tc_mode && (streamed || ncond != 1 || tc_mode < 1 || tc_mode > 2 || (kind == XS_VOIGT && !ov->tc_pw)))
        return fail(XS_ERR_INVALID, "per-temperature cache: one condition, S (and Voigt's power) arrays");
    if (lines->count > 0 && (!lines->nu || (!streamed && (!lines->energies || !lines->aif || !lines->gns))))
        return fail(XS_ERR_INVALID, "line arrays missing");
    if (kind == XS_VOIGT && lines->count > 0 && !streamed && (!lines->gamma || !lines->n))
        return fail(XS_ERR_INVALID, "VOIGT needs gamma and n");
    if (lines->count > size_t(INT32_MAX))
        return fail(XS_ERR_INVALID, "more than 2^31-1 lines in one call");
    for (int c = 0; c < ncond; ++c)
        if (!(conds[c].temperature > 0.0))
            return fail(XS_ERR_INVALID, "temperature must be > 0");
    const bool mixed = kind == XS_VOIGT && opt->precision == XS_MIXED;
    if (mixed && double(grid->npoints_total) > 15.0e6)
        return fail(XS_ERR_UNSUPPORTED, "mixed precision supports grids below 1.5e7 points");

    long n = long(lines->count);
    if (opt->convention == XS_CONV_CPU) n = cpu_covered_lines(n, opt->cpu_threads);
    if (n <= 0 || grid->points <= 0) return XS_OK;

    int P = opt->points_per_thread, W = opt->warps_per_block;
    int C = opt->conditions_per_warp;
    if (P == 0 && W == 0 && C == 0) {
        // a shape the autotuner measured for calls like this one
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(shape_key(*opt, conds, ncond, n, grid->points));
        if (it != g_tune.end()) {
            P = it->second.P;
            W = it->second.W;
            C = it->second.C;
        }
    }
    {
        int dP, dW;
        double cutmax = 0.0;
        for (int c = 0; c < ncond; ++c) cutmax = std::fmax(cutmax, make_cond(*opt, conds[c]).cut);
        default_shape(kind, mixed, 2.0 * cutmax / opt->dfreq, &dP, &dW);
        if (P == 0) P = dP;
        if (W == 0) W = dW;
    }
    if (kind == XS_VOIGT ? !(P == 1 || P == 2 || P == 4 || P == 8) : !(P == 1 || P == 2))
        return fail(XS_ERR_INVALID, "points_per_thread must be 1, 2, 4 or 8 (1 or 2 for erf profiles)");
    if (W != 4 && W != 8) return fail(XS_ERR_INVALID, "warps_per_block must be 4 or 8");

    // Multi-condition tiles (Voigt batches whose conditions share the cut).
    if (C < 0 || C == 3 || C > 8 || (C > 4 && C != 8))
        return fail(XS_ERR_INVALID, "conditions_per_warp must be 0, 1, 2, 4 or 8");
    // Order in which the conditions are evaluated (their results still go to
    // their own rows).  Voigt: by cut, then by decreasing Lorentz-to-Doppler
    // ratio (the gamma scale times (T_ref/T)^0.6, over the Doppler width per
    // unit wavenumber), so that the conditions sharing a multi-condition
    // group have similar core widths: a group's core run is set by its
    // widest core, and conditions whose y exceeds 15 have none.
    std::vector<int> order(static_cast<size_t>(ncond));
    for (int c = 0; c < ncond; ++c) order[size_t(c)] = c;
    if (kind == XS_VOIGT) {
        std::vector<double> cutv(order.size()), yv(order.size());
        for (int c = 0; c < ncond; ++c) {
            const CondDev d = make_cond(*opt, conds[c]);
            cutv[size_t(c)] = d.cut;
            const double yc = d.gamma_scale * std::pow(d.tratio, 0.6) / d.dpw;
            yv[size_t(c)] = std::isfinite(yc) ? yc : 0.0;
        }
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            if (cutv[size_t(x)] != cutv[size_t(y)]) return cutv[size_t(x)] < cutv[size_t(y)];
            return yv[size_t(x)] > yv[size_t(y)];
        });
    }
    {
        auto groups_ok = [&](int cg) {
            if (cg < 2 || ncond > kMaxCond || ncond % cg != 0) return false;
            for (int g0 = 0; g0 < ncond; g0 += cg) {
                const double cut0 = make_cond(*opt, conds[order[size_t(g0)]]).cut;
                for (int k = 1; k < cg; ++k)
                    if (make_cond(*opt, conds[order[size_t(g0 + k)]]).cut != cut0) return false;
            }
            return true;
        };
        if (kind != XS_VOIGT) {
            C = 1;
        } else if (C == 0) {
            // Measured on B200 (40-condition sweep, 0.1 cm-1 grid): two
            // conditions per warp is fastest for the mixed path; the FP64
            // path is faster with one condition and 32*P points per warp.
            C = (mixed && groups_ok(2)) ? 2 : 1;
        } else if (C > 1 && !groups_ok(C)) {
            return fail(XS_ERR_INVALID, "conditions_per_warp needs ncond <= 64 and, for every cut, a "
                                        "number of conditions that is a multiple of it");
        }
    }
    const int CG = C > 1 ? C : 0;
    if (opt->line_splits < 0 || opt->line_splits > kMaxSplits)
        return fail(XS_ERR_INVALID, "line_splits must be 0 (automatic) .. 64");

    std::lock_guard<std::mutex> lk(e->mu);
    DeviceGuard dg(e->device);

    // Scratch layout for one group of conditions.
    const int group = ncond < kMaxCond ? ncond : kMaxCond;
    const ScratchPlan plan = plan_scratch(kind, mixed, size_t(n), group, 0, CG);
    int occ = CG ? steptwo_mc_blocks_per_sm(mixed, CG, W)
                 : steptwo_blocks_per_sm(kind, opt->convention, mixed, P, W);
    if (occ < 1) {
        // e.g. 8 FP64 conditions per warp with 8 warps: more shared memory
        // than a block can have
        cudaGetLastError();
        return fail(XS_ERR_INVALID, "this launch shape cannot run on the device (shared memory)");
    }

    // Line splits.  Work items are taken dynamically, but an item is a whole
    // tile over all its lines: with fewer items than resident warps (short
    // or coarse grids over many lines) most of the GPU idles while each warp
    // walks a long line list, and with a few items per warp the last items
    // leave a tail.  Each tile's lines are then split into parts taken by
    // different warps -- enough for about 16 items per resident warp, at
    // least ~256 lines per part, the parts' buffer within kMaxPartBytes.
    // The count depends only on the call's sizes and the SM count.
    const int tile_pts = CG ? 32 : 32 * P;
    const int tiles = (grid->points + tile_pts - 1) / tile_pts;
    int S = opt->line_splits;
    if (ov && ov->scratch) S = 1;  // a fixed caller scratch holds no parts
    if (S == 0) {
        const long items = long(tiles) * (CG ? group / CG : group);
        const long warps = long(occ) * W * e->num_sms;
        S = 1;
        if (items < 16 * warps) {
            double cutmax = 0.0;
            for (int c = 0; c < ncond; ++c) cutmax = std::fmax(cutmax, make_cond(*opt, conds[c]).cut);
            const double span = double(grid->points) * opt->dfreq + 2.0 * cutmax;
            const double lpt = double(n) * (double(tile_pts) * opt->dfreq + 2.0 * cutmax) / span;
            long want = (16 * warps + items - 1) / items;
            want = std::min<long>(want, long(lpt / 256.0));
            const long cap = long(kMaxPartBytes / (sizeof(double) * size_t(group) * size_t(grid->points)));
            want = std::min<long>(want, std::min<long>(cap, kMaxSplits));
            if (want > 1) S = int(want);
        }
    }
    const size_t part_off = (plan.need + 255) & ~size_t(255);
    const size_t part_end = S > 1 ? part_off + sizeof(double) * size_t(S) * size_t(group) * size_t(grid->points)
                                  : plan.need;
    // sampled FP64 check (mixed Voigt): before/ref values and statistics
    const bool streamed_call = ov && ov->s32;
    const int tiles32 = (grid->points + 31) / 32;
    const int nchk = (mixed && kind == XS_VOIGT && !streamed_call && opt->check_rows > 0)
                         ? std::min(std::min(opt->check_rows, kMaxCheckRows), tiles32)
                         : 0;
    const size_t chk_off = (part_end + 255) & ~size_t(255);
    const size_t chk_bytes = nchk ? sizeof(double) * (size_t(2 * 32 * nchk) + 4) * size_t(ncond) : 0;
    const size_t need = nchk ? chk_off + chk_bytes : part_end;

    void* scratch = nullptr;
    unsigned* words = e->d_words;
    if (ov && ov->scratch) {
        if (need > ov->scratch_bytes)
            return fail(XS_ERR_NOMEM, "scratch larger than the caller-provided area");
        scratch = ov->scratch;
        if (ov->words) words = ov->words;
    } else {
        if (need > e->scratch_cap) {
            XS_CU(cudaStreamSynchronize(e->stream));
            cudaFree(e->scratch);
            e->scratch = nullptr;
            e->scratch_cap = 0;
            cudaError_t err = cudaMalloc(&e->scratch, need);
            if (err != cudaSuccess) {
                cudaGetLastError();
                return cuda_fail(err, "cudaMalloc(scratch)");
            }
            e->scratch_cap = need;
        }
        scratch = e->scratch;
    }
    if (ov && ov->alloc_only) return XS_OK;
    char* base = static_cast<char*>(scratch);
    e->bound_rel = error_bound(kind, mixed);
    e->chk_rows = nchk;
    e->chk_ncond = ncond;
    double* chk_before = nchk ? reinterpret_cast<double*>(base + chk_off) : nullptr;
    double* chk_ref = nchk ? chk_before + size_t(32 * nchk) * size_t(ncond) : nullptr;
    double* chk_stats = nchk ? chk_ref + size_t(32 * nchk) * size_t(ncond) : nullptr;
    e->chk_stats = chk_stats;

    GridDev G;
    G.freq = grid->freq;
    G.f0 = 0.0;  // kernels read freq[0] on the device
    G.df = opt->dfreq;
    G.npoints_total = grid->npoints_total;
    G.start = grid->start_idx;
    G.points = grid->points;

    LinesDev L;
    L.nu = lines->nu;
    L.energies = lines->energies;
    L.aif = lines->aif;
    L.gamma = lines->gamma;
    L.nexp = lines->n;
    L.gns = lines->gns;
    L.n = n;
    L.s32 = streamed ? ov->s32 : nullptr;
    L.gl32 = streamed ? ov->gl32 : nullptr;
    L.tc_s = tc_mode ? ov->tc_s : nullptr;
    L.tc_pw = tc_mode ? ov->tc_pw : nullptr;
    L.tc_mode = tc_mode;

    const cudaStream_t st = e->stream;
    if (h2d_pieces && !e->copy_stream) {
        XS_CU(cudaStreamCreateWithFlags(&e->copy_stream, cudaStreamNonBlocking));
        for (auto& ev : e->pev) XS_CU(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    const bool timing = !(ov && ov->no_timing);
    // Inside a stream capture the timing events must become event-record
    // nodes of the graph (cudaEventRecordExternal); outside one, a plain
    // record (the external flag is refused there).
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
        cudaGetLastError();
        cap = cudaStreamCaptureStatusNone;
    }
    const unsigned ev_flags = (cap == cudaStreamCaptureStatusActive) ? cudaEventRecordExternal : 0u;
    cudaError_t err = launch_grid_check(G, words, st);
    if (err != cudaSuccess) return cuda_fail(err, "grid check launch");
    int launched = G.npoints_total >= 2 ? 1 : 0;

    for (int c0 = 0; c0 < ncond; c0 += group) {
        const int nc = std::min(group, ncond - c0);
        PrepArgs pa;
        std::memset(&pa, 0, sizeof(pa));
        pa.L = L;
        pa.G = G;
        pa.ncond = nc;
        for (int c = 0; c < nc; ++c) {
            pa.cond[c] = make_cond(*opt, conds[order[size_t(c0 + c)]]);
            if (ov && ov->use_consts) {
                pa.cond[c].cmcoef = ov->cmcoef;
                pa.cond[c].beta = ov->beta;
            }
        }
        // temperature classes, numbered in order of first appearance
        pa.nclass = 0;
        for (int c = 0; c < nc; ++c) {
            pa.tclass[c] = -1;
            for (int t = 0; t < pa.nclass; ++t) {
                const CondDev& x = pa.cond[c];
                const CondDev& y = pa.cond[pa.class_rep[t]];
                if (x.cmcoef == y.cmcoef && x.beta == y.beta && x.partition == y.partition &&
                    x.tratio == y.tratio && x.dpw == y.dpw) {
                    pa.tclass[c] = t;
                    break;
                }
            }
            if (pa.tclass[c] < 0) {
                pa.tclass[c] = pa.nclass;
                pa.class_rep[pa.nclass++] = c;
            }
        }
        pa.rec = base + plan.off_rec;
        pa.wlo = reinterpret_cast<int*>(base + plan.off_wlo);
        pa.whi = reinterpret_cast<int*>(base + plan.off_whi);
        pa.mi = reinterpret_cast<int*>(base + plan.off_mi);
        pa.kc = reinterpret_cast<int*>(base + plan.off_kc);
        pa.err = words;
        pa.half_width = opt->half_width;
        pa.x0 = opt->dfreq * 0.5;
        if (kind == XS_GAUSSIAN) {
            pa.xg = std::sqrt(kLN2) / opt->half_width;
            pa.x0g = pa.xg * opt->dfreq * 0.5;
        }
        pa.mixed_tile_span = CG ? 32 : 32 * P;
        pa.group = CG;
        pa.lsh = base + plan.off_lsh;
        pa.civ = reinterpret_cast<CoreIv*>(base + plan.off_civ);
        pa.cyp = reinterpret_cast<float2*>(base + plan.off_cyp);
        // window slots: groups with the same cut (consecutive) share the
        // first one's window data
        for (int g = 0; CG && g < nc / CG; ++g)
            pa.wslot[g] = (g > 0 && pa.cond[g * CG].cut == pa.cond[(g - 1) * CG].cut) ? pa.wslot[g - 1] : g;

        if (timing && c0 == 0) cudaEventRecordWithFlags(e->ev[0], st, ev_flags);
        err = cudaMemsetAsync(pa.kc, 0, sizeof(int) * size_t(kKcWords), st);
        if (err != cudaSuccess) return cuda_fail(err, "core-width reset");
        if (c0 == 0 && h2d_pieces > 0) {
            // host lines: slice k is copied on the copy stream (after the
            // work already on this stream, which may still read the device
            // lines) and step one starts on it when its copy is done
            err = cudaEventRecord(e->pev[kMaxPieces], st);
            if (err == cudaSuccess) err = cudaStreamWaitEvent(e->copy_stream, e->pev[kMaxPieces], 0);
            const size_t total = lines->count;
            for (int k = 0; k < h2d_pieces && err == cudaSuccess; ++k) {
                const size_t a0 = total * size_t(k) / size_t(h2d_pieces);
                const size_t a1 = total * size_t(k + 1) / size_t(h2d_pieces);
                if (a1 <= a0) continue;
                auto cp = [&](const void* dst, const void* src, size_t elem) {
                    if (err == cudaSuccess && src && dst)
                        err = cudaMemcpyAsync(static_cast<char*>(const_cast<void*>(dst)) + a0 * elem,
                                              static_cast<const char*>(src) + a0 * elem, (a1 - a0) * elem,
                                              cudaMemcpyHostToDevice, e->copy_stream);
                };
                const xs_lines* hl = ov->h2d;
                cp(lines->nu, hl->nu, sizeof(double));
                cp(lines->energies, hl->energies, sizeof(double));
                cp(lines->aif, hl->aif, sizeof(double));
                cp(lines->gns, hl->gns, sizeof(int));
                cp(lines->gamma, hl->gamma, sizeof(double));
                cp(lines->n, hl->n, sizeof(double));
                if (err == cudaSuccess) err = cudaEventRecord(e->pev[k], e->copy_stream);
                if (err == cudaSuccess) err = cudaStreamWaitEvent(st, e->pev[k], 0);
                // the lines step one evaluates stop at n (CPU coverage rule)
                pa.line0 = long(std::min(a0, size_t(n)));
                pa.line1 = long(std::min(a1, size_t(n)));
                if (err == cudaSuccess && pa.line1 > pa.line0) {
                    err = launch_prep(kind, opt->convention, mixed, pa, st);
                    ++launched;
                }
            }
            pa.line0 = pa.line1 = 0;
            if (err != cudaSuccess) return cuda_fail(err, "host lines: copy or step one");
        } else {
            err = launch_prep(kind, opt->convention, mixed, pa, st);
            if (err != cudaSuccess) return cuda_fail(err, "step one launch");
            ++launched;
        }
        if (timing && c0 == 0) cudaEventRecordWithFlags(e->ev[1], st, ev_flags);

        StepArgs sa;
        std::memset(&sa, 0, sizeof(sa));
        sa.rec = pa.rec;
        sa.wlo = pa.wlo;
        sa.whi = pa.whi;
        sa.mi = pa.mi;
        sa.kc = pa.kc;
        sa.n = n;
        sa.out = out;
        sa.out_stride = out_stride;
        for (int c = 0; c < nc; ++c) sa.row[c] = order[size_t(c0 + c)];
        sa.G = G;
        sa.tiles_per_cond = (grid->points + 32 * P - 1) / (32 * P);
        sa.n_items = sa.tiles_per_cond * nc * S;
        sa.counter = words + 1;
        sa.splits = S;
        sa.part = S > 1 ? reinterpret_cast<double*>(base + part_off) : nullptr;
        sa.part_stride = size_t(grid->points);
        sa.x0 = pa.x0;
        sa.xg = pa.xg;
        sa.x0g = pa.x0g;
        err = cudaMemsetAsync(sa.counter, 0, sizeof(unsigned), st);
        if (err != cudaSuccess) return cuda_fail(err, "counter reset");
        for (int c = 0; c < nc; ++c) {
            const double k = 1.0 / pa.cond[c].dpw;
            sa.kx[c] = float(k);
            sa.kx2[c] = float(k * k);
        }
        if (CG) {
            sa.lsh = pa.lsh;
            for (int g = 0; g < nc / CG; ++g) sa.wslot[g] = pa.wslot[g];
            sa.group = CG;
            sa.tiles_per_cond = (grid->points + 31) / 32;
            sa.n_items = sa.tiles_per_cond * (nc / CG) * S;
        }
        CheckArgs ck;
        if (nchk) {
            std::memset(&ck, 0, sizeof(ck));
            ck.L = L;
            ck.G = G;
            ck.ncond = nc;
            ck.conv = opt->convention;
            for (int c = 0; c < nc; ++c) {
                ck.cond[c] = pa.cond[c];
                ck.row[c] = sa.row[c];
            }
            ck.out = out;
            ck.out_stride = out_stride;
            ck.nrows = nchk;
            for (int k = 0; k < nchk; ++k) {
                // evenly spaced rows of 32 points inside the chunk
                const long mid = long(grid->points) * (2 * k + 1) / (2 * nchk);
                long r0 = long(grid->start_idx) + mid - 16;
                if (r0 > long(grid->start_idx) + grid->points - 32) r0 = long(grid->start_idx) + grid->points - 32;
                if (r0 < grid->start_idx) r0 = grid->start_idx;
                ck.rows[k] = int(r0);
            }
            ck.before = chk_before + size_t(32 * nchk) * size_t(c0);
            ck.ref = chk_ref + size_t(32 * nchk) * size_t(c0);
            ck.stats = chk_stats + size_t(4) * size_t(c0);
            err = launch_check_snapshot(ck, st);
            if (err != cudaSuccess) return cuda_fail(err, "check snapshot launch");
            ++launched;
        }
        const long want = (long(sa.n_items) + W - 1) / W;
        const int blocks = int(std::min<long>(want, long(occ) * e->num_sms));
        err = CG ? launch_steptwo_mc(mixed, CG, W, blocks, sa, st)
                : launch_steptwo(kind, opt->convention, mixed, P, W, blocks, sa, st);
        if (err != cudaSuccess) return cuda_fail(err, "step two launch");
        if (blocks > 0 && sa.n_items > 0) ++launched;
        if (CG && mixed) {
            // the pairs inside the lines' region intervals (W4 regions II-IV),
            // into the split parts before they are added up
            CoreArgs ca;
            std::memset(&ca, 0, sizeof(ca));
            ca.civ = pa.civ;
            ca.cyp = pa.cyp;
            ca.lsh = static_cast<const LineShX*>(pa.lsh);
            ca.rec = pa.rec;
            ca.mi = pa.mi;
            ca.kc = pa.kc;
            ca.freq = G.freq;
            ca.n = n;
            ca.group = CG;
            ca.G = G;
            ca.out = out;
            ca.out_stride = out_stride;
            ca.splits = S;
            ca.part = sa.part;
            ca.part_stride = sa.part_stride;
            for (int c = 0; c < nc; ++c) {
                ca.kx[c] = sa.kx[c];
                ca.kx2[c] = sa.kx2[c];
                ca.row[c] = sa.row[c];
            }
            for (int g = 0; g < nc / CG; ++g) ca.wslot[g] = pa.wslot[g];
            err = launch_core_mcx(ca, nc, st);
            if (err != cudaSuccess) return cuda_fail(err, "core pass launch");
            ++launched;
        } else if (mixed) {
            // single-condition layout: the pairs inside the records' region
            // intervals (W4 regions II-IV), into the split parts if any
            err = launch_core_v32(sa, nc, st);
            if (err != cudaSuccess) return cuda_fail(err, "core pass launch");
            ++launched;
        }
        err = launch_reduce_splits(sa, nc, st);
        if (err != cudaSuccess) return cuda_fail(err, "split reduction launch");
        if (S > 1) ++launched;
        if (timing && c0 + nc >= ncond) {
            cudaEventRecordWithFlags(e->ev[2], st, ev_flags);
            e->timed = true;
        }
        if (nchk) {  // after the timed kernels: the check is not step two
            err = launch_check_rows(ck, st);
            if (err != cudaSuccess) return cuda_fail(err, "check launch");
            launched += 2;
        }
    }
    if (ov) ov->kernels += launched;
    return XS_OK;
}

int engine_reserve(xs_engine* e, size_t bytes) {
    if (!e) return fail(XS_ERR_INVALID, "engine_reserve: NULL engine");
    std::lock_guard<std::mutex> lk(e->mu);
    if (bytes <= e->scratch_cap) return XS_OK;
    DeviceGuard dg(e->device);
    XS_CU(cudaStreamSynchronize(e->stream));
    cudaFree(e->scratch);
    e->scratch = nullptr;
    e->scratch_cap = 0;
    cudaError_t err = cudaMalloc(&e->scratch, bytes);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(err, "cudaMalloc(scratch)");
    }
    e->scratch_cap = bytes;
    return XS_OK;
}

int engine_device(const xs_engine* e) { return e ? e->device : -1; }
void* engine_stream(const xs_engine* e) { return e ? static_cast<void*>(e->stream) : nullptr; }

}  // namespace xs

struct xs_graph {
    xs_engine* e = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

extern "C" {

int xs_engine_capture(xs_engine* e, const xs_options* opt, const xs_condition* conds, int ncond,
                      const xs_lines* lines, const xs_grid* grid, double* out, size_t out_stride,
                      int zero_out, xs_graph** out_graph) {
    if (!e || !out_graph || !grid || !out) return fail(XS_ERR_INVALID, "xs_engine_capture: NULL argument");
    *out_graph = nullptr;
    // Grow the scratch outside the capture (allocation is not a stream op).
    xs::ExecOverride pre;
    pre.alloc_only = true;
    int rc = xs::engine_execute(e, opt, conds, ncond, lines, grid, out, out_stride, &pre);
    if (rc) return rc;
    DeviceGuard dg(e->device);
    cudaStream_t cs = nullptr;
    XS_CU(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaStream_t saved;
    {
        std::lock_guard<std::mutex> lk(e->mu);
        saved = e->stream;
        e->stream = cs;
    }
    cudaGraph_t graph = nullptr;
    cudaError_t err = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (err == cudaSuccess && zero_out && grid->points > 0) {
        const size_t rows = size_t(ncond);
        const size_t pitch = (ncond > 1 ? out_stride : size_t(grid->npoints_total)) * sizeof(double);
        err = cudaMemset2DAsync(out + grid->start_idx, pitch, 0, size_t(grid->points) * sizeof(double),
                                rows, cs);
    }
    if (err == cudaSuccess) rc = xs::engine_execute(e, opt, conds, ncond, lines, grid, out, out_stride, nullptr);
    cudaError_t end = cudaStreamEndCapture(cs, &graph);
    {
        std::lock_guard<std::mutex> lk(e->mu);
        e->stream = saved;
    }
    cudaStreamDestroy(cs);
    if (err != cudaSuccess || end != cudaSuccess || rc != XS_OK) {
        if (graph) cudaGraphDestroy(graph);
        if (rc != XS_OK) return rc;
        return cuda_fail(err != cudaSuccess ? err : end, "stream capture");
    }
    auto* g = new xs_graph();
    g->e = e;
    g->graph = graph;
    err = cudaGraphInstantiate(&g->exec, graph, 0);
    if (err != cudaSuccess) {
        cudaGraphDestroy(graph);
        delete g;
        return cuda_fail(err, "cudaGraphInstantiate");
    }
    *out_graph = g;
    return XS_OK;
}

int xs_graph_launch(xs_graph* g, void* stream) {
    if (!g) return fail(XS_ERR_INVALID, "xs_graph_launch: NULL graph");
    DeviceGuard dg(g->e->device);
    XS_CU(cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream)));
    return XS_OK;
}

int xs_graph_kernel_count(const xs_graph* g, int* kernels) {
    if (!g || !kernels) return fail(XS_ERR_INVALID, "xs_graph_kernel_count: NULL argument");
    size_t n = 0;
    XS_CU(cudaGraphGetNodes(g->graph, nullptr, &n));
    std::vector<cudaGraphNode_t> nodes(n);
    if (n > 0) XS_CU(cudaGraphGetNodes(g->graph, nodes.data(), &n));
    int k = 0;
    for (cudaGraphNode_t node : nodes) {
        cudaGraphNodeType t;
        XS_CU(cudaGraphNodeGetType(node, &t));
        if (t == cudaGraphNodeTypeKernel) ++k;
    }
    *kernels = k;
    return XS_OK;
}

int xs_graph_destroy(xs_graph* g) {
    if (!g) return XS_OK;
    DeviceGuard dg(g->e->device);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return XS_OK;
}

}  // extern "C"

extern "C" {

int xs_engine_autotune(xs_engine* e, const xs_options* opt, const xs_condition* conds, int ncond,
                       const xs_lines* lines, const xs_grid* grid, double* out, size_t out_stride,
                       xs_tune_result* best) {
    if (!e || !opt || !conds || !lines || !grid || !out || ncond < 1)
        return fail(XS_ERR_INVALID, "xs_engine_autotune: NULL argument");
    const int kind = opt->profile;
    const bool mixed = kind == XS_VOIGT && opt->precision == XS_MIXED;
    struct Cand {
        int P, W, C;
    };
    std::vector<Cand> cands;
    const int Ps[4] = {1, 2, 4, 8};
    for (int W : {4, 8}) {
        for (int P : Ps) {
            if (kind != XS_VOIGT && P > 2) continue;
            if (kind == XS_VOIGT && !mixed && P > 4) continue;
            cands.push_back({P, W, kind == XS_VOIGT ? 1 : 0});
        }
        if (kind == XS_VOIGT && ncond > 1)
            for (int C : {2, 4, 8})
                if (ncond % C == 0 && ncond <= kMaxCond) cands.push_back({1, W, C});
    }
    long n = long(lines->count);
    if (opt->convention == XS_CONV_CPU) n = cpu_covered_lines(n, opt->cpu_threads);
    Shape pick{0, 0, 0, 1e300};
    for (const Cand& c : cands) {
        xs_options o = *opt;
        o.points_per_thread = c.P;
        o.warps_per_block = c.W;
        o.conditions_per_warp = c.C;
        o.check_rows = 0;  // time the computation alone
        double ms = 1e300;
        for (int rep = 0; rep < 2; ++rep) {
            int rc = xs::engine_execute(e, &o, conds, ncond, lines, grid, out, out_stride, nullptr);
            if (rc == XS_ERR_INVALID) break;  // a shape this call cannot take (e.g. unequal cuts)
            if (rc != XS_OK) return rc;
            rc = xs_engine_sync(e);
            if (rc != XS_OK) return rc;
            double pm = 0.0, sm = 0.0;
            rc = xs_engine_last_stats(e, &pm, &sm);
            if (rc != XS_OK) return rc;
            ms = pm + sm;  // the second run is the one kept (the first warms up)
        }
        if (ms < pick.ms) pick = Shape{c.P, c.W, c.C, ms};
    }
    if (pick.P == 0) return fail(XS_ERR_INVALID, "xs_engine_autotune: no launch shape fits this call");
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[shape_key(*opt, conds, ncond, n, grid->points)] = pick;
    }
    if (best) {
        best->points_per_thread = pick.P;
        best->warps_per_block = pick.W;
        best->conditions_per_warp = pick.C;
        best->ms = pick.ms;
        best->candidates = int(cands.size());
    }
    return XS_OK;
}

int xs_tune_save(const char* path) {
    if (!path) return fail(XS_ERR_INVALID, "xs_tune_save: NULL path");
    std::lock_guard<std::mutex> lk(g_tune_mu);
    FILE* f = std::fopen(path, "w");
    if (!f) return fail(XS_ERR_INVALID, std::string("xs_tune_save: cannot write ") + path);
    for (const auto& kv : g_tune)
        std::fprintf(f, "%s %d %d %d %.6f\n", kv.first.c_str(), kv.second.P, kv.second.W, kv.second.C,
                     kv.second.ms);
    std::fclose(f);
    return XS_OK;
}

int xs_tune_load(const char* path) {
    if (!path) return fail(XS_ERR_INVALID, "xs_tune_load: NULL path");
    FILE* f = std::fopen(path, "r");
    if (!f) return fail(XS_ERR_INVALID, std::string("xs_tune_load: cannot read ") + path);
    char key[96];
    Shape sh{};
    std::lock_guard<std::mutex> lk(g_tune_mu);
    while (std::fscanf(f, "%95s %d %d %d %lf", key, &sh.P, &sh.W, &sh.C, &sh.ms) == 5) {
        const bool ok = (sh.P == 1 || sh.P == 2 || sh.P == 4 || sh.P == 8) && (sh.W == 4 || sh.W == 8) &&
                        (sh.C == 0 || sh.C == 1 || sh.C == 2 || sh.C == 4 || sh.C == 8);
        if (ok) g_tune[key] = sh;
    }
    std::fclose(f);
    return XS_OK;
}

int xs_tune_clear(void) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.clear();
    return XS_OK;
}

}  // extern "C"
