// Allocation-free entry point: xs_execute_noalloc.
//
// Some callers cannot let this library call cudaMalloc.  A host that has
// already handed (nearly) all device memory to its own pool allocator would
// see the allocation fail or eat into its pool, and a latency-critical loop
// cannot afford the implicit device-wide synchronisation that cudaMalloc and
// cudaFree may cause.  xs_execute_noalloc runs the same kernels as
// xs_engine_execute -- grid check, step one, persistent step two, and in
// mixed precision the core pass -- for one condition, but takes its scratch
// (per-line records and windows, the error word and the work counter) from
// one fixed array compiled into the library,
// g_noalloc_scratch below.  It allocates nothing: no cudaMalloc, no cudaFree,
// no engine, no events, no library routine that allocates.
//
// The array is a file-scope __device__ variable, so every GPU that loads the
// library holds its kXsNoAllocScratchBytes until the process exits.  In host
// code its name is only a host-side stand-in: the device address comes from
// cudaGetSymbolAddress, with the device current.  Every call looks it up
// again (a host-side lookup that allocates nothing), so nothing cached goes
// stale when the caller resets the device or its primary context is torn
// down and recreated between calls.  The first call on a device may load the
// library's device code there, so it should come before any stream capture
// on that device.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>

#include "xs_engine.h"
#include "xs_internal.cuh"
#include "xsec_b200.h"

namespace {

constexpr size_t kXsNoAllocScratchBytes = size_t(XS_NOALLOC_SCRATCH_BYTES);
// First 256 bytes: [0] error bits, [1] work counter; the rest: records,
// windows, line grid indices and core widths, each section 256-byte aligned.
constexpr size_t kHeaderBytes = 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kXsNoAllocScratchBytes];

int noalloc_fail(int code, const char* msg) { return xs::set_error(code, msg); }

}  // namespace

extern "C" int xs_execute_noalloc(const xs_options* opt, const xs_condition* cond,
                                  const xs_lines* lines, const xs_grid* grid, double* out,
                                  void* stream) {
    if (!opt || !cond || !lines || !grid || !out)
        return noalloc_fail(XS_ERR_INVALID, "xs_execute_noalloc: NULL argument");
    const int kind = opt->profile;
    if (kind != XS_VOIGT && kind != XS_DOPPLER && kind != XS_GAUSSIAN)
        return noalloc_fail(XS_ERR_UNSUPPORTED, "xs_execute_noalloc: profile not supported");
    if (opt->convention != XS_CONV_GPU && opt->convention != XS_CONV_CPU)
        return noalloc_fail(XS_ERR_INVALID, "xs_execute_noalloc: unknown convention");
    if (kind == XS_GAUSSIAN && opt->convention == XS_CONV_CPU)
        return noalloc_fail(XS_ERR_UNSUPPORTED, "xs_execute_noalloc: no CPU-convention GAUSSIAN");
    if (opt->precision != XS_FP64 && opt->precision != XS_MIXED)
        return noalloc_fail(XS_ERR_INVALID, "xs_execute_noalloc: unknown precision");
    if (!(opt->dfreq > 0.0) || !(cond->temperature > 0.0) ||
        (kind != XS_GAUSSIAN && !(opt->mean_mass > 0.0)) ||
        (kind == XS_GAUSSIAN && !(opt->half_width > 0.0)))
        return noalloc_fail(XS_ERR_INVALID, "xs_execute_noalloc: bad constants");
    if (!grid->freq || grid->npoints_total < 1 || grid->start_idx < 0 || grid->points < 0 ||
        long(grid->start_idx) + long(grid->points) > long(grid->npoints_total))
        return noalloc_fail(XS_ERR_INVALID, "xs_execute_noalloc: grid chunk outside the grid");
    if (lines->count > 0 && (!lines->nu || !lines->energies || !lines->aif || !lines->gns ||
                             (kind == XS_VOIGT && (!lines->gamma || !lines->n))))
        return noalloc_fail(XS_ERR_INVALID, "xs_execute_noalloc: line arrays missing");
    const bool mixed = kind == XS_VOIGT && opt->precision == XS_MIXED;
    if (mixed && double(grid->npoints_total) > 15.0e6)
        return noalloc_fail(XS_ERR_UNSUPPORTED, "xs_execute_noalloc: grid too large for mixed");

    long n = long(lines->count);
    if (opt->convention == XS_CONV_CPU) n = xs::cpu_covered_lines(n, opt->cpu_threads);

    // Size check against the fixed array, before touching the device.
    const size_t nl = size_t(n > 0 ? n : 0);
    const xs::ScratchPlan plan = xs::plan_scratch(kind, mixed, nl, 1, kHeaderBytes);
    const size_t need = plan.need;
    if (need > kXsNoAllocScratchBytes) {
        const size_t per = xs::record_bytes(kind, mixed) + 3 * sizeof(int);
        char msg[256];
        std::snprintf(msg, sizeof(msg),
                      "xs_execute_noalloc: %zu lines need %zu scratch bytes; the fixed array holds "
                      "%zu bytes (at most about %zu lines for this profile and precision)",
                      nl, need, kXsNoAllocScratchBytes,
                      (kXsNoAllocScratchBytes - kHeaderBytes - 4 * 256) / per);
        return noalloc_fail(XS_ERR_INVALID, msg);
    }

    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        cudaGetLastError();
        return noalloc_fail(XS_ERR_NODEVICE, "xs_execute_noalloc: no current CUDA device");
    }
    int major = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
        major != 10)
        return noalloc_fail(XS_ERR_NODEVICE, "xs_execute_noalloc: the kernels are built for sm_100a");

    // The device address of the fixed array on this (current) device, looked
    // up on every call: after a device reset the module is loaded again and
    // the array may sit elsewhere.
    void* base_ptr = nullptr;
    {
        const cudaError_t e = cudaGetSymbolAddress(&base_ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !base_ptr) {
            cudaGetLastError();
            return noalloc_fail(XS_ERR_CUDA, "xs_execute_noalloc: cudaGetSymbolAddress failed");
        }
    }
    if (n <= 0 || grid->points <= 0) return XS_OK;

    char* base = static_cast<char*>(base_ptr);
    unsigned* words = reinterpret_cast<unsigned*>(base);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);

    int P = opt->points_per_thread, W = opt->warps_per_block;
    if (P == 0) P = (kind == XS_VOIGT) ? (mixed ? 4 : 2) : 1;
    if (W == 0) W = 8;
    if (kind == XS_VOIGT ? !(P == 1 || P == 2 || P == 4 || P == 8) : !(P == 1 || P == 2))
        return noalloc_fail(XS_ERR_INVALID, "xs_execute_noalloc: points_per_thread");
    if (W != 4 && W != 8) return noalloc_fail(XS_ERR_INVALID, "xs_execute_noalloc: warps_per_block");

    xs::GridDev G;
    G.freq = grid->freq;
    G.f0 = 0.0;
    G.df = opt->dfreq;
    G.npoints_total = grid->npoints_total;
    G.start = grid->start_idx;
    G.points = grid->points;

    xs::PrepArgs pa;
    std::memset(&pa, 0, sizeof(pa));
    pa.L.nu = lines->nu;
    pa.L.energies = lines->energies;
    pa.L.aif = lines->aif;
    pa.L.gamma = lines->gamma;
    pa.L.nexp = lines->n;
    pa.L.gns = lines->gns;
    pa.L.n = n;
    pa.G = G;
    pa.ncond = 1;
    pa.cond[0] = xs::make_cond(*opt, *cond);
    pa.rec = base + plan.off_rec;
    pa.wlo = reinterpret_cast<int*>(base + plan.off_wlo);
    pa.whi = reinterpret_cast<int*>(base + plan.off_whi);
    pa.mi = reinterpret_cast<int*>(base + plan.off_mi);
    pa.kc = reinterpret_cast<int*>(base + plan.off_kc);
    pa.err = words;
    pa.half_width = opt->half_width;
    pa.x0 = opt->dfreq * 0.5;
    if (kind == XS_GAUSSIAN) {
        pa.xg = std::sqrt(xs::kLN2) / opt->half_width;
        pa.x0g = pa.xg * opt->dfreq * 0.5;
    }
    pa.mixed_tile_span = 32 * P;

    xs::StepArgs sa;
    std::memset(&sa, 0, sizeof(sa));
    sa.rec = pa.rec;
    sa.wlo = pa.wlo;
    sa.whi = pa.whi;
    sa.mi = pa.mi;
    sa.kc = pa.kc;
    sa.n = n;
    sa.out = out;
    sa.out_stride = 0;
    sa.G = G;
    sa.tiles_per_cond = (grid->points + 32 * P - 1) / (32 * P);
    sa.n_items = sa.tiles_per_cond;
    sa.splits = 1;  // the fixed array holds no split parts
    sa.counter = words + 1;
    sa.x0 = pa.x0;
    sa.xg = pa.xg;
    sa.x0g = pa.x0g;
    sa.kx[0] = float(1.0 / pa.cond[0].dpw);

    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return noalloc_fail(XS_ERR_CUDA, "xs_execute_noalloc: device attribute");
    int occ = xs::steptwo_blocks_per_sm(kind, opt->convention, mixed, P, W);
    if (occ < 1) occ = 1;
    const long want = (long(sa.n_items) + W - 1) / W;
    const int blocks = int(want < long(occ) * sms ? want : long(occ) * sms);

    // The array keeps the previous call's contents: the error word, the
    // work counter and the core widths must start at zero; records, windows
    // and grid indices are rewritten.
    cudaError_t e = cudaMemsetAsync(words, 0, 2 * sizeof(unsigned), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(pa.kc, 0, sizeof(int) * size_t(xs::kKcWords), st);
    if (e == cudaSuccess) e = xs::launch_grid_check(G, words, st);
    if (e == cudaSuccess) e = xs::launch_prep(kind, opt->convention, mixed, pa, st);
    if (e == cudaSuccess) e = xs::launch_steptwo(kind, opt->convention, mixed, P, W, blocks, sa, st);
    if (e == cudaSuccess && mixed) e = xs::launch_core_v32(sa, 1, st);  // W4 regions II-IV
    // Wait for this call's kernels and report what they found.
    unsigned bits = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bits, words, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return noalloc_fail(XS_ERR_CUDA, cudaGetErrorString(e));
    }
    if (bits & xs::kErrUnsorted)
        return noalloc_fail(XS_ERR_UNSORTED, "xs_execute_noalloc: line centres not ascending");
    if (bits & xs::kErrGrid)
        return noalloc_fail(XS_ERR_GRID, "xs_execute_noalloc: grid not ascending/uniform");
    if (bits & xs::kErrReach)
        return noalloc_fail(XS_ERR_UNSUPPORTED, "xs_execute_noalloc: a line's core lies too far from "
                                                "its centre's grid index for mixed precision");
    return XS_OK;
}
