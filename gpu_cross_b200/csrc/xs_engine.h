// Internal engine entry shared by the C ABI files (launcher and manager
// levels).  Not part of the public ABI.
#pragma once

#include <cstddef>

#include "xsec_b200.h"

namespace xs {

struct CondDev;

// Optional knobs of one execute call.
struct ExecOverride {
    void* scratch = nullptr;      // caller-provided scratch area (device)
    size_t scratch_bytes = 0;
    unsigned* words = nullptr;    // caller-provided error word + counter (device)
    bool no_timing = false;       // skip the CUDA events
    bool alloc_only = false;      // only grow the engine scratch, launch nothing
    bool use_consts = false;      // take cmcoef and beta from below instead of
    double cmcoef = 0.0;          //   recomputing them from T (launcher level:
    double beta = 0.0;            //   the cross_section_data the caller copied)
    const float* s32 = nullptr;   // streamed Voigt lines: S(T) and gamma(T, P)
    const float* gl32 = nullptr;  //   per line (see LinesDev)
    // Line list in host memory, copied to the call's (device) lines in
    // h2d_pieces slices on the engine's copy stream; step one starts on each
    // slice as its copy completes.
    const xs_lines* h2d = nullptr;
    int h2d_pieces = 0;
    double* tc_s = nullptr;       // per-temperature cache of S(T) and
    double* tc_pw = nullptr;      //   (T_ref/T)^n (one condition; see
    int tc_mode = 0;              //   LinesDev)
    mutable int kernels = 0;      // out: kernels the call launched (added to)
};

int engine_execute(xs_engine* e, const xs_options* opt, const xs_condition* conds, int ncond,
                   const xs_lines* lines, const xs_grid* grid, double* out, size_t out_stride,
                   const ExecOverride* ov);

// Grows the engine's scratch to at least `bytes` (synchronises the engine's
// stream when it has to reallocate).
int engine_reserve(xs_engine* e, size_t bytes);
// The engine's device and stream.
int engine_device(const xs_engine* e);
void* engine_stream(const xs_engine* e);

int set_error(int code, const char* msg);
CondDev make_cond(const xs_options& o, const xs_condition& c);
long cpu_covered_lines(long n, int threads);

}  // namespace xs
