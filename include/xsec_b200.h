/*
 * xsec_b200 -- C ABI of the B200 cross-section engine.
 *
 * sigma(f_j) = sum_i S_i(T) * Phi_i(f_j - nu_i; T, P) over |f_j - nu_i| <= cut,
 * for Doppler, Gaussian and Voigt (Humlicek W4) line profiles on a uniform
 * wavenumber grid, computed by hand-written sm_100a kernels.
 *
 * Three levels, all plain C (pointers, sizes, int status codes; no C++ or
 * torch types):
 *
 *  1. Launcher level -- drop-in replacements for the reference's host
 *     launchers in cross_kernal.cuh (device pointers, default stream,
 *     constants set once per device).
 *  2. Engine level -- explicit handle, stream, profile, Doppler-width
 *     convention, precision (FP64 or mixed FP32/FP64) and batches of (T, P)
 *     conditions over one resident line list.
 *  3. Manager level -- the reference's BaseManager interface
 *     (BaseManager.h:22-30) over host buffers; the C++ classes in
 *     include/xsec/ (GpuManager, OpenMPManager, ...) sit on these calls.
 *
 * Every call returns XS_OK (0) or an XS_ERR_* code; xs_last_error() gives a
 * message for the calling thread.  Nothing here falls back to the CPU: a
 * machine without a usable sm_100 device gets XS_ERR_CUDA / XS_ERR_NODEVICE.
 */
#ifndef XSEC_B200_H
#define XSEC_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define XS_OK 0
#define XS_ERR_INVALID 1   /* bad argument or size */
#define XS_ERR_CUDA 2      /* a CUDA runtime call failed */
#define XS_ERR_NOMEM 3     /* device allocation failed / over budget */
#define XS_ERR_UNSORTED 4  /* line centres not ascending (the reference requires it) */
#define XS_ERR_GRID 5      /* grid not ascending or not uniform */
#define XS_ERR_STATE 6     /* call out of order (e.g. execute before upload) */
#define XS_ERR_NODEVICE 7  /* no usable sm_100 device */
#define XS_ERR_TIMEOUT 8   /* a bounded device-side wait ran out */
#define XS_ERR_UNSUPPORTED 9

/* ---- enums -------------------------------------------------------------- */
/* ProfileType, Input.h:9-15 (same order and values). */
#define XS_GAUSSIAN 0
#define XS_DOPPLER 1
#define XS_VOIGT 2
#define XS_PSUEDO_VOIGT 3

/* Which reference backend's arithmetic to reproduce.
 * XS_CONV_GPU: cross_kernal.cu -- Doppler width sqrt(2kT N_A/M)/c, window
 *   -cut <= nu - f <= cut, cut = min(25 P, 100) (Voigt) or 100 (Doppler).
 * XS_CONV_CPU: OpenMPManager.cpp -- width with an extra sqrt(ln 2), window
 *   [round((nu-cut-f0)/df), round((nu+cut-f0)/df)) clamped to the chunk. */
#define XS_CONV_GPU 0
#define XS_CONV_CPU 1

/* XS_FP64: every operation in double (matches the reference to <= 1e-10).
 * XS_MIXED: Voigt profile evaluation and accumulation in FP32 (compensated
 * per tile), line-centre offsets, intensities and the final per-tile sum in
 * FP64; Doppler and Gaussian stay FP64. */
#define XS_FP64 0
#define XS_MIXED 1

/* cross_section_data, cross_structs.cuh:3-17 (same fields, same order). */
typedef struct {
    double halfwidth;
    double mean_mass;
    double temperature;
    double pressure;
    double beta;
    double partition;
    double ln2;
    double ref_temp;
    double cmcoef;
    double dfreq;
} xs_cross_section_data;

/* One (T, P) condition of a run or sweep. */
typedef struct {
    double temperature;  /* K */
    double partition;    /* Q(T) */
    double pressure;     /* atm; sets the reference Voigt cut min(25 P, 100) */
    double gamma_scale;  /* multiplies the uploaded gamma (1.0 when gamma is
                            already pressure-scaled, as the readers do) */
    double cut;          /* > 0: window half width in cm-1; <= 0: reference rule */
} xs_condition;

/* Run options shared by all conditions of one call. */
typedef struct {
    int profile;      /* XS_DOPPLER / XS_VOIGT / XS_GAUSSIAN */
    int convention;   /* XS_CONV_GPU / XS_CONV_CPU */
    int precision;    /* XS_FP64 / XS_MIXED */
    int cpu_threads;  /* XS_CONV_CPU only: the OpenMPManager thread count; it
                         decides which lines the reference covers (blocks of
                         ceil(float(N)/float(threads)), OpenMPManager.cpp:186) */
    double mean_mass; /* amu */
    double ref_temp;  /* K, gamma(T) = gamma * (ref_temp / T)^n */
    double half_width;/* GAUSSIAN HWHM */
    double dfreq;     /* grid step (the reference's cross_constants.dfreq) */
    int points_per_thread; /* 0 = autotuned; else 1, 2, 4 or 8 */
    int warps_per_block;   /* 0 = autotuned; else 4 or 8 */
    int conditions_per_warp; /* VOIGT batches: 0 = automatic, 1 = one condition
                                per warp, 2/4/8 = that many conditions with the
                                same cut evaluated together by each warp */
    int line_splits;  /* 0 = automatic: when a call has too few grid tiles to
                         fill the GPU (short or coarse grids over many lines),
                         each tile's lines are split over up to 64 warps whose
                         partial sums are added in a fixed order; 1 = never;
                         N = N parts per tile.  The choice depends only on the
                         call's sizes and the device's SM count. */
    int check_rows;   /* XS_MIXED Voigt: 0 = no check; k > 0 = after the call,
                         re-evaluate k evenly spaced rows of 32 grid points
                         per condition (at most 16) in FP64 and compare
                         (xs_engine_accuracy). */
} xs_options;

/* Device-resident line list (structure of arrays, ascending nu). */
typedef struct {
    const double* nu;
    const double* energies; /* lower-state energy E'' (cm-1) */
    const double* aif;      /* Einstein A (s-1) */
    const int* gns;         /* upper-state degeneracy */
    const double* gamma;    /* Lorentz HWHM (cm-1); may be NULL unless VOIGT */
    const double* n;        /* temperature exponent; may be NULL unless VOIGT */
    size_t count;
} xs_lines;

/* Device grid: the reference's f_j = f0 + j*df array (BaseProfile.cpp:19). */
typedef struct {
    const double* freq;     /* npoints_total values, ascending, uniform step dfreq */
    int npoints_total;
    int start_idx;          /* first point of the chunk evaluated */
    int points;             /* points in the chunk */
} xs_grid;

typedef struct xs_engine xs_engine;

/* ---- general ------------------------------------------------------------ */
const char* xs_last_error(void);
const char* xs_version(void);
/* 1 if a usable sm_100 device is present (no context is created otherwise). */
int xs_device_available(void);
/* Number of visible CUDA devices (0 when there is no driver or device).  The
 * reference's MultiGpuManager (MultiGPUManager.cpp:5-16) makes one manager per
 * device; xs_manager_create reports XS_ERR_NODEVICE for a device that is not
 * sm_100. */
int xs_device_count(int* count);

/* ---- 1. launcher level: drop-in for cross_kernal.cuh -------------------- */
/* copy_intensity_info (cross_kernal.cuh:18): per-device constants used by the
 * launchers below (current device). */
int xs_copy_intensity_info(const xs_cross_section_data* cross_inf);
/* execute_two_step_kernal_voigt_block with gamma (cross_kernal.cuh:45):
 * g_intens[start_idx .. start_idx+Npoints) += Voigt sum over the first N_ener
 * lines, reference GPU convention, FP64, legacy default stream, asynchronous.
 * Unlike the reference, g_energies and g_gamma are not overwritten. */
int xs_execute_two_step_kernal_voigt_block(double* g_freq, double* g_intens, double* g_energies,
                                           double* g_nu, int* g_gns, double* g_aif,
                                           double* g_gamma, double* g_n, int Npoints, int N_ener,
                                           int start_idx);
/* execute_two_step_kernal_doppler_block (cross_kernal.cuh:52). */
int xs_execute_two_step_kernal_doppler_block(double* g_freq, double* g_intens,
                                             double* g_energies, double* g_nu, int* g_gns,
                                             double* g_aif, int Npoints, int N_ener,
                                             int start_idx);
/* execute_two_step_kernal_block (cross_kernal.cuh:35), GAUSSIAN with
 * ln2 = 0.69314718056 and the window |f - nu| <= 10 * halfwidth. */
int xs_execute_two_step_kernal_block(double* g_freq, double* g_intens, double* g_energies,
                                     double* g_nu, int* g_gns, double* g_aif, int Npoints,
                                     int N_ener, int start_idx);
/* Waits for the launcher-level work of the current device and reports
 * device-side errors (XS_ERR_UNSORTED, XS_ERR_GRID). */
int xs_launcher_sync(void);

/* ---- 2. engine level ---------------------------------------------------- */
int xs_engine_create(int device, xs_engine** out);
int xs_engine_destroy(xs_engine* e);
/* Stream for all later work of this engine (cudaStream_t; NULL = legacy). */
int xs_engine_set_stream(xs_engine* e, void* stream);
/* Waits for the engine's stream and reports device-side errors. */
int xs_engine_sync(xs_engine* e);
/* Device bytes held by the engine's scratch (records, windows, counters). */
int xs_engine_scratch_bytes(xs_engine* e, size_t* bytes);
/* Upper bound on scratch bytes xs_engine_execute needs for this shape. */
size_t xs_scratch_bytes_needed(const xs_options* opt, int ncond, size_t n_lines);

/* For each condition c: out[c*out_stride + j] += sigma_c(f_j) for j in
 * [grid.start_idx, grid.start_idx + grid.points).  With several conditions
 * out_stride must be at least grid.points (rows of a chunk-sized buffer are
 * addressed by passing out shifted back by start_idx elements).
 * Asynchronous on the engine's stream.  All pointers are device pointers. */
int xs_engine_execute(xs_engine* e, const xs_options* opt, const xs_condition* conds, int ncond,
                      const xs_lines* lines, const xs_grid* grid, double* out, size_t out_stride);

/* xs_engine_execute with the line list in host memory (pinned, for the
 * copies to overlap): host_lines is copied into dev_lines (the same count;
 * device arrays the call then evaluates, as in xs_engine_execute) in
 * `pieces` (1..16) slices on the engine's copy stream, and step one starts
 * on each slice as soon as its copy is done, so the copies overlap step one.
 * When host_out is not NULL, each condition's span [start_idx, start_idx +
 * points) of out is copied to the same place of host_out (rows out_stride
 * apart) after the call's work.  Asynchronous on the engine's stream:
 * xs_engine_sync before reading host_out or reusing the host arrays.  This is
 * the host-buffer form of the reference's GpuManager::TransferVectors ->
 * ExecuteCrossSection -> TransferResults sequence (GPUManager.cpp:87-106,
 * :107-121, :160-168). */
int xs_engine_execute_host(xs_engine* e, const xs_options* opt, const xs_condition* conds, int ncond,
                           const xs_lines* host_lines, const xs_lines* dev_lines, const xs_grid* grid,
                           double* out, size_t out_stride, double* host_out, int pieces);

/* Error statement of the last execute (or graph replay), against the FP64
 * arithmetic of the same reference convention (no counterpart in the
 * reference, which computes in FP64 only).
 *   bound_rel: a-priori bound on the relative error of every grid point of
 *     the result, and so of the band integral (every pair's true value is
 *     positive for non-negative intensities).  Mixed Voigt: 1024 * 2^-24 =
 *     6.1e-5, above the rounding-error analysis of the FP32 steps (region I:
 *     offset, u, u^2 + 2y^2, the shared reciprocal, 32-line FP32 partial sums
 *     folded with compensation, 76 * 2^-24; regions II-IV: the FP32 x and y
 *     through the profile's sensitivity, at most 2 x^2 = 60.5, the FP32 W4
 *     forms and, for several conditions at once, the region-I value that
 *     step two adds there and the core pass takes back, at most 1.21 W4 --
 *     about 690 * 2^-24).
 *     FP64 (every FP64 result, Doppler and Gaussian included): 1e-12,
 *     summation order only.
 *   sampled_*: with xs_options.check_rows > 0 (mixed Voigt), measured on
 *     the sampled rows of every condition -- the largest relative error on
 *     points above 1e-6 of the rows' FP64 peak, and the relative error of
 *     their sum -- as the worst over conditions; -1 when not measured.  What
 *     the call added is taken as out after minus out before the call.
 * Waits for the engine's stream. */
typedef struct {
    double bound_rel;
    double sampled_max_rel;
    double sampled_integrated_rel;
    int sampled_rows;  /* rows per condition measured (0: none) */
    int conditions;
} xs_accuracy;
int xs_engine_accuracy(xs_engine* e, xs_accuracy* acc);
/* The a-priori bound alone (xs_accuracy.bound_rel) for a profile and
 * precision: 1024 * 2^-24 for XS_MIXED Voigt, 1e-12 otherwise. */
double xs_error_bound(int profile, int precision);

/* Device time (ms, CUDA events on the engine's stream) of the step-one
 * (prep) and step-two launches of the last execute; waits for them. */
int xs_engine_last_stats(xs_engine* e, double* prep_ms, double* steptwo_ms);

/* Captures one xs_engine_execute (optionally preceded by zeroing the output
 * rows of the chunk) into a CUDA graph: grid check, step one for every
 * condition and the persistent step two, replayed by xs_graph_launch on any
 * stream.  The engine's scratch is sized before the capture; the buffers
 * named here must stay valid while the graph is used.  xs_engine_last_stats
 * reports the device times of the most recent replay. */
typedef struct xs_graph xs_graph;
int xs_engine_capture(xs_engine* e, const xs_options* opt, const xs_condition* conds, int ncond,
                      const xs_lines* lines, const xs_grid* grid, double* out, size_t out_stride,
                      int zero_out, xs_graph** graph);
int xs_graph_launch(xs_graph* graph, void* stream);
/* Kernel launches one replay of the graph makes (its kernel nodes). */
int xs_graph_kernel_count(const xs_graph* graph, int* kernels);
int xs_graph_destroy(xs_graph* graph);

/* Measured throughput of this device's FP32 FMA and FP64 FMA pipes
 * (TFLOP/s) and of the FP32 reciprocal (MUFU, Tops/s); the roofline
 * denominators of the step-two kernels. */
int xs_measure_peaks(int device, double* fp32_tflops, double* fp64_tflops, double* rcp32_tops);

/* Autotuner: runs the call below once per candidate launch shape (points
 * per thread, warps per block, conditions per warp; each twice, the second
 * timed), keeps the fastest for calls of the same signature (profile,
 * convention, precision, condition count, and the binary magnitudes of the
 * grid points and of the lines per point), and reports it.  Later calls with
 * points_per_thread = warps_per_block = conditions_per_warp = 0 use it.  `out`
 * is accumulated into many times: clear it afterwards.  The table lives in
 * the process; xs_tune_save / xs_tune_load keep it in a text file. */
typedef struct {
    int points_per_thread, warps_per_block, conditions_per_warp;
    double ms;       /* step one + step two of the chosen shape */
    int candidates;  /* shapes tried */
} xs_tune_result;
int xs_engine_autotune(xs_engine* e, const xs_options* opt, const xs_condition* conds, int ncond,
                       const xs_lines* lines, const xs_grid* grid, double* out, size_t out_stride,
                       xs_tune_result* best);
int xs_tune_save(const char* path);
int xs_tune_load(const char* path);
int xs_tune_clear(void);

/* Allocation-free variant of xs_engine_execute for ONE condition.  It has no
 * counterpart in the reference.  For callers that cannot let this library
 * allocate device memory: a host whose own pool allocator already holds the
 * device's memory (a cudaMalloc here would fail or shrink that pool), or a
 * latency-critical loop that cannot take the device-wide synchronisation
 * cudaMalloc/cudaFree may cause.  Inputs and outputs are the caller's
 * (device pointers, as for xs_engine_execute with ncond = 1 and `out`
 * accumulated); the scratch is one fixed array of XS_NOALLOC_SCRATCH_BYTES
 * compiled into the library, which every GPU that loads the library holds
 * until the process exits.  Line counts whose scratch would not fit (about
 * 320,000 lines for FP64 Voigt, 380,000 for mixed Voigt, 690,000 for
 * Doppler/Gaussian) are rejected with XS_ERR_INVALID before any device work.
 * Every call looks up the array's device address with the device current
 * (no allocation), so a device reset between calls invalidates nothing the
 * caller must redo; the first call on a device may load the library's device
 * code there, so make it before any stream capture on that device.  Work is
 * enqueued on `stream` (cudaStream_t; NULL = legacy) and the call waits for
 * it, then reports XS_ERR_UNSORTED / XS_ERR_GRID like xs_engine_sync.  Every
 * call shares the one array and it keeps the previous call's contents; calls
 * that overlap on the GPU (e.g. issued from two host threads at once) race on
 * it -- serialise them. */
#define XS_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)
int xs_execute_noalloc(const xs_options* opt, const xs_condition* cond, const xs_lines* lines,
                       const xs_grid* grid, double* out, void* stream);

/* Streamed Voigt line list (no counterpart in the reference, which hands the
 * manager one host chunk at a time and waits, VoigtProfile.cpp:56-103): the
 * lines stay in host memory -- pinned, for copies that overlap compute -- as
 * FP64 centres (ascending), FP32 intensities S(T) and FP32 Lorentz half widths
 * gamma(T, P) of the one condition `cond` (T, Q and P there only set the
 * Doppler width and the cut).  They are copied chunk_lines at a time into two
 * device buffers on a second stream while the previous chunk is evaluated on
 * the engine's stream; every chunk adds into `out` (the whole grid, device)
 * the points its lines reach.  VOIGT, GPU convention, FP64 or mixed.  Blocks
 * until done; `stats` (may be NULL) gets the device time of the whole
 * pipeline, the copy stream's span and the bytes copied. */
typedef struct {
    double total_ms;      /* first copy issued -> last chunk evaluated */
    double copy_span_ms;  /* first copy issued -> last copy done */
    double h2d_bytes;
    int chunks;
    int kernels;          /* kernels launched */
} xs_stream_stats;
int xs_stream_execute(xs_engine* e, const xs_options* opt, const xs_condition* cond,
                      const double* h_nu, const float* h_s, const float* h_gamma, size_t n,
                      const xs_grid* grid, double* out, size_t chunk_lines,
                      xs_stream_stats* stats);

/* Partition functions on the device: q[t] = sum_i gns[i] exp(-c2 E_i / T_t)
 * over a state list (host arrays; the sum of compute_partition,
 * exomol_functions.cpp:44-62, with its constants) for n_temps temperatures,
 * in a fixed summation order.  Blocks until q is written. */
int xs_partition_sum(int device, const double* energies, const int* gns, size_t n,
                     const double* temperatures, int n_temps, double* q);

/* ---- 3. manager level: BaseManager over host buffers --------------------- */
/* kind: 0 = GpuManager (reference GPU convention), 1 = OpenMPManager
 * (reference CPU convention, computed on the GPU). */
typedef struct xs_manager xs_manager;
int xs_manager_create(int kind, int profile, int gpu_id, int num_threads, size_t total_memory,
                      xs_manager** out);
int xs_manager_destroy(xs_manager* m);
int xs_manager_set_precision(xs_manager* m, int precision);
int xs_manager_initialize_vectors(xs_manager* m, int Npoints);
int xs_manager_initialize_constants(xs_manager* m, double half_width, double temperature,
                                    double partition, double dfreq, double meanmass,
                                    double pressure, double ref_temp);
int xs_manager_transfer_vectors(xs_manager* m, size_t Nener, const double* h_energies,
                                const double* h_nu, const double* h_aif, const int* h_gns,
                                const double* h_gamma, const double* h_n);
int xs_manager_transfer_freq(xs_manager* m, const double* h_freq, const double* h_intens, int N);
int xs_manager_execute_cross_section(xs_manager* m, int N, int N_ener, int start_idx);
int xs_manager_transfer_results(xs_manager* m, double* h_freq, double* h_intens, int N);
int xs_manager_cleanup(xs_manager* m);
int xs_manager_ready_for_work(xs_manager* m, int* ready);
int xs_manager_get_ntrans(xs_manager* m, size_t* ntrans);

/* ---- 4. server level: a continuous-batching request loop ----------------- */
/* No counterpart in the reference, which computes one .inp job per process.
 * Line lists stay resident in device memory; requests (molecule, T, Q(T), P,
 * profile, grid) arrive at any time from any thread and are admitted while
 * their memory fits the budgets.  Each request's grid is split into chunks
 * of whole 256-point tiles with bounded work; a scheduler thread interleaves
 * the chunks of all admitted requests over several streams (the request
 * with the least remaining work over all streams first, as many chunks in
 * flight as there are streams), so a request that arrives while a large one
 * runs does not wait for all of it.  A request's chunks depend
 * only on the request, so its result is the same alone and in any mix. */
typedef struct xs_server xs_server;

typedef struct {
    size_t device_budget; /* bytes of device memory for molecules, lane scratch
                             and admitted requests (0 = free memory - 2 GiB) */
    size_t host_budget;   /* pinned host bytes for results (0 = 1 GiB) */
    int lanes;            /* streams, each with its own engine (0 = 4) */
    int depth;            /* chunks in flight per lane (0 = 2) */
    double chunk_pairs;   /* target line-evals per chunk (0 = 4e9) */
    size_t chunk_lines;   /* most lines in one chunk's slice (0 = 2^22) */
    int policy;           /* which admitted request's chunk goes next:
                             XS_POLICY_LEAST_WORK (0, default): the one with
                             the least remaining work; XS_POLICY_ROUND_ROBIN:
                             each in turn (processor sharing by chunks);
                             XS_POLICY_DEADLINE: earliest deadline first, a
                             request's deadline being its submission time
                             plus its remaining work at 2e9 line-evals/ms */
    long long tcache_bytes; /* device bytes (within device_budget) for the
                             per-temperature intensity caches (0 = 4 GiB;
                             < 0: none).  A cache holds, for one molecule,
                             profile, T and Q(T), every line's S(T) and, for
                             Voigt, (T_ref/T)^n in FP64, exactly as step one
                             computes them; it is made on the second request
                             with that key, filled by the chunks that run, and
                             read by later chunks over the same lines instead
                             of recomputing (least recently used caches that
                             no request holds are dropped for room). */
} xs_server_config;
#define XS_POLICY_LEAST_WORK 0
#define XS_POLICY_ROUND_ROBIN 1
#define XS_POLICY_DEADLINE 2

typedef struct {
    int molecule;       /* id from xs_server_add_molecule */
    int profile;        /* XS_VOIGT or XS_DOPPLER */
    int precision;      /* XS_FP64 or XS_MIXED */
    double temperature; /* K */
    double partition;   /* Q(T); <= 0: from the molecule's states
                           (xs_server_add_states), computed on the device and
                           kept per temperature */
    double pressure;    /* atm: multiplies the molecule's gamma (given per atm)
                           and, when cut <= 0, sets the reference cut rule */
    double cut;         /* window half width in cm-1; <= 0: min(25 P, 100) for
                           Voigt, 100 for Doppler */
    double f0, df;      /* grid f_i = f0 + i*df ... */
    int npoints;        /* ... for i < npoints */
} xs_request;

typedef struct {
    int status;         /* XS_OK or the request's error */
    double latency_ms;  /* submit -> result in host memory */
    double queue_ms;    /* submit -> admitted */
    double run_ms;      /* admitted -> result in host memory */
    int chunks;
    double line_evals;  /* sum of window overlaps / df (an estimate) */
    size_t lines;       /* lines within the grid +/- cut */
    double err_bound;   /* a-priori bound on the relative error of every grid
                           point and of the band integral against the FP64
                           arithmetic (xs_error_bound of the request's profile
                           and precision) */
    int tcache_chunks;  /* chunks whose step one read the per-temperature
                           cache instead of computing S(T) */
} xs_request_info;

int xs_server_create(int device, const xs_server_config* cfg, xs_server** out);
/* Finishes the requests already submitted, then frees everything. */
int xs_server_destroy(xs_server* s);
/* Copies a nu-ascending line list to the device (gamma per atm at ref_temp);
 * at most 64 molecules. */
int xs_server_add_molecule(xs_server* s, const double* nu, const double* energies,
                           const double* aif, const int* gns, const double* gamma,
                           const double* n, size_t count, double mean_mass, double ref_temp,
                           int* molecule_id);
/* Optional lower-state list of a molecule (E in cm-1, total degeneracy g),
 * for requests that leave Q(T) to the server. */
int xs_server_add_states(xs_server* s, int molecule_id, const double* energies, const int* gns,
                         size_t count);
/* Non-blocking.  XS_ERR_NOMEM when the request alone exceeds a budget. */
int xs_server_submit(xs_server* s, const xs_request* r, unsigned long long* request_id);
/* Blocks until the request is done (timeout_ms < 0: no limit; on timeout
 * XS_ERR_TIMEOUT and the request stays), copies its npoints results to out
 * (may be NULL), fills info (may be NULL) and forgets the request. */
int xs_server_wait(xs_server* s, unsigned long long request_id, double* out, int npoints,
                   xs_request_info* info, int timeout_ms);
int xs_server_pending(xs_server* s, int* queued, int* active);
/* The server's chunk planner, on host arrays (no device needed): chunks of
 * whole 256-point tiles, each with at most max_pairs estimated line-evals
 * (unless one tile alone has more) and max_lines lines (0 = no limit).
 * Fills up to cap entries; *nchunks gets the count. */
int xs_plan_chunks(const double* nu, size_t n, double f0, double df, int npoints, double cut,
                   double max_pairs, size_t max_lines, int cap, int* start, int* points,
                   size_t* l0, size_t* l1, double* pairs, int* nchunks);
/* Grid-range split for several GPUs (no counterpart in the reference, whose
 * MultiGPUManager.cpp:61-83 shards the transitions and sums whole grids on
 * the host).  Grid tiles are independent, so rank `rank` of `nranks` takes
 * the grid points [*start, *start + *points) -- whole 256-point tiles, the
 * ranges contiguous, in rank order and balanced by estimated line-evals --
 * and only the lines [*l0, *l1) of the ascending host array `nu` whose
 * window (+-cut) can reach them.  Each rank computes its slice with no
 * reduction; the slices are concatenated (gpu_cross_b200.multigpu gathers
 * them over torch.distributed).  A rank with no work gets *points = 0.
 * *pairs (may be NULL): the rank's estimated line-evals.  Host only. */
int xs_split_grid(const double* nu, size_t n, double f0, double df, int npoints, double cut,
                  int nranks, int rank, int* start, int* points, size_t* l0, size_t* l1,
                  double* pairs);

#ifdef __cplusplus
}
#endif

#endif /* XSEC_B200_H */
