// Internal declarations shared by the kernels (xs_kernels.cu) and the host
// engine (xs_engine.cu).  Not part of the public C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace xs {

// Physical constants, defines.h:4-20 of the reference (the values must match
// bit-for-bit; GPUManager.cpp:28-31 uses the same literals).
constexpr double kLN2 = 0.69314718056;
constexpr double kISQRTPI = 0.564189584;
constexpr double kPI = 3.14159265359;
constexpr double kPLANCK = 6.6260693e-27;
constexpr double kVELLGT = 2.99792458e+10;
constexpr double kBOLTZ = 1.380658e-16;
constexpr double kNA = 6.0221412927e23;
constexpr double kDOPPLER_CUTOFF = 100.0;

// Region I constant of Humlicek's W4 (T * 0.5641896 / (0.5 + T^2)).
constexpr double kW4C = 0.5641896;

// |t| at and beyond which erf(t) is exactly +-1 in double precision
// (erfc(6) = 2.2e-17 < 2^-54); tests/test_gpu_parity.py checks the device erf
// against it.  Doppler/Gaussian pairs whose both erf arguments lie beyond it
// add exactly 0 in the reference and are skipped.
constexpr double kErfSat = 6.0;

enum Kind : int { kGauss = 0, kDoppler = 1, kVoigt = 2 };
enum Conv : int { kConvGpu = 0, kConvCpu = 1 };

// Device-side error bits (OR-ed into the engine's error word).
constexpr unsigned kErrUnsorted = 1u;
constexpr unsigned kErrGrid = 2u;
// A line's W4 region interval lies 3e7 or more grid points from the grid
// index of its centre (mixed precision; a grid step far below the cut over
// 3e7): the core pass, which finds lines by that index, could miss it.
constexpr unsigned kErrReach = 4u;

constexpr int kMaxCond = 64;  // conditions per launch (the sweep uses 40)
// Per-condition words step one reduces into (cleared before it runs): the
// widest core-candidate band and the core pass's reach.
constexpr int kKcWords = 2 * kMaxCond;
constexpr int kMaxSplits = 64;                      // line splits per tile
constexpr size_t kMaxPartBytes = size_t(64) << 20;  // automatic splits' part buffer

// Per-condition constants, computed on the host exactly as the selected
// reference backend computes them (GPUManager.cpp:24-47 for the GPU
// convention, OpenMPManager.cpp:57-67 and :146-147/:191-192 for the CPU one).
struct CondDev {
    double cmcoef;       // 1/(8 pi c)
    double beta;         // hc/kT
    double partition;    // Q(T)
    double tratio;       // ref_temp / T (base of the gamma temperature power)
    double dpw;          // Doppler width per unit wavenumber
    double cut;          // window half width (cm-1)
    double gamma_scale;  // multiplies the uploaded gamma
    double pad;
};

// Voigt records, one per (line, condition).  Region I of W4,
// Re[T c / (0.5 + T^2)] with T = y - ix, is evaluated as
//   Re w * pref = Pc (u + 1) / (u^2 + D2),  u = x^2 + Cy,
// with Cy = y^2 - 0.5, D2 = 2 y^2, Pc = pref c y (c = 0.5641896): the same
// rational as c y (0.5 + x^2 + y^2) / ((0.5 + y^2 - x^2)^2 + 4 x^2 y^2), since
// (0.5 + y^2 - x^2)^2 + 4 x^2 y^2 = (x^2 + y^2 - 0.5)^2 + 2 y^2.  In region I
// (|x| + y >= 15) u > 190, so nothing cancels.
// FP64 record: the first three 16-byte chunks are all the fast path reads.
struct __align__(16) RecV64 {
    double nu;     // line centre used for offsets
    double g;      // 1 / Doppler width
    double Cy, D2;
    double Pc, y;  // y = Lorentz / Doppler width ratio
    double pref;   // S * g
    double pad;
    int lo, hi;    // window [lo, hi) of grid indices
    int clo, chi;  // grid indices near the core (region I not guaranteed)
};
static_assert(sizeof(RecV64) == 80, "RecV64 layout");

// Mixed-precision record (FP32).  The offset of grid point j from the line
// centre is (m - j) * df + r in cm-1, with m the nearest grid index and
// |r| <= df/2 computed in FP64; stored scaled by g: x = (m - j) * dfa + ra.
// The first two 16-byte chunks are all the fast path reads.  [clo, chi]:
// the grid indices of the line's window where |x| + y < 15 (W4 regions
// II-IV, left to the core pass; empty: clo > chi), [lo55, hi55] those where
// |x| + y < 5.5.  A negative dfa marks a line whose x comes from its FP64
// centre (|m| >= 1.6e7, or offsets beyond the FP32 range over the window).
struct __align__(16) RecV32 {
    float m, ra, dfa, Cy;
    float D2, Pc, pref, y;
    float lo, hi, clo, chi;
    float lo55, hi55;
    double nu;
};
static_assert(sizeof(RecV32) == 64, "RecV32 layout");

// Multi-condition layout: a group of C conditions that share one window
// (same cut) is evaluated together, one 32-point row of the grid per warp
// and C accumulators per lane.  What the conditions share is stored once per
// line; the rest once per (line, condition), conditions innermost.
// Mixed-precision multi-condition layout.  The offset of grid point j from a
// line, in Doppler widths, factors into a condition-free part and a
// per-condition constant: the reference's gammaG = 1 / (nu dpw)
// (cross_kernal.cu:958), so x = (nu - f_j) / (nu dpw) = X k with
// X = (nu - f_j) / nu = (m - j) dfn + rn and k = 1 / dpw.  One X per
// (line, point) then serves every condition of the group, and
// u = x^2 + Cy = X^2 k^2 + Cy.
struct __align__(16) LineShX {
    float m;      // nearest grid index (exact below 2^24)
    float dfn;    // df / nu
    float rn;     // (nu - f0 - m df) / nu
    int flags;    // kLineWhole: X from nu in FP64 and every pair of the line
                  // tested; kLineWide: region-I products need the scaled
                  // shared reciprocal
    int lo, hi;   // window [lo, hi) of grid indices
    double nu;    // centre (whole lines)
};
static_assert(sizeof(LineShX) == 32, "LineShX layout");
constexpr int kLineWhole = 1;
constexpr int kLineWide = 2;
// Region-I constants of a line for the C conditions of its group, each
// array in condition order: conditions 2k and 2k+1 are one packed FP32x2
// operand, conditions 4k..4k+3 one 16-byte load.  This is all step two
// stages per (line, group) besides LineShX: 12 bytes per condition (C = 2 is
// padded to 32 bytes, a whole number of 16-byte copies).
template <int C>
struct __align__(16) LineR1 {
    float Cy[C], D2[C], Pc[C];
};
template <>
struct __align__(16) LineR1<2> {
    float Cy[2], D2[2], Pc[2], pad[2];
};
static_assert(sizeof(LineR1<8>) == 96 && sizeof(LineR1<4>) == 48 && sizeof(LineR1<2>) == 32,
              "LineR1 layout");
// Bytes per (line, group) of the mixed multi-condition region-I records.
constexpr size_t line_r1_bytes(int C) { return C == 8 ? 96 : (C == 4 ? 48 : 32); }
// Per (line, condition) of the mixed multi-condition layout, for the core
// pass: the grid indices of W4 regions II-IV [lo15, hi15] and III-IV
// [lo55, hi55] (empty: lo > hi) inside the line's window.  Step two adds
// the region-I rational at every pair of the window except, on the lines it
// takes as core candidates, the pairs where u = x^2 + y^2 - 0.5 < 1 in FP32
// (near the centre the rational can exceed W4 by up to 0.28 / y); the core
// pass makes the same choice and adds W4, less the rational where step two
// added it, over [lo15, hi15].
struct __align__(16) CoreIv {
    int lo15, hi15, lo55, hi55;
};
static_assert(sizeof(CoreIv) == 16, "CoreIv layout");
// FP64: core packs the core band around m: (m - clo) | (chi - m) << 16, each
// part at most 0x7fff (0x7fff: unbounded); -1: no core band.
struct __align__(16) LineSh64 {
    double nu;
    int lo, hi;
};
static_assert(sizeof(LineSh64) == 16, "LineSh64 layout");
struct __align__(16) CondRec64 {
    double g, Cy, D2, Pc, y, pref;
    int core, pad0, pad1, pad2;
};
static_assert(sizeof(CondRec64) == 64, "CondRec64 layout");

// Doppler / Gaussian record (FP64).
struct __align__(16) RecE64 {
    double nu;  // centre used for offsets
    double s;   // intensity
    double g;   // Doppler: 1 / (nu * dpw); Gaussian: unused
    double pad;
    int lo, hi;  // active window (reference window, minus pairs that add exactly 0)
    int pad0, pad1;
};
static_assert(sizeof(RecE64) == 48, "RecE64 layout");

struct GridDev {
    const double* freq;  // full grid
    double f0, df;       // analytic grid f_j ~ f0 + j * df (f0 = freq[0])
    int npoints_total;
    int start, points;   // chunk [start, start + points)
};

struct LinesDev {
    const double *nu, *energies, *aif, *gamma, *nexp;
    const int* gns;
    long n;  // lines evaluated (may be less than uploaded: CPU coverage rule)
    // Streamed lists (Voigt, GPU convention): the intensity S(T) and the
    // Lorentz half width gamma(T, P) of the condition, precomputed in FP32;
    // when set, energies, aif, gns, gamma and nexp are not read.
    const float* s32;
    const float* gl32;
    // Per-temperature cache (one condition, single-condition layouts): the
    // intensity S(T) and, for Voigt, the Lorentz temperature power
    // (T_ref/T)^n of each line as step one computes them, FP64.  tc_mode 1:
    // step one reads them instead of computing them (and reads no E'', A, g
    // or n); 2: it computes and stores them.
    double* tc_s;
    double* tc_pw;
    int tc_mode;
};

struct PrepArgs {
    LinesDev L;
    // Lines [line0, line1) of the list (line1 = 0: to L.n): step one can run
    // on a list in slices, each as soon as its copy to the device is done.
    long line0, line1;
    GridDev G;
    int ncond;
    CondDev cond[kMaxCond];
    void* rec;          // records, condition-major: rec + c * n
    int* wlo;           // windows, condition-major
    int* whi;
    int* mi;            // nearest grid index of each line (condition-free)
    int* kc;            // per condition: max core half-width in grid points
                        // (mixed multi-condition layout: the core-candidate
                        // reach plus one, 0 when no line has one);
                        // kc + kMaxCond: the core pass's reach (mixed
                        // multi-condition layout)
    unsigned* err;
    double half_width;  // Gaussian
    double x0;          // Doppler half bin: dfreq * 0.5
    double xg, x0g;     // Gaussian: sqrt(ln2)/HW, xg * dfreq * 0.5
    int mixed_tile_span;  // 32 * points_per_thread (mixed safety bound)
    int group;          // > 0: multi-condition layout with this many
                        // conditions per group (Voigt only)
    void* lsh;          // multi-condition: per-line shared records per group
                        // (LineShX mixed, LineSh64 FP64)
    CoreIv* civ;        // mixed multi-condition: region intervals and
    float2* cyp;        //   (y, pref) per (condition, line), condition-major
    // Multi-condition layouts: the window slot of each group -- groups with
    // the same cut (consecutive, conditions being ordered by cut) share one
    // copy of the per-line window data (LineShX / LineSh64, lo, hi), that of
    // the first group of their run.
    int wslot[kMaxCond];
    // Temperature classes: conditions of one class have the same cmcoef,
    // beta, Q, T_ref/T and Doppler width, so their intensity, Lorentz
    // temperature power and 1/Doppler width are the same numbers.  tclass[c]
    // in [0, nclass); class_rep[t]: a condition of class t.
    int nclass;
    int tclass[kMaxCond];
    int class_rep[kMaxCond];
};
// Temperature classes whose per-line values step one keeps in shared memory
// (more classes: each condition computes its own).
constexpr int kMaxClassCache = 16;

struct StepArgs {
    const void* rec;
    const int* wlo;
    const int* whi;
    const int* mi;
    const int* kc;
    long n;             // lines per condition
    double* out;
    size_t out_stride;  // elements between conditions
    GridDev G;
    const void* lsh;    // multi-condition layout (LineShX mixed, LineSh64 FP64)
    int wslot[kMaxCond];  // window slot of each group (PrepArgs::wslot)
    int group;          // conditions per group (multi-condition kernel)
    int tiles_per_cond;
    int n_items;
    unsigned* counter;
    double x0, xg, x0g;  // Doppler / Gaussian constants
    // Line splits: with splits > 1 every tile is taken by `splits` work
    // items, item s over the tile's 32-line groups s, s + splits, ...; it
    // stores its sums to part[(c * splits + s) * part_stride + j - G.start]
    // and k_reduce_splits adds the parts, in order, to out.
    int splits;
    double* part;
    size_t part_stride;
    // Mixed multi-condition kernel: per condition k = 1 / dpw and k^2.
    float kx[kMaxCond];
    float kx2[kMaxCond];
    // Output row of each condition of the launch: its sums go to
    // out + row[c] * out_stride.
    int row[kMaxCond];
};

// Kernel launchers (xs_kernels.cu).  All asynchronous on `stream`.
cudaError_t launch_grid_check(const GridDev& g, unsigned* err, cudaStream_t stream);
cudaError_t launch_prep(int kind, int conv, bool mixed, const PrepArgs& a, cudaStream_t stream);
// P = points per thread (1, 2, 4, 8), warps per block (4 or 8).
cudaError_t launch_steptwo(int kind, int conv, bool mixed, int P, int warps, int blocks,
                           const StepArgs& a, cudaStream_t stream);
// out[row[c]][G.start + j] += sum over s of part[(c * splits + s) * stride + j].
cudaError_t launch_reduce_splits(const StepArgs& a, int ncond_out, cudaStream_t stream);
// Resident blocks per SM for a step-two configuration.
int steptwo_blocks_per_sm(int kind, int conv, bool mixed, int P, int warps);
size_t record_bytes(int kind, bool mixed);

// Layout of the scratch one execute call needs: records and windows for
// `ncond` conditions of `n` lines, the per-line grid index and the
// per-condition core widths; sections 256-byte aligned from `base_off`.
struct ScratchPlan {
    size_t off_rec, off_wlo, off_whi, off_mi, off_kc, off_lsh, off_civ, off_cyp, need;
};
ScratchPlan plan_scratch(int kind, bool mixed, size_t n, int ncond, size_t base_off,
                         int group = 0);

// Core pass of the mixed multi-condition layout: for every (condition, row
// of 32 grid points), the W4 regions II-IV of the pairs inside the lines'
// region intervals, added to out + row[c] * out_stride in line order.
struct CoreArgs {
    const CoreIv* civ;
    const float2* cyp;
    const LineShX* lsh;
    const void* rec;    // LineR1<group> per (line, group): Cy of the condition
    const int* mi;
    const int* kc;
    const double* freq;
    long n;             // lines per condition
    int group;          // conditions per group (LineShX is per group)
    GridDev G;
    double* out;
    size_t out_stride;
    // Line splits as in StepArgs: with splits > 1 the warp of split s takes
    // the 32-line batches s, s + splits, ... of a row's candidate lines and
    // adds its sums to the step-two parts, which k_reduce_splits then adds in
    // order; with one split it adds to out.
    int splits;
    double* part;
    size_t part_stride;
    float kx[kMaxCond];   // 1 / dpw
    float kx2[kMaxCond];  // (1 / dpw)^2 as step two has it
    int row[kMaxCond];
    int wslot[kMaxCond];  // window slot of each group (PrepArgs::wslot)
};
cudaError_t launch_core_mcx(const CoreArgs& a, int ncond, cudaStream_t stream);
// The same for the single-condition mixed layout (RecV32 records; a.kx set;
// with line splits it adds to a.part).
cudaError_t launch_core_v32(const StepArgs& a, int ncond, cudaStream_t stream);

// Sampled FP64 re-evaluation of a mixed-precision Voigt result: for each
// condition and each of `nrows` sampled rows of 32 grid points, the FP64 sum
// of the selected convention (the reference's arithmetic: intensity, widths,
// window and W4 with its region choice), computed directly from the line
// arrays, then compared with what the call added to `out`.
constexpr int kMaxCheckRows = 16;
struct CheckArgs {
    LinesDev L;
    GridDev G;
    int ncond;
    int conv;
    CondDev cond[kMaxCond];
    int row[kMaxCond];      // output row of each condition
    double* out;
    size_t out_stride;
    int nrows;
    int rows[kMaxCheckRows];  // first grid index of each sampled row
    double* before;  // [c][k][32]: out at the sampled points before the call
    double* ref;     // [c][k][32]: the FP64 sums
    double* stats;   // [c][4]: max relative error (points above 1e-6 of the
                     // row's peak), sum of ref, sum of (got - ref), peak
};
// Copies out at the sampled points into `before` (launched before step two).
cudaError_t launch_check_snapshot(const CheckArgs& a, cudaStream_t stream);
// FP64 sums at the sampled points and the per-condition statistics
// (launched after the call's last kernel).
cudaError_t launch_check_rows(const CheckArgs& a, cudaStream_t stream);

// Multi-condition step two (Voigt): C conditions per warp, 32 points per warp.
cudaError_t launch_steptwo_mc(bool mixed, int C, int warps, int blocks, const StepArgs& a,
                              cudaStream_t stream);
int steptwo_mc_blocks_per_sm(bool mixed, int C, int warps);

}  // namespace xs
