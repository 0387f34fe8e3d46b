// sm_100a kernels of the cross-section engine.
//
//  k_grid_check   validates the grid (ascending, uniform step) once per run.
//  k_prep         "step one" per (line, condition): intensity S(T), Lorentz
//                 width, Doppler width, the exact window of grid indices each
//                 line reaches, and a packed record for step two.
//  k_steptwo_*    "step two": a persistent grid of warps takes work items
//                 (condition, tile of 32*P grid points) from an atomic
//                 counter.  A warp finds the lines whose windows meet its tile
//                 with a 32-way ballot search over the window arrays, streams
//                 their records through a per-warp double-buffered shared
//                 memory stage (cp.async), and accumulates its 32*P grid
//                 points in registers, line by line in ascending order: a
//                 fixed summation order, no atomics on the result.
//
// The reference computes the same sums with one CTA per grid point that scans
// the whole chunk (cross_kernal.cu:924-997, :654-723).
#include <cuda_runtime.h>

#include <cfloat>
#include <climits>
#include <cmath>
#include <type_traits>

#include "xs_internal.cuh"

namespace xs {
namespace {

// Depth of the per-warp cp.async staging pipeline (groups of 32 records).
constexpr int kStages = 3;

// Offsets (in Doppler widths) from which a line's every pair takes the
// per-pair path, x from its FP64 centre ("whole" lines): FP32 offsets and
// the region-I sums are exact enough below it.
constexpr double kWholeXMax = 1.0e8;
// Scale of the shared-reciprocal products of the region-I rational (2^-100).
// Where step two evaluates it (u >= 1), the denominators d = u^2 + 2 y^2
// lie in [1, 1e32] (|x| < 1e8 for lines that are not whole), so tau d lies
// in [7.9e-31, 79], tau dA dB in [7.9e-31, 7.9e33] and its reciprocal in
// [1.3e-34, 1.3e30]: all normal FP32 numbers.
constexpr float kPairTau = 7.88860905221011805e-31f;
// Lines whose x^2 + y^2 stays below kPairUMax over their tiles and whose
// |Pc| stays below kPairPcMax, for every condition of the group ("narrow"
// lines, the usual case), share reciprocals without the scaling: their
// denominators lie in [1, 6.3e18], so dA dB lies in [1, 4e37] and its
// reciprocal is a normal FP32 number, and the numerators |Pc (u + 1)| stay
// below 2.5e17, so the cross products nA dB of two lines stay below 1.6e36
// (and, d being >= 1, never fall below |n|).  Other lines are marked
// kLineWide.
constexpr double kPairUMax = 2.5e9;
constexpr double kPairPcMax = 1.0e8;


// ---------------------------------------------------------------------------
// Small complex arithmetic for the W4 regions II-IV.
// ---------------------------------------------------------------------------
struct cplx {
    double re, im;
};
__device__ __forceinline__ cplx operator+(double a, cplx b) { return {a + b.re, b.im}; }
__device__ __forceinline__ cplx operator-(double a, cplx b) { return {a - b.re, -b.im}; }
__device__ __forceinline__ cplx operator*(cplx a, cplx b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ cplx operator*(cplx a, double b) { return {a.re * b, a.im * b}; }
// Real part of a / b.
__device__ __forceinline__ double div_re(cplx a, cplx b) {
    return (a.re * b.re + a.im * b.im) / (b.re * b.re + b.im * b.im);
}

// Re w(x + iy) by Humlicek's W4 (JQSRT 27 (1982) 437): four regions chosen
// on s = |x| + y and y vs 0.195|x| - 0.176 (the region tests and the
// coefficient table are Humlicek's, as used by cross_kernal.cu:149-181 and
// profiles.cpp:9-42).  Region I is evaluated as a real rational, the others
// with complex Horner schemes.
__device__ double w4_re(double x, double y) {
    const double s = fabs(x) + y;
    if (s >= 15.0) {
        const double x2 = x * x, y2 = y * y;
        const double dr = 0.5 + y2 - x2;
        return kW4C * y * (0.5 + x2 + y2) / (dr * dr + 4.0 * x2 * y2);
    }
    const cplx t = {y, -x};
    if (s >= 5.5) {
        const cplx u = t * t;
        const cplx num = t * (1.410474 + u * .5641896);
        const cplx den = .75 + u * (3. + u);
        return div_re(num, den);
    }
    if (y >= 0.195 * fabs(x) - 0.176) {
        const cplx num = 16.4955 + t * (20.20933 + t * (11.96482 + t * (3.778987 + t * .5642236)));
        const cplx den =
            16.4955 + t * (38.82363 + t * (39.27121 + t * (21.69274 + t * (6.699398 + t))));
        return div_re(num, den);
    }
    const cplx u = t * t;
    double sn, cs;
    sincos(u.im, &sn, &cs);
    const double eu = exp(u.re);
    const cplx num =
        36183.31 - u * (3321.9905 - u * (1540.787 - u * (219.0313 - u * (35.76683 - u * (1.320522 - u * .56419)))));
    const cplx den =
        32066.6 - u * (24322.84 - u * (9022.228 - u * (2186.181 - u * (364.2191 - u * (61.57037 - u * (1.841439 - u))))));
    return eu * cs - div_re(t * num, den);
}

// First j in [s, e) with pred(j) true (pred monotone false..true), or e.
// Starts from a guess and walks; falls back to bisection after 8 steps.
template <class Pred>
__device__ int find_first(int s, int e, double guess, Pred pred) {
    long j;
    if (!(guess > double(s))) j = s;  // also catches NaN
    else if (guess > double(e)) j = e;
    else j = long(guess);
    for (int it = 0; it < 8; ++it) {
        if (j > s && pred(int(j - 1))) { --j; continue; }
        if (j < e && !pred(int(j))) { ++j; continue; }
        return int(j);
    }
    int lo = s, hi = e;
    while (lo < hi) {
        int mid = lo + (hi - lo) / 2;
        if (pred(mid)) hi = mid; else lo = mid + 1;
    }
    return lo;
}

__device__ __forceinline__ int clamp_index(double v, int lo, int hi) {
    if (!(v > double(lo))) return lo;  // NaN -> lo
    if (v > double(hi)) return hi;
    return int(v);
}

// ---------------------------------------------------------------------------
// Grid check.
// ---------------------------------------------------------------------------
__global__ void k_grid_check(GridDev g, unsigned* err) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (j >= g.npoints_total) return;
    const double f0 = g.freq[0];
    const double fj = g.freq[j];
    bool bad = !(fj > g.freq[j - 1]);
    bad |= !(fabs(fj - (f0 + double(j) * g.df)) <= 0.01 * g.df);
    if (bad) atomicOr(err, kErrGrid);
}

// ---------------------------------------------------------------------------
// Step one.
// ---------------------------------------------------------------------------
// Mixed multi-condition layout: outside x^2 + y^2 < kNearR2 the region-I
// rational stays below 2 Pc (u >= 1), so step two adds it there on every
// line; inside, only the lines within the core-candidate reach can have
// pairs, and step two tests u on them.
constexpr double kNearR2 = 1.5;
// Grid indices [jlo, jhi] of the window [lo, hi) where |x| + y < lim, with
// x = (nu - f_j) g in FP64 on the analytic grid f_j = f0 + j df: the region
// choice of the FP64 path (up to the grid's last-bit rounding), so that no
// pair changes region with the FP32 rounding of x.  Empty: jlo > jhi.
// md = (nu - f0) / df, q = 1 / (g df) and tb = |md| + (|nu| + |f0|) / df
// (the line's part of the rounding tolerance below) come precomputed; md and
// q place the interval's ends, and the region test itself decides where an
// end is close to a grid point.
__device__ __forceinline__ double region_tol_base(double nu, double f0, double df, double md) {
    return fabs(md) + (fabs(nu) + fabs(f0)) / df;
}
__device__ __forceinline__ void region_interval_q(double nu, double g, double y, double lim, int lo, int hi, double f0,
                                  double df, double md, double q, double tb, int& jlo, int& jhi) {
    jlo = 1;
    jhi = 0;
    if (!(y < lim) || lo >= hi) return;
    const double hq = (lim - y) * q;
    // x_j = (md - j) / q, so the points inside are the integers of
    // (md - hq, md + hq).  The region test's roundings (f_j, nu - f_j, the
    // product with g, md and hq themselves) move both ends by a few 1e-16 of
    // |md|, (|nu| + |f0|) / df and hq grid steps; where each end lies further
    // than `tol` (a thousand times that, and at least 1e-6) from an integer,
    // the exact region test of every point agrees with [ceil(md - hq),
    // ceil(md + hq) - 1], clamped to the window, and is not evaluated.
    // Otherwise the walks below decide.
    {
        const double bl = md - hq, bh = md + hq;
        const double tol = 1.0e-6 + 1.0e-13 * (tb + hq);
        if (fabs(bl) < 1.0e9 && fabs(bh) < 1.0e9 && fabs(bl - rint(bl)) > tol && fabs(bh - rint(bh)) > tol) {
            // ceil to int in one conversion, clamped in integers (lo < hi)
            const int jl = min(max(__double2int_ru(bl), lo), hi), jh = min(max(__double2int_ru(bh), lo), hi);
            if (jl < jh) {
                jlo = jl;
                jhi = jh - 1;
            }
            return;
        }
    }
    auto fa = [&](int j) { return fma(double(j), df, f0); };
    auto inside = [&](int j) { return !(fabs((nu - fa(j)) * g) + y >= lim); };
    const int jl = find_first(lo, hi, ceil(md - hq), [&](int j) { return fa(j) > nu || inside(j); });
    const int jh = find_first(lo, hi, floor(md + hq) + 1.0, [&](int j) { return fa(j) > nu && !inside(j); });
    if (jl < jh) {
        jlo = jl;
        jhi = jh - 1;
    }
}

// The intervals of region II-IV (|x| + y < 15) and of regions III-IV
// (|x| + y < 5.5), with md, q and tb computed once for both.
__device__ void region_intervals(double nu, double g, double y, int lo, int hi, double f0, double df, int& j15,
                                 int& k15, int& j55, int& k55) {
    const double md = (nu - f0) / df, q = 1.0 / (g * df);
    const double tb = region_tol_base(nu, f0, df, md);
    region_interval_q(nu, g, y, 15.0, lo, hi, f0, df, md, q, tb, j15, k15);
    region_interval_q(nu, g, y, 5.5, lo, hi, f0, df, md, q, tb, j55, k55);
}

// Step one of one (line, condition).  Returns the line's core half-width in
// grid points (Voigt; 0 otherwise).  `reach` (mixed Voigt): the largest
// distance, in grid points, from the line's nearest grid index to its region
// interval (the core pass's reach).  The mixed-precision multi-condition
// layout has its own step one (k_prep_lines_x); the FP64 one is written here.
template <int KIND, int CONV, bool MIXED>
__device__ __forceinline__ int prep_line(const PrepArgs& a, long i, int c, int* reach = nullptr) {
    const CondDev& C = a.cond[c];
    const double* F = a.G.freq;
    const double f0 = F[0];
    const double df = a.G.df;
    const int s = a.G.start, e = a.G.start + a.G.points;
    const double nu = a.L.nu[i];
    if (c == 0 && i > 0 && nu < a.L.nu[i - 1]) atomicOr(a.err, kErrUnsorted);
    const bool streamed = KIND == kVoigt && CONV == kConvGpu && a.L.s32 != nullptr;
    // per-temperature cache: read S(T) and (T_ref/T)^n, or compute and store
    const bool tc_read = a.L.tc_mode == 1, tc_write = a.L.tc_mode == 2;
    const bool from_lines = !streamed && !tc_read;
    const double ei = from_lines ? a.L.energies[i] : 0.0;
    const double aif = from_lines ? a.L.aif[i] : 0.0;
    const double gns = from_lines ? double(a.L.gns[i]) : 0.0;
    const double cut = C.cut;
    const size_t ci = size_t(c) * size_t(a.L.n) + size_t(i);
    int kcl = 0;

    // Intensity, centre used for offsets, and the reference window.
    double S, nu_p;
    int lo, hi;
    if (CONV == kConvGpu) {
        if (KIND == kVoigt) {
            // device_compute_cross_section_voigt_stepone, cross_kernal.cu:775-779
            double nu_if = nu;
            if (nu_if == 0) nu_if = 1e-6;
            if (streamed) {
                S = double(a.L.s32[i]);
            } else if (tc_read) {
                S = a.L.tc_s[i];
            } else {
                S = C.cmcoef * aif * gns * kISQRTPI * exp(-C.beta * ei) * (1.0 - exp(-C.beta * nu_if)) /
                    (nu_if * nu_if * C.partition);
                if (gns == -1) S = aif;
            }
        } else if (tc_read) {
            S = a.L.tc_s[i];
        } else {
            // doppler_stepone / stepone, cross_kernal.cu:645-648, :487-490
            S = C.cmcoef * aif * gns * exp(-C.beta * ei) * (1.0 - exp(-C.beta * nu)) /
                (nu * nu * C.partition);
            if (nu == 0) S = 0.0;
        }
        nu_p = nu;  // step two reads the uploaded centre (cross_kernal.cu:951)
        if (KIND == kGauss) {
            // |f - nu| <= cut with dnu = f - nu (cross_kernal.cu:599-602)
            lo = find_first(s, e, ceil((nu - cut - f0) / df),
                            [&](int j) { return !(F[j] - nu < -cut); });
            hi = find_first(s, e, ceil((nu + cut - f0) / df),
                            [&](int j) { return F[j] - nu > cut; });
        } else {
            // -cut <= nu - f <= cut (cross_kernal.cu:952-957, :684-687)
            lo = find_first(s, e, ceil((nu - cut - f0) / df),
                            [&](int j) { return !(nu - F[j] > cut); });
            hi = find_first(s, e, ceil((nu + cut - f0) / df),
                            [&](int j) { return nu - F[j] < -cut; });
        }
    } else {
        // OpenMPManager::ComputeVoigt / ComputeDoppler, OpenMPManager.cpp:196-208, :151-163
        double nu_if = nu;
        if (nu_if == 0) nu_if = 1e-6;
        if (tc_read)
            S = a.L.tc_s[i];
        else if (KIND == kVoigt)
            S = C.cmcoef * aif * gns * kISQRTPI * exp(-C.beta * ei) * (1.0 - exp(-C.beta * nu_if)) /
                (nu_if * nu_if * C.partition);
        else
            S = C.cmcoef * aif * gns * exp(-C.beta * ei) * (1.0 - exp(-C.beta * nu_if)) /
                (nu_if * nu_if * C.partition);
        nu_p = nu_if;
        const double rb = round((nu_if - cut - f0) / df);
        const double re = round((nu_if + cut - f0) / df);
        // ib = max(rb, start), ie = min(re, start + points); both clamped into
        // [s, e] so the arrays stay monotone (an empty range stays empty).
        lo = clamp_index(rb > double(s) ? rb : double(s), s, e);
        hi = clamp_index(re < double(e) ? re : double(e), s, e);
        // Lines with S == 0 are skipped (OpenMPManager.cpp:163, :208); they
        // keep their window (monotone arrays) and add exactly 0 below.
    }

    if (tc_write) a.L.tc_s[i] = S;
    if (KIND == kVoigt) {
        double pw = 0.0;
        if (!streamed) {
            pw = tc_read ? a.L.tc_pw[i] : pow(C.tratio, a.L.nexp[i]);
            if (tc_write) a.L.tc_pw[i] = pw;
        }
        const double gl = streamed ? double(a.L.gl32[i]) : a.L.gamma[i] * C.gamma_scale * pw;
        const double g = 1.0 / (nu_p * C.dpw);  // gammaG, cross_kernal.cu:958
        const double y = gl * g;
        const double pref = (CONV == kConvCpu && S == 0.0) ? 0.0 : S * g;
        const double y2 = y * y;
        const double Pc = pref * kW4C * y;
        const double Cy = y2 - 0.5;
        const double D2 = 2.0 * y2;
        const double m = rint((nu_p - f0) / df);
        // Grid indices where |x| + y < 15 is possible (region I not
        // guaranteed), with a margin of two points either side.
        double clo_d = 3.0e7, chi_d = -3.0e7;
        if (y < 15.0) {
            double h = (15.0 - y) / g;
            h = h * (1.0 + 1e-9) + 1e-12 * fabs(nu_p);
            clo_d = floor((nu_p - h - f0) / df) - 2.0;
            chi_d = ceil((nu_p + h - f0) / df) + 2.0;
            if (!(clo_d > -3.0e7)) clo_d = -3.0e7;
            if (!(chi_d < 3.0e7)) chi_d = 3.0e7;
        }
        // FP32 offsets need |m| < 2^24 and x below ~1e8 over the window;
        // otherwise every pair of the line takes the per-pair path.
        bool whole = false;
        if (MIXED) {
            const double xw = (cut + double(a.mixed_tile_span + 4) * df) * g;
            whole = !(fabs(m) < 16000000.0) || !(xw < kWholeXMax);
        }
        if (whole) {
            clo_d = -3.0e7;
            chi_d = 3.0e7;
            kcl = 30000000;
        } else if (chi_d >= clo_d) {
            const double w = fmax(m - clo_d, chi_d - m) + 1.0;
            kcl = w < 3.0e7 ? int(w) : 30000000;
        }
        if (c == 0) a.mi[i] = int(fmin(fmax(m, -1073741824.0), 1073741824.0));
        if (!MIXED && a.group > 0) {
            // FP64 multi-condition layout (conditions of a group share the
            // window).
            const int C = a.group;
            const int cg = c / C, cl = c - cg * C;
            const size_t gi = size_t(cg) * size_t(a.L.n) + size_t(i);
            int core = -1;
            if (whole) {
                core = 0x7fff | (0x7fff << 16);
            } else if (chi_d >= clo_d) {
                const int aa = int(fmin(m - clo_d, 32767.0));
                const int bb = int(fmin(chi_d - m, 32767.0));
                core = aa | (bb << 16);
            }
            {
                CondRec64 cr;
                cr.g = g;
                cr.Cy = Cy;
                cr.D2 = D2;
                cr.Pc = Pc;
                cr.y = y;
                cr.pref = pref;
                cr.core = core;
                cr.pad0 = cr.pad1 = cr.pad2 = 0;
                reinterpret_cast<CondRec64*>(a.rec)[gi * C + cl] = cr;
                if (cl == 0) {
                    LineSh64 ls;
                    ls.nu = nu_p;
                    ls.lo = lo;
                    ls.hi = hi;
                    reinterpret_cast<LineSh64*>(a.lsh)[gi] = ls;
                }
            }
            if (cl == 0) {
                a.wlo[gi] = lo;
                a.whi[gi] = hi;
            }
            return kcl;
        }
        if (MIXED) {
            RecV32 rr;
            rr.m = float(fabs(m) < 16000000.0 ? m : 0.0);
            rr.ra = float(((nu_p - f0) - m * df) * g);
            rr.dfa = float(whole ? -df * g : df * g);  // negative: x from the FP64 centre
            rr.Cy = float(Cy);
            rr.D2 = float(D2);
            rr.Pc = float(Pc);
            rr.pref = float(pref);
            rr.y = float(y);
            rr.lo = float(lo);
            rr.hi = float(hi);
            // exact intervals: step two leaves [clo, chi] to the core pass
            int j15, k15, j55, k55;
            region_intervals(nu_p, g, y, lo, hi, f0, df, j15, k15, j55, k55);
            int rch = 0;
            if (j15 <= k15) {
                const double w = fmax(m - double(j15), double(k15) - m);
                rch = w < 3.0e7 ? int(w) : 30000000;
                if (!(w < 3.0e7)) atomicOr(a.err, kErrReach);  // the core pass would not find it
            }
            if (reach) *reach = rch;
            kcl = whole ? 30000000 : rch;  // a whole line is a core candidate of every tile
            rr.clo = float(j15);
            rr.chi = float(k15);
            rr.lo55 = float(j55);
            rr.hi55 = float(k55);
            rr.nu = nu_p;
            reinterpret_cast<RecV32*>(a.rec)[ci] = rr;
        } else {
            RecV64 rr;
            rr.nu = nu_p;
            rr.g = g;
            rr.Cy = Cy;
            rr.D2 = D2;
            rr.Pc = Pc;
            rr.y = y;
            rr.pref = pref;
            rr.pad = 0.0;
            rr.lo = lo;
            rr.hi = hi;
            rr.clo = int(clo_d);
            rr.chi = int(chi_d);
            reinterpret_cast<RecV64*>(a.rec)[ci] = rr;
        }
    } else {
        // Doppler / Gaussian: pairs whose two erf arguments are both beyond
        // kErfSat on the same side add exactly 0; narrow the window to the
        // rest (with margins), keeping it monotone in nu.
        double g = 0.0, lo_f, hi_f;
        if (KIND == kDoppler) {
            g = 1.0 / (nu_p * C.dpw);
            const double w = kErfSat * C.dpw * (1.0 + 1e-6);
            const double abs_m = a.x0 * (1.0 + 1e-6) + 2.0 * df;
            lo_f = nu_p * (1.0 - w) - abs_m;
            hi_f = nu_p * (1.0 + w) + abs_m;
        } else {
            const double wg = (kErfSat + a.x0g) / a.xg * (1.0 + 1e-6) + 2.0 * df;
            lo_f = nu_p - wg;
            hi_f = nu_p + wg;
        }
        const int alo = clamp_index(floor((lo_f - f0) / df), s, e);
        const int ahi = clamp_index(ceil((hi_f - f0) / df) + 1.0, s, e);
        if (alo > lo) lo = alo;
        if (ahi < hi) hi = ahi;
        RecE64 rr;
        rr.nu = nu_p;
        rr.s = (CONV == kConvCpu && S == 0.0) ? 0.0 : S;
        rr.g = g;
        rr.pad = 0.0;
        rr.lo = lo;
        rr.hi = hi;
        rr.pad0 = rr.pad1 = 0;
        reinterpret_cast<RecE64*>(a.rec)[ci] = rr;
    }
    a.wlo[ci] = lo;
    a.whi[ci] = hi;
    return kcl;
}

template <int KIND, int CONV, bool MIXED>
__global__ void __launch_bounds__(256) k_prep(PrepArgs a) {
    const long i = a.line0 + long(blockIdx.x) * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    int kcl = 0, rch = 0;
    if (i < (a.line1 > 0 ? a.line1 : a.L.n)) kcl = prep_line<KIND, CONV, MIXED>(a, i, c, &rch);
    if (KIND == kVoigt) {
        // Block maxima of the core widths (kc) and, mixed, of the core pass's
        // reach (kc + kMaxCond), one atomic each per block.
        __shared__ int smax[2][8];
        kcl = __reduce_max_sync(0xffffffffu, kcl);
        rch = __reduce_max_sync(0xffffffffu, rch);
        if ((threadIdx.x & 31) == 0) {
            smax[0][threadIdx.x >> 5] = kcl;
            smax[1][threadIdx.x >> 5] = rch;
        }
        __syncthreads();
        if (threadIdx.x < 2) {
            int m = 0;
            for (int w = 0; w < int(blockDim.x >> 5); ++w) m = smax[threadIdx.x][w] > m ? smax[threadIdx.x][w] : m;
            if (m > 0) atomicMax(a.kc + threadIdx.x * kMaxCond + c, m);
        }
    }
}

// Step one of the mixed-precision multi-condition layout, one thread per line
// over every group of C conditions.  The line's data is read once; the
// intensity, the Lorentz temperature power and 1/Doppler width of each
// temperature class (conditions with the same beta, Q, T_ref/T and Doppler
// width; the 40-condition sweep has 10) are computed once per line and kept
// in shared memory (up to kMaxClassCache classes; beyond, each condition
// computes its own); what groups with the same cut share -- the window, the
// condition-free offsets (LineShX) -- is written once per run of such
// groups; the conditions follow in order, their loop not unrolled, which
// keeps the code small.  Each value takes the FP64 path's operations in the
// same order (the W4 region intervals are the FP64 region choice).  A
// line's LineR1 of a group is written by one thread within a short time, so
// whole sectors reach memory.  The core-candidate reach (kc) covers the
// pairs where x^2 + y^2 < kNearR2, at least one grid point beyond: there the
// region-I rational may exceed W4 by far, and step two tests u on the lines
// of that reach.
template <int CONV, int C>
__global__ void __launch_bounds__(256, 3) k_prep_lines_x(PrepArgs a) {
    static_assert(C % 2 == 0, "conditions come in pairs");
    extern __shared__ __align__(16) double cls[];  // [3][ncache][256]: S, (T_ref/T)^n, g
    __shared__ int smax[2][kMaxCond][8];
    const int ngroups = a.ncond / C;
    const long i = a.line0 + long(blockIdx.x) * 256 + threadIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool live = i < (a.line1 > 0 ? a.line1 : a.L.n);
    const double* F = a.G.freq;
    const double f0 = F[0];
    const double df = a.G.df;
    const int s = a.G.start, e = a.G.start + a.G.points;

    double nu = 0.0, ei = 0.0, aif = 0.0, gns = 0.0, gam = 0.0, nex = 0.0;
    if (live) {
        nu = a.L.nu[i];
        if (i > 0 && nu < a.L.nu[i - 1]) atomicOr(a.err, kErrUnsorted);
        ei = a.L.energies[i];
        aif = a.L.aif[i];
        gns = double(a.L.gns[i]);
        gam = a.L.gamma[i];
        nex = a.L.nexp[i];
    }
    double nu_if = nu;
    if (nu_if == 0) nu_if = 1e-6;
    // step two reads the uploaded centre in the GPU convention
    // (cross_kernal.cu:951), the nu = 0 guarded one in the CPU convention
    const double nu_p = CONV == kConvGpu ? nu : nu_if;
    const double md = (nu_p - f0) / df;
    const double m = rint(md);
    const double nu_df = nu_p / df;  // q = 1 / (g df) = nu_df * dpw
    const double tb = region_tol_base(nu_p, f0, df, md);
    const bool far_m = !(fabs(m) < 16000000.0);
    const int im = int(fmin(fmax(m, -1073741824.0), 1073741824.0));
    if (live) a.mi[i] = im;

    // device_compute_cross_section_voigt_stepone, cross_kernal.cu:775-779
    // (GPU); OpenMPManager.cpp:196-200 (CPU)
    auto class_values = [&](const CondDev& Cd, double& S, double& pw, double& g) {
        S = Cd.cmcoef * aif * gns * kISQRTPI * exp(-Cd.beta * ei) * (1.0 - exp(-Cd.beta * nu_if)) /
            (nu_if * nu_if * Cd.partition);
        if (CONV == kConvGpu && gns == -1) S = aif;
        pw = pow(Cd.tratio, nex);
        g = 1.0 / (nu_p * Cd.dpw);  // gammaG, cross_kernal.cu:958
    };
    const int ncache = a.nclass <= kMaxClassCache ? a.nclass : 0;
    double* cS = cls;
    double* cP = cls + ncache * 256;
    double* cG = cls + 2 * ncache * 256;
    if (live) {
        for (int t = 0; t < ncache; ++t)
            class_values(a.cond[a.class_rep[t]], cS[t * 256 + tid], cP[t * 256 + tid], cG[t * 256 + tid]);
    }

    // Window data (LineShX, lo, hi) once per run of groups with the same cut
    // (a.wslot), written when the run ends: its wide flag covers every
    // condition of the run.
    double cut_prev = -1.0;
    int lo = s, hi = s;
    int slot = -1;
    bool wide = false;
    auto flush_window = [&]() {
        if (!live || slot < 0) return;
        const size_t wi = size_t(slot) * size_t(a.L.n) + size_t(i);
        LineShX ls;
        ls.m = float(far_m ? 0.0 : m);
        ls.dfn = float(df / nu_p);
        ls.rn = float(((nu_p - f0) - m * df) / nu_p);
        ls.flags = (far_m ? kLineWhole : 0) | (wide ? kLineWide : 0);
        ls.lo = lo;
        ls.hi = hi;
        ls.nu = nu_p;
        reinterpret_cast<LineShX*>(a.lsh)[wi] = ls;
        a.wlo[wi] = lo;
        a.whi[wi] = hi;
    };
    for (int cg = 0; cg < ngroups; ++cg) {
        if (a.wslot[cg] != slot) {
            flush_window();
            slot = a.wslot[cg];
            wide = false;
            const double cut = a.cond[cg * C].cut;  // a run of groups shares its cut
            cut_prev = cut;
            if (live) {
                if (CONV == kConvGpu) {
                    // -cut <= nu - f <= cut (cross_kernal.cu:952-957)
                    lo = find_first(s, e, ceil((nu - cut - f0) / df), [&](int j) { return !(nu - F[j] > cut); });
                    hi = find_first(s, e, ceil((nu + cut - f0) / df), [&](int j) { return nu - F[j] < -cut; });
                } else {
                    // OpenMPManager.cpp:196-208
                    const double rb = round((nu_if - cut - f0) / df);
                    const double re = round((nu_if + cut - f0) / df);
                    lo = clamp_index(rb > double(s) ? rb : double(s), s, e);
                    hi = clamp_index(re < double(e) ? re : double(e), s, e);
                }
            }
        }
        const size_t gi = size_t(cg) * size_t(a.L.n) + size_t(live ? i : 0);
        LineR1<C>& lr = reinterpret_cast<LineR1<C>*>(a.rec)[gi];
        if constexpr (C == 2) {
            if (live) lr.pad[0] = lr.pad[1] = 0.0f;
        }
#pragma unroll 1
        for (int k = 0; k < C; ++k) {
            const int c = cg * C + k;
            const CondDev& Cd = a.cond[c];
            int kcl = 0, rch = 0;
            if (live) {
                double S, pw, g;
                if (ncache) {
                    const int t = a.tclass[c];
                    S = cS[t * 256 + tid];
                    pw = cP[t * 256 + tid];
                    g = cG[t * 256 + tid];
                } else {
                    class_values(Cd, S, pw, g);
                }
                const double gl = gam * Cd.gamma_scale * pw;
                const double y = gl * g;
                const double pref = (CONV == kConvCpu && S == 0.0) ? 0.0 : S * g;
                const double y2 = y * y;
                const double Pc = pref * kW4C * y;
                const double xw = (cut_prev + double(a.mixed_tile_span + 4) * df) * g;
                const bool whole = far_m || !(xw < kWholeXMax);
                // the shared reciprocals need the products in range
                wide = wide || !(xw * xw + y2 < kPairUMax) || !(fabs(Pc) < kPairPcMax);
                CoreIv iv;
                const double q = nu_df * Cd.dpw;
                region_interval_q(nu_p, g, y, 15.0, lo, hi, f0, df, md, q, tb, iv.lo15, iv.hi15);
                region_interval_q(nu_p, g, y, 5.5, lo, hi, f0, df, md, q, tb, iv.lo55, iv.hi55);
                if (iv.lo15 <= iv.hi15) {
                    // in integers where m is one (|m| < 1.6e7, grid indices
                    // below 1.5e7: no overflow)
                    bool over;
                    if (far_m) {
                        const double w = fmax(m - double(iv.lo15), double(iv.hi15) - m);
                        over = !(w < 3.0e7);
                        rch = over ? 30000000 : int(w);
                    } else {
                        rch = max(im - iv.lo15, iv.hi15 - im);
                        over = rch >= 30000000;
                        if (over) rch = 30000000;
                    }
                    if (over) atomicOr(a.err, kErrReach);  // the core pass would not find it
                    // |md - j| < sqrt(kNearR2 - y^2) q, |md - m| <= 1/2, one
                    // point of margin, plus one (0: none)
                    // (in FP32, widened by 1e-6 for its rounding)
                    if (y2 < kNearR2)
                        kcl = int(fminf(ceilf(sqrtf(float(kNearR2 - y2)) * float(q) * 1.000001f + 0.5f), 3.0e7f)) + 2;
                }
                if (whole) kcl = 30000000;  // a core candidate of every tile
                const size_t ci = size_t(c) * size_t(a.L.n) + size_t(i);
                a.civ[ci] = iv;
                a.cyp[ci] = make_float2(float(y), float(pref));
                lr.Cy[k] = float(y2 - 0.5);
                lr.D2[k] = float(2.0 * y2);
                lr.Pc[k] = float(Pc);
            }
            kcl = __reduce_max_sync(0xffffffffu, kcl);
            rch = __reduce_max_sync(0xffffffffu, rch);
            if (lane == 0) {
                smax[0][c][warp] = kcl;
                smax[1][c][warp] = rch;
            }
        }
    }
    flush_window();
    // block maxima of the core-candidate widths (kc) and of the core pass's
    // reach (kc + kMaxCond), one atomic each per block and condition
    __syncthreads();
    for (int idx = tid; idx < 2 * a.ncond; idx += 256) {
        const int which = idx / a.ncond, c = idx - which * a.ncond;
        int mx = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) mx = smax[which][c][w] > mx ? smax[which][c][w] : mx;
        if (mx > 0) atomicMax(a.kc + (which ? kMaxCond : 0) + c, mx);
    }
}

// ---------------------------------------------------------------------------
// Step two helpers.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// First i in [lo, hi) with pred(i) true (pred monotone), or hi; 32-way
// ballot search by one warp.  Lanes 0..30 probe the ends of 31 segments of
// `step` indices; lane 31 stands for the rest of the range and is taken as
// true, so the ballot is never empty inside the loop.
template <class Pred>
__device__ long warp_lower_bound(long lo, long hi, int lane, Pred pred) {
    while (hi - lo > 32) {
        const long step = (hi - lo + 31) / 32;
        const long q = lo + long(lane + 1) * step - 1;
        const bool v = (lane < 31 && q < hi) ? pred(q) : true;
        const unsigned b = __ballot_sync(0xffffffffu, v);
        const int f = __ffs(b) - 1;
        const long nlo = lo + long(f) * step;
        if (f < 31) {
            const long qf = lo + long(f + 1) * step - 1;
            hi = qf < hi ? qf : hi;
        }
        lo = nlo;
    }
    const long q = lo + lane;
    const bool v = (q < hi) ? pred(q) : true;
    const unsigned b = __ballot_sync(0xffffffffu, v);
    if (b == 0u) return hi;
    const long r = lo + (__ffs(b) - 1);
    return r < hi ? r : hi;
}

// Copy `cnt` records of REC (sizeof a multiple of 16) into shared memory,
// 16 bytes per lane per step.
template <class REC>
__device__ __forceinline__ void stage(REC* dst, const REC* src, int cnt, int lane) {
    constexpr int kChunks = sizeof(REC) / 16;
    const int total = cnt * kChunks;
    const char* s = reinterpret_cast<const char*>(src);
    char* d = reinterpret_cast<char*>(dst);
    for (int q = lane; q < total; q += 32) cp_async16(d + 16 * q, s + 16 * q);
}

struct WorkItem {
    int c, t0, t1, s;
};

// Items are (condition, tile, split), splits innermost: the parts of one
// tile run side by side and share its records in L2.
__device__ __forceinline__ bool next_item(const StepArgs& a, int P, int lane, WorkItem& w) {
    int item = 0;
    if (lane == 0) item = int(atomicAdd(a.counter, 1u));
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= a.n_items) return false;
    const int per_cond = a.tiles_per_cond * a.splits;
    w.c = item / per_cond;
    const int rem = item - w.c * per_cond;
    const int tile = rem / a.splits;
    w.s = rem - tile * a.splits;
    w.t0 = a.G.start + tile * 32 * P;
    const int end = a.G.start + a.G.points;
    w.t1 = w.t0 + 32 * P < end ? w.t0 + 32 * P : end;
    return true;
}

// Split s of `splits` takes the 32-line groups s, s + splits, s + 2 splits,
// ... of the tile's lines [La, Lb): interleaved, so that the costly lines
// near the tile (cores) are shared evenly between the splits.
__device__ __forceinline__ int split_groups(long nl, int splits, int s) {
    const int all = int((nl + 31) / 32);
    return all > s ? (all - s + splits - 1) / splits : 0;
}

// Where item (c, s) puts the sum of grid point j: added to out, or stored to
// its part when the tile is split.
__device__ __forceinline__ void put_result(const StepArgs& a, int c, int s, int j, double v) {
    if (a.splits <= 1)
        a.out[size_t(a.row[c]) * a.out_stride + size_t(j)] += v;
    else
        a.part[(size_t(c) * a.splits + s) * a.part_stride + size_t(j - a.G.start)] = v;
}

// ---------------------------------------------------------------------------
// Step two, Voigt.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float rcp_approx_f32(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// 1/x: the hardware approximation refined by one Newton-Raphson step
// (r <- r + r (1 - x r)), which squares its relative error.
__device__ __forceinline__ double rcp_refined_f64(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    const double e = fma(-x, r, 1.0);
    return fma(r, e, r);
}

struct fcplx {
    float re, im;
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2s(float a) { return make_float2(a, a); }
__device__ __forceinline__ fcplx operator+(float a, fcplx b) { return {a + b.re, b.im}; }
__device__ __forceinline__ fcplx operator*(fcplx a, fcplx b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}

// W4 region II (5.5 <= |x| + y < 15) as a real expression with the factor y
// explicit.  With T = y - ix, U = T^2 = Ur + i Ui, N = a + b U and
// D = c + U (3 + U):
//   Re[T N / D] = y [(a + b y^2 - 3 b x^2) Dr + 2 x^2 (3 + 2 Ur)(Nr + 2 b y^2)] / |D|^2
// (expanding Re[T N conj(D)]); a complex evaluation would cancel by a factor
// x / y in the wings of narrow lines.
// a / b for the FP32 W4 forms of regions II and III (no cancellation
// follows there): the hardware reciprocal and one product, within 2 ulp; the
// denominators lie between about 0.5 and 1e6, far from the range where the
// approximation fails.  Region IV, which subtracts, keeps the IEEE division.
__device__ __forceinline__ float region_div(float a, float b) { return __fdividef(a, b); }

template <class R>
__device__ __forceinline__ R w4_region2_re(R x, R y) {
    const R a = R(1.410474), b = R(.5641896), c = R(.75);
    const R x2 = x * x, y2 = y * y;
    const R ur = y2 - x2, ui = R(-2) * x * y;
    const R nr = a + b * ur;
    const R dr = c + R(3) * ur + ur * ur - ui * ui;
    const R di = ui * (R(3) + R(2) * ur);
    const R br = (a + b * y2 - R(3) * b * x2) * dr + R(2) * x2 * (R(3) + R(2) * ur) * (nr + R(2) * b * y2);
    return region_div(y * br, dr * dr + di * di);
}

// The region-I rational of W4 in FP32 per unit pref, as step two evaluates
// it: kW4C y (u + 1) / (u^2 + 2 y^2), u = x^2 + y^2 - 0.5.  The core pass
// takes it back off the pairs where step two added it.
__device__ __forceinline__ float w4_region1_re_f32(float x, float y) {
    const float y2 = y * y;
    const float u = fmaf(x, x, y2 - 0.5f);
    return region_div(float(kW4C) * y * (u + 1.0f), fmaf(u, u, 2.0f * y2));
}

// W4 region III in FP32 (there y >= 0.195|x| - 0.176, so Re w is not small
// next to |w| and the complex form keeps its accuracy).
__device__ __forceinline__ float w4_region3_re_f32(float x, float y) {
    const fcplx t = {y, -x};
    const fcplx num = 16.4955f + t * (20.20933f + t * (11.96482f + t * (3.778987f + t * fcplx{.5642236f, 0.f})));
    const fcplx den = 16.4955f + t * (38.82363f + t * (39.27121f + t * (21.69274f + t * (6.699398f + t))));
    return region_div(num.re * den.re + num.im * den.im, den.re * den.re + den.im * den.im);
}

// a - u p for the region IV Horner schemes.
__device__ __forceinline__ fcplx fms(float a, fcplx u, fcplx p) {
    return {a - (u.re * p.re - u.im * p.im), -(u.re * p.im + u.im * p.re)};
}

// W4 region IV in FP32: Re[exp(U) - T P(U) / Q(U)], U = T^2, with
// exp(U) = exp(y^2 - x^2) (cos 2xy + i ...).  Over the region (|x| + y < 5.5,
// y < 0.195|x| - 0.176) this stays within 7e-6 of the FP64 evaluation at the
// same FP32 x, y (sampled densely with y down to 1e-9).
__device__ float w4_region4_re_f32(float x, float y) {
    const float e = expf(fmaf(y, y, -x * x)) * cosf(2.0f * x * y);
    const fcplx t = {y, -x};
    const fcplx u = t * t;
    fcplx num = fms(1.320522f, u, fcplx{.56419f, 0.f});
    num = fms(35.76683f, u, num);
    num = fms(219.0313f, u, num);
    num = fms(1540.787f, u, num);
    num = fms(3321.9905f, u, num);
    num = fms(36183.31f, u, num);
    fcplx den = fms(1.841439f, u, fcplx{1.f, 0.f});
    den = fms(61.57037f, u, den);
    den = fms(364.2191f, u, den);
    den = fms(2186.181f, u, den);
    den = fms(9022.228f, u, den);
    den = fms(24322.84f, u, den);
    den = fms(32066.6f, u, den);
    const fcplx r = t * num;
    return e - (r.re * den.re + r.im * den.im) / (den.re * den.re + den.im * den.im);
}

// Persistent step two.  For a tile [t0, t1) the lines [La, Lb) meet it;
// since the window bounds lo[] and hi[] are ascending in line order, the
// lines covering the whole tile form one contiguous run [fs, fe), and among
// those the ones whose core may reach the tile ([E, F), from the ascending
// nearest-grid-index array mi[] and the condition's widest core kc) form
// another.  So every staged group splits into at most five contiguous runs:
//   partial [La, fs) | fast [fs, E) | core [E, F) | fast [F, fe) | partial [fe, Lb)
// Fast lines evaluate W4 region I on every pair with no test at all.  Core
// and partial lines classify whole rows (outside the window: skipped; inside
// and clear of the core band: as fast; otherwise lane by lane).  Pairs that
// need W4 regions II-IV are not evaluated in place -- that would run the
// union of the region code paths with a few lanes active -- but pushed to a
// per-warp queue in shared memory and evaluated 32 at a time, one per lane;
// each lane then adds the results addressed to it, in queue order, to a
// per-lane correction column.  The order of every sum is fixed.
template <class T>
struct CoreEntry {
    T x, y, pref;
    int dest;  // lane | (row << 5)
};

template <int P, bool MIXED>
struct WarpCoreQueue {
    using T = typename std::conditional<MIXED, float, double>::type;
    static constexpr int kCap = 32 * (P + 1);  // < 32 left + up to P rows of 32 (rows of
                                               // points, or conditions)
    CoreEntry<T> q[kCap];
    T corr[P][32];
};

// Evaluates the first k (<= 32) queued pairs, one per lane, adds each result
// to its destination lane's correction column in queue order, and moves the
// rest of the queue to the front.  Returns the new queue length.  Kept out of
// line: it runs once per 32 pairs and holds all of W4's regions II-IV.
template <int P, bool MIXED>
__device__ __noinline__ int core_queue_flush(WarpCoreQueue<P, MIXED>& cq, int qn, int k, int lane) {
    static_assert(!MIXED, "the mixed paths evaluate their core pairs in a core pass");
    using T = typename WarpCoreQueue<P, MIXED>::T;
    T v = T(0);
    int dest = 0;
    if (lane < k) {
        const CoreEntry<T> e = cq.q[lane];
        dest = e.dest;
        v = T(w4_re(double(e.x), double(e.y)) * double(e.pref));
    }
    // Each push queued a run of consecutive lanes of one row, so the queue is
    // a sequence of runs (entry s + i is lane first + i).  Runs are visited in
    // queue order and each lane takes at most one entry per run: every lane's
    // correction column gets its entries in queue order.
    const int prev = __shfl_up_sync(0xffffffffu, dest, 1);
    const bool start = lane < k && (lane == 0 || dest != prev + 1 || (dest & 31) == 0);
    unsigned starts = __ballot_sync(0xffffffffu, start);
    while (starts) {
        const int s0 = __ffs(starts) - 1;
        starts &= starts - 1;
        const int e0 = starts ? __ffs(starts) - 1 : k;
        const int d0 = __shfl_sync(0xffffffffu, dest, s0);
        const int first = d0 & 31, row = d0 >> 5;
        const T vv = __shfl_sync(0xffffffffu, v, (s0 + lane - first) & 31);
        if (lane >= first && lane < first + (e0 - s0)) cq.corr[row][lane] += vv;
    }
    __syncwarp();
    const int rem = qn - k;
    for (int base = 0; base < rem; base += 32) {
        CoreEntry<T> keep;
        const int i = base + lane;
        if (i < rem) keep = cq.q[k + i];
        __syncwarp();
        if (i < rem) cq.q[i] = keep;
        __syncwarp();
    }
    return rem;
}

// Resident blocks per SM the step-two Voigt kernel asks the compiler to fit
// (register budget), FP32 path at 4 warps per block: 28 warps per SM at 4
// points per thread (72 registers), 32 at 1 or 2 (64 registers; 8 blocks of
// 24.6 KB of staging fit in shared memory); 24 for its other shapes up to 4
// points per thread.
template <int P, int WARPS, bool MIXED>
constexpr int voigt_min_blocks() {
    return (MIXED && P == 4 && WARPS == 4) ? 7 : (MIXED && P <= 2 && WARPS == 4) ? 8 : (MIXED && P <= 4) ? 24 / WARPS : 1;
}

template <int P, int WARPS, bool MIXED>
__global__ void __launch_bounds__(WARPS * 32, (voigt_min_blocks<P, WARPS, MIXED>()))
    k_steptwo_voigt(StepArgs a) {
    using REC = typename std::conditional<MIXED, RecV32, RecV64>::type;
    using T = typename std::conditional<MIXED, float, double>::type;
    using Q = WarpCoreQueue<P, MIXED>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    REC* buf = reinterpret_cast<REC*>(smem_raw) + warp * 32 * kStages;
    // the core queue (FP64 only: the mixed path leaves regions II-IV to
    // k_core_v32 and has no queue in shared memory)
    Q& cq = reinterpret_cast<Q*>(smem_raw + size_t(WARPS) * 32 * kStages * sizeof(REC))[warp];
    const REC* recs_all = reinterpret_cast<const REC*>(a.rec);
    const double* F = a.G.freq;
    const unsigned lt_mask = (1u << lane) - 1u;

    if constexpr (!MIXED) {
#pragma unroll
        for (int p = 0; p < P; ++p) cq.corr[p][lane] = T(0);
    }
    int qn = 0;  // entries in the queue (warp-uniform)

    auto push = [&](bool need, T x, T y, T pref, int p) {
        const unsigned b = __ballot_sync(0xffffffffu, need);
        if (b == 0u) return;
        if (need) {
            CoreEntry<T> e;
            e.x = x;
            e.y = y;
            e.pref = pref;
            e.dest = lane | (p << 5);
            cq.q[qn + __popc(b & lt_mask)] = e;
        }
        qn += __popc(b);
        __syncwarp();
    };

    WorkItem w;
    while (next_item(a, P, lane, w)) {
        const size_t cbase = size_t(w.c) * size_t(a.n);
        const int* whi = a.whi + cbase;
        const int* wlo = a.wlo + cbase;
        const int* mi = a.mi;
        const int kc = a.kc[w.c];
        const int t0 = w.t0, t1 = w.t1, tl = t1 - 1;
        const long La = warp_lower_bound(0, a.n, lane, [&](long i) { return whi[i] > t0; });
        const long Lb = warp_lower_bound(La, a.n, lane, [&](long i) { return wlo[i] >= t1; });
        const long fs = warp_lower_bound(La, Lb, lane, [&](long i) { return whi[i] >= t1; });
        const long Cb = warp_lower_bound(La, Lb, lane, [&](long i) { return wlo[i] > t0; });
        const long fe = Cb > fs ? Cb : fs;
        const long E = warp_lower_bound(fs, fe, lane, [&](long i) { return mi[i] >= t0 - kc; });
        const long Fc = warp_lower_bound(E, fe, lane, [&](long i) { return mi[i] > tl + kc; });
        const REC* recs = recs_all + cbase;

        int jj[P];
        float jf[P];
        double fj[P];
        float accf[P], sumf[P], cmpf[P];
        double accd[P];
#pragma unroll
        for (int p = 0; p < P; ++p) {
            jj[p] = t0 + lane + 32 * p;
            jf[p] = float(jj[p]);
            fj[p] = MIXED ? 0.0 : F[jj[p] < t1 ? jj[p] : tl];
            accf[p] = sumf[p] = cmpf[p] = 0.0f;
            accd[p] = 0.0;
        }

        // Region I on every row: u = x^2 + Cy, acc += Pc (u + 1) / (u^2 + D2);
        // in FP32 two rows at a time as packed FP32x2 operations.
        auto fast_line = [&](const REC& r) {
            if (MIXED) {
                const float4* q = reinterpret_cast<const float4*>(&r);
                const float4 v0 = q[0], v1 = q[1];
                if constexpr (P % 2 == 0) {
#pragma unroll
                    for (int p = 0; p < P; p += 2) {
                        const float2 d = __fadd2_rn(f2s(v0.x), f2(-jf[p], -jf[p + 1]));
                        const float2 xs = __ffma2_rn(d, f2s(v0.z), f2s(v0.y));
                        const float2 u = __ffma2_rn(xs, xs, f2s(v0.w));
                        const float2 den = __ffma2_rn(u, u, f2s(v1.x));
                        const float2 num = __ffma2_rn(u, f2s(v1.y), f2s(v1.y));
                        const float2 acc = __ffma2_rn(num, f2(rcp_approx_f32(den.x), rcp_approx_f32(den.y)),
                                                      f2(accf[p], accf[p + 1]));
                        accf[p] = acc.x;
                        accf[p + 1] = acc.y;
                    }
                } else {
#pragma unroll
                    for (int p = 0; p < P; ++p) {
                        const float xs = fmaf(v0.x - jf[p], v0.z, v0.y);
                        const float u = fmaf(xs, xs, v0.w);
                        accf[p] = fmaf(fmaf(u, v1.y, v1.y), rcp_approx_f32(fmaf(u, u, v1.x)), accf[p]);
                    }
                }
            } else {
                const double2* q = reinterpret_cast<const double2*>(&r);
                const double2 v0 = q[0], v1 = q[1], v2 = q[2];
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    const double xs = (v0.x - fj[p]) * v0.y;
                    const double u = fma(xs, xs, v1.x);
                    accd[p] = fma(fma(u, v2.x, v2.x), rcp_refined_f64(fma(u, u, v1.y)), accd[p]);
                }
            }
        };
        // `full`: the line's window covers the whole tile.
        auto slow_line = [&](const REC& r, bool full) {
            if (MIXED) {
                // region I except the pairs of the region interval [clo, chi]
                // (the core pass takes those)
                const float4* q = reinterpret_cast<const float4*>(&r);
                const float4 v0 = q[0], v1 = q[1], v2 = q[2];
                const float m = v0.x, ra = v0.y, dfa = v0.z, Cy = v0.w;
                const float D2 = v1.x, Pc = v1.y;
                const float lo = v2.x, hi = v2.y, clo = v2.z, chi = v2.w;
                const bool whole = dfa < 0.0f;
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    const float r0 = float(t0 + 32 * p), r1 = r0 + 31.0f;
                    if (!full && (r0 >= hi || r1 < lo)) continue;
                    const bool row_in = full || (r0 >= lo && r1 < hi);
                    const bool row_core = whole || !(r1 < clo || r0 > chi);
                    const float xs = whole ? float((r.nu - F[jj[p] < t1 ? jj[p] : tl]) / r.nu) * a.kx[w.c]
                                           : fmaf(m - jf[p], dfa, ra);
                    const float u = fmaf(xs, xs, Cy);
                    const float num = fmaf(u, Pc, Pc);
                    const float rr = rcp_approx_f32(fmaf(u, u, D2));
                    if (row_in && !row_core) {
                        accf[p] = fmaf(num, rr, accf[p]);
                        continue;
                    }
                    const bool in = row_in || (jf[p] >= lo && jf[p] < hi);
                    const bool core = jf[p] >= clo && jf[p] <= chi;
                    // beyond x ~ 1e18 (whole lines only) region I is taken as 0
                    const bool keep = in && !core && fabsf(xs) < 1.0e18f;
                    accf[p] += keep ? num * rr : 0.0f;
                }
            } else {
                const double2* q = reinterpret_cast<const double2*>(&r);
                const double2 v0 = q[0], v1 = q[1], v2 = q[2], v3 = q[3];
                const int4 vi = reinterpret_cast<const int4*>(&r)[4];
                const double nu = v0.x, g = v0.y, Cy = v1.x, D2 = v1.y, Pc = v2.x, y = v2.y;
                const double pref = v3.x;
                const int lo = vi.x, hi = vi.y, clo = vi.z, chi = vi.w;
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    const int r0 = t0 + 32 * p, r1 = r0 + 31;
                    if (!full && (r0 >= hi || r1 < lo)) continue;
                    const bool row_in = full || (r0 >= lo && r1 < hi);
                    const bool row_core = !(r1 < clo || r0 > chi);
                    const double xs = (nu - fj[p]) * g;
                    if (row_in && !row_core) {
                        const double u = fma(xs, xs, Cy);
                        accd[p] = fma(fma(u, Pc, Pc), rcp_refined_f64(fma(u, u, D2)), accd[p]);
                        continue;
                    }
                    const bool in = row_in || (jj[p] >= lo && jj[p] < hi);
                    // x and y are bit-identical to the reference's, so the
                    // region choice below is the reference's.
                    const double ax = fabs(xs);
                    const bool exact = row_core && jj[p] >= clo && jj[p] <= chi && !(ax + y >= 15.0);
                    if (in && !exact) {
                        const double u = fma(xs, xs, Cy);
                        accd[p] = fma(fma(u, Pc, Pc), rcp_refined_f64(fma(u, u, D2)), accd[p]);
                    }
                    if (row_core) push(in && exact, ax, y, pref, p);
                }
            }
        };

        // A line whose window covers only part of the tile and whose core
        // band misses it: rows outside the window are skipped, the boundary
        // row is masked lane by lane.
        auto partial_line = [&](const REC& r) {
            if (MIXED) {
                const float4* q = reinterpret_cast<const float4*>(&r);
                const float4 v0 = q[0], v1 = q[1], v2 = q[2];
                const float lo = v2.x, hi = v2.y;
                // region interval reaching the tile, or a whole line
                if (v0.z < 0.0f || !(v2.w < float(t0) || v2.z > float(tl))) {
                    slow_line(r, false);
                    return;
                }
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    const float r0 = float(t0 + 32 * p), r1 = r0 + 31.0f;
                    if (r0 >= hi || r1 < lo) continue;
                    const float xs = fmaf(v0.x - jf[p], v0.z, v0.y);
                    const float u = fmaf(xs, xs, v0.w);
                    float rr = rcp_approx_f32(fmaf(u, u, v1.x));
                    if (!(r0 >= lo && r1 < hi)) rr = (jf[p] >= lo && jf[p] < hi) ? rr : 0.0f;
                    accf[p] = fmaf(fmaf(u, v1.y, v1.y), rr, accf[p]);
                }
            } else {
                const double2* q = reinterpret_cast<const double2*>(&r);
                const double2 v0 = q[0], v1 = q[1], v2 = q[2];
                const int4 vi = reinterpret_cast<const int4*>(&r)[4];
                const int lo = vi.x, hi = vi.y;
                if (!(vi.w < t0 || vi.z > tl)) {
                    slow_line(r, false);
                    return;
                }
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    const int r0 = t0 + 32 * p, r1 = r0 + 31;
                    if (r0 >= hi || r1 < lo) continue;
                    const double xs = (v0.x - fj[p]) * v0.y;
                    const double u = fma(xs, xs, v1.x);
                    double rr = rcp_refined_f64(fma(u, u, v1.y));
                    if (!(r0 >= lo && r1 < hi)) rr = (jj[p] >= lo && jj[p] < hi) ? rr : 0.0;
                    accd[p] = fma(fma(u, v2.x, v2.x), rr, accd[p]);
                }
            }
        };
        // A line whose window covers the tile and whose core band may reach
        // it: region I on every row except the band's pairs outside region
        // I, which are queued.
        auto core_line = [&](const REC& r) {
            if (MIXED) {
                const float4* q = reinterpret_cast<const float4*>(&r);
                const float4 v0 = q[0], v1 = q[1], v2 = q[2];
                const float clo = v2.z, chi = v2.w;
                const bool whole = v0.z < 0.0f;
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    const float r0 = float(t0 + 32 * p), r1 = r0 + 31.0f;
                    const float xs = whole ? float((r.nu - F[jj[p] < t1 ? jj[p] : tl]) / r.nu) * a.kx[w.c]
                                           : fmaf(v0.x - jf[p], v0.z, v0.y);
                    const float u = fmaf(xs, xs, v0.w);
                    const float num = fmaf(u, v1.y, v1.y);
                    const float rr = rcp_approx_f32(fmaf(u, u, v1.x));
                    if (!whole && (r1 < clo || r0 > chi)) {
                        accf[p] = fmaf(num, rr, accf[p]);
                        continue;
                    }
                    // region I except the pairs of the region interval
                    const bool core = jf[p] >= clo && jf[p] <= chi;
                    const bool keep = !core && fabsf(xs) < 1.0e18f;
                    accf[p] += keep ? num * rr : 0.0f;
                }
            } else {
                const double2* q = reinterpret_cast<const double2*>(&r);
                const double2 v0 = q[0], v1 = q[1], v2 = q[2], v3 = q[3];
                const int4 vi = reinterpret_cast<const int4*>(&r)[4];
                const int clo = vi.z, chi = vi.w;
                const double y = v2.y, pref = v3.x;
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    const int r0 = t0 + 32 * p, r1 = r0 + 31;
                    const double xs = (v0.x - fj[p]) * v0.y;
                    if (r1 < clo || r0 > chi) {
                        const double u = fma(xs, xs, v1.x);
                        accd[p] = fma(fma(u, v2.x, v2.x), rcp_refined_f64(fma(u, u, v1.y)), accd[p]);
                        continue;
                    }
                    const double ax = fabs(xs);
                    const bool exact = jj[p] >= clo && jj[p] <= chi && !(ax + y >= 15.0);
                    if (!exact) {
                        const double u = fma(xs, xs, v1.x);
                        accd[p] = fma(fma(u, v2.x, v2.x), rcp_refined_f64(fma(u, u, v1.y)), accd[p]);
                    }
                    push(exact, ax, y, pref, p);
                }
            }
        };

        // this item's groups of 32 lines: gi-th starts at La + 32 (s + gi S)
        const int ngroups = split_groups(Lb - La, a.splits, w.s);
        auto gstart = [&](int gi) { return La + 32L * (w.s + long(gi) * a.splits); };
        // kStages-deep cp.async pipeline: groups gi+1 .. gi+kStages-1 are in
        // flight while group gi is evaluated (one commit per step, empty
        // commits past the end keep the group count uniform).
        auto issue = [&](int g) {
            if (g < ngroups) {
                const long b = gstart(g);
                const long rem = Lb - b;
                stage(buf + (g % kStages) * 32, recs + b, int(rem < 32 ? rem : 32), lane);
            }
            cp_async_commit();
        };
#pragma unroll
        for (int g = 0; g < kStages - 1; ++g) issue(g);
        for (int gi = 0; gi < ngroups; ++gi) {
            issue(gi + kStages - 1);
            cp_async_wait<kStages - 1>();
            __syncwarp();
            const REC* R = buf + (gi % kStages) * 32;
            const long gb = gstart(gi);
            const long ge = Lb - gb < 32 ? Lb : gb + 32;
            auto lo_of = [&](long v) { return int((v < gb ? gb : (v > ge ? ge : v)) - gb); };
            const int a0 = lo_of(La), a1 = lo_of(fs);
            const int b1 = lo_of(E), c1 = lo_of(Fc), d1 = lo_of(fe), e1 = lo_of(Lb);
            // slow lines of the three slow runs, one loop: t in [a0, a1) and
            // [d1, e1) are partial, [b1, c1) cover the tile
            for (int t = a0; t < e1; ++t) {
                if (t == a1) t = b1;  // skip the first fast run
                if (t == c1) t = d1;  // skip the second fast run
                if (t >= e1) break;
                if (t >= b1 && t < c1) core_line(R[t]);
                else partial_line(R[t]);
                if constexpr (!MIXED)
                    while (qn >= 32) qn = core_queue_flush<P, MIXED>(cq, qn, 32, lane);
            }
            {
                int t = a1;
                for (; t + 1 < b1; t += 2) {
                    fast_line(R[t]);
                    fast_line(R[t + 1]);
                }
                if (t < b1) fast_line(R[t]);
                t = c1;
                for (; t + 1 < d1; t += 2) {
                    fast_line(R[t]);
                    fast_line(R[t + 1]);
                }
                if (t < d1) fast_line(R[t]);
            }
            if (MIXED) {
                // compensated (Kahan) fold of this group's FP32 partials
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    const float part = accf[p];
                    const float yk = part - cmpf[p];
                    const float tk = sumf[p] + yk;
                    cmpf[p] = (tk - sumf[p]) - yk;
                    sumf[p] = tk;
                    accf[p] = 0.0f;
                }
            }
            __syncwarp();
        }
        cp_async_wait<0>();
        __syncwarp();
        if constexpr (!MIXED) {
            while (qn > 0) qn = core_queue_flush<P, MIXED>(cq, qn, qn < 32 ? qn : 32, lane);
#pragma unroll
            for (int p = 0; p < P; ++p) {
                accd[p] += double(cq.corr[p][lane]);
                cq.corr[p][lane] = T(0);
            }
            __syncwarp();
        }
#pragma unroll
        for (int p = 0; p < P; ++p) {
            if (jj[p] < t1) {
                const double v = MIXED ? double(sumf[p]) - double(cmpf[p]) : accd[p];
                put_result(a, w.c, w.s, jj[p], v);
            }
        }
    }
}

// Multi-condition step two, FP64: a work item is (group of C conditions that
// share one window, row of 32 grid points); each lane owns one grid point and
// C accumulators.  The line runs are found as in k_steptwo_voigt (windows and
// grid indices are shared by the group; the core run uses the group's widest
// core), and every line loads its shared record once and one small record
// per condition.
template <int C, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_steptwo_voigt_mc(StepArgs a) {
    using Q = WarpCoreQueue<C, false>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    LineSh64* lsb = reinterpret_cast<LineSh64*>(smem_raw) + warp * 64;
    CondRec64* crb = reinterpret_cast<CondRec64*>(smem_raw + size_t(WARPS) * 64 * sizeof(LineSh64)) + warp * 64 * C;
    Q& cq = reinterpret_cast<Q*>(smem_raw + size_t(WARPS) * 64 * (sizeof(LineSh64) + C * sizeof(CondRec64)))[warp];
    const double* F = a.G.freq;
    const unsigned lt_mask = (1u << lane) - 1u;

#pragma unroll
    for (int c = 0; c < C; ++c) cq.corr[c][lane] = 0.0;
    int qn = 0;
    auto push = [&](bool need, double x, double y, double pref, int c) {
        const unsigned b = __ballot_sync(0xffffffffu, need);
        if (b == 0u) return;
        if (need) {
            CoreEntry<double> e;
            e.x = x;
            e.y = y;
            e.pref = pref;
            e.dest = lane | (c << 5);
            cq.q[qn + __popc(b & lt_mask)] = e;
        }
        qn += __popc(b);
        __syncwarp();
    };

    for (;;) {
        int item = 0;
        if (lane == 0) item = int(atomicAdd(a.counter, 1u));
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= a.n_items) break;
        const int per_cond = a.tiles_per_cond * a.splits;
        const int cg = item / per_cond;
        const int tile = (item - cg * per_cond) / a.splits;
        const int split = item - cg * per_cond - tile * a.splits;
        const int t0 = a.G.start + tile * 32;
        const int end = a.G.start + a.G.points;
        const int t1 = t0 + 32 < end ? t0 + 32 : end;
        const int tl = t1 - 1;
        const size_t gbase = size_t(cg) * size_t(a.n);
        const int* whi = a.whi + gbase;
        const int* wlo = a.wlo + gbase;
        const int* mi = a.mi;
        int kc = 0;
#pragma unroll
        for (int c = 0; c < C; ++c) kc = max(kc, a.kc[cg * C + c]);
        const long La = warp_lower_bound(0, a.n, lane, [&](long i) { return whi[i] > t0; });
        const long Lb = warp_lower_bound(La, a.n, lane, [&](long i) { return wlo[i] >= t1; });
        const long fs = warp_lower_bound(La, Lb, lane, [&](long i) { return whi[i] >= t1; });
        const long Cb = warp_lower_bound(La, Lb, lane, [&](long i) { return wlo[i] > t0; });
        const long fe = Cb > fs ? Cb : fs;
        // core candidates among all the tile's lines (partial ones included):
        // only lines in [E, Fc) can have a core band that reaches the row
        const long E = warp_lower_bound(La, Lb, lane, [&](long i) { return mi[i] >= t0 - kc; });
        const long Fc = warp_lower_bound(E, Lb, lane, [&](long i) { return mi[i] > tl + kc; });
        const LineSh64* lsh = reinterpret_cast<const LineSh64*>(a.lsh) + gbase;
        const CondRec64* crec = reinterpret_cast<const CondRec64*>(a.rec) + gbase * C;

        const int jj = t0 + lane;
        const double fj = F[jj < t1 ? jj : tl];
        double accd[C];
#pragma unroll
        for (int c = 0; c < C; ++c) accd[c] = 0.0;

        // x (in Doppler widths) of this lane's point for condition record r.
        auto offset = [&](const LineSh64& s, const CondRec64& r) { return (s.nu - fj) * r.g; };
        auto region1 = [&](double xs, const CondRec64& r, double mask, int c) {
            const double u = fma(xs, xs, r.Cy);
            accd[c] = fma(fma(u, r.Pc, r.Pc), rcp_refined_f64(fma(u, u, r.D2)) * mask, accd[c]);
        };
        // One condition of a partial line, or of a line whose core band may
        // reach this row; `in`: this lane's point lies in the line's window.
        auto core_cond = [&](const LineSh64& s, const CondRec64& r, int mline, bool in, int c) {
            const double xs = offset(s, r);
            const double ax = xs < 0.0 ? -xs : xs;
            const double sx = ax + r.y;
            bool band = false;
            if (r.core != -1) {
                const int aa = r.core & 0xffff, bb = (r.core >> 16) & 0xffff;
                const int rel = jj - mline;
                band = (aa == 0x7fff || rel >= -aa) && (bb == 0x7fff || rel <= bb);
            }
            // x and y are bit-identical to the reference's, so |x| + y < 15
            // is the reference's region choice.
            const bool special = in && band && sx < 15.0;
            if (!__any_sync(0xffffffffu, special)) {
                region1(xs, r, in ? 1.0 : 0.0, c);
                return;
            }
            region1(xs, r, (in && !special) ? 1.0 : 0.0, c);
            push(special, ax, r.y, r.pref, c);
        };

        // this item's groups of 32 lines: gi-th starts at La + 32 (s + gi S)
        const int ngroups = split_groups(Lb - La, a.splits, split);
        auto gstart = [&](int gi) { return La + 32L * (split + long(gi) * a.splits); };
        auto stage_group = [&](int bufi, long b, int cnt) {
            stage(lsb + bufi * 32, lsh + b, cnt, lane);
            stage(crb + bufi * 32 * C, crec + b * C, cnt * C, lane);
        };
        if (ngroups > 0) {
            const long b = gstart(0);
            stage_group(0, b, int(Lb - b < 32 ? Lb - b : 32));
            cp_async_commit();
        }
        for (int gi = 0; gi < ngroups; ++gi) {
            if (gi + 1 < ngroups) {
                const long b = gstart(gi + 1);
                const long rem = Lb - b;
                stage_group((gi + 1) & 1, b, int(rem < 32 ? rem : 32));
                cp_async_commit();
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncwarp();
            const LineSh64* SL = lsb + (gi & 1) * 32;
            const CondRec64* SC = crb + (gi & 1) * 32 * C;
            const long gb = gstart(gi);
            const long ge = Lb - gb < 32 ? Lb : gb + 32;
            auto lo_of = [&](long v) { return int((v < gb ? gb : (v > ge ? ge : v)) - gb); };
            const int a0 = lo_of(La), a1 = lo_of(fs), b1 = lo_of(E), c1 = lo_of(Fc), d1 = lo_of(fe),
                      e1 = lo_of(Lb);
            // Runs of this group: [a1, d1) cover the row (full), the rest
            // are partial; [b1, c1) are the core candidates.
            // Full lines away from every core: region I with no test.
            auto fast_run = [&](int x, int y) {
                for (int t = x; t < y; ++t) {
                    const LineSh64 s = SL[t];
#pragma unroll
                    for (int c = 0; c < C; ++c) region1(offset(s, SC[t * C + c]), SC[t * C + c], 1.0, c);
                }
            };
            // Partial lines away from every core: region I, the window as a
            // lane mask.
            auto masked_run = [&](int x, int y) {
                for (int t = x; t < y; ++t) {
                    const LineSh64 s = SL[t];
                    const double mask = (jj >= s.lo && jj < s.hi && jj < t1) ? 1.0 : 0.0;
#pragma unroll
                    for (int c = 0; c < C; ++c) region1(offset(s, SC[t * C + c]), SC[t * C + c], mask, c);
                }
            };
            // Core candidates.  Per condition: when its core band misses the
            // row, region I with the window as a lane mask; otherwise the
            // lane-by-lane core path.
            auto cand_run = [&](int x, int y) {
                for (int t = x; t < y; ++t) {
                    const LineSh64 s = SL[t];
                    const bool full = (t >= a1 && t < d1);
                    const bool in = full || (jj >= s.lo && jj < s.hi && jj < t1);
                    const double mask = in ? 1.0 : 0.0;
                    const int mline = mi[gb + t];
                    bool any_core = false;
#pragma unroll
                    for (int c = 0; c < C; ++c) {
                        const CondRec64& r = SC[t * C + c];
                        bool hit = false;
                        if (r.core != -1) {
                            const int aa = r.core & 0xffff, bb = (r.core >> 16) & 0xffff;
                            hit = (aa == 0x7fff || mline - aa <= tl) && (bb == 0x7fff || mline + bb >= t0);
                        }
                        if (!hit) {
                            region1(offset(s, r), r, mask, c);
                        } else {
                            core_cond(s, r, mline, in, c);
                            any_core = true;
                        }
                    }
                    if (any_core)
                        while (qn >= 32) qn = core_queue_flush<C, false>(cq, qn, 32, lane);
                }
            };
            fast_run(a1, min(d1, b1));
            fast_run(max(a1, c1), d1);
            masked_run(a0, min(a1, b1));
            masked_run(max(a0, c1), a1);
            masked_run(d1, min(e1, b1));
            masked_run(max(d1, c1), e1);
            cand_run(b1, c1);
            __syncwarp();
        }
        while (qn > 0) qn = core_queue_flush<C, false>(cq, qn, qn < 32 ? qn : 32, lane);
#pragma unroll
        for (int c = 0; c < C; ++c) {
            accd[c] += cq.corr[c][lane];
            cq.corr[c][lane] = 0.0;
        }
        __syncwarp();
        if (jj < t1) {
#pragma unroll
            for (int c = 0; c < C; ++c) put_result(a, cg * C + c, split, jj, accd[c]);
        }
    }
}

// ---------------------------------------------------------------------------
// Mixed-precision multi-condition step two (Voigt), packed FP32x2.
//
// Work items, line runs and the fixed summation order are those of
// k_steptwo_voigt_mc.  Per (line, point) one condition-free offset
// X = (m - j) dfn + rn and X^2 are formed; conditions are then taken in
// pairs, each pair one packed FP32x2 operation per step of the region-I
// rational (u = X^2 k^2 + Cy, u^2 + D2, Pc (u + 1), accumulate), so a
// region-I pair costs two FP32 operations and one reciprocal per condition
// and about three issue slots in all.  The rational is added at every pair
// of the window except, on core candidates, where u < 1; k_core_mcx adds W4
// less the rational (where it was added) inside the W4 region intervals
// (|x| + y < 15, from step one).
// ---------------------------------------------------------------------------
// Resident blocks per SM the mixed multi-condition kernel asks the compiler
// to fit: 24 warps per SM (about 80 registers a thread); 28 at 8 conditions
// and 4 warps per block (72 registers; 7 blocks of 30.7 KB of staging also
// fit in shared memory), and 16 at 8 conditions and 8 warps per block (124
// registers) -- the occupancy points the autotuner chooses between through
// the block size.
template <int C, int WARPS>
constexpr int voigt_mcx_min_blocks() {
    return (C == 8 && WARPS == 8) ? 2 : (C == 8 && WARPS == 4) ? 7 : 24 / WARPS;
}

template <int C, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, (voigt_mcx_min_blocks<C, WARPS>()))
    k_steptwo_voigt_mcx(StepArgs a) {
    static_assert(C % 2 == 0, "conditions come in pairs");
    constexpr int NP = C / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    using R1 = LineR1<C>;
    // staged per line: the offsets and flags of LineShX (16 B), its window
    // (8 B) and the group's region-I records; a whole line's FP64 centre is
    // read from memory when needed
    float4* lsb = reinterpret_cast<float4*>(smem_raw) + warp * 64;
    int2* lhb = reinterpret_cast<int2*>(smem_raw + size_t(WARPS) * 64 * sizeof(float4)) + warp * 64;
    R1* rb = reinterpret_cast<R1*>(smem_raw + size_t(WARPS) * 64 * (sizeof(float4) + sizeof(int2))) + warp * 64;

    for (;;) {
        int item = 0;
        if (lane == 0) item = int(atomicAdd(a.counter, 1u));
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= a.n_items) break;
        const int per_cond = a.tiles_per_cond * a.splits;
        const int cg = item / per_cond;
        const int tile = (item - cg * per_cond) / a.splits;
        const int split = item - cg * per_cond - tile * a.splits;
        const int t0 = a.G.start + tile * 32;
        const int end = a.G.start + a.G.points;
        const int t1 = t0 + 32 < end ? t0 + 32 : end;
        const int tl = t1 - 1;
        const size_t gbase = size_t(cg) * size_t(a.n);
        const size_t wbase = size_t(a.wslot[cg]) * size_t(a.n);  // the group's window data
        const int* whi = a.whi + wbase;
        const int* wlo = a.wlo + wbase;
        const int* mi = a.mi;
        int kc = 0;
#pragma unroll
        for (int c = 0; c < C; ++c) kc = max(kc, a.kc[cg * C + c]);
        // line indices fit 32 bits (at most 2^31 - 1 lines per call)
        const int La = int(warp_lower_bound(0, a.n, lane, [&](long i) { return whi[i] > t0; }));
        const int Lb = int(warp_lower_bound(La, a.n, lane, [&](long i) { return wlo[i] >= t1; }));
        const int fs = int(warp_lower_bound(La, Lb, lane, [&](long i) { return whi[i] >= t1; }));
        const int Cb = int(warp_lower_bound(La, Lb, lane, [&](long i) { return wlo[i] > t0; }));
        const int fe = Cb > fs ? Cb : fs;
        // core candidates [E, Fc): the lines whose near-centre pairs may
        // fall in the tile (kc: the group's widest reach plus one; 0: no
        // line of the group has such pairs)
        int E = La, Fc = La;
        if (kc > 0) {
            E = int(warp_lower_bound(La, Lb, lane, [&](long i) { return mi[i] >= t0 - (kc - 1); }));
            Fc = int(warp_lower_bound(E, Lb, lane, [&](long i) { return mi[i] > tl + (kc - 1); }));
        }
        const LineShX* lsh = reinterpret_cast<const LineShX*>(a.lsh) + wbase;
        const R1* r1 = reinterpret_cast<const R1*>(a.rec) + gbase;

        const int jj = t0 + lane;
        const float jf = float(jj);
        float2 k2[NP];
        float2 acc[NP], sum[NP], cmp[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            k2[p] = f2(a.kx2[cg * C + 2 * p], a.kx2[cg * C + 2 * p + 1]);
            acc[p] = sum[p] = cmp[p] = f2(0.0f, 0.0f);
        }

        // Region I of one pair of conditions: u = X^2 k^2 + Cy,
        // acc += Pc (u + 1) / (u^2 + D2).  Pairs where `keep` is false add
        // exactly zero: the reciprocal is replaced by 0 (not multiplied by a
        // mask, so that an infinite reciprocal of a skipped pair never
        // reaches the sum).  MODE 0: plain; 1: the product itself is selected,
        // for lines whose u may overflow; 2: as 1, and a pair is kept only
        // where u >= 1 (core candidates: the core pass takes u < 1).
        auto region1 = [&](auto mode, float X2, const R1& r, int p, bool keep0, bool keep1) {
            constexpr int MODE = decltype(mode)::value;
            const float2 cy = *reinterpret_cast<const float2*>(&r.Cy[2 * p]);
            const float2 d2 = *reinterpret_cast<const float2*>(&r.D2[2 * p]);
            const float2 pc = *reinterpret_cast<const float2*>(&r.Pc[2 * p]);
            const float2 u = __ffma2_rn(f2(X2, X2), k2[p], cy);
            if constexpr (MODE == 2) {
                keep0 = keep0 && !(u.x < 1.0f);
                keep1 = keep1 && !(u.y < 1.0f);
            }
            const float2 den = __ffma2_rn(u, u, d2);
            const float2 num = __ffma2_rn(u, pc, pc);
            const float2 rr = f2(keep0 ? rcp_approx_f32(den.x) : 0.0f, keep1 ? rcp_approx_f32(den.y) : 0.0f);
            if constexpr (MODE >= 1) {
                acc[p].x += keep0 ? num.x * rr.x : 0.0f;
                acc[p].y += keep1 ? num.y * rr.y : 0.0f;
            } else {
                acc[p] = __ffma2_rn(num, rr, acc[p]);
            }
        };
        const std::integral_constant<int, 0> plain;
        const std::integral_constant<int, 2> guarded_near;
        // Region I of two pairs of conditions (A, B) with one reciprocal per
        // two line-evals: lane h of A and lane h of B share 1 / (dA dB), so
        // 1/dA = dB / (dA dB) and 1/dB = dA / (dA dB).  For narrow lines the
        // product itself stays in range (kPairUMax); for wide ones both
        // factors are scaled by kPairTau first, 1/dA = (tau dB) / (tau dA dB).
        // pA = 2q, pB = 2q + 1: conditions 4q..4q+3, one 16-byte load for each
        // of Cy, D2 and Pc.  Pairs where `keep` is false add exactly zero.
        auto region1_ab = [&](auto narrow, float X2, const R1& r, int pA, int pB, bool keep) {
            const float4 cy = *reinterpret_cast<const float4*>(&r.Cy[2 * pA]);
            const float4 d2 = *reinterpret_cast<const float4*>(&r.D2[2 * pA]);
            const float4 pc = *reinterpret_cast<const float4*>(&r.Pc[2 * pA]);
            const float2 uA = __ffma2_rn(f2(X2, X2), k2[pA], f2(cy.x, cy.y));
            const float2 uB = __ffma2_rn(f2(X2, X2), k2[pB], f2(cy.z, cy.w));
            const float2 dA = __ffma2_rn(uA, uA, f2(d2.x, d2.y));
            const float2 dB = __ffma2_rn(uB, uB, f2(d2.z, d2.w));
            const float2 nA = __ffma2_rn(uA, f2(pc.x, pc.y), f2(pc.x, pc.y));
            const float2 nB = __ffma2_rn(uB, f2(pc.z, pc.w), f2(pc.z, pc.w));
            if constexpr (decltype(narrow)::value) {
                const float2 q = __fmul2_rn(dA, dB);
                const float2 rq = keep ? f2(rcp_approx_f32(q.x), rcp_approx_f32(q.y)) : f2(0.0f, 0.0f);
                acc[pA] = __ffma2_rn(nA, __fmul2_rn(dB, rq), acc[pA]);
                acc[pB] = __ffma2_rn(nB, __fmul2_rn(dA, rq), acc[pB]);
            } else {
                const float2 aA = __fmul2_rn(dA, f2s(kPairTau));
                const float2 bB = __fmul2_rn(dB, f2s(kPairTau));
                const float2 q = __fmul2_rn(aA, dB);
                const float2 rq = keep ? f2(rcp_approx_f32(q.x), rcp_approx_f32(q.y)) : f2(0.0f, 0.0f);
                acc[pA] = __ffma2_rn(nA, __fmul2_rn(bB, rq), acc[pA]);
                acc[pB] = __ffma2_rn(nB, __fmul2_rn(aA, rq), acc[pB]);
            }
        };
        const std::true_type narrow;
        const std::false_type scaled;
        // region1_ab for a narrow core-candidate line: a condition's pair is
        // kept where the point takes the line (`in`) and u >= 1 (the core
        // pass takes u < 1); a pair that is not kept enters the shared
        // product as 1 and adds exactly zero, so the kept ones keep their
        // ranges.
        auto region1_ab_near = [&](float X2, const R1& r, int pA, int pB, bool in) {
            const float4 cy = *reinterpret_cast<const float4*>(&r.Cy[2 * pA]);
            const float4 d2 = *reinterpret_cast<const float4*>(&r.D2[2 * pA]);
            const float4 pc = *reinterpret_cast<const float4*>(&r.Pc[2 * pA]);
            const float2 uA = __ffma2_rn(f2(X2, X2), k2[pA], f2(cy.x, cy.y));
            const float2 uB = __ffma2_rn(f2(X2, X2), k2[pB], f2(cy.z, cy.w));
            const bool q0 = in && !(uA.x < 1.0f), q1 = in && !(uA.y < 1.0f);
            const bool q2 = in && !(uB.x < 1.0f), q3 = in && !(uB.y < 1.0f);
            const float2 dA0 = __ffma2_rn(uA, uA, f2(d2.x, d2.y));
            const float2 dB0 = __ffma2_rn(uB, uB, f2(d2.z, d2.w));
            const float2 nA = __ffma2_rn(uA, f2(pc.x, pc.y), f2(pc.x, pc.y));
            const float2 nB = __ffma2_rn(uB, f2(pc.z, pc.w), f2(pc.z, pc.w));
            const float2 dA = f2(q0 ? dA0.x : 1.0f, q1 ? dA0.y : 1.0f);
            const float2 dB = f2(q2 ? dB0.x : 1.0f, q3 ? dB0.y : 1.0f);
            const float2 q = __fmul2_rn(dA, dB);
            const float2 rq = f2(rcp_approx_f32(q.x), rcp_approx_f32(q.y));
            const float2 iA = __fmul2_rn(dB, rq);
            const float2 iB = __fmul2_rn(dA, rq);
            acc[pA] = __ffma2_rn(nA, f2(q0 ? iA.x : 0.0f, q1 ? iA.y : 0.0f), acc[pA]);
            acc[pB] = __ffma2_rn(nB, f2(q2 ? iB.x : 0.0f, q3 ? iB.y : 0.0f), acc[pB]);
        };

        const int ngroups = split_groups(Lb - La, a.splits, split);
        auto gstart = [&](int gi) { return La + 32 * (split + gi * a.splits); };
        auto stage_group = [&](int bufi, int b, int cnt) {
            if (lane < cnt) {
                cp_async16(lsb + bufi * 32 + lane, lsh + b + lane);
                cp_async8(lhb + bufi * 32 + lane, &lsh[b + lane].lo);
            }
            stage(rb + bufi * 32, r1 + b, cnt, lane);
        };
        if (ngroups > 0) {
            const int b = gstart(0);
            stage_group(0, b, Lb - b < 32 ? Lb - b : 32);
            cp_async_commit();
        }
        for (int gi = 0; gi < ngroups; ++gi) {
            if (gi + 1 < ngroups) {
                const int b = gstart(gi + 1);
                const int rem = Lb - b;
                stage_group((gi + 1) & 1, b, rem < 32 ? rem : 32);
                cp_async_commit();
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncwarp();
            const float4* SL = lsb + (gi & 1) * 32;  // m, df/nu, r/nu, flags
            const int2* SW = lhb + (gi & 1) * 32;    // window [lo, hi)
            const R1* SR = rb + (gi & 1) * 32;
            const int gb = gstart(gi);
            const int ge = Lb - gb < 32 ? Lb : gb + 32;
            auto lo_of = [&](int v) { return (v < gb ? gb : (v > ge ? ge : v)) - gb; };
            const int a0 = lo_of(La), a1 = lo_of(fs), b1 = lo_of(E), c1 = lo_of(Fc), d1 = lo_of(fe),
                      e1 = lo_of(Lb);
            // One line's region I at this lane's point, conditions in pairs
            // of pairs (keep: the point takes the line).
            auto line_region1 = [&](float X2, const R1& r, bool wide, bool keep) {
                if constexpr (NP % 2 == 0) {
                    if (!wide) {
#pragma unroll
                        for (int p = 0; p < NP; p += 2) region1_ab(narrow, X2, r, p, p + 1, keep);
                    } else {
#pragma unroll
                        for (int p = 0; p < NP; p += 2) region1_ab(scaled, X2, r, p, p + 1, keep);
                    }
                } else {
#pragma unroll
                    for (int p = 0; p < NP; ++p) region1(plain, X2, r, p, keep, keep);
                }
            };
            // Full lines away from every core: region I with no test.
            // Two narrow lines A, B that are not core candidates, at once: per
            // condition one reciprocal for both lines, acc += (nA dB + nB dA)
            // / (dA dB) (u >= 1 on such lines, so dA, dB >= 1; narrow lines
            // keep dA dB and the products with Pc in range, kPairUMax).  inA,
            // inB: the point takes the line (a line left out adds exactly 0).
            auto pair_step = [&](float XA2, float XB2, float2 cyA, float2 d2A, float2 pcA, float2 cyB,
                                 float2 d2B, float2 pcB, int p, bool inA, bool inB) {
                const float2 uA = __ffma2_rn(f2(XA2, XA2), k2[p], cyA);
                const float2 uB = __ffma2_rn(f2(XB2, XB2), k2[p], cyB);
                const float2 dA = __ffma2_rn(uA, uA, d2A);
                const float2 dB = __ffma2_rn(uB, uB, d2B);
                float2 nA = __ffma2_rn(uA, pcA, pcA);
                float2 nB = __ffma2_rn(uB, pcB, pcB);
                if (!inA) nA = f2(0.0f, 0.0f);
                if (!inB) nB = f2(0.0f, 0.0f);
                const float2 q = __fmul2_rn(dA, dB);
                const float2 sn = __ffma2_rn(nB, dA, __fmul2_rn(nA, dB));
                acc[p] = __ffma2_rn(sn, f2(rcp_approx_f32(q.x), rcp_approx_f32(q.y)), acc[p]);
            };
            auto pair_region1 = [&](float XA2, float XB2, const R1& ra, const R1& rb, bool inA, bool inB) {
                if constexpr (NP % 2 == 0) {
                    // conditions 4q..4q+3: one 16-byte load per array and line
#pragma unroll
                    for (int p = 0; p < NP; p += 2) {
                        const float4 cyA = *reinterpret_cast<const float4*>(&ra.Cy[2 * p]);
                        const float4 d2A = *reinterpret_cast<const float4*>(&ra.D2[2 * p]);
                        const float4 pcA = *reinterpret_cast<const float4*>(&ra.Pc[2 * p]);
                        const float4 cyB = *reinterpret_cast<const float4*>(&rb.Cy[2 * p]);
                        const float4 d2B = *reinterpret_cast<const float4*>(&rb.D2[2 * p]);
                        const float4 pcB = *reinterpret_cast<const float4*>(&rb.Pc[2 * p]);
                        pair_step(XA2, XB2, f2(cyA.x, cyA.y), f2(d2A.x, d2A.y), f2(pcA.x, pcA.y), f2(cyB.x, cyB.y),
                                  f2(d2B.x, d2B.y), f2(pcB.x, pcB.y), p, inA, inB);
                        pair_step(XA2, XB2, f2(cyA.z, cyA.w), f2(d2A.z, d2A.w), f2(pcA.z, pcA.w), f2(cyB.z, cyB.w),
                                  f2(d2B.z, d2B.w), f2(pcB.z, pcB.w), p + 1, inA, inB);
                    }
                } else {
#pragma unroll
                    for (int p = 0; p < NP; ++p)
                        pair_step(XA2, XB2, *reinterpret_cast<const float2*>(&ra.Cy[2 * p]),
                                  *reinterpret_cast<const float2*>(&ra.D2[2 * p]),
                                  *reinterpret_cast<const float2*>(&ra.Pc[2 * p]),
                                  *reinterpret_cast<const float2*>(&rb.Cy[2 * p]),
                                  *reinterpret_cast<const float2*>(&rb.D2[2 * p]),
                                  *reinterpret_cast<const float2*>(&rb.Pc[2 * p]), p, inA, inB);
                }
            };
            // Lines [x, y) that are not core candidates, two at a time; `full`:
            // their windows cover the tile, else the window is a lane mask.
            auto pair_run = [&](int x, int y, auto full) {
                auto in_of = [&](int t) {
                    if constexpr (decltype(full)::value) return true;
                    else return jj >= SW[t].x && jj < SW[t].y && jj < t1;
                };
                int t = x;
                for (; t + 1 < y; t += 2) {
                    const float4 sA = SL[t];
                    const float4 sB = SL[t + 1];
                    const float XA = fmaf(sA.x - jf, sA.y, sA.z);
                    const float XB = fmaf(sB.x - jf, sB.y, sB.z);
                    const int fA = __float_as_int(sA.w), fB = __float_as_int(sB.w);
                    const bool inA = in_of(t), inB = in_of(t + 1);
                    if (!((fA | fB) & kLineWide)) {
                        pair_region1(XA * XA, XB * XB, SR[t], SR[t + 1], inA, inB);
                    } else {
                        line_region1(XA * XA, SR[t], (fA & kLineWide) != 0, inA);
                        line_region1(XB * XB, SR[t + 1], (fB & kLineWide) != 0, inB);
                    }
                }
                if (t < y) {
                    const float4 s = SL[t];
                    const float X = fmaf(s.x - jf, s.y, s.z);
                    line_region1(X * X, SR[t], (__float_as_int(s.w) & kLineWide) != 0, in_of(t));
                }
            };
            const std::true_type full_lines;
            const std::false_type partial_lines;
            // Full lines away from every core: region I with no test.
            auto fast_run = [&](int x, int y) { pair_run(x, y, full_lines); };
            // Partial lines away from every core: the window as a lane mask.
            auto masked_run = [&](int x, int y) { pair_run(x, y, partial_lines); };
            // Core candidates: region I where u >= 1, per condition (the
            // core pass takes the pairs with u < 1, deciding on the same FP32
            // u).
            auto cand_run = [&](int x, int y) {
                for (int t = x; t < y; ++t) {
                    const float4 s = SL[t];
                    const int flags = __float_as_int(s.w);
                    const bool full = (t >= a1 && t < d1);
                    const bool in = full || (jj >= SW[t].x && jj < SW[t].y && jj < t1);
                    if constexpr (NP % 2 == 0) {
                        if (!(flags & (kLineWhole | kLineWide))) {
                            // narrow: the shared reciprocal
                            const float X = fmaf(s.x - jf, s.y, s.z);
#pragma unroll
                            for (int p = 0; p < NP; p += 2) region1_ab_near(X * X, SR[t], p, p + 1, in);
                            continue;
                        }
                    }
                    // whole lines: X from the FP64 centre (rare; the grid
                    // value is read here rather than held for every line)
                    double nu = 0.0;
                    if (flags & kLineWhole) nu = lsh[gb + t].nu;
                    const float X = (flags & kLineWhole) ? float((nu - a.G.freq[jj < t1 ? jj : tl]) / nu)
                                                         : fmaf(s.x - jf, s.y, s.z);
                    const float X2 = X * X;
                    const float aX = fabsf(X);
#pragma unroll
                    for (int p = 0; p < NP; ++p) {
                        bool keep[2];
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int c = 2 * p + h;
                            // beyond x ~ 1e9 (lines far off the FP32 offset
                            // range) region I is taken as 0
                            keep[h] = in && aX * a.kx[cg * C + c] < 1.0e9f;
                        }
                        region1(guarded_near, X2, SR[t], p, keep[0], keep[1]);
                    }
                }
            };
            fast_run(a1, min(d1, b1));
            fast_run(max(a1, c1), d1);
            masked_run(a0, min(a1, b1));
            masked_run(max(a0, c1), a1);
            masked_run(d1, min(e1, b1));
            masked_run(max(d1, c1), e1);
            cand_run(b1, c1);
            // compensated (Kahan) fold of this group's FP32 partials
            auto kahan = [](float part, float& sm, float& cm) {
                const float yk = part - cm;
                const float tk = sm + yk;
                cm = (tk - sm) - yk;
                sm = tk;
            };
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                kahan(acc[p].x, sum[p].x, cmp[p].x);
                kahan(acc[p].y, sum[p].y, cmp[p].y);
                acc[p] = f2(0.0f, 0.0f);
            }
            __syncwarp();
        }
        if (jj < t1) {
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                put_result(a, cg * C + 2 * p, split, jj, double(sum[p].x) - double(cmp[p].x));
                put_result(a, cg * C + 2 * p + 1, split, jj, double(sum[p].y) - double(cmp[p].y));
            }
        }
    }
}

// The core passes' per-warp table: row = point of the 32-point row, column =
// line of the batch (stride kCoreRow floats keeps rows 16-byte aligned and a
// quarter-warp's 128-bit row reads on distinct banks).  It starts all zero;
// each lane writes its line's entries, every lane then sums its point's row in
// line order, and each lane clears what it wrote.
constexpr int kCoreRow = 36;
__device__ __forceinline__ void core_table_clear(float (*T)[kCoreRow], int lane) {
#pragma unroll
    for (int q = 0; q < 32; q += 4) *reinterpret_cast<float4*>(&T[lane][q]) = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncwarp();
}
// Sum of this lane's row in line order.  Entries of lines that wrote nothing
// are +0, so adding only the columns of `written` (the lines that wrote
// something; few in a sparse batch) gives the same sum.  Warp-uniform.
__device__ __forceinline__ float core_table_column(float (*T)[kCoreRow], int lane, unsigned written) {
    float part = 0.0f;
    if (__popc(written) <= 8) {
        for (unsigned m = written; m != 0u; m &= m - 1u) part += T[lane][__ffs(m) - 1];
        return part;
    }
#pragma unroll
    for (int q = 0; q < 32; q += 4) {
        const float4 v = *reinterpret_cast<const float4*>(&T[lane][q]);
        part += v.x;
        part += v.y;
        part += v.z;
        part += v.w;
    }
    return part;
}

// Core pass of the mixed multi-condition layout.  A warp takes a (condition,
// row of 32 grid points); the lines whose region interval may reach the row
// form one run (the nearest grid index mi[] is ascending; the condition's
// widest interval bounds the reach), taken 32 at a time: each lane evaluates
// W4 regions II-IV (region III-IV interval from step one, region III or IV
// by Humlicek's test on the FP32 x, y) at the row's points inside its line's
// interval, less the region-I rational where step two added it, and writes
// them to a per-warp table, then each lane adds its point's column in line
// order.  Sums are FP32 per batch of 32 lines and FP64
// across batches, in a fixed order.  With line splits (blockIdx.z = split) a
// row's batches are shared out as in step two and the sums go to the parts.
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_core_mcx(CoreArgs a) {
    __shared__ __align__(16) float tab[WARPS][32][kCoreRow];  // [point][line of the batch]
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    // blockIdx.x = condition, so that the blocks of one set of rows run
    // together and the lines' shared data (LineShX, mi) comes from DRAM once
    // for all conditions; blockIdx.y steps over the sets of WARPS rows.
    const int c = int(blockIdx.x);
    const int end = a.G.start + a.G.points;
    const int row_sets = (a.G.points + 32 * WARPS - 1) / (32 * WARPS);
    float (*T)[kCoreRow] = tab[warp];
    core_table_clear(T, lane);
    const int K = a.kc[kMaxCond + c];  // the condition's core-pass reach
    const int g = c / a.group, kg = c - g * a.group;
    const CoreIv* civ = a.civ + size_t(c) * size_t(a.n);
    const float2* cyp = a.cyp + size_t(c) * size_t(a.n);
    const LineShX* lsh = a.lsh + size_t(a.wslot[g]) * size_t(a.n);
    // Cy of this condition in the group's LineR1 records (step two's u)
    const size_t r1b = line_r1_bytes(a.group);
    const unsigned char* r1 = static_cast<const unsigned char*>(a.rec) + size_t(g) * size_t(a.n) * r1b +
                              sizeof(float) * size_t(kg);
    // step two's core candidates of a row: the group's reach (kc - 1)
    int kcg = 0;
    for (int q = 0; q < a.group; ++q) kcg = max(kcg, a.kc[g * a.group + q]);
    const float k = a.kx[c], k2 = a.kx2[c];
    const int split = int(blockIdx.z), S = a.splits;
    for (int rs = int(blockIdx.y); rs < row_sets; rs += int(gridDim.y)) {
        const int t0 = a.G.start + (rs * WARPS + warp) * 32;
        if (t0 >= end) break;  // warp-uniform; later sets start further on
        const int t1 = t0 + 32 < end ? t0 + 32 : end;
        const int tl = t1 - 1;
        const long E = warp_lower_bound(0, a.n, lane, [&](long i) { return a.mi[i] >= t0 - K; });
        const long F = warp_lower_bound(E, a.n, lane, [&](long i) { return a.mi[i] > tl + K; });
        double acc = 0.0;
        for (long b = E + 32L * split; b < F; b += 32L * S) {
            const long i = b + lane;
            int jlo = 1, jhi = 0;
            if (i < F) {
                const CoreIv iv = civ[i];
                jlo = max(iv.lo15, t0);
                jhi = min(iv.hi15, tl);
                if (jlo <= jhi) {
                    const LineShX s = lsh[i];
                    const float2 yp = cyp[i];
                    const int mline = a.mi[i];
                    const bool cand = kcg > 0 && mline >= t0 - (kcg - 1) && mline <= tl + (kcg - 1);
                    const float cy = cand ? *reinterpret_cast<const float*>(r1 + size_t(i) * r1b) : 0.0f;
                    for (int j = jlo; j <= jhi; ++j) {
                        const float X = (s.flags & kLineWhole) ? float((s.nu - a.freq[j]) / s.nu)
                                                               : fmaf(s.m - float(j), s.dfn, s.rn);
                        const float ax = fabsf(X) * k, y = yp.x;
                        float w;
                        if (j >= iv.lo55 && j <= iv.hi55)
                            w = (y >= fmaf(0.195f, ax, -0.176f)) ? w4_region3_re_f32(ax, y)
                                                                  : w4_region4_re_f32(ax, y);
                        else
                            w = w4_region2_re<float>(ax, y);
                        // step two added the region-I rational here unless the
                        // line was its core candidate and u < 1 (the same FP32 u)
                        if (!(cand && fmaf(X * X, k2, cy) < 1.0f)) w -= w4_region1_re_f32(ax, y);
                        T[j - t0][lane] = yp.y * w;
                    }
                }
            }
            const unsigned written = __ballot_sync(0xffffffffu, jlo <= jhi);
            if (written == 0u) continue;  // no pair in this batch
            __syncwarp();
            acc += double(core_table_column(T, lane, written));
            __syncwarp();
            for (int j = jlo; j <= jhi; ++j) T[j - t0][lane] = 0.0f;  // back to all zeros
        }
        const int jj = t0 + lane;
        if (jj < t1) {
            if (S <= 1)
                a.out[size_t(a.row[c]) * a.out_stride + size_t(jj)] += acc;
            else
                a.part[(size_t(c) * S + split) * a.part_stride + size_t(jj - a.G.start)] += acc;
        }
    }
}

// Core pass of the single-condition mixed layout (RecV32): as k_core_mcx,
// with the region intervals [clo, chi] and [lo55, hi55] of the records; a
// line marked whole (dfa < 0) takes x from its FP64 centre.
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_core_v32(StepArgs a) {
    __shared__ __align__(16) float tab[WARPS][32][kCoreRow];  // [point][line of the batch]
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int c = int(blockIdx.y);
    const int t0 = a.G.start + (int(blockIdx.x) * WARPS + warp) * 32;
    const int end = a.G.start + a.G.points;
    if (t0 >= end) return;
    float (*T)[kCoreRow] = tab[warp];
    core_table_clear(T, lane);
    const int t1 = t0 + 32 < end ? t0 + 32 : end;
    const int tl = t1 - 1;
    const int K = a.kc[kMaxCond + c];  // the condition's core-pass reach
    const long E = warp_lower_bound(0, a.n, lane, [&](long i) { return a.mi[i] >= t0 - K; });
    const long F = warp_lower_bound(E, a.n, lane, [&](long i) { return a.mi[i] > tl + K; });
    const RecV32* recs = reinterpret_cast<const RecV32*>(a.rec) + size_t(c) * size_t(a.n);
    const float k = a.kx[c];
    const int split = int(blockIdx.z), S = a.splits;
    double acc = 0.0;
    for (long b = E + 32L * split; b < F; b += 32L * S) {
        const long i = b + lane;
        int jlo = 1, jhi = 0;
        if (i < F) {
            const RecV32 r = recs[i];
            const bool whole = r.dfa < 0.0f;
            jlo = max(int(r.clo), t0);
            jhi = min(int(r.chi), tl);
            for (int j = jlo; j <= jhi; ++j) {
                const float xs = whole ? float((r.nu - a.G.freq[j]) / r.nu) * k : fmaf(r.m - float(j), r.dfa, r.ra);
                const float ax = fabsf(xs), y = r.y;
                float w;
                if (float(j) >= r.lo55 && float(j) <= r.hi55)
                    w = (y >= fmaf(0.195f, ax, -0.176f)) ? w4_region3_re_f32(ax, y) : w4_region4_re_f32(ax, y);
                else
                    w = w4_region2_re<float>(ax, y);
                T[j - t0][lane] = r.pref * w;
            }
        }
        const unsigned written = __ballot_sync(0xffffffffu, jlo <= jhi);
        if (written == 0u) continue;  // no pair in this batch
        __syncwarp();
        acc += double(core_table_column(T, lane, written));
        __syncwarp();
        for (int j = jlo; j <= jhi; ++j) T[j - t0][lane] = 0.0f;  // back to all zeros
    }
    const int jj = t0 + lane;
    if (jj < t1) {
        if (S <= 1)
            a.out[size_t(a.row[c]) * a.out_stride + size_t(jj)] += acc;
        else
            a.part[(size_t(c) * S + split) * a.part_stride + size_t(jj - a.G.start)] += acc;
    }
}

// ---------------------------------------------------------------------------
// Step two, Doppler and Gaussian (bin-integrated erf differences, FP64).
// ---------------------------------------------------------------------------
template <int KIND, int CONV, int P, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_steptwo_erf(StepArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    RecE64* buf = reinterpret_cast<RecE64*>(smem_raw) + warp * 64;
    const RecE64* recs_all = reinterpret_cast<const RecE64*>(a.rec);
    const double* F = a.G.freq;

    WorkItem w;
    while (next_item(a, P, lane, w)) {
        const size_t cbase = size_t(w.c) * size_t(a.n);
        const int* whi = a.whi + cbase;
        const int* wlo = a.wlo + cbase;
        const int t0 = w.t0, t1 = w.t1;
        const long La = warp_lower_bound(0, a.n, lane, [&](long i) { return whi[i] > t0; });
        const long Lb = warp_lower_bound(La, a.n, lane, [&](long i) { return wlo[i] >= t1; });
        const RecE64* recs = recs_all + cbase;
        int jj[P];
        double fj[P], acc[P];
#pragma unroll
        for (int p = 0; p < P; ++p) {
            jj[p] = t0 + lane + 32 * p;
            fj[p] = F[jj[p] < t1 ? jj[p] : t1 - 1];
            acc[p] = 0.0;
        }
        // this item's groups of 32 lines: gi-th starts at La + 32 (s + gi S)
        const int ngroups = split_groups(Lb - La, a.splits, w.s);
        auto gstart = [&](int gi) { return La + 32L * (w.s + long(gi) * a.splits); };
        if (ngroups > 0) {
            const long b = gstart(0);
            stage(buf, recs + b, int(Lb - b < 32 ? Lb - b : 32), lane);
            cp_async_commit();
        }
        for (int gi = 0; gi < ngroups; ++gi) {
            if (gi + 1 < ngroups) {
                const long b = gstart(gi + 1);
                const long rem = Lb - b;
                stage(buf + ((gi + 1) & 1) * 32, recs + b, int(rem < 32 ? rem : 32), lane);
                cp_async_commit();
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncwarp();
            const RecE64* R = buf + (gi & 1) * 32;
            const long gbase = gstart(gi);
            const int cnt = int(Lb - gbase < 32 ? Lb - gbase : 32);
            for (int t = 0; t < cnt; ++t) {
                const double2* q = reinterpret_cast<const double2*>(&R[t]);
                const double2 v0 = q[0], v1 = q[1];
                const int4 vi = reinterpret_cast<const int4*>(&R[t])[2];
                const double nu = v0.x, S = v0.y, g = v1.x;
                const int lo = vi.x, hi = vi.y;
                if (hi <= t0 || lo >= t1) continue;
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    if (jj[p] >= lo && jj[p] < hi) {
                        double xp, xm;
                        if (KIND == kDoppler) {
                            // cross_kernal.cu:684-698 (GPU), OpenMPManager.cpp:165-170 (CPU)
                            const double d = (CONV == kConvGpu) ? nu - fj[p] : fabs(nu - fj[p]);
                            xp = g * ((d) + a.x0);
                            xm = g * ((d) - a.x0);
                        } else {
                            // Gaussian erf bin with dnu = f - nu (cross_kernal.cu:599-609)
                            const double d = fj[p] - nu;
                            xp = a.xg * (d) + a.x0g;
                            xm = a.xg * (d) - a.x0g;
                        }
                        acc[p] += S * (erf(xp) - erf(xm));
                    }
                }
            }
            __syncwarp();
        }
#pragma unroll
        for (int p = 0; p < P; ++p)
            if (jj[p] < t1) put_result(a, w.c, w.s, jj[p], acc[p]);
    }
}

// ---------------------------------------------------------------------------
// Sampled FP64 re-evaluation (mixed-precision error statement).
// ---------------------------------------------------------------------------
__global__ void k_check_snapshot(CheckArgs a) {
    const int c = blockIdx.y, k = blockIdx.x, lane = threadIdx.x;
    const int j = a.rows[k] + lane;
    const bool in = j < a.G.start + a.G.points;
    a.before[(size_t(c) * a.nrows + k) * 32 + lane] =
        in ? a.out[size_t(a.row[c]) * a.out_stride + size_t(j)] : 0.0;
}

// One warp per (sampled row, condition).  The lines whose window may meet the
// row are taken 32 at a time, lane = line: each lane computes its line's
// intensity, widths and window in FP64 as step one does for the FP64 path
// (cross_kernal.cu:758-790 / OpenMPManager.cpp:183-208); then, line by line
// in order, every lane adds the line's W4 value at its own point (the
// reference's region choice, w4_re) when the point lies in the line's window.
template <int CONV>
__global__ void __launch_bounds__(32) k_check_rows(CheckArgs a) {
    const int k = blockIdx.x, c = blockIdx.y, lane = threadIdx.x;
    const CondDev& C = a.cond[c];
    const double* F = a.G.freq;
    const double f0 = F[0], df = a.G.df;
    const int s = a.G.start, e = a.G.start + a.G.points;
    const int t0 = a.rows[k];
    const int t1 = t0 + 32 < e ? t0 + 32 : e;
    const int j = t0 + lane;
    const bool mine = j < t1;
    const double fj = F[mine ? j : t1 - 1];
    const double cut = C.cut;
    // lines with nu in [F[t0] - cut - 2 df, F[t1 - 1] + cut + 2 df]
    const double lo_nu = F[t0] - cut - 2.0 * df, hi_nu = F[t1 - 1] + cut + 2.0 * df;
    const long La = warp_lower_bound(0, a.L.n, lane, [&](long i) { return a.L.nu[i] >= lo_nu; });
    const long Lb = warp_lower_bound(La, a.L.n, lane, [&](long i) { return a.L.nu[i] > hi_nu; });
    double acc = 0.0;
    for (long b = La; b < Lb; b += 32) {
        const long i = b + lane;
        double nu_p = 0.0, g = 0.0, y = 0.0, pref = 0.0;
        int ib = 0, ie = 0;
        if (i < Lb) {
            const double nu = a.L.nu[i];
            const double ei = a.L.energies[i], aif = a.L.aif[i], gns = double(a.L.gns[i]);
            double nu_if = nu;
            if (nu_if == 0) nu_if = 1e-6;
            double S = C.cmcoef * aif * gns * kISQRTPI * exp(-C.beta * ei) *
                       (1.0 - exp(-C.beta * nu_if)) / (nu_if * nu_if * C.partition);
            if (CONV == kConvGpu && gns == -1) S = aif;
            nu_p = CONV == kConvGpu ? nu : nu_if;
            const double gl = a.L.gamma[i] * C.gamma_scale * pow(C.tratio, a.L.nexp[i]);
            g = 1.0 / (nu_p * C.dpw);
            y = gl * g;
            pref = (CONV == kConvCpu && S == 0.0) ? 0.0 : S * g;
            if (CONV == kConvCpu) {
                const double rb = round((nu_if - cut - f0) / df);
                const double re = round((nu_if + cut - f0) / df);
                ib = clamp_index(rb > double(s) ? rb : double(s), s, e);
                ie = clamp_index(re < double(e) ? re : double(e), s, e);
            }
        }
        const int cnt = Lb - b < 32 ? int(Lb - b) : 32;
        for (int t = 0; t < cnt; ++t) {
            const double lnu = __shfl_sync(0xffffffffu, nu_p, t);
            const double lg = __shfl_sync(0xffffffffu, g, t);
            const double ly = __shfl_sync(0xffffffffu, y, t);
            const double lp = __shfl_sync(0xffffffffu, pref, t);
            const int lib = __shfl_sync(0xffffffffu, ib, t);
            const int lie = __shfl_sync(0xffffffffu, ie, t);
            const double d = lnu - fj;
            const bool in = CONV == kConvGpu ? (!(d > cut) && !(d < -cut)) : (j >= lib && j < lie);
            if (mine && in) acc += lp * w4_re(d * lg, ly);
        }
    }
    a.ref[(size_t(c) * a.nrows + k) * 32 + lane] = mine ? acc : 0.0;
}

// Per condition: the comparison of what the call added at the sampled
// points (out after minus out before) with the FP64 sums.
__global__ void __launch_bounds__(32) k_check_stats(CheckArgs a) {
    const int c = blockIdx.x, lane = threadIdx.x;
    const int e = a.G.start + a.G.points;
    double peak = 0.0;
    for (int k = 0; k < a.nrows; ++k) {
        const double r = a.ref[(size_t(c) * a.nrows + k) * 32 + lane];
        peak = fmax(peak, fabs(r));
    }
    for (int o = 16; o > 0; o >>= 1) peak = fmax(peak, __shfl_xor_sync(0xffffffffu, peak, o));
    double mx = 0.0, sr = 0.0, sd = 0.0;
    for (int k = 0; k < a.nrows; ++k) {
        const int j = a.rows[k] + lane;
        if (j >= e) continue;
        const size_t q = (size_t(c) * a.nrows + k) * 32 + lane;
        const double r = a.ref[q];
        const double got = a.out[size_t(a.row[c]) * a.out_stride + size_t(j)] - a.before[q];
        if (fabs(r) > 1e-6 * peak) mx = fmax(mx, fabs(got - r) / fabs(r));
        sr += r;
        sd += got - r;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        sd += __shfl_xor_sync(0xffffffffu, sd, o);
    }
    if (lane == 0) {
        a.stats[4 * c + 0] = mx;
        a.stats[4 * c + 1] = sr;
        a.stats[4 * c + 2] = sd;
        a.stats[4 * c + 3] = peak;
    }
}

// Sums the parts of split tiles in part order and adds them to out.
__global__ void k_reduce_splits(StepArgs a, int ncond_out) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    const long pts = a.G.points;
    if (i >= pts * ncond_out) return;
    const int c = int(i / pts);
    const long j = i - long(c) * pts;
    const double* p = a.part + size_t(c) * a.splits * a.part_stride + size_t(j);
    double v = 0.0;
    for (int s = 0; s < a.splits; ++s) v += p[size_t(s) * a.part_stride];
    a.out[size_t(a.row[c]) * a.out_stride + size_t(a.G.start + j)] += v;
}

template <class K>
int blocks_per_sm(K kernel, int threads, size_t smem) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess)
        return 1;
    return n > 0 ? n : 1;
}

template <int P, int WARPS, bool MIXED>
cudaError_t run_voigt(int blocks, const StepArgs& a, cudaStream_t st, int* occ) {
    using REC = typename std::conditional<MIXED, RecV32, RecV64>::type;
    const size_t smem = size_t(WARPS) * (32 * kStages * sizeof(REC) + (MIXED ? 0 : sizeof(WarpCoreQueue<P, MIXED>)));
    if (smem > 48 * 1024) {
        if (cudaFuncSetAttribute(k_steptwo_voigt<P, WARPS, MIXED>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
            return cudaGetLastError();
    }
    if (occ) {
        *occ = blocks_per_sm(k_steptwo_voigt<P, WARPS, MIXED>, WARPS * 32, smem);
        return cudaSuccess;
    }
    k_steptwo_voigt<P, WARPS, MIXED><<<blocks, WARPS * 32, smem, st>>>(a);
    return cudaGetLastError();
}

template <int C, int WARPS>
cudaError_t run_voigt_mc(int blocks, const StepArgs& a, cudaStream_t st, int* occ) {
    const size_t smem = size_t(WARPS) * (64 * (sizeof(LineSh64) + C * sizeof(CondRec64)) +
                                         sizeof(WarpCoreQueue<C, false>));
    if (smem > 48 * 1024) {
        if (cudaFuncSetAttribute(k_steptwo_voigt_mc<C, WARPS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem)) != cudaSuccess)
            return cudaGetLastError();
    }
    if (occ) {
        *occ = blocks_per_sm(k_steptwo_voigt_mc<C, WARPS>, WARPS * 32, smem);
        return cudaSuccess;
    }
    k_steptwo_voigt_mc<C, WARPS><<<blocks, WARPS * 32, smem, st>>>(a);
    return cudaGetLastError();
}

template <int C, int WARPS>
cudaError_t run_voigt_mcx(int blocks, const StepArgs& a, cudaStream_t st, int* occ) {
    const size_t smem = size_t(WARPS) * 64 * (sizeof(float4) + sizeof(int2) + sizeof(LineR1<C>));
    if (smem > 48 * 1024) {
        if (cudaFuncSetAttribute(k_steptwo_voigt_mcx<C, WARPS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem)) != cudaSuccess)
            return cudaGetLastError();
    }
    if (occ) {
        *occ = blocks_per_sm(k_steptwo_voigt_mcx<C, WARPS>, WARPS * 32, smem);
        return cudaSuccess;
    }
    k_steptwo_voigt_mcx<C, WARPS><<<blocks, WARPS * 32, smem, st>>>(a);
    return cudaGetLastError();
}

template <int WARPS, bool MIXED>
cudaError_t dispatch_mc_c(int C, int blocks, const StepArgs& a, cudaStream_t st, int* occ) {
    if (MIXED) {
        switch (C) {
            case 2: return run_voigt_mcx<2, WARPS>(blocks, a, st, occ);
            case 4: return run_voigt_mcx<4, WARPS>(blocks, a, st, occ);
            case 8: return run_voigt_mcx<8, WARPS>(blocks, a, st, occ);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (C) {
        case 2: return run_voigt_mc<2, WARPS>(blocks, a, st, occ);
        case 4: return run_voigt_mc<4, WARPS>(blocks, a, st, occ);
        case 8: return run_voigt_mc<8, WARPS>(blocks, a, st, occ);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t dispatch_mc(bool mixed, int C, int warps, int blocks, const StepArgs& a,
                        cudaStream_t st, int* occ) {
    if (warps == 4) return mixed ? dispatch_mc_c<4, true>(C, blocks, a, st, occ)
                                 : dispatch_mc_c<4, false>(C, blocks, a, st, occ);
    if (warps == 8) return mixed ? dispatch_mc_c<8, true>(C, blocks, a, st, occ)
                                 : dispatch_mc_c<8, false>(C, blocks, a, st, occ);
    return cudaErrorInvalidValue;
}

template <int KIND, int CONV, int P, int WARPS>
cudaError_t run_erf(int blocks, const StepArgs& a, cudaStream_t st, int* occ) {
    const size_t smem = size_t(WARPS) * 64 * sizeof(RecE64);
    if (occ) {
        *occ = blocks_per_sm(k_steptwo_erf<KIND, CONV, P, WARPS>, WARPS * 32, smem);
        return cudaSuccess;
    }
    k_steptwo_erf<KIND, CONV, P, WARPS><<<blocks, WARPS * 32, smem, st>>>(a);
    return cudaGetLastError();
}

template <int WARPS, bool MIXED>
cudaError_t dispatch_voigt_p(int P, int blocks, const StepArgs& a, cudaStream_t st, int* occ) {
    switch (P) {
        case 1: return run_voigt<1, WARPS, MIXED>(blocks, a, st, occ);
        case 2: return run_voigt<2, WARPS, MIXED>(blocks, a, st, occ);
        case 4: return run_voigt<4, WARPS, MIXED>(blocks, a, st, occ);
        case 8: return run_voigt<8, WARPS, MIXED>(blocks, a, st, occ);
        default: return cudaErrorInvalidValue;
    }
}

template <int KIND, int CONV, int WARPS>
cudaError_t dispatch_erf_p(int P, int blocks, const StepArgs& a, cudaStream_t st, int* occ) {
    switch (P) {
        case 1: return run_erf<KIND, CONV, 1, WARPS>(blocks, a, st, occ);
        case 2: return run_erf<KIND, CONV, 2, WARPS>(blocks, a, st, occ);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t dispatch_steptwo(int kind, int conv, bool mixed, int P, int warps, int blocks,
                             const StepArgs& a, cudaStream_t st, int* occ) {
    if (kind == kVoigt) {
        if (warps == 4) return mixed ? dispatch_voigt_p<4, true>(P, blocks, a, st, occ)
                                     : dispatch_voigt_p<4, false>(P, blocks, a, st, occ);
        if (warps == 8) return mixed ? dispatch_voigt_p<8, true>(P, blocks, a, st, occ)
                                     : dispatch_voigt_p<8, false>(P, blocks, a, st, occ);
        return cudaErrorInvalidValue;
    }
    if (warps != 4 && warps != 8) return cudaErrorInvalidValue;
    if (kind == kDoppler) {
        if (conv == kConvGpu)
            return warps == 4 ? dispatch_erf_p<kDoppler, kConvGpu, 4>(P, blocks, a, st, occ)
                              : dispatch_erf_p<kDoppler, kConvGpu, 8>(P, blocks, a, st, occ);
        return warps == 4 ? dispatch_erf_p<kDoppler, kConvCpu, 4>(P, blocks, a, st, occ)
                          : dispatch_erf_p<kDoppler, kConvCpu, 8>(P, blocks, a, st, occ);
    }
    if (kind == kGauss)
        return warps == 4 ? dispatch_erf_p<kGauss, kConvGpu, 4>(P, blocks, a, st, occ)
                          : dispatch_erf_p<kGauss, kConvGpu, 8>(P, blocks, a, st, occ);
    return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t launch_grid_check(const GridDev& g, unsigned* err, cudaStream_t stream) {
    if (g.npoints_total < 2) return cudaSuccess;
    const int n = g.npoints_total - 1;
    k_grid_check<<<(n + 255) / 256, 256, 0, stream>>>(g, err);
    return cudaGetLastError();
}

cudaError_t launch_check_snapshot(const CheckArgs& a, cudaStream_t stream) {
    if (a.nrows <= 0 || a.ncond <= 0) return cudaSuccess;
    k_check_snapshot<<<dim3(unsigned(a.nrows), unsigned(a.ncond)), 32, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_check_rows(const CheckArgs& a, cudaStream_t stream) {
    if (a.nrows <= 0 || a.ncond <= 0) return cudaSuccess;
    const dim3 grid(unsigned(a.nrows), unsigned(a.ncond));
    if (a.conv == kConvGpu) k_check_rows<kConvGpu><<<grid, 32, 0, stream>>>(a);
    else k_check_rows<kConvCpu><<<grid, 32, 0, stream>>>(a);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    k_check_stats<<<unsigned(a.ncond), 32, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_reduce_splits(const StepArgs& a, int ncond_out, cudaStream_t stream) {
    if (a.splits <= 1 || a.G.points <= 0 || ncond_out <= 0) return cudaSuccess;
    const long n = long(a.G.points) * ncond_out;
    k_reduce_splits<<<unsigned((n + 255) / 256), 256, 0, stream>>>(a, ncond_out);
    return cudaGetLastError();
}

cudaError_t launch_prep(int kind, int conv, bool mixed, const PrepArgs& a, cudaStream_t stream) {
    const long count = (a.line1 > 0 ? a.line1 : a.L.n) - a.line0;
    if (count <= 0 || a.ncond <= 0) return cudaSuccess;
    const dim3 grid(unsigned((count + 255) / 256), unsigned(a.ncond));
    if (kind == kVoigt && mixed && a.group > 0) {
        // (precomputed-intensity lists run one condition at a time)
        if (a.L.s32 != nullptr || a.ncond % a.group != 0) return cudaErrorInvalidValue;
        const unsigned nblk = unsigned((count + 255) / 256);
        const int ncache = a.nclass <= kMaxClassCache ? a.nclass : 0;
        const size_t smem = sizeof(double) * 3 * size_t(ncache) * 256;
        auto go = [&](auto kernel) {
            if (smem > 48 * 1024 &&
                cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
                return cudaGetLastError();
            kernel<<<nblk, 256, smem, stream>>>(a);
            return cudaGetLastError();
        };
        switch (a.group) {
            case 2: return conv == kConvGpu ? go(k_prep_lines_x<kConvGpu, 2>) : go(k_prep_lines_x<kConvCpu, 2>);
            case 4: return conv == kConvGpu ? go(k_prep_lines_x<kConvGpu, 4>) : go(k_prep_lines_x<kConvCpu, 4>);
            case 8: return conv == kConvGpu ? go(k_prep_lines_x<kConvGpu, 8>) : go(k_prep_lines_x<kConvCpu, 8>);
            default: return cudaErrorInvalidValue;
        }
    } else if (kind == kVoigt) {
        if (conv == kConvGpu) {
            if (mixed) k_prep<kVoigt, kConvGpu, true><<<grid, 256, 0, stream>>>(a);
            else k_prep<kVoigt, kConvGpu, false><<<grid, 256, 0, stream>>>(a);
        } else {
            if (mixed) k_prep<kVoigt, kConvCpu, true><<<grid, 256, 0, stream>>>(a);
            else k_prep<kVoigt, kConvCpu, false><<<grid, 256, 0, stream>>>(a);
        }
    } else if (kind == kDoppler) {
        if (conv == kConvGpu) k_prep<kDoppler, kConvGpu, false><<<grid, 256, 0, stream>>>(a);
        else k_prep<kDoppler, kConvCpu, false><<<grid, 256, 0, stream>>>(a);
    } else if (kind == kGauss) {
        k_prep<kGauss, kConvGpu, false><<<grid, 256, 0, stream>>>(a);
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_steptwo(int kind, int conv, bool mixed, int P, int warps, int blocks,
                           const StepArgs& a, cudaStream_t stream) {
    if (blocks <= 0 || a.n_items <= 0) return cudaSuccess;
    return dispatch_steptwo(kind, conv, mixed, P, warps, blocks, a, stream, nullptr);
}

int steptwo_blocks_per_sm(int kind, int conv, bool mixed, int P, int warps) {
    StepArgs dummy{};
    int occ = 0;
    if (dispatch_steptwo(kind, conv, mixed, P, warps, 0, dummy, nullptr, &occ) != cudaSuccess)
        return 0;
    return occ;
}

cudaError_t launch_core_v32(const StepArgs& a, int ncond, cudaStream_t stream) {
    if (a.n <= 0 || a.G.points <= 0 || ncond <= 0) return cudaSuccess;
    constexpr int W = 4;
    const int rows = (a.G.points + 31) / 32;
    const unsigned S = unsigned(a.splits > 1 ? a.splits : 1);
    k_core_v32<W><<<dim3(unsigned((rows + W - 1) / W), unsigned(ncond), S), W * 32, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_core_mcx(const CoreArgs& a, int ncond, cudaStream_t stream) {
    if (a.n <= 0 || a.G.points <= 0 || ncond <= 0) return cudaSuccess;
    constexpr int W = 4;
    const int rows = (a.G.points + 31) / 32;
    const unsigned S = unsigned(a.splits > 1 ? a.splits : 1);
    const int sets = (rows + W - 1) / W;
    k_core_mcx<W><<<dim3(unsigned(ncond), unsigned(sets < 65535 ? sets : 65535), S), W * 32, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_steptwo_mc(bool mixed, int C, int warps, int blocks, const StepArgs& a,
                              cudaStream_t stream) {
    if (blocks <= 0 || a.n_items <= 0) return cudaSuccess;
    return dispatch_mc(mixed, C, warps, blocks, a, stream, nullptr);
}

int steptwo_mc_blocks_per_sm(bool mixed, int C, int warps) {
    StepArgs dummy{};
    int occ = 0;
    if (dispatch_mc(mixed, C, warps, 0, dummy, nullptr, &occ) != cudaSuccess) return 0;
    return occ;
}

size_t record_bytes(int kind, bool mixed) {
    if (kind == kVoigt) return mixed ? sizeof(RecV32) : sizeof(RecV64);
    return sizeof(RecE64);
}

ScratchPlan plan_scratch(int kind, bool mixed, size_t n, int ncond, size_t base_off, int group) {
    auto al = [](size_t v) { return (v + 255) / 256 * 256; };
    ScratchPlan p;
    const size_t nwin = group > 0 ? size_t((ncond + group - 1) / group) : size_t(ncond);
    // records: per (line, condition), or for the mixed multi-condition layout
    // one LineR1<group> per (line, group)
    const size_t rec_bytes = group > 0 ? (mixed ? line_r1_bytes(group) * n * nwin
                                                : sizeof(CondRec64) * n * size_t(ncond))
                                       : record_bytes(kind, mixed) * n * size_t(ncond);
    p.off_rec = al(base_off);
    p.off_wlo = al(p.off_rec + rec_bytes);
    p.off_whi = al(p.off_wlo + sizeof(int) * n * nwin);
    p.off_mi = al(p.off_whi + sizeof(int) * n * nwin);
    p.off_kc = al(p.off_mi + sizeof(int) * n);
    p.off_lsh = al(p.off_kc + sizeof(int) * size_t(kKcWords));
    const size_t lsh = mixed ? sizeof(LineShX) : sizeof(LineSh64);
    p.off_civ = al(p.off_lsh + (group > 0 ? lsh * n * nwin : 0));
    const bool core = mixed && group > 0;
    p.off_cyp = al(p.off_civ + (core ? sizeof(CoreIv) * n * size_t(ncond) : 0));
    p.need = al(p.off_cyp + (core ? sizeof(float2) * n * size_t(ncond) : 0));
    return p;
}

}  // namespace xs
