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

// ---------------------------------------------------------------------------
// Small complex arithmetic for the W4 regions II-IV.
// ---------------------------------------------------------------------------
struct cplx {
    double re, im;
};
__device__ __forceinline__ cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
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
template <int KIND, int CONV, bool MIXED>
__global__ void __launch_bounds__(256) k_prep(PrepArgs a) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (i >= a.L.n) return;
    const CondDev& C = a.cond[c];
    const double* F = a.G.freq;
    const double f0 = F[0];
    const double df = a.G.df;
    const int s = a.G.start, e = a.G.start + a.G.points;
    const double nu = a.L.nu[i];
    if (c == 0 && i > 0 && nu < a.L.nu[i - 1]) atomicOr(a.err, kErrUnsorted);
    const double ei = a.L.energies[i];
    const double aif = a.L.aif[i];
    const double gns = double(a.L.gns[i]);
    const double cut = C.cut;
    const size_t ci = size_t(c) * size_t(a.L.n) + size_t(i);

    // Intensity, centre used for offsets, and the reference window.
    double S, nu_p;
    int lo, hi;
    if (CONV == kConvGpu) {
        if (KIND == kVoigt) {
            // device_compute_cross_section_voigt_stepone, cross_kernal.cu:775-779
            double nu_if = nu;
            if (nu_if == 0) nu_if = 1e-6;
            S = C.cmcoef * aif * gns * kISQRTPI * exp(-C.beta * ei) * (1.0 - exp(-C.beta * nu_if)) /
                (nu_if * nu_if * C.partition);
            if (gns == -1) S = aif;
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
        if (KIND == kVoigt)
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

    if (KIND == kVoigt) {
        const double gl = a.L.gamma[i] * C.gamma_scale * pow(C.tratio, a.L.nexp[i]);
        const double g = 1.0 / (nu_p * C.dpw);  // gammaG, cross_kernal.cu:958
        const double y = gl * g;
        const double pref = (CONV == kConvCpu && S == 0.0) ? 0.0 : S * g;
        const double y2 = y * y;
        const double Pc = pref * kW4C * y;
        const double Qc = Pc * (0.5 + y2);
        const double B = 2.0 * y2 - 1.0;
        const double A2 = (0.5 + y2) * (0.5 + y2);
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
        AuxV64* aux = reinterpret_cast<AuxV64*>(a.aux) + ci;
        *aux = AuxV64{nu_p, g, y, pref};
        if (MIXED) {
            const double m = rint((nu_p - f0) / df);
            const double r = (nu_p - f0) - m * df;
            // FP32 offsets need |m| < 2^24 and x below ~1e8 over the window.
            const double xw = (cut + double(a.mixed_tile_span + 4) * df) * g;
            if (!(fabs(m) < 16000000.0) || !(xw < 1.0e8)) {
                clo_d = -3.0e7;
                chi_d = 3.0e7;
            }
            RecV32 rr;
            rr.m = float(fabs(m) < 16000000.0 ? m : 0.0);
            rr.ra = float(r * g);
            rr.dfa = float(df * g);
            rr.B = float(B);
            rr.A2 = float(A2);
            rr.Pc = float(Pc);
            rr.Qc = float(Qc);
            rr.y = float(y);
            rr.lo = float(lo);
            rr.hi = float(hi);
            rr.clo = float(clo_d);
            rr.chi = float(chi_d);
            reinterpret_cast<RecV32*>(a.rec)[ci] = rr;
        } else {
            RecV64 rr;
            rr.nu = nu_p;
            rr.g = g;
            rr.B = B;
            rr.A2 = A2;
            rr.Pc = Pc;
            rr.Qc = Qc;
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
}

// ---------------------------------------------------------------------------
// Step two helpers.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
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

// Copy `cnt` records of REC (sizeof a multiple of 16) into shared memory.
template <class REC>
__device__ __forceinline__ void stage(REC* dst, const REC* src, int cnt, int lane) {
    constexpr int kChunks = sizeof(REC) / 16;
    const int total = cnt * kChunks;
    const char* s = reinterpret_cast<const char*>(src);
    char* d = reinterpret_cast<char*>(dst);
#pragma unroll
    for (int k = 0; k < kChunks; ++k) {
        const int q = lane + 32 * k;
        if (q < total) cp_async16(d + 16 * q, s + 16 * q);
    }
}

struct WorkItem {
    int c, t0, t1;
};

__device__ __forceinline__ bool next_item(const StepArgs& a, int P, int lane, WorkItem& w) {
    int item = 0;
    if (lane == 0) item = int(atomicAdd(a.counter, 1u));
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= a.n_items) return false;
    w.c = item / a.tiles_per_cond;
    const int tile = item - w.c * a.tiles_per_cond;
    w.t0 = a.G.start + tile * 32 * P;
    const int end = a.G.start + a.G.points;
    w.t1 = w.t0 + 32 * P < end ? w.t0 + 32 * P : end;
    return true;
}

// ---------------------------------------------------------------------------
// Step two, Voigt.
// ---------------------------------------------------------------------------
template <int P, int WARPS, bool MIXED>
__global__ void __launch_bounds__(WARPS * 32) k_steptwo_voigt(StepArgs a) {
    using REC = typename std::conditional<MIXED, RecV32, RecV64>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    REC* buf = reinterpret_cast<REC*>(smem_raw) + warp * 64;
    const REC* recs_all = reinterpret_cast<const REC*>(a.rec);
    const double* F = a.G.freq;

    WorkItem w;
    while (next_item(a, P, lane, w)) {
        const size_t cbase = size_t(w.c) * size_t(a.n);
        const int* whi = a.whi + cbase;
        const int* wlo = a.wlo + cbase;
        const int t0 = w.t0, t1 = w.t1;
        const long La = warp_lower_bound(0, a.n, lane, [&](long i) { return whi[i] > t0; });
        const long Lb = warp_lower_bound(La, a.n, lane, [&](long i) { return wlo[i] >= t1; });
        const REC* recs = recs_all + cbase;
        const AuxV64* aux = a.aux + cbase;

        int jj[P];
        float jf[P];
        double fj[P];
        float accf[P], sumf[P], cmpf[P];
        double accd[P];
#pragma unroll
        for (int p = 0; p < P; ++p) {
            jj[p] = t0 + lane + 32 * p;
            jf[p] = float(jj[p]);
            const int jc = jj[p] < t1 ? jj[p] : t1 - 1;
            fj[p] = MIXED ? 0.0 : F[jc];
            accf[p] = sumf[p] = cmpf[p] = 0.0f;
            accd[p] = 0.0;
        }
        const float t0f = float(t0), tlf = float(t1 - 1);

        const long nl = Lb - La;
        const int ngroups = int((nl + 31) / 32);
        if (ngroups > 0) {
            stage(buf, recs + La, int(nl < 32 ? nl : 32), lane);
            cp_async_commit();
        }
        for (int gi = 0; gi < ngroups; ++gi) {
            if (gi + 1 < ngroups) {
                const long b = La + 32L * (gi + 1);
                const long rem = Lb - b;
                stage(buf + ((gi + 1) & 1) * 32, recs + b, int(rem < 32 ? rem : 32), lane);
                cp_async_commit();
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncwarp();
            const REC* R = buf + (gi & 1) * 32;
            const long gbase = La + 32L * gi;
            const int cnt = int(Lb - gbase < 32 ? Lb - gbase : 32);
            for (int t = 0; t < cnt; ++t) {
                if (MIXED) {
                    const float4* q = reinterpret_cast<const float4*>(&R[t]);
                    const float4 v0 = q[0], v1 = q[1], v2 = q[2];
                    const float m = v0.x, ra = v0.y, dfa = v0.z, B = v0.w;
                    const float A2 = v1.x, Pc = v1.y, Qc = v1.z, y = v1.w;
                    const float lo = v2.x, hi = v2.y, clo = v2.z, chi = v2.w;
                    const bool fast = (lo <= t0f) && (tlf < hi) && ((tlf < clo) || (t0f > chi));
                    if (fast) {
#pragma unroll
                        for (int p = 0; p < P; ++p) {
                            const float xs = fmaf(m - jf[p], dfa, ra);
                            const float x2 = xs * xs;
                            const float den = fmaf(x2, x2 + B, A2);
                            const float num = fmaf(x2, Pc, Qc);
                            accf[p] += __fdividef(num, den);
                        }
                    } else {
#pragma unroll
                        for (int p = 0; p < P; ++p) {
                            if (jf[p] >= lo && jf[p] < hi) {
                                const float xs = fmaf(m - jf[p], dfa, ra);
                                const float ax = fabsf(xs);
                                const bool r1 = (jf[p] < clo || jf[p] > chi) && (ax + y >= 15.0f) &&
                                                (ax < 1.0e8f);
                                if (r1) {
                                    const float x2 = xs * xs;
                                    const float den = fmaf(x2, x2 + B, A2);
                                    const float num = fmaf(x2, Pc, Qc);
                                    accf[p] += __fdividef(num, den);
                                } else {
                                    const AuxV64 ax64 = aux[gbase + t];
                                    const double x = fabs(ax64.nu - F[jj[p]]) * ax64.g;
                                    accf[p] += float(w4_re(x, ax64.y) * ax64.pref);
                                }
                            }
                        }
                    }
                } else {
                    const double2* q = reinterpret_cast<const double2*>(&R[t]);
                    const double2 v0 = q[0], v1 = q[1], v2 = q[2];
                    const int4 vi = reinterpret_cast<const int4*>(&R[t])[3];
                    const double nu = v0.x, g = v0.y, B = v1.x, A2 = v1.y, Pc = v2.x, Qc = v2.y;
                    const int lo = vi.x, hi = vi.y, clo = vi.z, chi = vi.w;
                    const bool fast = (lo <= t0) && (t1 - 1 < hi) && ((t1 - 1 < clo) || (t0 > chi));
                    if (fast) {
#pragma unroll
                        for (int p = 0; p < P; ++p) {
                            const double xs = (nu - fj[p]) * g;
                            const double x2 = xs * xs;
                            const double den = fma(x2, x2 + B, A2);
                            const double num = fma(x2, Pc, Qc);
                            accd[p] += num / den;
                        }
                    } else {
#pragma unroll
                        for (int p = 0; p < P; ++p) {
                            if (jj[p] >= lo && jj[p] < hi) {
                                const AuxV64 ax64 = aux[gbase + t];
                                const double x = fabs(nu - fj[p]) * g;
                                accd[p] += w4_re(x, ax64.y) * ax64.pref;
                            }
                        }
                    }
                }
            }
            if (MIXED) {
                // Compensated (Kahan) fold of this group's FP32 partials.
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    const float yk = accf[p] - cmpf[p];
                    const float tk = sumf[p] + yk;
                    cmpf[p] = (tk - sumf[p]) - yk;
                    sumf[p] = tk;
                    accf[p] = 0.0f;
                }
            }
            __syncwarp();
        }
        double* out = a.out + size_t(w.c) * a.out_stride;
#pragma unroll
        for (int p = 0; p < P; ++p) {
            if (jj[p] < t1) {
                const double v = MIXED ? double(sumf[p]) - double(cmpf[p]) : accd[p];
                out[jj[p]] += v;
            }
        }
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
        const long nl = Lb - La;
        const int ngroups = int((nl + 31) / 32);
        if (ngroups > 0) {
            stage(buf, recs + La, int(nl < 32 ? nl : 32), lane);
            cp_async_commit();
        }
        for (int gi = 0; gi < ngroups; ++gi) {
            if (gi + 1 < ngroups) {
                const long b = La + 32L * (gi + 1);
                const long rem = Lb - b;
                stage(buf + ((gi + 1) & 1) * 32, recs + b, int(rem < 32 ? rem : 32), lane);
                cp_async_commit();
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncwarp();
            const RecE64* R = buf + (gi & 1) * 32;
            const long gbase = La + 32L * gi;
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
        double* out = a.out + size_t(w.c) * a.out_stride;
#pragma unroll
        for (int p = 0; p < P; ++p)
            if (jj[p] < t1) out[jj[p]] += acc[p];
    }
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
    const size_t smem = size_t(WARPS) * 64 * sizeof(REC);
    if (occ) {
        *occ = blocks_per_sm(k_steptwo_voigt<P, WARPS, MIXED>, WARPS * 32, smem);
        return cudaSuccess;
    }
    k_steptwo_voigt<P, WARPS, MIXED><<<blocks, WARPS * 32, smem, st>>>(a);
    return cudaGetLastError();
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

cudaError_t launch_prep(int kind, int conv, bool mixed, const PrepArgs& a, cudaStream_t stream) {
    if (a.L.n <= 0 || a.ncond <= 0) return cudaSuccess;
    const dim3 grid(unsigned((a.L.n + 255) / 256), unsigned(a.ncond));
    if (kind == kVoigt) {
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

size_t record_bytes(int kind, bool mixed) {
    if (kind == kVoigt) return mixed ? sizeof(RecV32) : sizeof(RecV64);
    return sizeof(RecE64);
}

size_t aux_bytes(int kind, bool mixed) {
    (void)mixed;
    return kind == kVoigt ? sizeof(AuxV64) : 0;
}

}  // namespace xs
