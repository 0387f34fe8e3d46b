/*
 * CPU oracle for the cross-section hot path.  TEST INFRASTRUCTURE ONLY:
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load this
 * library as the checker.  The product (gpu_cross_b200) never links or calls
 * it and has no CPU fallback.
 *
 * It restates, in plain C, the two backends of the reference
 * (ahmed-f-alrefaie/gpu_cross), whose arithmetic differs (see the notes at
 * each function):
 *
 *   "GPU convention"  cross_kernal.cu  step one + step two block kernels,
 *                     driven by GpuManager (GPUManager.cpp:24-47, 107-148).
 *   "CPU convention"  OpenMPManager.cpp ComputeVoigt / ComputeDoppler /
 *                     TransferResults.
 *
 * Pinning: the reference has no tests and no golden vectors.  The CPU
 * convention is pinned bit-for-bit against the reference's own OpenMPManager
 * compiled from its sources (oracle/Makefile -> oracle/_ref/libref_cpu.so,
 * fixtures in tests/golden/).  The GPU convention is pinned against the
 * reference's own kernels compiled for sm_100a (oracle/_ref/libref_gpu.so,
 * run on a B200; fixtures in tests/golden/).  The GAUSSIAN step two is NOT
 * pinned: the reference kernel reads a constant that GpuManager never sets
 * and stops early on ascending input (see oracle_gpu_gaussian).
 *
 * Physical constants are the reference's defines.h:4-20 values, and the
 * GpuManager host literals (GPUManager.cpp:28-31), which are equal.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* defines.h:4-20 */
#define O_LN2 0.69314718056
#define O_ISQRTPI 0.564189584
#define O_PI 3.14159265359
#define O_PLANCK 6.6260693e-27
#define O_VELLGT 2.99792458e+10
#define O_BOLTZ 1.380658e-16
#define O_NA 6.0221412927e23
#define O_DOPPLER_CUTOFF 100

/* Thread counts of the reference launchers (cross_kernal.cuh:9-16). */
#define O_VOIGT_BLOCK 128
#define O_BLOCK_SIZE 576

typedef struct {
    double half_width;
    double temperature;
    double partition;
    double dfreq;
    double mean_mass;
    double pressure;
    double ref_temp;
} oracle_consts;

/* ------------------------------------------------------------------------ */
/* Humlicek (1982) W4 rational approximation of Re w(x + iy).               */
/* The four regions and their coefficients are Humlicek's published table;  */
/* both reference backends use it (profiles.cpp:9-42 for the CPU,           */
/* cross_kernal.cu:149-181 for the GPU).  Operation order follows the       */
/* reference so the CPU restatement is bit-identical under the same gcc.    */
/* ------------------------------------------------------------------------ */
double oracle_humlic(double x, double y) {
    double complex t = y - x * I;
    double s = fabs(x) + y;
    if (s >= 15) {
        double complex w = t * 0.5641896 / (0.5 + t * t);
        return creal(w);
    }
    if (s >= 5.5) {
        double complex u = t * t;
        double complex w = t * (1.410474 + u * .5641896) / (.75 + u * (3. + u));
        return creal(w);
    }
    if (y >= 0.195 * fabs(x) - 0.176) {
        double complex w = (16.4955 + t * (20.20933 + t * (11.96482 + t * (3.778987 + t * .5642236)))) /
                           (16.4955 + t * (38.82363 + t * (39.27121 + t * (21.69274 + t * (6.699398 + t)))));
        return creal(w);
    }
    {
        double complex u = t * t;
        double complex w =
            cexp(u) - t * (36183.31 - u * (3321.9905 - u * (1540.787 - u * (219.0313 - u * (35.76683 - u * (1.320522 - u * .56419)))))) /
                          (32066.6 - u * (24322.84 - u * (9022.228 - u * (2186.181 - u * (364.2191 - u * (61.57037 - u * (1.841439 - u)))))));
        return creal(w);
    }
}

/* ------------------------------------------------------------------------ */
/* Step one (per line), GPU convention.                                     */
/* ------------------------------------------------------------------------ */

/* GpuManager::InitializeConstants, GPUManager.cpp:28-39: cmcoef uses
 * pi = acos(-1.0) (the OpenMPManager uses the 11-digit PI instead). */
static double gpu_cmcoef(void) { return 1.0 / (8.0 * acos(-1.0) * 2.99792458e10); }
static double gpu_beta(double t) { return 6.6260693e-27 * 2.99792458e10 / (1.380658e-16 * t); }

/* device_compute_cross_section_voigt_stepone (with gamma),
 * cross_kernal.cu:758-790.  Writes S and gammaL. */
void oracle_gpu_voigt_stepone(const oracle_consts* c, long n, const double* e, const double* nu,
                              const double* aif, const int* gns, const double* gamma,
                              const double* nexp, double* s_out, double* gl_out) {
    double cm = gpu_cmcoef(), beta = gpu_beta(c->temperature);
    for (long i = 0; i < n; ++i) {
        double ei = e[i], g = (double)gns[i], nu_if = nu[i], a = aif[i];
        if (nu_if == 0) nu_if = 1e-6;
        double s = cm * a * g * O_ISQRTPI * exp(-beta * ei) * (1.0 - exp(-beta * nu_if)) /
                   (nu_if * nu_if * c->partition);
        if (g == -1) s = a;
        s_out[i] = s;
        gl_out[i] = gamma[i] * pow(c->ref_temp / c->temperature, nexp[i]);
    }
}

/* device_compute_cross_section_doppler_stepone, cross_kernal.cu:629-653
 * (the GAUSSIAN step one, :471-495, is the same formula). */
void oracle_gpu_doppler_stepone(const oracle_consts* c, long n, const double* e, const double* nu,
                                const double* aif, const int* gns, double* s_out) {
    double cm = gpu_cmcoef(), beta = gpu_beta(c->temperature);
    for (long i = 0; i < n; ++i) {
        double ei = e[i], g = (double)gns[i], nu_if = nu[i], a = aif[i];
        double s = cm * a * g * exp(-beta * ei) * (1.0 - exp(-beta * nu_if)) /
                   (nu_if * nu_if * c->partition);
        if (nu_if == 0) s = 0.0;
        s_out[i] = s;
    }
}

static int is_sorted_nu(long n, const double* nu) {
    for (long i = 1; i < n; ++i)
        if (nu[i] < nu[i - 1]) return 0;
    return 1;
}

/* First index i in [0, n) with nu[i] >= v (nu ascending). */
static long lower_bound_d(const double* nu, long n, double v) {
    long lo = 0, hi = n;
    while (lo < hi) {
        long mid = lo + (hi - lo) / 2;
        if (nu[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

/* Step two of the GPU convention: CTA per grid point (blockIdx = b),
 * `nthr` threads each striding the lines from threadIdx, `continue` while
 * dnu < -cut, `break` once dnu > cut (dnu = nu - f), then a serial sum of
 * the per-thread partials by thread 0 and g_cs[start+b] += sum
 * (cross_kernal.cu:924-997 Voigt, :654-723 Doppler).
 * For ascending nu the lines a thread evaluates are exactly its stride
 * members inside [-cut, cut]; the loop below visits those directly.
 * kind: 2 Voigt, 1 Doppler. */
/* Window half width override for the GPU convention (cut > 0), as the
 * engine's xs_condition.cut; <= 0 restores the reference rule. */
static double g_cut_override = -1.0;
void oracle_set_cut(double cut) { g_cut_override = cut; }

static void gpu_steptwo(int kind, const oracle_consts* c, const double* freq, double* intens,
                        int points, int start_idx, long n, const double* nu, const double* s,
                        const double* gl, int nthr) {
    double dpw = sqrt(2.0 * O_BOLTZ * c->temperature * O_NA / (c->mean_mass)) / O_VELLGT;
    double cut = (kind == 2) ? fmin(25.0 * c->pressure, 100.0) : O_DOPPLER_CUTOFF;
    if (g_cut_override > 0.0) cut = g_cut_override;
    double x0d = c->dfreq * 0.5;
    int sorted = is_sorted_nu(n, nu);
    double* part = (double*)malloc(sizeof(double) * (size_t)nthr);
    for (int b = 0; b < points; ++b) {
        double f = freq[start_idx + b];
        for (int t = 0; t < nthr; ++t) part[t] = 0.0;
        long i0 = 0, i1 = n;
        if (sorted) {
            /* Lines with nu - f < -cut are skipped by `continue`; the first
             * line with nu - f > cut ends each thread's loop. */
            i0 = lower_bound_d(nu, n, f - cut - 1.0);
            while (i0 > 0 && !(nu[i0 - 1] - f < -cut)) --i0;
            while (i0 < n && nu[i0] - f < -cut) ++i0;
            i1 = i0;
            while (i1 < n && !(nu[i1] - f > cut)) ++i1;
        }
        for (int t = 0; t < nthr; ++t) {
            long first = i0 + ((t - i0 % nthr) % nthr + nthr) % nthr;
            for (long i = first; i < i1; i += nthr) {
                double d = nu[i] - f;
                if (d < -cut) continue;
                if (d > cut) break;
                double g = 1.0 / (nu[i] * dpw);
                if (kind == 2) {
                    double x = fabs(d) * g, y = gl[i] * g;
                    part[t] += s[i] * oracle_humlic(x, y) * g;
                } else {
                    double xp = g * ((d) + x0d), xm = g * ((d) - x0d);
                    part[t] += s[i] * (erf(xp) - erf(xm));
                }
            }
        }
        double sum = 0.0;
        for (int t = 0; t < nthr; ++t) sum += part[t];
        intens[start_idx + b] += sum;
    }
    free(part);
}

/* Reference GpuManager VOIGT path on one chunk: step one (in place in the
 * reference; into scratch here) then step two.  intens is accumulated. */
void oracle_gpu_voigt(const oracle_consts* c, const double* freq, double* intens, int points,
                      int start_idx, long n, const double* e, const double* nu, const double* aif,
                      const int* gns, const double* gamma, const double* nexp) {
    double* s = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    double* gl = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    oracle_gpu_voigt_stepone(c, n, e, nu, aif, gns, gamma, nexp, s, gl);
    gpu_steptwo(2, c, freq, intens, points, start_idx, n, nu, s, gl, O_VOIGT_BLOCK);
    free(s);
    free(gl);
}

/* Reference GpuManager DOPPLER path on one chunk (cross_kernal.cu:240-253). */
void oracle_gpu_doppler(const oracle_consts* c, const double* freq, double* intens, int points,
                        int start_idx, long n, const double* e, const double* nu, const double* aif,
                        const int* gns) {
    double* s = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    oracle_gpu_doppler_stepone(c, n, e, nu, aif, gns, s);
    gpu_steptwo(1, c, freq, intens, points, start_idx, n, nu, s, NULL, O_BLOCK_SIZE);
    free(s);
}

/* GAUSSIAN, INTENDED formula (parity unpinned).  The reference kernel
 * device_compute_cross_section_steptwo_block (cross_kernal.cu:567-625)
 * computes x_ = sqrt(ln2)/halfwidth from cross_constants.ln2, which
 * GpuManager never sets (GPUManager.cpp:38 is commented out), and with
 * dnu = f - nu it `break`s on the first line below f - 10*HW, i.e. at once
 * for ascending input.  Restated here with ln2 = LN2 (defines.h:4) and the
 * symmetric window |f - nu| <= 10*HW. */
void oracle_gpu_gaussian(const oracle_consts* c, const double* freq, double* intens, int points,
                         int start_idx, long n, const double* e, const double* nu,
                         const double* aif, const int* gns) {
    double* s = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    oracle_gpu_doppler_stepone(c, n, e, nu, aif, gns, s);
    double* part = (double*)malloc(sizeof(double) * O_BLOCK_SIZE);
    double cut = c->half_width * 10.0;
    double xg = sqrt(O_LN2) / c->half_width;
    double x0g = xg * c->dfreq * 0.5;
    for (int b = 0; b < points; ++b) {
        double f = freq[start_idx + b];
        for (int t = 0; t < O_BLOCK_SIZE; ++t) part[t] = 0.0;
        for (long i = 0; i < n; ++i) {
            double d = f - nu[i];
            if (d < -cut || d > cut) continue;
            double xp = xg * (d) + x0g, xm = xg * (d) - x0g;
            part[i % O_BLOCK_SIZE] += s[i] * (erf(xp) - erf(xm));
        }
        double sum = 0.0;
        for (int t = 0; t < O_BLOCK_SIZE; ++t) sum += part[t];
        intens[start_idx + b] += sum;
    }
    free(part);
    free(s);
}

/* ------------------------------------------------------------------------ */
/* CPU convention: OpenMPManager.                                           */
/* ------------------------------------------------------------------------ */

/* OpenMPManager::ComputeVoigt (OpenMPManager.cpp:183-224) and
 * ComputeDoppler (:138-181) for all `nthreads` workers, then
 * TransferResults (:118-131).
 *
 *  - Lines are split in blocks of ceil(float(N)/float(threads)) (a float
 *    division: for N > 2^24 the last lines can fall outside every block).
 *  - Each worker adds into a private copy of the initial grid (TransferFreq,
 *    :82-88), in line order.
 *  - The Doppler width carries sqrt(LN2) (:146,191), unlike the GPU kernels.
 *  - The window is [round((nu-cut-f0)/df), round((nu+cut-f0)/df)) clamped
 *    to [start_idx, start_idx+points) (:160-161, :205-206), f0 = freq[0].
 *  - nu == 0 becomes 1e-6 everywhere; lines with S == 0 are skipped.
 *  - The result is 0 + grid_0 + grid_1 + ... over the whole grid (g_intens
 *    is a fresh, zeroed allocation in a new process).
 * kind: 2 Voigt, 1 Doppler.  intens: initial grid in, result out. */
static void cpu_compute(int kind, const oracle_consts* c, int nthreads, int npoints_total,
                        const double* freq, double* intens, int points, int start_idx, long n,
                        const double* e, const double* nu, const double* aif, const int* gns,
                        const double* gamma, const double* nexp) {
    double m_cmcoef = 1.0 / (8.0 * O_PI * O_VELLGT);
    double m_beta = O_PLANCK * O_VELLGT / (O_BOLTZ * c->temperature);
    double dpwcoef = sqrt(2.0 * O_LN2 * O_BOLTZ * c->temperature * O_NA / (c->mean_mass)) / O_VELLGT;
    double lorentz_cutoff = fmin(25.0 * c->pressure, 100.0);
    double x0 = c->dfreq * 0.5;
    double start_nu = freq[0];
    int nener = (int)n;
    int for_block = (int)ceilf((float)nener / (float)nthreads);
    double* total = (double*)calloc((size_t)npoints_total, sizeof(double));
    double* grid = (double*)malloc(sizeof(double) * (size_t)npoints_total);
    for (int id = 0; id < nthreads; ++id) {
        memcpy(grid, intens, sizeof(double) * (size_t)npoints_total);
        int start = id * for_block;
        int end = id * for_block + for_block < nener ? id * for_block + for_block : nener;
        for (int i = start; i < end; ++i) {
            double nu_if = nu[i];
            if (nu_if == 0) nu_if = 1e-6;
            if (kind == 2) {
                double abscoef = m_cmcoef * aif[i] * gns[i] * O_ISQRTPI * exp(-m_beta * e[i]) *
                                 (1.0 - exp(-m_beta * nu_if)) / (nu_if * nu_if * c->partition);
                double gammaL = gamma[i] * pow(c->ref_temp / c->temperature, nexp[i]);
                double rb = round((nu_if - lorentz_cutoff - start_nu) / c->dfreq);
                double re = round((nu_if + lorentz_cutoff - start_nu) / c->dfreq);
                int ib = (int)(rb > (double)start_idx ? rb : (double)start_idx);
                int ie = (int)(re < (double)(points + start_idx) ? re : (double)(points + start_idx));
                if (abscoef == 0.0) continue;
                for (int j = ib; j < ie; ++j) {
                    double gammaG = 1.0 / (nu_if * dpwcoef);
                    double dfreq_ = nu_if - freq[j];
                    double x = fabs(dfreq_) * gammaG;
                    double y = gammaL * gammaG;
                    grid[j] += abscoef * oracle_humlic(x, y) * gammaG;
                }
            } else {
                double abscoef = m_cmcoef * aif[i] * gns[i] * exp(-m_beta * e[i]) *
                                 (1.0 - exp(-m_beta * nu_if)) / (nu_if * nu_if * c->partition);
                double rb = round((nu_if - O_DOPPLER_CUTOFF - start_nu) / c->dfreq);
                double re = round((nu_if + O_DOPPLER_CUTOFF - start_nu) / c->dfreq);
                int ib = (int)(rb > (double)start_idx ? rb : (double)start_idx);
                int ie = (int)(re < (double)(points + start_idx) ? re : (double)(points + start_idx));
                if (abscoef == 0.0) continue;
                for (int j = ib; j < ie; ++j) {
                    double gammaG = 1.0 / (nu_if * dpwcoef);
                    double dfreq_ = fabs(nu_if - freq[j]);
                    double xp = gammaG * ((dfreq_) + x0);
                    double xm = gammaG * ((dfreq_) - x0);
                    grid[j] += abscoef * (erf(xp) - erf(xm));
                }
            }
        }
        for (int j = 0; j < npoints_total; ++j) total[j] += grid[j];
    }
    memcpy(intens, total, sizeof(double) * (size_t)npoints_total);
    free(grid);
    free(total);
}

void oracle_cpu_voigt(const oracle_consts* c, int nthreads, int npoints_total, const double* freq,
                      double* intens, int points, int start_idx, long n, const double* e,
                      const double* nu, const double* aif, const int* gns, const double* gamma,
                      const double* nexp) {
    cpu_compute(2, c, nthreads, npoints_total, freq, intens, points, start_idx, n, e, nu, aif, gns,
                gamma, nexp);
}

void oracle_cpu_doppler(const oracle_consts* c, int nthreads, int npoints_total, const double* freq,
                        double* intens, int points, int start_idx, long n, const double* e,
                        const double* nu, const double* aif, const int* gns) {
    cpu_compute(1, c, nthreads, npoints_total, freq, intens, points, start_idx, n, e, nu, aif, gns,
                NULL, NULL);
}
