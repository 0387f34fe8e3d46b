// Test infrastructure only: drives the UNMODIFIED reference GPU kernels
// (cross_kernal.cu, compiled from the reference tree by oracle/Makefile for
// sm_100a) through their own host launchers (cross_kernal.cuh:18-52).
// Nothing in the product links or loads this file.
//
// GpuManager (GPUManager.cpp) is not used: its InitializeVectors sizes the
// line buffers from all of device memory (GPUManager.cpp:12,55-58).  This
// harness allocates exactly the buffers one chunk needs, fills the constant
// block the way GpuManager::InitializeConstants does (GPUManager.cpp:24-47)
// and calls the same launcher GpuManager::ExecuteCrossSection would
// (GPUManager.cpp:107-121, 139-148).
#include "cross_kernal.cuh"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>

namespace {

// Constant block as GpuManager::InitializeConstants builds it
// (GPUManager.cpp:24-47).  `ln2` is left unset there; it is set to 0 here so
// the copy is at least deterministic.
void fill_constants(cross_section_data* c, double half_width, double temperature,
                    double partition, double dfreq, double mean_mass,
                    double pressure, double ref_temp) {
    const double planck = 6.6260693e-27;
    const double vellgt = 2.99792458e10;
    const double boltz = 1.380658e-16;
    const double pi = std::acos(-1.0);
    c->halfwidth = half_width;
    c->beta = planck * vellgt / (boltz * temperature);
    c->partition = partition;
    c->ref_temp = ref_temp;
    c->cmcoef = 1.0 / (8.0 * pi * vellgt);
    c->dfreq = dfreq;
    c->temperature = temperature;
    c->mean_mass = mean_mass;
    c->pressure = pressure;
    c->ln2 = 0.0;
}

#define RG_CHECK(call)                                        \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) {                              \
            fprintf(stderr, "ref_gpu_harness: %s: %s\n", #call, \
                    cudaGetErrorString(e_));                  \
            rc = 3;                                           \
            goto done;                                        \
        }                                                     \
    } while (0)

}  // namespace

extern "C" {

// Same arguments as ref_cpu_run.  `chunks` > 1 splits the line list into
// that many equal consecutive chunks, each executed over the grid slice its
// lines reach (the span rule of BaseProfile::PerformCrossSection,
// BaseProfile.cpp:55-57), the way BaseProfile feeds a manager.  `kernel_ms`
// (may be NULL) receives the summed device time of all launches.
int ref_gpu_run(int profile, int npoints_total, double* freq, double* intens,
                long n_lines, const double* energies, const double* nu,
                const double* aif, const int* gns, const double* gamma,
                const double* n, double half_width, double temperature,
                double partition, double dfreq, double mean_mass,
                double pressure, double ref_temp, int points, int start_idx,
                int chunks, float* kernel_ms) {
    int rc = 0;
    double *d_freq = nullptr, *d_intens = nullptr, *d_e = nullptr, *d_nu = nullptr,
           *d_aif = nullptr, *d_gamma = nullptr, *d_n = nullptr;
    int* d_gns = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float total_ms = 0.0f;
    size_t nb = size_t(n_lines) * sizeof(double);
    size_t nl = n_lines > 0 ? size_t(n_lines) : 1;
    cross_section_data c;
    fill_constants(&c, half_width, temperature, partition, dfreq, mean_mass,
                   pressure, ref_temp);
    if (chunks < 1) chunks = 1;

    RG_CHECK(cudaMalloc(&d_freq, sizeof(double) * size_t(npoints_total)));
    RG_CHECK(cudaMalloc(&d_intens, sizeof(double) * size_t(npoints_total)));
    RG_CHECK(cudaMalloc(&d_e, nl * sizeof(double)));
    RG_CHECK(cudaMalloc(&d_nu, nl * sizeof(double)));
    RG_CHECK(cudaMalloc(&d_aif, nl * sizeof(double)));
    RG_CHECK(cudaMalloc(&d_gns, nl * sizeof(int)));
    RG_CHECK(cudaMalloc(&d_gamma, nl * sizeof(double)));
    RG_CHECK(cudaMalloc(&d_n, nl * sizeof(double)));
    RG_CHECK(cudaMemcpy(d_freq, freq, sizeof(double) * size_t(npoints_total), cudaMemcpyHostToDevice));
    RG_CHECK(cudaMemcpy(d_intens, intens, sizeof(double) * size_t(npoints_total), cudaMemcpyHostToDevice));
    RG_CHECK(cudaMemcpy(d_e, energies, nb, cudaMemcpyHostToDevice));
    RG_CHECK(cudaMemcpy(d_nu, nu, nb, cudaMemcpyHostToDevice));
    RG_CHECK(cudaMemcpy(d_aif, aif, nb, cudaMemcpyHostToDevice));
    RG_CHECK(cudaMemcpy(d_gns, gns, size_t(n_lines) * sizeof(int), cudaMemcpyHostToDevice));
    if (gamma && n) {
        RG_CHECK(cudaMemcpy(d_gamma, gamma, nb, cudaMemcpyHostToDevice));
        RG_CHECK(cudaMemcpy(d_n, n, nb, cudaMemcpyHostToDevice));
    }
    copy_intensity_info(&c);
    RG_CHECK(cudaGetLastError());
    RG_CHECK(cudaEventCreate(&ev0));
    RG_CHECK(cudaEventCreate(&ev1));

    {
        long per = (n_lines + chunks - 1) / chunks;
        double cut = (profile == 2) ? std::fmin(25.0 * pressure, 100.0) : 100.0;
        for (int k = 0; k < chunks; ++k) {
            long a = long(k) * per;
            long b = a + per < n_lines ? a + per : n_lines;
            if (b <= a) break;
            int n_ener = int(b - a);
            int ib = start_idx, np = points;
            if (chunks > 1) {
                // BaseProfile.cpp:55-57 with HW = the profile's cut.
                double min_nu = nu[a], max_nu = nu[b - 1];
                ib = int(std::fmax(std::round((min_nu - cut - freq[0]) / dfreq), 0.0));
                int ie = int(std::fmin(std::round((max_nu + cut - freq[0]) / dfreq),
                                       double(npoints_total)));
                np = ie - ib;
                if (np <= 0) continue;
            }
            RG_CHECK(cudaEventRecord(ev0));
            if (profile == 2) {
                execute_two_step_kernal_voigt_block(d_freq, d_intens, d_e + a, d_nu + a, d_gns + a,
                                                    d_aif + a, d_gamma + a, d_n + a, np, n_ener, ib);
            } else if (profile == 1) {
                execute_two_step_kernal_doppler_block(d_freq, d_intens, d_e + a, d_nu + a, d_gns + a,
                                                      d_aif + a, np, n_ener, ib);
            } else {
                execute_two_step_kernal_block(d_freq, d_intens, d_e + a, d_nu + a, d_gns + a,
                                              d_aif + a, np, n_ener, ib);
            }
            RG_CHECK(cudaEventRecord(ev1));
            RG_CHECK(cudaEventSynchronize(ev1));
            RG_CHECK(cudaGetLastError());
            float ms = 0.0f;
            RG_CHECK(cudaEventElapsedTime(&ms, ev0, ev1));
            total_ms += ms;
        }
    }
    RG_CHECK(cudaMemcpy(intens, d_intens, sizeof(double) * size_t(npoints_total), cudaMemcpyDeviceToHost));
    if (kernel_ms) *kernel_ms = total_ms;

done:
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    cudaFree(d_freq);
    cudaFree(d_intens);
    cudaFree(d_e);
    cudaFree(d_nu);
    cudaFree(d_aif);
    cudaFree(d_gns);
    cudaFree(d_gamma);
    cudaFree(d_n);
    return rc;
}

}  // extern "C"
