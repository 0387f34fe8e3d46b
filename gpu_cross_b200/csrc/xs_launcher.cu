// Launcher level of the C ABI: drop-in replacements for the reference's host
// launchers (cross_kernal.cuh:18-52).  They keep the reference's calling
// convention -- per-device constants set once by copy_intensity_info, device
// pointers, asynchronous work on the legacy default stream, accumulation into
// g_intens[start_idx, start_idx + Npoints) -- and run the engine's kernels
// (reference GPU convention, FP64).
#include <cuda_runtime.h>

#include <mutex>

#include "xs_engine.h"
#include "xsec_b200.h"

namespace {

constexpr int kMaxDevices = 64;

struct DeviceState {
    bool have_consts = false;
    xs_cross_section_data consts{};
    xs_engine* engine = nullptr;
};

std::mutex g_mu;
DeviceState g_dev[kMaxDevices];

int current_device(int* dev) {
    if (cudaGetDevice(dev) != cudaSuccess || *dev < 0 || *dev >= kMaxDevices) {
        cudaGetLastError();
        return xs::set_error(XS_ERR_NODEVICE, "no current CUDA device");
    }
    return XS_OK;
}

int run_block(int profile, double* g_freq, double* g_intens, double* g_energies, double* g_nu,
              int* g_gns, double* g_aif, double* g_gamma, double* g_n, int Npoints, int N_ener,
              int start_idx) {
    int dev = 0;
    int rc = current_device(&dev);
    if (rc) return rc;
    if (Npoints < 0 || N_ener < 0 || start_idx < 0)
        return xs::set_error(XS_ERR_INVALID, "negative size");
    xs_engine* eng = nullptr;
    xs_cross_section_data c{};
    {
        std::lock_guard<std::mutex> lk(g_mu);
        DeviceState& s = g_dev[dev];
        if (!s.have_consts)
            return xs::set_error(XS_ERR_STATE, "xs_copy_intensity_info was not called on this device");
        if (!s.engine) {
            rc = xs_engine_create(dev, &s.engine);
            if (rc) return rc;
        }
        eng = s.engine;
        c = s.consts;
    }
    xs_options o{};
    o.profile = profile;
    o.convention = XS_CONV_GPU;
    o.precision = XS_FP64;
    o.mean_mass = c.mean_mass;
    o.ref_temp = c.ref_temp;
    o.half_width = c.halfwidth;
    o.dfreq = c.dfreq;
    xs_condition cond{};
    cond.temperature = c.temperature;
    cond.partition = c.partition;
    cond.pressure = c.pressure;
    cond.gamma_scale = 1.0;
    cond.cut = -1.0;
    xs_lines L{g_nu, g_energies, g_aif, g_gns, g_gamma, g_n, size_t(N_ener)};
    xs_grid G{g_freq, start_idx + Npoints, start_idx, Npoints};
    xs::ExecOverride ov;
    ov.use_consts = true;
    ov.cmcoef = c.cmcoef;
    ov.beta = c.beta;
    return xs::engine_execute(eng, &o, &cond, 1, &L, &G, g_intens, 0, &ov);
}

}  // namespace

extern "C" {

int xs_copy_intensity_info(const xs_cross_section_data* cross_inf) {
    if (!cross_inf) return xs::set_error(XS_ERR_INVALID, "NULL constants");
    int dev = 0;
    int rc = current_device(&dev);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(g_mu);
    g_dev[dev].consts = *cross_inf;
    g_dev[dev].have_consts = true;
    return XS_OK;
}

int xs_execute_two_step_kernal_voigt_block(double* g_freq, double* g_intens, double* g_energies,
                                           double* g_nu, int* g_gns, double* g_aif,
                                           double* g_gamma, double* g_n, int Npoints, int N_ener,
                                           int start_idx) {
    return run_block(XS_VOIGT, g_freq, g_intens, g_energies, g_nu, g_gns, g_aif, g_gamma, g_n,
                     Npoints, N_ener, start_idx);
}

int xs_execute_two_step_kernal_doppler_block(double* g_freq, double* g_intens,
                                             double* g_energies, double* g_nu, int* g_gns,
                                             double* g_aif, int Npoints, int N_ener,
                                             int start_idx) {
    return run_block(XS_DOPPLER, g_freq, g_intens, g_energies, g_nu, g_gns, g_aif, nullptr,
                     nullptr, Npoints, N_ener, start_idx);
}

int xs_execute_two_step_kernal_block(double* g_freq, double* g_intens, double* g_energies,
                                     double* g_nu, int* g_gns, double* g_aif, int Npoints,
                                     int N_ener, int start_idx) {
    return run_block(XS_GAUSSIAN, g_freq, g_intens, g_energies, g_nu, g_gns, g_aif, nullptr,
                     nullptr, Npoints, N_ener, start_idx);
}

int xs_launcher_sync(void) {
    int dev = 0;
    int rc = current_device(&dev);
    if (rc) return rc;
    xs_engine* eng = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        eng = g_dev[dev].engine;
    }
    if (!eng) {
        if (cudaDeviceSynchronize() != cudaSuccess)
            return xs::set_error(XS_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
        return XS_OK;
    }
    return xs_engine_sync(eng);
}

}  // extern "C"
