// Manager level of the C ABI: the reference's BaseManager interface
// (BaseManager.h:22-30) over host buffers.  Two kinds, both computed on the
// B200 by the engine:
//   kind 0  GpuManager semantics and arithmetic (GPUManager.cpp, reference
//           GPU convention);
//   kind 1  OpenMPManager semantics and arithmetic (OpenMPManager.cpp,
//           reference CPU convention: sqrt(ln2) Doppler width, rounded index
//           windows, thread-block line coverage) -- on the GPU, not the CPU.
// The C++ classes of include/xsec/ are thin wrappers over these calls.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <string>
#include <vector>

#include "xs_engine.h"
#include "xsec_b200.h"

namespace {

int mfail(int code, const std::string& msg) { return xs::set_error(code, msg.c_str()); }

#define XM_CU(call)                                                                       \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            cudaGetLastError();                                                           \
            return mfail(e_ == cudaErrorMemoryAllocation ? XS_ERR_NOMEM : XS_ERR_CUDA,    \
                         std::string(#call) + ": " + cudaGetErrorString(e_));             \
        }                                                                                 \
    } while (0)

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DevGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// GetNtrans of the GPU kind: lines that fit in free device memory next to the
// engine's scratch, capped so the host-side chunk arrays a caller sizes from
// it (VoigtProfile.cpp:30-36) stay moderate.
constexpr size_t kGpuNtransCap = size_t(1) << 26;

}  // namespace

struct xs_manager {
    int kind = 0;
    int profile = XS_VOIGT;
    int gpu_id = 0;
    int num_threads = 1;
    size_t total_memory = 0;
    int precision = XS_FP64;
    xs_engine* eng = nullptr;

    double* d_freq = nullptr;
    double* d_intens = nullptr;
    int npoints = 0;
    std::vector<double> init_intens;

    double *d_nu = nullptr, *d_e = nullptr, *d_aif = nullptr, *d_gamma = nullptr, *d_n = nullptr;
    int* d_gns = nullptr;
    size_t cap = 0, nlines = 0;
    bool have_gamma = false;

    bool have_consts = false;
    double half_width = 0, temperature = 0, partition = 0, dfreq = 0, mean_mass = 0,
           pressure = 0, ref_temp = 296.0;
    size_t ntrans = 0;

    void free_lines() {
        cudaFree(d_nu);
        cudaFree(d_e);
        cudaFree(d_aif);
        cudaFree(d_gamma);
        cudaFree(d_n);
        cudaFree(d_gns);
        d_nu = d_e = d_aif = d_gamma = d_n = nullptr;
        d_gns = nullptr;
        cap = nlines = 0;
    }
};

extern "C" {

int xs_manager_create(int kind, int profile, int gpu_id, int num_threads, size_t total_memory,
                      xs_manager** out) {
    if (!out) return mfail(XS_ERR_INVALID, "xs_manager_create: out is NULL");
    *out = nullptr;
    if (kind != 0 && kind != 1) return mfail(XS_ERR_INVALID, "manager kind must be 0 (GPU) or 1 (OpenMP)");
    if (profile == XS_PSUEDO_VOIGT || (kind == 1 && profile == XS_GAUSSIAN))
        return mfail(XS_ERR_UNSUPPORTED, "Profile not implemented (as in the reference)");
    if (profile != XS_VOIGT && profile != XS_DOPPLER && profile != XS_GAUSSIAN)
        return mfail(XS_ERR_INVALID, "unknown profile");
    if (kind == 1 && num_threads < 1) return mfail(XS_ERR_INVALID, "num_threads < 1");
    auto* m = new xs_manager();
    m->kind = kind;
    m->profile = profile;
    m->gpu_id = gpu_id;
    m->num_threads = num_threads < 1 ? 1 : num_threads;
    m->total_memory = total_memory;
    int rc = xs_engine_create(gpu_id, &m->eng);
    if (rc) {
        delete m;
        return rc;
    }
    *out = m;
    return XS_OK;
}

int xs_manager_cleanup(xs_manager* m) {
    if (!m) return mfail(XS_ERR_INVALID, "NULL manager");
    DevGuard g(m->gpu_id);
    cudaDeviceSynchronize();
    cudaFree(m->d_freq);
    cudaFree(m->d_intens);
    m->d_freq = m->d_intens = nullptr;
    m->npoints = 0;
    m->free_lines();
    return XS_OK;
}

int xs_manager_destroy(xs_manager* m) {
    if (!m) return XS_OK;
    xs_manager_cleanup(m);
    xs_engine_destroy(m->eng);
    delete m;
    return XS_OK;
}

int xs_manager_set_precision(xs_manager* m, int precision) {
    if (!m) return mfail(XS_ERR_INVALID, "NULL manager");
    if (precision != XS_FP64 && precision != XS_MIXED) return mfail(XS_ERR_INVALID, "precision");
    m->precision = precision;
    return XS_OK;
}

int xs_manager_initialize_vectors(xs_manager* m, int Npoints) {
    if (!m || Npoints < 1) return mfail(XS_ERR_INVALID, "InitializeVectors: bad arguments");
    DevGuard g(m->gpu_id);
    cudaFree(m->d_freq);
    cudaFree(m->d_intens);
    m->d_freq = m->d_intens = nullptr;
    XM_CU(cudaMalloc(&m->d_freq, sizeof(double) * size_t(Npoints)));
    XM_CU(cudaMalloc(&m->d_intens, sizeof(double) * size_t(Npoints)));
    XM_CU(cudaMemset(m->d_intens, 0, sizeof(double) * size_t(Npoints)));
    m->npoints = Npoints;
    // bytes per line: nu, E, A, gns (+ gamma, n for Voigt), GPUManager.cpp:55-58
    // and OpenMPManager.cpp:32-35
    const size_t raw = (m->profile == XS_VOIGT) ? 44 : 28;
    if (m->kind == 1) {
        // OpenMPManager::InitializeVectors (OpenMPManager.cpp:9, 19-35): half
        // of total_memory, minus the grids, divided by the bytes per line.
        const size_t budget = m->total_memory / 2;
        const size_t grids = size_t(Npoints) * sizeof(double) * size_t(2 + m->num_threads);
        m->ntrans = budget > grids ? (budget - grids) / raw : 0;
    } else {
        size_t free_b = 0, total_b = 0;
        XM_CU(cudaMemGetInfo(&free_b, &total_b));
        xs_options o{};
        o.profile = m->profile;
        o.precision = XS_FP64;
        const size_t per = raw + xs_scratch_bytes_needed(&o, 1, 1024) / 1024;
        const size_t reserve = size_t(1) << 30;
        const size_t avail = free_b > reserve ? free_b - reserve : 0;
        m->ntrans = std::min(avail / per, kGpuNtransCap);
    }
    return XS_OK;
}

int xs_manager_initialize_constants(xs_manager* m, double half_width, double temperature,
                                    double partition, double dfreq, double meanmass,
                                    double pressure, double ref_temp) {
    if (!m) return mfail(XS_ERR_INVALID, "NULL manager");
    m->half_width = half_width;
    m->temperature = temperature;
    m->partition = partition;
    m->dfreq = dfreq;
    m->mean_mass = meanmass;
    m->pressure = pressure;
    m->ref_temp = ref_temp;
    m->have_consts = true;
    return XS_OK;
}

int xs_manager_transfer_freq(xs_manager* m, const double* h_freq, const double* h_intens, int N) {
    if (!m || !h_freq || !h_intens || N < 1) return mfail(XS_ERR_INVALID, "TransferFreq: bad arguments");
    if (N > m->npoints) return mfail(XS_ERR_STATE, "TransferFreq: N exceeds InitializeVectors(Npoints)");
    DevGuard g(m->gpu_id);
    XM_CU(cudaMemcpy(m->d_freq, h_freq, sizeof(double) * size_t(N), cudaMemcpyHostToDevice));
    XM_CU(cudaMemcpy(m->d_intens, h_intens, sizeof(double) * size_t(N), cudaMemcpyHostToDevice));
    if (m->kind == 1) m->init_intens.assign(h_intens, h_intens + N);
    return XS_OK;
}

int xs_manager_transfer_vectors(xs_manager* m, size_t Nener, const double* h_energies,
                                const double* h_nu, const double* h_aif, const int* h_gns,
                                const double* h_gamma, const double* h_n) {
    if (!m) return mfail(XS_ERR_INVALID, "NULL manager");
    if (Nener > 0 && (!h_energies || !h_nu || !h_aif || !h_gns))
        return mfail(XS_ERR_INVALID, "TransferVectors: NULL line array");
    if (m->ntrans && Nener > m->ntrans)
        return mfail(XS_ERR_INVALID, "TransferVectors: more lines than GetNtrans()");
    DevGuard g(m->gpu_id);
    // Like the reference, wait for the previous chunk before reusing buffers
    // (GPUManager.cpp:89, OpenMPManager.cpp:70).
    int rc = xs_engine_sync(m->eng);
    if (rc) return rc;
    const bool with_gamma = h_gamma && h_n;
    if (Nener > m->cap || (with_gamma && !m->d_gamma)) {
        m->free_lines();
        const size_t c = std::max<size_t>(Nener, 1);
        XM_CU(cudaMalloc(&m->d_nu, c * sizeof(double)));
        XM_CU(cudaMalloc(&m->d_e, c * sizeof(double)));
        XM_CU(cudaMalloc(&m->d_aif, c * sizeof(double)));
        XM_CU(cudaMalloc(&m->d_gns, c * sizeof(int)));
        if (with_gamma || m->profile == XS_VOIGT) {
            XM_CU(cudaMalloc(&m->d_gamma, c * sizeof(double)));
            XM_CU(cudaMalloc(&m->d_n, c * sizeof(double)));
        }
        m->cap = c;
    }
    // The reference needs ascending nu (its kernels `break` on the first
    // line past the window); sort a copy when the caller's chunk is not.
    bool sorted = true;
    for (size_t i = 1; i < Nener && sorted; ++i) sorted = !(h_nu[i] < h_nu[i - 1]);
    std::vector<size_t> order;
    std::vector<double> tmp_d;
    std::vector<int> tmp_i;
    auto put_d = [&](double* dst, const double* src) -> cudaError_t {
        if (sorted) return cudaMemcpy(dst, src, Nener * sizeof(double), cudaMemcpyHostToDevice);
        tmp_d.resize(Nener);
        for (size_t i = 0; i < Nener; ++i) tmp_d[i] = src[order[i]];
        return cudaMemcpy(dst, tmp_d.data(), Nener * sizeof(double), cudaMemcpyHostToDevice);
    };
    if (!sorted) {
        order.resize(Nener);
        std::iota(order.begin(), order.end(), size_t(0));
        std::stable_sort(order.begin(), order.end(),
                         [&](size_t a, size_t b) { return h_nu[a] < h_nu[b]; });
    }
    if (Nener > 0) {
        XM_CU(put_d(m->d_nu, h_nu));
        XM_CU(put_d(m->d_e, h_energies));
        XM_CU(put_d(m->d_aif, h_aif));
        if (sorted) {
            XM_CU(cudaMemcpy(m->d_gns, h_gns, Nener * sizeof(int), cudaMemcpyHostToDevice));
        } else {
            tmp_i.resize(Nener);
            for (size_t i = 0; i < Nener; ++i) tmp_i[i] = h_gns[order[i]];
            XM_CU(cudaMemcpy(m->d_gns, tmp_i.data(), Nener * sizeof(int), cudaMemcpyHostToDevice));
        }
        if (with_gamma) {
            XM_CU(put_d(m->d_gamma, h_gamma));
            XM_CU(put_d(m->d_n, h_n));
        }
    }
    m->nlines = Nener;
    m->have_gamma = with_gamma;
    return XS_OK;
}

int xs_manager_execute_cross_section(xs_manager* m, int N, int N_ener, int start_idx) {
    if (!m) return mfail(XS_ERR_INVALID, "NULL manager");
    if (!m->have_consts) return mfail(XS_ERR_STATE, "ExecuteCrossSection before InitializeConstants");
    if (!m->d_freq) return mfail(XS_ERR_STATE, "ExecuteCrossSection before InitializeVectors");
    if (N_ener < 0 || size_t(N_ener) > m->nlines)
        return mfail(XS_ERR_INVALID, "ExecuteCrossSection: N_ener exceeds the uploaded lines");
    if (N < 0 || start_idx < 0 || long(start_idx) + long(N) > long(m->npoints))
        return mfail(XS_ERR_INVALID, "ExecuteCrossSection: chunk outside the grid");
    if (m->profile == XS_VOIGT && N_ener > 0 && !m->have_gamma)
        return mfail(XS_ERR_STATE, "VOIGT needs gamma and n in TransferVectors");
    xs_options o{};
    o.profile = m->profile;
    o.convention = m->kind == 1 ? XS_CONV_CPU : XS_CONV_GPU;
    o.precision = m->precision;
    o.cpu_threads = m->num_threads;
    o.mean_mass = m->mean_mass;
    o.ref_temp = m->ref_temp;
    o.half_width = m->half_width;
    o.dfreq = m->dfreq;
    xs_condition c{};
    c.temperature = m->temperature;
    c.partition = m->partition;
    c.pressure = m->pressure;
    c.gamma_scale = 1.0;
    c.cut = -1.0;
    xs_lines L{m->d_nu, m->d_e, m->d_aif, m->d_gns, m->d_gamma, m->d_n, size_t(N_ener)};
    xs_grid G{m->d_freq, m->npoints, start_idx, N};
    return xs_engine_execute(m->eng, &o, &c, 1, &L, &G, m->d_intens, 0);
}

int xs_manager_transfer_results(xs_manager* m, double* h_freq, double* h_intens, int N) {
    if (!m || !h_intens || N < 1 || N > m->npoints)
        return mfail(XS_ERR_INVALID, "TransferResults: bad arguments");
    DevGuard g(m->gpu_id);
    int rc = xs_engine_sync(m->eng);
    if (rc) return rc;
    XM_CU(cudaMemcpy(h_intens, m->d_intens, sizeof(double) * size_t(N), cudaMemcpyDeviceToHost));
    if (m->kind == 0) {
        // GpuManager copies the grid back too (GPUManager.cpp:163).
        if (h_freq)
            XM_CU(cudaMemcpy(h_freq, m->d_freq, sizeof(double) * size_t(N), cudaMemcpyDeviceToHost));
    } else if (m->num_threads > 1 && !m->init_intens.empty()) {
        // OpenMPManager sums one private copy of the initial grid per thread
        // (OpenMPManager.cpp:84-86, 123-127): the initial values count
        // num_threads times.
        const double k = double(m->num_threads - 1);
        const size_t nn = std::min(size_t(N), m->init_intens.size());
        for (size_t j = 0; j < nn; ++j) h_intens[j] += k * m->init_intens[j];
    }
    return XS_OK;
}

int xs_manager_ready_for_work(xs_manager* m, int* ready) {
    if (!m || !ready) return mfail(XS_ERR_INVALID, "NULL argument");
    DevGuard g(m->gpu_id);
    const cudaError_t q = cudaStreamQuery(nullptr);
    if (q != cudaSuccess && q != cudaErrorNotReady) {
        cudaGetLastError();
        return mfail(XS_ERR_CUDA, cudaGetErrorString(q));
    }
    *ready = (q == cudaSuccess) ? 1 : 0;
    return XS_OK;
}

int xs_manager_get_ntrans(xs_manager* m, size_t* ntrans) {
    if (!m || !ntrans) return mfail(XS_ERR_INVALID, "NULL argument");
    *ntrans = m->ntrans;
    return XS_OK;
}

}  // extern "C"
