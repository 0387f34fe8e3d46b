// The reference's BaseManager family on the manager level of the C ABI
// (xs_manager_*).  Every compute step runs on the B200; errors throw xs_error.
#include <algorithm>
#include <climits>
#include <thread>

#include "xsec/xsec.h"

BaseManager::~BaseManager() {}

bool BaseManager::ReadyForWork() { return true; }

size_t BaseManager::GetNtrans() { return N_trans; }

void BaseManager::SetPrecision(int precision) {
    if (precision != XS_FP64)
        throw xs_error(XS_ERR_UNSUPPORTED, "SetPrecision: this manager computes in FP64 only");
}

// ---------------------------------------------------------------------------
EngineManager::EngineManager(ProfileType p, int kind, int gpu_id, int num_threads,
                             size_t total_memory)
    : BaseManager(p) {
    xs_throw_if(xs_manager_create(kind, int(p), gpu_id, num_threads, total_memory, &m_),
                kind == 1 ? "OpenMPManager" : "GpuManager");
}

EngineManager::~EngineManager() { xs_manager_destroy(m_); }

void EngineManager::InitializeVectors(int Npoints) {
    xs_throw_if(xs_manager_initialize_vectors(m_, Npoints), "InitializeVectors");
    xs_throw_if(xs_manager_get_ntrans(m_, &N_trans), "GetNtrans");
}

void EngineManager::InitializeConstants(double half_width, double temperature, double partition,
                                        double dfreq, double meanmass, double pressure,
                                        double ref_temp) {
    xs_throw_if(xs_manager_initialize_constants(m_, half_width, temperature, partition, dfreq,
                                                meanmass, pressure, ref_temp),
                "InitializeConstants");
}

void EngineManager::TransferVectors(size_t Nener, double* h_energies, double* h_nu,
                                    double* h_aif, int* h_gns, double* h_gamma, double* h_n) {
    xs_throw_if(xs_manager_transfer_vectors(m_, Nener, h_energies, h_nu, h_aif, h_gns, h_gamma, h_n),
                "TransferVectors");
}

void EngineManager::TransferFreq(double* h_freq, double* h_intens, int N) {
    xs_throw_if(xs_manager_transfer_freq(m_, h_freq, h_intens, N), "TransferFreq");
}

void EngineManager::ExecuteCrossSection(int N, int N_ener, int start_idx) {
    xs_throw_if(xs_manager_execute_cross_section(m_, N, N_ener, start_idx), "ExecuteCrossSection");
}

void EngineManager::TransferResults(double* h_freq, double* h_intens, int N) {
    xs_throw_if(xs_manager_transfer_results(m_, h_freq, h_intens, N), "TransferResults");
}

void EngineManager::Cleanup() { xs_throw_if(xs_manager_cleanup(m_), "Cleanup"); }

bool EngineManager::ReadyForWork() {
    int ready = 0;
    xs_throw_if(xs_manager_ready_for_work(m_, &ready), "ReadyForWork");
    return ready != 0;
}

void EngineManager::SetPrecision(int precision) {
    xs_throw_if(xs_manager_set_precision(m_, precision), "SetPrecision");
}

GpuManager::GpuManager(ProfileType pProfile, int gpu_id)
    : EngineManager(pProfile, 0, gpu_id, 1, 0) {}

OpenMPManager::OpenMPManager(ProfileType pprofile, int num_threads, size_t total_memory)
    : EngineManager(pprofile, 1, 0, num_threads, total_memory) {}

// ---------------------------------------------------------------------------
// MultiGPUManager.cpp:5-16: one GpuManager per device (devices that are not
// sm_100 are skipped).
MultiGpuManager::MultiGpuManager(ProfileType pProfile) : BaseManager(pProfile) {
    int n = 0;
    xs_throw_if(xs_device_count(&n), "MultiGpuManager");
    for (int d = 0; d < n; ++d) {
        try {
            gpus_.push_back(new GpuManager(pProfile, d));
        } catch (const xs_error& e) {
            if (e.code() != XS_ERR_NODEVICE) {
                for (auto* g : gpus_) delete g;
                throw;
            }
        }
    }
    if (gpus_.empty()) throw xs_error(XS_ERR_NODEVICE, "MultiGpuManager: no sm_100 device");
    selected_ = gpus_[0];
}

MultiGpuManager::~MultiGpuManager() {
    for (auto* g : gpus_) delete g;
}

// MultiGPUManager.cpp:27-37: N_trans of the first device.
void MultiGpuManager::InitializeVectors(int Npoints) {
    for (auto* g : gpus_) g->InitializeVectors(Npoints);
    N_trans = gpus_[0]->GetNtrans();
}

void MultiGpuManager::InitializeConstants(double half_width, double temperature, double partition,
                                          double dfreq, double meanmass, double pressure,
                                          double ref_temp) {
    for (auto* g : gpus_)
        g->InitializeConstants(half_width, temperature, partition, dfreq, meanmass, pressure,
                               ref_temp);
}

// SwitchGPU (MultiGPUManager.cpp:91-103): scan from device 1 for an idle one.
void MultiGpuManager::TransferVectors(size_t Nener, double* h_energies, double* h_nu,
                                      double* h_aif, int* h_gns, double* h_gamma, double* h_n) {
    const int n = int(gpus_.size());
    for (int i = 1 % n;; i = (i + 1) % n) {
        if (gpus_[size_t(i)]->ReadyForWork()) {
            selected_ = gpus_[size_t(i)];
            break;
        }
        if (i == 0) std::this_thread::yield();
    }
    selected_->TransferVectors(Nener, h_energies, h_nu, h_aif, h_gns, h_gamma, h_n);
}

void MultiGpuManager::TransferFreq(double* h_freq, double* h_intens, int N) {
    for (auto* g : gpus_) g->TransferFreq(h_freq, h_intens, N);
}

void MultiGpuManager::ExecuteCrossSection(int N, int N_ener, int start_idx) {
    selected_->ExecuteCrossSection(N, N_ener, start_idx);
}

// MultiGPUManager.cpp:61-83: every device's grid is added into h_intens.
void MultiGpuManager::TransferResults(double* h_freq, double* h_intens, int N) {
    std::vector<double> f(size_t(std::max(N, 0))), v(size_t(std::max(N, 0)));
    for (auto* g : gpus_) {
        g->TransferResults(f.data(), v.data(), N);
        for (int j = 0; j < N; ++j) h_intens[j] += v[size_t(j)];
    }
    (void)h_freq;
}

void MultiGpuManager::Cleanup() {
    for (auto* g : gpus_) g->Cleanup();
}

bool MultiGpuManager::ReadyForWork() {
    bool any = false;
    for (auto* g : gpus_) any = g->ReadyForWork() || any;
    return any;
}

void MultiGpuManager::SetPrecision(int precision) {
    for (auto* g : gpus_) g->SetPrecision(precision);
}

// ---------------------------------------------------------------------------
HybridManager::HybridManager(ProfileType pProfile, int num_threads, size_t total_memory)
    : BaseManager(pProfile) {
    workers_.push_back(new OpenMPManager(pProfile, num_threads, total_memory));
    current_ = workers_[0];
}

HybridManager::~HybridManager() {
    for (auto* w : workers_) delete w;
}

// HybridManager.cpp:24-34: the smallest N_trans of the workers.
void HybridManager::InitializeVectors(int Npoints) {
    N_trans = size_t(INT_MAX);
    for (auto* w : workers_) w->InitializeVectors(Npoints);
    for (auto* w : workers_) N_trans = std::min(w->GetNtrans(), N_trans);
}

void HybridManager::InitializeConstants(double half_width, double temperature, double partition,
                                        double dfreq, double meanmass, double pressure,
                                        double ref_temp) {
    for (auto* w : workers_)
        w->InitializeConstants(half_width, temperature, partition, dfreq, meanmass, pressure,
                               ref_temp);
}

void HybridManager::TransferVectors(size_t Nener, double* h_energies, double* h_nu, double* h_aif,
                                    int* h_gns, double* h_gamma, double* h_n) {
    current_ = workers_[0];
    current_->TransferVectors(Nener, h_energies, h_nu, h_aif, h_gns, h_gamma, h_n);
}

void HybridManager::TransferFreq(double* h_freq, double* h_intens, int N) {
    for (auto* w : workers_) w->TransferFreq(h_freq, h_intens, N);
}

void HybridManager::ExecuteCrossSection(int N, int N_ener, int start_idx) {
    current_->ExecuteCrossSection(N, N_ener, start_idx);
}

// HybridManager.cpp:58-80: every worker's grid is added into h_intens.
void HybridManager::TransferResults(double* h_freq, double* h_intens, int N) {
    std::vector<double> f(size_t(std::max(N, 0))), v(size_t(std::max(N, 0)));
    for (auto* w : workers_) {
        std::fill(v.begin(), v.end(), 0.0);
        w->TransferResults(f.data(), v.data(), N);
        for (int j = 0; j < N; ++j) h_intens[j] += v[size_t(j)];
    }
    (void)h_freq;
}

void HybridManager::Cleanup() {
    for (auto* w : workers_) w->Cleanup();
}

bool HybridManager::ReadyForWork() { return workers_[0]->ReadyForWork(); }

void HybridManager::SetPrecision(int precision) {
    for (auto* w : workers_) w->SetPrecision(precision);
}
