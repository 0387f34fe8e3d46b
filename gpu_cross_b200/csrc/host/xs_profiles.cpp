// BaseProfile, VoigtProfile, DopplerProfile: the reference's driver loop
// (BaseProfile.cpp, VoigtProfile.cpp, DopplerProfile.cpp).  Lines are read
// from the transition files, kept when inside [nu_start - cut, nu_end + cut],
// and handed to the manager in chunks; each chunk is evaluated over the grid
// points its lines can reach.
//
// Differences from the reference: host line arrays grow with the chunk
// instead of being allocated at GetNtrans() lines up front; a missing
// BROADENERS block means default broadening (the reference indexes an empty
// vector); DopplerProfile sets its profile to DOPPLER (the reference leaves
// it unset, DopplerProfile.cpp:4-33); progress messages go to stderr so that
// stdout holds only the spectrum.
#include <algorithm>
#include <cmath>
#include <cstdint>

#include "xsec/xsec.h"

// BaseProfile.cpp:3-24: f_j = start + j * (end - start) / Npoints.
BaseProfile::BaseProfile(Input* pInput) : input(pInput) {
    start_nu = input->GetNuStart();
    end_nu = input->GetNuEnd();
    Npoints = input->GetNpoints();
    dfreq = (end_nu - start_nu) / double(Npoints);
    freq.resize(size_t(Npoints));
    intens.assign(size_t(Npoints), 0.0);
    for (int i = 0; i < Npoints; ++i) freq[size_t(i)] = start_nu + double(i) * dfreq;
}

BaseProfile::~BaseProfile() {
    delete manager;
    delete state_reader;
}

void BaseProfile::SetBackend(const std::string& backend, int precision) {
    if (backend != "hybrid" && backend != "gpu" && backend != "openmp" && backend != "multigpu")
        throw xs_error(XS_ERR_INVALID, "unknown backend " + backend);
    if (precision != XS_FP64 && precision != XS_MIXED)
        throw xs_error(XS_ERR_INVALID, "precision must be XS_FP64 or XS_MIXED");
    backend_ = backend;
    precision_ = precision;
}

BaseManager* BaseProfile::MakeManager(ProfileType p) {
    BaseManager* m = nullptr;
    if (backend_ == "gpu")
        m = new GpuManager(p, 0);
    else if (backend_ == "openmp")
        m = new OpenMPManager(p, input->GetNumThreads(), input->GetMemory());
    else if (backend_ == "multigpu")
        m = new MultiGpuManager(p);
    else
        m = new HybridManager(p, input->GetNumThreads(), input->GetMemory());
    if (precision_ != XS_FP64) {
        try {
            m->SetPrecision(precision_);
        } catch (...) {
            delete m;
            throw;
        }
    }
    return m;
}

void BaseProfile::Initialize() {
    InitializeProfile();
    transition_files = input->GetTransFiles();
}

// BaseProfile.cpp:49-62: upload the chunk, evaluate it over the grid points
// [round((min_nu - HW - f0)/df), round((max_nu + HW - f0)/df)) clamped.
void BaseProfile::PerformCrossSection(double HW) {
    manager->TransferVectors(size_t(Ntrans), h_energies.data(), h_nu.data(), h_aif.data(),
                             h_gns.data(), h_gammaL.empty() ? nullptr : h_gammaL.data(),
                             h_n.empty() ? nullptr : h_n.data());
    ib = int(std::max(std::round((min_nu - HW - start_nu) / dfreq), 0.0));
    ie = int(std::min(std::round((max_nu + HW - start_nu) / dfreq), double(Npoints)));
    points = ie - ib;
    if (points > 0) manager->ExecuteCrossSection(points, Ntrans, ib);
    lines_used_ += size_t(Ntrans);
    ++chunks_;
    std::fprintf(stderr, "chunk %d: %d lines, points [%d, %d)\n", chunks_, Ntrans, ib, ie);
}

// BaseProfile.cpp:65-71.
void BaseProfile::OutputProfile(FILE* out) {
    std::fill(intens.begin(), intens.end(), 0.0);
    manager->TransferResults(freq.data(), intens.data(), Npoints);
    for (int i = 0; i < Npoints; ++i) std::fprintf(out, "%12.6f %13.8E\n", freq[size_t(i)], intens[size_t(i)]);
}

void BaseProfile::OutputProfileBinary(FILE* out) {
    std::fill(intens.begin(), intens.end(), 0.0);
    manager->TransferResults(freq.data(), intens.data(), Npoints);
    const char magic[8] = {'X', 'S', 'E', 'C', 'B', 'I', 'N', '1'};
    const int64_t n = Npoints;
    bool ok = std::fwrite(magic, 1, 8, out) == 8 && std::fwrite(&n, sizeof(n), 1, out) == 1;
    if (ok && n > 0)
        ok = std::fwrite(freq.data(), sizeof(double), size_t(n), out) == size_t(n) &&
             std::fwrite(intens.data(), sizeof(double), size_t(n), out) == size_t(n);
    if (!ok) throw xs_error(XS_ERR_INVALID, "OutputProfileBinary: write failed");
}

// ---------------------------------------------------------------------------
namespace {

void reserve_chunk(std::vector<double>& v, int n) { v.reserve(size_t(std::min(n, 1 << 22))); }

}  // namespace

// VoigtProfile.cpp:4-36.  HITRAN gamma is referred to 296 K, ExoMol to 500 K.
void VoigtProfile::InitializeProfile() {
    profile = VOIGT;
    double ref_temp = 296.0;
    if (input->GetFileType() == HITRAN_TYPE) {
        const auto files = input->GetTransFiles();
        if (files.empty()) throw xs_error(XS_ERR_INVALID, "HITRAN input without TRANS-FILES");
        state_reader = new HITRANStateReader(files[0], input->GetPartition(), input->GetPressure(),
                                             input->GetTemperature(), input->GetHitranMixture());
    } else {
        const auto broad = input->GetBroadeners();
        state_reader = new ExomolStateReader(input->GetStateFile(), input->GetPartition(),
                                             input->GetPressure(), broad.empty() ? "" : broad[0],
                                             input->GetGammaAir(), input->GetNAir());
        ref_temp = 500.0;
    }
    manager = MakeManager(profile);
    manager->InitializeVectors(Npoints);
    manager->TransferFreq(freq.data(), intens.data(), Npoints);
    num_trans_fit = int(std::min<size_t>(manager->GetNtrans(), size_t(INT32_MAX)));
    if (num_trans_fit < 1) throw xs_error(XS_ERR_NOMEM, "no room for transitions");
    manager->InitializeConstants(input->GetHalfWidth(), input->GetTemperature(),
                                 state_reader->ComputePartition(input->GetTemperature()), dfreq,
                                 input->GetMeanMass(), input->GetPressure(), ref_temp);
}

// VoigtProfile.cpp:38-119: cut = min(25 P, 100); a chunk closes when it
// holds GetNtrans() lines or would span more than MAX-POINTS grid points.
void VoigtProfile::ExecuteCrossSection() {
    Ntrans = 0;
    lines_used_ = 0;
    chunks_ = 0;
    double t_nu = 0, t_ei = 0, t_aif = 0, t_gns = 0, t_gammaL = 0, t_n = 0;
    max_nu = 0.0;
    min_nu = 99999.0;
    const double gammaHW = std::min(25.0 * input->GetPressure(), 100.0);
    const int max_points = int(input->GetMaxPoints());
    for (auto* v : {&h_energies, &h_nu, &h_aif, &h_gammaL, &h_n}) {
        v->clear();
        reserve_chunk(*v, num_trans_fit);
    }
    h_gns.clear();
    auto flush = [&]() {
        PerformCrossSection(gammaHW);
        max_nu = 0.0;
        min_nu = 99999.0;
        Ntrans = 0;
        for (auto* v : {&h_energies, &h_nu, &h_aif, &h_gammaL, &h_n}) v->clear();
        h_gns.clear();
    };
    for (const auto& file : transition_files) {
        state_reader->OpenFile(file);
        while (state_reader->ReadNextState(t_nu, t_gns, t_ei, t_aif, t_gammaL, t_n)) {
            if (t_nu < start_nu - gammaHW) continue;
            if (t_nu > end_nu + gammaHW) break;
            h_energies.push_back(t_ei);
            h_nu.push_back(t_nu);
            h_gns.push_back(int(t_gns));
            h_aif.push_back(t_aif);
            h_gammaL.push_back(t_gammaL);
            h_n.push_back(t_n);
            min_nu = std::min(min_nu, t_nu);
            max_nu = std::max(max_nu, t_nu);
            const int tib = int(std::max(std::round((min_nu - gammaHW - start_nu) / dfreq), 0.0));
            const int tie = int(std::min(std::round((max_nu + gammaHW - start_nu) / dfreq), double(Npoints)));
            ++Ntrans;
            if (Ntrans >= num_trans_fit || tie - tib > max_points) flush();
        }
        state_reader->CloseFile();
    }
    if (Ntrans > 0) flush();
}

// DopplerProfile.cpp:6-33.
void DopplerProfile::InitializeProfile() {
    profile = DOPPLER;
    if (input->GetFileType() == HITRAN_TYPE) {
        const auto files = input->GetTransFiles();
        if (files.empty()) throw xs_error(XS_ERR_INVALID, "HITRAN input without TRANS-FILES");
        state_reader = new HITRANStateReader(files[0], input->GetPartition(), input->GetPressure(),
                                             input->GetTemperature(), input->GetHitranMixture());
    } else {
        state_reader = new ExomolStateReader(input->GetStateFile(), input->GetPartition(),
                                             input->GetPressure());
    }
    manager = MakeManager(profile);
    manager->InitializeVectors(Npoints);
    manager->TransferFreq(freq.data(), intens.data(), Npoints);
    num_trans_fit = int(std::min<size_t>(manager->GetNtrans(), size_t(INT32_MAX)));
    if (num_trans_fit < 1) throw xs_error(XS_ERR_NOMEM, "no room for transitions");
    manager->InitializeConstants(input->GetHalfWidth(), input->GetTemperature(),
                                 state_reader->ComputePartition(input->GetTemperature()), dfreq,
                                 input->GetMeanMass(), input->GetPressure(), 296.0);
}

// DopplerProfile.cpp:35-101: cut 100 cm-1; chunks of GetNtrans() lines.
void DopplerProfile::ExecuteCrossSection() {
    const double dopplerHW = 100.0;
    Ntrans = 0;
    lines_used_ = 0;
    chunks_ = 0;
    double t_nu = 0, t_ei = 0, t_aif = 0, t_gns = 0;
    max_nu = 0.0;
    min_nu = 99999.0;
    for (auto* v : {&h_energies, &h_nu, &h_aif}) {
        v->clear();
        reserve_chunk(*v, num_trans_fit);
    }
    h_gns.clear();
    h_gammaL.clear();
    h_n.clear();
    auto flush = [&]() {
        PerformCrossSection(dopplerHW);
        max_nu = 0.0;
        min_nu = 99999.0;
        Ntrans = 0;
        for (auto* v : {&h_energies, &h_nu, &h_aif}) v->clear();
        h_gns.clear();
    };
    for (const auto& file : transition_files) {
        state_reader->OpenFile(file);
        while (state_reader->ReadNextState(t_nu, t_gns, t_ei, t_aif)) {
            if (t_nu < start_nu - dopplerHW) continue;
            if (t_nu > end_nu + dopplerHW) break;
            h_energies.push_back(t_ei);
            h_nu.push_back(t_nu);
            h_gns.push_back(int(t_gns));
            h_aif.push_back(t_aif);
            min_nu = std::min(min_nu, t_nu);
            max_nu = std::max(max_nu, t_nu);
            ++Ntrans;
            if (Ntrans >= num_trans_fit) flush();
        }
        state_reader->CloseFile();
    }
    if (Ntrans > 0) flush();
}
