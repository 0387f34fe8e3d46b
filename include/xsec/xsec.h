// C++ host layer of the B200 cross-section engine: the reference's classes
// (ahmed-f-alrefaie/gpu_cross) with their names and signatures, implemented
// on the C ABI of include/xsec_b200.h.  All compute runs on the GPU; there
// is no CPU path.
//
//   Input                .inp keyword file (Input.h:22-82, Input.cpp:98-182)
//   StateReader          line sources (StateReader.h:7-19)
//     ExomolStateReader  .states + .trans[.bz2] + .broad (ExomolStateReader.h)
//     HITRANStateReader  160-character HITRAN records (HITRANStateReader.h)
//   BaseManager          backend interface (BaseManager.h:6-33)
//     GpuManager         reference GPU arithmetic (GPUManager.h:12-43)
//     OpenMPManager      reference CPU arithmetic, computed on the GPU
//                        (OpenMPManager.h:13-50)
//     MultiGpuManager    one GpuManager per device (MultiGPUManager.h)
//     HybridManager      OpenMPManager arithmetic (HybridManager.h)
//   BaseProfile          grid, chunking, output (BaseProfile.h:14-46)
//     VoigtProfile, DopplerProfile
//
// Errors throw xs_error (the reference prints and calls exit(-1)); the CLI
// (csrc/host/main.cpp) turns them into that behaviour.
#pragma once

#include <cstddef>
#include <cstdio>
#include <istream>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "xsec_b200.h"

// Input.h:9-20 (same order and values as XS_GAUSSIAN..XS_PSUEDO_VOIGT).
enum ProfileType { GAUSSIAN = 0, DOPPLER = 1, VOIGT = 2, PSUEDO_VOIGT = 3 };
enum FileType { HITRAN_TYPE, EXOMOL_TYPE };

class xs_error : public std::runtime_error {
public:
    xs_error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

// Throws xs_error for a non-XS_OK status of the C ABI.
void xs_throw_if(int rc, const char* where);

// ---------------------------------------------------------------------------
class Input {
public:
    Input();
    ProfileType profile;
    // Input::ReadInputII (Input.cpp:98-182): first line HITRAN or EXOMOL, then
    // keywords; reads std::cin, or the given stream.
    void ReadInputII();
    void ReadInputII(std::istream& in);
    double GetHalfWidth() { return half_width; }
    double GetMeanMass() { return mean_mass; }
    double GetTemperature() { return temperature; }
    double GetNuStart() { return nu_start; }
    double GetNuEnd() { return nu_end; }
    double GetPartition() { return partition; }
    double GetPressure() { return pressure; }
    double GetHitranMixture() { return hitran_mixture_air; }
    double GetMaxPoints() { return max_points; }
    double GetGammaAir() { return gamma_air; }
    double GetNAir() { return n_air; }
    int GetNumThreads() { return num_threads; }
    size_t GetMemory() { return memory; }
    FileType GetFileType() { return which_file; }
    int GetNpoints() { return Npoints; }
    std::string GetStateFile() { return state_file; }
    std::vector<std::string> GetTransFiles() { return trans_files; }
    std::vector<std::string> GetBroadeners() { return broadener_files; }

private:
    double half_width, mean_mass, temperature, partition, pressure, nu_start, nu_end;
    int Npoints;
    double gamma_air, n_air, hitran_mixture_air;
    size_t memory;
    int num_threads, max_points;
    FileType which_file;
    std::vector<std::string> trans_files, broadener_files;
    std::string state_file;
};

// ---------------------------------------------------------------------------
class StateReader {
public:
    StateReader(std::string pFilename = "", double pPartition = -1.0)
        : m_filename(pFilename), partition(pPartition) {}
    virtual ~StateReader() {}
    virtual bool OpenFile(std::string pFilename) = 0;
    virtual bool CloseFile() = 0;
    virtual bool ReadNextState(double& nu, double& gns, double& e_i, double& aif, double& gam,
                               double& n) = 0;
    virtual bool ReadNextState(double& nu, double& gns, double& e_i, double& aif) = 0;
    virtual double ComputePartition(double temperature) = 0;

protected:
    std::string m_filename;
    double partition;
};

// Text lines from a plain or bzip2 (multi-stream) file.
class LineSource {
public:
    LineSource() = default;
    ~LineSource();
    bool open(const std::string& path);
    bool next(std::string& line);
    void close();

private:
    FILE* f_ = nullptr;
    void* bz_ = nullptr;
    bool bz2_ = false;
    std::string buf_;
    size_t pos_ = 0;
    bool eof_ = false;
    bool fill();
};

class ExomolStateReader : public StateReader {
public:
    // ExomolStateReader.cpp:61-69: states from pFilename; broadening from the
    // .broad file (keys a1 Ji Jf, then a0 Ji); gamma is multiplied by pressure.
    ExomolStateReader(std::string pFilename = "", double partition = -1.0, double pressure = 1.0,
                      std::string broadeners = "", double default_gamma = 0.05,
                      double default_n = 0.4);
    bool OpenFile(std::string pFilename) override;
    bool CloseFile() override;
    bool ReadNextState(double& nu, double& gns, double& e_i, double& aif, double& gam,
                       double& n) override;
    bool ReadNextState(double& nu, double& gns, double& e_i, double& aif) override;
    double ComputePartition(double temperature) override;
    size_t NumStates() const { return energy_.size(); }

private:
    std::vector<double> energy_;
    std::vector<int> gns_, J_;
    std::map<std::string, std::pair<double, double>> broad_;
    double m_pressure, default_gamma_, default_n_;
    LineSource src_;
    bool open_ = false;
};

class HITRANStateReader : public StateReader {
public:
    // HITRANStateReader.cpp:41-65.  Q(T) must be given (partition > 0): the
    // TIPS sums are not part of this build.  ref_partition: Q(296 K), only
    // needed to rebuild A from S for records with A == 0.
    HITRANStateReader(std::string pFilename = "", double partition = -1.0, double pressure = 1.0,
                      double temperature = 296.0, double hitran_air_mixture = 1.0,
                      double ref_partition = -1.0);
    bool OpenFile(std::string pFilename) override;
    bool CloseFile() override;
    bool ReadNextState(double& nu, double& gns, double& e_i, double& aif, double& gam,
                       double& n) override;
    bool ReadNextState(double& nu, double& gns, double& e_i, double& aif) override;
    double ComputePartition(double temperature) override;

private:
    FILE* file_ = nullptr;
    double m_pressure, m_mixture, m_temperature, ref_partition_;
};

// ---------------------------------------------------------------------------
class BaseManager {
public:
    virtual ~BaseManager();
    virtual void InitializeVectors(int Npoints) = 0;
    virtual void InitializeConstants(double half_width, double temperature, double partition,
                                     double dfreq, double meanmass, double pressure = 10.0,
                                     double ref_temp = 296.0) = 0;
    virtual void TransferVectors(size_t Nener, double* h_energies, double* h_nu, double* h_aif,
                                 int* h_gns, double* h_gamma = NULL, double* h_n = NULL) = 0;
    virtual void TransferFreq(double* h_freq, double* h_intens, int N) = 0;
    virtual void ExecuteCrossSection(int N, int N_ener, int start_idx) = 0;
    virtual void TransferResults(double* h_freq, double* h_intens, int N) = 0;
    virtual void Cleanup() = 0;
    virtual bool ReadyForWork();
    size_t GetNtrans();
    // Not in the reference: XS_FP64 (default) or XS_MIXED for the step-two
    // arithmetic of every later ExecuteCrossSection.  Not pure, so that a
    // BaseManager subclass written against the reference's BaseManager.h:6-33
    // still compiles: this default accepts XS_FP64 and throws xs_error for
    // anything else.
    virtual void SetPrecision(int precision);

protected:
    explicit BaseManager(ProfileType pprofile) : N_trans(0), profile(pprofile) {}
    size_t N_trans;
    ProfileType profile;
};

// The manager level of the C ABI behind the BaseManager virtuals.
class EngineManager : public BaseManager {
public:
    void InitializeVectors(int Npoints) override;
    void InitializeConstants(double half_width, double temperature, double partition,
                             double dfreq, double meanmass, double pressure = 10.0,
                             double ref_temp = 296.0) override;
    void TransferVectors(size_t Nener, double* h_energies, double* h_nu, double* h_aif,
                         int* h_gns, double* h_gamma = NULL, double* h_n = NULL) override;
    void TransferFreq(double* h_freq, double* h_intens, int N) override;
    void ExecuteCrossSection(int N, int N_ener, int start_idx) override;
    void TransferResults(double* h_freq, double* h_intens, int N) override;
    void Cleanup() override;
    bool ReadyForWork() override;
    void SetPrecision(int precision) override;
    ~EngineManager() override;

protected:
    EngineManager(ProfileType p, int kind, int gpu_id, int num_threads, size_t total_memory);
    xs_manager* m_ = nullptr;
};

// GPUManager.cpp: the reference GPU kernels' arithmetic on device gpu_id.
class GpuManager : public EngineManager {
public:
    GpuManager(ProfileType pProfile, int gpu_id = 0);
};

// OpenMPManager.cpp: the reference CPU backend's arithmetic (sqrt(ln2)
// Doppler width, rounded windows, lines covered in blocks of
// ceil(float(N)/float(num_threads))), computed on device 0.
class OpenMPManager : public EngineManager {
public:
    OpenMPManager(ProfileType pprofile, int num_threads, size_t total_memory);
};

// MultiGPUManager.cpp: one GpuManager per visible sm_100 device; each chunk
// goes to the first idle device scanning from device 1, and TransferResults
// adds every device's grid into h_intens.
class MultiGpuManager : public BaseManager {
public:
    explicit MultiGpuManager(ProfileType pProfile);
    ~MultiGpuManager() override;
    void InitializeVectors(int Npoints) override;
    void InitializeConstants(double half_width, double temperature, double partition,
                             double dfreq, double meanmass, double pressure = 10.0,
                             double ref_temp = 296.0) override;
    void TransferVectors(size_t Nener, double* h_energies, double* h_nu, double* h_aif,
                         int* h_gns, double* h_gamma = NULL, double* h_n = NULL) override;
    void TransferFreq(double* h_freq, double* h_intens, int N) override;
    void ExecuteCrossSection(int N, int N_ener, int start_idx) override;
    void TransferResults(double* h_freq, double* h_intens, int N) override;
    void Cleanup() override;
    bool ReadyForWork() override;
    void SetPrecision(int precision) override;
    int NumDevices() const { return int(gpus_.size()); }

private:
    std::vector<GpuManager*> gpus_;
    GpuManager* selected_ = nullptr;
};

// HybridManager.cpp: the reference hands each chunk to its first idle
// worker, worker 0 being OpenMPManager (the only one in a build without a
// GPU) and worker 1 MultiGpuManager, so which arithmetic a chunk gets
// depends on timing.  Here every chunk gets worker 0's, OpenMPManager's,
// arithmetic, computed on the B200: the output of the reference's
// deterministic (CPU-only) build.  TransferResults adds into h_intens.
class HybridManager : public BaseManager {
public:
    HybridManager(ProfileType pProfile, int num_threads, size_t total_memory);
    ~HybridManager() override;
    void InitializeVectors(int Npoints) override;
    void InitializeConstants(double half_width, double temperature, double partition,
                             double dfreq, double meanmass, double pressure = 10.0,
                             double ref_temp = 296.0) override;
    void TransferVectors(size_t Nener, double* h_energies, double* h_nu, double* h_aif,
                         int* h_gns, double* h_gamma = NULL, double* h_n = NULL) override;
    void TransferFreq(double* h_freq, double* h_intens, int N) override;
    void ExecuteCrossSection(int N, int N_ener, int start_idx) override;
    void TransferResults(double* h_freq, double* h_intens, int N) override;
    void Cleanup() override;
    bool ReadyForWork() override;
    void SetPrecision(int precision) override;

private:
    std::vector<BaseManager*> workers_;
    BaseManager* current_ = nullptr;
};

// ---------------------------------------------------------------------------
class BaseProfile {
public:
    virtual ~BaseProfile();
    void Initialize();
    virtual void ExecuteCrossSection() = 0;
    // Writes "%12.6f %13.8E" per grid point (BaseProfile.cpp:65-71).
    void OutputProfile(FILE* out = stdout);
    // Not in the reference: the same grid and cross-section in binary, with
    // every bit of the FP64 values (the text keeps nine digits).  Layout,
    // little-endian: the 8 bytes "XSECBIN1", int64 N, double freq[N],
    // double sigma[N].
    void OutputProfileBinary(FILE* out);
    const std::vector<double>& Frequencies() const { return freq; }
    const std::vector<double>& Intensities() const { return intens; }
    // Not in the reference: the manager Initialize() makes, "hybrid" (the
    // reference's HybridManager, default), "gpu", "openmp" or "multigpu",
    // and its precision, XS_FP64 (default) or XS_MIXED.  Call before
    // Initialize().
    void SetBackend(const std::string& backend, int precision = XS_FP64);
    // Lines of the last ExecuteCrossSection and the chunks they went in.
    size_t LinesUsed() const { return lines_used_; }
    int Chunks() const { return chunks_; }

protected:
    explicit BaseProfile(Input* pInput);
    virtual void PerformCrossSection(double HW);
    virtual void InitializeProfile() = 0;
    BaseManager* MakeManager(ProfileType p);

    BaseManager* manager = nullptr;
    StateReader* state_reader = nullptr;
    Input* input;
    ProfileType profile = VOIGT;
    std::vector<double> freq, intens;
    double dfreq;
    int ib = 0, ie = 0;
    std::vector<double> h_energies, h_nu, h_aif, h_gammaL, h_n;
    std::vector<int> h_gns;
    int Npoints;
    int num_trans_fit = 0;
    int Ntrans = 0;
    int points = 0;
    double start_nu, end_nu, min_nu = 0.0, max_nu = 0.0;
    std::vector<std::string> transition_files;
    std::string backend_ = "hybrid";
    int precision_ = XS_FP64;
    size_t lines_used_ = 0;
    int chunks_ = 0;
};

class VoigtProfile : public BaseProfile {
public:
    explicit VoigtProfile(Input* pInput) : BaseProfile(pInput) {}
    void ExecuteCrossSection() override;

protected:
    void InitializeProfile() override;
};

class DopplerProfile : public BaseProfile {
public:
    explicit DopplerProfile(Input* pInput) : BaseProfile(pInput) {}
    void ExecuteCrossSection() override;

protected:
    void InitializeProfile() override;
};
