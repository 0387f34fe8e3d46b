// Line sources: ExoMol (.states + .trans[.bz2] + .broad) and HITRAN
// 160-character records, the reference's StateReader family
// (ExomolStateReader.cpp, HITRANStateReader.cpp, exomol_functions.cpp,
// bz2_compression/read_compress_trans.c).
//
// Differences from the reference, each a fix of undefined or unintended
// behaviour there:
//  * broadening keys are (code, J'', J') tuples; the reference concatenates
//    the numbers into one string, so ("a1", 1, 12) and ("a1", 11, 2) collide;
//  * the a0 fallback works (ExomolStateReader.cpp:21-22 appends to the a1 key
//    instead of replacing it, so a0 entries never match) and a transition
//    with neither entry gets the default gamma * pressure and n, where the
//    reference leaves the caller's previous (or uninitialised) values;
//  * transition records are read line by line, three numbers each; extra
//    columns are ignored and blank lines skipped;
//  * HITRANStateReader::OpenFile opens the file it is given (the reference
//    re-opens the constructor's file, HITRANStateReader.cpp:74);
//  * state ids out of range and unreadable files are errors.
// .bz2 transition files are decompressed through libbz2's public stream API,
// loaded at run time, including files made of several concatenated streams.
#include <dlfcn.h>

#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>

#include "xsec/xsec.h"

namespace {

// libbz2's public decompression interface (bzlib.h of bzip2 1.0).
struct BzStream {
    char* next_in;
    unsigned int avail_in;
    unsigned int total_in_lo32;
    unsigned int total_in_hi32;
    char* next_out;
    unsigned int avail_out;
    unsigned int total_out_lo32;
    unsigned int total_out_hi32;
    void* state;
    void* (*bzalloc)(void*, int, int);
    void (*bzfree)(void*, void*);
    void* opaque;
};
constexpr int kBzOk = 0;
constexpr int kBzStreamEnd = 4;

struct Bz2Api {
    int (*init)(BzStream*, int, int) = nullptr;
    int (*step)(BzStream*) = nullptr;
    int (*end)(BzStream*) = nullptr;
    bool ok = false;
};

const Bz2Api& bz2_api() {
    static Bz2Api api;
    static std::once_flag once;
    std::call_once(once, [] {
        const char* names[] = {"libbz2.so.1.0", "libbz2.so.1", "libbz2.so"};
        for (const char* n : names) {
            void* h = dlopen(n, RTLD_NOW | RTLD_LOCAL);
            if (!h) continue;
            api.init = reinterpret_cast<int (*)(BzStream*, int, int)>(dlsym(h, "BZ2_bzDecompressInit"));
            api.step = reinterpret_cast<int (*)(BzStream*)>(dlsym(h, "BZ2_bzDecompress"));
            api.end = reinterpret_cast<int (*)(BzStream*)>(dlsym(h, "BZ2_bzDecompressEnd"));
            api.ok = api.init && api.step && api.end;
            if (api.ok) break;
        }
    });
    return api;
}

struct Bz2State {
    BzStream s{};
    std::vector<char> in;
    bool active = false;
};

bool ends_with(const std::string& s, const std::string& suf) {
    return s.size() >= suf.size() && s.compare(s.size() - suf.size(), suf.size(), suf) == 0;
}

bool blank(const std::string& s) {
    return s.find_first_not_of(" \t\r\n\f\v") == std::string::npos;
}

// Physical constants of the readers (exomol_functions.cpp:49-53,
// HITRANStateReader.cpp:223-227).
constexpr double kPlanck = 6.6260693e-27;
constexpr double kVellgt = 2.99792458e10;
constexpr double kBoltz = 1.380658e-16;

}  // namespace

// ---------------------------------------------------------------------------
LineSource::~LineSource() { close(); }

bool LineSource::open(const std::string& path) {
    close();
    f_ = std::fopen(path.c_str(), "rb");
    if (!f_) return false;
    bz2_ = ends_with(path, ".bz2");
    if (bz2_) {
        const Bz2Api& api = bz2_api();
        if (!api.ok) {
            close();
            throw xs_error(XS_ERR_UNSUPPORTED, "libbz2 is not available to read " + path);
        }
        auto* st = new Bz2State();
        st->in.resize(1 << 20);
        bz_ = st;
    }
    buf_.clear();
    pos_ = 0;
    eof_ = false;
    return true;
}

void LineSource::close() {
    if (bz_) {
        auto* st = static_cast<Bz2State*>(bz_);
        if (st->active) bz2_api().end(&st->s);
        delete st;
        bz_ = nullptr;
    }
    if (f_) std::fclose(f_);
    f_ = nullptr;
    buf_.clear();
    pos_ = 0;
    eof_ = true;
}

// Appends the next block of (decompressed) text to buf_; false at the end.
bool LineSource::fill() {
    if (eof_ || !f_) return false;
    const size_t kChunk = 1 << 20;
    if (!bz2_) {
        const size_t old = buf_.size();
        buf_.resize(old + kChunk);
        const size_t got = std::fread(&buf_[old], 1, kChunk, f_);
        buf_.resize(old + got);
        if (got == 0) eof_ = true;
        return got > 0;
    }
    auto* st = static_cast<Bz2State*>(bz_);
    const Bz2Api& api = bz2_api();
    std::vector<char> out(kChunk);
    for (;;) {
        if (st->s.avail_in == 0) {
            const size_t got = std::fread(st->in.data(), 1, st->in.size(), f_);
            if (got == 0) {
                if (st->active) throw xs_error(XS_ERR_INVALID, "truncated bzip2 stream");
                eof_ = true;
                return false;
            }
            st->s.next_in = st->in.data();
            st->s.avail_in = unsigned(got);
        }
        if (!st->active) {
            // A new stream starts here (the file may hold several, one after
            // another, as the reference's reader expects).
            char* nin = st->s.next_in;
            const unsigned ain = st->s.avail_in;
            std::memset(&st->s, 0, sizeof(st->s));
            if (api.init(&st->s, 0, 0) != kBzOk) throw xs_error(XS_ERR_INVALID, "bzip2 init failed");
            st->s.next_in = nin;
            st->s.avail_in = ain;
            st->active = true;
        }
        st->s.next_out = out.data();
        st->s.avail_out = unsigned(out.size());
        const int rc = api.step(&st->s);
        const size_t produced = out.size() - st->s.avail_out;
        if (rc == kBzStreamEnd) {
            char* nin = st->s.next_in;
            const unsigned ain = st->s.avail_in;
            api.end(&st->s);
            st->active = false;
            st->s.next_in = nin;
            st->s.avail_in = ain;
        } else if (rc != kBzOk) {
            throw xs_error(XS_ERR_INVALID, "corrupt bzip2 data (code " + std::to_string(rc) + ")");
        }
        if (produced) {
            buf_.append(out.data(), produced);
            return true;
        }
    }
}

bool LineSource::next(std::string& line) {
    for (;;) {
        const size_t nl = buf_.find('\n', pos_);
        if (nl != std::string::npos) {
            line.assign(buf_, pos_, nl - pos_);
            pos_ = nl + 1;
            return true;
        }
        if (pos_ > 0) {
            buf_.erase(0, pos_);
            pos_ = 0;
        }
        if (!fill()) {
            if (buf_.empty()) return false;
            line.swap(buf_);
            buf_.clear();
            return true;
        }
    }
}

// ---------------------------------------------------------------------------
// initialize_states (exomol_functions.cpp:6-40): one state per line, "id E
// gns J ..."; the state with id k is the k-th line (ExoMol .states files
// are numbered 1..N in order, ExomolStateReader.cpp:156-160).
ExomolStateReader::ExomolStateReader(std::string pFilename, double partition, double pressure,
                                     std::string broadeners, double default_gamma,
                                     double default_n)
    : StateReader(pFilename, partition),
      m_pressure(pressure),
      default_gamma_(default_gamma),
      default_n_(default_n) {
    LineSource src;
    if (!src.open(pFilename)) throw xs_error(XS_ERR_INVALID, "cannot open state file " + pFilename);
    std::string line;
    while (src.next(line)) {
        if (blank(line)) continue;
        const char* p = line.c_str();
        char* q = nullptr;
        std::strtol(p, &q, 10);  // id: the line order is the index
        const double e = std::strtod(q, &q);
        const long g = std::strtol(q, &q, 10);
        const long J = std::strtol(q, &q, 10);
        energy_.push_back(e);
        gns_.push_back(int(g));
        J_.push_back(int(J));
    }
    if (broadeners.empty()) return;
    // InitializeBroadener (ExomolStateReader.cpp:39-80): "code gamma n J'' [J']".
    std::ifstream in(broadeners);
    if (!in) throw xs_error(XS_ERR_INVALID, "cannot open broadener file " + broadeners);
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::vector<std::string> t;
        std::string w;
        while (ls >> w) t.push_back(w);
        if (t.empty()) continue;
        const bool a1 = t[0] == "a1";
        if (t.size() < (a1 ? 5u : 4u))
            throw xs_error(XS_ERR_INVALID, "malformed broadener line: " + line);
        const int Ji = std::atoi(t[3].c_str());
        const int Jf = a1 ? std::atoi(t[4].c_str()) : -1;
        std::ostringstream key;
        key << (a1 ? "a1" : "a0") << ':' << Ji << ':' << Jf;
        broad_[key.str()] = {std::atof(t[1].c_str()), std::atof(t[2].c_str())};
    }
}

bool ExomolStateReader::OpenFile(std::string pFilename) {
    if (!src_.open(pFilename)) throw xs_error(XS_ERR_INVALID, "cannot open transition file " + pFilename);
    m_filename = pFilename;
    open_ = true;
    return true;
}

bool ExomolStateReader::CloseFile() {
    src_.close();
    open_ = false;
    return true;
}

// ExomolStateReader::ReadNextState (ExomolStateReader.cpp:130-167) and
// GetGammaN (:7-37).
bool ExomolStateReader::ReadNextState(double& nu, double& gns, double& e_i, double& aif,
                                      double& gam, double& n) {
    if (!open_) return false;
    std::string line;
    for (;;) {
        if (!src_.next(line)) return false;
        if (!blank(line)) break;
    }
    const char* p = line.c_str();
    char* q = nullptr;
    const long id_f = std::strtol(p, &q, 10) - 1;
    const long id_i = std::strtol(q, &q, 10) - 1;
    aif = std::strtod(q, &q);
    const long ns = long(energy_.size());
    if (id_f < 0 || id_f >= ns || id_i < 0 || id_i >= ns)
        throw xs_error(XS_ERR_INVALID, "transition refers to a state outside the state file: " + line);
    nu = energy_[id_f] - energy_[id_i];
    e_i = energy_[id_i];
    gns = gns_[id_f];
    const int Ji = J_[id_i], Jf = J_[id_f];
    std::ostringstream k1, k0;
    k1 << "a1:" << Ji << ':' << Jf;
    auto it = broad_.find(k1.str());
    if (it == broad_.end()) {
        k0 << "a0:" << Ji << ":-1";
        it = broad_.find(k0.str());
    }
    if (it != broad_.end()) {
        gam = it->second.first * m_pressure;
        n = it->second.second;
    } else {
        gam = default_gamma_ * m_pressure;
        n = default_n_;
    }
    return true;
}

bool ExomolStateReader::ReadNextState(double& nu, double& gns, double& e_i, double& aif) {
    double g = 0.0, n = 0.0;
    return ReadNextState(nu, gns, e_i, aif, g, n);
}

// compute_partition (exomol_functions.cpp:44-62): Q = sum gns exp(-beta E).
double ExomolStateReader::ComputePartition(double temperature) {
    if (partition < 0.0) {
        const double beta = kPlanck * kVellgt / (kBoltz * temperature);
        double q = 0.0;
        for (size_t i = 0; i < energy_.size(); ++i) q += gns_[i] * std::exp(-beta * energy_[i]);
        partition = q;
    }
    return partition;
}

// ---------------------------------------------------------------------------
namespace {

// HITRAN 160-character record, field widths of HITRANStateReader.cpp:4.
constexpr int kHitranWidths[] = {2, 1, 12, 10, 10, 5, 5, 10, 4, 8, 15, 15, 15, 15, 6, 12, 1, 7, 7};

std::string hitran_field(const std::string& rec, int field) {
    int start = 0;
    for (int i = 0; i < field; ++i) start += kHitranWidths[i];
    const int len = std::min(kHitranWidths[field], 12);  // GetField keeps 12 characters
    if (start >= int(rec.size())) return std::string();
    return rec.substr(size_t(start), size_t(len));
}

}  // namespace

HITRANStateReader::HITRANStateReader(std::string pFilename, double partition, double pressure,
                                     double temperature, double hitran_air_mixture,
                                     double ref_partition)
    : StateReader(pFilename, partition),
      m_pressure(pressure),
      m_mixture(hitran_air_mixture),
      m_temperature(temperature),
      ref_partition_(ref_partition) {
    // Q(T) at 296 K is the reference partition the A-from-S rebuild needs.
    if (ref_partition_ <= 0.0 && partition > 0.0 && temperature == 296.0) ref_partition_ = partition;
}

bool HITRANStateReader::OpenFile(std::string pFilename) {
    if (pFilename.empty()) return false;
    CloseFile();
    file_ = std::fopen(pFilename.c_str(), "r");
    if (!file_) throw xs_error(XS_ERR_INVALID, "cannot open HITRAN file " + pFilename);
    m_filename = pFilename;
    return true;
}

bool HITRANStateReader::CloseFile() {
    if (file_) std::fclose(file_);
    file_ = nullptr;
    return true;
}

// HITRANStateReader::ReadNextState (HITRANStateReader.cpp:137-250).
bool HITRANStateReader::ReadNextState(double& nu, double& gns, double& e_i, double& aif,
                                      double& gam, double& n) {
    if (!file_) return false;
    char buffer[1024];
    std::string rec;
    for (;;) {
        if (!std::fgets(buffer, sizeof(buffer), file_)) return false;
        rec = buffer;
        if (!blank(rec)) break;
    }
    nu = std::atof(hitran_field(rec, 2).c_str());
    const double intens = std::atof(hitran_field(rec, 3).c_str());
    aif = std::atof(hitran_field(rec, 4).c_str());
    const double gam_air = std::atof(hitran_field(rec, 5).c_str());
    const double self = std::atof(hitran_field(rec, 6).c_str());
    e_i = std::atof(hitran_field(rec, 7).c_str());
    n = std::atof(hitran_field(rec, 8).c_str());
    gns = std::atoi(hitran_field(rec, 17).c_str());
    gam = (gam_air * m_mixture + self * (1.0 - m_mixture)) * m_pressure;
    if (aif == 0.0) {
        // Old records carry only S(296 K): rebuild gns*A from it with Q(296).
        if (ref_partition_ <= 0.0)
            throw xs_error(XS_ERR_UNSUPPORTED,
                           "HITRAN record without an Einstein A needs Q(296 K); the TIPS "
                           "tables are not part of this build");
        const double pi = std::acos(-1.0);
        const double beta = kPlanck * kVellgt / (kBoltz * 296.0);
        aif = intens * 8.0 * pi * kVellgt * ref_partition_ * nu * nu /
              (std::exp(-beta * e_i) * (1.0 - std::exp(-beta * nu)));
        gns = 1.0;
    }
    return true;
}

bool HITRANStateReader::ReadNextState(double& nu, double& gns, double& e_i, double& aif) {
    double g = 0.0, n = 0.0;
    return ReadNextState(nu, gns, e_i, aif, g, n);
}

double HITRANStateReader::ComputePartition(double temperature) {
    (void)temperature;
    if (partition <= 0.0)
        throw xs_error(XS_ERR_UNSUPPORTED,
                       "HITRAN input needs PARTITION > 0 (the TIPS partition sums of "
                       "HITRANStateReader.cpp:62 are not part of this build)");
    return partition;
}
