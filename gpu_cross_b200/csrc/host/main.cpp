// xsec_cross: the reference's main (main.cpp:17-44) on the B200 engine.
//
//   xsec_cross [--input FILE] [--output FILE] [--format text|binary]
//              [--backend hybrid|gpu|openmp|multigpu] [--precision fp64|mixed]
//              [--settings] [--list-lines]
//
// Reads the .inp keyword file (stdin by default), computes the cross-section
// and prints "%12.6f %13.8E" per grid point, like the reference; with
// --format binary it writes BaseProfile::OutputProfileBinary's layout
// instead ("XSECBIN1", int64 N, N FP64 wavenumbers, N FP64 values).  Progress
// goes to stderr.  --settings prints the parsed input and --list-lines the
// lines the readers return (nu, gns, E'', A, gamma, n), both without a GPU.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>
#include <string>

#include "xsec/xsec.h"

namespace {

int usage() {
    std::fprintf(stderr,
                 "usage: xsec_cross [--input FILE] [--output FILE] [--format text|binary] "
                 "[--backend hybrid|gpu|openmp|multigpu] [--precision fp64|mixed] "
                 "[--settings] [--list-lines]\n");
    return 2;
}

void print_settings(Input& in) {
    const char* prof[] = {"GAUSSIAN", "DOPPLER", "VOIGT", "PSUEDO_VOIGT"};
    std::printf("file-type %s\n", in.GetFileType() == HITRAN_TYPE ? "HITRAN" : "EXOMOL");
    std::printf("profile %s\n", prof[int(in.profile)]);
    std::printf("temperature %.17g\npressure %.17g\npartition %.17g\n", in.GetTemperature(),
                in.GetPressure(), in.GetPartition());
    std::printf("mean-mass %.17g\nhalf-width %.17g\nhitran-mixture-air %.17g\n", in.GetMeanMass(),
                in.GetHalfWidth(), in.GetHitranMixture());
    std::printf("gamma-air %.17g\nn-air %.17g\n", in.GetGammaAir(), in.GetNAir());
    std::printf("nu-range %.17g %.17g\nn-points %d\nmax-points %d\n", in.GetNuStart(),
                in.GetNuEnd(), in.GetNpoints(), int(in.GetMaxPoints()));
    std::printf("num-threads %d\nmemory %zu\n", in.GetNumThreads(), in.GetMemory());
    std::printf("state-file %s\n", in.GetStateFile().c_str());
    for (const auto& f : in.GetTransFiles()) std::printf("trans-file %s\n", f.c_str());
    for (const auto& f : in.GetBroadeners()) std::printf("broadener %s\n", f.c_str());
}

// The readers exactly as the profiles drive them (same reader, same
// arguments), without the window filter.
void list_lines(Input& in) {
    std::unique_ptr<StateReader> r;
    const bool voigt = in.profile == VOIGT;
    const auto files = in.GetTransFiles();
    if (in.GetFileType() == HITRAN_TYPE) {
        if (files.empty()) throw xs_error(XS_ERR_INVALID, "HITRAN input without TRANS-FILES");
        r.reset(new HITRANStateReader(files[0], in.GetPartition(), in.GetPressure(),
                                      in.GetTemperature(), in.GetHitranMixture()));
    } else {
        const auto b = in.GetBroadeners();
        r.reset(new ExomolStateReader(in.GetStateFile(), in.GetPartition(), in.GetPressure(),
                                      voigt && !b.empty() ? b[0] : "", in.GetGammaAir(),
                                      in.GetNAir()));
    }
    try {
        std::printf("partition %.17g\n", r->ComputePartition(in.GetTemperature()));
    } catch (const xs_error& e) {
        std::printf("partition unavailable (%s)\n", e.what());
    }
    double nu, gns, e, a, g = 0.0, n = 0.0;
    for (const auto& f : files) {
        r->OpenFile(f);
        while (voigt ? r->ReadNextState(nu, gns, e, a, g, n) : r->ReadNextState(nu, gns, e, a))
            std::printf("%.17g %d %.17g %.17g %.17g %.17g\n", nu, int(gns), e, a, g, n);
        r->CloseFile();
    }
}

}  // namespace

int main(int argc, char** argv) {
    std::string input_path, output_path, backend = "hybrid";
    int precision = XS_FP64;
    bool settings = false, lines = false, binary = false;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&]() -> std::string {
            if (i + 1 >= argc) throw xs_error(XS_ERR_INVALID, a + " needs a value");
            return argv[++i];
        };
        try {
            if (a == "--input")
                input_path = next();
            else if (a == "--output")
                output_path = next();
            else if (a == "--backend")
                backend = next();
            else if (a == "--format") {
                const std::string f = next();
                if (f == "binary")
                    binary = true;
                else if (f != "text")
                    return usage();
            }
            else if (a == "--precision") {
                const std::string p = next();
                if (p == "fp64")
                    precision = XS_FP64;
                else if (p == "mixed")
                    precision = XS_MIXED;
                else
                    return usage();
            } else if (a == "--settings")
                settings = true;
            else if (a == "--list-lines")
                lines = true;
            else
                return usage();
        } catch (const xs_error&) {
            return usage();
        }
    }
    try {
        Input in;
        if (input_path.empty()) {
            in.ReadInputII();
        } else {
            std::ifstream f(input_path);
            if (!f) throw xs_error(XS_ERR_INVALID, "cannot open " + input_path);
            in.ReadInputII(f);
        }
        if (settings || lines) {
            if (settings) print_settings(in);
            if (lines) list_lines(in);
            return 0;
        }
        std::unique_ptr<BaseProfile> profile;
        if (in.profile == VOIGT)
            profile.reset(new VoigtProfile(&in));
        else if (in.profile == DOPPLER)
            profile.reset(new DopplerProfile(&in));
        else
            throw xs_error(XS_ERR_UNSUPPORTED, "Selected unimplemented profile");
        profile->SetBackend(backend, precision);
        profile->Initialize();
        profile->ExecuteCrossSection();
        FILE* out = stdout;
        if (!output_path.empty()) {
            out = std::fopen(output_path.c_str(), binary ? "wb" : "w");
            if (!out) throw xs_error(XS_ERR_INVALID, "cannot write " + output_path);
        }
        if (binary)
            profile->OutputProfileBinary(out);
        else
            profile->OutputProfile(out);
        if (out != stdout) std::fclose(out);
        std::fprintf(stderr, "%zu lines in %d chunks\n", profile->LinesUsed(), profile->Chunks());
        // the error statement of the result against the FP64 arithmetic
        std::fprintf(stderr,
                     "error bound (%s): every grid point and the band integral within %.3e "
                     "relative of the FP64 result\n",
                     precision == XS_MIXED && in.profile == VOIGT ? "mixed FP32/FP64" : "FP64",
                     xs_error_bound(int(in.profile), precision));
    } catch (const xs_error& e) {
        std::fprintf(stderr, "xsec_cross: %s\n", e.what());
        return 1;
    }
    return 0;
}
