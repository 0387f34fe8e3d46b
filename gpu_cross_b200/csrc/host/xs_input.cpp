// Input: the reference's .inp keyword reader (Input.cpp:98-182).
//
// First line HITRAN or EXOMOL; then one keyword per line, the value(s)
// after it separated by whitespace.  TRANS-FILES and BROADENERS take the
// following lines up to END.  Unknown keywords are ignored, as in the
// reference.  A keyword without its value is an error here (the reference
// reads past the end of its token vector).
#include <cstdlib>
#include <iostream>
#include <sstream>

#include "xsec/xsec.h"

namespace {

std::string trimmed(const std::string& s) {
    const char* ws = " \t\r\n\f\v";
    const size_t b = s.find_first_not_of(ws);
    if (b == std::string::npos) return std::string();
    const size_t e = s.find_last_not_of(ws);
    return s.substr(b, e - b + 1);
}

std::vector<std::string> tokens(const std::string& s) {
    std::istringstream in(s);
    std::vector<std::string> out;
    std::string t;
    while (in >> t) out.push_back(t);
    return out;
}

// Input::StringToProfile (Input.cpp:85-96): anything else is PSUEDO_VOIGT.
ProfileType profile_from(const std::string& s) {
    if (s == "GAUSSIAN") return GAUSSIAN;
    if (s == "DOPPLER") return DOPPLER;
    if (s == "VOIGT") return VOIGT;
    return PSUEDO_VOIGT;
}

}  // namespace

void xs_throw_if(int rc, const char* where) {
    if (rc == XS_OK) return;
    throw xs_error(rc, std::string(where) + ": " + xs_last_error());
}

// Defaults of Input::Input (Input.cpp:2-15); ReadInputII then sets partition
// -1, one thread and 1 GB (Input.cpp:112-114).
Input::Input()
    : profile(VOIGT),
      half_width(0.1),
      mean_mass(10.0),
      temperature(296.0),
      partition(1000.0),
      pressure(1.0),
      nu_start(0.0),
      nu_end(100.0),
      Npoints(1000),
      gamma_air(0.05),
      n_air(0.4),
      hitran_mixture_air(1.0),
      memory(1000000000ul),
      num_threads(1),
      max_points(80000),
      which_file(EXOMOL_TYPE) {}

void Input::ReadInputII() { ReadInputII(std::cin); }

void Input::ReadInputII(std::istream& in) {
    std::string line;
    if (!std::getline(in, line)) throw xs_error(XS_ERR_INVALID, "Input: empty input");
    const std::string kind = trimmed(line);
    if (kind == "HITRAN")
        which_file = HITRAN_TYPE;
    else if (kind == "EXOMOL")
        which_file = EXOMOL_TYPE;
    else
        throw xs_error(XS_ERR_INVALID, "Input: file type " + kind + " not supported");

    partition = -1.0;
    num_threads = 1;
    memory = 1000000000ul;
    auto value = [](const std::vector<std::string>& t, size_t i) -> const char* {
        if (t.size() <= i) throw xs_error(XS_ERR_INVALID, "Input: " + t[0] + " needs a value");
        return t[i].c_str();
    };
    auto block = [&](std::vector<std::string>& dst) {
        while (std::getline(in, line)) {
            const std::string t = trimmed(line);
            if (t == "END") break;
            dst.push_back(t);
        }
    };
    while (std::getline(in, line)) {
        const std::vector<std::string> t = tokens(line);
        if (t.empty()) continue;
        const std::string& key = t[0];
        if (key == "PRESSURE")
            pressure = std::atof(value(t, 1));
        else if (key == "TEMPERATURE")
            temperature = std::atof(value(t, 1));
        else if (key == "MEAN-MASS")
            mean_mass = std::atof(value(t, 1));
        else if (key == "HITRAN-MIXTURE-AIR")
            hitran_mixture_air = std::atof(value(t, 1));
        else if (key == "PARTITION")
            partition = std::atof(value(t, 1));
        else if (key == "HALF-WIDTH")
            half_width = std::atof(value(t, 1));
        else if (key == "GAMMA-AIR")
            gamma_air = std::atof(value(t, 1));
        else if (key == "N-AIR")
            n_air = std::atof(value(t, 1));
        else if (key == "MAX-POINTS")
            max_points = std::atoi(value(t, 1));
        else if (key == "STATE-FILE")
            state_file = value(t, 1);
        else if (key == "TRANS-FILES")
            block(trans_files);
        else if (key == "BROADENERS")
            block(broadener_files);
        else if (key == "PROFILE")
            profile = profile_from(value(t, 1));
        else if (key == "N-POINTS")
            Npoints = std::atoi(value(t, 1));
        else if (key == "NU-RANGE") {
            nu_start = std::atof(value(t, 1));
            nu_end = std::atof(value(t, 2));
        } else if (key == "MEMORY")
            memory = size_t(std::atoi(value(t, 1))) * 1000000000ul;
        else if (key == "NUM-THREADS")
            num_threads = std::atoi(value(t, 1));
    }
    if (Npoints < 1) throw xs_error(XS_ERR_INVALID, "Input: N-POINTS must be >= 1");
    if (!(nu_end > nu_start)) throw xs_error(XS_ERR_INVALID, "Input: NU-RANGE must be ascending");
    if (num_threads < 1) throw xs_error(XS_ERR_INVALID, "Input: NUM-THREADS must be >= 1");
}
