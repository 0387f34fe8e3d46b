// Test infrastructure only: the two symbols the reference's CPU-only main
// program needs that its C++ sources do not define, for oracle/_ref/ref_main
// (built by oracle/Makefile from the reference's own main.cpp, Input.cpp,
// BaseProfile.cpp, VoigtProfile.cpp, DopplerProfile.cpp, HybridManager.cpp,
// OpenMPManager.cpp, the readers and the bzip2 transition reader).
//
//  * humlic: profiles.cpp is C99 (double complex) and is compiled as C under
//    the name humlic_c; this forwards the C++ declaration of profiles.h.
//  * bd_tips_2011_: the HITRAN TIPS partition sums are Fortran
//    (HITRAN_files/BD_TIPS_2011_v1p0.for) and no Fortran compiler is
//    available.  The stand-in returns Q = $REF_TIPS_Q (0 when unset) for any
//    molecule and temperature; the end-to-end cases give PARTITION explicitly
//    and carry Einstein A coefficients, so the sums are not used for results.
#include <cstdlib>

extern "C" double humlic_c(double x, double y);
double humlic(double x, double y) { return humlic_c(x, y); }

extern "C" void bd_tips_2011_(int* mol, double* temp, int* iso, double* gi, double* qt) {
    (void)mol;
    (void)temp;
    (void)iso;
    const char* q = std::getenv("REF_TIPS_Q");
    *gi = 0.0;
    *qt = q ? std::atof(q) : 0.0;
}
