// Test infrastructure only: drives the UNMODIFIED reference CPU backend
// (OpenMPManager.cpp + BaseManager.cpp + profiles.cpp, compiled from the
// reference tree by oracle/Makefile) through its own BaseManager interface
// (BaseManager.h:6-33).  Nothing in the product links or loads this file.
//
// Call order mirrors what BaseProfile/VoigtProfile do with a manager
// (VoigtProfile.cpp:20-26, BaseProfile.cpp:49-62, BaseProfile.cpp:65-67):
//   InitializeVectors -> TransferFreq -> InitializeConstants ->
//   TransferVectors -> ExecuteCrossSection -> TransferResults.
#include "OpenMPManager.h"

#include <fcntl.h>
#include <malloc.h>
#include <unistd.h>

#include <cstdio>

// profiles.cpp is C99 (double complex); it is compiled as C with
// -Dhumlic=humlic_c and reached from the C++ declaration in profiles.h here.
extern "C" double humlic_c(double x, double y);
double humlic(double x, double y) { return humlic_c(x, y); }

namespace {

// The reference prints progress to stdout on every call; keep the caller's
// stdout clean while the reference runs.
struct QuietStdout {
    int saved = -1;
    explicit QuietStdout(bool enable) {
        if (!enable) return;
        fflush(stdout);
        saved = dup(1);
        int devnull = open("/dev/null", O_WRONLY);
        if (devnull >= 0) {
            dup2(devnull, 1);
            close(devnull);
        }
    }
    ~QuietStdout() {
        if (saved < 0) return;
        fflush(stdout);
        dup2(saved, 1);
        close(saved);
    }
};

}  // namespace

extern "C" {

// profile: 0 GAUSSIAN, 1 DOPPLER, 2 VOIGT (Input.h:9-15 order).
// freq/intens: the full grid (npoints_total).  intens is the initial grid on
// input and the reference's TransferResults output on return.
// One chunk (points, start_idx) of n_lines lines is executed, as
// BaseProfile::PerformCrossSection does.  Returns 0 on success.
int ref_cpu_run(int profile, int num_threads, int npoints_total,
                double* freq, double* intens, long n_lines,
                const double* energies, const double* nu, const double* aif,
                const int* gns, const double* gamma, const double* n,
                double half_width, double temperature, double partition,
                double dfreq, double mean_mass, double pressure,
                double ref_temp, int points, int start_idx, int quiet) {
    if (num_threads < 1 || npoints_total < 1 || n_lines < 0) return 1;
    QuietStdout q(quiet != 0);
    // OpenMPManager::TransferResults adds the thread grids into g_intens,
    // which InitializeVectors allocates with new[] and never clears
    // (OpenMPManager.cpp:23,123-127).  While the manager allocates, have
    // malloc fill every new block with zero bytes (M_PERTURB with 0xff fills
    // allocations with the complement, 0x00), so the result does not depend
    // on whatever the heap held before.
    mallopt(M_PERTURB, 0xff);
    // OpenMPManager budgets half of total_memory (OpenMPManager.cpp:9); size
    // it so that N_trans >= n_lines.
    size_t per_line = 6 * sizeof(double) + sizeof(int);
    size_t grid_bytes = size_t(npoints_total) * sizeof(double) * size_t(2 + num_threads);
    size_t total = 2 * (grid_bytes + size_t(n_lines + 16) * per_line + 4096);
    int rc = 0;
    {
        OpenMPManager mgr(static_cast<ProfileType>(profile), num_threads, total);
        mgr.InitializeVectors(npoints_total);
        mallopt(M_PERTURB, 0);
        if (mgr.GetNtrans() < size_t(n_lines)) {
            rc = 2;
        } else {
            mgr.TransferFreq(freq, intens, npoints_total);
            mgr.InitializeConstants(half_width, temperature, partition, dfreq,
                                    mean_mass, pressure, ref_temp);
            mgr.TransferVectors(size_t(n_lines), const_cast<double*>(energies),
                                const_cast<double*>(nu), const_cast<double*>(aif),
                                const_cast<int*>(gns), const_cast<double*>(gamma),
                                const_cast<double*>(n));
            mgr.ExecuteCrossSection(points, int(n_lines), start_idx);
            mgr.TransferResults(freq, intens, npoints_total);
        }
        // OpenMPManager has no destructor that frees its arrays; the harness
        // process is short-lived, so they are left to the OS like the
        // reference's own main() does.
    }
    return rc;
}

}  // extern "C"
