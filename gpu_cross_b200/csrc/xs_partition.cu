// Partition functions on the device: Q(T) = sum over states g_i exp(-c2 E_i / T)
// for a batch of temperatures, the sum compute_partition takes over an ExoMol
// state list on the host (exomol_functions.cpp:44-62), with that file's
// constants.  Each block sums a fixed slice of the states (strided per thread,
// then a fixed tree), a second pass adds the block sums in block order, so
// the result does not depend on scheduling.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "xs_engine.h"
#include "xsec_b200.h"

namespace {

constexpr int kThreads = 256;
constexpr int kBlocks = 296;  // two per SM of a B200

__global__ void k_partition_blocks(const double* __restrict__ e, const int* __restrict__ g, long n,
                                   const double* __restrict__ beta, double* __restrict__ part) {
    __shared__ double red[kThreads];
    const int t = blockIdx.y;
    const double b = beta[t];
    const long per = (n + gridDim.x - 1) / gridDim.x;
    const long lo = long(blockIdx.x) * per;
    const long hi = lo + per < n ? lo + per : n;
    double acc = 0.0;
    for (long i = lo + threadIdx.x; i < hi; i += blockDim.x) acc += double(g[i]) * exp(-b * e[i]);
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[size_t(t) * gridDim.x + blockIdx.x] = red[0];
}

__global__ void k_partition_sum(const double* __restrict__ part, int nblocks, int ntemps,
                                double* __restrict__ q) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntemps) return;
    double s = 0.0;
    for (int k = 0; k < nblocks; ++k) s += part[size_t(t) * nblocks + k];
    q[t] = s;
}

int pfail(int code, const std::string& m) { return xs::set_error(code, m.c_str()); }

}  // namespace

namespace xs {

// Device arrays in, device q out, on `stream`; `work` holds
// partition_work_doubles(n_temps) doubles.
cudaError_t partition_on_stream(const double* d_e, const int* d_g, long n, const double* d_beta,
                                int n_temps, double* d_q, double* work, cudaStream_t stream) {
    const dim3 grid(kBlocks, unsigned(n_temps));
    k_partition_blocks<<<grid, kThreads, 0, stream>>>(d_e, d_g, n, d_beta, work);
    k_partition_sum<<<(n_temps + 127) / 128, 128, 0, stream>>>(work, kBlocks, n_temps, d_q);
    return cudaGetLastError();
}

size_t partition_work_doubles(int n_temps) { return size_t(n_temps) * kBlocks; }

double partition_beta(double temperature) {
    // exomol_functions.cpp:49-53
    const double planck = 6.6260693e-27, vellgt = 2.99792458e10, boltz = 1.380658e-16;
    return planck * vellgt / (boltz * temperature);
}

}  // namespace xs

extern "C" int xs_partition_sum(int device, const double* energies, const int* gns, size_t n,
                                const double* temperatures, int n_temps, double* q) {
    if ((n > 0 && (!energies || !gns)) || !temperatures || !q || n_temps < 1 || n_temps > 65535)
        return pfail(XS_ERR_INVALID, "xs_partition_sum: bad arguments");
    for (int t = 0; t < n_temps; ++t)
        if (!(temperatures[t] > 0.0)) return pfail(XS_ERR_INVALID, "xs_partition_sum: T must be > 0");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return pfail(XS_ERR_NODEVICE, "xs_partition_sum: no such CUDA device");
    }
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != device) cudaSetDevice(device);
    std::vector<double> beta(static_cast<size_t>(n_temps));
    for (int t = 0; t < n_temps; ++t) beta[size_t(t)] = xs::partition_beta(temperatures[t]);
    double *d_e = nullptr, *d_b = nullptr, *d_q = nullptr, *d_w = nullptr;
    int* d_g = nullptr;
    const size_t nn = n > 0 ? n : 1;
    cudaError_t err = cudaMalloc(&d_e, nn * sizeof(double));
    if (err == cudaSuccess) err = cudaMalloc(&d_g, nn * sizeof(int));
    if (err == cudaSuccess) err = cudaMalloc(&d_b, size_t(n_temps) * sizeof(double));
    if (err == cudaSuccess) err = cudaMalloc(&d_q, size_t(n_temps) * sizeof(double));
    if (err == cudaSuccess) err = cudaMalloc(&d_w, xs::partition_work_doubles(n_temps) * sizeof(double));
    if (err == cudaSuccess && n > 0) err = cudaMemcpy(d_e, energies, n * sizeof(double), cudaMemcpyHostToDevice);
    if (err == cudaSuccess && n > 0) err = cudaMemcpy(d_g, gns, n * sizeof(int), cudaMemcpyHostToDevice);
    if (err == cudaSuccess)
        err = cudaMemcpy(d_b, beta.data(), size_t(n_temps) * sizeof(double), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = xs::partition_on_stream(d_e, d_g, long(n), d_b, n_temps, d_q, d_w, nullptr);
    if (err == cudaSuccess)
        err = cudaMemcpy(q, d_q, size_t(n_temps) * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d_e);
    cudaFree(d_g);
    cudaFree(d_b);
    cudaFree(d_q);
    cudaFree(d_w);
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return pfail(err == cudaErrorMemoryAllocation ? XS_ERR_NOMEM : XS_ERR_CUDA,
                     std::string("xs_partition_sum: ") + cudaGetErrorString(err));
    }
    return XS_OK;
}
