// Allocation-free variant of the conservation-totals reduction.
//
// Some callers cannot allocate device memory: an embedding application
// whose device memory is entirely owned by its own allocator (a framework's
// caching pool or a fixed arena handed out at start-up), or a solver loop
// that must not allocate once it runs.  rkdg_conservation_totals_noalloc
// serves them: the caller passes its own device inputs and output, and the
// reduction's per-block partial sums live in the file-scope device array
// below instead of memory from cudaMalloc.
//
// The array is static device memory of this library: every GPU that loads
// librkdg.so holds it (kMaxBlocks * 4 doubles = 128 KiB) until the process
// exits.  Host code may not use the symbol as a pointer; its device address
// is looked up once per device with cudaGetSymbolAddress (on the first call
// made with that device current) and passed to the kernels.  The address
// belongs to the context that was current then, so a device reset between
// calls (which unloads the module) is not supported.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "rkdg_internal.hpp"

namespace {

constexpr int kBlock = 256;
constexpr int kMaxBlocks = 4096;  // largest mesh: kMaxBlocks * kBlock elements
constexpr int kMaxDevices = 64;

// Per-block partial sums of the four totals (one copy per GPU).  Every call
// writes the slots of the blocks it launches before reading them, so the
// contents a previous call left behind are never read and nothing has to be
// cleared; calls that overlap on the same GPU (on different streams, or from
// different host threads) share the array and race on it.
static __device__ __align__(256) double g_partials[kMaxBlocks * 4];

__global__ void __launch_bounds__(kBlock) partial_kernel(int T, const double* __restrict__ means,
                                                         int ld, const double* __restrict__ area,
                                                         double* __restrict__ partial) {
    __shared__ double s[4][kBlock];
    const int e = blockIdx.x * kBlock + threadIdx.x;
    for (int v = 0; v < 4; ++v) s[v][threadIdx.x] = e < T ? area[e] * means[(size_t)v * ld + e] : 0.0;
    __syncthreads();
    for (int o = kBlock / 2; o > 0; o >>= 1) {  // fixed-order tree: deterministic
        if (threadIdx.x < o)
            for (int v = 0; v < 4; ++v) s[v][threadIdx.x] += s[v][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int v = 0; v < 4; ++v) partial[(size_t)4 * blockIdx.x + v] = s[v][0];
}

__global__ void __launch_bounds__(kBlock) final_kernel(int n, const double* __restrict__ partial,
                                                       double* __restrict__ out) {
    __shared__ double s[4][kBlock];
    double acc[4] = {0, 0, 0, 0};
    for (int i = threadIdx.x; i < n; i += kBlock)
        for (int v = 0; v < 4; ++v) acc[v] += partial[(size_t)4 * i + v];
    for (int v = 0; v < 4; ++v) s[v][threadIdx.x] = acc[v];
    __syncthreads();
    for (int o = kBlock / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int v = 0; v < 4; ++v) s[v][threadIdx.x] += s[v][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int v = 0; v < 4; ++v) out[v] = s[v][0];
}

std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

// Device address of g_partials on the current device, looked up once per device.
double* partials_address(int dev) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_partials);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw rkdg::Error{RKDG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e)};
        }
        g_addr[dev] = static_cast<double*>(p);
    }
    return g_addr[dev];
}

}  // namespace

extern "C" int rkdg_conservation_totals_noalloc(int32_t ntri, const double* d_means, int32_t ld,
                                                const double* d_area, double* d_totals,
                                                void* stream) {
    try {
        if (ntri <= 0 || ld < ntri || !d_means || !d_area || !d_totals)
            throw rkdg::Error{RKDG_ERR_INVALID, "rkdg_conservation_totals_noalloc: bad arguments"};
        const int nblocks = (ntri + kBlock - 1) / kBlock;
        if (nblocks > kMaxBlocks)
            throw rkdg::Error{RKDG_ERR_INVALID,
                              "rkdg_conservation_totals_noalloc: ntri = " + std::to_string(ntri) +
                                  " exceeds the maximum of " + std::to_string(kMaxBlocks * kBlock) +
                                  " triangles (static scratch of " + std::to_string(kMaxBlocks) +
                                  " block partials)"};
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw rkdg::Error{RKDG_ERR_NODEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e)};
        }
        if (dev < 0 || dev >= kMaxDevices) throw rkdg::Error{RKDG_ERR_INVALID, "device index out of range"};
        double* partial = partials_address(dev);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        partial_kernel<<<nblocks, kBlock, 0, s>>>(ntri, d_means, ld, d_area, partial);
        final_kernel<<<1, kBlock, 0, s>>>(nblocks, partial, d_totals);
        e = cudaGetLastError();
        if (e != cudaSuccess)
            throw rkdg::Error{RKDG_ERR_CUDA, std::string("rkdg_conservation_totals_noalloc launch: ") +
                                                 cudaGetErrorString(e)};
        return RKDG_OK;
    } catch (const rkdg::Error& err) {
        rkdg::set_error(err.msg);
        return err.code;
    }
}
