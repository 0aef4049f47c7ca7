// Stored-energy reduction for callers that cannot allocate device memory.
//
// fitb_energy() keeps its block partial sums in scratch that the engine
// handle allocated with cudaMalloc.  Some callers of this library cannot
// allocate at all while they run: a host process that embeds the engine in
// a real-time loop with a fixed device-memory budget, a framework that owns
// every device byte through its own pool, or code that must not trigger the
// implicit device synchronisation cudaMalloc/cudaFree may cause in the
// middle of a time step.  fitb_energy_noalloc() serves them: the caller
// passes the field and mass arrays and the output slot (all device memory it
// already owns), and the partial sums live in the fixed array below, which
// is part of the loaded library image on every device that uses it.
//
// Rules of use:
//   * The first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture that would record it.
//   * All calls share the one array.  Calls whose launches overlap on the
//     GPU (different streams, or host threads racing) corrupt each other's
//     partial sums: serialise them.
//   * The array keeps the previous call's contents; each call writes every
//     slot it later reads, so nothing has to start at zero.
//   * A CUDA error still pending from earlier work on the calling thread
//     makes the call fail without launching; the error is left in place for
//     the code that caused it.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/fitb200.h"

namespace fitb {
void set_last_error(const std::string& msg);
}

namespace {

constexpr int kThreads = 256;
constexpr int kItemsPerThread = 16;
constexpr long long kItemsPerBlock = (long long)kThreads * kItemsPerThread;  // 4096
constexpr int kMaxPartials = 131072;  // 1 MiB of float64 partial sums
constexpr int kMaxDevices = 64;

// Per-block partial sums of the most recent call (see the rules above).
static __device__ __align__(256) double g_energy_partials[kMaxPartials];

double* g_partials_addr[kMaxDevices] = {};
std::mutex g_partials_mutex;

template <typename T>
__global__ void k_energy_blocks(const T* __restrict__ f, const T* __restrict__ m, long long n,
                                double* __restrict__ partials) {
    // Fixed element -> block mapping and a fixed in-block tree: the result
    // does not depend on scheduling.
    const long long base = (long long)blockIdx.x * kItemsPerBlock;
    double acc = 0.0;
#pragma unroll
    for (int q = 0; q < kItemsPerThread; ++q) {
        const long long t = base + (long long)q * kThreads + threadIdx.x;
        if (t < n) {
            const double v = (double)f[t];
            acc += (double)m[t] * v * v;
        }
    }
    __shared__ double red[kThreads];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

__global__ void k_energy_finish(const double* __restrict__ partials, int n, double* __restrict__ out) {
    __shared__ double red[kThreads];
    double acc = 0.0;
    for (int t = threadIdx.x; t < n; t += kThreads) acc += partials[t];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = 0.5 * red[0];
}

int fail_with(int code, const char* msg) {
    fitb::set_last_error(msg);
    return code;
}

}  // namespace

extern "C" int fitb_energy_noalloc(const void* e, const void* h, const void* m_eps, const void* m_mu,
                                   int64_t n_e, int64_t n_h, int32_t precision, double* out,
                                   void* stream) {
    if (precision != 4 && precision != 8) return fail_with(FITB_ERR_ARG, "precision must be 4 or 8");
    if (n_e < 0 || n_h < 0) return fail_with(FITB_ERR_ARG, "array lengths must be >= 0");
    // block counts without rounding overflow: lengths near INT64_MAX must
    // still end in the limit error below
    const long long nb_e = n_e / kItemsPerBlock + (n_e % kItemsPerBlock != 0);
    const long long nb_h = n_h / kItemsPerBlock + (n_h % kItemsPerBlock != 0);
    if (nb_e > kMaxPartials || nb_h > kMaxPartials || nb_e + nb_h > kMaxPartials) {
        char buf[256];
        snprintf(buf, sizeof(buf),
                 "fitb_energy_noalloc: n_e + n_h needs %lld partial sums, the fixed scratch holds %d "
                 "(at most %lld elements per array pair)",
                 nb_e + nb_h, kMaxPartials, (long long)kMaxPartials * kItemsPerBlock);
        return fail_with(FITB_ERR_LIMIT, buf);
    }
    if (!out || (n_e > 0 && (!e || !m_eps)) || (n_h > 0 && (!h || !m_mu)))
        return fail_with(FITB_ERR_ARG, "fitb_energy_noalloc: null device pointer");
    // An error left by earlier work on this thread is the caller's: report
    // it without launching and without clearing it.
    cudaError_t err = cudaPeekAtLastError();
    if (err != cudaSuccess) {
        char buf[256];
        snprintf(buf, sizeof(buf),
                 "fitb_energy_noalloc: a CUDA error from earlier work is pending (%s); nothing was launched",
                 cudaGetErrorString(err));
        return fail_with(FITB_ERR_CUDA, buf);
    }
    int dev = 0;
    err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return fail_with(FITB_ERR_CUDA, cudaGetErrorString(err));
    if (dev < 0 || dev >= kMaxDevices) return fail_with(FITB_ERR_LIMIT, "device ordinal beyond the supported range");
    double* partials = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_partials_mutex);
        if (!g_partials_addr[dev]) {
            void* p = nullptr;
            err = cudaGetSymbolAddress(&p, g_energy_partials);
            if (err != cudaSuccess) return fail_with(FITB_ERR_CUDA, cudaGetErrorString(err));
            g_partials_addr[dev] = static_cast<double*>(p);
        }
        partials = g_partials_addr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // each launch's own error, checked right after it
    auto launched = [](const char* what) {
        const cudaError_t le = cudaGetLastError();
        if (le == cudaSuccess) return true;
        char buf[256];
        snprintf(buf, sizeof(buf), "fitb_energy_noalloc: %s launch failed: %s", what, cudaGetErrorString(le));
        fitb::set_last_error(buf);
        return false;
    };
    if (nb_e) {
        if (precision == 4)
            k_energy_blocks<float><<<(int)nb_e, kThreads, 0, s>>>((const float*)e, (const float*)m_eps, n_e, partials);
        else
            k_energy_blocks<double><<<(int)nb_e, kThreads, 0, s>>>((const double*)e, (const double*)m_eps, n_e, partials);
        if (!launched("E partial sums")) return FITB_ERR_CUDA;
    }
    if (nb_h) {
        if (precision == 4)
            k_energy_blocks<float><<<(int)nb_h, kThreads, 0, s>>>((const float*)h, (const float*)m_mu, n_h, partials + nb_e);
        else
            k_energy_blocks<double><<<(int)nb_h, kThreads, 0, s>>>((const double*)h, (const double*)m_mu, n_h, partials + nb_e);
        if (!launched("H partial sums")) return FITB_ERR_CUDA;
    }
    k_energy_finish<<<1, kThreads, 0, s>>>(partials, (int)(nb_e + nb_h), out);
    if (!launched("final sum")) return FITB_ERR_CUDA;
    return FITB_OK;
}
