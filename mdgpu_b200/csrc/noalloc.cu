// Solve entry point that allocates no device memory.
//
// mdgpu_solve_device allocates its work vectors (permuted right-hand sides and
// the per-front vectors of the multifrontal sweep) on first use.  Some callers
// cannot do that at solve time: host frameworks whose own caching allocator
// owns the device memory (an allocation behind its back can fail or fragment
// its pool), and latency-bound loops that cannot afford cudaMalloc's
// implicit device synchronization.  This variant takes its work vectors from a fixed
// file-scope device array instead.
//
// Limits and sharing:
//   * the array holds kNoAllocScratchDoubles doubles (32 MiB) on every GPU
//     that loads this library, for the life of the process;
//   * one call needs (n + solve_work_rows) * min(nrhs, 64) doubles (work
//     rows: front vectors and backward partial sums), one more when
//     n * min(nrhs, 64) is odd (the work rows start on 16 bytes); larger
//     requests are rejected with MDGPU_ERR_INVALID and a message giving both
//     numbers;
//   * all calls share the array, and it keeps the last call's contents: calls
//     whose kernels overlap on the GPU (different streams, threads or
//     handles on one device) race on it and must be serialized by the caller;
//   * every scratch entry is written before it is read within a call (the
//     gather fills the permuted right-hand sides, each front vector is formed
//     before use), so nothing needs clearing between calls.
// The array's address is looked up once per device with
// cudaGetSymbolAddress, with that device current: by the analysis that
// uploads a plan to the device (so the module holding the array is loaded
// and its memory committed then, not inside a solve), else by the first
// no-allocation solve on the device (make it before any stream capture).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "kernels.hpp"

namespace mdgpu {

constexpr long long kNoAllocScratchDoubles = 4ll << 20;  // 32 MiB

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double* g_scratch_ptr[kMaxDevices] = {};
}  // namespace

long long noalloc_scratch_capacity() { return kNoAllocScratchDoubles; }

// Device address of the scratch array on the current device (set up on first
// use).  Returns nullptr and fills msg on failure.
double* noalloc_scratch(std::string& msg) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        msg = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            msg = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
            return nullptr;
        }
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    return g_scratch_ptr[dev];
}

}  // namespace mdgpu
