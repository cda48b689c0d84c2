// Projector on caller-owned device vectors with no allocation at all.
//
// Some callers of the PCPG building blocks cannot call cudaMalloc at the
// moment they project: a serving loop that admits work against a fixed
// device-memory budget must not grow its footprint per call, and a
// latency-bound loop that shares the GPU with other streams cannot afford
// the device-wide synchronisation an allocation may cause.  For them the
// reduction scratch of the projector (6 partial sums per Gf chunk) lives in
// the static array below instead of the context's own buffer.
//
// The array is HTF_NOALLOC_SCRATCH_DOUBLES doubles (8 MiB); every GPU that
// loads the library holds it until the process exits.  All calls share it
// and it keeps the last call's contents; each call overwrites every entry it
// reads before reading it, so nothing needs to start at zero.  Calls whose
// kernels overlap on the GPU (different streams without ordering) race on
// the array and must be serialised by the caller.  The first call on a
// device looks the array's device address up (once per device, with that
// device current) and should come before any stream capture.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "engine.hpp"

namespace htf {

static __device__ __align__(256) double g_noalloc_scratch[HTF_NOALLOC_SCRATCH_DOUBLES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_addr[kMaxDevices] = {nullptr};
}  // namespace

// Device address of the static scratch on the current device, looked up once
// per device (the first call on a device does the lookup, so it must come
// before any stream capture that contains later calls).
int noalloc_scratch(double **ptr, size_t *cap, std::string &err) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        err = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
        return HTF_ECUDA;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        double *p = nullptr;
        e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            err = std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e);
            return HTF_ECUDA;
        }
        g_addr[dev] = p;
    }
    *ptr = g_addr[dev];
    *cap = HTF_NOALLOC_SCRATCH_DOUBLES;
    return HTF_OK;
}

}  // namespace htf
