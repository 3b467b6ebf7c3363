// The action without any device allocation (a43g_action_multiply_noalloc).
//
// Some callers cannot let a library call cudaMalloc: hosts that hand out all device memory
// through their own pool and forbid allocations behind their back, processes that have already
// claimed nearly all of the GPU's memory, and latency-bound loops where the device-wide
// synchronization of cudaMalloc/cudaFree would stall other streams.  The ordinary
// a43g_action_multiply allocates the projector coefficient scratch of a plan on its first call;
// this variant keeps that scratch in one fixed array in device memory instead, compiled into the
// library: kScratchBytes (16 MiB) on every GPU that loads the library, held until the process
// exits.  Plans whose projector coefficients need more are rejected with an error.
//
// The array is shared by every call on a device and keeps the data of the last call.  The part
// the projection accumulates into is zeroed by each call; everything else is overwritten before
// it is read.  Calls whose GPU work overlaps (on different streams, from different threads or
// for different plans) therefore race on the array and must be serialized by the caller.
//
// The device address of the array is looked up once per device and kept.  A cudaDeviceReset
// destroys the context that holds the array; the kept address is then stale, so this entry point
// must not be used on a device after the caller has reset it.
#include "device.cuh"
#include "noalloc.hpp"

#include <mutex>

namespace a43g {

namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_lookup;
void *g_address[kMaxDevices] = {};

size_t round256(size_t n) { return (n + 255) & ~size_t(255); }

} // namespace

size_t noalloc_capacity() { return kScratchBytes; }

size_t noalloc_required(DevicePlan const &dp, size_t real_bytes) {
    if (dp.nAI < 1 || dp.nCols < 1) return 0;
    size_t const nI = size_t(dp.ncoeffI)*dp.nCols*128, nA = size_t(dp.ncoeffA)*dp.nCols*128;
    return 2*round256(nI*real_bytes) + 2*round256(nA*sizeof(double));
}

bool noalloc_scratch_address(void **address) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (cudaSuccess != e) { set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e)); return false; }
    if (dev < 0 || dev >= kMaxDevices) { set_error("device ordinal beyond the supported 64"); return false; }
    std::lock_guard<std::mutex> lock(g_lookup);
    if (!g_address[dev]) {
        // the host-side name of the array is not a device address: ask the runtime, once per device
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (cudaSuccess != e || !p) {
            set_error(std::string("cudaGetSymbolAddress of the scratch array: ") + cudaGetErrorString(e));
            return false;
        }
        g_address[dev] = p;
    }
    *address = g_address[dev];
    return true;
}

template <typename T>
bool action_noalloc(DevicePlan &dp, T *y, T const *x, uint16_t const *colIndex, cudaStream_t st) {
    size_t const need = noalloc_required(dp, sizeof(T));
    if (need > kScratchBytes) {
        set_error("the projector coefficients of this plan need " + std::to_string(need) +
                  " bytes of scratch, more than the " + std::to_string(kScratchBytes) +
                  " bytes of the allocation-free entry point; use a43g_action_multiply");
        return false;
    }
    DyadicScratch sc{nullptr, nullptr, nullptr, nullptr};
    if (need) {
        void *base = nullptr;
        if (!noalloc_scratch_address(&base)) return false;
        char *p = static_cast<char*>(base);
        size_t const nI = size_t(dp.ncoeffI)*dp.nCols*128, nA = size_t(dp.ncoeffA)*dp.nCols*128;
        sc.apc = p;  p += round256(nI*sizeof(T));
        sc.cad = p;  p += round256(nI*sizeof(T));
        sc.aac = reinterpret_cast<double*>(p);  p += round256(nA*sizeof(double));
        sc.cadd = reinterpret_cast<double*>(p);
    }
    return launch_action_scratch<T>(dp, y, x, colIndex, st, sc);
}

template bool action_noalloc<double>(DevicePlan &, double *, double const *, uint16_t const *, cudaStream_t);
template bool action_noalloc<float>(DevicePlan &, float *, float const *, uint16_t const *, cudaStream_t);

} // namespace a43g
