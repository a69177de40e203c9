// Fixed device buffer for the allocation-free field read-back
// (fdf_get_field_noalloc), for callers that may not allocate device memory
// once they are running: a service that sizes all of its GPU memory up front,
// or code that shares the GPU under an external memory budget.
//
// The buffer is a file-scope device array sized at compile time; every GPU
// that loads the library holds it until the process exits.  In host code its
// name is only a host-side stand-in, so its device address is looked up with
// cudaGetSymbolAddress -- once per device, with that device made current, on
// the first allocation-free call on that device (make that first call before
// any stream capture) -- and cached.  Nothing here calls cudaMalloc or
// cudaFree.
#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>
#include <string>

#include "noalloc.hpp"

namespace fdf {

namespace {

// FDF_NOALLOC_MAX_VALUES doubles (8 MiB), shared by every handle on a device
static __device__ __align__(256) double g_noalloc_values[FDF_NOALLOC_MAX_VALUES];

constexpr int kMaxDevices = 64;
std::mutex g_lock;
double* g_addr[kMaxDevices] = {};

}  // namespace

double* noalloc_field_buffer(int device) {
    if (device < 0 || device >= kMaxDevices) throw std::invalid_argument("device ordinal out of range");
    std::lock_guard<std::mutex> g(g_lock);
    if (!g_addr[device]) {
        // the symbol's address is per device: look it up with `device` current
        int prev = 0;
        cudaError_t e = cudaGetDevice(&prev);
        if (e == cudaSuccess && prev != device) e = cudaSetDevice(device);
        void* p = nullptr;
        if (e == cudaSuccess) e = cudaGetSymbolAddress(&p, g_noalloc_values);
        if (prev != device) cudaSetDevice(prev);
        if (e != cudaSuccess)
            throw std::runtime_error(std::string("CUDA error in cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_addr[device] = static_cast<double*>(p);
    }
    return g_addr[device];
}

}  // namespace fdf
