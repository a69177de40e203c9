// Fixed device buffer for the allocation-free field read-back
// (fdf_get_field_noalloc).  The buffer is a file-scope device array sized at
// compile time; its device address is looked up once per device and cached.
// Nothing here calls cudaMalloc or cudaFree.
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
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_values);
        if (e != cudaSuccess)
            throw std::runtime_error(std::string("CUDA error in cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_addr[device] = static_cast<double*>(p);
    }
    return g_addr[device];
}

}  // namespace fdf
