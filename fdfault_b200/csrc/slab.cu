// Ghost-plane exchange of an x slab: the copy between the field buffer and a
// contiguous exchange buffer.  The reference's fields::exchange_neighbors
// (src/fields.cpp:276-291) sends each MPI neighbour the planes next to the
// shared face through derived datatypes; here the planes of one side are, per
// component, one contiguous range of the field buffer (x is the slowest
// index), so a side is `ncomp` ranges of `len` elements, and one kernel moves
// them to or from a buffer that a collective library sends as it is.
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>

#include "kernels.hpp"

namespace fdf {

namespace {

// element e of the buffer is component e / len, offset e % len of the range
// that starts at `off` in every component; 16-byte vectors when every range
// start and length allows it
template <typename V>
__global__ void __launch_bounds__(256) k_ghost_copy(V* __restrict__ field, long long cstride, int ncomp, long long off,
                                                    long long len, V* __restrict__ buf, int unpack) {
    const long long n = (long long)ncomp * len;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long c = e / len, r = e - c * len;
        V* f = field + c * cstride + off + r;
        if (unpack)
            *f = buf[e];
        else
            buf[e] = *f;
    }
}

template <typename V>
void launch_as(void* field, long long cstride, int ncomp, long long off, long long len, void* buf, int unpack,
               cudaStream_t s) {
    const long long n = (long long)ncomp * len;
    long long grid = (n + 255) / 256;
    if (grid > 148 * 16) grid = 148 * 16;
    if (grid < 1) grid = 1;
    k_ghost_copy<V><<<(unsigned)grid, 256, 0, s>>>((V*)field, cstride, ncomp, off, len, (V*)buf, unpack);
}

}  // namespace

void launch_ghost_copy(void* field, int elem_bytes, long long cstride, int ncomp, long long off, long long len,
                       void* buf, int unpack, cudaStream_t s) {
    if (elem_bytes != 4 && elem_bytes != 8) throw std::runtime_error("ghost copy: element size is 4 or 8 bytes");
    if (len <= 0 || ncomp <= 0) return;
    const int vec = 16 / elem_bytes;   // elements per 16-byte vector
    const bool aligned = (cstride % vec == 0) && (off % vec == 0) && (len % vec == 0) &&
                         ((reinterpret_cast<uintptr_t>(field) | reinterpret_cast<uintptr_t>(buf)) % 16 == 0);
    if (aligned)
        launch_as<int4>(field, cstride / vec, ncomp, off / vec, len / vec, buf, unpack, s);
    else if (elem_bytes == 8)
        launch_as<double>(field, cstride, ncomp, off, len, buf, unpack, s);
    else
        launch_as<float>(field, cstride, ncomp, off, len, buf, unpack, s);
}

}  // namespace fdf
