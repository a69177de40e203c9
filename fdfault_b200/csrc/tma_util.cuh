// Helpers shared by the kernels that stage planes through shared memory with
// TMA tensor copies (cp.async.bulk.tensor) and count their completion on
// mbarriers: barrier set-up, bounded waits, the copy instructions, and the
// host-side tensor-map encoder (fetched from the driver at first use).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

namespace fdf {

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint32_t bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(1) : "memory");
}
__device__ __forceinline__ void bar_init_count(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
// one arrival (release semantics at CTA scope)
__device__ __forceinline__ void bar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void bar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void bar_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool bar_test(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// polls of a drain wait (copies in flight before an early exit): independent
// of the consumers' limit, so a CTA never leaves with a copy still landing
constexpr long long TMA_DRAIN_LIMIT = 1LL << 24;
// wait for phase `parity` of the barrier; false when `limit` polls pass first.
// The first poll never blocks, the later ones may suspend the thread for a
// while (mbarrier.try_wait), so a limit of 1 is one immediate test; a
// negative limit gives up at once without looking (the expiry path on demand).
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity, long long limit) {
    if (limit < 0) return false;
    if (bar_test(bar, parity)) return true;
    for (long long it = 1; it < limit; it++)
        if (bar_try(bar, parity)) return true;
    return false;
}
// generic-proxy accesses of shared memory before this point are ordered
// before later asynchronous-proxy (TMA) writes to it
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void tma4(uint32_t dst, const CUtensorMap* map, int x, int y, int z, int w, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
        "[%2];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y), "r"(z), "r"(w)
        : "memory");
}
__device__ __forceinline__ void tma3(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
        "[%2];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y), "r"(z)
        : "memory");
}

using TmaEncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline TmaEncodeFn tma_encode_fn() {
    static TmaEncodeFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p)
            throw std::runtime_error("CUDA driver entry point cuTensorMapEncodeTiled is unavailable");
        fn = reinterpret_cast<TmaEncodeFn>(p);
    }
    return fn;
}

// FP32 tiled tensor map: dims[0] innermost; strides in bytes for dims 1..rank-1;
// parts of a box outside dims are filled with zeros
inline void tma_encode(CUtensorMap* m, const float* base, cuuint32_t rank, const cuuint64_t* dims,
                       const cuuint64_t* strides, const cuuint32_t* box) {
    const cuuint32_t es[4] = {1, 1, 1, 1};
    const CUresult r = tma_encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, const_cast<float*>(base), dims,
                                       strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                       CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw std::runtime_error("CUDA error in cuTensorMapEncodeTiled: " + std::to_string((int)r));
}

}  // namespace fdf
