// Volume stage kernel in the reference's operation order (compiled with
// -fmad=false).  One thread per node of a block computes, for that node,
// exactly the sequence of roundings the reference performs across
//   fields::scale_df           src/fields.cpp:293-300
//   block::calc_df_3d          src/block.cpp:1541-2050
//   block::calc_df_mode2/_szz  src/block.cpp:1048-1294
//   block::calc_df_mode3       src/block.cpp:1384-1539
//   boundary::apply_bcs        src/boundary.cpp:265-503
//   fields::update             src/fields.cpp:302-309
// fused into one pass: df is scaled, the x, y (and z) derivative taps are
// accumulated in the reference's tap order, then the outer-face SATs of the
// faces the node sits on, in face order.  Nodes on interface faces keep
// their rate for the interface kernel, which adds the interface SAT and
// finishes the update; every other node finishes here (RK update, and on the
// last stage the return map and the absolute-stress round trip).
#include <cuda_runtime.h>

#include "stage_exact.cuh"

namespace fdf {

namespace {

template <typename T, int NDIM, int MODE, bool HET>
__global__ void __launch_bounds__(128) k_volume_exact(VolumeArgs<T> a, BlockDev B, StageArgs sa) {
    volume_node<T, NDIM, MODE, HET>(a, B, sa, blockIdx.x * (long long)blockDim.x + threadIdx.x);
}

// Every block of a problem in one launch: thread t takes node t - start[b] of
// the block b whose range holds t, with the same per-node arithmetic as the
// per-block launch (the block table is read from device memory).  Small
// problems, whose per-block launches each fill a fraction of one wave, then
// overlap their blocks.
template <typename T, int NDIM, int MODE, bool HET>
__global__ void __launch_bounds__(128) k_volume_exact_all(VolumeArgs<T> a, const BlockDev* __restrict__ blks,
                                                          BlockRanges r, StageArgs sa) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= r.start[FDF_ALLB_MAX]) return;
    int b = 0;
    long long s = 0;
#pragma unroll
    for (int q = 1; q < FDF_ALLB_MAX; q++)
        if (t >= r.start[q]) {
            b = q;
            s = r.start[q];
        }
    volume_node<T, NDIM, MODE, HET>(a, blks[b], sa, t - s);
}

}  // namespace

template <typename T>
void launch_volume_exact(const VolumeArgs<T>& a, const BlockDev& b, const StageArgs& sa, cudaStream_t s) {
    long long nn = (long long)(b.xe - b.xb) * b.n[1] * b.n[2];
    if (nn <= 0) return;
    unsigned grid = (unsigned)((nn + 127) / 128);
    // heterogeneous material: modes II and 3D (mode III is rejected at input)
    if (a.L.ndim == 3) {
        if (b.mat)
            k_volume_exact<T, 3, 2, true><<<grid, 128, 0, s>>>(a, b, sa);
        else
            k_volume_exact<T, 3, 2, false><<<grid, 128, 0, s>>>(a, b, sa);
    } else if (a.L.mode == 2) {
        if (b.mat)
            k_volume_exact<T, 2, 2, true><<<grid, 128, 0, s>>>(a, b, sa);
        else
            k_volume_exact<T, 2, 2, false><<<grid, 128, 0, s>>>(a, b, sa);
    } else {
        k_volume_exact<T, 2, 3, false><<<grid, 128, 0, s>>>(a, b, sa);
    }
}

template <typename T>
void launch_volume_exact_all(const VolumeArgs<T>& a, const BlockDev* blks_dev, const BlockDev* blks, int nb,
                             const StageArgs& sa, cudaStream_t s) {
    BlockRanges r{};
    long long n = 0;
    for (int b = 0; b < FDF_ALLB_MAX; b++) {
        r.start[b] = n;
        if (b < nb) n += (long long)(blks[b].xe - blks[b].xb) * blks[b].n[1] * blks[b].n[2];
    }
    r.start[FDF_ALLB_MAX] = n;   // ranges of absent blocks are empty and never selected
    if (n <= 0) return;
    const unsigned grid = (unsigned)((n + 127) / 128);
    const bool het = nb > 0 && blks[0].mat != nullptr;   // one material array for all blocks
    if (a.L.ndim == 3) {
        if (het)
            k_volume_exact_all<T, 3, 2, true><<<grid, 128, 0, s>>>(a, blks_dev, r, sa);
        else
            k_volume_exact_all<T, 3, 2, false><<<grid, 128, 0, s>>>(a, blks_dev, r, sa);
    } else if (a.L.mode == 2) {
        if (het)
            k_volume_exact_all<T, 2, 2, true><<<grid, 128, 0, s>>>(a, blks_dev, r, sa);
        else
            k_volume_exact_all<T, 2, 2, false><<<grid, 128, 0, s>>>(a, blks_dev, r, sa);
    } else {
        k_volume_exact_all<T, 2, 3, false><<<grid, 128, 0, s>>>(a, blks_dev, r, sa);
    }
}

template void launch_volume_exact_all<double>(const VolumeArgs<double>&, const BlockDev*, const BlockDev*, int,
                                              const StageArgs&, cudaStream_t);
template void launch_volume_exact_all<float>(const VolumeArgs<float>&, const BlockDev*, const BlockDev*, int,
                                             const StageArgs&, cudaStream_t);
template void launch_volume_exact<double>(const VolumeArgs<double>&, const BlockDev&, const StageArgs&, cudaStream_t);
template void launch_volume_exact<float>(const VolumeArgs<float>&, const BlockDev&, const StageArgs&, cudaStream_t);

}  // namespace fdf
