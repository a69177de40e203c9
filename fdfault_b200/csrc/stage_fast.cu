// Tiled FP32 volume kernel for 3D blocks (placeholder dispatch: the tiled
// kernel is not enabled for any layout yet, so FP32 problems run the
// one-thread-per-node kernel).
#include <cuda_runtime.h>

#include "kernels.hpp"

namespace fdf {

bool fast3d_supported(const Layout& L, const BlockDev& b, int order) {
    (void)L;
    (void)b;
    (void)order;
    return false;
}

void launch_volume_fast3d(const VolumeArgs<float>& a, const BlockDev& b, const StageArgs& sa, cudaStream_t s) {
    launch_volume_exact<float>(a, b, sa, s);
}

}  // namespace fdf
