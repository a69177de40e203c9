// Host-callable launchers for the device kernels of the fdfault B200 path.
#pragma once

#include <cuda_runtime.h>

#include "fdf_types.hpp"

namespace fdf {

// block geometry for the set-up kernels
struct GeoBlock {
    int lo[3], n[3];
    double dx[3];
    const double* surf[6];   // bounding surfaces, [ndim][sn0][sn1]
    int sn0[6], sn1[6];
};

void launch_transfinite(const Layout& L, const GeoBlock& g, double* X, cudaStream_t s);
void launch_metrics(const Layout& L, const GeoBlock& g, int order, const double* X, double* M, double* J, int* status,
                    cudaStream_t s);
void launch_face_normals(const Layout& L, int d, int at, int lo0, int n0, int lo1, int n1, int flip, double h0dx,
                         const double* M, double* nx[3], double* dl, double* dl2, int at2, double h0dx2,
                         cudaStream_t s);
// largest cs |grad xi_l| / dxi_l over the block; cs per node from mat
// (rho, lambda, G planes) when mat is not null
void launch_max_speed(const Layout& L, const GeoBlock& g, double cs, const double* M, const double* mat,
                      unsigned long long* out, cudaStream_t s);
template <typename T>
void launch_stress_roundtrip(const Layout& L, T* F, const double* S, const double s0[6], cudaStream_t s);
void launch_to_float(const double* a, float* b, long long n, cudaStream_t s);

// arguments of the volume (rate + outer SAT + RK update) kernel
template <typename T>
struct VolumeArgs {
    Layout L;
    int order;
    double cdiss;
    double s0[6];
    const T* F;        // fields at the start of the stage
    T* Fn;             // fields at the end of the stage
    T* DF;             // RK rate register, updated in place
    const T* M;        // metric, [ndim*ndim][cstride]
    const T* J;        // Jacobian
    T* FP;             // plastic-only fields, updated in place on the last stage
    const double* S;   // heterogeneous initial stress or null
    double* ABS;       // absolute-stress staging for output, or null
    int plastic_tensor;
};

// exact-order kernel: one thread per node, reference operation order
template <typename T>
void launch_volume_exact(const VolumeArgs<T>& a, const BlockDev& b, const StageArgs& sa, cudaStream_t s);

// the exact-order kernel over all nb <= FDF_ALLB_MAX blocks in one launch;
// blks_dev is a device copy of the host table blks
constexpr int FDF_ALLB_MAX = 8;
struct BlockRanges {
    long long start[FDF_ALLB_MAX + 1];   // first node of each block in the launch; start[MAX] = total
};
template <typename T>
void launch_volume_exact_all(const VolumeArgs<T>& a, const BlockDev* blks_dev, const BlockDev* blks, int nb,
                             const StageArgs& sa, cudaStream_t s);

// optimised FP32 3D kernel (2.5D tiles marching along x, shared-memory halos)
void launch_volume_fast3d(const VolumeArgs<float>& a, const BlockDev& b, const StageArgs& sa, cudaStream_t s);
bool fast3d_supported(const Layout& L, const BlockDev& b, int order);

// optimised FP32 2D kernel (mode II / mode III elastic; one warp per 32-column
// tile marching along x); plastic or dissipative stages go to the exact kernel
void launch_volume_fast2d(const VolumeArgs<float>& a, const BlockDev& b, const StageArgs& sa, cudaStream_t s);
bool fast2d_supported(const Layout& L, const BlockDev& b, int order);
// staged FP32 3D kernel (planes brought into shared memory by TMA tensor copies)
struct StagedMapsHost;
StagedMapsHost* make_staged_maps(const Layout& L, const float* F0, const float* F1, const float* M, const float* J,
                                 int order);
void free_staged_maps(StagedMapsHost* h);
void launch_volume_staged3d(const VolumeArgs<float>& a, const BlockDev& b, const StageArgs& sa, int* status,
                            const StagedMapsHost* maps, cudaStream_t s);
bool staged3d_supported(const Layout& L, const BlockDev& b, int order);
// register-window FP32 3D kernel (x window in registers, tile planes staged by TMA)
struct RegMapsHost;
// (allocates, per block, the k-face SAT increment buffer of 18 x n0 x n1 floats)
RegMapsHost* make_reg_maps(const Layout& L, const float* F0, const float* F1, const float* M, const float* J,
                           const float* DF, const BlockDev* blocks, int nblocks);
void free_reg_maps(RegMapsHost* h);
void launch_volume_reg3d(const VolumeArgs<float>& a, const BlockDev& b, int bi, const StageArgs& sa, int* status,
                         const RegMapsHost* maps, cudaStream_t s);
bool reg3d_supported(const Layout& L, const BlockDev& b, int order);
// the register-window kernel's pre-passes (k-face SAT increments, closure-plane
// x derivatives) of blocks b0 .. b0+nb-1 (nb <= FDF_ALLB_MAX) in one launch,
// before the blocks' marches; blks_dev is the device copy of the block table
void launch_prepass_reg3d(const VolumeArgs<float>& a, const BlockDev* blks_dev, const BlockDev* blks, int b0,
                          int nb, const StageArgs& sa, const RegMapsHost* maps, cudaStream_t s);
// outer SATs and RK update of the face nodes of a 3D block, after a marching
// kernel wrote their rate without the SAT (kdone: the k-face SATs are already
// in the rate and nodes on k faces only are finished); plastic: the last
// stage's return map too
void launch_faces3d(const VolumeArgs<float>& a, const BlockDev& b, const StageArgs& sa, bool kdone, bool plastic,
                    cudaStream_t s);
// return map of a 3D block's nodes off the x and y faces after a marching
// kernel (kall: nodes on k faces included, except interface faces)
void launch_return_map3(const VolumeArgs<float>& a, const BlockDev& b, const StageArgs& sa, bool kall,
                        cudaStream_t s);

// interface kernels
template <typename T>
struct IfaceArgs {
    Layout L;
    double s0[6];
    const T* F;
    T* Fn;
    T* DF;
    T* FP;
    const double* S;
    double* ABS;
    int plastic_tensor;
    int* status;
    const BlockDev* blocks;   // host copy indices resolved into b1/b2 below
};

template <typename T>
void launch_interface(const IfaceArgs<T>& a, const IfaceDev& itf, const BlockDev& b1, const BlockDev& b2,
                      const StageArgs& sa, int no_sat, cudaStream_t s);

// output helpers
struct OutWindow {   // strided index window of an output unit (global node indices)
    int xm[3], xs[3], n[3];
};
template <typename T>
void launch_gather_window(const Layout& L, const T* F, int comp, int add_stress, const double s0[6], const double* S,
                          const OutWindow& w, double* out, cudaStream_t s);
void launch_gather_fault(const double* arr, long long offset, int n1, int fa, int fb, int base_a, int base_b,
                         const OutWindow& w, double* out, cudaStream_t s);
template <typename T>
void launch_fetch_component(const Layout& L, const T* F, int comp, int add_stress, const double s0[6],
                            const double* S, double* out, cudaStream_t s);
template <typename T>
void launch_store_component(const Layout& L, T* F, int comp, const double* in, cudaStream_t s);
void launch_front(const IfaceDev& itf, double t, double value, cudaStream_t s);
void launch_step_advance(int* step, cudaStream_t s);
// x-slab ghost exchange: ncomp ranges of len elements at c * cstride + off of
// the field buffer to (unpack 0) or from (unpack 1) a contiguous buffer
void launch_ghost_copy(void* field, int elem_bytes, long long cstride, int ncomp, long long off, long long len,
                       void* buf, int unpack, cudaStream_t s);
void launch_set_step(int* step, int value, cudaStream_t s);

}  // namespace fdf
