// FP64 energy diagnostics of the elastic fields (energy.cu).
#pragma once

#include <cuda_runtime.h>

#include "fdf_types.hpp"

namespace fdf {

// diagonal SBP norm weights of the boundary rows (h[0..nb-1]; 1 elsewhere)
void norm_weights(int order, double h[8], int* nb);

template <typename T>
struct EnergyArgs {
    Layout L;
    const T* F;        // fields
    const T* R;        // rates L(f), or null
    const T* J;        // Jacobian
};

// adds kinetic energy, strain energy, their rate along R and the sum of the
// rate terms' magnitudes over block b to out[0..3]
template <typename T>
void launch_energy(const EnergyArgs<T>& a, const BlockDev& b, int order, double* out, cudaStream_t s);
// adds the frictional power (face area element x traction . slip rate) of
// interface I to out[0]; J, M the Jacobian and metric
template <typename T>
void launch_fault_power(const Layout& L, const IfaceDev& I, const BlockDev& b1, int order, const T* J, const T* M,
                        double* out, cudaStream_t s);

}  // namespace fdf
