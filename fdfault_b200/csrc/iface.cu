// Interface kernel: one thread per fault node (compiled with -fmad=false so
// the FP64 arithmetic rounds as the reference's does).  Per node and stage it
// performs, in the reference's order,
//   friction::scale_df                      src/friction.cpp:444-463
//   interface::apply_bcs (incl. SAT)        src/interface.cpp:573-970
//     interface::solve_interface (locked)   src/interface.cpp:972-1028
//     friction::solve_interface/_friction   src/friction.cpp:259-398
//     friction::solve_fs / slipweak / stz   src/friction.cpp:400-442,
//                                           src/slipweak.cpp:206-308,
//                                           src/stz.cpp:263-356
//     solve_newton (bracketed Newton)       src/utilities.cpp:89-179
//   friction::calc_df, friction::update     src/friction.cpp:465-505
// and then finishes the RK update of the two fault-plane nodes (the volume
// kernel leaves those to this kernel).  Fault-plane parameters that the
// reference recomputes from parametric perturbations every stage
// (src/pert.cpp:45-136) use precomputed spatial shapes times the same
// scalar value and time ramp, which rounds identically.
#include <cuda_runtime.h>

#include "iface_dev.cuh"

namespace fdf {

namespace {

// five 128-thread CTAs per SM (at most 96 registers, some spilled): the
// 80,601 nodes of a 401 x 201 fault fit in one wave (at 128 registers four
// CTAs per SM left 38 CTAs to a second wave: 66 against 43 us per stage)
template <typename T, bool LEARN>
__global__ void __launch_bounds__(128, 5) k_interface(IfaceArgs<T> a, IfaceDev I, BlockDev B1, BlockDev B2, StageArgs sa,
                                                   int no_sat) {
    interface_node<T, LEARN>(a, I, B1, B2, sa, no_sat, blockIdx.x * (long long)blockDim.x + threadIdx.x);
}

template <typename T>
__global__ void k_fetch(Layout L, const T* __restrict__ F, int comp, int add_stress, double s0v,
                        const double* __restrict__ S, int scomp, double* __restrict__ out) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long nn = (long long)L.nx[0] * L.nx[1] * L.nx[2];
    if (t >= nn) return;
    int k = (int)(t % L.nx[2]);
    int j = (int)((t / L.nx[2]) % L.nx[1]);
    int i = (int)(t / ((long long)L.nx[2] * L.nx[1]));
    long long id = node_index(L, i, j, k);
    double v = (double)F[comp * L.cstride + id];
    if (add_stress) {
        v += s0v;
        if (S) v += S[scomp * L.cstride + id];
    }
    out[t] = v;
}

// one output unit's window of a field component: out[(a*ny + b)*nz + c] =
// F at node (xm0 + a xs0, xm1 + b xs1, xm2 + c xs2), plus the initial stress
// when add_stress (the same conversion as k_fetch)
template <typename T>
__global__ void k_gather_window(Layout L, const T* __restrict__ F, int comp, int add_stress, double s0v,
                                const double* __restrict__ S, int scomp, OutWindow w, double* __restrict__ out) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long nn = (long long)w.n[0] * w.n[1] * w.n[2];
    if (t >= nn) return;
    const int c = (int)(t % w.n[2]), b = (int)((t / w.n[2]) % w.n[1]), a = (int)(t / ((long long)w.n[2] * w.n[1]));
    const long long id = node_index(L, w.xm[0] + a * w.xs[0], w.xm[1] + b * w.xs[1], w.xm[2] + c * w.xs[2]);
    double v = (double)F[comp * L.cstride + id];
    if (add_stress) {
        v += s0v;
        if (S) v += S[scomp * L.cstride + id];
    }
    out[t] = v;
}

// one output unit's window of a fault array (face node (p_a, p_b) at
// offset + (p_a - base_a) * n1 + (p_b - base_b))
__global__ void k_gather_fault(const double* __restrict__ arr, long long offset, int n1, int fa, int fb, int base_a,
                               int base_b, OutWindow w, double* __restrict__ out) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long nn = (long long)w.n[0] * w.n[1] * w.n[2];
    if (t >= nn) return;
    const int c = (int)(t % w.n[2]), b = (int)((t / w.n[2]) % w.n[1]), a = (int)(t / ((long long)w.n[2] * w.n[1]));
    const int pos[3] = {w.xm[0] + a * w.xs[0], w.xm[1] + b * w.xs[1], w.xm[2] + c * w.xs[2]};
    out[t] = arr[offset + (long long)(pos[fa] - base_a) * n1 + (pos[fb] - base_b)];
}

template <typename T>
__global__ void k_store(Layout L, T* __restrict__ F, int comp, const double* __restrict__ in) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long nn = (long long)L.nx[0] * L.nx[1] * L.nx[2];
    if (t >= nn) return;
    int k = (int)(t % L.nx[2]);
    int j = (int)((t / L.nx[2]) % L.nx[1]);
    int i = (int)(t / ((long long)L.nx[2] * L.nx[1]));
    F[comp * L.cstride + node_index(L, i, j, k)] = (T)in[t];
}

__global__ void k_front(IfaceDev I, double t, double value) {
    long long ij = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (ij >= (long long)I.n0 * I.n1) return;
    if (I.tfront[ij] < 0. && I.v[ij] >= value) I.tfront[ij] = t;
}

}  // namespace

__global__ void k_step_advance(int* step) { *step += 1; }
__global__ void k_set_step(int* step, int value) { *step = value; }

void launch_step_advance(int* step, cudaStream_t s) { k_step_advance<<<1, 1, 0, s>>>(step); }
void launch_set_step(int* step, int value, cudaStream_t s) { k_set_step<<<1, 1, 0, s>>>(step, value); }

template <typename T>
void launch_interface(const IfaceArgs<T>& a, const IfaceDev& itf, const BlockDev& b1, const BlockDev& b2,
                      const StageArgs& sa, int no_sat, cudaStream_t s) {
    long long nn = (long long)itf.n0 * itf.n1;
    const unsigned nb = (unsigned)((nn + 127) / 128);
    if (itf.kind == 3 && itf.stz.learned)
        k_interface<T, true><<<nb, 128, 0, s>>>(a, itf, b1, b2, sa, no_sat);
    else
        k_interface<T, false><<<nb, 128, 0, s>>>(a, itf, b1, b2, sa, no_sat);
}
template void launch_interface<double>(const IfaceArgs<double>&, const IfaceDev&, const BlockDev&, const BlockDev&,
                                       const StageArgs&, int, cudaStream_t);
template void launch_interface<float>(const IfaceArgs<float>&, const IfaceDev&, const BlockDev&, const BlockDev&,
                                      const StageArgs&, int, cudaStream_t);

template <typename T>
void launch_fetch_component(const Layout& L, const T* F, int comp, int add_stress, const double s0[6],
                            const double* S, double* out, cudaStream_t s) {
    long long nn = (long long)L.nx[0] * L.nx[1] * L.nx[2];
    int sc = comp - L.nv;
    double s0v = (add_stress && sc >= 0 && sc < L.ns) ? s0[L.sidx[sc]] : 0.;
    int add = add_stress && sc >= 0 && sc < L.ns;
    k_fetch<T><<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(L, F, comp, add, s0v, add ? S : nullptr, sc, out);
}
template void launch_fetch_component<double>(const Layout&, const double*, int, int, const double*, const double*,
                                             double*, cudaStream_t);
template void launch_fetch_component<float>(const Layout&, const float*, int, int, const double*, const double*,
                                            double*, cudaStream_t);

template <typename T>
void launch_gather_window(const Layout& L, const T* F, int comp, int add_stress, const double s0[6], const double* S,
                          const OutWindow& w, double* out, cudaStream_t s) {
    const long long nn = (long long)w.n[0] * w.n[1] * w.n[2];
    int sc = comp - L.nv;
    double s0v = (add_stress && sc >= 0 && sc < L.ns) ? s0[L.sidx[sc]] : 0.;
    int add = add_stress && sc >= 0 && sc < L.ns;
    k_gather_window<T><<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(L, F, comp, add, s0v, add ? S : nullptr, sc, w,
                                                                      out);
}
template void launch_gather_window<double>(const Layout&, const double*, int, int, const double*, const double*,
                                           const OutWindow&, double*, cudaStream_t);
template void launch_gather_window<float>(const Layout&, const float*, int, int, const double*, const double*,
                                          const OutWindow&, double*, cudaStream_t);

void launch_gather_fault(const double* arr, long long offset, int n1, int fa, int fb, int base_a, int base_b,
                         const OutWindow& w, double* out, cudaStream_t s) {
    const long long nn = (long long)w.n[0] * w.n[1] * w.n[2];
    k_gather_fault<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(arr, offset, n1, fa, fb, base_a, base_b, w, out);
}

template <typename T>
void launch_store_component(const Layout& L, T* F, int comp, const double* in, cudaStream_t s) {
    long long nn = (long long)L.nx[0] * L.nx[1] * L.nx[2];
    k_store<T><<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(L, F, comp, in);
}
template void launch_store_component<double>(const Layout&, double*, int, const double*, cudaStream_t);
template void launch_store_component<float>(const Layout&, float*, int, const double*, cudaStream_t);

void launch_front(const IfaceDev& itf, double t, double value, cudaStream_t s) {
    long long nn = (long long)itf.n0 * itf.n1;
    k_front<<<(unsigned)((nn + 127) / 128), 128, 0, s>>>(itf, t, value);
}

}  // namespace fdf
