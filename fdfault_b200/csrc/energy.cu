// FP64 energy diagnostics of the elastic fields, in the discrete norm of the
// SBP operator.
//
// The reference's operator (src/fd.cpp:33-155) is summation-by-parts with a
// diagonal norm H: H D + D^T H = diag(-1, 0, ..., 0, 1).  The reference keeps
// only its first entry h0 (src/fd.cpp:119-120); the others follow from the
// SBP property row by row (h_i D_i0 = -h0 D_0i), and for the three orders are
// the rationals in norm_weights() below.  The discrete energy of a block is
//   E = sum_nodes  w_ijk J_ijk ( 1/2 rho |v|^2  +  1/2 sigma : S : sigma ),
//   w_ijk = H_i H_j H_k dxi dxeta dzeta,
// S the isotropic compliance of the node's material (plane strain: sigma_zz = nu (sigma_xx + sigma_yy);
// antiplane: sigma_xz and sigma_yz only), J the Jacobian of the block's map.
// Its rate under the semi-discrete operator L (volume terms, outer SATs and
// interface conditions together) is
//   dE/dt = sum_nodes w J ( rho v . L_v(f) + sigma : S : L_sigma(f) ),
// which the SBP property makes a sum of face terms; outer SATs and the
// interfaces can only remove energy (frictional slip, absorbed waves, and
// the penalty on any violation of a boundary condition).  Every sum is
// accumulated in FP64 on the device, whatever the precision of the fields.
#include <cuda_runtime.h>

#include "energy.hpp"
#include "stage_common.cuh"

namespace fdf {

void norm_weights(int order, double h[8], int* nb) {
    for (int i = 0; i < 8; i++) h[i] = 1.;
    if (order == 2) {
        h[0] = 0.5;
        *nb = 1;
    } else if (order == 3) {
        const double w[4] = {17. / 48., 59. / 48., 43. / 48., 49. / 48.};
        for (int i = 0; i < 4; i++) h[i] = w[i];
        *nb = 4;
    } else {
        const double w[6] = {13649. / 43200., 12013. / 8640., 2711. / 4320.,
                             5359. / 4320.,   7877. / 8640.,  43801. / 43200.};
        for (int i = 0; i < 6; i++) h[i] = w[i];
        *nb = 6;
    }
}

namespace {

struct NormW {
    double h[8];
    int nb;
};

__device__ __forceinline__ double hw(const NormW& W, int i, int n) {
    if (i < W.nb) return W.h[i];
    if (i >= n - W.nb) return W.h[n - 1 - i];
    return 1.;
}

// strain energy density 1/2 sigma : S : sigma (3D stress components) and its
// derivative sigma : S : r along the stress rate r
__device__ __forceinline__ void strain_terms(double lam, double g, const double s[6], const double r[6], double* w,
                                             double* wr) {
    // S sigma = (sigma - lam / (3 lam + 2 g) tr(sigma) I) / (2 g); components xx, xy, xz, yy, yz, zz
    const double c = lam / (3. * lam + 2. * g);
    const double trs = s[0] + s[3] + s[5], trr = r[0] + r[3] + r[5];
    const double ss = s[0] * s[0] + s[3] * s[3] + s[5] * s[5] + 2. * (s[1] * s[1] + s[2] * s[2] + s[4] * s[4]);
    const double sr = s[0] * r[0] + s[3] * r[3] + s[5] * r[5] + 2. * (s[1] * r[1] + s[2] * r[2] + s[4] * r[4]);
    *w = 0.25 / g * (ss - c * trs * trs);
    *wr = 0.5 / g * (sr - c * trs * trr);
}

template <typename T>
__global__ void __launch_bounds__(256) k_energy(EnergyArgs<T> a, BlockDev B, NormW W, double* out) {
    const Layout& L = a.L;
    const int n0 = B.n[0], n1 = B.n[1], n2 = (L.ndim == 3) ? B.n[2] : 1;
    const long long total = (long long)n0 * n1 * n2;
    const long long cs = L.cstride;
    double ek = 0., es = 0., er = 0., scale = 0.;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % n2), j = (int)((t / n2) % n1), i = (int)(t / ((long long)n2 * n1));
        if (i < B.xb || i >= B.xe) continue;   // plane summed by the process that updates it
        const long long id = (L.ndim == 3) ? node_index(L, B.lo[0] + i, B.lo[1] + j, B.lo[2] + k)
                                           : node_index(L, B.lo[0] + i, B.lo[1] + j, 0);
        double w = hw(W, i, n0) * hw(W, j, n1) * B.dx[0] * B.dx[1] * (double)a.J[id];
        if (L.ndim == 3) w *= hw(W, k, n2) * B.dx[2];
        double rho = B.rho, lam = B.lam, g = B.g;
        if (B.mat) {   // heterogeneous material
            rho = B.mat[id];
            lam = B.mat[B.matstride + id];
            g = B.mat[2 * B.matstride + id];
        }
        double v[3] = {0., 0., 0.}, rv[3] = {0., 0., 0.}, s[6] = {0., 0., 0., 0., 0., 0.}, rs[6] = {0., 0., 0., 0., 0., 0.};
        auto f = [&](int c) { return (double)a.F[c * cs + id]; };
        auto d = [&](int c) { return a.R ? (double)a.R[c * cs + id] : 0.; };
        if (L.ndim == 3) {
            for (int c = 0; c < 3; c++) {
                v[c] = f(c);
                rv[c] = d(c);
            }
            for (int c = 0; c < 6; c++) {
                s[c] = f(3 + c);
                rs[c] = d(3 + c);
            }
        } else if (L.mode == 2) {   // vx, vy, sxx, sxy, syy; plane strain
            v[0] = f(0), v[1] = f(1), rv[0] = d(0), rv[1] = d(1);
            s[0] = f(2), s[1] = f(3), s[3] = f(4);
            rs[0] = d(2), rs[1] = d(3), rs[3] = d(4);
            const double nu = 0.5 * lam / (lam + g);
            s[5] = nu * (s[0] + s[3]);
            rs[5] = nu * (rs[0] + rs[3]);
        } else {   // mode III: vz, sxz, syz
            v[2] = f(0), rv[2] = d(0);
            s[2] = f(1), s[4] = f(2);
            rs[2] = d(1), rs[4] = d(2);
        }
        const double kin = 0.5 * rho * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        const double kr = rho * (v[0] * rv[0] + v[1] * rv[1] + v[2] * rv[2]);
        double ws, wr;
        strain_terms(lam, g, s, rs, &ws, &wr);
        ek += w * kin;
        es += w * ws;
        er += w * (kr + wr);
        scale += w * (fabs(kr) + fabs(wr));
    }
    for (int o = 16; o > 0; o >>= 1) {
        ek += __shfl_xor_sync(0xffffffffu, ek, o);
        es += __shfl_xor_sync(0xffffffffu, es, o);
        er += __shfl_xor_sync(0xffffffffu, er, o);
        scale += __shfl_xor_sync(0xffffffffu, scale, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out + 0, ek);
        atomicAdd(out + 1, es);
        atomicAdd(out + 2, er);
        atomicAdd(out + 3, scale);
    }
}

// frictional power on one interface: sum over its nodes of the face area
// element (minus side) times traction . slip rate
template <typename T>
__global__ void __launch_bounds__(256) k_fault_power(Layout L, IfaceDev I, BlockDev B1, NormW W, const T* J,
                                                     const T* M, double* out) {
    const int nf = I.n0 * I.n1;
    const int D = I.direction;
    const int o0 = (D == 0) ? 1 : 0, o1 = (D == 2) ? 1 : 2;
    double p = 0.;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nf; t += gridDim.x * blockDim.x) {
        const int a = t / I.n1, b = t % I.n1;
        int g[3] = {I.mlb[0], I.mlb[1], I.mlb[2]};
        g[o0] += a;
        if (L.ndim == 3) g[o1] += b;
        if (g[0] - B1.lo[0] < B1.xb || g[0] - B1.lo[0] >= B1.xe) continue;   // another process's plane
        const long long id = (L.ndim == 3) ? node_index(L, g[0], g[1], g[2]) : node_index(L, g[0], g[1], 0);
        double gn = 0.;
        for (int m = 0; m < L.ndim; m++) {
            const double q = (double)M[(D * L.ndim + m) * L.cstride + id];
            gn += q * q;
        }
        double w = (double)J[id] * sqrt(gn) * hw(W, a, B1.n[o0]) * B1.dx[o0];
        if (L.ndim == 3) w *= hw(W, b, B1.n[o1]) * B1.dx[o1];
        double sv = 0.;
        for (int c = 0; c < L.ndim - 1; c++) sv += I.sx[c * nf + t] * I.vx[c * nf + t];
        p += w * sv;
    }
    for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, p);
}

}  // namespace

template <typename T>
void launch_energy(const EnergyArgs<T>& a, const BlockDev& b, int order, double* out, cudaStream_t s) {
    NormW W;
    norm_weights(order, W.h, &W.nb);
    const long long n = (long long)b.n[0] * b.n[1] * (a.L.ndim == 3 ? b.n[2] : 1);
    long long grid = (n + 255) / 256;
    if (grid > 4096) grid = 4096;
    k_energy<T><<<(unsigned)grid, 256, 0, s>>>(a, b, W, out);
}

template void launch_energy<float>(const EnergyArgs<float>&, const BlockDev&, int, double*, cudaStream_t);
template void launch_energy<double>(const EnergyArgs<double>&, const BlockDev&, int, double*, cudaStream_t);

template <typename T>
void launch_fault_power(const Layout& L, const IfaceDev& I, const BlockDev& b1, int order, const T* J, const T* M,
                        double* out, cudaStream_t s) {
    NormW W;
    norm_weights(order, W.h, &W.nb);
    const int nf = I.n0 * I.n1;
    int grid = (nf + 255) / 256;
    if (grid > 1024) grid = 1024;
    k_fault_power<T><<<grid, 256, 0, s>>>(L, I, b1, W, J, M, out);
}

template void launch_fault_power<float>(const Layout&, const IfaceDev&, const BlockDev&, int, const float*,
                                        const float*, double*, cudaStream_t);
template void launch_fault_power<double>(const Layout&, const IfaceDev&, const BlockDev&, int, const double*,
                                         const double*, double*, cudaStream_t);

}  // namespace fdf
