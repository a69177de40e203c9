// Device set-up of the curvilinear grid, in FP64 with the reference's
// operation order (this file is compiled with -fmad=false, so every product
// and sum rounds exactly as in the reference's x86-64 build):
//  - transfinite interpolation of the block's bounding surfaces
//    (src/block.cpp:795-829);
//  - SBP derivatives of the coordinates, Jacobian and metric
//    (src/block.cpp:831-1014);
//  - outer-face and interface unit normals and SAT grid factors
//    (src/boundary.cpp:173-240, src/interface.cpp:414-534);
//  - the CFL length scale min(dx/cs) (src/block.cpp:368-403);
//  - the absolute-stress add/subtract replay applied after every write of the
//    output list (src/fields.cpp:184-220, src/problem.cpp:74-78).
#include <cuda_runtime.h>

#include "fdf_types.hpp"
#include "kernels.hpp"
#include "sbp_coeffs.cuh"

namespace fdf {

namespace {

__device__ __forceinline__ long long nidx(const Layout& L, int i, int j, int k) {
    return (long long)i * L.s0 + (long long)j * L.s1 + (long long)k * L.s2;
}

__device__ __forceinline__ double surf_x(const GeoBlock& g, int f, int c, int a, int b) {
    return g.surf[f][((long long)c * g.sn0[f] + a) * g.sn1[f] + b];
}

__global__ void k_transfinite(Layout L, GeoBlock g, double* __restrict__ X) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long nn = (long long)g.n[0] * g.n[1] * g.n[2];
    if (t >= nn) return;
    int ll = (int)(t % g.n[2]);
    int kk = (int)((t / g.n[2]) % g.n[1]);
    int jj = (int)(t / ((long long)g.n[2] * g.n[1]));
    const int ny = g.n[1], nz = g.n[2];
    double p = (double)jj * g.dx[0];
    double q = (double)kk * g.dx[1];
    double r = (double)ll * g.dx[2];
    long long id = nidx(L, g.lo[0] + jj, g.lo[1] + kk, g.lo[2] + ll);
    for (int i = 0; i < L.ndim; i++) {
        double x = ((1. - p) * surf_x(g, 0, i, kk, ll) + p * surf_x(g, 1, i, kk, ll) +
                    (1. - q) * surf_x(g, 2, i, jj, ll) + q * surf_x(g, 3, i, jj, ll));
        if (L.ndim == 3) x += (1. - r) * surf_x(g, 4, i, jj, kk) + r * surf_x(g, 5, i, jj, kk);
        x -= ((1. - q) * (1. - p) * surf_x(g, 0, i, 0, ll) + (1. - q) * p * surf_x(g, 1, i, 0, ll) +
              q * (1. - p) * surf_x(g, 0, i, ny - 1, ll) + q * p * surf_x(g, 1, i, ny - 1, ll));
        if (L.ndim == 3) {
            x -= ((1. - p) * (1. - r) * surf_x(g, 0, i, kk, 0) + p * (1. - r) * surf_x(g, 1, i, kk, 0) +
                  (1. - q) * (1. - r) * surf_x(g, 2, i, jj, 0) + q * (1. - r) * surf_x(g, 3, i, jj, 0) +
                  (1. - p) * r * surf_x(g, 0, i, kk, nz - 1) + p * r * surf_x(g, 1, i, kk, nz - 1) +
                  (1. - q) * r * surf_x(g, 2, i, jj, nz - 1) + q * r * surf_x(g, 3, i, jj, nz - 1));
            x += ((1. - p) * (1. - q) * (1. - r) * surf_x(g, 0, i, 0, 0) +
                  p * (1. - q) * (1. - r) * surf_x(g, 1, i, 0, 0) +
                  (1. - p) * q * (1. - r) * surf_x(g, 0, i, ny - 1, 0) +
                  (1. - p) * (1. - q) * r * surf_x(g, 0, i, 0, nz - 1) +
                  p * q * (1. - r) * surf_x(g, 1, i, ny - 1, 0) +
                  p * (1. - q) * r * surf_x(g, 1, i, 0, nz - 1) +
                  (1. - p) * q * r * surf_x(g, 0, i, ny - 1, nz - 1) +
                  p * q * r * surf_x(g, 1, i, ny - 1, nz - 1));
        }
        X[i * L.cstride + id] = x;
    }
}

// xp[l][d] = d x_l / d xi_d by the SBP operator, then Jacobian and metric
__global__ void k_metrics(Layout L, GeoBlock g, int order, const double* __restrict__ X,
                          double* __restrict__ M, double* __restrict__ J, int* __restrict__ status) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long nn = (long long)g.n[0] * g.n[1] * g.n[2];
    if (t >= nn) return;
    int pos[3];
    pos[2] = (int)(t % g.n[2]);
    pos[1] = (int)((t / g.n[2]) % g.n[1]);
    pos[0] = (int)(t / ((long long)g.n[2] * g.n[1]));
    const int nb = 2 * (order - 1);
    double xp[3][3];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) xp[a][b] = (a == b) ? 1. : 0.;
    long long id = nidx(L, g.lo[0] + pos[0], g.lo[1] + pos[1], g.lo[2] + pos[2]);
    const long long st[3] = {L.s0, L.s1, L.s2};
    for (int d = 0; d < L.ndim; d++) {
        const int p = pos[d], n = g.n[d];
        for (int l = 0; l < L.ndim; l++) {
            const double* Xl = X + l * L.cstride;
            double acc = 0.;
            if (p < nb) {
                long long base = id - (long long)p * st[d];
                for (int m = 0; m < 3 * (order - 1); m++)
                    acc += sbp_coef<double>(order, p + 1, m) * Xl[base + m * st[d]] / g.dx[d];
            } else if (p < n - nb) {
                long long base = id - (long long)(order - 1) * st[d];
                for (int m = 0; m < 2 * order - 1; m++)
                    acc += sbp_coef<double>(order, 0, m) * Xl[base + m * st[d]] / g.dx[d];
            } else {
                long long base = id + (long long)(n - 1 - p) * st[d];
                for (int m = 0; m < 3 * (order - 1); m++)
                    acc -= sbp_coef<double>(order, n - p, m) * Xl[base - m * st[d]] / g.dx[d];
            }
            xp[l][d] = acc;
        }
    }
    double jac = (xp[0][0] * (xp[1][1] * xp[2][2] - xp[1][2] * xp[2][1]) -
                  xp[1][0] * (xp[0][1] * xp[2][2] - xp[0][2] * xp[2][1]) +
                  xp[2][0] * (xp[0][1] * xp[1][2] - xp[0][2] * xp[1][1]));
    J[id] = jac;
    if (!(jac > 0.)) atomicOr(status, (int)FDF_ERR_JACOBIAN);
    for (int l = 0; l < L.ndim; l++)
        for (int m = 0; m < L.ndim; m++)
            M[(l * L.ndim + m) * L.cstride + id] =
                ((xp[(m + 1) % 3][(l + 1) % 3] * xp[(m + 2) % 3][(l + 2) % 3] -
                  xp[(m + 1) % 3][(l + 2) % 3] * xp[(m + 2) % 3][(l + 1) % 3]) /
                 jac);
}

// unit normal and grid factor on a face of constant xi_d at global index `at`
__global__ void k_face_normals(Layout L, int d, int at, int lo0, int n0, int lo1, int n1, int flip, double h0dx,
                               const double* __restrict__ M, double* __restrict__ nx0, double* __restrict__ nx1,
                               double* __restrict__ nx2, double* __restrict__ dl, double* __restrict__ dl2,
                               int at2, double h0dx2) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n0 * n1) return;
    int a = t / n1, b = t % n1;
    int pos[3];
    int o0 = (d == 0) ? 1 : 0, o1 = (d == 2) ? 1 : 2;
    pos[d] = at;
    pos[o0] = lo0 + a;
    pos[o1] = lo1 + b;
    long long id = nidx(L, pos[0], pos[1], pos[2]);
    double* nxp[3] = {nx0, nx1, nx2};
    double s = 0., v[3];
    for (int k = 0; k < L.ndim; k++) {
        double m = M[(d * L.ndim + k) * L.cstride + id];
        s += m * m;
        v[k] = m;
    }
    s = sqrt(s);
    for (int k = 0; k < L.ndim; k++) {
        double w = v[k] / s;
        nxp[k][t] = flip ? -w : w;
    }
    dl[t] = s / h0dx;
    if (dl2) {
        pos[d] = at2;
        long long id2 = nidx(L, pos[0], pos[1], pos[2]);
        double s2 = 0.;
        for (int k = 0; k < L.ndim; k++) {
            double m = M[(d * L.ndim + k) * L.cstride + id2];
            s2 += m * m;
        }
        s2 = sqrt(s2);
        dl2[t] = s2 / h0dx2;
    }
}

__global__ void k_max_speed(Layout L, GeoBlock g, double cs, const double* __restrict__ M,
                            const double* __restrict__ mat, unsigned long long* __restrict__ out) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long nn = (long long)g.n[0] * g.n[1] * g.n[2];
    double best = 0.;
    if (t < nn) {
        int k = (int)(t % g.n[2]);
        int j = (int)((t / g.n[2]) % g.n[1]);
        int i = (int)(t / ((long long)g.n[2] * g.n[1]));
        long long id = nidx(L, g.lo[0] + i, g.lo[1] + j, g.lo[2] + k);
        if (mat) cs = sqrt(mat[2 * L.cstride + id] / mat[id]);   // block.cpp:387-388
        for (int l = 0; l < L.ndim; l++) {
            double s = 0.;
            for (int m = 0; m < L.ndim; m++) {
                double v = M[(l * L.ndim + m) * L.cstride + id];
                s += v * v;
            }
            s = cs * sqrt(s) / g.dx[l];
            if (s > best) best = s;
        }
    }
    // max of non-negative doubles == max of their bit patterns
    unsigned long long bits = (unsigned long long)__double_as_longlong(best);
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long w = __shfl_down_sync(0xffffffffu, bits, o);
        bits = w > bits ? w : bits;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(out, bits);
}

template <typename T>
__global__ void k_stress_roundtrip(Layout L, int n0, int n1, int n2, T* __restrict__ F, const double* __restrict__ S,
                                   double s00, double s01, double s02, double s03, double s04, double s05) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long nn = (long long)n0 * n1 * n2;
    if (t >= nn) return;
    int k = (int)(t % n2);
    int j = (int)((t / n2) % n1);
    int i = (int)(t / ((long long)n2 * n1));
    long long id = nidx(L, i, j, k);
    const double s0[6] = {s00, s01, s02, s03, s04, s05};
    for (int c = 0; c < L.ns; c++) {
        T* p = F + (L.nv + c) * L.cstride + id;
        double v = (double)*p;
        v += s0[L.sidx[c]];
        if (S) v += S[c * L.cstride + id];
        v -= s0[L.sidx[c]];
        if (S) v -= S[c * L.cstride + id];
        *p = (T)v;
    }
}

__global__ void k_to_float(const double* __restrict__ a, float* __restrict__ b, long long n) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t < n) b[t] = (float)a[t];
}

inline unsigned nblk(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

void launch_transfinite(const Layout& L, const GeoBlock& g, double* X, cudaStream_t s) {
    long long nn = (long long)g.n[0] * g.n[1] * g.n[2];
    k_transfinite<<<nblk(nn, 256), 256, 0, s>>>(L, g, X);
}

void launch_metrics(const Layout& L, const GeoBlock& g, int order, const double* X, double* M, double* J, int* status,
                    cudaStream_t s) {
    long long nn = (long long)g.n[0] * g.n[1] * g.n[2];
    k_metrics<<<nblk(nn, 128), 128, 0, s>>>(L, g, order, X, M, J, status);
}

void launch_face_normals(const Layout& L, int d, int at, int lo0, int n0, int lo1, int n1, int flip, double h0dx,
                         const double* M, double* nx[3], double* dl, double* dl2, int at2, double h0dx2,
                         cudaStream_t s) {
    k_face_normals<<<nblk((long long)n0 * n1, 256), 256, 0, s>>>(L, d, at, lo0, n0, lo1, n1, flip, h0dx, M, nx[0],
                                                                 nx[1], nx[2], dl, dl2, at2, h0dx2);
}

void launch_max_speed(const Layout& L, const GeoBlock& g, double cs, const double* M, const double* mat,
                      unsigned long long* out, cudaStream_t s) {
    long long nn = (long long)g.n[0] * g.n[1] * g.n[2];
    k_max_speed<<<nblk(nn, 256), 256, 0, s>>>(L, g, cs, M, mat, out);
}

template <typename T>
void launch_stress_roundtrip(const Layout& L, T* F, const double* S, const double s0[6], cudaStream_t s) {
    long long nn = (long long)L.nx[0] * L.nx[1] * L.nx[2];
    k_stress_roundtrip<T><<<nblk(nn, 256), 256, 0, s>>>(L, L.nx[0], L.nx[1], L.nx[2], F, S, s0[0], s0[1], s0[2], s0[3],
                                                        s0[4], s0[5]);
}
template void launch_stress_roundtrip<double>(const Layout&, double*, const double*, const double*, cudaStream_t);
template void launch_stress_roundtrip<float>(const Layout&, float*, const double*, const double*, cudaStream_t);

void launch_to_float(const double* a, float* b, long long n, cudaStream_t s) {
    k_to_float<<<nblk(n, 256), 256, 0, s>>>(a, b, n);
}

}  // namespace fdf
