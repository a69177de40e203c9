#pragma once
// One node of the volume stage in the reference's operation order; used by the
// per-block kernel (stage_exact.cu) and the batched ensemble kernel
// (ensemble.cu).  Both are compiled with -fmad=false.
//
// The node follows, in one pass, the roundings the reference performs across
//   fields::scale_df           src/fields.cpp:293-300
//   block::calc_df_3d          src/block.cpp:1541-2050
//   block::calc_df_mode2/_szz  src/block.cpp:1048-1294
//   block::calc_df_mode3       src/block.cpp:1384-1539
//   boundary::apply_bcs        src/boundary.cpp:265-503
//   fields::update             src/fields.cpp:302-309
#include "kernels.hpp"
#include "sbp_coeffs.cuh"
#include "stage_common.cuh"

namespace fdf {

// HET: the problem has a heterogeneous material (per-node moduli); kept out
// of the common instantiation, whose register budget it would raise
template <typename T, int NDIM, int MODE, bool HET = false>
__device__ __forceinline__ void volume_node(const VolumeArgs<T>& a, const BlockDev& B, const StageArgs& sa,
                                            long long t) {
    const Layout& L = a.L;
    // t counts the nodes of the planes this process updates (xb <= p[0] < xe)
    const long long nn = (long long)(B.xe - B.xb) * B.n[1] * B.n[2];
    if (t >= nn) return;
    int p[3];
    p[2] = (int)(t % B.n[2]);
    p[1] = (int)((t / B.n[2]) % B.n[1]);
    p[0] = B.xb + (int)(t / ((long long)B.n[2] * B.n[1]));
    const long long id = node_index(L, B.lo[0] + p[0], B.lo[1] + p[1], B.lo[2] + p[2]);
    const long long cs = L.cstride;
    const int order = a.order;
    const int nb = 2 * (order - 1);
    constexpr int NF = (NDIM == 3) ? 9 : ((MODE == 2) ? 5 : 3);
    const bool plastic = sa.plastic != 0;
    const int nfd = L.nfields;   // includes szz for mode II plastic
    const T* __restrict__ F = a.F;
    const T* __restrict__ M = a.M;
    const T* __restrict__ J = a.J;
    T df[9];
    const T A = (T)sa.A;
    for (int q = 0; q < nfd; q++) df[q] = a.DF[q * cs + id] * A;
    const long long st[3] = {L.s0, L.s1, L.s2};
    const T cdiss = (T)a.cdiss;
    const T jc = J[id];
    for (int d = 0; d < NDIM; d++) {
        T invrho = (T)B.coef[d][0], g2lam = (T)B.coef[d][1], g = (T)B.coef[d][2], lambda = (T)B.coef[d][3];
        if (HET) {   // per-node material (block.cpp:1061-1065 and the other passes)
            const double rho = B.mat[id], lm = B.mat[cs + id], gg = B.mat[2 * cs + id];
            invrho = (T)(sa.dt / rho / B.dx[d]);
            g2lam = (T)(sa.dt * (2. * gg + lm) / B.dx[d]);
            g = (T)(sa.dt * gg / B.dx[d]);
            lambda = (T)(sa.dt * lm / B.dx[d]);
        }
        const T invjac = invrho / jc;
        const int pp = p[d], n = B.n[d];
        int row, ntap;
        long long base, step;
        bool minus;
        if (pp < nb) {
            row = pp + 1;
            ntap = 3 * (order - 1);
            base = id - (long long)pp * st[d];
            step = st[d];
            minus = false;
        } else if (pp < n - nb) {
            row = 0;
            ntap = 2 * order - 1;
            base = id - (long long)(order - 1) * st[d];
            step = st[d];
            minus = false;
        } else {
            row = n - pp;
            ntap = 3 * (order - 1);
            base = id + (long long)(n - 1 - pp) * st[d];
            step = -st[d];
            minus = true;
        }
        const T* md = M + (long long)(d * NDIM) * cs;
        const T ca = md[id], cb = md[cs + id];
        const T cc = (NDIM == 3) ? md[2 * cs + id] : T(0.);
        for (int m = 0; m < ntap; m++) {
            const long long i2 = base + (long long)m * step;
            const T c = sbp_coef<T>(order, row, m);
            T tv[9];
            if (NDIM == 3) {
                const T ma = md[i2], mb = md[cs + i2], mc = md[2 * cs + i2];
                const T jt = J[i2];
                tv[0] = (invjac * c * jt * (ma * F[3 * cs + i2] + mb * F[4 * cs + i2] + mc * F[5 * cs + i2]));
                tv[1] = (invjac * c * jt * (ma * F[4 * cs + i2] + mb * F[6 * cs + i2] + mc * F[7 * cs + i2]));
                tv[2] = (invjac * c * jt * (ma * F[5 * cs + i2] + mb * F[7 * cs + i2] + mc * F[8 * cs + i2]));
                const T vx = F[i2], vy = F[cs + i2], vz = F[2 * cs + i2];
                tv[3] = c * (g2lam * ca * vx + lambda * (cb * vy + cc * vz));
                tv[4] = c * g * (ca * vy + cb * vx);
                tv[5] = c * g * (ca * vz + cc * vx);
                tv[6] = c * (g2lam * cb * vy + lambda * (ca * vx + cc * vz));
                tv[7] = c * g * (cb * vz + cc * vy);
                tv[8] = c * (g2lam * cc * vz + lambda * (ca * vx + cb * vy));
            } else if (MODE == 2) {
                const T ma = md[i2], mb = md[cs + i2];
                const T jt = J[i2];
                tv[0] = (invjac * c * jt * (ma * F[2 * cs + i2] + mb * F[3 * cs + i2]));
                tv[1] = (invjac * c * jt * (ma * F[3 * cs + i2] + mb * F[4 * cs + i2]));
                const T vx = F[i2], vy = F[cs + i2];
                tv[2] = c * (g2lam * ca * vx + lambda * cb * vy);
                tv[3] = g * c * (ca * vy + cb * vx);
                tv[4] = c * (g2lam * cb * vy + lambda * ca * vx);
            } else {
                const T ma = md[i2], mb = md[cs + i2];
                const T jt = J[i2];
                tv[0] = invjac * c * jt * (ma * F[cs + i2] + mb * F[2 * cs + i2]);
                const T vz = F[i2];
                tv[1] = g * ca * c * vz;
                tv[2] = g * cb * c * vz;
            }
            if (minus) {
#pragma unroll
                for (int q = 0; q < NF; q++) df[q] -= tv[q];
            } else {
#pragma unroll
                for (int q = 0; q < NF; q++) df[q] += tv[q];
            }
            if (cdiss > T(0.)) {
                const T dcf = diss_coef<T>(order, row, m);
                const T jt = J[i2];
#pragma unroll
                for (int q = 0; q < NF; q++) df[q] += cdiss * (dcf * jt * F[q * cs + i2]) / jc;
            }
        }
    }
    if (NDIM == 2 && MODE == 2 && plastic) {
        T nu = (T)B.nu;
        if (HET) {
            // block.cpp:1289-1291 reads lambda at the node and, as its second
            // term, the material array one x row further on (mat[nxd[1] + index]):
            // rho of node (i+1, j), or past the last row lambda of (0, j)
            const int gi = B.lo[0] + p[0], gj = B.lo[1] + p[1], ny = L.nx[1];
            const long long q = (long long)gi * ny + gj + ny, nxy = (long long)L.nx[0] * ny;
            const long long qc = q / nxy, qr = q % nxy;
            const double other = B.mat[qc * cs + node_index(L, (int)(qr / ny), (int)(qr % ny), 0)];
            const double lm = B.mat[cs + id];
            nu = (T)(0.5 * lm / (lm + other));
        }
        df[5] = nu * (df[2] + df[4]);
    }
    // outer-face SATs (block::set_boundaries: faces in order)
    bool defer = false;
    bool onface = false;
    for (int f = 0; f < 2 * NDIM; f++) {
        const int d = f / 2;
        const bool at = (f % 2 == 0) ? (p[d] == 0) : (p[d] == B.n[d] - 1);
        if (!at) continue;
        onface = true;
        if (B.defer[f]) defer = true;
        if (!B.bactive[f]) continue;
        int fa, fb;
        if (d == 0) {
            fa = p[1];
            fb = p[2];
        } else if (d == 1) {
            fa = p[0];
            fb = p[2];
        } else {
            fa = p[0];
            fb = p[1];
        }
        T fv[9];
#pragma unroll
        for (int q = 0; q < NF; q++) fv[q] = F[q * cs + id];
        boundary_sat<T, NDIM, MODE>(B, f, fa, fb, (T)sa.dt, fv, df, plastic, HET ? id : -1);
    }
    (void)onface;
    for (int q = 0; q < nfd; q++) a.DF[q * cs + id] = df[q];
    if (defer) return;
    T fn[9];
    const T Bc = (T)sa.B;
    for (int q = 0; q < nfd; q++) fn[q] = F[q * cs + id] + Bc * df[q];
    finish_node<T>(L, B, sa, a.s0, a.S, a.ABS, a.FP, a.plastic_tensor, id, fn, false);
    for (int q = 0; q < nfd; q++) a.Fn[q * cs + id] = fn[q];
}


}  // namespace fdf
