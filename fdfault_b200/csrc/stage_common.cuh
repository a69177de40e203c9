// Device helpers shared by the stage kernels: node indexing, the outer
// boundary SAT (src/boundary.cpp:265-568), the Drucker-Prager return map
// (src/block.cpp:591-697) and the end-of-stage update with the reference's
// absolute-stress bookkeeping (src/domain.cpp:269-299, src/problem.cpp:160-164,
// src/fields.cpp:184-220).  Arithmetic follows the reference's operation
// order; files that need bit-exact FP64 results compile with -fmad=false.
#pragma once

#include "fdf_types.hpp"
#include "kernels.hpp"

namespace fdf {

__device__ __forceinline__ long long node_index(const Layout& L, int i, int j, int k) {
    return (long long)i * L.s0 + (long long)j * L.s1 + (long long)k * L.s2;
}

template <typename T>
struct BF {
    T v1, v2, v3, s11, s12, s13, s22, s23, s33;
};

template <typename T>
__device__ __forceinline__ BF<T> rot_xy_nt(const BF<T>& b, const T nn[3], const T t1[3], const T t2[3]) {
    BF<T> o;
    o.v1 = nn[0] * b.v1 + nn[1] * b.v2 + nn[2] * b.v3;
    o.v2 = t1[0] * b.v1 + t1[1] * b.v2 + t1[2] * b.v3;
    o.v3 = t2[0] * b.v1 + t2[1] * b.v2 + t2[2] * b.v3;
    o.s11 = (nn[0] * (b.s11 * nn[0] + b.s12 * nn[1] + b.s13 * nn[2]) + nn[1] * (b.s12 * nn[0] + b.s22 * nn[1] + b.s23 * nn[2]) +
             nn[2] * (b.s13 * nn[0] + b.s23 * nn[1] + b.s33 * nn[2]));
    o.s12 = (nn[0] * (b.s11 * t1[0] + b.s12 * t1[1] + b.s13 * t1[2]) + nn[1] * (b.s12 * t1[0] + b.s22 * t1[1] + b.s23 * t1[2]) +
             nn[2] * (b.s13 * t1[0] + b.s23 * t1[1] + b.s33 * t1[2]));
    o.s13 = (nn[0] * (b.s11 * t2[0] + b.s12 * t2[1] + b.s13 * t2[2]) + nn[1] * (b.s12 * t2[0] + b.s22 * t2[1] + b.s23 * t2[2]) +
             nn[2] * (b.s13 * t2[0] + b.s23 * t2[1] + b.s33 * t2[2]));
    o.s22 = (t1[0] * (b.s11 * t1[0] + b.s12 * t1[1] + b.s13 * t1[2]) + t1[1] * (b.s12 * t1[0] + b.s22 * t1[1] + b.s23 * t1[2]) +
             t1[2] * (b.s13 * t1[0] + b.s23 * t1[1] + b.s33 * t1[2]));
    o.s23 = (t1[0] * (b.s11 * t2[0] + b.s12 * t2[1] + b.s13 * t2[2]) + t1[1] * (b.s12 * t2[0] + b.s22 * t2[1] + b.s23 * t2[2]) +
             t1[2] * (b.s13 * t2[0] + b.s23 * t2[1] + b.s33 * t2[2]));
    o.s33 = (t2[0] * (b.s11 * t2[0] + b.s12 * t2[1] + b.s13 * t2[2]) + t2[1] * (b.s12 * t2[0] + b.s22 * t2[1] + b.s23 * t2[2]) +
             t2[2] * (b.s13 * t2[0] + b.s23 * t2[1] + b.s33 * t2[2]));
    return o;
}

template <typename T>
__device__ __forceinline__ BF<T> rot_nt_xy(const BF<T>& b, const T nn[3], const T t1[3], const T t2[3]) {
    BF<T> o;
    o.v1 = nn[0] * b.v1 + t1[0] * b.v2 + t2[0] * b.v3;
    o.v2 = nn[1] * b.v1 + t1[1] * b.v2 + t2[1] * b.v3;
    o.v3 = nn[2] * b.v1 + t1[2] * b.v2 + t2[2] * b.v3;
    o.s11 = (nn[0] * (b.s11 * nn[0] + b.s12 * t1[0] + b.s13 * t2[0]) + t1[0] * (b.s12 * nn[0] + b.s22 * t1[0] + b.s23 * t2[0]) +
             t2[0] * (b.s13 * nn[0] + b.s23 * t1[0] + b.s33 * t2[0]));
    o.s12 = (nn[0] * (b.s11 * nn[1] + b.s12 * t1[1] + b.s13 * t2[1]) + t1[0] * (b.s12 * nn[1] + b.s22 * t1[1] + b.s23 * t2[1]) +
             t2[0] * (b.s13 * nn[1] + b.s23 * t1[1] + b.s33 * t2[1]));
    o.s13 = (nn[0] * (b.s11 * nn[2] + b.s12 * t1[2] + b.s13 * t2[2]) + t1[0] * (b.s12 * nn[2] + b.s22 * t1[2] + b.s23 * t2[2]) +
             t2[0] * (b.s13 * nn[2] + b.s23 * t1[2] + b.s33 * t2[2]));
    o.s22 = (nn[1] * (b.s11 * nn[1] + b.s12 * t1[1] + b.s13 * t2[1]) + t1[1] * (b.s12 * nn[1] + b.s22 * t1[1] + b.s23 * t2[1]) +
             t2[1] * (b.s13 * nn[1] + b.s23 * t1[1] + b.s33 * t2[1]));
    o.s23 = (nn[1] * (b.s11 * nn[2] + b.s12 * t1[2] + b.s13 * t2[2]) + t1[1] * (b.s12 * nn[2] + b.s22 * t1[2] + b.s23 * t2[2]) +
             t2[1] * (b.s13 * nn[2] + b.s23 * t1[2] + b.s33 * t2[2]));
    o.s33 = (nn[2] * (b.s11 * nn[2] + b.s12 * t1[2] + b.s13 * t2[2]) + t1[2] * (b.s12 * nn[2] + b.s22 * t1[2] + b.s23 * t2[2]) +
             t2[2] * (b.s13 * nn[2] + b.s23 * t1[2] + b.s33 * t2[2]));
    return o;
}

// wave speeds, impedances and gamma = 1 - 2 (cs/cp)^2 of one node of a
// heterogeneous material (planes rho, lambda, G at stride st), in the
// reference's expressions (boundary.cpp:303-314, interface.cpp:614-638)
struct NodeMat {
    double cp, cs, zp, zs, gamma;
};
__device__ __forceinline__ NodeMat node_material(const double* mat, long long st, long long id) {
    NodeMat m;
    const double rho = mat[id], lm = mat[st + id], gg = mat[2 * st + id];
    m.cp = sqrt((lm + 2. * gg) / rho);
    m.cs = sqrt(gg / rho);
    m.zp = rho * m.cp;
    m.zs = rho * m.cs;
    m.gamma = 1. - 2. * ((m.cs / m.cp) * (m.cs / m.cp));
    return m;
}

// Outer-boundary SAT on face `face` of block b for the node at (a,b) in the
// face arrays; f holds the node's stage-start fields, df its rate register.
template <typename T, int NDIM, int MODE>
__device__ __forceinline__ void boundary_sat(const BlockDev& B, int face, int fa, int fb, T dt, const T* f, T* df,
                                             bool plastic, long long id = -1) {
    const long long ij = (long long)fa * B.fn1[face] + fb;
    T nn[3] = {T(0.), T(0.), T(0.)}, t1[3], t2[3];
    for (int l = 0; l < NDIM; l++) nn[l] = (T)B.fnx[face][l][ij];
    const T h = dt * (T)B.fdl[face][ij];
    T cp = (T)B.cp, cs = (T)B.cs, zp = (T)B.zp, zs = (T)B.zs, gamma = (T)B.gamma;
    const T r = (T)B.r[face];
    if (B.mat && id >= 0) {   // per-node material; id is the node
        const NodeMat m = node_material(B.mat, B.matstride, id);
        cp = (T)m.cp;
        cs = (T)m.cs;
        zp = (T)m.zp;
        zs = (T)m.zs;
        gamma = (T)m.gamma;
    }
    if (fabs(nn[0]) > fabs(nn[1]) && fabs(nn[0]) > fabs(nn[2])) {
        t1[2] = T(0.);
        t1[1] = nn[0] / sqrt(nn[0] * nn[0] + nn[1] * nn[1]);
        t1[0] = -nn[1] / sqrt(nn[0] * nn[0] + nn[1] * nn[1]);
    } else if (fabs(nn[1]) > fabs(nn[2])) {
        t1[2] = T(0.);
        t1[0] = nn[1] / sqrt(nn[0] * nn[0] + nn[1] * nn[1]);
        t1[1] = -nn[0] / sqrt(nn[0] * nn[0] + nn[1] * nn[1]);
    } else {
        t1[1] = T(0.);
        t1[0] = nn[2] / sqrt(nn[0] * nn[0] + nn[2] * nn[2]);
        t1[2] = -nn[0] / sqrt(nn[0] * nn[0] + nn[2] * nn[2]);
    }
    t2[0] = nn[1] * t1[2] - nn[2] * t1[1];
    t2[1] = nn[2] * t1[0] - nn[0] * t1[2];
    t2[2] = nn[0] * t1[1] - nn[1] * t1[0];
    BF<T> b;
    if (NDIM == 3) {
        b = {f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8]};
    } else if (MODE == 2) {
        b = {f[0], f[1], T(0.), f[2], f[3], T(0.), f[4], T(0.), T(0.)};
    } else {
        b = {T(0.), T(0.), f[0], T(0.), T(0.), f[1], T(0.), f[2], T(0.)};
    }
    BF<T> brot = rot_xy_nt(b, nn, t1, t2);
    BF<T> brots = brot;
    const T hps = (r + T(1.)) * T(0.5) * (brot.s11 - zp * brot.v1), hpv = (r - T(1.)) * T(0.5) * (brot.s11 / zp - brot.v1);
    const T h1s = (r + T(1.)) * T(0.5) * (brot.s12 - zs * brot.v2), h1v = (r - T(1.)) * T(0.5) * (brot.s12 / zs - brot.v2);
    const T h2s = (r + T(1.)) * T(0.5) * (brot.s13 - zs * brot.v3), h2v = (r - T(1.)) * T(0.5) * (brot.s13 / zs - brot.v3);
    brot.v1 -= hpv;
    brot.v2 = T(0.);
    brot.v3 = T(0.);
    brot.s22 = gamma * (brot.s11 - hps);
    brot.s33 = gamma * (brot.s11 - hps);
    brot.s11 -= hps;
    brot.s12 = T(0.);
    brot.s13 = T(0.);
    brot.s23 = T(0.);
    b = rot_nt_xy(brot, nn, t1, t2);
    const T alpha = (T)B.alpha[face], theta = (T)B.theta[face];
    if (NDIM == 3) {
        df[0] -= alpha * cp * h * b.v1;
        df[1] -= alpha * cp * h * b.v2;
        df[2] -= alpha * cp * h * b.v3;
        df[3] -= theta * cp * h * b.s11;
        df[4] -= theta * cp * h * b.s12;
        df[5] -= theta * cp * h * b.s13;
        df[6] -= theta * cp * h * b.s22;
        df[7] -= theta * cp * h * b.s23;
        df[8] -= theta * cp * h * b.s33;
    } else if (MODE == 2) {
        df[0] -= cp * h * b.v1;
        df[1] -= cp * h * b.v2;
        df[2] -= cp * h * b.s11;
        df[3] -= cp * h * b.s12;
        df[4] -= cp * h * b.s22;
        if (plastic) df[5] -= cp * h * b.s33;
    }
    brots.v1 = T(0.);
    brots.v2 -= h1v;
    brots.v3 -= h2v;
    brots.s11 = T(0.);
    brots.s12 -= h1s;
    brots.s13 -= h2s;
    brots.s22 = T(0.);
    brots.s23 = T(0.);
    brots.s33 = T(0.);
    b = rot_nt_xy(brots, nn, t1, t2);
    if (NDIM == 3) {
        df[0] -= alpha * cs * h * b.v1;
        df[1] -= alpha * cs * h * b.v2;
        df[2] -= alpha * cs * h * b.v3;
        df[3] -= theta * cs * h * b.s11;
        df[4] -= theta * cs * h * b.s12;
        df[5] -= theta * cs * h * b.s13;
        df[6] -= theta * cs * h * b.s22;
        df[7] -= theta * cs * h * b.s23;
        df[8] -= theta * cs * h * b.s33;
    } else if (MODE == 2) {
        df[0] -= cs * h * b.v1;
        df[1] -= cs * h * b.v2;
        df[2] -= cs * h * b.s11;
        df[3] -= cs * h * b.s12;
        df[4] -= cs * h * b.s22;
    } else {
        df[0] -= cs * h * b.v3;
        df[1] -= cs * h * b.s13;
        df[2] -= cs * h * b.s23;
    }
}

struct Plastp {
    double sxx, sxy, sxz, syy, syz, szz, gammap, lambda, epxx, epxy, epxz, epyy, epyz, epzz;
};

// Drucker-Prager viscoplastic return map, block.cpp:591-697 (always FP64)
__device__ __forceinline__ Plastp plastic_flow(const BlockDev& B, double dt, const Plastp& in, double k, double g) {
    double sigma = (in.sxx + in.syy + in.szz) / 3.;
    double tau = sqrt(((in.sxx - in.syy) * (in.sxx - in.syy) + (in.syy - in.szz) * (in.syy - in.szz) +
                       (in.szz - in.sxx) * (in.szz - in.sxx)) / 6. +
                      in.sxy * in.sxy + in.sxz * in.sxz + in.syz * in.syz);
    double yf = B.coh - B.mu * sigma;
    if (yf < 0.) yf = 0.;
    Plastp out = in;
    if (tau - yf <= 0.) {
        out.lambda = 0.;
        return out;
    }
    if (tau * B.mu * B.beta * k > (B.mu * sigma - B.coh) * g)
        out.lambda = (tau + B.mu * sigma - B.coh) / (B.eta + dt * (g + B.mu * B.beta * k));
    else
        out.lambda = tau / (B.eta + dt * g);
    out.gammap = in.gammap + dt * out.lambda;
    double sd[6] = {in.sxx - sigma, in.sxy, in.sxz, in.syy - sigma, in.syz, in.szz - sigma};
    tau -= dt * out.lambda * g;
    sigma -= dt * out.lambda * B.beta * k;
    for (int i = 0; i < 6; i++) sd[i] *= tau / (tau + dt * out.lambda * g);
    out.sxx = sd[0] + sigma;
    out.sxy = sd[1];
    out.sxz = sd[2];
    out.syy = sd[3] + sigma;
    out.syz = sd[4];
    out.szz = sd[5] + sigma;
    out.epxx = in.epxx + dt * out.lambda * (sd[0] / (2. * tau) + (B.beta / 3.));
    out.epxy = in.epxy + dt * out.lambda * (sd[1] / (2. * tau));
    out.epxz = in.epxz + dt * out.lambda * (sd[2] / (2. * tau));
    out.epyy = in.epyy + dt * out.lambda * (sd[3] / (2. * tau) + (B.beta / 3.));
    out.epyz = in.epyz + dt * out.lambda * (sd[4] / (2. * tau));
    out.epzz = in.epzz + dt * out.lambda * (sd[5] / (2. * tau) + (B.beta / 3.));
    return out;
}

// End-of-stage update of one node: f_new = f + B*df, then on the last stage
// the return map (plastic) and the absolute-stress round trip.  `fn` holds
// the node's nf updated fields on return; plastic-only fields are updated in
// place in FP.  With stop_before_output the last-stage sequence stops after
// the return map (the caller re-solves the interface first).
template <typename T>
__device__ __forceinline__ void finish_node(const Layout& L, const BlockDev& B, const StageArgs& sa, const double s0[6],
                                            const double* S, double* ABS, T* FP, int plastic_tensor, long long id,
                                            T* fn, bool stop_before_output) {
    if (!sa.last) return;
    double sv[6];
    if (sa.plastic) {
        // set_stress -> calc_plastic -> remove_stress
        for (int c = 0; c < L.ns; c++) {
            T v = fn[L.nv + c];
            v += (T)s0[L.sidx[c]];
            if (S) v += (T)S[c * L.cstride + id];
            sv[c] = (double)v;
        }
        if (sizeof(T) == 4) {
            // FP32 fields: form the absolute stress in FP64
            for (int c = 0; c < L.ns; c++) {
                double v = (double)fn[L.nv + c] + s0[L.sidx[c]];
                if (S) v += S[c * L.cstride + id];
                sv[c] = v;
            }
        }
        Plastp in;
        const int o = L.nfields;
        if (L.ndim == 3) {
            in.sxx = sv[0]; in.sxy = sv[1]; in.sxz = sv[2]; in.syy = sv[3]; in.syz = sv[4]; in.szz = sv[5];
        } else if (L.mode == 2) {
            in.sxx = sv[0]; in.sxy = sv[1]; in.sxz = 0.; in.syy = sv[2]; in.syz = 0.; in.szz = sv[3];
        } else {
            in.sxx = s0[0]; in.sxy = 0.; in.sxz = sv[0]; in.syy = s0[3]; in.syz = sv[1]; in.szz = s0[5];
        }
        in.lambda = (double)FP[0 * L.cstride + id];
        in.gammap = (double)FP[1 * L.cstride + id];
        in.epxx = in.epxy = in.epxz = in.epyy = in.epyz = in.epzz = 0.;
        if (plastic_tensor) {
            in.epxx = (double)FP[2 * L.cstride + id]; in.epxy = (double)FP[3 * L.cstride + id];
            in.epxz = (double)FP[4 * L.cstride + id]; in.epyy = (double)FP[5 * L.cstride + id];
            in.epyz = (double)FP[6 * L.cstride + id]; in.epzz = (double)FP[7 * L.cstride + id];
        }
        (void)o;
        double lm = B.lam, gg = B.g;
        if (B.mat) {   // block.cpp:519-521
            lm = B.mat[L.cstride + id];
            gg = B.mat[2 * L.cstride + id];
        }
        double k = lm + 2. / 3. * gg;
        if (B.ptrunc) k = (double)(int)k;   // the int loop index holds it (block.cpp:519-524)
        bool visit = true;
        if (B.pvisit == 1)
            visit = (int)(id % L.s1) == B.lo[2];
        else if (B.pvisit == 2)
            visit = B.pmask[id] != 0;
        // a node the loop skips keeps its stress (through the absolute-stress
        // round trip below) and its plastic fields
        Plastp out = visit ? plastic_flow(B, sa.dt, in, k, gg) : in;
        if (L.ndim == 3) {
            sv[0] = out.sxx; sv[1] = out.sxy; sv[2] = out.sxz; sv[3] = out.syy; sv[4] = out.syz; sv[5] = out.szz;
        } else if (L.mode == 2) {
            sv[0] = out.sxx; sv[1] = out.sxy; sv[2] = out.syy; sv[3] = out.szz;
        } else {
            sv[0] = out.sxz; sv[1] = out.syz;
        }
        if (visit) {
            FP[0 * L.cstride + id] = (T)out.lambda;
            FP[1 * L.cstride + id] = (T)out.gammap;
            if (plastic_tensor) {
                FP[2 * L.cstride + id] = (T)out.epxx; FP[3 * L.cstride + id] = (T)out.epxy;
                FP[4 * L.cstride + id] = (T)out.epxz; FP[5 * L.cstride + id] = (T)out.epyy;
                FP[6 * L.cstride + id] = (T)out.epyz; FP[7 * L.cstride + id] = (T)out.epzz;
            }
        }
        for (int c = 0; c < L.ns; c++) {
            if (sizeof(T) == 8) {
                T v = (T)sv[c];
                v -= (T)s0[L.sidx[c]];
                if (S) v -= (T)S[c * L.cstride + id];
                fn[L.nv + c] = v;
            } else {
                double v = sv[c] - s0[L.sidx[c]];
                if (S) v -= S[c * L.cstride + id];
                fn[L.nv + c] = (T)v;
            }
        }
        if (stop_before_output) return;
    }
    if (!sa.roundtrip) return;
    // output on absolute stress, then back (problem.cpp:160-164)
    for (int c = 0; c < L.ns; c++) {
        T v = fn[L.nv + c];
        v += (T)s0[L.sidx[c]];
        if (S) v += (T)S[c * L.cstride + id];
        if (ABS) ABS[c * L.cstride + id] = (double)v;
        v -= (T)s0[L.sidx[c]];
        if (S) v -= (T)S[c * L.cstride + id];
        fn[L.nv + c] = v;
    }
}

}  // namespace fdf
