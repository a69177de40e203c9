#pragma once
// Device side of the interface stage: one thread per fault node, in the
// reference's order (FP64 arithmetic; every file that includes this header
// is compiled with -fmad=false so it rounds as the reference does):
//   friction::scale_df                      src/friction.cpp:444-463
//   interface::apply_bcs (incl. SAT)        src/interface.cpp:573-970
//     interface::solve_interface (locked)   src/interface.cpp:972-1028
//     friction::solve_interface/_friction   src/friction.cpp:259-398
//     friction::solve_fs / slipweak / stz   src/friction.cpp:400-442,
//                                           src/slipweak.cpp:206-308,
//                                           src/stz.cpp:263-356
//     solve_newton (bracketed Newton)       src/utilities.cpp:89-179
//   friction::calc_df, friction::update     src/friction.cpp:465-505
// then the finish of the RK update of the two fault-plane nodes (the volume
// stage leaves those to the interface stage).  Fault-plane parameters that the
// reference recomputes from parametric perturbations every stage
// (src/pert.cpp:45-136) use precomputed spatial shapes times the same scalar
// value and time ramp, which rounds identically.  Used by the per-interface
// kernel (iface.cu) and the batched ensemble kernel (ensemble.cu).
#include <cuda_runtime.h>

#include "kernels.hpp"
#include "mlp_dev.cuh"
#include "stage_common.cuh"

namespace fdf {

namespace {

__device__ __forceinline__ double pert_value(const PertDev& q, int k, long long ij, double t) {
    double xy = q.shaped ? q.xy[ij] : 1.;
    double tf = (t >= q.t0) ? 1. : t / q.t0;
    return q.val[k] * xy * tf;
}

__device__ __forceinline__ double pert_sum(const IfaceDev& I, int k, long long ij, double t) {
    double acc = 0.;
    for (int m = 0; m < I.nperts; m++) acc += pert_value(I.perts[m], k, ij, t);
    return acc;
}

// slipweak::calc_mu: slip weakening combined with time weakening
__device__ double sw_calc_mu(const IfaceDev& I, long long ij, double t) {
    double dct = 0., must = 0., mudt = 0., trupt = 0., tct = 0.;
    for (int m = 0; m < I.nperts; m++) {
        const PertDev& q = I.perts[m];
        dct += pert_value(q, 0, ij, t);
        must += pert_value(q, 1, ij, t);
        mudt += pert_value(q, 2, ij, t);
        trupt += pert_value(q, 4, ij, t);
        tct += pert_value(q, 5, ij, t);
    }
    if (I.param_file) {
        dct += I.par[0][ij];
        must += I.par[1][ij];
        mudt += I.par[2][ij];
        trupt += I.par[4][ij];
        tct += I.par[5][ij];
    }
    const double u = I.u[ij];
    double f1, f2;
    if (dct == 0. || u >= dct)
        f1 = 1.;
    else
        f1 = u / dct;
    if (trupt <= 0. || t < trupt)
        f2 = 0.;
    else if (t >= trupt && t < trupt + tct)
        f2 = (tct == 0.) ? 1. : (t - trupt) / tct;
    else
        f2 = 1.;
    return (f1 >= f2) ? must + (mudt - must) * f1 : must + (mudt - must) * f2;
}

struct StzPar {
    double phi, eta, snc, chi, v0, f0, a, muy;
};

__device__ __forceinline__ double stz_vpl(double mu, const StzPar& p) {
    if (mu <= p.muy) return 0.;
    return p.v0 * exp(-p.f0 + mu / p.a - 1. / p.chi) * (1. - p.muy / mu);
}
// derivative as coded in the reference (stz.cpp:479); the bracketing keeps
// the root the same, and reproducing it keeps the iteration sequence
__device__ __forceinline__ double stz_dvpldmu(double mu, const StzPar& p) {
    if (mu <= p.muy) return 0.;
    return stz_vpl(mu, p) * (1. / p.a - p.muy / mu / (mu - p.muy));
}
__device__ __forceinline__ double stz_func(double mu, const StzPar& p) {
    return p.eta * stz_vpl(mu, p) - p.snc * mu - p.phi;
}
__device__ __forceinline__ double stz_der(double mu, const StzPar& p) { return p.eta * stz_dvpldmu(mu, p) - p.snc; }
// exact derivative of the root function: dV/dmu = V (1/a + muy / (mu (mu - muy)))
__device__ __forceinline__ double stz_der_exact(double mu, const StzPar& p) {
    const double dv = (mu <= p.muy) ? 0. : stz_vpl(mu, p) * (1. / p.a + p.muy / mu / (mu - p.muy));
    return p.eta * dv - p.snc;
}

// bracketed Newton with bisection fallback; returns a status bit on failure and
// the number of iterations taken in *iters
__device__ int solve_newton(double xmin, double xmax, const StzPar& p, double* out, int* iters, bool exact = false) {
    const int nmax = 100;
    const double tol = 2.e-16;
    double func, der, x, xl, xh, fh, dx, dxold, temp;
    x = 0.5 * (xmin + xmax);
    xh = xmax;
    xl = xmin;
    func = stz_func(x, p);
    fh = stz_func(xh, p);
    if (isinf(fh)) {
        int guard = 0;
        while (true) {
            if (!isinf(func)) {
                if (func > 0.) {
                    xh = x;
                    break;
                } else {
                    xl = x;
                }
            } else {
                xh = x;
            }
            x = 0.5 * (xh + xl);
            func = stz_func(x, p);
            if (++guard > 4096) {
                *out = x;
                *iters = guard;
                return FDF_ERR_NEWTON;
            }
        }
        *iters = guard;
    } else {
        *iters = 0;
    }
    x = 0.5 * (xh + xl);
    func = stz_func(x, p);
    der = exact ? stz_der_exact(x, p) : stz_der(x, p);
    dx = fabs(xh - xl);
    dxold = dx;
    int i = 0;
    while (i < nmax) {
        if (der == 0.) {
            *out = x;
            *iters += i;
            return FDF_ERR_ZERO_DERIV;
        }
        if ((((x - xh) * der - func) * ((x - xl) * der - func) > 0.) || fabs(2. * func) > fabs(dxold * der)) {
            dxold = dx;
            dx = 0.5 * (xh - xl);
            x = xl + dx;
            if (xl == x) break;
        } else {
            dxold = dx;
            dx = func / der;
            temp = x;
            x = x - dx;
            if (temp == x) break;
        }
        if (fabs(dx) < tol) break;
        func = stz_func(x, p);
        der = exact ? stz_der_exact(x, p) : stz_der(x, p);
        if (func < 0.)
            xl = x;
        else
            xh = x;
        i++;
    }
    *out = x;
    *iters += i;
    return (i == nmax) ? FDF_ERR_NEWTON : 0;
}

// The same bracketed iteration started from x0 (the learned guess) instead of
// the bracket midpoint: the bracket [xmin, xmax] is first narrowed by the sign
// of f(x0) (a guess where f overflows becomes the new upper end and the start
// moves to the midpoint, as in the plain solve).  Returns FDF_ERR_NEWTON if it
// does not converge; the caller then falls back to the plain solve.
__device__ int solve_newton_from(double xmin, double xmax, double x0, const StzPar& p, double* out, int* iters,
                                 bool exact = false) {
    const int nmax = 100;
    const double tol = 2.e-16;
    double xl = xmin, xh = xmax, x = x0;
    double func = stz_func(x, p);
    int guard = 0;
    while (isinf(func) || isnan(func)) {
        xh = x;
        x = 0.5 * (xl + xh);
        func = stz_func(x, p);
        if (++guard > 4096) {
            *iters = guard;
            *out = x;
            return FDF_ERR_NEWTON;
        }
    }
    if (func < 0.)
        xl = x;
    else
        xh = x;
    double der = exact ? stz_der_exact(x, p) : stz_der(x, p);
    double dx = fabs(xh - xl), dxold = dx, temp;
    int i = 0;
    while (i < nmax) {
        if (der == 0.) break;
        if ((((x - xh) * der - func) * ((x - xl) * der - func) > 0.) || fabs(2. * func) > fabs(dxold * der)) {
            dxold = dx;
            dx = 0.5 * (xh - xl);
            x = xl + dx;
            if (xl == x) break;
        } else {
            dxold = dx;
            dx = func / der;
            temp = x;
            x = x - dx;
            if (temp == x) break;
        }
        if (fabs(dx) < tol) break;
        func = stz_func(x, p);
        der = exact ? stz_der_exact(x, p) : stz_der(x, p);
        if (func < 0.)
            xl = x;
        else
            xh = x;
        i++;
    }
    *out = x;
    *iters = guard + i;
    return (i == nmax || der == 0.) ? FDF_ERR_NEWTON : 0;
}

__device__ inline void stz_par(const IfaceDev& I, double phi, double eta, double snc, long long ij, double t,
                               StzPar& p) {
    p.phi = phi;
    p.eta = eta;
    p.snc = snc;
    p.chi = I.state[ij];
    p.v0 = pert_sum(I, 0, ij, t);
    p.f0 = pert_sum(I, 1, ij, t);
    p.a = pert_sum(I, 2, ij, t);
    p.muy = pert_sum(I, 3, ij, t);
    if (I.param_file) {
        p.v0 += I.par[0][ij];
        p.f0 += I.par[1][ij];
        p.a += I.par[2][ij];
        p.muy += I.par[3][ij];
    }
}

// counters and training samples of one STZ Newton solve
__device__ inline void stz_record(const IfaceDev& I, const StzPar& p, double mu, int iters, bool midpoint, int st,
                                  const float* x) {
    if (I.stz.stats) {   // one atomic per counter per warp
        const unsigned mask = __activemask();
        const unsigned n = __popc(mask);
        const unsigned it = __reduce_add_sync(mask, (unsigned)iters);
        const unsigned mid = __reduce_add_sync(mask, midpoint ? 1u : 0u);
        if ((threadIdx.x & 31) == __ffs(mask) - 1) {
            atomicAdd(&I.stz.stats[0], (unsigned long long)n);
            atomicAdd(&I.stz.stats[1], (unsigned long long)it);
            if (mid) atomicAdd(&I.stz.stats[2], (unsigned long long)mid);
        }
    }
    if (I.stz.samples && st == 0) {
        float xs[MLP_IN];
        bool ok = true;
        if (x) {
            for (int i = 0; i < MLP_IN; i++) xs[i] = x[i];
        } else {
            ok = stz_features(p.phi, p.snc, p.chi, p.eta, p.v0, p.f0, p.a, p.muy, xs);
        }
        const double mh = -p.phi / p.snc;
        if (ok) {
            const unsigned long long k = atomicAdd(I.stz.nsamples, 1ULL);
            if (k < I.stz.cap) {
                // target t = logit(s)/20 with s and 1 - s each taken from its own
                // difference (both ends of the bracket resolved)
                const double w = mh - p.muy;
                const double lo = fmax((mu - p.muy) / w, 1e-16), hi = fmax((mh - mu) / w, 1e-16);
                float* o = I.stz.samples + 8 * k;
                for (int i = 0; i < MLP_IN; i++) o[i] = xs[i];
                o[6] = (float)((log(lo) - log(hi)) / 20.);
                o[7] = (float)mu;
            }
        }
    }
}

// friction::solve_fs (frictionless / stz) and slipweak::solve_fs
template <bool LEARN>
__device__ int solve_fs(const IfaceDev& I, double phi, double eta, double snc, long long ij, double t, double* bv,
                        double* bs) {
    int st = 0;
    if (I.kind == 2) {
        double c0t = 0.;
        for (int m = 0; m < I.nperts; m++) c0t += pert_value(I.perts[m], 3, ij, t);
        if (I.param_file) c0t += I.par[3][ij];
        if (snc < 0.) {
            double mu = sw_calc_mu(I, ij, t);
            if (c0t + mu * fabs(snc) > phi) {
                *bv = 0.;
                *bs = phi;
            } else {
                *bs = c0t + mu * fabs(snc);
                *bv = (phi - *bs) / eta;
            }
        } else {
            if (phi > c0t) {
                *bs = c0t;
                *bv = (phi - *bs) / eta;
            } else {
                *bv = 0.;
                *bs = phi;
            }
        }
        return 0;
    }
    if (LEARN && I.kind == 3) {
        // learned start: every lane evaluates the network (a full warp on the
        // tensor cores) before the per-node branches
        StzPar p;
        stz_par(I, phi, eta, snc, ij, t, p);
        float x[MLP_IN];
        // only nodes that reach the Newton solve need the network
        const bool need = (snc < 0.) && (p.muy < -phi / snc);
        const bool feat = need && stz_features(phi, snc, p.chi, eta, p.v0, p.f0, p.a, p.muy, x);
        if (!feat)
            for (int i = 0; i < MLP_IN; i++) x[i] = 0.f;
        float y = 0.f;
        const unsigned act = __activemask();
        if (act == 0xffffffffu) {
            __syncwarp();
            if (__any_sync(0xffffffffu, feat)) y = mlp_eval_warp(I.stz.mlp, x);
        } else if (feat) {
            y = mlp_eval_thread(I.stz.mlp, x);
        }
        double mu = 0.;
        if (snc < 0.) {
            const double mh = -phi / snc;
            if (p.muy >= mh) {
                mu = mh;
            } else {
                int iters = 0, s1 = FDF_ERR_NEWTON;
                bool midpoint = true;
                // the network predicts t = logit(s)/20, s = (mu - muy)/(mh - muy):
                // roots of creeping nodes sit within 1e-7 of the bracket's upper
                // end, of fast-slipping nodes near its lower end.  The start is
                // mh - q (mh - muy) with q = 1 - s, formed without cancellation.
                if (feat && isfinite(y)) {
                    const float z = fminf(fmaxf(20.f * y, -36.f), 36.f);
                    const double q = (double)(1.f / (1.f + __expf(z)));
                    const double x0 = fmin(fmax(mh - q * (mh - p.muy), p.muy), mh);
                    s1 = solve_newton_from(p.muy, mh, x0, p, &mu, &iters);
                    midpoint = s1 != 0;
                }
                if (s1 != 0) {   // the plain solve judges and replaces a failed start
                    int it2 = 0;
                    s1 = solve_newton(p.muy, mh, p, &mu, &it2);
                    iters += it2;
                }
                st |= s1;
                if (I.stz.stats || I.stz.samples) stz_record(I, p, mu, iters, midpoint, s1, feat ? x : nullptr);
            }
            if (mu * fabs(snc) > phi) {
                *bv = 0.;
                *bs = phi;
            } else {
                *bs = mu * fabs(snc);
                *bv = (phi - *bs) / eta;
            }
        } else {
            *bs = 0.;
            *bv = phi / eta;
        }
    } else if (snc < 0.) {
        double mu = 0.;
        if (I.kind == 3) {
            StzPar p;
            p.phi = phi;
            p.eta = eta;
            p.snc = snc;
            p.chi = I.state[ij];
            p.v0 = pert_sum(I, 0, ij, t);
            p.f0 = pert_sum(I, 1, ij, t);
            p.a = pert_sum(I, 2, ij, t);
            p.muy = pert_sum(I, 3, ij, t);
            if (I.param_file) {
                p.v0 += I.par[0][ij];
                p.f0 += I.par[1][ij];
                p.a += I.par[2][ij];
                p.muy += I.par[3][ij];
            }
            const double mh = -phi / snc;
            if (p.muy >= mh) {
                mu = mh;
            } else {
                int iters = 0, s1 = FDF_ERR_NEWTON;
                bool midpoint = true;
                if (I.stz.start == 2 && I.stz.mu_prev) {   // warm start from this node's last root
                    const double x0 = I.stz.mu_prev[ij];
                    if (x0 > p.muy && x0 < mh) {
                        s1 = solve_newton_from(p.muy, mh, x0, p, &mu, &iters);
                        midpoint = s1 != 0;
                    }
                }
                if (s1 != 0) {
                    int it2 = 0;
                    s1 = solve_newton(p.muy, mh, p, &mu, &it2, I.stz.start == 3);
                    iters += it2;
                }
                st |= s1;
                if (I.stz.start == 2 && I.stz.mu_prev) I.stz.mu_prev[ij] = mu;
                if (I.stz.stats || I.stz.samples) stz_record(I, p, mu, iters, midpoint, s1, nullptr);
            }
        }
        if (mu * fabs(snc) > phi) {
            *bv = 0.;
            *bs = phi;
        } else {
            *bs = mu * fabs(snc);
            *bv = (phi - *bs) / eta;
        }
    } else {
        *bs = 0.;
        *bv = phi / eta;
    }
    if (I.kind == 3) {
        // stz::calc_dstatedt with chihat
        double c0t = pert_sum(I, 4, ij, t), Rt = pert_sum(I, 5, ij, t), betat = pert_sum(I, 6, ij, t);
        double chiwt = pert_sum(I, 7, ij, t), v1t = pert_sum(I, 8, ij, t);
        if (I.param_file) {
            c0t += I.par[4][ij];
            Rt += I.par[5][ij];
            betat += I.par[6][ij];
            chiwt += I.par[7][ij];
            v1t += I.par[8][ij];
        }
        if (*bv > v1t) st |= FDF_ERR_MELT;
        double chihat = (*bv == 0.) ? chiwt : chiwt / log(v1t / *bv);
        const double chi = I.state[ij];
        I.dstatedt[ij] = *bv * *bs / c0t * (1. - chi / chihat) - Rt * exp(-betat / chi);
    }
    return st;
}

template <typename T>
__device__ __forceinline__ void load_abs(const IfaceArgs<T>& a, const T* F, long long id, BF<double>& b) {
    const Layout& L = a.L;
    const long long cs = L.cstride;
    const double* s0 = a.s0;
    const double* S = a.S;
    if (L.ndim == 3) {
        b.v1 = (double)F[id];
        b.v2 = (double)F[cs + id];
        b.v3 = (double)F[2 * cs + id];
        b.s11 = (double)F[3 * cs + id] + s0[0];
        b.s12 = (double)F[4 * cs + id] + s0[1];
        b.s13 = (double)F[5 * cs + id] + s0[2];
        b.s22 = (double)F[6 * cs + id] + s0[3];
        b.s23 = (double)F[7 * cs + id] + s0[4];
        b.s33 = (double)F[8 * cs + id] + s0[5];
        if (S) {
            b.s11 += S[id];
            b.s12 += S[cs + id];
            b.s13 += S[2 * cs + id];
            b.s22 += S[3 * cs + id];
            b.s23 += S[4 * cs + id];
            b.s33 += S[5 * cs + id];
        }
    } else if (L.mode == 2) {
        b.v1 = (double)F[id];
        b.v2 = (double)F[cs + id];
        b.v3 = 0.;
        b.s11 = (double)F[2 * cs + id] + s0[0];
        b.s12 = (double)F[3 * cs + id] + s0[1];
        b.s13 = 0.;
        b.s22 = (double)F[4 * cs + id] + s0[3];
        b.s23 = 0.;
        b.s33 = 0.;
        if (S) {
            b.s11 += S[id];
            b.s12 += S[cs + id];
            b.s22 += S[2 * cs + id];
        }
    } else {
        b.v1 = 0.;
        b.v2 = 0.;
        b.v3 = (double)F[id];
        b.s11 = s0[0];
        b.s12 = 0.;
        b.s13 = (double)F[cs + id] + s0[2];
        b.s22 = s0[3];
        b.s23 = (double)F[2 * cs + id] + s0[4];
        b.s33 = 0.;
        if (S) {
            b.s13 += S[id];
            b.s23 += S[cs + id];
        }
    }
}

// df -= coef * h * (SAT vector), in the component order of the field layout
template <typename T>
__device__ __forceinline__ void sat_sub(const Layout& L, bool plastic, T* DF, long long id, double ch, const BF<double>& b,
                                        bool normal) {
    const long long cs = L.cstride;
    if (L.ndim == 3) {
        const double v[9] = {b.v1, b.v2, b.v3, b.s11, b.s12, b.s13, b.s22, b.s23, b.s33};
        for (int q = 0; q < 9; q++) DF[q * cs + id] = (T)((double)DF[q * cs + id] - ch * v[q]);
    } else if (L.mode == 2) {
        const double v[5] = {b.v1, b.v2, b.s11, b.s12, b.s22};
        for (int q = 0; q < 5; q++) DF[q * cs + id] = (T)((double)DF[q * cs + id] - ch * v[q]);
        if (normal && plastic) DF[5 * cs + id] = (T)((double)DF[5 * cs + id] - ch * b.s33);
    } else if (!normal) {
        const double v[3] = {b.v3, b.s13, b.s23};
        for (int q = 0; q < 3; q++) DF[q * cs + id] = (T)((double)DF[q * cs + id] - ch * v[q]);
    }
}

template <typename T>
__device__ __forceinline__ void finish_fault_node(const IfaceArgs<T>& a, const BlockDev& B, const StageArgs& sa,
                                                  long long id, int no_sat) {
    const Layout& L = a.L;
    const long long cs = L.cstride;
    const int nf = L.nfields;
    T fn[9];
    if (!no_sat) {
        const T Bc = (T)sa.B;
        for (int q = 0; q < nf; q++) fn[q] = a.F[q * cs + id] + Bc * a.DF[q * cs + id];
        // plastic problems stop after the return map: the interface is
        // re-solved on the updated fields before the output round trip
        finish_node<T>(L, B, sa, a.s0, a.S, a.ABS, a.FP, a.plastic_tensor, id, fn, true);
    } else {
        for (int q = 0; q < nf; q++) fn[q] = a.Fn[q * cs + id];
        StageArgs s2 = sa;
        s2.plastic = 0;   // return map already applied
        finish_node<T>(L, B, s2, a.s0, a.S, a.ABS, a.FP, a.plastic_tensor, id, fn, false);
    }
    for (int q = 0; q < nf; q++) a.Fn[q * cs + id] = fn[q];
}

// one fault node ij of interface I (both sides' volume nodes, the friction
// solve, the SATs, the fault RK update and the finish of the two nodes)
template <typename T, bool LEARN>
__device__ __forceinline__ void interface_node(const IfaceArgs<T>& a, const IfaceDev& I, const BlockDev& B1,
                                               const BlockDev& B2, const StageArgs& sa, int no_sat, long long ij) {
    const long long nn = (long long)I.n0 * I.n1;
    if (ij >= nn) return;
    const Layout& L = a.L;
    const int D = I.direction;
    const int ii = (int)(ij / I.n1), jj = (int)(ij % I.n1);
    int pos[3] = {I.mlb[0], I.mlb[1], I.mlb[2]};
    const int o0 = (D == 0) ? 1 : 0, o1 = (D == 2) ? 1 : 2;
    pos[o0] += ii;
    pos[o1] += jj;
    // fault nodes on x planes that another process updates are left to it
    // (an x-normal fault goes with the minus side's last plane)
    if (pos[0] - B1.lo[0] < B1.xb || pos[0] - B1.lo[0] >= B1.xe) return;
    const long long st[3] = {L.s0, L.s1, L.s2};
    const long long i1 = node_index(L, pos[0], pos[1], pos[2]);
    const long long i2 = i1 + st[D];
    const double dt = sa.dt;
    double t = sa.t, tfront = sa.tfront;
    if (sa.step_dev) {
        const int sd = *sa.step_dev;
        t = (double)sd * dt + sa.cst * dt;
        tfront = (double)(sd + 1) * dt;
    }
    const bool fric = I.kind >= 1;
    const bool plastic = sa.plastic != 0;
    const T* F = no_sat ? a.Fn : a.F;
    if (fric && !no_sat) {
        // friction::scale_df
        const double A = sa.A;
        for (int c = 0; c < L.ndim - 1; c++) I.dux[c * nn + ij] *= A;
        I.du[ij] *= A;
        if (I.kind == 3) I.dstate[ij] *= A;
    }
    const double h1 = dt * I.dl1[ij], h2 = dt * I.dl2[ij];
    double nv[3] = {0., 0., 0.}, t1[3], t2[3];
    for (int l = 0; l < L.ndim; l++) nv[l] = I.nx[l][ij];
    switch (D) {
        case 0:
            t1[2] = 0.;
            t1[1] = nv[0] / sqrt(nv[0] * nv[0] + nv[1] * nv[1]);
            t1[0] = -nv[1] / sqrt(nv[0] * nv[0] + nv[1] * nv[1]);
            break;
        case 1:
            t1[2] = 0.;
            t1[0] = nv[1] / sqrt(nv[0] * nv[0] + nv[1] * nv[1]);
            t1[1] = -nv[0] / sqrt(nv[0] * nv[0] + nv[1] * nv[1]);
            break;
        default:
            t1[1] = 0.;
            t1[0] = nv[2] / sqrt(nv[0] * nv[0] + nv[2] * nv[2]);
            t1[2] = -nv[0] / sqrt(nv[0] * nv[0] + nv[2] * nv[2]);
    }
    t2[0] = nv[1] * t1[2] - nv[2] * t1[1];
    t2[1] = nv[2] * t1[0] - nv[0] * t1[2];
    t2[2] = nv[0] * t1[1] - nv[1] * t1[0];
    if (D == 1) {
        t2[0] = -t2[0];
        t2[1] = -t2[1];
        t2[2] = -t2[2];
    }
    BF<double> b1, b2;
    load_abs(a, F, i1, b1);
    load_abs(a, F, i2, b2);
    BF<double> br1 = rot_xy_nt(b1, nv, t1, t2), br2 = rot_xy_nt(b2, nv, t1, t2);
    BF<double> bs1 = br1, bs2 = br2;
    double zp1 = I.zp1, zs1 = I.zs1, zp2 = I.zp2, zs2 = I.zs2;
    double cp1 = I.cp1, cs1 = I.cs1, cp2 = I.cp2, cs2 = I.cs2, gamma1 = I.gamma1, gamma2 = I.gamma2;
    if (B1.mat) {   // heterogeneous material: both sides' nodes (interface.cpp:614-638)
        const NodeMat m1 = node_material(B1.mat, B1.matstride, i1), m2 = node_material(B2.mat, B2.matstride, i2);
        cp1 = m1.cp, cs1 = m1.cs, zp1 = m1.zp, zs1 = m1.zs, gamma1 = m1.gamma;
        cp2 = m2.cp, cs2 = m2.cs, zp2 = m2.zp, zs2 = m2.zs, gamma2 = m2.gamma;
    }
    // normal characteristic: locked solve (interface.cpp:1017-1028)
    double hs11 = (zp2 * (br1.s11 - zp1 * br1.v1) + zp1 * (br2.s11 + zp2 * br2.v1)) / (zp1 + zp2);
    double hv11 = (hs11 - br1.s11) / zp1 + br1.v1;
    double hs21 = hs11, hv21 = hv11;
    double hs12, hs22, hs13, hs23, hv12, hv22, hv13, hv23;
    int status = 0;
    if (!fric) {
        hs12 = (zs2 * (br1.s12 - zs1 * br1.v2) + zs1 * (br2.s12 + zs2 * br2.v2)) / (zs1 + zs2);
        hv12 = (hs12 - br1.s12) / zs1 + br1.v2;
        hs22 = hs12;
        hv22 = hv12;
        hs13 = (zs2 * (br1.s13 - zs1 * br1.v3) + zs1 * (br2.s13 + zs2 * br2.v3)) / (zs1 + zs2);
        hv13 = (hs13 - br1.s13) / zs1 + br1.v3;
        hs23 = hs13;
        hv23 = hv13;
    } else {
        // friction::solve_friction
        double snc = hs11;
        double is12 = br1.s12, is22 = br2.s12, is13 = br1.s13, is23 = br2.s13;
        const double iv12 = br1.v2, iv22 = br2.v2, iv13 = br1.v3, iv23 = br2.v3;
        const double eta = zs1 * zs2 / (zs1 + zs2);
        if (I.load_file) {
            snc += I.s1[ij];
            is12 += I.s2[ij];
            is22 += I.s2[ij];
            is13 += I.s3[ij];
            is23 += I.s3[ij];
        }
        for (int k = 0; k < I.nloads; k++) {
            const PertDev& q = I.loads[k];
            snc += pert_value(q, 0, ij, t);
            is12 += pert_value(q, 1, ij, t);
            is22 += pert_value(q, 1, ij, t);
            is13 += pert_value(q, 2, ij, t);
            is23 += pert_value(q, 2, ij, t);
        }
        const double phi2 = eta * (is12 / zs1 - iv12 + is22 / zs2 + iv22);
        const double phi3 = eta * (is13 / zs1 - iv13 + is23 / zs2 + iv23);
        const double phi = sqrt(phi2 * phi2 + phi3 * phi3);
        double bv, bs;
        status |= solve_fs<LEARN>(I, phi, eta, snc, ij, t, &bv, &bs);
        double v2, v3;
        if (bv == 0.) {
            v2 = 0.;
            v3 = 0.;
        } else {
            v2 = bv * phi2 / (eta * bv + bs);
            v3 = bv * phi3 / (eta * bv + bs);
        }
        hs12 = phi2 - eta * v2;
        hs22 = hs12;
        hs13 = phi3 - eta * v3;
        hs23 = hs13;
        hv12 = (hs12 - is12) / zs1 + iv12;
        hv22 = (-hs22 + is22) / zs2 + iv22;
        hv13 = (hs13 - is13) / zs1 + iv13;
        hv23 = (-hs23 + is23) / zs2 + iv23;
        I.v[ij] = bv;
        I.s[ij] = bs;
        I.sn[ij] = snc;
        if (L.ndim == 3) {
            I.vx[ij] = v2;
            I.vx[nn + ij] = v3;
            I.sx[ij] = hs12;
            I.sx[nn + ij] = hs13;
        } else if (L.mode == 2) {
            I.vx[ij] = v2;
            I.sx[ij] = hs12;
        } else {
            I.vx[ij] = v3;
            I.sx[ij] = hs13;
        }
        if (I.load_file) {
            hs12 -= I.s2[ij];
            hs22 -= I.s2[ij];
            hs13 -= I.s3[ij];
            hs23 -= I.s3[ij];
        }
        for (int k = 0; k < I.nloads; k++) {
            const PertDev& q = I.loads[k];
            hs12 -= pert_value(q, 1, ij, t);
            hs22 -= pert_value(q, 1, ij, t);
            hs13 -= pert_value(q, 2, ij, t);
            hs23 -= pert_value(q, 2, ij, t);
        }
    }
    if (!isfinite(hs12) || !isfinite(hv12)) status |= FDF_ERR_NONFINITE;
    if (status) atomicOr(a.status, status);
    if (!no_sat) {
        br1.v1 -= hv11;
        br1.v2 = 0.;
        br1.v3 = 0.;
        br1.s22 = gamma1 * (br1.s11 - hs11);
        br1.s33 = gamma1 * (br1.s11 - hs11);
        br1.s11 -= hs11;
        br1.s12 = 0.;
        br1.s13 = 0.;
        br1.s23 = 0.;
        br2.v1 -= hv21;
        br2.v2 = 0.;
        br2.v3 = 0.;
        br2.s22 = gamma2 * (br2.s11 - hs21);
        br2.s33 = gamma2 * (br2.s11 - hs21);
        br2.s11 -= hs21;
        br2.s12 = 0.;
        br2.s13 = 0.;
        br2.s23 = 0.;
        b1 = rot_nt_xy(br1, nv, t1, t2);
        b2 = rot_nt_xy(br2, nv, t1, t2);
        sat_sub<T>(L, plastic, a.DF, i1, cp1 * h1, b1, true);
        sat_sub<T>(L, plastic, a.DF, i2, cp2 * h2, b2, true);
        bs1.v1 = 0.;
        bs1.v2 -= hv12;
        bs1.v3 -= hv13;
        bs1.s11 = 0.;
        bs1.s12 -= hs12;
        bs1.s13 -= hs13;
        bs1.s22 = 0.;
        bs1.s23 = 0.;
        bs1.s33 = 0.;
        bs2.v1 = 0.;
        bs2.v2 -= hv22;
        bs2.v3 -= hv23;
        bs2.s11 = 0.;
        bs2.s12 -= hs22;
        bs2.s13 -= hs23;
        bs2.s22 = 0.;
        bs2.s23 = 0.;
        bs2.s33 = 0.;
        b1 = rot_nt_xy(bs1, nv, t1, t2);
        b2 = rot_nt_xy(bs2, nv, t1, t2);
        sat_sub<T>(L, plastic, a.DF, i1, cs1 * h1, b1, false);
        sat_sub<T>(L, plastic, a.DF, i2, cs2 * h2, b2, false);
        if (fric) {
            // friction::calc_df and friction::update
            const double Bc = sa.B;
            for (int c = 0; c < L.ndim - 1; c++) {
                I.dux[c * nn + ij] += dt * I.vx[c * nn + ij];
                I.ux[c * nn + ij] += Bc * I.dux[c * nn + ij];
            }
            I.du[ij] += dt * I.v[ij];
            I.u[ij] += Bc * I.du[ij];
            if (I.kind == 3) {
                I.dstate[ij] += dt * I.dstatedt[ij];
                I.state[ij] += Bc * I.dstate[ij];
            }
        }
    }
    if (!no_sat || plastic) {
        if (I.fin1[ij]) finish_fault_node(a, B1, sa, i1, no_sat);
        if (I.fin2[ij]) finish_fault_node(a, B2, sa, i2, no_sat);
    }
    // front::set_front after the step (front.cpp:103-125; the U field never records)
    if (fric && sa.front_on && sa.last && (no_sat || !plastic)) {
        if (I.tfront[ij] < 0. && I.v[ij] >= sa.front_value) I.tfront[ij] = tfront;
    }
}

}  // namespace

}  // namespace fdf
