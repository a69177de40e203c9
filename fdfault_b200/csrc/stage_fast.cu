// Tiled FP32 volume kernel for 3D blocks.
//
// Same discrete operator as the reference's calc_df_3d (src/block.cpp:
// 1541-2050) plus the outer SAT (src/boundary.cpp:265-503) and the RK update
// (src/fields.cpp:293-309), reorganised for bandwidth:
//  * each CTA owns a TJ x TK tile of (j, k) columns of one block and marches
//    along x through a chunk of planes;
//  * the x-derivative inputs of a column -- the x fluxes F_x,c = J (m_x . sigma_c)
//    paired with the velocity v_c -- are formed once per plane when the plane
//    enters the stencil window and kept in a per-thread shared-memory ring
//    deep enough for the 9-tap boundary closure rows;
//  * the y and z derivative inputs (F_y,c | v_c and F_z,c | v_c pairs) of the
//    current plane go into shared tiles with a halo of order-1 nodes;
//  * the centre values, rate register and halo node of the next plane are
//    loaded at the end of the current plane's iteration (two resident CTAs
//    per SM overlap one CTA's loads with the other's arithmetic);
//  * interior stencils are unrolled with immediate coefficients in the
//    antisymmetric form c1 (u+1 - u-1) + c2 (u+2 - u-2) + c3 (u+3 - u-3);
//    x and y closure rows (whole planes, whole warps) use the tabulated rows;
//    in the two k-edge tiles of a block every lane evaluates one NTB-tap row
//    whose weights and columns it set up once (interior lanes carry the
//    centred row padded with zero weights), so no warp diverges on k;
//  * the rate is accumulated in registers and written once; nodes on a block
//    face are finished by a small second kernel (k_faces3d) that adds the
//    outer SATs in face order and performs the RK update there, so the
//    marching kernel carries no face code.
// Momentum rates use sum_d (dt/rho/dx_d)/J * D_d(J m_d . sigma), which is
// algebraically the reference's conservative form; stress rates are formed
// from the velocity gradient e_ab = sum_d (dt/dx_d) m_d,b D_d v_a as
// lambda tr(e) delta_ab + G (e_ab + e_ba), algebraically the reference's
// sum over directions of the same non-conservative terms.  Arithmetic is FP32
// with FMA contraction; the FP64 exact-order kernel is stage_exact.cu.
#include <cuda_runtime.h>

#include <atomic>

#include "kernels.hpp"
#include "sbp_coeffs.cuh"
#include "stage_common.cuh"

namespace fdf {

namespace {

constexpr int TJ = 8, TK = 32, NT = TJ * TK;

template <int ORDER>
struct FastCfg {
    static constexpr int H = ORDER - 1;
    static constexpr int NB = 2 * H;        // closure rows per side
    static constexpr int NTB = 3 * H;       // taps of a closure row
    static constexpr int R = NTB + 1;       // ring depth
    static constexpr int HN = 2 * H * (TK + TJ);   // halo nodes per plane
    static constexpr int VH = TJ + 2 * H, VW = TK + 2 * H;
    static constexpr int RING = R * 3 * NT;   // float2 entries
    static constexpr int TY = 3 * VH * TK;    // float2
    static constexpr int TZ = 3 * TJ * VW;    // float2
    static constexpr int WROWS = 2 * NB + 1;  // k-edge weight rows: centred, left closure, right closure (negated)
    static constexpr int WTAB = ((WROWS * NTB + 3) / 4) * 4;   // floats
    static constexpr size_t SMEM = sizeof(float2) * (RING + TY + TZ) + sizeof(float) * WTAB;
};

// interior first-derivative weights in antisymmetric form (src/fd.cpp:53-83):
// D u_p = sum_n c_n (u_{p+n} - u_{p-n})
template <int ORDER>
__device__ __forceinline__ constexpr float inner_c(int n) {
    return ORDER == 4 ? (n == 1 ? 0.75f : (n == 2 ? -0.15f : 1.f / 60.f))
                      : (ORDER == 3 ? (n == 1 ? 2.f / 3.f : -1.f / 12.f) : 0.5f);
}

// fluxes J*(m_d . sigma_c) for c = x, y, z; s = sxx, sxy, sxz, syy, syz, szz
__device__ __forceinline__ void fluxes(float J, float m0, float m1, float m2, const float s[6], float F[3]) {
    F[0] = J * (m0 * s[0] + m1 * s[1] + m2 * s[2]);
    F[1] = J * (m0 * s[1] + m1 * s[3] + m2 * s[4]);
    F[2] = J * (m0 * s[2] + m1 * s[4] + m2 * s[5]);
}

struct RingPlane {   // raw values of one column at one plane, for the x ring
    float s[6], v[3], m[3], J;
};
struct HaloNode {
    float s[6], v[3], m[3], J;
};

template <int ORDER>
__global__ void __launch_bounds__(NT, 2) k_fast3d(VolumeArgs<float> a, BlockDev B, StageArgs sa, int chunk) {
    using C = FastCfg<ORDER>;
    constexpr int H = C::H, R = C::R, NB = C::NB, NTB = C::NTB, VH = C::VH, VW = C::VW;
    extern __shared__ float2 smem2[];
    float2* ring = smem2;              // [R][3][NT]   (F_x,c , v_c)
    float2* ty = ring + C::RING;       // [3][VH][TK]  (F_y,c , v_c)
    float2* tz = ty + C::TY;           // [3][TJ][VW]  (F_z,c , v_c)
    float* wtab = (float*)(tz + C::TZ);   // [WROWS][NTB]

    const Layout& L = a.L;
    const int cs = (int)L.cstride;
    const int n0 = B.n[0], n1 = B.n[1], n2 = B.n[2];
    const int tid = threadIdx.x;
    const int tk = tid % TK, tj = tid / TK;
    // The last tile in j and in k is shifted to end on the block face so it
    // holds every right-closure row together with all of that row's taps;
    // closure rows near a face are written by the face tile only, other rows
    // by their natural tile (rows computed twice are written once).
    const bool lastk = blockIdx.x == gridDim.x - 1, lastj = blockIdx.y == gridDim.y - 1;
    const int k0 = lastk ? n2 - TK : blockIdx.x * TK;
    const int j0 = lastj ? n1 - TJ : blockIdx.y * TJ;
    const int k = k0 + tk, j = j0 + tj;
    const bool ownk = (k >= n2 - NB) ? lastk : (k / TK == (int)blockIdx.x);
    const bool ownj = (j >= n1 - NB) ? lastj : (j / TJ == (int)blockIdx.y);
    const bool owner = ownk && ownj;
    const int ib = blockIdx.z * chunk;
    const int ie = min(n0, ib + chunk);
    if (ib >= ie) return;

    // k-edge tiles (first and last in k): one NTB-tap row per lane
    const bool kedge = (blockIdx.x == 0) || lastk;
    if (kedge && tid < C::WROWS * NTB) {
        const int r = tid / NTB, n = tid % NTB;
        float w;
        if (r == 0)
            w = (n <= 2 * H) ? sbp_coef<float>(ORDER, 0, n) : 0.f;
        else if (r <= NB)
            w = sbp_coef<float>(ORDER, r, n);
        else
            w = -sbp_coef<float>(ORDER, r - NB, n);
        wtab[tid] = w;
    }
    // this lane's row: tap n reads column kb + ks * min(n, kmax) of its tz row
    int kb = tk, ks = 1, kmax = 2 * H, kw = 0;
    if (ownk && k < NB) {
        kb = H - k0;
        kmax = NTB - 1;
        kw = (k + 1) * NTB;
    } else if (ownk && k >= n2 - NB) {
        kb = (n2 - 1 - k0) + H;
        ks = -1;
        kmax = NTB - 1;
        kw = (NB + n2 - k) * NTB;
    }

    const int s0 = (int)L.s0;
    const int colbase = B.lo[0] * s0 + (B.lo[1] + j) * (int)L.s1 + (B.lo[2] + k);
    const float* __restrict__ F = a.F;
    const float* __restrict__ M = a.M;
    const float* __restrict__ Jg = a.J;
    float* __restrict__ DFg = a.DF;
    float* __restrict__ Fn = a.Fn;

    // halo node handled by this thread (fixed for the whole march)
    int hj = 0, hk = 0, hkind = -1;   // 0: j-halo (F_y), 1: k-halo (F_z)
    if (tid < C::HN) {
        if (tid < 2 * H * TK) {
            const int r = tid / TK, c = tid % TK;
            hj = (r < H) ? (r - H) : (TJ + r - H);
            hk = c;
            hkind = 0;
        } else {
            const int t2 = tid - 2 * H * TK;
            const int r = t2 / (2 * H), c = t2 % (2 * H);
            hj = r;
            hk = (c < H) ? (c - H) : (TK + c - H);
            hkind = 1;
        }
        const int gj = j0 + hj, gk = k0 + hk;
        if (gj < 0 || gj >= n1 || gk < 0 || gk >= n2) hkind = -1;
    }
    const int hbase = B.lo[0] * s0 + (B.lo[1] + j0 + hj) * (int)L.s1 + (B.lo[2] + k0 + hk);
    const int hrow = (hkind == 0) ? 3 : 6;   // metric row y or z

    float crho[3], sd[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        crho[d] = (float)B.coef[d][0];
        sd[d] = (float)(sa.dt / B.dx[d]);
    }
    const float lamc = (float)B.lam, gc = (float)B.g, g2c = (float)(2. * B.g);
    const float Acoef = (float)sa.A, Bcoef = (float)sa.B;
    const bool jint = (j >= NB) && (j < n1 - NB);
    const bool face = (j == 0) | (j == n1 - 1) | (k == 0) | (k == n2 - 1);

    auto mintap = [&](int i) { return i < NB ? 0 : (i >= n0 - NB ? n0 - NTB : i - H); };
    auto maxtap = [&](int i) { return i < NB ? NTB - 1 : (i >= n0 - NB ? n0 - 1 : i + H); };

    auto load_ring = [&](int q, RingPlane& r) {
        const int id = colbase + q * s0;
#pragma unroll
        for (int c = 0; c < 6; c++) r.s[c] = __ldg(F + (3 + c) * cs + id);
#pragma unroll
        for (int c = 0; c < 3; c++) r.v[c] = __ldg(F + c * cs + id);
#pragma unroll
        for (int c = 0; c < 3; c++) r.m[c] = __ldg(M + c * cs + id);
        r.J = __ldg(Jg + id);
    };
    auto store_ring = [&](int qslot, const RingPlane& r) {
        float Fx[3];
        fluxes(r.J, r.m[0], r.m[1], r.m[2], r.s, Fx);
        float2* slot = ring + qslot * 3 * NT + tid;
#pragma unroll
        for (int c = 0; c < 3; c++) slot[c * NT] = make_float2(Fx[c], r.v[c]);
    };
    auto load_center = [&](int i, float f[9], float m[9], float& Jc, float df[9]) {
        const int id = colbase + i * s0;
#pragma unroll
        for (int c = 0; c < 9; c++) f[c] = __ldg(F + c * cs + id);
#pragma unroll
        for (int c = 0; c < 9; c++) m[c] = __ldg(M + c * cs + id);
        Jc = __ldg(Jg + id);
#pragma unroll
        for (int c = 0; c < 9; c++) df[c] = DFg[c * cs + id];
    };
    auto load_halo = [&](int i, HaloNode& h) {
        if (hkind < 0) return;
        const int id = hbase + i * s0;
#pragma unroll
        for (int c = 0; c < 6; c++) h.s[c] = __ldg(F + (3 + c) * cs + id);
#pragma unroll
        for (int c = 0; c < 3; c++) h.v[c] = __ldg(F + c * cs + id);
#pragma unroll
        for (int c = 0; c < 3; c++) h.m[c] = __ldg(M + (hrow + c) * cs + id);
        h.J = __ldg(Jg + id);
    };

    // prologue: the x window of the first plane, and the first plane's loads
    int loaded = mintap(ib);
    int lslot = loaded % R;
    {
        const int need = maxtap(ib);
        while (loaded <= need) {
            RingPlane r;
            load_ring(loaded, r);
            store_ring(lslot, r);
            loaded++;
            lslot = (lslot + 1 == R) ? 0 : lslot + 1;
        }
    }
    int islot = ib % R;
    const int rslot = (n0 - 1) % R;
    float f[9], m[9], Jc, df[9];
    load_center(ib, f, m, Jc, df);
    HaloNode hn;
    load_halo(ib, hn);

    for (int i = ib; i < ie; i++) {
        // ---- complete the x window for plane i
        {
            const int need = maxtap(i);
            while (loaded <= need) {   // only near the block's x faces
                RingPlane r;
                load_ring(loaded, r);
                store_ring(lslot, r);
                loaded++;
                lslot = (lslot + 1 == R) ? 0 : lslot + 1;
            }
        }
        // ---- shared tiles of plane i: centre and halo node
        {
            float Fy[3], Fz[3];
            fluxes(Jc, m[3], m[4], m[5], f + 3, Fy);
            fluxes(Jc, m[6], m[7], m[8], f + 3, Fz);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                ty[(c * VH + tj + H) * TK + tk] = make_float2(Fy[c], f[c]);
                tz[(c * TJ + tj) * VW + tk + H] = make_float2(Fz[c], f[c]);
            }
        }
        if (hkind >= 0) {
            float Fh[3];
            fluxes(hn.J, hn.m[0], hn.m[1], hn.m[2], hn.s, Fh);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                if (hkind == 0)
                    ty[(c * VH + hj + H) * TK + hk] = make_float2(Fh[c], hn.v[c]);
                else
                    tz[(c * TJ + hj) * VW + hk + H] = make_float2(Fh[c], hn.v[c]);
            }
        }
        const bool more = i + 1 < ie;
        __syncthreads();

        // ---- derivatives: DFl[d][c] of the fluxes, Dv[d][c] of the velocities
        float DFl[3][3], Dv[3][3];
        if (i >= NB && i < n0 - NB) {
            const float2* c0 = ring + tid;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float af = 0.f, av = 0.f;
#pragma unroll
                for (int n = 1; n <= H; n++) {
                    const int sp = (islot + n >= R) ? islot + n - R : islot + n;
                    const int sq = (islot - n < 0) ? islot - n + R : islot - n;
                    const float2 p = c0[(sp * 3 + c) * NT];
                    const float2 q = c0[(sq * 3 + c) * NT];
                    af = fmaf(inner_c<ORDER>(n), p.x - q.x, af);
                    av = fmaf(inner_c<ORDER>(n), p.y - q.y, av);
                }
                DFl[0][c] = af;
                Dv[0][c] = av;
            }
        } else {
            const bool left = i < NB;
            const int row = left ? i + 1 : n0 - i;
            const float sg = left ? 1.f : -1.f;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float af = 0.f, av = 0.f;
                for (int n = 0; n < NTB; n++) {
                    const float cf = sbp_coef<float>(ORDER, row, n);
                    int sl = left ? n : rslot - n;
                    if (sl < 0) sl += R;
                    const float2 p = ring[(sl * 3 + c) * NT + tid];
                    af = fmaf(cf, p.x, af);
                    av = fmaf(cf, p.y, av);
                }
                DFl[0][c] = sg * af;
                Dv[0][c] = sg * av;
            }
        }
        // closure rows this tile does not write (another tile owns them) may
        // have taps outside the tile: give them the interior form, whose taps
        // always lie in the tile and its halo, and discard the result
        const bool jskip = !jint && !ownj;
        if (jint || jskip) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float af = 0.f, av = 0.f;
#pragma unroll
                for (int n = 1; n <= H; n++) {
                    const float2 p = ty[(c * VH + tj + H + n) * TK + tk];
                    const float2 q = ty[(c * VH + tj + H - n) * TK + tk];
                    af = fmaf(inner_c<ORDER>(n), p.x - q.x, af);
                    av = fmaf(inner_c<ORDER>(n), p.y - q.y, av);
                }
                DFl[1][c] = af;
                Dv[1][c] = av;
            }
        } else {
            const bool left = j < NB;
            const int row = left ? j + 1 : n1 - j;
            const int base = (left ? 0 : n1 - 1) - j0 + H, step = left ? 1 : -1;
            const float sg = left ? 1.f : -1.f;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float af = 0.f, av = 0.f;
                for (int n = 0; n < NTB; n++) {
                    const float cf = sbp_coef<float>(ORDER, row, n);
                    const float2 p = ty[(c * VH + base + n * step) * TK + tk];
                    af = fmaf(cf, p.x, af);
                    av = fmaf(cf, p.y, av);
                }
                DFl[1][c] = sg * af;
                Dv[1][c] = sg * av;
            }
        }
        if (!kedge) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float af = 0.f, av = 0.f;
#pragma unroll
                for (int n = 1; n <= H; n++) {
                    const float2 p = tz[(c * TJ + tj) * VW + tk + H + n];
                    const float2 q = tz[(c * TJ + tj) * VW + tk + H - n];
                    af = fmaf(inner_c<ORDER>(n), p.x - q.x, af);
                    av = fmaf(inner_c<ORDER>(n), p.y - q.y, av);
                }
                DFl[2][c] = af;
                Dv[2][c] = av;
            }
        } else {
            float af[3] = {0.f, 0.f, 0.f}, av[3] = {0.f, 0.f, 0.f};
            const float2* trow = tz + tj * VW;
#pragma unroll
            for (int n = 0; n < NTB; n++) {
                const float w = wtab[kw + n];
                const int col = kb + ks * min(n, kmax);
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const float2 p = trow[c * TJ * VW + col];
                    af[c] = fmaf(w, p.x, af[c]);
                    av[c] = fmaf(w, p.y, av[c]);
                }
            }
#pragma unroll
            for (int c = 0; c < 3; c++) {
                DFl[2][c] = af[c];
                Dv[2][c] = av[c];
            }
        }
        __syncthreads();   // shared tiles are rewritten for the next plane

        // ---- rate: df = A df + L(f)
        const float iJ = __frcp_rn(Jc);
        {
            const float w0 = crho[0] * iJ, w1 = crho[1] * iJ, w2 = crho[2] * iJ;
#pragma unroll
            for (int c = 0; c < 3; c++)
                df[c] = fmaf(w2, DFl[2][c], fmaf(w1, DFl[1][c], fmaf(w0, DFl[0][c], Acoef * df[c])));
        }
        {
            // velocity gradient e[a][b] = d v_a / d x_b (times dt)
#pragma unroll
            for (int d = 0; d < 3; d++)
#pragma unroll
                for (int c = 0; c < 3; c++) Dv[d][c] *= sd[d];
            float e[3][3];
#pragma unroll
            for (int va = 0; va < 3; va++)
#pragma unroll
                for (int b = 0; b < 3; b++) e[va][b] = fmaf(m[6 + b], Dv[2][va], fmaf(m[3 + b], Dv[1][va], m[b] * Dv[0][va]));
            const float lt = lamc * (e[0][0] + e[1][1] + e[2][2]);
            df[3] = fmaf(Acoef, df[3], fmaf(g2c, e[0][0], lt));
            df[4] = fmaf(Acoef, df[4], gc * (e[0][1] + e[1][0]));
            df[5] = fmaf(Acoef, df[5], gc * (e[0][2] + e[2][0]));
            df[6] = fmaf(Acoef, df[6], fmaf(g2c, e[1][1], lt));
            df[7] = fmaf(Acoef, df[7], gc * (e[1][2] + e[2][1]));
            df[8] = fmaf(Acoef, df[8], fmaf(g2c, e[2][2], lt));
        }
        if (owner) {
            const int id = colbase + i * s0;
#pragma unroll
            for (int c = 0; c < 9; c++) DFg[c * cs + id] = df[c];
            // face nodes: k_faces3d adds the outer SATs and finishes them
            if (!(face | (i == 0) | (i == n0 - 1))) {
#pragma unroll
                for (int c = 0; c < 9; c++) Fn[c * cs + id] = fmaf(Bcoef, df[c], f[c]);
            }
        }
        if (more) {
            load_center(i + 1, f, m, Jc, df);
            load_halo(i + 1, hn);
        }
        islot = (islot + 1 == R) ? 0 : islot + 1;
    }
}

// Face nodes of a 3D block, after k_fast3d wrote their rate without the
// outer SAT: add the SAT of every face the node lies on, in face order
// (block::set_boundaries), write the rate, and unless a face is an interface
// (whose kernel finishes the node) perform the RK update.  blockIdx.z is the
// face; threadIdx.x runs along the face's k extent (its j extent on the two
// k faces), threadIdx.y along the other.  A node on several faces is handled
// by its first face.  With kdone the marching kernel has already added the
// k-face SATs and finished the nodes that lie on k faces only: the grid then
// covers the x and y faces, and k-face SATs are not added again.
template <bool PLASTIC>
__global__ void __launch_bounds__(128) k_faces3d(VolumeArgs<float> a, BlockDev B, StageArgs sa, int kdone) {
    const int fc = blockIdx.z, d = fc >> 1;
    const int n0 = B.n[0], n1 = B.n[1], n2 = B.n[2];
    const int nb = (d == 2) ? n1 : n2;
    const int na = (d == 0) ? n1 : n0;
    const int ub = blockIdx.x * 32 + threadIdx.x, ua = blockIdx.y * 4 + threadIdx.y;
    if (ub >= nb || ua >= na) return;
    const int at = (fc & 1) ? ((d == 0) ? n0 : ((d == 1) ? n1 : n2)) - 1 : 0;
    int i, j, k;
    if (d == 0) {
        i = at;
        j = ua;
        k = ub;
    } else if (d == 1) {
        i = ua;
        j = at;
        k = ub;
    } else {
        i = ua;
        j = ub;
        k = at;
    }
    if (i < B.xb || i >= B.xe) return;                // plane updated by another process
    if (d >= 1 && (i == 0 || i == n0 - 1)) return;   // belongs to an x face
    if (d == 2 && (j == 0 || j == n1 - 1)) return;   // belongs to a y face
    const Layout& L = a.L;
    const long long cs = L.cstride;
    const long long id = node_index(L, B.lo[0] + i, B.lo[1] + j, B.lo[2] + k);
    float f[9], df[9];
#pragma unroll
    for (int c = 0; c < 9; c++) {
        f[c] = a.F[c * cs + id];
        df[c] = a.DF[c * cs + id];
    }
    const bool on[6] = {i == 0, i == n0 - 1, j == 0, j == n1 - 1, k == 0, k == n2 - 1};
    bool defer = false;
#pragma unroll
    for (int f2 = 0; f2 < 6; f2++) {
        if (!on[f2]) continue;
        if (B.defer[f2]) defer = true;
        if (!B.bactive[f2] || (kdone && f2 >= 4)) continue;
        const int fa = (f2 < 2) ? j : i;
        const int fb = (f2 >= 4) ? j : k;
        boundary_sat<float, 3, 2>(B, f2, fa, fb, (float)sa.dt, f, df, false);
    }
#pragma unroll
    for (int c = 0; c < 9; c++) a.DF[c * cs + id] = df[c];
    if (defer) return;
    const float Bcoef = (float)sa.B;
    float fn[9];
#pragma unroll
    for (int c = 0; c < 9; c++) fn[c] = fmaf(Bcoef, df[c], f[c]);
    if (PLASTIC && sa.last) finish_node<float>(L, B, sa, a.s0, a.S, nullptr, a.FP, a.plastic_tensor, id, fn, false);
#pragma unroll
    for (int c = 0; c < 9; c++) a.Fn[c * cs + id] = fn[c];
}

// Drucker-Prager return map (finish_node on the last stage) of the interior
// nodes of a block, after a marching kernel wrote their updated fields: face
// nodes were finished by k_faces3d and fault nodes by the interface kernel.
// With kall the nodes on the k faces are included (the register-window kernel
// finishes them itself), except on k faces that an interface finishes.  Kept
// out of the marching kernels, whose register budget the FP64 return map
// would exceed.
__global__ void __launch_bounds__(256) k_return_map3(VolumeArgs<float> a, BlockDev B, StageArgs sa, int kall) {
    const int n1i = B.n[1] - 2, n2i = kall ? B.n[2] : B.n[2] - 2;
    // interior planes this process updates: max(1, xb) <= i < min(n0 - 1, xe)
    const int i0 = max(1, B.xb), i1 = min(B.n[0] - 1, B.xe);
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)(i1 - i0) * n1i * n2i) return;
    const int k = (kall ? 0 : 1) + (int)(t % n2i), j = 1 + (int)((t / n2i) % n1i),
              i = i0 + (int)(t / ((long long)n2i * n1i));
    if ((k == 0 && B.defer[4]) || (k == B.n[2] - 1 && B.defer[5])) return;
    const Layout& L = a.L;
    const long long cs = L.cstride;
    const long long id = node_index(L, B.lo[0] + i, B.lo[1] + j, B.lo[2] + k);
    float fn[9];
#pragma unroll
    for (int c = 0; c < 9; c++) fn[c] = a.Fn[c * cs + id];
    finish_node<float>(L, B, sa, a.s0, a.S, nullptr, a.FP, a.plastic_tensor, id, fn, false);
#pragma unroll
    for (int c = 3; c < 9; c++) a.Fn[c * cs + id] = fn[c];
}

template <int ORDER, bool PLASTIC>
void launch_order(const VolumeArgs<float>& a, const BlockDev& b, const StageArgs& sa, cudaStream_t s) {
    using C = FastCfg<ORDER>;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    // the shared-memory opt-in is a per-device function attribute: set it once per device
    static std::atomic<unsigned> configured{0};
    const unsigned bit = 1u << (dev & 31);
    if (!(configured.load() & bit)) {
        cudaFuncSetAttribute(k_fast3d<ORDER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
        configured.fetch_or(bit);
    }
    const int tk = (b.n[2] + TK - 1) / TK, tj = (b.n[1] + TJ - 1) / TJ;
    // split the x march into chunks so the grid fills the GPU a few times over
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int slots = 2 * nsm;
    int chunks = (4 * slots + tk * tj - 1) / (tk * tj);
    if (chunks < 1) chunks = 1;
    int chunk = (b.n[0] + chunks - 1) / chunks;
    if (chunk < 16) chunk = 16;
    chunks = (b.n[0] + chunk - 1) / chunk;
    dim3 grid(tk, tj, chunks);
    k_fast3d<ORDER><<<grid, NT, C::SMEM, s>>>(a, b, sa, chunk);
    const int nbmax = b.n[2] > b.n[1] ? b.n[2] : b.n[1], namax = b.n[0] > b.n[1] ? b.n[0] : b.n[1];
    k_faces3d<PLASTIC><<<dim3((nbmax + 31) / 32, (namax + 3) / 4, 6), dim3(32, 4), 0, s>>>(a, b, sa, 0);
    if (PLASTIC && sa.last) launch_return_map3(a, b, sa, false, s);
}

template <bool PLASTIC>
void launch_plastic(const VolumeArgs<float>& a, const BlockDev& b, const StageArgs& sa, cudaStream_t s) {
    switch (a.order) {
        case 2: launch_order<2, PLASTIC>(a, b, sa, s); break;
        case 3: launch_order<3, PLASTIC>(a, b, sa, s); break;
        default: launch_order<4, PLASTIC>(a, b, sa, s); break;
    }
}

}  // namespace

bool fast3d_supported(const Layout& L, const BlockDev& b, int order) {
    if (b.mat) return false;   // one material per block
    if (L.ndim != 3 || L.nfields != 9) return false;
    if (order < 2 || order > 4) return false;
    if (b.n[1] < TJ || b.n[2] < TK) return false;
    if (b.n[0] < 4 * order - 3) return false;
    if (L.cstride * 9 >= (1LL << 31)) return false;   // 32-bit element offsets
    return true;
}

void launch_faces3d(const VolumeArgs<float>& a, const BlockDev& b, const StageArgs& sa, bool kdone, bool plastic,
                    cudaStream_t s) {
    const int nbmax = b.n[2] > b.n[1] ? b.n[2] : b.n[1], namax = b.n[0] > b.n[1] ? b.n[0] : b.n[1];
    const dim3 grid((nbmax + 31) / 32, (namax + 3) / 4, kdone ? 4 : 6);
    if (plastic)
        k_faces3d<true><<<grid, dim3(32, 4), 0, s>>>(a, b, sa, kdone ? 1 : 0);
    else
        k_faces3d<false><<<grid, dim3(32, 4), 0, s>>>(a, b, sa, kdone ? 1 : 0);
}

void launch_return_map3(const VolumeArgs<float>& a, const BlockDev& b, const StageArgs& sa, bool kall,
                        cudaStream_t s) {
    const int i0 = b.xb > 1 ? b.xb : 1, i1 = b.xe < b.n[0] - 1 ? b.xe : b.n[0] - 1;
    const long long nin = (long long)(i1 - i0) * (b.n[1] - 2) * (kall ? b.n[2] : b.n[2] - 2);
    if (nin <= 0) return;
    k_return_map3<<<(unsigned)((nin + 255) / 256), 256, 0, s>>>(a, b, sa, kall ? 1 : 0);
}

void launch_volume_fast3d(const VolumeArgs<float>& a, const BlockDev& b, const StageArgs& sa, cudaStream_t s) {
    if (a.cdiss > 0.) {
        launch_volume_exact<float>(a, b, sa, s);   // artificial dissipation: exact-order kernel
        return;
    }
    if (sa.plastic)
        launch_plastic<true>(a, b, sa, s);
    else
        launch_plastic<false>(a, b, sa, s);
}

}  // namespace fdf
