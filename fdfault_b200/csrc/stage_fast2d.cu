// Tiled FP32 volume kernel for 2D blocks (mode II and mode III, elastic).
//
// Same discrete operator as the reference's calc_df_mode2 (src/block.cpp:
// 1048-1278) and calc_df_mode3 (src/block.cpp:1384-1539), plus the outer SAT
// (src/boundary.cpp:265-503) and the RK update (src/fields.cpp:293-309):
//  * one warp owns a tile of 32 consecutive j columns (the contiguous
//    direction) of one block and marches along x through a chunk of rows;
//  * the x-derivative inputs of a column -- the x fluxes F_x,c = J (m_x . sigma_c)
//    paired with the velocities v_c -- enter a per-warp shared ring when a
//    row enters the stencil window (deep enough for the 9-tap closure rows);
//  * the y-derivative inputs (F_y,c | v_c) of the current row go to a shared
//    row with a halo of order-1 columns on each side;
//  * interior stencils use the antisymmetric form; x closure rows (whole
//    rows) use the tabulated rows; in the first and last j tile of a block
//    every lane evaluates one NTB-tap row set up once per tile, so no lane
//    diverges on j;
//  * x-face rows get their outer SAT inline (every lane of the row is on the
//    face); y-face nodes (one lane in an edge tile) leave f and df in a
//    per-warp stash, and every KB2 rows 32 lanes add the y-face SATs of the
//    stashed nodes and write them.  A corner node gets its x SAT first and its
//    y SAT second, the reference's face order.
// Momentum rates use sum_d (dt/rho/dx_d)/J D_d(J m_d . sigma); stress rates
// come from the velocity gradient e_ab = sum_d (dt/dx_d) m_d,b D_d v_a
// (mode II: lambda (e_xx + e_yy) + 2G e_aa, G (e_xy + e_yx); mode III:
// G e_zx, G e_zy), algebraically the reference's per-direction terms.
//
// The per-tile routine tile2d() is shared by the per-block kernel and the
// ensemble's batched kernel, both in this file and compiled with the same
// flags, so an ensemble member's result is bit-identical to the same problem
// run alone with this kernel.  No result depends on the chunking in x.
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "ensemble.hpp"
#include "kernels.hpp"
#include "sbp_coeffs.cuh"
#include "stage_common.cuh"

namespace fdf {

namespace {

constexpr int TJ2 = 32;     // columns per tile (one warp)
constexpr int KB2 = 16;     // rows per y-face batch (2 sides x 16 rows = 32 lanes)
constexpr int NW2 = 4;      // warps (tiles) per CTA
constexpr int MINB2 = 4;    // resident CTAs per SM the register budget is sized for

template <int ORDER, int MODE>
struct F2 {
    static constexpr int H = ORDER - 1;
    static constexpr int NB = 2 * H;          // closure rows per side
    static constexpr int NTB = 3 * H;         // taps of a closure row
    static constexpr int R = NTB + 1;         // ring depth
    static constexpr int NC = (MODE == 2) ? 2 : 1;   // (flux, velocity) pairs per node
    static constexpr int NS = (MODE == 2) ? 3 : 2;   // stress components
    static constexpr int NF = NC + NS;               // fields
    static constexpr int VW = TJ2 + 2 * H;
    static constexpr int WROWS = 2 * NB + 1;  // centred, left closure, right closure (negated)
};

template <int ORDER, int MODE>
struct WarpSmem {
    using C = F2<ORDER, MODE>;
    float2 ring[C::R][C::NC][TJ2];   // (F_x,c , v_c)
    float2 trow[C::NC][C::VW];       // (F_y,c , v_c)
    float stash[KB2][2][2 * C::NF];  // y-face nodes: f, df per batch row and side
};

template <int ORDER>
__device__ __forceinline__ constexpr float inner_c2(int n) {
    return ORDER == 4 ? (n == 1 ? 0.75f : (n == 2 ? -0.15f : 1.f / 60.f))
                      : (ORDER == 3 ? (n == 1 ? 2.f / 3.f : -1.f / 12.f) : 0.5f);
}

// fluxes J (m0, m1) . sigma_c: mode II s = (sxx, sxy, syy), c = x, y;
// mode III s = (sxz, syz), one flux
template <int MODE>
__device__ __forceinline__ void flux2(float J, float m0, float m1, const float* s, float* Fo) {
    if (MODE == 2) {
        Fo[0] = J * (m0 * s[0] + m1 * s[1]);
        Fo[1] = J * (m0 * s[1] + m1 * s[2]);
    } else {
        Fo[0] = J * (m0 * s[0] + m1 * s[1]);
    }
}

// k-edge style weight table: row 0 centred (padded with zeros), rows 1..NB
// left closure, rows NB+1..2NB right closure negated
template <int ORDER, int MODE>
__device__ __forceinline__ void fill_wtab2(float* wtab) {
    using C = F2<ORDER, MODE>;
    for (int t = threadIdx.x; t < C::WROWS * C::NTB; t += blockDim.x) {
        const int r = t / C::NTB, n = t % C::NTB;
        float w;
        if (r == 0)
            w = (n <= 2 * C::H) ? sbp_coef<float>(ORDER, 0, n) : 0.f;
        else if (r <= C::NB)
            w = sbp_coef<float>(ORDER, r, n);
        else
            w = -sbp_coef<float>(ORDER, r - C::NB, n);
        wtab[t] = w;
    }
}

// One warp: tile jt of block B, rows [ib, ie).
template <int ORDER, int MODE>
__device__ __forceinline__ void tile2d(const VolumeArgs<float>& a, const BlockDev& B, const StageArgs& sa, int jt,
                                       int ib, int ie, WarpSmem<ORDER, MODE>& S, const float* wtab) {
    using C = F2<ORDER, MODE>;
    constexpr int H = C::H, NB = C::NB, NTB = C::NTB, R = C::R, NC = C::NC, NS = C::NS, NF = C::NF;
    const Layout& L = a.L;
    const int cs = (int)L.cstride;
    const int n0 = B.n[0], n1 = B.n[1];
    const int lane = threadIdx.x & 31;
    const int ntj = (n1 + TJ2 - 1) / TJ2;
    // the last tile is shifted to end on the block face; closure rows near a
    // face are written by the face tile, other columns by their natural tile
    const bool lastj = jt == ntj - 1;
    const int j0 = lastj ? n1 - TJ2 : jt * TJ2;
    const int j = j0 + lane;
    const bool own = (j >= n1 - NB) ? lastj : (j / TJ2 == jt);
    const bool jedge = (jt == 0) || lastj;
    int kb = lane, ks = 1, kmax = 2 * H, kw = 0;   // this lane's y row in an edge tile
    if (own && j < NB) {
        kb = H - j0;
        kmax = NTB - 1;
        kw = (j + 1) * NTB;
    } else if (own && j >= n1 - NB) {
        kb = (n1 - 1 - j0) + H;
        ks = -1;
        kmax = NTB - 1;
        kw = (NB + n1 - j) * NTB;
    }
    const int s0 = (int)L.s0;
    const int colbase = B.lo[0] * s0 + B.lo[1] + j;   // s1 == 1 in 2D
    // halo column of lanes [0, 2H)
    int hj = -1;
    if (lane < 2 * H) {
        hj = (lane < H) ? (j0 - H + lane) : (j0 + TJ2 + lane - H);
        if (hj < 0 || hj >= n1) hj = -1;
    }
    const int hcol = (lane < H) ? lane : (TJ2 + lane);
    const int hbase = B.lo[0] * s0 + B.lo[1] + hj;

    const float* __restrict__ F = a.F;
    const float* __restrict__ M = a.M;
    const float* __restrict__ Jg = a.J;
    float* __restrict__ DFg = a.DF;
    float* __restrict__ Fn = a.Fn;
    const float crho0 = (float)B.coef[0][0], crho1 = (float)B.coef[1][0];
    const float sd0 = (float)(sa.dt / B.dx[0]), sd1 = (float)(sa.dt / B.dx[1]);
    const float lamc = (float)B.lam, gc = (float)B.g, g2c = (float)(2. * B.g);
    const float Acoef = (float)sa.A, Bcoef = (float)sa.B, dtf = (float)sa.dt;

    auto mintap = [&](int i) { return i < NB ? 0 : (i >= n0 - NB ? n0 - NTB : i - H); };
    auto maxtap = [&](int i) { return i < NB ? NTB - 1 : (i >= n0 - NB ? n0 - 1 : i + H); };
    auto push_ring = [&](int q, int slot) {
        const int id = colbase + q * s0;
        float s[NS], v[NC], Fx[NC];
#pragma unroll
        for (int c = 0; c < NS; c++) s[c] = __ldg(F + (NC + c) * cs + id);
#pragma unroll
        for (int c = 0; c < NC; c++) v[c] = __ldg(F + c * cs + id);
        const float mx0 = __ldg(M + id), mx1 = __ldg(M + cs + id), Jq = __ldg(Jg + id);
        flux2<MODE>(Jq, mx0, mx1, s, Fx);
#pragma unroll
        for (int c = 0; c < NC; c++) S.ring[slot][c][lane] = make_float2(Fx[c], v[c]);
    };
    float f[NF], m[4], Jc, df[NF];
    float hs[NS], hv[NC], hm0 = 0.f, hm1 = 0.f, hJ = 0.f;
    auto load_center = [&](int i) {
        const int id = colbase + i * s0;
#pragma unroll
        for (int c = 0; c < NF; c++) f[c] = __ldg(F + c * cs + id);
#pragma unroll
        for (int c = 0; c < 4; c++) m[c] = __ldg(M + c * cs + id);
        Jc = __ldg(Jg + id);
#pragma unroll
        for (int c = 0; c < NF; c++) df[c] = DFg[c * cs + id];
        if (hj >= 0) {
            const int hid = hbase + i * s0;
#pragma unroll
            for (int c = 0; c < NS; c++) hs[c] = __ldg(F + (NC + c) * cs + hid);
#pragma unroll
            for (int c = 0; c < NC; c++) hv[c] = __ldg(F + c * cs + hid);
            hm0 = __ldg(M + 2 * cs + hid);
            hm1 = __ldg(M + 3 * cs + hid);
            hJ = __ldg(Jg + hid);
        }
    };

    int loaded = mintap(ib);
    int lslot = loaded % R;
    {
        const int need = maxtap(ib);
        while (loaded <= need) {
            push_ring(loaded, lslot);
            loaded++;
            lslot = (lslot + 1 == R) ? 0 : lslot + 1;
        }
    }
    int islot = ib % R;
    const int rslot = (n0 - 1) % R;
    int kbat = ib;
    load_center(ib);

    for (int i = ib; i < ie; i++) {
        {
            const int need = maxtap(i);
            while (loaded <= need) {   // near the block's x faces only
                push_ring(loaded, lslot);
                loaded++;
                lslot = (lslot + 1 == R) ? 0 : lslot + 1;
            }
        }
        {
            float Fy[NC];
            flux2<MODE>(Jc, m[2], m[3], f + NC, Fy);
#pragma unroll
            for (int c = 0; c < NC; c++) S.trow[c][lane + H] = make_float2(Fy[c], f[c]);
            if (hj >= 0) {
                float Fh[NC];
                flux2<MODE>(hJ, hm0, hm1, hs, Fh);
#pragma unroll
                for (int c = 0; c < NC; c++) S.trow[c][hcol] = make_float2(Fh[c], hv[c]);
            }
        }
        __syncwarp();
        float DFx[NC], Dvx[NC], DFy[NC], Dvy[NC];
        if (i >= NB && i < n0 - NB) {
#pragma unroll
            for (int c = 0; c < NC; c++) {
                float af = 0.f, av = 0.f;
#pragma unroll
                for (int n = 1; n <= H; n++) {
                    const int sp = (islot + n >= R) ? islot + n - R : islot + n;
                    const int sq = (islot - n < 0) ? islot - n + R : islot - n;
                    const float2 p = S.ring[sp][c][lane];
                    const float2 q = S.ring[sq][c][lane];
                    af = fmaf(inner_c2<ORDER>(n), p.x - q.x, af);
                    av = fmaf(inner_c2<ORDER>(n), p.y - q.y, av);
                }
                DFx[c] = af;
                Dvx[c] = av;
            }
        } else {
            const bool left = i < NB;
            const int row = left ? i + 1 : n0 - i;
            const float sg = left ? 1.f : -1.f;
#pragma unroll
            for (int c = 0; c < NC; c++) {
                float af = 0.f, av = 0.f;
                for (int n = 0; n < NTB; n++) {
                    const float cf = sbp_coef<float>(ORDER, row, n);
                    int sl = left ? n : rslot - n;
                    if (sl < 0) sl += R;
                    const float2 p = S.ring[sl][c][lane];
                    af = fmaf(cf, p.x, af);
                    av = fmaf(cf, p.y, av);
                }
                DFx[c] = sg * af;
                Dvx[c] = sg * av;
            }
        }
        if (!jedge) {
#pragma unroll
            for (int c = 0; c < NC; c++) {
                float af = 0.f, av = 0.f;
#pragma unroll
                for (int n = 1; n <= H; n++) {
                    const float2 p = S.trow[c][lane + H + n];
                    const float2 q = S.trow[c][lane + H - n];
                    af = fmaf(inner_c2<ORDER>(n), p.x - q.x, af);
                    av = fmaf(inner_c2<ORDER>(n), p.y - q.y, av);
                }
                DFy[c] = af;
                Dvy[c] = av;
            }
        } else {
            float af[NC], av[NC];
#pragma unroll
            for (int c = 0; c < NC; c++) af[c] = av[c] = 0.f;
#pragma unroll
            for (int n = 0; n < NTB; n++) {
                const float w = wtab[kw + n];
                const int col = kb + ks * min(n, kmax);
#pragma unroll
                for (int c = 0; c < NC; c++) {
                    const float2 p = S.trow[c][col];
                    af[c] = fmaf(w, p.x, af[c]);
                    av[c] = fmaf(w, p.y, av[c]);
                }
            }
#pragma unroll
            for (int c = 0; c < NC; c++) {
                DFy[c] = af[c];
                Dvy[c] = av[c];
            }
        }
        __syncwarp();   // the shared row is rewritten for the next row

        // ---- rate: df = A df + L(f)
        const float iJ = __frcp_rn(Jc);
        const float w0 = crho0 * iJ, w1 = crho1 * iJ;
#pragma unroll
        for (int c = 0; c < NC; c++) df[c] = fmaf(w1, DFy[c], fmaf(w0, DFx[c], Acoef * df[c]));
#pragma unroll
        for (int c = 0; c < NC; c++) {
            Dvx[c] *= sd0;
            Dvy[c] *= sd1;
        }
        if (MODE == 2) {
            const float exx = fmaf(m[2], Dvy[0], m[0] * Dvx[0]), exy = fmaf(m[3], Dvy[0], m[1] * Dvx[0]);
            const float eyx = fmaf(m[2], Dvy[1], m[0] * Dvx[1]), eyy = fmaf(m[3], Dvy[1], m[1] * Dvx[1]);
            const float lt = lamc * (exx + eyy);
            df[2] = fmaf(Acoef, df[2], fmaf(g2c, exx, lt));
            df[3] = fmaf(Acoef, df[3], gc * (exy + eyx));
            df[NF - 1] = fmaf(Acoef, df[NF - 1], fmaf(g2c, eyy, lt));
        } else {
            const float ezx = fmaf(m[2], Dvy[0], m[0] * Dvx[0]), ezy = fmaf(m[3], Dvy[0], m[1] * Dvx[0]);
            df[1] = fmaf(Acoef, df[1], gc * ezx);
            df[NF - 1] = fmaf(Acoef, df[NF - 1], gc * ezy);
        }
        // ---- x-face rows: outer SAT on every lane of the row
        bool deferx = false;
        if ((i == 0) | (i == n0 - 1)) {
            const int fc = (i == 0) ? 0 : 1;
            deferx = B.defer[fc] != 0;
            if (B.bactive[fc]) {
                float fl[NF], dl[NF];
#pragma unroll
                for (int c = 0; c < NF; c++) {
                    fl[c] = f[c];
                    dl[c] = df[c];
                }
                boundary_sat<float, 2, MODE>(B, fc, j, 0, dtf, fl, dl, false);
#pragma unroll
                for (int c = 0; c < NF; c++) df[c] = dl[c];
            }
        }
        if (own && ((j == 0) | (j == n1 - 1))) {   // y-face node: finished by the batch pass
            float* st = S.stash[i - kbat][j == 0 ? 0 : 1];
#pragma unroll
            for (int c = 0; c < NF; c++) {
                st[c] = f[c];
                st[NF + c] = df[c];
            }
        } else if (own) {
            const int id = colbase + i * s0;
#pragma unroll
            for (int c = 0; c < NF; c++) DFg[c * cs + id] = df[c];
            if (!deferx) {
#pragma unroll
                for (int c = 0; c < NF; c++) Fn[c * cs + id] = fmaf(Bcoef, df[c], f[c]);
            }
        }
        if (i - kbat == KB2 - 1 || i == ie - 1) {
            __syncwarp();
            const int q = lane >> 1, side = lane & 1;
            const int ip = kbat + q;
            if (ip <= i && (side == 0 ? jt == 0 : lastj)) {
                const int jr = side ? n1 - 1 : 0, fc = 2 + side;
                const float* st = S.stash[q][side];
                float fl[NF], dl[NF];
#pragma unroll
                for (int c = 0; c < NF; c++) {
                    fl[c] = st[c];
                    dl[c] = st[NF + c];
                }
                if (B.bactive[fc]) boundary_sat<float, 2, MODE>(B, fc, ip, 0, dtf, fl, dl, false);
                const int id = (B.lo[0] + ip) * s0 + B.lo[1] + jr;
#pragma unroll
                for (int c = 0; c < NF; c++) DFg[c * cs + id] = dl[c];
                const bool dx = ((ip == 0) && B.defer[0]) || ((ip == n0 - 1) && B.defer[1]);
                if (!B.defer[fc] && !dx) {
#pragma unroll
                    for (int c = 0; c < NF; c++) Fn[c * cs + id] = fmaf(Bcoef, dl[c], fl[c]);
                }
            }
            kbat = i + 1;
        }
        if (i + 1 < ie) load_center(i + 1);
        islot = (islot + 1 == R) ? 0 : islot + 1;
    }
}

template <int ORDER, int MODE>
__global__ void __launch_bounds__(NW2 * 32, MINB2) k_fast2d(VolumeArgs<float> a, BlockDev B, StageArgs sa, int chunk,
                                                     int nitems) {
    using C = F2<ORDER, MODE>;
    __shared__ WarpSmem<ORDER, MODE> S[NW2];
    __shared__ float wtab[C::WROWS * C::NTB];
    fill_wtab2<ORDER, MODE>(wtab);
    __syncthreads();
    const int w = threadIdx.x >> 5;
    const int item = blockIdx.x * NW2 + w;
    if (item >= nitems) return;
    const int ntj = (B.n[1] + TJ2 - 1) / TJ2;
    const int jt = item % ntj, ch = item / ntj;
    const int ib = ch * chunk, ie = min(B.n[0], ib + chunk);
    tile2d<ORDER, MODE>(a, B, sa, jt, ib, ie, S[w], wtab);
}

// the per-stage scalars of one ensemble member, as the single-problem solver
// forms them (only dt, A, B and last reach the volume kernel)
__device__ __forceinline__ StageArgs member_stage2(const EnsMember& M, const EnsRK& rk, int st) {
    StageArgs sa{};
    sa.dt = M.dt;
    sa.A = rk.A[st];
    sa.B = rk.B[st];
    sa.t = __dadd_rn(__dmul_rn((double)M.step, M.dt), __dmul_rn(rk.C[st], M.dt));
    sa.last = (st + 1 == rk.nstages);
    sa.cst = rk.C[st];
    return sa;
}

template <int ORDER, int MODE>
__global__ void __launch_bounds__(NW2 * 32, MINB2) k_ens_fast2d(const EnsMember* __restrict__ mem,
                                                         const Ens2dItem* __restrict__ items, int nitems, EnsRK rk,
                                                         int st) {
    using C = F2<ORDER, MODE>;
    __shared__ WarpSmem<ORDER, MODE> S[NW2];
    __shared__ float wtab[C::WROWS * C::NTB];
    fill_wtab2<ORDER, MODE>(wtab);
    __syncthreads();
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int it = blockIdx.x * nw + w; it < nitems; it += gridDim.x * nw) {
        const Ens2dItem t = items[it];
        const EnsMember& Mb = mem[t.m];
        if (Mb.step >= Mb.nt) continue;
        const StageArgs sa = member_stage2(Mb, rk, st);
        VolumeArgs<float> va = Mb.va;
        const int par = Mb.cur ^ (st & 1);
        va.F = Mb.buf[par];
        va.Fn = Mb.buf[par ^ 1];
        tile2d<ORDER, MODE>(va, Mb.blk[t.part], sa, t.jt, t.ib, t.ie, S[w], wtab);
    }
}

template <int ORDER, int MODE>
void launch2(const VolumeArgs<float>& a, const BlockDev& b, const StageArgs& sa, cudaStream_t s) {
    const int ntj = (b.n[1] + TJ2 - 1) / TJ2;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // enough warps to fill the GPU a few times over, chunks of at least 32 rows
    const long long want = 8LL * nsm * 16;
    int chunks = (int)((want + ntj - 1) / ntj);
    int chunk = (b.n[0] + chunks - 1) / chunks;
    if (chunk < 32) chunk = 32;
    chunks = (b.n[0] + chunk - 1) / chunk;
    const int nitems = ntj * chunks;
    k_fast2d<ORDER, MODE><<<(nitems + NW2 - 1) / NW2, NW2 * 32, 0, s>>>(a, b, sa, chunk, nitems);
}

template <int ORDER, int MODE>
void launch_ens2(int grid, const EnsMember* mem, const Ens2dItem* items, int nitems, const EnsRK& rk, int st,
                 cudaStream_t s) {
    k_ens_fast2d<ORDER, MODE><<<grid, NW2 * 32, 0, s>>>(mem, items, nitems, rk, st);
}

}  // namespace

bool fast2d_supported(const Layout& L, const BlockDev& b, int order) {
    if (b.mat) return false;   // one material per block
    if (L.ndim != 2) return false;
    if (!((L.mode == 2 && L.nfields == 5) || (L.mode == 3 && L.nfields == 3))) return false;   // elastic only
    if (order < 2 || order > 4) return false;
    if (b.n[1] < TJ2) return false;
    if (b.n[0] < 4 * order - 3) return false;
    if (L.cstride * L.nfields >= (1LL << 31)) return false;   // 32-bit element offsets
    return true;
}

void launch_volume_fast2d(const VolumeArgs<float>& a, const BlockDev& b, const StageArgs& sa, cudaStream_t s) {
    if (a.cdiss > 0. || sa.plastic) {
        launch_volume_exact<float>(a, b, sa, s);   // dissipation / plasticity: reference-order kernel
        return;
    }
    if (a.L.mode == 2) {
        switch (a.order) {
            case 2: launch2<2, 2>(a, b, sa, s); break;
            case 3: launch2<3, 2>(a, b, sa, s); break;
            default: launch2<4, 2>(a, b, sa, s); break;
        }
    } else {
        switch (a.order) {
            case 2: launch2<2, 3>(a, b, sa, s); break;
            case 3: launch2<3, 3>(a, b, sa, s); break;
            default: launch2<4, 3>(a, b, sa, s); break;
        }
    }
}

int fast2d_ensemble_grid(int order, int mode, int device) {
    int nsm = 148, occ = 1;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e;
    if (mode == 2)
        e = order == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_ens_fast2d<2, 2>, NW2 * 32, 0)
            : order == 3 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_ens_fast2d<3, 2>, NW2 * 32, 0)
                         : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_ens_fast2d<4, 2>, NW2 * 32, 0);
    else
        e = order == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_ens_fast2d<2, 3>, NW2 * 32, 0)
            : order == 3 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_ens_fast2d<3, 3>, NW2 * 32, 0)
                         : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_ens_fast2d<4, 3>, NW2 * 32, 0);
    if (e != cudaSuccess) throw std::runtime_error(std::string("occupancy query: ") + cudaGetErrorString(e));
    return nsm * (occ > 0 ? occ : 1);
}

void fast2d_ensemble_launch(int order, int mode, int grid, const EnsMember* mem, const Ens2dItem* items,
                            int nitems, const EnsRK& rk, int st, cudaStream_t s) {
    if (mode == 2) {
        switch (order) {
            case 2: launch_ens2<2, 2>(grid, mem, items, nitems, rk, st, s); break;
            case 3: launch_ens2<3, 2>(grid, mem, items, nitems, rk, st, s); break;
            default: launch_ens2<4, 2>(grid, mem, items, nitems, rk, st, s); break;
        }
    } else {
        switch (order) {
            case 2: launch_ens2<2, 3>(grid, mem, items, nitems, rk, st, s); break;
            case 3: launch_ens2<3, 3>(grid, mem, items, nitems, rk, st, s); break;
            default: launch_ens2<4, 3>(grid, mem, items, nitems, rk, st, s); break;
        }
    }
}

}  // namespace fdf
