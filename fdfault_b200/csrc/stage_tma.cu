// Staged FP32 3D volume kernel: the operator of the tiled kernel
// (stage_fast.cu: calc_df_3d src/block.cpp:1541-2050, outer SAT
// src/boundary.cpp:265-503, RK update src/fields.cpp:293-309), with every
// plane's data brought into shared memory by asynchronous bulk copies
// (TMA tensor copies, cp.async.bulk.tensor, completion counted on an
// mbarrier) a plane or two before it is needed, so no thread waits on a
// global load of its own:
//  * one CTA of 8 x 32 (j, k) columns per SM marches along x through a chunk
//    of planes;
//  * centre stream: plane i's fields, y/z metric rows, Jacobian (with the
//    order-1 halo in y and z) and x/z metric rows of the tile, double-buffered;
//  * ring stream: plane i+H's fields, x metric row and Jacobian of the tile,
//    double-buffered, from which the x fluxes J (m_x . sigma_c) and v_c enter
//    the per-thread x ring (deep enough for the 9-tap closure rows);
//  * y/z fluxes of the current plane go to shared tiles with a halo;
//  * the rate register df is read with ordinary loads one plane ahead.
// Each staged box is one tensor copy over a (k, j, i, component) tensor map of
// the field, metric or Jacobian array; its k origin is the 16-byte boundary at
// or below the first needed column (so the x coordinate times 4 bytes is a
// multiple of 16), and parts outside the arrays are filled with zeros.  Only
// results that are discarded read values from outside the block.  Every wait
// on an mbarrier is bounded: on expiry the CTA records FDF_ERR_TIMEOUT, drains
// its own copies in flight (bounded) and returns as a whole.
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "kernels.hpp"
#include "sbp_coeffs.cuh"
#include "stage_common.cuh"
#include "tma_util.cuh"

namespace fdf {

// tensor maps of one problem's FP32 arrays, with box shapes for the staged
// kernel of its operator order (Fc/Fr per field buffer: centre and ring boxes;
// My: y metric rows with halo; Mt: three metric rows of the tile; Mr: x
// metric rows of the ring; Jc/Jr: Jacobian)
struct StagedMaps {
    CUtensorMap Fc[2], Fr[2], My, Mt, Mr, Jc, Jr;
};

struct StagedMapsHost {
    StagedMaps m;
    const float* F0;
    int order;
};

namespace {

constexpr int TJ = 8, TK = 32, NT = TJ * TK;
constexpr int CW = 44;   // staged centre row, floats: TK + 2H + alignment slack, multiple of 4
constexpr int RW = 36;   // staged ring row, floats: TK + alignment slack, multiple of 4

constexpr int up32(int n) { return (n + 31) / 32 * 32; }   // 128-byte boundaries for every box

template <int ORDER>
struct StCfg {
    static constexpr int H = ORDER - 1;
    static constexpr int NB = 2 * H;
    static constexpr int NTB = 3 * H;
    static constexpr int R = NTB + 1;
    static constexpr int VH = TJ + 2 * H, VW = TK + 2 * H;
    // centre staging, floats: F[9][VH][CW], My[3][VH][CW], Mx[3][TJ][CW], Mz[3][TJ][CW], J[VH][CW]
    static constexpr int CF = 0, CMY = up32(9 * VH * CW), CMX = CMY + up32(3 * VH * CW),
                         CMZ = CMX + up32(3 * TJ * CW), CJ = CMZ + up32(3 * TJ * CW);
    static constexpr int CSZ = CJ + up32(VH * CW);
    static constexpr uint32_t CBYTES = 4u * (9 * VH * CW + 3 * VH * CW + 6 * TJ * CW + VH * CW);
    // ring staging, floats: F[9][TJ][RW], Mx[3][TJ][RW], J[TJ][RW]
    static constexpr int RMX = up32(9 * TJ * RW), RJ = RMX + up32(3 * TJ * RW), RSZ = RJ + up32(TJ * RW);
    static constexpr uint32_t RBYTES = 4u * 13 * TJ * RW;
    static constexpr int RING = R * 3 * NT, TY = 3 * VH * TK, TZ = 3 * TJ * VW;   // float2
    static constexpr size_t SMEM = sizeof(float) * (2 * CSZ + 2 * RSZ) + sizeof(float2) * (RING + TY + TZ) + 64;
};

template <int ORDER>
__device__ __forceinline__ constexpr float inner_c(int n) {
    return ORDER == 4 ? (n == 1 ? 0.75f : (n == 2 ? -0.15f : 1.f / 60.f))
                      : (ORDER == 3 ? (n == 1 ? 2.f / 3.f : -1.f / 12.f) : 0.5f);
}

__device__ __forceinline__ void fluxes(float J, float m0, float m1, float m2, const float s[6], float F[3]) {
    F[0] = J * (m0 * s[0] + m1 * s[1] + m2 * s[2]);
    F[1] = J * (m0 * s[1] + m1 * s[3] + m2 * s[4]);
    F[2] = J * (m0 * s[2] + m1 * s[4] + m2 * s[5]);
}

template <int ORDER>
__global__ void __launch_bounds__(NT, 1)
    k_tma3d(VolumeArgs<float> a, BlockDev B, StageArgs sa, int chunk, int* status,
            const __grid_constant__ StagedMaps maps, int fsel) {
    using C = StCfg<ORDER>;
    constexpr int H = C::H, R = C::R, NB = C::NB, NTB = C::NTB, VH = C::VH, VW = C::VW;
    extern __shared__ __align__(128) float smem[];
    float* cst0 = smem;                   // centre staging, two buffers
    float* rst0 = smem + 2 * C::CSZ;      // ring staging, two buffers
    float2* ring = reinterpret_cast<float2*>(rst0 + 2 * C::RSZ);   // [R][3][NT] (F_x,c , v_c)
    float2* ty = ring + C::RING;          // [3][VH][TK]  (F_y,c , v_c)
    float2* tz = ty + C::TY;              // [3][TJ][VW]  (F_z,c , v_c)
    uint64_t* bars = reinterpret_cast<uint64_t*>(tz + C::TZ);   // centre 0, 1; ring 0, 1

    const Layout& L = a.L;
    const int cs = (int)L.cstride;
    const int n0 = B.n[0], n1 = B.n[1], n2 = B.n[2];
    const int tid = threadIdx.x;
    const int tk = tid % TK, tj = tid / TK;
    // tiles, ownership and the shifted last tiles as in the tiled kernel
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
    const long long wlim = sa.wait_limit != 0 ? sa.wait_limit : (1LL << 22);

    const int s0 = (int)L.s0, s1 = (int)L.s1;
    const int colbase = B.lo[0] * s0 + (B.lo[1] + j) * s1 + (B.lo[2] + k);
    float* __restrict__ DFg = a.DF;
    float* __restrict__ Fn = a.Fn;

    // staged box origins: global k at the 16-byte boundary at or below the
    // first needed column (may be negative: zero fill), global j and i
    const int kgc = B.lo[2] + k0 - H;
    const int kofs = ((kgc % 4) + 4) % 4;
    const int kgb = kgc - kofs;
    const int kgr = B.lo[2] + k0;
    const int kofr = kgr % 4;
    const int krs = kgr - kofr;
    const int jgc = B.lo[1] + j0 - H, jgr = B.lo[1] + j0;
    const CUtensorMap* mFc = &maps.Fc[fsel];
    const CUtensorMap* mFr = &maps.Fr[fsel];

    const uint32_t bar_c[2] = {saddr(bars), saddr(bars + 1)};
    const uint32_t bar_r[2] = {saddr(bars + 2), saddr(bars + 3)};
    if (tid == 0) {
        for (int b = 0; b < 4; b++) bar_init(saddr(bars + b));
        bar_init_fence();
    }
    __syncthreads();

    // one thread: plane q of the centre stream into buffer b
    auto issue_centre = [&](int q, int b) {
        float* dst = cst0 + b * C::CSZ;
        const int ig = B.lo[0] + q;
        fence_proxy_async();
        bar_expect(bar_c[b], C::CBYTES);
        tma4(saddr(dst + C::CF), mFc, kgb, jgc, ig, 0, bar_c[b]);
        tma4(saddr(dst + C::CMY), &maps.My, kgb, jgc, ig, 3, bar_c[b]);
        tma4(saddr(dst + C::CMX), &maps.Mt, kgb, jgr, ig, 0, bar_c[b]);
        tma4(saddr(dst + C::CMZ), &maps.Mt, kgb, jgr, ig, 6, bar_c[b]);
        tma3(saddr(dst + C::CJ), &maps.Jc, kgb, jgc, ig, bar_c[b]);
    };
    // one thread: plane q of the ring stream into buffer b
    auto issue_ring = [&](int q, int b) {
        float* dst = rst0 + b * C::RSZ;
        const int ig = B.lo[0] + q;
        fence_proxy_async();
        bar_expect(bar_r[b], C::RBYTES);
        tma4(saddr(dst), mFr, krs, jgr, ig, 0, bar_r[b]);
        tma4(saddr(dst + C::RMX), &maps.Mr, krs, jgr, ig, 0, bar_r[b]);
        tma3(saddr(dst + C::RJ), &maps.Jr, krs, jgr, ig, bar_r[b]);
    };

    float crho[3], cg2l[3], cg[3], clam[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        crho[d] = (float)B.coef[d][0];
        cg2l[d] = (float)B.coef[d][1];
        cg[d] = (float)B.coef[d][2];
        clam[d] = (float)B.coef[d][3];
    }
    const float Acoef = (float)sa.A, Bcoef = (float)sa.B;
    const bool jint = (j >= NB) && (j < n1 - NB);
    const bool kint = (k >= NB) && (k < n2 - NB);
    auto mintap = [&](int i) { return i < NB ? 0 : (i >= n0 - NB ? n0 - NTB : i - H); };
    auto maxtap = [&](int i) { return i < NB ? NTB - 1 : (i >= n0 - NB ? n0 - 1 : i + H); };

    const int q0 = mintap(ib), qmax = maxtap(ie - 1);
    int r_issue = q0, r_cons = q0, c_issue = ib;
    if (tid == 0) {
        for (int n = 0; n < 2; n++) {
            if (r_issue + n <= qmax) issue_ring(r_issue + n, (r_issue + n - q0) & 1);
            if (c_issue + n < ie) issue_centre(c_issue + n, (c_issue + n - ib) & 1);
        }
    }
    r_issue = min(q0 + 2, qmax + 1);
    c_issue = min(ib + 2, ie);

    // bounded wait for every copy this CTA still has in flight, before an early
    // exit: ring planes from r_first (the one whose wait gave up, if any) and
    // centre planes from i_cons
    auto drain = [&](int r_first, int i_cons) {
        for (int q = r_first; q < r_issue; q++) bar_wait(bar_r[(q - q0) & 1], ((q - q0) >> 1) & 1, TMA_DRAIN_LIMIT);
        for (int q = i_cons; q < c_issue; q++) bar_wait(bar_c[(q - ib) & 1], ((q - ib) >> 1) & 1, TMA_DRAIN_LIMIT);
    };

    int lslot = q0 % R;
    int islot = ib % R;
    const int rslot = (n0 - 1) % R;
    const float* pDF = DFg + colbase;
    float dfn[9];
#pragma unroll
    for (int c = 0; c < 9; c++) dfn[c] = __ldcs(pDF + c * cs + ib * s0);

    for (int i = ib; i < ie; i++) {
        // ---- x window: ring planes up to maxtap(i) from the ring stream
        const int need = maxtap(i);
        while (r_cons <= need) {   // uniform: one plane per iteration in the interior
            const int b = (r_cons - q0) & 1;
            const bool ok = bar_wait(bar_r[b], ((r_cons - q0) >> 1) & 1, wlim);
            const float* rs = rst0 + b * C::RSZ + tj * RW + tk + kofr;
            float s[6], v[3];
#pragma unroll
            for (int c = 0; c < 6; c++) s[c] = rs[(3 + c) * TJ * RW];
#pragma unroll
            for (int c = 0; c < 3; c++) v[c] = rs[c * TJ * RW];
            float Fx[3];
            fluxes(rs[C::RJ], rs[C::RMX], rs[C::RMX + TJ * RW], rs[C::RMX + 2 * TJ * RW], s, Fx);
            float2* slot = ring + lslot * 3 * NT + tid;
#pragma unroll
            for (int c = 0; c < 3; c++) slot[c * NT] = make_float2(Fx[c], v[c]);
            r_cons++;
            lslot = (lslot + 1 == R) ? 0 : lslot + 1;
            if (__syncthreads_or(!ok)) {   // staging buffer b is free for the plane two ahead
                if (tid == 0) atomicOr(status, FDF_ERR_TIMEOUT);
                drain(r_cons - 1, i);   // the plane whose copy may still land, and every later one
                return;
            }
            if (r_issue <= qmax && r_issue < r_cons + 2) {
                if (tid == 0) issue_ring(r_issue, (r_issue - q0) & 1);
                r_issue++;
            }
        }
        // ---- centre plane i: flux tiles (tile and halo) and this node's values
        const int cb = (i - ib) & 1;
        const bool okc = bar_wait(bar_c[cb], ((i - ib) >> 1) & 1, wlim);
        const float* cs_ = cst0 + cb * C::CSZ;
        for (int e = tid; e < VH * TK; e += NT) {   // y fluxes: all VH rows, tile columns
            const int r = e / TK, kk = e % TK;
            const int col = kk + H + kofs;
            float sv[6];
#pragma unroll
            for (int c = 0; c < 6; c++) sv[c] = cs_[C::CF + ((3 + c) * VH + r) * CW + col];
            float Fy[3];
            fluxes(cs_[C::CJ + r * CW + col], cs_[C::CMY + (0 * VH + r) * CW + col], cs_[C::CMY + (1 * VH + r) * CW + col],
                   cs_[C::CMY + (2 * VH + r) * CW + col], sv, Fy);
#pragma unroll
            for (int c = 0; c < 3; c++) ty[(c * VH + r) * TK + kk] = make_float2(Fy[c], cs_[C::CF + (c * VH + r) * CW + col]);
        }
        for (int e = tid; e < TJ * VW; e += NT) {   // z fluxes: tile rows, all VW columns
            const int rr = e / VW, w = e % VW;
            const int r = rr + H, col = w + kofs;
            float sv[6];
#pragma unroll
            for (int c = 0; c < 6; c++) sv[c] = cs_[C::CF + ((3 + c) * VH + r) * CW + col];
            float Fz[3];
            fluxes(cs_[C::CJ + r * CW + col], cs_[C::CMZ + (0 * TJ + rr) * CW + col],
                   cs_[C::CMZ + (1 * TJ + rr) * CW + col], cs_[C::CMZ + (2 * TJ + rr) * CW + col], sv, Fz);
#pragma unroll
            for (int c = 0; c < 3; c++) tz[(c * TJ + rr) * VW + w] = make_float2(Fz[c], cs_[C::CF + (c * VH + r) * CW + col]);
        }
        float f[9], m[9];
        {
            const int col = tk + H + kofs, r = tj + H;
#pragma unroll
            for (int c = 0; c < 9; c++) f[c] = cs_[C::CF + (c * VH + r) * CW + col];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                m[c] = cs_[C::CMX + (c * TJ + tj) * CW + col];
                m[3 + c] = cs_[C::CMY + (c * VH + r) * CW + col];
                m[6 + c] = cs_[C::CMZ + (c * TJ + tj) * CW + col];
            }
        }
        const float Jc = cs_[C::CJ + (tj + H) * CW + tk + H + kofs];
        if (__syncthreads_or(!okc)) {   // flux tiles ready; centre buffer cb free
            if (tid == 0) atomicOr(status, FDF_ERR_TIMEOUT);
            drain(r_cons, i);
            return;
        }
        if (c_issue < ie) {
            if (tid == 0) issue_centre(c_issue, (c_issue - ib) & 1);
            c_issue++;
        }

        // ---- derivatives
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
        // closure rows this tile does not write may have taps outside the tile:
        // they take the interior form (taps in the tile and its halo), discarded
        const bool jskip = !jint && !ownj;
        const bool kskip = !kint && !ownk;
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
        if (kint || kskip) {
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
            const bool left = k < NB;
            const int row = left ? k + 1 : n2 - k;
            const int base = (left ? 0 : n2 - 1) - k0 + H, step = left ? 1 : -1;
            const float sg = left ? 1.f : -1.f;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float af = 0.f, av = 0.f;
                for (int n = 0; n < NTB; n++) {
                    const float cf = sbp_coef<float>(ORDER, row, n);
                    const float2 p = tz[(c * TJ + tj) * VW + base + n * step];
                    af = fmaf(cf, p.x, af);
                    av = fmaf(cf, p.y, av);
                }
                DFl[2][c] = sg * af;
                Dv[2][c] = sg * av;
            }
        }
        __syncthreads();   // flux tiles are rewritten for the next plane

        // ---- rate: df = A df + L(f), outer SATs, RK update
        float df[9];
#pragma unroll
        for (int c = 0; c < 9; c++) df[c] = dfn[c] * Acoef;
        if (i + 1 < ie) {   // rate register of the next plane
#pragma unroll
            for (int c = 0; c < 9; c++) dfn[c] = __ldcs(pDF + c * cs + (i + 1) * s0);
        }
        const float iJ = __frcp_rn(Jc);
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const float w = crho[d] * iJ;
            const float ma = m[3 * d], mb = m[3 * d + 1], mc = m[3 * d + 2];
            df[0] = fmaf(w, DFl[d][0], df[0]);
            df[1] = fmaf(w, DFl[d][1], df[1]);
            df[2] = fmaf(w, DFl[d][2], df[2]);
            const float dvx = Dv[d][0], dvy = Dv[d][1], dvz = Dv[d][2];
            df[3] += cg2l[d] * ma * dvx + clam[d] * (mb * dvy + mc * dvz);
            df[4] += cg[d] * (ma * dvy + mb * dvx);
            df[5] += cg[d] * (ma * dvz + mc * dvx);
            df[6] += cg2l[d] * mb * dvy + clam[d] * (ma * dvx + mc * dvz);
            df[7] += cg[d] * (mb * dvz + mc * dvy);
            df[8] += cg2l[d] * mc * dvz + clam[d] * (ma * dvx + mb * dvy);
        }
        bool defer = false;
        const bool face = (i == 0) | (i == n0 - 1) | (j == 0) | (j == n1 - 1) | (k == 0) | (k == n2 - 1);
        if (face) {
            const int pos[3] = {i, j, k};
#pragma unroll
            for (int fc = 0; fc < 6; fc++) {
                const int d = fc / 2;
                const bool at = (fc % 2 == 0) ? (pos[d] == 0) : (pos[d] == B.n[d] - 1);
                if (!at) continue;
                if (B.defer[fc]) defer = true;
                if (!B.bactive[fc]) continue;
                const int fa = (d == 0) ? j : i;
                const int fb = (d == 2) ? j : k;
                // the SAT reads and writes through pointers: work on copies so that
                // f and df stay in registers on every other node
                float fl[9], dl[9];
#pragma unroll
                for (int c = 0; c < 9; c++) {
                    fl[c] = f[c];
                    dl[c] = df[c];
                }
                boundary_sat<float, 3, 2>(B, fc, fa, fb, (float)sa.dt, fl, dl, false);
#pragma unroll
                for (int c = 0; c < 9; c++) df[c] = dl[c];
            }
        }
        if (owner) {
            const int id = colbase + i * s0;
#pragma unroll
            for (int c = 0; c < 9; c++) __stcs(DFg + c * cs + id, df[c]);
            if (!defer) {
                float fn[9];
#pragma unroll
                for (int c = 0; c < 9; c++) fn[c] = fmaf(Bcoef, df[c], f[c]);
                if (sa.last && sa.plastic) {   // return map: indexes its copy by the layout
                    float fl[9];
#pragma unroll
                    for (int c = 0; c < 9; c++) fl[c] = fn[c];
                    finish_node<float>(L, B, sa, a.s0, a.S, nullptr, a.FP, a.plastic_tensor, id, fl, false);
#pragma unroll
                    for (int c = 0; c < 9; c++) fn[c] = fl[c];
                }
#pragma unroll
                for (int c = 0; c < 9; c++) __stcs(Fn + c * cs + id, fn[c]);
            }
        }
        islot = (islot + 1 == R) ? 0 : islot + 1;
    }
}

template <int ORDER>
void launch_order(const VolumeArgs<float>& a, const BlockDev& b, const StageArgs& sa, int* status,
                  const StagedMapsHost& mh, cudaStream_t s) {
    using C = StCfg<ORDER>;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    // the shared-memory opt-in is a per-device function attribute: set it once per device
    static std::atomic<unsigned> configured{0};
    const unsigned bit = 1u << (dev & 31);
    if (!(configured.load() & bit)) {
        cudaFuncSetAttribute(k_tma3d<ORDER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
        configured.fetch_or(bit);
    }
    const int tk = (b.n[2] + TK - 1) / TK, tj = (b.n[1] + TJ - 1) / TJ;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // one resident CTA per SM: enough x chunks for a few waves
    int chunks = (3 * nsm + tk * tj - 1) / (tk * tj);
    if (chunks < 1) chunks = 1;
    int chunk = (b.n[0] + chunks - 1) / chunks;
    if (chunk < 16) chunk = 16;
    chunks = (b.n[0] + chunk - 1) / chunk;
    dim3 grid(tk, tj, chunks);
    const int fsel = (a.F == mh.F0) ? 0 : 1;
    k_tma3d<ORDER><<<grid, NT, C::SMEM, s>>>(a, b, sa, chunk, status, mh.m, fsel);
}

}  // namespace

StagedMapsHost* make_staged_maps(const Layout& L, const float* F0, const float* F1, const float* M, const float* J,
                                 int order) {
    const int H = order - 1, VH = TJ + 2 * H;
    StagedMapsHost* h = new StagedMapsHost;
    h->F0 = F0;
    h->order = order;
    const cuuint64_t d4[4] = {(cuuint64_t)L.s1, (cuuint64_t)L.nx[1], (cuuint64_t)L.nx[0], 9};
    const cuuint64_t s4[3] = {(cuuint64_t)L.s1 * 4, (cuuint64_t)L.s0 * 4, (cuuint64_t)L.cstride * 4};
    const cuuint64_t d3[3] = {(cuuint64_t)L.s1, (cuuint64_t)L.nx[1], (cuuint64_t)L.nx[0]};
    const cuuint32_t bFc[4] = {CW, (cuuint32_t)VH, 1, 9}, bFr[4] = {RW, TJ, 1, 9};
    const cuuint32_t bMy[4] = {CW, (cuuint32_t)VH, 1, 3}, bMt[4] = {CW, TJ, 1, 3}, bMr[4] = {RW, TJ, 1, 3};
    const cuuint32_t bJc[3] = {CW, (cuuint32_t)VH, 1}, bJr[3] = {RW, TJ, 1};
    try {
        const float* F[2] = {F0, F1};
        for (int b = 0; b < 2; b++) {
            tma_encode(&h->m.Fc[b], F[b], 4, d4, s4, bFc);
            tma_encode(&h->m.Fr[b], F[b], 4, d4, s4, bFr);
        }
        tma_encode(&h->m.My, M, 4, d4, s4, bMy);
        tma_encode(&h->m.Mt, M, 4, d4, s4, bMt);
        tma_encode(&h->m.Mr, M, 4, d4, s4, bMr);
        tma_encode(&h->m.Jc, J, 3, d3, s4, bJc);
        tma_encode(&h->m.Jr, J, 3, d3, s4, bJr);
    } catch (...) {
        delete h;
        throw;
    }
    return h;
}

void free_staged_maps(StagedMapsHost* h) { delete h; }

bool staged3d_supported(const Layout& L, const BlockDev& b, int order) {
    if (b.mat) return false;   // one material per block
    if (L.ndim != 3 || L.nfields != 9) return false;
    if (order < 2 || order > 4) return false;
    if (b.n[1] < TJ || b.n[2] < TK) return false;
    if (b.n[0] < 4 * order - 3) return false;
    if (L.cstride * 9 >= (1LL << 31)) return false;   // 32-bit element offsets of the stores
    if (L.s1 % 4 != 0 || L.s0 % 4 != 0 || L.cstride % 4 != 0) return false;   // 16-byte row starts
    return true;
}

void launch_volume_staged3d(const VolumeArgs<float>& a, const BlockDev& b, const StageArgs& sa, int* status,
                            const StagedMapsHost* maps, cudaStream_t s) {
    if (a.cdiss > 0.) {
        launch_volume_exact<float>(a, b, sa, s);   // artificial dissipation: exact-order kernel
        return;
    }
    if (!maps || maps->order != a.order) throw std::runtime_error("staged kernel: tensor maps missing");
    switch (a.order) {
        case 2: launch_order<2>(a, b, sa, status, *maps, s); break;
        case 3: launch_order<3>(a, b, sa, status, *maps, s); break;
        default: launch_order<4>(a, b, sa, status, *maps, s); break;
    }
}

}  // namespace fdf
