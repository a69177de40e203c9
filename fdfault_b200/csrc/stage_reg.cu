// Register-window FP32 volume kernel for 3D blocks (volume kernel kind 3).
//
// Same discrete operator as the reference's calc_df_3d (src/block.cpp:
// 1541-2050), outer SAT (src/boundary.cpp:265-503) and RK update
// (src/fields.cpp:293-309) as the tiled kernel in stage_fast.cu, with the
// memory traffic organised so that no thread waits on a DRAM load of its own:
//  * each CTA owns an 8 x 32 tile of (j, k) columns of one block (12 x 16 over
//    the last k columns when n2 mod 32 is small) and marches along x through
//    a chunk of planes; two CTAs share an SM;
//  * every plane's tile data arrives by TMA tensor copies into one of two
//    shared-memory stages, issued by one thread a plane ahead and counted on
//    an mbarrier: the centre plane i (fields, metric, Jacobian, rate register)
//    and the leading plane i+H (fields, x metric row, Jacobian) from which
//    the x fluxes J (m_x . sigma_c) and velocities enter the x window;
//  * the x window of the interior stencil (planes i-H .. i+H of the thread's
//    own column: three fluxes and three velocities each) lives in registers,
//    so shared memory holds only the two stages and the y/z flux tiles; a
//    chunk fills its window by tensor copies through its second stage;
//  * the y and z derivative inputs of the centre plane go to shared tiles
//    with an (order-1) halo.  The centre boxes are staged 4 columns wider on
//    each side, so the k halo comes from the stage; the j halo rows are loaded
//    a plane ahead into registers by the threads that own them;
//  * interior stencils are unrolled in the antisymmetric form with immediate
//    coefficients; y closure rows use the tabulated rows and the k-edge
//    tiles use one tap row per lane, as in stage_fast.cu;
//  * the 2(order-1) planes at each x face, whose closure rows reach 3(order-1)
//    planes, take their x derivatives from a pre-pass (k_prepass3d) that
//    forms them from the stage-start fields in global memory;
//  * plastic stages: the face-node kernel applies the return map to face
//    nodes and k_return_map3 to the others on the last stage;
//  * outer SATs: the same pre-pass (one thread per k-face node) evaluates
//    the SAT increments of the two k faces from the stage-start fields into a
//    compact per-block buffer; the k-edge tiles stage their rows of it with
//    the plane and finish k-face nodes themselves, so their stores stay whole
//    rows; nodes on x or y faces are written without those faces' SATs and
//    finished by the face-node kernel of stage_fast.cu (coalesced along k).
// Each staged box is one tensor copy over a (k, j, i, component) map.  Tiles
// start on 4-column (16-byte) boundaries: the last tile of a row is moved up
// to one and its columns past the block face are computed and dropped.  Every
// mbarrier wait is bounded: on expiry the CTA records FDF_ERR_TIMEOUT, waits
// (bounded) for the copies it still has in flight and returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels.hpp"
#include "sbp_coeffs.cuh"
#include "stage_common.cuh"
#include "tma_util.cuh"

namespace fdf {

// tensor maps of the FP32 arrays for kind 3 (F: both field buffers; M9: the
// nine metric rows; M3: the x metric rows; DF: the rate register)
struct RegMaps {
    CUtensorMap F[2], M9, J;        // centre plane: 4 halo columns on each side
    CUtensorMap FL[2], M3, JL, DF;  // leading plane and rate register: the tile's columns
};

struct RegMapsHost {
    RegMaps m, me;   // boxes of the main tiles and of the narrower last-column tiles
    const float* F0;
    // per block: k-face SAT increments [side][c][i][jp] and their tensor maps (both tile heights)
    std::vector<float*> ksat;
    std::vector<int> jp;
    std::vector<CUtensorMap> kmap, ekmap;
    // per block: x derivatives of the closure planes [slot][q][j][k] (see xcl_block)
    std::vector<float*> xcl;
    ~RegMapsHost() {
        for (float* p : ksat)
            if (p) cudaFree(p);
        for (float* p : xcl)
            if (p) cudaFree(p);
    }
};

namespace {

// tile shapes (j rows x k columns): the main tiles, and the narrower tile
// that covers the last k columns of a block when n2 mod 32 is small (12 x 16,
// 192 of the launch's 256 threads), so those columns are not computed twice
constexpr int TJM = 8, TKM = 32, TJE = 12, TKE = 16;
constexpr int NTL = 256;          // threads per CTA of the launch
constexpr int KH = 4;             // halo columns staged on each side of the centre boxes (>= H, 16 bytes)

constexpr int up32(int n) { return (n + 31) / 32 * 32; }   // every box on a 128-byte boundary

template <int ORDER, int TJ_ = TJM, int TK_ = TKM>
struct RgCfg {
    static constexpr int TJ = TJ_, TK = TK_, NT = TJ * TK;
    static constexpr int SWC = TK + 2 * KH;  // staged centre row
    static constexpr int SWD = TK;           // staged row of the rate register and the leading plane
    static constexpr int KBJ = TJ + 4;       // staged k-face row: 16-byte boundary at or below the first j
    static constexpr int H = ORDER - 1, NB = 2 * H, NTB = 3 * H, W = 2 * H + 1;
    static constexpr int VH = TJ + 2 * H, VW = TK + 2 * H;
    static constexpr int BOXC = TJ * SWC, BOXD = TJ * SWD;   // floats of one staged component
    // stage layout, floats: centre F[9], M[9], J (BOXC each); DF[9], leading
    // F[9], Mx[3], J (BOXD each).  k-edge tiles also stage their rows of the
    // k-face SAT increments: per face side one box of KBJ j x 9 components
    static constexpr int CF = 0, CM = CF + up32(9 * BOXC), CJ = CM + up32(9 * BOXC), CD = CJ + up32(BOXC),
                         LF = CD + up32(9 * BOXD), LM = LF + up32(9 * BOXD), LJ = LM + up32(3 * BOXD),
                         KSW = up32(9 * KBJ), KS = LJ + up32(BOXD), SSZ = KS + 2 * KSW;
    static constexpr uint32_t BYTES = 4u * (19 * BOXC + 22 * BOXD), KBYTES = 4u * 9 * KBJ;
    // window fill of a chunk: leading-plane boxes (13 components) of up to PR
    // planes at a time in one stage
    static constexpr uint32_t LBYTES = 4u * 13 * BOXD;
    static constexpr int PR = SSZ / (13 * BOXD) < 3 ? SSZ / (13 * BOXD) : 3;
    static constexpr int TY = 3 * VH * TK, TZ = 3 * TJ * VW;   // float2
    static constexpr int WROWS = 2 * NB + 1;
    static constexpr int WTAB = ((WROWS * NTB + 3) / 4) * 4;
    static constexpr size_t SMEM =
        sizeof(float) * 2 * SSZ + sizeof(float2) * (TY + TZ) + sizeof(float) * WTAB + 7 * sizeof(uint64_t);
};
// dynamic shared memory of a launch: the larger of the two shapes
template <int ORDER>
constexpr size_t reg_smem() {
    return RgCfg<ORDER, TJM, TKM>::SMEM > RgCfg<ORDER, TJE, TKE>::SMEM ? RgCfg<ORDER, TJM, TKM>::SMEM
                                                                         : RgCfg<ORDER, TJE, TKE>::SMEM;
}

// one CTA's tile: origin, tile indices, the last tiles in k and j, and the k
// columns it owns away from the closure rows
struct RegTile {
    int k0, j0, bx, by, kown0, kown1;
    bool lastk, lastj;
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

struct HaloNode {
    float s[6], v[3], m[3], J;
};

// (flux, velocity) pairs go through the paired FP32 instructions of sm_100
// (each lane rounds as the scalar instruction would)
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 fma2(float a, float2 x, float2 acc) { return __ffma2_rn(make_float2(a, a), x, acc); }

template <int ORDER, int TJ, int TK>
__device__ __forceinline__ void reg_march(const VolumeArgs<float>& a, const BlockDev& B, const StageArgs& sa,
                                          int chunk, int* status, const RegMaps& maps, int fsel,
                                          const CUtensorMap& kmap, const float* __restrict__ xcl, const RegTile& T) {
    using C = RgCfg<ORDER, TJ, TK>;
    constexpr int H = C::H, NB = C::NB, NTB = C::NTB, W = C::W, VH = C::VH, VW = C::VW, BOXC = C::BOXC,
                  BOXD = C::BOXD;
    constexpr int NT = C::NT, SWC = C::SWC, SWD = C::SWD, KBJ = C::KBJ;
    extern __shared__ __align__(128) float smem[];
    float* stg = smem;                                            // two stages of C::SSZ floats
    float2* ty = reinterpret_cast<float2*>(smem + 2 * C::SSZ);   // [3][VH][TK]  (F_y,c , v_c)
    float2* tz = ty + C::TY;                                     // [3][TJ][VW]  (F_z,c , v_c)
    float* wtab = reinterpret_cast<float*>(tz + C::TZ);          // [WROWS][NTB]
    uint64_t* bars = reinterpret_cast<uint64_t*>(wtab + C::WTAB);

    const Layout& L = a.L;
    const int cs = (int)L.cstride;
    const int n0 = B.n[0], n1 = B.n[1], n2 = B.n[2];
    const int tid = threadIdx.x;   // threads from NT on (the narrower tile) only share the set-up barriers
    const int tk = tid % TK, tj = tid / TK;
    // tiles and ownership as in stage_fast.cu: the last tile in j ends on the
    // block face, the last tile in k at or up to 3 columns past it (its first
    // column on a 4-column boundary); each owns the closure rows near its face
    const bool lastk = T.lastk, lastj = T.lastj;
    const int k0 = T.k0, j0 = T.j0;
    const int k = k0 + tk, j = j0 + tj;
    const bool ownk = (k >= n2) ? false : (k >= n2 - NB) ? lastk : (k >= T.kown0 && k < T.kown1);
    const bool ownj = (j >= n1 - NB) ? lastj : (j / TJ == T.by);
    const bool owner = ownk && ownj;
    // chunks tile the planes this process updates, [xb, xe); the x window and
    // the closure tests stay in block coordinates
    const int ib = B.xb + blockIdx.z * chunk;
    const int ie = min(B.xe, ib + chunk);
    if (ib >= ie) return;
    const long long wlim = sa.wait_limit != 0 ? sa.wait_limit : (1LL << 22);

    // staged boxes: the tile's first column kg is on a 16-byte boundary (the
    // block's first k is, by the support check); centre boxes start KH before it
    const int kg = B.lo[2] + k0;
    const int jg = B.lo[1] + j0;
    const CUtensorMap* mF = &maps.F[fsel];
    const CUtensorMap* mFL = &maps.FL[fsel];
    const uint32_t bar0 = saddr(bars), bar1 = saddr(bars + 1);
    // warp-arrival barriers of the march (one arrival per warp and plane):
    // flux tiles written, flux tiles read, stage consumed
    constexpr uint32_t NWARP = NT / 32;
    const uint32_t barT = saddr(bars + 2), barR = saddr(bars + 3), barS = saddr(bars + 4);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 5);
    const int lane = tid & 31;

    const bool kedge = (T.bx == 0) || lastk;
    // k faces whose SAT increments this tile stages (outer faces with a SAT)
    const bool kf0 = (T.bx == 0) && B.bactive[4], kf1 = lastk && B.bactive[5];
    const int kjb = j0 & ~3;   // k-face box origin in j (block coordinates)
    const uint32_t bytes = C::BYTES + (kf0 ? C::KBYTES : 0u) + (kf1 ? C::KBYTES : 0u);
    if (tid == 0) {
        bar_init(bar0);
        bar_init(bar1);
        bar_init(saddr(bars + 6));   // window fill
        bar_init_count(barT, NWARP);
        bar_init_count(barR, NWARP);
        bar_init_count(barS, NWARP);
        *abort_flag = 0;
        bar_init_fence();
    }
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
    __syncthreads();

    // one thread: centre plane i and leading plane i+H into stage b
    auto issue = [&](int i, int b) {
        float* st = stg + b * C::SSZ;
        const uint32_t bar = b ? bar1 : bar0;
        const int ig = B.lo[0] + i;
        fence_proxy_async();
        bar_expect(bar, bytes);
        tma4(saddr(st + C::CF), mF, kg - KH, jg, ig, 0, bar);
        tma4(saddr(st + C::CM), &maps.M9, kg - KH, jg, ig, 0, bar);
        tma3(saddr(st + C::CJ), &maps.J, kg - KH, jg, ig, bar);
        tma4(saddr(st + C::CD), &maps.DF, kg, jg, ig, 0, bar);
        tma4(saddr(st + C::LF), mFL, kg, jg, ig + H, 0, bar);
        tma4(saddr(st + C::LM), &maps.M3, kg, jg, ig + H, 0, bar);
        tma3(saddr(st + C::LJ), &maps.JL, kg, jg, ig + H, bar);
        if (kf0) tma3(saddr(st + C::KS), &kmap, kjb, i, 0, bar);
        if (kf1) tma3(saddr(st + C::KS + C::KSW), &kmap, kjb, i, 9, bar);
    };
    // a chunk that starts past the left closure rows fills its x window first
    // through stage 1 (below), which takes plane ib+1 after that
    const bool prefill = ib >= NB && ib < n0 - NB;
    if (tid == 0) {
        issue(ib, 0);
        if (ib + 1 < ie && !prefill) issue(ib + 1, 1);
    }
    int issued = min(ie, ib + 2);   // planes whose stage was issued (uniform over the CTA)

    // this lane's k-edge row: tap n reads column kb + ks * min(n, kmax) of its tz row
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
    if (tid < 2 * H * (TK + TJ)) {
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
    // j-halo nodes: loaded a plane ahead from global memory (metric rows 3-5)
    auto load_halo = [&](int i, HaloNode& h) {
        if (hkind != 0) return;
        const int id = hbase + i * s0;
#pragma unroll
        for (int c = 0; c < 6; c++) h.s[c] = __ldg(F + (3 + c) * cs + id);
#pragma unroll
        for (int c = 0; c < 3; c++) h.v[c] = __ldg(F + c * cs + id);
#pragma unroll
        for (int c = 0; c < 3; c++) h.m[c] = __ldg(M + (3 + c) * cs + id);
        h.J = __ldg(Jg + id);
    };

    float crho[3], sd[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        crho[d] = (float)B.coef[d][0];
        sd[d] = (float)(sa.dt / B.dx[d]);
    }
    const float lamc = (float)B.lam, gc = (float)B.g, g2c = (float)(2. * B.g);
    const float Acoef = (float)sa.A, Bcoef = (float)sa.B;
    const bool jint = (j >= NB) && (j < n1 - NB);
    const bool facexy = (j == 0) | (j == n1 - 1);   // (x faces: planes 0 and n0-1)
    // this node's k face: 0 none, 1 SAT increment staged, 2 interface (finished there)
    int kface = 0, kside = 0;
    if (k == 0 || k == n2 - 1) {
        kside = (k == 0) ? 0 : 1;
        kface = B.defer[4 + kside] ? 2 : (B.bactive[4 + kside] ? 1 : 0);
    }

    const int sod = tj * SWD + tk;   // this node in a staged rate or leading-plane component
    // x window: after the insert at plane i, w[m][c] holds the pair
    // (F_x,c , v_c) of plane i - H + m.  A chunk that starts past the left
    // closure rows fills planes ib-H..ib+H-1 first: tensor copies of their
    // leading-plane boxes, up to PR planes per round, through stage 1 (free
    // until plane ib+1 is issued into it); the first chunk builds its window
    // from the inserts.
    float2 w[W][3];
#pragma unroll
    for (int m = 0; m < W; m++)
#pragma unroll
        for (int c = 0; c < 3; c++) w[m][c] = make_float2(0.f, 0.f);
    if (prefill) {
        constexpr int NPF = W - 1, PR = C::PR, PLN = 13 * BOXD;
        float* pst = stg + C::SSZ;
        const uint32_t barP = saddr(bars + 6);
#pragma unroll
        for (int t = 0; t < NPF; t++) {
            const int p = t % PR, round = t / PR;
            if (p == 0) {
                const int np = min(PR, NPF - t);
                if (tid == 0) {
                    fence_proxy_async();
                    bar_expect(barP, (uint32_t)np * C::LBYTES);
                    for (int q = 0; q < np; q++) {
                        const int ig = B.lo[0] + ib - H + t + q;
                        float* d = pst + q * PLN;
                        tma4(saddr(d), mFL, kg, jg, ig, 0, barP);
                        tma4(saddr(d + 9 * BOXD), &maps.M3, kg, jg, ig, 0, barP);
                        tma3(saddr(d + 12 * BOXD), &maps.JL, kg, jg, ig, barP);
                    }
                }
                if (!bar_wait(barP, round & 1, wlim)) *abort_flag = 1;
                // the issuing thread also sees the copies land before it reuses the space
                if (tid == 0 && !bar_wait(barP, round & 1, TMA_DRAIN_LIMIT)) *abort_flag = 1;
            }
            if (tid < NT) {
                const float* d = pst + p * PLN;
                float s[6], Fx[3];
#pragma unroll
                for (int c = 0; c < 6; c++) s[c] = d[(3 + c) * BOXD + sod];
                fluxes(d[12 * BOXD + sod], d[9 * BOXD + sod], d[10 * BOXD + sod], d[11 * BOXD + sod], s, Fx);
#pragma unroll
                for (int c = 0; c < 3; c++) w[t + 1][c] = make_float2(Fx[c], d[c * BOXD + sod]);
            }
            if (p == PR - 1 || t == NPF - 1) __syncthreads();   // round read before the space is refilled
        }
        if (tid == 0 && ib + 1 < ie) issue(ib + 1, 1);
    }
    if (tid >= NT) return;   // no part in the march (its barriers count NT / 32 warps)
    HaloNode hn;
    load_halo(ib, hn);

    const int so = tj * SWC + tk + KH;   // this node in a staged centre component
    const int hso = hj * SWC + hk + KH;  // the k-halo node in a staged centre component
    for (int i = ib; i < ie; i++) {
        const int kk = i - ib;
        const int b = kk & 1;
        const float* st = stg + b * C::SSZ;
        if (kk > 0) {
            // every warp has read plane i-1's flux tiles (they are rewritten below);
            // once every warp is also done with plane i-1's stage, plane i+1 goes into it
            if (!bar_wait(barR, (kk - 1) & 1, TMA_DRAIN_LIMIT)) *abort_flag = 1;
            if (tid == 0 && issued < ie) {
                if (bar_wait(barS, (kk - 1) & 1, TMA_DRAIN_LIMIT))
                    issue(issued, (issued - ib) & 1);
                else
                    *abort_flag = 1;
            }
            if (issued < ie) issued++;
        }
        if (!bar_wait(b ? bar1 : bar0, (kk >> 1) & 1, wlim)) *abort_flag = 1;
        // ---- centre plane i: y/z flux tiles of the tile and of this thread's halo node
        {
            float s[6], Fy[3], Fz[3];
#pragma unroll
            for (int c = 0; c < 6; c++) s[c] = st[C::CF + (3 + c) * BOXC + so];
            const float Jc = st[C::CJ + so];
            fluxes(Jc, st[C::CM + 3 * BOXC + so], st[C::CM + 4 * BOXC + so], st[C::CM + 5 * BOXC + so], s, Fy);
            fluxes(Jc, st[C::CM + 6 * BOXC + so], st[C::CM + 7 * BOXC + so], st[C::CM + 8 * BOXC + so], s, Fz);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float v = st[C::CF + c * BOXC + so];
                ty[(c * VH + tj + H) * TK + tk] = make_float2(Fy[c], v);
                tz[(c * TJ + tj) * VW + tk + H] = make_float2(Fz[c], v);
            }
        }
        if (hkind == 0) {
            float Fh[3];
            fluxes(hn.J, hn.m[0], hn.m[1], hn.m[2], hn.s, Fh);
#pragma unroll
            for (int c = 0; c < 3; c++) ty[(c * VH + hj + H) * TK + hk] = make_float2(Fh[c], hn.v[c]);
        } else if (hkind == 1) {   // k halo: from the staged centre boxes
            float s[6], Fh[3];
#pragma unroll
            for (int c = 0; c < 6; c++) s[c] = st[C::CF + (3 + c) * BOXC + hso];
            fluxes(st[C::CJ + hso], st[C::CM + 6 * BOXC + hso], st[C::CM + 7 * BOXC + hso],
                   st[C::CM + 8 * BOXC + hso], s, Fh);
#pragma unroll
            for (int c = 0; c < 3; c++)
                tz[(c * TJ + hj) * VW + hk + H] = make_float2(Fh[c], st[C::CF + c * BOXC + hso]);
        }
        __syncwarp();
        if (lane == 0) bar_arrive(barT);
        // work that the flux tiles do not wait for: the next halo node's loads
        // and the leading plane's entry into the x window
        if (i + 1 < ie) load_halo(i + 1, hn);
        // ---- leading plane i+H enters the x window
        if (i + H < n0) {
            float s[6], v[3], Fx[3];
#pragma unroll
            for (int c = 0; c < 6; c++) s[c] = st[C::LF + (3 + c) * BOXD + sod];
#pragma unroll
            for (int c = 0; c < 3; c++) v[c] = st[C::LF + c * BOXD + sod];
            fluxes(st[C::LJ + sod], st[C::LM + sod], st[C::LM + BOXD + sod], st[C::LM + 2 * BOXD + sod], s, Fx);
#pragma unroll
            for (int m = 0; m < W - 1; m++)
#pragma unroll
                for (int c = 0; c < 3; c++) w[m][c] = w[m + 1][c];
#pragma unroll
            for (int c = 0; c < 3; c++) w[W - 1][c] = make_float2(Fx[c], v[c]);
        }

        // ---- derivatives: D[d][c] = (d/dxi_d of the flux F_d,c , of the velocity v_c)
        float2 D[3][3];
        if (i >= NB && i < n0 - NB) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float2 acc = make_float2(0.f, 0.f);
#pragma unroll
                for (int n = 1; n <= H; n++) acc = fma2(inner_c<ORDER>(n), sub2(w[H + n][c], w[H - n][c]), acc);
                D[0][c] = acc;
            }
        } else {   // x closure rows: from the pre-pass
            const int slot = (i < NB) ? i : NB + i - (n0 - NB);
            const long long pl = (long long)n1 * n2;
            const float* xc = xcl + (long long)slot * 6 * pl + (long long)j * n2 + min(k, n2 - 1);
#pragma unroll
            for (int c = 0; c < 3; c++) D[0][c] = make_float2(xc[2 * c * pl], xc[(2 * c + 1) * pl]);
        }
        // flux tiles of plane i complete; a wait that ran out anywhere ends the CTA
        if (!bar_wait(barT, kk & 1, TMA_DRAIN_LIMIT) || *abort_flag) {
            if (tid == 0) {
                atomicOr(status, FDF_ERR_TIMEOUT);
                // wait for the copies still in flight before the CTA leaves
                for (int q = i; q < issued; q++)
                    bar_wait((q - ib) & 1 ? bar1 : bar0, ((q - ib) >> 1) & 1, TMA_DRAIN_LIMIT);
            }
            return;
        }
        // closure rows this tile does not write may have taps outside the tile:
        // they take the interior form (taps in the tile and its halo), discarded
        const bool jskip = !jint && !ownj;
        if (jint || jskip) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float2 acc = make_float2(0.f, 0.f);
#pragma unroll
                for (int n = 1; n <= H; n++)
                    acc = fma2(inner_c<ORDER>(n),
                               sub2(ty[(c * VH + tj + H + n) * TK + tk], ty[(c * VH + tj + H - n) * TK + tk]), acc);
                D[1][c] = acc;
            }
        } else {
            const bool left = j < NB;
            const int row = left ? j + 1 : n1 - j;
            const int base = (left ? 0 : n1 - 1) - j0 + H, step = left ? 1 : -1;
            const float sg = left ? 1.f : -1.f;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float2 acc = make_float2(0.f, 0.f);
                for (int n = 0; n < NTB; n++)
                    acc = fma2(sbp_coef<float>(ORDER, row, n), ty[(c * VH + base + n * step) * TK + tk], acc);
                D[1][c] = __fmul2_rn(make_float2(sg, sg), acc);
            }
        }
        if (!kedge) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float2 acc = make_float2(0.f, 0.f);
#pragma unroll
                for (int n = 1; n <= H; n++)
                    acc = fma2(inner_c<ORDER>(n),
                               sub2(tz[(c * TJ + tj) * VW + tk + H + n], tz[(c * TJ + tj) * VW + tk + H - n]), acc);
                D[2][c] = acc;
            }
        } else {
            float2 acc[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
            const float2* trow = tz + tj * VW;
#pragma unroll
            for (int n = 0; n < NTB; n++) {
                const float wt = wtab[kw + n];
                const int col = kb + ks * min(n, kmax);
#pragma unroll
                for (int c = 0; c < 3; c++) acc[c] = fma2(wt, trow[c * TJ * VW + col], acc[c]);
            }
#pragma unroll
            for (int c = 0; c < 3; c++) D[2][c] = acc[c];
        }
        float DFl[3][3], Dv[3][3];
#pragma unroll
        for (int d = 0; d < 3; d++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                DFl[d][c] = D[d][c].x;
                Dv[d][c] = D[d][c].y;
            }
        __syncwarp();
        if (lane == 0) bar_arrive(barR);   // this warp is done with the flux tiles

        // ---- rate: df = A df + L(f), then the RK update
        float df[9];
#pragma unroll
        for (int c = 0; c < 9; c++) df[c] = st[C::CD + c * BOXD + sod];
        const float iJ = __frcp_rn(st[C::CJ + so]);
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
            float m[9];
#pragma unroll
            for (int c = 0; c < 9; c++) m[c] = st[C::CM + c * BOXC + so];
            float e[3][3];
#pragma unroll
            for (int va = 0; va < 3; va++)
#pragma unroll
                for (int bb = 0; bb < 3; bb++)
                    e[va][bb] = fmaf(m[6 + bb], Dv[2][va], fmaf(m[3 + bb], Dv[1][va], m[bb] * Dv[0][va]));
            const float lt = lamc * (e[0][0] + e[1][1] + e[2][2]);
            df[3] = fmaf(Acoef, df[3], fmaf(g2c, e[0][0], lt));
            df[4] = fmaf(Acoef, df[4], gc * (e[0][1] + e[1][0]));
            df[5] = fmaf(Acoef, df[5], gc * (e[0][2] + e[2][0]));
            df[6] = fmaf(Acoef, df[6], fmaf(g2c, e[1][1], lt));
            df[7] = fmaf(Acoef, df[7], gc * (e[1][2] + e[2][1]));
            df[8] = fmaf(Acoef, df[8], fmaf(g2c, e[2][2], lt));
        }
        if (kface == 1) {   // k-face SAT increment staged by the pre-pass
            const float* ks = st + C::KS + kside * C::KSW + (j - kjb);
#pragma unroll
            for (int c = 0; c < 9; c++) df[c] += ks[c * KBJ];
        }
        if (owner) {
            const int id = colbase + i * s0;
#pragma unroll
            for (int c = 0; c < 9; c++) DFg[c * cs + id] = df[c];
            // x/y face nodes: k_faces3d adds those SATs and finishes them
            if (!(facexy | (i == 0) | (i == n0 - 1) | (kface == 2))) {
#pragma unroll
                for (int c = 0; c < 9; c++) Fn[c * cs + id] = fmaf(Bcoef, df[c], st[C::CF + c * BOXC + so]);
            }
        }
        __syncwarp();
        if (lane == 0) bar_arrive(barS);   // this warp is done with the stage of plane i
    }
}

// One launch per block and stage: blockIdx.x < tkm are the main tiles along k
// (8 x 32); with `edge` set, blockIdx.x == tkm is the column of narrower tiles
// (12 x 16) over the last k columns, which owns k >= 32 tkm.
template <int ORDER>
__global__ void __launch_bounds__(NTL, 2)
    k_reg3d(VolumeArgs<float> a, BlockDev B, StageArgs sa, int chunk, int* status, int tkm, int edge,
            const __grid_constant__ RegMaps maps, const __grid_constant__ RegMaps emaps, int fsel,
            const __grid_constant__ CUtensorMap kmap, const __grid_constant__ CUtensorMap ekmap,
            const float* __restrict__ xcl) {
    const int n1 = B.n[1], n2 = B.n[2];
    RegTile T;
    T.bx = blockIdx.x;
    T.by = blockIdx.y;
    if (edge && T.bx == tkm) {
        const int tje = (n1 + TJE - 1) / TJE;
        if (T.by >= tje) return;
        T.lastk = true;
        T.lastj = T.by == tje - 1;
        T.k0 = (n2 - TKE + 3) & ~3;
        T.j0 = T.lastj ? n1 - TJE : T.by * TJE;
        T.kown0 = tkm * TKM;
        T.kown1 = n2;
        reg_march<ORDER, TJE, TKE>(a, B, sa, chunk, status, emaps, fsel, ekmap, xcl, T);
    } else {
        const int tjm = (n1 + TJM - 1) / TJM;
        if (T.by >= tjm) return;
        T.lastk = !edge && T.bx == tkm - 1;
        T.lastj = T.by == tjm - 1;
        T.k0 = T.lastk ? ((n2 - TKM + 3) & ~3) : T.bx * TKM;
        T.j0 = T.lastj ? n1 - TJM : T.by * TJM;
        T.kown0 = T.bx * TKM;
        T.kown1 = T.kown0 + TKM;
        reg_march<ORDER, TJM, TKM>(a, B, sa, chunk, status, maps, fsel, kmap, xcl, T);
    }
}

// SAT increments of the two k faces of a block from the stage-start fields:
// ks[side][c][i][jp] = the change the face's SAT makes to the rate of node
// (i, j, k = 0 or n2-1).  One thread per face node, threads along j.
// (bx, by, side): the 32 x 4 thread block's place in the (j, i, side) grid.
__device__ __forceinline__ void ksat_block(const VolumeArgs<float>& a, const BlockDev& B, const StageArgs& sa,
                                           float* ks, int jp, int bx, int by, int side) {
    if (!B.bactive[4 + side]) return;
    const int j = bx * 32 + threadIdx.x, i = by * 4 + threadIdx.y;
    const int n1 = B.n[1];
    if (j >= n1 || i < B.xb || i >= B.xe) return;   // planes this process updates
    const int n0 = B.n[0];
    const int k = side ? B.n[2] - 1 : 0;
    const long long cs = a.L.cstride;
    const long long id = node_index(a.L, B.lo[0] + i, B.lo[1] + j, B.lo[2] + k);
    float f[9], d[9];
#pragma unroll
    for (int c = 0; c < 9; c++) {
        f[c] = a.F[c * cs + id];
        d[c] = 0.f;
    }
    boundary_sat<float, 3, 2>(B, 4 + side, i, j, (float)sa.dt, f, d, false);
    float* o = ks + (long long)side * 9 * n0 * jp + (long long)i * jp + j;
#pragma unroll
    for (int c = 0; c < 9; c++) o[(long long)c * n0 * jp] = d[c];
}

// x derivatives of the (F_x,c , v_c) pairs on the 2(order-1) closure planes
// at each x face of a block, from the stage-start fields:
// xcl[slot][q][j][k], slot 0..NB-1 planes 0..NB-1, slot NB+m plane n0-NB+m,
// q = 2c (flux) or 2c+1 (velocity).  One thread per (j, k) and face: each of
// the 3(order-1) planes the closure rows reach is loaded once.
// (bx, by, side): the 32 x 4 thread block's place in the (k, j, face) grid.
template <int ORDER>
__device__ __forceinline__ void xcl_block(const VolumeArgs<float>& a, const BlockDev& B, float* __restrict__ xcl,
                                          int bx, int by, int side) {
    constexpr int H = ORDER - 1, NB = 2 * H, NTB = 3 * H;
    const int n0 = B.n[0], n1 = B.n[1], n2 = B.n[2];
    const int k = bx * 32 + threadIdx.x, j = by * 4 + threadIdx.y;
    const bool left = side == 0;
    if (k >= n2 || j >= n1) return;
    if (B.xe <= B.xb || (left ? B.xb >= NB : B.xe <= n0 - NB)) return;   // no closure plane of this face updated here
    const float sg = left ? 1.f : -1.f;
    const int cs = (int)a.L.cstride, s0 = (int)a.L.s0;
    const int colbase = B.lo[0] * s0 + (B.lo[1] + j) * (int)a.L.s1 + (B.lo[2] + k);
    float2 acc[NB][3];
#pragma unroll
    for (int r = 0; r < NB; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) acc[r][c] = make_float2(0.f, 0.f);
#pragma unroll
    for (int n = 0; n < NTB; n++) {
        const int id = colbase + (left ? n : n0 - 1 - n) * s0;
        float s[6], v[3], Fx[3];
#pragma unroll
        for (int c = 0; c < 6; c++) s[c] = __ldg(a.F + (3 + c) * cs + id);
#pragma unroll
        for (int c = 0; c < 3; c++) v[c] = __ldg(a.F + c * cs + id);
        fluxes(__ldg(a.J + id), __ldg(a.M + id), __ldg(a.M + cs + id), __ldg(a.M + 2 * cs + id), s, Fx);
        // closure row r+1 of the plane r from the face (left: plane r, right: plane n0-1-r)
#pragma unroll
        for (int r = 0; r < NB; r++) {
            const float cf = sbp_coef<float>(ORDER, r + 1, n);
#pragma unroll
            for (int c = 0; c < 3; c++) acc[r][c] = fma2(cf, make_float2(Fx[c], v[c]), acc[r][c]);
        }
    }
    const long long pl = (long long)n1 * n2;
#pragma unroll
    for (int r = 0; r < NB; r++) {
        const int slot = left ? r : 2 * NB - 1 - r;   // right face: plane n0-1-r
        float* o = xcl + (long long)slot * 6 * pl + (long long)j * n2 + k;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const float2 d = __fmul2_rn(make_float2(sg, sg), acc[r][c]);
            o[2 * c * pl] = d.x;
            o[(2 * c + 1) * pl] = d.y;
        }
    }
}

// Both pre-passes of every block of a stage in one launch (each reads only the
// stage-start fields): thread block t belongs to the block b with
// start[b] <= t < start[b+1]; within it the first nk[b] evaluate the k-face
// SAT increments (grid kx x ky x 2), the others the closure-plane x
// derivatives (grid xx x xy x 2).  The block table is read from device memory.
struct PrepTable {
    int nblk;
    int start[FDF_ALLB_MAX + 1];
    int kx[FDF_ALLB_MAX], ky[FDF_ALLB_MAX], nk[FDF_ALLB_MAX], xx[FDF_ALLB_MAX], xy[FDF_ALLB_MAX],
        jp[FDF_ALLB_MAX];
    float* ks[FDF_ALLB_MAX];
    float* xcl[FDF_ALLB_MAX];
};

template <int ORDER>
__global__ void __launch_bounds__(128) k_prepass3d(VolumeArgs<float> a, const BlockDev* __restrict__ blks,
                                                   StageArgs sa, const __grid_constant__ PrepTable P) {
    int b = 0;
    for (int q = 1; q < P.nblk; q++)
        if ((int)blockIdx.x >= P.start[q]) b = q;
    int t = blockIdx.x - P.start[b];
    const BlockDev& B = blks[b];
    if (t < P.nk[b]) {
        ksat_block(a, B, sa, P.ks[b], P.jp[b], t % P.kx[b], (t / P.kx[b]) % P.ky[b], t / (P.kx[b] * P.ky[b]));
    } else {
        t -= P.nk[b];
        xcl_block<ORDER>(a, B, P.xcl[b], t % P.xx[b], (t / P.xx[b]) % P.xy[b], t / (P.xx[b] * P.xy[b]));
    }
}

// choose the x chunk: the grid of tiles x chunks runs in whole waves of
// `slots` resident CTAs; each chunk also pays about H planes of window set-up
int pick_chunk(int n0, int tiles, int slots, int H) {
    int best = n0, bestcost = 1 << 30;
    for (int chunks = 1; chunks <= 64; chunks++) {
        const int chunk = (n0 + chunks - 1) / chunks;
        if (chunk < 16 && chunks > 1) break;
        const int nc = (n0 + chunk - 1) / chunk;
        const int waves = (tiles * nc + slots - 1) / slots;
        const int cost = waves * (chunk + H + 1);
        if (cost < bestcost) {
            bestcost = cost;
            best = chunk;
        }
    }
    return best;
}

template <int ORDER>
void launch_order(const VolumeArgs<float>& a, const BlockDev& b, int bi, const StageArgs& sa, int* status,
                  const RegMapsHost& mh, cudaStream_t s) {
    constexpr size_t SMEM = reg_smem<ORDER>();
    constexpr int NB = 2 * (ORDER - 1);
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    // the shared-memory opt-in is a per-device function attribute: set it once per device
    static std::atomic<unsigned> configured{0};
    static int occ[32] = {0};
    const unsigned bit = 1u << (dev & 31);
    if (!(configured.load() & bit)) {
        cudaFuncSetAttribute(k_reg3d<ORDER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
        int o = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_reg3d<ORDER>, NTL, SMEM);
        occ[dev & 31] = o > 0 ? o : 1;
        configured.fetch_or(bit);
    }
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // the narrower tiles take the last k columns when n2 mod 32 leaves between
    // NB (its closure rows) and 16 columns
    const int rem = b.n[2] % TKM;
    const int edge = (rem >= NB && rem <= TKE && b.n[2] > TKM && b.n[1] >= TJE) ? 1 : 0;
    const int tkm = edge ? b.n[2] / TKM : (b.n[2] + TKM - 1) / TKM;
    const int tjm = (b.n[1] + TJM - 1) / TJM, tje = (b.n[1] + TJE - 1) / TJE;
    const int tiles = tkm * tjm + (edge ? tje : 0);
    const int nown = b.xe - b.xb;   // planes this process updates
    if (nown <= 0) return;
    const int chunk = pick_chunk(nown, tiles, occ[dev & 31] * nsm, ORDER - 1);
    const int chunks = (nown + chunk - 1) / chunk;
    dim3 grid(tkm + edge, edge ? (tjm > tje ? tjm : tje) : tjm, chunks);
    const int fsel = (a.F == mh.F0) ? 0 : 1;
    k_reg3d<ORDER><<<grid, NTL, SMEM, s>>>(a, b, sa, chunk, status, tkm, edge, mh.m, mh.me, fsel, mh.kmap[bi],
                                           mh.ekmap[bi], mh.xcl[bi]);
    // plasticity: face nodes get the return map in the face-node kernel, the
    // others (k-face nodes included, finished by the march) in their own pass
    launch_faces3d(a, b, sa, true, sa.plastic != 0, s);
    if (sa.plastic && sa.last) launch_return_map3(a, b, sa, true, s);
}

}  // namespace

RegMapsHost* make_reg_maps(const Layout& L, const float* F0, const float* F1, const float* M, const float* J,
                           const float* DF, const BlockDev* blocks, int nblocks) {
    RegMapsHost* h = new RegMapsHost;
    h->F0 = F0;
    const cuuint64_t d4[4] = {(cuuint64_t)L.s1, (cuuint64_t)L.nx[1], (cuuint64_t)L.nx[0], 9};
    const cuuint64_t s4[3] = {(cuuint64_t)L.s1 * 4, (cuuint64_t)L.s0 * 4, (cuuint64_t)L.cstride * 4};
    const cuuint64_t d3[3] = {(cuuint64_t)L.s1, (cuuint64_t)L.nx[1], (cuuint64_t)L.nx[0]};
    // one set of maps per tile shape (box tj rows; centre rows tk + 2 KH wide, others tk)
    auto encode = [&](RegMaps& m, cuuint32_t tj, cuuint32_t tk) {
        const cuuint32_t swc = tk + 2 * KH;
        const cuuint32_t c9[4] = {swc, tj, 1, 9}, c1[3] = {swc, tj, 1};
        const cuuint32_t d9[4] = {tk, tj, 1, 9}, d3b[4] = {tk, tj, 1, 3}, d1[3] = {tk, tj, 1};
        tma_encode(&m.F[0], F0, 4, d4, s4, c9);
        tma_encode(&m.F[1], F1, 4, d4, s4, c9);
        tma_encode(&m.M9, M, 4, d4, s4, c9);
        tma_encode(&m.J, J, 3, d3, s4, c1);
        tma_encode(&m.FL[0], F0, 4, d4, s4, d9);
        tma_encode(&m.FL[1], F1, 4, d4, s4, d9);
        tma_encode(&m.M3, M, 4, d4, s4, d3b);
        tma_encode(&m.JL, J, 3, d3, s4, d1);
        tma_encode(&m.DF, DF, 4, d4, s4, d9);
    };
    try {
        encode(h->m, TJM, TKM);
        encode(h->me, TJE, TKE);
        h->ksat.assign(nblocks, nullptr);
        h->xcl.assign(nblocks, nullptr);
        h->jp.assign(nblocks, 0);
        h->kmap.resize(nblocks);
        h->ekmap.resize(nblocks);
        for (int b = 0; b < nblocks; b++) {
            const int n0 = blocks[b].n[0], jp = (blocks[b].n[1] + 3) / 4 * 4;
            h->jp[b] = jp;
            const size_t bytes = sizeof(float) * 18 * (size_t)n0 * jp;
            const cudaError_t e = cudaMalloc(&h->ksat[b], bytes);
            if (e != cudaSuccess)
                throw std::runtime_error(std::string("CUDA error in cudaMalloc (k-face SAT buffer): ") +
                                         cudaGetErrorString(e));
            cudaMemset(h->ksat[b], 0, bytes);
            // closure-plane x derivatives: up to 12 planes (order 4) x 6 values per node
            const size_t xbytes = sizeof(float) * 12 * 6 * (size_t)blocks[b].n[1] * blocks[b].n[2];
            const cudaError_t ex = cudaMalloc(&h->xcl[b], xbytes);
            if (ex != cudaSuccess)
                throw std::runtime_error(std::string("CUDA error in cudaMalloc (closure-plane buffer): ") +
                                         cudaGetErrorString(ex));
            const cuuint64_t dk[3] = {(cuuint64_t)jp, (cuuint64_t)n0, 18};
            const cuuint64_t sk[2] = {(cuuint64_t)jp * 4, (cuuint64_t)n0 * jp * 4};
            const cuuint32_t bk[3] = {TJM + 4, 1, 9}, bke[3] = {TJE + 4, 1, 9};
            tma_encode(&h->kmap[b], h->ksat[b], 3, dk, sk, bk);
            tma_encode(&h->ekmap[b], h->ksat[b], 3, dk, sk, bke);
        }
    } catch (...) {
        delete h;
        throw;
    }
    return h;
}

void free_reg_maps(RegMapsHost* h) { delete h; }

bool reg3d_supported(const Layout& L, const BlockDev& b, int order) {
    if (b.mat) return false;   // one material per block
    if (L.ndim != 3 || L.nfields != 9) return false;
    if (order < 2 || order > 4) return false;
    if (b.n[1] < TJM || b.n[2] < TKM) return false;
    if (b.n[0] < 4 * order - 3) return false;
    if (L.cstride * 9 >= (1LL << 31)) return false;   // 32-bit element offsets
    if (L.s1 % 4 != 0 || L.s0 % 4 != 0 || L.cstride % 4 != 0) return false;   // 16-byte row starts
    if (b.lo[2] % 4 != 0) return false;   // tiles start on 16-byte boundaries
    return true;
}

void launch_prepass_reg3d(const VolumeArgs<float>& a, const BlockDev* blks_dev, const BlockDev* blks, int b0,
                          int nb, const StageArgs& sa, const RegMapsHost* maps, cudaStream_t s) {
    if (nb > FDF_ALLB_MAX || nb < 1 || !maps) throw std::runtime_error("register-window pre-pass: bad block range");
    PrepTable P{};
    P.nblk = nb;
    int t = 0;
    for (int b = 0; b < nb; b++) {
        const BlockDev& B = blks[b0 + b];
        P.start[b] = t;
        P.kx[b] = (B.n[1] + 31) / 32;
        P.ky[b] = (B.n[0] + 3) / 4;
        P.nk[b] = (B.bactive[4] || B.bactive[5]) ? P.kx[b] * P.ky[b] * 2 : 0;
        P.xx[b] = (B.n[2] + 31) / 32;
        P.xy[b] = (B.n[1] + 3) / 4;
        P.jp[b] = maps->jp[b0 + b];
        P.ks[b] = maps->ksat[b0 + b];
        P.xcl[b] = maps->xcl[b0 + b];
        t += P.nk[b] + P.xx[b] * P.xy[b] * 2;
    }
    P.start[nb] = t;
    switch (a.order) {
        case 2: k_prepass3d<2><<<t, dim3(32, 4), 0, s>>>(a, blks_dev + b0, sa, P); break;
        case 3: k_prepass3d<3><<<t, dim3(32, 4), 0, s>>>(a, blks_dev + b0, sa, P); break;
        default: k_prepass3d<4><<<t, dim3(32, 4), 0, s>>>(a, blks_dev + b0, sa, P); break;
    }
}

void launch_volume_reg3d(const VolumeArgs<float>& a, const BlockDev& b, int bi, const StageArgs& sa, int* status,
                         const RegMapsHost* maps, cudaStream_t s) {
    if (a.cdiss > 0.) {   // artificial dissipation: the tiled kernel of stage_fast.cu
        launch_volume_fast3d(a, b, sa, s);
        return;
    }
    if (!maps) throw std::runtime_error("register-window kernel: tensor maps missing");
    switch (a.order) {
        case 2: launch_order<2>(a, b, bi, sa, status, *maps, s); break;
        case 3: launch_order<3>(a, b, bi, sa, status, *maps, s); break;
        default: launch_order<4>(a, b, bi, sa, status, *maps, s); break;
    }
}

}  // namespace fdf
