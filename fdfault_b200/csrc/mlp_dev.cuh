#pragma once
// Learned initial guess for the STZ friction Newton solve: a 6 -> 64 -> 64 -> 1
// multilayer perceptron (ReLU hidden layers) with BF16 weights and
// activations and FP32 accumulation.
//
// Inference runs warp-cooperatively on the tensor cores: a warp evaluates the
// network for its 32 fault nodes with mma.m16n8k16 (BF16 in, FP32
// accumulate) -- two 16-row tiles; the FP32 accumulator of one layer,
// after bias and ReLU, is repacked in registers as the BF16 A operand of the
// next layer.  A warp whose lanes are not all present (the tail of the fault)
// uses the per-thread path, which rounds the same operands to BF16 and
// accumulates in FP32.
//
// Weight layout (device, BF16 row-major [out][in], inputs zero-padded):
//   w1[64][16] (6 real inputs), w2[64][64], w3[8][64] (row 0 real);
// biases FP32: b1[64], b2[64], b3[1].
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "fdf_types.hpp"

namespace fdf {

constexpr int MLP_IN = 6, MLP_H = 64;

__device__ __forceinline__ unsigned mlp_pack(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<unsigned*>(&v);
}

__device__ __forceinline__ float mlp_bf16(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ float mlp_w(const unsigned short* w, int idx) {
    return __bfloat162float(__ushort_as_bfloat16(w[idx]));
}

__device__ __forceinline__ void mma_bf16_16816(float d[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                               unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ unsigned mlp_ld2(const unsigned short* w, int idx) {
    return __ldg(reinterpret_cast<const unsigned*>(w + idx));   // idx even: 4-byte aligned pair
}

// Per-thread evaluation (FP32 accumulation of BF16-rounded operands).
__device__ inline float mlp_eval_thread(const MlpDev& m, const float x[MLP_IN]) {
    float xb[MLP_IN];
#pragma unroll
    for (int i = 0; i < MLP_IN; i++) xb[i] = mlp_bf16(x[i]);
    float h1[MLP_H];
    for (int o = 0; o < MLP_H; o++) {
        float acc = 0.f;
#pragma unroll
        for (int i = 0; i < MLP_IN; i++) acc = fmaf(mlp_w(m.w1, o * 16 + i), xb[i], acc);
        acc += m.b1[o];
        h1[o] = mlp_bf16(fmaxf(acc, 0.f));
    }
    float y = 0.f;
    for (int o = 0; o < MLP_H; o++) {
        float acc = 0.f;
        for (int i = 0; i < MLP_H; i++) acc = fmaf(mlp_w(m.w2, o * MLP_H + i), h1[i], acc);
        acc += m.b2[o];
        y = fmaf(mlp_w(m.w3, o), mlp_bf16(fmaxf(acc, 0.f)), y);
    }
    return y + m.b3[0];
}

// Warp-cooperative evaluation; every lane of the warp must call it together
// (full mask).  Each lane passes its own node's inputs and gets its output.
__device__ inline float mlp_eval_warp(const MlpDev& m, const float x[MLP_IN]) {
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, tig = lane & 3;
    const unsigned p0 = mlp_pack(x[0], x[1]), p1 = mlp_pack(x[2], x[3]), p2 = mlp_pack(x[4], x[5]);
    float yt[2][2];
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
        // ---- layer 1: A = inputs of nodes 16mt+g (row g) and 16mt+g+8 (row g+8)
        const int s0 = 16 * mt + g, s1 = s0 + 8;
        const unsigned u0 = __shfl_sync(0xffffffffu, p0, s0), u1 = __shfl_sync(0xffffffffu, p1, s0),
                       u2 = __shfl_sync(0xffffffffu, p2, s0);
        const unsigned w0 = __shfl_sync(0xffffffffu, p0, s1), w1 = __shfl_sync(0xffffffffu, p1, s1),
                       w2 = __shfl_sync(0xffffffffu, p2, s1);
        const unsigned a0 = tig == 0 ? u0 : (tig == 1 ? u1 : (tig == 2 ? u2 : 0u));
        const unsigned a1 = tig == 0 ? w0 : (tig == 1 ? w1 : (tig == 2 ? w2 : 0u));
        unsigned A[4][4];   // layer-2 A fragments, k-tiles 0..3
#pragma unroll
        for (int jp = 0; jp < 4; jp++) {
            float c[2][4];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int j = 2 * jp + h, n = 8 * j + g;
                c[h][0] = c[h][1] = c[h][2] = c[h][3] = 0.f;
                mma_bf16_16816(c[h], a0, a1, 0u, 0u, mlp_ld2(m.w1, n * 16 + 2 * tig), mlp_ld2(m.w1, n * 16 + 8 + 2 * tig));
                const int col = 8 * j + 2 * tig;
                const float bb0 = m.b1[col], bb1 = m.b1[col + 1];
                c[h][0] = fmaxf(c[h][0] + bb0, 0.f);
                c[h][1] = fmaxf(c[h][1] + bb1, 0.f);
                c[h][2] = fmaxf(c[h][2] + bb0, 0.f);
                c[h][3] = fmaxf(c[h][3] + bb1, 0.f);
            }
            A[jp][0] = mlp_pack(c[0][0], c[0][1]);
            A[jp][1] = mlp_pack(c[0][2], c[0][3]);
            A[jp][2] = mlp_pack(c[1][0], c[1][1]);
            A[jp][3] = mlp_pack(c[1][2], c[1][3]);
        }
        // ---- layer 2 (64 x 64), then layer 3 fragments
        unsigned A3[4][4];
#pragma unroll
        for (int jp = 0; jp < 4; jp++) {
            float c[2][4];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int j = 2 * jp + h, n = 8 * j + g;
                c[h][0] = c[h][1] = c[h][2] = c[h][3] = 0.f;
#pragma unroll
                for (int t = 0; t < 4; t++)
                    mma_bf16_16816(c[h], A[t][0], A[t][1], A[t][2], A[t][3],
                                   mlp_ld2(m.w2, n * MLP_H + 16 * t + 2 * tig),
                                   mlp_ld2(m.w2, n * MLP_H + 16 * t + 8 + 2 * tig));
                const int col = 8 * j + 2 * tig;
                const float bb0 = m.b2[col], bb1 = m.b2[col + 1];
                c[h][0] = fmaxf(c[h][0] + bb0, 0.f);
                c[h][1] = fmaxf(c[h][1] + bb1, 0.f);
                c[h][2] = fmaxf(c[h][2] + bb0, 0.f);
                c[h][3] = fmaxf(c[h][3] + bb1, 0.f);
            }
            A3[jp][0] = mlp_pack(c[0][0], c[0][1]);
            A3[jp][1] = mlp_pack(c[0][2], c[0][3]);
            A3[jp][2] = mlp_pack(c[1][0], c[1][1]);
            A3[jp][3] = mlp_pack(c[1][2], c[1][3]);
        }
        // ---- layer 3 (1 real output column; w3 rows 1..7 are zero)
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int t = 0; t < 4; t++)
            mma_bf16_16816(c, A3[t][0], A3[t][1], A3[t][2], A3[t][3], mlp_ld2(m.w3, g * MLP_H + 16 * t + 2 * tig),
                           mlp_ld2(m.w3, g * MLP_H + 16 * t + 8 + 2 * tig));
        yt[mt][0] = c[0];   // (row g, col 2tig): column 0 lives in lanes with tig == 0
        yt[mt][1] = c[2];   // (row g+8, col 2tig)
    }
    const int r = lane & 15, src = (r & 7) * 4;
    const float y00 = __shfl_sync(0xffffffffu, yt[0][0], src), y01 = __shfl_sync(0xffffffffu, yt[0][1], src);
    const float y10 = __shfl_sync(0xffffffffu, yt[1][0], src), y11 = __shfl_sync(0xffffffffu, yt[1][1], src);
    const float y = (lane < 16) ? (r < 8 ? y00 : y01) : (r < 8 ? y10 : y11);
    return y + m.b3[0];
}

// Network inputs for the STZ solve of one fault node.  With the root mu in
// [muy, phi/|sn|], eta*V(mu) = phi - |sn|*mu and
// log(phi/|sn| - mu) = q + mu/a + log(1 - muy/mu),  q = log(eta*v0/|sn|) - f0 - 1/chi,
// so (phi/|sn|, muy, a, q) fix the root; |sn| and 1/chi are given as well.
// The network predicts t = log(s / (1 - s)) / 20 with s = (mu - muy) / (phi/|sn| - muy).
// Returns false when an input is not finite (the caller then starts from the
// bracket midpoint).
__device__ inline bool stz_features(double phi, double snc, double chi, double eta, double v0, double f0, double a,
                                    double muy, float x[MLP_IN]) {
    // inputs only steer the start of the solve: single precision is enough
    const float asn = (float)fmax(fabs(snc), 1e-30);
    const float la = __logf(asn);
    const float q = __logf((float)(eta * v0)) - la - (float)f0 - (float)(1. / chi);
    const float v[MLP_IN] = {(float)(phi / fabs(snc)), (float)muy, (float)(a / 0.02), (q + 40.f) / 10.f, la / 5.f,
                             (float)(1. / chi) / 20.f};
    bool ok = true;
#pragma unroll
    for (int i = 0; i < MLP_IN; i++) {
        ok = ok && isfinite(v[i]) && fabsf(v[i]) < 1e4f;
        x[i] = ok ? v[i] : 0.f;
    }
    if (!ok) {
#pragma unroll
        for (int i = 0; i < MLP_IN; i++) x[i] = 0.f;
    }
    return ok;
}

}  // namespace fdf
