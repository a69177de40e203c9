// Training and inference kernels of the learned STZ initial guess
// (6 -> 64 -> 64 -> 1, ReLU, BF16 weights and activations, FP32 accumulate).
//
// Forward pass: inputs, weights and hidden activations are rounded to BF16,
// products are accumulated in FP32 and the biases are FP32 -- the same
// numerics as the inference path inside the interface kernel.  Backward pass:
// FP32, from the BF16 activations and weights of the forward pass (the
// gradient of the function the forward pass computes, with the roundings
// treated as identities).  Master weights and Adam moments are FP32.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "mlp.hpp"
#include "mlp_dev.cuh"

namespace fdf {

namespace {

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

// per-sample activations of a batch, sample-major
struct Act {
    float *x, *h1, *h2, *dz1, *dz2, *dy, *loss;
};

__global__ void k_mlp_to_bf16(const float* __restrict__ P, unsigned short* __restrict__ wb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 64 * 16) {
        const int o = t / 16, i = t % 16;
        const float w = i < MLP_IN ? P[MLP_OFF_W1 + o * MLP_IN + i] : 0.f;
        wb[t] = __bfloat16_as_ushort(__float2bfloat16_rn(w));
    } else if (t < 64 * 16 + 64 * 64) {
        const int q = t - 64 * 16;
        wb[t] = __bfloat16_as_ushort(__float2bfloat16_rn(P[MLP_OFF_W2 + q]));
    } else if (t < 64 * 16 + 64 * 64 + 8 * 64) {
        const int q = t - 64 * 16 - 64 * 64;
        const int r = q / 64, i = q % 64;
        const float w = r == 0 ? P[MLP_OFF_W3 + i] : 0.f;
        wb[t] = __bfloat16_as_ushort(__float2bfloat16_rn(w));
    }
}

constexpr int WB_TOTAL = 64 * 16 + 64 * 64 + 8 * 64;

// inference: x [n][xs] rows (first 6 values used); all lanes of every warp take
// part (rows past n are evaluated on zeros and dropped)
__global__ void __launch_bounds__(128) k_mlp_infer(MlpDev m, const float* __restrict__ x, int xs, long long n,
                                                   float* __restrict__ y, int force_thread) {
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    float in[MLP_IN];
#pragma unroll
    for (int i = 0; i < MLP_IN; i++) in[i] = s < n ? x[s * xs + i] : 0.f;
    const float out = force_thread ? mlp_eval_thread(m, in) : mlp_eval_warp(m, in);
    if (s < n) y[s] = out;
}

__global__ void __launch_bounds__(128) k_mlp_fwd_bwd(MlpDev m, const float* __restrict__ samples,
                                                     const int* __restrict__ idx, int n, float inv_n, Act a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float* smp = samples + 8LL * (idx ? idx[s] : s);
    float x[MLP_IN];
#pragma unroll
    for (int i = 0; i < MLP_IN; i++) x[i] = mlp_bf16(smp[i]);
    const float tgt = smp[6];
    float z1[MLP_H], h1[MLP_H];
    for (int o = 0; o < MLP_H; o++) {
        float acc = 0.f;
#pragma unroll
        for (int i = 0; i < MLP_IN; i++) acc = fmaf(mlp_w(m.w1, o * 16 + i), x[i], acc);
        z1[o] = acc + m.b1[o];
        h1[o] = mlp_bf16(fmaxf(z1[o], 0.f));
    }
    float y = 0.f;
    float* h2o = a.h2 + (long long)s * MLP_H;
    float* dz2o = a.dz2 + (long long)s * MLP_H;
    // z2 is only needed through its sign and h2: keep h2 in the output row,
    // the sign in dz2's row until dy is known
    for (int o = 0; o < MLP_H; o++) {
        float acc = 0.f;
        for (int i = 0; i < MLP_H; i++) acc = fmaf(mlp_w(m.w2, o * MLP_H + i), h1[i], acc);
        const float z2 = acc + m.b2[o];
        const float h2 = mlp_bf16(fmaxf(z2, 0.f));
        h2o[o] = h2;
        dz2o[o] = z2 > 0.f ? 1.f : 0.f;
        y = fmaf(mlp_w(m.w3, o), h2, y);
    }
    y += m.b3[0];
    const float e = y - tgt;
    a.loss[s] = 0.5f * e * e;
    const float dy = e * inv_n;
    a.dy[s] = dy;
    for (int o = 0; o < MLP_H; o++) dz2o[o] *= dy * mlp_w(m.w3, o);
    float* dz1o = a.dz1 + (long long)s * MLP_H;
    for (int i = 0; i < MLP_H; i++) {
        float acc = 0.f;
        for (int o = 0; o < MLP_H; o++) acc = fmaf(mlp_w(m.w2, o * MLP_H + i), dz2o[o], acc);
        dz1o[i] = z1[i] > 0.f ? acc : 0.f;
    }
    float* h1o = a.h1 + (long long)s * MLP_H;
    for (int i = 0; i < MLP_H; i++) h1o[i] = h1[i];
    float* xo = a.x + (long long)s * 8;
#pragma unroll
    for (int i = 0; i < MLP_IN; i++) xo[i] = x[i];
}

// one thread per parameter, sequential FP32 sum over the batch (deterministic)
__global__ void k_mlp_wgrad(Act a, int n, float* __restrict__ g) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= MLP_NPARAM) return;
    float acc = 0.f;
    if (p < MLP_OFF_B1) {
        const int o = p / MLP_IN, i = p % MLP_IN;
        for (int s = 0; s < n; s++) acc = fmaf(a.dz1[(long long)s * MLP_H + o], a.x[(long long)s * 8 + i], acc);
    } else if (p < MLP_OFF_W2) {
        const int o = p - MLP_OFF_B1;
        for (int s = 0; s < n; s++) acc += a.dz1[(long long)s * MLP_H + o];
    } else if (p < MLP_OFF_B2) {
        const int q = p - MLP_OFF_W2, o = q / MLP_H, i = q % MLP_H;
        for (int s = 0; s < n; s++) acc = fmaf(a.dz2[(long long)s * MLP_H + o], a.h1[(long long)s * MLP_H + i], acc);
    } else if (p < MLP_OFF_W3) {
        const int o = p - MLP_OFF_B2;
        for (int s = 0; s < n; s++) acc += a.dz2[(long long)s * MLP_H + o];
    } else if (p < MLP_OFF_B3) {
        const int o = p - MLP_OFF_W3;
        for (int s = 0; s < n; s++) acc = fmaf(a.dy[s], a.h2[(long long)s * MLP_H + o], acc);
    } else {
        for (int s = 0; s < n; s++) acc += a.dy[s];
    }
    g[p] = acc;
}

__global__ void k_mlp_adam(float* __restrict__ P, float* __restrict__ m, float* __restrict__ v,
                           const float* __restrict__ g, float lr, float c1, float c2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= MLP_NPARAM) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float gi = g[p];
    const float mi = b1 * m[p] + (1.f - b1) * gi;
    const float vi = b2 * v[p] + (1.f - b2) * gi * gi;
    m[p] = mi;
    v[p] = vi;
    P[p] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

struct ActBuf {
    Act a{};
    float* base = nullptr;
    explicit ActBuf(long long n) {
        const long long per = 8 + 4 * MLP_H + 2;
        ck(cudaMalloc(&base, (size_t)(per * n) * sizeof(float)), "cudaMalloc mlp activations");
        a.x = base;
        a.h1 = a.x + 8 * n;
        a.h2 = a.h1 + MLP_H * n;
        a.dz1 = a.h2 + MLP_H * n;
        a.dz2 = a.dz1 + MLP_H * n;
        a.dy = a.dz2 + MLP_H * n;
        a.loss = a.dy + n;
    }
    ~ActBuf() { cudaFree(base); }
};

void refresh_bf16(MlpState& s, cudaStream_t st) {
    k_mlp_to_bf16<<<(WB_TOTAL + 255) / 256, 256, 0, st>>>(s.P, s.wb);
    ck(cudaGetLastError(), "k_mlp_to_bf16");
}

}  // namespace

MlpDev MlpState::dev() const {
    MlpDev d{};
    d.w1 = wb;
    d.w2 = wb + 64 * 16;
    d.w3 = wb + 64 * 16 + 64 * 64;
    d.b1 = P + MLP_OFF_B1;
    d.b2 = P + MLP_OFF_B2;
    d.b3 = P + MLP_OFF_B3;
    return d;
}

void mlp_alloc(MlpState& s) {
    if (s.P) return;
    ck(cudaMalloc(&s.P, 4 * MLP_NPARAM * sizeof(float)), "cudaMalloc mlp");
    s.m = s.P + MLP_NPARAM;
    s.v = s.m + MLP_NPARAM;
    s.grad = s.v + MLP_NPARAM;
    ck(cudaMalloc(&s.wb, WB_TOTAL * sizeof(unsigned short)), "cudaMalloc mlp bf16");
    ck(cudaMemset(s.P, 0, 4 * MLP_NPARAM * sizeof(float)), "mlp clear");
}

void mlp_free(MlpState& s) {
    if (s.P) cudaFree(s.P);
    if (s.wb) cudaFree(s.wb);
    s = MlpState{};
}

void mlp_set_params(MlpState& s, const float* host, cudaStream_t st) {
    mlp_alloc(s);
    ck(cudaMemcpyAsync(s.P, host, MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice, st), "mlp params");
    ck(cudaMemsetAsync(s.m, 0, 2 * MLP_NPARAM * sizeof(float), st), "mlp moments");
    s.adam_t = 0;
    refresh_bf16(s, st);
    ck(cudaStreamSynchronize(st), "mlp params");
    s.ready = true;
}

void mlp_get_params(const MlpState& s, float* host, cudaStream_t st) {
    if (!s.ready) throw std::runtime_error("network parameters are not set");
    ck(cudaMemcpyAsync(host, s.P, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, st), "mlp params");
    ck(cudaStreamSynchronize(st), "mlp params");
}

void mlp_init(MlpState& s, unsigned long long seed, cudaStream_t st) {
    std::vector<float> p(MLP_NPARAM, 0.f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> nd(0., 1.);
    for (int q = 0; q < 64 * MLP_IN; q++) p[MLP_OFF_W1 + q] = (float)(nd(rng) * std::sqrt(2.0 / MLP_IN));
    for (int q = 0; q < 64 * 64; q++) p[MLP_OFF_W2 + q] = (float)(nd(rng) * std::sqrt(2.0 / MLP_H));
    for (int q = 0; q < 64; q++) p[MLP_OFF_W3 + q] = (float)(nd(rng) * std::sqrt(1.0 / MLP_H));
    p[MLP_OFF_B3] = 0.f;   // logit 0: the middle of the bracket
    mlp_set_params(s, p.data(), st);
}

void mlp_infer(const MlpState& s, const float* x, long long n, float* y, int force_thread, cudaStream_t st) {
    if (!s.ready) throw std::runtime_error("network parameters are not set");
    if (n <= 0) return;
    float *dx = nullptr, *dy = nullptr;
    ck(cudaMalloc(&dx, (size_t)n * MLP_IN * sizeof(float)), "cudaMalloc mlp input");
    ck(cudaMalloc(&dy, (size_t)n * sizeof(float)), "cudaMalloc mlp output");
    ck(cudaMemcpyAsync(dx, x, (size_t)n * MLP_IN * sizeof(float), cudaMemcpyHostToDevice, st), "mlp input");
    k_mlp_infer<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(s.dev(), dx, MLP_IN, n, dy, force_thread);
    ck(cudaGetLastError(), "k_mlp_infer");
    ck(cudaMemcpyAsync(y, dy, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, st), "mlp output");
    ck(cudaStreamSynchronize(st), "mlp infer");
    cudaFree(dx);
    cudaFree(dy);
}

void mlp_gradients(MlpState& s, const float* x, const float* t, long long n, float* grads, double* loss,
                   cudaStream_t st) {
    if (!s.ready) throw std::runtime_error("network parameters are not set");
    if (n <= 0 || n > (1LL << 24)) throw std::invalid_argument("sample count out of range");
    std::vector<float> smp((size_t)n * 8, 0.f);
    for (long long i = 0; i < n; i++) {
        for (int c = 0; c < MLP_IN; c++) smp[i * 8 + c] = x[i * MLP_IN + c];
        smp[i * 8 + 6] = t[i];
    }
    float* ds = nullptr;
    ck(cudaMalloc(&ds, smp.size() * sizeof(float)), "cudaMalloc mlp samples");
    ck(cudaMemcpyAsync(ds, smp.data(), smp.size() * sizeof(float), cudaMemcpyHostToDevice, st), "mlp samples");
    ActBuf ab(n);
    k_mlp_fwd_bwd<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(s.dev(), ds, nullptr, (int)n,
                                                                1.f / (float)n, ab.a);
    ck(cudaGetLastError(), "k_mlp_fwd_bwd");
    k_mlp_wgrad<<<(MLP_NPARAM + 127) / 128, 128, 0, st>>>(ab.a, (int)n, s.grad);
    ck(cudaGetLastError(), "k_mlp_wgrad");
    std::vector<float> l((size_t)n);
    ck(cudaMemcpyAsync(grads, s.grad, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, st), "mlp grads");
    ck(cudaMemcpyAsync(l.data(), ab.a.loss, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, st), "mlp loss");
    ck(cudaStreamSynchronize(st), "mlp gradients");
    cudaFree(ds);
    double sum = 0.;
    for (float v : l) sum += v;
    *loss = sum / (double)n;
}

void mlp_train(MlpState& s, const float* dsamples, long long count, int epochs, int batch, float lr,
               unsigned long long seed, double* train_loss, double* val_loss, cudaStream_t st) {
    if (!s.ready) throw std::runtime_error("network parameters are not set");
    if (count < 16) throw std::invalid_argument("too few samples to train on");
    if (batch <= 0 || epochs < 0) throw std::invalid_argument("invalid batch or epoch count");
    std::mt19937_64 rng(seed);
    std::vector<int> perm((size_t)count);
    std::iota(perm.begin(), perm.end(), 0);
    std::shuffle(perm.begin(), perm.end(), rng);
    const long long nval = std::max<long long>(1, count / 10);
    const long long ntr = count - nval;
    std::vector<int> tr(perm.begin(), perm.begin() + ntr), va(perm.begin() + ntr, perm.end());
    const int B = (int)std::min<long long>(batch, ntr);
    int *didx = nullptr, *dval = nullptr;
    ck(cudaMalloc(&didx, (size_t)ntr * sizeof(int)), "cudaMalloc mlp index");
    ck(cudaMalloc(&dval, (size_t)nval * sizeof(int)), "cudaMalloc mlp index");
    ck(cudaMemcpyAsync(dval, va.data(), (size_t)nval * sizeof(int), cudaMemcpyHostToDevice, st), "mlp index");
    ActBuf ab(std::max<long long>(B, nval));
    std::vector<float> l;
    double last = 0.;
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(tr.begin(), tr.end(), rng);
        ck(cudaMemcpyAsync(didx, tr.data(), (size_t)ntr * sizeof(int), cudaMemcpyHostToDevice, st), "mlp index");
        double sum = 0.;
        long long seen = 0;
        for (long long b0 = 0; b0 + B <= ntr; b0 += B) {
            k_mlp_fwd_bwd<<<(B + 127) / 128, 128, 0, st>>>(s.dev(), dsamples, didx + b0, B,
                                                           1.f / (float)B, ab.a);
            k_mlp_wgrad<<<(MLP_NPARAM + 127) / 128, 128, 0, st>>>(ab.a, B, s.grad);
            s.adam_t++;
            const float c1 = 1.f - std::pow(0.9f, (float)s.adam_t), c2 = 1.f - std::pow(0.999f, (float)s.adam_t);
            k_mlp_adam<<<(MLP_NPARAM + 127) / 128, 128, 0, st>>>(s.P, s.m, s.v, s.grad, lr, c1, c2);
            refresh_bf16(s, st);
            if (ep == epochs - 1) {
                l.resize((size_t)B);
                ck(cudaMemcpyAsync(l.data(), ab.a.loss, (size_t)B * sizeof(float), cudaMemcpyDeviceToHost, st),
                   "mlp loss");
                ck(cudaStreamSynchronize(st), "mlp loss");
                for (float v : l) sum += v;
                seen += B;
            }
        }
        ck(cudaGetLastError(), "mlp training");
        if (ep == epochs - 1 && seen) last = sum / (double)seen;
    }
    // held-out loss with the final weights
    k_mlp_fwd_bwd<<<(unsigned)((nval + 127) / 128), 128, 0, st>>>(s.dev(), dsamples, dval, (int)nval,
                                                                   1.f / (float)nval, ab.a);
    ck(cudaGetLastError(), "mlp validation");
    l.resize((size_t)nval);
    ck(cudaMemcpyAsync(l.data(), ab.a.loss, (size_t)nval * sizeof(float), cudaMemcpyDeviceToHost, st), "mlp loss");
    ck(cudaStreamSynchronize(st), "mlp training");
    double vs = 0.;
    for (float v : l) vs += v;
    *train_loss = last;
    *val_loss = vs / (double)nval;
    cudaFree(didx);
    cudaFree(dval);
}

}  // namespace fdf
