#pragma once
// Host side of the learned STZ initial guess: parameters, training and
// inference of the 6 -> 64 -> 64 -> 1 network on the GPU.
//
// Flat FP32 parameter vector (MLP_NPARAM values), in this order:
//   W1[64][6], b1[64], W2[64][64], b2[64], W3[64], b3[1]
// The device keeps BF16 copies of W1 (zero-padded to [64][16]), W2 and W3
// (zero-padded to [8][64]) for the forward pass; biases stay FP32.
#include <cuda_runtime.h>

#include "fdf_types.hpp"

namespace fdf {

constexpr int MLP_OFF_W1 = 0, MLP_OFF_B1 = 384, MLP_OFF_W2 = 448, MLP_OFF_B2 = 4544, MLP_OFF_W3 = 4608,
              MLP_OFF_B3 = 4672, MLP_NPARAM = 4673;

struct MlpState {
    float* P = nullptr;              // master parameters (FP32)
    float* m = nullptr;              // Adam first moments
    float* v = nullptr;              // Adam second moments
    float* grad = nullptr;           // last batch gradient
    unsigned short* wb = nullptr;    // BF16 copies: w1 [64*16], w2 [64*64], w3 [8*64]
    long long adam_t = 0;
    bool ready = false;
    MlpDev dev() const;
};

void mlp_alloc(MlpState& s);
void mlp_free(MlpState& s);
// He-normal initialisation from a seeded generator (host), zero biases
void mlp_init(MlpState& s, unsigned long long seed, cudaStream_t st);
void mlp_set_params(MlpState& s, const float* host, cudaStream_t st);
void mlp_get_params(const MlpState& s, float* host, cudaStream_t st);
// network outputs for n input rows x[n][6] (host arrays); force_thread
// selects the per-thread path instead of the tensor-core warp path
void mlp_infer(const MlpState& s, const float* x, long long n, float* y, int force_thread, cudaStream_t st);
// gradient of 0.5 * mean((y - t)^2) over n samples (host arrays): grads[MLP_NPARAM], loss
void mlp_gradients(MlpState& s, const float* x, const float* t, long long n, float* grads, double* loss,
                   cudaStream_t st);
// Adam training on device samples [count][8] (6 inputs, target, mu): the
// last tenth of a seeded permutation is held out; returns the mean training
// loss of the last epoch and the held-out loss
void mlp_train(MlpState& s, const float* dsamples, long long count, int epochs, int batch, float lr,
               unsigned long long seed, double* train_loss, double* val_loss, cudaStream_t st);

}  // namespace fdf
