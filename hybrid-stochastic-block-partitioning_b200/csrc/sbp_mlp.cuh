// The learned proposal's network: 64 features -> 128 -> 128 -> 16 logits (ReLU between),
// BF16 weights and activations, FP32 accumulation, on the 5th-generation tensor cores
// (tcgen05.mma with the accumulators in tensor memory).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace sbpb {

constexpr int kMlpIn = 64;
constexpr int kMlpHid = 128;
constexpr int kMlpOut = 16;      // 14 candidate slots + escape + one always-masked pad
constexpr int kMlpSlots = 14;    // candidate neighbour blocks per vertex
constexpr int kMlpEscape = 14;   // logit index of "uniformly random block"
constexpr int kMlpTile = 128;    // rows (vertices) per CTA tile = the MMA's M

// Parameter vector (FP32 master copy), in this order.
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpHid * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpHid;
constexpr int kOffB2 = kOffW2 + kMlpHid * kMlpHid;
constexpr int kOffW3 = kOffB2 + kMlpHid;
constexpr int kOffB3 = kOffW3 + kMlpOut * kMlpHid;
constexpr int kMlpParams = kOffB3 + kMlpOut;   // 26,896

struct MlpWeights {                 // device copies used by the kernels
  const __nv_bfloat16* W1;         // [128][64]  row-major [out][in]
  const __nv_bfloat16* W2;         // [128][128]
  const __nv_bfloat16* W3;         // [16][128]
  const float* b1;                 // [128]
  const float* b2;                 // [128]
  const float* b3;                 // [16]
};

// logits[n][16] = MLP(features[n][64]); rows are independent.  status[0] |= 64 when a
// tensor-core completion wait gave up.
void mlp_forward(const __nv_bfloat16* features, long long n, MlpWeights w, float* logits, int* status, int sms,
                 cudaStream_t s);

// Gradients of the mean masked cross-entropy over n rows, accumulated (atomically) into
// grads[kMlpParams] (zeroed by the caller); loss_sum[0] += sum of row losses.
// target[i] in [0,15) or -1 (row ignored); nvalid[i] = number of valid candidate slots
// (slots >= nvalid and logit 15 are masked out; the escape logit is always valid).
void mlp_gradients(const __nv_bfloat16* features, const int* target, const int* nvalid, long long n, float inv_count,
                   MlpWeights w, float* grads, double* loss_sum, int* status, cudaStream_t s);

// Adam step on the FP32 master parameters; refreshes the BF16 weight copies and FP32 biases.
void mlp_adam(float* params, float* m, float* v, const float* grads, int step, float lr, float beta1, float beta2,
              float eps, __nv_bfloat16* W1, __nv_bfloat16* W2, __nv_bfloat16* W3, float* bias, cudaStream_t s);

// BF16 weight copies and biases from the FP32 parameter vector.
void mlp_publish(const float* params, __nv_bfloat16* W1, __nv_bfloat16* W2, __nv_bfloat16* W3, float* bias,
                 cudaStream_t s);

void float_to_bf16(const float* in, __nv_bfloat16* out, long long n, cudaStream_t s);

constexpr int kErrTensorWait = 64;

}  // namespace sbpb
