// The dispatch cost model: a 6 -> 32 -> 32 -> 4 fp32 MLP (ReLU hidden layers)
// predicting, for one segment, the log-cost of each of the four kernel
// variants.  Parameters are one flat float array in this order:
//   W1[32][6], b1[32], W2[32][32], b2[32], W3[4][32], b3[4].
#pragma once
#include <cstdint>

namespace lpa_mlp {

constexpr int kIn = 6, kH = 32, kOut = 4;
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kH * kIn;
constexpr int kOffW2 = kOffB1 + kH;
constexpr int kOffB2 = kOffW2 + kH * kH;
constexpr int kOffW3 = kOffB2 + kH;
constexpr int kOffB3 = kOffW3 + kOut * kH;
constexpr int kParams = kOffB3 + kOut;  // 1412

// Forward pass; h1/h2 receive the hidden activations (after ReLU).
__host__ __device__ inline void forward(const float *P, const float *x, float *h1, float *h2, float *y) {
  for (int j = 0; j < kH; j++) {
    float s = P[kOffB1 + j];
    for (int i = 0; i < kIn; i++) s += P[kOffW1 + j * kIn + i] * x[i];
    h1[j] = s > 0.f ? s : 0.f;
  }
  for (int j = 0; j < kH; j++) {
    float s = P[kOffB2 + j];
    for (int i = 0; i < kH; i++) s += P[kOffW2 + j * kH + i] * h1[i];
    h2[j] = s > 0.f ? s : 0.f;
  }
  for (int o = 0; o < kOut; o++) {
    float s = P[kOffB3 + o];
    for (int i = 0; i < kH; i++) s += P[kOffW3 + o * kH + i] * h2[i];
    y[o] = s;
  }
}

}  // namespace lpa_mlp
