// jp_mlp.cuh -- the weight surrogate network shared by training (jp_mlp.cu) and the
// force-scaling step (jp_integrate.cu): nin -> 64 -> 64 -> nout, tanh hidden layers, linear
// output, FP32 parameters in one flat vector
//   [W1 64 x nin | b1 64 | W2 64 x 64 | b2 64 | W3 nout x 64 | b3 nout |
//    x offset nin | x scale nin | y offset nout | y scale nout]
// evaluated as y = yoff + yscale * net((x - xoff) * xscale).
#pragma once
#include "jpgpu.h"

namespace jp {

constexpr int kMlpH = JP_MLP_HIDDEN;

struct MlpLayout {
  int w1, b1, w2, b2, w3, b3, xo, xs, yo, ys, n;
};

__host__ __device__ __forceinline__ MlpLayout mlp_layout(int nin, int nout) {
  MlpLayout L;
  L.w1 = 0;
  L.b1 = L.w1 + kMlpH * nin;
  L.w2 = L.b1 + kMlpH;
  L.b2 = L.w2 + kMlpH * kMlpH;
  L.w3 = L.b2 + kMlpH;
  L.b3 = L.w3 + nout * kMlpH;
  L.xo = L.b3 + nout;
  L.xs = L.xo + nin;
  L.yo = L.xs + nin;
  L.ys = L.yo + nout;
  L.n = L.ys + nout;
  return L;
}

// One forward pass by a full warp (lane j holds hidden units j and j + 32).  p: parameters
// (any memory space), x[nin]; y[nout] is returned in every lane.
__device__ __forceinline__ void mlp_forward_warp(const float* __restrict__ p, int nin, int nout,
                                                 const float* x, float* y) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const MlpLayout L = mlp_layout(nin, nout);
  float xn[JP_MLP_MAXIO];
  for (int i = 0; i < nin; ++i) xn[i] = (x[i] - p[L.xo + i]) * p[L.xs + i];
  float h1[2];
  for (int r = 0; r < 2; ++r) {
    const int j = lane + 32 * r;
    float z = p[L.b1 + j];
    for (int i = 0; i < nin; ++i) z = fmaf(p[L.w1 + j * nin + i], xn[i], z);
    h1[r] = tanhf(z);
  }
  float h2[2];
  for (int r = 0; r < 2; ++r) {
    const int j = lane + 32 * r;
    float z = p[L.b2 + j];
    for (int k = 0; k < kMlpH; ++k) {
      const float hk = __shfl_sync(full, h1[k >> 5], k & 31);
      z = fmaf(p[L.w2 + j * kMlpH + k], hk, z);
    }
    h2[r] = tanhf(z);
  }
  for (int o = 0; o < nout; ++o) {
    float s = p[L.w3 + o * kMlpH + lane] * h2[0] + p[L.w3 + o * kMlpH + lane + 32] * h2[1];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(full, s, off);
    y[o] = p[L.yo + o] + p[L.ys + o] * (s + p[L.b3 + o]);
  }
}

}  // namespace jp
