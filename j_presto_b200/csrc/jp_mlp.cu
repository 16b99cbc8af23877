// jp_mlp.cu -- training and batch inference of the weight surrogate network (jp_mlp.cuh).
//
// The network stands in for GEprep's windowed polynomial fit of d lnN/dE (and, with two
// inputs and outputs, of the ALSD weight in (E, lambda)): it is trained on the same data the
// polynomial fit takes -- points (x, y) with weights w -- by full-batch Adam on the weighted
// mean squared error of the normalised targets, sum_s w_s (net(x_s) - (y_s - yoff)/yscale)^2
// / sum_s w_s.
//
// One CUDA block trains one network, so the networks of many replicas train in one launch.
// Each epoch runs as block-wide phases separated by __syncthreads: forward (activations of
// all samples in a global scratch slice), output error, back-propagation, the gradient
// sums over samples, Adam.  Every gradient entry is one thread's sequential sum over the
// samples, so training is deterministic.  Parameters, gradients and Adam moments live in
// shared memory.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "jp_common.cuh"
#include "jp_mlp.cuh"

namespace jp {
namespace {

constexpr int kMlpThreads = 256;

struct MlpTrainArgs {
  const float *x, *y, *w;     // [total][nin], [total][nout], [total]
  const int *off;             // [nnet + 1] sample ranges
  int nin, nout, epochs;
  float lr;
  float *params;              // [nnet][np] in/out
  float *grad;                // nullable: [nnet][np] gradient at the final parameters
  float *loss;                // [nnet] loss at the final parameters
  float *scratch;             // per sample 4 * 64 + 2 floats
};

__global__ void __launch_bounds__(kMlpThreads) k_mlp_train(MlpTrainArgs a) {
  extern __shared__ float sm[];
  const MlpLayout L = mlp_layout(a.nin, a.nout);
  const int np = L.n, H = kMlpH, nin = a.nin, nout = a.nout;
  const int net = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  const int s0 = a.off[net], n = a.off[net + 1] - s0;
  float* p = sm;
  float* g = p + np;
  float* m1 = g + np;
  float* m2 = m1 + np;
  float* red = m2 + np;                       // [kMlpThreads]
  float* prm = a.params + (size_t)net * np;
  for (int i = tid; i < np; i += nt) { p[i] = prm[i]; m1[i] = 0.f; m2[i] = 0.f; }
  const float* X = a.x + (size_t)s0 * nin;
  const float* Y = a.y + (size_t)s0 * nout;
  const float* W = a.w + s0;
  float* H1 = a.scratch + (size_t)s0 * (4 * H + 2);
  float* H2 = H1 + (size_t)n * H;
  float* D2 = H2 + (size_t)n * H;
  float* D1 = D2 + (size_t)n * H;
  float* G3 = D1 + (size_t)n * H;             // [n][nout]
  // sum of weights
  float sw = 0.f;
  for (int s = tid; s < n; s += nt) sw += W[s];
  red[tid] = sw;
  __syncthreads();
  if (tid == 0) {
    float t = 0.f;
    for (int i = 0; i < nt; ++i) t += red[i];
    red[0] = t > 0.f ? 1.f / t : 0.f;
  }
  __syncthreads();
  const float isw = red[0];
  __syncthreads();
  float b1t = 1.f, b2t = 1.f;
  const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
  for (int ep = 0; ep <= a.epochs; ++ep) {
    const bool last = ep == a.epochs;
    // forward
    for (int idx = tid; idx < n * H; idx += nt) {
      const int s = idx / H, j = idx - s * H;
      float z = p[L.b1 + j];
      for (int i = 0; i < nin; ++i)
        z = fmaf(p[L.w1 + j * nin + i], (X[s * nin + i] - p[L.xo + i]) * p[L.xs + i], z);
      H1[idx] = tanhf(z);
    }
    __syncthreads();
    for (int idx = tid; idx < n * H; idx += nt) {
      const int s = idx / H, j = idx - s * H;
      float z = p[L.b2 + j];
      const float* h = H1 + (size_t)s * H;
      for (int k = 0; k < H; ++k) z = fmaf(p[L.w2 + j * H + k], h[k], z);
      H2[idx] = tanhf(z);
    }
    __syncthreads();
    // output error dL/do (normalised units) and the loss
    float lsum = 0.f;
    for (int idx = tid; idx < n * nout; idx += nt) {
      const int s = idx / nout, o = idx - s * nout;
      float z = p[L.b3 + o];
      const float* h = H2 + (size_t)s * H;
      for (int k = 0; k < H; ++k) z = fmaf(p[L.w3 + o * H + k], h[k], z);
      const float e = z - (Y[idx] - p[L.yo + o]) / p[L.ys + o];
      lsum += W[s] * e * e;
      G3[idx] = 2.f * W[s] * e * isw;
    }
    red[tid] = lsum;
    __syncthreads();
    if (last) {
      if (tid == 0) {
        float t = 0.f;
        for (int i = 0; i < nt; ++i) t += red[i];
        a.loss[net] = t * isw;
      }
      if (!a.grad) break;
    }
    // back-propagation through layer 3 and 2
    for (int idx = tid; idx < n * H; idx += nt) {
      const int s = idx / H, k = idx - s * H;
      float d = 0.f;
      for (int o = 0; o < nout; ++o) d = fmaf(p[L.w3 + o * H + k], G3[s * nout + o], d);
      const float h = H2[idx];
      D2[idx] = d * (1.f - h * h);
    }
    __syncthreads();
    for (int idx = tid; idx < n * H; idx += nt) {
      const int s = idx / H, k = idx - s * H;
      float d = 0.f;
      const float* dz = D2 + (size_t)s * H;
      for (int j = 0; j < H; ++j) d = fmaf(p[L.w2 + j * H + k], dz[j], d);
      const float h = H1[idx];
      D1[idx] = d * (1.f - h * h);
    }
    __syncthreads();
    // gradient: each entry one thread's sum over the samples
    for (int q = tid; q < L.xo; q += nt) {
      float acc = 0.f;
      if (q < L.b1) {                       // W1[j][i]
        const int j = q / nin, i = q - j * nin;
        for (int s = 0; s < n; ++s)
          acc = fmaf(D1[s * H + j], (X[s * nin + i] - p[L.xo + i]) * p[L.xs + i], acc);
      } else if (q < L.w2) {                // b1[j]
        const int j = q - L.b1;
        for (int s = 0; s < n; ++s) acc += D1[s * H + j];
      } else if (q < L.b2) {                // W2[j][k]
        const int j = (q - L.w2) / H, k = (q - L.w2) - j * H;
        for (int s = 0; s < n; ++s) acc = fmaf(D2[s * H + j], H1[s * H + k], acc);
      } else if (q < L.w3) {                // b2[j]
        const int j = q - L.b2;
        for (int s = 0; s < n; ++s) acc += D2[s * H + j];
      } else if (q < L.b3) {                // W3[o][k]
        const int o = (q - L.w3) / H, k = (q - L.w3) - o * H;
        for (int s = 0; s < n; ++s) acc = fmaf(G3[s * nout + o], H2[s * H + k], acc);
      } else {                              // b3[o]
        const int o = q - L.b3;
        for (int s = 0; s < n; ++s) acc += G3[s * nout + o];
      }
      g[q] = acc;
    }
    __syncthreads();
    if (last) {
      for (int q = tid; q < L.xo; q += nt) a.grad[(size_t)net * np + q] = g[q];
      break;
    }
    // Adam (the normalisation entries are not trained)
    b1t *= beta1;
    b2t *= beta2;
    const float c1 = 1.f / (1.f - b1t), c2 = 1.f / (1.f - b2t);
    for (int q = tid; q < L.xo; q += nt) {
      const float gq = g[q];
      const float mq = beta1 * m1[q] + (1.f - beta1) * gq;
      const float vq = beta2 * m2[q] + (1.f - beta2) * gq * gq;
      m1[q] = mq;
      m2[q] = vq;
      p[q] -= a.lr * (mq * c1) / (sqrtf(vq * c2) + eps);
    }
    __syncthreads();
  }
  __syncthreads();
  for (int i = tid; i < np; i += nt) prm[i] = p[i];
}

// batch inference: one warp per sample
__global__ void k_mlp_forward(const float* __restrict__ params, int nin, int nout,
                              const float* __restrict__ x, int n, float* __restrict__ y) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int s = warp; s < n; s += nw) {   // warp-uniform
    float out[JP_MLP_MAXIO];
    mlp_forward_warp(params, nin, nout, x + (size_t)s * nin, out);
    if ((threadIdx.x & 31) == 0)
      for (int o = 0; o < nout; ++o) y[(size_t)s * nout + o] = out[o];
  }
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

struct DevBuf {
  std::vector<void*> p;
  ~DevBuf() { for (void* q : p) cudaFree(q); }
  template <class T> T* get(size_t n) {
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(1, n) * sizeof(T)) != cudaSuccess) return nullptr;
    p.push_back(q);
    return static_cast<T*>(q);
  }
};

}  // namespace
}  // namespace jp

using namespace jp;

extern "C" int32_t jp_mlp_nparam(int32_t nin, int32_t nout) {
  if (nin < 1 || nin > JP_MLP_MAXIO || nout < 1 || nout > JP_MLP_MAXIO) return JP_E_INVALID;
  return mlp_layout(nin, nout).n;
}

extern "C" int jp_mlp_init(int32_t nin, int32_t nout, int32_t nnet, const float *x, const float *y,
                           const int32_t *off, uint64_t seed, float *params) {
  const int np = jp_mlp_nparam(nin, nout);
  if (np < 0 || nnet < 1 || !x || !y || !off || !params) return JP_E_INVALID;
  const MlpLayout L = mlp_layout(nin, nout);
  uint64_t st = seed;
  auto uni = [&]() { return (double)(splitmix(st) >> 11) * (1.0 / 9007199254740992.0); };
  for (int net = 0; net < nnet; ++net) {
    float* p = params + (size_t)net * np;
    const int s0 = off[net], n = off[net + 1] - s0;
    if (n < 1) return JP_E_INVALID;
    // Glorot-uniform weights, zero biases
    auto fill = [&](int o, int cnt, int fan_in, int fan_out) {
      const double lim = std::sqrt(6.0 / (fan_in + fan_out));
      for (int i = 0; i < cnt; ++i) p[o + i] = (float)((2.0 * uni() - 1.0) * lim);
    };
    fill(L.w1, kMlpH * nin, nin, kMlpH);
    fill(L.w2, kMlpH * kMlpH, kMlpH, kMlpH);
    fill(L.w3, kMlpH * nout, kMlpH, nout);
    for (int i = 0; i < kMlpH; ++i) { p[L.b1 + i] = 0.f; p[L.b2 + i] = 0.f; }
    for (int o = 0; o < nout; ++o) p[L.b3 + o] = 0.f;
    // inputs mapped to [-1, 1] over their range, targets to zero mean and unit spread
    for (int i = 0; i < nin; ++i) {
      double lo = 1e300, hi = -1e300;
      for (int s = s0; s < s0 + n; ++s) { lo = std::min(lo, (double)x[s * nin + i]); hi = std::max(hi, (double)x[s * nin + i]); }
      const double half = hi > lo ? 0.5 * (hi - lo) : 1.0;
      p[L.xo + i] = (float)(0.5 * (lo + hi));
      p[L.xs + i] = (float)(1.0 / half);
    }
    for (int o = 0; o < nout; ++o) {
      double m = 0.0, v = 0.0;
      for (int s = s0; s < s0 + n; ++s) m += y[s * nout + o];
      m /= n;
      for (int s = s0; s < s0 + n; ++s) v += (y[s * nout + o] - m) * (y[s * nout + o] - m);
      const double sd = std::sqrt(v / n);
      p[L.yo + o] = (float)m;
      p[L.ys + o] = (float)(sd > 0.0 ? sd : 1.0);
    }
  }
  return JP_OK;
}

extern "C" int jp_mlp_train(int32_t nin, int32_t nout, int32_t nnet, const float *x, const float *y,
                            const float *w, const int32_t *off, int32_t epochs, float lr,
                            int32_t device, float *params, float *loss, float *grad) {
  const int np = jp_mlp_nparam(nin, nout);
  if (np < 0 || nnet < 1 || !x || !y || !w || !off || !params || !loss || epochs < 0 || !(lr > 0.f))
    return JP_E_INVALID;
  const int total = off[nnet];
  for (int i = 0; i < nnet; ++i)
    if (off[i + 1] <= off[i]) return JP_E_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return JP_E_NO_DEVICE;
  DevBuf B;
  float* dx = B.get<float>((size_t)total * nin);
  float* dy = B.get<float>((size_t)total * nout);
  float* dw = B.get<float>(total);
  int* doff = B.get<int>(nnet + 1);
  float* dp = B.get<float>((size_t)nnet * np);
  float* dl = B.get<float>(nnet);
  float* dg = grad ? B.get<float>((size_t)nnet * np) : nullptr;
  float* scr = B.get<float>((size_t)total * (4 * kMlpH + 2));
  if (!dx || !dy || !dw || !doff || !dp || !dl || !scr || (grad && !dg)) return JP_E_CUDA;
  cudaMemcpy(dx, x, sizeof(float) * total * nin, cudaMemcpyHostToDevice);
  cudaMemcpy(dy, y, sizeof(float) * total * nout, cudaMemcpyHostToDevice);
  cudaMemcpy(dw, w, sizeof(float) * total, cudaMemcpyHostToDevice);
  cudaMemcpy(doff, off, sizeof(int) * (nnet + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(dp, params, sizeof(float) * nnet * np, cudaMemcpyHostToDevice);
  if (dg) cudaMemset(dg, 0, sizeof(float) * nnet * np);
  MlpTrainArgs a{dx, dy, dw, doff, nin, nout, epochs, lr, dp, dg, dl, scr};
  const size_t smem = sizeof(float) * (4 * np + kMlpThreads);
  if (cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return JP_E_CUDA;
  k_mlp_train<<<nnet, kMlpThreads, smem>>>(a);
  if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return JP_E_CUDA;
  cudaMemcpy(params, dp, sizeof(float) * nnet * np, cudaMemcpyDeviceToHost);
  cudaMemcpy(loss, dl, sizeof(float) * nnet, cudaMemcpyDeviceToHost);
  if (grad) cudaMemcpy(grad, dg, sizeof(float) * nnet * np, cudaMemcpyDeviceToHost);
  for (int i = 0; i < nnet; ++i)
    if (!std::isfinite(loss[i])) return JP_E_NONFINITE;
  return cudaGetLastError() == cudaSuccess ? JP_OK : JP_E_CUDA;
}

extern "C" int jp_mlp_forward(int32_t nin, int32_t nout, const float *params, const float *x,
                              int32_t n, int32_t device, float *y) {
  const int np = jp_mlp_nparam(nin, nout);
  if (np < 0 || n < 1 || !params || !x || !y) return JP_E_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return JP_E_NO_DEVICE;
  DevBuf B;
  float* dp = B.get<float>(np);
  float* dx = B.get<float>((size_t)n * nin);
  float* dy = B.get<float>((size_t)n * nout);
  if (!dp || !dx || !dy) return JP_E_CUDA;
  cudaMemcpy(dp, params, sizeof(float) * np, cudaMemcpyHostToDevice);
  cudaMemcpy(dx, x, sizeof(float) * n * nin, cudaMemcpyHostToDevice);
  const int blocks = std::min(1024, (n + 7) / 8);
  k_mlp_forward<<<blocks, 256>>>(dp, nin, nout, dx, n, dy);
  if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return JP_E_CUDA;
  cudaMemcpy(y, dy, sizeof(float) * n * nout, cudaMemcpyDeviceToHost);
  return JP_OK;
}
