// gearmlp.cu - the learned gear controller's network: a 16 -> 64 -> 64 -> 4
// FP32 MLP (ReLU hidden layers, linear output = predicted SNR per gear),
// with hand-written forward, backward and Adam kernels.
//
// Parameter layout (GM_PARAMS floats): W1[64][16], b1[64], W2[64][64],
// b2[64], W3[4][64], b3[4].  Loss: mean over the batch of
// sum_o mask[b][o] (y[b][o] - t[b][o])^2.  Gradient reductions over the batch
// are done by one thread per parameter (no atomics), so results are
// deterministic and reproducible run to run.
#include "dispatch.cuh"

constexpr int GM_IN = 16, GM_H = 64, GM_OUT = 4;
constexpr int GM_W1 = 0, GM_B1 = GM_W1 + GM_H * GM_IN, GM_W2 = GM_B1 + GM_H,
              GM_B2 = GM_W2 + GM_H * GM_H, GM_W3 = GM_B2 + GM_H, GM_B3 = GM_W3 + GM_OUT * GM_H,
              GM_PARAMS = GM_B3 + GM_OUT;
constexpr int GM_CACHE = 2 * GM_H;  // per sample: h1, h2 (post-ReLU)

__global__ void __launch_bounds__(128)
    k_gm_forward(const float* __restrict__ P, const float* __restrict__ x, float* __restrict__ y,
                 float* __restrict__ cache, int batch) {
  __shared__ float sp[GM_PARAMS];
  for (int i = threadIdx.x; i < GM_PARAMS; i += blockDim.x) sp[i] = P[i];
  __syncthreads();
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  float xi[GM_IN];
#pragma unroll
  for (int i = 0; i < GM_IN; ++i) xi[i] = x[(size_t)b * GM_IN + i];
  float h1[GM_H];
#pragma unroll
  for (int k = 0; k < GM_H; ++k) {
    float s = sp[GM_B1 + k];
#pragma unroll
    for (int i = 0; i < GM_IN; ++i) s = fmaf(sp[GM_W1 + k * GM_IN + i], xi[i], s);
    h1[k] = fmaxf(s, 0.f);
    if (cache) cache[(size_t)b * GM_CACHE + k] = h1[k];
  }
  float out[GM_OUT];
#pragma unroll
  for (int o = 0; o < GM_OUT; ++o) out[o] = sp[GM_B3 + o];
#pragma unroll 4
  for (int j = 0; j < GM_H; ++j) {
    float s = sp[GM_B2 + j];
#pragma unroll
    for (int k = 0; k < GM_H; ++k) s = fmaf(sp[GM_W2 + j * GM_H + k], h1[k], s);
    const float h2 = fmaxf(s, 0.f);
    if (cache) cache[(size_t)b * GM_CACHE + GM_H + j] = h2;
#pragma unroll
    for (int o = 0; o < GM_OUT; ++o) out[o] = fmaf(sp[GM_W3 + o * GM_H + j], h2, out[o]);
  }
#pragma unroll
  for (int o = 0; o < GM_OUT; ++o) y[(size_t)b * GM_OUT + o] = out[o];
}

// per sample: dy, dh2 (pre-activation), dh1 (pre-activation) -> dcache [b][4 + 64 + 64]
constexpr int GM_DC = GM_OUT + 2 * GM_H;

__global__ void __launch_bounds__(128)
    k_gm_backprop(const float* __restrict__ P, const float* __restrict__ cache,
                  const float* __restrict__ y, const float* __restrict__ t,
                  const float* __restrict__ mask, float* __restrict__ dcache, int batch) {
  __shared__ float sp[GM_PARAMS];
  for (int i = threadIdx.x; i < GM_PARAMS; i += blockDim.x) sp[i] = P[i];
  __syncthreads();
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  const float inv_b = 1.0f / (float)batch;
  float dy[GM_OUT];
#pragma unroll
  for (int o = 0; o < GM_OUT; ++o) {
    const float m = mask ? mask[(size_t)b * GM_OUT + o] : 1.0f;
    dy[o] = 2.0f * m * (y[(size_t)b * GM_OUT + o] - t[(size_t)b * GM_OUT + o]) * inv_b;
    dcache[(size_t)b * GM_DC + o] = dy[o];
  }
  const float* h1 = cache + (size_t)b * GM_CACHE;
  const float* h2 = h1 + GM_H;
  float dh2[GM_H];
#pragma unroll
  for (int j = 0; j < GM_H; ++j) {
    float s = 0.f;
#pragma unroll
    for (int o = 0; o < GM_OUT; ++o) s = fmaf(dy[o], sp[GM_W3 + o * GM_H + j], s);
    dh2[j] = h2[j] > 0.f ? s : 0.f;
    dcache[(size_t)b * GM_DC + GM_OUT + j] = dh2[j];
  }
#pragma unroll 4
  for (int k = 0; k < GM_H; ++k) {
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < GM_H; ++j) s = fmaf(dh2[j], sp[GM_W2 + j * GM_H + k], s);
    dcache[(size_t)b * GM_DC + GM_OUT + GM_H + k] = h1[k] > 0.f ? s : 0.f;
  }
}

// one thread per parameter: sum over the batch
__global__ void k_gm_grad(const float* __restrict__ x, const float* __restrict__ cache,
                          const float* __restrict__ dcache, float* __restrict__ grad, int batch) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= GM_PARAMS) return;
  float s = 0.f;
  if (p < GM_B1) {  // W1[k][i]: dh1[k] * x[i]
    const int k = p / GM_IN, i = p % GM_IN;
    for (int b = 0; b < batch; ++b)
      s = fmaf(dcache[(size_t)b * GM_DC + GM_OUT + GM_H + k], x[(size_t)b * GM_IN + i], s);
  } else if (p < GM_W2) {
    const int k = p - GM_B1;
    for (int b = 0; b < batch; ++b) s += dcache[(size_t)b * GM_DC + GM_OUT + GM_H + k];
  } else if (p < GM_B2) {  // W2[j][k]: dh2[j] * h1[k]
    const int j = (p - GM_W2) / GM_H, k = (p - GM_W2) % GM_H;
    for (int b = 0; b < batch; ++b)
      s = fmaf(dcache[(size_t)b * GM_DC + GM_OUT + j], cache[(size_t)b * GM_CACHE + k], s);
  } else if (p < GM_W3) {
    const int j = p - GM_B2;
    for (int b = 0; b < batch; ++b) s += dcache[(size_t)b * GM_DC + GM_OUT + j];
  } else if (p < GM_B3) {  // W3[o][j]: dy[o] * h2[j]
    const int o = (p - GM_W3) / GM_H, j = (p - GM_W3) % GM_H;
    for (int b = 0; b < batch; ++b)
      s = fmaf(dcache[(size_t)b * GM_DC + o], cache[(size_t)b * GM_CACHE + GM_H + j], s);
  } else {
    const int o = p - GM_B3;
    for (int b = 0; b < batch; ++b) s += dcache[(size_t)b * GM_DC + o];
  }
  grad[p] = s;
}

__global__ void k_gm_adam(float* __restrict__ P, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, float lr, float b1, float b2, float eps, float c1,
                          float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= GM_PARAMS) return;
  const float gp = g[p];
  const float mp = b1 * m[p] + (1.f - b1) * gp;
  const float vp = b2 * v[p] + (1.f - b2) * gp * gp;
  m[p] = mp;
  v[p] = vp;
  P[p] -= lr * (mp / c1) / (sqrtf(vp / c2) + eps);
}

extern "C" int ckks_gear_mlp_param_count(void) { return GM_PARAMS; }

extern "C" int ckks_gear_mlp_forward(const float* params, const float* x, float* y, float* cache,
                                     int batch, void* stream) {
  CKKS_REQUIRE(batch >= 0, "ckks_gear_mlp_forward: batch < 0");
  CKKS_REQUIRE(params && x && y, "ckks_gear_mlp_forward: NULL argument");
  if (batch == 0) return CKKS_OK;
  k_gm_forward<<<(batch + 127) / 128, 128, 0, as_stream(stream)>>>(params, x, y, cache, batch);
  return ckks_check_launch("ckks_gear_mlp_forward");
}

extern "C" int ckks_gear_mlp_backward(const float* params, const float* x, const float* cache,
                                      const float* y, const float* target, const float* mask,
                                      float* grad, float* dcache, int batch, void* stream) {
  CKKS_REQUIRE(batch >= 1, "ckks_gear_mlp_backward: batch < 1");
  CKKS_REQUIRE(params && x && cache && y && target && grad && dcache,
               "ckks_gear_mlp_backward: NULL argument");
  cudaStream_t st = as_stream(stream);
  k_gm_backprop<<<(batch + 127) / 128, 128, 0, st>>>(params, cache, y, target, mask, dcache, batch);
  if (int rc = ckks_check_launch("ckks_gear_mlp_backward")) return rc;
  k_gm_grad<<<(GM_PARAMS + 127) / 128, 128, 0, st>>>(x, cache, dcache, grad, batch);
  return ckks_check_launch("ckks_gear_mlp_backward");
}

extern "C" int ckks_gear_mlp_adam(float* params, const float* grad, float* m, float* v, int step,
                                  float lr, float beta1, float beta2, float eps, void* stream) {
  CKKS_REQUIRE(step >= 1, "ckks_gear_mlp_adam: step must start at 1");
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  k_gm_adam<<<(GM_PARAMS + 127) / 128, 128, 0, as_stream(stream)>>>(params, grad, m, v, lr, beta1,
                                                                   beta2, eps, c1, c2);
  return ckks_check_launch("ckks_gear_mlp_adam");
}
