// Learned join order: a 16 -> 64 -> 64 -> 1 MLP (ReLU) with BF16 weights
// and FP32 accumulation, trained and evaluated by the kernels below, and the
// planner kernel that uses it to choose a vertex order on the device.
//
// Training keeps FP32 master weights and Adam moments; every forward pass
// reads the BF16 copy (round to nearest even), activations and sums are
// FP32, and gradients are taken with respect to the BF16 weights and applied
// to the masters. Loss: mean squared error on the step's log2 expansion.
//
// The layers are tiny (5,313 parameters), so the kernels are plain FMA
// loops with the weights staged in shared memory; there is no dense
// contraction large enough to pay for tensor-core tiles.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.h"
#include "learned.h"
#include "rng.h"

namespace gpsm {

// ---------------------------------------------------------------------------
// shared helpers
// ---------------------------------------------------------------------------
struct MlpSmem {
  float w1[kHidden * kFeat];
  float b1[kHidden];
  float w2[kHidden * kHidden];
  float b2[kHidden];
  float w3[kHidden];
  float b3;
};

__device__ __forceinline__ void stage_weights(MlpSmem& S, const __nv_bfloat16* __restrict__ wb,
                                              const float* __restrict__ wf) {
  // weights come from the bf16 copy, biases from the fp32 masters
  for (int i = threadIdx.x; i < kHidden * kFeat; i += blockDim.x) S.w1[i] = __bfloat162float(wb[kW1 + i]);
  for (int i = threadIdx.x; i < kHidden * kHidden; i += blockDim.x) S.w2[i] = __bfloat162float(wb[kW2 + i]);
  for (int i = threadIdx.x; i < kHidden; i += blockDim.x) {
    S.b1[i] = wf[kB1 + i];
    S.b2[i] = wf[kB2 + i];
    S.w3[i] = __bfloat162float(wb[kW3 + i]);
  }
  if (threadIdx.x == 0) S.b3 = wf[kB3];
}

__device__ __forceinline__ float mlp_eval(const MlpSmem& S, const float* x, float* h1, float* h2) {
#pragma unroll 4
  for (int j = 0; j < kHidden; ++j) {
    float a = S.b1[j];
#pragma unroll
    for (int k = 0; k < kFeat; ++k) a = fmaf(S.w1[j * kFeat + k], x[k], a);
    h1[j] = a > 0.f ? a : 0.f;
  }
#pragma unroll 2
  for (int j = 0; j < kHidden; ++j) {
    float a = S.b2[j];
#pragma unroll 8
    for (int k = 0; k < kHidden; ++k) a = fmaf(S.w2[j * kHidden + k], h1[k], a);
    h2[j] = a > 0.f ? a : 0.f;
  }
  float o = S.b3;
#pragma unroll 8
  for (int k = 0; k < kHidden; ++k) o = fmaf(S.w3[k], h2[k], o);
  return o;
}

// ---------------------------------------------------------------------------
// training and inference kernels
// ---------------------------------------------------------------------------
// Forward over n samples (rows of x selected by idx, or 0..n-1 when idx is
// null). Stores H1, H2 for the backward pass when h1/h2 are non-null, the
// output in out, and, when y is given, dO = (out - y) * scale and the loss.
__global__ void __launch_bounds__(128) k_mlp_forward(const float* __restrict__ x, const float* __restrict__ y,
                                                     const uint32_t* __restrict__ idx, uint32_t n,
                                                     const __nv_bfloat16* __restrict__ wb,
                                                     const float* __restrict__ wf, float* __restrict__ h1o,
                                                     float* __restrict__ h2o, float* __restrict__ out,
                                                     float* __restrict__ dout, float scale,
                                                     float* __restrict__ loss) {
  __shared__ MlpSmem S;
  stage_weights(S, wb, wf);
  __syncthreads();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (i < n) {
    const uint32_t r = idx ? idx[i] : i;
    float xv[kFeat], h1[kHidden], h2[kHidden];
#pragma unroll
    for (int k = 0; k < kFeat; ++k) xv[k] = x[(size_t)r * kFeat + k];
    const float o = mlp_eval(S, xv, h1, h2);
    if (h1o)
      for (int k = 0; k < kHidden; ++k) h1o[(size_t)i * kHidden + k] = h1[k];
    if (h2o)
      for (int k = 0; k < kHidden; ++k) h2o[(size_t)i * kHidden + k] = h2[k];
    if (out) out[i] = o;
    if (y) {
      const float d = o - y[r];
      if (dout) dout[i] = d * scale;
      l = 0.5f * d * d * scale;
    }
  }
  if (loss) {
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.f) atomicAdd(loss, l);
  }
}

// dH2 = dO * W3 * [H2 > 0]; dH1 = (dH2 W2) * [H1 > 0]; one thread per sample.
__global__ void __launch_bounds__(128) k_mlp_backward_data(const float* __restrict__ h1, const float* __restrict__ h2,
                                                           const float* __restrict__ dout, uint32_t n,
                                                           const __nv_bfloat16* __restrict__ wb,
                                                           const float* __restrict__ wf, float* __restrict__ dh1,
                                                           float* __restrict__ dh2) {
  __shared__ MlpSmem S;
  stage_weights(S, wb, wf);
  __syncthreads();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float d = dout[i];
  float g2[kHidden];
#pragma unroll 8
  for (int j = 0; j < kHidden; ++j) {
    g2[j] = h2[(size_t)i * kHidden + j] > 0.f ? d * S.w3[j] : 0.f;
    dh2[(size_t)i * kHidden + j] = g2[j];
  }
  for (int k = 0; k < kHidden; ++k) {
    float a = 0.f;
#pragma unroll 8
    for (int j = 0; j < kHidden; ++j) a = fmaf(g2[j], S.w2[j * kHidden + k], a);
    dh1[(size_t)i * kHidden + k] = h1[(size_t)i * kHidden + k] > 0.f ? a : 0.f;
  }
}

// Weight gradient of one dense layer: dW[m][k] = sum_s dC[s][m] * A[s][k],
// db[m] = sum_s dC[s][m]. One block per output row m. A rows are selected
// by idx when given (the layer-1 input is the gathered minibatch).
template <int K>
__global__ void __launch_bounds__(256) k_mlp_wgrad(const float* __restrict__ dc, uint32_t ldc,
                                                   const float* __restrict__ a, const uint32_t* __restrict__ idx,
                                                   uint32_t n, float* __restrict__ dw, float* __restrict__ db) {
  const uint32_t m = blockIdx.x;
  float acc[K];
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = 0.f;
  float accb = 0.f;
  for (uint32_t s = threadIdx.x; s < n; s += blockDim.x) {
    const float g = dc[(size_t)s * ldc + m];
    if (g == 0.f) continue;
    const uint32_t r = idx ? idx[s] : s;
    accb += g;
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = fmaf(g, a[(size_t)r * K + k], acc[k]);
  }
  __shared__ float red[8][K + 1];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    float v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[wid][k] = v;
  }
  for (int o = 16; o > 0; o >>= 1) accb += __shfl_xor_sync(0xffffffffu, accb, o);
  if (lane == 0) red[wid][K] = accb;
  __syncthreads();
  if (threadIdx.x <= (unsigned)K) {
    float v = 0.f;
    for (int w = 0; w < 8; ++w) v += red[w][threadIdx.x];
    if (threadIdx.x < (unsigned)K) dw[(size_t)m * K + threadIdx.x] = v;
    else if (db) db[m] = v;
  }
}

__global__ void k_mlp_adam(float* __restrict__ w, __nv_bfloat16* __restrict__ wb, const float* __restrict__ g,
                           float* __restrict__ m1, float* __restrict__ m2, uint32_t n, float lr, float b1, float b2,
                           float eps, float bc1, float bc2) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float upd = lr * (a / bc1) / (sqrtf(b / bc2) + eps);
    w[i] -= upd;
    wb[i] = __float2bfloat16_rn(w[i]);
  }
}

__global__ void k_mlp_to_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    wb[i] = __float2bfloat16_rn(w[i]);
}

// ---------------------------------------------------------------------------
// planner: one warp per start vertex runs the greedy order.
// ---------------------------------------------------------------------------
constexpr int kPlanWarps = 9;  // up to 8 greedy starts + the scored plain order (one block each)
constexpr int kPlanTeam = 8;   // warps of a plan's block: frontier candidates scored 8 at a time
struct PlanOut {
  int32_t order[kMaxPlanQ];
  float work;     // predicted sum of 2^{L_k} over the intermediate tables (widths 1 .. n-1)
  float peak;     // predicted max_k 2^{L_k} * 4 * (k + 1) bytes (the largest whole table)
  float pad[2];
  float logsize[kMaxPlanQ];  // L_k: predicted log2 rows of the table of width k + 1
};

// Weights for the planner, laid out for lane-parallel evaluation: lane j of
// a warp computes hidden units j and j + 32, so layer weights are stored
// input-major (w1t[k][j] = W1[j][k]): a warp's 32 loads of one input row
// hit 32 consecutive words.
struct PlanSmem {
  float w1t[kFeat][kHidden];
  float b1[kHidden];
  float w2t[kHidden][kHidden];
  float b2[kHidden];
  float w3[kHidden];
  float b3;
  float x[kPlanTeam][kFeat];    // features of the candidate a warp scores
  float h1[kPlanTeam][kHidden];
  float h2[kPlanTeam][kHidden];
  float best[kPlanTeam];        // each warp's best candidate of the step
  uint32_t bv[kPlanTeam];
};

// One block per start vertex builds a greedy order; when `fixed` is given,
// block `nstarts` scores that order instead (same predictions, no choice).
// Each step, the block's warps score the frontier candidates, eight at a
// time (the i-th candidate in vertex order goes to warp i mod 8), lanes
// splitting the hidden units; each unit's sum runs over its inputs in the
// same order as mlp_eval, and lane 0 forms the output sum in order, so the
// predictions equal mlp_eval's. The step takes the smallest prediction,
// ties to the smallest vertex, as a scan in vertex order would.
__global__ void __launch_bounds__(32 * kPlanTeam, 1) k_plan(const PlanQuery* __restrict__ Qp,
                                                          const PlanEdges* __restrict__ E,
                                                          const uint32_t* __restrict__ starts, uint32_t nstarts,
                                                          const int32_t* __restrict__ fixed,
                                                          const __nv_bfloat16* __restrict__ wb,
                                                          const float* __restrict__ wf, PlanOut* __restrict__ outs) {
  __shared__ PlanSmem S;
  for (int i = threadIdx.x; i < kHidden * kFeat; i += blockDim.x) {
    const int j = i / kFeat, k = i % kFeat;
    S.w1t[k][j] = __bfloat162float(wb[kW1 + i]);
  }
  for (int i = threadIdx.x; i < kHidden * kHidden; i += blockDim.x) {
    const int j = i / kHidden, k = i % kHidden;
    S.w2t[k][j] = __bfloat162float(wb[kW2 + i]);
  }
  for (int i = threadIdx.x; i < kHidden; i += blockDim.x) {
    S.b1[i] = wf[kB1 + i];
    S.b2[i] = wf[kB2 + i];
    S.w3[i] = __bfloat162float(wb[kW3 + i]);
  }
  if (threadIdx.x == 0) S.b3 = wf[kB3];
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5, plan = blockIdx.x;
  const bool follow = fixed && plan == nstarts;
  if (plan >= nstarts && !follow) return;  // block-uniform
  const PlanQuery& Q = *Qp;
  const uint32_t n = Q.n;
  PlanOut& O = outs[plan];
  uint64_t P[2] = {0, 0};
  const uint32_t v0 = follow ? (uint32_t)fixed[0] : starts[plan];
  P[v0 >> 6] |= 1ULL << (v0 & 63);
  if (threadIdx.x == 0) O.order[0] = (int32_t)v0;
  float L = Q.log_cand[v0];
  if (threadIdx.x == 0) O.logsize[0] = L;
  float work = exp2f(L), peak = exp2f(L) * 4.f;
  float* x = S.x[wid];
  float* h1 = S.h1[wid];
  float* h2 = S.h2[wid];
  for (uint32_t k = 1; k < n; ++k) {
    float best = 1e30f;
    uint32_t bv = 0xffffffffu;
    uint32_t seen = 0;                   // frontier candidates so far (block-uniform)
    for (uint32_t v = 0; v < n; ++v) {  // block-uniform
      if (pq_has(P, v)) continue;
      if (!((Q.adj[v][0] & P[0]) | (Q.adj[v][1] & P[1]))) continue;
      if (follow && v != (uint32_t)fixed[k]) continue;
      if ((seen++ % kPlanTeam) != wid) continue;  // another warp scores it (warp-uniform)
      if (lane == 0) step_features(Q, *E, P, k, v, x);
      __syncwarp();
      float a0 = S.b1[lane], a1 = S.b1[lane + 32];
#pragma unroll
      for (int f = 0; f < kFeat; ++f) {
        const float xf = x[f];
        a0 = fmaf(S.w1t[f][lane], xf, a0);
        a1 = fmaf(S.w1t[f][lane + 32], xf, a1);
      }
      h1[lane] = a0 > 0.f ? a0 : 0.f;
      h1[lane + 32] = a1 > 0.f ? a1 : 0.f;
      __syncwarp();
      float c0 = S.b2[lane], c1 = S.b2[lane + 32];
#pragma unroll 16
      for (int f = 0; f < kHidden; ++f) {
        const float hf = h1[f];
        c0 = fmaf(S.w2t[f][lane], hf, c0);
        c1 = fmaf(S.w2t[f][lane + 32], hf, c1);
      }
      h2[lane] = c0 > 0.f ? c0 : 0.f;
      h2[lane + 32] = c1 > 0.f ? c1 : 0.f;
      __syncwarp();
      float d = 0.f;
      if (lane == 0) {
        float o = S.b3;
        for (int f = 0; f < kHidden; ++f) o = fmaf(S.w3[f], h2[f], o);
        d = o;
      }
      d = __shfl_sync(0xffffffffu, d, 0);
      __syncwarp();  // x, h1, h2 are rewritten for the next candidate
      if (d < best || (d == best && v < bv)) {
        best = d;
        bv = v;
      }
    }
    // the block's best: the smallest prediction, ties to the smallest vertex
    if (lane == 0) {
      S.best[wid] = best;
      S.bv[wid] = bv;
    }
    __syncthreads();
    best = 1e30f;
    bv = 0xffffffffu;
    for (int w = 0; w < kPlanTeam; ++w)
      if (S.bv[w] != 0xffffffffu && (S.best[w] < best || (S.best[w] == best && S.bv[w] < bv))) {
        best = S.best[w];
        bv = S.bv[w];
      }
    __syncthreads();  // S.best / S.bv are rewritten next step
    if (bv == 0xffffffffu) break;  // disconnected (rejected earlier)
    P[bv >> 6] |= 1ULL << (bv & 63);
    if (threadIdx.x == 0) O.order[k] = (int32_t)bv;
    L += best;
    L = L < 0.f ? 0.f : L;
    if (threadIdx.x == 0) O.logsize[k] = L;
    const float rows = exp2f(L);
    // the final table holds the embeddings, the same in every order (and,
    // under a cap, the same number of rows): it does not rank orders
    if (k + 1 < n) work += rows;
    peak = fmaxf(peak, rows * 4.f * (float)(k + 1));
  }
  if (threadIdx.x == 0) {
    O.work = work;
    O.peak = peak;
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct Model {
  int device = 0;
  float* w = nullptr;            // fp32 masters
  __nv_bfloat16* wb = nullptr;   // bf16 copy used by every forward pass
  float* m1 = nullptr;
  float* m2 = nullptr;
  float* g = nullptr;
  uint64_t step = 0;
};

Model* model_create(int device, uint64_t seed) {
  GPSM_CUDA(cudaSetDevice(device));
  Model* M = new Model();
  M->device = device;
  GPSM_CUDA(cudaMalloc(&M->w, kParams * sizeof(float)));
  GPSM_CUDA(cudaMalloc(&M->wb, kParams * sizeof(__nv_bfloat16)));
  GPSM_CUDA(cudaMalloc(&M->m1, kParams * sizeof(float)));
  GPSM_CUDA(cudaMalloc(&M->m2, kParams * sizeof(float)));
  GPSM_CUDA(cudaMalloc(&M->g, kParams * sizeof(float)));
  // He-style uniform initialisation from a seeded stream
  std::vector<float> w(kParams, 0.f);
  Rng r(seed, 0x317);
  auto fill = [&](int off, int fan_in, int count) {
    const float lim = std::sqrt(6.f / (float)fan_in);
    for (int i = 0; i < count; ++i) w[off + i] = (float)((r.uniform() * 2.0 - 1.0) * lim);
  };
  fill(kW1, kFeat, kHidden * kFeat);
  fill(kW2, kHidden, kHidden * kHidden);
  fill(kW3, kHidden, kHidden);
  GPSM_CUDA(cudaMemcpy(M->w, w.data(), kParams * sizeof(float), cudaMemcpyHostToDevice));
  GPSM_CUDA(cudaMemset(M->m1, 0, kParams * sizeof(float)));
  GPSM_CUDA(cudaMemset(M->m2, 0, kParams * sizeof(float)));
  k_mlp_to_bf16<<<(kParams + 255) / 256, 256>>>(M->w, M->wb, kParams);
  GPSM_LAUNCHED();
  GPSM_CUDA(cudaDeviceSynchronize());
  return M;
}

void model_free(Model* M) {
  if (!M) return;
  cudaSetDevice(M->device);
  cudaFree(M->w);
  cudaFree(M->wb);
  cudaFree(M->m1);
  cudaFree(M->m2);
  cudaFree(M->g);
  delete M;
}

void model_set(Model* M, const float* w) {
  GPSM_CUDA(cudaSetDevice(M->device));
  GPSM_CUDA(cudaMemcpy(M->w, w, kParams * sizeof(float), cudaMemcpyHostToDevice));
  GPSM_CUDA(cudaMemset(M->m1, 0, kParams * sizeof(float)));
  GPSM_CUDA(cudaMemset(M->m2, 0, kParams * sizeof(float)));
  M->step = 0;
  k_mlp_to_bf16<<<(kParams + 255) / 256, 256>>>(M->w, M->wb, kParams);
  GPSM_LAUNCHED();
  GPSM_CUDA(cudaDeviceSynchronize());
}

void model_get(Model* M, float* w) {
  GPSM_CUDA(cudaSetDevice(M->device));
  GPSM_CUDA(cudaMemcpy(w, M->w, kParams * sizeof(float), cudaMemcpyDeviceToHost));
}

namespace {
struct DevBuf {
  void* p = nullptr;
  explicit DevBuf(size_t bytes) { GPSM_CUDA(cudaMalloc(&p, std::max<size_t>(bytes, 16))); }
  ~DevBuf() { cudaFree(p); }
  template <class T>
  T* as() const {
    return (T*)p;
  }
};

// forward + backward of one minibatch (rows idx[0..nb)) into M->g; returns nothing (loss accumulates)
void grad_batch(Model* M, const float* dx, const float* dy, const uint32_t* didx, uint32_t nb, float* h1, float* h2,
                float* out, float* dout, float* dh1, float* dh2, float* dloss, cudaStream_t s) {
  const uint32_t blocks = (nb + 127) / 128;
  k_mlp_forward<<<blocks, 128, 0, s>>>(dx, dy, didx, nb, M->wb, M->w, h1, h2, out, dout, 1.f / (float)nb, dloss);
  GPSM_LAUNCHED();
  k_mlp_backward_data<<<blocks, 128, 0, s>>>(h1, h2, dout, nb, M->wb, M->w, dh1, dh2);
  GPSM_LAUNCHED();
  k_mlp_wgrad<kHidden><<<1, 256, 0, s>>>(dout, 1, h2, nullptr, nb, M->g + kW3, M->g + kB3);
  GPSM_LAUNCHED();
  k_mlp_wgrad<kHidden><<<kHidden, 256, 0, s>>>(dh2, kHidden, h1, nullptr, nb, M->g + kW2, M->g + kB2);
  GPSM_LAUNCHED();
  k_mlp_wgrad<kFeat><<<kHidden, 256, 0, s>>>(dh1, kHidden, dx, didx, nb, M->g + kW1, M->g + kB1);
  GPSM_LAUNCHED();
}
}  // namespace

// Mean-squared-error gradient over all n samples (no update): grad[kParams].
float model_grad(Model* M, const float* x, const float* y, uint32_t n, float* grad) {
  GPSM_CUDA(cudaSetDevice(M->device));
  DevBuf dx((size_t)n * kFeat * 4), dy((size_t)n * 4), h1((size_t)n * kHidden * 4), h2((size_t)n * kHidden * 4),
      out((size_t)n * 4), dout((size_t)n * 4), dh1((size_t)n * kHidden * 4), dh2((size_t)n * kHidden * 4), dl(4);
  GPSM_CUDA(cudaMemcpy(dx.p, x, (size_t)n * kFeat * 4, cudaMemcpyHostToDevice));
  GPSM_CUDA(cudaMemcpy(dy.p, y, (size_t)n * 4, cudaMemcpyHostToDevice));
  GPSM_CUDA(cudaMemset(dl.p, 0, 4));
  grad_batch(M, dx.as<float>(), dy.as<float>(), nullptr, n, h1.as<float>(), h2.as<float>(), out.as<float>(),
             dout.as<float>(), dh1.as<float>(), dh2.as<float>(), dl.as<float>(), 0);
  GPSM_CUDA(cudaDeviceSynchronize());
  GPSM_CUDA(cudaMemcpy(grad, M->g, kParams * 4, cudaMemcpyDeviceToHost));
  float loss = 0;
  GPSM_CUDA(cudaMemcpy(&loss, dl.p, 4, cudaMemcpyDeviceToHost));
  return loss;
}

// Adam on minibatches; returns the mean loss of the last epoch.
float model_train(Model* M, const float* x, const float* y, uint32_t n, uint32_t epochs, uint32_t batch, float lr,
                  uint64_t seed) {
  GPSM_CUDA(cudaSetDevice(M->device));
  batch = std::max<uint32_t>(1, std::min(batch, n));
  DevBuf dx((size_t)n * kFeat * 4), dy((size_t)n * 4), didx((size_t)n * 4), h1((size_t)batch * kHidden * 4),
      h2((size_t)batch * kHidden * 4), out((size_t)batch * 4), dout((size_t)batch * 4),
      dh1((size_t)batch * kHidden * 4), dh2((size_t)batch * kHidden * 4), dl(4);
  GPSM_CUDA(cudaMemcpy(dx.p, x, (size_t)n * kFeat * 4, cudaMemcpyHostToDevice));
  GPSM_CUDA(cudaMemcpy(dy.p, y, (size_t)n * 4, cudaMemcpyHostToDevice));
  std::vector<uint32_t> perm(n);
  for (uint32_t i = 0; i < n; ++i) perm[i] = i;
  Rng r(seed, 0x7a1);
  float last = 0.f;
  for (uint32_t ep = 0; ep < epochs; ++ep) {
    for (uint32_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[r.below(i + 1)]);
    GPSM_CUDA(cudaMemcpy(didx.p, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice));
    GPSM_CUDA(cudaMemset(dl.p, 0, 4));
    uint32_t nbatches = 0;
    for (uint32_t b0 = 0; b0 < n; b0 += batch) {
      const uint32_t nb = std::min(batch, n - b0);
      grad_batch(M, dx.as<float>(), dy.as<float>(), didx.as<uint32_t>() + b0, nb, h1.as<float>(), h2.as<float>(),
                 out.as<float>(), dout.as<float>(), dh1.as<float>(), dh2.as<float>(), dl.as<float>(), 0);
      ++M->step;
      const float bc1 = 1.f - std::pow(0.9f, (float)M->step), bc2 = 1.f - std::pow(0.999f, (float)M->step);
      k_mlp_adam<<<(kParams + 255) / 256, 256>>>(M->w, M->wb, M->g, M->m1, M->m2, kParams, lr, 0.9f, 0.999f, 1e-8f,
                                                  bc1, bc2);
      GPSM_LAUNCHED();
      ++nbatches;
    }
    GPSM_CUDA(cudaMemcpy(&last, dl.p, 4, cudaMemcpyDeviceToHost));
    last /= (float)std::max<uint32_t>(nbatches, 1);
  }
  GPSM_CUDA(cudaDeviceSynchronize());
  return last;
}

void model_predict(Model* M, const float* x, uint32_t n, float* y) {
  GPSM_CUDA(cudaSetDevice(M->device));
  DevBuf dx((size_t)n * kFeat * 4), out((size_t)n * 4);
  GPSM_CUDA(cudaMemcpy(dx.p, x, (size_t)n * kFeat * 4, cudaMemcpyHostToDevice));
  k_mlp_forward<<<(n + 127) / 128, 128>>>(dx.as<float>(), nullptr, nullptr, n, M->wb, M->w, nullptr, nullptr,
                                          out.as<float>(), nullptr, 1.f, nullptr);
  GPSM_LAUNCHED();
  GPSM_CUDA(cudaMemcpy(y, out.p, (size_t)n * 4, cudaMemcpyDeviceToHost));
}

// Runs the planner for `nstarts` start vertices on `stream`; d_q, d_e, d_starts
// and d_out are device buffers (workspace memory). Asynchronous.
// d_fixed (or null): an order of the n query vertices to score; its result
// is written after the nstarts greedy plans.
void launch_plan(cudaStream_t s, const Model* M, const PlanQuery* d_q, const PlanEdges* d_e, const uint32_t* d_starts,
                 uint32_t nstarts, const int32_t* d_fixed, void* d_out) {
  nstarts = std::min<uint32_t>(nstarts, kPlanWarps - 1);
  const uint32_t plans = std::max<uint32_t>(1, nstarts + (d_fixed ? 1 : 0));
  k_plan<<<plans, 32 * kPlanTeam, 0, s>>>(d_q, d_e, d_starts, nstarts, d_fixed, M->wb, M->w, (PlanOut*)d_out);
  GPSM_LAUNCHED();
}

size_t plan_out_bytes() { return sizeof(PlanOut); }

}  // namespace gpsm
