// Learned join order: features and the MLP shape, shared by the host
// (training-sample construction) and the device (planner kernel).
//
// The model predicts, for one join step that adds query vertex v to the set
// P of already-placed vertices, the step's log expansion
//     delta = log2((rows_out + 1) / (rows_in + 1)),
// so a vertex order's predicted prefix sizes are
//     L_1 = log2(1 + |C(v_0)|),  L_{k+1} = L_k + delta_k,
// and its predicted work is sum_k 2^{L_k}. The planner picks the order with
// the smallest predicted work (greedy per start, a few starts); it only
// reorders joins, so the embedding set does not change.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define GPSM_HD __host__ __device__ __forceinline__
#else
#define GPSM_HD inline
#endif

namespace gpsm {

constexpr int kFeat = 16;        // input features
constexpr int kHidden = 64;      // two hidden layers of 64
constexpr int kMaxPlanQ = 128;   // query vertices the planner handles
// parameter layout (fp32 master / bf16 copy): W1[64][16] b1[64] W2[64][64] b2[64] W3[64] b3
constexpr int kW1 = 0, kB1 = kW1 + kHidden * kFeat, kW2 = kB1 + kHidden, kB2 = kW2 + kHidden * kHidden,
              kW3 = kB2 + kHidden, kB3 = kW3 + kHidden, kParams = kB3 + 1;

// Per-query inputs of the feature function (all host-computable after the
// filter stage; the planner receives the same struct on the device).
struct PlanQuery {
  uint32_t n;                        // query vertices (<= kMaxPlanQ)
  uint32_t pad;
  uint64_t adj[kMaxPlanQ][2];        // adjacency bitsets
  uint32_t label[kMaxPlanQ];
  uint32_t qdeg[kMaxPlanQ];
  float log_cand[kMaxPlanQ];         // log2(1 + |C(v)|) after refinement
  float log_labdeg[kMaxPlanQ];       // log2(1 + #data vertices with label(v), degree >= deg(v))
  float log_label[kMaxPlanQ];        // log2(1 + #data vertices with label(v))
};

// Directed candidate-edge statistics, dense [w][v]: log2(1 + size(w->v))
// and log2(1 + size(w->v) / |C(w)|) (the average list length).
struct PlanEdges {
  float log_size[kMaxPlanQ * kMaxPlanQ];
  float log_avg[kMaxPlanQ * kMaxPlanQ];
};

GPSM_HD bool pq_has(const uint64_t* bits, uint32_t v) { return (bits[v >> 6] >> (v & 63)) & 1ULL; }

// Features of the step adding v to P (bitset over query vertices).
GPSM_HD void step_features(const PlanQuery& Q, const PlanEdges& E, const uint64_t P[2], uint32_t psize, uint32_t v,
                           float* f) {
  float mn_avg = 1e30f, mx_avg = -1e30f, sum_avg = 0.f, mn_size = 1e30f, mn_cand_w = 1e30f;
  uint32_t b = 0, same = 0;
  for (uint32_t w = 0; w < Q.n; ++w) {
    if (!pq_has(P, w)) continue;
    if (Q.label[w] == Q.label[v]) ++same;
    if (!pq_has(Q.adj[v], w)) continue;
    ++b;
    const float a = E.log_avg[w * kMaxPlanQ + v];
    const float s = E.log_size[w * kMaxPlanQ + v];
    mn_avg = a < mn_avg ? a : mn_avg;
    mx_avg = a > mx_avg ? a : mx_avg;
    sum_avg += a;
    mn_size = s < mn_size ? s : mn_size;
    mn_cand_w = Q.log_cand[w] < mn_cand_w ? Q.log_cand[w] : mn_cand_w;
  }
  if (b == 0) {
    mn_avg = mx_avg = 0.f;
    mn_size = 0.f;
    mn_cand_w = 0.f;
  }
  f[0] = Q.log_cand[v] / 16.f;
  f[1] = (float)b / 8.f;
  f[2] = mn_avg / 8.f;
  f[3] = (b ? sum_avg / (float)b : 0.f) / 8.f;
  f[4] = mx_avg / 8.f;
  f[5] = mn_size / 32.f;
  f[6] = Q.log_label[v] / 24.f;
  f[7] = (float)Q.qdeg[v] / 8.f;
  f[8] = (float)psize / 32.f;
  f[9] = (float)same / 8.f;
  f[10] = (float)(Q.qdeg[v] - b) / 8.f;
  f[11] = (Q.log_labdeg[v] - Q.log_cand[v]) / 8.f;
  f[12] = (float)Q.n / 64.f;
  f[13] = b > 1 ? 1.f : 0.f;
  f[14] = mn_cand_w / 16.f;
  f[15] = (Q.log_cand[v] - mn_avg) / 16.f;
}

}  // namespace gpsm
