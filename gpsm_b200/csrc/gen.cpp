// Seeded synthetic workloads: Erdos-Renyi G(n, m) and R-MAT data graphs,
// uniform and Zipf vertex labels, undirected CSR construction with sorted
// adjacency, and random-walk query extraction.
//
// The reference reads its graphs from text files (io/IO.cpp:46-128) and
// builds the undirected CSR on the host (graph/Graph.cpp:30-65: in- and
// out-lists merged, each list sorted ascending). gpsm_csr_from_edges
// produces the same arrays from an edge list in which every undirected edge
// appears once, which is the file convention the reference assumes
// (README.md: "A->B and B->A" create parallel edges).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "gpsm.h"
#include "rng.h"

namespace gpsm {

static int hw_threads() {
  unsigned t = std::thread::hardware_concurrency();
  return t == 0 ? 1 : (int)std::min(t, 64u);
}

template <class F>
static void parallel_for(int64_t n, int threads, F f) {
  if (threads <= 1 || n < 4096) {
    f(0, n, 0);
    return;
  }
  std::vector<std::thread> ts;
  int64_t chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    int64_t b = t * chunk, e = std::min<int64_t>(n, b + chunk);
    if (b >= e) break;
    ts.emplace_back([=] { f(b, e, t); });
  }
  for (auto& th : ts) th.join();
}

// LSD radix sort of 64-bit keys on the low `bits` bits, 16 bits per pass.
static void radix_sort_u64(std::vector<uint64_t>& a, int bits) {
  std::vector<uint64_t> tmp(a.size());
  const int threads = hw_threads();
  for (int shift = 0; shift < bits; shift += 16) {
    const int64_t n = (int64_t)a.size();
    const int T = (n < (1 << 20)) ? 1 : threads;
    std::vector<std::vector<uint64_t>> hist(T, std::vector<uint64_t>(65536, 0));
    int64_t chunk = (n + T - 1) / T;
    auto count = [&](int t) {
      int64_t b = t * chunk, e = std::min<int64_t>(n, b + chunk);
      auto& h = hist[t];
      for (int64_t i = b; i < e; ++i) h[(a[i] >> shift) & 0xffff]++;
    };
    {
      std::vector<std::thread> ts;
      for (int t = 0; t < T; ++t) ts.emplace_back(count, t);
      for (auto& th : ts) th.join();
    }
    uint64_t run = 0;
    for (int d = 0; d < 65536; ++d)
      for (int t = 0; t < T; ++t) {
        uint64_t c = hist[t][d];
        hist[t][d] = run;
        run += c;
      }
    auto scatter = [&](int t) {
      int64_t b = t * chunk, e = std::min<int64_t>(n, b + chunk);
      auto& h = hist[t];
      for (int64_t i = b; i < e; ++i) tmp[h[(a[i] >> shift) & 0xffff]++] = a[i];
    };
    {
      std::vector<std::thread> ts;
      for (int t = 0; t < T; ++t) ts.emplace_back(scatter, t);
      for (auto& th : ts) th.join();
    }
    a.swap(tmp);
  }
}

static void sort_unique(std::vector<uint64_t>& keys, int bits) {
  radix_sort_u64(keys, bits);
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
}

// Keep exactly m of the (sorted, unique) keys: the m with the smallest
// seeded hash. The kept keys stay sorted.
static void select_m(std::vector<uint64_t>& keys, uint64_t m, uint64_t seed) {
  if (keys.size() <= m) return;
  std::vector<uint64_t> h(keys.size());
  parallel_for((int64_t)keys.size(), hw_threads(), [&](int64_t b, int64_t e, int) {
    for (int64_t i = b; i < e; ++i) h[i] = mix64(seed ^ 0x5e1ec7ULL, keys[i]);
  });
  std::vector<uint64_t> hc(h);
  std::nth_element(hc.begin(), hc.begin() + (m - 1), hc.end());
  const uint64_t thr = hc[m - 1];
  uint64_t below = 0;
  for (uint64_t x : h) below += (x < thr);
  uint64_t ties_left = m - below;  // keys hashing exactly to thr that are kept
  std::vector<uint64_t> out;
  out.reserve(m);
  for (size_t i = 0; i < keys.size(); ++i) {
    if (h[i] < thr) {
      out.push_back(keys[i]);
    } else if (h[i] == thr && ties_left > 0) {
      out.push_back(keys[i]);
      --ties_left;
    }
  }
  keys.swap(out);
}

static void keys_to_edges(const std::vector<uint64_t>& keys, int vbits, uint32_t* edges) {
  const uint64_t mask = (vbits >= 32) ? 0xffffffffULL : ((1ULL << vbits) - 1);
  parallel_for((int64_t)keys.size(), hw_threads(), [&](int64_t b, int64_t e, int) {
    for (int64_t i = b; i < e; ++i) {
      edges[2 * i] = (uint32_t)(keys[i] >> vbits);
      edges[2 * i + 1] = (uint32_t)(keys[i] & mask);
    }
  });
}

static int bits_for(uint64_t n) {
  int b = 1;
  while ((1ULL << b) < n) ++b;
  return b;
}

}  // namespace gpsm

using namespace gpsm;

extern "C" int gpsm_gen_er(uint32_t n, uint64_t m, uint64_t seed, uint32_t* edges) {
  if (n < 2 || edges == nullptr) return GPSM_ERR_INVALID;
  if (m > (uint64_t)n * (n - 1) / 2) return GPSM_ERR_INVALID;
  const int vb = bits_for(n);
  std::vector<uint64_t> keys;
  keys.reserve(m + m / 8 + 16);
  uint64_t round = 0;
  while (keys.size() < m) {
    Rng r(seed, 0xe5000000ULL + round++);
    uint64_t need = (m - keys.size()) + (m - keys.size()) / 8 + 16;
    for (uint64_t i = 0; i < need; ++i) {
      uint32_t a = (uint32_t)r.below(n), b = (uint32_t)r.below(n);
      if (a == b) continue;
      if (a > b) std::swap(a, b);
      keys.push_back(((uint64_t)a << vb) | b);
    }
    sort_unique(keys, 2 * vb);
  }
  select_m(keys, m, seed);
  keys_to_edges(keys, vb, edges);
  return GPSM_OK;
}

// R-MAT (Chakrabarti, Zhan, Faloutsos 2004): each edge descends `scale`
// levels of the adjacency matrix choosing quadrant a/b/c/d. Self loops are
// dropped, pairs are made undirected (min, max) and deduplicated; sampling
// continues until m unique edges exist and exactly m are kept. Vertex ids are
// then randomly permuted (as Graph500 does) so hubs are not clustered at 0.
extern "C" int gpsm_gen_rmat(int scale, uint64_t m, double a, double b, double c, uint64_t seed,
                             uint32_t* edges) {
  if (scale < 2 || scale > 30 || edges == nullptr) return GPSM_ERR_INVALID;
  const uint64_t n = 1ULL << scale;
  if (m > n * (n - 1) / 2) return GPSM_ERR_INVALID;
  const uint32_t ta = (uint32_t)std::lround(a * 65536.0);
  const uint32_t tb = (uint32_t)std::lround((a + b) * 65536.0);
  const uint32_t tc = (uint32_t)std::lround((a + b + c) * 65536.0);
  const int threads = hw_threads();
  std::vector<uint64_t> keys;
  uint64_t round = 0;
  while (keys.size() < m) {
    uint64_t missing = m - keys.size();
    uint64_t need = missing + missing / 4 + 1024;
    size_t base = keys.size();
    keys.resize(base + need);
    const int64_t chunks = 256;
    std::atomic<int64_t> next_chunk(0);
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; ++t)
      ts.emplace_back([&, t] {
        (void)t;
        for (;;) {
          int64_t ch = next_chunk.fetch_add(1);
          if (ch >= chunks) break;
          uint64_t lo = need * ch / chunks, hi = need * (ch + 1) / chunks;
          Rng r(seed, (round << 20) + 0xa7000 + ch);
          for (uint64_t i = lo; i < hi; ++i) {
            uint64_t u = 0, v = 0;
            uint64_t bitsrc = 0;
            int avail = 0;
            for (int lev = 0; lev < scale; ++lev) {
              if (avail == 0) {
                bitsrc = r.next();
                avail = 4;
              }
              uint32_t x = (uint32_t)(bitsrc & 0xffff);
              bitsrc >>= 16;
              --avail;
              u <<= 1;
              v <<= 1;
              if (x < ta) {
              } else if (x < tb) {
                v |= 1;
              } else if (x < tc) {
                u |= 1;
              } else {
                u |= 1;
                v |= 1;
              }
            }
            if (u == v) {
              keys[base + i] = ~0ULL;  // removed below
              continue;
            }
            if (u > v) std::swap(u, v);
            keys[base + i] = (u << scale) | v;
          }
        }
      });
    for (auto& th : ts) th.join();
    sort_unique(keys, 2 * scale + 1);
    while (!keys.empty() && keys.back() == ~0ULL) keys.pop_back();
    // ~0ULL sorts last only when all bits participate; the radix pass above
    // covers 2*scale+1 bits so the marker (all ones) still sorts last.
    ++round;
  }
  select_m(keys, m, seed);
  // permute vertex ids
  std::vector<uint32_t> perm(n);
  for (uint64_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
  Rng pr(seed, 0x9e7a);
  for (uint64_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[pr.below(i + 1)]);
  parallel_for((int64_t)keys.size(), threads, [&](int64_t lo, int64_t hi, int) {
    const uint64_t mask = (1ULL << scale) - 1;
    for (int64_t i = lo; i < hi; ++i) {
      uint32_t u = perm[keys[i] >> scale], v = perm[keys[i] & mask];
      if (u > v) std::swap(u, v);
      edges[2 * i] = u;
      edges[2 * i + 1] = v;
    }
  });
  return GPSM_OK;
}

extern "C" int gpsm_gen_labels(uint32_t n, uint32_t num_labels, double zipf_s, uint64_t seed,
                               uint32_t* labels) {
  if (num_labels == 0 || labels == nullptr) return GPSM_ERR_INVALID;
  std::vector<double> cdf(num_labels);
  double acc = 0;
  for (uint32_t k = 0; k < num_labels; ++k) {
    acc += (zipf_s == 0.0) ? 1.0 : std::pow((double)(k + 1), -zipf_s);
    cdf[k] = acc;
  }
  for (auto& x : cdf) x /= acc;
  cdf[num_labels - 1] = 1.0;
  const int64_t chunk = 1 << 16;
  const int64_t nch = ((int64_t)n + chunk - 1) / chunk;
  parallel_for(nch, hw_threads(), [&](int64_t b, int64_t e, int) {
    for (int64_t ch = b; ch < e; ++ch) {
      Rng r(seed, 0x1abe1000ULL + ch);
      int64_t lo = ch * chunk, hi = std::min<int64_t>((int64_t)n, lo + chunk);
      for (int64_t i = lo; i < hi; ++i) {
        double x = r.uniform();
        uint32_t k = (uint32_t)(std::upper_bound(cdf.begin(), cdf.end(), x) - cdf.begin());
        if (k >= num_labels) k = num_labels - 1;
        labels[i] = k + 1;  // labels are 1-based (README.md "labels start from 1")
      }
    }
  });
  return GPSM_OK;
}

// Undirected CSR with every adjacency list sorted ascending (graph/Graph.cpp:30-65).
// edges: m pairs (u, v), each undirected edge once. Parallel edges and self
// loops are kept exactly as given, like the reference.
extern "C" int gpsm_csr_from_edges(uint32_t n, uint64_t m, const uint32_t* edges, uint32_t* offsets,
                                   uint32_t* cols) {
  if (offsets == nullptr || (m > 0 && (edges == nullptr || cols == nullptr))) return GPSM_ERR_INVALID;
  if (2 * m > 0xffffffffULL) return GPSM_ERR_INVALID;
  std::vector<uint32_t> deg(n + 1, 0);
  for (uint64_t i = 0; i < m; ++i) {
    uint32_t u = edges[2 * i], v = edges[2 * i + 1];
    if (u >= n || v >= n) return GPSM_ERR_INVALID;
    deg[u]++;
    deg[v]++;
  }
  offsets[0] = 0;
  for (uint32_t i = 0; i < n; ++i) offsets[i + 1] = offsets[i] + deg[i];
  std::vector<uint32_t> pos(offsets, offsets + n);
  for (uint64_t i = 0; i < m; ++i) {
    uint32_t u = edges[2 * i], v = edges[2 * i + 1];
    cols[pos[u]++] = v;
    cols[pos[v]++] = u;
  }
  parallel_for((int64_t)n, hw_threads(), [&](int64_t b, int64_t e, int) {
    for (int64_t i = b; i < e; ++i) {
      uint32_t* p = cols + offsets[i];
      uint32_t* q = cols + offsets[i + 1];
      if (!std::is_sorted(p, q)) std::sort(p, q);
    }
  });
  return GPSM_OK;
}

static inline bool adjacent(const uint32_t* off, const uint32_t* cols, uint32_t a, uint32_t b) {
  const uint32_t *p = cols + off[a], *q = cols + off[a + 1];
  return std::binary_search(p, q, b);
}

// Random-walk query extraction. A walk from a random non-isolated vertex runs
// until it has visited qn distinct vertices (restarting when stuck); query
// vertex i is the i-th newly visited data vertex, so the identity walk is one
// embedding and every query has at least one match.
//   mode 0 (induced): every data edge among the visited vertices;
//   mode 1 (tree):    only the walk's discovery edges (qn-1 edges);
//   mode 2 (dense):   discovery edges plus each other induced edge kept with
//                     probability p_extra.
// Queries whose average degree 2m/qn is below min_avg_degree are redrawn.
// q_edges must hold qn*(qn-1)/2 pairs; edges are written sorted by
// (min, max) as (min, max). Returns the number of query edges, or <0.
extern "C" int64_t gpsm_gen_query(uint32_t n, const uint32_t* offsets, const uint32_t* cols,
                                  const uint32_t* labels, uint32_t qn, int mode, double p_extra,
                                  double min_avg_degree, uint64_t seed, uint32_t* q_labels,
                                  uint32_t* q_edges, uint32_t* q_data_ids) {
  if (qn < 1 || qn > 4096 || n == 0 || q_labels == nullptr || q_edges == nullptr) return GPSM_ERR_INVALID;
  Rng r(seed, 0x9e11e5ULL);
  std::vector<uint32_t> visited;
  std::vector<std::pair<uint32_t, uint32_t>> tree;  // (parent idx, child idx)
  for (int attempt = 0; attempt < 100000; ++attempt) {
    uint32_t start = (uint32_t)r.below(n);
    if (offsets[start + 1] == offsets[start] && qn > 1) continue;
    visited.assign(1, start);
    tree.clear();
    uint32_t cur = 0;  // index into visited
    uint64_t steps = 0;
    while (visited.size() < qn && steps < 200ULL * qn) {
      uint32_t cv = visited[cur];
      uint32_t d = offsets[cv + 1] - offsets[cv];
      if (d == 0) break;
      uint32_t nxt = cols[offsets[cv] + (uint32_t)r.below(d)];
      ++steps;
      auto it = std::find(visited.begin(), visited.end(), nxt);
      if (it == visited.end()) {
        tree.emplace_back(cur, (uint32_t)visited.size());
        visited.push_back(nxt);
        cur = (uint32_t)visited.size() - 1;
      } else {
        cur = (uint32_t)(it - visited.begin());
      }
    }
    if (visited.size() < qn) continue;
    std::vector<uint64_t> ek;
    auto key = [&](uint32_t x, uint32_t y) {
      if (x > y) std::swap(x, y);
      return ((uint64_t)x << 32) | y;
    };
    std::vector<uint64_t> tk;
    for (auto& e : tree) tk.push_back(key(e.first, e.second));
    std::sort(tk.begin(), tk.end());
    for (uint32_t i = 0; i < qn; ++i)
      for (uint32_t j = i + 1; j < qn; ++j) {
        if (!adjacent(offsets, cols, visited[i], visited[j])) continue;
        uint64_t k = key(i, j);
        bool is_tree = std::binary_search(tk.begin(), tk.end(), k);
        if (mode == 0 || is_tree) {
          ek.push_back(k);
        } else if (mode == 2) {
          if (r.uniform() < p_extra) ek.push_back(k);
        }
      }
    if (qn > 1 && 2.0 * (double)ek.size() / (double)qn < min_avg_degree) continue;
    std::sort(ek.begin(), ek.end());
    for (uint32_t i = 0; i < qn; ++i) {
      q_labels[i] = labels[visited[i]];
      if (q_data_ids) q_data_ids[i] = visited[i];
    }
    for (size_t i = 0; i < ek.size(); ++i) {
      q_edges[2 * i] = (uint32_t)(ek[i] >> 32);
      q_edges[2 * i + 1] = (uint32_t)(ek[i] & 0xffffffffULL);
    }
    return (int64_t)ek.size();
  }
  return GPSM_ERR_NOT_FOUND;
}
