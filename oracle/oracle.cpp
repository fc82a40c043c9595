// ORACLE - test infrastructure only. Nothing in the product links this file;
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// the shared library built from it.
//
// Two independent checkers of the subgraph-matching path:
//
// 1. oracle_enumerate: a backtracking matcher written from the definition of
//    a non-induced, injective, undirected, edge-unlabelled embedding (labels
//    equal, every query edge maps to a data edge, distinct query vertices map
//    to distinct data vertices). It shares no code or order with the engine.
//
// 2. oracle_ref_*: a CPU restatement of the reference GpSM pipeline, step for
//    step, so that intermediate products can be compared bit for bit:
//      edge list ............ match/Match.cu:1738-1754
//      root + BFS order ..... match/Match.cu:339-429  (generateSpanningTree)
//      candidate init ....... match/Match.cu:431-461, 528-719 (check/explore)
//      simplified graph ..... match/Match.cu:721-759
//      refinement ........... match/Match.cu:761-890  (4 rounds + 1 check)
//      candidate edges ...... match/Match.cu:892-1139 (count/examine)
//      join order + joins ... match/Match.cu:1141-1708 (table/join/expand/link)
//      host verify .......... io/IO.cpp:146-180        (IO::verify)
//    The reference's expand step may pick an edge with neither endpoint
//    visited (match/Match.cu:1639-1650, then vpos = -1 at :1680); the
//    restatement reports that as a defect instead of reading out of bounds.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <climits>
#include <cstring>
#include <queue>
#include <thread>
#include <vector>

namespace {

struct DataGraph {
  uint32_t n;
  const uint32_t* off;
  const uint32_t* col;
  const uint32_t* lab;
  inline uint32_t deg(uint32_t x) const { return off[x + 1] - off[x]; }
  inline bool adj(uint32_t a, uint32_t b) const {
    return std::binary_search(col + off[a], col + off[a + 1], b);
  }
};

// Every adjacency list again, ordered by (neighbour label, id), with a
// directory of label runs per vertex: lets the ordered search scan only the
// neighbours that carry the next query vertex's label. Built here on host
// threads, apart from the engine's own (device-built) label runs.
struct LabelIndex {
  uint32_t n = 0;
  const uint32_t* off = nullptr;  // the graph's CSR offsets (lcol uses the same segments)
  std::vector<uint32_t> lcol;
  std::vector<uint64_t> run_off;  // [n+1] runs of vertex x: run_off[x] .. run_off[x+1]-1
  std::vector<uint32_t> run_lab, run_beg;  // label and first lcol index of each run
  // [b, e) of lcol: x's neighbours with label l (empty when none)
  void run_of(uint32_t x, uint32_t l, uint32_t* b, uint32_t* e) const {
    const uint32_t* lo = run_lab.data() + run_off[x];
    const uint32_t* hi = run_lab.data() + run_off[x + 1];
    const uint32_t* it = std::lower_bound(lo, hi, l);
    if (it == hi || *it != l) {
      *b = *e = 0;
      return;
    }
    const uint64_t k = (uint64_t)(it - run_lab.data());
    *b = run_beg[k];
    *e = k + 1 < run_off[x + 1] ? run_beg[k + 1] : off[x + 1];
  }
};

static void build_label_index(LabelIndex& L, uint32_t n, const uint32_t* off, const uint32_t* col,
                              const uint32_t* lab, int threads) {
  L.n = n;
  L.off = off;
  L.lcol.assign(col, col + off[n]);
  std::vector<uint64_t> runs(n, 0);
  auto sort_part = [&](uint32_t a, uint32_t b) {
    for (uint32_t x = a; x < b; ++x) {
      uint32_t* p = L.lcol.data() + off[x];
      uint32_t* q = L.lcol.data() + off[x + 1];
      std::stable_sort(p, q, [&](uint32_t u, uint32_t v) { return lab[u] < lab[v]; });  // ids stay ascending
      uint64_t r = 0;
      for (uint32_t* t = p; t < q; ++t) r += (t == p || lab[*t] != lab[t[-1]]);
      runs[x] = r;
    }
  };
  if (threads < 1) threads = 1;
  std::vector<std::thread> ts;
  const uint32_t chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    const uint32_t a = std::min<uint64_t>((uint64_t)t * chunk, n), b = std::min<uint64_t>((uint64_t)a + chunk, n);
    if (a < b) ts.emplace_back(sort_part, a, b);
  }
  for (auto& th : ts) th.join();
  L.run_off.assign(n + 1, 0);
  for (uint32_t x = 0; x < n; ++x) L.run_off[x + 1] = L.run_off[x] + runs[x];
  L.run_lab.resize(L.run_off[n]);
  L.run_beg.resize(L.run_off[n]);
  for (uint32_t x = 0; x < n; ++x) {
    uint64_t k = L.run_off[x];
    for (uint32_t i = off[x]; i < off[x + 1]; ++i)
      if (i == off[x] || lab[L.lcol[i]] != lab[L.lcol[i - 1]]) {
        L.run_lab[k] = lab[L.lcol[i]];
        L.run_beg[k] = i;
        ++k;
      }
  }
}

// ---------------------------------------------------------------------------
// 1. independent backtracking oracle
// ---------------------------------------------------------------------------
struct Enumerator {
  const DataGraph& g;
  uint32_t qn;
  std::vector<uint32_t> qlab, qdeg;
  std::vector<std::vector<uint32_t>> qadj;  // undirected, deduplicated
  std::vector<uint32_t> order;               // matching order
  std::vector<std::vector<uint32_t>> back;   // earlier-ordered neighbours per position
  std::vector<uint32_t> f;                   // current partial map (by query vertex)
  std::vector<uint8_t> used;                 // data vertices in use
  uint64_t count = 0, cap;
  uint32_t* out;
  uint64_t out_cap;

  Enumerator(const DataGraph& g_, uint32_t qn_, const uint32_t* ql, uint32_t qm, const uint32_t* qe,
             uint64_t cap_, uint32_t* out_, uint64_t out_cap_)
      : g(g_), qn(qn_), qlab(ql, ql + qn_), qdeg(qn_, 0), qadj(qn_), cap(cap_), out(out_),
        out_cap(out_cap_) {
    for (uint32_t i = 0; i < qm; ++i) {
      uint32_t a = qe[2 * i], b = qe[2 * i + 1];
      if (a == b) continue;
      qadj[a].push_back(b);
      qadj[b].push_back(a);
    }
    for (uint32_t u = 0; u < qn; ++u) {
      std::sort(qadj[u].begin(), qadj[u].end());
      qadj[u].erase(std::unique(qadj[u].begin(), qadj[u].end()), qadj[u].end());
      qdeg[u] = (uint32_t)qadj[u].size();
    }
  }

  uint64_t label_count(uint32_t u) const {
    uint64_t c = 0;
    for (uint32_t x = 0; x < g.n; ++x) c += (g.lab[x] == qlab[u] && g.deg(x) >= qdeg[u]);
    return c;
  }

  // A given matching order (a connected permutation): rows then come out in
  // lexicographic order of their values taken in that order, the order in
  // which the engine emits a join in that vertex order.
  std::vector<uint32_t> given;
  uint64_t work = 0, work_cap = ~0ULL;  // nodes and candidates visited; optional bound
  bool out_by_pos = false;              // write rows in order position, not by query vertex
  uint64_t digest = 0;                  // rows_digest of the rows found, in order (by position)
  const LabelIndex* lidx = nullptr;     // optional: scan label runs instead of whole lists
  // with lidx: arc-consistent candidate sets, one bitset per query vertex
  std::vector<std::vector<uint64_t>> cand;

  bool in_cand(uint32_t u, uint32_t y) const { return (cand[u][y >> 6] >> (y & 63)) & 1u; }

  // Candidate sets by arc consistency, written from the definition of an
  // embedding: x stays a candidate of u only while, for every query
  // neighbour w of u, x has a neighbour that is a candidate of w. An
  // embedding maps every vertex to a vertex that passes this test forever,
  // so no embedding is lost; rounds repeat until nothing changes.
  void filter_candidates() {
    const size_t words = (g.n + 63) / 64;
    cand.assign(qn, std::vector<uint64_t>(words, 0));
    for (uint32_t u = 0; u < qn; ++u)
      for (uint32_t x = 0; x < g.n; ++x)
        if (g.lab[x] == qlab[u] && g.deg(x) >= qdeg[u]) cand[u][x >> 6] |= 1ull << (x & 63);
    const uint32_t* L = lidx->lcol.data();
    for (bool changed = true; changed;) {
      changed = false;
      for (uint32_t u = 0; u < qn; ++u)
        for (size_t wd = 0; wd < words; ++wd)
          for (uint64_t bits = cand[u][wd]; bits; bits &= bits - 1) {
            const uint32_t x = (uint32_t)(wd * 64 + __builtin_ctzll(bits));
            for (uint32_t w : qadj[u]) {
              uint32_t b, e;
              lidx->run_of(x, qlab[w], &b, &e);
              bool any = false;
              for (uint32_t i = b; i < e && !any; ++i) any = in_cand(w, L[i]);
              if (!any) {
                cand[u][wd] &= ~(1ull << (x & 63));
                changed = true;
                break;
              }
            }
          }
    }
  }

  void make_order() {
    if (!given.empty()) {
      order = given;
      set_back();
      return;
    }
    std::vector<uint64_t> cnt(qn);
    for (uint32_t u = 0; u < qn; ++u) cnt[u] = label_count(u);
    std::vector<uint8_t> in(qn, 0);
    std::vector<uint32_t> conn(qn, 0);
    for (uint32_t k = 0; k < qn; ++k) {
      int best = -1;
      for (uint32_t u = 0; u < qn; ++u) {
        if (in[u]) continue;
        if (best < 0) {
          best = (int)u;
          continue;
        }
        uint32_t b = (uint32_t)best;
        if (conn[u] != conn[b] ? conn[u] > conn[b] : (cnt[u] != cnt[b] ? cnt[u] < cnt[b] : u < b))
          best = (int)u;
      }
      uint32_t u = (uint32_t)best;
      in[u] = 1;
      order.push_back(u);
      for (uint32_t w : qadj[u]) conn[w]++;
    }
    set_back();
  }

  void set_back() {
    back.assign(qn, {});
    std::vector<uint8_t> placed(qn, 0);
    for (uint32_t i = 0; i < qn; ++i) {
      uint32_t u = order[i];
      for (uint32_t w : qadj[u])
        if (placed[w]) back[i].push_back(w);
      placed[u] = 1;
    }
  }

  bool fits(uint32_t pos, uint32_t y) const {
    uint32_t u = order[pos];
    if (g.lab[y] != qlab[u] || g.deg(y) < qdeg[u] || used[y]) return false;
    for (uint32_t w : back[pos])
      if (!g.adj(f[w], y)) return false;
    return true;
  }

  void emit() {
    if (out != nullptr && count < out_cap) {
      uint32_t* r = out + count * qn;
      for (uint32_t u = 0; u < qn; ++u) r[u] = out_by_pos ? f[order[u]] : f[u];
    }
    if (out_by_pos) digest += row_hash(f, order) * (count + 1);
    ++count;
  }

  // Hash of one row, values taken in position order: a splitmix64-style
  // fold of (value | position << 32); oracle.rows_digest restates it in numpy.
  static uint64_t fold(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
  }
  static uint64_t row_hash(const std::vector<uint32_t>& f, const std::vector<uint32_t>& order) {
    uint64_t h = 0x243f6a8885a308d3ULL;
    for (uint32_t p = 0; p < order.size(); ++p) h = fold(h ^ ((uint64_t)f[order[p]] | ((uint64_t)p << 32)));
    return h;
  }

  void dfs(uint32_t pos) {
    if (count >= cap) return;
    if (++work > work_cap) {
      cap = count;  // stop everywhere; the caller sees the bound was hit
      return;
    }
    if (pos == qn) {
      emit();
      return;
    }
    uint32_t u = order[pos];
    if (back[pos].empty()) {
      for (uint32_t y = 0; y < g.n && count < cap; ++y) {
        if (++work > work_cap) {  // every candidate examined counts
          cap = count;
          return;
        }
        if (lidx ? !in_cand(u, y) : !fits(pos, y)) continue;
        f[u] = y;
        used[y] = 1;
        dfs(pos + 1);
        used[y] = 0;
      }
      return;
    }
    if (lidx) {
      dfs_runs(pos, u);
      return;
    }
    // scan the smallest adjacency among mapped neighbours
    uint32_t p = back[pos][0];
    for (uint32_t w : back[pos])
      if (g.deg(f[w]) < g.deg(f[p])) p = w;
    const uint32_t* a = g.col + g.off[f[p]];
    const uint32_t* e = g.col + g.off[f[p] + 1];
    uint32_t prev = 0xffffffffu;
    for (; a < e && count < cap; ++a) {
      if (++work > work_cap) {
        cap = count;
        return;
      }
      uint32_t y = *a;
      if (y == prev) continue;  // parallel data edges give one embedding
      prev = y;
      if (!fits(pos, y)) continue;
      f[u] = y;
      used[y] = 1;
      dfs(pos + 1);
      used[y] = 0;
    }
  }

  // dfs step with the label index: the shortest label run among the placed
  // neighbours drives (ascending ids), the others are binary-searched.
  void dfs_runs(uint32_t pos, uint32_t u) {
    const auto& bk = back[pos];
    const size_t nb = bk.size();
    uint32_t rb[128], re[128];  // query vertices < 128
    size_t d = 0;
    for (size_t k = 0; k < nb; ++k) {
      lidx->run_of(f[bk[k]], qlab[u], &rb[k], &re[k]);
      if (re[k] - rb[k] < re[d] - rb[d]) d = k;
    }
    const uint32_t* L = lidx->lcol.data();
    uint32_t prev = 0xffffffffu;
    for (uint32_t i = rb[d]; i < re[d] && count < cap; ++i) {
      if (++work > work_cap) {
        cap = count;
        return;
      }
      const uint32_t y = L[i];
      if (y == prev) continue;  // parallel data edges give one embedding
      prev = y;
      if (!in_cand(u, y) || used[y]) continue;
      bool ok = true;
      for (size_t k = 0; ok && k < nb; ++k)
        if (k != d) ok = std::binary_search(L + rb[k], L + re[k], y);
      if (!ok) continue;
      f[u] = y;
      used[y] = 1;
      dfs(pos + 1);
      used[y] = 0;
    }
  }

  void run() {
    if (qn == 0) return;
    make_order();
    if (lidx) filter_candidates();
    f.assign(qn, 0);
    used.assign(g.n, 0);
    dfs(0);
  }
};

static bool row_less(const uint32_t* a, const uint32_t* b, uint32_t w) {
  for (uint32_t i = 0; i < w; ++i)
    if (a[i] != b[i]) return a[i] < b[i];
  return false;
}

static void sort_rows(uint32_t* rows, uint64_t nrows, uint32_t w) {
  if (nrows < 2 || w == 0) return;
  std::vector<uint64_t> idx(nrows);
  for (uint64_t i = 0; i < nrows; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(),
            [&](uint64_t x, uint64_t y) { return row_less(rows + x * w, rows + y * w, w); });
  std::vector<uint32_t> tmp(rows, rows + nrows * w);
  for (uint64_t i = 0; i < nrows; ++i) memcpy(rows + i * w, tmp.data() + idx[i] * w, 4 * w);
}

// ---------------------------------------------------------------------------
// 2. restatement of the reference pipeline
// ---------------------------------------------------------------------------
struct RefQuery {
  uint32_t n = 0;
  std::vector<uint32_t> lab;
  std::vector<std::vector<uint32_t>> in, out;  // file-order directed lists (Graph::addEdge)
  std::vector<uint32_t> roff, rcol;             // undirected CSR, sorted lists
  std::vector<uint32_t> qm_from, qm_to;         // file edges (for verify)
  void build(uint32_t qn, const uint32_t* ql, uint32_t qm, const uint32_t* qe) {
    n = qn;
    lab.assign(ql, ql + qn);
    in.assign(qn, {});
    out.assign(qn, {});
    for (uint32_t i = 0; i < qm; ++i) {
      uint32_t a = qe[2 * i], b = qe[2 * i + 1];
      out[a].push_back(b);  // graph/Graph.cpp:20-24
      in[b].push_back(a);
      qm_from.push_back(a);
      qm_to.push_back(b);
    }
    roff.assign(qn + 1, 0);
    for (uint32_t i = 0; i < qn; ++i) roff[i + 1] = roff[i] + (uint32_t)(in[i].size() + out[i].size());
    rcol.resize(roff[qn]);
    for (uint32_t i = 0; i < qn; ++i) {
      uint32_t p = roff[i];
      for (uint32_t x : in[i]) rcol[p++] = x;
      for (uint32_t x : out[i]) rcol[p++] = x;
      std::sort(rcol.begin() + roff[i], rcol.begin() + roff[i + 1]);
    }
  }
  uint32_t deg(uint32_t u) const { return roff[u + 1] - roff[u]; }
};

enum RefStatus : int32_t {
  REF_OK = 0,
  REF_EMPTY_INIT = 1,      // Match.cu:1768-1779
  REF_EMPTY_REFINE = 2,    // Match.cu:1806-1814
  REF_EMPTY_JOIN = 3,      // JoinCandidateEdges returned false (Match.cu:1696-1699)
  REF_DISCONNECTED = 4,    // filter order does not reach every vertex (undefined in the reference)
  REF_NO_EDGES = 5,        // edge_num == 0: Match.cu:383 reads edge_from[-1]
  REF_EMPTY_CEDGE = 6,     // a C(u) collected empty in FindCandidateEdges: zero-size grid, exit(1)
};

struct RefPlan {
  RefQuery q;
  uint32_t m = 0;
  std::vector<uint32_t> efrom, eto;  // edge ids, Match.cu:1738-1754
  std::vector<uint32_t> order;       // filter order (BFS)
  std::vector<uint8_t> cand_init, cand;  // qn x N
  int32_t status = REF_OK;
  // candidate edges: per edge id and direction, [C(u) ids][offsets n+1][nbrs]
  std::vector<std::vector<uint32_t>> cedge_fwd, cedge_rev;
  std::vector<uint64_t> size_fwd, size_rev;
  std::vector<uint32_t> num_fwd, num_rev;
  // plain order
  struct Step {
    uint32_t edge;
    int32_t mode;    // 0 seed, 1 join (check), 2 expand fwd (u visited), 3 expand rev (v visited)
    int32_t defect;  // 1 when the reference's pick had neither endpoint visited
  };
  std::vector<Step> steps;
  std::vector<int32_t> pos2id, id2pos;
  int32_t defect = 0;
  // a vertex keeps its table column once added, so the final map serves every step
  int32_t id2pos_at(uint32_t id) const { return id2pos[id]; }
};

static void ref_edges(RefPlan& P) {
  // Match.cu:1738-1754: for each vertex i, its in-neighbours in file order
  for (uint32_t i = 0; i < P.q.n; ++i)
    for (uint32_t a : P.q.in[i]) {
      P.efrom.push_back(std::min(a, i));
      P.eto.push_back(std::max(a, i));
    }
  P.m = (uint32_t)P.efrom.size();
}

static void ref_spanning_order(const DataGraph& g, RefPlan& P) {
  const RefQuery& q = P.q;
  // label frequencies of the data graph (Graph::inverse_num, graph/Graph.cpp:66-102)
  std::vector<float> score(q.n);
  for (uint32_t i = 0; i < q.n; ++i) {
    float num = 0.0f;
    uint64_t c = 0;
    for (uint32_t x = 0; x < g.n; ++x) c += (g.lab[x] == q.lab[i]);
    num = (float)c;
    int degree = (int)(q.in[i].size() + q.out[i].size());
    score[i] = (float)(((double)degree + 0.0) / (double)num);  // Match.cu:360
  }
  float maxv = 0.0f;
  int maxi = -1;
  for (uint32_t i = 0; i < P.m; ++i) {
    float tmp = score[P.efrom[i]] + score[P.eto[i]];
    if (tmp > maxv) {
      maxv = tmp;
      maxi = (int)i;
    }
  }
  if (maxi < 0) maxi = 0;  // all scores 0 cannot happen for connected queries with present labels
  uint32_t from = P.efrom[maxi], to = P.eto[maxi];
  uint32_t start = from;
  if (score[to] > score[from]) start = to;
  std::vector<uint8_t> visit(q.n, 0);
  P.order.clear();
  P.order.push_back(start);
  visit[start] = 1;
  std::queue<uint32_t> tq;
  tq.push(start);
  while (!tq.empty()) {
    uint32_t t = tq.front();
    tq.pop();
    for (uint32_t i = q.roff[t]; i < q.roff[t + 1]; ++i) {
      uint32_t a = q.rcol[i];
      if (visit[a]) continue;
      tq.push(a);
      P.order.push_back(a);
      visit[a] = 1;
    }
  }
}

static bool ref_collect(const std::vector<uint8_t>& C, uint32_t N, uint32_t u, std::vector<uint32_t>& arr) {
  arr.clear();
  const uint8_t* row = C.data() + (size_t)u * N;
  for (uint32_t x = 0; x < N; ++x)
    if (row[x]) arr.push_back(x);
  return !arr.empty();
}

static void ref_filter(const DataGraph& g, RefPlan& P) {
  const RefQuery& q = P.q;
  const uint32_t N = g.n;
  std::vector<uint8_t>& C = P.cand;
  C.assign((size_t)q.n * N, 0);
  std::vector<uint8_t> initialized(q.n, 0);
  std::vector<uint32_t> arr;
  for (uint32_t i = 0; i < q.n; ++i) {
    uint32_t u = P.order[i];
    if (!initialized[u]) {  // check_kernel, Match.cu:431-446
      for (uint32_t x = 0; x < N; ++x)
        if (g.lab[x] == q.lab[u] && g.deg(x) >= q.deg(u)) C[(size_t)u * N + x] = 1;
      initialized[u] = 1;
    }
    if (!ref_collect(C, N, u, arr)) {
      P.status = REF_EMPTY_INIT;
      return;
    }
    // explore_kernel, Match.cu:528-601 (targets built at :603-641)
    std::vector<uint32_t> tv;
    for (uint32_t k = q.roff[u]; k < q.roff[u + 1]; ++k)
      if (!initialized[q.rcol[k]]) tv.push_back(q.rcol[k]);
    if (!tv.empty()) {
      for (uint32_t mu : arr) {
        for (uint32_t v : tv) {
          bool any = false;
          const uint32_t lv = q.lab[v], dv = q.deg(v);
          for (uint32_t e = g.off[mu]; e < g.off[mu + 1]; ++e) {
            uint32_t mv = g.col[e];
            if (g.lab[mv] == lv && g.deg(mv) >= dv) {
              C[(size_t)v * N + mv] = 1;
              any = true;
            }
          }
          if (!any) {
            C[(size_t)u * N + mu] = 0;
            break;
          }
        }
      }
    }
    for (uint32_t k = q.roff[u]; k < q.roff[u + 1]; ++k) initialized[q.rcol[k]] = 1;
  }
  P.cand_init = C;
  // generateSimplifiedGraph, Match.cu:721-759 (degree threshold 1, :852)
  std::vector<uint32_t> sv;
  std::vector<uint8_t> valid(q.n, 0);
  for (uint32_t i = 0; i < q.n; ++i)
    if (q.deg(i) > 1) {
      valid[i] = 1;
      sv.push_back(i);
    }
  std::vector<std::vector<uint32_t>> se(sv.size());
  for (size_t i = 0; i < sv.size(); ++i) {
    for (uint32_t x : q.in[sv[i]])
      if (valid[x]) se[i].push_back(x);
    for (uint32_t x : q.out[sv[i]])
      if (valid[x]) se[i].push_back(x);
  }
  // RefineCandidateVertices, Match.cu:848-890: 5 rounds, last is a check
  for (int k = 0; k < 5; ++k) {
    for (size_t i = 0; i < sv.size(); ++i) {
      uint32_t u = sv[i];
      if (!ref_collect(C, N, u, arr)) {
        P.status = REF_EMPTY_REFINE;
        return;
      }
      if (k == 4 || se[i].empty()) continue;
      for (uint32_t mu : arr) {
        for (uint32_t v : se[i]) {
          bool any = false;
          const uint8_t* cv = C.data() + (size_t)v * N;
          for (uint32_t e = g.off[mu]; e < g.off[mu + 1] && !any; ++e) any = cv[g.col[e]] != 0;
          if (!any) {
            C[(size_t)u * N + mu] = 0;
            break;
          }
        }
      }
    }
  }
}

static bool ref_cedges(const DataGraph& g, RefPlan& P, bool reverse) {
  const uint32_t N = g.n;
  auto& bufs = reverse ? P.cedge_rev : P.cedge_fwd;
  auto& sizes = reverse ? P.size_rev : P.size_fwd;
  auto& nums = reverse ? P.num_rev : P.num_fwd;
  bufs.assign(P.m, {});
  sizes.assign(P.m, 0);
  nums.assign(P.m, 0);
  std::vector<uint32_t> arr;
  for (uint32_t i = 0; i < P.m; ++i) {
    uint32_t u = reverse ? P.eto[i] : P.efrom[i];
    uint32_t v = reverse ? P.efrom[i] : P.eto[i];
    if (!ref_collect(P.cand, N, u, arr)) return false;
    const uint32_t na = (uint32_t)arr.size();
    std::vector<uint32_t>& b = bufs[i];
    b.assign(arr.begin(), arr.end());
    b.resize(2 * (size_t)na + 1);
    std::vector<uint32_t> nb;
    const uint8_t* cv = P.cand.data() + (size_t)v * N;
    for (uint32_t k = 0; k < na; ++k) {
      b[na + k] = (uint32_t)nb.size();
      uint32_t mu = arr[k];
      for (uint32_t e = g.off[mu]; e < g.off[mu + 1]; ++e)
        if (cv[g.col[e]]) nb.push_back(g.col[e]);
    }
    b[2 * na] = (uint32_t)nb.size();
    b.insert(b.end(), nb.begin(), nb.end());
    sizes[i] = nb.size();
    nums[i] = na;
  }
  return true;
}

static void ref_order(const DataGraph& g, RefPlan& P) {
  const uint32_t qn = P.q.n;
  std::vector<uint8_t> vv(qn, 0), ve(P.m, 0);
  P.pos2id.assign(qn, -1);
  P.id2pos.assign(qn, -1);
  int cur = 0;
  auto add = [&](uint32_t id) {
    P.pos2id[cur] = (int32_t)id;
    P.id2pos[id] = cur;
    ++cur;
  };
  uint64_t minv = (uint64_t)g.off[g.n] + 1;
  uint32_t minx = 0;
  for (uint32_t i = 0; i < P.m; ++i)
    if (P.size_fwd[i] < minv) {
      minv = P.size_fwd[i];
      minx = i;
    }
  vv[P.efrom[minx]] = vv[P.eto[minx]] = 1;
  ve[minx] = 1;
  P.steps.push_back({minx, 0, 0});
  add(P.efrom[minx]);
  add(P.eto[minx]);
  for (uint32_t cnt = 1; cnt < P.m; ++cnt) {
    std::vector<uint32_t> next;
    bool expand = false;
    for (uint32_t i = 0; i < P.m; ++i)
      if (!ve[i] && vv[P.efrom[i]] && vv[P.eto[i]]) next.push_back(i);
    int defect = 0;
    if (next.empty()) {
      expand = true;
      // the reference considers every unvisited edge (Match.cu:1641-1650);
      // record whether its pick would have had no visited endpoint
      uint64_t rv = (uint64_t)g.off[g.n] + 1;
      uint32_t rx = 0;
      for (uint32_t i = 0; i < P.m; ++i)
        if (!ve[i] && P.size_fwd[i] < rv) {
          rv = P.size_fwd[i];
          rx = i;
        }
      if (!vv[P.efrom[rx]] && !vv[P.eto[rx]]) defect = 1;
      for (uint32_t i = 0; i < P.m; ++i)
        if (!ve[i] && (vv[P.efrom[i]] || vv[P.eto[i]])) next.push_back(i);
    }
    uint64_t nv = (uint64_t)g.off[g.n] + 1;
    uint32_t nx = 0;
    for (uint32_t e : next)
      if (P.size_fwd[e] < nv) {
        nv = P.size_fwd[e];
        nx = e;
      }
    uint32_t u = P.efrom[nx], v = P.eto[nx];
    int mode = 1;
    if (expand) {
      if (vv[u]) {
        mode = 2;
        add(v);
      } else {
        mode = 3;
        add(u);
      }
    }
    P.steps.push_back({nx, mode, defect});
    if (defect) P.defect = 1;
    vv[u] = vv[v] = 1;
    ve[nx] = 1;
  }
}

// Lookup of mu's candidate neighbours in a candidate-edge buffer.
static inline bool cedge_lookup(const std::vector<uint32_t>& b, uint32_t na, uint32_t mu,
                                const uint32_t** beg, const uint32_t** end) {
  const uint32_t* ids = b.data();
  const uint32_t* p = std::lower_bound(ids, ids + na, mu);
  if (p == ids + na || *p != mu) return false;
  size_t k = (size_t)(p - ids);
  *beg = b.data() + 2 * (size_t)na + 1 + b[na + k];
  *end = b.data() + 2 * (size_t)na + 1 + b[na + k + 1];
  return true;
}

// Joins in the plain order. injective=false reproduces the reference table
// (homomorphisms, Match.cu:1141-1569); injective=true drops rows that repeat
// a data vertex as soon as the repeat appears. Rows come out in the
// reference's order (lexicographic by table column). Stops counting at cap.
struct RefJoin {
  const RefPlan& P;
  bool injective;
  uint64_t cap;
  std::vector<uint64_t> level_rows;  // rows alive after each step
  std::vector<uint32_t>* out;        // row-major, pos order (nullable)
  uint64_t final_rows = 0;
  bool capped = false;
  uint64_t work = 0, work_cap = ~0ULL;  // DFS nodes visited; optional bound
  const std::atomic<int>* abort_flag = nullptr;  // set by the caller's deadline
  bool aborted = false;
  std::vector<uint32_t> row;

  RefJoin(const RefPlan& p, bool inj, uint64_t c, std::vector<uint32_t>* o)
      : P(p), injective(inj), cap(c), out(o) {}

  bool used(uint32_t x, int ncols) const {
    for (int i = 0; i < ncols; ++i)
      if (row[i] == x) return true;
    return false;
  }

  void rec(size_t s, int ncols) {
    if (capped) return;
    if (++work >= work_cap) {
      capped = true;
      return;
    }
    if (abort_flag && (work & 0xFFFF) == 0 && abort_flag->load(std::memory_order_relaxed)) {
      capped = true;
      aborted = true;
      return;
    }
    level_rows[s - 1]++;
    if (s == P.steps.size()) {
      if (out) out->insert(out->end(), row.begin(), row.begin() + ncols);
      if (++final_rows >= cap) capped = true;
      return;
    }
    const auto& st = P.steps[s];
    uint32_t e = st.edge;
    uint32_t u = P.efrom[e], v = P.eto[e];
    if (st.mode == 1) {
      const uint32_t *b, *en;
      uint32_t mu = row[P.id2pos_at(u)], mv = row[P.id2pos_at(v)];
      if (!cedge_lookup(P.cedge_fwd[e], P.num_fwd[e], mu, &b, &en)) return;
      for (; b < en; ++b)
        if (*b == mv) {
          rec(s + 1, ncols);
          return;
        }
      return;
    }
    const bool fwd = st.mode == 2;
    const auto& buf = fwd ? P.cedge_fwd[e] : P.cedge_rev[e];
    const uint32_t na = fwd ? P.num_fwd[e] : P.num_rev[e];
    uint32_t anchor = fwd ? u : v;
    const uint32_t *b, *en;
    if (!cedge_lookup(buf, na, row[P.id2pos_at(anchor)], &b, &en)) return;
    for (; b < en && !capped; ++b) {
      if (injective && used(*b, ncols)) continue;
      row[ncols] = *b;
      rec(s + 1, ncols + 1);
    }
  }

  void run() {
    level_rows.assign(P.steps.size(), 0);
    row.assign(P.q.n, 0);
    uint32_t e = P.steps[0].edge;
    const auto& buf = P.cedge_fwd[e];
    const uint32_t na = P.num_fwd[e];
    for (uint32_t k = 0; k < na && !capped; ++k) {
      row[0] = buf[k];
      for (uint32_t j = buf[na + k]; j < buf[na + k + 1] && !capped; ++j) {
        row[1] = buf[2 * (size_t)na + 1 + j];
        if (injective && row[1] == row[0]) continue;
        rec(1, 2);
      }
    }
  }
};

}  // namespace

// ---------------------------------------------------------------------------
// C ABI for the Python test harness
// ---------------------------------------------------------------------------
extern "C" {

// Independent oracle. Writes up to out_cap sorted rows (query-vertex order)
// when out != NULL. Returns the number of embeddings (capped at cap).
int64_t oracle_enumerate(uint32_t n, const uint32_t* off, const uint32_t* col, const uint32_t* lab,
                         uint32_t qn, const uint32_t* qlab, uint32_t qm, const uint32_t* qe,
                         uint64_t cap, uint32_t* out, uint64_t out_cap) {
  DataGraph g{n, off, col, lab};
  Enumerator en(g, qn, qlab, qm, qe, cap, out, out_cap);
  en.run();
  if (out != nullptr) sort_rows(out, std::min(en.count, out_cap), qn);
  return (int64_t)en.count;
}

// The same backtracking in a given vertex order (pos2id: a connected
// permutation of the query vertices). Candidates of each position are taken
// in ascending data-vertex order, so rows are found in lexicographic order
// of (row[pos2id[0]], row[pos2id[1]], ...): the first `cap` rows are the
// first `cap` of that order. Rows are written in position order (column p =
// query vertex pos2id[p]), unsorted, up to out_cap of them; *digest gets an
// order-sensitive digest of all `count` rows (sum over rows i of
// (i + 1) * hash(row i), mod 2^64). Returns the count (at most cap), or -1
// when work_cap search steps (nodes and candidates examined) came first (0 = no bound); then
// *partial gets the rows found so far.
// lidx: a handle from oracle_label_index (or NULL: scan whole lists).
int64_t oracle_enumerate_ordered(uint32_t n, const uint32_t* off, const uint32_t* col, const uint32_t* lab,
                                 uint32_t qn, const uint32_t* qlab, uint32_t qm, const uint32_t* qe,
                                 const int32_t* pos2id, uint64_t cap, uint32_t* out, uint64_t out_cap,
                                 uint64_t work_cap, uint64_t* partial, uint64_t* digest, const void* lidx) {
  DataGraph g{n, off, col, lab};
  Enumerator en(g, qn, qlab, qm, qe, cap, out, out_cap);
  en.lidx = (const LabelIndex*)lidx;
  std::vector<uint8_t> seen(qn, 0);
  for (uint32_t p = 0; p < qn; ++p) {
    const int32_t u = pos2id[p];
    if (u < 0 || (uint32_t)u >= qn || seen[u]) return -2;
    seen[u] = 1;
    en.given.push_back((uint32_t)u);
  }
  en.out_by_pos = true;
  if (work_cap) en.work_cap = work_cap;
  en.run();
  if (partial) *partial = en.count;
  if (digest) *digest = en.digest;
  if (en.work > en.work_cap) return -1;
  return (int64_t)en.count;
}

// The label-run index of a graph for oracle_enumerate_ordered (the graph's
// arrays must outlive it); free with oracle_label_index_free.
void* oracle_label_index(uint32_t n, const uint32_t* off, const uint32_t* col, const uint32_t* lab, int threads) {
  LabelIndex* L = new LabelIndex();
  build_label_index(*L, n, off, col, lab, threads);
  return L;
}

void oracle_label_index_free(void* h) { delete (LabelIndex*)h; }

// ---- restatement of the reference pipeline --------------------------------
// Runs edge list, spanning order, init, refinement, candidate edges (both
// directions) and the plain join order. *status gets a RefStatus.
void* oracle_ref_plan(uint32_t n, const uint32_t* off, const uint32_t* col, const uint32_t* lab,
                      uint32_t qn, const uint32_t* qlab, uint32_t qm, const uint32_t* qe,
                      int32_t* status) {
  DataGraph g{n, off, col, lab};
  RefPlan* P = new RefPlan();
  P->q.build(qn, qlab, qm, qe);
  ref_edges(*P);
  if (P->m == 0) {
    P->status = REF_NO_EDGES;
  } else {
    ref_spanning_order(g, *P);
    if (P->order.size() != qn) {
      P->status = REF_DISCONNECTED;
    } else {
      ref_filter(g, *P);
      if (P->status == REF_OK) {
        if (!ref_cedges(g, *P, false) || !ref_cedges(g, *P, true)) {
          P->status = REF_EMPTY_CEDGE;
        } else {
          ref_order(g, *P);
        }
      }
    }
  }
  if (status) *status = P->status;
  return P;
}

void oracle_ref_free(void* h) { delete (RefPlan*)h; }

void oracle_ref_info(void* h, uint32_t* m, uint32_t* nsteps, int32_t* defect, uint32_t* norder) {
  RefPlan* P = (RefPlan*)h;
  if (m) *m = P->m;
  if (nsteps) *nsteps = (uint32_t)P->steps.size();
  if (defect) *defect = P->defect;
  if (norder) *norder = (uint32_t)P->order.size();
}

void oracle_ref_edges(void* h, uint32_t* efrom, uint32_t* eto) {
  RefPlan* P = (RefPlan*)h;
  for (uint32_t i = 0; i < P->m; ++i) efrom[i] = P->efrom[i], eto[i] = P->eto[i];
}

void oracle_ref_order(void* h, uint32_t* order) {
  RefPlan* P = (RefPlan*)h;
  for (size_t i = 0; i < P->order.size(); ++i) order[i] = P->order[i];
}

// which: 0 = after init (explore), 1 = after refinement. out: qn*N bytes.
int oracle_ref_cand(void* h, int which, uint8_t* out) {
  RefPlan* P = (RefPlan*)h;
  const std::vector<uint8_t>& c = which == 0 ? P->cand_init : P->cand;
  if (c.empty()) return -1;
  memcpy(out, c.data(), c.size());
  return 0;
}

void oracle_ref_cedge_sizes(void* h, uint64_t* size_fwd, uint32_t* num_fwd, uint64_t* size_rev,
                            uint32_t* num_rev) {
  RefPlan* P = (RefPlan*)h;
  for (uint32_t i = 0; i < P->m && i < P->size_fwd.size(); ++i) {
    size_fwd[i] = P->size_fwd[i];
    num_fwd[i] = P->num_fwd[i];
    size_rev[i] = P->size_rev[i];
    num_rev[i] = P->num_rev[i];
  }
}

uint64_t oracle_ref_cedge_len(void* h, uint32_t e, int rev) {
  RefPlan* P = (RefPlan*)h;
  return (rev ? P->cedge_rev : P->cedge_fwd)[e].size();
}

void oracle_ref_cedge_copy(void* h, uint32_t e, int rev, uint32_t* out) {
  RefPlan* P = (RefPlan*)h;
  const auto& b = (rev ? P->cedge_rev : P->cedge_fwd)[e];
  memcpy(out, b.data(), b.size() * 4);
}

void oracle_ref_steps(void* h, uint32_t* edge, int32_t* mode, int32_t* defect) {
  RefPlan* P = (RefPlan*)h;
  for (size_t i = 0; i < P->steps.size(); ++i) {
    edge[i] = P->steps[i].edge;
    mode[i] = P->steps[i].mode;
    defect[i] = P->steps[i].defect;
  }
}

void oracle_ref_mapping(void* h, int32_t* id2pos, int32_t* pos2id) {
  RefPlan* P = (RefPlan*)h;
  for (uint32_t i = 0; i < P->q.n; ++i) {
    id2pos[i] = P->id2pos.empty() ? -1 : P->id2pos[i];
    pos2id[i] = P->pos2id.empty() ? -1 : P->pos2id[i];
  }
}

// Joins in the plain order. injective=0: the reference's homomorphism table;
// injective=1: rows repeating a data vertex are dropped. level_rows (nsteps)
// gets the rows alive after each step (capped run: partial). Rows are
// written in table-column order when out != NULL (up to out_cap rows).
// Returns the number of final rows (at most cap).
int64_t oracle_ref_join(void* h, int injective, uint64_t cap, uint64_t* level_rows, uint32_t* out,
                        uint64_t out_cap, int* capped, uint64_t work_cap) {
  RefPlan* P = (RefPlan*)h;
  if (P->status != REF_OK || P->steps.empty()) {
    if (capped) *capped = 0;
    return 0;
  }
  std::vector<uint32_t> rows;
  RefJoin J(*P, injective != 0, cap, out ? &rows : nullptr);
  if (work_cap) J.work_cap = work_cap;
  J.run();
  if (level_rows)
    for (size_t i = 0; i < J.level_rows.size(); ++i) level_rows[i] = J.level_rows[i];
  if (out) {
    uint64_t nr = std::min<uint64_t>(J.final_rows, out_cap);
    memcpy(out, rows.data(), nr * P->q.n * 4);
  }
  if (capped) *capped = J.capped ? 1 : 0;
  return (int64_t)J.final_rows;
}

// IO::verify (io/IO.cpp:146-180) for one row in table-column order: the row
// must be injective and every query edge (from -> to, file order) must be a
// data edge stored as from -> to in the data file. data_from/data_to hold the
// data file's edges sorted by (from, to).
int oracle_ref_verify(void* h, const int32_t* id2pos, const uint32_t* row, uint64_t dm,
                      const uint32_t* data_edges_sorted) {
  RefPlan* P = (RefPlan*)h;
  const uint32_t n = P->q.n;
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t j = i + 1; j < n; ++j)
      if (row[i] == row[j]) return 0;
  for (size_t k = 0; k < P->q.qm_from.size(); ++k) {
    uint32_t a = row[id2pos[P->q.qm_from[k]]], b = row[id2pos[P->q.qm_to[k]]];
    uint64_t key = ((uint64_t)a << 32) | b;
    uint64_t lo = 0, hi = dm;
    bool found = false;
    while (lo < hi) {
      uint64_t mid = (lo + hi) / 2;
      uint64_t mk = ((uint64_t)data_edges_sorted[2 * mid] << 32) | data_edges_sorted[2 * mid + 1];
      if (mk == key) {
        found = true;
        break;
      }
      if (mk < key) lo = mid + 1;
      else hi = mid;
    }
    if (!found) return 0;
  }
  return 1;
}

// CPU port of the whole path, for the baseline: for each query, the
// restated filter, refinement, candidate edges and plain-order joins with
// the injectivity check (counting embeddings, at most cap per query).
// Queries are spread over `threads` host threads. Query k has vertices
// q_voff[k]..q_voff[k+1] (labels in qlab) and edges q_eoff[k]..q_eoff[k+1]
// (pairs in qe). counts[k] gets the embedding count, -(RefStatus) for a
// query the reference cannot run, or INT64_MIN when the deadline (seconds,
// 0 = none) stopped it first. Returns elapsed seconds.
double oracle_cpu_pipeline(uint32_t n, const uint32_t* off, const uint32_t* col, const uint32_t* lab,
                           uint32_t nq, const uint32_t* q_voff, const uint32_t* qlab,
                           const uint64_t* q_eoff, const uint32_t* qe, int threads, uint64_t cap,
                           int64_t* counts, double deadline_s) {
  auto t0 = std::chrono::steady_clock::now();
  std::atomic<uint32_t> next(0);
  std::atomic<int> abort_flag(0);
  auto work = [&] {
    for (;;) {
      if (abort_flag.load()) break;
      uint32_t k = next.fetch_add(1);
      if (k >= nq) break;
      uint32_t qn = q_voff[k + 1] - q_voff[k];
      uint32_t qm = (uint32_t)(q_eoff[k + 1] - q_eoff[k]);
      int32_t st = 0;
      RefPlan* P = (RefPlan*)oracle_ref_plan(n, off, col, lab, qn, qlab + q_voff[k], qm,
                                             qe + 2 * q_eoff[k], &st);
      if (st != REF_OK) {
        counts[k] = (st == REF_EMPTY_INIT || st == REF_EMPTY_REFINE) ? 0 : -(int64_t)st;
      } else {
        RefJoin J(*P, true, cap, nullptr);
        J.abort_flag = &abort_flag;
        J.run();
        counts[k] = J.aborted ? INT64_MIN : (int64_t)J.final_rows;
      }
      delete P;
    }
  };
  for (uint32_t k = 0; k < nq; ++k) counts[k] = INT64_MIN;
  if (threads < 1) threads = 1;
  std::vector<std::thread> ts;
  for (int t = 0; t < threads; ++t) ts.emplace_back(work);
  // watchdog: raises the abort flag at the deadline; joined before return
  // (it reads this frame's locals)
  std::atomic<int> workers_done(0);
  std::thread watchdog;
  if (deadline_s > 0)
    watchdog = std::thread([&] {
      while (!workers_done.load()) {
        double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el >= deadline_s) {
          abort_flag.store(1);
          break;
        }
        std::this_thread::sleep_for(std::chrono::milliseconds(20));
      }
    });
  for (auto& th : ts) th.join();
  double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  workers_done.store(1);
  if (watchdog.joinable()) watchdog.join();
  return el;
}

}  // extern "C"
