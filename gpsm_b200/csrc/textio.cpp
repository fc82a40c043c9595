// The reference's graph text format at full speed (io/IO.cpp:46-128 reads
// it with one fscanf per token, which takes minutes for a 256M-edge file).
//
// Format: `t # <id>` starts a graph (id -1 ends the file), then a line of
// four counts (ignored, as the reference ignores them), `v <id> <label>` per
// vertex (the id is ignored: vertices are numbered in file order, as
// Graph::addVertex does), `e <from> <to> <label>` per edge in file order.
//
// The file is memory-mapped; graph boundaries are found by one scan for
// "\nt"; within a graph, lines are split into per-thread chunks at line
// starts, each thread counts its `v`/`e` lines, and a second pass parses
// into the exact output positions.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "gpsm.h"
#include "internal.h"

struct gpsm_text_s {
  const char* data = nullptr;
  size_t size = 0;
  int fd = -1;
  struct G {
    int32_t id;
    size_t begin, end;  // byte range after the header lines
    uint32_t n = 0;
    uint64_t m = 0;
    bool counted = false;
    std::vector<size_t> chunk;           // chunk start offsets (line starts)
    std::vector<uint32_t> nv;            // vertices per chunk
    std::vector<uint64_t> ne;            // edges per chunk
  };
  std::vector<G> graphs;
};

namespace {

int threads_for(size_t bytes) {
  unsigned t = std::thread::hardware_concurrency();
  if (t == 0) t = 1;
  size_t by_size = bytes / (1u << 20) + 1;  // at least 1 MiB per thread
  return (int)std::min<size_t>(std::min<unsigned>(t, 64), by_size);
}

inline const char* skip_ws(const char* p, const char* e) {
  while (p < e && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
  return p;
}

inline const char* parse_i64(const char* p, const char* e, long long* out) {
  p = skip_ws(p, e);
  bool neg = false;
  if (p < e && *p == '-') {
    neg = true;
    ++p;
  }
  long long v = 0;
  const char* s = p;
  while (p < e && *p >= '0' && *p <= '9') v = v * 10 + (*p++ - '0');
  if (p == s) return nullptr;
  *out = neg ? -v : v;
  return p;
}

inline const char* next_line(const char* p, const char* e) {
  while (p < e && *p != '\n') ++p;
  return p < e ? p + 1 : e;
}

void count_graph(gpsm_text_s::G& g, const char* base) {
  const size_t len = g.end - g.begin;
  const int T = threads_for(len);
  g.chunk.assign(T + 1, g.end);
  g.chunk[0] = g.begin;
  for (int t = 1; t < T; ++t) {
    const char* p = base + g.begin + len * t / T;
    const char* e = base + g.end;
    // advance to the next line start
    if (p > base + g.begin && p[-1] != '\n') p = next_line(p, e);
    g.chunk[t] = std::max<size_t>(p - base, g.chunk[t - 1]);
  }
  g.nv.assign(T, 0);
  g.ne.assign(T, 0);
  std::vector<std::thread> th;
  for (int t = 0; t < T; ++t)
    th.emplace_back([&, t] {
      const char* p = base + g.chunk[t];
      const char* e = base + g.chunk[t + 1];
      uint32_t nv = 0;
      uint64_t ne = 0;
      while (p < e) {
        const char* q = skip_ws(p, e);
        if (q < e) {
          if (*q == 'v') ++nv;
          else if (*q == 'e') ++ne;
        }
        p = next_line(q, e);
      }
      g.nv[t] = nv;
      g.ne[t] = ne;
    });
  for (auto& x : th) x.join();
  uint64_t nv = 0, ne = 0;
  for (int t = 0; t < T; ++t) {
    nv += g.nv[t];
    ne += g.ne[t];
  }
  g.n = (uint32_t)nv;
  g.m = ne;
  g.counted = true;
}

}  // namespace

extern "C" {

int gpsm_text_open(const char* path, gpsm_text_t* out) {
  if (!path || !out) return GPSM_ERR_INVALID;
  int fd = open(path, O_RDONLY);
  if (fd < 0) {
    gpsm::set_last_error(std::string("cannot open ") + path);
    return GPSM_ERR_INVALID;
  }
  struct stat st;
  if (fstat(fd, &st) != 0) {
    close(fd);
    return GPSM_ERR_INVALID;
  }
  gpsm_text_s* h = new gpsm_text_s();
  h->fd = fd;
  h->size = (size_t)st.st_size;
  if (h->size) {
    void* m = mmap(nullptr, h->size, PROT_READ, MAP_PRIVATE, fd, 0);
    if (m == MAP_FAILED) {
      close(fd);
      delete h;
      return GPSM_ERR_NOMEM;
    }
    h->data = (const char*)m;
  }
  // graph headers: a line whose first non-blank character is 't'
  const char* p = h->data;
  const char* e = h->data + h->size;
  gpsm_text_s::G* cur = nullptr;
  while (p < e) {
    const char* q = skip_ws(p, e);
    const char* nl = next_line(q, e);
    if (q < e && *q == 't') {
      if (cur) cur->end = (size_t)(p - h->data);
      const char* r = q + 1;
      r = skip_ws(r, e);
      if (r < e && *r == '#') ++r;
      long long id = 0;
      if (!parse_i64(r, nl, &id)) {
        gpsm::set_last_error("malformed graph header");
        gpsm_text_close(h);
        return GPSM_ERR_INVALID;
      }
      if (id == -1) {
        cur = nullptr;
        break;
      }
      h->graphs.emplace_back();
      cur = &h->graphs.back();
      cur->id = (int32_t)id;
      // skip the counts line that follows the header
      const char* after = nl;
      cur->begin = (size_t)(next_line(after, e) - h->data);
      p = h->data + cur->begin;
      continue;
    }
    p = nl;
  }
  if (cur) cur->end = h->size;  // no `t # -1`: the last graph runs to the end of the file
  *out = h;
  return GPSM_OK;
}

int gpsm_text_count(gpsm_text_t h, uint32_t* ngraphs) {
  if (!h || !ngraphs) return GPSM_ERR_INVALID;
  *ngraphs = (uint32_t)h->graphs.size();
  return GPSM_OK;
}

int gpsm_text_graph_info(gpsm_text_t h, uint32_t k, uint32_t* n, uint64_t* m, int32_t* id) {
  if (!h || k >= h->graphs.size()) return GPSM_ERR_INVALID;
  auto& g = h->graphs[k];
  if (!g.counted) count_graph(g, h->data);
  if (n) *n = g.n;
  if (m) *m = g.m;
  if (id) *id = g.id;
  return GPSM_OK;
}

// labels[n]; edges[2m] (from, to) in file order; edge_labels[m] or NULL.
int gpsm_text_graph_read(gpsm_text_t h, uint32_t k, uint32_t* labels, uint32_t* edges, uint32_t* edge_labels) {
  if (!h || k >= h->graphs.size()) return GPSM_ERR_INVALID;
  auto& g = h->graphs[k];
  if (!g.counted) count_graph(g, h->data);
  if ((g.n && !labels) || (g.m && !edges)) return GPSM_ERR_INVALID;
  const int T = (int)g.nv.size();
  std::vector<uint64_t> vbase(T + 1, 0), ebase(T + 1, 0);
  for (int t = 0; t < T; ++t) {
    vbase[t + 1] = vbase[t] + g.nv[t];
    ebase[t + 1] = ebase[t] + g.ne[t];
  }
  std::vector<int> bad(T, 0);
  std::vector<std::thread> th;
  for (int t = 0; t < T; ++t)
    th.emplace_back([&, t] {
      const char* p = h->data + g.chunk[t];
      const char* e = h->data + g.chunk[t + 1];
      uint64_t vi = vbase[t], ei = ebase[t];
      while (p < e) {
        const char* q = skip_ws(p, e);
        const char* nl = next_line(q, e);
        if (q < e && (*q == 'v' || *q == 'e')) {
          long long a = 0, b = 0, c = 0;
          const char* r = parse_i64(q + 1, nl, &a);
          if (r) r = parse_i64(r, nl, &b);
          if (*q == 'v') {
            if (!r) {
              bad[t] = 1;
              return;
            }
            labels[vi++] = (uint32_t)b;
          } else {
            if (r) r = parse_i64(r, nl, &c);
            if (!r || a < 0 || b < 0) {
              bad[t] = 1;
              return;
            }
            edges[2 * ei] = (uint32_t)a;
            edges[2 * ei + 1] = (uint32_t)b;
            if (edge_labels) edge_labels[ei] = (uint32_t)c;
            ++ei;
          }
        } else if (q < e && *q != '\n' && *q != '#') {
          bad[t] = 1;  // the reference stops on any other leading character
          return;
        }
        p = nl;
      }
    });
  for (auto& x : th) x.join();
  for (int t = 0; t < T; ++t)
    if (bad[t]) {
      gpsm::set_last_error("malformed vertex or edge line");
      return GPSM_ERR_INVALID;
    }
  for (uint64_t i = 0; i < g.m; ++i)
    if (edges[2 * i] >= g.n || edges[2 * i + 1] >= g.n) {
      gpsm::set_last_error("edge endpoint out of range");
      return GPSM_ERR_INVALID;
    }
  return GPSM_OK;
}

int gpsm_text_close(gpsm_text_t h) {
  if (!h) return GPSM_ERR_INVALID;
  if (h->data) munmap((void*)h->data, h->size);
  if (h->fd >= 0) close(h->fd);
  delete h;
  return GPSM_OK;
}

// Appends (append != 0) or writes one graph; terminate != 0 adds `t # -1`.
int gpsm_text_write(const char* path, int append, int32_t id, uint32_t n, const uint32_t* labels, uint64_t m,
                    const uint32_t* edges, const uint32_t* edge_labels, int terminate) {
  if (!path || (n && !labels) || (m && !edges)) return GPSM_ERR_INVALID;
  FILE* f = fopen(path, append ? "ab" : "wb");
  if (!f) return GPSM_ERR_INVALID;
  std::vector<char> buf(1 << 22);
  setvbuf(f, buf.data(), _IOFBF, buf.size());
  uint32_t nl = 0;
  if (n) {
    std::vector<uint32_t> l(labels, labels + n);
    std::sort(l.begin(), l.end());
    nl = (uint32_t)(std::unique(l.begin(), l.end()) - l.begin());
  }
  fprintf(f, "t # %d\n%u %llu %u 1\n", id, n, (unsigned long long)m, nl);
  char line[96];
  for (uint32_t i = 0; i < n; ++i) {
    int k = snprintf(line, sizeof(line), "v %u %u\n", i, labels[i]);
    fwrite(line, 1, k, f);
  }
  for (uint64_t i = 0; i < m; ++i) {
    int k = snprintf(line, sizeof(line), "e %u %u %u\n", edges[2 * i], edges[2 * i + 1],
                     edge_labels ? edge_labels[i] : 1u);
    fwrite(line, 1, k, f);
  }
  if (terminate) fputs("t # -1\n", f);
  const int rc = fclose(f) == 0 ? GPSM_OK : GPSM_ERR_INVALID;
  return rc;
}

}  // extern "C"
