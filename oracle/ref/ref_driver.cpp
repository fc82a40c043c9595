// ORACLE (test infrastructure): a driver linked against the reference's own
// objects (built from the unmodified sources by oracle/ref.mk). For every
// query it calls the reference's Match::match and dumps the raw result table
// BEFORE IO::verify's directed/edge-label filter (io/IO.cpp:146-180), so the
// reference's undirected matches can be compared with the oracle's.
//
//   ref_driver DATA QUERY OUT.bin [dev]
// OUT.bin records, per query: int32 qid, uint32 rows, uint32 cols,
// float match_ms, int32 id_map[cols], uint32 table[rows*cols].
#include "io/IO.h"
#include "match/Match.h"

#include <chrono>

int main(int argc, const char* argv[]) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s data query out.bin [dev]\n", argv[0]);
    return 2;
  }
  int dev = argc >= 5 ? atoi(argv[4]) : 0;
  Match::initGPU(dev);
  IO io = IO(argv[2], argv[1], "/dev/null");
  std::vector<Graph*> qs;
  io.input(qs);
  Graph* data = NULL;
  if (!io.input(data)) {
    fprintf(stderr, "no data graph\n");
    return 3;
  }
  FILE* f = fopen(argv[3], "wb");
  if (!f) return 4;
  for (size_t i = 0; i < qs.size(); ++i) {
    Match m(qs[i], data);
    unsigned* fr = NULL;
    unsigned rows = 0, cols = 0;
    int* idm = NULL;
    auto t0 = std::chrono::steady_clock::now();
    m.match(io, fr, rows, cols, idm);
    auto t1 = std::chrono::steady_clock::now();
    float ms = std::chrono::duration<float, std::milli>(t1 - t0).count();
    int32_t qid = (int32_t)i;
    uint32_t r = fr ? rows : 0, c = qs[i]->vertex_num;
    fwrite(&qid, 4, 1, f);
    fwrite(&r, 4, 1, f);
    fwrite(&c, 4, 1, f);
    fwrite(&ms, 4, 1, f);
    for (uint32_t j = 0; j < c; ++j) {
      int32_t x = idm ? idm[j] : -1;
      fwrite(&x, 4, 1, f);
    }
    if (r) fwrite(fr, 4, (size_t)r * c, f);
    delete[] fr;
    fflush(f);
  }
  fclose(f);
  return 0;
}
