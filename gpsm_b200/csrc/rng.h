// Deterministic pseudo-random streams for the synthetic workload generators.
// splitmix64 seeds xoshiro256** (Blackman & Vigna, "Scrambled linear
// pseudorandom number generators", 2018). Every generator derives one stream
// per (seed, purpose, chunk) so results do not depend on thread count.
#pragma once
#include <cstdint>

namespace gpsm {

static inline uint64_t splitmix64(uint64_t& x) {
  uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

static inline uint64_t mix64(uint64_t a, uint64_t b) {
  uint64_t s = a * 0x9e3779b97f4a7c15ULL + b;
  return splitmix64(s);
}

struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed, uint64_t stream = 0) {
    uint64_t x = seed ^ (stream * 0xd1b54a32d192ed03ULL);
    for (int i = 0; i < 4; ++i) s[i] = splitmix64(x);
  }
  static inline uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
  inline uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  // uniform double in [0, 1) with 53 random bits
  inline double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  // uniform integer in [0, n) by 128-bit multiply (Lemire); n > 0
  inline uint64_t below(uint64_t n) {
    return (uint64_t)(((unsigned __int128)next() * (unsigned __int128)n) >> 64);
  }
};

}  // namespace gpsm
