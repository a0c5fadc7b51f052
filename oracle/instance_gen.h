// Seeded planted 3-SAT formulas and uniform initial states for the CPU reference runs.
//
// TEST INFRASTRUCTURE ONLY.  A restatement of the library's generator
// (dmm_cnf_generate_planted) and uniform initial state (dmm_initial_state_uniform), so that
// a process timing the reference integrator can build the same formula and starting state
// without loading the library it is compared with.  tests/test_oracle.py checks that both
// produce identical arrays for the same arguments.
//
// Random numbers: xoshiro256** seeded through splitmix64 (Blackman & Vigna, public-domain
// algorithms); a uniform double takes the top 53 bits; a uniform integer in [0, k) rejects
// draws at or above the largest multiple of k.
#pragma once

#include <cstdint>
#include <vector>

namespace oracle_gen {

struct Xoshiro {
  uint64_t s[4];
  explicit Xoshiro(uint64_t seed) {
    uint64_t z = seed;
    for (int i = 0; i < 4; i++) {
      z += 0x9e3779b97f4a7c15ull;
      uint64_t x = z;
      x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
      x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
      s[i] = x ^ (x >> 31);
    }
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t out = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return out;
  }
  double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  uint64_t below(uint64_t k) {
    const uint64_t lim = UINT64_MAX - UINT64_MAX % k;
    for (;;) {
      const uint64_t x = next();
      if (x < lim) return x % k;
    }
  }
};

// Planted 3-SAT: the planted sign of each variable from the top bit of one draw; per clause
// three distinct variables, then one uniform draw choosing how many literals agree with the
// planted assignment (3 below p0, 1 below p0 + p1, else 2) and, for 1 or 2, one draw for
// the position that differs from the rest.  lits: 3m entries, clause_off: m + 1.
inline void planted(int32_t n, int32_t m, double p0, double p1, uint64_t seed, int32_t* lits,
                    int64_t* clause_off, int8_t* sigma_out) {
  Xoshiro r(seed);
  std::vector<int8_t> sigma(n);
  for (int32_t i = 0; i < n; i++) sigma[i] = (r.next() >> 63) ? 1 : -1;
  for (int32_t c = 0; c < m; c++) {
    int32_t v0 = (int32_t)r.below(n), v1, v2;
    do v1 = (int32_t)r.below(n);
    while (v1 == v0);
    do v2 = (int32_t)r.below(n);
    while (v2 == v0 || v2 == v1);
    const double u = r.unit();
    bool agree[3] = {true, true, true};
    if (u >= p0) {
      if (u < p0 + p1) {  // exactly one literal agrees
        const int k = (int)r.below(3);
        for (int j = 0; j < 3; j++) agree[j] = j == k;
      } else {  // exactly two agree
        agree[r.below(3)] = false;
      }
    }
    const int32_t v[3] = {v0, v1, v2};
    for (int j = 0; j < 3; j++) {
      const int s = agree[j] ? sigma[v[j]] : -sigma[v[j]];
      lits[3 * (int64_t)c + j] = s * (v[j] + 1);
    }
    clause_off[c] = 3 * (int64_t)c;
  }
  clause_off[m] = 3 * (int64_t)m;
  if (sigma_out)
    for (int32_t i = 0; i < n; i++) sigma_out[i] = sigma[i];
}

// V ~ U[-1, 1] (unit-clause variables pinned to their sign), Xs ~ U[0, 1], Xl = 1; the
// draws go to V first, then Xs, in index order.
inline void uniform_state(const int32_t* lits, const int64_t* clause_off, int32_t n, int32_t m,
                          uint64_t seed, double* x) {
  std::vector<int8_t> pin(n, 0);
  for (int32_t c = 0; c < m; c++)
    if (clause_off[c + 1] - clause_off[c] == 1) {
      const int32_t l = lits[clause_off[c]];
      pin[(l < 0 ? -l : l) - 1] = l > 0 ? 1 : -1;
    }
  Xoshiro r(seed);
  for (int32_t j = 0; j < n; j++) x[j] = pin[j] != 0 ? (double)pin[j] : 2.0 * r.unit() - 1.0;
  for (int32_t j = 0; j < m; j++) x[n + j] = r.unit();
  for (int32_t j = 0; j < m; j++) x[(int64_t)n + m + j] = 1.0;
}

}  // namespace oracle_gen
