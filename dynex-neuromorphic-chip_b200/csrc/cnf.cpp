// Host-side formula handling: DIMACS reader/writer, planted generator, strict-sign
// checker and initial states.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "dmm_pack.h"

namespace dmm {

// xoshiro256** seeded through splitmix64 (Blackman & Vigna, public-domain algorithms).
struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
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
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  // uniform integer in [0, k) by rejection (unbiased)
  uint64_t below(uint64_t k) {
    const uint64_t lim = UINT64_MAX - UINT64_MAX % k;
    uint64_t x;
    do x = next();
    while (x >= lim);
    return x % k;
  }
};

static dmm_status alloc_cnf(int32_t n, int32_t m, int64_t nlits, dmm_cnf** out) {
  dmm_cnf* c = static_cast<dmm_cnf*>(std::calloc(1, sizeof(dmm_cnf)));
  if (!c) return DMM_ERR_NOMEM;
  c->n = n;
  c->m = m;
  c->nlits = nlits;
  c->lits = static_cast<int32_t*>(std::malloc(std::max<int64_t>(nlits, 1) * sizeof(int32_t)));
  c->clause_off = static_cast<int64_t*>(std::malloc((size_t)(m + 1) * sizeof(int64_t)));
  if (!c->lits || !c->clause_off) {
    std::free(c->lits);
    std::free(c->clause_off);
    std::free(c);
    return DMM_ERR_NOMEM;
  }
  *out = c;
  return DMM_OK;
}

static void occurrences(dmm_cnf* c) {
  std::vector<int32_t> occ(c->n + 1, 0);
  int32_t mx = 0;
  for (int64_t i = 0; i < c->nlits; i++) mx = std::max(mx, ++occ[std::abs(c->lits[i])]);
  c->max_occurrence = mx;
}

}  // namespace dmm

using namespace dmm;

extern "C" {

void dmm_cnf_free(dmm_cnf* c) {
  if (!c) return;
  std::free(c->lits);
  std::free(c->clause_off);
  std::free(c);
}

// DIMACS reader (dynex.cc:2306-2392): tokens before `p` are skipped (comment lines),
// `p cnf n m`, then m clauses of 0-terminated literals where a `c` token inside the
// clause section skips the rest of its line.  A clause longer than DMM_MAX_CLAUSE_LITS is
// an error as in the reference.  A file that ends before m clauses is an error here
// (the reference would read empty clauses).
dmm_status dmm_cnf_read(const char* path, dmm_cnf** out) {
  clear_error();
  if (!path || !out) return DMM_ERR_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error("cannot open %s", path);
    return DMM_ERR_IO;
  }
  std::string buf;
  {
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (sz < 0) sz = 0;
    buf.resize((size_t)sz);
    if (sz > 0 && std::fread(&buf[0], 1, (size_t)sz, f) != (size_t)sz) {
      std::fclose(f);
      set_error("read error on %s", path);
      return DMM_ERR_IO;
    }
    std::fclose(f);
  }
  const char* p = buf.data();
  const char* e = p + buf.size();
  auto skip_ws = [&]() {
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r' || *p == '\f' || *p == '\v'))
      p++;
  };
  auto token = [&](const char** b, const char** te) -> bool {
    skip_ws();
    if (p >= e) return false;
    *b = p;
    while (p < e && !(*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r' || *p == '\f' || *p == '\v'))
      p++;
    *te = p;
    return true;
  };
  const char *tb, *te;
  bool found = false;
  while (token(&tb, &te)) {
    if (te - tb == 1 && *tb == 'p') {
      found = true;
      break;
    }
  }
  if (!found) {
    set_error("%s: no `p cnf` header", path);
    return DMM_ERR_PARSE;
  }
  if (!token(&tb, &te) || std::string(tb, te) != "cnf") {
    set_error("%s: expected `p cnf n m`", path);
    return DMM_ERR_PARSE;
  }
  long long nn = 0, mm = 0;
  {
    if (!token(&tb, &te)) return DMM_ERR_PARSE;
    nn = std::atoll(std::string(tb, te).c_str());
    if (!token(&tb, &te)) return DMM_ERR_PARSE;
    mm = std::atoll(std::string(tb, te).c_str());
  }
  if (nn <= 0 || nn > 0x7fffffffll || mm < 0 || mm > 0x7fffffffll) {
    set_error("%s: bad header n=%lld m=%lld", path, nn, mm);
    return DMM_ERR_PARSE;
  }
  std::vector<int32_t> lits;
  std::vector<int64_t> off;
  lits.reserve((size_t)mm * 3);
  off.reserve((size_t)mm + 1);
  off.push_back(0);
  for (long long i = 0; i < mm; i++) {
    int len = 0;
    for (;;) {
      if (!token(&tb, &te)) {
        set_error("%s: file ends after %lld of %lld clauses", path, i, mm);
        return DMM_ERR_PARSE;
      }
      if (te - tb == 1 && *tb == 'c') {
        while (p < e && *p != '\n') p++;
        continue;
      }
      char* endp = nullptr;
      std::string tok(tb, te);
      const long long v = std::strtoll(tok.c_str(), &endp, 10);
      if (endp == tok.c_str() || *endp != '\0') {
        set_error("%s: bad literal `%s` in clause %lld", path, tok.c_str(), i);
        return DMM_ERR_PARSE;
      }
      if (v == 0) break;
      if (v > nn || v < -nn) {
        set_error("%s: literal %lld out of range in clause %lld", path, v, i);
        return DMM_ERR_LITERAL;
      }
      if (++len > DMM_MAX_CLAUSE_LITS) {
        set_error("CLAUSE %lld HAS MORE THAN %d LITERALS.", i, DMM_MAX_CLAUSE_LITS);
        return DMM_ERR_CLAUSE_LEN;
      }
      lits.push_back((int32_t)v);
    }
    off.push_back((int64_t)lits.size());
  }
  dmm_cnf* c = nullptr;
  dmm_status st = alloc_cnf((int32_t)nn, (int32_t)mm, (int64_t)lits.size(), &c);
  if (st != DMM_OK) return st;
  std::memcpy(c->lits, lits.data(), lits.size() * sizeof(int32_t));
  std::memcpy(c->clause_off, off.data(), off.size() * sizeof(int64_t));
  occurrences(c);
  *out = c;
  return DMM_OK;
}

dmm_status dmm_cnf_from_arrays(const int32_t* lits, const int64_t* clause_off, int32_t n,
                               int32_t m, dmm_cnf** out) {
  clear_error();
  if (!out) return DMM_ERR_ARG;
  bool k3;
  dmm_status st = validate_formula(lits, clause_off, n, m, &k3);
  if (st != DMM_OK) return st;
  dmm_cnf* c = nullptr;
  st = alloc_cnf(n, m, clause_off[m], &c);
  if (st != DMM_OK) return st;
  if (clause_off[m] > 0) std::memcpy(c->lits, lits, (size_t)clause_off[m] * sizeof(int32_t));
  std::memcpy(c->clause_off, clause_off, (size_t)(m + 1) * sizeof(int64_t));
  occurrences(c);
  *out = c;
  return DMM_OK;
}

dmm_status dmm_cnf_write(const dmm_cnf* c, const char* path, const int8_t* planted) {
  clear_error();
  if (!c || !path) return DMM_ERR_ARG;
  FILE* f = std::fopen(path, "w");
  if (!f) {
    set_error("cannot write %s", path);
    return DMM_ERR_IO;
  }
  if (planted) {
    std::fprintf(f, "c [");
    for (int32_t i = 0; i < c->n; i++) std::fprintf(f, " %d", planted[i] > 0 ? i + 1 : -(i + 1));
    std::fprintf(f, " ]\n");
  }
  std::fprintf(f, "p cnf %d %d\n", c->n, c->m);
  for (int32_t i = 0; i < c->m; i++) {
    for (int64_t j = c->clause_off[i]; j < c->clause_off[i + 1]; j++) std::fprintf(f, "%d ", c->lits[j]);
    std::fprintf(f, "0\n");
  }
  const bool ok = std::fclose(f) == 0;
  return ok ? DMM_OK : DMM_ERR_IO;
}

dmm_status dmm_state_write(const char* path, const double* x, int32_t n, int32_t m, double t) {
  clear_error();
  if (!path || !x || n < 0 || m < 0) return DMM_ERR_ARG;
  FILE* f = std::fopen(path, "w");
  if (!f) {
    set_error("cannot write %s", path);
    return DMM_ERR_IO;
  }
  const int64_t N = (int64_t)n + 2 * (int64_t)m;
  for (int64_t j = 0; j < N; j++) std::fprintf(f, "%.15f, ", x[j]);
  std::fprintf(f, "%.15f ", t);
  const bool ok = std::fclose(f) == 0;
  if (!ok) set_error("writing %s failed", path);
  return ok ? DMM_OK : DMM_ERR_IO;
}

dmm_status dmm_state_read(const char* path, int32_t n, int32_t m, int32_t reference_rounding,
                          double* x, double* t) {
  clear_error();
  if (!path || !x || !t || n < 0 || m < 0) return DMM_ERR_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error("cannot read %s", path);
    return DMM_ERR_IO;
  }
  std::string text;
  char buf[1 << 16];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, got);
  std::fclose(f);
  const int64_t N = (int64_t)n + 2 * (int64_t)m;
  const char* p = text.c_str();
  for (int64_t k = 0; k <= N; k++) {
    while (*p == ',' || std::isspace((unsigned char)*p)) p++;
    char* end = nullptr;
    // the reference reads each value with fscanf("%f") into a float
    const double v = reference_rounding ? (double)std::strtof(p, &end) : std::strtod(p, &end);
    if (end == p) {
      set_error("%s: %lld numbers where the state needs %lld (n + 2m values and t)", path,
                (long long)k, (long long)(N + 1));
      return DMM_ERR_PARSE;
    }
    p = end;
    if (k < N) x[k] = v;
    else *t = v;
  }
  return DMM_OK;
}

dmm_status dmm_cnf_generate_planted(int32_t n, int32_t m, double p0, double p1, uint64_t seed,
                                    dmm_cnf** out, int8_t* planted) {
  clear_error();
  if (!out || n < 3 || m < 0 || p0 < 0 || p1 < 0 || p0 + p1 > 1.0) {
    set_error("generate_planted: need n >= 3, m >= 0, p0, p1 >= 0, p0 + p1 <= 1");
    return DMM_ERR_ARG;
  }
  dmm_cnf* c = nullptr;
  dmm_status st = alloc_cnf(n, m, 3 * (int64_t)m, &c);
  if (st != DMM_OK) return st;
  Rng r(seed);
  std::vector<int8_t> sigma(n);
  for (int32_t i = 0; i < n; i++) sigma[i] = (r.next() >> 63) ? 1 : -1;
  for (int32_t i = 0; i < m; i++) {
    int32_t v[3];
    v[0] = (int32_t)r.below(n);
    do v[1] = (int32_t)r.below(n);
    while (v[1] == v[0]);
    do v[2] = (int32_t)r.below(n);
    while (v[2] == v[0] || v[2] == v[1]);
    const double x = r.uniform();
    const int agree = x < p0 ? 3 : (x < p0 + p1 ? 1 : 2);
    bool ag[3] = {true, true, true};
    if (agree == 1) {
      ag[0] = ag[1] = ag[2] = false;
      ag[r.below(3)] = true;
    } else if (agree == 2) {
      ag[r.below(3)] = false;
    }
    for (int j = 0; j < 3; j++) {
      const int s = ag[j] ? sigma[v[j]] : -sigma[v[j]];
      c->lits[3 * (int64_t)i + j] = s * (v[j] + 1);
    }
    c->clause_off[i] = 3 * (int64_t)i;
  }
  c->clause_off[m] = 3 * (int64_t)m;
  occurrences(c);
  if (planted) std::memcpy(planted, sigma.data(), n);
  *out = c;
  return DMM_OK;
}

int64_t dmm_check_assignment(const int32_t* lits, const int64_t* clause_off, int32_t m, int32_t n,
                             const int8_t* assign) {
  if (!clause_off || !assign || m < 0 || n <= 0) return -1;
  int64_t bad = 0;
  for (int32_t c = 0; c < m; c++) {
    bool sat = false;
    for (int64_t j = clause_off[c]; j < clause_off[c + 1]; j++) {
      const int32_t l = lits[j];
      const int32_t v = std::abs(l);
      if (v < 1 || v > n) return -1;
      const int8_t a = assign[v - 1];
      if ((a > 0 && l > 0) || (a < 0 && l < 0)) {
        sat = true;
        break;
      }
    }
    bad += !sat;
  }
  return bad;
}

static std::vector<int8_t> unit_pins(const int32_t* lits, const int64_t* off, int32_t n, int32_t m) {
  std::vector<int8_t> u(n, 0);
  for (int32_t c = 0; c < m; c++)
    if (off[c + 1] - off[c] == 1) {
      const int32_t l = lits[off[c]];
      u[std::abs(l) - 1] = l > 0 ? 1 : -1;
    }
  return u;
}

dmm_status dmm_initial_state_reference(const int32_t* lits, const int64_t* clause_off, int32_t n,
                                       int32_t m, int32_t seed, int32_t replica, double* x,
                                       int32_t* alpha_div) {
  clear_error();
  bool k3;
  dmm_status st = validate_formula(lits, clause_off, n, m, &k3);
  if (st != DMM_OK) return st;
  if (!x || replica < 0) return DMM_ERR_ARG;
  const std::vector<int8_t> unit = unit_pins(lits, clause_off, n, m);
  const int64_t N = (int64_t)n + 2 * (int64_t)m;
  // dynex.cc:2635-2700: one mt19937 shared by the replicas in order.
  std::mt19937 gen(seed);
  std::uniform_int_distribution<int> rand_v(-1, 1);
  for (int32_t i = 0; i <= replica; i++) {
    if (i <= 2 && seed == 0) {
      const double val = (i == 0) ? 1.0 : (i == 1 ? 0.0 : -1.0);
      for (int64_t j = 0; j < N; j++) x[j] = val;
    } else {
      for (int32_t j = 0; j < n; j++) x[j] = (double)rand_v(gen);
      for (int64_t j = n; j < n + (int64_t)m; j++) x[j] = 0.0;
      for (int64_t j = n + (int64_t)m; j < N; j++) x[j] = 1.0;
    }
    if (seed == -1)
      for (int32_t j = 0; j < n; j++) x[j] = 0.0;
    if (seed == -2)
      for (int32_t j = 0; j < n; j++) x[j] = -1.0;
    for (int32_t j = 0; j < n; j++)
      if (unit[j] != 0) x[j] = unit[j];
  }
  if (alpha_div) *alpha_div = replica > 0 ? replica : 1;
  return DMM_OK;
}

dmm_status dmm_initial_state_uniform(const int32_t* lits, const int64_t* clause_off, int32_t n,
                                     int32_t m, uint64_t seed, double* x) {
  clear_error();
  bool k3;
  dmm_status st = validate_formula(lits, clause_off, n, m, &k3);
  if (st != DMM_OK) return st;
  if (!x) return DMM_ERR_ARG;
  const std::vector<int8_t> unit = unit_pins(lits, clause_off, n, m);
  Rng r(seed);
  for (int32_t j = 0; j < n; j++) x[j] = unit[j] != 0 ? unit[j] : 2.0 * r.uniform() - 1.0;
  for (int32_t j = 0; j < m; j++) x[n + j] = r.uniform();
  for (int32_t j = 0; j < m; j++) x[(int64_t)n + m + j] = 1.0;
  return DMM_OK;
}

}  // extern "C"
