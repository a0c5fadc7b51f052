// Host-side formula handling: DIMACS reader/writer, planted generator, strict-sign
// checker and initial states.
#include <algorithm>
#include <charconv>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

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

// ---- clause section of a DIMACS file, tokenized in chunks --------------------------------
//
// The clause section is cut at line starts into chunks that threads tokenize on their own:
// each turns its tokens into values (a `c` token skips the rest of its line, which never
// crosses a chunk) and stops at its first token that is not a literal, recording it.  The
// tokens of all chunks in order are the tokens the sequential reader sees, so one pass over
// them afterwards applies the clause rules in file order and stops after the m-th clause;
// a chunk's recorded error counts only if that pass reaches it.

inline bool is_ws(char c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f' || c == '\v';
}

struct CnfChunk {
  std::vector<int32_t> vals;  // literal values and 0 terminators, in file order
  int end = 0;                // what follows vals: 0 the chunk's end, 1 a token that is not
                              // an integer (bad_tok), 2 an integer beyond int32 (big)
  std::string bad_tok;
  int64_t big = 0;
};

// Tokenizes [p, e): integers as strtoll reads them (optional sign, decimal digits, the whole
// token; values beyond int64 saturate as strtoll's do), `c` tokens skip to the end of the
// line; a token that is not an integer, or an integer outside int32 (never a literal),
// ends the chunk.
static void tokenize_chunk(const char* p, const char* e, CnfChunk* out) {
  std::vector<int32_t>& v = out->vals;
  v.reserve((size_t)(e - p) / 6 + 16);
  while (p < e) {
    while (p < e && is_ws(*p)) p++;
    if (p >= e) break;
    const char* tb = p;
    while (p < e && !is_ws(*p)) p++;
    const char* te = p;
    if (te - tb == 1 && *tb == 'c') {
      while (p < e && *p != '\n') p++;
      continue;
    }
    const char* q = tb;
    bool neg = false;
    if (*q == '+' || *q == '-') neg = *q++ == '-';
    if (q == te) {
      out->end = 1;
      out->bad_tok.assign(tb, te);
      return;
    }
    uint64_t x = 0;
    bool sat = false;
    for (; q < te; q++) {
      const unsigned d = (unsigned)(*q - '0');
      if (d > 9) {
        out->end = 1;
        out->bad_tok.assign(tb, te);
        return;
      }
      if (x > (UINT64_MAX - d) / 10) sat = true;
      else x = 10 * x + d;
    }
    int64_t val;
    if (neg) val = (sat || x > (uint64_t)INT64_MAX + 1) ? INT64_MIN : (int64_t)(0 - x);
    else val = (sat || x > (uint64_t)INT64_MAX) ? INT64_MAX : (int64_t)x;
    if (val > INT32_MAX || val < -(int64_t)INT32_MAX) {
      out->end = 2;
      out->big = val;
      return;
    }
    v.push_back((int32_t)val);
  }
}

// Runs f(k) for k in [0, count) on up to `count` threads (this one included); the tasks
// whose thread cannot be started run on this thread.
template <class F>
static void parallel_for(int count, F f) {
  std::vector<std::thread> pool;
  int started = 1;
  try {
    for (; started < count; started++) pool.emplace_back(f, started);
  } catch (...) {
  }
  for (int k = started; k < count; k++) f(k);
  if (count > 0) f(0);
  for (auto& t : pool) t.join();
}

// Literal and clause counts of a chunk's values: zeros, non-zeros, and the non-zeros after
// its last zero (all of them when it has none).
struct ChunkCounts {
  int64_t zeros = 0, lits = 0, trailing = 0;
};
static ChunkCounts count_chunk(const std::vector<int32_t>& v) {
  ChunkCounts c;
  for (const int32_t x : v) {
    if (x == 0) {
      c.zeros++;
      c.trailing = 0;
    } else {
      c.lits++;
      c.trailing++;
    }
  }
  return c;
}

// A file's bytes: mapped read-only when possible, else read into memory.
struct FileBytes {
  const char* p = nullptr;
  size_t n = 0;
  void* map = nullptr;
  std::vector<char> buf;
  ~FileBytes() {
    if (map) munmap(map, n);
  }
  bool open(const char* path) {
    const int fd = ::open(path, O_RDONLY);
    if (fd < 0) return false;
    struct stat sb;
    if (fstat(fd, &sb) == 0 && S_ISREG(sb.st_mode) && sb.st_size > 0) {
      void* m = mmap(nullptr, (size_t)sb.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
      if (m != MAP_FAILED) {
        map = m;
        n = (size_t)sb.st_size;
        p = static_cast<const char*>(m);
        ::close(fd);
        return true;
      }
    }
    char tmp[1 << 16];
    for (;;) {
      const ssize_t r = ::read(fd, tmp, sizeof tmp);
      if (r < 0) {
        ::close(fd);
        return false;
      }
      if (r == 0) break;
      buf.insert(buf.end(), tmp, tmp + r);
    }
    ::close(fd);
    p = buf.data();
    n = buf.size();
    return true;
  }
};

// Largest occurrence count of a variable; `threads` > 1 counts slices of the literals in
// parallel with atomic increments (the counts, and so the result, do not depend on it).
static void occurrences(dmm_cnf* c, int threads = 1) {
  std::vector<int32_t> occ(c->n + 1, 0);
  if (threads <= 1 || c->nlits < (1 << 20)) {
    int32_t mx = 0;
    for (int64_t i = 0; i < c->nlits; i++) mx = std::max(mx, ++occ[std::abs(c->lits[i])]);
    c->max_occurrence = mx;
    return;
  }
  int32_t* o = occ.data();
  const int64_t per = (c->nlits + threads - 1) / threads;
  parallel_for(threads, [&](int k) {
    const int64_t lo = std::min(c->nlits, per * k), hi = std::min(c->nlits, lo + per);
    for (int64_t i = lo; i < hi; i++) __atomic_fetch_add(o + std::abs(c->lits[i]), 1, __ATOMIC_RELAXED);
  });
  c->max_occurrence = *std::max_element(occ.begin(), occ.end());
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
// (the reference would read empty clauses).  Whatever follows the m-th clause is not read.
// The clause section is tokenized and checked in chunks on several threads; the result,
// and the error reported (the first in file order), are those of reading it in sequence.
dmm_status dmm_cnf_read(const char* path, dmm_cnf** out) {
  clear_error();
  if (!path || !out) return DMM_ERR_ARG;
  FileBytes file;
  if (!file.open(path)) {
    set_error("cannot open %s", path);
    return DMM_ERR_IO;
  }
  const char* p = file.p;
  const char* e = p + file.n;
  auto token = [&](const char** b, const char** te) -> bool {
    while (p < e && is_ws(*p)) p++;
    if (p >= e) return false;
    *b = p;
    while (p < e && !is_ws(*p)) p++;
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
  // the clause section in chunks cut at line starts (one per MB at least, at most 32),
  // tokenized by one thread each
  const size_t rest = (size_t)(e - p);
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int nchunk =
      (int)std::min<size_t>({(size_t)std::min(hw, 32u), rest / (1u << 20) + 1});
  std::vector<const char*> cut(nchunk + 1);
  cut[0] = p;
  cut[nchunk] = e;
  for (int k = 1; k < nchunk; k++) {
    const char* q = std::max(cut[k - 1], p + rest / nchunk * k);
    while (q < e && *q != '\n') q++;
    cut[k] = q < e ? q + 1 : e;
  }
  std::vector<CnfChunk> chunks(nchunk);
  std::vector<ChunkCounts> cnt(nchunk);
  parallel_for(nchunk, [&](int k) {
    tokenize_chunk(cut[k], cut[k + 1], &chunks[k]);
    cnt[k] = count_chunk(chunks[k].vals);
  });
  // where each chunk starts: its first clause, its first literal, and the literals of the
  // clause open at its start (for the length rule); the chunk that holds the m-th clause end
  // and the values of it up to there
  std::vector<int64_t> c0(nchunk + 1, 0), l0(nchunk + 1, 0), open(nchunk + 1, 0);
  for (int k = 0; k < nchunk; k++) {
    c0[k + 1] = c0[k] + cnt[k].zeros;
    l0[k + 1] = l0[k] + cnt[k].lits;
    open[k + 1] = cnt[k].zeros > 0 ? cnt[k].trailing : open[k] + cnt[k].lits;
  }
  int last = nchunk - 1;  // the last chunk read
  size_t used_last = chunks[last].vals.size();
  for (int k = 0; k < nchunk; k++) {
    if (c0[k + 1] >= mm) {
      last = k;
      int64_t z = c0[k];
      size_t j = 0;
      const std::vector<int32_t>& v = chunks[k].vals;
      while (z < mm) z += v[j++] == 0;  // past the m-th clause's terminator
      used_last = j;
      break;
    }
  }
  // every chunk up to `last` checks the clause rules on its values and writes its literals
  // and clause ends in place; the first violation in file order is the one reported
  struct Fault {
    size_t at = SIZE_MAX;  // value index of the chunk
    int kind = 0;          // 1 literal out of range, 2 clause too long
    int64_t clause = 0;
    long long value = 0;
  };
  std::vector<Fault> fault(nchunk);
  const bool complete = c0[nchunk] >= mm;
  const int64_t nlits = complete ? l0[last] + [&] {
    int64_t c = 0;
    for (size_t j = 0; j < used_last; j++) c += chunks[last].vals[j] != 0;
    return c;
  }() : 0;
  // (a file that ends early is still checked: a violation before its end is reported as
  // such, as the sequential reading would)
  dmm_cnf* c = nullptr;
  if (complete) {
    dmm_status st = alloc_cnf((int32_t)nn, (int32_t)mm, nlits, &c);
    if (st != DMM_OK) return st;
    c->clause_off[0] = 0;
  }
  parallel_for(last + 1, [&](int k) {
    const std::vector<int32_t>& v = chunks[k].vals;
    const size_t nv = k == last ? used_last : v.size();
    int64_t cl = c0[k], li = l0[k], len = open[k];
    for (size_t j = 0; j < nv; j++) {
      const int32_t x = v[j];
      if (x == 0) {
        cl++;
        if (c) c->clause_off[cl] = li;
        len = 0;
        continue;
      }
      if (x > nn || x < -nn) {
        fault[k] = {j, 1, cl, (long long)x};
        return;
      }
      if (++len > DMM_MAX_CLAUSE_LITS) {
        fault[k] = {j, 2, cl, 0};
        return;
      }
      if (c) c->lits[li] = x;
      li++;
    }
  });
  // the first violation in file order: a clause rule, or the token that ended a chunk
  for (int k = 0; k <= last; k++) {
    const Fault& f = fault[k];
    if (f.kind == 1 || f.kind == 2) {
      dmm_cnf_free(c);
      if (f.kind == 1) {
        set_error("%s: literal %lld out of range in clause %lld", path, f.value,
                  (long long)f.clause);
        return DMM_ERR_LITERAL;
      }
      set_error("CLAUSE %lld HAS MORE THAN %d LITERALS.", (long long)f.clause,
                DMM_MAX_CLAUSE_LITS);
      return DMM_ERR_CLAUSE_LEN;
    }
    const bool ends_here = !(complete && k == last);  // the m-th clause ended before it
    if (ends_here && chunks[k].end == 1) {
      dmm_cnf_free(c);
      set_error("%s: bad literal `%s` in clause %lld", path, chunks[k].bad_tok.c_str(),
                (long long)c0[k + 1]);
      return DMM_ERR_PARSE;
    }
    if (ends_here && chunks[k].end == 2) {
      dmm_cnf_free(c);
      set_error("%s: literal %lld out of range in clause %lld", path, (long long)chunks[k].big,
                (long long)c0[k + 1]);
      return DMM_ERR_LITERAL;
    }
  }
  if (!complete) {
    set_error("%s: file ends after %lld of %lld clauses", path, (long long)c0[nchunk], mm);
    return DMM_ERR_PARSE;
  }
  occurrences(c, nchunk);
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
  // the text in blocks of about 1 MB: integers formatted with to_chars, one fwrite per block
  std::vector<char> buf(1 << 20);
  size_t used = 0;
  bool ok = true;
  auto flush = [&]() {
    if (used && std::fwrite(buf.data(), 1, used, f) != used) ok = false;
    used = 0;
  };
  auto put = [&](const char* s, size_t len) {
    if (used + len > buf.size()) flush();
    std::memcpy(buf.data() + used, s, len);
    used += len;
  };
  auto put_int = [&](long long v, char sep_before, char sep_after) {
    if (used + 24 > buf.size()) flush();
    char* q = buf.data() + used;
    if (sep_before) *q++ = sep_before;
    q = std::to_chars(q, q + 21, v).ptr;
    if (sep_after) *q++ = sep_after;
    used = (size_t)(q - buf.data());
  };
  if (planted) {
    put("c [", 3);
    for (int32_t i = 0; i < c->n; i++) put_int(planted[i] > 0 ? i + 1 : -(i + 1), ' ', 0);
    put(" ]\n", 3);
  }
  char head[64];
  const int hl = std::snprintf(head, sizeof head, "p cnf %d %d\n", c->n, c->m);
  put(head, (size_t)hl);
  for (int32_t i = 0; i < c->m; i++) {
    for (int64_t j = c->clause_off[i]; j < c->clause_off[i + 1]; j++) put_int(c->lits[j], 0, ' ');
    put("0\n", 2);
  }
  flush();
  ok = std::fclose(f) == 0 && ok;
  if (!ok) set_error("write error on %s", path);
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
