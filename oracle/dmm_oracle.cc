// CPU restatement of the reference DMM integrator hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity checker: tests, the golden-vector
// script and bench.py's CPU-baseline leg load it (oracle/_build/liboracle.so); the
// product never does.  It is pinned against the unmodified reference (oracle/_ref/,
// built from dynex.cc by oracle/Makefile) and against the reference CLI's known answers
// committed under tests/golden/.
//
// Two arithmetic modes:
//  * FP64 "reference" mode restates dynex.cc exactly: per-clause terms in double with
//    no FMA contraction, per-variable sums over the non-zero contributions sorted
//    ascending and accumulated left to right from +0.0 (dynex.cc:408-410, 527-530).
//  * FP32 "production" mode restates the CUDA FP32 path: the same formulas in float,
//    and each variable's contributions summed in a fixed canonical order: 32 strided
//    partial sums over the variable's clause slots in ascending slot order, combined
//    by a 5-round xor butterfly (offsets 16, 8, 4, 2, 1).  The adaptive step test uses
//    the exact double difference of the float values.
//
// Reference lines followed:
//   right-hand side          dynex.cc:362-530 (3-SAT 371-418, 2-SAT 420-454, k-SAT 457-494)
//   loc / energy             dynex.cc:497-499
//   dXs / dXl                dynex.cc:503, 506
//   Euler step + clamps      dynex.cc:301-327
//   adaptive controller      dynex.cc:1389-1417
//   solve + verification     dynex.cc:662-703, reported assignment 1420-1427
//   unit clauses             dynex.cc:2459-2469
//   initial state            dynex.cc:2635-2700
//   Xl bound                 dynex.cc:2358-2359
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <random>
#include <type_traits>
#include <vector>

namespace {

struct Formula {
  int n = 0, m = 0;
  std::vector<int32_t> lits;      // flat signed literals
  std::vector<int64_t> coff;      // m+1 clause offsets into lits
  std::vector<int8_t> unit;       // n: +1/-1 for unit-clause variables, else 0
  std::vector<int64_t> vptr;      // n+1: variable -> slot CSR offsets
  std::vector<int64_t> vslot;     // slots of each variable, ascending
  std::vector<double> alpha_cm;   // m
  double alpha = 2.5, beta = 20.0, gamma = 0.25, delta = 0.05, eps = 0.1, zeta = 0.1;
  double xl_max = 0.0;
  int precision = 1;              // 1 = FP64 reference mode, 0 = FP32 production mode
};

// dynex.cc:2358-2359: xl_max = xl_max * m in 32-bit int arithmetic; <= 0 means INT_MAX.
double effective_xl_max(int factor, int m) {
  int32_t v = (int32_t)((uint32_t)factor * (uint32_t)m);
  if (v <= 0) v = INT_MAX;
  return (double)v;
}

template <class T>
inline T clampv(T x, T lo, T hi) {
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}

// Canonical FP32 sum: 32 strided partials in slot order, then xor butterfly.
float tree32_sum(const float* vals, int64_t d) {
  float p[32];
  for (int l = 0; l < 32; l++) p[l] = 0.0f;
  for (int64_t j = 0; j < d; j++) p[j & 31] = p[j & 31] + vals[j];
  for (int off = 16; off >= 1; off >>= 1) {
    float q[32];
    for (int l = 0; l < 32; l++) q[l] = p[l] + p[l ^ off];
    for (int l = 0; l < 32; l++) p[l] = q[l];
  }
  return p[0];
}

// Right-hand side.  x: n+2m (T).  dxdt: n+2m (T).  Returns loc; energy via pointer.
template <class T>
int rhs(const Formula& F, const T* x, T* dxdt, double* energy, std::vector<T>& u) {
  const int n = F.n, m = F.m;
  const T one = T(1), half = T(0.5), two = T(2);
  const T xlmax = T(F.xl_max);
  const T zeta = T(F.zeta), beta = T(F.beta), gamma = T(F.gamma), delta = T(F.delta),
          eps = T(F.eps);
  u.assign(F.lits.size(), T(0));
  int loc = m;
  double e = 0.0;
  T av[64];
  for (int c = 0; c < m; c++) {
    const int64_t b = F.coff[c];
    const int k = (int)(F.coff[c + 1] - b);
    T Xs = clampv(x[n + c], T(0), one);
    T Xl = clampv(x[n + m + c], one, xlmax);
    T C;
    if (k == 1) {
      C = T(0);  // no branch of dynex.cc:371-494 runs for a unit clause
    } else if (k == 0) {
      C = T((double)INT_MAX) / two;  // dynex.cc:460-468 with an empty literal loop
    } else {
      // a_i = 1 - q_i v_i with v clamped on read (dynex.cc:377-383, 464-467)
      T cmin = T((double)INT_MAX);
      for (int j = 0; j < k; j++) {
        int l = F.lits[b + j];
        T q = l > 0 ? one : -one;
        T v = clampv(x[std::abs(l) - 1], -one, one);
        av[j] = one - q * v;
        if (av[j] < cmin) cmin = av[j];
      }
      C = cmin / two;
      const T xlxs = Xl * Xs;
      const T rfac = (one + zeta * Xl) * (one - Xs);
      for (int j = 0; j < k; j++) {
        int l = F.lits[b + j];
        T q = l > 0 ? one : -one;
        T v = clampv(x[std::abs(l) - 1], -one, one);
        T gmin = T((double)INT_MAX);
        for (int jj = 0; jj < k; jj++)
          if (jj != j && av[jj] < gmin) gmin = av[jj];
        T G = q * gmin / two;
        T R = (C == av[j] / two) ? (q - v) / two : T(0);
        u[b + j] = xlxs * G + rfac * R;
      }
    }
    e += (double)C;
    if (C < half) loc--;
    dxdt[n + c] = beta * (Xs + eps) * (C - gamma);
    dxdt[n + m + c] = T(F.alpha_cm[c]) * (C - delta);
  }
  // per-variable sums
  std::vector<T> tmp;
  for (int v = 0; v < n; v++) {
    const int64_t s0 = F.vptr[v], s1 = F.vptr[v + 1];
    tmp.clear();
    if constexpr (std::is_same<T, double>::value) {
      for (int64_t s = s0; s < s1; s++) {
        T val = u[F.vslot[s]];
        if (val != T(0)) tmp.push_back(val);
      }
      std::sort(tmp.begin(), tmp.end());
      T acc = T(0);
      for (T val : tmp) acc = acc + val;
      dxdt[v] = acc;
    } else {
      for (int64_t s = s0; s < s1; s++) tmp.push_back(u[F.vslot[s]]);
      dxdt[v] = tree32_sum(tmp.data(), (int64_t)tmp.size());
    }
  }
  if (energy) *energy = e;
  return loc;
}

// Euler step with unit pin and clamps, dynex.cc:301-327.
template <class T>
void dostep(const Formula& F, const T* x, const T* dxdt, double h, T* xo) {
  const int n = F.n, m = F.m;
  const T hh = T(h), one = T(1), xlmax = T(F.xl_max);
  for (int i = 0; i < n; i++) {
    T v = x[i] + hh * dxdt[i];
    if (F.unit[i] != 0) v = T(F.unit[i]);
    xo[i] = clampv(v, -one, one);
  }
  for (int i = n; i < n + m; i++) xo[i] = clampv(x[i] + hh * dxdt[i], T(0), one);
  for (int i = n + m; i < n + 2 * m; i++) xo[i] = clampv(x[i] + hh * dxdt[i], one, xlmax);
}

// Strict-sign clause check of dynex.cc:674-687 on raw V.  Returns #unsatisfied clauses.
template <class T>
int verify(const Formula& F, const T* x) {
  int bad = 0;
  for (int c = 0; c < F.m; c++) {
    bool sat = false;
    for (int64_t j = F.coff[c]; j < F.coff[c + 1]; j++) {
      int l = F.lits[j];
      T v = x[std::abs(l) - 1];
      if ((v > 0 && l > 0) || (v < 0 && l < 0)) { sat = true; break; }
    }
    if (!sat) bad++;
  }
  return bad;
}

struct RunResult {
  int steps;
  int solved;
  int solve_step;
  int pad;
  double t;
  double solve_t;
};

template <class T>
int run(const Formula& F, const double* x0, int max_steps, double* dump, int dump_every,
        int* loc_trace, double* energy_trace, signed char* pre, signed char* post,
        RunResult* res) {
  const int n = F.n;
  const size_t N = (size_t)F.n + 2 * (size_t)F.m;
  std::vector<T> x(N), dx(N), xt(N), u;
  for (size_t i = 0; i < N; i++) x[i] = T(x0[i]);
  if (dump && dump_every > 0)
    for (size_t i = 0; i < N; i++) dump[i] = (double)x[i];
  int steps = 0, solved = 0, solve_step = -1;
  double t = 0.0, solve_t = -1.0;
  while (!solved && steps < max_steps) {
    double energy = 0.0;
    int loc = rhs<T>(F, x.data(), dx.data(), &energy, u);
    if (loc_trace) loc_trace[steps] = loc;
    if (energy_trace) energy_trace[steps] = energy;
    if (loc == 0 && verify<T>(F, x.data()) == 0) {
      solved = 1;
      solve_step = steps;
      solve_t = t;
      if (pre)
        for (int i = 0; i < n; i++) pre[i] = x[i] > 0 ? 1 : (x[i] < 0 ? -1 : 0);
    }
    // adaptive controller, dynex.cc:1395-1412: trials at h = 1/8, 1/16, 1/32, 1/64;
    // when the last trial also fails, its state is kept and t advances by 1/128.
    double h = 0.125;
    for (;;) {
      dostep<T>(F, x.data(), dx.data(), h, xt.data());
      bool reject = false;
      for (int i = 0; i < n; i++)
        if (std::fabs((double)xt[i] - (double)x[i]) >= 1.0) { reject = true; break; }
      if (reject) h = h * 0.5;
      if (!reject || h <= 0.0078125) break;
    }
    x.swap(xt);
    steps++;
    t = t + h;
    if (dump && dump_every > 0 && steps % dump_every == 0)
      for (size_t i = 0; i < N; i++) dump[(size_t)(steps / dump_every) * N + i] = (double)x[i];
    if (solved && post)
      for (int i = 0; i < n; i++) post[i] = x[i] > 0 ? 1 : -1;
  }
  if (res) {
    res->steps = steps;
    res->solved = solved;
    res->solve_step = solve_step;
    res->pad = 0;
    res->t = t;
    res->solve_t = solve_t;
  }
  return 0;
}

}  // namespace

extern "C" {

// Creates an oracle for one formula.  params: alpha beta gamma delta epsilon zeta.
// alpha_cm: per-clause alpha (m) or NULL for all = alpha.  precision: 1 FP64, 0 FP32.
// Returns NULL for a literal out of range.
void* oracle_create(int n, int m, const int32_t* lits, const int64_t* clause_off,
                    const double* params, int xl_max_factor, const double* alpha_cm,
                    int precision) {
  Formula* F = new Formula();
  F->n = n;
  F->m = m;
  F->coff.assign(clause_off, clause_off + m + 1);
  F->lits.assign(lits, lits + clause_off[m]);
  F->unit.assign(n, 0);
  for (int32_t l : F->lits)
    if (l == 0 || l > n || l < -n) { delete F; return nullptr; }
  for (int c = 0; c < m; c++)
    if (F->coff[c + 1] - F->coff[c] == 1) {
      int l = F->lits[F->coff[c]];
      F->unit[std::abs(l) - 1] = l > 0 ? 1 : -1;
    }
  F->vptr.assign(n + 1, 0);
  for (int32_t l : F->lits) F->vptr[std::abs(l)]++;
  for (int v = 0; v < n; v++) F->vptr[v + 1] += F->vptr[v];
  F->vslot.assign(F->lits.size(), 0);
  std::vector<int64_t> fill(F->vptr.begin(), F->vptr.end() - 1);
  for (int64_t s = 0; s < (int64_t)F->lits.size(); s++)
    F->vslot[fill[std::abs(F->lits[s]) - 1]++] = s;
  F->alpha = params[0];
  F->beta = params[1];
  F->gamma = params[2];
  F->delta = params[3];
  F->eps = params[4];
  F->zeta = params[5];
  F->alpha_cm.assign(m, F->alpha);
  if (alpha_cm) F->alpha_cm.assign(alpha_cm, alpha_cm + m);
  F->xl_max = effective_xl_max(xl_max_factor, m);
  F->precision = precision;
  return F;
}

void oracle_destroy(void* h) { delete static_cast<Formula*>(h); }

double oracle_xl_max(void* h) { return static_cast<Formula*>(h)->xl_max; }

// dxdt of state x (both n+2m doubles; FP32 mode rounds x to float first).
int oracle_rhs(void* h, const double* x, double* dxdt, int* loc, double* energy) {
  const Formula& F = *static_cast<Formula*>(h);
  const size_t N = (size_t)F.n + 2 * (size_t)F.m;
  int l;
  if (F.precision == 1) {
    std::vector<double> u;
    l = rhs<double>(F, x, dxdt, energy, u);
  } else {
    std::vector<float> xf(N), df(N), u;
    for (size_t i = 0; i < N; i++) xf[i] = (float)x[i];
    l = rhs<float>(F, xf.data(), df.data(), energy, u);
    for (size_t i = 0; i < N; i++) dxdt[i] = df[i];
  }
  if (loc) *loc = l;
  return 0;
}

int oracle_dostep(void* h, const double* x, const double* dxdt, double step, double* xo) {
  const Formula& F = *static_cast<Formula*>(h);
  const size_t N = (size_t)F.n + 2 * (size_t)F.m;
  if (F.precision == 1) {
    dostep<double>(F, x, dxdt, step, xo);
  } else {
    std::vector<float> xf(N), df(N), of(N);
    for (size_t i = 0; i < N; i++) { xf[i] = (float)x[i]; df[i] = (float)dxdt[i]; }
    dostep<float>(F, xf.data(), df.data(), step, of.data());
    for (size_t i = 0; i < N; i++) xo[i] = of[i];
  }
  return 0;
}

int oracle_run(void* h, const double* x0, int max_steps, double* dump, int dump_every,
               int* loc_trace, double* energy_trace, signed char* pre, signed char* post,
               RunResult* res) {
  const Formula& F = *static_cast<Formula*>(h);
  if (F.precision == 1)
    return run<double>(F, x0, max_steps, dump, dump_every, loc_trace, energy_trace, pre, post,
                       res);
  return run<float>(F, x0, max_steps, dump, dump_every, loc_trace, energy_trace, pre, post,
                    res);
}

// Unsatisfied clauses of a +1/-1/0 assignment under strict signs (dynex.cc:674-687).
int oracle_check(void* h, const signed char* assign) {
  const Formula& F = *static_cast<Formula*>(h);
  std::vector<double> x(F.n);
  for (int i = 0; i < F.n; i++) x[i] = assign[i];
  return verify<double>(F, x.data());
}

// Initial state of replica `replica` for CLI seed `seed` (dynex.cc:2635-2700, default
// flags: no solution/assignment file).  Draws for all earlier replicas are replayed
// because the reference shares one generator across replicas.  x: n+2m doubles.
// Returns the replica's alpha divisor (1 for replica 0, else replica).
int oracle_init_state(void* h, int seed, int replica, double* x) {
  const Formula& F = *static_cast<Formula*>(h);
  const int n = F.n, m = F.m;
  const size_t N = (size_t)n + 2 * (size_t)m;
  std::mt19937 gen(seed);
  std::uniform_int_distribution<int> rand_v(-1, 1);
  for (int i = 0; i <= replica; i++) {
    if (i <= 2 && seed == 0) {
      double val = (i == 0) ? 1.0 : (i == 1 ? 0.0 : -1.0);
      for (size_t j = 0; j < N; j++) x[j] = val;
    } else {
      for (int j = 0; j < n; j++) x[j] = (double)rand_v(gen);
      for (int j = n; j < n + m; j++) x[j] = 0.0;
      for (int j = n + m; j < n + 2 * m; j++) x[j] = 1.0;
    }
    if (seed == -1)
      for (int j = 0; j < n; j++) x[j] = 0.0;
    if (seed == -2)
      for (int j = 0; j < n; j++) x[j] = -1.0;
    for (int j = 0; j < n; j++)
      if (F.unit[j] != 0) x[j] = F.unit[j];
  }
  return replica > 0 ? replica : 1;
}

}  // extern "C"
