// Per-step driver around the UNMODIFIED reference integrator (dynex.cc).
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile into oracle/_ref/libdynex_ref.so
// with the reference source included verbatim from its read-only location (the recipe
// passes its path as DYNEX_REF_SRC; nothing of it is copied into this repository).  The
// reference's own main() is renamed so that this file can set the reference's globals
// for one replica (node 0), inject an explicit initial state, and call the reference's
// own functions:
//   dmm_generate_dxdt  dynex.cc:332-720   (right-hand side, loc/energy, solve + verify)
//   dmm_dostep         dynex.cc:301-327   (Euler step, unit pin, clamps)
// The adaptive step-size loop that dmm() wraps around them (dynex.cc:1389-1417) is
// restated in ref_run() below, line for line in behaviour, because dmm() itself has no
// step cap and no per-step hook.  Only tests, the golden-vector script and bench.py's
// CPU-baseline leg load this library.
#include <fcntl.h>
#include <unistd.h>

#include <cstdint>
#include <cstdio>
#include <cstring>

#define main dynex_ref_main
#include DYNEX_REF_SRC
#undef main

#include "instance_gen.h"

namespace {

int g_ready = 0;
int g_n = 0, g_m = 0;

// Silences the reference's console output (it prints even in quiet mode,
// e.g. dynex.cc:636 and dynex.cc:664-703) while a harness call runs.
struct StdoutMute {
  int saved = -1;
  StdoutMute() {
    std::fflush(stdout);
    std::cout.flush();
    saved = dup(1);
    int dn = open("/dev/null", O_WRONLY);
    if (dn >= 0) {
      dup2(dn, 1);
      close(dn);
    }
  }
  ~StdoutMute() {
    std::fflush(stdout);
    std::cout.flush();
    if (saved >= 0) {
      dup2(saved, 1);
      close(saved);
    }
  }
};

void free_globals() {
  free(cls); cls = nullptr;
  free(clauseSizes); clauseSizes = nullptr;
  free(unit_clause_vars); unit_clause_vars = nullptr;
  free(v_best); v_best = nullptr;
  free(loc_thread); loc_thread = nullptr;
  free(energy_thread); energy_thread = nullptr;
  free(energy_thread_min); energy_thread_min = nullptr;
  free(global_thread); global_thread = nullptr;
  free(global_all_runs_thread); global_all_runs_thread = nullptr;
  free(time_thread); time_thread = nullptr;
  free(time_thread_actual); time_thread_actual = nullptr;
  free(walltime_thread); walltime_thread = nullptr;
  free(t_init); t_init = nullptr;
  free(t_begin_thread); t_begin_thread = nullptr;
  free(t_end_thread); t_end_thread = nullptr;
  free(stepcounter); stepcounter = nullptr;
  free(dmm_alpha_cm); dmm_alpha_cm = nullptr;
  g_ready = 0;
}

// Per-run resets mirroring dmm() (dynex.cc:1187-1202) for replica 0.
void reset_run_state() {
  solved = 0;
  global = m;
  global_energy = m;
  quiet = true;
  global_best_thread = 0;
  stepcounter[0] = 0;
  global_thread[0] = m;
  global_all_runs_thread[0] = m;
  time_thread[0] = 0.0;
  walltime_thread[0] = 0.0;
  energy_thread[0] = m;
  energy_thread_min[0] = m;
  t_init[0] = 0.0;
  t_begin_thread[0] = pt::microsec_clock::local_time().time_of_day().total_milliseconds();
}

}  // namespace

extern "C" {

// Loads one formula into the reference's globals (the part of main(), dynex.cc:2354-2469,
// that the integrator reads).  lits/clause_off: flat signed literals, clause i is
// lits[clause_off[i] .. clause_off[i+1]).  params: alpha beta gamma delta epsilon zeta.
// Returns 0, or -1 for a clause longer than MAX_LITS_SYSTEM (dynex.cc:2388) or a bad literal.
int ref_setup(int nv, int mc, const int* lits, const long long* clause_off, const double* params,
              int xl_max_factor) {
  if (g_ready) free_globals();
  n = nv;
  m = mc;
  g_n = nv;
  g_m = mc;
  THREAD_COUNT = 1;
  // dynex.cc:2358-2359 (int arithmetic, as the reference does it)
  xl_max = xl_max_factor;
  xl_max = xl_max * m;
  if (xl_max <= 0) xl_max = INT_MAX;
  cls = (int*)calloc((size_t)m * MAX_LITS_SYSTEM, sizeof(int));
  clauseSizes = (int*)calloc((size_t)m, sizeof(int));
  for (int i = 0; i < m; i++) {
    long long b = clause_off[i], e = clause_off[i + 1];
    if (e - b > MAX_LITS_SYSTEM) { free_globals(); return -1; }
    for (long long j = b; j < e; j++) {
      int l = lits[j];
      if (l == 0 || l > n || l < -n) { free_globals(); return -1; }
      cls[(size_t)i * MAX_LITS_SYSTEM + (j - b)] = l;
    }
    clauseSizes[i] = (int)(e - b);
  }
  v_best = (TFloat*)calloc((size_t)(n + m * 2), sizeof(TFloat));
  loc_thread = (int*)calloc(1, sizeof(int));
  unit_clause_vars = (int*)calloc((size_t)n + 1, sizeof(int));
  energy_thread = (TFloat*)calloc(1, sizeof(TFloat));
  energy_thread_min = (TFloat*)calloc(1, sizeof(TFloat));
  global_thread = (int*)calloc(1, sizeof(int));
  global_all_runs_thread = (int*)calloc(1, sizeof(int));
  time_thread = (TFloat*)calloc(1, sizeof(TFloat));
  time_thread_actual = (TFloat*)calloc(1, sizeof(TFloat));
  walltime_thread = (double*)calloc(1, sizeof(double));
  t_init = (TFloat*)calloc(1, sizeof(TFloat));
  t_begin_thread = (double*)calloc(1, sizeof(double));
  t_end_thread = (double*)calloc(1, sizeof(double));
  stepcounter = (int*)calloc(1, sizeof(int));
  dmm_alpha_cm = (TFloat*)calloc((size_t)m, sizeof(TFloat));
  // unit clauses, dynex.cc:2459-2469
  unit_clauses = false;
  for (int i = 0; i < m; i++) {
    if (clauseSizes[i] == 1) {
      unit_clauses = true;
      int lit = cls[(size_t)i * MAX_LITS_SYSTEM];
      if (lit > 0) unit_clause_vars[abs(lit)] = 1;
      if (lit < 0) unit_clause_vars[abs(lit)] = -1;
    }
  }
  dmm_alpha = params[0];
  dmm_beta = params[1];
  dmm_gamma = params[2];
  dmm_delta = params[3];
  dmm_epsilon = params[4];
  dmm_zeta = params[5];
  for (int i = 0; i < m; i++) dmm_alpha_cm[i] = dmm_alpha;  // dynex.cc:1200-1202
  walltime_timeout = INT_MAX;
  g_ready = 1;
  return 0;
}

void ref_teardown(void) {
  if (g_ready) free_globals();
}

// Effective Xl upper bound the reference uses after ref_setup.
double ref_xl_max(void) { return (double)xl_max; }

// One call of the reference right-hand side on state x (n+2m) at time t.
// Writes dxdt (n+2m), the unsatisfied-clause count and the energy.
int ref_rhs(const double* x, double t, double* dxdt, int* loc, double* energy) {
  if (!g_ready) return -1;
  StdoutMute mute;
  reset_run_state();
  std::snprintf(SOLUTION_FILE, sizeof(SOLUTION_FILE), "/dev/null");
  std::vector<TFloat> xv(x, x + (size_t)(n + 2 * m));
  std::vector<TFloat> d = dmm_generate_dxdt(0, xv, t);
  std::memcpy(dxdt, d.data(), sizeof(double) * (size_t)(n + 2 * m));
  if (loc) *loc = loc_thread[0];
  if (energy) *energy = energy_thread[0];
  solved = 0;
  return 0;
}

// One reference Euler step dmm_dostep(x, dxdt, h).
int ref_dostep(const double* x, const double* dxdt, double h, double* x_out) {
  if (!g_ready) return -1;
  std::vector<TFloat> xv(x, x + (size_t)(n + 2 * m));
  std::vector<TFloat> dv(dxdt, dxdt + (size_t)(n + 2 * m));
  std::vector<TFloat> r = dmm_dostep(0, xv, dv, h);
  std::memcpy(x_out, r.data(), sizeof(double) * (size_t)(n + 2 * m));
  return 0;
}

// Integrates from x0 with the reference functions and the adaptive controller of dmm()
// (dynex.cc:1387-1427) until the reference reports a verified solution or max_steps
// accepted steps were taken.
//   dump: if non-NULL, row r (n+2m doubles) receives x after r*dump_every accepted steps,
//         for r = 0 .. max_steps/dump_every (row 0 = x0).
//   loc_trace: if non-NULL, loc_trace[s] = loc of the right-hand side evaluated at step s.
//   out_pre:  sign of V when the solution was found (the printed list, dynex.cc:667-670):
//             +1, -1, or 0 for V == 0.
//   out_post: the reported assignment node->optimal after the final step (dynex.cc:1420-1427,
//             printed at dynex.cc:1506-1512): +1 or -1.
// Returns 0 on success.
struct RefResult {
  int steps;       // accepted steps (stepcounter) when the run ended
  int solved;      // 1 if the reference reported SAT (VERIFIED)
  int solve_step;  // stepcounter when the solving right-hand side ran, -1 if unsolved
  int pad;
  double t;        // simulated time when the run ended
  double solve_t;  // T printed with SOLUTION FOUND (dynex.cc:666), -1 if unsolved
};

int ref_run(const double* x0, int max_steps, double* dump, int dump_every, int* loc_trace,
            double* energy_trace, signed char* out_pre, signed char* out_post, RefResult* res) {
  if (!g_ready) return -1;
  StdoutMute mute;
  reset_run_state();
  std::snprintf(SOLUTION_FILE, sizeof(SOLUTION_FILE), "/dev/null");
  const size_t N = (size_t)(n + 2 * m);
  state_type x(x0, x0 + N);
  if (dump && dump_every > 0) std::memcpy(dump, x.data(), sizeof(double) * N);
  TFloat t = 0.0;
  TFloat h = 0.125;
  int solved_flag = 0, solve_step = -1;
  double solve_t = -1.0;
  while (solved != 1 && stepcounter[0] < max_steps) {
    int step_before = stepcounter[0];
    auto dxdt = dmm_generate_dxdt(0, x, t);
    if (loc_trace) loc_trace[step_before] = loc_thread[0];
    if (energy_trace) energy_trace[step_before] = energy_thread[0];
    if (solved == 1) {
      solve_step = step_before;
      solve_t = t;
      if (out_pre)
        for (int i = 0; i < n; i++) out_pre[i] = (x[i] > 0) ? 1 : ((x[i] < 0) ? -1 : 0);
    }
    bool adaptive_accepted = false;
    TFloat h_min = 0.0078125;
    h = 0.125;
    auto x_tmp = x;
    int varchanges2;
    while (!adaptive_accepted) {
      x_tmp = dmm_dostep(0, x, dxdt, h);
      varchanges2 = 0;
      for (int i = 0; i < n; i++) {
        if (fabs(x_tmp[i] - x[i]) >= 1) varchanges2++;
      }
      if (varchanges2 > 0) { h = h * 1 / 2; } else { adaptive_accepted = true; }
      stepcounter[0]--;
      if (h <= h_min) adaptive_accepted = true;
    }
    x = x_tmp;
    stepcounter[0]++;
    t = t + h;
    int s = stepcounter[0];
    if (dump && dump_every > 0 && s % dump_every == 0)
      std::memcpy(dump + (size_t)(s / dump_every) * N, x.data(), sizeof(double) * N);
    if (solved == 1) {
      solved_flag = 1;
      if (out_post)
        for (int i = 0; i < n; i++) out_post[i] = (x[i] > 0) ? 1 : -1;
    }
  }
  if (res) {
    res->steps = stepcounter[0];
    res->solved = solved_flag;
    res->solve_step = solve_step;
    res->pad = 0;
    res->t = t;
    res->solve_t = solve_t;
  }
  solved = 0;
  return 0;
}

// The seeded planted 3-SAT formula and uniform initial state of the library's generator
// (instance_gen.h), so that a process timing the reference builds its input without the
// library.  lits: 3m entries; clause_off: m + 1; sigma (optional): n planted signs;
// x: n + 2m.
int ref_generate_planted(int nv, int mc, double p0, double p1, unsigned long long seed,
                         int* lits, long long* clause_off, signed char* sigma) {
  if (nv < 3 || mc < 0 || p0 < 0 || p1 < 0 || p0 + p1 > 1.0 || !lits || !clause_off) return -1;
  oracle_gen::planted(nv, mc, p0, p1, seed, lits, reinterpret_cast<int64_t*>(clause_off),
                      reinterpret_cast<int8_t*>(sigma));
  return 0;
}

int ref_initial_state_uniform(const int* lits, const long long* clause_off, int nv, int mc,
                              unsigned long long seed, double* x) {
  if (!lits || !clause_off || !x || nv <= 0 || mc < 0) return -1;
  oracle_gen::uniform_state(lits, reinterpret_cast<const int64_t*>(clause_off), nv, mc, seed, x);
  return 0;
}

}  // extern "C"
