// dynex: drop-in command line of the reference solver (dynex.cc:2204-2296, report
// dynex.cc:1480-1533 and 662-703), running the integrator on the GPU through libdmm.
//
//   dynex -i file.cnf [-l seed] [-w replicas] [-u walltime] [-z maxsteps]
//         [-c alpha] [-b beta] [-n gamma] [-h delta] [-j epsilon] [-k zeta] [-m xl_max]
//         [-q 0|1] [-p 0|1] [-P fp64|fp32] [-D device] [-L 0|1] [-S 0|1]
//         [-t 1 [-s iterations] [-v switchfraction] [-g 0|1|2] [-x err1] [-y err2] [-d init_dt]]
//
// Defaults follow the reference (FP64 arithmetic, seed 0, one replica); with them the
// reported step count, T and assignment equal the reference's.  -P fp32 selects the
// production FP32 path.  Replicas (-w) start from the reference's per-replica initial
// states with alpha / i (dynex.cc:2643-2700) and run together in one batch; the replica
// that solves at the lowest step wins.  -p 1 runs the reference's alpha heuristic every
// 10^4 steps (with replicas, on each replica in turn).  Options of the reference that select modes outside the
// default integrator (-o, -t, -e, ...) are accepted and reported as unsupported when they
// ask for anything but the default.  -S 1 writes the final state of the reported replica
// to <cnf>.assignment.txt in the reference's checkpoint format (dynex.cc:2131-2135); -L 1
// starts every replica from that file, at its time t, as the reference's load_assignment
// does (dynex.cc:2521-2532, 2688-2692; a compile-time switch there).  -t 1 runs the
// reference's simulated-annealing parameter tuner with the replicas as its chains.
#include <getopt.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "dmm.h"

namespace {

struct Opts {
  std::string input;
  int seed = 0;
  int replicas = 1;
  double walltime = 0.0;
  int max_steps = 0;
  bool quiet = false;
  bool heuristics = false;
  dmm_precision prec = DMM_FP64;
  int device = 0;
  bool load_state = false;  // -L: start from <cnf>.assignment.txt
  bool save_state = false;  // -S: write the final state to <cnf>.assignment.txt
  dmm_params p{};
};

// V of unit-clause variables pinned to the clause's sign, the last unit clause of a
// variable winning (dynex.cc:2459-2469, applied to every initial state at :2694-2698).
void pin_units(const dmm_cnf* cnf, std::vector<double>& x) {
  for (int32_t c = 0; c < cnf->m; c++)
    if (cnf->clause_off[c + 1] - cnf->clause_off[c] == 1) {
      const int32_t l = cnf->lits[cnf->clause_off[c]];
      x[std::abs(l) - 1] = l > 0 ? 1.0 : -1.0;
    }
}

constexpr int kHeuristicEvery = 10000;  // dynex.cc:1430

struct HeuristicCounts {
  int up = 0, down = 0, max = 0;
  double median = 0.0;
};

// The reference's alpha heuristic (dynex.cc:1429-1457) on the state x after an accepted
// step: clause alpha x1.1 where Xl is above the "median", x0.9 at or below it, floored at
// the replica's alpha; a clause whose Xl reached xl_max gets the replica's alpha back and
// Xl = alpha.  The median is the reference's own: nth_element around m/2, then the element
// at index n, the variable count (dynex.cc:1108-1113).
HeuristicCounts alpha_heuristic(std::vector<double>& x, std::vector<double>& acm, int n, int m,
                                double alpha_replica, double alpha, double xl_max) {
  HeuristicCounts h;
  std::vector<double> v(x.begin() + n + m, x.begin() + n + 2 * (size_t)m);
  const size_t nq = v.size() / 2;
  std::nth_element(v.begin(), v.begin() + nq, v.end());
  h.median = v[std::min<size_t>((size_t)n, v.size() - 1)];  // the reference reads v[n]
  for (int i = 0; i < m; i++) {
    const double xl = x[(size_t)n + m + i];
    if (xl > h.median) {
      acm[i] *= 1.1;
      h.up++;
    }
    if (xl <= h.median) {
      acm[i] *= 0.9;
      h.down++;
    }
    if (acm[i] < alpha_replica) acm[i] = alpha_replica;
    if (x[(size_t)n + m + i] >= xl_max) {
      acm[i] = alpha_replica;
      x[(size_t)n + m + i] = alpha;
      h.max++;
    }
  }
  return h;
}

// xl_max after the reference's `xl_max *= m` in int arithmetic (dynex.cc:2358)
double effective_xl_max(int32_t factor, int32_t m) {
  int32_t v = (int32_t)((uint32_t)factor * (uint32_t)m);
  if (v <= 0) v = INT32_MAX;
  return (double)v;
}

void usage(const char* argv0) {
  std::printf("c Syntax: %s -i file.cnf [options]\n", argv0);
  std::printf(
      "c   -i file     input CNF (DIMACS)\n"
      "c   -l int      seed (0: replica 0 starts at 1.0; other seeds: V in {-1,0,1})\n"
      "c   -w int      replicas run together on the GPU (reference: threads)\n"
      "c   -u sec      wall-time limit\n"
      "c   -z int      accepted-step limit\n"
      "c   -c -b -n -h -j -k float   alpha beta gamma delta epsilon zeta\n"
      "c   -m int      Xl bound factor (bound = factor * m)\n"
      "c   -q 0|1      quiet\n"
      "c   -P fp64|fp32  arithmetic (default fp64, the reference's)\n"
      "c   -D int      CUDA device\n"
      "c   -L 0|1      start from <file>.assignment.txt (V, Xs, Xl and t)\n"
      "c   -S 0|1      write the final state to <file>.assignment.txt\n"
      "c   -t 1        tune the parameters (simulated annealing, one chain per replica):\n"
      "c               -s iterations, -v switchfraction, -g 0|1|2 params, -z steps per run\n");
}

bool fail(dmm_status st, const char* what) {
  if (st == DMM_OK) return false;
  std::fprintf(stderr, "c ERROR: %s: %s (%s)\n", what, dmm_status_string(st), dmm_last_error());
  return true;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ---- parameter tuner (-t 1) ---------------------------------------------------------------
// The reference's simulated-annealing tuner (dynex.cc:1575-2201) in its default form
// (tune_mode 0: every iteration starts the replicas from their original states, perturbed by
// `switchfraction`).  Replicas are Metropolis chains over the nine parameters (alpha .. zeta,
// the two Runge-Kutta tolerances and init_dt; the default integrator uses the first six);
// a chain's objective is the lowest loc its replica reaches in a run (dynex.cc:537, 640).
// Proposals, acceptance and the random-number use follow the reference step by step (one
// std::mt19937 seeded with -l, the same distributions drawn in the same order), so the
// parameter sequence depends only on the objectives.  Each iteration runs all replicas as one
// batch on the GPU, each to the step cap (-z) or its solution; the reference's threads also
// stop when any of them solves, a race that is not reproduced here.  The initial objective
// is the loc of each replica's initial state (the reference takes one Euler step through
// odeint, dynex.cc:1711-1716, whose one right-hand side sees that state).
struct TuneOpts {
  int iterations = INT_MAX;       // -s
  double switchfraction = 0.0001; // -v
  int params = 2;                 // -g: 0 alpha..zeta, 1 the integrator's, 2 all
  double err1 = 0.52, err2 = 0.10, init_dt = 0.15;  // -x -y -d (dynex.cc:151-153)
};

constexpr int kParams = 9;
enum { kLBH = 0, kHBH = 1, kLBS = 2, kHBS = 3 };  // dynex.cc:72-75

int run_tuner(const Opts& o, const TuneOpts& to, const dmm_cnf* cnf) {
  const int n = cnf->n, m = cnf->m, R = o.replicas;
  const int64_t N = (int64_t)n + 2 * (int64_t)m;
  // default (large) bounds, dynex.cc:1607-1634: {hard low, hard high, soft low, soft high}
  const double bounds[kParams][4] = {
      {1e-15, 100.0, 0.01, 1.0},  {1e-15, 100.0, 0.01, 1.0},  {1e-15, 0.5, 0.01, 0.25},
      {1e-15, 1.0, 0.01, 0.25},   {1e-15, 0.5, 0.01, 0.25},   {1e-15, 1.0, 0.01, 0.25},
      {1e-15, 1.0, 0.01, 1.0},    {1e-15, 1.0, 0.01, 1.0},    {1e-15, 1.0, 1e-15, 0.00001}};
  std::vector<double> par((size_t)R * kParams), rem_par((size_t)R * kParams);
  std::vector<double> rem_x((size_t)R * N), x0((size_t)R * N);
  for (int i = 0; i < R; i++) {
    int32_t div = 1;
    if (fail(dmm_initial_state_reference(cnf->lits, cnf->clause_off, n, m, o.seed, i,
                                         rem_x.data() + (size_t)i * N, &div), "initial state"))
      return EXIT_FAILURE;
    const double p[kParams] = {o.p.alpha / div, o.p.beta, o.p.gamma, o.p.delta, o.p.epsilon,
                               o.p.zeta, to.err1, to.err2, to.init_dt};
    std::copy(p, p + kParams, par.begin() + (size_t)i * kParams);
  }
  std::mt19937 gen(o.seed);  // dynex.cc:1684
  int p_low = 0, p_high = kParams - 1;
  if (to.params == 0) p_high = 5;
  if (to.params == 1) p_low = 6;
  std::uniform_int_distribution<int> rand_param(p_low, p_high);
  std::uniform_real_distribution<double> rand_r(0.0, 1.0);
  std::uniform_int_distribution<int> rand_switch(0, n - 1);
  std::uniform_int_distribution<int> rand_v(-1, 1);
  std::uniform_int_distribution<int> rand_mode(0, 2);
  std::vector<double> best(R), curr(R), cand(R), ssf(R, 100.0);
  std::vector<int> no_impr(R, 0), nchange(R, 0), best_loc(R, m), loc_zero(R, 0);
  std::vector<int> tune_p((size_t)R * kParams, -1), rem_tune_p((size_t)R * kParams, -1);
  // one batch run of every replica from x0 with its parameters: lowest loc of each
  auto evaluate = [&](int max_steps, double wall) -> bool {
    dmm_batch* b = nullptr;
    if (fail(dmm_batch_create(o.prec, o.device, R, (int64_t)n * R, (int64_t)m * R,
                              cnf->nlits * R, &b), "creating the batch"))
      return false;
    bool ok = true;
    for (int i = 0; i < R && ok; i++) {
      dmm_params p = o.p;
      const double* q = par.data() + (size_t)i * kParams;
      p.alpha = q[0]; p.beta = q[1]; p.gamma = q[2]; p.delta = q[3]; p.epsilon = q[4]; p.zeta = q[5];
      int32_t idx = 0;
      ok = !fail(dmm_batch_add(b, cnf->lits, cnf->clause_off, n, m, &p, x0.data() + (size_t)i * N,
                               max_steps, &idx), "adding a replica");
    }
    dmm_batch_stats st{};
    ok = ok && !fail(dmm_batch_run(b, wall, &st), "integration");
    for (int i = 0; i < R && ok; i++) {
      dmm_report rep{};
      ok = !fail(dmm_batch_result(b, i, &rep, nullptr), "result");
      best_loc[i] = rep.best_loc;
      loc_zero[i] = rep.status == DMM_SOLVED;
    }
    dmm_batch_destroy(b);
    return ok;
  };
  const bool q = o.quiet;
  if (!q) {
    std::printf("c [TUNE] MODE           : 0\n");
    std::printf("c [TUNE] N_ITERATIONS   : %d\n", to.iterations);
    std::printf("c [TUNE] SWITCHFRACTION : %.15f\n", to.switchfraction);
    std::printf("c [TUNE] INITIAL OBJECTIVE...\n");
  }
  // initial objective: loc of each replica's initial state (energy = loc when tuning)
  {
    dmm_instance* inst = nullptr;
    if (fail(dmm_instance_create(cnf->lits, cnf->clause_off, n, m, o.prec, o.device, &inst),
             "creating the instance"))
      return EXIT_FAILURE;
    std::vector<double> dx(N);
    for (int i = 0; i < R; i++) {
      int32_t loc = 0;
      double e = 0.0;
      if (fail(dmm_instance_rhs(inst, rem_x.data() + (size_t)i * N, dx.data(), &loc, &e), "rhs")) {
        dmm_instance_destroy(inst);
        return EXIT_FAILURE;
      }
      best[i] = curr[i] = std::min(loc, m);
    }
    dmm_instance_destroy(inst);
    if (!q) {  // the reference's line after its initial objective (dynex.cc:1717-1722)
      std::printf("c [TUNE] E: ");
      for (int i = 0; i < R; i++) std::printf("[%.2f]", best[i]);
      std::printf("\n");
    }
  }
  const std::string tuning_file = o.input + ".tuning.txt";
  if (FILE* f = std::fopen(tuning_file.c_str(), "w")) {  // dynex.cc:2719-2726
    std::fprintf(f, "ITERATION;INSTANCE;PARAM_01;PARAM_02;PARAM_03;PARAM_04;PARAM_05;PARAM_06;"
                    "PARAM_07;ENERGY\n");
    std::fclose(f);
  }
  double tune_global = m;
  int max_steps = o.max_steps;
  double wall = o.walltime;
  bool change_params = false, solved = false;
  int switch_count = 0;
  for (int iter = 0; iter < to.iterations && !solved; iter++) {
    std::printf("c [TUNE] ITERATION %d. GLOBAL=%g\n", iter, tune_global);
    int min_no_impr = INT_MAX;
    for (int i = 0; i < R; i++) {
      min_no_impr = std::min(min_no_impr, no_impr[i]);
      std::copy(par.begin() + (size_t)i * kParams, par.begin() + (size_t)(i + 1) * kParams,
                rem_par.begin() + (size_t)i * kParams);
      double* xi = x0.data() + (size_t)i * N;
      std::copy(rem_x.begin() + (size_t)i * N, rem_x.begin() + (size_t)(i + 1) * N, xi);
      if (iter > 0) {  // switchfraction (dynex.cc:1858-1866)
        switch_count = (int)std::abs(n * to.switchfraction);
        if (to.switchfraction > 0 && switch_count == 0) switch_count = 1;
        for (int j = 0; j < switch_count; j++) {
          const int v = rand_switch(gen);
          xi[v] = rand_v(gen);
        }
      }
    }
    if (min_no_impr >= 25) {  // dynex.cc:1870-1917 (tune_mode 0 part)
      wall *= 2;
      max_steps = max_steps > 0 ? (int)std::min<int64_t>(2 * (int64_t)max_steps, INT_MAX) : 0;
      if (!q) std::printf("c [TUNE] NOTHING IMPROVED SINCE 25 ITERATIONS. maxsteps TO %d\n", max_steps);
      std::fill(no_impr.begin(), no_impr.end(), 0);
      std::fill(ssf.begin(), ssf.end(), 100.0);
      change_params = false;
    }
    for (int i = 0; i < R; i++) {
      nchange[i] = 0;
      for (int k = 0; k < kParams; k++) rem_tune_p[(size_t)i * kParams + k] = -1;
    }
    if (change_params) {
      for (int i = 0; i < R; i++) {
        double* pi = par.data() + (size_t)i * kParams;
        if (no_impr[i] > 0 && no_impr[i] % 10 == 0) ssf[i] = std::min(ssf[i] * 10, 1e12);
        const int mode = rand_mode(gen);
        std::lognormal_distribution<double> rand_num(0.0, 0.5);
        int nc = (int)rand_num(gen);
        nc = std::max(1, std::min(nc, kParams));
        nchange[i] = nc;
        for (int k = 0; k < nc; k++) {
          int& tp = tune_p[(size_t)i * kParams + k];
          int& rtp = rem_tune_p[(size_t)i * kParams + k];
          tp = rtp == -1 ? rand_param(gen) : rtp;
          rtp = tp;
          const double* bd = bounds[tp];
          double c = pi[tp];
          if (mode == 0) {  // small move (dynex.cc:1972-1995)
            const double soft = bd[kHBS] - bd[kLBS];
            std::uniform_real_distribution<double> rand_p(0, soft);
            (void)rand_p(gen);  // drawn and overwritten in the reference
            std::uniform_real_distribution<double> rand_move(-1.5, 1.5);
            const double move = rand_move(gen);
            c = pi[tp] + pi[tp] * move / ssf[i];
            if (c <= 0.0) c = 1e-8;
          } else {  // a point within the soft (1) or hard (2) bounds (dynex.cc:1998-2058)
            const double lo = mode == 1 ? bd[kLBS] : bd[kLBH];
            const double hi = mode == 1 ? bd[kHBS] : bd[kHBH];
            std::uniform_real_distribution<double> rand_b(lo, hi);
            c = rand_b(gen);
            if (tp == 4 && c >= pi[2]) c = pi[2] - 0.1;
          }
          pi[tp] = c;
        }
        if (!q) {
          std::printf("c [TUNE] [%d] -c=%.15f -b=%.15f -n=%.15f -h=%.15f -j=%.15f -k=%.15f "
                      "-x=%.15f -y=%.15f -d=%.15f\n", i, pi[0], pi[1], pi[2], pi[3], pi[4], pi[5],
                      pi[6], pi[7], pi[8]);
        }
      }
    }
    change_params = true;
    if (!evaluate(max_steps, wall > 0 ? wall : 0.0)) return EXIT_FAILURE;
    for (int i = 0; i < R; i++) {
      cand[i] = best_loc[i];
      if (cand[i] < tune_global) {
        tune_global = cand[i];
        const double* pi = par.data() + (size_t)i * kParams;
        if (FILE* f = std::fopen(tuning_file.c_str(), "a")) {  // dynex.cc:2127-2129
          std::fprintf(f, "%d;%d;%.15f;%.15f;%.15f;%.15f;%.15f;%.15f;%.15f;%.15f\n", iter, i,
                       pi[0], pi[1], pi[2], pi[3], pi[4], pi[5], pi[8], tune_global);
          std::fclose(f);
        }
        if (!q) std::printf("c [TUNE] [%d] NEW GLOBAL %g\n", i, tune_global);
      }
    }
    for (int i = 0; i < R; i++) {  // Metropolis (dynex.cc:2149-2184)
      if (cand[i] < best[i]) {
        best[i] = cand[i];
        if (loc_zero[i] || best_loc[i] == 0) {
          solved = true;
          break;
        }
      }
      const double diff = cand[i] - curr[i] + 1.0;
      const double temp = 1.0 / double(iter + 1);
      const double metropolis = std::exp(-diff / temp);
      if (diff < 0 || rand_r(gen) < metropolis) {
        std::printf("c [TUNE] [%d] %d CANDIDATES ACCEPTED (E=%g, temp=%g)\n", i, nchange[i], cand[i],
                    temp);
        curr[i] = cand[i];
        no_impr[i] = 0;
      } else {
        for (int k = 0; k < nchange[i]; k++) {
          const int tp = tune_p[(size_t)i * kParams + k];
          par[(size_t)i * kParams + tp] = rem_par[(size_t)i * kParams + tp];
          rem_tune_p[(size_t)i * kParams + k] = -1;
        }
        std::printf("c [TUNE] [%d] CANDIDATE REJECTED (E=%g, temp=%g)\n", i, cand[i], temp);
        no_impr[i]++;
      }
    }
  }
  std::printf(solved ? "c [TUNE] SOLUTION FOUND.\nc [TUNE] FINISHED.\n" : "c [TUNE] FINISHED.\n");
  std::printf("%g", tune_global);
  std::fflush(stdout);
  return EXIT_SUCCESS;
}

}  // namespace

int main(int argc, char** argv) {
  Opts o;
  dmm_params_default(&o.p);
  TuneOpts to;
  bool tune = false;
  int c;
  while ((c = getopt(argc, argv, "i:l:w:u:z:c:b:n:h:j:k:m:q:P:D:L:S:o:t:p:e:f:g:r:v:x:y:d:a:s:")) != -1) {
    const char* a = optarg;
    if (a && a[0] == '=') a++;  // the reference accepts -x=value (dynex.cc:2208)
    switch (c) {
      case 'i': o.input = a; break;
      case 'l': o.seed = std::atoi(a); break;
      case 'w': o.replicas = std::atoi(a); break;
      case 'u': o.walltime = std::atof(a); break;
      case 'z': o.max_steps = std::atoi(a); break;
      case 'c': o.p.alpha = std::atof(a); break;
      case 'b': o.p.beta = std::atof(a); break;
      case 'n': o.p.gamma = std::atof(a); break;
      case 'h': o.p.delta = std::atof(a); break;
      case 'j': o.p.epsilon = std::atof(a); break;
      case 'k': o.p.zeta = std::atof(a); break;
      case 'm': o.p.xl_max = std::atoi(a); break;
      case 'q': o.quiet = std::atoi(a) != 0; break;
      case 'P': o.prec = std::strcmp(a, "fp32") == 0 ? DMM_FP32 : DMM_FP64; break;
      case 'D': o.device = std::atoi(a); break;
      case 'L': o.load_state = std::atoi(a) != 0; break;
      case 'S': o.save_state = std::atoi(a) != 0; break;
      case 'o':
        if (std::atoi(a) != 6) std::fprintf(stderr, "c -o %s: only the default integrator (6) is available\n", a);
        break;
      case 't': tune = std::atoi(a) != 0; break;
      case 's': to.iterations = (int)std::atof(a); break;
      case 'v': to.switchfraction = std::atof(a); break;
      case 'g': to.params = std::atoi(a); break;
      case 'x': to.err1 = std::atof(a); break;
      case 'y': to.err2 = std::atof(a); break;
      case 'd': to.init_dt = std::atof(a); break;
      case 'p': o.heuristics = std::atoi(a) != 0; break;
      default:
        break;  // other reference options only affect modes outside the default path
    }
  }
  if (o.input.empty() || o.replicas < 1) {
    usage(argv[0]);
    return EXIT_FAILURE;
  }
  dmm_cnf* cnf = nullptr;
  dmm_status st = dmm_cnf_read(o.input.c_str(), &cnf);
  if (st != DMM_OK) {
    if (st == DMM_ERR_CLAUSE_LEN) std::printf("c ERROR: %s\n", dmm_last_error());
    else fail(st, "reading the formula");
    return EXIT_FAILURE;
  }
  const int n = cnf->n, m = cnf->m;
  if (!o.quiet) {
    std::printf("c --------------------------------------------\n");
    std::printf("c DMM INTEGRATOR ON B200 (sm_100a)\n");
    std::printf("c --------------------------------------------\n");
    std::printf("c INSTANCE  : %s\n", o.input.c_str());
    std::printf("c VARIABLES : %d\n", n);
    std::printf("c CLAUSES   : %d\n", m);
    std::printf("c RATIO     : %lf\n", (double)m / n);
    std::printf("c MAX VARIABLE OCCURENCE: %d\n", cnf->max_occurrence);
    std::printf("c PRECISION : %s\n", o.prec == DMM_FP64 ? "FP64" : "FP32");
    std::printf("c REPLICAS  : %d\n", o.replicas);
    std::printf("c HEURISTICS: %d\n", o.heuristics ? 1 : 0);
    std::printf("c ALPHA %.15f BETA %.15f GAMMA %.15f DELTA %.15f EPSILON %.15f ZETA %.15f\n",
                o.p.alpha, o.p.beta, o.p.gamma, o.p.delta, o.p.epsilon, o.p.zeta);
    std::printf("c SEED      : %d\n", o.seed);
  }
  if (tune) {
    if (!o.quiet) std::printf("c [TUNE] TUNING CIRCUIT...\n");
    const int rc = run_tuner(o, to, cnf);
    dmm_cnf_free(cnf);
    return rc;
  }
  const int64_t N = (int64_t)n + 2 * (int64_t)m;
  std::vector<double> x(N);
  const std::string state_file = o.input + ".assignment.txt";
  // -L: the checkpoint replaces every replica's initial state; read as the reference's
  // loader reads it (each value through a float)
  std::vector<double> x_loaded;
  double t_loaded = 0.0;
  if (o.load_state) {
    x_loaded.resize(N);
    if (dmm_state_read(state_file.c_str(), n, m, 1, x_loaded.data(), &t_loaded) == DMM_OK) {
      pin_units(cnf, x_loaded);
      if (!o.quiet)
        std::printf("c ASSIGNMENT %s LOADED, WILL START AT t=%g\n", state_file.c_str(), t_loaded);
    } else {
      std::fprintf(stderr, "c -L: %s not loaded (%s)\n", state_file.c_str(), dmm_last_error());
      x_loaded.clear();
      t_loaded = 0.0;
    }
  }
  const double t0 = now_s();
  dmm_report rep{};
  std::vector<int8_t> pre(n), post(n);
  int winner = 0;
  bool solved = false;
  if (o.replicas == 1 || o.heuristics) {
    // One replica, or replicas with the alpha heuristic (which needs each replica's state
    // every 10^4 steps): every replica on its own instance, one after another.  A later
    // replica runs at most to the best solving step so far (only an earlier solve wins), and
    // each replica has the whole wall-time limit, as each of the reference's threads has.
    dmm_instance* keep = nullptr;
    auto drop = [&](dmm_instance* i) { dmm_instance_destroy(i); };
    for (int r = 0; r < o.replicas; r++) {
      if (solved && rep.solved_step <= 0) break;  // solved by an initial state: nothing is earlier
      dmm_instance* inst = nullptr;
      int32_t div = 1;
      dmm_params pr = o.p;
      const bool set_up =
          !fail(dmm_instance_create(cnf->lits, cnf->clause_off, n, m, o.prec, o.device, &inst),
                "creating the instance") &&
          !fail(dmm_initial_state_reference(cnf->lits, cnf->clause_off, n, m, o.seed, r, x.data(),
                                            &div), "initial state");
      pr.alpha = o.p.alpha / div;  // dynex.cc:2657
      if (!set_up || fail(dmm_instance_set_params(inst, &pr, nullptr), "parameters") ||
          fail(x_loaded.empty() ? dmm_instance_set_state(inst, x.data())
                                : dmm_instance_set_state_at(inst, x_loaded.data(), t_loaded, 0),
               "state")) {
        drop(inst);
        drop(keep);
        dmm_cnf_free(cnf);
        return EXIT_FAILURE;
      }
      int cap = o.max_steps;
      if (solved) cap = cap > 0 ? std::min(cap, rep.solved_step) : rep.solved_step;
      if (!o.quiet) std::printf("c [%d] STARTING ODE...\n", r);
      const double tr = now_s();
      dmm_report rr{};
      bool ok = true;
      if (!o.heuristics) {
        dmm_limits lim{cap, 0, o.walltime};
        ok = !fail(dmm_instance_solve(inst, &lim, &rr), "integration");
      } else {
        // integrate to every 10^4-th step, apply the heuristic to the state there, continue
        std::vector<double> acm((size_t)m, pr.alpha);  // dmm_alpha_cm (dynex.cc:1201)
        const double xl_max = effective_xl_max(o.p.xl_max, m);
        ok = !fail(dmm_instance_set_params(inst, &pr, acm.data()), "parameters");
        while (ok) {
          dmm_report cur{};
          ok = !fail(dmm_instance_report(inst, &cur), "report");
          int target = (cur.steps / kHeuristicEvery + 1) * kHeuristicEvery;
          if (cap > 0) target = std::min(target, cap);
          double wall = 0.0;
          if (o.walltime > 0) {
            wall = o.walltime - (now_s() - tr);
            if (wall <= 0) break;
          }
          dmm_limits lim{target, 0, wall};
          if (!ok || fail(dmm_instance_solve(inst, &lim, &rr), "integration")) {
            ok = false;
            break;
          }
          if (rr.status != DMM_STEP_LIMIT || rr.steps != target || (cap > 0 && rr.steps >= cap))
            break;  // solved, out of time, or at the step cap
          double t = 0.0;
          if (fail(dmm_instance_get_state(inst, x.data(), &t), "state")) {
            ok = false;
            break;
          }
          // floor: the replica's alpha; Xl reset: -c (dynex.cc:1446-1450)
          const HeuristicCounts hc = alpha_heuristic(x, acm, n, m, pr.alpha, o.p.alpha, xl_max);
          std::printf("c [%d] alpha heuristic changed %d up, %d down, %d max reached (median = %.2f)\n",
                      r, hc.up, hc.down, hc.max, hc.median);
          ok = !fail(dmm_instance_set_params(inst, &pr, acm.data()), "parameters") &&
               !fail(dmm_instance_set_state_at(inst, x.data(), t, rr.steps), "state");
        }
      }
      if (!ok) {
        drop(inst);
        drop(keep);
        dmm_cnf_free(cnf);
        return EXIT_FAILURE;
      }
      const bool won = rr.status == DMM_SOLVED && (!solved || rr.solved_step < rep.solved_step);
      if (r == 0 || won) {
        drop(keep);
        keep = inst;
        rep = rr;
        winner = r;
        solved = rr.status == DMM_SOLVED;
      } else {
        drop(inst);
      }
    }
    double t_end = 0.0;
    if (fail(dmm_instance_assignment(keep, solved ? pre.data() : nullptr, post.data()),
             "assignment") ||
        (o.save_state && (fail(dmm_instance_get_state(keep, x.data(), &t_end), "state") ||
                          fail(dmm_state_write(state_file.c_str(), x.data(), n, m, t_end),
                               "writing the state")))) {
      drop(keep);
      dmm_cnf_free(cnf);
      return EXIT_FAILURE;
    }
    drop(keep);
  } else {
    dmm_batch* b = nullptr;
    const int R = o.replicas;
    if (fail(dmm_batch_create(o.prec, o.device, R, (int64_t)n * R, (int64_t)m * R,
                              cnf->nlits * R, &b), "creating the batch")) {
      dmm_cnf_free(cnf);
      return EXIT_FAILURE;
    }
    for (int r = 0; r < R; r++) {
      int32_t div = 1, idx = 0;
      dmm_params pr = o.p;
      if (fail(dmm_initial_state_reference(cnf->lits, cnf->clause_off, n, m, o.seed, r, x.data(), &div),
               "initial state"))
        return EXIT_FAILURE;
      pr.alpha = o.p.alpha / div;  // dynex.cc:2657
      const double* xr = x_loaded.empty() ? x.data() : x_loaded.data();
      if (fail(dmm_batch_add(b, cnf->lits, cnf->clause_off, n, m, &pr, xr, o.max_steps, &idx),
               "adding a replica"))
        return EXIT_FAILURE;
      if (!x_loaded.empty() && t_loaded != 0.0 &&
          fail(dmm_batch_set_state_at(b, idx, xr, t_loaded, 0), "state"))
        return EXIT_FAILURE;
    }
    if (!o.quiet) std::printf("c [*] STARTING ODE ON %d REPLICAS...\n", R);
    dmm_batch_stats stats{};
    if (fail(dmm_batch_run_until(b, o.walltime, 1, &stats), "integration")) return EXIT_FAILURE;
    int best = -1;
    dmm_report rr{};
    for (int r = 0; r < R; r++) {
      dmm_batch_result(b, r, &rr, nullptr);
      if (rr.status == DMM_SOLVED && (best < 0 || rr.solved_step < rep.solved_step)) {
        best = r;
        rep = rr;
      }
    }
    if (best < 0) {
      dmm_batch_result(b, 0, &rep, nullptr);
      best = 0;
    }
    winner = best;
    solved = rep.status == DMM_SOLVED;
    dmm_batch_assignment(b, best, solved ? pre.data() : nullptr, post.data());
    double t_end = 0.0;
    if (o.save_state && (fail(dmm_batch_state(b, best, x.data(), &t_end), "state") ||
                         fail(dmm_state_write(state_file.c_str(), x.data(), n, m, t_end),
                              "writing the state")))
      return EXIT_FAILURE;
    dmm_batch_destroy(b);
  }
  const double spent = now_s() - t0;
  if (solved) {
    std::printf("\nc [%d] T=%.2f SOLUTION FOUND\n", winner, rep.solved_t);
    for (int i = 0; i < n; i++)
      if (pre[i] != 0) std::printf("%d ", pre[i] > 0 ? i + 1 : -(i + 1));
    std::printf("\nc [%d] VERIFYING...\n", winner);
    const int64_t bad = dmm_check_assignment(cnf->lits, cnf->clause_off, m, n, pre.data());
    if (bad == 0) {
      std::printf("c [%d] SAT (VERIFIED)\n", winner);
      const std::string sol = o.input + ".solution.txt";
      if (FILE* f = std::fopen(sol.c_str(), "w")) {
        for (int i = 0; i < n; i++) std::fprintf(f, "%d, ", pre[i] >= 0 ? i + 1 : -(i + 1));
        std::fclose(f);
      }
    } else {
      std::printf("c [%d] UNSAT (VERIFIED)\n", winner);
    }
  }
  if (!o.quiet) {
    std::printf("c [%d] TIME SPENT: %.5fs\n", winner, spent);
    std::printf("c [%d] STEPS = %d (T = %.5f)\n", winner, solved ? rep.solved_step : rep.steps,
                solved ? rep.solved_t : rep.t);
    std::printf("c [%d] BEST LOC = %d (GLOBAL %d) **\n", winner, rep.best_loc, rep.best_loc);
  }
  if (solved) {
    std::printf("\ns [%d] SATISFIABLE", winner);
    for (int i = 0; i < n; i++) {
      if (i % 20 == 0) std::printf("\nv ");
      std::printf("%i ", post[i] > 0 ? (i + 1) : -(i + 1));
    }
    std::printf("0\n");
  } else {
    std::printf("\ns [%d] UNKNOWN\n", winner);
  }
  std::printf("%d", solved ? 0 : rep.best_loc);
  std::fflush(stdout);
  dmm_cnf_free(cnf);
  return EXIT_SUCCESS;
}
