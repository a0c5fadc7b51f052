// dynex: drop-in command line of the reference solver (dynex.cc:2204-2296, report
// dynex.cc:1480-1533 and 662-703), running the integrator on the GPU through libdmm.
//
//   dynex -i file.cnf [-l seed] [-w replicas] [-u walltime] [-z maxsteps]
//         [-c alpha] [-b beta] [-n gamma] [-h delta] [-j epsilon] [-k zeta] [-m xl_max]
//         [-q 0|1] [-p 0|1] [-P fp64|fp32] [-D device] [-L 0|1] [-S 0|1]
//
// Defaults follow the reference (FP64 arithmetic, seed 0, one replica); with them the
// reported step count, T and assignment equal the reference's.  -P fp32 selects the
// production FP32 path.  Replicas (-w) start from the reference's per-replica initial
// states with alpha / i (dynex.cc:2643-2700) and run together in one batch; the replica
// that solves at the lowest step wins.  -p 1 runs the reference's alpha heuristic every
// 10^4 steps (one replica).  Options of the reference that select modes outside the
// default integrator (-o, -t, -e, ...) are accepted and reported as unsupported when they
// ask for anything but the default.  -S 1 writes the final state of the reported replica
// to <cnf>.assignment.txt in the reference's checkpoint format (dynex.cc:2131-2135); -L 1
// starts every replica from that file, at its time t, as the reference's load_assignment
// does (dynex.cc:2521-2532, 2688-2692; a compile-time switch there).
#include <getopt.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
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
      "c   -S 0|1      write the final state to <file>.assignment.txt\n");
}

bool fail(dmm_status st, const char* what) {
  if (st == DMM_OK) return false;
  std::fprintf(stderr, "c ERROR: %s: %s (%s)\n", what, dmm_status_string(st), dmm_last_error());
  return true;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

int main(int argc, char** argv) {
  Opts o;
  dmm_params_default(&o.p);
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
      case 't':
        if (std::atoi(a) != 0) std::fprintf(stderr, "c -t %s: tuning mode is not available\n", a);
        break;
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
  if (o.replicas == 1) {
    dmm_instance* inst = nullptr;
    int32_t div = 1;
    if (fail(dmm_instance_create(cnf->lits, cnf->clause_off, n, m, o.prec, o.device, &inst),
             "creating the instance") ||
        fail(dmm_initial_state_reference(cnf->lits, cnf->clause_off, n, m, o.seed, 0, x.data(), &div),
             "initial state") ||
        fail(dmm_instance_set_params(inst, &o.p, nullptr), "parameters") ||
        fail(x_loaded.empty() ? dmm_instance_set_state(inst, x.data())
                              : dmm_instance_set_state_at(inst, x_loaded.data(), t_loaded, 0),
             "state")) {
      dmm_instance_destroy(inst);
      dmm_cnf_free(cnf);
      return EXIT_FAILURE;
    }
    if (!o.quiet) std::printf("c [0] STARTING ODE...\n");
    bool ok = true;
    if (!o.heuristics) {
      dmm_limits lim{o.max_steps, 0, o.walltime};
      ok = !fail(dmm_instance_solve(inst, &lim, &rep), "integration");
    } else {
      // integrate to every 10^4-th step, apply the heuristic to the state there, continue
      std::vector<double> acm((size_t)m, o.p.alpha);  // dmm_alpha_cm (dynex.cc:1201)
      const double xl_max = effective_xl_max(o.p.xl_max, m);
      ok = !fail(dmm_instance_set_params(inst, &o.p, acm.data()), "parameters");
      while (ok) {
        dmm_report cur{};
        ok = !fail(dmm_instance_report(inst, &cur), "report");
        int target = (cur.steps / kHeuristicEvery + 1) * kHeuristicEvery;
        if (o.max_steps > 0) target = std::min(target, o.max_steps);
        double wall = 0.0;
        if (o.walltime > 0) {
          wall = o.walltime - (now_s() - t0);
          if (wall <= 0) break;
        }
        dmm_limits lim{target, 0, wall};
        if (!ok || fail(dmm_instance_solve(inst, &lim, &rep), "integration")) {
          ok = false;
          break;
        }
        if (rep.status != DMM_STEP_LIMIT || rep.steps != target ||
            (o.max_steps > 0 && rep.steps >= o.max_steps))
          break;  // solved, out of time, or at the step cap
        double t = 0.0;
        if (fail(dmm_instance_get_state(inst, x.data(), &t), "state")) {
          ok = false;
          break;
        }
        const HeuristicCounts hc = alpha_heuristic(x, acm, n, m, o.p.alpha, o.p.alpha, xl_max);
        std::printf("c [0] alpha heuristic changed %d up, %d down, %d max reached (median = %.2f)\n",
                    hc.up, hc.down, hc.max, hc.median);
        ok = !fail(dmm_instance_set_params(inst, &o.p, acm.data()), "parameters") &&
             !fail(dmm_instance_set_state_at(inst, x.data(), t, rep.steps), "state");
      }
    }
    if (!ok) {
      dmm_instance_destroy(inst);
      dmm_cnf_free(cnf);
      return EXIT_FAILURE;
    }
    solved = rep.status == DMM_SOLVED;
    double t_end = 0.0;
    if (fail(dmm_instance_assignment(inst, solved ? pre.data() : nullptr, post.data()),
             "assignment") ||
        (o.save_state && (fail(dmm_instance_get_state(inst, x.data(), &t_end), "state") ||
                          fail(dmm_state_write(state_file.c_str(), x.data(), n, m, t_end),
                               "writing the state")))) {
      dmm_instance_destroy(inst);
      dmm_cnf_free(cnf);
      return EXIT_FAILURE;
    }
    dmm_instance_destroy(inst);
  } else {
    dmm_batch* b = nullptr;
    const int R = o.replicas;
    if (o.heuristics)
      std::fprintf(stderr, "c -p: the alpha heuristic runs with one replica (-w 1) only\n");
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
