/*
 * dmm.h — C ABI of the B200-native digital-memcomputing (DMM) SAT integrator.
 *
 * The reference (dynex.cc) exposes no library interface: its surface is the CLI
 * `dynex -i file.cnf` (dynex.cc:2204-2296) and, inside the program, the function pair
 *   std::vector<TFloat> dmm_generate_dxdt(int node, std::vector<TFloat> x, TFloat t)  dynex.cc:332
 *   std::vector<TFloat> dmm_dostep(int node, std::vector<TFloat> x,
 *                                  std::vector<TFloat> dxdt, TFloat h)                dynex.cc:301
 * driven by the adaptive loop of dmm() (dynex.cc:1381-1459) over process globals filled by
 * the DIMACS loader (dynex.cc:2306-2469).  Each entry point below names the reference
 * interface it replaces.
 *
 * Conventions
 *  - Plain C types only.  Host buffers are owned by the caller; device buffers by the
 *    library.  Every call returns dmm_status; nothing exits, aborts or traps.
 *  - A state vector x has n + 2m doubles laid out as in the reference (dynex.cc:304-321):
 *    [ V_0..V_{n-1} | Xs_0..Xs_{m-1} | Xl_0..Xl_{m-1} ].
 *  - A formula is given as flat signed literals (DIMACS numbering, 1..n) plus m+1 clause
 *    offsets: clause i is lits[clause_off[i] .. clause_off[i+1]).
 *  - Handles are not thread-safe; distinct handles are independent.  Each handle owns one
 *    CUDA stream on its device.
 */
#ifndef DMM_H
#define DMM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DMM_ABI_VERSION 1
/* Longest clause accepted, as in the reference (MAX_LITS_SYSTEM, dynex.cc:69). */
#define DMM_MAX_CLAUSE_LITS 25

typedef enum dmm_status {
  DMM_OK = 0,
  DMM_ERR_ARG = 1,          /* invalid argument (null pointer, bad size, bad index)          */
  DMM_ERR_CUDA = 2,         /* a CUDA runtime call failed; see dmm_last_error()              */
  DMM_ERR_NOMEM = 3,        /* device or host allocation failed                             */
  DMM_ERR_NO_DEVICE = 4,    /* no usable CUDA device                                         */
  DMM_ERR_LITERAL = 5,      /* literal 0 inside a clause list or |literal| > n               */
  DMM_ERR_CLAUSE_LEN = 6,   /* clause longer than DMM_MAX_CLAUSE_LITS (dynex.cc:2388-2391)   */
  DMM_ERR_PARSE = 7,        /* malformed DIMACS                                              */
  DMM_ERR_IO = 8,           /* file could not be opened / written                            */
  DMM_ERR_BUDGET = 9,       /* request larger than the configured device-memory budget      */
  DMM_ERR_STATE = 10,       /* call not valid in the handle's current state                  */
  DMM_ERR_BUILD = 11        /* library built without the CUDA kernels for this device        */
} dmm_status;

typedef enum dmm_precision {
  DMM_FP32 = 0, /* production: state and right-hand side in FP32, step-size test, loc and
                   energy reductions in FP64 / integers                                      */
  DMM_FP64 = 1  /* parity: the reference's arithmetic (FP64, sorted per-variable sums)       */
} dmm_precision;

/* Run status of an integration (dmm_report.status). */
typedef enum dmm_run_status {
  DMM_RUNNING = 0,
  DMM_SOLVED = 1,      /* loc == 0 and the strict-sign check passed (dynex.cc:662-703)        */
  DMM_STEP_LIMIT = 2,  /* max_steps accepted steps taken without a solution                  */
  DMM_TIME_LIMIT = 3,  /* wall-clock limit (the reference's -u, dynex.cc:340-345)             */
  DMM_CANCELLED = 4
} dmm_run_status;

/* ODE parameters, defaults from dynex.cc:132-140 (dmm_params_default). */
typedef struct dmm_params {
  double alpha;    /* growth rate of Xl                (-c) */
  double beta;     /* growth rate of Xs                (-b) */
  double gamma;    /* Xs threshold on C_m              (-n) */
  double delta;    /* Xl threshold on C_m              (-h) */
  double epsilon;  /* Xs offset                        (-j) */
  double zeta;     /* rigidity weight                  (-k) */
  int32_t xl_max;  /* Xl bound factor (-m); bound = xl_max * m in 32-bit arithmetic,
                      INT_MAX when that is <= 0 (dynex.cc:2358-2359)                        */
  int32_t reserved;
} dmm_params;

/* Result and progress of an integration. */
typedef struct dmm_report {
  int32_t status;       /* dmm_run_status                                                    */
  int32_t steps;        /* accepted steps taken (the reference's stepcounter)                */
  double t;             /* simulated time after the last accepted step                      */
  int32_t loc;          /* unsatisfied clauses (C_m >= 1/2) at the last evaluated RHS        */
  int32_t best_loc;     /* lowest loc seen                                                   */
  double energy;        /* sum of C_m at the last evaluated RHS (FP64)                       */
  int32_t solved_step;  /* stepcounter printed with SOLUTION FOUND, -1 if unsolved            */
  int32_t reserved;
  double solved_t;      /* T printed with SOLUTION FOUND, -1 if unsolved                      */
  double wall_s;        /* wall time of the last solve/step call                             */
} dmm_report;

typedef struct dmm_limits {
  int32_t max_steps;    /* accepted-step cap (<= 0: no cap)                                  */
  int32_t reserved;
  double wall_s;        /* wall-clock cap in seconds (<= 0: no cap), checked between launches */
} dmm_limits;

/* Launch shape; 0 in a field selects the default.  Results never depend on it: per-variable
 * sums use a fixed canonical order for every var_group, and tiles never straddle instances. */
typedef struct dmm_tuning {
  int32_t clause_tile;      /* clauses per clause tile (multiple of 4, >= 256; 0: balanced
                               over the grid for one instance, else 4 x block size)          */
  int32_t var_group;        /* lanes per variable in the dV reduction: 1,2,4,8,16,32         */
  int32_t var_tile;         /* variables per variable tile (>= 32; 0: as clause_tile)         */
  int32_t steps_per_graph;  /* steps per launch: per cooperative launch, or per CUDA graph   */
  int32_t blocks_per_sm;    /* two-kernel form: persistent blocks per SM (0: occupancy)      */
  int32_t launch_mode;      /* 0: automatic (cooperative launches running steps_per_graph
                               steps with grid barriers between phases; one block per small
                               formula when there are enough of them); 1: one kernel per
                               phase, CUDA graphs; 2: cooperative only; 3: one block per
                               formula for every formula that fits                          */
  int32_t u_layout;         /* storage of the per-literal contributions: 0 default (slot-major
                               on the tile paths, variable-major in the one-block-per-formula
                               kernel), 1 slot-major (gathered through the CSR), 2 variable-
                               major (scattered through the slot positions)                  */
  int32_t l2_policy;        /* staged form with several tiles per block (launch form 6), two
                               bits: 0 default (tables and clause memories marked evict-first
                               in L2, the phase-A staging areas evict-last); bit 0 set: no
                               eviction hints; bit 1 set: one warp per block also prefetches
                               the block's next clause tile into L2 (measured slower: 71.5
                               vs 65.8 us per step at n = 300k)                             */
} dmm_tuning;

/* A DIMACS formula held in host memory (allocated by the library). */
typedef struct dmm_cnf {
  int32_t n;               /* variables                                                      */
  int32_t m;               /* clauses                                                        */
  int64_t nlits;           /* total literals                                                 */
  int32_t* lits;           /* nlits signed literals                                          */
  int64_t* clause_off;     /* m + 1 offsets                                                  */
  int32_t max_occurrence;  /* largest variable occurrence count (dynex.cc:2381-2383)         */
  int32_t reserved;
} dmm_cnf;

/* ---- library ------------------------------------------------------------------------ */
int32_t dmm_abi_version(void);
const char* dmm_status_string(dmm_status s);
/* Text of the last error raised on the calling thread ("" if none). */
const char* dmm_last_error(void);
void dmm_params_default(dmm_params* p);
/* Number of CUDA devices this library can use (0 when none). */
int32_t dmm_device_count(void);
/* No counterpart in the reference.  Instances and batches take their device buffers from a
 * process-wide cache: a destroyed instance's buffers are kept (up to 8 GiB per device) and
 * reused by the next instance of a similar size, so that creating and destroying instances
 * does not go through cudaMalloc/cudaFree (which synchronize the device).  This call returns
 * every cached block to the driver; live instances keep theirs. */
void dmm_release_cached_memory(void);

/* ---- formulas (host) ----------------------------------------------------------------- */
/* DIMACS loader: replaces the parser in main(), dynex.cc:2306-2392 (comment lines skipped,
 * `p cnf n m` header, 0-terminated clauses, at most DMM_MAX_CLAUSE_LITS literals each). */
dmm_status dmm_cnf_read(const char* path, dmm_cnf** out);
/* Builds a formula from caller arrays (validated, copied). */
dmm_status dmm_cnf_from_arrays(const int32_t* lits, const int64_t* clause_off, int32_t n,
                               int32_t m, dmm_cnf** out);
void dmm_cnf_free(dmm_cnf* cnf);
/* Writes DIMACS; planted (n signs, may be NULL) is written as a `c [ ... ]` first line
 * like the first line of the reference's fixture files. */
dmm_status dmm_cnf_write(const dmm_cnf* cnf, const char* path, const int8_t* planted);
/* Planted random k=3 SAT: a planted assignment is drawn from `seed`; each clause has 3
 * distinct variables; literal signs are drawn so that the number of literals agreeing with
 * the planted assignment is 3 with probability p0, 1 with probability p1, else 2.
 * planted (n entries of +1/-1) may be NULL.  Not in the reference (its instances come from
 * an external generator); used for the synthetic workloads. */
dmm_status dmm_cnf_generate_planted(int32_t n, int32_t m, double p0, double p1, uint64_t seed,
                                    dmm_cnf** out, int8_t* planted);
/* Strict-sign clause check (dynex.cc:674-687): number of clauses with no literal whose sign
 * matches assign[var] (+1 true, -1 false, 0 matches nothing).  -1 on bad arguments. */
int64_t dmm_check_assignment(const int32_t* lits, const int64_t* clause_off, int32_t m,
                             int32_t n, const int8_t* assign);
/* State checkpoint file in the reference's `<cnf>.assignment.txt` format (writer
 * dynex.cc:2131-2135): the n + 2m state values [V | Xs | Xl] each printed as "%.15f, ",
 * then the simulated time t as "%.15f ". */
dmm_status dmm_state_write(const char* path, const double* x, int32_t n, int32_t m, double t);
/* Reads that format (loader dynex.cc:2521-2532): n + 2m values, then t; values may be
 * separated by commas and white space, anything after t is ignored.  reference_rounding = 1
 * rounds every value to float, as the reference's loader does (it reads each one with "%f"
 * into a float); 0 keeps the printed decimals in double precision.  DMM_ERR_IO when the
 * file cannot be read, DMM_ERR_PARSE when it holds fewer than n + 2m + 1 numbers. */
dmm_status dmm_state_read(const char* path, int32_t n, int32_t m, int32_t reference_rounding,
                          double* x, double* t);
/* Initial state of replica `replica` for CLI seed `seed` (dynex.cc:2635-2700, default flags).
 * x: n + 2m doubles.  *alpha_div receives the replica's alpha divisor (dynex.cc:2657). */
dmm_status dmm_initial_state_reference(const int32_t* lits, const int64_t* clause_off,
                                       int32_t n, int32_t m, int32_t seed, int32_t replica,
                                       double* x, int32_t* alpha_div);
/* Initial state V ~ U[-1,1], Xs ~ U[0,1], Xl = 1 from a 64-bit seed (unit-clause variables
 * pinned).  Not in the reference; the synthetic workloads' initial state. */
dmm_status dmm_initial_state_uniform(const int32_t* lits, const int64_t* clause_off, int32_t n,
                                     int32_t m, uint64_t seed, double* x);

/* ---- one formula on one GPU (the plain path) ---------------------------------------- */
typedef struct dmm_instance dmm_instance;

/* Uploads the formula and builds the variable->clause-slot CSR on the device.
 * Replaces the loader globals of dynex.cc:2354-2469 and the occurrence table
 * (dynex.cc:2413-2422). */
dmm_status dmm_instance_create(const int32_t* lits, const int64_t* clause_off, int32_t n,
                               int32_t m, dmm_precision precision, int32_t device,
                               dmm_instance** out);
void dmm_instance_destroy(dmm_instance* inst);
/* Parameters (dynex.cc:132-140, CLI -c -b -n -h -j -k -m).  alpha_cm: per-clause alpha (m
 * doubles, dmm_alpha_cm of dynex.cc:133/1200) or NULL for alpha everywhere.  Applies from
 * the next step on. */
dmm_status dmm_instance_set_params(dmm_instance* inst, const dmm_params* p,
                                   const double* alpha_cm);
dmm_status dmm_instance_set_tuning(dmm_instance* inst, const dmm_tuning* t);
dmm_status dmm_instance_get_tuning(const dmm_instance* inst, dmm_tuning* t);
/* Sets the state x (n + 2m doubles) at t = 0, step 0 (the initial_assignments of
 * dynex.cc:1216). */
dmm_status dmm_instance_set_state(dmm_instance* inst, const double* x);
/* Sets the state x with the integration continuing at simulated time t after `step`
 * accepted steps, keeping the best unsatisfied count seen so far: the reference's
 * continuation after its alpha heuristic rewrites Xl in the running state
 * (dynex.cc:1429-1457), and its start from a loaded assignment at t_init
 * (dynex.cc:2515-2540). */
dmm_status dmm_instance_set_state_at(dmm_instance* inst, const double* x, double t,
                                     int32_t step);
/* Reads the current state (after the last accepted step) and simulated time. */
dmm_status dmm_instance_get_state(dmm_instance* inst, double* x, double* t);
/* Right-hand side of state x: replaces dmm_generate_dxdt (dynex.cc:332-720) without its
 * console side effects.  dxdt: n + 2m doubles; loc/energy may be NULL.  Like
 * dmm_instance_set_state, it leaves the instance at state x, t = 0, step 0. */
dmm_status dmm_instance_rhs(dmm_instance* inst, const double* x, double* dxdt, int32_t* loc,
                            double* energy);
/* One Euler step with unit pin and clamps: replaces dmm_dostep (dynex.cc:301-327).
 * Leaves the integration state unchanged. */
dmm_status dmm_instance_dostep(dmm_instance* inst, const double* x, const double* dxdt,
                               double h, double* x_out);
/* Advances up to nsteps accepted steps of the adaptive integrator (dynex.cc:1387-1417),
 * stopping early at a verified solution.  rep may be NULL. */
dmm_status dmm_instance_step(dmm_instance* inst, int32_t nsteps, dmm_report* rep);
/* Integrates until solved or a limit is hit: replaces dmm() (dynex.cc:1182-1474). */
dmm_status dmm_instance_solve(dmm_instance* inst, const dmm_limits* lim, dmm_report* rep);
dmm_status dmm_instance_report(dmm_instance* inst, dmm_report* rep);
/* Assignments after a solve (n entries each, may be NULL):
 *  pre:  sign of V when SOLUTION FOUND was detected (+1/-1, 0 for V == 0; the literal list
 *        of dynex.cc:667-670 and the solution file of dynex.cc:693-699),
 *  post: the reported assignment after the final step (+1/-1; `v` lines, dynex.cc:1506-1512). */
dmm_status dmm_instance_assignment(dmm_instance* inst, int8_t* pre, int8_t* post);
/* No counterpart in the reference.  The kernel that dmm_instance_step / _solve launch for
 * this instance with its current tuning:
 *   1  two kernels per step (clause tiles, then variable tiles), CUDA graphs
 *   2  one cooperative kernel for several steps, three grid barriers per step
 *   3  the same for a single formula (FP64, or FP32 without the staged tables): two grid
 *      barriers per step
 *   4  the staged single-formula kernel (FP32, 3-literal clauses, tables fit)
 *   6  the staged kernel with several clause and variable tiles per block (formulas whose
 *      tiles are too large for one of each per block)
 *   5  one block per formula
 * or a negative dmm_status. */
int32_t dmm_instance_launch_form(const dmm_instance* inst);
/* No counterpart in the reference.  Test hook for the failure path of the cooperative step
 * kernels: one launch whose first grid barrier waits for one arrival more than the grid has,
 * so every block's bounded wait runs out (a few seconds); returns the status the library
 * reports for it (DMM_ERR_CUDA, "grid barrier wait gave up ...").  The device context stays
 * usable; the instance's state is undefined afterwards (set a state before stepping). */
dmm_status dmm_instance_test_barrier_timeout(dmm_instance* inst);
/* Benchmark helper: runs nsteps steps as plain launches with CUDA events around each of
 * the two step kernels; before each step it writes flush_bytes of scratch (0: none) so
 * the step starts with a cold L2.  Returns the summed device times (ms). */
dmm_status dmm_instance_profile(dmm_instance* inst, int32_t nsteps, int64_t flush_bytes,
                                double* clause_ms, double* var_ms);
/* Benchmark helper: device time (ms) of nsteps steps launched as the solver launches them
 * (CUDA-graph chunks, state resident on the device), one event pair around all of them. */
dmm_status dmm_instance_time_steps(dmm_instance* inst, int32_t nsteps, double* ms);
/* Benchmark helper: nsteps steps, each launched on its own (one cooperative launch per
 * step, or the two phase kernels) after writing flush_bytes of scratch so that it starts
 * with a cold L2; returns the summed device time of the steps (ms, flushes excluded). */
dmm_status dmm_instance_time_steps_flushed(dmm_instance* inst, int32_t nsteps,
                                           int64_t flush_bytes, double* ms);
/* Benchmark helper: one cooperative launch of nsteps steps with a device timer read by
 * every block at 10 points of each step (start, clause tile loaded, voltages gathered,
 * phase A done, past grid barrier 1, variable tile loaded, contributions gathered, phase B
 * done, past barrier 2, step decision done).  out[23]: out[2k], out[2k+1] = mean and max
 * over blocks of the microseconds from point k to point k+1 (point 10: the next step's
 * start), averaged over steps; out[20] = the SM clock (MHz) over the traced steps;
 * out[21], out[22] = mean microseconds from kernel entry to the first step (launch set-up)
 * and from the last step's end to kernel exit (staged kernel; 0 for the others).
 * DMM_ERR_STATE on the two-kernel launch form. */
dmm_status dmm_instance_trace_phases(dmm_instance* inst, int32_t nsteps, double* out);

/* ---- right-hand side without device allocation ----------------------------------------- */
/* No counterpart in the reference.  For callers that may not allocate device memory (a
 * host framework whose caching allocator owns the GPU, a plug-in limited to the buffers it
 * is given): the FP32 right-hand side of a formula whose clauses all have three literals,
 * from DEVICE buffers the caller owns:
 *   lits  3m signed literals,  x  n + 2m floats (V | Xs | Xl),
 *   dxdt  n + 2m floats out,   loc  one int32 out (clauses with C_m >= 1/2),
 *   p     host parameters (NULL: defaults; the scalar alpha, no per-clause alpha),
 *   stream  a cudaStream_t (NULL: default stream).
 * Intermediates live in one fixed __device__ array (about 2.1 MB per GPU, held until the
 * process exits), so n <= 32768, m <= 65536 and at most 1024 literal slots per variable;
 * larger formulas are rejected with DMM_ERR_ARG, literals outside [-n, n] or zero with
 * DMM_ERR_LITERAL.  These checks run on the device and the call waits for the stream twice
 * to read their counters, so it blocks the calling thread; the right-hand side is then
 * queued on the stream.  The first call on a device looks up the array's address.  Calls
 * share the array: calls that overlap on the GPU race and must be serialized by the
 * caller.  Results equal dmm_instance_rhs on an FP32 instance. */
dmm_status dmm_rhs3_f32_noalloc(const int32_t* lits, int32_t n, int32_t m, const float* x,
                                const dmm_params* p, float* dxdt, int32_t* loc, void* stream);

/* ---- many formulas in one launch (batched path) -------------------------------------- */
typedef struct dmm_batch dmm_batch;

typedef struct dmm_batch_stats {
  int64_t clause_updates;  /* sum over instances of m_i x accepted steps                     */
  int64_t steps_launched;  /* graph steps launched                                           */
  int32_t solved;          /* instances solved                                               */
  int32_t unsolved;        /* instances stopped by a limit                                   */
  double wall_s;           /* wall time of the run                                           */
  double device_ms;        /* device time of the run (CUDA events)                           */
} dmm_batch_stats;

/* Capacities bound the device arrays allocated once at creation. */
dmm_status dmm_batch_create(dmm_precision precision, int32_t device, int32_t max_instances,
                            int64_t max_vars, int64_t max_clauses, int64_t max_lits,
                            dmm_batch** out);
void dmm_batch_destroy(dmm_batch* b);
dmm_status dmm_batch_set_tuning(dmm_batch* b, const dmm_tuning* t);
/* Adds one formula with its parameters (NULL: defaults) and initial state x0 (n + 2m
 * doubles).  max_steps <= 0: no cap.  *index receives the instance index. */
dmm_status dmm_batch_add(dmm_batch* b, const int32_t* lits, const int64_t* clause_off,
                         int32_t n, int32_t m, const dmm_params* p, const double* x0,
                         int32_t max_steps, int32_t* index);
/* Integrates every instance until each is solved or hits its limit (or wall_s passes). */
dmm_status dmm_batch_run(dmm_batch* b, double wall_s, dmm_batch_stats* stats);
/* Like dmm_batch_run, but returns once at least stop_after instances have finished
 * (solved or at their step cap) during this call; instances still running are stopped
 * with DMM_CANCELLED.  Replaces the reference's replica race (`-w`, dynex.cc:2738-2801:
 * the first replica to solve ends the run). */
dmm_status dmm_batch_run_until(dmm_batch* b, double wall_s, int32_t stop_after,
                               dmm_batch_stats* stats);
dmm_status dmm_batch_result(dmm_batch* b, int32_t index, dmm_report* rep, int8_t* post);
/* Assignments of one instance, as dmm_instance_assignment. */
dmm_status dmm_batch_assignment(dmm_batch* b, int32_t index, int8_t* pre, int8_t* post);
/* State of instance `index` in the reference layout [V | Xs | Xl] and its time t. */
dmm_status dmm_batch_state(dmm_batch* b, int32_t index, double* x, double* t);
/* Restarts instance `index` from state x at simulated time t after `step` accepted steps,
 * as dmm_instance_set_state_at: a replica resumed from a checkpoint file starts at the
 * file's t (the reference's t_init, dynex.cc:2531, 1229). */
dmm_status dmm_batch_set_state_at(dmm_batch* b, int32_t index, const double* x, double t,
                                  int32_t step);

/* ---- continuous-batching server ------------------------------------------------------- */
typedef struct dmm_server dmm_server;

typedef struct dmm_server_config {
  int32_t precision;        /* dmm_precision                                                 */
  int32_t device;
  int64_t budget_bytes;     /* device-memory budget for resident instances, reserved at
                               creation (DMM_ERR_BUDGET when it exceeds the device's free
                               memory less 1 GiB)                                            */
  int32_t max_slots;        /* most instances resident at once                               */
  int32_t steps_per_launch; /* steps between admission/retire points                         */
} dmm_server_config;

typedef struct dmm_server_result {
  int64_t ticket;
  dmm_report report;
  double submit_s;          /* times on the server's monotonic clock                         */
  double admit_s;
  double finish_s;
} dmm_server_result;

dmm_status dmm_server_create(const dmm_server_config* cfg, dmm_server** out);
void dmm_server_destroy(dmm_server* s);
/* Queues a request (the formula is copied).  x0: n + 2m doubles or NULL for the uniform
 * initial state from init_seed.  *ticket identifies the result. */
dmm_status dmm_server_submit(dmm_server* s, const int32_t* lits, const int64_t* clause_off,
                             int32_t n, int32_t m, const dmm_params* p, const double* x0,
                             uint64_t init_seed, int32_t max_steps, int64_t* ticket);
/* One scheduling round: admits queued requests that fit, launches steps_per_launch steps
 * for every resident instance, retires finished ones and frees their slots. */
dmm_status dmm_server_pump(dmm_server* s, int32_t* resident, int32_t* queued);
/* Moves up to cap finished results out; *count receives how many. */
dmm_status dmm_server_take(dmm_server* s, dmm_server_result* out, int32_t cap, int32_t* count);
/* Reported assignment of a finished ticket (n entries, +1/-1).  Each ticket's assignment
 * can be read once; reading it releases it. */
dmm_status dmm_server_assignment(dmm_server* s, int64_t ticket, int8_t* post, int32_t n);
double dmm_server_clock(dmm_server* s);

#ifdef __cplusplus
}
#endif

#endif /* DMM_H */
