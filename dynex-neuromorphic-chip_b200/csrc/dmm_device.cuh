// Device-side data layout and arithmetic of the DMM integrator (sm_100a).
//
// A *pack* holds one or many formulas in shared device arrays.  Every formula (an
// "instance") owns a contiguous range in three index spaces:
//   variables [var0, var0+n)   : candidate voltages, unit pins, CSR ends
//   clauses   [cls0, cls0+m)   : Xs, Xl, C of the last right-hand side, per-clause alpha
//   slots     [slot0, slot0+L) : one per literal occurrence: literal, contribution u,
//                                and (in variable order) the CSR list of slots
// The work of one step is cut into clause tiles and variable tiles that never straddle
// instances, so an instance's arithmetic is identical alone or packed with others.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace dmm {

constexpr int kMaxK = 25;          // longest clause (MAX_LITS_SYSTEM, dynex.cc:69)
constexpr int kThreads = 256;      // block size of every tile kernel (fixed: reductions
                                   // over a block are part of the result definition)
constexpr int kTrials = 4;         // adaptive trials h = 1/8, 1/16, 1/32, 1/64
constexpr int kTraceK = 10;        // trace points per step of the cooperative kernel

// Read-only description of one instance.
struct InstDesc {
  int32_t n, m;
  int64_t var0, cls0, slot0;
  int32_t nslots;
  int32_t k3;            // every clause has exactly 3 literals: slot of clause c is 3c
  int32_t has_alpha_cm;  // per-clause alpha array present
  int32_t max_steps;     // accepted-step cap, <= 0: none
  int32_t ctile0, nctile, vtile0, nvtile;
  double alpha, beta, gamma, delta, eps, zeta, xl_max;
};

// Mutable integration state of one instance (written by the finalize step).
struct InstCtrl {
  int32_t done;         // dmm_run_status; 0 while running
  int32_t step;         // accepted steps (reference stepcounter)
  int32_t set;          // candidate set holding V(step)
  int32_t kcur;         // trial slot of V(step) in that set
  int32_t pending;      // Xs/Xl Euler update of the previous step not yet applied
  int32_t loc;          // loc of the last right-hand side
  int32_t best_loc;
  int32_t solved_step;  // step at which the solving right-hand side ran, -1
  int32_t sol_set, sol_k;
  int32_t vfail;        // strict-sign failures of the last right-hand side
  int32_t pad0;
  double t;             // simulated time
  double h_state;       // h of the pending Xs/Xl update
  double energy;        // energy of the last right-hand side
  double solved_t;
  double best_t;
  // per-step accumulators, zeroed by the finalize step
  int32_t acc_loc, acc_vfail, acc_kmax, vtiles_done;
};

// Accumulators of one step of a single formula on the cooperative form (two per formula,
// alternating by step): every block reads them after the step's last grid barrier.
struct StepAcc {
  int32_t loc, vfail, kmax, pad;
  unsigned long long energy;  // FP32 energy in units of 2^-25 (exact)
  unsigned long long arrive;  // grid-barrier arrivals carrying trial indices (staged form)
};

struct Tile {
  int32_t inst;
  int32_t begin;  // local clause / variable index
  int32_t count;
  int32_t pad;
};

template <class T>
struct PackView {
  T* Xs;
  T* Xl;
  T* Cp;                    // C_m of the last right-hand side (for the deferred update)
  const T* alpha_cm;        // per-clause alpha (may be null)
  const int32_t* coff;      // general layout: local slot offset of each clause
  const int32_t* lit;       // local signed literal of each slot (1-based variable)
  T* u;                     // contribution of each slot
  const int32_t* vslot;     // variable-ordered slot list (local slot indices)
  const int32_t* vend;      // inclusive end of each variable's slot list (local)
  T* cand;                  // candidates: cand[(set*4 + k) * var_cap + v]
  int64_t var_cap;
  const int8_t* unit;       // +1/-1 pin of unit-clause variables, else 0
  double* epart;            // energy partial of each clause tile
  const InstDesc* inst;
  InstCtrl* ctrl;
  const Tile* ctiles;
  const Tile* vtiles;
  const int32_t* ntiles;    // [0] clause tiles, [1] variable tiles
  int32_t* queue;           // [0] clause-tile counter, [1] variable-tile counter
  int32_t* active;          // instances still running
  int32_t* ring;            // finished instances (ring buffer)
  int32_t* ring_tail;
  int32_t ring_cap;
  const int32_t* live;      // indices of the instances with tiles
  int32_t live0;            // live[0] when the host knows it (single-formula forms), else -1
  const int32_t* nlive;
  const int32_t* upos;      // variable-major position of each slot (null: u is slot-major)
  StepAcc* acc2;            // [2] step accumulators of the single-formula cooperative form
  // staged form (FP32, one formula of 3-literal clauses, cooperative launch, one clause
  // tile and one variable tile per block; xdlist null when off).  Clause tile t gathers
  // the voltages of its distinct variables (ascending; xdlist from xdoff[2t], xdoff[2t+1]
  // entries, 16-byte aligned) into shared memory, reads
  // them through the tile-local literals xllit (+-(1 + position in the list)), stages each
  // contribution at xspos in a shared area grouped by destination variable tile (chunks
  // padded to 8 entries) and writes the area to ux[xubase[t] ..).  Variable tile b reads
  // bucket positions [xboff[b], xboff[b + 1]) (ux index of every 8 positions in xsrc8)
  // and scatters them to their variable-major positions xdst in shared memory.
  const int32_t* xdlist;
  const int32_t* xdoff;     // [2 * clause tiles]: start, count
  const int16_t* xllit;     // per slot of the formula
  const uint16_t* xspos;    // per slot of the formula
  T* ux;
  const int32_t* xubase;    // [clause tiles + 1], multiples of 8
  const int32_t* xboff;     // [variable tiles + 1], multiples of 8
  const int32_t* xsrc8;     // per 8 bucket positions
  const uint16_t* xdst;     // per bucket position; 0xFFFF for padding
  int32_t xsv_cap, xbk_cap, xtv_cap;  // shared-memory capacities (entries)
  int32_t xst_cap;          // staging-area capacity of the several-tiles-per-block form
  int32_t xl2_plain;        // that form without L2 eviction hints
  int32_t xprefetch;        // that form prefetching each block's next clause tile into L2 (off
                            // by default: measured slower)
  // phase trace of the cooperative kernel (null when off): trace[(s * kTraceK + k) * grid +
  // block] = %globaltimer at step s's point k: 0 start, 1 clause tile loaded, 2 voltages
  // gathered, 3 phase A done, 4 past barrier 1, 5 variable tile loaded, 6 bucket filled,
  // 7 phase B done, 8 past barrier 2, 9 phase F done; followed by the same layout of SM
  // clock counts
  long long* trace;
  int32_t trace_steps;
  // test hook: arrivals the first grid barrier of a launch waits for beyond the grid (0
  // normally; 1 makes every block's bounded wait run out)
  int32_t barrier_extra;
};

// ---- exactly rounded arithmetic (no FMA contraction: the reference has none) ----------
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

template <class T>
__device__ __forceinline__ T clampv(T x, T lo, T hi) {
  x = (x < lo) ? lo : x;
  return (x > hi) ? hi : x;
}

template <class T>
__device__ __forceinline__ T inf_val();
template <>
__device__ __forceinline__ float inf_val<float>() { return __int_as_float(0x7f800000); }
template <>
__device__ __forceinline__ double inf_val<double>() {
  return __longlong_as_double(0x7ff0000000000000ll);
}

}  // namespace dmm
