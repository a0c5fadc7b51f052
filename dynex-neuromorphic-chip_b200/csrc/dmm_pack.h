// Host side of a pack: device arrays for one or many formulas, the device-built CSR,
// tile tables, and the CUDA-graph step loop.  Used by the single-instance API, the
// batched API and the server.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "../../include/dmm.h"
#include "dmm_device.cuh"

namespace dmm {

// Thread-local error text behind dmm_last_error().
void set_error(const char* fmt, ...);
void clear_error();
const char* last_error();

#define DMM_CUDA(call)                                                                     \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      ::dmm::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,  \
                       __LINE__);                                                          \
      return (e_ == cudaErrorMemoryAllocation) ? DMM_ERR_NOMEM : DMM_ERR_CUDA;             \
    }                                                                                      \
  } while (0)

#define DMM_TRY(call)                     \
  do {                                    \
    dmm_status s_ = (call);               \
    if (s_ != DMM_OK) return s_;          \
  } while (0)

// Makes `dev` the calling thread's current device for the scope of a library call and
// restores the caller's device afterwards (every entry point that takes a handle).
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      prev = -1;
    }
    if (dev >= 0 && dev != prev) cudaSetDevice(dev);
  }
  ~DeviceScope() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// Validates a formula given as flat literals + offsets.  Sets *k3 when every clause has
// exactly three literals, and *may_have_units (if given) unless every clause has two or more.
// check_literals = false skips the pass over the literals (the caller checks them on the
// device, see Pack::add).
dmm_status validate_formula(const int32_t* lits, const int64_t* clause_off, int32_t n,
                            int32_t m, bool* k3, bool* may_have_units = nullptr,
                            bool check_literals = true);
// First literal of lits[0, len) outside [-n, n] or zero: sets the error text and returns
// DMM_ERR_LITERAL; DMM_OK when there is none.
dmm_status locate_bad_literal(const int32_t* lits, int64_t len, int32_t n);
// The checks of validate_formula that do not read the clauses or literals (shape of the
// arrays and the slot count); the rest is checked when the formula is added to a pack.
dmm_status validate_shape(const int32_t* lits, const int64_t* clause_off, int32_t n, int32_t m);

// First-fit allocator of aligned ranges in [0, cap).
class RangeAlloc {
 public:
  void reset(int64_t cap);
  // Returns the start or -1 when no free range fits.
  int64_t alloc(int64_t len);
  void free(int64_t start, int64_t len);
  int64_t largest_free() const;
  static int64_t round(int64_t len) { return (len + 31) & ~int64_t(31); }

 private:
  std::map<int64_t, int64_t> free_;  // start -> length
};

struct PackCaps {
  int32_t insts = 1;
  int64_t vars = 0, clauses = 0, slots = 0;
};

struct StepTimes {
  double clause_ms = 0, var_ms = 0, step_ms = 0;
  int64_t launches = 0;
};

class Pack {
 public:
  Pack(dmm_precision prec, int device) : prec_(prec), dev_(device) {}
  ~Pack();
  Pack(const Pack&) = delete;
  Pack& operator=(const Pack&) = delete;

  // fixed_grid: size the persistent grids for the whole device instead of the current
  // tile count (the server changes tiles between launches without re-capturing).
  dmm_status init(const PackCaps& caps, bool with_alpha_cm, bool fixed_grid);
  static int64_t bytes_per(dmm_precision prec, int64_t n, int64_t m, int64_t slots,
                           bool with_alpha_cm);

  // x0 (n+2m doubles, optional): the instance starts runnable from this state, as after
  // set_state, with no read-back of its control record.
  // device_literal_check: the literals are range-checked by the device CSR build instead of
  // a host pass (large formulas); a bad literal is then reported by the next
  // commit_tiles(), which the caller runs before using the formula.
  dmm_status add(const int32_t* lits, const int64_t* clause_off, int32_t n, int32_t m,
                 const dmm_params* p, const double* alpha_cm, int32_t max_steps, int32_t* idx,
                 const double* x0 = nullptr, bool device_literal_check = false);
  dmm_status remove(int32_t idx);
  dmm_status set_params(int32_t idx, const dmm_params* p, const double* alpha_cm);
  dmm_status set_max_steps(int32_t idx, int32_t max_steps);
  // State x (n+2m doubles) at t = 0, step 0; the instance becomes runnable.
  dmm_status set_state(int32_t idx, const double* x);
  // The state x, the integration continuing at simulated time t after `step` accepted
  // steps; keep_best keeps the best unsatisfied count seen so far.
  dmm_status set_state_at(int32_t idx, const double* x, double t, int32_t step, bool keep_best);
  dmm_status get_state(int32_t idx, double* x, double* t);
  dmm_status rhs(int32_t idx, const double* x, double* dxdt, int32_t* loc, double* energy);
  dmm_status dostep(int32_t idx, const double* x, const double* dxdt, double h, double* xo);
  dmm_status assignment(int32_t idx, int8_t* pre, int8_t* post);
  dmm_status read_ctrl(int32_t idx, InstCtrl* c);
  dmm_status read_ctrls(std::vector<InstCtrl>* out);
  // Forces a running instance to stop with the given status (between launches).
  dmm_status stop(int32_t idx, int32_t status);

  dmm_status set_tuning(const dmm_tuning* t);
  dmm_tuning tuning() const { return tun_; }
  // Rebuilds the tile tables after adds/removes.
  dmm_status commit_tiles();
  // Enqueues nsteps steps (CUDA-graph chunks of steps_per_graph, plain launches for the rest).
  dmm_status launch_steps(int32_t nsteps);
  // Enqueues one step as plain launches with CUDA events around each kernel, optionally
  // after writing flush_bytes of scratch (cold L2); accumulates into *t after sync.
  dmm_status profile_steps(int32_t nsteps, int64_t flush_bytes, StepTimes* t);
  // nsteps steps each launched alone after an L2 flush; summed device time of the steps.
  dmm_status time_steps_flushed(int32_t nsteps, int64_t flush_bytes, double* ms);
  // One cooperative launch of nsteps steps with %globaltimer stamps at kTraceK points of
  // every step; out[2k], out[2k+1] = mean and max over blocks of the microseconds from
  // point k to point k+1 (point kTraceK: the next step's start), averaged over steps;
  // out[2 kTraceK] = SM clock (MHz); out[2 kTraceK + 1], [+ 2] = launch prologue and epilogue
  // (staged kernel).
  dmm_status trace_phases(int32_t nsteps, double* out);
  // Kernel used by launch_steps: 1 two-kernel, 2 cooperative, 3 cooperative single formula,
  // 4 staged, 5 one block per formula (dmm_instance_launch_form).
  int launch_form() const;
  // Test hook: one cooperative launch whose first grid barrier waits for one arrival more
  // than the grid has; returns what check_error reports (DMM_ERR_CUDA).
  dmm_status test_barrier_timeout();
  // Loads every kernel this pack's precision and tuning can launch (the driver otherwise
  // loads a kernel at its first launch, which would stall a running service).
  dmm_status preload_kernels();
  // Raises DMM_ERR_CUDA when a cooperative launch reported a grid-barrier timeout.
  dmm_status check_error();
  dmm_status read_active(int32_t* active);
  // Launches step chunks until no instance is running, or wall_s (> 0) seconds pass, or
  // (stop_after > 0) that many instances finished during the call; keeps one chunk in
  // flight while checking the previous one.  *timed_out tells whether time ran out.
  dmm_status run(double wall_s, int64_t* steps_launched, bool* timed_out, int32_t stop_after = 0);
  // Makes an instance stopped by its step cap runnable again.
  dmm_status resume(int32_t idx);
  // Finished instance indices since the last call.
  dmm_status drain_finished(std::vector<int32_t>* out);
  dmm_status sync();
  cudaStream_t stream() const { return stream_; }
  int device() const { return dev_; }
  dmm_precision precision() const { return prec_; }
  const InstDesc& desc(int32_t idx) const { return inst_h_[idx]; }
  bool live(int32_t idx) const { return idx >= 0 && idx < (int32_t)live_.size() && live_[idx]; }
  int32_t num_live() const;
  int64_t free_vars() const { return var_alloc_.largest_free(); }
  int64_t free_clauses() const { return cls_alloc_.largest_free(); }
  int64_t free_slots() const { return slot_alloc_.largest_free(); }
  int32_t free_insts() const;
  int64_t tile_count(int which) const {
    return which == 0 ? (int64_t)ctiles_h_.size() : (int64_t)vtiles_h_.size();
  }
  int sm_count() const { return sms_; }

 private:
  dmm_status build_csr(const InstDesc& I, const int32_t* lits);
  // sorts the slot lists longer than the device sorter (reported by the CSR builds since
  // the last call); runs before the CSR is first used
  dmm_status resolve_long_lists();
  dmm_status ensure_stage(int64_t doubles);
  dmm_status capture(int32_t steps);
  dmm_status launch_persist(int32_t nsteps);
  dmm_status launch_inst(int32_t nsteps);
  dmm_status prepare_xpose(int32_t idx, int TC, int TV, bool mt, bool* ok);
  // several-tiles-per-block staged form for a formula too large for one tile per block:
  // retiles formula idx and builds the tables for the first tiling that fits
  dmm_status prepare_xpose_mt(int32_t idx, bool* ok);
  dmm_status set_tiles(int32_t idx, int TC, int TV);
  dmm_status ensure_flush(int64_t bytes);
  const void* persist_fn() const;
  dmm_status enqueue_step(bool rhs_only, void* dv_out);
  dmm_status enqueue_clause();
  dmm_status enqueue_var(bool rhs_only, void* dv_out);
  template <class T>
  void fill_view(void* view) const;
  dmm_status upload_desc(int32_t idx);
  dmm_status write_ctrl(int32_t idx, const InstCtrl& c);
  dmm_status add_active(int32_t delta);
  dmm_status upload_state(const InstDesc& I, const double* x);
  static InstCtrl running_ctrl(const InstDesc& I, double t, int32_t step);
  void retire(void* p);  // dev_free after this pack's queued work

  dmm_precision prec_;
  int dev_;
  cudaStream_t stream_ = nullptr;
  int sms_ = 148;
  PackCaps caps_;
  size_t tsize_ = 4;
  bool with_alpha_cm_ = false;
  bool fixed_grid_ = false;
  int64_t ctile_cap_ = 0, vtile_cap_ = 0;

  // device arrays
  void* Xs_ = nullptr;
  void* Xl_ = nullptr;
  void* Cp_ = nullptr;
  void* alpha_cm_ = nullptr;
  void* u_ = nullptr;
  void* cand_ = nullptr;
  int32_t* coff_ = nullptr;
  int32_t* lit_ = nullptr;
  int32_t* vslot_ = nullptr;
  int32_t* upos_ = nullptr;  // variable-major position of each slot
  // staged form (single FP32 formula of 3-literal clauses on the cooperative path)
  std::vector<int8_t> unit_h_;  // unit pins of the formula being added
  bool xp_active_ = false;
  bool one_active_ = false;
  bool launch_area_clean_ = false;  // cooperative launch area zeroed (see leave_launch)
  int32_t barrier_extra_ = 0;       // test_barrier_timeout
  // which formula placement and tiling the staged tables were built for
  struct XpKey {
    int32_t idx;
    int64_t var0, slot0;
    int32_t n, m, tc, tv, g;
    bool mt;
    uint64_t serial;
    bool operator==(const XpKey& o) const {
      return idx == o.idx && var0 == o.var0 && slot0 == o.slot0 && n == o.n && m == o.m &&
             tc == o.tc && tv == o.tv && g == o.g && mt == o.mt && serial == o.serial;
    }
  };
  XpKey xp_key_{};
  bool xp_key_valid_ = false;
  std::vector<uint64_t> add_serial_;  // per slot: which add() placed the formula there
  uint64_t add_counter_ = 0;  // single FP32 formula on the cooperative path
  enum { kXpDlist, kXpDoff, kXpLlit, kXpSpos, kXpUx, kXpUbase, kXpBoff, kXpSrc8, kXpDst,
         kXpScratch, kXpBufs };
  void* xbuf_[kXpBufs] = {};
  int64_t xbuf_cap_[kXpBufs] = {};
  int32_t xsv_cap_ = 0, xbk_cap_ = 0, xtv_cap_ = 0, xst_cap_ = 0, xsmem_ = 0;
  bool xp_mt_ = false;  // the staged form runs several tiles per block
  int32_t live0_ = -1;  // the live formula when exactly one has tiles
  long long* trace_ = nullptr;
  int64_t trace_cap_ = 0;
  bool trace_on_ = false;
  int32_t trace_steps_ = 0;
  int32_t* vend_ = nullptr;
  int32_t* fill_ = nullptr;
  int8_t* unit_ = nullptr;
  double* epart_ = nullptr;
  InstDesc* inst_d_ = nullptr;
  InstCtrl* ctrl_d_ = nullptr;
  Tile* ctiles_d_ = nullptr;
  Tile* vtiles_d_ = nullptr;
  int32_t* ntiles_d_ = nullptr;  // [0..1] main tables, [2..3] auxiliary
  int32_t* queue_d_ = nullptr;
  int32_t* active_d_ = nullptr;
  int32_t* ring_d_ = nullptr;
  int32_t* ring_tail_d_ = nullptr;
  int32_t* scan_tmp_ = nullptr;
  int64_t scan_tmp_cap_ = 0;
  int32_t* longv_d_ = nullptr;
  int32_t longv_cap_ = 0;
  bool long_pending_ = false;  // CSR builds since the last resolve_long_lists()
  double* stage_ = nullptr;
  int64_t stage_cap_ = 0;
  Tile* aux_ctiles_d_ = nullptr;
  Tile* aux_vtiles_d_ = nullptr;
  int64_t aux_cap_ = 0;
  void* flush_ = nullptr;
  int64_t flush_cap_ = 0;
  cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};
  int32_t* pinned_ = nullptr;  // host copies of the running count and finished-ring tail
  int32_t* live_d_ = nullptr;  // indices of the instances with tiles
  int32_t* misc_d_ = nullptr;  // [0] live count, [1] barrier error, [2] barrier counter,
                               // [3] formula queue of the one-block-per-formula kernel
  int32_t* order_d_ = nullptr; // formulas run one block each, largest first
  int32_t n_small_ = 0;
  int grid_p_ = 148;           // blocks of the cooperative step kernel

  // host mirrors
  std::vector<InstDesc> inst_h_;
  std::vector<uint8_t> live_;
  RangeAlloc var_alloc_, cls_alloc_, slot_alloc_;
  std::vector<Tile> ctiles_h_, vtiles_h_;
  dmm_tuning tun_{};
  int32_t ring_read_ = 0;

  // graph of steps_per_graph steps
  cudaGraphExec_t graph_exec_ = nullptr;
  cudaGraph_t graph_ = nullptr;
  int32_t graph_steps_ = 0;
  bool graph_stale_ = true;
  int grid_c_ = 1, grid_v_ = 1;
  bool use_aux_ = false;  // route the next launches through the auxiliary tile tables
};

}  // namespace dmm
