// extern "C" entry points of include/dmm.h: library, single instance, batch.
#include <chrono>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "devmem.h"
#include "dmm_pack.h"

using dmm::InstCtrl;
using dmm::Pack;

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void fill_report(const InstCtrl& c, dmm_report* r) {
  std::memset(r, 0, sizeof *r);
  r->status = c.done;
  r->steps = c.step;
  r->t = c.t;
  r->loc = c.loc;
  r->best_loc = c.best_loc;
  r->energy = c.energy;
  r->solved_step = c.solved_step;
  r->solved_t = c.solved_t;
}

}  // namespace

struct dmm_instance {
  std::unique_ptr<Pack> pack;
  int32_t idx = -1;
  int32_t n = 0, m = 0;
  double last_wall = 0.0;
};

struct dmm_batch {
  std::unique_ptr<Pack> pack;
  std::vector<int32_t> idx;
  std::vector<int32_t> m;
  bool dirty = true;
};

extern "C" {

int32_t dmm_abi_version(void) { return DMM_ABI_VERSION; }

const char* dmm_status_string(dmm_status s) {
  switch (s) {
    case DMM_OK: return "ok";
    case DMM_ERR_ARG: return "invalid argument";
    case DMM_ERR_CUDA: return "CUDA error";
    case DMM_ERR_NOMEM: return "out of memory";
    case DMM_ERR_NO_DEVICE: return "no CUDA device";
    case DMM_ERR_LITERAL: return "literal out of range";
    case DMM_ERR_CLAUSE_LEN: return "clause too long";
    case DMM_ERR_PARSE: return "malformed DIMACS";
    case DMM_ERR_IO: return "I/O error";
    case DMM_ERR_BUDGET: return "over the device-memory budget";
    case DMM_ERR_STATE: return "invalid in the current state";
    case DMM_ERR_BUILD: return "library built without kernels for this device";
  }
  return "unknown status";
}

const char* dmm_last_error(void) { return dmm::last_error(); }

void dmm_params_default(dmm_params* p) {
  if (!p) return;
  p->alpha = 2.5;   // dynex.cc:132
  p->beta = 20.0;   // dynex.cc:134
  p->gamma = 0.25;  // dynex.cc:135
  p->delta = 0.05;  // dynex.cc:136
  p->epsilon = 0.1; // dynex.cc:137
  p->zeta = 0.1;    // dynex.cc:138
  p->xl_max = 10000;  // dynex.cc:140
  p->reserved = 0;
}

void dmm_release_cached_memory(void) { dmm::release_cached(); }

int32_t dmm_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// ---- single instance ----------------------------------------------------------------------

dmm_status dmm_instance_create(const int32_t* lits, const int64_t* clause_off, int32_t n, int32_t m,
                               dmm_precision precision, int32_t device, dmm_instance** out) {
  dmm::clear_error();
  if (!out || (precision != DMM_FP32 && precision != DMM_FP64)) return DMM_ERR_ARG;
  *out = nullptr;
  dmm::DeviceScope device_scope(device);
  DMM_TRY(dmm::validate_shape(lits, clause_off, n, m));  // the rest is checked by add()
  auto* inst = new (std::nothrow) dmm_instance();
  if (!inst) return DMM_ERR_NOMEM;
  inst->pack.reset(new (std::nothrow) Pack(precision, device));
  if (!inst->pack) {
    delete inst;
    return DMM_ERR_NOMEM;
  }
  dmm::PackCaps caps;
  caps.insts = 1;
  caps.vars = n;
  caps.clauses = m;
  caps.slots = clause_off[m];
  dmm_status st = inst->pack->init(caps, true, false);
  // the literals are range-checked by the device CSR build (a host pass over a large
  // formula costs milliseconds); commit_tiles reports a bad one
  if (st == DMM_OK)
    st = inst->pack->add(lits, clause_off, n, m, nullptr, nullptr, 0, &inst->idx, nullptr, true);
  if (st == DMM_OK) st = inst->pack->commit_tiles();
  if (st != DMM_OK) {
    delete inst;
    return st;
  }
  inst->n = n;
  inst->m = m;
  *out = inst;
  return DMM_OK;
}

void dmm_instance_destroy(dmm_instance* inst) {
  if (!inst) return;
  dmm::DeviceScope device_scope(inst->pack ? inst->pack->device() : -1);
  delete inst;
}

dmm_status dmm_instance_set_params(dmm_instance* inst, const dmm_params* p, const double* alpha_cm) {
  dmm::clear_error();
  if (!inst || !p) return DMM_ERR_ARG;
  return inst->pack->set_params(inst->idx, p, alpha_cm);
}

dmm_status dmm_instance_set_tuning(dmm_instance* inst, const dmm_tuning* t) {
  dmm::clear_error();
  if (!inst || !t) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  return inst->pack->set_tuning(t);
}

dmm_status dmm_instance_get_tuning(const dmm_instance* inst, dmm_tuning* t) {
  if (!inst || !t) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  *t = inst->pack->tuning();
  return DMM_OK;
}

dmm_status dmm_instance_set_state(dmm_instance* inst, const double* x) {
  dmm::clear_error();
  if (!inst || !x) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  return inst->pack->set_state(inst->idx, x);
}

dmm_status dmm_instance_set_state_at(dmm_instance* inst, const double* x, double t,
                                     int32_t step) {
  dmm::clear_error();
  if (!inst || !x || step < 0) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  return inst->pack->set_state_at(inst->idx, x, t, step, true);
}

dmm_status dmm_instance_get_state(dmm_instance* inst, double* x, double* t) {
  dmm::clear_error();
  if (!inst) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  return inst->pack->get_state(inst->idx, x, t);
}

dmm_status dmm_instance_rhs(dmm_instance* inst, const double* x, double* dxdt, int32_t* loc,
                            double* energy) {
  dmm::clear_error();
  if (!inst || !x || !dxdt) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  return inst->pack->rhs(inst->idx, x, dxdt, loc, energy);
}

dmm_status dmm_instance_dostep(dmm_instance* inst, const double* x, const double* dxdt, double h,
                               double* x_out) {
  dmm::clear_error();
  if (!inst || !x || !dxdt || !x_out) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  return inst->pack->dostep(inst->idx, x, dxdt, h, x_out);
}

dmm_status dmm_instance_report(dmm_instance* inst, dmm_report* rep) {
  dmm::clear_error();
  if (!inst || !rep) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  InstCtrl c;
  DMM_TRY(inst->pack->read_ctrl(inst->idx, &c));
  fill_report(c, rep);
  rep->wall_s = inst->last_wall;
  return DMM_OK;
}

dmm_status dmm_instance_step(dmm_instance* inst, int32_t nsteps, dmm_report* rep) {
  dmm::clear_error();
  if (!inst || nsteps < 0) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  const double t0 = now_s();
  InstCtrl c;
  DMM_TRY(inst->pack->read_ctrl(inst->idx, &c));
  if (c.done == 0 && nsteps > 0) {
    const int32_t cap = c.step + nsteps;
    DMM_TRY(inst->pack->set_max_steps(inst->idx, cap));
    // exactly nsteps: whole graph chunks, then plain launches for the rest
    DMM_TRY(inst->pack->launch_steps(nsteps));
    DMM_TRY(inst->pack->sync());
    DMM_TRY(inst->pack->read_ctrl(inst->idx, &c));
    if (c.done == DMM_STEP_LIMIT && c.step == cap) DMM_TRY(inst->pack->resume(inst->idx));
    DMM_TRY(inst->pack->set_max_steps(inst->idx, 0));
  }
  inst->last_wall = now_s() - t0;
  if (rep) return dmm_instance_report(inst, rep);
  return DMM_OK;
}

dmm_status dmm_instance_solve(dmm_instance* inst, const dmm_limits* lim, dmm_report* rep) {
  dmm::clear_error();
  if (!inst) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  const double t0 = now_s();
  const int32_t max_steps = lim && lim->max_steps > 0 ? lim->max_steps : 0;
  const double wall = lim ? lim->wall_s : 0.0;
  DMM_TRY(inst->pack->set_max_steps(inst->idx, max_steps));
  bool timed_out = false;
  int64_t launched = 0;
  DMM_TRY(inst->pack->run(wall, &launched, &timed_out));
  if (timed_out) DMM_TRY(inst->pack->stop(inst->idx, DMM_TIME_LIMIT));
  inst->last_wall = now_s() - t0;
  if (rep) return dmm_instance_report(inst, rep);
  return DMM_OK;
}

dmm_status dmm_instance_assignment(dmm_instance* inst, int8_t* pre, int8_t* post) {
  dmm::clear_error();
  if (!inst) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  return inst->pack->assignment(inst->idx, pre, post);
}

dmm_status dmm_instance_profile(dmm_instance* inst, int32_t nsteps, int64_t flush_bytes,
                                double* clause_ms, double* var_ms) {
  dmm::clear_error();
  if (!inst || nsteps < 0 || flush_bytes < 0) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  dmm::StepTimes t;
  DMM_TRY(inst->pack->profile_steps(nsteps, flush_bytes, &t));
  if (clause_ms) *clause_ms = t.clause_ms;
  if (var_ms) *var_ms = t.var_ms;
  return DMM_OK;
}

dmm_status dmm_instance_time_steps(dmm_instance* inst, int32_t nsteps, double* ms) {
  dmm::clear_error();
  if (!inst || nsteps < 0 || !ms) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  cudaEvent_t e0, e1;
  DMM_CUDA(cudaEventCreate(&e0));
  DMM_CUDA(cudaEventCreate(&e1));
  DMM_CUDA(cudaEventRecord(e0, inst->pack->stream()));
  dmm_status st = inst->pack->launch_steps(nsteps);
  DMM_CUDA(cudaEventRecord(e1, inst->pack->stream()));
  DMM_CUDA(cudaEventSynchronize(e1));
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = t;
  return st;
}

dmm_status dmm_instance_time_steps_flushed(dmm_instance* inst, int32_t nsteps,
                                           int64_t flush_bytes, double* ms) {
  dmm::clear_error();
  if (!inst || nsteps < 0 || flush_bytes < 0 || !ms) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  return inst->pack->time_steps_flushed(nsteps, flush_bytes, ms);
}

dmm_status dmm_instance_test_barrier_timeout(dmm_instance* inst) {
  dmm::clear_error();
  if (!inst) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  return inst->pack->test_barrier_timeout();
}

int32_t dmm_instance_launch_form(const dmm_instance* inst) {
  if (!inst) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  return inst->pack->launch_form();
}

dmm_status dmm_instance_trace_phases(dmm_instance* inst, int32_t nsteps, double* out) {
  dmm::clear_error();
  if (!inst || nsteps <= 0 || !out) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(inst->pack->device());
  return inst->pack->trace_phases(nsteps, out);
}

// ---- batch ---------------------------------------------------------------------------------

dmm_status dmm_batch_create(dmm_precision precision, int32_t device, int32_t max_instances,
                            int64_t max_vars, int64_t max_clauses, int64_t max_lits,
                            dmm_batch** out) {
  dmm::clear_error();
  if (!out || max_instances <= 0 || max_vars <= 0 || max_clauses < 0 || max_lits < 0 ||
      (precision != DMM_FP32 && precision != DMM_FP64))
    return DMM_ERR_ARG;
  *out = nullptr;
  dmm::DeviceScope device_scope(device);
  auto* b = new (std::nothrow) dmm_batch();
  if (!b) return DMM_ERR_NOMEM;
  b->pack.reset(new (std::nothrow) Pack(precision, device));
  dmm::PackCaps caps;
  caps.insts = max_instances;
  caps.vars = max_vars;
  caps.clauses = max_clauses;
  caps.slots = max_lits;
  dmm_status st = b->pack ? b->pack->init(caps, false, false) : DMM_ERR_NOMEM;
  if (st != DMM_OK) {
    delete b;
    return st;
  }
  *out = b;
  return DMM_OK;
}

void dmm_batch_destroy(dmm_batch* b) {
  if (!b) return;
  dmm::DeviceScope device_scope(b->pack ? b->pack->device() : -1);
  delete b;
}

dmm_status dmm_batch_set_tuning(dmm_batch* b, const dmm_tuning* t) {
  dmm::clear_error();
  if (!b || !t) return DMM_ERR_ARG;
  b->dirty = true;
  return b->pack->set_tuning(t);
}

dmm_status dmm_batch_add(dmm_batch* b, const int32_t* lits, const int64_t* clause_off, int32_t n,
                         int32_t m, const dmm_params* p, const double* x0, int32_t max_steps,
                         int32_t* index) {
  dmm::clear_error();
  if (!b || !x0 || !index) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(b->pack->device());
  int32_t idx = -1;
  DMM_TRY(b->pack->add(lits, clause_off, n, m, p, nullptr, max_steps, &idx, x0));
  *index = (int32_t)b->idx.size();
  b->idx.push_back(idx);
  b->m.push_back(m);
  b->dirty = true;
  return DMM_OK;
}

dmm_status dmm_batch_run(dmm_batch* b, double wall_s, dmm_batch_stats* stats) {
  return dmm_batch_run_until(b, wall_s, 0, stats);
}

dmm_status dmm_batch_run_until(dmm_batch* b, double wall_s, int32_t stop_after,
                               dmm_batch_stats* stats) {
  dmm::clear_error();
  if (!b || stop_after < 0) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(b->pack->device());
  if (b->dirty) {
    DMM_TRY(b->pack->commit_tiles());
    b->dirty = false;
  }
  std::vector<InstCtrl> before;
  DMM_TRY(b->pack->read_ctrls(&before));
  cudaEvent_t e0, e1;
  DMM_CUDA(cudaEventCreate(&e0));
  DMM_CUDA(cudaEventCreate(&e1));
  const double t0 = now_s();
  DMM_CUDA(cudaEventRecord(e0, b->pack->stream()));
  bool timed_out = false;
  int64_t launched = 0;
  dmm_status st = b->pack->run(wall_s, &launched, &timed_out, stop_after);
  DMM_CUDA(cudaEventRecord(e1, b->pack->stream()));
  DMM_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  DMM_TRY(st);
  const double wall = now_s() - t0;
  std::vector<InstCtrl> after;
  DMM_TRY(b->pack->read_ctrls(&after));
  if (timed_out || stop_after > 0)
    for (int32_t i : b->idx)
      if (after[i].done == 0) {
        DMM_TRY(b->pack->stop(i, timed_out ? DMM_TIME_LIMIT : DMM_CANCELLED));
        after[i].done = timed_out ? DMM_TIME_LIMIT : DMM_CANCELLED;
      }
  if (stats) {
    std::memset(stats, 0, sizeof *stats);
    for (size_t k = 0; k < b->idx.size(); k++) {
      const InstCtrl& a = after[b->idx[k]];
      stats->clause_updates += (int64_t)b->m[k] * (a.step - before[b->idx[k]].step);
      if (a.done == DMM_SOLVED) stats->solved++;
      else stats->unsolved++;
    }
    stats->steps_launched = launched;
    stats->wall_s = wall;
    stats->device_ms = ms;
  }
  return DMM_OK;
}

dmm_status dmm_batch_result(dmm_batch* b, int32_t index, dmm_report* rep, int8_t* post) {
  dmm::clear_error();
  if (!b || index < 0 || index >= (int32_t)b->idx.size()) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(b->pack->device());
  const int32_t i = b->idx[index];
  if (rep) {
    InstCtrl c;
    DMM_TRY(b->pack->read_ctrl(i, &c));
    fill_report(c, rep);
  }
  if (post) DMM_TRY(b->pack->assignment(i, nullptr, post));
  return DMM_OK;
}

dmm_status dmm_batch_assignment(dmm_batch* b, int32_t index, int8_t* pre, int8_t* post) {
  dmm::clear_error();
  if (!b || index < 0 || index >= (int32_t)b->idx.size()) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(b->pack->device());
  return b->pack->assignment(b->idx[index], pre, post);
}

dmm_status dmm_batch_state(dmm_batch* b, int32_t index, double* x, double* t) {
  dmm::clear_error();
  if (!b || index < 0 || index >= (int32_t)b->idx.size()) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(b->pack->device());
  return b->pack->get_state(b->idx[index], x, t);
}

dmm_status dmm_batch_set_state_at(dmm_batch* b, int32_t index, const double* x, double t,
                                  int32_t step) {
  dmm::clear_error();
  if (!b || !x || index < 0 || index >= (int32_t)b->idx.size() || step < 0) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(b->pack->device());
  return b->pack->set_state_at(b->idx[index], x, t, step, false);
}

}  // extern "C"
