// Continuous-batching server: requests are admitted into one resident pack as slots and
// device memory free up, every resident instance advances together in CUDA-graph chunks,
// and finished instances are retired and their ranges reused.  Results of an instance do
// not depend on what else is resident: tiles never straddle instances and every
// per-instance reduction has a fixed order.
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <new>
#include <vector>

#include "dmm_pack.h"

using dmm::InstCtrl;
using dmm::Pack;

namespace {

struct Request {
  int64_t ticket = 0;
  std::vector<int32_t> lits;
  std::vector<int64_t> off;
  int32_t n = 0, m = 0;
  dmm_params p{};
  std::vector<double> x0;
  uint64_t seed = 0;
  int32_t max_steps = 0;
  double submit_s = 0;
  int64_t bytes = 0;
};

struct Resident {
  int64_t ticket = 0;
  int32_t n = 0, m = 0;
  double submit_s = 0, admit_s = 0;
  int64_t bytes = 0;
};

}  // namespace

struct dmm_server {
  dmm_server_config cfg{};
  std::unique_ptr<Pack> pack;
  std::deque<Request> queue;
  std::map<int32_t, Resident> resident;  // pack index -> request
  std::vector<dmm_server_result> finished;
  std::map<int64_t, std::vector<int8_t>> assignments;
  int64_t next_ticket = 1;
  int64_t used_bytes = 0;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double clock() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

extern "C" {

dmm_status dmm_server_create(const dmm_server_config* cfg, dmm_server** out) {
  dmm::clear_error();
  if (!cfg || !out || cfg->budget_bytes <= 0 || cfg->max_slots <= 0 ||
      (cfg->precision != DMM_FP32 && cfg->precision != DMM_FP64))
    return DMM_ERR_ARG;
  *out = nullptr;
  dmm::DeviceScope device_scope(cfg->device);
  // the arena below is reserved up front: the budget must fit the device's free memory,
  // with headroom for the per-launch buffers and other users of the device
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    cudaGetLastError();
    dmm::set_error("server: cannot read the device's free memory");
    return DMM_ERR_CUDA;
  }
  constexpr int64_t kHeadroom = int64_t(1) << 30;
  if (cfg->budget_bytes > (int64_t)free_b - kHeadroom) {
    dmm::set_error("server: budget of %lld bytes exceeds the device's free memory (%lld of %lld "
                   "bytes) less 1 GiB of headroom",
                   (long long)cfg->budget_bytes, (long long)free_b, (long long)total_b);
    return DMM_ERR_BUDGET;
  }
  auto* s = new (std::nothrow) dmm_server();
  if (!s) return DMM_ERR_NOMEM;
  s->cfg = *cfg;
  if (s->cfg.steps_per_launch <= 0) s->cfg.steps_per_launch = 32;
  s->pack.reset(new (std::nothrow) Pack((dmm_precision)cfg->precision, cfg->device));
  // Arena capacities from the budget: a 3-literal clause costs 3t+4 bytes plus 3 slots of
  // 12+t (Pack::bytes_per); variables get a quarter of the budget so formulas down to ratio
  // ~2 fit.
  const int64_t t = cfg->precision == DMM_FP64 ? 8 : 4;
  const int64_t per_clause = 3 * t + 4 + 3 * (12 + t);
  const int64_t per_var = 8 * t + 9;
  dmm::PackCaps caps;
  caps.insts = cfg->max_slots;
  caps.clauses = std::max<int64_t>(1024, (cfg->budget_bytes * 3 / 4) / per_clause);
  caps.slots = 3 * caps.clauses;
  caps.vars = std::max<int64_t>(1024, (cfg->budget_bytes / 4) / per_var);
  dmm_status st = s->pack ? s->pack->init(caps, false, true) : DMM_ERR_NOMEM;
  if (st != DMM_OK) {
    delete s;
    return st;
  }
  dmm_tuning tun{};
  tun.steps_per_graph = s->cfg.steps_per_launch;
  st = s->pack->set_tuning(&tun);
  if (st == DMM_OK) st = s->pack->preload_kernels();
  if (st != DMM_OK) {
    delete s;
    return st;
  }
  *out = s;
  return DMM_OK;
}

void dmm_server_destroy(dmm_server* s) {
  if (!s) return;
  dmm::DeviceScope device_scope(s->pack ? s->pack->device() : -1);
  delete s;
}

double dmm_server_clock(dmm_server* s) { return s ? s->clock() : 0.0; }

dmm_status dmm_server_submit(dmm_server* s, const int32_t* lits, const int64_t* clause_off,
                             int32_t n, int32_t m, const dmm_params* p, const double* x0,
                             uint64_t init_seed, int32_t max_steps, int64_t* ticket) {
  dmm::clear_error();
  if (!s || !ticket) return DMM_ERR_ARG;
  bool k3;
  DMM_TRY(dmm::validate_formula(lits, clause_off, n, m, &k3));
  Request r;
  r.bytes = Pack::bytes_per((dmm_precision)s->cfg.precision, n, m, clause_off[m], false);
  if (r.bytes > s->cfg.budget_bytes) {
    dmm::set_error("request needs %lld bytes, budget is %lld", (long long)r.bytes,
                   (long long)s->cfg.budget_bytes);
    return DMM_ERR_BUDGET;
  }
  r.ticket = s->next_ticket++;
  r.lits.assign(lits, lits + clause_off[m]);
  r.off.assign(clause_off, clause_off + m + 1);
  r.n = n;
  r.m = m;
  if (p) r.p = *p;
  else dmm_params_default(&r.p);
  if (x0) r.x0.assign(x0, x0 + (int64_t)n + 2 * (int64_t)m);
  r.seed = init_seed;
  r.max_steps = max_steps;
  r.submit_s = s->clock();
  *ticket = r.ticket;
  s->queue.push_back(std::move(r));
  return DMM_OK;
}

static dmm_status retire(dmm_server* s) {
  std::vector<int32_t> fin;
  DMM_TRY(s->pack->drain_finished(&fin));
  const double now = s->clock();
  for (int32_t idx : fin) {
    auto it = s->resident.find(idx);
    if (it == s->resident.end()) continue;
    InstCtrl c;
    DMM_TRY(s->pack->read_ctrl(idx, &c));
    dmm_server_result res;
    std::memset(&res, 0, sizeof res);
    res.ticket = it->second.ticket;
    res.report.status = c.done;
    res.report.steps = c.step;
    res.report.t = c.t;
    res.report.loc = c.loc;
    res.report.best_loc = c.best_loc;
    res.report.energy = c.energy;
    res.report.solved_step = c.solved_step;
    res.report.solved_t = c.solved_t;
    res.report.wall_s = now - it->second.admit_s;
    res.submit_s = it->second.submit_s;
    res.admit_s = it->second.admit_s;
    res.finish_s = now;
    std::vector<int8_t> post(it->second.n);
    DMM_TRY(s->pack->assignment(idx, nullptr, post.data()));
    s->assignments[res.ticket] = std::move(post);
    s->finished.push_back(res);
    s->used_bytes -= it->second.bytes;
    DMM_TRY(s->pack->remove(idx));
    s->resident.erase(it);
  }
  return DMM_OK;
}

static dmm_status admit(dmm_server* s, bool* changed) {
  for (auto it = s->queue.begin(); it != s->queue.end();) {
    Request& r = *it;
    const bool fits = s->used_bytes + r.bytes <= s->cfg.budget_bytes && s->pack->free_insts() > 0 &&
                      s->pack->free_vars() >= r.n && s->pack->free_clauses() >= r.m &&
                      s->pack->free_slots() >= (int64_t)r.lits.size();
    if (!fits) {
      ++it;
      continue;
    }
    if (r.x0.empty()) {
      r.x0.resize((size_t)r.n + 2 * (size_t)r.m);
      DMM_TRY(dmm_initial_state_uniform(r.lits.data(), r.off.data(), r.n, r.m, r.seed, r.x0.data()));
    }
    int32_t idx = -1;
    dmm_status st = s->pack->add(r.lits.data(), r.off.data(), r.n, r.m, &r.p, nullptr,
                                 r.max_steps, &idx, r.x0.data());
    if (st == DMM_ERR_BUDGET) {  // fragmented arena: try again after retirements
      ++it;
      continue;
    }
    DMM_TRY(st);
    Resident res;
    res.ticket = r.ticket;
    res.n = r.n;
    res.m = r.m;
    res.submit_s = r.submit_s;
    res.admit_s = s->clock();
    res.bytes = r.bytes;
    s->resident[idx] = res;
    s->used_bytes += r.bytes;
    *changed = true;
    it = s->queue.erase(it);
  }
  return DMM_OK;
}

dmm_status dmm_server_pump(dmm_server* s, int32_t* resident, int32_t* queued) {
  dmm::clear_error();
  if (!s) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(s->pack->device());
  DMM_TRY(retire(s));
  bool changed = false;
  DMM_TRY(admit(s, &changed));
  if (changed || s->pack->tile_count(0) + s->pack->tile_count(1) == 0 ||
      (int64_t)s->resident.size() != (int64_t)s->pack->num_live())
    DMM_TRY(s->pack->commit_tiles());
  if (!s->resident.empty()) {
    DMM_TRY(s->pack->launch_steps(s->cfg.steps_per_launch));
    DMM_TRY(s->pack->sync());
    DMM_TRY(retire(s));
    bool ch2 = false;
    DMM_TRY(admit(s, &ch2));
    if (ch2 || !s->resident.empty()) DMM_TRY(s->pack->commit_tiles());
  }
  if (resident) *resident = (int32_t)s->resident.size();
  if (queued) *queued = (int32_t)s->queue.size();
  return DMM_OK;
}

dmm_status dmm_server_take(dmm_server* s, dmm_server_result* out, int32_t cap, int32_t* count) {
  dmm::clear_error();
  if (!s || !count || cap < 0 || (cap > 0 && !out)) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(s->pack->device());
  const int32_t k = std::min<int32_t>(cap, (int32_t)s->finished.size());
  for (int32_t i = 0; i < k; i++) out[i] = s->finished[i];
  s->finished.erase(s->finished.begin(), s->finished.begin() + k);
  *count = k;
  return DMM_OK;
}

dmm_status dmm_server_assignment(dmm_server* s, int64_t ticket, int8_t* post, int32_t n) {
  dmm::clear_error();
  if (!s || !post) return DMM_ERR_ARG;
  dmm::DeviceScope device_scope(s->pack->device());
  auto it = s->assignments.find(ticket);
  if (it == s->assignments.end()) {
    dmm::set_error("no finished assignment for ticket %lld", (long long)ticket);
    return DMM_ERR_STATE;
  }
  if ((int32_t)it->second.size() != n) return DMM_ERR_ARG;
  std::memcpy(post, it->second.data(), n);
  s->assignments.erase(it);
  return DMM_OK;
}

}  // extern "C"
