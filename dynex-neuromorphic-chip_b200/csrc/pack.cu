// Pack: device arrays, device-built CSR, tile tables and the CUDA-graph step loop.
#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "dmm_inst.cuh"
#include "dmm_step.cuh"
#include "dmm_xprep.cuh"
#include "dmm_pack.h"
#include "devmem.h"

namespace dmm {

// ---- errors --------------------------------------------------------------------------------
static thread_local std::string g_err;
void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
}
void clear_error() { g_err.clear(); }
const char* last_error() { return g_err.c_str(); }

dmm_status validate_shape(const int32_t* lits, const int64_t* clause_off, int32_t n, int32_t m) {
  if (n <= 0 || m < 0 || clause_off == nullptr) {
    set_error("formula: need n > 0, m >= 0 and clause offsets");
    return DMM_ERR_ARG;
  }
  if (clause_off[0] != 0) {
    set_error("formula: clause_off[0] must be 0");
    return DMM_ERR_ARG;
  }
  const int64_t L = clause_off[m];
  if (L < 0 || L > 0x7fffffffll - 64) {
    set_error("formula: %lld literals outside the 2^31 slot limit", (long long)L);
    return DMM_ERR_ARG;
  }
  if (L > 0 && lits == nullptr) {
    set_error("formula: literals missing");
    return DMM_ERR_ARG;
  }
  return DMM_OK;
}

// Runs f(lo, hi, t) over the chunks t of [0, len) on up to kValidateThreads host threads
// when len is large (these passes are bound by memory bandwidth, which one core does not
// reach); returns the number of chunks.  Falls back to one chunk on the calling thread
// when no thread can be started.
constexpr int kValidateThreads = 8;
constexpr int64_t kValidateChunk = int64_t(1) << 18;  // elements per thread at least
template <class F>
static int host_parallel(int64_t len, F&& f) {
  const int64_t hw = std::max(1u, std::thread::hardware_concurrency());
  const int T = (int)std::max<int64_t>(
      1, std::min<int64_t>({(int64_t)kValidateThreads, hw, len / kValidateChunk}));
  if (T <= 1) {
    f(int64_t(0), len, 0);
    return 1;
  }
  const int64_t per = (len + T - 1) / T;
  std::vector<std::thread> th;
  try {
    for (int t = 1; t < T; t++)
      th.emplace_back([&f, t, per, len] { f(t * per, std::min(len, (t + 1) * per), t); });
  } catch (...) {
    for (auto& x : th) x.join();
    f(int64_t(0), len, 0);
    return 1;
  }
  f(int64_t(0), std::min(len, per), 0);
  for (auto& x : th) x.join();
  return T;
}

dmm_status locate_bad_literal(const int32_t* lits, int64_t len, int32_t n) {
  for (int64_t s = 0; s < len; s++) {
    const int32_t l = lits[s];
    if (l == 0 || l > n || l < -n) {
      set_error("formula: literal %d at position %lld out of range for n=%d", l, (long long)s, n);
      return DMM_ERR_LITERAL;
    }
  }
  return DMM_OK;
}

dmm_status validate_formula(const int32_t* lits, const int64_t* clause_off, int32_t n, int32_t m,
                            bool* k3, bool* may_have_units, bool check_literals) {
  if (n <= 0 || m < 0 || clause_off == nullptr) {
    set_error("formula: need n > 0, m >= 0 and clause offsets");
    return DMM_ERR_ARG;
  }
  if (clause_off[0] != 0) {
    set_error("formula: clause_off[0] must be 0");
    return DMM_ERR_ARG;
  }
  // branch-free passes (they vectorize), split over host threads for large formulas; the
  // slow loops below only locate an error
  int64_t lmin_t[kValidateThreads], lmax_t[kValidateThreads];
  const int nt_c = host_parallel(m, [&](int64_t lo, int64_t hi, int t) {
    int64_t a = INT64_MAX, b = INT64_MIN;
    for (int64_t c = lo; c < hi; c++) {
      const int64_t len = clause_off[c + 1] - clause_off[c];
      a = len < a ? len : a;
      b = len > b ? len : b;
    }
    lmin_t[t] = a;
    lmax_t[t] = b;
  });
  int64_t lmin = INT64_MAX, lmax = INT64_MIN;
  for (int t = 0; t < nt_c; t++) {
    lmin = std::min(lmin, lmin_t[t]);
    lmax = std::max(lmax, lmax_t[t]);
  }
  if (m > 0 && (lmin < 0 || lmax > DMM_MAX_CLAUSE_LITS)) {
    for (int32_t c = 0; c < m; c++) {
      const int64_t len = clause_off[c + 1] - clause_off[c];
      if (len < 0) {
        set_error("formula: clause offsets decrease at clause %d", c);
        return DMM_ERR_ARG;
      }
      if (len > DMM_MAX_CLAUSE_LITS) {
        set_error("CLAUSE %d HAS MORE THAN %d LITERALS", c, DMM_MAX_CLAUSE_LITS);
        return DMM_ERR_CLAUSE_LEN;
      }
    }
  }
  const int64_t L = clause_off[m];
  if (L > 0x7fffffffll - 64) {
    set_error("formula: %lld literals exceed the 2^31 slot limit", (long long)L);
    return DMM_ERR_ARG;
  }
  if (L > 0 && lits == nullptr) {
    set_error("formula: literals missing");
    return DMM_ERR_ARG;
  }
  // -n <= l <= n, l != 0: (unsigned)l + n lies in [0, 2n]
  const uint32_t un = (uint32_t)n, span = 2u * (uint32_t)n;
  uint32_t bad_t[kValidateThreads];
  const int nt_l = host_parallel(check_literals ? L : 0, [&](int64_t lo, int64_t hi, int t) {
    uint32_t bad = 0;
    for (int64_t s = lo; s < hi; s++) {
      const int32_t l = lits[s];
      bad |= (uint32_t)(l == 0) | (uint32_t)((uint32_t)l + un > span);
    }
    bad_t[t] = bad;
  });
  uint32_t bad = 0;
  for (int t = 0; t < nt_l; t++) bad |= bad_t[t];
  if (bad) DMM_TRY(locate_bad_literal(lits, L, n));
  *k3 = m > 0 && lmin == 3 && lmax == 3;
  if (may_have_units) *may_have_units = m > 0 && lmin <= 1;
  return DMM_OK;
}

// ---- range allocator ---------------------------------------------------------------------------
void RangeAlloc::reset(int64_t cap) {
  free_.clear();
  if (cap > 0) free_[0] = cap;
}

int64_t RangeAlloc::alloc(int64_t len) {
  len = round(std::max<int64_t>(len, 1));
  for (auto it = free_.begin(); it != free_.end(); ++it) {
    if (it->second >= len) {
      const int64_t start = it->first, rest = it->second - len;
      free_.erase(it);
      if (rest > 0) free_[start + len] = rest;
      return start;
    }
  }
  return -1;
}

void RangeAlloc::free(int64_t start, int64_t len) {
  len = round(std::max<int64_t>(len, 1));
  auto it = free_.emplace(start, len).first;
  auto nx = std::next(it);
  if (nx != free_.end() && it->first + it->second == nx->first) {
    it->second += nx->second;
    free_.erase(nx);
  }
  if (it != free_.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == it->first) {
      pv->second += it->second;
      free_.erase(it);
    }
  }
}

int64_t RangeAlloc::largest_free() const {
  int64_t b = 0;
  for (auto& kv : free_) b = std::max(b, kv.second);
  return b;
}

// ---- pack ------------------------------------------------------------------------------------

namespace {
inline int blocks_for(int64_t work, int per = kThreads, int cap = 148 * 16) {
  int64_t b = (work + per - 1) / per;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (int)b;
}
constexpr int kMinClauseTile = 256;  // smallest clause tile (bounds the tile tables)
constexpr int kMinVarTile = 32;      // smallest variable tile
constexpr int kPersistThreads = 1024;  // block size of the cooperative step kernel
// FP64: 512 threads, so that the sorted sums and the clause code fit in registers without
// spilling (measured 74.3 vs 76.4 us per n=100k step with 1024 threads)
constexpr int kPersistThreads64 = 512;
constexpr int kStagedThreads = 1024;  // block size of the staged form
static int persist_threads(dmm_precision prec) {
  return prec == DMM_FP64 ? kPersistThreads64 : kPersistThreads;
}
constexpr int kSlotPad = 8;             // entries past the last slot of vslot and u
constexpr int kXpSmemMax = 220 * 1024;  // dynamic shared memory of the staged form, at most
// ... and of its several-tiles-per-block form: beyond about 195 KB a block takes the largest
// shared-memory carve-out, and the L1 left to the gathers shrinks (measured at 0.4-1.5 million
// variables: every tiling above the cap ran 8-30 % slower than the best one below it)
constexpr int kXpSmemMaxMT = 193 * 1024;  // with the form's ~1.4 KB of static shared memory
constexpr int kXpMaxTiles = 1 << 14;    // clause or variable tiles of the staged form, at most
constexpr int kMiscInts = 48;            // misc_d_: 192 bytes
constexpr int kMiscLaunch = 16;          // misc_d_ index of the per-launch area (byte 64)
constexpr int kMiscAcc2 = 20;            // misc_d_ index of the StepAcc pair (byte 80)
}  // namespace

int64_t Pack::bytes_per(dmm_precision prec, int64_t n, int64_t m, int64_t slots,
                        bool with_alpha_cm) {
  const int64_t t = prec == DMM_FP64 ? 8 : 4;
  n = RangeAlloc::round(std::max<int64_t>(n, 1));
  m = RangeAlloc::round(std::max<int64_t>(m, 1));
  slots = RangeAlloc::round(std::max<int64_t>(slots, 1));
  // per slot: literal, CSR entry, variable-major position (4 each) and the contribution
  int64_t b = m * (3 * t + 4 + (with_alpha_cm ? t : 0)) + slots * (12 + t) + n * (8 * t + 9);
  b += (m / kMinClauseTile + 1) * (8 + 16) + (n / kMinVarTile + 1) * 16;
  b += sizeof(InstDesc) + sizeof(InstCtrl) + 8;
  return b;
}

Pack::~Pack() {
  if (dev_ >= 0) cudaSetDevice(dev_);
  if (stream_) cudaStreamSynchronize(stream_);
  if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
  if (graph_) cudaGraphDestroy(graph_);
  void* ptrs[] = {Xs_,      Xl_,        Cp_,      alpha_cm_,   u_,         cand_,
                  coff_,    lit_,       vslot_,   vend_,       fill_,      unit_,
                  epart_,   inst_d_,    ctrl_d_,  ctiles_d_,   vtiles_d_,  ntiles_d_,
                  queue_d_, active_d_,  ring_d_,  ring_tail_d_, scan_tmp_, longv_d_,
                  stage_,   aux_ctiles_d_, aux_vtiles_d_, flush_, live_d_, misc_d_, order_d_,
                  upos_,    trace_};
  for (void* p : ptrs)
    if (p) dev_free(p);
  for (void* p : xbuf_)
    if (p) dev_free(p);
  for (auto& e : ev_)
    if (e) cudaEventDestroy(e);
  if (pinned_) pinned_free(pinned_);
  if (stream_) cudaStreamDestroy(stream_);
}

dmm_status Pack::init(const PackCaps& caps_in, bool with_alpha_cm, bool fixed_grid) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("no CUDA device");
    return DMM_ERR_NO_DEVICE;
  }
  if (dev_ < 0 || dev_ >= ndev) {
    set_error("device %d out of range (%d devices)", dev_, ndev);
    return DMM_ERR_ARG;
  }
  DMM_CUDA(cudaSetDevice(dev_));
  DMM_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  DMM_CUDA(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev_));
  for (auto& e : ev_) DMM_CUDA(cudaEventCreate(&e));
  with_alpha_cm_ = with_alpha_cm;
  fixed_grid_ = fixed_grid;
  tsize_ = prec_ == DMM_FP64 ? 8 : 4;
  caps_ = caps_in;
  if (caps_.insts < 1) caps_.insts = 1;
  caps_.vars = RangeAlloc::round(caps_.vars) + 32 * (int64_t)caps_.insts;
  caps_.clauses = RangeAlloc::round(caps_.clauses) + 32 * (int64_t)caps_.insts;
  caps_.slots = RangeAlloc::round(caps_.slots) + 32 * (int64_t)caps_.insts;
  const int64_t V = caps_.vars, C = caps_.clauses, S = caps_.slots, I = caps_.insts;
  ctile_cap_ = C / kMinClauseTile + I + 1;
  vtile_cap_ = V / kMinVarTile + I + 1;
  DMM_CUDA(dev_alloc(&Xs_, C * tsize_));
  DMM_CUDA(dev_alloc(&Xl_, C * tsize_));
  DMM_CUDA(dev_alloc(&Cp_, C * tsize_));
  if (with_alpha_cm) DMM_CUDA(dev_alloc(&alpha_cm_, C * tsize_));
  DMM_CUDA(dev_alloc(&coff_, C * 4));
  DMM_CUDA(dev_alloc(&lit_, S * 4));
  // the per-variable lists are read in aligned 16-byte words: padding past the last slot
  DMM_CUDA(dev_alloc(&vslot_, (S + kSlotPad) * 4));
  DMM_CUDA(dev_alloc(&upos_, S * 4));
  DMM_CUDA(dev_alloc(&u_, (S + kSlotPad) * tsize_));
  DMM_CUDA(dev_alloc(&cand_, 2 * kTrials * V * tsize_));
  DMM_CUDA(dev_alloc(&vend_, V * 4));
  DMM_CUDA(dev_alloc(&fill_, V * 4));
  DMM_CUDA(dev_alloc(&unit_, V));
  DMM_CUDA(dev_alloc(&epart_, ctile_cap_ * sizeof(double)));
  DMM_CUDA(dev_alloc(&inst_d_, I * sizeof(InstDesc)));
  DMM_CUDA(dev_alloc(&ctrl_d_, I * sizeof(InstCtrl)));
  DMM_CUDA(dev_alloc(&ctiles_d_, ctile_cap_ * sizeof(Tile)));
  DMM_CUDA(dev_alloc(&vtiles_d_, vtile_cap_ * sizeof(Tile)));
  DMM_CUDA(dev_alloc(&ntiles_d_, 4 * sizeof(int32_t)));
  DMM_CUDA(dev_alloc(&queue_d_, 2 * sizeof(int32_t)));
  DMM_CUDA(dev_alloc(&active_d_, sizeof(int32_t)));
  DMM_CUDA(dev_alloc(&ring_d_, I * sizeof(int32_t)));
  DMM_CUDA(dev_alloc(&ring_tail_d_, 4 * sizeof(int32_t)));
  longv_cap_ = (int32_t)(S / kSortCap + 2);
  DMM_CUDA(dev_alloc(&longv_d_, longv_cap_ * sizeof(int32_t)));
  DMM_CUDA(dev_alloc(&live_d_, I * sizeof(int32_t)));
  DMM_CUDA(dev_alloc(&order_d_, I * sizeof(int32_t)));
  // [0] live formulas, [1] error flag, [3] k_inst queue; bytes 64..191: grid-barrier
  // counter and the two step accumulators of the single-formula form (zeroed per launch)
  DMM_CUDA(dev_alloc(&misc_d_, kMiscInts * sizeof(int32_t)));
  DMM_CUDA(cudaMemsetAsync(misc_d_, 0, kMiscInts * sizeof(int32_t), stream_));
  DMM_CUDA(cudaMemsetAsync(ctrl_d_, 0, I * sizeof(InstCtrl), stream_));
  DMM_CUDA(cudaMemsetAsync(ntiles_d_, 0, 4 * sizeof(int32_t), stream_));
  DMM_CUDA(cudaMemsetAsync(queue_d_, 0, 2 * sizeof(int32_t), stream_));
  DMM_CUDA(cudaMemsetAsync(active_d_, 0, sizeof(int32_t), stream_));
  DMM_CUDA(cudaMemsetAsync(ring_tail_d_, 0, 4 * sizeof(int32_t), stream_));
  DMM_CUDA(cudaMemsetAsync(cand_, 0, 2 * kTrials * V * tsize_, stream_));
  var_alloc_.reset(V);
  cls_alloc_.reset(C);
  slot_alloc_.reset(S);
  inst_h_.assign(I, InstDesc{});
  live_.assign(I, 0);
  add_serial_.assign(I, 0);
  tun_ = dmm_tuning{};
  DMM_TRY(set_tuning(&tun_));
  DMM_CUDA(cudaStreamSynchronize(stream_));
  return DMM_OK;
}

dmm_status Pack::set_tuning(const dmm_tuning* t) {
  dmm_tuning n = *t;
  if (n.clause_tile < 0 || (n.clause_tile > 0 && (n.clause_tile % 4 || n.clause_tile < kMinClauseTile))) {
    set_error("clause_tile must be 0 (balanced) or a multiple of 4 that is >= %d", kMinClauseTile);
    return DMM_ERR_ARG;
  }
  if (n.var_tile < 0 || (n.var_tile > 0 && n.var_tile < kMinVarTile)) {
    set_error("var_tile must be 0 (balanced) or >= %d", kMinVarTile);
    return DMM_ERR_ARG;
  }
  if (prec_ == DMM_FP64) {
    if (n.var_group != 0 && n.var_group != 32) {
      set_error("FP64 mode reduces with one warp per variable (var_group 32)");
      return DMM_ERR_ARG;
    }
    n.var_group = 32;
  } else {
    if (n.var_group <= 0) n.var_group = 4;
    if (n.var_group != 1 && n.var_group != 2 && n.var_group != 4 && n.var_group != 8 &&
        n.var_group != 16 && n.var_group != 32) {
      set_error("var_group must be 1, 2, 4, 8, 16 or 32");
      return DMM_ERR_ARG;
    }
  }
  if (n.steps_per_graph <= 0) n.steps_per_graph = 32;
  if (n.steps_per_graph > 4096) n.steps_per_graph = 4096;
  if (n.blocks_per_sm < 0 || n.blocks_per_sm > 32) {
    set_error("blocks_per_sm out of range");
    return DMM_ERR_ARG;
  }
  if (n.l2_policy < 0 || n.l2_policy > 3) {
    set_error("l2_policy must be 0..3 (bit 0: no eviction hints, bit 1: L2 prefetch)");
    return DMM_ERR_ARG;
  }
  if (n.u_layout < 0 || n.u_layout > 2) {
    set_error("u_layout must be 0 (default), 1 (slot-major, no staging) or 2 (variable-major)");
    return DMM_ERR_ARG;
  }
  if (n.launch_mode < 0 || n.launch_mode > 3) {
    set_error("launch_mode must be 0 (auto), 1 (kernel per phase), 2 (cooperative tiles) or "
              "3 (one block per small formula)");
    return DMM_ERR_ARG;
  }
  tun_ = n;
  graph_stale_ = true;
  if (!ctiles_h_.empty() || !vtiles_h_.empty()) return commit_tiles();
  return DMM_OK;
}

int32_t Pack::num_live() const {
  int32_t c = 0;
  for (auto l : live_) c += l;
  return c;
}

int32_t Pack::free_insts() const {
  int32_t c = 0;
  for (auto l : live_) c += !l;
  return c;
}

dmm_status Pack::ensure_stage(int64_t doubles) {
  if (doubles <= stage_cap_) return DMM_OK;
  if (stage_) retire(stage_);
  stage_ = nullptr;
  stage_cap_ = 0;
  DMM_CUDA(dev_alloc(&stage_, doubles * sizeof(double)));
  stage_cap_ = doubles;
  return DMM_OK;
}

void Pack::retire(void* p) {
  // the block may still be read by work queued on this pack's stream, and the cache can
  // hand it to another stream at once
  cudaStreamSynchronize(stream_);
  dev_free(p);
}

// Small records travel as kernel arguments: stream-ordered, no host staging, no wait.
__global__ void k_put_desc(InstDesc* dst, InstDesc d) { *dst = d; }
__global__ void k_put_ctrl(InstCtrl* dst, InstCtrl c) { *dst = c; }

// Signs of V on the device (the control record says which candidate holds it), so that
// one byte per variable crosses to the host: pre from the solving step's V (0 for V == 0;
// flag[0] = 1 when the formula is not solved), post from the current V (+1 / -1).
template <class T>
__global__ void k_signs(const InstCtrl* __restrict__ ctrl, const T* __restrict__ cand,
                        int64_t var_cap, int64_t var0, int n, int8_t* pre, int8_t* post,
                        int32_t* flag) {
  const InstCtrl c = *ctrl;
  if (pre && c.solved_step < 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *flag = 1;
    pre = nullptr;
  }
  const T* vs = cand + (int64_t)(c.sol_set * kTrials + c.sol_k) * var_cap + var0;
  const T* vc = cand + (int64_t)(c.set * kTrials + c.kcur) * var_cap + var0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (pre) {
      const T v = vs[i];
      pre[i] = v > T(0) ? 1 : (v < T(0) ? -1 : 0);
    }
    if (post) post[i] = vc[i] > T(0) ? 1 : -1;
  }
}


dmm_status Pack::upload_desc(int32_t idx) {
  k_put_desc<<<1, 1, 0, stream_>>>(inst_d_ + idx, inst_h_[idx]);
  DMM_CUDA(cudaGetLastError());
  return DMM_OK;
}

dmm_status Pack::write_ctrl(int32_t idx, const InstCtrl& c) {
  k_put_ctrl<<<1, 1, 0, stream_>>>(ctrl_d_ + idx, c);
  DMM_CUDA(cudaGetLastError());
  return DMM_OK;
}

__global__ void k_active_add(int32_t* a, int32_t d) { atomicAdd(a, d); }

dmm_status Pack::add_active(int32_t delta) {
  k_active_add<<<1, 1, 0, stream_>>>(active_d_, delta);
  DMM_CUDA(cudaGetLastError());
  return DMM_OK;
}

dmm_status Pack::read_ctrl(int32_t idx, InstCtrl* c) {
  if (!live(idx)) {
    set_error("instance %d is not live", idx);
    return DMM_ERR_ARG;
  }
  DMM_CUDA(cudaMemcpyAsync(c, ctrl_d_ + idx, sizeof(InstCtrl), cudaMemcpyDeviceToHost, stream_));
  DMM_CUDA(cudaStreamSynchronize(stream_));
  return DMM_OK;
}

dmm_status Pack::read_ctrls(std::vector<InstCtrl>* out) {
  out->resize(caps_.insts);
  DMM_CUDA(cudaMemcpyAsync(out->data(), ctrl_d_, caps_.insts * sizeof(InstCtrl),
                           cudaMemcpyDeviceToHost, stream_));
  DMM_CUDA(cudaStreamSynchronize(stream_));
  return DMM_OK;
}

static dmm_status scan_inclusive(int32_t* a, int64_t len, int32_t* tmp, cudaStream_t s) {
  constexpr int per = kThreads * 8;
  const int64_t nb = (len + per - 1) / per;
  if (nb <= 1) {
    k_scan_block<<<1, kThreads, 0, s>>>(a, (int)len, nullptr);
    DMM_CUDA(cudaGetLastError());
    return DMM_OK;
  }
  k_scan_block<<<(unsigned)nb, kThreads, 0, s>>>(a, (int)len, tmp);
  DMM_CUDA(cudaGetLastError());
  DMM_TRY(scan_inclusive(tmp, nb, tmp + nb, s));
  k_scan_add<<<(unsigned)nb, kThreads, 0, s>>>(a, (int)len, tmp);
  DMM_CUDA(cudaGetLastError());
  return DMM_OK;
}

dmm_status Pack::build_csr(const InstDesc& I, const int32_t* lits_host) {
  const int n = I.n, L = I.nslots;
  int32_t* vend = vend_ + I.var0;
  int32_t* fill = fill_ + I.var0;
  const int32_t* lit = lit_ + I.slot0;
  int32_t* vsl = vslot_ + I.slot0;
  DMM_CUDA(cudaMemsetAsync(vend, 0, (size_t)n * 4, stream_));
  if (L > 0) {
    k_count<<<blocks_for(L), kThreads, 0, stream_>>>(lit, L, n, vend, ring_tail_d_ + 3);
    DMM_CUDA(cudaGetLastError());
  }
  const int64_t need = n / (kThreads * 8) + 64;
  if (need > scan_tmp_cap_) {
    if (scan_tmp_) retire(scan_tmp_);
    scan_tmp_ = nullptr;
    DMM_CUDA(dev_alloc(&scan_tmp_, need * 2 * sizeof(int32_t)));
    scan_tmp_cap_ = need;
  }
  DMM_TRY(scan_inclusive(vend, n, scan_tmp_, stream_));
  k_fill_start<<<blocks_for(n), kThreads, 0, stream_>>>(vend, n, fill);
  DMM_CUDA(cudaGetLastError());
  if (L > 0) {
    k_scatter<<<blocks_for(L), kThreads, 0, stream_>>>(lit, L, n, fill, vsl);
    DMM_CUDA(cudaGetLastError());
  }
  // lists longer than the shared-memory sorter are appended to longv_d_ (count at
  // ring_tail_d_[2]) and sorted by resolve_long_lists() before the CSR is first used, so
  // that adding a formula needs no host synchronization
  const size_t smem = (kThreads / 32) * kSortCap * sizeof(int32_t);
  k_sort_lists<<<blocks_for(n, kThreads / 32), kThreads, smem, stream_>>>(
      vend, n, vsl, longv_d_, ring_tail_d_ + 2, (int32_t)I.var0, longv_cap_);
  DMM_CUDA(cudaGetLastError());
  long_pending_ = true;
  if (L > 0) {
    // variable-major position of every slot (the inverse of the sorted CSR)
    k_invert<<<blocks_for(L), kThreads, 0, stream_>>>(vsl, L, upos_ + I.slot0);
    DMM_CUDA(cudaGetLastError());
  }
  (void)lits_host;
  return DMM_OK;
}

dmm_status Pack::resolve_long_lists() {
  if (!long_pending_) return DMM_OK;
  int32_t counts[2] = {0, 0};  // long lists, literals the CSR build found out of range
  DMM_CUDA(cudaMemcpyAsync(counts, ring_tail_d_ + 2, sizeof counts, cudaMemcpyDeviceToHost,
                           stream_));
  DMM_CUDA(cudaStreamSynchronize(stream_));
  const int32_t nlong = counts[0];
  if (counts[1] > 0) {
    // a formula admitted with device_literal_check holds a bad literal: name it as the host
    // check would, then leave the counters for the caller to discard the pack
    for (int32_t i = 0; i < (int32_t)live_.size(); i++) {
      if (!live_[i]) continue;
      const InstDesc& I = inst_h_[i];
      std::vector<int32_t> h(I.nslots);
      DMM_CUDA(cudaMemcpy(h.data(), lit_ + I.slot0, (size_t)I.nslots * 4, cudaMemcpyDeviceToHost));
      DMM_TRY(locate_bad_literal(h.data(), I.nslots, I.n));
    }
    set_error("formula: %d literals out of range", counts[1]);
    return DMM_ERR_LITERAL;
  }
  if (nlong > 0) {
    // sorted on the host (setup only); an entry whose formula was removed meanwhile is
    // skipped, one whose range a later formula took is sorted again (harmless).  Past the
    // list's capacity (formulas with long lists added and removed repeatedly before a
    // commit) every long list of every live formula is taken.
    std::vector<int32_t> ids;
    if (nlong <= longv_cap_) {
      ids.resize(nlong);
      DMM_CUDA(cudaMemcpy(ids.data(), longv_d_, nlong * 4, cudaMemcpyDeviceToHost));
    } else {
      for (int32_t i = 0; i < (int32_t)live_.size(); i++) {
        if (!live_[i]) continue;
        const InstDesc& I = inst_h_[i];
        std::vector<int32_t> ends(I.n);
        DMM_CUDA(cudaMemcpy(ends.data(), vend_ + I.var0, (size_t)I.n * 4, cudaMemcpyDeviceToHost));
        for (int32_t v = 0; v < I.n; v++)
          if (ends[v] - (v > 0 ? ends[v - 1] : 0) > kSortCap) ids.push_back((int32_t)I.var0 + v);
      }
    }
    std::vector<int32_t> redo;
    std::vector<int32_t> seg;
    for (int32_t g : ids) {
      int32_t owner = -1;
      for (int32_t i = 0; i < (int32_t)live_.size(); i++)
        if (live_[i] && g >= inst_h_[i].var0 && g < inst_h_[i].var0 + inst_h_[i].n) owner = i;
      if (owner < 0) continue;
      const InstDesc& I = inst_h_[owner];
      const int32_t v = g - (int32_t)I.var0;
      int32_t e[2] = {0, 0};
      if (v > 0)
        DMM_CUDA(cudaMemcpy(e, vend_ + I.var0 + v - 1, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost));
      else
        DMM_CUDA(cudaMemcpy(e + 1, vend_ + I.var0, sizeof(int32_t), cudaMemcpyDeviceToHost));
      int32_t* vsl = vslot_ + I.slot0;
      seg.resize(e[1] - e[0]);
      DMM_CUDA(cudaMemcpy(seg.data(), vsl + e[0], seg.size() * 4, cudaMemcpyDeviceToHost));
      std::sort(seg.begin(), seg.end());
      DMM_CUDA(cudaMemcpy(vsl + e[0], seg.data(), seg.size() * 4, cudaMemcpyHostToDevice));
      if (std::find(redo.begin(), redo.end(), owner) == redo.end()) redo.push_back(owner);
    }
    for (int32_t i : redo) {
      const InstDesc& I = inst_h_[i];
      k_invert<<<blocks_for(I.nslots), kThreads, 0, stream_>>>(vslot_ + I.slot0, I.nslots,
                                                               upos_ + I.slot0);
      DMM_CUDA(cudaGetLastError());
    }
    DMM_CUDA(cudaMemsetAsync(ring_tail_d_ + 2, 0, sizeof(int32_t), stream_));
  }
  long_pending_ = false;
  return DMM_OK;
}

static double effective_xl_max(int32_t factor, int32_t m) {
  int32_t v = (int32_t)((uint32_t)factor * (uint32_t)m);  // dynex.cc:2358 in int arithmetic
  if (v <= 0) v = 0x7fffffff;
  return (double)v;
}

static void fill_params(InstDesc& I, const dmm_params* p) {
  dmm_params d;
  dmm_params_default(&d);
  if (!p) p = &d;
  I.alpha = p->alpha;
  I.beta = p->beta;
  I.gamma = p->gamma;
  I.delta = p->delta;
  I.eps = p->epsilon;
  I.zeta = p->zeta;
  I.xl_max = effective_xl_max(p->xl_max, I.m);
}

// Copies from pageable host memory have read their source when cudaMemcpyAsync returns;
// from page-locked memory they run later, so a call that copies from a caller's
// page-locked buffer waits for its stream before returning (the caller may reuse it).
static bool page_locked(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;  // unknown: treat as page-locked
  }
  return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeManaged;
}

template <class T>
static dmm_status upload_alpha(T* dst, const double* a, int32_t m, cudaStream_t s) {
  std::vector<T> h(m);
  for (int32_t i = 0; i < m; i++) h[i] = T(a[i]);
  DMM_CUDA(cudaMemcpyAsync(dst, h.data(), (size_t)m * sizeof(T), cudaMemcpyHostToDevice, s));
  DMM_CUDA(cudaStreamSynchronize(s));
  return DMM_OK;
}

dmm_status Pack::add(const int32_t* lits, const int64_t* clause_off, int32_t n, int32_t m,
                     const dmm_params* p, const double* alpha_cm, int32_t max_steps,
                     int32_t* idx_out, const double* x0, bool device_literal_check) {
  DMM_TRY(validate_shape(lits, clause_off, n, m));
  if (alpha_cm && !with_alpha_cm_) {
    set_error("this pack was created without per-clause alpha storage");
    return DMM_ERR_ARG;
  }
  DMM_CUDA(cudaSetDevice(dev_));
  int32_t idx = -1;
  for (int32_t i = 0; i < (int32_t)live_.size(); i++)
    if (!live_[i]) {
      idx = i;
      break;
    }
  if (idx < 0) {
    set_error("pack is full (%d instances)", caps_.insts);
    return DMM_ERR_BUDGET;
  }
  const int64_t L = clause_off[m];
  const int64_t var0 = var_alloc_.alloc(n);
  const int64_t cls0 = var0 < 0 ? -1 : cls_alloc_.alloc(m);
  const int64_t slot0 = cls0 < 0 ? -1 : slot_alloc_.alloc(L);
  if (var0 < 0 || cls0 < 0 || slot0 < 0) {
    if (var0 >= 0) var_alloc_.free(var0, n);
    if (cls0 >= 0) cls_alloc_.free(cls0, m);
    set_error("pack capacity exhausted (n=%d m=%d literals=%lld)", n, m, (long long)L);
    return DMM_ERR_BUDGET;
  }
  // the literal upload runs while the host checks the clauses (and literals)
  if (L > 0)
    DMM_CUDA(cudaMemcpyAsync(lit_ + slot0, lits, (size_t)L * 4, cudaMemcpyHostToDevice, stream_));
  InstDesc I{};
  I.n = n;
  I.m = m;
  I.var0 = var0;
  I.cls0 = cls0;
  I.slot0 = slot0;
  I.nslots = (int32_t)L;
  // with the literals checked on the device the occurrence lists need nothing from the
  // host pass: they build while the host checks the clause offsets
  if (device_literal_check) DMM_TRY(build_csr(I, lits));
  bool k3 = false, units = true;
  const dmm_status vst =
      validate_formula(lits, clause_off, n, m, &k3, &units, !device_literal_check);
  if (vst != DMM_OK) {
    cudaStreamSynchronize(stream_);
    var_alloc_.free(var0, n);
    cls_alloc_.free(cls0, m);
    slot_alloc_.free(slot0, L);
    return vst;
  }
  I.k3 = k3 ? 1 : 0;
  I.has_alpha_cm = alpha_cm ? 1 : 0;
  I.max_steps = max_steps;
  fill_params(I, p);
  std::vector<int32_t> coff_local;
  if (!k3 && m > 0) {
    coff_local.resize(m);
    for (int32_t c = 0; c < m; c++) coff_local[c] = (int32_t)clause_off[c];
    DMM_CUDA(cudaMemcpyAsync(coff_ + cls0, coff_local.data(), (size_t)m * 4,
                             cudaMemcpyHostToDevice, stream_));
  }
  // unit clauses (dynex.cc:2459-2469: the last unit clause of a variable wins)
  if (units) {
    unit_h_.assign(n, 0);
    for (int32_t c = 0; c < m; c++)
      if (clause_off[c + 1] - clause_off[c] == 1) {
        const int32_t l = lits[clause_off[c]];
        if (l == 0 || l > n || l < -n) continue;  // unchecked literal: the device check reports it
        unit_h_[std::abs(l) - 1] = l > 0 ? 1 : -1;
      }
    DMM_CUDA(cudaMemcpyAsync(unit_ + var0, unit_h_.data(), n, cudaMemcpyHostToDevice, stream_));
  } else {
    DMM_CUDA(cudaMemsetAsync(unit_ + var0, 0, n, stream_));
  }
  if (alpha_cm) {
    if (prec_ == DMM_FP64)
      DMM_TRY(upload_alpha(static_cast<double*>(alpha_cm_) + cls0, alpha_cm, m, stream_));
    else
      DMM_TRY(upload_alpha(static_cast<float*>(alpha_cm_) + cls0, alpha_cm, m, stream_));
  }
  if (!device_literal_check) DMM_TRY(build_csr(I, lits));
  inst_h_[idx] = I;
  live_[idx] = 1;
  add_serial_[idx] = ++add_counter_;
  DMM_TRY(upload_desc(idx));
  InstCtrl c{};
  c.done = DMM_CANCELLED;  // not runnable until a state is set
  c.best_loc = m;
  c.loc = m;
  c.solved_step = -1;
  c.solved_t = -1.0;
  c.h_state = 0.125;
  if (x0) {
    // runnable at once: the state set_state would upload, without reading the control
    // record back (it is the one written here)
    const dmm_status st = upload_state(I, x0);
    if (st != DMM_OK) {
      write_ctrl(idx, c);
      var_alloc_.free(var0, n);
      cls_alloc_.free(cls0, m);
      slot_alloc_.free(slot0, L);
      live_[idx] = 0;
      return st;
    }
    DMM_TRY(write_ctrl(idx, running_ctrl(I, 0.0, 0)));
    DMM_TRY(add_active(+1));
  } else {
    DMM_TRY(write_ctrl(idx, c));
  }
  if (!fixed_grid_) graph_stale_ = true;
  if (page_locked(lits) || page_locked(x0)) DMM_CUDA(cudaStreamSynchronize(stream_));
  *idx_out = idx;
  return DMM_OK;
}

dmm_status Pack::remove(int32_t idx) {
  if (!live(idx)) {
    set_error("instance %d is not live", idx);
    return DMM_ERR_ARG;
  }
  InstCtrl c;
  DMM_TRY(read_ctrl(idx, &c));
  if (c.done == 0) {
    DMM_TRY(add_active(-1));
    c.done = DMM_CANCELLED;
    DMM_TRY(write_ctrl(idx, c));
  }
  const InstDesc& I = inst_h_[idx];
  var_alloc_.free(I.var0, I.n);
  cls_alloc_.free(I.cls0, I.m);
  slot_alloc_.free(I.slot0, I.nslots);
  live_[idx] = 0;
  if (!fixed_grid_) graph_stale_ = true;
  return DMM_OK;
}

dmm_status Pack::set_params(int32_t idx, const dmm_params* p, const double* alpha_cm) {
  if (!live(idx)) return DMM_ERR_ARG;
  if (alpha_cm && !with_alpha_cm_) {
    set_error("this pack was created without per-clause alpha storage");
    return DMM_ERR_ARG;
  }
  InstDesc& I = inst_h_[idx];
  fill_params(I, p);
  I.has_alpha_cm = alpha_cm ? 1 : 0;
  if (alpha_cm) {
    if (prec_ == DMM_FP64)
      DMM_TRY(upload_alpha(static_cast<double*>(alpha_cm_) + I.cls0, alpha_cm, I.m, stream_));
    else
      DMM_TRY(upload_alpha(static_cast<float*>(alpha_cm_) + I.cls0, alpha_cm, I.m, stream_));
  }
  DMM_TRY(upload_desc(idx));
  DMM_CUDA(cudaStreamSynchronize(stream_));
  return DMM_OK;
}

dmm_status Pack::set_max_steps(int32_t idx, int32_t max_steps) {
  if (!live(idx)) return DMM_ERR_ARG;
  inst_h_[idx].max_steps = max_steps;
  DMM_TRY(upload_desc(idx));
  return DMM_OK;
}

dmm_status Pack::set_state(int32_t idx, const double* x) {
  return set_state_at(idx, x, 0.0, 0, false);
}

dmm_status Pack::set_state_at(int32_t idx, const double* x, double t, int32_t step,
                              bool keep_best) {
  if (!live(idx) || !x || step < 0) {
    set_error("set_state: bad instance or null state");
    return DMM_ERR_ARG;
  }
  const InstDesc& I = inst_h_[idx];
  InstCtrl old;
  DMM_TRY(read_ctrl(idx, &old));
  DMM_TRY(upload_state(I, x));
  InstCtrl c = running_ctrl(I, t, step);
  if (keep_best) {
    c.best_loc = old.best_loc;
    c.best_t = old.best_t;
  }
  if (old.done != 0) DMM_TRY(add_active(+1));
  DMM_TRY(write_ctrl(idx, c));
  if (page_locked(x)) DMM_CUDA(cudaStreamSynchronize(stream_));
  return DMM_OK;
}

dmm_status Pack::upload_state(const InstDesc& I, const double* x) {
  const int64_t N = (int64_t)I.n + 2 * (int64_t)I.m;
  DMM_TRY(ensure_stage(3 * N));
  DMM_CUDA(cudaMemcpyAsync(stage_, x, N * sizeof(double), cudaMemcpyHostToDevice, stream_));
  if (prec_ == DMM_FP64) {
    double* V = static_cast<double*>(cand_) + I.var0;
    k_set_state<double><<<blocks_for(N), kThreads, 0, stream_>>>(
        stage_, I.n, I.m, V, static_cast<double*>(Xs_) + I.cls0, static_cast<double*>(Xl_) + I.cls0);
  } else {
    float* V = static_cast<float*>(cand_) + I.var0;
    k_set_state<float><<<blocks_for(N), kThreads, 0, stream_>>>(
        stage_, I.n, I.m, V, static_cast<float*>(Xs_) + I.cls0, static_cast<float*>(Xl_) + I.cls0);
  }
  DMM_CUDA(cudaGetLastError());
  return DMM_OK;
}

InstCtrl Pack::running_ctrl(const InstDesc& I, double t, int32_t step) {
  InstCtrl c{};
  c.done = 0;
  c.step = step;
  c.t = t;
  c.loc = I.m;
  c.best_loc = I.m;
  c.best_t = 0.0;
  c.solved_step = -1;
  c.solved_t = -1.0;
  c.h_state = 0.125;
  return c;
}

dmm_status Pack::get_state(int32_t idx, double* x, double* t) {
  if (!live(idx)) return DMM_ERR_ARG;
  const InstDesc& I = inst_h_[idx];
  const int64_t N = (int64_t)I.n + 2 * (int64_t)I.m;
  DMM_TRY(ensure_stage(3 * N));
  if (prec_ == DMM_FP64) {
    k_get_state<double><<<blocks_for(N), kThreads, 0, stream_>>>(
        inst_d_, ctrl_d_, idx, static_cast<double*>(cand_), caps_.vars, static_cast<double*>(Xs_),
        static_cast<double*>(Xl_), static_cast<double*>(Cp_), static_cast<double*>(alpha_cm_), stage_);
  } else {
    k_get_state<float><<<blocks_for(N), kThreads, 0, stream_>>>(
        inst_d_, ctrl_d_, idx, static_cast<float*>(cand_), caps_.vars, static_cast<float*>(Xs_),
        static_cast<float*>(Xl_), static_cast<float*>(Cp_), static_cast<float*>(alpha_cm_), stage_);
  }
  DMM_CUDA(cudaGetLastError());
  if (x) DMM_CUDA(cudaMemcpyAsync(x, stage_, N * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  DMM_CUDA(cudaStreamSynchronize(stream_));
  if (t) {
    InstCtrl c;
    DMM_TRY(read_ctrl(idx, &c));
    *t = c.t;
  }
  return DMM_OK;
}

template <class T>
void Pack::fill_view(void* vv) const {
  PackView<T>& v = *static_cast<PackView<T>*>(vv);
  v.Xs = static_cast<T*>(Xs_);
  v.Xl = static_cast<T*>(Xl_);
  v.Cp = static_cast<T*>(Cp_);
  v.alpha_cm = static_cast<const T*>(alpha_cm_);
  v.coff = coff_;
  v.lit = lit_;
  v.u = static_cast<T*>(u_);
  v.vslot = vslot_;
  v.vend = vend_;
  v.cand = static_cast<T*>(cand_);
  v.var_cap = caps_.vars;
  v.unit = unit_;
  v.epart = epart_;
  v.inst = inst_d_;
  v.ctrl = ctrl_d_;
  v.ctiles = use_aux_ ? aux_ctiles_d_ : ctiles_d_;
  v.vtiles = use_aux_ ? aux_vtiles_d_ : vtiles_d_;
  v.ntiles = use_aux_ ? ntiles_d_ + 2 : ntiles_d_;
  v.queue = queue_d_;
  v.active = active_d_;
  v.ring = ring_d_;
  v.ring_tail = ring_tail_d_;
  v.ring_cap = caps_.insts;
  v.live = live_d_;
  v.live0 = live0_;
  v.nlive = misc_d_;
  v.acc2 = reinterpret_cast<StepAcc*>(misc_d_ + kMiscAcc2);
  // tile paths: slot-major unless asked (measured faster there); the one-block-per-formula
  // kernel switches to variable-major by default in launch_inst
  v.upos = tun_.u_layout == 2 ? upos_ : nullptr;
  v.xdlist = xp_active_ ? static_cast<const int32_t*>(xbuf_[kXpDlist]) : nullptr;
  v.xdoff = static_cast<const int32_t*>(xbuf_[kXpDoff]);
  v.xllit = static_cast<const int16_t*>(xbuf_[kXpLlit]);
  v.xspos = static_cast<const uint16_t*>(xbuf_[kXpSpos]);
  v.ux = static_cast<T*>(xbuf_[kXpUx]);
  v.xubase = static_cast<const int32_t*>(xbuf_[kXpUbase]);
  v.xboff = static_cast<const int32_t*>(xbuf_[kXpBoff]);
  v.xsrc8 = static_cast<const int32_t*>(xbuf_[kXpSrc8]);
  v.xdst = static_cast<const uint16_t*>(xbuf_[kXpDst]);
  v.xsv_cap = xsv_cap_;
  v.xbk_cap = xbk_cap_;
  v.xtv_cap = xtv_cap_;
  v.xst_cap = xst_cap_;
  v.xl2_plain = tun_.l2_policy & 1;
  v.xprefetch = (tun_.l2_policy & 2) != 0;
  v.barrier_extra = barrier_extra_;
  v.trace = trace_on_ ? trace_ : nullptr;
  v.trace_steps = trace_on_ ? trace_steps_ : 0;
}

dmm_status Pack::enqueue_clause() {
  if (prec_ == DMM_FP64) {
    PackView<double> v;
    fill_view<double>(&v);
    k_clause<double, false><<<grid_c_, kThreads, 0, stream_>>>(v);
  } else {
    PackView<float> v;
    fill_view<float>(&v);
    k_clause<float, true><<<grid_c_, kThreads, 0, stream_>>>(v);
  }
  DMM_CUDA(cudaGetLastError());
  return DMM_OK;
}

template <int MODE>
static void launch_var_f32(int G, int grid, cudaStream_t s, const PackView<float>& v, double* dv) {
  switch (G) {
    case 1: k_var<float, 1, false, MODE><<<grid, kThreads, 0, s>>>(v, dv); break;
    case 2: k_var<float, 2, false, MODE><<<grid, kThreads, 0, s>>>(v, dv); break;
    case 4: k_var<float, 4, false, MODE><<<grid, kThreads, 0, s>>>(v, dv); break;
    case 8: k_var<float, 8, false, MODE><<<grid, kThreads, 0, s>>>(v, dv); break;
    case 16: k_var<float, 16, false, MODE><<<grid, kThreads, 0, s>>>(v, dv); break;
    default: k_var<float, 32, false, MODE><<<grid, kThreads, 0, s>>>(v, dv); break;
  }
}

dmm_status Pack::enqueue_var(bool rhs_only, void* dv_out) {
  double* dv = static_cast<double*>(dv_out);
  if (prec_ == DMM_FP64) {
    PackView<double> v;
    fill_view<double>(&v);
    if (rhs_only)
      k_var<double, 32, true, 1><<<grid_v_, kThreads, 0, stream_>>>(v, dv);
    else
      k_var<double, 32, true, 0><<<grid_v_, kThreads, 0, stream_>>>(v, dv);
  } else {
    PackView<float> v;
    fill_view<float>(&v);
    if (rhs_only)
      launch_var_f32<1>(tun_.var_group, grid_v_, stream_, v, dv);
    else
      launch_var_f32<0>(tun_.var_group, grid_v_, stream_, v, dv);
  }
  DMM_CUDA(cudaGetLastError());
  return DMM_OK;
}

dmm_status Pack::enqueue_step(bool rhs_only, void* dv_out) {
  DMM_TRY(enqueue_clause());
  DMM_TRY(enqueue_var(rhs_only, dv_out));
  return DMM_OK;
}

static int occupancy_blocks(const void* fn, int threads, size_t smem = 0) {
  int b = 1;
  if (smem > 0 &&
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, threads, smem) != cudaSuccess) {
    cudaGetLastError();
    b = 4;
  }
  return std::max(1, b);
}

// ONE: single-formula form
template <bool ONE>
static const void* persist_fn_x(dmm_precision prec, int G) {
  if (prec == DMM_FP64)
    return (const void*)k_persist<double, 32, true, false, kPersistThreads64, ONE>;
  switch (G) {
    case 1: return (const void*)k_persist<float, 1, false, true, kPersistThreads, ONE>;
    case 2: return (const void*)k_persist<float, 2, false, true, kPersistThreads, ONE>;
    case 4: return (const void*)k_persist<float, 4, false, true, kPersistThreads, ONE>;
    case 8: return (const void*)k_persist<float, 8, false, true, kPersistThreads, ONE>;
    case 16: return (const void*)k_persist<float, 16, false, true, kPersistThreads, ONE>;
    default: return (const void*)k_persist<float, 32, false, true, kPersistThreads, ONE>;
  }
}

// the staged form (FP32, single formula); mt: several tiles per block
template <bool MT>
static const void* staged_fn_x(int G) {
  switch (G) {
    case 1: return (const void*)k_staged<1, kStagedThreads, MT>;
    case 2: return (const void*)k_staged<2, kStagedThreads, MT>;
    case 4: return (const void*)k_staged<4, kStagedThreads, MT>;
    case 8: return (const void*)k_staged<8, kStagedThreads, MT>;
    case 16: return (const void*)k_staged<16, kStagedThreads, MT>;
    default: return (const void*)k_staged<32, kStagedThreads, MT>;
  }
}
static const void* staged_fn(int G, bool mt) {
  return mt ? staged_fn_x<true>(G) : staged_fn_x<false>(G);
}

const void* Pack::persist_fn() const {
  if (xp_active_) return staged_fn(tun_.var_group, xp_mt_);
  if (one_active_) return persist_fn_x<true>(prec_, tun_.var_group);
  return persist_fn_x<false>(prec_, tun_.var_group);
}

// Tables of the staged form (dmm_xpose.cuh) for formula idx with clause tiles of TC and
// variable tiles of TV, built on the device (dmm_xprep.cuh); mt: the several-tiles-per-block
// form (the tile lists must hold that tiling).  Leaves *ok false (and the plain tile code in
// use) when the formula or its tiles do not fit the form's 16-bit indices or shared memory.
dmm_status Pack::prepare_xpose(int32_t idx, int TC, int TV, bool mt, bool* ok) {
  *ok = false;
  const InstDesc& I = inst_h_[idx];
  if (prec_ != DMM_FP32 || !I.k3) return DMM_OK;
  // the tables of the same formula at the same place with the same tiles are still valid
  // (only this function writes them, and a live formula's device arrays do not change)
  const XpKey key{idx, I.var0, I.slot0, I.n, I.m, TC, TV, tun_.var_group, mt, add_serial_[idx]};
  if (xp_key_valid_ && key == xp_key_) {
    *ok = true;
    return DMM_OK;
  }
  xp_key_valid_ = false;
  const int m = I.m, n = I.n, L = I.nslots;
  const int nct = (m + TC - 1) / TC, nvt = (n + TV - 1) / TV;
  if (nct <= 0 || nvt <= 0) return DMM_OK;
  if (!mt && (nct > grid_p_ || nvt > grid_p_)) return DMM_OK;
  if (nct > kXpMaxTiles || nvt > kXpMaxTiles) return DMM_OK;
  const int W = (n + 31) / 32;
  const int RW = std::min(W, kXpRangeWords);
  const int smem_k = (nvt + 2 * RW) * 4;
  if (smem_k > kXpSmemMax) return DMM_OK;
  const int64_t pairs = (int64_t)nct * nvt;
  const int64_t ux_cap = (int64_t)L + 8 * pairs;  // sector padding: < 8 per chunk
  if (ux_cap > INT32_MAX / 2) return DMM_OK;
  // scratch: cnt, sb, bt (pairs each), st, dcnt (nct each), btot (nvt), out (8)
  const int64_t scratch_ints = 3 * pairs + 2 * (int64_t)nct + nvt + 8;
  const int64_t bytes[kXpBufs] = {
      ((int64_t)L + 4 * nct) * 4,  // dlist
      2 * (int64_t)nct * 4,        // doff
      (int64_t)L * 2,              // llit
      (int64_t)L * 2,              // spos
      ux_cap * 4,                  // ux
      ((int64_t)nct + 1) * 4,      // ubase
      ((int64_t)nvt + 1) * 4,      // boff
      (ux_cap / 8 + 1) * 4,        // src8
      ux_cap * 2,                  // dst
      scratch_ints * 4};           // scratch
  for (int i = 0; i < kXpBufs; i++) {
    const int64_t want = std::max<int64_t>(bytes[i], 16);
    if (want > xbuf_cap_[i]) {
      if (xbuf_[i]) retire(xbuf_[i]);
      xbuf_[i] = nullptr;
      xbuf_cap_[i] = 0;
      DMM_CUDA(dev_alloc(&xbuf_[i], want));
      xbuf_cap_[i] = want;
    }
  }
  int* scr = static_cast<int*>(xbuf_[kXpScratch]);
  int* cnt = scr;
  int* sb = cnt + pairs;
  int* bt = sb + pairs;
  int* st = bt + pairs;
  int* dcnt = st + nct;
  int* btot = dcnt + nct;
  int* out = btot + nvt;
  auto* dlist = static_cast<int32_t*>(xbuf_[kXpDlist]);
  auto* doff = static_cast<int32_t*>(xbuf_[kXpDoff]);
  auto* llit = static_cast<int16_t*>(xbuf_[kXpLlit]);
  auto* spos = static_cast<uint16_t*>(xbuf_[kXpSpos]);
  auto* ubase = static_cast<int32_t*>(xbuf_[kXpUbase]);
  auto* boff = static_cast<int32_t*>(xbuf_[kXpBoff]);
  auto* src8 = static_cast<int32_t*>(xbuf_[kXpSrc8]);
  auto* dst = static_cast<uint16_t*>(xbuf_[kXpDst]);
  const int32_t* lit = lit_ + I.slot0;
  const int32_t* upos = upos_ + I.slot0;
  const int32_t* vend = vend_ + I.var0;
  DMM_CUDA(cudaMemsetAsync(dlist, 0, bytes[kXpDlist], stream_));
  DMM_CUDA(cudaMemsetAsync(dst, 0xFF, bytes[kXpDst], stream_));
  if (smem_k > 48 * 1024) {
    DMM_CUDA(cudaFuncSetAttribute(k_xp_count<kXprepThreads>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, smem_k));
    DMM_CUDA(cudaFuncSetAttribute(k_xp_fill<kXprepThreads>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, smem_k));
  }
  k_xp_count<kXprepThreads><<<nct, kXprepThreads, smem_k, stream_>>>(lit, L, TC, TV, nvt, n, RW,
                                                                     cnt, sb, st, dcnt, spos);
  k_xp_scan<kXprepThreads><<<1, kXprepThreads, 0, stream_>>>(nct, nvt, cnt, st, dcnt, ubase,
                                                             doff, bt, boff, btot, out);
  k_xp_fill<kXprepThreads><<<nct, kXprepThreads, smem_k, stream_>>>(
      lit, upos, vend, L, TC, TV, nct, nvt, n, RW, sb, ubase, doff, bt, boff, dlist, llit, spos,
      dst, src8);
  DMM_CUDA(cudaGetLastError());
  int h[8];
  DMM_CUDA(cudaMemcpyAsync(h, out, sizeof h, cudaMemcpyDeviceToHost, stream_));
  DMM_CUDA(cudaStreamSynchronize(stream_));
  if (h[0] != 0) return DMM_OK;
  const int sv_cap = std::max(h[1], 4);
  const int st_cap = std::max(h[6], 8);
  const int bk_cap = mt ? std::max(h[7], 8) : std::max(h[2], 8);
  const int smem = mt ? xp_layout_mt(sv_cap, st_cap, bk_cap, TV).total
                      : xp_layout(sv_cap, bk_cap, TV).total;
  if (smem > (mt ? kXpSmemMaxMT : kXpSmemMax)) return DMM_OK;
  if (occupancy_blocks(staged_fn(tun_.var_group, mt), kStagedThreads, smem) * sms_ != grid_p_)
    return DMM_OK;
  xsv_cap_ = sv_cap;
  xst_cap_ = st_cap;
  xbk_cap_ = bk_cap;
  xtv_cap_ = TV;
  xsmem_ = smem;
  xp_mt_ = mt;
  xp_key_ = key;
  xp_key_valid_ = true;
  *ok = true;
  return DMM_OK;
}

// Tile lists of the single live formula idx (the only entries of the tables).
dmm_status Pack::set_tiles(int32_t idx, int TC, int TV) {
  InstDesc& I = inst_h_[idx];
  ctiles_h_.clear();
  vtiles_h_.clear();
  I.ctile0 = 0;
  for (int32_t b = 0; b < I.m; b += TC) ctiles_h_.push_back(Tile{idx, b, std::min(TC, I.m - b), 0});
  I.nctile = (int32_t)ctiles_h_.size();
  I.vtile0 = 0;
  for (int32_t b = 0; b < I.n; b += TV) vtiles_h_.push_back(Tile{idx, b, std::min(TV, I.n - b), 0});
  I.nvtile = (int32_t)vtiles_h_.size();
  if ((int64_t)ctiles_h_.size() > ctile_cap_ || (int64_t)vtiles_h_.size() > vtile_cap_) {
    set_error("tile tables overflow");
    return DMM_ERR_BUDGET;
  }
  return upload_desc(idx);
}

// The several-tiles-per-block staged form: k_c clause tiles and k_v variable tiles per block
// (tile counts multiples of the grid, so that every block has the same number).  Candidate
// tilings whose estimated shared memory fits are ordered by an estimate of their step time
// (a fixed cost per tile a block visits, plus the bytes of the tiles' variable lists and of
// the chunk padding at the measured HBM rate); the first one whose tables build and fit is
// kept.  Leaves *ok false, with the tile lists in an unspecified state, when none fits.
dmm_status Pack::prepare_xpose_mt(int32_t idx, bool* ok) {
  *ok = false;
  const InstDesc& I = inst_h_[idx];
  if (prec_ != DMM_FP32 || !I.k3) return DMM_OK;
  const double n = I.n, m = I.m;
  const int grid = grid_p_;
  struct Cand {
    int TC, TV;
    double cost;
  };
  std::vector<Cand> cands;
  for (int kc = 1; kc <= 64; kc++) {
    const int TC = (int)(((int64_t)std::ceil(m / (kc * (double)grid)) + 3) & ~int64_t(3));
    if (TC < kMinClauseTile) break;
    const double nct = std::ceil(m / TC);
    const double distinct = n * (1.0 - std::exp(-3.0 * TC / n));
    for (int kv = 1; kv <= 64; kv++) {
      const int TV = (int)(((int64_t)std::ceil(n / (kv * (double)grid)) + 3) & ~int64_t(3));
      if (TV < kMinVarTile) break;
      const double nvt = std::ceil(n / TV);
      const double stage = 3.0 * TC + 3.5 * nvt;
      const double bucket = 3.0 * m / nvt * 1.08 + 3.5 * nct;
      if (distinct > 30000 || stage > 60000 || bucket > 60000) continue;
      const double smem = 4.0 * std::max(distinct * 1.03 + stage, bucket) + 0.5 * bucket +
                          9.0 * TV + 4096;
      if (smem > kXpSmemMaxMT + 7 * 1024) continue;  // the estimate runs up to ~6 KB high
      const double bytes = 4.0 * distinct * nct + 8.0 * 3.5 * nct * nvt;
      cands.push_back({TC, TV, 2.0 * (kc + kv) + bytes / 6.0e6});
    }
  }
  std::sort(cands.begin(), cands.end(), [](const Cand& a, const Cand& b) { return a.cost < b.cost; });
  for (size_t k = 0; k < cands.size() && k < 8; k++) {
    DMM_TRY(set_tiles(idx, cands[k].TC, cands[k].TV));
    DMM_TRY(prepare_xpose(idx, cands[k].TC, cands[k].TV, true, ok));
    if (*ok) return DMM_OK;
  }
  return DMM_OK;
}

dmm_status Pack::commit_tiles() {
  DMM_TRY(resolve_long_lists());
  xp_active_ = false;
  one_active_ = false;
  ctiles_h_.clear();
  vtiles_h_.clear();
  std::vector<int32_t> live_list;
  // formulas that one block integrates alone (FP32, V and dV fit in shared memory): used
  // when there are enough of them to fill the GPU (auto) or when forced (launch_mode 3)
  std::vector<int32_t> small_list;
  {
    std::vector<int32_t> eligible, others;
    for (int32_t i = 0; i < (int32_t)live_.size(); i++) {
      if (!live_[i]) continue;
      const bool ok = prec_ == DMM_FP32 && inst_h_[i].n <= kInstVCap &&
                      (tun_.launch_mode == 0 || tun_.launch_mode == 3);
      (ok ? eligible : others).push_back(i);
    }
    const bool use_small = tun_.launch_mode == 3 || (int64_t)eligible.size() >= sms_;
    if (use_small) {
      small_list = eligible;
    } else {
      others.insert(others.end(), eligible.begin(), eligible.end());
      std::sort(others.begin(), others.end());
    }
    live_list = others;
    std::stable_sort(small_list.begin(), small_list.end(),
                     [&](int32_t a, int32_t b) { return inst_h_[a].m > inst_h_[b].m; });
  }
  for (int32_t i : small_list) {
    inst_h_[i].ctile0 = inst_h_[i].nctile = inst_h_[i].vtile0 = inst_h_[i].nvtile = 0;
    DMM_TRY(upload_desc(i));
  }
  if (!small_list.empty())
    DMM_CUDA(cudaMemcpyAsync(order_d_, small_list.data(), small_list.size() * sizeof(int32_t),
                             cudaMemcpyHostToDevice, stream_));
  n_small_ = (int32_t)small_list.size();
  // grids
  int bc, bv;
  if (prec_ == DMM_FP64) {
    bc = occupancy_blocks((const void*)k_clause<double, false>, kThreads);
    bv = occupancy_blocks((const void*)k_var<double, 32, true, 0>, kThreads);
  } else {
    bc = occupancy_blocks((const void*)k_clause<float, true>, kThreads);
    bv = occupancy_blocks((const void*)k_var<float, 8, false, 0>, kThreads);
  }
  if (tun_.blocks_per_sm > 0) {
    bc = std::min(bc, tun_.blocks_per_sm);
    bv = std::min(bv, tun_.blocks_per_sm);
  }
  grid_p_ = occupancy_blocks(persist_fn(), persist_threads(prec_)) * sms_;
  const bool coop = tun_.launch_mode != 1;
  const int block = coop ? persist_threads(prec_) : kThreads;
  const int64_t spread = coop ? grid_p_ : (int64_t)bc * sms_;
  // tile sizes: balanced over the grid for a single instance, else fixed
  int TC = tun_.clause_tile, TV = tun_.var_tile;
  if (TC == 0) {
    TC = 4 * block;
    if (live_list.size() == 1) {
      const int64_t m = inst_h_[live_list[0]].m;
      TC = (int)std::max<int64_t>(kMinClauseTile, ((m + spread - 1) / spread + 3) & ~int64_t(3));
    }
  }
  if (TV == 0) {
    TV = block;
    if (live_list.size() == 1) {
      const int64_t n = inst_h_[live_list[0]].n;
      // a multiple of 4 (not of a warp) so that every block gets a variable tile
      TV = (int)std::max<int64_t>(kMinVarTile, ((n + spread - 1) / spread + 3) & ~int64_t(3));
    }
  }
  for (int32_t i : live_list) {
    InstDesc& I = inst_h_[i];
    I.ctile0 = (int32_t)ctiles_h_.size();
    for (int32_t b = 0; b < I.m; b += TC) ctiles_h_.push_back(Tile{i, b, std::min(TC, I.m - b), 0});
    I.nctile = (int32_t)ctiles_h_.size() - I.ctile0;
    I.vtile0 = (int32_t)vtiles_h_.size();
    for (int32_t b = 0; b < I.n; b += TV) vtiles_h_.push_back(Tile{i, b, std::min(TV, I.n - b), 0});
    I.nvtile = (int32_t)vtiles_h_.size() - I.vtile0;
    DMM_TRY(upload_desc(i));
  }
  if ((int64_t)ctiles_h_.size() > ctile_cap_ || (int64_t)vtiles_h_.size() > vtile_cap_) {
    set_error("tile tables overflow");
    return DMM_ERR_BUDGET;
  }
  // one formula on the cooperative path: two grid barriers per step; FP32 with the
  // default layout and tiles: the staged form when it fits
  one_active_ = coop && live_list.size() == 1 && small_list.empty();
  if (one_active_ && prec_ == DMM_FP32 && tun_.u_layout == 0 && tun_.clause_tile == 0 &&
      tun_.var_tile == 0) {
    DMM_TRY(prepare_xpose(live_list[0], TC, TV, false, &xp_active_));
    // too large for one tile per block: several tiles per block, else the tiles above
    if (!xp_active_) {
      DMM_TRY(prepare_xpose_mt(live_list[0], &xp_active_));
      if (!xp_active_) DMM_TRY(set_tiles(live_list[0], TC, TV));
    }
  }
  if (!ctiles_h_.empty())
    DMM_CUDA(cudaMemcpyAsync(ctiles_d_, ctiles_h_.data(), ctiles_h_.size() * sizeof(Tile),
                             cudaMemcpyHostToDevice, stream_));
  if (!vtiles_h_.empty())
    DMM_CUDA(cudaMemcpyAsync(vtiles_d_, vtiles_h_.data(), vtiles_h_.size() * sizeof(Tile),
                             cudaMemcpyHostToDevice, stream_));
  live0_ = live_list.size() == 1 ? live_list[0] : -1;
  if (!live_list.empty())
    DMM_CUDA(cudaMemcpyAsync(live_d_, live_list.data(), live_list.size() * sizeof(int32_t),
                             cudaMemcpyHostToDevice, stream_));
  int32_t nt[2] = {(int32_t)ctiles_h_.size(), (int32_t)vtiles_h_.size()};
  int32_t nl = (int32_t)live_list.size();
  DMM_CUDA(cudaMemcpyAsync(ntiles_d_, nt, sizeof nt, cudaMemcpyHostToDevice, stream_));
  DMM_CUDA(cudaMemcpyAsync(misc_d_, &nl, sizeof nl, cudaMemcpyHostToDevice, stream_));
  const int gc = bc * sms_, gv = bv * sms_;
  const int new_c = fixed_grid_ ? gc : std::max(1, std::min<int>(gc, nt[0]));
  const int new_v = fixed_grid_ ? gv : std::max(1, std::min<int>(gv, nt[1]));
  if (new_c != grid_c_ || new_v != grid_v_) graph_stale_ = true;
  grid_c_ = new_c;
  grid_v_ = new_v;
  if (!fixed_grid_) graph_stale_ = true;
  DMM_CUDA(cudaStreamSynchronize(stream_));
  return DMM_OK;
}

dmm_status Pack::launch_persist(int32_t nsteps) {
  PackView<float> vf;
  PackView<double> vd;
  void* view;
  if (prec_ == DMM_FP64) {
    fill_view<double>(&vd);
    view = &vd;
  } else {
    fill_view<float>(&vf);
    view = &vf;
  }
  static_assert(kMiscAcc2 * 4 + 2 * sizeof(StepAcc) <= kMiscInts * 4, "misc area");
  static_assert(kMiscInts - kMiscLaunch == kLaunchAreaInts, "launch area");
  unsigned int* bar = reinterpret_cast<unsigned int*>(misc_d_ + kMiscLaunch);
  int* err = misc_d_ + 1;
  // a completed launch leaves its area zeroed (leave_launch); after an error or before the
  // first launch it is zeroed here
  if (!launch_area_clean_)
    DMM_CUDA(cudaMemsetAsync(bar, 0, kLaunchAreaInts * sizeof(int32_t), stream_));
  launch_area_clean_ = true;
  void* args[] = {view, &nsteps, &bar, &err};
  const size_t smem = xp_active_ ? (size_t)xsmem_ : 0;
  if (smem)
    DMM_CUDA(cudaFuncSetAttribute(persist_fn(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int block = xp_active_ ? kStagedThreads : persist_threads(prec_);
  DMM_CUDA(cudaLaunchCooperativeKernel(persist_fn(), dim3(grid_p_), dim3(block), args, smem,
                                       stream_));
  return DMM_OK;
}

template <int G>
static dmm_status launch_inst_g(const PackView<float>& v, const int32_t* order, int count,
                                int nsteps, int* queue, int grid, cudaStream_t s) {
  // function attributes are per device: set it on the current one (a cheap driver call)
  DMM_CUDA(cudaFuncSetAttribute(k_inst<G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kInstSmem));
  k_inst<G><<<grid, kInstThreads, kInstSmem, s>>>(v, order, count, nsteps, queue);
  DMM_CUDA(cudaGetLastError());
  return DMM_OK;
}

dmm_status Pack::launch_inst(int32_t nsteps) {
  PackView<float> v;
  fill_view<float>(&v);
  // variable-major contributions by default here: scattered into shared memory, then read
  // contiguously per variable (measured 1.5x faster than gathering through the CSR)
  v.upos = tun_.u_layout == 1 ? nullptr : upos_;
  int* queue = misc_d_ + 3;
  DMM_CUDA(cudaMemsetAsync(queue, 0, sizeof(int32_t), stream_));
  const int grid = std::max(1, std::min(sms_, (int)n_small_));
  switch (tun_.var_group) {
    case 1: return launch_inst_g<1>(v, order_d_, n_small_, nsteps, queue, grid, stream_);
    case 2: return launch_inst_g<2>(v, order_d_, n_small_, nsteps, queue, grid, stream_);
    case 4: return launch_inst_g<4>(v, order_d_, n_small_, nsteps, queue, grid, stream_);
    case 8: return launch_inst_g<8>(v, order_d_, n_small_, nsteps, queue, grid, stream_);
    case 16: return launch_inst_g<16>(v, order_d_, n_small_, nsteps, queue, grid, stream_);
    default: return launch_inst_g<32>(v, order_d_, n_small_, nsteps, queue, grid, stream_);
  }
}

dmm_status Pack::check_error() {
  int32_t e = 0;
  DMM_CUDA(cudaMemcpyAsync(&e, misc_d_ + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, stream_));
  DMM_CUDA(cudaStreamSynchronize(stream_));
  if (e) {
    launch_area_clean_ = false;
    DMM_CUDA(cudaMemsetAsync(misc_d_ + 1, 0, sizeof(int32_t), stream_));  // reported once
    DMM_CUDA(cudaStreamSynchronize(stream_));
    set_error("grid barrier wait gave up in the cooperative step kernel");
    return DMM_ERR_CUDA;
  }
  return DMM_OK;
}

dmm_status Pack::test_barrier_timeout() {
  DMM_CUDA(cudaSetDevice(dev_));
  if (tun_.launch_mode == 1 || (ctiles_h_.empty() && vtiles_h_.empty())) {
    set_error("the barrier test needs the cooperative launch of tile-path formulas");
    return DMM_ERR_STATE;
  }
  barrier_extra_ = 1;
  const dmm_status st = launch_persist(1);
  barrier_extra_ = 0;
  DMM_TRY(st);
  DMM_CUDA(cudaStreamSynchronize(stream_));
  return check_error();
}

dmm_status Pack::capture(int32_t steps) {
  if (graph_exec_) {
    DMM_CUDA(cudaGraphExecDestroy(graph_exec_));
    graph_exec_ = nullptr;
  }
  if (graph_) {
    DMM_CUDA(cudaGraphDestroy(graph_));
    graph_ = nullptr;
  }
  DMM_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
  dmm_status st = DMM_OK;
  for (int32_t s = 0; s < steps && st == DMM_OK; s++) st = enqueue_step(false, nullptr);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(stream_, &g);
  if (st != DMM_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  DMM_CUDA(e);
  graph_ = g;
  DMM_CUDA(cudaGraphInstantiate(&graph_exec_, graph_, 0));
  graph_steps_ = steps;
  graph_stale_ = false;
  return DMM_OK;
}

dmm_status Pack::launch_steps(int32_t nsteps) {
  DMM_CUDA(cudaSetDevice(dev_));
  if (ctiles_h_.empty() && vtiles_h_.empty() && n_small_ == 0) return DMM_OK;
  const int32_t S = tun_.steps_per_graph;
  if (tun_.launch_mode != 1) {
    while (nsteps > 0) {
      const int32_t k = std::min(nsteps, S);
      if (!ctiles_h_.empty() || !vtiles_h_.empty()) DMM_TRY(launch_persist(k));
      if (n_small_ > 0) DMM_TRY(launch_inst(k));
      nsteps -= k;
    }
    return DMM_OK;
  }
  while (nsteps >= S) {
    if (graph_stale_ || graph_steps_ != S || !graph_exec_) DMM_TRY(capture(S));
    DMM_CUDA(cudaGraphLaunch(graph_exec_, stream_));
    nsteps -= S;
  }
  for (int32_t s = 0; s < nsteps; s++) DMM_TRY(enqueue_step(false, nullptr));
  return DMM_OK;
}

dmm_status Pack::ensure_flush(int64_t flush_bytes) {
  if (flush_bytes > flush_cap_) {
    if (flush_) retire(flush_);
    flush_ = nullptr;
    DMM_CUDA(dev_alloc(&flush_, flush_bytes));
    flush_cap_ = flush_bytes;
  }
  return DMM_OK;
}

dmm_status Pack::time_steps_flushed(int32_t nsteps, int64_t flush_bytes, double* ms) {
  DMM_CUDA(cudaSetDevice(dev_));
  DMM_TRY(ensure_flush(flush_bytes));
  double total = 0.0;
  for (int32_t s = 0; s < nsteps; s++) {
    if (flush_bytes > 0) {
      k_flush<<<sms_ * 4, kThreads, 0, stream_>>>(static_cast<int4*>(flush_), flush_bytes / 16, s);
      DMM_CUDA(cudaGetLastError());
    }
    DMM_CUDA(cudaEventRecord(ev_[0], stream_));
    DMM_TRY(launch_steps(1));
    DMM_CUDA(cudaEventRecord(ev_[1], stream_));
    DMM_CUDA(cudaEventSynchronize(ev_[1]));
    float a = 0;
    DMM_CUDA(cudaEventElapsedTime(&a, ev_[0], ev_[1]));
    total += a;
  }
  *ms = total;
  return check_error();
}

dmm_status Pack::preload_kernels() {
  DMM_CUDA(cudaSetDevice(dev_));
  const int G = tun_.var_group;
  std::vector<const void*> fns = {
      persist_fn_x<false>(prec_, G), (const void*)k_count, (const void*)k_scan_block,
      (const void*)k_scan_add, (const void*)k_fill_start, (const void*)k_scatter,
      (const void*)k_sort_lists, (const void*)k_invert, (const void*)k_active_add,
      (const void*)k_put_desc,   (const void*)k_put_ctrl};
  if (prec_ == DMM_FP64) {
    fns.push_back((const void*)k_set_state<double>);
    fns.push_back((const void*)k_get_state<double>);
    fns.push_back((const void*)k_signs<double>);
    fns.push_back(persist_fn_x<true>(prec_, G));
  } else {
    fns.push_back((const void*)k_set_state<float>);
    fns.push_back((const void*)k_get_state<float>);
    fns.push_back((const void*)k_signs<float>);
    fns.push_back(persist_fn_x<true>(prec_, G));
    fns.push_back(staged_fn(G, false));
    fns.push_back(staged_fn(G, true));
    fns.push_back((const void*)k_xp_count<kXprepThreads>);
    fns.push_back((const void*)k_xp_scan<kXprepThreads>);
    fns.push_back((const void*)k_xp_fill<kXprepThreads>);
    switch (G) {
      case 1: fns.push_back((const void*)k_inst<1>); break;
      case 2: fns.push_back((const void*)k_inst<2>); break;
      case 4: fns.push_back((const void*)k_inst<4>); break;
      case 8: fns.push_back((const void*)k_inst<8>); break;
      case 16: fns.push_back((const void*)k_inst<16>); break;
      default: fns.push_back((const void*)k_inst<32>); break;
    }
  }
  for (const void* f : fns) {
    cudaFuncAttributes a;
    DMM_CUDA(cudaFuncGetAttributes(&a, f));
  }
  return DMM_OK;
}

int Pack::launch_form() const {
  if (tun_.launch_mode == 1) return 1;
  if (ctiles_h_.empty() && vtiles_h_.empty() && n_small_ > 0) return 5;
  if (xp_active_) return xp_mt_ ? 6 : 4;
  if (one_active_) return 3;
  return 2;
}

dmm_status Pack::trace_phases(int32_t nsteps, double* out) {
  DMM_CUDA(cudaSetDevice(dev_));
  if (tun_.launch_mode == 1 || n_small_ > 0 || nsteps <= 0) {
    set_error("phase tracing needs the cooperative launch of tile-path formulas");
    return DMM_ERR_STATE;
  }
  constexpr int K = kTraceK;
  const int64_t half = (int64_t)nsteps * K * grid_p_;
  const int64_t need = 2 * half;  // timer stamps, then clock counts
  if (need > trace_cap_) {
    if (trace_) retire(trace_);
    trace_ = nullptr;
    DMM_CUDA(dev_alloc(&trace_, need * sizeof(long long)));
    trace_cap_ = need;
  }
  DMM_CUDA(cudaMemsetAsync(trace_, 0, need * sizeof(long long), stream_));
  trace_on_ = true;
  trace_steps_ = nsteps;
  dmm_status st = launch_persist(nsteps);  // one launch: trace step s = launch step s
  trace_on_ = false;
  DMM_TRY(st);
  std::vector<long long> h(need);
  DMM_CUDA(cudaMemcpyAsync(h.data(), trace_, need * sizeof(long long), cudaMemcpyDeviceToHost, stream_));
  DMM_CUDA(cudaStreamSynchronize(stream_));
  DMM_TRY(check_error());
  const int G = grid_p_;
  auto at = [&](int64_t s, int k, int b) { return h[(s * K + k) * G + b]; };
  double mean[K] = {}, mx[K] = {};
  int used = 0;
  // a step counts when every block stamped its start and the next step's start exists
  for (int32_t s = 0; s + 1 < nsteps; s++) {
    bool ok = true;
    for (int b = 0; b < G && ok; b++) ok = at(s, 0, b) != 0 && at(s + 1, 0, b) != 0;
    if (!ok) break;
    double sm[K] = {}, smx[K] = {};
    for (int b = 0; b < G; b++) {
      long long pts[K + 1];
      for (int k = 0; k < K; k++) {
        const long long v = at(s, k, b);
        pts[k] = v != 0 ? v : pts[k - 1];  // a block without a tile of the phase
      }
      pts[K] = at(s + 1, 0, b);
      for (int k = 0; k < K; k++) {
        const double d = (double)(pts[k + 1] - pts[k]);
        sm[k] += d;
        smx[k] = std::max(smx[k], d);
      }
    }
    for (int k = 0; k < K; k++) {
      mean[k] += sm[k] / G;
      mx[k] += smx[k];
    }
    used++;
  }
  for (int k = 0; k < K; k++) {
    out[2 * k] = used ? mean[k] / used / 1000.0 : 0.0;  // microseconds
    out[2 * k + 1] = used ? mx[k] / used / 1000.0 : 0.0;
  }
  // SM clock of block 0 over the traced steps
  out[2 * K] = 0.0;
  if (used > 0) {
    const long long t0 = at(0, 0, 0), t1 = at(used, 0, 0);
    const long long c0 = h[half + 0], c1 = h[half + (int64_t)used * K * G];
    if (t1 > t0) out[2 * K] = (double)(c1 - c0) / (double)(t1 - t0) * 1000.0;  // MHz
  }
  return DMM_OK;
}

dmm_status Pack::profile_steps(int32_t nsteps, int64_t flush_bytes, StepTimes* t) {
  DMM_CUDA(cudaSetDevice(dev_));
  if (flush_bytes > flush_cap_) {
    if (flush_) retire(flush_);
    flush_ = nullptr;
    DMM_CUDA(dev_alloc(&flush_, flush_bytes));
    flush_cap_ = flush_bytes;
  }
  for (int32_t s = 0; s < nsteps; s++) {
    if (flush_bytes > 0) {
      k_flush<<<sms_ * 4, kThreads, 0, stream_>>>(static_cast<int4*>(flush_), flush_bytes / 16, s);
      DMM_CUDA(cudaGetLastError());
    }
    DMM_CUDA(cudaEventRecord(ev_[0], stream_));
    DMM_TRY(enqueue_clause());
    DMM_CUDA(cudaEventRecord(ev_[1], stream_));
    DMM_TRY(enqueue_var(false, nullptr));
    DMM_CUDA(cudaEventRecord(ev_[2], stream_));
    DMM_CUDA(cudaEventSynchronize(ev_[2]));
    float a = 0, b = 0;
    DMM_CUDA(cudaEventElapsedTime(&a, ev_[0], ev_[1]));
    DMM_CUDA(cudaEventElapsedTime(&b, ev_[1], ev_[2]));
    t->clause_ms += a;
    t->var_ms += b;
    t->step_ms += a + b;
    t->launches += 2;
  }
  return DMM_OK;
}

dmm_status Pack::read_active(int32_t* active) {
  DMM_CUDA(cudaMemcpyAsync(active, active_d_, sizeof(int32_t), cudaMemcpyDeviceToHost, stream_));
  DMM_CUDA(cudaStreamSynchronize(stream_));
  return DMM_OK;
}

dmm_status Pack::run(double wall_s, int64_t* steps_launched, bool* timed_out,
                     int32_t stop_after) {
  DMM_CUDA(cudaSetDevice(dev_));
  *timed_out = false;
  if (steps_launched) *steps_launched = 0;
  if (!pinned_) DMM_CUDA(pinned_alloc(&pinned_, 4 * sizeof(int32_t)));
  const auto t0 = std::chrono::steady_clock::now();
  auto elapsed = [&]() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  };
  int32_t active = 0, tail0 = 0;
  DMM_TRY(read_active(&active));
  DMM_CUDA(cudaMemcpyAsync(&tail0, ring_tail_d_, sizeof(int32_t), cudaMemcpyDeviceToHost, stream_));
  DMM_CUDA(cudaStreamSynchronize(stream_));
  if (active <= 0) return DMM_OK;
  const int32_t S = tun_.steps_per_graph;
  // chunk k: S steps, then copies of the running count and the finished-ring tail
  auto chunk = [&](int slot) -> dmm_status {
    DMM_TRY(launch_steps(S));
    DMM_CUDA(cudaMemcpyAsync(pinned_ + slot, active_d_, sizeof(int32_t), cudaMemcpyDeviceToHost,
                             stream_));
    DMM_CUDA(cudaMemcpyAsync(pinned_ + 2 + slot, ring_tail_d_, sizeof(int32_t),
                             cudaMemcpyDeviceToHost, stream_));
    DMM_CUDA(cudaEventRecord(ev_[slot], stream_));
    if (steps_launched) *steps_launched += S;
    return DMM_OK;
  };
  int cur = 0;
  DMM_TRY(chunk(cur));
  for (;;) {
    const int nxt = cur ^ 1;
    DMM_TRY(chunk(nxt));
    DMM_CUDA(cudaEventSynchronize(ev_[cur]));
    if (pinned_[cur] <= 0) break;
    if (stop_after > 0 && pinned_[2 + cur] - tail0 >= stop_after) break;
    if (wall_s > 0 && elapsed() > wall_s) {
      *timed_out = true;
      break;
    }
    cur = nxt;
  }
  DMM_CUDA(cudaStreamSynchronize(stream_));
  return check_error();
}

dmm_status Pack::resume(int32_t idx) {
  InstCtrl c;
  DMM_TRY(read_ctrl(idx, &c));
  if (c.done != DMM_STEP_LIMIT) return DMM_OK;
  c.done = 0;
  DMM_TRY(add_active(+1));
  DMM_TRY(write_ctrl(idx, c));
  return DMM_OK;
}

dmm_status Pack::drain_finished(std::vector<int32_t>* out) {
  out->clear();
  int32_t tail = 0;
  DMM_CUDA(cudaMemcpyAsync(&tail, ring_tail_d_, sizeof(int32_t), cudaMemcpyDeviceToHost, stream_));
  DMM_CUDA(cudaStreamSynchronize(stream_));
  if (tail == ring_read_) return DMM_OK;
  std::vector<int32_t> ring(caps_.insts);
  DMM_CUDA(cudaMemcpy(ring.data(), ring_d_, caps_.insts * sizeof(int32_t), cudaMemcpyDeviceToHost));
  for (int32_t p = ring_read_; p < tail; p++) out->push_back(ring[p % caps_.insts]);
  ring_read_ = tail;
  return DMM_OK;
}

dmm_status Pack::stop(int32_t idx, int32_t status) {
  InstCtrl c;
  DMM_TRY(read_ctrl(idx, &c));
  if (c.done != 0) return DMM_OK;
  c.done = status;
  DMM_TRY(add_active(-1));
  DMM_TRY(write_ctrl(idx, c));
  return DMM_OK;
}

dmm_status Pack::sync() {
  DMM_CUDA(cudaStreamSynchronize(stream_));
  return check_error();
}

dmm_status Pack::rhs(int32_t idx, const double* x, double* dxdt, int32_t* loc, double* energy) {
  if (!live(idx) || !x || !dxdt) return DMM_ERR_ARG;
  DMM_TRY(resolve_long_lists());
  DMM_TRY(set_state(idx, x));
  const InstDesc& I = inst_h_[idx];
  const int64_t N = (int64_t)I.n + 2 * (int64_t)I.m;
  // tiles of this instance only
  std::vector<Tile> ct, vt;
  // the right-hand side runs the kernel-per-phase form with its own fixed tiles
  const int TC = 4 * kThreads, TV = kThreads;
  for (int32_t b = 0; b < I.m; b += TC) ct.push_back(Tile{idx, b, std::min(TC, I.m - b), 0});
  for (int32_t b = 0; b < I.n; b += TV) vt.push_back(Tile{idx, b, std::min(TV, I.n - b), 0});
  const int64_t need = std::max<int64_t>(std::max(ct.size(), vt.size()), 1);
  if (need > aux_cap_) {
    if (aux_ctiles_d_) retire(aux_ctiles_d_);
    if (aux_vtiles_d_) retire(aux_vtiles_d_);
    aux_ctiles_d_ = aux_vtiles_d_ = nullptr;
    DMM_CUDA(dev_alloc(&aux_ctiles_d_, need * sizeof(Tile)));
    DMM_CUDA(dev_alloc(&aux_vtiles_d_, need * sizeof(Tile)));
    aux_cap_ = need;
  }
  if (!ct.empty())
    DMM_CUDA(cudaMemcpyAsync(aux_ctiles_d_, ct.data(), ct.size() * sizeof(Tile),
                             cudaMemcpyHostToDevice, stream_));
  DMM_CUDA(cudaMemcpyAsync(aux_vtiles_d_, vt.data(), vt.size() * sizeof(Tile),
                           cudaMemcpyHostToDevice, stream_));
  int32_t nt[2] = {(int32_t)ct.size(), (int32_t)vt.size()};
  DMM_CUDA(cudaMemcpyAsync(ntiles_d_ + 2, nt, sizeof nt, cudaMemcpyHostToDevice, stream_));
  // the finalize of a right-hand side reads the epart of the auxiliary tiles
  InstDesc Iaux = I;
  Iaux.ctile0 = 0;
  Iaux.nctile = nt[0];
  DMM_CUDA(cudaMemcpyAsync(inst_d_ + idx, &Iaux, sizeof(InstDesc), cudaMemcpyHostToDevice, stream_));
  const int gc = grid_c_, gv = grid_v_;
  grid_c_ = std::max(1, std::min(nt[0], sms_ * 8));
  grid_v_ = std::max(1, std::min(nt[1], sms_ * 8));
  use_aux_ = true;
  dmm_status st = enqueue_step(true, stage_);
  use_aux_ = false;
  grid_c_ = gc;
  grid_v_ = gv;
  DMM_TRY(st);
  if (prec_ == DMM_FP64)
    k_clause_dx<double><<<blocks_for(I.m), kThreads, 0, stream_>>>(
        inst_d_, idx, static_cast<double*>(Xs_), static_cast<double*>(Cp_),
        static_cast<double*>(alpha_cm_), stage_);
  else
    k_clause_dx<float><<<blocks_for(I.m), kThreads, 0, stream_>>>(
        inst_d_, idx, static_cast<float*>(Xs_), static_cast<float*>(Cp_),
        static_cast<float*>(alpha_cm_), stage_);
  DMM_CUDA(cudaGetLastError());
  k_rhs_finish<<<1, kThreads, 0, stream_>>>(inst_d_, ctrl_d_, idx, epart_);
  DMM_CUDA(cudaGetLastError());
  DMM_TRY(upload_desc(idx));
  DMM_CUDA(cudaMemcpyAsync(dxdt, stage_, N * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  InstCtrl c;
  DMM_TRY(read_ctrl(idx, &c));
  if (loc) *loc = c.loc;
  if (energy) *energy = c.energy;
  return DMM_OK;
}

dmm_status Pack::dostep(int32_t idx, const double* x, const double* dxdt, double h, double* xo) {
  if (!live(idx) || !x || !dxdt || !xo) return DMM_ERR_ARG;
  const InstDesc& I = inst_h_[idx];
  const int64_t N = (int64_t)I.n + 2 * (int64_t)I.m;
  DMM_TRY(ensure_stage(3 * N));
  DMM_CUDA(cudaMemcpyAsync(stage_, x, N * sizeof(double), cudaMemcpyHostToDevice, stream_));
  DMM_CUDA(cudaMemcpyAsync(stage_ + N, dxdt, N * sizeof(double), cudaMemcpyHostToDevice, stream_));
  if (prec_ == DMM_FP64)
    k_dostep<double><<<blocks_for(N), kThreads, 0, stream_>>>(inst_d_, idx, unit_, stage_,
                                                              stage_ + N, h, stage_ + 2 * N);
  else
    k_dostep<float><<<blocks_for(N), kThreads, 0, stream_>>>(inst_d_, idx, unit_, stage_,
                                                             stage_ + N, h, stage_ + 2 * N);
  DMM_CUDA(cudaGetLastError());
  DMM_CUDA(cudaMemcpyAsync(xo, stage_ + 2 * N, N * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  DMM_CUDA(cudaStreamSynchronize(stream_));
  return DMM_OK;
}

dmm_status Pack::assignment(int32_t idx, int8_t* pre, int8_t* post) {
  if (!live(idx)) return DMM_ERR_ARG;
  if (!pre && !post) return DMM_OK;
  const InstDesc& I = inst_h_[idx];
  // [flag | pre (n) | post (n)] in the staging buffer
  DMM_TRY(ensure_stage(1 + (2 * (int64_t)I.n + 7) / 8));
  int32_t* flag = reinterpret_cast<int32_t*>(stage_);
  int8_t* dpre = reinterpret_cast<int8_t*>(stage_) + 8;
  int8_t* dpost = dpre + I.n;
  DMM_CUDA(cudaMemsetAsync(flag, 0, sizeof(int32_t), stream_));
  if (prec_ == DMM_FP64)
    k_signs<double><<<blocks_for(I.n), kThreads, 0, stream_>>>(
        ctrl_d_ + idx, static_cast<const double*>(cand_), caps_.vars, I.var0, I.n,
        pre ? dpre : nullptr, post ? dpost : nullptr, flag);
  else
    k_signs<float><<<blocks_for(I.n), kThreads, 0, stream_>>>(
        ctrl_d_ + idx, static_cast<const float*>(cand_), caps_.vars, I.var0, I.n,
        pre ? dpre : nullptr, post ? dpost : nullptr, flag);
  DMM_CUDA(cudaGetLastError());
  int32_t not_solved = 0;
  DMM_CUDA(cudaMemcpyAsync(&not_solved, flag, sizeof(int32_t), cudaMemcpyDeviceToHost, stream_));
  if (pre) DMM_CUDA(cudaMemcpyAsync(pre, dpre, I.n, cudaMemcpyDeviceToHost, stream_));
  if (post) DMM_CUDA(cudaMemcpyAsync(post, dpost, I.n, cudaMemcpyDeviceToHost, stream_));
  DMM_CUDA(cudaStreamSynchronize(stream_));
  if (pre && not_solved) {
    set_error("instance %d is not solved", idx);
    return DMM_ERR_STATE;
  }
  return DMM_OK;
}

}  // namespace dmm
