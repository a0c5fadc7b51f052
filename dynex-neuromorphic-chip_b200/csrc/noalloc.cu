// Right-hand side of a 3-SAT formula for callers that cannot allocate device memory.
//
// Some callers run where cudaMalloc is not available to them: inside a host framework
// whose caching allocator owns all device memory (a second allocator would fragment it or
// fail), or in a plug-in that may only touch the buffers it is handed.
// dmm_rhs3_f32_noalloc serves them: the caller passes device inputs and outputs, and the
// intermediate data (per-literal contributions, clause values, the variable->slot CSR and
// counters) lives in one file-scope __device__ array of fixed size, so the call performs
// no device allocation of its own.
//
// The array, g_na_scratch, is NA_SCRATCH_BYTES (about 2.1 MB) on every GPU that loads the
// library, for the life of the process.  It bounds the formula: at most NA_MAX_VARS
// variables and NA_MAX_CLAUSES clauses of exactly three literals, each variable in at
// most NA_MAX_OCC literal slots.  The clause memory rate is the scalar alpha of the
// parameters (no per-clause alpha).
//
// The call validates the formula on the device and reads two counters back (literals out
// of range, over-long variable lists), waiting for the caller's stream each time, so it
// blocks the calling thread until the work queued before it and its own checks finish; the
// right-hand side itself is then queued on the stream without waiting for it.
//
// Every call uses the same array and leaves its contents behind; each call clears the
// parts that must start at zero.  Calls whose work overlaps on the GPU (different streams,
// or different host threads on one device) race on the array and must be serialized by
// the caller.
//
// Host code cannot use g_na_scratch's name as a device address.  On its first call on a
// device, the entry point looks the address up with cudaGetSymbolAddress while that
// device is current and keeps it for later calls on that device.
//
// The arithmetic is the production FP32 path's (the same clause and canonical-sum device
// functions), so the output equals dmm_instance_rhs on an FP32 instance bit for bit.
#include <mutex>

#include "dmm_kernels.cuh"
#include "dmm_pack.h"

namespace dmm {
namespace {

constexpr int NA_MAX_VARS = 1 << 15;
constexpr int NA_MAX_CLAUSES = 1 << 16;
constexpr int NA_MAX_SLOTS = 3 * NA_MAX_CLAUSES;
constexpr int NA_MAX_OCC = kSortCap;  // longest per-variable slot list the sorter handles
constexpr int NA_THREADS = 256;
constexpr int NA_MAX_DEVICES = 64;

struct NaScratch {
  float u[NA_MAX_SLOTS];        // contribution of each literal slot
  int32_t vslot[NA_MAX_SLOTS];  // variable-ordered slot lists
  float C[NA_MAX_CLAUSES];      // C_m of each clause
  int32_t vend[NA_MAX_VARS];    // inclusive ends of the slot lists
  int32_t fill[NA_MAX_VARS];    // scatter cursors
  int32_t longv[NA_MAX_SLOTS / kSortCap + 2];  // variables with too many occurrences
  int32_t counters[8];          // [0] unsatisfied clauses, [1] long lists, [2] bad literals
};
constexpr size_t NA_SCRATCH_BYTES = sizeof(NaScratch);

__device__ __align__(256) NaScratch g_na_scratch;

std::mutex g_na_mu;
NaScratch* g_na_addr[NA_MAX_DEVICES] = {nullptr};

// Clears the counters and degree array (everything that accumulates).
__global__ void k_na_clear(NaScratch* s, int n) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    s->vend[v] = 0;
  if (blockIdx.x == 0 && threadIdx.x < 8) s->counters[threadIdx.x] = 0;
}

// Inclusive scan of vend[0..n) (n <= NA_MAX_VARS) in one block of NA_THREADS threads: the
// block walks the array in chunks of NA_THREADS consecutive entries (coalesced loads and
// stores), scans each chunk with warp shuffles and carries the running total forward.
__global__ void k_na_scan(NaScratch* s, int n) {
  __shared__ int32_t wsum[NA_THREADS / 32];
  __shared__ int32_t carry;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += NA_THREADS) {
    const int i = base + threadIdx.x;
    const int32_t v = i < n ? s->vend[i] : 0;
    int32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    int32_t before = carry;
    for (int k = 0; k < w; k++) before += wsum[k];
    if (i < n) s->vend[i] = before + x;
    __syncthreads();  // every thread has read carry and wsum
    if (threadIdx.x == NA_THREADS - 1) carry = before + x;
    __syncthreads();
  }
}

// Counts literals outside [-n, n] \ {0} (the caller's buffer is never indexed before this).
__global__ void k_na_check(NaScratch* s, const int32_t* __restrict__ lits, int L, int n) {
  int bad = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L; i += gridDim.x * blockDim.x) {
    const int32_t l = lits[i];
    bad += (l == 0 || l > n || l < -n);
  }
  bad = warp_sum_i(bad);
  if ((threadIdx.x & 31) == 0 && bad) atomicAdd(&s->counters[2], bad);
}

__global__ void k_na_clause(NaScratch* s, const int32_t* __restrict__ lits, int n, int m,
                            const float* __restrict__ x, ClauseConsts<float> kc) {
  int unsat = 0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < m; c += gridDim.x * blockDim.x) {
    const int l0 = lits[3 * c], l1 = lits[3 * c + 1], l2 = lits[3 * c + 2];
    float u0, u1, u2;
    bool ss;
    const float C = clause3(l0, l1, l2, x[abs(l0) - 1], x[abs(l1) - 1], x[abs(l2) - 1], x[n + c],
                            x[n + m + c], kc, u0, u1, u2, ss);
    s->u[3 * c] = u0;
    s->u[3 * c + 1] = u1;
    s->u[3 * c + 2] = u2;
    s->C[c] = C;
    unsat += !(C < 0.5f);
  }
  unsat = warp_sum_i(unsat);
  if ((threadIdx.x & 31) == 0 && unsat) atomicAdd(&s->counters[0], unsat);
}

// dV of every variable in the canonical order (8 lanes per variable), then dXs / dXl.
__global__ void k_na_var(NaScratch* s, int n, int m, const float* __restrict__ x,
                         ClauseConsts<float> kc, float* __restrict__ dxdt) {
  constexpr int G = 8;
  const int lane = threadIdx.x % G;
  const int warps_total = gridDim.x * (blockDim.x / G);
  const int rounds = (n + warps_total - 1) / warps_total;
  for (int r = 0; r < rounds; r++) {
    const int v = r * warps_total + blockIdx.x * (blockDim.x / G) + threadIdx.x / G;
    int s0 = 0, s1 = 0;
    if (v < n) {
      s1 = s->vend[v];
      s0 = v > 0 ? s->vend[v - 1] : 0;
    }
    const float dv = tree_sum<float, G>(s->u, s->vslot + s0, s1 - s0, lane);
    if (v < n && lane == 0) dxdt[v] = dv;
  }
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < m; c += gridDim.x * blockDim.x) {
    const float xs = clampv(x[n + c], 0.f, 1.f);
    const float C = s->C[c];
    dxdt[n + c] = mul(mul(kc.beta, add(xs, kc.eps)), sub(C, kc.gamma));
    dxdt[n + m + c] = mul(kc.alpha, sub(C, kc.delta));
  }
}

}  // namespace
}  // namespace dmm

using namespace dmm;

extern "C" dmm_status dmm_rhs3_f32_noalloc(const int32_t* lits, int32_t n, int32_t m,
                                           const float* x, const dmm_params* p, float* dxdt,
                                           int32_t* loc, void* stream) {
  clear_error();
  if (!lits || !x || !dxdt || !loc || n <= 0 || m < 0) {
    set_error("dmm_rhs3_f32_noalloc: null buffer or bad size");
    return DMM_ERR_ARG;
  }
  if (n > NA_MAX_VARS || m > NA_MAX_CLAUSES) {
    set_error("dmm_rhs3_f32_noalloc: n=%d m=%d exceeds the fixed scratch (at most %d variables "
              "and %d clauses)", n, m, NA_MAX_VARS, NA_MAX_CLAUSES);
    return DMM_ERR_ARG;
  }
  int dev = 0;
  DMM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NA_MAX_DEVICES) {
    set_error("dmm_rhs3_f32_noalloc: device %d out of range", dev);
    return DMM_ERR_ARG;
  }
  NaScratch* s = nullptr;
  {
    std::lock_guard<std::mutex> g(g_na_mu);
    if (!g_na_addr[dev]) {
      void* a = nullptr;
      DMM_CUDA(cudaGetSymbolAddress(&a, g_na_scratch));
      g_na_addr[dev] = static_cast<NaScratch*>(a);
    }
    s = g_na_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  dmm_params d;
  dmm_params_default(&d);
  if (!p) p = &d;
  ClauseConsts<float> kc;
  kc.beta = float(p->beta);
  kc.gamma = float(p->gamma);
  kc.delta = float(p->delta);
  kc.eps = float(p->epsilon);
  kc.zeta = float(p->zeta);
  kc.alpha = float(p->alpha);
  kc.h = 0.f;
  {
    int32_t v = (int32_t)((uint32_t)p->xl_max * (uint32_t)m);  // dynex.cc:2358-2359
    if (v <= 0) v = 0x7fffffff;
    kc.xlmax = float((double)v);
  }
  const int L = 3 * m;
  const int gb = (std::max(L, n) + NA_THREADS - 1) / NA_THREADS;
  const int grid = std::max(1, std::min(gb, 148 * 8));
  k_na_clear<<<grid, NA_THREADS, 0, st>>>(s, n);
  if (L > 0) k_na_check<<<grid, NA_THREADS, 0, st>>>(s, lits, L, n);
  DMM_CUDA(cudaGetLastError());
  int32_t nbad = 0;
  DMM_CUDA(cudaMemcpyAsync(&nbad, &s->counters[2], sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  DMM_CUDA(cudaStreamSynchronize(st));
  if (nbad > 0) {
    set_error("dmm_rhs3_f32_noalloc: %d literals outside [-n, n] or zero", nbad);
    return DMM_ERR_LITERAL;
  }
  if (L > 0) k_count<<<grid, NA_THREADS, 0, st>>>(lits, L, n, s->vend, nullptr);
  k_na_scan<<<1, NA_THREADS, 0, st>>>(s, n);
  k_fill_start<<<grid, NA_THREADS, 0, st>>>(s->vend, n, s->fill);
  if (L > 0) k_scatter<<<grid, NA_THREADS, 0, st>>>(lits, L, n, s->fill, s->vslot);
  k_sort_lists<<<grid, kThreads, (kThreads / 32) * kSortCap * sizeof(int32_t), st>>>(
      s->vend, n, s->vslot, s->longv, &s->counters[1], 0, NA_MAX_SLOTS / kSortCap + 2);
  DMM_CUDA(cudaGetLastError());
  int32_t nlong = 0;
  DMM_CUDA(cudaMemcpyAsync(&nlong, &s->counters[1], sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  DMM_CUDA(cudaStreamSynchronize(st));
  if (nlong > 0) {
    set_error("dmm_rhs3_f32_noalloc: a variable occurs in more than %d literal slots", NA_MAX_OCC);
    return DMM_ERR_ARG;
  }
  if (m > 0) k_na_clause<<<grid, NA_THREADS, 0, st>>>(s, lits, n, m, x, kc);
  k_na_var<<<grid, NA_THREADS, 0, st>>>(s, n, m, x, kc, dxdt);
  DMM_CUDA(cudaMemcpyAsync(loc, &s->counters[0], sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
  DMM_CUDA(cudaGetLastError());
  return DMM_OK;
}
