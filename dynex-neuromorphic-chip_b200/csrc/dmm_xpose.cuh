// Staged form of the integration step: FP32, one formula of 3-literal clauses, one
// cooperative launch with one clause tile and one variable tile per block.
//
// The plain tile code issues one L2 request per literal occurrence in each phase (phase A
// gathers V[|l|-1] per literal, phase B gathers u through the variable->slot list), each
// behind a dependent global load.  The staged form moves both gathers into shared memory:
//
//   A  the clause tile's distinct variables (ascending, kept in shared memory for the whole
//      launch) have their voltages gathered by asynchronous copies into shared memory;
//      the clauses read them through 16-bit tile-local literals.  Each contribution is
//      written to a shared staging area grouped by destination variable tile (one chunk
//      per variable tile, padded to 8 entries = one sector) and the area is written to
//      global memory with 16-byte stores.
//   B  a variable tile loads its chunk of every clause tile (contiguous, sector-aligned)
//      with 16-byte loads and stores each value to its variable-major position in shared
//      memory, then reduces each variable from there; the lanes of a variable's group form
//      one Euler candidate each.
//
// Grid barriers are split (arrive ... wait) so that loads that do not depend on the other
// blocks (the voltages of phase B's variables; at barrier 2 the step's phase-A counts) are
// in flight during the wait.
// Barrier 2 carries the step decision: a block arrives by adding 1 << (12 k) to the step's
// arrival word, k = the largest trial index of its variables, so that the word that ends
// the wait also holds the step's largest trial index.  The step's unsatisfied count and
// strict-sign failures (complete at barrier 1) are read during that wait.  Every block applies
// the decision to its own copy of the control state; block 0 writes it for the host.
//
// Every clause value and every per-variable sum is computed from the same operands in the
// same order as the plain tile code, so results are identical to it.
//
// Several tiles per block (MT): formulas too large for one clause tile and one variable
// tile per block (the tiles' 16-bit indices and shared memory bound them) are cut into
// more tiles than blocks; block b takes clause tiles b, b + grid, ... in phase A and
// variable tiles b, b + grid, ... in phase B, loading each tile's tables when it starts
// it.  In phase B the bucket overlays the voltage and staging areas of phase A, so a
// variable tile may hold more contributions than a clause tile stages.  The per-block
// counts are summed over its tiles before the one update of the step accumulators.
#pragma once

namespace dmm {

constexpr uint16_t kXpPad = 0xFFFF;  // xdst of a padding entry
constexpr int kArriveBits = 12;      // width of one trial's arrival count (> grid size)
constexpr int kPollSleepNs = 64;     // back-off between polls of a barrier word


__host__ __device__ constexpr int xp_align16(int bytes) { return (bytes + 15) & ~15; }

// Dynamic shared-memory layout of the staged form (byte offsets).
struct XpLayout {
  int sd, sv, bk, src8, vend, cur, unit, total;
};

__host__ __device__ inline XpLayout xp_layout(int sv_cap, int bk_cap, int tv_cap) {
  XpLayout L;
  int o = 0;
  L.sd = o;                                       // (unused: the list is read per step)
  L.sv = o;   o += xp_align16(4 * sv_cap);        // the tile's variables, then their voltages
  L.bk = o;   o += xp_align16(4 * bk_cap);        // staging area (A) / bucket (B)
  L.src8 = o; o += xp_align16(4 * (bk_cap / 8));  // ux index of every 8 bucket positions
  L.vend = o; o += xp_align16(4 * (tv_cap + 1));  // tile-local CSR ends of the variable tile
  L.cur = o;  o += xp_align16(4 * tv_cap);        // V of the variable tile
  L.unit = o; o += xp_align16(tv_cap);            // unit pins of the variable tile
  L.total = o;
  return L;
}

// Layout of the several-tiles-per-block form: phase A's voltages (sv_cap) and staging area
// (st_cap) side by side at L.sv and L.bk; phase B's bucket (bk_cap entries) from L.sv over
// both; the tables of the current variable tile after the larger of the two.
__host__ __device__ inline XpLayout xp_layout_mt(int sv_cap, int st_cap, int bk_cap, int tv_cap) {
  XpLayout L;
  L.sd = 0;
  L.sv = 0;
  L.bk = xp_align16(4 * sv_cap);
  int o = L.bk + xp_align16(4 * st_cap);
  if (xp_align16(4 * bk_cap) > o) o = xp_align16(4 * bk_cap);
  L.src8 = o; o += xp_align16(4 * (bk_cap / 8 + 1));
  L.vend = o; o += xp_align16(4 * (tv_cap + 1));
  L.cur = o;  o += xp_align16(4 * tv_cap);
  L.unit = o; o += xp_align16(tv_cap);
  L.total = o;
  return L;
}

// Asynchronous global->shared copies (completed by cp_async_wait_all + a block barrier).
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Entry k (0..11) of twelve 16-bit values held in three 8-byte words; k must fold to a
// constant (unrolled loops), so the words stay in registers.
__device__ __forceinline__ int i16_at(const int2 (&w)[3], int k) {
  const int word = (k & 2) ? w[k >> 2].y : w[k >> 2].x;
  return (k & 1) ? (word >> 16) : (int)(short)(word & 0xffff);
}
__device__ __forceinline__ int u16_at(const uint2 (&w)[3], int k) {
  const unsigned word = (k & 2) ? w[k >> 2].y : w[k >> 2].x;
  return (int)((k & 1) ? (word >> 16) : (word & 0xffffu));
}
__device__ __forceinline__ float f4_at(const float4& v, int i) {
  return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}

// L2 eviction policies for the several-tiles-per-block form, whose per-step working set
// exceeds the L2: the streamed tables and clause memories are marked evict-first, the
// staging areas written in phase A and read back in phase B evict-last, so that the
// staging traffic stays in L2 as far as it fits.
struct L2Pol {
  uint64_t first, last;
};
__device__ __forceinline__ L2Pol make_l2pol(bool plain) {
  L2Pol p;
  if (plain) {  // the same accesses with the default priority
    asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p.first));
    p.last = p.first;
  } else {
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p.first));
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p.last));
  }
  return p;
}
__device__ __forceinline__ float4 ld_hint4(const float* a, uint64_t pol) {
  float4 v;
  asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ void st_hint4(float* a, float4 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(a),
               "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "l"(pol)
               : "memory");
}
__device__ __forceinline__ int2 ld_hint_i2(const void* a, uint64_t pol) {
  int2 v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.s32 {%0, %1}, [%2], %3;"
               : "=r"(v.x), "=r"(v.y)
               : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ void cp_async16_hint(void* smem, const void* gmem, uint64_t pol) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(sa),
               "l"(gmem), "l"(pol)
               : "memory");
}

// Prefetch of the byte range [lo, hi) of `base` into L2 (the bulk prefetch needs a 16-byte
// aligned start and a size that is a multiple of 16: both ends are rounded down, so the range
// never reaches past the array), in pieces of 4 KB spread over the lanes of one warp.
__device__ __forceinline__ void prefetch_l2(const void* base, int64_t lo, int64_t hi, int lane) {
  lo &= ~int64_t(15);
  hi &= ~int64_t(15);
  for (int64_t o = lo + 4096 * (int64_t)lane; o < hi; o += 32 * 4096) {
    const unsigned sz = (unsigned)(hi - o < 4096 ? hi - o : 4096);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(
                     static_cast<const char*>(base) + o),
                 "r"(sz)
                 : "memory");
  }
}

// Several-tiles form: each block's first kXpMetaTiles clause and variable tiles keep their
// ranges and table offsets in shared memory for the whole launch, so a tile starts without a
// dependent global load (tiles past those read them from global memory as they start).
constexpr int kXpMetaTiles = 16;
struct XpMetaC {
  int begin, count, dbeg, dcnt, ubase, ulen;
};
struct XpMetaV {
  int begin, count, bbeg, blen, jb;  // jb: CSR end before the tile
};

// The block's copy of the control state of the formula.
struct StagedCtrl {
  int done, step, set, kcur, pending, best_loc;
  double h, t, best_t;
};

// Operands of one group of 4 clauses.
struct Group4 {
  int2 lw[3];   // 12 tile-local literals
  uint2 qw[3];  // 12 staging positions
  float4 xs, xl, cp, al;
};

__device__ __forceinline__ void load_words4(Group4& q, const int16_t* ll, const uint16_t* sp,
                                            int g) {
  const int2* L2 = reinterpret_cast<const int2*>(ll + 3 * g);
  const uint2* Q2 = reinterpret_cast<const uint2*>(sp + 3 * g);
#pragma unroll
  for (int r = 0; r < 3; r++) {
    q.lw[r] = __ldg(L2 + r);
    q.qw[r] = __ldg(Q2 + r);
  }
}

__device__ __forceinline__ void load_state4(Group4& q, const float* Xs, const float* Xl,
                                            const float* Cp, const float* acm, float alpha,
                                            bool pending, int g) {
  q.xs = *reinterpret_cast<const float4*>(Xs + g);
  q.xl = *reinterpret_cast<const float4*>(Xl + g);
  q.cp = pending ? *reinterpret_cast<const float4*>(Cp + g) : make_float4(0.f, 0.f, 0.f, 0.f);
  q.al = acm ? *reinterpret_cast<const float4*>(acm + g) : make_float4(alpha, alpha, alpha, alpha);
}

// The same loads marked evict-first in L2 (several-tiles-per-block form).
__device__ __forceinline__ void load_words4_hint(Group4& q, const int16_t* ll, const uint16_t* sp,
                                                 int g, uint64_t pol) {
#pragma unroll
  for (int r = 0; r < 3; r++) {
    q.lw[r] = ld_hint_i2(ll + 3 * g + 4 * r, pol);
    const int2 w = ld_hint_i2(sp + 3 * g + 4 * r, pol);
    q.qw[r] = make_uint2((unsigned)w.x, (unsigned)w.y);
  }
}
__device__ __forceinline__ void load_state4_hint(Group4& q, const float* Xs, const float* Xl,
                                                 const float* Cp, const float* acm, float alpha,
                                                 bool pending, int g, uint64_t pol) {
  q.xs = ld_hint4(Xs + g, pol);
  q.xl = ld_hint4(Xl + g, pol);
  q.cp = pending ? ld_hint4(Cp + g, pol) : make_float4(0.f, 0.f, 0.f, 0.f);
  q.al = acm ? ld_hint4(acm + g, pol) : make_float4(alpha, alpha, alpha, alpha);
}

template <int G, int NT, bool MT>
__global__ void __launch_bounds__(NT, 1)
    k_staged(PackView<float> P, int nsteps, unsigned int* bar, int* err) {
  using T = float;
  extern __shared__ __align__(16) unsigned char staged_smem[];
  __shared__ InstDesc I;
  __shared__ StagedCtrl lc;
  __shared__ Tile ctile, vtile;
  __shared__ int dbeg, dcnt, ubase, ulen, bbeg, blen;
  __shared__ XpMetaC s_mc[MT ? kXpMetaTiles : 1];
  __shared__ XpMetaV s_mv[MT ? kXpMetaTiles : 1];
  __shared__ double red[NT / 32];
  __shared__ int cnt[2][NT / 32];
  __shared__ int s_ok;
  const XpLayout LY = MT ? xp_layout_mt(P.xsv_cap, P.xst_cap, P.xbk_cap, P.xtv_cap)
                        : xp_layout(P.xsv_cap, P.xbk_cap, P.xtv_cap);
  T* sV = reinterpret_cast<T*>(staged_smem + LY.sv);
  T* stage = reinterpret_cast<T*>(staged_smem + LY.bk);  // phase A
  T* bucket = MT ? sV : stage;                            // phase B
  int* s_src8 = reinterpret_cast<int*>(staged_smem + LY.src8);
  int* s_vend = reinterpret_cast<int*>(staged_smem + LY.vend);
  T* s_cur = reinterpret_cast<T*>(staged_smem + LY.cur);
  int8_t* s_unit = reinterpret_cast<int8_t*>(staged_smem + LY.unit);
  const int b = blockIdx.x, tid = threadIdx.x;
  const int nct = P.ntiles[0], nvt = P.ntiles[1];
  const bool has_c = b < nct, has_v = b < nvt;
  const int ii = P.live0 >= 0 ? P.live0 : P.live[0];
  L2Pol pol{0, 0};
  if constexpr (MT) pol = make_l2pol(P.xl2_plain != 0);

  trace_launch(P, 0);
  // ---- launch setup: description, control state, ranges, launch-constant tables
  if (tid == 0) {
    I = P.inst[ii];
    const volatile InstCtrl* S = P.ctrl + ii;
    lc.done = S->done;
    lc.step = S->step;
    lc.set = S->set;
    lc.kcur = S->kcur;
    lc.pending = S->pending;
    lc.best_loc = S->best_loc;
    lc.h = S->h_state;
    lc.t = S->t;
    lc.best_t = S->best_t;
    dbeg = dcnt = ubase = ulen = bbeg = blen = 0;
    if (!MT && has_c) {
      ctile = P.ctiles[b];
      dbeg = __ldg(P.xdoff + 2 * b);
      dcnt = __ldg(P.xdoff + 2 * b + 1);
      ubase = __ldg(P.xubase + b);
      ulen = __ldg(P.xubase + b + 1) - ubase;
    }
    if (!MT && has_v) {
      vtile = P.vtiles[b];
      bbeg = __ldg(P.xboff + b);
      blen = __ldg(P.xboff + b + 1) - bbeg;
    }
  }
  __syncthreads();
  if (!MT && has_v) {
    // phase B's tables arrive by asynchronous copies that the first wait of phase A
    // completes, so they load alongside phase A's first reads: the raw CSR ends (s_vend[0]
    // = the end before the tile, subtracted where they are read) and the unit pins as
    // 4-byte words (the tile starts at a multiple of 4 variables of a 32-aligned range,
    // and the pin array has slack past its last variable)
    const int32_t* vend = P.vend + I.var0;
    for (int g = tid; g < blen / 8; g += NT) cp_async4(s_src8 + g, P.xsrc8 + bbeg / 8 + g);
    for (int i = tid; i <= vtile.count; i += NT) {
      if (i > 0 || vtile.begin > 0) cp_async4(s_vend + i, vend + vtile.begin + i - 1);
      else s_vend[0] = 0;
    }
    for (int w = tid; 4 * w < vtile.count; w += NT)
      cp_async4(s_unit + 4 * w, P.unit + I.var0 + vtile.begin + 4 * w);
  }
  if constexpr (MT) {
    if (tid < kXpMetaTiles) {
      const int k = tid, ct = b + k * (int)gridDim.x, vt = ct;
      if (ct < nct) {
        XpMetaC& mc = s_mc[k];
        mc.begin = P.ctiles[ct].begin;
        mc.count = P.ctiles[ct].count;
        mc.dbeg = __ldg(P.xdoff + 2 * ct);
        mc.dcnt = __ldg(P.xdoff + 2 * ct + 1);
        mc.ubase = __ldg(P.xubase + ct);
        mc.ulen = __ldg(P.xubase + ct + 1) - mc.ubase;
      }
      if (vt < nvt) {
        XpMetaV& mv = s_mv[k];
        mv.begin = P.vtiles[vt].begin;
        mv.count = P.vtiles[vt].count;
        mv.bbeg = __ldg(P.xboff + vt);
        mv.blen = __ldg(P.xboff + vt + 1) - mv.bbeg;
        mv.jb = mv.begin > 0 ? __ldg(P.vend + I.var0 + mv.begin - 1) : 0;
      }
    }
  }
  if (!MT && tid == 32 && lc.done == 0) {
    // the voltages of the first step: this block's share of them toward L2 (later steps
    // read the candidates the previous step wrote, still in L2)
    const T* V0 = P.cand + (int64_t)(lc.set * kTrials + lc.kcur) * P.var_cap + I.var0;
    const int64_t per = ((int64_t)I.n + gridDim.x - 1) / gridDim.x;
    const int64_t lo = min((int64_t)I.n, per * b), hi = min((int64_t)I.n, lo + per);
    if (hi > lo) prefetch_l2(V0, 4 * lo, 4 * hi, 0);
  }
  __syncthreads();

  unsigned int target = 0;

  for (int s = 0; s < nsteps; s++) {
    if (lc.done != 0) break;  // grid-uniform: every block applies the same decisions
    trace_stamp(P, s, 0);
    StepAcc* acc = P.acc2 + (s & 1);
    const int set = lc.set, kcur = lc.kcur;
    const bool pending = lc.pending != 0;
    const ClauseConsts<T> kc = make_consts<T>(I, lc.h);
    const T* V = P.cand + (int64_t)(set * kTrials + kcur) * P.var_cap + I.var0;
    trace_stamp(P, s, 1);

    // ---- phase A
    int unsat = 0, vfail = 0;
    double e = 0.0;
    // the block's clause tiles: b, b + grid, ... (one, b, without MT)
    for (int ct = b; ct < nct; ct += MT ? (int)gridDim.x : nct) {
      if constexpr (MT) {
        const int k = (ct - b) / (int)gridDim.x;
        if (tid == 0) {
          if (k < kXpMetaTiles) {
            const XpMetaC& mc = s_mc[k];
            ctile.begin = mc.begin;
            ctile.count = mc.count;
            dbeg = mc.dbeg;
            dcnt = mc.dcnt;
            ubase = mc.ubase;
            ulen = mc.ulen;
          } else {
            ctile = P.ctiles[ct];
            dbeg = __ldg(P.xdoff + 2 * ct);
            dcnt = __ldg(P.xdoff + 2 * ct + 1);
            ubase = __ldg(P.xubase + ct);
            ulen = __ldg(P.xubase + ct + 1) - ubase;
          }
        }
        __syncthreads();
        // one warp asks L2 for the block's next clause tile (its variable list, local
        // literals, staging positions and clause memories) while this one is processed
        const int nt = ct + (int)gridDim.x;
        if (P.xprefetch && nt < nct && tid < 32) {
          const Tile tn = P.ctiles[nt];
          const int db = __ldg(P.xdoff + 2 * nt), dc = __ldg(P.xdoff + 2 * nt + 1);
          const int64_t c0 = tn.begin, c1 = (int64_t)tn.begin + tn.count;
          prefetch_l2(P.xdlist, 4 * (int64_t)db, 4 * (int64_t)(db + ((dc + 3) & ~3)), tid);
          prefetch_l2(P.xllit, 6 * c0, 6 * c1, tid);
          prefetch_l2(P.xspos, 6 * c0, 6 * c1, tid);
          prefetch_l2(P.Xs + I.cls0, 4 * c0, 4 * c1, tid);
          prefetch_l2(P.Xl + I.cls0, 4 * c0, 4 * c1, tid);
          if (lc.pending) prefetch_l2(P.Cp + I.cls0, 4 * c0, 4 * c1, tid);
          if (I.has_alpha_cm) prefetch_l2(P.alpha_cm + I.cls0, 4 * c0, 4 * c1, tid);
        }
      }
      T* __restrict__ Xs = P.Xs + I.cls0;
      T* __restrict__ Xl = P.Xl + I.cls0;
      T* __restrict__ Cp = P.Cp + I.cls0;
      const T* __restrict__ acm = I.has_alpha_cm ? P.alpha_cm + I.cls0 : nullptr;
      const int16_t* __restrict__ ll = P.xllit;
      const uint16_t* __restrict__ sp = P.xspos;
      // the tile's variable list (padded to 4 entries), then each entry replaced in place
      // by its voltage: two rounds of asynchronous copies with every load in flight
      int* sVi = reinterpret_cast<int*>(sV);
      for (int q = tid; 4 * q < dcnt; q += NT) {
        if constexpr (MT) cp_async16_hint(sVi + 4 * q, P.xdlist + dbeg + 4 * q, pol.first);
        else cp_async16(sVi + 4 * q, P.xdlist + dbeg + 4 * q);
      }
      cp_async_wait_all();
      __syncthreads();
      for (int i = tid; i < dcnt; i += NT) cp_async4(sV + i, V + sVi[i]);
      const int c_begin = ctile.begin, c_end = ctile.begin + ctile.count;
      const int g0 = c_begin + 4 * tid;
      if (!MT && s == 0 && (tid >> 5) == 1) {
        // first step of a launch, when the tables may be cold: while the voltages gather,
        // one warp asks L2 for the tile's local literals, staging positions and clause
        // memories (read next) and for phase B's bucket destinations
        const int64_t c0 = c_begin, c1 = c_end;
        prefetch_l2(P.xllit, 6 * c0, 6 * c1, tid & 31);
        prefetch_l2(P.xspos, 6 * c0, 6 * c1, tid & 31);
        prefetch_l2(P.Xs + I.cls0, 4 * c0, 4 * c1, tid & 31);
        prefetch_l2(P.Xl + I.cls0, 4 * c0, 4 * c1, tid & 31);
        if (pending) prefetch_l2(P.Cp + I.cls0, 4 * c0, 4 * c1, tid & 31);
        if (I.has_alpha_cm) prefetch_l2(P.alpha_cm + I.cls0, 4 * c0, 4 * c1, tid & 31);
        if (has_v) prefetch_l2(P.xdst, 2 * (int64_t)bbeg, 2 * ((int64_t)bbeg + blen), tid & 31);
      }
      cp_async_wait_all();
      __syncthreads();
      trace_stamp(P, s, 2);
      auto one = [&](int l0, int l1, int l2, int p0, int p1, int p2, T& xs, T& xl, T cp,
                     T al) -> T {
        if (pending) advance_memory(xs, xl, cp, al, kc);
        bool ss;
        T u0, u1, u2;
        const T C = clause3(l0, l1, l2, sV[abs(l0) - 1], sV[abs(l1) - 1], sV[abs(l2) - 1], xs,
                            xl, kc, u0, u1, u2, ss);
        stage[p0] = u0;
        stage[p1] = u1;
        stage[p2] = u2;
        unsat += !(C < T(0.5));
        vfail += !ss;
        e += (double)C;  // exact: multiples of 2^-25, scaled once per block
        return C;
      };
      auto group = [&](const Group4& q, int g) {
        T xs[4] = {q.xs.x, q.xs.y, q.xs.z, q.xs.w};
        T xl[4] = {q.xl.x, q.xl.y, q.xl.z, q.xl.w};
        T cc[4];
#pragma unroll
        for (int i = 0; i < 4; i++)
          cc[i] = one(i16_at(q.lw, 3 * i), i16_at(q.lw, 3 * i + 1), i16_at(q.lw, 3 * i + 2),
                      u16_at(q.qw, 3 * i), u16_at(q.qw, 3 * i + 1), u16_at(q.qw, 3 * i + 2), xs[i],
                      xl[i], f4_at(q.cp, i), f4_at(q.al, i));
        if constexpr (MT) {
          st_hint4(Xs + g, make_float4(xs[0], xs[1], xs[2], xs[3]), pol.first);
          st_hint4(Xl + g, make_float4(xl[0], xl[1], xl[2], xl[3]), pol.first);
          st_hint4(Cp + g, make_float4(cc[0], cc[1], cc[2], cc[3]), pol.first);
        } else {
          *reinterpret_cast<float4*>(Xs + g) = make_float4(xs[0], xs[1], xs[2], xs[3]);
          *reinterpret_cast<float4*>(Xl + g) = make_float4(xl[0], xl[1], xl[2], xl[3]);
          *reinterpret_cast<float4*>(Cp + g) = make_float4(cc[0], cc[1], cc[2], cc[3]);
        }
      };
      auto single = [&](int c) {
        T xs = Xs[c], xl = Xl[c];
        const T cp = pending ? Cp[c] : T(0);
        const T al = acm ? acm[c] : kc.alpha;
        Cp[c] = one(__ldg(ll + 3 * c), __ldg(ll + 3 * c + 1), __ldg(ll + 3 * c + 2),
                    __ldg(sp + 3 * c), __ldg(sp + 3 * c + 1), __ldg(sp + 3 * c + 2), xs, xl, cp,
                    al);
        Xs[c] = xs;
        Xl[c] = xl;
      };
      // rounds of 4-clause groups (one per thread); a remainder of at most 2 NT clauses
      // goes out as pairs, so that the last round spreads over twice as many threads with
      // half the work each
      const int count = c_end - c_begin;
      const int full_end = c_begin + count / (4 * NT) * (4 * NT);
      const int rem = c_end - full_end;
      const bool pairs = rem <= 2 * NT;
      const int g_end = pairs ? full_end : full_end + (rem & ~3);
      for (int g = g0; g < g_end; g += 4 * NT) {
        Group4 q;
        if constexpr (MT) {
          load_words4_hint(q, ll, sp, g, pol.first);
          load_state4_hint(q, Xs, Xl, Cp, acm, kc.alpha, pending, g, pol.first);
        } else {
          load_words4(q, ll, sp, g);
          load_state4(q, Xs, Xl, Cp, acm, kc.alpha, pending, g);
        }
        group(q, g);
      }
      if (pairs) {
        const int c = full_end + 2 * tid;  // even: 4-byte aligned words, 8-byte state
        if (c + 2 <= c_end) {
          const int* L3 = reinterpret_cast<const int*>(ll + 3 * c);
          const unsigned* Q3 = reinterpret_cast<const unsigned*>(sp + 3 * c);
          int lw[3];
          unsigned qw[3];
#pragma unroll
          for (int r = 0; r < 3; r++) {
            lw[r] = __ldg(L3 + r);
            qw[r] = __ldg(Q3 + r);
          }
          auto lit = [&](int k) {
            return (k & 1) ? (lw[k >> 1] >> 16) : (int)(short)(lw[k >> 1] & 0xffff);
          };
          auto pos = [&](int k) { return (int)((k & 1) ? (qw[k >> 1] >> 16) : (qw[k >> 1] & 0xffffu)); };
          const float2 xs2 = *reinterpret_cast<const float2*>(Xs + c);
          const float2 xl2 = *reinterpret_cast<const float2*>(Xl + c);
          const float2 cp2 = pending ? *reinterpret_cast<const float2*>(Cp + c) : make_float2(0.f, 0.f);
          const float2 al2 = acm ? *reinterpret_cast<const float2*>(acm + c)
                                 : make_float2(kc.alpha, kc.alpha);
          T xs[2] = {xs2.x, xs2.y}, xl[2] = {xl2.x, xl2.y}, cc[2];
          cc[0] = one(lit(0), lit(1), lit(2), pos(0), pos(1), pos(2), xs[0], xl[0], cp2.x, al2.x);
          cc[1] = one(lit(3), lit(4), lit(5), pos(3), pos(4), pos(5), xs[1], xl[1], cp2.y, al2.y);
          *reinterpret_cast<float2*>(Xs + c) = make_float2(xs[0], xs[1]);
          *reinterpret_cast<float2*>(Xl + c) = make_float2(xl[0], xl[1]);
          *reinterpret_cast<float2*>(Cp + c) = make_float2(cc[0], cc[1]);
        } else if (c < c_end) {
          single(c);
        }
      } else if (g_end + tid < c_end) {
        single(g_end + tid);  // fewer than 4 clauses
      }
      if constexpr (MT) {
        __syncthreads();  // the staging area is complete
        const float4* src = reinterpret_cast<const float4*>(stage);
        for (int i = tid; i < ulen / 4; i += NT) st_hint4(P.ux + ubase + 4 * i, src[i], pol.last);
        __syncthreads();  // before the next tile reuses the voltage and staging areas
        continue;
      }
      unsat = warp_sum_i(unsat);
      vfail = warp_sum_i(vfail);
      if ((tid & 31) == 0) {
        cnt[0][tid >> 5] = unsat;
        cnt[1][tid >> 5] = vfail;
      }
      const double et = block_sum<NT>(e, red) * kEnergyUnitF32;  // also completes the staging area
      {
        float4* __restrict__ dst = reinterpret_cast<float4*>(P.ux + ubase);
        const float4* src = reinterpret_cast<const float4*>(stage);
        for (int i = tid; i < ulen / 4; i += NT) dst[i] = src[i];
      }
      if (tid == 0) {
        int tu = 0, tv = 0;
#pragma unroll
        for (int i = 0; i < NT / 32; i++) {
          tu += cnt[0][i];
          tv += cnt[1][i];
        }
        if (tu) atomicAdd(&acc->loc, tu);
        if (tv) atomicAdd(&acc->vfail, tv);
        atomicAdd(&acc->energy, (unsigned long long)et);
      }
    }
    if constexpr (MT) {
      if (has_c) {  // the counts of all the block's clause tiles, once
        unsat = warp_sum_i(unsat);
        vfail = warp_sum_i(vfail);
        if ((tid & 31) == 0) {
          cnt[0][tid >> 5] = unsat;
          cnt[1][tid >> 5] = vfail;
        }
        const double et = block_sum<NT>(e, red) * kEnergyUnitF32;
        if (tid == 0) {
          int tu = 0, tv = 0;
#pragma unroll
          for (int i = 0; i < NT / 32; i++) {
            tu += cnt[0][i];
            tv += cnt[1][i];
          }
          if (tu) atomicAdd(&acc->loc, tu);
          if (tv) atomicAdd(&acc->vfail, tv);
          atomicAdd(&acc->energy, (unsigned long long)et);
        }
      }
    }
    trace_stamp(P, s, 3);

    // ---- barrier 1 (split): the variable tile's voltages load during the wait
    __syncthreads();
    if (tid == 0) {
      red_release(bar, 1u);
    }
    target += gridDim.x + (s == 0 ? P.barrier_extra : 0);
    T cv = T(0);
    if (has_v) {  // V(step) of the (first) variable tile's variables
      const Tile t0 = MT ? P.vtiles[b] : vtile;
      if (tid < t0.count) cv = V[t0.begin + tid];
    }
    if (tid == 0) {
      int ok = 1;
      long long it = 0;
      while (ld_acquire(bar) < target) {
        if (++it > kBarrierSpinLimit) {
          ok = 0;
          atomicExch(err, 1);
          break;
        }
        __nanosleep(kPollSleepNs);
      }
      s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) {
      leave_launch(bar);  // every block gives up in turn; the last one clears the area
      return;
    }
    trace_stamp(P, s, 4);

    // every block has finished step s-1, whose barrier 2 read the other slot last
    if (tid == 0 && b == 0) {
      StepAcc* z = P.acc2 + ((s + 1) & 1);
      z->loc = 0;
      z->vfail = 0;
      z->kmax = 0;
      z->energy = 0ull;
      z->arrive = 0ull;
    }
    trace_stamp(P, s, 5);

    // ---- phase B
    int kmax_b = 0;
    // the block's variable tiles: b, b + grid, ... (one, b, without MT)
    for (int vt = b; vt < nvt; vt += MT ? (int)gridDim.x : nvt) {
      if constexpr (MT) {
        const int k = (vt - b) / (int)gridDim.x;
        if (tid == 0) {
          if (k < kXpMetaTiles) {
            const XpMetaV& mv = s_mv[k];
            vtile.begin = mv.begin;
            vtile.count = mv.count;
            bbeg = mv.bbeg;
            blen = mv.blen;
          } else {
            vtile = P.vtiles[vt];
            bbeg = __ldg(P.xboff + vt);
            blen = __ldg(P.xboff + vt + 1) - bbeg;
          }
        }
        __syncthreads();
        const int32_t* vend = P.vend + I.var0;
        const int jb = k < kXpMetaTiles ? s_mv[k].jb
                                        : vtile.begin > 0 ? __ldg(vend + vtile.begin - 1) : 0;
        for (int g = tid; g < blen / 8; g += NT) s_src8[g] = __ldg(P.xsrc8 + bbeg / 8 + g);
        for (int i = tid; i <= vtile.count; i += NT)
          s_vend[i] = i == 0 ? 0 : __ldg(vend + vtile.begin + i - 1) - jb;
        for (int i = tid; i < vtile.count; i += NT) s_unit[i] = P.unit[I.var0 + vtile.begin + i];
        __syncthreads();
      }
      const int nv = vtile.count, v0 = vtile.begin;
      // the tile's chunks, 4 values per thread and pass: one 16-byte load of a chunk (L2,
      // written by other blocks this step) and four shared stores to the values'
      // variable-major positions
      {
        const uint2* __restrict__ xd4 = reinterpret_cast<const uint2*>(P.xdst + bbeg);
        const int nb4 = blen / 4;
#pragma unroll 4
        for (int q = tid; q < nb4; q += NT) {
          const int p = 4 * q;
          float4 val;
          uint2 w;
          if constexpr (MT) {
            val = ld_hint4(P.ux + s_src8[p >> 3] + (p & 7), pol.first);
            const int2 wi = ld_hint_i2(xd4 + q, pol.first);
            w = make_uint2((unsigned)wi.x, (unsigned)wi.y);
          } else {
            val = __ldcg(reinterpret_cast<const float4*>(P.ux + s_src8[p >> 3] + (p & 7)));
            w = __ldg(xd4 + q);
          }
          const unsigned d0 = w.x & 0xffffu, d1 = w.x >> 16, d2 = w.y & 0xffffu, d3 = w.y >> 16;
          if (d0 != kXpPad) bucket[d0] = val.x;
          if (d1 != kXpPad) bucket[d1] = val.y;
          if (d2 != kXpPad) bucket[d2] = val.z;
          if (d3 != kXpPad) bucket[d3] = val.w;
        }
      }
      if (vt == b) {
        if (tid < nv) s_cur[tid] = cv;
        for (int i = tid + NT; i < nv; i += NT) s_cur[i] = V[v0 + i];
      } else {
        for (int i = tid; i < nv; i += NT) s_cur[i] = V[v0 + i];
      }
      __syncthreads();
      trace_stamp(P, s, 6);
      T* __restrict__ nxt = P.cand + (int64_t)((set ^ 1) * kTrials) * P.var_cap + I.var0;
      constexpr int VPP = NT / G;
      const int grp = tid / G, lane = tid % G;
      for (int vb = 0; vb < nv; vb += VPP) {
        const int i = vb + grp;
        const bool valid = i < nv;
        int s0 = 0, s1 = 0;
        if (valid) {
          s0 = s_vend[i] - s_vend[0];
          s1 = s_vend[i + 1] - s_vend[0];
        }
        const T dv = tree_sum<T, G, true, int32_t>(bucket + s0, nullptr, s1 - s0, lane);
        if constexpr (G >= kTrials) {
          // every lane of the group holds dv: lane k forms candidate k, and the group's
          // first accepted trial is the lowest accepting lane (one ballot per warp)
          bool acc_k = false;
          if (valid && lane < kTrials) {
            const T Vv = s_cur[i];
            const int8_t un = s_unit[i];
            const T h = lane == 0 ? T(0.125) : lane == 1 ? T(0.0625) : lane == 2 ? T(0.03125)
                                                                            : T(0.015625);
            T c = add(Vv, mul(h, dv));
            if (un != 0) c = T(un);
            c = clampv(c, T(-1), T(1));
            nxt[(int64_t)lane * P.var_cap + v0 + i] = c;
            acc_k = !(fabs((double)c - (double)Vv) >= 1.0);
          }
          const unsigned bal = __ballot_sync(0xffffffffu, acc_k);
          const unsigned gb = (bal >> ((tid & 31) & ~(G - 1))) & ((1u << kTrials) - 1u);
          if (valid) kmax_b = max(kmax_b, gb ? __ffs(gb) - 1 : kTrials);
        } else if (valid && lane == 0) {
          const T Vv = s_cur[i];
          const int8_t un = s_unit[i];
          const int v = v0 + i;
          int kv = kTrials;
#pragma unroll
          for (int k = 0; k < kTrials; k++) {
            const T h = T(0.125 / (double)(1 << k));
            T c = add(Vv, mul(h, dv));
            if (un != 0) c = T(un);
            c = clampv(c, T(-1), T(1));
            nxt[(int64_t)k * P.var_cap + v] = c;
            const bool fail = fabs((double)c - (double)Vv) >= 1.0;
            if (!fail && kv == kTrials) kv = k;
          }
          kmax_b = max(kmax_b, kv);
        }
      }
      if constexpr (MT) __syncthreads();  // before the next tile reuses the shared tables
    }
    if (has_v) {
      kmax_b = warp_max_i(kmax_b);
      if ((tid & 31) == 0) cnt[0][tid >> 5] = kmax_b;
    }
    trace_stamp(P, s, 7);

    // ---- barrier 2 (carries the largest trial index) and the step decision
    __syncthreads();
    if (tid == 0) {
      int km = 0;
      if (has_v) {
#pragma unroll
        for (int i = 0; i < NT / 32; i++) km = max(km, cnt[0][i]);
      }
      red_release64(&acc->arrive, 1ull << (kArriveBits * km));
      // the step's counts of phase A (complete since barrier 1) load during the wait
      const volatile StepAcc* A = acc;
      const int loc = A->loc, vfail = A->vfail;
      const unsigned long long energy = b == 0 ? A->energy : 0ull;
      int ok = 1, kmax = 0;
      long long it = 0;
      for (;;) {
        const unsigned long long a = ld_acquire64(&acc->arrive);
        unsigned int n = 0;
        kmax = 0;
#pragma unroll
        for (int k = 0; k <= kTrials; k++) {
          const unsigned int f =
              (unsigned int)(a >> (kArriveBits * k)) & ((1u << kArriveBits) - 1);
          n += f;
          if (f) kmax = k;
        }
        if (n >= gridDim.x) break;
        if (++it > kBarrierSpinLimit) {
          ok = 0;
          atomicExch(err, 1);
          break;
        }
        __nanosleep(kPollSleepNs);
      }
      s_ok = ok;
      trace_stamp(P, s, 8);
      const StepDecision d = decide(loc, vfail, kmax, lc.step, I.max_steps);
      if (b == 0) {
        InstCtrl* S = P.ctrl + ii;
        if (loc < lc.best_loc) {
          S->best_loc = loc;
          S->best_t = lc.t;
          lc.best_loc = loc;
          lc.best_t = lc.t;
        }
        if (d.status == 1) {
          S->solved_step = lc.step;
          S->solved_t = lc.t;
          S->sol_set = set;
          S->sol_k = kcur;
        }
        S->loc = loc;
        S->vfail = vfail;
        S->energy = (double)energy * (1.0 / kEnergyUnitF32);
        S->t = __dadd_rn(lc.t, d.ht);
        S->step = lc.step + 1;
        S->set = set ^ 1;
        S->kcur = d.kacc;
        S->h_state = d.hs;
        S->pending = 1;
        if (d.status) {
          S->done = d.status;
          atomicSub(P.active, 1);
          const int pos = atomicAdd(P.ring_tail, 1);
          P.ring[pos % P.ring_cap] = ii;
        }
        __threadfence();
      }
      lc.t = __dadd_rn(lc.t, d.ht);
      lc.done = d.status;
      lc.step += 1;
      lc.set = set ^ 1;
      lc.kcur = d.kacc;
      lc.h = d.hs;
      lc.pending = 1;
    }
    __syncthreads();
    if (!s_ok) {
      leave_launch(bar);  // every block gives up in turn; the last one clears the area
      return;
    }
    trace_stamp(P, s, 9);
  }
  cp_async_wait_all();  // a launch on a finished formula left the prologue's copies pending
  leave_launch(bar);
  trace_launch(P, 1);
}

}  // namespace dmm
