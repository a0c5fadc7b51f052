// One accepted integration step of the reference integrator (dmm_generate_dxdt and the
// adaptive dmm_dostep loop, dynex.cc:332-530, 301-327, 1389-1417) as three phases:
//
//   A  clause tiles   apply the previous step's deferred Euler update to Xs/Xl (the
//                     accepted h is only known after every variable is reduced), evaluate
//                     C_m, G, R and the per-literal contributions u (stored per literal
//                     slot), count unsatisfied clauses (C_m >= 1/2) and strict-sign
//                     failures, energy partial per tile.
//   B  variable tiles reduce each variable's contributions over the variable->slot CSR in
//                     a fixed order (no atomics), form the four Euler candidates
//                     V + h dV for h = 1/8 .. 1/64 with unit pin and clamps, and the first
//                     trial each variable accepts; max over the tile by integer atomic.
//   F  per instance   accepted trial = max over variables; t += h; solved / step limit.
//
// The four candidates replace the reference's retry loop: |clamp(V + h dV) - V| is
// monotone in h, so the first h the reference accepts is the largest h every variable
// accepts, i.e. trial max_v k_v; when no trial passes the reference keeps the 1/64 state
// and advances t by 1/128 (dynex.cc:1401-1411).
//
// Two launch forms share the tile code:
//   k_clause + k_var     one kernel per phase (F runs in the last variable tile of each
//                        instance); persistent blocks pull tiles from an atomic queue.
//   k_persist            one cooperative launch runs many steps; each block owns a static
//                        set of tiles and the phases are separated by grid barriers.
//
// Results never depend on the launch form or shape: clause work is per clause,
// per-variable sums use one canonical order for every lane grouping, tiles never straddle
// instances, cross-block combinations are integer atomics or fixed-order reductions, and
// the FP32 energy is summed as exact integers in units of 2^-25.
#pragma once

#include "dmm_kernels.cuh"

namespace dmm {

constexpr double kEnergyUnitF32 = 33554432.0;  // 2^25: every FP32 C_m is a multiple of 2^-25

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red) {
  v = warp_sum_d(v);
  const int w = threadIdx.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x < 32) {
    r = (threadIdx.x < NT / 32) ? red[threadIdx.x] : 0.0;
    r = warp_sum_d(r);
  }
  return r;
}

// Records %globaltimer at trace point k of step s (thread 0; no-op unless tracing).
template <class T>
__device__ __forceinline__ void trace_stamp(const PackView<T>& P, int s, int k) {
  if (P.trace && threadIdx.x == 0 && s < P.trace_steps) {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    const int64_t at = ((int64_t)s * kTraceK + k) * gridDim.x + blockIdx.x;
    P.trace[at] = t;
    P.trace[at + (int64_t)P.trace_steps * kTraceK * gridDim.x] = clock64();
  }
}

// Records %globaltimer at kernel entry (which 0) or exit (which 1) of this block, after
// the step stamps and clock counts (thread 0; no-op unless tracing).
template <class T>
__device__ __forceinline__ void trace_launch(const PackView<T>& P, int which) {
  if (P.trace && threadIdx.x == 0) {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    P.trace[(int64_t)2 * P.trace_steps * kTraceK * gridDim.x + which * gridDim.x + blockIdx.x] = t;
  }
}

struct TileSnap {
  int32_t done, pending, set, kcur;
  double h;
};

template <int NT>
struct TileSmem {
  InstDesc inst;
  TileSnap snap;
  Tile tile;
  int cached;  // instance whose description + snapshot are loaded, -1 for none
  StepAcc* acc;  // step accumulators (single-formula cooperative form), else null
  int ti;
  int flag;
  int vnext;  // next 32-variable group of the sorted sums (reset by the tile loaders)
  double red[NT / 32];
  int cnt[2][NT / 32];
};

// Loads tile `ti` and, when its instance differs from the cached one, the instance
// description and control snapshot.  Block-wide.  The leading barrier keeps thread 0 from
// overwriting the previous tile's state while other warps still read it: a tile of a
// finished formula returns from the tile code at once, with no block barrier of its own, so
// without it a warp could take the next tile's state for the previous tile and the block's
// barriers would fall out of step.
template <class T, int NT>
__device__ __forceinline__ void load_tile(TileSmem<NT>& sm, const PackView<T>& P, const Tile* tiles,
                                          int ti) {
  __syncthreads();
  if (threadIdx.x == 0) {
    sm.tile = tiles[ti];
    const int ii = sm.tile.inst;
    if (ii != sm.cached) {
      sm.inst = P.inst[ii];
      const InstCtrl* S = P.ctrl + ii;
      sm.snap.done = S->done;
      sm.snap.pending = S->pending;
      sm.snap.set = S->set;
      sm.snap.kcur = S->kcur;
      sm.snap.h = S->h_state;
      sm.cached = ii;
    }
    sm.vnext = 0;
  }
  __syncthreads();
}

// Adds a clause tile's unsatisfied count, strict-sign failures and energy partial to the
// step's accumulators (thread 0).
template <class T, int NT>
__device__ __forceinline__ void add_clause_counts(const PackView<T>& P, TileSmem<NT>& sm, int ti,
                                                  int tu, int tv, double et) {
  if (sm.acc) {
    if (tu) atomicAdd(&sm.acc->loc, tu);
    if (tv) atomicAdd(&sm.acc->vfail, tv);
    if (sizeof(T) == 4) atomicAdd(&sm.acc->energy, (unsigned long long)et);  // exact units
    else P.epart[ti] = et;  // FP64: summed in a fixed order (energy_sum)
  } else {
    InstCtrl* S = P.ctrl + sm.tile.inst;
    if (tu) atomicAdd(&S->acc_loc, tu);
    if (tv) atomicAdd(&S->acc_vfail, tv);
    P.epart[ti] = et;
  }
}

// ---- phase A -------------------------------------------------------------------------------
template <class T, bool VEC, int NT>
__device__ void clause_tile(const PackView<T>& P, TileSmem<NT>& sm, int ti) {
  if (sm.snap.done != 0) return;  // block-uniform
  const InstDesc& I = sm.inst;
  const ClauseConsts<T> kc = make_consts<T>(I, sm.snap.h);
  const bool pending = sm.snap.pending != 0;
  const T* V =
      P.cand + (int64_t)(sm.snap.set * kTrials + sm.snap.kcur) * P.var_cap + I.var0;
  T* __restrict__ Xs = P.Xs + I.cls0;
  T* __restrict__ Xl = P.Xl + I.cls0;
  T* __restrict__ Cp = P.Cp + I.cls0;
  const T* __restrict__ acm = I.has_alpha_cm ? P.alpha_cm + I.cls0 : nullptr;
  const int32_t* __restrict__ lit = P.lit + I.slot0;
  T* __restrict__ u = P.u + I.slot0;
  // variable-major storage: contribution of slot s goes to u[upos[s]]
  const int32_t* __restrict__ upos = P.upos ? P.upos + I.slot0 : nullptr;
  const int c_begin = sm.tile.begin, c_end = sm.tile.begin + sm.tile.count;
  // FP32: energy in exact integer units of 2^-25 (order-independent); FP64: plain sum
  const double escale = sizeof(T) == 4 ? kEnergyUnitF32 : 1.0;
  int unsat = 0, vfail = 0;
  double e = 0.0;
  auto one_clause = [&](int c) {
    T xs = Xs[c], xl = Xl[c];
    const T al = acm ? acm[c] : kc.alpha;
    if (pending) advance_memory(xs, xl, Cp[c], al, kc);
    bool ss;
    T C;
    if (I.k3) {
      const int l0 = __ldg(lit + 3 * c), l1 = __ldg(lit + 3 * c + 1), l2 = __ldg(lit + 3 * c + 2);
      T u0, u1, u2;
      C = clause3(l0, l1, l2, V[abs(l0) - 1], V[abs(l1) - 1], V[abs(l2) - 1], xs, xl, kc, u0, u1,
                  u2, ss);
      if (upos) {
        u[__ldg(upos + 3 * c)] = u0;
        u[__ldg(upos + 3 * c + 1)] = u1;
        u[__ldg(upos + 3 * c + 2)] = u2;
      } else {
        u[3 * c] = u0;
        u[3 * c + 1] = u1;
        u[3 * c + 2] = u2;
      }
    } else {
      const int s0 = P.coff[I.cls0 + c];
      const int s1 = (c + 1 < I.m) ? P.coff[I.cls0 + c + 1] : I.nslots;
      C = clause_general(lit + s0, s1 - s0, V, xs, xl, kc, upos ? u : u + s0,
                         upos ? upos + s0 : nullptr, ss);
    }
    Xs[c] = xs;
    Xl[c] = xl;
    Cp[c] = C;
    unsat += !(C < T(0.5));
    vfail += !ss;
    e += (double)C * escale;
  };
  if constexpr (!VEC) {
    for (int c = c_begin + threadIdx.x; c < c_end; c += NT) one_clause(c);
  } else if (!I.k3) {
    for (int c = c_begin + threadIdx.x; c < c_end; c += NT) one_clause(c);
  } else {
    // 4 consecutive clauses per thread: 16-byte loads of 12 literals and of Xs, Xl, C;
    // 16-byte stores of 12 contributions and of Xs, Xl, C.
    for (int g = c_begin + 4 * threadIdx.x; g < c_end; g += 4 * NT) {
      if (g + 4 <= c_end) {
        const int4* L4 = reinterpret_cast<const int4*>(lit + 3 * g);
        const int4 A = __ldg(L4), B = __ldg(L4 + 1), Cc = __ldg(L4 + 2);
        const int L[12] = {A.x, A.y, A.z, A.w, B.x, B.y, B.z, B.w, Cc.x, Cc.y, Cc.z, Cc.w};
        const float4 xs4 = *reinterpret_cast<const float4*>(Xs + g);
        const float4 xl4 = *reinterpret_cast<const float4*>(Xl + g);
        float4 cp4 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (pending) cp4 = *reinterpret_cast<const float4*>(Cp + g);
        float4 al4 = make_float4(kc.alpha, kc.alpha, kc.alpha, kc.alpha);
        if (acm) al4 = *reinterpret_cast<const float4*>(acm + g);
        float xs[4] = {xs4.x, xs4.y, xs4.z, xs4.w};
        float xl[4] = {xl4.x, xl4.y, xl4.z, xl4.w};
        const float cp[4] = {cp4.x, cp4.y, cp4.z, cp4.w};
        const float al[4] = {al4.x, al4.y, al4.z, al4.w};
        float vv[12];
#pragma unroll
        for (int i = 0; i < 12; i++) vv[i] = V[abs(L[i]) - 1];
        float uu[12], cc[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
          if (pending) advance_memory(xs[i], xl[i], T(cp[i]), T(al[i]), kc);
          bool ss;
          T u0, u1, u2;
          const T C = clause3(L[3 * i], L[3 * i + 1], L[3 * i + 2], T(vv[3 * i]), T(vv[3 * i + 1]),
                              T(vv[3 * i + 2]), T(xs[i]), T(xl[i]), kc, u0, u1, u2, ss);
          uu[3 * i] = u0;
          uu[3 * i + 1] = u1;
          uu[3 * i + 2] = u2;
          cc[i] = C;
          unsat += !(C < T(0.5));
          vfail += !ss;
          e += (double)C * escale;
        }
        if (upos) {
          const int4* Q4 = reinterpret_cast<const int4*>(upos + 3 * g);
          const int4 QA = __ldg(Q4), QB = __ldg(Q4 + 1), QC = __ldg(Q4 + 2);
          const int Q[12] = {QA.x, QA.y, QA.z, QA.w, QB.x, QB.y, QB.z, QB.w, QC.x, QC.y, QC.z, QC.w};
#pragma unroll
          for (int i = 0; i < 12; i++) u[Q[i]] = uu[i];
        } else {
          float4* U4 = reinterpret_cast<float4*>(u + 3 * g);
          U4[0] = make_float4(uu[0], uu[1], uu[2], uu[3]);
          U4[1] = make_float4(uu[4], uu[5], uu[6], uu[7]);
          U4[2] = make_float4(uu[8], uu[9], uu[10], uu[11]);
        }
        *reinterpret_cast<float4*>(Xs + g) = make_float4(xs[0], xs[1], xs[2], xs[3]);
        *reinterpret_cast<float4*>(Xl + g) = make_float4(xl[0], xl[1], xl[2], xl[3]);
        *reinterpret_cast<float4*>(Cp + g) = make_float4(cc[0], cc[1], cc[2], cc[3]);
      } else {
        for (int c = g; c < c_end; c++) one_clause(c);
      }
    }
  }
  const int w = threadIdx.x >> 5;
  unsat = warp_sum_i(unsat);
  vfail = warp_sum_i(vfail);
  if ((threadIdx.x & 31) == 0) {
    sm.cnt[0][w] = unsat;
    sm.cnt[1][w] = vfail;
  }
  const double et = block_sum<NT>(e, sm.red);
  if (threadIdx.x == 0) {
    int tu = 0, tv = 0;
#pragma unroll
    for (int i = 0; i < NT / 32; i++) {
      tu += sm.cnt[0][i];
      tv += sm.cnt[1][i];
    }
    add_clause_counts(P, sm, ti, tu, tv, et);
  }
  __syncthreads();
}

// ---- phase B -------------------------------------------------------------------------------
// MODE 0: integration step (candidates, trial index).  MODE 1: right-hand side only (dV
// to dv_out, local variable index).  Returns after a block-wide barrier.
template <class T, int G, bool SORTED, int MODE, int NT>
__device__ void var_tile(const PackView<T>& P, TileSmem<NT>& sm, double* __restrict__ dv_out) {
  if (sm.snap.done != 0) return;  // block-uniform
  const InstDesc& I = sm.inst;
  const T* u = P.u + I.slot0;
  const int32_t* __restrict__ vsl = P.vslot + I.slot0;
  const int32_t* __restrict__ vend = P.vend + I.var0;
  const T* cur =
      P.cand + (int64_t)(sm.snap.set * kTrials + sm.snap.kcur) * P.var_cap + I.var0;
  T* __restrict__ nxt = P.cand + (int64_t)((sm.snap.set ^ 1) * kTrials) * P.var_cap + I.var0;
  const int8_t* __restrict__ unit = P.unit + I.var0;
  constexpr int VPP = NT / G;
  const int grp = threadIdx.x / G, lane = threadIdx.x % G;
  const int v_end = sm.tile.begin + sm.tile.count;
  int kmax = 0;
  // candidates and trial index of variable v from its sum dv (lane 0 of its group)
  auto finish = [&](int v, T dv) {
    if (MODE == 1) {
      dv_out[v] = (double)dv;
    } else {
      const T V = cur[v];
      const int8_t un = unit[v];
      int kv = kTrials;
#pragma unroll
      for (int k = 0; k < kTrials; k++) {
        const T h = T(0.125 / (double)(1 << k));
        T c = add(V, mul(h, dv));
        if (un != 0) c = T(un);
        c = clampv(c, T(-1), T(1));
        nxt[(int64_t)k * P.var_cap + v] = c;
        const bool fail = fabs((double)c - (double)V) >= 1.0;
        if (!fail && kv == kTrials) kv = k;
      }
      kmax = max(kmax, kv);
    }
  };
  if constexpr (SORTED) {
    // FP64 reference sums, one thread per variable: a lane loads its variable's list (up to
    // 32 entries, +inf beyond its length) into registers, sorts it with a fixed network and
    // adds it left to right, so a warp keeps the loads of 32 lists in flight and needs no
    // shuffles.  Lists longer than 32 are queued for the block and summed afterwards, four
    // per warp.  Warps take their groups from shared counters: each variable's sum is
    // computed by one thread, one 8-lane segment or one warp alone, so the assignment does
    // not change any result.
    static_assert(G == 32, "the sorted sum is organized per warp");
    constexpr int R = 32;
    __shared__ int s_nlong, s_lnext;          // queued long lists; next queue group
    __shared__ int32_t s_long[kLongQueue];
    if (threadIdx.x == 0) s_nlong = s_lnext = 0;
    __syncthreads();
    const double* ud = reinterpret_cast<const double*>(u);
    const double pinf = inf_val<double>();
    (void)VPP;
    (void)grp;
    for (;;) {
      int gi = 0;
      if (lane == 0) gi = atomicAdd(&sm.vnext, 1);
      const int vb = sm.tile.begin + 32 * __shfl_sync(0xffffffffu, gi, 0);
      if (vb >= v_end) break;
      const int v = vb + lane;
      const bool valid = v < v_end;
      int s0 = 0, d = 0;
      if (valid) {
        const int s1 = __ldg(vend + v);
        s0 = v > 0 ? __ldg(vend + v - 1) : 0;
        d = s1 - s0;
      }
      const bool small = valid && d <= R;
      const int ds = small ? d : 0;
      // A variable-major list is read with 16-byte loads from the even position at or below
      // s0 (the instance's arrays start 16-byte aligned and u ends with padding, so the
      // words past the list stay in the allocation); entry r is word entry (s0 & 1) + r.
      double a[R];
      if (P.upos) {  // variable-major contributions: the list itself, two per load
        const int off = s0 & 1;
        const double2* w2 = reinterpret_cast<const double2*>(ud + (s0 - off));
        const int nw = (off + ds + 1) >> 1;
        double2 w[R / 2 + 1];
#pragma unroll
        for (int j = 0; j < R / 2 + 1; j++) w[j] = j < nw ? w2[j] : make_double2(pinf, pinf);
#pragma unroll
        for (int r = 0; r < R; r++) {
          const double e0 = (r & 1) ? w[r >> 1].y : w[r >> 1].x;        // offset 0
          const double e1 = (r & 1) ? w[(r + 1) >> 1].x : w[r >> 1].y;  // offset 1
          a[r] = r < ds ? (off ? e1 : e0) : pinf;
        }
      } else {  // slot-major contributions: gathers through the slot list
        int q[R];
#pragma unroll
        for (int r = 0; r < R; r++) q[r] = r < ds ? __ldg(vsl + s0 + r) : 0;
#pragma unroll
        for (int r = 0; r < R; r++) a[r] = r < ds ? ud[q[r]] : pinf;
      }
      sort_net<R>(a);
      double acc = 0.0;
#pragma unroll
      for (int r = 0; r < R; r++)
        if (r < ds) acc = __dadd_rn(acc, a[r]);
      if (small) finish(v, T(acc));
      // longer lists wait in the block's queue (the ones past its end are summed here)
      int qs = kLongQueue;
      if (valid && !small) qs = atomicAdd(&s_nlong, 1);
      unsigned over = __ballot_sync(0xffffffffu, valid && !small && qs >= kLongQueue);
      if (valid && !small && qs < kLongQueue) s_long[qs] = v;
      while (over) {  // warp-uniform
        const int vl = vb + __ffs(over) - 1;
        over &= over - 1;
        const int e1 = __ldg(vend + vl), e0 = vl > 0 ? __ldg(vend + vl - 1) : 0;
        const double dv = P.upos ? sorted_sum<true, int32_t>(ud + e0, nullptr, e1 - e0, lane)
                                 : sorted_sum<false>(ud, vsl + e0, e1 - e0, lane);
        if (lane == 0) finish(vl, T(dv));
      }
    }
    // the queued lists, four per warp: eight lanes and eight registers per list (up to 64
    // entries, one bitonic network for the four); longer ones warp-wide
    __syncthreads();
    const int nq = min(s_nlong, kLongQueue);
    constexpr int SEG = 8, RQ = 8;
    const int seg = lane / SEG, sl = lane % SEG;
    for (;;) {
      int gi = 0;
      if (lane == 0) gi = atomicAdd(&s_lnext, 1);
      const int q0 = 4 * __shfl_sync(0xffffffffu, gi, 0);
      if (q0 >= nq) break;
      const bool valid = q0 + seg < nq;
      const int vq = valid ? s_long[q0 + seg] : 0;
      int s0 = 0, d = 0;
      if (valid) {
        const int s1 = __ldg(vend + vq);
        s0 = vq > 0 ? __ldg(vend + vq - 1) : 0;
        d = s1 - s0;
      }
      const bool mid = valid && d <= SEG * RQ;
      double a[RQ];
#pragma unroll
      for (int r = 0; r < RQ; r++) {
        const int e = sl + SEG * r;
        a[r] = (mid && e < d) ? (P.upos ? ud[s0 + e] : ud[__ldg(vsl + s0 + e)]) : pinf;
      }
      const double acc = seg_sort_sum<SEG, RQ>(a, mid ? d : 0, lane);
      if (mid && sl == 0) finish(vq, T(acc));
      unsigned big = __ballot_sync(0xffffffffu, valid && !mid && sl == 0);
      while (big) {  // warp-uniform
        const int vl = s_long[q0 + (__ffs(big) - 1) / SEG];
        big &= big - 1;
        const int e1 = __ldg(vend + vl), e0 = vl > 0 ? __ldg(vend + vl - 1) : 0;
        const double dv = P.upos ? sorted_sum<true, int32_t>(ud + e0, nullptr, e1 - e0, lane)
                                 : sorted_sum<false>(ud, vsl + e0, e1 - e0, lane);
        if (lane == 0) finish(vl, T(dv));
      }
    }
  } else {
  for (int vb = sm.tile.begin; vb < v_end; vb += VPP) {
    const int v = vb + grp;
    const bool valid = v < v_end;
    int s0 = 0, s1 = 0;
    if (valid) {
      s1 = __ldg(vend + v);
      s0 = v > 0 ? __ldg(vend + v - 1) : 0;
    }
    const T dv = P.upos ? tree_sum<T, G, true, int32_t>(u + s0, nullptr, s1 - s0, lane)
                        : tree_sum<T, G, false>(u, vsl + s0, s1 - s0, lane);
    if (valid && lane == 0) finish(v, dv);
  }
  }
  if (MODE == 0) {
    kmax = warp_max_i(kmax);
    if ((threadIdx.x & 31) == 0) sm.cnt[0][threadIdx.x >> 5] = kmax;
    __syncthreads();
    if (threadIdx.x == 0) {
      int km = 0;
#pragma unroll
      for (int i = 0; i < NT / 32; i++) km = max(km, sm.cnt[0][i]);
      if (km) atomicMax(sm.acc ? &sm.acc->kmax : &P.ctrl[sm.tile.inst].acc_kmax, km);
    }
  }
  __syncthreads();
}

// ---- phase F -------------------------------------------------------------------------------
// The reference's step decision (dynex.cc:1389-1417) from a step's accumulators: accepted
// trial, h of the deferred memory update, time advance, status after the step.
struct StepDecision {
  int kacc;   // trial slot of the accepted candidates
  double hs;  // h of the accepted trial (1/64 when none passed)
  double ht;  // time advance (1/128 when none passed)
  int status; // 0 running, 1 solved, 2 step limit
};

__device__ __forceinline__ StepDecision decide(int loc, int vfail, int kmax, int step,
                                               int max_steps) {
  StepDecision d;
  d.kacc = kmax < kTrials - 1 ? kmax : kTrials - 1;
  d.hs = 0.125 / (double)(1 << d.kacc);
  d.ht = kmax < kTrials ? d.hs : 0.0078125;
  d.status = (loc == 0 && vfail == 0) ? 1 : (max_steps > 0 && step + 1 >= max_steps) ? 2 : 0;
  return d;
}

// Writes the control state after step S->step of instance ii (one thread).
template <class T>
__device__ void commit_step(const PackView<T>& P, const InstDesc& I, int ii, int loc, int vfail,
                            int kmax, double e) {
  InstCtrl* S = P.ctrl + ii;
  volatile InstCtrl* vS = S;
  InstCtrl c;
  // one burst of loads, then one burst of stores
  c.step = vS->step;
  c.set = vS->set;
  c.kcur = vS->kcur;
  c.best_loc = vS->best_loc;
  c.t = vS->t;
  c.best_t = vS->best_t;
  const StepDecision d = decide(loc, vfail, kmax, c.step, I.max_steps);
  if (loc < c.best_loc) {
    S->best_loc = loc;
    S->best_t = c.t;
  }
  if (d.status == 1) {
    S->solved_step = c.step;
    S->solved_t = c.t;
    S->sol_set = c.set;
    S->sol_k = c.kcur;
  }
  S->loc = loc;
  S->vfail = vfail;
  S->energy = e;
  S->t = __dadd_rn(c.t, d.ht);
  S->step = c.step + 1;
  S->set = c.set ^ 1;
  S->kcur = d.kacc;
  S->h_state = d.hs;
  S->pending = 1;
  if (d.status) {
    S->done = d.status;
    atomicSub(P.active, 1);
    const int pos = atomicAdd(P.ring_tail, 1);
    P.ring[pos % P.ring_cap] = ii;
  }
}

// A formula's energy from its clause tiles' partials, by one warp in a fixed order (lane-
// strided sums, then a butterfly), the same in the single-formula and the multi-formula
// cooperative forms: for a given tiling the value does not depend on the form (FP32
// partials are exact integers, so there it does not depend on the tiling either); valid in
// every lane.  The partials were written by other blocks before a grid barrier: read past L1.
template <class T>
__device__ __forceinline__ double energy_sum(const PackView<T>& P, int ctile0, int nctile) {
  double e = 0.0;
  for (int i = threadIdx.x & 31; i < nctile; i += 32) e = __dadd_rn(e, __ldcg(P.epart + ctile0 + i));
  return warp_sum_d(e);
}

// Finalizes one instance's step (block-wide).  Reads the accumulators of the step, writes
// the new control state, zeroes the accumulators.
template <class T, int NT>
__device__ void finalize_step(const PackView<T>& P, const InstDesc& I, int ii, double* red) {
  (void)red;
  double e = 0.0;
  if (threadIdx.x < 32) e = energy_sum(P, I.ctile0, I.nctile);
  if (threadIdx.x == 0) {
    if (sizeof(T) == 4) e = e * (1.0 / kEnergyUnitF32);
    InstCtrl* S = P.ctrl + ii;
    volatile InstCtrl* vS = S;
    const int loc = vS->acc_loc;
    const int vfail = vS->acc_vfail;
    const int kmax = vS->acc_kmax;
    commit_step(P, I, ii, loc, vfail, kmax, e);
    S->acc_loc = 0;
    S->acc_vfail = 0;
    S->acc_kmax = 0;
    S->vtiles_done = 0;
    __threadfence();
  }
}

// ---- two-kernel form -------------------------------------------------------------------------

template <class T, bool VEC>
__global__ void __launch_bounds__(kThreads) k_clause(PackView<T> P) {
  __shared__ TileSmem<kThreads> sm;
  if (threadIdx.x == 0) {
    sm.cached = -1;
    sm.acc = nullptr;
    if (blockIdx.x == 0) P.queue[1] = 0;  // the variable-tile queue is idle
  }
  const int ntiles = P.ntiles[0];
  for (;;) {
    if (threadIdx.x == 0) sm.ti = atomicAdd(&P.queue[0], 1);
    __syncthreads();
    const int ti = sm.ti;
    if (ti >= ntiles) break;
    load_tile<T, kThreads>(sm, P, P.ctiles, ti);
    clause_tile<T, VEC, kThreads>(P, sm, ti);
  }
}

template <class T, int G, bool SORTED, int MODE>
__global__ void __launch_bounds__(kThreads) k_var(PackView<T> P, double* __restrict__ dv_out) {
  __shared__ TileSmem<kThreads> sm;
  if (threadIdx.x == 0) {
    sm.cached = -1;
    sm.acc = nullptr;
    if (blockIdx.x == 0) P.queue[0] = 0;  // the clause-tile queue is idle
  }
  const int ntiles = P.ntiles[1];
  for (;;) {
    if (threadIdx.x == 0) sm.ti = atomicAdd(&P.queue[1], 1);
    __syncthreads();
    const int ti = sm.ti;
    if (ti >= ntiles) break;
    load_tile<T, kThreads>(sm, P, P.vtiles, ti);
    if (sm.snap.done != 0) continue;
    var_tile<T, G, SORTED, MODE, kThreads>(P, sm, dv_out);
    if (MODE == 0) {
      // the last variable tile of an instance finalizes its step
      if (threadIdx.x == 0) {
        __threadfence();
        const int prev = atomicAdd(&P.ctrl[sm.tile.inst].vtiles_done, 1);
        sm.flag = (prev == sm.inst.nvtile - 1);
      }
      __syncthreads();
      if (sm.flag) {
        __threadfence();
        finalize_step<T, kThreads>(P, sm.inst, sm.tile.inst, sm.red);
      }
      __syncthreads();
    }
  }
}

// ---- persistent form -------------------------------------------------------------------------

// Grid barrier for a cooperative launch: a monotonic arrival counter (zero at launch),
// release-ordered arrivals, acquire-ordered polls and a bounded wait.  Returns false, after
// raising *err, when the wait gives up (the co-residency of a cooperative launch makes this
// unreachable in practice; the bound keeps a fault from turning into a hang).
constexpr long long kBarrierSpinLimit = 1ll << 22;  // x ~0.3-1 us per poll: about a second

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Arrival with release semantics: after the block barrier that precedes it, it makes the
// whole block's earlier writes visible to a block that acquires the counter (release is
// cumulative over what the thread has observed, and the block barrier orders the other
// threads' writes before it).
__device__ __forceinline__ void red_release(unsigned int* p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void red_release64(unsigned long long* p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

template <int NT>
__device__ __forceinline__ bool grid_barrier(unsigned int* bar, unsigned int& target, int* err,
                                             int* s_ok) {
  __syncthreads();
  target += gridDim.x;
  if (threadIdx.x == 0) {
    red_release(bar, 1u);
    int ok = 1;
    long long it = 0;
    while (ld_acquire(bar) < target) {
      if (++it > kBarrierSpinLimit) {
        ok = 0;
        atomicExch(err, 1);
        break;
      }
      __nanosleep(64);
    }
    *s_ok = ok;  // the acquire load that saw the count orders everything after it
  }
  __syncthreads();
  return *s_ok != 0;
}

// Tile load of the single-formula form: description loaded once per launch, snapshot from
// the block's own copy of the control state.
struct LocalSnap {
  int done, step, set, kcur, pending;
  double h;
};

template <int NT>
__device__ __forceinline__ void load_tile_one(TileSmem<NT>& sm, const LocalSnap& ls,
                                              const Tile* tiles, int ti) {
  __syncthreads();  // as in load_tile: the previous tile's state is no longer read
  if (threadIdx.x == 0) {
    sm.tile = tiles[ti];
    sm.snap.done = ls.done;
    sm.snap.pending = ls.pending;
    sm.snap.set = ls.set;
    sm.snap.kcur = ls.kcur;
    sm.snap.h = ls.h;
    sm.vnext = 0;
  }
  __syncthreads();
}

// Number of ints at `bar` that a cooperative launch uses (barrier counter, exit counter,
// the StepAcc pair) and leaves zeroed for the next launch.
constexpr int kLaunchAreaInts = 32;

// Called by every block of a cooperative launch that did not give up at a barrier, after its
// last read of the launch area: the last block to leave zeroes the area (the barrier
// counter, this exit counter at bar[1], the step accumulators), so that the next launch on
// the stream starts from zero without a separate memset.
__device__ __forceinline__ void leave_launch(unsigned int* bar) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int prev = atomicAdd(bar + 1, 1u);
    if (prev == gridDim.x - 1) {
      volatile unsigned int* a = bar;
      for (int i = 0; i < kLaunchAreaInts; i++) a[i] = 0u;
      __threadfence();
    }
  }
}

// nsteps integration steps in one cooperative launch.  Blocks own tiles statically
// (tile ti -> block ti % gridDim.x); phases A | B | F are separated by grid barriers.
// ONE (a single formula): two grid barriers per step.  The step's counts go to the
// accumulators acc2[s & 1] (zeroed before the launch; slot (s+1) & 1 is zeroed by block 0
// once barrier 1 of step s has passed, after every block has read it in step s-1); after
// barrier 2 every block reads them and applies the step decision to its own copy of the
// control state, and block 0 writes the control state for the host.
template <class T, int G, bool SORTED, bool VEC, int NT, bool ONE = false>
__global__ void __launch_bounds__(NT, 1)
    k_persist(PackView<T> P, int nsteps, unsigned int* bar, int* err) {
  __shared__ TileSmem<NT> sm;
  __shared__ LocalSnap ls;
  __shared__ int s_ok, s_active;
  unsigned int target = 0;
  const int nct = P.ntiles[0], nvt = P.ntiles[1], nlive = *P.nlive;
  auto stamp = [&](int s, int k) { trace_stamp(P, s, k); };
  if (threadIdx.x == 0) {
    sm.acc = nullptr;
    sm.cached = -1;
    if (ONE) {
      const int ii = P.live[0];
      sm.inst = P.inst[ii];
      sm.cached = ii;
      const volatile InstCtrl* S = P.ctrl + ii;
      ls.done = S->done;
      ls.step = S->step;
      ls.set = S->set;
      ls.kcur = S->kcur;
      ls.pending = S->pending;
      ls.h = S->h_state;
    }
  }
  __syncthreads();
  for (int s = 0; s < nsteps; s++) {
    if constexpr (ONE) {
      if (ls.done != 0) break;  // grid-uniform: every block applies the same decisions
      if (threadIdx.x == 0) sm.acc = P.acc2 + (s & 1);
    } else {
      if (threadIdx.x == 0) {
        s_active = *(volatile int*)P.active;
        sm.cached = -1;
      }
      __syncthreads();
      if (s_active <= 0) break;  // grid-uniform: read after a barrier, written before one
    }
    stamp(s, 0);
    for (int ti = blockIdx.x; ti < nct; ti += gridDim.x) {
      if (ONE) load_tile_one<NT>(sm, ls, P.ctiles, ti);
      else load_tile<T, NT>(sm, P, P.ctiles, ti);
      stamp(s, 1);
      stamp(s, 2);
      clause_tile<T, VEC, NT>(P, sm, ti);
    }
    stamp(s, 3);
    if (s == 0) target += P.barrier_extra;
    if (!grid_barrier<NT>(bar, target, err, &s_ok)) {
      leave_launch(bar);  // every block gives up in turn; the last one clears the area
      return;
    }
    stamp(s, 4);
    if (ONE && blockIdx.x == 0 && threadIdx.x == 0) {
      StepAcc* z = P.acc2 + ((s + 1) & 1);
      z->loc = 0;
      z->vfail = 0;
      z->kmax = 0;
      z->energy = 0ull;
      z->arrive = 0ull;
    }
    for (int ti = blockIdx.x; ti < nvt; ti += gridDim.x) {
      if (ONE) load_tile_one<NT>(sm, ls, P.vtiles, ti);
      else load_tile<T, NT>(sm, P, P.vtiles, ti);
      stamp(s, 5);
      stamp(s, 6);
      var_tile<T, G, SORTED, 0, NT>(P, sm, nullptr);
    }
    stamp(s, 7);
    if (!grid_barrier<NT>(bar, target, err, &s_ok)) {
      leave_launch(bar);  // every block gives up in turn; the last one clears the area
      return;
    }
    stamp(s, 8);
    if constexpr (ONE) {
      double e64 = 0.0;  // FP64: the clause tiles' energy partials, summed by warp 0 of block 0
      if (sizeof(T) == 8 && blockIdx.x == 0 && threadIdx.x < 32)
        e64 = energy_sum(P, sm.inst.ctile0, sm.inst.nctile);
      if (threadIdx.x == 0) {
        const volatile StepAcc* A = P.acc2 + (s & 1);
        const int loc = A->loc, vfail = A->vfail, kmax = A->kmax;
        if (blockIdx.x == 0) {
          const double e = sizeof(T) == 4 ? (double)A->energy * (1.0 / kEnergyUnitF32) : e64;
          commit_step(P, sm.inst, P.live[0], loc, vfail, kmax, e);
          __threadfence();
        }
        const StepDecision d = decide(loc, vfail, kmax, ls.step, sm.inst.max_steps);
        ls.done = d.status;
        ls.step += 1;
        ls.set ^= 1;
        ls.kcur = d.kacc;
        ls.h = d.hs;
        ls.pending = 1;
      }
      __syncthreads();
      stamp(s, 9);
    } else {
      for (int k = blockIdx.x; k < nlive; k += gridDim.x) {
        if (threadIdx.x == 0) {
          const int ii = P.live[k];
          sm.inst = P.inst[ii];
          sm.flag = (*(volatile int*)&P.ctrl[ii].done == 0);
          sm.ti = ii;
        }
        __syncthreads();
        if (sm.flag) finalize_step<T, NT>(P, sm.inst, sm.ti, sm.red);
        __syncthreads();
      }
      stamp(s, 9);
      if (!grid_barrier<NT>(bar, target, err, &s_ok)) {
      leave_launch(bar);  // every block gives up in turn; the last one clears the area
      return;
    }
    }
  }
  leave_launch(bar);
}

}  // namespace dmm

#include "dmm_xpose.cuh"
