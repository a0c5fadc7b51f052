// One block per formula for batches of small formulas (FP32 production path).
//
// A block takes a formula from a work queue (largest first) and runs many steps of it on
// its own: V and dV of the formula live in shared memory, and so do the per-literal
// contributions when they fit; the formula's literals, CSR and clause memories are re-read
// from L2, where they stay across the block's steps.  No grid-wide synchronization is
// needed, because the step decision (the accepted trial) is a block reduction.
//
// The arithmetic is the tile path's (same clause, canonical-sum and candidate code), and
// the control state is written back in the same layout, so a formula's results do not
// depend on which path or batch ran it.
#pragma once

#include "dmm_step.cuh"

namespace dmm {

constexpr int kInstThreads = 1024;
constexpr int kInstVCap = 8192;    // variables whose V and dV fit in shared memory
// literal slots whose contributions fit in shared memory: V, dV and these make 190 KB per
// block, under the carve-out step (about 195 KB) past which the L1 shrinks to a fraction
// (the 4096-formula batch ran 7 % slower with 36,864 slots, 213 KB)
constexpr int kInstUCap = 32256;
constexpr size_t kInstSmem = (2 * (size_t)kInstVCap + kInstUCap) * sizeof(float);

struct InstBlockCtl {
  InstDesc I;
  int ii, k, done, step, set, kcur, pending, best_loc, solved_step, sol_set, sol_k, loc, vfail;
  int kacc, stop;
  double t, h_state, best_t, solved_t, energy;
  double red[kInstThreads / 32];
  int cnt[3][kInstThreads / 32];
};

template <int G>
__global__ void __launch_bounds__(kInstThreads, 1)
    k_inst(PackView<float> P, const int32_t* __restrict__ order, int count, int nsteps,
           int* queue) {
  constexpr int NT = kInstThreads;
  extern __shared__ __align__(16) float dyn[];
  __shared__ InstBlockCtl sc;
  float* sV = dyn;
  float* sdV = dyn + kInstVCap;
  float* sU = dyn + 2 * kInstVCap;
  for (;;) {
    if (threadIdx.x == 0) sc.k = atomicAdd(queue, 1);
    __syncthreads();
    if (sc.k >= count) break;
    if (threadIdx.x == 0) {
      const int ii = order[sc.k];
      sc.ii = ii;
      sc.I = P.inst[ii];
      const InstCtrl* S = P.ctrl + ii;
      sc.done = S->done;
      sc.step = S->step;
      sc.set = S->set;
      sc.kcur = S->kcur;
      sc.pending = S->pending;
      sc.best_loc = S->best_loc;
      sc.solved_step = S->solved_step;
      sc.sol_set = S->sol_set;
      sc.sol_k = S->sol_k;
      sc.loc = S->loc;
      sc.vfail = S->vfail;
      sc.t = S->t;
      sc.h_state = S->h_state;
      sc.best_t = S->best_t;
      sc.solved_t = S->solved_t;
      sc.energy = S->energy;
      sc.stop = 0;
    }
    __syncthreads();
    if (sc.done != 0) continue;  // block-uniform
    const InstDesc& I = sc.I;
    const int n = I.n, m = I.m;
    float* u = I.nslots <= kInstUCap ? sU : P.u + I.slot0;
    // variable-major storage: contribution of slot s goes to u[upos[s]]
    const int32_t* __restrict__ upos = P.upos ? P.upos + I.slot0 : nullptr;
    const int32_t* __restrict__ lit = P.lit + I.slot0;
    const int32_t* __restrict__ vsl = P.vslot + I.slot0;
    const int32_t* __restrict__ vend = P.vend + I.var0;
    const int8_t* __restrict__ unit = P.unit + I.var0;
    float* __restrict__ Xs = P.Xs + I.cls0;
    float* __restrict__ Xl = P.Xl + I.cls0;
    float* __restrict__ Cp = P.Cp + I.cls0;
    const float* __restrict__ acm = I.has_alpha_cm ? P.alpha_cm + I.cls0 : nullptr;
    {
      const float* cur = P.cand + (int64_t)(sc.set * kTrials + sc.kcur) * P.var_cap + I.var0;
      for (int v = threadIdx.x; v < n; v += NT) sV[v] = cur[v];
    }
    __syncthreads();
    for (int s = 0; s < nsteps; s++) {
      // ---- A: clauses ------------------------------------------------------------------
      const ClauseConsts<float> kc = make_consts<float>(I, sc.h_state);
      const bool pending = sc.pending != 0;
      int unsat = 0, vfail = 0;
      double e = 0.0;
      auto one_clause = [&](int c) {
        float xs = Xs[c], xl = Xl[c];
        const float al = acm ? acm[c] : kc.alpha;
        if (pending) advance_memory(xs, xl, Cp[c], al, kc);
        bool ss;
        float C;
        if (I.k3) {
          const int l0 = __ldg(lit + 3 * c), l1 = __ldg(lit + 3 * c + 1), l2 = __ldg(lit + 3 * c + 2);
          float u0, u1, u2;
          C = clause3(l0, l1, l2, sV[abs(l0) - 1], sV[abs(l1) - 1], sV[abs(l2) - 1], xs, xl, kc,
                      u0, u1, u2, ss);
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
          const int s1 = (c + 1 < m) ? P.coff[I.cls0 + c + 1] : I.nslots;
          C = clause_general(lit + s0, s1 - s0, sV, xs, xl, kc, upos ? u : u + s0,
                             upos ? upos + s0 : nullptr, ss);
        }
        Xs[c] = xs;
        Xl[c] = xl;
        Cp[c] = C;
        unsat += !(C < 0.5f);
        vfail += !ss;
        e += (double)C * kEnergyUnitF32;
      };
      if (!I.k3) {
        for (int c = threadIdx.x; c < m; c += NT) one_clause(c);
      } else {
        for (int g = 4 * threadIdx.x; g < m; g += 4 * NT) {
          if (g + 4 <= m) {
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
            float uu[12], cc[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
              if (pending) advance_memory(xs[i], xl[i], cp[i], al[i], kc);
              bool ss;
              float u0, u1, u2;
              const int l0 = L[3 * i], l1 = L[3 * i + 1], l2 = L[3 * i + 2];
              const float C = clause3(l0, l1, l2, sV[abs(l0) - 1], sV[abs(l1) - 1], sV[abs(l2) - 1],
                                      xs[i], xl[i], kc, u0, u1, u2, ss);
              uu[3 * i] = u0;
              uu[3 * i + 1] = u1;
              uu[3 * i + 2] = u2;
              cc[i] = C;
              unsat += !(C < 0.5f);
              vfail += !ss;
              e += (double)C * kEnergyUnitF32;
            }
            if (upos) {
              const int4* Q4 = reinterpret_cast<const int4*>(upos + 3 * g);
              const int4 QA = __ldg(Q4), QB = __ldg(Q4 + 1), QC = __ldg(Q4 + 2);
              const int Q[12] = {QA.x, QA.y, QA.z, QA.w, QB.x, QB.y,
                                 QB.z, QB.w, QC.x, QC.y, QC.z, QC.w};
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
            for (int c = g; c < m; c++) one_clause(c);
          }
        }
      }
      const int w = threadIdx.x >> 5;
      unsat = warp_sum_i(unsat);
      vfail = warp_sum_i(vfail);
      if ((threadIdx.x & 31) == 0) {
        sc.cnt[0][w] = unsat;
        sc.cnt[1][w] = vfail;
      }
      const double et = block_sum<NT>(e, sc.red);  // ends with the block's u visible
      // ---- B: variables ----------------------------------------------------------------
      constexpr int VPP = NT / G;
      const int grp = threadIdx.x / G, lane = threadIdx.x % G;
      int kmax = 0;
      for (int vb = 0; vb < n; vb += VPP) {
        const int v = vb + grp;
        const bool valid = v < n;
        int s0 = 0, s1 = 0;
        if (valid) {
          s1 = __ldg(vend + v);
          s0 = v > 0 ? __ldg(vend + v - 1) : 0;
        }
        const float dv = upos ? tree_sum<float, G, true, int32_t>(u + s0, nullptr, s1 - s0, lane)
                              : tree_sum<float, G, false>(u, vsl + s0, s1 - s0, lane);
        if (valid && lane == 0) {
          sdV[v] = dv;
          const float V = sV[v];
          const int8_t un = unit[v];
          int kv = kTrials;
#pragma unroll
          for (int k = 0; k < kTrials; k++) {
            const float h = float(0.125 / (double)(1 << k));
            float c = add(V, mul(h, dv));
            if (un != 0) c = float(un);
            c = clampv(c, -1.f, 1.f);
            const bool fail = fabs((double)c - (double)V) >= 1.0;
            if (!fail && kv == kTrials) kv = k;
          }
          kmax = max(kmax, kv);
        }
      }
      kmax = warp_max_i(kmax);
      if ((threadIdx.x & 31) == 0) sc.cnt[2][w] = kmax;
      __syncthreads();
      // ---- F: step decision ------------------------------------------------------------
      if (threadIdx.x == 0) {
        int loc = 0, vf = 0, km = 0;
#pragma unroll
        for (int i = 0; i < NT / 32; i++) {
          loc += sc.cnt[0][i];
          vf += sc.cnt[1][i];
          km = max(km, sc.cnt[2][i]);
        }
        const bool solved = (loc == 0 && vf == 0);
        const int kacc = km < kTrials - 1 ? km : kTrials - 1;
        const double hs = 0.125 / (double)(1 << kacc);
        const double ht = km < kTrials ? hs : 0.0078125;
        if (loc < sc.best_loc) {
          sc.best_loc = loc;
          sc.best_t = sc.t;
        }
        if (solved) {
          sc.solved_step = sc.step;
          sc.solved_t = sc.t;
          sc.sol_set = sc.set;
          sc.sol_k = sc.kcur;
        }
        sc.loc = loc;
        sc.vfail = vf;
        sc.energy = et * (1.0 / kEnergyUnitF32);
        sc.t = __dadd_rn(sc.t, ht);
        sc.step += 1;
        sc.kacc = kacc;
        sc.h_state = hs;
        sc.pending = 1;
        int st = 0;
        if (solved) st = 1;
        else if (I.max_steps > 0 && sc.step >= I.max_steps) st = 2;
        sc.done = st;
        sc.stop = st != 0;
      }
      __syncthreads();
      // ---- the accepted candidate (same arithmetic as the tile path's trial kacc) ----------
      {
        const int kacc = sc.kacc;
        const float h = float(0.125 / (double)(1 << kacc));
        float* nxt = P.cand + (int64_t)((sc.set ^ 1) * kTrials + kacc) * P.var_cap + I.var0;
        for (int v = threadIdx.x; v < n; v += NT) {
          float c = add(sV[v], mul(h, sdV[v]));
          const int8_t un = unit[v];
          if (un != 0) c = float(un);
          c = clampv(c, -1.f, 1.f);
          sV[v] = c;
          nxt[v] = c;
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        sc.set ^= 1;
        sc.kcur = sc.kacc;
      }
      __syncthreads();
      if (sc.stop) break;
    }
    if (threadIdx.x == 0) {
      InstCtrl* S = P.ctrl + sc.ii;
      S->step = sc.step;
      S->set = sc.set;
      S->kcur = sc.kcur;
      S->pending = sc.pending;
      S->best_loc = sc.best_loc;
      S->solved_step = sc.solved_step;
      S->sol_set = sc.sol_set;
      S->sol_k = sc.sol_k;
      S->loc = sc.loc;
      S->vfail = sc.vfail;
      S->t = sc.t;
      S->h_state = sc.h_state;
      S->best_t = sc.best_t;
      S->solved_t = sc.solved_t;
      S->energy = sc.energy;
      if (sc.done != 0) {
        S->done = sc.done;
        atomicSub(P.active, 1);
        const int pos = atomicAdd(P.ring_tail, 1);
        P.ring[pos % P.ring_cap] = sc.ii;
      }
      __threadfence();
    }
    __syncthreads();
  }
}

}  // namespace dmm
