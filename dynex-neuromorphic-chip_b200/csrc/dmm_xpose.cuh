// Staged form of phases A and B (FP32, one formula of 3-literal clauses, cooperative launch
// with one clause tile and one variable tile per block).
//
// The plain tile code issues one L2 request per literal occurrence in each phase (phase A
// gathers V[|l|-1] per literal, phase B gathers u through the variable->slot list), and each
// request sits behind a dependent global load.  The staged form moves both gathers into
// shared memory:
//
//   A  the voltages of the clause tile's distinct variables are gathered once, in ascending
//      variable order (neighbouring lanes share 32-byte sectors), into shared memory; the
//      clauses read them through 16-bit tile-local literals.  Each contribution is written
//      to a shared staging area grouped by destination variable tile (one chunk per
//      variable tile, padded to 8 entries = one sector) and the area is written to global
//      memory with 16-byte stores.
//   B  a variable tile copies its chunk from every clause tile (coalesced: chunks are
//      contiguous and sector-aligned) and scatters the values into shared memory at their
//      variable-major positions, then reduces each variable from there.
//
// Every clause value and every per-variable sum is computed from the same operands in the
// same order as the plain tile code, so results are identical to it.
#pragma once

#include "dmm_kernels.cuh"

namespace dmm {

constexpr int kXpUnroll = 8;            // independent loads per thread in the staged gathers
constexpr uint16_t kXpPad = 0xFFFF;     // xdst of a padding entry

__host__ __device__ constexpr int xp_align16(int bytes) { return (bytes + 15) & ~15; }

// Dynamic shared-memory layout of the staged form (byte offsets).
struct XpLayout {
  int sv, bk, src8, vend, cur, unit, total;
};

__host__ __device__ inline XpLayout xp_layout(int sv_cap, int bk_cap, int tv_cap) {
  XpLayout L;
  int o = 0;
  L.sv = o;   o += xp_align16(4 * sv_cap);        // voltages of the clause tile's variables
  L.bk = o;   o += xp_align16(4 * bk_cap);        // staging area (A) / bucket (B)
  L.src8 = o; o += xp_align16(4 * (bk_cap / 8));  // ux index of every 8 bucket positions
  L.vend = o; o += xp_align16(4 * (tv_cap + 1));  // tile-local CSR ends of the variable tile
  L.cur = o;  o += xp_align16(4 * tv_cap);        // V of the variable tile
  L.unit = o; o += xp_align16(tv_cap);            // unit pins of the variable tile
  L.total = o;
  return L;
}

// Per-block ranges of the staged form (constant for a launch).
struct XpTile {
  int dbeg, dcnt;   // distinct variables of the clause tile: xdlist[dbeg, dbeg + dcnt)
  int ubase, ulen;  // staging area of the clause tile: ux[ubase, ubase + ulen)
  int bbeg, blen;   // bucket of the variable tile: positions [bbeg, bbeg + blen)
};

// Loads the launch-constant tables of block b's variable tile into shared memory.
template <int NT>
__device__ void xp_setup(const PackView<float>& P, XpTile& sx, unsigned char* dyn, int nct,
                         int nvt) {
  const XpLayout L = xp_layout(P.xsv_cap, P.xbk_cap, P.xtv_cap);
  const int b = blockIdx.x;
  if (threadIdx.x == 0) {
    XpTile x = {0, 0, 0, 0, 0, 0};
    if (b < nct) {
      x.dbeg = __ldg(P.xdoff + b);
      x.dcnt = __ldg(P.xdoff + b + 1) - x.dbeg;
      x.ubase = __ldg(P.xubase + b);
      x.ulen = __ldg(P.xubase + b + 1) - x.ubase;
    }
    if (b < nvt) {
      x.bbeg = __ldg(P.xboff + b);
      x.blen = __ldg(P.xboff + b + 1) - x.bbeg;
    }
    sx = x;
  }
  __syncthreads();
  if (b < nvt) {
    const Tile vt = P.vtiles[b];
    const int64_t var0 = P.inst[vt.inst].var0;
    const int32_t* __restrict__ vend = P.vend + var0;
    const int jb = vt.begin > 0 ? __ldg(vend + vt.begin - 1) : 0;
    int32_t* s_src8 = reinterpret_cast<int32_t*>(dyn + L.src8);
    int32_t* s_vend = reinterpret_cast<int32_t*>(dyn + L.vend);
    int8_t* s_unit = reinterpret_cast<int8_t*>(dyn + L.unit);
    const int32_t* __restrict__ src8 = P.xsrc8 + sx.bbeg / 8;
    for (int g = threadIdx.x; g < sx.blen / 8; g += NT) s_src8[g] = __ldg(src8 + g);
    for (int i = threadIdx.x; i <= vt.count; i += NT)
      s_vend[i] = i == 0 ? 0 : __ldg(vend + vt.begin + i - 1) - jb;
    for (int i = threadIdx.x; i < vt.count; i += NT) s_unit[i] = P.unit[var0 + vt.begin + i];
  }
  __syncthreads();
}

__device__ __forceinline__ void unpack_i16x4(int2 w, int* out) {
  out[0] = (int)(short)(w.x & 0xffff);
  out[1] = w.x >> 16;
  out[2] = (int)(short)(w.y & 0xffff);
  out[3] = w.y >> 16;
}

__device__ __forceinline__ void unpack_u16x4(uint2 w, int* out) {
  out[0] = (int)(w.x & 0xffffu);
  out[1] = (int)(w.x >> 16);
  out[2] = (int)(w.y & 0xffffu);
  out[3] = (int)(w.y >> 16);
}

// ---- phase A, staged -------------------------------------------------------------------------
template <int NT>
__device__ void clause_tile_xp(const PackView<float>& P, TileSmem<NT>& sm, const XpTile& X,
                               unsigned char* dyn, int ti, int step) {
  if (sm.snap.done != 0) return;  // block-uniform
  using T = float;
  const XpLayout LY = xp_layout(P.xsv_cap, P.xbk_cap, P.xtv_cap);
  T* sV = reinterpret_cast<T*>(dyn + LY.sv);
  T* stage = reinterpret_cast<T*>(dyn + LY.bk);
  const InstDesc& I = sm.inst;
  const ClauseConsts<T> kc = make_consts<T>(I, sm.snap.h);
  const bool pending = sm.snap.pending != 0;
  const T* V = P.cand + (int64_t)(sm.snap.set * kTrials + sm.snap.kcur) * P.var_cap + I.var0;
  {
    const int32_t* __restrict__ dl = P.xdlist + X.dbeg;
    const int nd = X.dcnt;
    for (int i0 = threadIdx.x; i0 < nd; i0 += kXpUnroll * NT) {
      T val[kXpUnroll];
#pragma unroll
      for (int k = 0; k < kXpUnroll; k++) {
        const int i = i0 + k * NT;
        if (i < nd) val[k] = V[__ldg(dl + i)];
      }
#pragma unroll
      for (int k = 0; k < kXpUnroll; k++) {
        const int i = i0 + k * NT;
        if (i < nd) sV[i] = val[k];
      }
    }
  }
  __syncthreads();
  trace_stamp(P, step, 2);
  T* __restrict__ Xs = P.Xs + I.cls0;
  T* __restrict__ Xl = P.Xl + I.cls0;
  T* __restrict__ Cp = P.Cp + I.cls0;
  const T* __restrict__ acm = I.has_alpha_cm ? P.alpha_cm + I.cls0 : nullptr;
  const int16_t* __restrict__ ll = P.xllit;
  const uint16_t* __restrict__ sp = P.xspos;
  const int c_begin = sm.tile.begin, c_end = sm.tile.begin + sm.tile.count;
  int unsat = 0, vfail = 0;
  double e = 0.0;
  for (int g = c_begin + 4 * threadIdx.x; g < c_end; g += 4 * NT) {
    const int nc = min(4, c_end - g);
    int L[12], Q[12];
    T xs[4], xl[4], cp[4], al[4];
    if (nc == 4) {
      const int2* L2 = reinterpret_cast<const int2*>(ll + 3 * g);
      const uint2* Q2 = reinterpret_cast<const uint2*>(sp + 3 * g);
#pragma unroll
      for (int r = 0; r < 3; r++) {
        unpack_i16x4(__ldg(L2 + r), L + 4 * r);
        unpack_u16x4(__ldg(Q2 + r), Q + 4 * r);
      }
      const float4 xs4 = *reinterpret_cast<const float4*>(Xs + g);
      const float4 xl4 = *reinterpret_cast<const float4*>(Xl + g);
      float4 cp4 = make_float4(0.f, 0.f, 0.f, 0.f);
      if (pending) cp4 = *reinterpret_cast<const float4*>(Cp + g);
      float4 al4 = make_float4(kc.alpha, kc.alpha, kc.alpha, kc.alpha);
      if (acm) al4 = *reinterpret_cast<const float4*>(acm + g);
      xs[0] = xs4.x; xs[1] = xs4.y; xs[2] = xs4.z; xs[3] = xs4.w;
      xl[0] = xl4.x; xl[1] = xl4.y; xl[2] = xl4.z; xl[3] = xl4.w;
      cp[0] = cp4.x; cp[1] = cp4.y; cp[2] = cp4.z; cp[3] = cp4.w;
      al[0] = al4.x; al[1] = al4.y; al[2] = al4.z; al[3] = al4.w;
    } else {
#pragma unroll
      for (int i = 0; i < 4; i++) {
        xs[i] = xl[i] = cp[i] = T(0);
        al[i] = kc.alpha;
#pragma unroll
        for (int j = 0; j < 3; j++) L[3 * i + j] = Q[3 * i + j] = 0;
        if (i < nc) {
          const int c = g + i;
#pragma unroll
          for (int j = 0; j < 3; j++) {
            L[3 * i + j] = __ldg(ll + 3 * c + j);
            Q[3 * i + j] = __ldg(sp + 3 * c + j);
          }
          xs[i] = Xs[c];
          xl[i] = Xl[c];
          if (pending) cp[i] = Cp[c];
          if (acm) al[i] = acm[c];
        }
      }
    }
    T cc[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      cc[i] = T(0);
      if (i < nc) {
        if (pending) advance_memory(xs[i], xl[i], cp[i], al[i], kc);
        bool ss;
        T u0, u1, u2;
        const T C = clause3(L[3 * i], L[3 * i + 1], L[3 * i + 2], sV[abs(L[3 * i]) - 1],
                            sV[abs(L[3 * i + 1]) - 1], sV[abs(L[3 * i + 2]) - 1], xs[i], xl[i],
                            kc, u0, u1, u2, ss);
        stage[Q[3 * i]] = u0;
        stage[Q[3 * i + 1]] = u1;
        stage[Q[3 * i + 2]] = u2;
        cc[i] = C;
        unsat += !(C < T(0.5));
        vfail += !ss;
        e += (double)C * kEnergyUnitF32;
      }
    }
    if (nc == 4) {
      *reinterpret_cast<float4*>(Xs + g) = make_float4(xs[0], xs[1], xs[2], xs[3]);
      *reinterpret_cast<float4*>(Xl + g) = make_float4(xl[0], xl[1], xl[2], xl[3]);
      *reinterpret_cast<float4*>(Cp + g) = make_float4(cc[0], cc[1], cc[2], cc[3]);
    } else {
      for (int i = 0; i < nc; i++) {
        Xs[g + i] = xs[i];
        Xl[g + i] = xl[i];
        Cp[g + i] = cc[i];
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
  const double et = block_sum<NT>(e, sm.red);  // also completes the staging area
  {
    float4* __restrict__ dst = reinterpret_cast<float4*>(P.ux + X.ubase);
    const float4* src = reinterpret_cast<const float4*>(stage);
    for (int i = threadIdx.x; i < X.ulen / 4; i += NT) dst[i] = src[i];
  }
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

// ---- phase B, staged -------------------------------------------------------------------------
template <int G, int NT>
__device__ void var_tile_xp(const PackView<float>& P, TileSmem<NT>& sm, const XpTile& X,
                            unsigned char* dyn, int step) {
  if (sm.snap.done != 0) return;  // block-uniform
  using T = float;
  const XpLayout LY = xp_layout(P.xsv_cap, P.xbk_cap, P.xtv_cap);
  T* bucket = reinterpret_cast<T*>(dyn + LY.bk);
  const int32_t* s_src8 = reinterpret_cast<const int32_t*>(dyn + LY.src8);
  const int32_t* s_vend = reinterpret_cast<const int32_t*>(dyn + LY.vend);
  T* s_cur = reinterpret_cast<T*>(dyn + LY.cur);
  const int8_t* s_unit = reinterpret_cast<const int8_t*>(dyn + LY.unit);
  const InstDesc& I = sm.inst;
  const T* cur = P.cand + (int64_t)(sm.snap.set * kTrials + sm.snap.kcur) * P.var_cap + I.var0;
  T* __restrict__ nxt = P.cand + (int64_t)((sm.snap.set ^ 1) * kTrials) * P.var_cap + I.var0;
  const int v0 = sm.tile.begin, nv = sm.tile.count;
  // the tile's voltages and its chunk of every clause tile, with all loads in flight
  T cv = T(0);
  if (threadIdx.x < nv) cv = cur[v0 + threadIdx.x];
  {
    const uint16_t* __restrict__ xd = P.xdst + X.bbeg;
    const T* ux = P.ux;
    const int nb = X.blen;
    for (int p0 = threadIdx.x; p0 < nb; p0 += kXpUnroll * NT) {
      T val[kXpUnroll];
      int d[kXpUnroll];
#pragma unroll
      for (int k = 0; k < kXpUnroll; k++) {
        const int p = p0 + k * NT;
        d[k] = kXpPad;
        if (p < nb) {
          val[k] = ux[s_src8[p >> 3] + (p & 7)];
          d[k] = __ldg(xd + p);
        }
      }
#pragma unroll
      for (int k = 0; k < kXpUnroll; k++)
        if (d[k] != kXpPad) bucket[d[k]] = val[k];
    }
  }
  if (threadIdx.x < nv) s_cur[threadIdx.x] = cv;
  for (int i = threadIdx.x + NT; i < nv; i += NT) s_cur[i] = cur[v0 + i];
  __syncthreads();
  trace_stamp(P, step, 6);
  constexpr int VPP = NT / G;
  const int grp = threadIdx.x / G, lane = threadIdx.x % G;
  int kmax = 0;
  for (int vb = 0; vb < nv; vb += VPP) {
    const int i = vb + grp;
    const bool valid = i < nv;
    int s0 = 0, s1 = 0;
    if (valid) {
      s0 = s_vend[i];
      s1 = s_vend[i + 1];
    }
    const T dv = tree_sum<T, G, true, int32_t>(bucket + s0, nullptr, s1 - s0, lane);
    if (valid && lane == 0) {
      const T V = s_cur[i];
      const int8_t un = s_unit[i];
      const int v = v0 + i;
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
  }
  kmax = warp_max_i(kmax);
  if ((threadIdx.x & 31) == 0) sm.cnt[0][threadIdx.x >> 5] = kmax;
  __syncthreads();
  if (threadIdx.x == 0) {
    int km = 0;
#pragma unroll
    for (int i = 0; i < NT / 32; i++) km = max(km, sm.cnt[0][i]);
    if (km) atomicMax(sm.acc ? &sm.acc->kmax : &P.ctrl[sm.tile.inst].acc_kmax, km);
  }
  __syncthreads();
}

}  // namespace dmm
