// Device construction of the staged form's tables (dmm_xpose.cuh) for one formula of
// 3-literal clauses with clause tiles of TC clauses and variable tiles of TV variables.
//
//   k_xp_count  (one block per clause tile t) rank of every slot within its chunk (t, b),
//               b = variable tile of its literal (slot order inside a chunk is arbitrary:
//               both sides of the transpose use the same rank, and each value lands at its
//               canonical variable-major position); chunk sizes and the sector-padded
//               staging offsets sb[t][b]; number of distinct variables.
//   k_xp_scan   (one block) offsets over tiles: staging areas, variable lists, buckets;
//               the capacities and the 16-bit range checks.
//   k_xp_fill   (one block per clause tile t) the ascending variable list, tile-local
//               literals, staging positions, bucket destinations and source table.
//
// A tile's variables are marked in a shared-memory bitmap; a variable's local index is its
// rank among the marked bits (word prefix counts + popcount).  The bitmap covers at most
// kXpRangeWords * 32 variables at a time: larger formulas are marked range by range, each
// range's ranks continuing from the marked count of the ranges before it.
#pragma once

namespace dmm {

constexpr int kXprepThreads = 1024;
constexpr int kXpRangeWords = 8192;  // bitmap words per pass (262,144 variables)

__device__ __forceinline__ int pad8i(int x) { return (x + 7) & ~7; }

// Block-wide exclusive scan of one value per thread (NT threads); returns the exclusive
// prefix and stores the total in *total.
template <int NT>
__device__ int block_exscan(int v, int* wsum, int* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = lane < NT / 32 ? wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    wsum[lane] = s;  // inclusive over warps
  }
  __syncthreads();
  const int before = (w > 0 ? wsum[w - 1] : 0) + x - v;
  *total = wsum[NT / 32 - 1];
  __syncthreads();
  return before;
}

// Marks the variables in [r0, r0 + 32 RW) of slots [s_lo, s_hi) in bits[RW] and builds the
// exclusive prefix of the words' popcounts in wpre[RW]; returns the number of marked
// variables.
template <int NT>
__device__ int xp_bitmap(const int32_t* lit, int s_lo, int s_hi, unsigned* bits, int* wpre,
                         int r0, int RW, int* wsum) {
  for (int w = threadIdx.x; w < RW; w += NT) bits[w] = 0u;
  __syncthreads();
  for (int s = s_lo + threadIdx.x; s < s_hi; s += NT) {
    const int v = abs(__ldg(lit + s)) - 1 - r0;
    if (v >= 0 && v < 32 * RW) atomicOr(&bits[v >> 5], 1u << (v & 31));
  }
  __syncthreads();
  int carry = 0;
  for (int w0 = 0; w0 < RW; w0 += NT) {
    const int w = w0 + threadIdx.x;
    const int c = w < RW ? __popc(bits[w]) : 0;
    int tot;
    const int ex = block_exscan<NT>(c, wsum, &tot);
    if (w < RW) wpre[w] = carry + ex;
    carry += tot;
  }
  __syncthreads();
  return carry;
}

template <int NT>
__global__ void __launch_bounds__(NT) k_xp_count(const int32_t* __restrict__ lit, int L, int TC,
                                                 int TV, int nvt, int n, int RW,
                                                 int* __restrict__ cnt, int* __restrict__ sb,
                                                 int* __restrict__ st, int* __restrict__ dcnt,
                                                 uint16_t* __restrict__ rank) {
  extern __shared__ __align__(16) int xp_smem[];
  __shared__ int wsum[32];
  int* c_s = xp_smem;                                            // [nvt]
  unsigned* bits = reinterpret_cast<unsigned*>(xp_smem + nvt);   // [RW]
  int* wpre = xp_smem + nvt + RW;                                // [RW]
  const int t = blockIdx.x;
  const int s_lo = 3 * t * TC, s_hi = min(L, 3 * (t + 1) * TC);
  for (int b = threadIdx.x; b < nvt; b += NT) c_s[b] = 0;
  __syncthreads();
  for (int s = s_lo + threadIdx.x; s < s_hi; s += NT) {
    const int b = (abs(__ldg(lit + s)) - 1) / TV;
    rank[s] = (uint16_t)atomicAdd(&c_s[b], 1);
  }
  int nd = 0;
  for (int r0 = 0; r0 < n; r0 += 32 * RW) nd += xp_bitmap<NT>(lit, s_lo, s_hi, bits, wpre, r0, RW, wsum);
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int b = 0; b < nvt; b++) {
      cnt[(int64_t)t * nvt + b] = c_s[b];
      sb[(int64_t)t * nvt + b] = acc;
      acc += pad8i(c_s[b]);
    }
    st[t] = acc;
    dcnt[t] = nd;
  }
}

// out[0] status (0 ok, else the number of the check that failed), [1] largest padded
// variable-list length, [2] staging / bucket capacity, [3] ux entries, [4] bucket
// positions, [5] variable-list entries, [6] largest staging area, [7] largest bucket.
// btot[nvt]: scratch for the bucket size of every variable tile.
template <int NT>
__global__ void __launch_bounds__(NT) k_xp_scan(int nct, int nvt, const int* __restrict__ cnt,
                                                const int* __restrict__ st,
                                                const int* __restrict__ dcnt,
                                                int* __restrict__ ubase, int* __restrict__ doff,
                                                int* __restrict__ bt, int* __restrict__ boff,
                                                int* __restrict__ btot, int* __restrict__ out) {
  __shared__ int s_bad;
  if (threadIdx.x == 0) {
    int64_t acc = 0, dacc = 0;
    int stmax = 0, dmax = 0, bad = 0;
    for (int t = 0; t < nct; t++) {
      ubase[t] = (int)acc;
      acc += st[t];
      stmax = max(stmax, st[t]);
      const int nd = dcnt[t];
      if (nd > 32767) bad = 1;  // 16-bit signed local literals
      doff[2 * t] = (int)dacc;
      doff[2 * t + 1] = nd;
      dacc += (nd + 3) & ~3;
      dmax = max(dmax, (nd + 3) & ~3);
    }
    ubase[nct] = (int)acc;
    if (stmax > 65535) bad = 2;  // 16-bit staging positions
    if (acc > INT32_MAX / 2 || dacc > INT32_MAX / 2) bad = 4;
    out[1] = dmax;
    out[2] = stmax;
    out[3] = (int)acc;
    out[5] = (int)dacc;
    out[6] = stmax;
    s_bad = bad;
  }
  __syncthreads();
  // bucket offsets: one thread per variable tile
  for (int b = threadIdx.x; b < nvt; b += NT) {
    int acc = 0, slots = 0;
    for (int t = 0; t < nct; t++) {
      bt[(int64_t)b * nct + t] = acc;
      acc += pad8i(cnt[(int64_t)t * nvt + b]);
      slots += cnt[(int64_t)t * nvt + b];
    }
    btot[b] = acc;
    if (slots >= 65535) atomicExch(&s_bad, 3);  // 16-bit bucket destinations
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t acc = 0;
    int bmax = 0;
    for (int b = 0; b < nvt; b++) {
      boff[b] = (int)acc;
      acc += btot[b];
      bmax = max(bmax, btot[b]);
    }
    boff[nvt] = (int)acc;
    if (acc > INT32_MAX / 2) s_bad = 4;
    out[2] = max(out[2], bmax);
    out[4] = (int)acc;
    out[7] = bmax;
    out[0] = s_bad;
  }
}

template <int NT>
__global__ void __launch_bounds__(NT) k_xp_fill(const int32_t* __restrict__ lit,
                                                const int32_t* __restrict__ upos,
                                                const int32_t* __restrict__ vend, int L, int TC,
                                                int TV, int nct, int nvt, int n, int RW,
                                                const int* __restrict__ sb,
                                                const int* __restrict__ ubase,
                                                const int* __restrict__ doff,
                                                const int* __restrict__ bt,
                                                const int* __restrict__ boff,
                                                int32_t* __restrict__ dlist,
                                                int16_t* __restrict__ llit,
                                                uint16_t* __restrict__ spos,  // in: ranks
                                                uint16_t* __restrict__ dst,
                                                int32_t* __restrict__ src8) {
  extern __shared__ __align__(16) int xp_smem[];
  __shared__ int wsum[32];
  unsigned* bits = reinterpret_cast<unsigned*>(xp_smem);  // [RW]
  int* wpre = xp_smem + RW;                               // [RW]
  int* s_sb = xp_smem + 2 * RW;                           // [nvt]
  const int t = blockIdx.x;
  const int s_lo = 3 * t * TC, s_hi = min(L, 3 * (t + 1) * TC);
  for (int b = threadIdx.x; b < nvt; b += NT) s_sb[b] = sb[(int64_t)t * nvt + b];
  __syncthreads();
  // per slot: staging position and bucket destination
  for (int s = s_lo + threadIdx.x; s < s_hi; s += NT) {
    const int v = abs(__ldg(lit + s)) - 1;
    const int b = v / TV;
    const int r = spos[s];
    spos[s] = (uint16_t)(s_sb[b] + r);
    const int jb = b * TV > 0 ? __ldg(vend + b * TV - 1) : 0;
    dst[boff[b] + bt[(int64_t)b * nct + t] + r] = (uint16_t)(__ldg(upos + s) - jb);
  }
  // the tile's variable list (ascending) and tile-local literals, range by range
  const int d0 = doff[2 * t];
  int before = 0;  // variables of the tile in the ranges already done
  for (int r0 = 0; r0 < n; r0 += 32 * RW) {
    const int nr = xp_bitmap<NT>(lit, s_lo, s_hi, bits, wpre, r0, RW, wsum);
    for (int w = threadIdx.x; w < RW; w += NT) {
      unsigned x = bits[w];
      int j = d0 + before + wpre[w];
      while (x) {
        const int bit = __ffs(x) - 1;
        dlist[j++] = r0 + 32 * w + bit;
        x &= x - 1;
      }
    }
    for (int s = s_lo + threadIdx.x; s < s_hi; s += NT) {
      const int l = __ldg(lit + s);
      const int v = abs(l) - 1 - r0;
      if (v < 0 || v >= 32 * RW) continue;
      const int loc = before + wpre[v >> 5] + __popc(bits[v >> 5] & ((1u << (v & 31)) - 1u));
      llit[s] = (int16_t)(l > 0 ? loc + 1 : -(loc + 1));
    }
    before += nr;
    __syncthreads();  // the next range rebuilds bits / wpre
  }
  // ux index of every 8 bucket positions: group g of the staging area lies in the chunk b
  // with sb[b] <= 8 g < sb[b] + pad8(cnt[t][b]), i.e. the last b with sb[b] <= 8 g (empty
  // chunks before it share its start; those after it start past 8 g)
  const int ng = (ubase[t + 1] - ubase[t]) / 8;
  for (int g = threadIdx.x; g < ng; g += NT) {
    int lo = 0, hi = nvt;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (s_sb[mid] <= 8 * g) lo = mid;
      else hi = mid;
    }
    const int k = g - s_sb[lo] / 8;
    src8[(boff[lo] + bt[(int64_t)lo * nct + t]) / 8 + k] = ubase[t] + 8 * g;
  }
}

}  // namespace dmm
