// opeval.cuh - device evaluation of the declarative query operator and the
// warp-aggregated int64 group-by.
//
// Reference op functors: s1op..s4op (ssb/lambdas.cuh:19-152) and the synthetic
// _op (synth/synthdemo.cu:7-53): re-check the predicates of uncertain rows,
// probe dimension arrays through foreign keys, compute a dense mixed-radix
// group index and a value.  mb_op (merle_b200.h) states the same computation as
// data so it crosses the C ABI; this evaluator interprets it per selected row.
// The aggregation follows primitive.cuh:386-389 (__match_any_sync peers,
// __reduce_add_sync, leader atomicAdd) widened to int64: a 64-bit value is
// summed over the peers as three 32-bit reductions (bits 0-15, 16-31 and the
// high word), which cannot overflow for 32 lanes.
#pragma once
#include "common.cuh"

namespace mb {

__device__ __forceinline__ bool src_value(const mb_src &s, uint32_t row, uint64_t &v) {
  if (s.fk == nullptr) {
    v = load_width(s.col, row, s.width);
    return true;
  }
  const uint32_t key = __ldg(s.fk + row);
  if (s.dimsz != 0 && key >= s.dimsz) return false;
  v = load_width(s.col, key, s.width);
  return true;
}

// The op on one row; returns true if the row is kept (value, group set).
// Clause `passed` (if < nclause) is known to hold and is not re-evaluated.
__device__ __forceinline__ bool op_eval(const mb_op &O, uint32_t row, bool chk, uint32_t nr_grp,
                                        int64_t &value, uint32_t &group, uint32_t passed = ~0u) {
  if (chk) {
    uint32_t t = 0;
    for (uint32_t c = 0; c < O.nclause; ++c) {
      bool any = c == passed;
      const uint32_t len = O.clause_len[c];
      for (uint32_t k = 0; k < len; ++k, ++t) {
        if (any) continue;
        const mb_term &tm = O.terms[t];
        uint64_t v;
        if (src_value(O.src[tm.src], row, v) && v >= tm.lo && v < tm.hi) any = true;
      }
      if (!any) return false;
    }
  }
  uint32_t g = 0;
  for (uint32_t k = 0; k < O.nkey; ++k) {
    const mb_key &kk = O.keys[k];
    uint64_t v;
    if (!src_value(O.src[kk.src], row, v)) return false;
    uint32_t x = (uint32_t)v;
    if (kk.xform == MB_X_DIV) x = (uint32_t)(v / kk.div);
    else if (kk.xform == MB_X_YEAR) x = date_to_year((uint32_t)v);
    g += kk.mul * (x - kk.base);
  }
  if (g >= nr_grp) return false;
  uint64_t a = 0, b = 0;
  switch (O.vkind) {
  case MB_V_ONE: value = 1; break;
  case MB_V_COL:
    if (!src_value(O.src[O.va], row, a)) return false;
    value = (int64_t)a;
    break;
  case MB_V_MUL:
    if (!src_value(O.src[O.va], row, a) || !src_value(O.src[O.vb], row, b)) return false;
    value = (int64_t)(a * b);
    break;
  default:
    if (!src_value(O.src[O.va], row, a) || !src_value(O.src[O.vb], row, b)) return false;
    value = (int64_t)a - (int64_t)b;
    break;
  }
  group = g;
  return true;
}

// Sum of a 64-bit value over the lanes of `peers` (all of which call this).
__device__ __forceinline__ uint64_t peer_sum64(uint32_t peers, uint64_t v) {
  const uint32_t s0 = __reduce_add_sync(peers, (uint32_t)(v & 0xffffu));
  const uint32_t s1 = __reduce_add_sync(peers, (uint32_t)((v >> 16) & 0xffffu));
  const uint32_t s2 = __reduce_add_sync(peers, (uint32_t)(v >> 32));
  return (uint64_t)s0 + ((uint64_t)s1 << 16) + ((uint64_t)s2 << 32);
}

// Group-by strategies (template parameter GS).
enum { GS_SCALAR = 0, GS_SHARED = 1, GS_GLOBAL = 2, GS_HASH = 3 };

constexpr uint32_t HASH_EMPTY = 0xffffffffu;
constexpr uint32_t HASH_PROBES = 32;

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  return x ^ (x >> 16);
}

// Group counts from which a lane adds its row straight into the table
// instead of finding its peers first (match + three reductions, then one
// atomic per group and warp).  Measured on the 64-query mix at 120M rows
// (plain path): peers first below 256 groups 4.26 ms, below 64 4.19 ms,
// never 4.10 ms; the same-address atomics of a few groups cost less than
// the match.
constexpr uint32_t GRP_DIRECT_MIN = 2;

// Per-CTA group-by state in shared memory.
struct GrpCtx {
  unsigned long long *table;  // GS_SHARED: nr_grp sums; GS_HASH: hash sums
  uint32_t *keys;             // GS_HASH: keys (HASH_EMPTY = free)
  uint32_t hcap;              // GS_HASH: capacity (power of two)
  bool direct;                // GS_SHARED / GS_GLOBAL: one atomic per row (nr_grp >= GRP_DIRECT_MIN)
  unsigned long long *gout;   // global output
};

__device__ __forceinline__ void hash_add(const GrpCtx &G, uint32_t grp, uint64_t s) {
  uint32_t h = hash32(grp) & (G.hcap - 1);
  for (uint32_t p = 0; p < HASH_PROBES; ++p) {
    uint32_t k = G.keys[h];
    if (k == HASH_EMPTY) k = atomicCAS(&G.keys[h], HASH_EMPTY, grp);
    if (k == HASH_EMPTY || k == grp) {
      atomicAdd(&G.table[h], (unsigned long long)s);
      return;
    }
    h = (h + 1) & (G.hcap - 1);
  }
  atomicAdd(&G.gout[grp], (unsigned long long)s);  // table crowded: go global
}

// Warp-collective aggregation of one (kept, group, value) per lane.  All 32
// lanes must call it.
template <int GS>
__device__ __forceinline__ void aggregate(const GrpCtx &G, bool kept, uint32_t grp, int64_t val,
                                          int64_t &acc) {
  if (GS == GS_SCALAR) {
    if (kept) acc += val;
    return;
  }
  if ((GS == GS_SHARED || GS == GS_GLOBAL) && G.direct) {  // uniform over the warp
    if (kept) atomicAdd(GS == GS_SHARED ? &G.table[grp] : &G.gout[grp], (unsigned long long)val);
    return;
  }
  const uint32_t key = kept ? grp : 0xffffffffu;
  const uint32_t peers = __match_any_sync(0xffffffffu, key);
  if (!kept) return;
  const uint64_t s = peer_sum64(peers, (uint64_t)val);
  if ((threadIdx.x & 31) != (uint32_t)(__ffs(peers) - 1)) return;
  if (GS == GS_SHARED) atomicAdd(&G.table[grp], (unsigned long long)s);
  else if (GS == GS_GLOBAL) atomicAdd(&G.gout[grp], (unsigned long long)s);
  else hash_add(G, grp, s);
}

// Shared-memory bytes of the group state.
__host__ __device__ inline size_t grp_smem_bytes(int gs, uint32_t nr_grp, uint32_t hcap) {
  if (gs == GS_SHARED) return (size_t)nr_grp * 8;
  if (gs == GS_HASH) return (size_t)hcap * 12;
  return 0;
}

// Carves the group state out of `smem` and zeroes it (block-collective;
// callers __syncthreads() afterwards).
template <int GS>
__device__ __forceinline__ GrpCtx grp_init(uint8_t *smem, uint32_t nr_grp, uint32_t hcap,
                                           unsigned long long *gout) {
  GrpCtx G;
  G.gout = gout;
  G.hcap = hcap;
  G.direct = nr_grp >= GRP_DIRECT_MIN;
  G.table = reinterpret_cast<unsigned long long *>(smem);
  G.keys = reinterpret_cast<uint32_t *>(smem + (size_t)hcap * 8);
  if (GS == GS_SHARED)
    for (uint32_t i = threadIdx.x; i < nr_grp; i += blockDim.x) G.table[i] = 0;
  if (GS == GS_HASH)
    for (uint32_t i = threadIdx.x; i < hcap; i += blockDim.x) {
      G.table[i] = 0;
      G.keys[i] = HASH_EMPTY;
    }
  return G;
}

// Block reduction of two 64-bit values; result valid in thread 0.
__device__ __forceinline__ void block_sum2(uint64_t &a, uint64_t &b, uint64_t *scratch /*2*32*/) {
  for (int d = 16; d; d >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, d);
    b += __shfl_down_sync(0xffffffffu, b, d);
  }
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) {
    scratch[warp] = a;
    scratch[32 + warp] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (uint32_t w = 1; w < nw; ++w) {
      a += scratch[w];
      b += scratch[32 + w];
    }
  }
}

// Flushes the per-CTA state and the per-thread scalar sum / row count to
// global memory (block-collective).
template <int GS>
__device__ __forceinline__ void grp_flush(const GrpCtx &G, uint32_t nr_grp, int64_t acc, uint64_t cnt,
                                          unsigned long long *nqual, uint64_t *scratch) {
  uint64_t a = (uint64_t)acc, c = cnt;
  block_sum2(a, c, scratch);
  if (threadIdx.x == 0) {
    if (GS == GS_SCALAR && a) atomicAdd(&G.gout[0], (unsigned long long)a);
    if (c) atomicAdd(nqual, (unsigned long long)c);
  }
  if (GS == GS_SHARED)
    for (uint32_t i = threadIdx.x; i < nr_grp; i += blockDim.x) {
      const unsigned long long v = G.table[i];
      if (v) atomicAdd(&G.gout[i], v);
    }
  if (GS == GS_HASH)
    for (uint32_t i = threadIdx.x; i < G.hcap; i += blockDim.x) {
      const uint32_t k = G.keys[i];
      if (k != HASH_EMPTY && G.table[i]) atomicAdd(&G.gout[k], G.table[i]);
    }
}

}  // namespace mb
