// wah.cu - WAH (word-aligned hybrid) compressed bitmaps: conversion between
// this library's bitmaps and the WAH streams of the reference's
// compressed-bitmap baseline, AND / OR / XOR between streams, and the
// reference's WAH file layout.
//
// Stream layout (merle/host/wahCpu.c:20-24, merle/host/wahConv.c:36-57): the
// rows are cut into 31-bit groups; a literal word (bit 31 clear) holds one
// group in its low 31 bits; a fill word (bit 31 set) stands for a run of
// groups that are all 0 (bit 30 clear) or all 0x7fffffff (bit 30 set), the
// run length in bits 0..29.  Streams written here are canonical: every run
// of equal all-0 / all-1 groups is one fill (wahCmprsCPU's output).
//
// The reference builds its GPU side from moderngpu passes (transform_scan,
// transform_lbs, transform_compact; merle/wahGpuCmprs.cu).  Here:
//   encode  (1) per-block count of stream words (a group starts a word when
//           it is a literal or differs in kind from the group before it);
//           (2) one CTA scans the block counts; (3) each block writes its
//           words, each with its starting group in a side array; (4) a
//           fill's run = the next word's starting group minus its own.
//   decode  (1)-(2) the exclusive scan of the words' group counts (what
//           wahCntExcScan computes, merle/wahGpuCmprs.cu:6-14); (3) for each
//           block of output words, the stream words covering its groups by
//           binary search over that scan; (4) each output word w holds rows
//           32w .. 32w+31 = the tail of group floor(32w/31) and the head of
//           the next one: the block stages its stream words in shared memory
//           and each thread finds its two groups there.
// All passes are HBM-bound integer work: no tensor cores.
#include <string.h>
#include <stdio.h>
#include <vector>
#include "common.cuh"

namespace mb {
namespace {

constexpr uint32_t WT = 256;          // threads of the counting / writing passes
constexpr uint32_t WI = 8;            // groups (encode) or stream words (decode) per thread
constexpr uint32_t WB = WT * WI;      // per block
constexpr uint32_t EW = WB * 31 / 32;  // bitmap words an encode block covers (2048 groups = 1984 words)
constexpr uint32_t DT = 256;          // threads of a decode block
constexpr uint32_t DV = 8;            // output words a decode thread writes
constexpr uint32_t DW = DT * DV;      // output words a decode block writes
constexpr uint32_t DCAP = 2304;       // stream words a decode block stages
constexpr uint32_t DGRP = DW * 32 / 31 + 3;  // groups a decode block's words span
constexpr uint32_t DLONG = 64;        // runs longer than 32 groups a decode block fills together
constexpr uint32_t FILL = 0x80000000u, ONES = 0x40000000u, CNT = 0x3fffffffu, LIT = 0x7fffffffu;
constexpr uint64_t MAX_GROUPS = CNT;  // a run must fit the 30-bit count
constexpr uint32_t WAH_MAGIC = 0x44f8a1efu;

// Groups of one bitmap, or of op(a, b) over two (0 AND, 1 OR, 2 XOR).
struct EncSrc {
  const uint32_t *a, *b;
  uint32_t op, order;
  uint64_t nrows, nw;  // rows; words of a (and b): ceil(nrows / 32)
};

__device__ __forceinline__ uint32_t enc_word(const EncSrc &S, uint64_t i) {
  if (i >= S.nw) return 0u;
  uint32_t v = __ldg(S.a + i);
  if (S.b) {
    const uint32_t u = __ldg(S.b + i);
    v = S.op == 0 ? v & u : S.op == 1 ? v | u : v ^ u;
  }
  return v;
}

__device__ __forceinline__ uint32_t kind_of(uint32_t v) { return v == 0 ? 0u : v == LIT ? 1u : 2u; }

// Block-wide exclusive scan of one value per thread; returns the thread's
// prefix and sets *total.  All WT threads call it.
template <typename T>
__device__ __forceinline__ T block_excl_scan(T x, T *total) {
  __shared__ T warp_sum[WT / 32];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T inc = x;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const T y = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= (uint32_t)d) inc += y;
  }
  if (lane == 31) warp_sum[warp] = inc;
  __syncthreads();
  T before = 0, all = 0;
#pragma unroll
  for (uint32_t i = 0; i < WT / 32; ++i) {
    if (i < warp) before += warp_sum[i];
    all += warp_sum[i];
  }
  __syncthreads();  // warp_sum is reused by the next call
  *total = all;
  return before + inc - x;
}

// Stages the bitmap words of encode block b (groups [WB b, WB (b + 1)) are
// rows [63488 b, 63488 (b + 1)) = words [EW b, EW (b + 1))) in shared memory:
// st[0] = word EW b - 1 (the group before the block ends in it), st[1 + i] =
// word EW b + i, st[EW + 1] = the word after.  Rows >= nrows read as 0.
__device__ __forceinline__ void enc_stage(const EncSrc &S, uint64_t b, uint32_t *st) {
  constexpr uint32_t R = (EW + 2 + WT - 1) / WT;
  const int64_t base = (int64_t)(b * EW) - 1;
  uint32_t v[R];
#pragma unroll
  for (uint32_t r = 0; r < R; ++r) {  // every load issued before the first store
    const uint32_t i = r * WT + threadIdx.x;
    const int64_t w = base + i;
    v[r] = i < EW + 2 && w >= 0 && (uint64_t)w < S.nw ? enc_word(S, (uint64_t)w) : 0u;
  }
#pragma unroll
  for (uint32_t r = 0; r < R; ++r) {
    const uint32_t i = r * WT + threadIdx.x;
    if (i >= EW + 2) break;
    const int64_t w = base + i;
    const uint64_t r0 = (uint64_t)w * 32;
    if (w >= 0 && (uint64_t)w < S.nw && r0 + 32 > S.nrows) v[r] &= (1u << (S.nrows - r0)) - 1u;
    st[i] = v[r];
  }
  __syncthreads();
}

// Local group j (-1 = the group before the block) from the staged words.
__device__ __forceinline__ uint32_t enc_group(const uint32_t *st, int32_t j, uint32_t order) {
  const uint32_t bit = (uint32_t)(32 + 31 * j), w = bit >> 5;
  uint32_t v = __funnelshift_r(st[w], st[w + 1], bit & 31) & LIT;
  if (order) v = __brev(v) >> 1;
  return v;
}

// Whether local group j (global gbase + j < G) starts a stream word: a
// literal, the first group, or a kind unlike the group before.  Threads take
// groups j = i * WT + t in round i, so neighbouring lanes read neighbouring
// shared-memory words.
__device__ __forceinline__ uint32_t enc_flag(const uint32_t *st, int32_t j, uint64_t gbase, uint64_t G,
                                             uint32_t order, uint32_t *v) {
  *v = enc_group(st, j, order);
  const uint32_t k = kind_of(*v);
  // the kind of group j - 1: lane - 1 holds it; lane 0 extracts it
  uint32_t kp = __shfl_up_sync(0xffffffffu, k, 1);
  if ((threadIdx.x & 31) == 0) kp = kind_of(enc_group(st, j - 1, order));
  const uint64_t g = gbase + (uint64_t)j;
  if (g >= G) return 0u;
  if (k == 2u || g == 0) return 1u;
  return k != kp ? 1u : 0u;
}

// Exclusive prefix of one flag per thread over the block (lane order within
// warps, warps in order); *total = the block's flags.  All WT threads call it.
__device__ __forceinline__ uint32_t block_flag_scan(uint32_t f, uint32_t *total) {
  __shared__ uint32_t wsum[WT / 32];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t bal = __ballot_sync(0xffffffffu, f);
  if (lane == 0) wsum[warp] = __popc(bal);
  __syncthreads();
  uint32_t before = 0, all = 0;
#pragma unroll
  for (uint32_t i = 0; i < WT / 32; ++i) {
    if (i < warp) before += wsum[i];
    all += wsum[i];
  }
  __syncthreads();
  *total = all;
  return before + __popc(bal & ((1u << lane) - 1u));
}

// (1) stream words each block of WB groups starts.
__global__ void __launch_bounds__(WT) wah_enc_count(const EncSrc S, uint64_t G, uint64_t *bcnt) {
  __shared__ uint32_t st[EW + 2];
  enc_stage(S, blockIdx.x, st);
  const uint64_t gbase = (uint64_t)blockIdx.x * WB;
  uint32_t c = 0, v;
#pragma unroll
  for (uint32_t i = 0; i < WI; ++i) c += enc_flag(st, (int32_t)(i * WT + threadIdx.x), gbase, G, S.order, &v);
  uint64_t total;
  block_excl_scan<uint64_t>(c, &total);
  if (threadIdx.x == 0) bcnt[blockIdx.x] = total;
}

// (2) exclusive scan of n block values in place (one CTA, four values a
// thread per round); v[n] = total.
__global__ void __launch_bounds__(1024) wah_scan_blocks(uint64_t *v, uint64_t n) {
  __shared__ uint64_t part[32];
  __shared__ uint64_t carry;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint64_t base = 0; base < n; base += 4096) {
    const uint64_t i0 = base + 4ull * threadIdx.x;
    uint64_t x[4], sum = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) x[j] = i0 + j < n ? v[i0 + j] : 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) sum += x[j];
    uint64_t inc = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint64_t y = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= (uint32_t)d) inc += y;
    }
    if (lane == 31) part[warp] = inc;
    __syncthreads();
    uint64_t at = carry, all = 0;
    for (uint32_t k = 0; k < 32; ++k) {
      if (k < warp) at += part[k];
      all += part[k];
    }
    at += inc - sum;
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (i0 + j < n) v[i0 + j] = at, at += x[j];
    __syncthreads();
    if (threadIdx.x == 0) carry += all;
    __syncthreads();
  }
  if (threadIdx.x == 0) v[n] = carry;
}

// (3) the stream words: literals in full, fills with their kind only; each
// word's starting group into pos.
__global__ void __launch_bounds__(WT) wah_enc_write(const EncSrc S, uint64_t G, const uint64_t *boff, uint32_t *out,
                                                    uint32_t *pos) {
  __shared__ uint32_t st[EW + 2];
  enc_stage(S, blockIdx.x, st);
  const uint64_t gbase = (uint64_t)blockIdx.x * WB;
  uint64_t at = boff[blockIdx.x];
#pragma unroll 1
  for (uint32_t i = 0; i < WI; ++i) {
    const int32_t j = (int32_t)(i * WT + threadIdx.x);
    uint32_t v, total;
    const uint32_t f = enc_flag(st, j, gbase, G, S.order, &v);
    const uint32_t ex = block_flag_scan(f, &total);
    if (f) {
      const uint32_t k = kind_of(v);
      out[at + ex] = k == 2u ? v : (k == 1u ? FILL | ONES : FILL);
      pos[at + ex] = (uint32_t)(gbase + (uint64_t)j);
    }
    at += total;
  }
}

// (4) fill runs.
__global__ void wah_enc_fills(uint32_t *out, const uint32_t *pos, uint64_t K, uint64_t G) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t w = out[k];
    if (w & FILL) {
      const uint64_t next = k + 1 < K ? pos[k + 1] : G;
      out[k] = w + (uint32_t)(next - pos[k]);
    }
  }
}

__device__ __forceinline__ uint64_t word_groups(uint32_t w) { return (w & FILL) ? (w & CNT) : 1u; }

// decode (1): group counts per block of WB stream words (word i * WT + t of
// the block in round i: coalesced).
__global__ void __launch_bounds__(WT) wah_dec_count(const uint32_t *wah, uint64_t n, uint64_t *bsum) {
  const uint64_t kbase = (uint64_t)blockIdx.x * WB;
  uint64_t c = 0;
#pragma unroll
  for (uint32_t i = 0; i < WI; ++i) {
    const uint64_t k = kbase + i * WT + threadIdx.x;
    if (k < n) c += word_groups(__ldg(wah + k));
  }
  uint64_t total;
  block_excl_scan<uint64_t>(c, &total);
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// decode (2b): the exclusive scan of every word's group count; S[n] = total.
// S is stored saturated at 2^32 - 1: decoding looks up groups below 2^30
// only, and min(x, cap) keeps the order of every prefix below the cap.
__device__ __forceinline__ uint32_t sat32(uint64_t x) { return x > 0xffffffffull ? 0xffffffffu : (uint32_t)x; }

__global__ void __launch_bounds__(WT) wah_dec_scan(const uint32_t *wah, uint64_t n, const uint64_t *boff,
                                                   uint64_t nblk, uint32_t *S) {
  // counts in round order (coalesced loads), regrouped through shared
  // memory so that each thread owns WI consecutive words: one block scan
  __shared__ uint32_t xs[WB + WB / 32];  // padded: index i at i + i / 32
  const uint64_t kbase = (uint64_t)blockIdx.x * WB;
  uint32_t c[WI];
#pragma unroll
  for (uint32_t i = 0; i < WI; ++i) {
    const uint64_t k = kbase + i * WT + threadIdx.x;
    c[i] = k < n ? (uint32_t)word_groups(__ldg(wah + k)) : 0u;
  }
#pragma unroll
  for (uint32_t i = 0; i < WI; ++i) {
    const uint32_t l = i * WT + threadIdx.x;
    xs[l + l / 32] = c[i];
  }
  __syncthreads();
  uint64_t sum = 0;
#pragma unroll
  for (uint32_t i = 0; i < WI; ++i) {
    const uint32_t l = threadIdx.x * WI + i;
    c[i] = xs[l + l / 32];
    sum += c[i];
  }
  uint64_t total;
  uint64_t at = boff[blockIdx.x] + block_excl_scan<uint64_t>(sum, &total);
#pragma unroll
  for (uint32_t i = 0; i < WI; ++i) {
    const uint32_t l = threadIdx.x * WI + i;
    xs[l + l / 32] = sat32(at);
    at += c[i];
  }
  __syncthreads();
#pragma unroll
  for (uint32_t i = 0; i < WI; ++i) {
    const uint32_t l = i * WT + threadIdx.x;
    const uint64_t k = kbase + l;
    if (k < n) S[k] = xs[l + l / 32];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) S[n] = sat32(boff[nblk]);
}

// Largest k in [lo, hi] with S[k] <= g (S ascending, S[lo] <= g).
__device__ __forceinline__ uint64_t last_le(const uint32_t *S, uint64_t lo, uint64_t hi, uint64_t g) {
  while (lo < hi) {
    const uint64_t mid = lo + (hi - lo + 1) / 2;
    if (S[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// decode (3): for output block b (words [DW b, DW (b + 1))), the stream
// words covering its groups.
__global__ void wah_dec_partition(const uint32_t *S, uint64_t n, uint64_t nblk, uint64_t *kb, uint64_t *ke) {
  const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblk) return;
  const uint64_t total = S[n];
  const uint64_t w0 = b * DW, w1 = w0 + DW - 1;
  const uint64_t ga = (32 * w0) / 31, gz = (32 * w1) / 31 + 1;
  if (ga >= total) {
    kb[b] = 1, ke[b] = 0;  // past the stream: an empty range
    return;
  }
  const uint64_t s = last_le(S, 0, n - 1, ga);
  kb[b] = s;
  ke[b] = last_le(S, s, n - 1, gz < total ? gz : total - 1);
}

__device__ __forceinline__ uint32_t group_value(uint32_t word, uint32_t order) {
  uint32_t x = (word & FILL) ? ((word & ONES) ? LIT : 0u) : (word & LIT);
  return order ? __brev(x) >> 1 : x;
}

// decode (4): the block expands its staged stream words into its groups in
// shared memory (0 groups are the default; runs longer than 32 groups are
// filled by all threads together), then each thread composes output words
// w = DW b + i DT + t from the two groups each spans.
__global__ void __launch_bounds__(DT) wah_dec_emit(const uint32_t *wah, const uint32_t *S, uint64_t n,
                                                   const uint64_t *kb, const uint64_t *ke, uint32_t order,
                                                   uint64_t nrows, uint64_t nw, uint64_t stride, uint32_t *bm) {
  __shared__ uint32_t s_S[DCAP + 1];
  __shared__ uint32_t s_w[DCAP];
  __shared__ uint32_t grp[DGRP];
  __shared__ uint32_t long_lo[DLONG], long_hi[DLONG], long_v[DLONG];
  __shared__ uint32_t nlong;
  const uint32_t t = threadIdx.x;
  const uint64_t b = blockIdx.x, wbase = b * DW;
  const uint64_t ga0 = (32 * wbase) / 31;
  const uint64_t lo = kb[b], hi = ke[b], total = S[n];
  const bool empty = lo > hi, staged = !empty && hi - lo + 1 <= DCAP;
  const uint32_t cnt = staged ? (uint32_t)(hi - lo + 1) : 0u;
  const uint64_t wend = wbase + DW < nw ? wbase + DW : nw;
  const uint32_t ng = wend > wbase ? (uint32_t)((32 * (wend - 1)) / 31 + 2 - ga0) : 0u;
  const uint64_t gcap = ga0 + ng < total ? ga0 + ng : total;  // groups with a value: [ga0, gcap)
  for (uint32_t j = t; j < ng; j += DT) grp[j] = 0;
  if (t == 0) nlong = 0;
  if (staged) {
    constexpr uint32_t R = (DCAP + DT - 1) / DT;
    uint32_t a[R], c[R];
#pragma unroll
    for (uint32_t r = 0; r < R; ++r) {  // every load issued before the first store
      const uint32_t i = r * DT + t;
      if (i < cnt) a[r] = S[lo + i], c[r] = __ldg(wah + lo + i);
    }
#pragma unroll
    for (uint32_t r = 0; r < R; ++r) {
      const uint32_t i = r * DT + t;
      if (i < cnt) s_S[i] = a[r], s_w[i] = c[r];
    }
    if (t == 0) s_S[cnt] = S[hi + 1];
  }
  __syncthreads();
  if (staged) {
    // local group range of the block: [0, lcap); S values are < 2^32 here
    const uint32_t g_lo = (uint32_t)ga0, lcap = (uint32_t)(gcap > ga0 ? gcap - ga0 : 0);
    for (uint32_t i = t; i < cnt; i += DT) {
      const uint32_t x = group_value(s_w[i], order);
      if (!x) continue;
      const uint32_t a = s_S[i] > g_lo ? s_S[i] - g_lo : 0u, e0 = s_S[i + 1] > g_lo ? s_S[i + 1] - g_lo : 0u;
      const uint32_t e = e0 < lcap ? e0 : lcap;
      if (a >= e) continue;
      if (e - a <= 32) {
        for (uint32_t j = a; j < e; ++j) grp[j] = x;
      } else {
        const uint32_t r = atomicAdd(&nlong, 1u);
        if (r < DLONG) long_lo[r] = a, long_hi[r] = e, long_v[r] = x;
        else
          for (uint32_t j = a; j < e; ++j) grp[j] = x;
      }
    }
  }
  __syncthreads();
  const uint32_t nl = nlong < DLONG ? nlong : DLONG;
  for (uint32_t r = 0; r < nl; ++r)
    for (uint32_t j = long_lo[r] + t; j < long_hi[r]; j += DT) grp[j] = long_v[r];
  __syncthreads();
  // word wbase + l holds rows from local group (rb + 32 l) / 31 at bit
  // (rb + 32 l) % 31 on, rb = 32 wbase - 31 ga0 (< 31): 32-bit arithmetic
  const uint32_t rb = (uint32_t)(32 * wbase - 31 * ga0);
#pragma unroll 1
  for (uint32_t i = 0; i < DV; ++i) {
    const uint32_t l = i * DT + t;
    const uint64_t w = wbase + l;
    if (w >= stride) break;
    uint32_t o = 0;
    if (!empty && w < nw) {
      const uint32_t q = rb + 32 * l, la = q / 31, sa = q - 31 * la;
      uint32_t va, vb;
      if (staged) {
        va = grp[la];
        vb = grp[la + 1];
      } else {  // more stream words than the stage holds (runs of 0 groups): search
        const uint64_t ga = ga0 + la;
        va = ga < total ? group_value(__ldg(wah + last_le(S, lo, hi, ga)), order) : 0u;
        vb = ga + 1 < total ? group_value(__ldg(wah + last_le(S, lo, hi, ga + 1)), order) : 0u;
      }
      o = (va >> sa) | (vb << (31 - sa));
      const uint64_t r0 = 32 * w;
      if (r0 + 32 > nrows) o &= nrows > r0 ? (1u << (nrows - r0)) - 1u : 0u;
    }
    bm[w] = o;
  }
}

// Encodes the groups of S into out (capacity words); *nwords = words of the
// stream, also when it does not fit (nothing is written then).
mb_status encode(const EncSrc &S, uint32_t *out, uint64_t capacity, uint64_t *nwords, cudaStream_t st,
                 const char *who) {
  const uint64_t G = ceil_div(S.nrows, 31);
  *nwords = 0;
  if (G == 0) return MB_OK;
  const uint64_t nblk = ceil_div(G, WB);
  Scratch sc(st);
  uint64_t *boff;
  MB_CHECK(sc.get(&boff, nblk + 1));
  wah_enc_count<<<(unsigned)nblk, WT, 0, st>>>(S, G, boff);
  MB_LAUNCH_CHECK("wah_enc_count");
  wah_scan_blocks<<<1, 1024, 0, st>>>(boff, nblk);
  MB_LAUNCH_CHECK("wah_scan_blocks");
  uint64_t K = 0;
  MB_CUDA(cudaMemcpyAsync(&K, boff + nblk, 8, cudaMemcpyDeviceToHost, st));
  MB_CUDA(cudaStreamSynchronize(st));
  *nwords = K;
  if (!out) return MB_OK;  // a size query
  if (K > capacity) return fail(MB_ERR_INVALID, "%s: the stream has %llu words, the output holds %llu", who,
                                (unsigned long long)K, (unsigned long long)capacity);
  uint32_t *pos;
  MB_CHECK(sc.get(&pos, K));
  wah_enc_write<<<(unsigned)nblk, WT, 0, st>>>(S, G, boff, out, pos);
  MB_LAUNCH_CHECK("wah_enc_write");
  const unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(K, 256), (uint64_t)dev_info().sms * 8);
  wah_enc_fills<<<grid, 256, 0, st>>>(out, pos, K, G);
  MB_LAUNCH_CHECK("wah_enc_fills");
  return MB_OK;
}

// The exclusive scan of the stream's group counts into a new scratch array
// S[0..n] (S[n] = the groups the stream stands for).
mb_status group_scan(const uint32_t *wah, uint64_t n, Scratch &sc, uint32_t **S_out, cudaStream_t st) {
  const uint64_t nblk = ceil_div(n, WB);
  uint64_t *boff;
  uint32_t *S;
  MB_CHECK(sc.get(&boff, nblk + 1));
  MB_CHECK(sc.get(&S, n + 1));
  wah_dec_count<<<(unsigned)nblk, WT, 0, st>>>(wah, n, boff);
  MB_LAUNCH_CHECK("wah_dec_count");
  wah_scan_blocks<<<1, 1024, 0, st>>>(boff, nblk);
  MB_LAUNCH_CHECK("wah_scan_blocks");
  wah_dec_scan<<<(unsigned)nblk, WT, 0, st>>>(wah, n, boff, nblk, S);
  MB_LAUNCH_CHECK("wah_dec_scan");
  *S_out = S;
  return MB_OK;
}

mb_status decode(const uint32_t *wah, uint64_t n, uint32_t order, uint64_t nrows, uint32_t *bm, cudaStream_t st) {
  const uint64_t stride = mb_bitmap_stride(nrows), nw = mb_bitmap_words(nrows);
  if (stride == 0) return MB_OK;
  if (n == 0) {
    MB_CUDA(cudaMemsetAsync(bm, 0, stride * 4, st));
    return MB_OK;
  }
  Scratch sc(st);
  uint32_t *S;
  MB_CHECK(group_scan(wah, n, sc, &S, st));
  const uint64_t nblk = ceil_div(stride, DW);
  uint64_t *kb, *ke;
  MB_CHECK(sc.get(&kb, nblk));
  MB_CHECK(sc.get(&ke, nblk));
  wah_dec_partition<<<(unsigned)ceil_div(nblk, 256), 256, 0, st>>>(S, n, nblk, kb, ke);
  MB_LAUNCH_CHECK("wah_dec_partition");
  wah_dec_emit<<<(unsigned)nblk, DT, 0, st>>>(wah, S, n, kb, ke, order, nrows, nw, stride, bm);
  MB_LAUNCH_CHECK("wah_dec_emit");
  return MB_OK;
}

bool aligned4(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 3) == 0; }

// ----------------------------------------------- direct (compressed) ops
// The reference's direct operations (wahAnd / wahOr / wahXor,
// merle/wahGpuDirect.cu) never expand the streams: the runs of both are cut
// at the union of their word boundaries and each piece is combined whole.
// Here: (1) the group scans SA, SB of both streams (saturated, clamped to G);
// (2) a merge of the two boundary lists by rank (an A boundary's rank is its
// index plus the B boundaries below it, a B boundary's its index plus the A
// boundaries at or below it); (3) piece r is [m[r], m[r+1]) (the last one
// ends at G), its value op(A's word, B's word) at its first group; a piece
// starts an output word when its value is a literal or its kind differs from
// the kind at the group before it; (4) fill runs as in the encoder.
struct DirectSrc {
  const uint32_t *a, *b, *SA, *SB;  // streams and their exclusive group scans
  uint64_t na, nb, G;
  uint32_t op;
};

// Value (31 bits) of op(A, B) at group g (< G), with its kind.
__device__ __forceinline__ uint32_t direct_value(const DirectSrc &D, uint64_t g) {
  uint32_t va = 0, vb = 0;
  if (D.na && g < D.SA[D.na]) va = group_value(__ldg(D.a + last_le(D.SA, 0, D.na - 1, g)), 0);
  if (D.nb && g < D.SB[D.nb]) vb = group_value(__ldg(D.b + last_le(D.SB, 0, D.nb - 1, g)), 0);
  return D.op == 0 ? va & vb : D.op == 1 ? va | vb : va ^ vb;
}

__device__ __forceinline__ uint32_t clamp_g(uint32_t x, uint64_t G) { return x < G ? x : (uint32_t)G; }

// (2) the merged boundary list m[0 .. na + nb + 1].
__global__ void wah_direct_merge(const DirectSrc D, uint32_t *m) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i <= D.na) {
    const uint32_t v = clamp_g(D.SA[i], D.G);
    uint64_t lo = 0, hi = D.nb + 1;  // B boundaries < v
    while (lo < hi) {
      const uint64_t mid = (lo + hi) / 2;
      if (clamp_g(D.SB[mid], D.G) < v) lo = mid + 1;
      else hi = mid;
    }
    m[i + lo] = v;
  } else if (i <= D.na + 1 + D.nb) {
    const uint64_t j = i - D.na - 1;
    const uint32_t v = clamp_g(D.SB[j], D.G);
    uint64_t lo = 0, hi = D.na + 1;  // A boundaries <= v
    while (lo < hi) {
      const uint64_t mid = (lo + hi) / 2;
      if (clamp_g(D.SA[mid], D.G) <= v) lo = mid + 1;
      else hi = mid;
    }
    m[j + lo] = v;
  }
}

// Piece r starts an output word: *v = its value, *x = its first group.
__device__ __forceinline__ bool direct_flag(const DirectSrc &D, const uint32_t *m, uint64_t M, uint64_t r,
                                            uint32_t *v, uint64_t *x) {
  if (r >= M) return false;
  const uint64_t x0 = m[r], y0 = r + 1 < M ? m[r + 1] : D.G;
  *x = x0;
  if (x0 >= y0 || x0 >= D.G) return false;
  *v = direct_value(D, x0);
  const uint32_t k = kind_of(*v);
  if (k == 2u || x0 == 0) return true;
  return k != kind_of(direct_value(D, x0 - 1));
}

// (3a) output words per block of WB pieces.
__global__ void __launch_bounds__(WT) wah_direct_count(const DirectSrc D, const uint32_t *m, uint64_t M,
                                                       uint64_t *bcnt) {
  uint32_t c = 0, v;
  uint64_t x;
#pragma unroll
  for (uint32_t i = 0; i < WI; ++i)
    c += direct_flag(D, m, M, (uint64_t)blockIdx.x * WB + i * WT + threadIdx.x, &v, &x) ? 1u : 0u;
  uint64_t total;
  block_excl_scan<uint64_t>(c, &total);
  if (threadIdx.x == 0) bcnt[blockIdx.x] = total;
}

// (3b) the words, in piece order; each word's first group into pos.
__global__ void __launch_bounds__(WT) wah_direct_write(const DirectSrc D, const uint32_t *m, uint64_t M,
                                                       const uint64_t *boff, uint32_t *out, uint32_t *pos) {
  uint64_t at = boff[blockIdx.x];
#pragma unroll 1
  for (uint32_t i = 0; i < WI; ++i) {
    uint32_t v = 0, total;
    uint64_t x = 0;
    const bool f = direct_flag(D, m, M, (uint64_t)blockIdx.x * WB + i * WT + threadIdx.x, &v, &x);
    const uint32_t ex = block_flag_scan(f ? 1u : 0u, &total);
    if (f) {
      const uint32_t k = kind_of(v);
      out[at + ex] = k == 2u ? v : (k == 1u ? FILL | ONES : FILL);
      pos[at + ex] = (uint32_t)x;
    }
    at += total;
  }
}

mb_status direct_op(uint32_t op, const uint32_t *a, uint64_t na, const uint32_t *b, uint64_t nb, uint64_t G,
                    uint32_t *out, uint64_t capacity, uint64_t *nwords, cudaStream_t st) {
  Scratch sc(st);
  DirectSrc D{a, b, nullptr, nullptr, na, nb, G, op};
  uint32_t *SA, *SB, *m;
  const uint32_t zero = 0;
  if (na) {
    MB_CHECK(group_scan(a, na, sc, &SA, st));
  } else {
    MB_CHECK(sc.get(&SA, 1));
    MB_CUDA(cudaMemcpyAsync(SA, &zero, 4, cudaMemcpyHostToDevice, st));
  }
  if (nb) {
    MB_CHECK(group_scan(b, nb, sc, &SB, st));
  } else {
    MB_CHECK(sc.get(&SB, 1));
    MB_CUDA(cudaMemcpyAsync(SB, &zero, 4, cudaMemcpyHostToDevice, st));
  }
  D.SA = SA, D.SB = SB;
  const uint64_t M = na + nb + 2;
  MB_CHECK(sc.get(&m, M));
  wah_direct_merge<<<(unsigned)ceil_div(M, 256), 256, 0, st>>>(D, m);
  MB_LAUNCH_CHECK("wah_direct_merge");
  const uint64_t nblk = ceil_div(M, WB);
  uint64_t *boff;
  MB_CHECK(sc.get(&boff, nblk + 1));
  wah_direct_count<<<(unsigned)nblk, WT, 0, st>>>(D, m, M, boff);
  MB_LAUNCH_CHECK("wah_direct_count");
  wah_scan_blocks<<<1, 1024, 0, st>>>(boff, nblk);
  MB_LAUNCH_CHECK("wah_scan_blocks");
  uint64_t K = 0;
  MB_CUDA(cudaMemcpyAsync(&K, boff + nblk, 8, cudaMemcpyDeviceToHost, st));
  MB_CUDA(cudaStreamSynchronize(st));
  *nwords = K;
  if (!out) return MB_OK;
  if (K > capacity) return fail(MB_ERR_INVALID, "mb_wah_op: the stream has %llu words, the output holds %llu",
                                (unsigned long long)K, (unsigned long long)capacity);
  uint32_t *pos;
  MB_CHECK(sc.get(&pos, K));
  wah_direct_write<<<(unsigned)nblk, WT, 0, st>>>(D, m, M, boff, out, pos);
  MB_LAUNCH_CHECK("wah_direct_write");
  const unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(K, 256), (uint64_t)dev_info().sms * 8);
  wah_enc_fills<<<grid, 256, 0, st>>>(out, pos, K, G);
  MB_LAUNCH_CHECK("wah_enc_fills");
  return MB_OK;
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" uint64_t mb_wah_groups(uint64_t nrows) { return ceil_div(nrows, 31); }

extern "C" mb_status mb_wah_encode(const uint32_t *bitmap, uint64_t nrows, uint32_t order, uint32_t *wah,
                                   uint64_t capacity, uint64_t *nwords, void *stream) {
  NvtxRange nvtx_("mb_wah_encode");
  if (!nwords) return fail(MB_ERR_INVALID, "mb_wah_encode: NULL word count");
  *nwords = 0;
  if (nrows && !bitmap) return fail(MB_ERR_INVALID, "mb_wah_encode: NULL bitmap");
  if (order > 1) return fail(MB_ERR_INVALID, "mb_wah_encode: order %u (0 or 1)", order);
  if (ceil_div(nrows, 31) > MAX_GROUPS)
    return fail(MB_ERR_INVALID, "mb_wah_encode: %llu rows exceed the 30-bit run count", (unsigned long long)nrows);
  if (!aligned4(bitmap) || !aligned4(wah)) return fail(MB_ERR_INVALID, "mb_wah_encode: misaligned pointer");
  const EncSrc S{bitmap, nullptr, 0, order, nrows, mb_bitmap_words(nrows)};
  return encode(S, wah, capacity, nwords, as_stream(stream), "mb_wah_encode");
}

extern "C" mb_status mb_wah_decode(const uint32_t *wah, uint64_t nwords, uint32_t order, uint64_t nrows,
                                   uint32_t *bitmap, void *stream) {
  NvtxRange nvtx_("mb_wah_decode");
  if (nwords && !wah) return fail(MB_ERR_INVALID, "mb_wah_decode: NULL stream");
  if (nrows && !bitmap) return fail(MB_ERR_INVALID, "mb_wah_decode: NULL bitmap");
  if (order > 1) return fail(MB_ERR_INVALID, "mb_wah_decode: order %u (0 or 1)", order);
  if (!aligned4(bitmap) || !aligned4(wah)) return fail(MB_ERR_INVALID, "mb_wah_decode: misaligned pointer");
  return decode(wah, nwords, order, nrows, bitmap, as_stream(stream));
}

extern "C" mb_status mb_wah_ngroups(const uint32_t *wah, uint64_t nwords, uint64_t *ngroups, void *stream) {
  if (!ngroups || (nwords && !wah)) return fail(MB_ERR_INVALID, "mb_wah_ngroups: NULL argument");
  *ngroups = 0;
  if (nwords == 0) return MB_OK;
  cudaStream_t st = as_stream(stream);
  Scratch sc(st);
  const uint64_t nblk = ceil_div(nwords, WB);
  uint64_t *boff;
  MB_CHECK(sc.get(&boff, nblk + 1));
  wah_dec_count<<<(unsigned)nblk, WT, 0, st>>>(wah, nwords, boff);
  MB_LAUNCH_CHECK("wah_dec_count");
  wah_scan_blocks<<<1, 1024, 0, st>>>(boff, nblk);
  MB_LAUNCH_CHECK("wah_scan_blocks");
  MB_CUDA(cudaMemcpyAsync(ngroups, boff + nblk, 8, cudaMemcpyDeviceToHost, st));
  MB_CUDA(cudaStreamSynchronize(st));
  return MB_OK;
}

extern "C" mb_status mb_wah_op(uint32_t op, const uint32_t *a, uint64_t na, const uint32_t *b, uint64_t nb,
                               uint64_t ngroups, uint32_t *out, uint64_t capacity, uint64_t *nwords, void *stream) {
  return mb_wah_op_ex(op, a, na, b, nb, ngroups, MB_WAH_AUTO, out, capacity, nwords, stream);
}

extern "C" mb_status mb_wah_op_ex(uint32_t op, const uint32_t *a, uint64_t na, const uint32_t *b, uint64_t nb,
                                  uint64_t ngroups, uint32_t method, uint32_t *out, uint64_t capacity,
                                  uint64_t *nwords, void *stream) {
  NvtxRange nvtx_("mb_wah_op");
  if (!nwords) return fail(MB_ERR_INVALID, "mb_wah_op: NULL word count");
  *nwords = 0;
  if (op > MB_WAH_XOR) return fail(MB_ERR_INVALID, "mb_wah_op: op %u", op);
  if (method > MB_WAH_DIRECT) return fail(MB_ERR_INVALID, "mb_wah_op: method %u", method);
  if ((na && !a) || (nb && !b)) return fail(MB_ERR_INVALID, "mb_wah_op: NULL stream");
  if (ngroups > MAX_GROUPS) return fail(MB_ERR_INVALID, "mb_wah_op: %llu groups exceed the 30-bit run count",
                                        (unsigned long long)ngroups);
  if (ngroups == 0) return MB_OK;
  cudaStream_t st = as_stream(stream);
  // direct when the streams are short next to the groups: its work follows
  // the words (with a binary search per piece), the explicit form's the rows
  if (method == MB_WAH_DIRECT || (method == MB_WAH_AUTO && 8 * (na + nb) < ngroups))
    return direct_op(op, a, na, b, nb, ngroups, out, capacity, nwords, st);
  // decode both (the order is immaterial: both sides and the result keep
  // the streams' own), then encode op(x, y)
  const uint64_t nrows = 31 * ngroups, stride = mb_bitmap_stride(nrows);
  Scratch sc(st);
  uint32_t *x, *y;
  MB_CHECK(sc.get(&x, stride));
  MB_CHECK(sc.get(&y, stride));
  MB_CHECK(decode(a, na, 0, nrows, x, st));
  MB_CHECK(decode(b, nb, 0, nrows, y, st));
  const EncSrc S{x, y, op, 0, nrows, mb_bitmap_words(nrows)};
  return encode(S, out, capacity, nwords, st, "mb_wah_op");
}

// The reference's WAH file (struct wahHost_s, merle/host/wahCpu.h:10-15, read
// whole by loadWahFile, merle/host/wahConv.c:93-109): has1Fill (bool, then 3
// pad bytes), magic 0x44f8a1ef, cmprsNrWord, decmprsNrWord (uint64 each),
// then the stream words.
namespace {
struct WahFileHdr {
  uint8_t has1fill, pad[3];
  uint32_t magic;
  uint64_t cmprs, decmprs;
};
static_assert(sizeof(WahFileHdr) == 24, "the reference's header is 24 bytes");
}  // namespace

extern "C" mb_status mb_wah_save(const char *path, const uint32_t *words, uint64_t nwords, uint64_t ngroups) {
  if (!path || (nwords && !words)) return fail(MB_ERR_INVALID, "mb_wah_save: NULL argument");
  WahFileHdr h{};
  h.magic = WAH_MAGIC;
  h.cmprs = nwords;
  h.decmprs = ngroups;
  for (uint64_t i = 0; i < nwords; ++i)
    if ((words[i] >> 30) == 3u) {
      h.has1fill = 1;
      break;
    }
  FILE *f = fopen(path, "wb");
  if (!f) return fail(MB_ERR_IO, "mb_wah_save: cannot open %s", path);
  bool ok = fwrite(&h, sizeof(h), 1, f) == 1 && (nwords == 0 || fwrite(words, 4, nwords, f) == nwords);
  ok = fclose(f) == 0 && ok;
  return ok ? MB_OK : fail(MB_ERR_IO, "mb_wah_save: write to %s failed", path);
}

extern "C" mb_status mb_wah_load(const char *path, uint32_t *words, uint64_t capacity, uint64_t *nwords,
                                 uint64_t *ngroups) {
  if (!path || !nwords) return fail(MB_ERR_INVALID, "mb_wah_load: NULL argument");
  FILE *f = fopen(path, "rb");
  if (!f) return fail(MB_ERR_IO, "mb_wah_load: cannot open %s", path);
  WahFileHdr h{};
  mb_status st = MB_OK;
  long size = -1;
  if (fread(&h, sizeof(h), 1, f) != 1) st = fail(MB_ERR_IO, "mb_wah_load: %s: short header", path);
  else if (h.magic != WAH_MAGIC) st = fail(MB_ERR_IO, "mb_wah_load: %s: bad magic 0x%08x", path, h.magic);
  else if (fseek(f, 0, SEEK_END) != 0 || (size = ftell(f)) < 0 || h.cmprs > ((uint64_t)size) / 4 ||
           (uint64_t)size != sizeof(h) + 4 * h.cmprs)
    st = fail(MB_ERR_IO, "mb_wah_load: %s: %ld bytes for %llu words", path, size, (unsigned long long)h.cmprs);
  if (st == MB_OK) {
    *nwords = h.cmprs;
    if (ngroups) *ngroups = h.decmprs;
    if (words) {
      if (capacity < h.cmprs)
        st = fail(MB_ERR_INVALID, "mb_wah_load: %llu words, the buffer holds %llu", (unsigned long long)h.cmprs,
                  (unsigned long long)capacity);
      else if (fseek(f, sizeof(h), SEEK_SET) != 0 ||
               (h.cmprs && fread(words, 4, h.cmprs, f) != h.cmprs))
        st = fail(MB_ERR_IO, "mb_wah_load: %s: short read", path);
    }
  }
  fclose(f);
  return st;
}
