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
constexpr uint32_t DT = 256;          // output words per decode block (one per thread)
constexpr uint32_t DCAP = 1024;       // stream words a decode block stages
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

// Group g (< ceil(nrows / 31)) as stored in a stream: row 31g + j at bit j
// (order 0) or at bit 30 - j (order 1); rows >= nrows are 0.
__device__ __forceinline__ uint32_t group_of(const EncSrc &S, uint64_t g) {
  const uint64_t r0 = 31 * g, w = r0 >> 5;
  const uint32_t s = (uint32_t)(r0 & 31);
  const uint64_t two = (uint64_t)enc_word(S, w) | ((uint64_t)enc_word(S, w + 1) << 32);
  uint32_t v = (uint32_t)(two >> s) & LIT;
  const uint64_t left = S.nrows - r0;
  if (left < 31) v &= (1u << left) - 1u;
  if (S.order) v = __brev(v) >> 1;
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

// (1) stream words each block of WB groups starts.
__global__ void __launch_bounds__(WT) wah_enc_count(const EncSrc S, uint64_t G, uint64_t *bcnt) {
  const uint64_t g0 = (uint64_t)blockIdx.x * WB + (uint64_t)threadIdx.x * WI;
  uint32_t c = 0;
  if (g0 < G) {
    uint32_t prev = g0 ? kind_of(group_of(S, g0 - 1)) : 3u;
#pragma unroll
    for (uint32_t i = 0; i < WI; ++i) {
      const uint64_t g = g0 + i;
      if (g >= G) break;
      const uint32_t k = kind_of(group_of(S, g));
      c += (k == 2u || k != prev) ? 1u : 0u;
      prev = k;
    }
  }
  uint64_t total;
  block_excl_scan<uint64_t>(c, &total);
  if (threadIdx.x == 0) bcnt[blockIdx.x] = total;
}

// (2) exclusive scan of n block values in place (one CTA); v[n] = total.
__global__ void __launch_bounds__(1024) wah_scan_blocks(uint64_t *v, uint64_t n) {
  __shared__ uint64_t part[32];
  __shared__ uint64_t carry;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint64_t base = 0; base < n; base += 1024) {
    const uint64_t i = base + threadIdx.x;
    const uint64_t x = i < n ? v[i] : 0;
    uint64_t inc = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint64_t y = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= (uint32_t)d) inc += y;
    }
    if (lane == 31) part[warp] = inc;
    __syncthreads();
    uint64_t before = carry, all = 0;
    for (uint32_t k = 0; k < 32; ++k) {
      if (k < warp) before += part[k];
      all += part[k];
    }
    if (i < n) v[i] = before + inc - x;
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
  const uint64_t g0 = (uint64_t)blockIdx.x * WB + (uint64_t)threadIdx.x * WI;
  uint32_t v[WI], head = 0, c = 0;
  if (g0 < G) {
    uint32_t prev = g0 ? kind_of(group_of(S, g0 - 1)) : 3u;
#pragma unroll
    for (uint32_t i = 0; i < WI; ++i) {
      const uint64_t g = g0 + i;
      v[i] = g < G ? group_of(S, g) : 0u;
      const uint32_t k = kind_of(v[i]);
      if (g < G && (k == 2u || k != prev)) head |= 1u << i, ++c;
      prev = k;
    }
  }
  uint64_t total;
  uint64_t at = boff[blockIdx.x] + block_excl_scan<uint64_t>(c, &total);
#pragma unroll
  for (uint32_t i = 0; i < WI; ++i)
    if (head >> i & 1u) {
      const uint32_t k = kind_of(v[i]);
      out[at] = k == 2u ? v[i] : (k == 1u ? FILL | ONES : FILL);
      pos[at] = (uint32_t)(g0 + i);
      ++at;
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

// decode (1): group counts per block of WB stream words.
__global__ void __launch_bounds__(WT) wah_dec_count(const uint32_t *wah, uint64_t n, uint64_t *bsum) {
  const uint64_t k0 = (uint64_t)blockIdx.x * WB + (uint64_t)threadIdx.x * WI;
  uint64_t c = 0;
#pragma unroll
  for (uint32_t i = 0; i < WI; ++i)
    if (k0 + i < n) c += word_groups(__ldg(wah + k0 + i));
  uint64_t total;
  block_excl_scan<uint64_t>(c, &total);
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// decode (2b): the exclusive scan of every word's group count; S[n] = total.
__global__ void __launch_bounds__(WT) wah_dec_scan(const uint32_t *wah, uint64_t n, const uint64_t *boff,
                                                   uint64_t nblk, uint64_t *S) {
  const uint64_t k0 = (uint64_t)blockIdx.x * WB + (uint64_t)threadIdx.x * WI;
  uint32_t c[WI];
  uint64_t sum = 0;
#pragma unroll
  for (uint32_t i = 0; i < WI; ++i) {
    c[i] = k0 + i < n ? (uint32_t)word_groups(__ldg(wah + k0 + i)) : 0u;
    sum += c[i];
  }
  uint64_t total;
  uint64_t at = boff[blockIdx.x] + block_excl_scan<uint64_t>(sum, &total);
#pragma unroll
  for (uint32_t i = 0; i < WI; ++i)
    if (k0 + i < n) S[k0 + i] = at, at += c[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) S[n] = boff[nblk];
}

// Largest k in [lo, hi] with S[k] <= g (S ascending, S[lo] <= g).
__device__ __forceinline__ uint64_t last_le(const uint64_t *S, uint64_t lo, uint64_t hi, uint64_t g) {
  while (lo < hi) {
    const uint64_t mid = lo + (hi - lo + 1) / 2;
    if (S[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// decode (3): for output block b, the stream words covering its groups.
__global__ void wah_dec_partition(const uint64_t *S, uint64_t n, uint64_t nblk, uint64_t *kb, uint64_t *ke) {
  const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblk) return;
  const uint64_t total = S[n];
  const uint64_t w0 = b * DT, w1 = w0 + DT - 1;
  const uint64_t ga = (32 * w0) / 31, gz = (32 * w1) / 31 + 1;
  if (ga >= total) {
    kb[b] = 1, ke[b] = 0;  // past the stream: an empty range
    return;
  }
  const uint64_t s = last_le(S, 0, n - 1, ga);
  kb[b] = s;
  ke[b] = last_le(S, s, n - 1, gz < total ? gz : total - 1);
}

// decode (4): output words, one per thread.
__global__ void __launch_bounds__(DT) wah_dec_emit(const uint32_t *wah, const uint64_t *S, uint64_t n,
                                                   const uint64_t *kb, const uint64_t *ke, uint32_t order,
                                                   uint64_t nrows, uint64_t nw, uint64_t stride, uint32_t *bm) {
  __shared__ uint64_t s_S[DCAP];
  __shared__ uint32_t s_w[DCAP];
  const uint64_t b = blockIdx.x, w = b * DT + threadIdx.x;
  const uint64_t lo = kb[b], hi = ke[b], total = S[n];
  const bool empty = lo > hi, staged = !empty && hi - lo + 1 <= DCAP;
  if (staged)
    for (uint64_t i = threadIdx.x; i <= hi - lo; i += DT) s_S[i] = S[lo + i], s_w[i] = __ldg(wah + lo + i);
  __syncthreads();
  if (w >= stride) return;
  uint32_t out = 0;
  if (!empty && w < nw) {
    const uint64_t ga = (32 * w) / 31;
    const uint32_t sa = (uint32_t)(32 * w - 31 * ga);
    uint32_t v[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const uint64_t g = ga + h;
      uint32_t x = 0;
      if (g < total) {
        uint32_t word;
        if (staged) {
          uint32_t l = 0, r = (uint32_t)(hi - lo);
          while (l < r) {
            const uint32_t m = l + (r - l + 1) / 2;
            if (s_S[m] <= g) l = m;
            else r = m - 1;
          }
          word = s_w[l];
        } else {
          word = __ldg(wah + last_le(S, lo, hi, g));
        }
        x = (word & FILL) ? ((word & ONES) ? LIT : 0u) : (word & LIT);
        if (order) x = __brev(x) >> 1;
      }
      v[h] = x;
    }
    out = (v[0] >> sa) | (v[1] << (31 - sa));
    const uint64_t r0 = 32 * w;
    if (r0 + 32 > nrows) out &= nrows > r0 ? (1u << (nrows - r0)) - 1u : 0u;
  }
  bm[w] = out;
}

// Device scratch freed on scope exit (stream-ordered).
struct Scratch {
  cudaStream_t st;
  std::vector<void *> ptrs;
  explicit Scratch(cudaStream_t s) : st(s) {}
  ~Scratch() {
    for (void *p : ptrs) cudaFreeAsync(p, st);
  }
  template <typename T>
  mb_status get(T **p, uint64_t count) {
    void *q = nullptr;
    const cudaError_t e = cudaMallocAsync(&q, count ? count * sizeof(T) : sizeof(T), st);
    if (e != cudaSuccess) return cuda_fail(e, "wah: scratch allocation");
    ptrs.push_back(q);
    *p = static_cast<T *>(q);
    return MB_OK;
  }
};

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
mb_status group_scan(const uint32_t *wah, uint64_t n, Scratch &sc, uint64_t **S_out, cudaStream_t st) {
  const uint64_t nblk = ceil_div(n, WB);
  uint64_t *boff, *S;
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
  uint64_t *S;
  MB_CHECK(group_scan(wah, n, sc, &S, st));
  const uint64_t nblk = ceil_div(stride, DT);
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
  uint64_t *S;
  MB_CHECK(group_scan(wah, nwords, sc, &S, st));
  MB_CUDA(cudaMemcpyAsync(ngroups, S + nwords, 8, cudaMemcpyDeviceToHost, st));
  MB_CUDA(cudaStreamSynchronize(st));
  return MB_OK;
}

extern "C" mb_status mb_wah_op(uint32_t op, const uint32_t *a, uint64_t na, const uint32_t *b, uint64_t nb,
                               uint64_t ngroups, uint32_t *out, uint64_t capacity, uint64_t *nwords, void *stream) {
  NvtxRange nvtx_("mb_wah_op");
  if (!nwords) return fail(MB_ERR_INVALID, "mb_wah_op: NULL word count");
  *nwords = 0;
  if (op > MB_WAH_XOR) return fail(MB_ERR_INVALID, "mb_wah_op: op %u", op);
  if ((na && !a) || (nb && !b)) return fail(MB_ERR_INVALID, "mb_wah_op: NULL stream");
  if (ngroups > MAX_GROUPS) return fail(MB_ERR_INVALID, "mb_wah_op: %llu groups exceed the 30-bit run count",
                                        (unsigned long long)ngroups);
  if (ngroups == 0) return MB_OK;
  cudaStream_t st = as_stream(stream);
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
  else if (fseek(f, 0, SEEK_END) != 0 || (size = ftell(f)) < 0 ||
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
