// bitmap.cu - one-pass multi-bin bitmap-index creation (mb_bitmap_create).
//
// Reference: create_bin (bmpidx_create.cu:14-56) launching the multi-bin
// bmpcreate kernel (primitive.cuh:102-118): one thread per row, one
// __ballot_sync per (row-word, bin), lane 0 storing each word to HBM.
//
// B200 design:
//  - Persistent CTAs (SMs x occupancy) walk 4096-row tiles.  A 3-stage ring of
//    column tiles is filled by 1-D TMA bulk copies (cp.async.bulk) with mbarrier
//    completion, so HBM reads stream ahead of the compute.  For join bitmaps the
//    staged column is the foreign key and the dimension value is gathered from
//    the (L2-resident) dimension array.
//  - Bins that partition a value range (equal-width, or sorted and disjoint)
//    cost one bin lookup per row plus one __match_any_sync per 32-row word: the
//    peer mask of a bin IS that bin's word.  Arbitrary (overlapping) bins fall
//    back to one ballot per bin, as the reference does.
//  - Words are assembled in a shared-memory tile [bin][128 words] and written
//    out with coalesced 128-bit stores, instead of one 4-byte store per word.
//  - The tail is exact: bits of rows >= n are zero (the reference's
//    single-predicate kernel writes past the bitmap end, primitive.cuh:94-99,
//    and its multi-bin kernel breaks out of a full-mask ballot,
//    primitive.cuh:110-113; neither happens here).
#include <stddef.h>
#include <string.h>
#include <algorithm>
#include <type_traits>
#include "common.cuh"
#include "tma.cuh"

namespace mb {

constexpr int BC_THREADS = 256;
constexpr int BC_TILE_ROWS = 4096;
constexpr int BC_TILE_WORDS = BC_TILE_ROWS / 32;  // 128
constexpr int BC_STAGES = 3;
constexpr int BC_MAXBINS = 256;
constexpr uint32_t BC_NOBIN = 0xffffffffu;

enum { BC_BALLOT = 0, BC_EQUAL = 1, BC_SORTED = 2 };

struct BinSpec {
  uint32_t nbins;
  uint32_t pad_;
  uint64_t lo0, width;  // BC_EQUAL: bin = (v - lo0) / width
  uint64_t lo[BC_MAXBINS], hi[BC_MAXBINS];
};

// Bin of v: BC_EQUAL by arithmetic, BC_SORTED by binary search over the lower
// bounds staged in shared memory (divergent lanes read shared memory at bank
// speed; the same search over the kernel-parameter array serialises per
// distinct address in the constant cache).
template <int MODE>
__device__ __forceinline__ uint32_t find_bin(const BinSpec &S, const uint64_t *slo, const uint64_t *shi,
                                             uint64_t v) {
  if (MODE == BC_EQUAL) {
    if (v < S.lo0) return BC_NOBIN;
    uint64_t d = v - S.lo0;
    uint64_t b = S.width == 1 ? d : d / S.width;
    return b < S.nbins ? (uint32_t)b : BC_NOBIN;
  } else {  // BC_SORTED: last bin with lo <= v, then v < hi
    if (v < slo[0]) return BC_NOBIN;
    uint32_t lo = 0, hi = S.nbins - 1;
    while (lo < hi) {
      uint32_t mid = (lo + hi + 1) >> 1;
      if (slo[mid] <= v) lo = mid; else hi = mid - 1;
    }
    return v < shi[lo] ? lo : BC_NOBIN;
  }
}

template <int W>
__device__ __forceinline__ uint64_t ld_smem_w(const uint8_t *p, uint32_t i) {
  if (W == 1) return p[i];
  if (W == 2) return reinterpret_cast<const uint16_t *>(p)[i];
  if (W == 4) return reinterpret_cast<const uint32_t *>(p)[i];
  return reinterpret_cast<const unsigned long long *>(p)[i];
}

// Word wi of bin b in the shared tile: groups of 4 words are XOR-swizzled by
// the bin so that leaders of different bins storing the same word index hit
// different banks, while each bin's 4-word groups stay contiguous.
__device__ __forceinline__ uint32_t tile_word(uint32_t b, uint32_t wi) {
  return b * BC_TILE_WORDS + ((((wi >> 2) ^ b) & 31u) << 2) + (wi & 3u);
}

// W: bytes of the staged column element (4 for join: the foreign key);
// DW: bytes of the dimension element (join only).
template <int W, bool JOIN, int DW, int MODE>
__global__ void __launch_bounds__(BC_THREADS)
bitmap_create_kernel(const __grid_constant__ BinSpec S, const void *__restrict__ col,
                     const void *__restrict__ dim, uint64_t dimsz, uint64_t n,
                     uint32_t *__restrict__ out, uint64_t stride,
                     unsigned long long *__restrict__ pop, uint32_t *errw) {
  extern __shared__ __align__(128) uint8_t smem[];
  constexpr uint32_t STAGE_BYTES = BC_TILE_ROWS * W;
  uint8_t *stage = smem;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + BC_STAGES * STAGE_BYTES);
  uint32_t *obuf = reinterpret_cast<uint32_t *>(smem + BC_STAGES * STAGE_BYTES + 128);
  unsigned long long *cnt = reinterpret_cast<unsigned long long *>(obuf + S.nbins * BC_TILE_WORDS);
  uint64_t *slo = reinterpret_cast<uint64_t *>(cnt + S.nbins);
  uint64_t *shi = slo + S.nbins;

  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t nwords = (n + 31) / 32;
  const uint64_t ntiles = (n + BC_TILE_ROWS - 1) / BC_TILE_ROWS;
  const uint8_t *colb = reinterpret_cast<const uint8_t *>(col);

  for (uint32_t b = tid; b < S.nbins; b += BC_THREADS) {
    cnt[b] = 0;
    slo[b] = S.lo[b];
    shi[b] = S.hi[b];
  }
  if (MODE != BC_BALLOT)
    for (uint32_t i = tid; i < S.nbins * BC_TILE_WORDS; i += BC_THREADS) obuf[i] = 0;
  if (tid == 0) {
    for (int s = 0; s < BC_STAGES; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  // Bytes of tile t that the bulk copy moves: whole 16-byte chunks only.
  auto tile_bulk_bytes = [&](uint64_t t) -> uint32_t {
    uint64_t rows = n - t * BC_TILE_ROWS;
    if (rows > BC_TILE_ROWS) rows = BC_TILE_ROWS;
    return (uint32_t)((rows * W) & ~(uint64_t)15);
  };
  auto issue = [&](uint64_t t, int s) {
    uint32_t bytes = tile_bulk_bytes(t);
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&bars[s], bytes);
    if (bytes) bulk_g2s(stage + s * STAGE_BYTES, colb + t * (uint64_t)STAGE_BYTES, bytes, &bars[s]);
  };

  if (tid == 0) {
    uint64_t t = blockIdx.x;
    for (int s = 0; s < BC_STAGES && t < ntiles; ++s, t += gridDim.x) issue(t, s);
  }

  uint32_t it = 0;
  for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
    const int s = it % BC_STAGES;
    const uint32_t parity = (it / BC_STAGES) & 1u;
    // Every thread waits (bounded) for the stage; the block leaves together if
    // any wait ran out, after one more bounded wait for the copy in flight.
    const bool arrived = mbar_wait_bounded(&bars[s], parity, errw, MB_DEVERR_TMA_WAIT);
    if (!__syncthreads_and(arrived)) {
      if (tid == 0) mbar_wait_bounded(&bars[s], parity, nullptr, 0, 1u << 16);
      return;
    }
    const uint8_t *sp = stage + s * STAGE_BYTES;
    const uint32_t bulk_rows = tile_bulk_bytes(t) / W;
    const uint64_t row0 = t * BC_TILE_ROWS;

    for (uint32_t wi = warp; wi < BC_TILE_WORDS; wi += BC_THREADS / 32) {
      const uint32_t r = wi * 32 + lane;
      const uint64_t row = row0 + r;
      bool valid = row < n;
      uint64_t v = 0;
      if (valid) {
        uint64_t x = r < bulk_rows ? ld_smem_w<W>(sp, r) : load_width(col, row, W);
        if (JOIN) {
          if (dimsz != 0 && x >= dimsz) valid = false;
          else v = load_width(dim, x, DW);
        } else {
          v = x;
        }
      }
      if (MODE == BC_BALLOT) {
        for (uint32_t b = 0; b < S.nbins; ++b) {
          uint32_t m = __ballot_sync(0xffffffffu, valid && v >= slo[b] && v < shi[b]);
          if (lane == (b & 31)) obuf[tile_word(b, wi)] = m;
        }
      } else {
        uint32_t bin = valid ? find_bin<MODE>(S, slo, shi, v) : BC_NOBIN;
        uint32_t peers = __match_any_sync(0xffffffffu, bin);
        if (bin != BC_NOBIN && lane == (uint32_t)(__ffs(peers) - 1)) obuf[tile_word(bin, wi)] = peers;
      }
    }
    __syncthreads();  // stage s fully read, obuf complete

    if (tid == 0 && t + (uint64_t)BC_STAGES * gridDim.x < ntiles)
      issue(t + (uint64_t)BC_STAGES * gridDim.x, s);

    // Coalesced write-out: per bin 128 consecutive words = 32 x uint4.  A
    // warp covers exactly one bin per iteration (i / 32 is warp-uniform).
    const uint64_t w0 = t * BC_TILE_WORDS;
    for (uint32_t i = tid; i < S.nbins * (BC_TILE_WORDS / 4); i += BC_THREADS) {
      const uint32_t b = i / (BC_TILE_WORDS / 4), q = i % (BC_TILE_WORDS / 4);
      const uint64_t w = w0 + q * 4;
      uint32_t c = 0;
      if (w < nwords) {  // obuf beyond the last word is never written
        uint4 *src = reinterpret_cast<uint4 *>(&obuf[tile_word(b, q * 4)]);
        const uint4 v4 = *src;
        if (MODE != BC_BALLOT) *src = make_uint4(0, 0, 0, 0);  // zeroed for the next tile
        uint32_t *dst = out + b * stride + w;
        if (w + 4 <= nwords) {
          *reinterpret_cast<uint4 *>(dst) = v4;
        } else {
          dst[0] = v4.x;
          if (w + 1 < nwords) dst[1] = v4.y;
          if (w + 2 < nwords) dst[2] = v4.z;
        }
        c = __popc(v4.x) + __popc(v4.y) + __popc(v4.z) + __popc(v4.w);
      }
      if (pop) {
        c = __reduce_add_sync(0xffffffffu, c);
        if (lane == 0 && c) atomicAdd(&cnt[b], (unsigned long long)c);
      }
    }
    __syncthreads();  // obuf reused by the next tile
  }
  if (pop) {
    __syncthreads();
    for (uint32_t b = tid; b < S.nbins; b += BC_THREADS)
      if (cnt[b]) atomicAdd(&pop[b], cnt[b]);
  }
}

// ---------------------------------------------------------------- levels
// One column pass for several levels of bins (years and months of a date,
// regions and nations of a city): each row's bin in every level comes from
// one 4-byte lookup (byte l = the bin of level l) in a shared-memory table
// over the column's value domain, so the column is read once however many
// levels it has.  Each row ORs its bit into its bin's word of the level with
// one shared-memory atomic; rows without a bin OR into the level's spare row
// of words, which is never written out, so the inner loop has no branch.
// The write-out clears the words it reads.  (Measured against one ballot per
// bin and word, against ballots of the bin index's bits, and against the peer
// masks of __match_any_sync: the atomics issue the fewest instructions and
// were the fastest, 1.7x the bit-sliced ballots over a 600M-row index.)
// Words are written out as coalesced 16-byte stores, one warp per bin.
constexpr int BL_THREADS = 512;
constexpr int BL_MAXLEVELS = MB_MAXLEVELS;
constexpr uint32_t BL_LUT_VALUES = 6144;  // value domain of the lookup table (24 KB)
constexpr uint32_t BL_NOBIN = 0xff;       // (lookup table bytes of values outside a level)

struct LevelSpec {
  uint32_t nlevels, nrows_tile;  // levels; rows of words in the tile (bins + one spare row a level)
  uint32_t nb[BL_MAXLEVELS];     // bins of each level (<= 254)
  uint32_t row0[BL_MAXLEVELS];   // first tile row of each level; row0[l] + nb[l] is its spare row
  uint32_t nobin;                // lookup entry of a row in no bin: byte l = nb[l]
  uint32_t dom_n;                // values [dom_lo, dom_lo + dom_n) in the table
  uint64_t dom_lo;
  uint32_t *out[BL_MAXLEVELS];
  unsigned long long *pop[BL_MAXLEVELS];
  uint32_t lut[BL_LUT_VALUES];   // value v: byte l of lut[v - dom_lo] = bin of level l (nb[l]: none)
};

// Word wi of tile row j: XOR-swizzled by the row so that lanes ORing word wi
// of different bins hit different banks, while each row's words stay in one
// 128-word row (read back as 16-byte groups, permuted).
__device__ __forceinline__ uint32_t lv_word(uint32_t j, uint32_t wi) {
  return j * BC_TILE_WORDS + (wi ^ (j & 31u));
}

// Join output of the levels pass: the dimension value of every row (0 where
// the key leaves the dimension) written to dout, and the rows whose key
// leaves it counted in *bad; both optional.
struct LevelsJoinOut {
  void *dout;
  unsigned long long *bad;
};

// The dimension value of key x (JOIN) or x itself; ok false for a key
// outside the dimension.
template <bool JOIN, int DW>
__device__ __forceinline__ uint64_t lv_value(const void *dim, uint64_t dimsz, uint64_t x, bool &ok) {
  if (!JOIN) return x;
  ok = dimsz == 0 || x < dimsz;
  return ok ? load_width(dim, x, DW) : 0;
}

template <int DW>
__device__ __forceinline__ void lv_store(void *dout, uint64_t row, uint64_t v) {
  if (DW == 1) reinterpret_cast<uint8_t *>(dout)[row] = (uint8_t)v;
  else if (DW == 2) reinterpret_cast<uint16_t *>(dout)[row] = (uint16_t)v;
  else if (DW == 4) reinterpret_cast<uint32_t *>(dout)[row] = (uint32_t)v;
  else reinterpret_cast<unsigned long long *>(dout)[row] = v;
}

// (A join pass holds its dimension reads in flight: two CTAs an SM, at most
// 64 registers; three CTAs at 42 registers spilled and measured 27 % slower.)
template <int W, bool JOIN, int DW, int NLC>
__global__ void __launch_bounds__(BL_THREADS, JOIN ? 2 : 1)
bitmap_levels_kernel(const __grid_constant__ LevelSpec S, const void *__restrict__ col,
                     const void *__restrict__ dim, uint64_t dimsz, uint64_t n, uint64_t stride, uint32_t *errw,
                     LevelsJoinOut jo) {
  extern __shared__ __align__(128) uint8_t smem[];
  constexpr uint32_t STAGE_BYTES = BC_TILE_ROWS * W;
  uint8_t *stage = smem;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + BC_STAGES * STAGE_BYTES);
  unsigned long long *cnt = reinterpret_cast<unsigned long long *>(smem + BC_STAGES * STAGE_BYTES + 64);
  uint32_t *tiles = reinterpret_cast<uint32_t *>(cnt + ((S.nrows_tile + 1) & ~1u));  // 16-byte aligned
  uint32_t *lut = tiles + S.nrows_tile * BC_TILE_WORDS;
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = BL_THREADS / 32;
  const uint64_t nwords = (n + 31) / 32;
  const uint64_t ntiles = (n + BC_TILE_ROWS - 1) / BC_TILE_ROWS;
  const uint8_t *colb = reinterpret_cast<const uint8_t *>(col);
  const uint32_t NL = S.nlevels, bit = 1u << lane;
  uint32_t rw[NLC];  // first tile row of each level
#pragma unroll
  for (int l = 0; l < NLC; ++l) rw[l] = S.row0[l];
  uint32_t nbad = 0;  // rows of this thread whose key leaves the dimension (JOIN)

  for (uint32_t i = tid; i < S.dom_n; i += BL_THREADS) lut[i] = S.lut[i];
  for (uint32_t b = tid; b < S.nrows_tile; b += BL_THREADS) cnt[b] = 0;
  for (uint32_t i = tid; i < S.nrows_tile * BC_TILE_WORDS; i += BL_THREADS) tiles[i] = 0;
  if (tid == 0) {
    for (int s = 0; s < BC_STAGES; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  auto tile_bulk_bytes = [&](uint64_t t) -> uint32_t {
    uint64_t rows = n - t * BC_TILE_ROWS;
    if (rows > BC_TILE_ROWS) rows = BC_TILE_ROWS;
    return (uint32_t)((rows * W) & ~(uint64_t)15);
  };
  auto issue = [&](uint64_t t, int s) {
    const uint32_t bytes = tile_bulk_bytes(t);
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&bars[s], bytes);
    if (bytes) bulk_g2s(stage + s * STAGE_BYTES, colb + t * (uint64_t)STAGE_BYTES, bytes, &bars[s]);
  };
  if (tid == 0) {
    uint64_t t = blockIdx.x;
    for (int s = 0; s < BC_STAGES && t < ntiles; ++s, t += gridDim.x) issue(t, s);
  }

  uint32_t it = 0;
  for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
    const int s = it % BC_STAGES;
    const uint32_t parity = (it / BC_STAGES) & 1u;
    const bool arrived = mbar_wait_bounded(&bars[s], parity, errw, MB_DEVERR_TMA_WAIT);
    if (!__syncthreads_and(arrived)) {
      if (tid == 0)  // let this CTA's copies in flight land (this tile and the next stages' tiles)
        for (uint32_t k = 0; k < (uint32_t)BC_STAGES; ++k)
          if (t + (uint64_t)k * gridDim.x < ntiles)
            mbar_wait_bounded(&bars[(it + k) % BC_STAGES], ((it + k) / BC_STAGES) & 1u, nullptr, 0, 1u << 16);
      return;
    }
    const uint8_t *sp = stage + s * STAGE_BYTES;
    const uint32_t bulk_rows = tile_bulk_bytes(t) / W;
    const uint64_t row0 = t * BC_TILE_ROWS;
    const uint32_t rows_here = n - row0 < (uint64_t)BC_TILE_ROWS ? (uint32_t)(n - row0) : (uint32_t)BC_TILE_ROWS;

    if (rows_here == (uint32_t)BC_TILE_ROWS && bulk_rows == (uint32_t)BC_TILE_ROWS) {
      // an interior tile: the warp's PER values (and dimension reads) first,
      // then their bins
      constexpr uint32_t PER = BC_TILE_WORDS / (BL_THREADS / 32);
      using VT = typename std::conditional<((JOIN ? DW : W) <= 4), uint32_t, uint64_t>::type;
      VT v[PER];
      bool ok[PER];
#pragma unroll
      for (uint32_t k = 0; k < PER; ++k) {
        ok[k] = true;
        v[k] = (VT)lv_value<JOIN, DW>(dim, dimsz, ld_smem_w<W>(sp, (warp + k * nwarps) * 32 + lane), ok[k]);
      }
#pragma unroll
      for (uint32_t k = 0; k < PER; ++k) {
        const uint32_t wi = warp + k * nwarps;
        if (JOIN) {
          if (jo.dout) lv_store<DW>(jo.dout, row0 + wi * 32 + lane, v[k]);
          nbad += ok[k] ? 0u : 1u;
        }
        const uint32_t bins =
            (ok[k] && (uint64_t)v[k] - S.dom_lo < (uint64_t)S.dom_n) ? lut[(uint32_t)((uint64_t)v[k] - S.dom_lo)] : S.nobin;
#pragma unroll
        for (int l = 0; l < NLC; ++l) atomicOr(&tiles[lv_word(rw[l] + ((bins >> (8 * l)) & 0xffu), wi)], bit);
      }
    } else {
      for (uint32_t wi = warp; wi < BC_TILE_WORDS; wi += nwarps) {
        const uint32_t r = wi * 32 + lane;
        uint32_t bins = S.nobin;
        if (r < rows_here) {
          const uint64_t x = r < bulk_rows ? ld_smem_w<W>(sp, r) : load_width(col, row0 + r, W);
          bool ok = true;
          const uint64_t v = lv_value<JOIN, DW>(dim, dimsz, x, ok);
          if (JOIN) {
            if (jo.dout) lv_store<DW>(jo.dout, row0 + r, v);
            nbad += ok ? 0u : 1u;
          }
          if (ok && v - S.dom_lo < (uint64_t)S.dom_n) bins = lut[(uint32_t)(v - S.dom_lo)];
        }
#pragma unroll
        for (int l = 0; l < NLC; ++l) atomicOr(&tiles[lv_word(rw[l] + ((bins >> (8 * l)) & 0xffu), wi)], bit);
      }
    }
    __syncthreads();  // stage s fully read, tiles complete

    if (tid == 0 && t + (uint64_t)BC_STAGES * gridDim.x < ntiles) issue(t + (uint64_t)BC_STAGES * gridDim.x, s);

    // write-out: warp g takes tile row g, its 128 words as 32 lanes x uint4
    // (lane L's group holds words 4L + (q ^ (g & 3))); spare rows are only
    // cleared
    const uint64_t w = t * BC_TILE_WORDS + lane * 4;
    for (uint32_t g = warp; g < S.nrows_tile; g += nwarps) {
      uint4 *src = reinterpret_cast<uint4 *>(tiles + g * BC_TILE_WORDS + 4 * (lane ^ ((g & 31u) >> 2)));
      uint4 v4 = *src;
      *src = make_uint4(0, 0, 0, 0);
      uint32_t l = 0;
#pragma unroll
      for (uint32_t k = 1; k < (uint32_t)BL_MAXLEVELS; ++k) l += (k < NL && g >= S.row0[k]) ? 1u : 0u;
      const uint32_t b = g - S.row0[l];
      if (b >= S.nb[l]) continue;  // the spare row (warp-uniform)
      if (g & 1u) v4 = make_uint4(v4.y, v4.x, v4.w, v4.z);
      if (g & 2u) v4 = make_uint4(v4.z, v4.w, v4.x, v4.y);
      uint32_t c = 0;
      if (w < nwords) {
        uint32_t *dst = S.out[l] + b * stride + w;
        if (w + 4 <= nwords) {
          *reinterpret_cast<uint4 *>(dst) = v4;
        } else {
          dst[0] = v4.x;
          if (w + 1 < nwords) dst[1] = v4.y;
          if (w + 2 < nwords) dst[2] = v4.z;
        }
        c = __popc(v4.x) + __popc(v4.y) + __popc(v4.z) + __popc(v4.w);
      }
      c = __reduce_add_sync(0xffffffffu, c);
      if (lane == 0 && c) cnt[g] += c;  // this warp owns row g in this tile
    }
    __syncthreads();  // tiles reused by the next tile
  }
  if (JOIN && jo.bad) {
    nbad = __reduce_add_sync(0xffffffffu, nbad);
    if (lane == 0 && nbad) atomicAdd(jo.bad, (unsigned long long)nbad);
  }
  __syncthreads();
  for (uint32_t g = tid; g < S.nrows_tile; g += BL_THREADS) {
    uint32_t l = 0;
    for (uint32_t k = 1; k < NL; ++k) l += g >= S.row0[k] ? 1u : 0u;
    const uint32_t b = g - S.row0[l];
    if (b < S.nb[l] && S.pop[l] && cnt[g]) atomicAdd(&S.pop[l][b], cnt[g]);
  }
}

// ---------------------------------------------------------------- host
template <int W, bool JOIN, int DW, int MODE>
static mb_status launch_bc(const BinSpec &S, const mb_src *src, uint64_t n, uint32_t *out,
                           uint64_t stride, uint64_t *pop, cudaStream_t st) {
  auto kern = bitmap_create_kernel<W, JOIN, DW, MODE>;
  size_t smem = (size_t)BC_STAGES * BC_TILE_ROWS * W + 128 +
                (size_t)S.nbins * BC_TILE_WORDS * 4 + (size_t)S.nbins * 24;
  MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, BC_THREADS, smem));
  if (occ < 1) return fail(MB_ERR_INVALID, "bitmap_create: %u bins do not fit in shared memory", S.nbins);
  uint64_t ntiles = ceil_div(n, BC_TILE_ROWS);
  uint64_t grid = (uint64_t)dev_info().sms * occ;
  if (grid > ntiles) grid = ntiles;
  uint32_t *errw = device_error_word();
  if (!errw) return fail(MB_ERR_OOM, "bitmap_create: device error word");
  const void *colp = JOIN ? (const void *)src->fk : src->col;
  const void *dimp = JOIN ? src->col : nullptr;
  kern<<<(unsigned)grid, BC_THREADS, smem, st>>>(S, colp, dimp, src->dimsz, n, out, stride,
                                                 reinterpret_cast<unsigned long long *>(pop), errw);
  MB_LAUNCH_CHECK("bitmap_create_kernel");
  return MB_OK;
}

template <int W, bool JOIN, int DW>
static mb_status dispatch_mode(int mode, const BinSpec &S, const mb_src *src, uint64_t n,
                               uint32_t *out, uint64_t stride, uint64_t *pop, cudaStream_t st) {
  switch (mode) {
  case BC_EQUAL: return launch_bc<W, JOIN, DW, BC_EQUAL>(S, src, n, out, stride, pop, st);
  case BC_SORTED: return launch_bc<W, JOIN, DW, BC_SORTED>(S, src, n, out, stride, pop, st);
  default: return launch_bc<W, JOIN, DW, BC_BALLOT>(S, src, n, out, stride, pop, st);
  }
}

template <bool JOIN, int DW>
static mb_status dispatch_w(uint32_t w, int mode, const BinSpec &S, const mb_src *src, uint64_t n,
                            uint32_t *out, uint64_t stride, uint64_t *pop, cudaStream_t st) {
  switch (w) {
  case 1: return dispatch_mode<1, JOIN, DW>(mode, S, src, n, out, stride, pop, st);
  case 2: return dispatch_mode<2, JOIN, DW>(mode, S, src, n, out, stride, pop, st);
  case 4: return dispatch_mode<4, JOIN, DW>(mode, S, src, n, out, stride, pop, st);
  default: return dispatch_mode<8, JOIN, DW>(mode, S, src, n, out, stride, pop, st);
  }
}


// ---------------------------------------------------------------- levels host
// Shared memory of bitmap_levels_kernel<W>: column stages, barriers, row
// counts, the word tiles and the lookup table.
static size_t levels_smem(const LevelSpec &S, int W) {
  return (size_t)BC_STAGES * BC_TILE_ROWS * W + 64 + (size_t)((S.nrows_tile + 1) & ~1u) * 8 +
         (size_t)S.nrows_tile * BC_TILE_WORDS * 4 + (size_t)S.dom_n * 4;
}

template <int W, bool JOIN, int DW>
static mb_status launch_levels(const LevelSpec &S, const mb_src *src, uint64_t n, uint64_t stride, cudaStream_t st,
                               LevelsJoinOut jo) {
  auto kern = S.nlevels == 1   ? bitmap_levels_kernel<W, JOIN, DW, 1>
              : S.nlevels == 2 ? bitmap_levels_kernel<W, JOIN, DW, 2>
              : S.nlevels == 3 ? bitmap_levels_kernel<W, JOIN, DW, 3>
                               : bitmap_levels_kernel<W, JOIN, DW, 4>;
  const size_t smem = levels_smem(S, W);
  MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, BL_THREADS, smem));
  if (occ < 1) return fail(MB_ERR_INVALID, "bitmap_create_levels: %u tile rows do not fit in shared memory", S.nrows_tile);
  uint64_t grid = (uint64_t)dev_info().sms * occ;
  const uint64_t ntiles = ceil_div(n, BC_TILE_ROWS);
  if (grid > ntiles) grid = ntiles;
  uint32_t *errw = device_error_word();
  if (!errw) return fail(MB_ERR_OOM, "bitmap_create_levels: device error word");
  const void *colp = JOIN ? (const void *)src->fk : src->col;
  const void *dimp = JOIN ? src->col : nullptr;
  kern<<<(unsigned)grid, BL_THREADS, smem, st>>>(S, colp, dimp, src->dimsz, n, stride, errw, jo);
  MB_LAUNCH_CHECK("bitmap_levels_kernel");
  return MB_OK;
}

// The levels as one LevelSpec, if the fast path takes them: each level
// sorted and disjoint with at most 254 bins, the value domain within the
// lookup table (the caller checks that the tiles fit in shared memory).
static bool levels_spec(const mb_level *lv, uint32_t nl, LevelSpec &S) {
  if (nl == 0 || nl > (uint32_t)BL_MAXLEVELS) return false;
  memset(&S, 0, offsetof(LevelSpec, lut));
  S.nlevels = nl;
  uint64_t dlo = ~0ull, dhi = 0;
  for (uint32_t l = 0; l < nl; ++l) {
    const mb_level &L = lv[l];
    if (L.nbins == 0 || L.nbins >= BL_NOBIN || !L.lo || !L.hi || !L.out) return false;
    for (uint32_t j = 0; j < L.nbins; ++j) {
      if (L.hi[j] <= L.lo[j]) return false;
      if (j + 1 < L.nbins && L.lo[j + 1] < L.hi[j]) return false;
    }
    dlo = std::min<uint64_t>(dlo, L.lo[0]);
    dhi = std::max<uint64_t>(dhi, L.hi[L.nbins - 1]);
    S.nb[l] = L.nbins;
    S.row0[l] = S.nrows_tile;
    S.nrows_tile += L.nbins + 1;
    S.nobin |= L.nbins << (8 * l);
    S.out[l] = L.out;
    S.pop[l] = reinterpret_cast<unsigned long long *>(L.popcounts);
  }
  if (dhi - dlo > BL_LUT_VALUES) return false;
  S.dom_lo = dlo;
  S.dom_n = (uint32_t)(dhi - dlo);
  for (uint32_t i = 0; i < S.dom_n; ++i) S.lut[i] = S.nobin;
  for (uint32_t l = 0; l < nl; ++l) {
    const mb_level &L = lv[l];
    for (uint32_t j = 0; j < L.nbins; ++j)
      for (uint64_t v = L.lo[j]; v < L.hi[j]; ++v) {
        uint32_t &e = S.lut[v - dlo];
        e = (e & ~(0xffu << (8 * l))) | (j << (8 * l));
      }
  }
  return true;
}

static int classify_bins(const uint64_t *lo, const uint64_t *hi, uint32_t nb, uint64_t *lo0,
                         uint64_t *width) {
  if (nb <= 4) return BC_BALLOT;
  bool equal = true, sorted = true;
  uint64_t w = hi[0] - lo[0];
  for (uint32_t j = 0; j < nb; ++j) {
    if (hi[j] <= lo[j]) return BC_BALLOT;  // empty bins: keep the generic path
    if (hi[j] - lo[j] != w) equal = false;
    if (j + 1 < nb) {
      if (lo[j + 1] != hi[j]) equal = false;
      if (lo[j + 1] < hi[j]) sorted = false;
    }
  }
  if (equal) {
    *lo0 = lo[0];
    *width = w;
    return BC_EQUAL;
  }
  return sorted ? BC_SORTED : BC_BALLOT;
}

}  // namespace mb

using namespace mb;

extern "C" mb_status mb_bitmap_create(const mb_src *src, uint64_t nrows, const uint64_t *lo,
                                      const uint64_t *hi, uint32_t nbins, uint32_t *out,
                                      uint64_t stride_words, uint64_t *popcounts, void *stream) {
  if (!src || !lo || !hi || !out) return fail(MB_ERR_INVALID, "mb_bitmap_create: NULL argument");
  if (nbins == 0) return MB_OK;
  uint32_t w = src->width;
  if (w != 1 && w != 2 && w != 4 && w != 8)
    return fail(MB_ERR_INVALID, "mb_bitmap_create: width %u not in {1,2,4,8}", w);
  if (!src->col) return fail(MB_ERR_INVALID, "mb_bitmap_create: column is NULL");
  if (stride_words < mb_bitmap_words(nrows) || (stride_words & 3) != 0)
    return fail(MB_ERR_INVALID, "mb_bitmap_create: stride %llu < words or not a multiple of 4",
                (unsigned long long)stride_words);
  if (((uintptr_t)out & 15) != 0)
    return fail(MB_ERR_INVALID, "mb_bitmap_create: output not 16-byte aligned");
  const void *staged = src->fk ? (const void *)src->fk : src->col;
  if (((uintptr_t)staged & 15) != 0)
    return fail(MB_ERR_INVALID, "mb_bitmap_create: staged column not 16-byte aligned");
  if (nrows == 0) return MB_OK;
  cudaStream_t st = as_stream(stream);
  // More bins than one shared-memory tile holds: split into passes.
  // 8-byte staged columns leave room for 224 bins next to the 3 stages
  const uint32_t maxb = (w == 8 && src->fk == nullptr) ? 224u : (uint32_t)BC_MAXBINS;
  for (uint32_t b0 = 0; b0 < nbins; b0 += maxb) {
    uint32_t nb = nbins - b0 < maxb ? nbins - b0 : maxb;
    BinSpec S;
    memset(&S, 0, sizeof(S));
    S.nbins = nb;
    for (uint32_t j = 0; j < nb; ++j) {
      S.lo[j] = lo[b0 + j];
      S.hi[j] = hi[b0 + j];
    }
    int mode = classify_bins(S.lo, S.hi, nb, &S.lo0, &S.width);
    uint32_t *o = out + (uint64_t)b0 * stride_words;
    uint64_t *p = popcounts ? popcounts + b0 : nullptr;
    mb_status r;
    if (src->fk == nullptr) {
      r = dispatch_w<false, 1>(w, mode, S, src, nrows, o, stride_words, p, st);
    } else {
      switch (w) {  // staged column is the 4-byte key; w is the dimension width
      case 1: r = dispatch_mode<4, true, 1>(mode, S, src, nrows, o, stride_words, p, st); break;
      case 2: r = dispatch_mode<4, true, 2>(mode, S, src, nrows, o, stride_words, p, st); break;
      case 4: r = dispatch_mode<4, true, 4>(mode, S, src, nrows, o, stride_words, p, st); break;
      default: r = dispatch_mode<4, true, 8>(mode, S, src, nrows, o, stride_words, p, st); break;
      }
    }
    if (r != MB_OK) return r;
  }
  return MB_OK;
}

mb_status mb::bitmap_create_levels_join(const mb_src *src, uint64_t nrows, const mb_level *levels,
                                        uint32_t nlevels, uint64_t stride_words, void *stream, void *dout,
                                        unsigned long long *bad) {
  if (!src || (!levels && nlevels)) return fail(MB_ERR_INVALID, "mb_bitmap_create_levels: NULL argument");
  if (nlevels == 0) return MB_OK;
  const uint32_t w = src->width;
  if (w != 1 && w != 2 && w != 4 && w != 8)
    return fail(MB_ERR_INVALID, "mb_bitmap_create_levels: width %u not in {1,2,4,8}", w);
  if (!src->col) return fail(MB_ERR_INVALID, "mb_bitmap_create_levels: column is NULL");
  if (stride_words < mb_bitmap_words(nrows) || (stride_words & 3) != 0)
    return fail(MB_ERR_INVALID, "mb_bitmap_create_levels: stride %llu < words or not a multiple of 4",
                (unsigned long long)stride_words);
  for (uint32_t l = 0; l < nlevels; ++l)
    if (levels[l].nbins && (!levels[l].out || ((uintptr_t)levels[l].out & 15) != 0))
      return fail(MB_ERR_INVALID, "mb_bitmap_create_levels: level %u output NULL or not 16-byte aligned", l);
  const void *staged = src->fk ? (const void *)src->fk : src->col;
  if (((uintptr_t)staged & 15) != 0)
    return fail(MB_ERR_INVALID, "mb_bitmap_create_levels: staged column not 16-byte aligned");
  const bool join_out = dout || bad;
  if (join_out && !src->fk) return fail(MB_ERR_INVALID, "bitmap levels: join outputs without a foreign key");
  if (nrows == 0) return MB_OK;
  cudaStream_t st = as_stream(stream);
  static thread_local LevelSpec S;  // 24 KB lookup table: not on the stack
  const int staged_w = src->fk ? 4 : (int)w;
  const bool fast = levels_spec(levels, nlevels, S) && (w <= 4 || src->fk) &&
                    levels_smem(S, staged_w) <= (size_t)dev_info().max_smem_optin;
  if (!fast) {  // one pass per level
    if (join_out) return fail(MB_ERR_INVALID, "bitmap levels: join outputs need the one-pass form");
    for (uint32_t l = 0; l < nlevels; ++l)
      MB_CHECK(mb_bitmap_create(src, nrows, levels[l].lo, levels[l].hi, levels[l].nbins, levels[l].out, stride_words,
                                levels[l].popcounts, stream));
    return MB_OK;
  }
  const LevelsJoinOut jo = {dout, bad};
  if (src->fk == nullptr) {
    switch (w) {
    case 1: return launch_levels<1, false, 1>(S, src, nrows, stride_words, st, jo);
    case 2: return launch_levels<2, false, 1>(S, src, nrows, stride_words, st, jo);
    default: return launch_levels<4, false, 1>(S, src, nrows, stride_words, st, jo);
    }
  }
  switch (w) {  // staged column is the 4-byte key; w is the dimension width
  case 1: return launch_levels<4, true, 1>(S, src, nrows, stride_words, st, jo);
  case 2: return launch_levels<4, true, 2>(S, src, nrows, stride_words, st, jo);
  case 4: return launch_levels<4, true, 4>(S, src, nrows, stride_words, st, jo);
  default: return launch_levels<4, true, 8>(S, src, nrows, stride_words, st, jo);
  }
}

extern "C" mb_status mb_bitmap_create_levels(const mb_src *src, uint64_t nrows, const mb_level *levels,
                                             uint32_t nlevels, uint64_t stride_words, void *stream) {
  return mb::bitmap_create_levels_join(src, nrows, levels, nlevels, stride_words, stream, nullptr, nullptr);
}
