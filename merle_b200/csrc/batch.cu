// batch.cu - the batched scan kernel (see batch.cuh for the design).
//
// Reference: the per-query fused kernel vprg_grpby (primitive.cuh:340-445)
// and its op functors (ssb/lambdas.cuh:19-152) define what each query of a
// batch computes; the batch evaluates the same programs with the same
// candidate-check semantics, so every query's groups and row count equal what
// it gets alone.
//
// A CTA walks its row tiles (T = 32 * V words), S tiles in flight in shared
// memory.  One producer warp fills the stages: the index is one slab of
// bitmap rows, so a tile of the rows the batch reads is staged by one 2-D
// tensor copy per run of rows (TMA, box = run x T words), the payload
// columns the batch reads densely either by bulk copies into the same stage
// or by L2 prefetches, all completing on the stage's "full" mbarrier.  The
// other warps work: on a staged tile each takes queries off the stage's
// counter, costliest first, and leaves the tile (an arrival on its "empty"
// mbarrier, which lets the producer refill it) when none is left, so warps
// move between tiles independently.
//
// For its query a warp evaluates the conjunctive chain on the staged words
// (each lane V consecutive words) and then runs the query's op on the
// selected rows of the tile itself, one row per lane per round: up to 256
// rows compacted in row order through the warp's buffer, denser queries by
// the lowest selected bit of each lane's words.  The op's constants sit in
// registers for the whole tile; the four query templates have compiled
// drains, any other op the generic one.  Nothing is queued across tiles: a
// tile's payload rows are read while they are staged or in L2.
//
// Group sums: a query whose estimated rows outweigh its group count by far
// sums into a group table in shared memory (per CTA, flushed to the output
// at the end); other multi-group queries add to the output with one global
// atomic per row; 1-group sums and row counts accumulate per CTA with shared
// atomics (two warps can hold one query on two tiles at once).
//
// Every wait is bounded: a stage whose copies do not arrive, or that its
// workers do not release, within the launch's try limit makes the CTA
// record (code, block) in the device error word, let its copies in flight
// land, and exit.
#include <cudaTypedefs.h>
#include <string.h>
#include <mutex>
#include <vector>
#include "batch.cuh"
#include "opeval.cuh"
#include "tma.cuh"
#include "vbp.cuh"

namespace mb {

namespace {

constexpr uint32_t BT_THREADS_MAX = BW_MAX * 32;
constexpr uint32_t BT_NOTABLE = 0xffffffffu;

constexpr uint32_t BT_BUF = 256;  // rows of a warp's chunk buffer (or 1024 where shared memory allows)


// Shared-memory layout of one launch (identical on host and device).
struct BLayout {
  uint32_t off_Q, off_src, off_sum, off_cnt, off_toff, off_bar, off_ctr, off_order, off_chain, off_conj, off_stab,
      off_buf, off_stage, stage_words, total, buf;
};

__host__ __device__ inline uint32_t align_up(uint32_t x, uint32_t a) { return (x + a - 1) / a * a; }

__host__ __device__ inline BLayout blayout(uint32_t nq, uint32_t nchain, uint32_t nconj, uint32_t nu, uint32_t S,
                                           uint32_t T, uint32_t nstab, uint32_t nw, uint32_t buf) {
  BLayout L;
  L.buf = buf ? buf : BT_BUF;
  uint32_t o = 0;
  L.off_Q = o;
  o += nq * BQD_WORDS * 4;
  L.off_src = o = align_up(o, 16);
  o += BS_MAX * 24;  // col[] and fk[] (8 bytes), dimsz[] and width[] (4 bytes)
  L.off_sum = o = align_up(o, 16);
  o += nq * 8;  // per query: 1-group sum
  L.off_cnt = o;
  o += nq * 8;  // per query: kept rows
  L.off_toff = o;
  o += nq * 4;  // per query: first slot of its shared group table, or BT_NOTABLE
  L.off_bar = o = align_up(o, 8);
  o += 16 * S;  // full[S], empty[S]
  L.off_ctr = o;
  o += 4 * S + 4;  // per stage: the query counter; the abort flag
  L.off_order = o;
  o += nq;
  L.off_chain = o = align_up(o, 16);
  o += align_up(nchain * 2, 16);
  L.off_conj = o;
  o += nconj * 4;
  L.off_stab = o = align_up(o, 16);  // 64-bit atomics: 8-byte aligned at least
  o += nstab * 8;
  L.off_buf = o = align_up(o, 16);
  o += nw * L.buf * 4;
  L.off_stage = o = align_up(o, 128);
  L.stage_words = nu * T;
  o += S * L.stage_words * 4;
  L.total = o;
  return L;
}

struct BParams {
  uint64_t nrows, nwords;
  uint32_t nq, nu, nsrc, nchain, nconj, pf_mask, S, nstab;
  uint32_t ncopy;
  uint32_t wait_tries;   // mbarrier try_wait limit of a stage wait
  uint32_t skip_stage0;  // 1: stage 0 is armed but never filled (its wait runs out: tests only)
  uint32_t copy[BCP_MAX];  // BatchHdr::copy
  BLayout L;
};

// The batch's tables as a warp sees them (shared memory).
struct BCtx {
  const uint32_t *Qd;
  const unsigned long long *scol, *sfk;
  const uint32_t *sdim;
  const uint32_t *toff;
  unsigned long long *out;
  unsigned long long *qsum;  // per query: 1-group sum (this CTA)
  unsigned long long *qcnt;  // per query: kept rows (this CTA)
  unsigned long long *stab;  // shared group tables
};

// A predicated 32-bit read-only load: 0 where pred is false.  Written out so
// that a drain's loads form one straight run the warp issues back to back.
__device__ __forceinline__ uint32_t ldg_pred(const void *p, bool pred) {
  uint32_t v;
  asm volatile(
      "{\n .reg .pred q;\n setp.ne.b32 q, %2, 0;\n mov.b32 %0, 0;\n @q ld.global.nc.b32 %0, [%1];\n}\n"
      : "=r"(v)
      : "l"(p), "r"(pred ? 1u : 0u));
  return v;
}

// Adds one round's results of query q (warp-uniform), R rows per lane: row
// counts and 1-group sums into the CTA's slots, group sums into the query's
// shared table or, without one, the output.  All 32 lanes call it.
template <int R>
__device__ __forceinline__ void b_accumulate(const BCtx &C, uint32_t q, const uint32_t *d, const bool (&keep)[R],
                                             const uint32_t (&g)[R], const uint64_t (&x)[R]) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t kept = 0;
#pragma unroll
  for (int j = 0; j < R; ++j) kept += __popc(__ballot_sync(0xffffffffu, keep[j]));
  if ((d[0] >> 8) & 1u) {  // one group: a warp sum
    uint64_t v = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) v += keep[j] ? x[j] : 0;
    const uint64_t s = peer_sum64(0xffffffffu, v);
    if (lane == 0 && s) atomicAdd(&C.qsum[q], (unsigned long long)s);
  } else {
    const uint32_t t = C.toff[q];
#pragma unroll
    for (int j = 0; j < R; ++j)
      if (keep[j]) {
        if (t != BT_NOTABLE) atomicAdd(&C.stab[t + g[j]], (unsigned long long)x[j]);
        else atomicAdd(&C.out[d[2] + g[j]], (unsigned long long)x[j]);
      }
  }
  if (lane == 0 && kept) atomicAdd(&C.qcnt[q], (unsigned long long)kept);
}

// Query q's op on R rows per lane (act: the lane has the row; unc: the row
// is uncertain and must pass the candidate check): the per-slot descriptor
// of batch.cuh, read as data, so every query of the batch runs the same code
// (one small body for all warps keeps the instruction cache warm).  The
// slots a round needs are known to the whole warp: every row's value slots,
// the filter slots only when some row of the round is uncertain.  All
// addresses are formed and all loads of the R rows issued before any value
// is used, so a round waits for one memory round trip (two for a source read
// through a foreign key) with R x slots loads in flight per lane.  Staged
// payload columns are read from the tile's copy in shared memory.
template <int R>
__device__ __noinline__ void b_round(const BCtx &C, uint32_t q, const bool (&act)[R], const uint32_t (&r)[R],
                                     const bool (&unc)[R]) {
  const uint32_t *d = C.Qd + q * BQD_WORDS;
  const uint32_t h0 = d[0], roles = d[5], fkm = d[7];
  const uint32_t nslot = h0 & 0xffu, kv = roles & 0xffu, filt = (roles >> 8) & 0xffu, keym = (roles >> 16) & 0xffu,
                 termm = roles >> 24;
  bool c[R], anyl = false;
#pragma unroll
  for (int j = 0; j < R; ++j) c[j] = act[j] && unc[j], anyl = anyl || c[j];
  const bool anyc = __any_sync(0xffffffffu, anyl);
  const uint32_t need = (kv | (anyc ? filt : 0u)) & ((1u << nslot) - 1u);
  // foreign keys first (the column read needs the key)
  uint32_t key[R][BSLOT], bad[R];
#pragma unroll
  for (int j = 0; j < R; ++j) {
    bad[j] = 0;
#pragma unroll
    for (uint32_t s = 0; s < BSLOT; ++s) {
      key[j][s] = r[j];
      if (((need & fkm) >> s) & 1u) {
        const uint32_t t = d[BQD_SLOT0 + BQD_SLOTW * s] & 0xffu;
        const bool l = act[j] && (((kv >> s) & 1u) || c[j]);
        key[j][s] = ldg_pred(reinterpret_cast<const uint32_t *>(C.sfk[t]) + r[j], l);
      }
    }
  }
  if (need & fkm) {
#pragma unroll
    for (int j = 0; j < R; ++j)
#pragma unroll
      for (uint32_t s = 0; s < BSLOT; ++s)
        if (((need & fkm) >> s) & 1u) {
          const uint32_t dz = C.sdim[d[BQD_SLOT0 + BQD_SLOTW * s] & 0xffu];
          if (dz && key[j][s] >= dz) bad[j] |= 1u << s;
        }
  }
  uint32_t sh[R][BSLOT], raw[R][BSLOT];
#pragma unroll
  for (uint32_t s = 0; s < BSLOT; ++s) {
#pragma unroll
    for (int j = 0; j < R; ++j) sh[j][s] = 0, raw[j][s] = 0;
    if ((need >> s) & 1u) {
      const uint32_t e = d[BQD_SLOT0 + BQD_SLOTW * s], t = e & 0xffu, w = (e >> 8) & 0xffu;
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const bool l = act[j] && (((kv >> s) & 1u) || c[j]) && !((bad[j] >> s) & 1u);
        const uintptr_t a = (uintptr_t)C.scol[t] + (uintptr_t)key[j][s] * w;
        raw[j][s] = ldg_pred(reinterpret_cast<const void *>(a & ~(uintptr_t)3), l);
        sh[j][s] = (uint32_t)(a & 3) * 8;
      }
    }
  }
  bool keep[R];
  uint32_t g[R];
  uint64_t x[R];
  const uint32_t vkind = (h0 >> 16) & 15u, va = (h0 >> 20) & 15u, vb = (h0 >> 24) & 15u;
#pragma unroll
  for (int j = 0; j < R; ++j) {
    uint32_t v[BSLOT];
#pragma unroll
    for (uint32_t s = 0; s < BSLOT; ++s) {
      const uint32_t w = (d[BQD_SLOT0 + BQD_SLOTW * s] >> 8) & 0xffu;
      const uint32_t mask = w >= 4 ? 0xffffffffu : ((1u << (8 * w)) - 1u);
      v[s] = (raw[j][s] >> sh[j][s]) & mask;
    }
    bool k = act[j];
    if (termm && anyc) {  // candidate check of uncertain rows: single-term clauses, bounds intersected per slot
#pragma unroll
      for (uint32_t s = 0; s < BSLOT; ++s)
        if ((termm >> s) & 1u) {
          const uint32_t lo = d[BQD_SLOT0 + BQD_SLOTW * s + 1], hi = d[BQD_SLOT0 + BQD_SLOTW * s + 2];
          k = k && (!c[j] || (!((bad[j] >> s) & 1u) && v[s] >= lo && v[s] <= hi));
        }
    }
    uint32_t gg = 0;
#pragma unroll
    for (uint32_t s = 0; s < BSLOT; ++s)
      if ((keym >> s) & 1u) {
        const uint32_t *sl = d + BQD_SLOT0 + BQD_SLOTW * s;
        const uint32_t e = sl[0], xf = (e >> 16) & 0xffu;
        k = k && !((bad[j] >> s) & 1u);
        uint32_t xv = v[s];
        if (xf == MB_X_DIV) xv = div_by_magic(xv, sl[3], (e >> 24) & 15u, e >> 28);
        else if (xf == MB_X_YEAR) xv = date_to_year(xv);
        gg += sl[5] * (xv - sl[4]);
      }
    k = k && gg < d[1];
    uint64_t xx = 1;
    if (vkind != MB_V_ONE) {
      uint64_t xa = 0, xb = 0;
#pragma unroll
      for (uint32_t s = 0; s < BSLOT; ++s) {
        if (s == va) xa = v[s];
        if (s == vb) xb = v[s];
      }
      k = k && !((bad[j] >> va) & 1u);
      if (vkind == MB_V_COL) {
        xx = xa;
      } else {
        k = k && !((bad[j] >> vb) & 1u);
        xx = vkind == MB_V_MUL ? xa * xb : (uint64_t)((int64_t)xa - (int64_t)xb);
      }
    }
    keep[j] = k, g[j] = gg, x[j] = xx;
  }
  b_accumulate<R>(C, q, d, keep, g, x);
}

// The op of a compiled shape SH with the query's constants in registers:
// set up once per (query, tile), then each round is straight-line code over
// the shape's slots (every row's value slots, the filter slots of uncertain
// rows), R rows per lane with all their loads issued before any use.
template <int SH>
struct BDrain {
  static constexpr BShape sh = BSHAPES[SH];
  const uint8_t *col[BSLOT];   // by slot: the column
  uint32_t w[BSLOT];           // element bytes
  uint32_t msk[BSLOT];         // value mask of an element read as the aligned 32-bit word holding it
  uint32_t lo[BSLOT], hi[BSLOT];  // candidate-check bounds (inclusive)
  uint32_t km[BSLOT], ks[BSLOT], kb[BSLOT], kmul[BSLOT];  // key divisor magic and shifts, base, multiplier
  uint32_t ng, obase, toff, single;

  __device__ __forceinline__ BDrain(const BCtx &C, uint32_t q, const uint32_t *d) {
#pragma unroll
    for (uint32_t s = 0; s < BSLOT; ++s) {
      if (s < sh.ns && (((sh.kv | sh.filt) >> s) & 1u)) {
        const uint32_t e = d[BQD_SLOT0 + BQD_SLOTW * s];
        w[s] = (e >> 8) & 0xffu;
        msk[s] = w[s] >= 4 ? 0xffffffffu : ((1u << (8 * w[s])) - 1u);
        col[s] = reinterpret_cast<const uint8_t *>(C.scol[e & 0xffu]);
        if ((sh.filt >> s) & 1u) lo[s] = d[BQD_SLOT0 + BQD_SLOTW * s + 1], hi[s] = d[BQD_SLOT0 + BQD_SLOTW * s + 2];
        if ((sh.keym >> s) & 1u) {
          ks[s] = e >> 24;
          km[s] = d[BQD_SLOT0 + BQD_SLOTW * s + 3];
          kb[s] = d[BQD_SLOT0 + BQD_SLOTW * s + 4];
          kmul[s] = d[BQD_SLOT0 + BQD_SLOTW * s + 5];
        }
      }
    }
    ng = d[1], obase = d[2], single = (d[0] >> 8) & 1u, toff = C.toff[q];
  }

  template <int R>
  __device__ __forceinline__ void round(const BCtx &C, uint32_t q, const bool (&act)[R], const uint32_t (&r)[R],
                                        const bool (&unc)[R]) const {
    bool c[R], anyl = false;
#pragma unroll
    for (int j = 0; j < R; ++j) c[j] = act[j] && unc[j], anyl = anyl || c[j];
    const bool anyc = sh.filt ? __any_sync(0xffffffffu, anyl) : false;
    uint32_t raw[R][BSLOT], shf[R][BSLOT];
#pragma unroll
    for (uint32_t s = 0; s < BSLOT; ++s) {
#pragma unroll
      for (int j = 0; j < R; ++j) raw[j][s] = 0, shf[j][s] = 0;
      if (s < sh.ns && (((sh.kv | sh.filt) >> s) & 1u)) {
        const bool kvs = (sh.kv >> s) & 1u;
        if (kvs || anyc) {
#pragma unroll
          for (int j = 0; j < R; ++j) {
            const bool l = act[j] && (kvs || c[j]);
            const uintptr_t a = (uintptr_t)col[s] + (uintptr_t)r[j] * w[s];
            raw[j][s] = ldg_pred(reinterpret_cast<const void *>(a & ~(uintptr_t)3), l);
            shf[j][s] = (uint32_t)(a & 3) * 8;
          }
        }
      }
    }
    bool keep[R];
    uint32_t g[R];
    uint64_t x[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      uint32_t v[BSLOT];
#pragma unroll
      for (uint32_t s = 0; s < BSLOT; ++s) {
        v[s] = 0;
        if (s < sh.ns && (((sh.kv | sh.filt) >> s) & 1u)) v[s] = (raw[j][s] >> shf[j][s]) & msk[s];
      }
      bool k = act[j];
      if (sh.filt && anyc) {
#pragma unroll
        for (uint32_t s = 0; s < BSLOT; ++s)
          if ((sh.filt >> s) & 1u) k = k && (!c[j] || (v[s] >= lo[s] && v[s] <= hi[s]));
      }
      uint32_t gg = 0;
#pragma unroll
      for (uint32_t s = 0; s < BSLOT; ++s)
        if ((sh.keym >> s) & 1u) {
          const uint32_t xv = ((sh.yearm >> s) & 1u) ? date_to_year(v[s]) : div_by_magic(v[s], km[s], ks[s] & 15u, ks[s] >> 4);
          gg += kmul[s] * (xv - kb[s]);
        }
      k = k && gg < ng;
      uint64_t xx = 1;
      if (sh.vk == MB_V_COL) xx = v[sh.va];
      else if (sh.vk == MB_V_MUL) xx = (uint64_t)v[sh.va] * (uint64_t)v[sh.vb];
      else if (sh.vk == MB_V_SUB) xx = (uint64_t)((int64_t)v[sh.va] - (int64_t)v[sh.vb]);
      keep[j] = k, g[j] = gg, x[j] = xx;
    }
    const uint32_t lane = threadIdx.x & 31;
    uint32_t kept = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) kept += __popc(__ballot_sync(0xffffffffu, keep[j]));
    if (single) {
      uint64_t sv = 0;
#pragma unroll
      for (int j = 0; j < R; ++j) sv += keep[j] ? x[j] : 0;
      const uint64_t tot = peer_sum64(0xffffffffu, sv);
      if (lane == 0 && tot) atomicAdd(&C.qsum[q], (unsigned long long)tot);
    } else {
#pragma unroll
      for (int j = 0; j < R; ++j)
        if (keep[j]) {
          if (toff != BT_NOTABLE) atomicAdd(&C.stab[toff + g[j]], (unsigned long long)x[j]);
          else atomicAdd(&C.out[obase + g[j]], (unsigned long long)x[j]);
        }
    }
    if (lane == 0 && kept) atomicAdd(&C.qcnt[q], (unsigned long long)kept);
  }
};

// The generic drain as a round functor.
struct BDrainAny {
  __device__ __forceinline__ BDrainAny(const BCtx &, uint32_t, const uint32_t *) {}
  template <int R>
  __device__ __forceinline__ void round(const BCtx &C, uint32_t q, const bool (&act)[R], const uint32_t (&r)[R],
                                        const bool (&unc)[R]) const {
    b_round<R>(C, q, act, r, unc);
  }
};

// The op of query q over its selected rows in this tile (bits p[k], uncertain
// u[k] of the lane's words: rows rowbase + 32 k + b), R rows per lane per
// round (the kernel takes R = 1: two rows a lane measured 9 % slower).  The
// rows go through the warp's buffer in chunks: each lane adds up to CH of
// its remaining rows, word by word (a prefix sum of the lanes' counts places
// them), then full rounds of 32 rows drain the chunk, so every round but a
// chunk's last is full however unevenly the rows fall on the lanes, and a
// round's rows lie close together (one lane's span).  On the
// selectivity-spanning mix: 6 % faster than draining dense words by each
// lane's lowest set bit; filling word by word 5 % faster than through a
// select chain over the lane's words; CH = 32 (1,024-row buffers) 2 % faster
// than CH = 8.
template <class DR, int V, int R, int CH>
__device__ __forceinline__ void b_rows(const BCtx &C, uint32_t q, uint32_t (&p)[V], const uint32_t (&u)[V],
                                       uint32_t rowbase, uint32_t *buf) {
  // CH: rows a lane adds to the buffer per chunk (the buffer holds 32 * CH)
  const uint32_t lane = threadIdx.x & 31;
  uint32_t cnt = 0;
#pragma unroll
  for (int k = 0; k < V; ++k) cnt += __popc(p[k]);
  if (__reduce_add_sync(0xffffffffu, cnt) == 0) return;
  const DR dr(C, q, C.Qd + q * BQD_WORDS);
  while (true) {
    // each lane's next min(cnt, CH) rows, placed by a prefix sum of the counts
    const uint32_t take = cnt < CH ? cnt : CH;
    uint32_t incl = take;
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, dd);
      if (lane >= (uint32_t)dd) incl += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0) break;
    uint32_t pos = incl - take;
    cnt -= take;
    uint32_t left = take;
#pragma unroll
    for (int kk = 0; kk < V; ++kk) {
      uint32_t mm = p[kk];
      while (mm && left) {
        const uint32_t b = __ffs(mm) - 1;
        mm &= mm - 1;
        --left;
        buf[pos++] = (rowbase + kk * 32 + b) | (((u[kk] >> b) & 1u) << 31);
      }
      p[kk] = mm;
    }
    __syncwarp();
    for (uint32_t i0 = 0; i0 < total; i0 += 32 * R) {
      bool act[R], unc[R];
      uint32_t row[R];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const uint32_t i = i0 + 32 * j + lane;
        act[j] = i < total;
        const uint32_t e = act[j] ? buf[i] : 0u;
        row[j] = e & 0x7fffffffu, unc[j] = e >> 31;
      }
      dr.template round<R>(C, q, act, row, unc);
    }
    __syncwarp();
  }
}

template <int V>
__device__ __forceinline__ void lds_words(const uint32_t *p, uint32_t (&x)[V]) {
  if (V == 6) {  // 24 bytes a lane: three 8-byte loads
    const uint2 a = reinterpret_cast<const uint2 *>(p)[0], b = reinterpret_cast<const uint2 *>(p)[1],
                c = reinterpret_cast<const uint2 *>(p)[2];
    x[0] = a.x, x[1] = a.y, x[2 % V] = b.x, x[3 % V] = b.y, x[4 % V] = c.x, x[5 % V] = c.y;
  } else if (V == 4) {
    const uint4 t = *reinterpret_cast<const uint4 *>(p);
    x[0] = t.x, x[1] = t.y, x[2] = t.z, x[3] = t.w;
  } else if (V == 2) {
    const uint2 t = *reinterpret_cast<const uint2 *>(p);
    x[0] = t.x, x[1] = t.y;
  } else {
    x[0] = p[0];
  }
}

// Query q on the staged tile (words w0 + lane*V + k of the table; word
// lane*V + k of the stage): the conjunctive chain, then the op on its
// selected rows.
template <int V, int CH>
__device__ __forceinline__ void b_query(const BCtx &C, const uint16_t *chain, const uint32_t *conj,
                                        const uint32_t *stage, uint64_t w0,
                                        uint64_t nwords, uint32_t tail, uint32_t q, uint32_t *buf) {
  constexpr uint32_t T = 32 * V;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t ch = C.Qd[q * BQD_WORDS + 4], j0 = ch & 0xffffu, nj = ch >> 16;
  // the program, a conjunct at a time: the OR of its middle bins and of its
  // edge bins (four loads issued together), then the AND into the result
  uint32_t acc[V], unc[V];
#pragma unroll
  for (int k = 0; k < V; ++k) acc[k] = 0xffffffffu, unc[k] = 0;
  const uint32_t *sl = stage + lane * V;
  for (uint32_t jj = 0; jj < nj; ++jj) {
    const uint32_t h = conj[j0 + jj];
    const uint16_t *e = chain + (h & BJ_FIRST);
    const uint32_t nm = (h >> BJ_NMID_SHIFT) & 0xffu, ne = (h >> BJ_NEDGE_SHIFT) & 0xfu;
    uint32_t cm[V], cx[V];
#pragma unroll
    for (int k = 0; k < V; ++k) cm[k] = 0, cx[k] = 0;
    uint32_t i = 0;
    for (; i + 4 <= nm; i += 4) {
      uint32_t x[4][V];
#pragma unroll
      for (int j = 0; j < 4; ++j) lds_words<V>(sl + e[i + j] * T, x[j]);
#pragma unroll
      for (int k = 0; k < V; ++k) cm[k] |= (x[0][k] | x[1][k]) | (x[2][k] | x[3][k]);
    }
    for (; i < nm + ne; ++i) {  // the last middle bins, then the edge bins
      uint32_t x[V];
      lds_words<V>(sl + e[i] * T, x);
      if (i < nm) {
#pragma unroll
        for (int k = 0; k < V; ++k) cm[k] |= x[k];
      } else {
#pragma unroll
        for (int k = 0; k < V; ++k) cx[k] |= x[k];
      }
    }
    if (h & BJ_NEG) {
#pragma unroll
      for (int k = 0; k < V; ++k) acc[k] &= ~(cm[k] | cx[k]);
    } else {
#pragma unroll
      for (int k = 0; k < V; ++k) acc[k] &= cm[k] | cx[k], unc[k] |= cx[k];
    }
  }
  uint32_t p[V], u[V];
  if (w0 + T <= nwords && (tail == 0 || w0 + T < nwords)) {  // an interior tile: no mask
#pragma unroll
    for (int k = 0; k < V; ++k) p[k] = acc[k], u[k] = unc[k] & acc[k];
  } else {
#pragma unroll
    for (int k = 0; k < V; ++k) {
      const uint64_t w = w0 + lane * V + k;
      uint32_t m = w < nwords ? 0xffffffffu : 0u;
      if (tail && w + 1 == nwords) m = (1u << tail) - 1u;
      p[k] = acc[k] & m;
      u[k] = unc[k] & p[k];
    }
  }
  const uint32_t rowbase = (uint32_t)((w0 + lane * V) * 32);  // first row of the lane's words
  // word 7: slots read through a foreign key (generic drain); word 6: shape
  switch (C.Qd[q * BQD_WORDS + 7] ? 0u : C.Qd[q * BQD_WORDS + 6]) {
  case 1: b_rows<BDrain<0>, V, 1, CH>(C, q, p, u, rowbase, buf); break;
  case 2: b_rows<BDrain<1>, V, 1, CH>(C, q, p, u, rowbase, buf); break;
  case 3: b_rows<BDrain<2>, V, 1, CH>(C, q, p, u, rowbase, buf); break;
  case 4: b_rows<BDrain<3>, V, 1, CH>(C, q, p, u, rowbase, buf); break;
  default: b_rows<BDrainAny, V, 1, CH>(C, q, p, u, rowbase, buf); break;
  }
}

template <int V, int CH>
__global__ void __launch_bounds__(BT_THREADS_MAX, 1)
batch_scan_kernel(const BatchHdr *__restrict__ H, const __grid_constant__ BParams P,
                  const CUtensorMap *__restrict__ maps, unsigned long long *__restrict__ out,
                  unsigned long long *__restrict__ nqual, uint32_t *errw) {
  constexpr uint32_t T = 32 * V;
  extern __shared__ __align__(128) uint8_t smem[];
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  const BLayout &L = P.L;
  uint32_t *Qd = reinterpret_cast<uint32_t *>(smem + L.off_Q);
  unsigned long long *scol = reinterpret_cast<unsigned long long *>(smem + L.off_src);
  unsigned long long *sfk = scol + BS_MAX;
  uint32_t *sdim = reinterpret_cast<uint32_t *>(sfk + BS_MAX), *swid = sdim + BS_MAX;
  unsigned long long *qsum = reinterpret_cast<unsigned long long *>(smem + L.off_sum);
  unsigned long long *qcnt = reinterpret_cast<unsigned long long *>(smem + L.off_cnt);
  uint32_t *toff = reinterpret_cast<uint32_t *>(smem + L.off_toff);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + L.off_bar), *empty = full + P.S;
  uint32_t *qctr = reinterpret_cast<uint32_t *>(smem + L.off_ctr), *abort_ = qctr + P.S;
  uint8_t *order = smem + L.off_order;
  uint16_t *chain = reinterpret_cast<uint16_t *>(smem + L.off_chain);
  uint32_t *conj = reinterpret_cast<uint32_t *>(smem + L.off_conj);
  unsigned long long *stab = reinterpret_cast<unsigned long long *>(smem + L.off_stab);
  uint32_t *wbuf = reinterpret_cast<uint32_t *>(smem + L.off_buf) + warp * L.buf;
  uint32_t *stages = reinterpret_cast<uint32_t *>(smem + L.off_stage);

  for (uint32_t i = tid; i < P.nq * BQD_WORDS; i += blockDim.x) Qd[i] = H->Qd[i];
  for (uint32_t i = tid; i < P.nq; i += blockDim.x) qsum[i] = 0, qcnt[i] = 0, toff[i] = H->toff[i];
  for (uint32_t i = tid; i < P.nstab; i += blockDim.x) stab[i] = 0;
  for (uint32_t i = tid; i < P.nchain; i += blockDim.x) chain[i] = H->chain[i];
  for (uint32_t i = tid; i < P.nconj; i += blockDim.x) conj[i] = H->conj[i];
  for (uint32_t i = tid; i < P.nq; i += blockDim.x) order[i] = H->order[i];
  if (tid < BS_MAX) {
    scol[tid] = reinterpret_cast<unsigned long long>(H->src[tid].col);
    sfk[tid] = reinterpret_cast<unsigned long long>(H->src[tid].fk);
    sdim[tid] = H->src[tid].dimsz;
    swid[tid] = H->src[tid].width;
  }
  if (tid <= P.S) qctr[tid] = 0;  // the counters and the abort flag
  if (tid == 0) {
    for (uint32_t s = 0; s < P.S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], nw - 1);  // the workers
    }
    fence_mbar_init();
  }
  __syncthreads();

  BCtx C;
  C.Qd = Qd;
  C.scol = scol;
  C.sfk = sfk;
  C.sdim = sdim;
  C.toff = toff;
  C.out = out;
  C.qsum = qsum;
  C.qcnt = qcnt;
  C.stab = stab;

  const uint64_t ntiles = (P.nwords + T - 1) / T;
  // tiles of this CTA (fewer than 2^32: a table has fewer than 2^31 rows)
  const uint32_t nit = blockIdx.x < ntiles ? (uint32_t)((ntiles - 1 - blockIdx.x) / gridDim.x + 1) : 0u;
  const uint32_t tail = (uint32_t)(P.nrows & 31u);

  if (warp == nw - 1) {
    // ------------------------------------------------------------ producer
    // stage j % S <- the CTA's j-th tile, once the workers have left the
    // tile it held: reset the stage's query counter, arm the stage with its
    // byte count, then the tensor copies of the staged bitmap rows x T words
    // (copy c by lane c % 32); the tile's rows of the dense payload columns
    // into L2.
    uint32_t issued = 0;
    bool ok = true;
    // stage s of tile j = j % S; the workers released its previous tile in
    // phase (j / S - 1) of empty[s]: epar, flipped at every wrap after the first
    uint32_t s = 0, epar = 0;
    for (uint32_t j = 0; j < nit && ok; ++j, s = s + 1 == P.S ? 0u : s + 1u) {
      if (j >= P.S && s == 0 && j > P.S) epar ^= 1u;
      if (j >= P.S) {
        ok = mbar_wait_bounded(&empty[s], epar, errw, MB_DEVERR_IDLE_WAIT, P.wait_tries);
        ok = __all_sync(0xffffffffu, ok);
        if (!ok || __any_sync(0xffffffffu, *(volatile uint32_t *)abort_ != 0)) break;
      }
      const uint64_t w0 = ((uint64_t)blockIdx.x + (uint64_t)j * gridDim.x) * T, r0 = w0 * 32;
      const bool skip = P.skip_stage0 && j == 0;
      if (lane == 0) {
        qctr[s] = 0;
        mbar_arrive_expect_tx(&full[s], P.nu * T * 4);  // (release: the counter reset is seen with the phase)
      }
      __syncwarp();
      fence_proxy_async_smem();
      uint32_t *dst = stages + (size_t)s * L.stage_words;
      if (!skip)
        for (uint32_t c = lane; c < P.ncopy; c += 32) {
          const uint32_t e = P.copy[c];
          tma_load_2d(dst + ((e >> 12) & 0xfffu) * T, maps + (e >> 24), (int)w0, (int)(e & 0xfffu), &full[s]);
        }
      if (lane < P.nsrc && ((P.pf_mask >> lane) & 1u) && r0 < P.nrows) {
        const uint64_t nr = P.nrows - r0 < T * 32 ? P.nrows - r0 : T * 32;
        const bool viafk = sfk[lane] != 0;
        const uint32_t w = viafk ? 4u : swid[lane];
        const uint8_t *base = reinterpret_cast<const uint8_t *>(viafk ? sfk[lane] : scol[lane]) + r0 * w;
        const uint32_t pb = (uint32_t)(nr * w) & ~15u;
        if (pb) prefetch_l2(base, pb);
      }
      ++issued;
    }
    if (!ok && lane == 0) atomicExch(abort_, 1u);
    if (*(volatile uint32_t *)abort_ && lane == 0) {
      // let the copies still in flight land before the CTA exits
      for (uint32_t j = issued > P.S ? issued - P.S : 0; j < issued; ++j)
        mbar_wait_bounded(&full[j % P.S], (j / P.S) & 1u, nullptr, 0, 1u << 16);  // (32-bit, error path only)
    }
  } else {
    // ------------------------------------------------------------- workers
    // tile `it` of the CTA: wait for its stage, take queries off the
    // stage's counter (costliest first) until none is left, then release the
    // stage to the producer.  Warps move on to the next staged tile without
    // waiting for each other.
    uint32_t s = 0, par = 0;  // stage it % S and the parity of its phase, (it / S) & 1
    for (uint32_t it = 0; it < nit; ++it, par ^= (s + 1 == P.S) ? 1u : 0u, s = s + 1 == P.S ? 0u : s + 1u) {
      const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(&full[s], par, errw, MB_DEVERR_TMA_WAIT, P.wait_tries));
      if (!ok) {
        if (lane == 0) atomicExch(abort_, 1u);
        break;
      }
      if (__any_sync(0xffffffffu, *(volatile uint32_t *)abort_ != 0)) break;
      const uint64_t w0 = ((uint64_t)blockIdx.x + (uint64_t)it * gridDim.x) * T;
      const uint32_t *st = stages + (size_t)s * L.stage_words;
      while (true) {
        uint32_t qi = 0;
        if (lane == 0) qi = atomicAdd(&qctr[s], 1u);
        qi = __shfl_sync(0xffffffffu, qi, 0);
        if (qi >= P.nq) break;
        b_query<V, CH>(C, chain, conj, st, w0, P.nwords, tail, order[qi], wbuf);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
  }
  __syncthreads();
  if (*(volatile uint32_t *)abort_) return;
  for (uint32_t q = tid; q < P.nq; q += blockDim.x) {
    const uint32_t *d = Qd + q * BQD_WORDS;
    if (qsum[q]) atomicAdd(&out[d[2]], qsum[q]);
    if (qcnt[q]) atomicAdd(&nqual[d[3]], qcnt[q]);
  }
  // the shared group tables, one warp per query
  for (uint32_t q = warp; q < P.nq; q += nw) {
    const uint32_t t = toff[q];
    if (t == BT_NOTABLE) continue;
    const uint32_t *d = Qd + q * BQD_WORDS;
    for (uint32_t g = lane; g < d[1]; g += 32)
      if (stab[t + g]) atomicAdd(&out[d[2] + g], stab[t + g]);
  }
}

}  // namespace

size_t batch_smem(const BatchHdr &h, const BatchCfg &c) {
  if (c.V != 1 && c.V != 2 && c.V != 4 && c.V != 6) return 0;
  if (c.warps < 2 || c.warps > BW_MAX || c.stages == 0 || c.stages > 4) return 0;  // a producer and workers
  if (c.buf != 0 && c.buf != BT_BUF && c.buf != 1024) return 0;
  return blayout(h.nq, h.nchain, h.nconj, h.nu, c.stages, 32 * c.V, h.nstab, c.warps, c.buf).total;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).
mb_status batch_encode_maps(const uint32_t *slab, uint64_t stride, uint32_t nslab, uint32_t T, void *host_maps) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  if (!encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    MB_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !fn) return fail(MB_ERR_CUDA, "batch: cuTensorMapEncodeTiled not found");
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  static_assert(sizeof(CUtensorMap) == BMAP_BYTES, "tensor map size");
  if (T == 0 || T > 256 || (T * 4) % 16 != 0 || ((uintptr_t)slab & 15) != 0 || (stride * 4) % 16 != 0)
    return fail(MB_ERR_INVALID, "batch: tensor map shape (T %u, stride %llu)", T, (unsigned long long)stride);
  CUtensorMap *m = static_cast<CUtensorMap *>(host_maps);
  const cuuint64_t dim[2] = {stride, nslab};
  const cuuint64_t gstride[1] = {stride * 4};
  const cuuint32_t estride[2] = {1, 1};
  for (uint32_t h = 1; h <= BMAP_COUNT; ++h) {
    const cuuint32_t box[2] = {T, h};
    const CUresult r = encode(&m[h - 1], CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, const_cast<uint32_t *>(slab), dim,
                              gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(MB_ERR_CUDA, "batch: cuTensorMapEncodeTiled failed (%d)", (int)r);
  }
  return MB_OK;
}

template <int V>
static mb_status launch_bs(const BatchHdr &h, const BatchHdr *dh, const BatchCfg &c, const void *maps, int64_t *out,
                           uint64_t *nqual, cudaStream_t st) {
  auto kern = c.buf == 1024 ? batch_scan_kernel<V, 32> : batch_scan_kernel<V, BT_BUF / 32>;
  BParams P;
  memset(&P, 0, sizeof(P));
  P.nrows = h.nrows;
  P.nwords = h.nwords;
  P.nq = h.nq;
  P.nu = h.nu;
  P.ncopy = h.ncopy;
  memcpy(P.copy, h.copy, sizeof(P.copy));
  P.nsrc = h.nsrc;
  P.nchain = h.nchain;
  P.nconj = h.nconj;
  P.pf_mask = h.pf_mask;
  P.nstab = h.nstab;
  P.S = c.stages;
  P.wait_tries = c.wait_tries ? c.wait_tries : (1u << 20);
  P.skip_stage0 = c.skip_stage0;
  P.L = blayout(h.nq, h.nchain, h.nconj, h.nu, c.stages, 32 * V, h.nstab, c.warps, c.buf);
  // the 64-bit areas (sums, counts, group tables, mbarriers) must be 8-byte
  // aligned, the stage 128-byte aligned (tensor copies): refuse a layout that
  // is not, rather than launch it
  if ((P.L.off_sum | P.L.off_cnt | P.L.off_stab | P.L.off_bar | P.L.off_src) & 7u || (P.L.off_stage & 127u) ||
      (P.L.off_buf & 15u) || (P.L.off_conj & 3u) || (P.L.off_toff & 3u) || (P.L.off_ctr & 3u))
    return fail(MB_ERR_INVALID, "batch: shared-memory layout misaligned");
  const DevInfo &di = dev_info();
  const size_t smem = P.L.total;
  if (smem > (size_t)di.max_smem_optin) return fail(MB_ERR_UNSUPPORTED, "batch: %zu bytes of shared memory", smem);
  MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, (int)(c.warps * 32), smem));
  if (occ < 1) return fail(MB_ERR_UNSUPPORTED, "batch: kernel does not fit on an SM");
  if (c.cps && (int)c.cps < occ) occ = (int)c.cps;
  const uint64_t ntiles = (h.nwords + 32 * V - 1) / (32 * V);
  uint64_t grid = (uint64_t)di.sms * occ;
  if (grid > ntiles) grid = ntiles;
  uint32_t *errw = device_error_word();
  if (!errw) return fail(MB_ERR_OOM, "batch: device error word");
  kern<<<(unsigned)grid, c.warps * 32, smem, st>>>(dh, P, static_cast<const CUtensorMap *>(maps),
                                                   reinterpret_cast<unsigned long long *>(out),
                                                   reinterpret_cast<unsigned long long *>(nqual), errw);
  MB_LAUNCH_CHECK("batch_scan_kernel");
  return MB_OK;
}

mb_status batch_scan(const BatchHdr &h, const BatchHdr *dh, const BatchCfg &c, const void *maps, int64_t *out,
                     uint64_t *nqual, cudaStream_t st) {
  if (h.nq == 0 || h.nrows == 0) return MB_OK;
  if (h.nq > BQ_MAX || h.nu > BU_MAX || h.nsrc > BS_MAX || h.nchain > BC_MAX || h.nconj > BJ_MAX)
    return fail(MB_ERR_INVALID, "batch: descriptor over its limits");
  // every program within the chain and its stage rows within the stage
  for (uint32_t q = 0; q < h.nq; ++q) {
    const uint32_t w4 = h.Qd[(size_t)q * BQD_WORDS + 4], j0 = w4 & 0xffffu, nj = w4 >> 16;
    if (j0 + nj > h.nconj) return fail(MB_ERR_INVALID, "batch: query %u program out of range", q);
    for (uint32_t j = j0; j < j0 + nj; ++j) {
      const uint32_t c = h.conj[j], f = c & BJ_FIRST, n = ((c >> BJ_NMID_SHIFT) & 0xffu) + ((c >> BJ_NEDGE_SHIFT) & 0xfu);
      if (f + n > h.nchain) return fail(MB_ERR_INVALID, "batch: conjunct %u out of range", j);
      for (uint32_t i = f; i < f + n; ++i)
        if (h.chain[i] >= h.nu) return fail(MB_ERR_INVALID, "batch: chain row %u not staged", (uint32_t)h.chain[i]);
    }
  }
  // shared group tables: each within the table area, of its query's size
  for (uint32_t q = 0; q < h.nq; ++q) {
    const uint32_t t = h.toff[q], ng = h.Qd[(size_t)q * BQD_WORDS + 1];
    if (t != 0xffffffffu && ((uint64_t)t + ng > h.nstab || ((h.Qd[(size_t)q * BQD_WORDS] >> 8) & 1u)))
      return fail(MB_ERR_INVALID, "batch: group table of query %u (slots %u+%u of %u)", q, t, ng, h.nstab);
  }
  if (h.stride % 32 != 0 || h.stride < h.nwords || ((uintptr_t)h.slab & 15) != 0 || h.nslab > 4096 ||
      h.nrows >= (1ull << 31))
    return fail(MB_ERR_INVALID, "batch: bitmap slab (stride %llu, %u rows) over %llu table rows",
                (unsigned long long)h.stride, h.nslab, (unsigned long long)h.nrows);
  // the copies must tile stage rows [0, nu) exactly, from rows of the slab
  if (h.nu == 0 || h.ncopy == 0 || h.ncopy > BCP_MAX) return fail(MB_ERR_INVALID, "batch: %u staging copies", h.ncopy);
  if (!maps || ((uintptr_t)maps & 63) != 0) return fail(MB_ERR_INVALID, "batch: tensor maps not 64-byte aligned");
  {
    uint32_t next = 0;
    for (uint32_t i = 0; i < h.ncopy; ++i) {
      const uint32_t e = h.copy[i], r0 = e & 0xfffu, t0 = (e >> 12) & 0xfffu, hh = (e >> 24) + 1;
      if (t0 != next || r0 + hh > h.nslab)
        return fail(MB_ERR_INVALID, "batch: staging copy %u (rows %u+%u to %u)", i, r0, hh, t0);
      next = t0 + hh;
    }
    if (next != h.nu) return fail(MB_ERR_INVALID, "batch: staging copies cover %u of %u rows", next, h.nu);
  }
  if (batch_smem(h, c) == 0) return fail(MB_ERR_INVALID, "batch: launch shape V=%u warps=%u stages=%u", c.V,
                                         c.warps, c.stages);
  switch (c.V) {
  case 6: return launch_bs<6>(h, dh, c, maps, out, nqual, st);
  case 4: return launch_bs<4>(h, dh, c, maps, out, nqual, st);
  case 2: return launch_bs<2>(h, dh, c, maps, out, nqual, st);
  default: return launch_bs<1>(h, dh, c, maps, out, nqual, st);
  }
}

}  // namespace mb
