// batch.cu - the batched scan kernel (see batch.cuh for the design).
//
// Reference: the per-query fused kernel vprg_grpby (primitive.cuh:340-445)
// and its op functors (ssb/lambdas.cuh:19-152) define what each query of a
// batch computes; the batch evaluates the same programs with the same
// candidate-check semantics, so every query's groups and row count equal what
// it gets alone.
//
// A CTA's warps split into producers and consumers.
//
// Producers walk the CTA's row tiles (T = 32 * V words), S tiles of the
// bitmaps in flight: the index is one slab of bitmap rows, so a tile of the
// rows the batch reads is staged by one 2-D tensor copy per run of rows
// (TMA, box = run x T words, all completing on the stage's mbarrier; the
// copies are issued by lane 0 of every producer warp in turn) and the tile's
// payload rows are prefetched into L2.  On a tile,
// producers take the batch's queries off a counter, costliest first; for its
// query a producer evaluates the conjunctive chain on the staged words and
// appends the selected rows to the query's own row queue.  Every 64 queued
// rows become a job in a ring in shared memory.  A producer barrier closes
// the tile (then its stage is refilled), so a query is on one producer at a
// time and its queue, which outlives the tile, needs no atomics.
//
// Consumers take jobs off the ring and run the op on their 64 rows: one
// query per job, so every descriptor read is a broadcast and every branch on
// the descriptor uniform (a compiled drain for the engine's op shapes, the
// generic one otherwise).  Drains wait on payload gathers; on their own
// warps that latency overlaps the producers' bitmap work instead of stalling
// the tile.  A producer that finds the ring full runs the drain itself.
// 1-group sums and row counts accumulate per warp (plain adds) and are
// folded at the end.
//
// Job states move FREE -> FILL -> READY -> RUN -> FREE by compare-and-swap.
// Every wait is bounded: a stage that does not arrive, or consumers idle for
// too long, record the block in the device error word; the block then stops
// and lets its copies land before exiting.
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
constexpr uint32_t BQQ = 96;  // a query's queue: < 64 pending + one 32-entry round
constexpr uint32_t BJ = 64;   // jobs in the ring
constexpr uint32_t CONSUMER_IDLE_TRIES = 1u << 24;  // x 128 ns sleeps, about two seconds
enum : uint32_t { JOB_FREE = 0, JOB_FILL = 1, JOB_READY = 2, JOB_RUN = 3 };
struct Job {
  uint32_t state, q, n, pad_;
  uint32_t rows[64];
};

// Shared-memory layout of one launch (identical on host and device).
struct BLayout {
  uint32_t off_Q, off_src, off_sum, off_cnt, off_len, off_bar, off_ctr, off_order, off_chain, off_qbuf, off_jobs,
      off_stage, total;
};

__host__ __device__ inline uint32_t align_up(uint32_t x, uint32_t a) { return (x + a - 1) / a * a; }

__host__ __device__ inline BLayout blayout(uint32_t nq, uint32_t nchain, uint32_t nu, uint32_t warps, uint32_t S,
                                           uint32_t T) {
  BLayout L;
  uint32_t o = 0;
  L.off_Q = o;
  o += nq * BQD_WORDS * 4;
  L.off_src = o = align_up(o, 16);
  o += BS_MAX * 24;  // col[] and fk[] (8 bytes), dimsz[] and width[] (4 bytes)
  L.off_sum = o = align_up(o, 16);
  o += warps * nq * 8;  // per warp and query: 1-group sum
  L.off_cnt = o;
  o += warps * nq * 4;  // per warp and query: kept rows
  L.off_len = o;
  o += nq * 4;  // per query: rows queued
  L.off_bar = o = align_up(o, 8);
  o += 8 * S;
  L.off_ctr = o;
  o += 6 * 4;  // qctr[2], tiles issued, producers done, producer error, consumer error
  L.off_order = o;
  o += nq;
  L.off_chain = o = align_up(o, 16);
  o += align_up(nchain * 2, 16);
  L.off_qbuf = o;
  o += nq * BQQ * 4;
  L.off_jobs = o = align_up(o, 16);
  o += BJ * (uint32_t)sizeof(Job);
  L.off_stage = o = align_up(o, 128);
  o += S * nu * T * 4;
  L.total = o;
  return L;
}

struct BParams {
  uint64_t nrows, nwords;
  uint32_t nq, nu, nsrc, nchain, pf_mask, S, np;  // np: producer warps
  uint32_t ncopy;
  uint32_t copy[BCP_MAX];  // BatchHdr::copy
  BLayout L;
};


// The batch's tables as a warp sees them (shared memory).
struct BCtx {
  const uint32_t *Qd;
  const unsigned long long *scol, *sfk;
  const uint32_t *sdim;
  unsigned long long *out;
  unsigned long long *usum;  // this warp's 1-group sums, per query
  uint32_t *ucnt;            // this warp's kept rows, per query
  Job *jobs;
};

// Value of a 1-, 2- or 4-byte element without a branch on the width: the
// aligned 32-bit word holding it, shifted and masked.  The word lies in the
// same 4-byte block (hence the same page) as the element itself.
__device__ __forceinline__ uint32_t b_ldw(const void *col, uint32_t i, uint32_t w) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(col) + (uintptr_t)i * w;
  const uint32_t word = __ldg(reinterpret_cast<const uint32_t *>(a & ~(uintptr_t)3));
  const uint32_t sh = (uint32_t)(a & 3) * 8;
  const uint32_t mask = w >= 4 ? 0xffffffffu : ((1u << (8 * w)) - 1u);
  return (word >> sh) & mask;
}

// Runs query q's op on the first n (<= 64) entries of qe (row | uncertain
// << 31), two rows per lane, and accumulates them: 1-group sums (a warp
// reduction) and kept rows into the warp's own slots, group sums by one
// global atomic add per row.  q is warp-uniform: descriptor reads are broadcasts, branches on
// the descriptor uniform, and the slots unrolled, so no value is picked by
// a run-time index.  All 32 lanes call it.
__device__ __forceinline__ void b_drain(const BCtx &C, uint32_t q, const uint32_t *qe, uint32_t n) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t *d = C.Qd + q * BQD_WORDS;
  const uint32_t h0 = d[0], roles = d[5];
  const uint32_t nslot = h0 & 0xffu, kv = roles & 0xffu, filt = (roles >> 8) & 0xffu, keym = (roles >> 16) & 0xffu,
                 termm = roles >> 24;
  const bool ok0 = lane < n, ok1 = lane + 32 < n;
  const uint32_t e0 = ok0 ? qe[lane] : 0u, e1 = ok1 ? qe[lane + 32] : 0u;
  const bool c0 = ok0 && (e0 >> 31), c1 = ok1 && (e1 >> 31);
  const uint32_t r0 = e0 & 0x7fffffffu, r1 = e1 & 0x7fffffffu;
  uint32_t v0[BSLOT], v1[BSLOT], bad0 = 0, bad1 = 0;
#pragma unroll
  for (uint32_t s = 0; s < BSLOT; ++s) {
    v0[s] = v1[s] = 0;
    if (s < nslot) {
      const uint32_t a = d[BQD_SLOT0 + BQD_SLOTW * s], t = a & 0xffu, w = (a >> 8) & 0xffu;
      const bool kvs = (kv >> s) & 1u, fs = (filt >> s) & 1u;
      bool l0 = ok0 && (kvs || (c0 && fs)), l1 = ok1 && (kvs || (c1 && fs));
      uint32_t k0 = r0, k1 = r1;
      const uint32_t *fk = reinterpret_cast<const uint32_t *>(C.sfk[t]);
      if (fk) {
        if (l0) k0 = __ldg(fk + r0);
        if (l1) k1 = __ldg(fk + r1);
        const uint32_t dz = C.sdim[t];
        if (dz) {
          if (l0 && k0 >= dz) bad0 |= 1u << s, l0 = false;
          if (l1 && k1 >= dz) bad1 |= 1u << s, l1 = false;
        }
      }
      const void *col = reinterpret_cast<const void *>(C.scol[t]);
      if (l0) v0[s] = b_ldw(col, k0, w);
      if (l1) v1[s] = b_ldw(col, k1, w);
    }
  }
  bool keep0 = ok0, keep1 = ok1;
  // candidate check of uncertain rows: the single-term clauses, bounds
  // intersected per slot
  if (termm && __any_sync(0xffffffffu, c0 || c1)) {
#pragma unroll
    for (uint32_t s = 0; s < BSLOT; ++s)
      if ((termm >> s) & 1u) {
        const uint32_t lo = d[BQD_SLOT0 + BQD_SLOTW * s + 1], hi = d[BQD_SLOT0 + BQD_SLOTW * s + 2];
        keep0 = keep0 && (!c0 || (!((bad0 >> s) & 1u) && v0[s] >= lo && v0[s] <= hi));
        keep1 = keep1 && (!c1 || (!((bad1 >> s) & 1u) && v1[s] >= lo && v1[s] <= hi));
      }
  }
  // group key: sum over key slots of mul * (xform(value) - base)
  uint32_t g0 = 0, g1 = 0;
#pragma unroll
  for (uint32_t s = 0; s < BSLOT; ++s)
    if ((keym >> s) & 1u) {
      const uint32_t *sl = d + BQD_SLOT0 + BQD_SLOTW * s;
      const uint32_t a = sl[0], xf = (a >> 16) & 0xffu;
      keep0 = keep0 && !((bad0 >> s) & 1u);
      keep1 = keep1 && !((bad1 >> s) & 1u);
      uint32_t x0 = v0[s], x1 = v1[s];
      if (xf == MB_X_DIV) {
        const uint32_t m = sl[3], sh1 = (a >> 24) & 15u, sh2 = a >> 28;
        x0 = div_by_magic(x0, m, sh1, sh2);
        x1 = div_by_magic(x1, m, sh1, sh2);
      } else if (xf == MB_X_YEAR) {
        x0 = date_to_year(x0);
        x1 = date_to_year(x1);
      }
      const uint32_t base = sl[4], mul = sl[5];
      g0 += mul * (x0 - base);
      g1 += mul * (x1 - base);
    }
  const uint32_t ng = d[1];
  keep0 = keep0 && g0 < ng;
  keep1 = keep1 && g1 < ng;
  // value
  const uint32_t vkind = (h0 >> 16) & 15u, va = (h0 >> 20) & 15u, vb = (h0 >> 24) & 15u;
  uint64_t x0 = 1, x1 = 1;
  if (vkind != MB_V_ONE) {
    uint64_t a0 = 0, a1 = 0, b0 = 0, b1 = 0;
#pragma unroll
    for (uint32_t s = 0; s < BSLOT; ++s) {
      if (s == va) a0 = v0[s], a1 = v1[s];
      if (s == vb) b0 = v0[s], b1 = v1[s];
    }
    keep0 = keep0 && !((bad0 >> va) & 1u);
    keep1 = keep1 && !((bad1 >> va) & 1u);
    if (vkind == MB_V_COL) {
      x0 = a0, x1 = a1;
    } else {
      keep0 = keep0 && !((bad0 >> vb) & 1u);
      keep1 = keep1 && !((bad1 >> vb) & 1u);
      x0 = vkind == MB_V_MUL ? a0 * b0 : (uint64_t)((int64_t)a0 - (int64_t)b0);
      x1 = vkind == MB_V_MUL ? a1 * b1 : (uint64_t)((int64_t)a1 - (int64_t)b1);
    }
  }
  const uint32_t kept = __popc(__ballot_sync(0xffffffffu, keep0)) + __popc(__ballot_sync(0xffffffffu, keep1));
  if ((h0 >> 8) & 1u) {  // one group: a warp sum into the warp's slot
    const uint64_t s = peer_sum64(0xffffffffu, (keep0 ? x0 : 0) + (keep1 ? x1 : 0));
    if (lane == 0) C.usum[q] += s;
  } else {
    // one atomic add per kept row: the rows of a chunk spread over many
    // groups, and grouping peers first (match + reduce per group) costs more
    // than it saves
    const uint32_t base = d[2];
    if (keep0) atomicAdd(&C.out[base + g0], (unsigned long long)x0);
    if (keep1) atomicAdd(&C.out[base + g1], (unsigned long long)x1);
  }
  if (lane == 0) C.ucnt[q] += kept;
  __syncwarp();
}

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

// b_drain for a compiled shape SH (BSHAPES) whose sources are fact columns
// (no foreign keys): the slots, their roles and the key transforms are known
// at compile time; only the columns, bounds and key constants are read from
// the descriptor.  Every address is formed first and every load issued in
// one run, so a drain waits for one memory round trip, not one per slot.
// Same results as b_drain.
template <int SH>
__device__ __forceinline__ void b_drain_s(const BCtx &C, uint32_t q, const uint32_t *qe, uint32_t n) {
  constexpr BShape sh = BSHAPES[SH];
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t *d = C.Qd + q * BQD_WORDS;
  const bool ok0 = lane < n, ok1 = lane + 32 < n;
  const uint32_t e0 = ok0 ? qe[lane] : 0u, e1 = ok1 ? qe[lane + 32] : 0u;
  const bool c0 = ok0 && (e0 >> 31), c1 = ok1 && (e1 >> 31);
  const uint32_t r0 = e0 & 0x7fffffffu, r1 = e1 & 0x7fffffffu;
  // addresses
  uintptr_t a0[BSLOT], a1[BSLOT];
  uint32_t wd[BSLOT];
  bool l0[BSLOT], l1[BSLOT];
#pragma unroll
  for (uint32_t s = 0; s < BSLOT; ++s) {
    a0[s] = a1[s] = 0;
    wd[s] = 4;
    l0[s] = l1[s] = false;
    if (s < sh.ns && (((sh.kv | sh.filt) >> s) & 1u)) {
      const bool kvs = (sh.kv >> s) & 1u;
      const uint32_t a = d[BQD_SLOT0 + BQD_SLOTW * s], t = a & 0xffu;
      wd[s] = (a >> 8) & 0xffu;
      const uintptr_t col = (uintptr_t)C.scol[t];
      l0[s] = ok0 && (kvs || c0);
      l1[s] = ok1 && (kvs || c1);
      a0[s] = col + (uintptr_t)r0 * wd[s];
      a1[s] = col + (uintptr_t)r1 * wd[s];
    }
  }
  // loads: the aligned words holding the values, all issued before any use
  uint32_t raw0[BSLOT], raw1[BSLOT];
#pragma unroll
  for (uint32_t s = 0; s < BSLOT; ++s) {
    raw0[s] = raw1[s] = 0;
    if (s < sh.ns && (((sh.kv | sh.filt) >> s) & 1u)) {
      raw0[s] = ldg_pred(reinterpret_cast<const void *>(a0[s] & ~(uintptr_t)3), l0[s]);
      raw1[s] = ldg_pred(reinterpret_cast<const void *>(a1[s] & ~(uintptr_t)3), l1[s]);
    }
  }
  uint32_t v0[BSLOT], v1[BSLOT];
#pragma unroll
  for (uint32_t s = 0; s < BSLOT; ++s) {
    const uint32_t mask = wd[s] >= 4 ? 0xffffffffu : ((1u << (8 * wd[s])) - 1u);
    v0[s] = (raw0[s] >> ((uint32_t)(a0[s] & 3) * 8)) & mask;
    v1[s] = (raw1[s] >> ((uint32_t)(a1[s] & 3) * 8)) & mask;
  }
  const uint32_t bad0 = 0, bad1 = 0;
  bool keep0 = ok0, keep1 = ok1;
  if (sh.filt && __any_sync(0xffffffffu, c0 || c1)) {
#pragma unroll
    for (uint32_t s = 0; s < BSLOT; ++s)
      if ((sh.filt >> s) & 1u) {
        const uint32_t lo = d[BQD_SLOT0 + BQD_SLOTW * s + 1], hi = d[BQD_SLOT0 + BQD_SLOTW * s + 2];
        keep0 = keep0 && (!c0 || (!((bad0 >> s) & 1u) && v0[s] >= lo && v0[s] <= hi));
        keep1 = keep1 && (!c1 || (!((bad1 >> s) & 1u) && v1[s] >= lo && v1[s] <= hi));
      }
  }
  uint32_t g0 = 0, g1 = 0;
#pragma unroll
  for (uint32_t s = 0; s < BSLOT; ++s)
    if ((sh.keym >> s) & 1u) {
      const uint32_t *sl = d + BQD_SLOT0 + BQD_SLOTW * s;
      keep0 = keep0 && !((bad0 >> s) & 1u);
      keep1 = keep1 && !((bad1 >> s) & 1u);
      uint32_t x0 = v0[s], x1 = v1[s];
      constexpr uint32_t XDIV = 1, XYEAR = 2;
      const uint32_t xf = (sh.xf >> (2 * s)) & 3u;
      if (xf == XDIV) {
        const uint32_t a = sl[0], m = sl[3], sh1 = (a >> 24) & 15u, sh2 = a >> 28;
        x0 = div_by_magic(x0, m, sh1, sh2);
        x1 = div_by_magic(x1, m, sh1, sh2);
      } else if (xf == XYEAR) {
        x0 = date_to_year(x0);
        x1 = date_to_year(x1);
      }
      const uint32_t base = sl[4], mul = sl[5];
      g0 += mul * (x0 - base);
      g1 += mul * (x1 - base);
    }
  const uint32_t ng = d[1];
  keep0 = keep0 && g0 < ng;
  keep1 = keep1 && g1 < ng;
  uint64_t x0 = 1, x1 = 1;
  if (sh.vk != MB_V_ONE) {
    keep0 = keep0 && !((bad0 >> sh.va) & 1u);
    keep1 = keep1 && !((bad1 >> sh.va) & 1u);
    const uint64_t a0 = v0[sh.va], a1 = v1[sh.va];
    if (sh.vk == MB_V_COL) {
      x0 = a0, x1 = a1;
    } else {
      keep0 = keep0 && !((bad0 >> sh.vb) & 1u);
      keep1 = keep1 && !((bad1 >> sh.vb) & 1u);
      const uint64_t b0 = v0[sh.vb], b1 = v1[sh.vb];
      x0 = sh.vk == MB_V_MUL ? a0 * b0 : (uint64_t)((int64_t)a0 - (int64_t)b0);
      x1 = sh.vk == MB_V_MUL ? a1 * b1 : (uint64_t)((int64_t)a1 - (int64_t)b1);
    }
  }
  const uint32_t kept = __popc(__ballot_sync(0xffffffffu, keep0)) + __popc(__ballot_sync(0xffffffffu, keep1));
  if ((d[0] >> 8) & 1u) {  // one group: a warp sum into the query's slot
    const uint64_t s = peer_sum64(0xffffffffu, (keep0 ? x0 : 0) + (keep1 ? x1 : 0));
    if (lane == 0) C.usum[q] += s;
  } else {
    // one atomic add per kept row: the rows of a chunk spread over many
    // groups, and grouping peers first (match + reduce per group) costs more
    // than it saves
    const uint32_t base = d[2];
    if (keep0) atomicAdd(&C.out[base + g0], (unsigned long long)x0);
    if (keep1) atomicAdd(&C.out[base + g1], (unsigned long long)x1);
  }
  if (lane == 0) C.ucnt[q] += kept;
  __syncwarp();
}

// The drain for query q: its compiled shape (fact-column sources only), or
// the generic one.  One out-of-line copy serves every call site.
__device__ __noinline__ void b_drain_any(const BCtx C, uint32_t q, const uint32_t *qe, uint32_t n) {
  switch (C.Qd[q * BQD_WORDS + 7] ? 0u : C.Qd[q * BQD_WORDS + 6]) {  // word 7: slots read through a foreign key
  case 1: b_drain_s<0>(C, q, qe, n); break;
  case 2: b_drain_s<1>(C, q, qe, n); break;
  case 3: b_drain_s<2>(C, q, qe, n); break;
  case 4: b_drain_s<3>(C, q, qe, n); break;
  case 5: b_drain_s<4>(C, q, qe, n); break;
  case 6: b_drain_s<5>(C, q, qe, n); break;
  case 7: b_drain_s<6>(C, q, qe, n); break;
  case 8: b_drain_s<7>(C, q, qe, n); break;
  default: b_drain(C, q, qe, n); break;
  }
}

// Posts the n (<= 64) rows at qe of query q as a job; false if every slot
// is taken (the caller drains them itself).  Warp-collective.
__device__ __forceinline__ bool job_post(const BCtx &C, uint32_t q, const uint32_t *qe, uint32_t n) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t slot = 0xffffffffu;
  for (uint32_t base = 0; base < BJ && slot == 0xffffffffu; base += 32) {
    const uint32_t st = *(volatile uint32_t *)&C.jobs[base + lane].state;
    uint32_t freem = __ballot_sync(0xffffffffu, st == JOB_FREE);
    if (lane == 0)
      while (freem) {
        const uint32_t j = base + __ffs(freem) - 1;
        freem &= freem - 1;
        if (atomicCAS(&C.jobs[j].state, JOB_FREE, JOB_FILL) == JOB_FREE) {
          slot = j;
          break;
        }
      }
    slot = __shfl_sync(0xffffffffu, slot, 0);
  }
  if (slot == 0xffffffffu) return false;
  Job &J = C.jobs[slot];
  if (lane < n) J.rows[lane] = qe[lane];
  if (lane + 32 < n) J.rows[lane + 32] = qe[lane + 32];
  if (lane == 0) J.q = q, J.n = n;
  __syncwarp();
  if (lane == 0) {
    __threadfence_block();
    atomicExch(&J.state, JOB_READY);
  }
  __syncwarp();
  return true;
}

__device__ __noinline__ void b_drain_any(const BCtx C, uint32_t q, const uint32_t *qe, uint32_t n);

// Runs one posted job, if there is one; returns whether it did.
// Warp-collective.
__device__ __forceinline__ bool job_run(const BCtx &C) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t slot = 0xffffffffu;
  for (uint32_t base = 0; base < BJ && slot == 0xffffffffu; base += 32) {
    const uint32_t st = *(volatile uint32_t *)&C.jobs[base + lane].state;
    uint32_t readym = __ballot_sync(0xffffffffu, st == JOB_READY);
    if (lane == 0) {
      while (readym) {
        const uint32_t j = base + __ffs(readym) - 1;
        readym &= readym - 1;
        if (atomicCAS(&C.jobs[j].state, JOB_READY, JOB_RUN) == JOB_READY) {
          slot = j;
          break;
        }
      }
      __threadfence_block();
    }
    slot = __shfl_sync(0xffffffffu, slot, 0);
  }
  __syncwarp();
  if (slot == 0xffffffffu) return false;
  Job &J = C.jobs[slot];
  b_drain_any(C, J.q, J.rows, J.n);
  __syncwarp();
  if (lane == 0) {
    __threadfence_block();
    atomicExch(&J.state, JOB_FREE);
  }
  __syncwarp();
  return true;
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
// lane*V + k of the stage): the conjunctive chain, then the selected rows
// into the query's queue; every 64 become a job.
template <int V>
__device__ __forceinline__ void b_query(const BCtx &C, const uint16_t *chain, const uint32_t *stage, uint64_t w0,
                                        uint64_t nwords, uint32_t tail, uint32_t q, uint32_t *queue,
                                        uint32_t *qlen) {
  constexpr uint32_t T = 32 * V;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t ch = C.Qd[q * BQD_WORDS + 4], c0 = ch & 0xffffu, nc = ch >> 16;
  // the chain: one entry per bin, stage row | edge | last of its conjunct |
  // conjunct negated (BCH_*); four entries per step, their loads issued
  // together
  uint32_t acc[V], unc[V], cm[V], cx[V];
#pragma unroll
  for (int k = 0; k < V; ++k) acc[k] = 0xffffffffu, unc[k] = 0, cm[k] = 0, cx[k] = 0;
  const uint32_t *sl = stage + lane * V;
  for (uint32_t i = 0; i < nc; i += 4) {
    uint32_t e[4], x[4][V];
#pragma unroll
    for (int j = 0; j < 4; ++j) e[j] = i + j < nc ? chain[c0 + i + j] : 0u;
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (i + j < nc) lds_words<V>(sl + (e[j] & BCH_ROW) * T, x[j]);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (i + j >= nc) break;
      if (e[j] & BCH_EDGE) {
#pragma unroll
        for (int k = 0; k < V; ++k) cx[k] |= x[j][k];
      } else {
#pragma unroll
        for (int k = 0; k < V; ++k) cm[k] |= x[j][k];
      }
      if (e[j] & BCH_LAST) {
        if (e[j] & BCH_NEG) {
#pragma unroll
          for (int k = 0; k < V; ++k) acc[k] &= ~(cm[k] | cx[k]);
        } else {
#pragma unroll
          for (int k = 0; k < V; ++k) acc[k] &= cm[k] | cx[k], unc[k] |= cx[k];
        }
#pragma unroll
        for (int k = 0; k < V; ++k) cm[k] = 0, cx[k] = 0;
      }
    }
  }
  uint32_t p[V], u[V], pc = 0;
  if (w0 + T <= nwords && (tail == 0 || w0 + T < nwords)) {  // an interior tile: no mask
#pragma unroll
    for (int k = 0; k < V; ++k) p[k] = acc[k], u[k] = unc[k] & acc[k], pc += __popc(p[k]);
  } else {
#pragma unroll
    for (int k = 0; k < V; ++k) {
      const uint64_t w = w0 + lane * V + k;
      uint32_t m = w < nwords ? 0xffffffffu : 0u;
      if (tail && w + 1 == nwords) m = (1u << tail) - 1u;
      p[k] = acc[k] & m;
      u[k] = unc[k] & p[k];
      pc += __popc(p[k]);
    }
  }
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t rowbase = (uint32_t)((w0 + lane * V) * 32);  // first row of the lane's words
  uint32_t qn = *qlen;
  // fast path: every selected row fits the queue at once (a prefix sum of
  // the lanes' counts places them)
  uint32_t incl = pc;
#pragma unroll
  for (int dd = 1; dd < 32; dd <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, dd);
    if (lane >= (uint32_t)dd) incl += y;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  if (qn + total <= BQQ) {
    uint32_t pos = qn + incl - pc;
#pragma unroll
    for (int k = 0; k < V; ++k) {
      uint32_t m = p[k];
      while (m) {
        const uint32_t b = __ffs(m) - 1;
        m &= m - 1;
        queue[pos++] = (rowbase + k * 32 + b) | (((u[k] >> b) & 1u) << 31);
      }
    }
    qn += total;
    __syncwarp();
    if (qn >= 64) {
      qn -= 64;
      if (!job_post(C, q, queue + qn, 64)) b_drain_any(C, q, queue + qn, 64);
    }
    if (lane == 0) *qlen = qn;
    return;
  }
  // otherwise one row per lane per round, draining every 64
  while (true) {
    bool has = false;
    uint32_t e = 0;
#pragma unroll
    for (int k = 0; k < V; ++k) {
      if (!has && p[k]) {
        const uint32_t b = __ffs(p[k]) - 1;
        p[k] &= p[k] - 1;
        has = true;
        e = (rowbase + k * 32 + b) | (((u[k] >> b) & 1u) << 31);
      }
    }
    const uint32_t bal = __ballot_sync(0xffffffffu, has);
    if (!bal) break;
    if (has) queue[qn + __popc(bal & lt)] = e;
    qn += __popc(bal);
    if (qn >= 64) {
      __syncwarp();
      qn -= 64;
      if (!job_post(C, q, queue + qn, 64)) b_drain_any(C, q, queue + qn, 64);
    }
  }
  __syncwarp();
  if (lane == 0) *qlen = qn;
}

template <int V>
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
  unsigned long long *usum = reinterpret_cast<unsigned long long *>(smem + L.off_sum);
  uint32_t *ucnt = reinterpret_cast<uint32_t *>(smem + L.off_cnt);
  uint32_t *qlen = reinterpret_cast<uint32_t *>(smem + L.off_len);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + L.off_bar);
  uint32_t *qctr = reinterpret_cast<uint32_t *>(smem + L.off_ctr), *issued = qctr + 2, *pdone = qctr + 3,
           *perr = qctr + 4, *cerr = qctr + 5;
  uint8_t *order = smem + L.off_order;
  uint16_t *chain = reinterpret_cast<uint16_t *>(smem + L.off_chain);
  uint32_t *qbuf = reinterpret_cast<uint32_t *>(smem + L.off_qbuf);
  Job *jobs = reinterpret_cast<Job *>(smem + L.off_jobs);
  uint32_t *stages = reinterpret_cast<uint32_t *>(smem + L.off_stage);
  const uint32_t np = P.np;  // warps 0 .. np-1 produce, the others consume

  for (uint32_t i = tid; i < P.nq * BQD_WORDS; i += blockDim.x) Qd[i] = H->Qd[i];
  for (uint32_t i = tid; i < BJ; i += blockDim.x) jobs[i].state = JOB_FREE;
  for (uint32_t i = tid; i < nw * P.nq; i += blockDim.x) usum[i] = 0, ucnt[i] = 0;
  for (uint32_t i = tid; i < P.nchain; i += blockDim.x) chain[i] = H->chain[i];
  for (uint32_t i = tid; i < P.nq; i += blockDim.x) order[i] = H->order[i];
  for (uint32_t i = tid; i < P.nq; i += blockDim.x) qlen[i] = 0;
  if (tid < BS_MAX) {
    scol[tid] = reinterpret_cast<unsigned long long>(H->src[tid].col);
    sfk[tid] = reinterpret_cast<unsigned long long>(H->src[tid].fk);
    sdim[tid] = H->src[tid].dimsz;
    swid[tid] = H->src[tid].width;
  }
  if (tid < 6) qctr[tid] = 0;
  if (tid == 0) {
    for (uint32_t s = 0; s < P.S; ++s) mbar_init(&full[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  BCtx C;
  C.Qd = Qd;
  C.scol = scol;
  C.sfk = sfk;
  C.sdim = sdim;
  C.out = out;
  C.usum = usum + (size_t)warp * P.nq;
  C.ucnt = ucnt + (size_t)warp * P.nq;
  C.jobs = jobs;

  const uint64_t ntiles = (P.nwords + T - 1) / T;
  const uint64_t nit = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  // stage j % S <- the CTA's j-th tile: the tensor copies of the staged
  // rows x T words (copy c by lane 0 of producer warp c % np; thread 0 sets
  // the stage's byte count, and a copy landing before that only takes the
  // count below zero for a while), zeros past the table's end; the payload
  // rows of the tile into L2 (threads < nsrc).  Called by every producer.
  auto fill = [&](uint64_t j) {
    const uint32_t s = (uint32_t)(j % P.S);
    const uint64_t w0 = ((uint64_t)blockIdx.x + j * gridDim.x) * T;
    if (lane == 0) {
      if (warp == 0) {
        ++*issued;
        mbar_arrive_expect_tx(&full[s], P.nu * T * 4);
      }
      fence_proxy_async_smem();
      uint32_t *dst = stages + (size_t)s * P.nu * T;
      for (uint32_t c = warp; c < P.ncopy; c += np) {
        const uint32_t e = P.copy[c];
        tma_load_2d(dst + ((e >> 12) & 0xfffu) * T, maps + (e >> 24), (int)w0, (int)(e & 0xfffu), &full[s]);
      }
    }
    if (tid < P.nsrc && ((P.pf_mask >> tid) & 1u)) {
      const uint64_t r0 = w0 * 32;
      if (r0 < P.nrows) {
        const uint64_t nr = P.nrows - r0 < T * 32 ? P.nrows - r0 : T * 32;
        const bool viafk = sfk[tid] != 0;
        const uint32_t w = viafk ? 4u : swid[tid];
        const uint8_t *base = reinterpret_cast<const uint8_t *>(viafk ? sfk[tid] : scol[tid]) + r0 * w;
        const uint32_t pb = (uint32_t)(nr * w) & ~15u;
        if (pb) prefetch_l2(base, pb);
      }
    }
  };
  auto pbar = [&]() { asm volatile("bar.sync 1, %0;" ::"r"(np * 32) : "memory"); };  // producers only

  if (warp < np) {
    // ---------------------------------------------------------- producers
    for (uint64_t j = 0; j < P.S && j < nit; ++j) fill(j);
    const uint32_t tail = (uint32_t)(P.nrows & 31u);
    for (uint64_t it = 0; it < nit; ++it) {
      const uint32_t s = (uint32_t)(it % P.S), par = (uint32_t)((it / P.S) & 1u), b = (uint32_t)(it & 1u);
      if (!mbar_wait_bounded(&full[s], par, errw, MB_DEVERR_TMA_WAIT)) atomicOr(perr, 1u);
      pbar();
      if (*(volatile uint32_t *)perr) break;
      if (tid == 0) qctr[b ^ 1u] = 0;  // last used on the previous tile; next used after this tile's barrier
      const uint64_t w0 = ((uint64_t)blockIdx.x + it * gridDim.x) * T;
      const uint32_t *st = stages + (size_t)s * P.nu * T;
      while (true) {
        uint32_t qi = 0;
        if (lane == 0) qi = atomicAdd(&qctr[b], 1u);
        qi = __shfl_sync(0xffffffffu, qi, 0);
        if (qi >= P.nq) break;
        const uint32_t q = order[qi];
        b_query<V>(C, chain, st, w0, P.nwords, tail, q, qbuf + (size_t)q * BQQ, &qlen[q]);
      }
      pbar();  // the stage is consumed: refill it
      if (it + P.S < nit) fill(it + P.S);
    }
    if (*(volatile uint32_t *)perr) {
      // a wait ran out: let the copies still in flight land before exiting
      if (tid == 0)
        for (uint32_t j = *issued > P.S ? *issued - P.S : 0; j < *issued; ++j)
          mbar_wait_bounded(&full[j % P.S], (j / P.S) & 1u, nullptr, 0, 1u << 16);
    } else {
      // every query's last rows become jobs
      for (uint32_t q = warp; q < P.nq; q += np) {
        const uint32_t n = qlen[q];
        if (n && !job_post(C, q, qbuf + (size_t)q * BQQ, n)) b_drain_any(C, q, qbuf + (size_t)q * BQQ, n);
      }
    }
    __syncwarp();
    if (lane == 0) {
      __threadfence_block();
      atomicAdd(pdone, 1u);
    }
  } else {
    // ---------------------------------------------------------- consumers
    uint32_t idle = 0;
    while (true) {
      if (job_run(C)) {
        idle = 0;
        continue;
      }
      if (*(volatile uint32_t *)pdone == np) {
        __threadfence_block();
        if (!job_run(C)) break;  // nothing posted after the last producer finished
        continue;
      }
      if (++idle >= CONSUMER_IDLE_TRIES) {
        if (lane == 0) {
          atomicOr(cerr, 1u);
          if (atomicCAS(errw, 0u, 1u) == 0u) {
            errw[1] = MB_DEVERR_IDLE_WAIT;
            errw[2] = blockIdx.x;
          }
        }
        break;
      }
      __nanosleep(128);
    }
  }
  __syncthreads();
  if (*(volatile uint32_t *)perr || *(volatile uint32_t *)cerr) return;
  for (uint32_t q = tid; q < P.nq; q += blockDim.x) {
    unsigned long long sum = 0, cnt = 0;
    for (uint32_t w = 0; w < nw; ++w) sum += usum[w * P.nq + q], cnt += ucnt[w * P.nq + q];
    if (sum) atomicAdd(&out[Qd[q * BQD_WORDS + 2]], sum);
    if (cnt) atomicAdd(&nqual[Qd[q * BQD_WORDS + 3]], cnt);
  }
}

}  // namespace

size_t batch_smem(const BatchHdr &h, const BatchCfg &c) {
  if (c.V != 1 && c.V != 2 && c.V != 4 && c.V != 6) return 0;
  if (c.warps < 2 || c.warps > BW_MAX || c.stages == 0 || c.stages > 4 || c.drainers == 0 || c.drainers >= c.warps)
    return 0;
  return blayout(h.nq, h.nchain, h.nu, c.warps, c.stages, 32 * c.V).total;
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
  auto kern = batch_scan_kernel<V>;
  BParams P;
  P.nrows = h.nrows;
  P.nwords = h.nwords;
  P.nq = h.nq;
  P.nu = h.nu;
  P.ncopy = h.ncopy;
  memcpy(P.copy, h.copy, sizeof(P.copy));
  P.nsrc = h.nsrc;
  P.nchain = h.nchain;
  P.pf_mask = h.pf_mask;
  P.S = c.stages;
  P.np = c.warps - c.drainers;
  P.L = blayout(h.nq, h.nchain, h.nu, c.warps, c.stages, 32 * V);
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
  kern<<<(unsigned)grid, c.warps * 32, smem, st>>>(dh, P, static_cast<const CUtensorMap *>(maps), reinterpret_cast<unsigned long long *>(out),
                                                   reinterpret_cast<unsigned long long *>(nqual), errw);
  MB_LAUNCH_CHECK("batch_scan_kernel");
  return MB_OK;
}

mb_status batch_scan(const BatchHdr &h, const BatchHdr *dh, const BatchCfg &c, const void *maps, int64_t *out,
                     uint64_t *nqual, cudaStream_t st) {
  if (h.nq == 0 || h.nrows == 0) return MB_OK;
  if (h.nq > BQ_MAX || h.nu > BU_MAX || h.nsrc > BS_MAX || h.nchain > BC_MAX)
    return fail(MB_ERR_INVALID, "batch: descriptor over its limits");
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
