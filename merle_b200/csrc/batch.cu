// batch.cu - the batched scan kernel (see batch.cuh for the design).
//
// Reference: the per-query fused kernel vprg_grpby (primitive.cuh:340-445)
// and its op functors (ssb/lambdas.cuh:19-152) define what each query of a
// batch computes; the batch evaluates the same programs with the same
// candidate-check semantics, so every query's groups and row count equal what
// it gets alone.
//
// A CTA walks its row tiles (T = 32 * V words); per tile, with S stages of
// the union bitmaps in flight:
//   phase A  warps take the batch's queries off a counter (costliest first),
//            evaluate each query's conjunctive chain on the staged words and
//            append its selected rows - entry = row in tile << 8 | uncertain
//            << 7 | query - to one tile-wide row list in shared memory, each
//            query's rows reserved as one contiguous run;
//   barrier  the stage is consumed: its refill with tile j + S starts (every
//            thread issues its share of 16-byte cp.async copies, completing
//            on the stage's mbarrier), plus an L2 prefetch of the tile's
//            payload rows;
//   phase B  warps take 64-entry chunks of the row list and run the ops, two
//            rows per lane, each lane reading its own row's query descriptor
//            (a chunk spans few queries, so most reads are broadcasts); the
//            payload rows of the tile were prefetched into L2, and every
//            query of the batch gathers from the same lines;
//   barrier  the list is consumed.
// 1-group sums and row counts accumulate per warp (plain adds by one leader
// lane per query, no shared-memory atomics) and are folded at the end.  A
// query whose rows do not fit the list (a dense query on a full list) runs
// them through the warp's own 64-row queue instead.  Every wait is bounded: a
// stage that does not arrive records the block in the device error word, and
// the block stops walking and waits for its own copies before exiting.
#include <string.h>
#include "batch.cuh"
#include "opeval.cuh"
#include "tma.cuh"
#include "vbp.cuh"

namespace mb {

namespace {

constexpr uint32_t BT_THREADS_MAX = BW_MAX * 32;
constexpr uint32_t BL_CAP = 4096;  // entries of the tile row list
constexpr uint32_t BWQ = 96;       // a warp's own queue: < 64 pending + one 32-entry round

// Shared-memory layout of one launch (identical on host and device).
struct BLayout {
  uint32_t nqs;  // query stride of the per-warp accumulators
  uint32_t off_Q, off_src, off_ubmp, off_sum, off_cnt, off_bar, off_ctr, off_order, off_chain, off_list, off_wq,
      off_stage, total;
};

__host__ __device__ inline uint32_t align_up(uint32_t x, uint32_t a) { return (x + a - 1) / a * a; }

__host__ __device__ inline BLayout blayout(uint32_t nq, uint32_t nchain, uint32_t nu, uint32_t warps, uint32_t S,
                                           uint32_t T) {
  BLayout L;
  uint32_t o = 0;
  L.nqs = align_up(nq, 2);
  L.off_Q = o;
  o += nq * BQD_WORDS * 4;
  L.off_src = o = align_up(o, 16);
  o += BS_MAX * 24;  // col[] and fk[] (8 bytes), dimsz[] and width[] (4 bytes)
  L.off_ubmp = o;
  o += nu * 8;
  L.off_sum = o = align_up(o, 16);
  o += warps * L.nqs * 8;  // per warp and query: 1-group sum
  L.off_cnt = o;
  o += warps * L.nqs * 4;  // per warp and query: kept rows
  L.off_bar = o = align_up(o, 8);
  o += 8 * S;
  L.off_ctr = o;
  o += 4 * 8;  // qctr[2], lcnt[2], cctr[2]
  L.off_order = o;
  o += nq;
  L.off_chain = o = align_up(o, 16);
  o += align_up(nchain * 2, 16);
  L.off_list = o;
  o += BL_CAP * 4;
  L.off_wq = o;
  o += warps * BWQ * 4;
  L.off_stage = o = align_up(o, 128);
  o += S * nu * T * 4;
  L.total = o;
  return L;
}

struct BParams {
  uint64_t nrows, nwords, stride;
  uint32_t nq, nu, nsrc, nchain, pf_mask, S;
  BLayout L;
};

// The batch's tables as a warp sees them (shared memory).
struct BCtx {
  const uint32_t *Qd;
  const unsigned long long *scol, *sfk;
  const uint32_t *sdim;
  unsigned long long *out;
  unsigned long long *wsum;  // this warp's 1-group sums, per query
  uint32_t *wcnt;            // this warp's kept rows, per query
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

// One row's share of the op: everything per lane (the row's own query).
struct BRow {
  bool ok, chk;
  uint32_t q, row;
  const uint32_t *d;
};

// Runs the ops of the first n (<= 64) entries of ents, two rows per lane;
// each lane reads its own row's query descriptor.  Accumulates 1-group sums
// and kept rows into the warp's own slots (plain adds by one leader lane per
// query), group sums by warp-aggregated global atomics.  All 32 lanes call it.
__device__ __forceinline__ void b_drain(const BCtx &C, const uint32_t *ents, uint32_t n, uint32_t row0) {
  const uint32_t lane = threadIdx.x & 31;
  BRow R[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t i = lane + 32 * h;
    R[h].ok = i < n;
    const uint32_t e = R[h].ok ? ents[i] : 0u;
    R[h].q = e & 0x7fu;
    R[h].chk = R[h].ok && ((e >> 7) & 1u);
    R[h].row = row0 + (e >> 8);
    R[h].d = C.Qd + R[h].q * BQD_WORDS;
  }
  // loads: foreign keys, then values, of every slot of both rows
  uint32_t key[2][BSLOT], v[2][BSLOT], bad[2] = {0, 0};
  bool ld[2][BSLOT];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t h0 = R[h].d[0], roles = R[h].d[5];
    const uint32_t nslot = h0 & 0xffu, kv = roles & 0xffu, filt = (roles >> 8) & 0xffu;
#pragma unroll
    for (uint32_t s = 0; s < BSLOT; ++s) {
      key[h][s] = R[h].row;
      ld[h][s] = R[h].ok && s < nslot && (((kv >> s) & 1u) || (R[h].chk && ((filt >> s) & 1u)));
      if (ld[h][s]) {
        const uint32_t t = R[h].d[BQD_SLOT0 + BQD_SLOTW * s] & 0xffu;
        const uint32_t *fk = reinterpret_cast<const uint32_t *>(C.sfk[t]);
        if (fk) key[h][s] = __ldg(fk + R[h].row);
      }
    }
  }
#pragma unroll
  for (int h = 0; h < 2; ++h) {
#pragma unroll
    for (uint32_t s = 0; s < BSLOT; ++s) {
      v[h][s] = 0;
      if (ld[h][s]) {
        const uint32_t a = R[h].d[BQD_SLOT0 + BQD_SLOTW * s], t = a & 0xffu, w = (a >> 8) & 0xffu;
        const uint32_t dz = C.sdim[t];
        if (C.sfk[t] && dz && key[h][s] >= dz) bad[h] |= 1u << s;
        else v[h][s] = b_ldw(reinterpret_cast<const void *>(C.scol[t]), key[h][s], w);
      }
    }
  }
  bool keep[2], scal[2];
  uint32_t slot[2];
  uint64_t val[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t *d = R[h].d;
    const uint32_t h0 = d[0], roles = d[5];
    const uint32_t keym = (roles >> 16) & 0xffu, termm = roles >> 24;
    bool kp = R[h].ok;
    // candidate check of an uncertain row: the single-term clauses, bounds
    // intersected per slot
    if (R[h].chk) {
#pragma unroll
      for (uint32_t s = 0; s < BSLOT; ++s)
        if ((termm >> s) & 1u) {
          const uint32_t lo = d[BQD_SLOT0 + BQD_SLOTW * s + 1], hi = d[BQD_SLOT0 + BQD_SLOTW * s + 2];
          kp = kp && !((bad[h] >> s) & 1u) && v[h][s] >= lo && v[h][s] <= hi;
        }
    }
    // group key: sum over key slots of mul * (xform(value) - base); the
    // transforms are computed branch-free and selected
    uint32_t g = 0;
#pragma unroll
    for (uint32_t s = 0; s < BSLOT; ++s)
      if ((keym >> s) & 1u) {
        const uint32_t *sl = d + BQD_SLOT0 + BQD_SLOTW * s;
        const uint32_t a = sl[0], xf = (a >> 16) & 0xffu, x = v[h][s];
        kp = kp && !((bad[h] >> s) & 1u);
        const uint32_t xd = div_by_magic(x, sl[3], (a >> 24) & 15u, a >> 28), xy = date_to_year(x);
        const uint32_t xx = xf == MB_X_DIV ? xd : (xf == MB_X_YEAR ? xy : x);
        g += sl[5] * (xx - sl[4]);
      }
    kp = kp && g < d[1];
    const uint32_t vkind = (h0 >> 16) & 15u, va = (h0 >> 20) & 15u, vb = (h0 >> 24) & 15u;
    uint64_t x = 1;
    if (vkind != MB_V_ONE) {
      uint64_t av = 0, bv = 0;
#pragma unroll
      for (uint32_t s = 0; s < BSLOT; ++s) {
        if (s == va) av = v[h][s];
        if (s == vb) bv = v[h][s];
      }
      kp = kp && !((bad[h] >> va) & 1u);
      if (vkind == MB_V_COL) {
        x = av;
      } else {
        kp = kp && !((bad[h] >> vb) & 1u);
        x = vkind == MB_V_MUL ? av * bv : (uint64_t)((int64_t)av - (int64_t)bv);
      }
    }
    keep[h] = kp;
    val[h] = x;
    scal[h] = (h0 >> 8) & 1u;
    slot[h] = d[2] + g;
  }
  // aggregation: peers share a 1-group query (summed into the warp's slot)
  // or an output slot (global atomics); rows are counted per query
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    if (h == 1 && n <= 32) break;
    const uint32_t key2 = keep[h] ? (scal[h] ? (0x80000000u | R[h].q) : slot[h]) : 0xffffffffu;
    const uint32_t peers = __match_any_sync(0xffffffffu, key2);
    if (keep[h]) {
      const uint64_t s = peer_sum64(peers, val[h]);
      if (lane == (uint32_t)(__ffs(peers) - 1)) {
        if (scal[h]) C.wsum[R[h].q] += s;
        else atomicAdd(&C.out[slot[h]], (unsigned long long)s);
      }
    }
    const uint32_t qpeers = __match_any_sync(0xffffffffu, keep[h] ? R[h].q : 0xffffffffu);
    if (keep[h] && lane == (uint32_t)(__ffs(qpeers) - 1)) C.wcnt[R[h].q] += __popc(qpeers);
    __syncwarp();
  }
}

template <int V>
__device__ __forceinline__ void lds_words(const uint32_t *p, uint32_t (&x)[V]) {
  if (V == 4) {
    const uint4 t = *reinterpret_cast<const uint4 *>(p);
    x[0] = t.x, x[1] = t.y, x[2] = t.z, x[3] = t.w;
  } else if (V == 2) {
    const uint2 t = *reinterpret_cast<const uint2 *>(p);
    x[0] = t.x, x[1] = t.y;
  } else {
    x[0] = p[0];
  }
}

// Phase A for query q on the staged tile (words w0 + lane*V + k of the
// table; word lane*V + k of the stage): the conjunctive chain, then the
// selected rows appended to the tile list (or, if they do not fit, run
// through the warp's own queue).
template <int V>
__device__ __forceinline__ void b_query(const BCtx &C, const uint16_t *chain, const uint32_t *stage, uint64_t w0,
                                        uint64_t nwords, uint32_t tail, uint32_t q, uint32_t *list, uint32_t *lcnt,
                                        uint32_t *wq) {
  constexpr uint32_t T = 32 * V;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t ch = C.Qd[q * BQD_WORDS + 4], c0 = ch & 0xffffu, nc = ch >> 16;
  uint32_t acc[V], cur[V], ce[V], unc[V];
#pragma unroll
  for (int k = 0; k < V; ++k) acc[k] = 0xffffffffu, cur[k] = ce[k] = unc[k] = 0;
  const uint32_t *sl = stage + lane * V;
  for (uint32_t i = 0; i < nc; ++i) {
    const uint32_t e = chain[c0 + i];
    uint32_t x[V];
    lds_words<V>(sl + (e & 0xffu) * T, x);
    const uint32_t em = (e & (CNF_EDGE << 8)) ? 0xffffffffu : 0u;
#pragma unroll
    for (int k = 0; k < V; ++k) {
      cur[k] |= x[k];
      ce[k] |= x[k] & em;
    }
    if (e & (CNF_END << 8)) {
      const bool neg = (e & (CNF_NEG << 8)) != 0;
#pragma unroll
      for (int k = 0; k < V; ++k) {
        acc[k] &= neg ? ~cur[k] : cur[k];
        if (!neg) unc[k] |= ce[k];
        cur[k] = ce[k] = 0;
      }
    }
  }
  uint32_t p[V], u[V], pc = 0;
#pragma unroll
  for (int k = 0; k < V; ++k) {
    const uint64_t w = w0 + lane * V + k;
    uint32_t m = w < nwords ? 0xffffffffu : 0u;
    if (tail && w + 1 == nwords) m = (1u << tail) - 1u;
    p[k] = acc[k] & m;
    u[k] = unc[k] & p[k];
    pc += __popc(p[k]);
  }
  // exclusive prefix of the lanes' row counts
  uint32_t incl = pc;
#pragma unroll
  for (int dd = 1; dd < 32; dd <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, dd);
    if (lane >= (uint32_t)dd) incl += y;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  if (total == 0) return;
  uint32_t base = 0;
  if (lane == 0) {
    // a reservation that would pass the end is taken back; while it is out,
    // every other reservation fails too, so the granted runs stay contiguous
    base = atomicAdd(lcnt, total);
    if (base + total > BL_CAP) {
      atomicSub(lcnt, total);
      base = 0xffffffffu;
    }
  }
  base = __shfl_sync(0xffffffffu, base, 0);
  const uint32_t lrow = lane * V * 32;  // first row of the lane's words within the tile
  if (base != 0xffffffffu) {
    uint32_t pos = base + incl - pc;
#pragma unroll
    for (int k = 0; k < V; ++k) {
      uint32_t m = p[k];
      while (m) {
        const uint32_t b = __ffs(m) - 1;
        m &= m - 1;
        list[pos++] = ((lrow + k * 32 + b) << 8) | (((u[k] >> b) & 1u) << 7) | q;
      }
    }
    return;
  }
  // the list is full: the rows through the warp's queue, one per lane per round
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t row0 = (uint32_t)(w0 * 32);
  uint32_t qn = 0;
  while (true) {
    bool has = false;
    uint32_t e = 0;
#pragma unroll
    for (int k = 0; k < V; ++k) {
      if (!has && p[k]) {
        const uint32_t b = __ffs(p[k]) - 1;
        p[k] &= p[k] - 1;
        has = true;
        e = ((lrow + k * 32 + b) << 8) | (((u[k] >> b) & 1u) << 7) | q;
      }
    }
    const uint32_t bal = __ballot_sync(0xffffffffu, has);
    if (!bal) break;
    if (has) wq[qn + __popc(bal & lt)] = e;
    qn += __popc(bal);
    if (qn >= 64) {
      __syncwarp();
      qn -= 64;
      b_drain(C, wq + qn, 64, row0);
      __syncwarp();
    }
  }
  __syncwarp();
  if (qn) b_drain(C, wq, qn, row0);
  __syncwarp();
}

template <int V>
__global__ void __launch_bounds__(BT_THREADS_MAX)
batch_scan_kernel(const BatchHdr *__restrict__ H, const __grid_constant__ BParams P, unsigned long long *__restrict__ out,
                  unsigned long long *__restrict__ nqual, uint32_t *errw) {
  constexpr uint32_t T = 32 * V;
  extern __shared__ __align__(128) uint8_t smem[];
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  const BLayout &L = P.L;
  uint32_t *Qd = reinterpret_cast<uint32_t *>(smem + L.off_Q);
  unsigned long long *scol = reinterpret_cast<unsigned long long *>(smem + L.off_src);
  unsigned long long *sfk = scol + BS_MAX;
  uint32_t *sdim = reinterpret_cast<uint32_t *>(sfk + BS_MAX), *swid = sdim + BS_MAX;
  const uint32_t **ubmp = reinterpret_cast<const uint32_t **>(smem + L.off_ubmp);
  unsigned long long *usum = reinterpret_cast<unsigned long long *>(smem + L.off_sum);  // [warp][nqs]
  uint32_t *ucnt = reinterpret_cast<uint32_t *>(smem + L.off_cnt);                      // [warp][nqs]
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + L.off_bar);
  uint32_t *qctr = reinterpret_cast<uint32_t *>(smem + L.off_ctr), *lcnt = qctr + 2, *cctr = qctr + 4;
  uint8_t *order = smem + L.off_order;
  uint16_t *chain = reinterpret_cast<uint16_t *>(smem + L.off_chain);
  uint32_t *list = reinterpret_cast<uint32_t *>(smem + L.off_list);
  uint32_t *wq = reinterpret_cast<uint32_t *>(smem + L.off_wq) + (size_t)warp * BWQ;
  uint32_t *stages = reinterpret_cast<uint32_t *>(smem + L.off_stage);

  for (uint32_t i = tid; i < P.nq * BQD_WORDS; i += blockDim.x) Qd[i] = H->Qd[i];
  for (uint32_t i = tid; i < P.nchain; i += blockDim.x) chain[i] = H->chain[i];
  for (uint32_t i = tid; i < P.nu; i += blockDim.x) ubmp[i] = H->ubmp[i];
  for (uint32_t i = tid; i < P.nq; i += blockDim.x) order[i] = H->order[i];
  for (uint32_t i = tid; i < nw * L.nqs; i += blockDim.x) usum[i] = 0, ucnt[i] = 0;
  if (tid < BS_MAX) {
    scol[tid] = reinterpret_cast<unsigned long long>(H->src[tid].col);
    sfk[tid] = reinterpret_cast<unsigned long long>(H->src[tid].fk);
    sdim[tid] = H->src[tid].dimsz;
    swid[tid] = H->src[tid].width;
  }
  if (tid < 6) qctr[tid] = 0;
  if (tid == 0) {
    for (uint32_t s = 0; s < P.S; ++s) mbar_init(&full[s], blockDim.x);
    fence_mbar_init();
  }
  __syncthreads();

  BCtx C;
  C.Qd = Qd;
  C.scol = scol;
  C.sfk = sfk;
  C.sdim = sdim;
  C.out = out;
  C.wsum = usum + (size_t)warp * L.nqs;
  C.wcnt = ucnt + (size_t)warp * L.nqs;

  const uint64_t ntiles = (P.nwords + T - 1) / T;
  const uint64_t nit = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  // block-collective: stage j % S <- the CTA's j-th tile; every thread's
  // copies complete one arrival on full[j % S]
  auto fill = [&](uint64_t j) {
    const uint32_t s = (uint32_t)(j % P.S);
    const uint64_t w0 = ((uint64_t)blockIdx.x + j * gridDim.x) * T;
    const uint64_t avail = P.stride - w0;  // a multiple of 32 words
    const uint32_t cpb = (uint32_t)(avail < T ? avail : T) / 4;  // 16-byte chunks per bitmap
    uint32_t *st = stages + (size_t)s * P.nu * T;
    const uint32_t total = P.nu * cpb;
    for (uint32_t i = tid; i < total; i += blockDim.x) {
      const uint32_t u = i / cpb, c = i - u * cpb;
      cp_async16(st + u * T + c * 4, ubmp[u] + w0 + c * 4);
    }
    cp_async_mbar_arrive(&full[s]);
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
  for (uint64_t j = 0; j < P.S && j < nit; ++j) fill(j);

  bool err = false;
  const uint32_t tail = (uint32_t)(P.nrows & 31u);
  for (uint64_t it = 0; it < nit; ++it) {
    const uint32_t s = (uint32_t)(it % P.S), par = (uint32_t)((it / P.S) & 1u), b = (uint32_t)(it & 1u);
    const bool ok = mbar_wait_bounded(&full[s], par, errw, MB_DEVERR_TMA_WAIT);
    if (!__syncthreads_and(ok ? 1 : 0)) {
      err = true;
      break;
    }
    if (tid == 0) cctr[b] = 0;  // last used two tiles ago; next used after the barrier below
    const uint64_t w0 = ((uint64_t)blockIdx.x + it * gridDim.x) * T;
    const uint32_t *st = stages + (size_t)s * P.nu * T;
    // phase A: the queries' chains into the tile row list
    while (true) {
      uint32_t qi = 0;
      if (lane == 0) qi = atomicAdd(&qctr[b], 1u);
      qi = __shfl_sync(0xffffffffu, qi, 0);
      if (qi >= P.nq) break;
      b_query<V>(C, chain, st, w0, P.nwords, tail, order[qi], list, &lcnt[b], wq);
    }
    __syncthreads();
    // the stage is consumed: refill it; then the next tile's counters
    if (it + P.S < nit) fill(it + P.S);
    const uint32_t n = lcnt[b];
    __syncthreads();  // every thread has read n before the next tile's counters are reset
    if (tid == 0) qctr[b ^ 1u] = 0, lcnt[b ^ 1u] = 0;
    // phase B: the ops over 64-entry chunks of the list
    const uint32_t nch = (n + 63) / 64;
    const uint32_t row0 = (uint32_t)(w0 * 32);
    while (true) {
      uint32_t c = 0;
      if (lane == 0) c = atomicAdd(&cctr[b], 1u);
      c = __shfl_sync(0xffffffffu, c, 0);
      if (c >= nch) break;
      b_drain(C, list + 64 * c, n - 64 * c < 64 ? n - 64 * c : 64, row0);
    }
    __syncthreads();  // the list is consumed
  }
  if (err) {
    cp_async_wait_all();  // copies this thread issued land before the block exits
    __syncthreads();
    return;
  }
  __syncthreads();
  for (uint32_t q = tid; q < P.nq; q += blockDim.x) {
    unsigned long long sum = 0, cnt = 0;
    for (uint32_t w = 0; w < nw; ++w) sum += usum[w * L.nqs + q], cnt += ucnt[w * L.nqs + q];
    if (sum) atomicAdd(&out[Qd[q * BQD_WORDS + 2]], sum);
    if (cnt) atomicAdd(&nqual[Qd[q * BQD_WORDS + 3]], cnt);
  }
}

}  // namespace

size_t batch_smem(const BatchHdr &h, const BatchCfg &c) {
  if (c.V != 1 && c.V != 2 && c.V != 4) return 0;
  if (c.warps == 0 || c.warps > BW_MAX || c.stages == 0 || c.stages > 4) return 0;
  return blayout(h.nq, h.nchain, h.nu, c.warps, c.stages, 32 * c.V).total;
}

template <int V>
static mb_status launch_bs(const BatchHdr &h, const BatchHdr *dh, const BatchCfg &c, int64_t *out, uint64_t *nqual,
                           cudaStream_t st) {
  auto kern = batch_scan_kernel<V>;
  BParams P;
  P.nrows = h.nrows;
  P.nwords = h.nwords;
  P.stride = h.stride;
  P.nq = h.nq;
  P.nu = h.nu;
  P.nsrc = h.nsrc;
  P.nchain = h.nchain;
  P.pf_mask = h.pf_mask;
  P.S = c.stages;
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
  kern<<<(unsigned)grid, c.warps * 32, smem, st>>>(dh, P, reinterpret_cast<unsigned long long *>(out),
                                                   reinterpret_cast<unsigned long long *>(nqual), errw);
  MB_LAUNCH_CHECK("batch_scan_kernel");
  return MB_OK;
}

mb_status batch_scan(const BatchHdr &h, const BatchHdr *dh, const BatchCfg &c, int64_t *out, uint64_t *nqual,
                     cudaStream_t st) {
  if (h.nq == 0 || h.nrows == 0) return MB_OK;
  if (h.nq > BQ_MAX || h.nu > BU_MAX || h.nsrc > BS_MAX || h.nchain > BC_MAX)
    return fail(MB_ERR_INVALID, "batch: descriptor over its limits");
  if (h.stride % 32 != 0 || h.stride < h.nwords) return fail(MB_ERR_INVALID, "batch: bitmap stride %llu",
                                                              (unsigned long long)h.stride);
  if (batch_smem(h, c) == 0) return fail(MB_ERR_INVALID, "batch: launch shape V=%u warps=%u stages=%u", c.V,
                                         c.warps, c.stages);
  switch (c.V) {
  case 4: return launch_bs<4>(h, dh, c, out, nqual, st);
  case 2: return launch_bs<2>(h, dh, c, out, nqual, st);
  default: return launch_bs<1>(h, dh, c, out, nqual, st);
  }
}

}  // namespace mb
