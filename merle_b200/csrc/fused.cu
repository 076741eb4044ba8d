// fused.cu - the TMA-staged fused kernel: program -> compaction -> op ->
// group-by, with every operand bitmap of a tile staged in shared memory.
//
// Reference: vprg_grpby (primitive.cuh:340-445).  The reference reads each
// operand word with a dependent chain of __ldcs loads per thread; here one
// thread per CTA streams the tile of EVERY bitmap of the program into shared
// memory with 1-D TMA bulk copies (cp.async.bulk, mbarrier completion, two
// stages), so HBM reads run ahead of the compute without occupying warps:
//
//   stage s ready -> phase A: all warps evaluate the program from shared
//   memory into a per-CTA result tile -> __syncthreads -> thread 0 refills
//   stage s with the tile after next -> phase B: each warp compacts 32-word
//   chunks of the result tile into its own row queue, while the other stage
//   streams in.
//
// A warp runs the op only on full 64-row batches of its queue (two rows per
// lane), carrying fewer than 64 rows over to the next chunk or tile, so lanes
// stay busy at any selectivity; sums commute, so the queue is drained from
// its end.  The op's sources are loaded for both rows at once, foreign keys
// first and then every column / dimension value, keeping several independent
// gathers in flight per lane; filter-only sources are read only for uncertain
// rows (chk), as the reference's functors do.
//
// Bounded waits: every mbarrier wait gives up after 2^20 tries, records the
// block in the device error word and leaves the loop block-uniformly.
#include <string.h>
#include "common.cuh"
#include "opeval.cuh"
#include "tma.cuh"
#include "vbp.cuh"

namespace mb {

constexpr uint32_t FT_THREADS = 256;
constexpr uint32_t FT_WARPS = FT_THREADS / 32;

OpNeeds op_needs(const mb_op &O) {
  OpNeeds n{0, 0};
  for (uint32_t k = 0; k < O.nkey; ++k) n.kv_mask |= 1u << O.keys[k].src;
  if (O.vkind != MB_V_ONE) n.kv_mask |= 1u << O.va;
  if (O.vkind == MB_V_MUL || O.vkind == MB_V_SUB) n.kv_mask |= 1u << O.vb;
  uint32_t nt = 0;
  for (uint32_t c = 0; c < O.nclause; ++c) nt += O.clause_len[c];
  for (uint32_t t = 0; t < nt; ++t) n.filt_mask |= 1u << O.terms[t].src;
  return n;
}

__device__ __forceinline__ uint32_t ld_w32(const void *p, uint64_t i, uint32_t w) {
  switch (w) {
  case 1: return __ldg(reinterpret_cast<const uint8_t *>(p) + i);
  case 2: return __ldg(reinterpret_cast<const uint16_t *>(p) + i);
  default: return __ldg(reinterpret_cast<const uint32_t *>(p) + i);
  }
}

// v[s] for a warp-uniform runtime s without dynamic register indexing.
__device__ __forceinline__ uint32_t pick(const uint32_t (&v)[MB_MAXSRC], uint32_t s) {
  uint32_t r = v[0];
#pragma unroll
  for (uint32_t i = 1; i < MB_MAXSRC; ++i) r = (s == i) ? v[i] : r;
  return r;
}

// Loads every needed source of one row: foreign keys first, then values.
// bad: bit s set if source s's key is out of its dimension.
__device__ __forceinline__ void load_row(const mb_op &O, uint32_t need, uint32_t row, uint32_t (&v)[MB_MAXSRC],
                                         uint32_t &bad) {
  uint32_t key[MB_MAXSRC];
#pragma unroll
  for (uint32_t s = 0; s < MB_MAXSRC; ++s) {
    key[s] = row;
    if (s < O.nsrc && ((need >> s) & 1u) && O.src[s].fk) key[s] = __ldg(O.src[s].fk + row);
  }
  bad = 0;
#pragma unroll
  for (uint32_t s = 0; s < MB_MAXSRC; ++s) {
    v[s] = 0;
    if (s < O.nsrc && ((need >> s) & 1u)) {
      const mb_src &S = O.src[s];
      if (S.fk && S.dimsz != 0 && key[s] >= S.dimsz) bad |= 1u << s;
      else v[s] = ld_w32(S.col, key[s], S.width);
    }
  }
}

// The op over loaded values (the same semantics as op_eval in opeval.cuh).
__device__ __forceinline__ bool eval_row(const mb_op &O, const uint32_t (&v)[MB_MAXSRC], uint32_t bad, bool chk,
                                         uint32_t nr_grp, int64_t &value, uint32_t &group) {
  if (chk) {
    uint32_t t = 0;
    for (uint32_t c = 0; c < O.nclause; ++c) {
      bool any = false;
      const uint32_t len = O.clause_len[c];
      for (uint32_t k = 0; k < len; ++k, ++t) {
        const mb_term &tm = O.terms[t];
        const uint64_t x = pick(v, tm.src);
        any |= !((bad >> tm.src) & 1u) && x >= tm.lo && x < tm.hi;
      }
      if (!any) return false;
    }
  }
  uint32_t g = 0;
  for (uint32_t k = 0; k < O.nkey; ++k) {
    const mb_key &kk = O.keys[k];
    if ((bad >> kk.src) & 1u) return false;
    uint32_t x = pick(v, kk.src);
    if (kk.xform == MB_X_DIV) x = x / kk.div;
    else if (kk.xform == MB_X_YEAR) x = date_to_year(x);
    g += kk.mul * (x - kk.base);
  }
  if (g >= nr_grp) return false;
  if (O.vkind == MB_V_ONE) {
    value = 1;
  } else {
    if ((bad >> O.va) & 1u) return false;
    const uint64_t a = pick(v, O.va);
    if (O.vkind == MB_V_COL) {
      value = (int64_t)a;
    } else {
      if ((bad >> O.vb) & 1u) return false;
      const uint64_t b = pick(v, O.vb);
      value = O.vkind == MB_V_MUL ? (int64_t)(a * b) : (int64_t)a - (int64_t)b;
    }
  }
  group = g;
  return true;
}

// Word lw of bitmap b in the staged tile; words past the bulk-copied part of
// the last tile come from global memory, words past the bitmap are 0.
struct TileView {
  const uint32_t *stage;  // nb x T words
  uint32_t T, copied, valid;
  uint64_t w0;
};

// The stage holds all T words of every bitmap (the last tile's tail words are
// completed by the threads before phase A), so reads need no bounds checks.
__device__ __forceinline__ uint32_t tword(const DevPrg &P, const TileView &tv, uint32_t b, uint32_t lw) {
  (void)P;
  return tv.stage[b * tv.T + lw];
}

// The conjunctive form on word lw: p = AND of (negated) operand ORs,
// u = OR of the positive operands' edge bins, masked by p.
template <bool CHK>
__device__ __forceinline__ void cnf_eval(const DevPrg &P, const TileView &tv, uint32_t lw, uint32_t &p,
                                         uint32_t &u) {
  uint32_t acc = 0xffffffffu, unc = 0;
  for (uint32_t c = 0; c < MB_MAXCOLS; ++c) {
    if (!((P.cmask >> c) & 1u)) continue;
    const uint32_t first = P.off[c], nm = P.nmid[c], ne = P.nedge[c];
    uint32_t cm = 0, ce = 0;
    for (uint32_t b = 0; b < nm; ++b) cm |= tv.stage[(first + b) * tv.T + lw];
    for (uint32_t b = 0; b < ne; ++b) ce |= tv.stage[(first + nm + b) * tv.T + lw];
    if ((P.neg >> c) & 1u) {
      acc &= ~(cm | ce);
    } else {
      acc &= cm | ce;
      if (CHK) unc |= ce;
    }
  }
  const uint64_t w = tv.w0 + lw;
  uint32_t m = w < P.nwords ? 0xffffffffu : 0u;
  const uint32_t tail = (uint32_t)(P.nrows & 31u);
  if (tail && w + 1 == P.nwords) m = (1u << tail) - 1u;
  p = acc & m;
  u = CHK ? (unc & p) : 0u;
}

__device__ __forceinline__ void or_bins_s(const DevPrg &P, const TileView &tv, int first, int cnt, uint32_t lw,
                                          uint32_t &acc) {
  acc = 0;
  for (int b = 0; b < cnt; ++b) acc |= tword(P, tv, first + b, lw);
}

// The program on words lw[k] of the staged tile (same algebra as vbp_eval).
template <int V, bool CHK>
__device__ __forceinline__ void vbp_eval_staged(const DevPrg &P, const TileView &tv, const uint32_t (&lw)[V],
                                                uint32_t (&p)[V], uint32_t (&u)[V]) {
  Regs<V> R, U;
#pragma unroll
  for (int i = 0; i < MB_NREGS; ++i)
#pragma unroll
    for (int k = 0; k < V; ++k) R.r[i][k] = U.r[i][k] = 0;
  for (uint32_t i = 0; i < P.ninstr; ++i) {
    const mb_instr in = P.ins[i];
    uint32_t dp[V], du[V], sp[V], su[V];
    rget(R, in.dstreg, dp);
    if (CHK) rget(U, in.dstreg, du);
    switch (in.opcode) {
    case MB_AND:
      rget(R, in.src1, sp);
      if (CHK) rget(U, in.src1, su);
#pragma unroll
      for (int k = 0; k < V; ++k) {
        dp[k] &= sp[k];
        if (CHK) du[k] = (du[k] | su[k]) & dp[k];
      }
      break;
    case MB_OR:
      rget(R, in.src1, sp);
      if (CHK) rget(U, in.src1, su);
#pragma unroll
      for (int k = 0; k < V; ++k) {
        if (CHK) du[k] = (du[k] & ~(sp[k] & ~su[k])) | (su[k] & ~dp[k]);
        dp[k] |= sp[k];
      }
      break;
    case MB_NOT:
      rget(R, in.src1, sp);
#pragma unroll
      for (int k = 0; k < V; ++k) dp[k] = ~sp[k];
      if (CHK && in.dstreg != in.src1) rget(U, in.src1, du);
      break;
    case MB_ANDM:
    case MB_ORM: {
      const int c = in.src1;
#pragma unroll
      for (int k = 0; k < V; ++k) {
        uint32_t cm, ce;
        or_bins_s(P, tv, P.off[c], P.nmid[c], lw[k], cm);
        or_bins_s(P, tv, P.off[c] + P.nmid[c], P.nedge[c], lw[k], ce);
        if (in.opcode == MB_ANDM) {
          if (CHK) {
            const uint32_t np = dp[k] & (ce | cm);
            du[k] = dp[k] ? ((du[k] | ce) & np) : du[k];  // primitive.cuh:292
            dp[k] = np;
          } else {
            dp[k] &= (cm | ce);
          }
        } else {
          if (CHK) du[k] = (du[k] & ~cm) | (ce & ~dp[k]);
          dp[k] |= ce | cm;
        }
      }
      break;
    }
    default: break;
    }
    rset(R, in.dstreg, dp);
    if (CHK) rset(U, in.dstreg, du);
  }
  const uint32_t tail = (uint32_t)(P.nrows & 31u);
#pragma unroll
  for (int k = 0; k < V; ++k) {
    const uint64_t w = tv.w0 + lw[k];
    uint32_t m = w < P.nwords ? 0xffffffffu : 0u;
    if (tail && w + 1 == P.nwords) m = (1u << tail) - 1u;
    p[k] = R.r[0][k] & m;
    u[k] = CHK ? (U.r[0][k] & m) : 0u;
  }
}

// Runs the op over 64 queued rows (two per lane) and aggregates them.
template <bool CHK, int GS>
__device__ __forceinline__ void drain64(const mb_op &O, const OpNeeds &N, const uint32_t *q, uint32_t nrows_avail,
                                        uint32_t nr_grp, const GrpCtx &G, int64_t &acc, uint64_t &cnt) {
  const uint32_t lane = threadIdx.x & 31;
  const bool ok0 = lane < nrows_avail, ok1 = lane + 32 < nrows_avail;
  const uint32_t e0 = ok0 ? q[lane] : 0u, e1 = ok1 ? q[lane + 32] : 0u;
  const bool c0 = CHK && (e0 >> 31), c1 = CHK && (e1 >> 31);
  uint32_t v0[MB_MAXSRC], v1[MB_MAXSRC], bad0, bad1;
  load_row(O, ok0 ? (N.kv_mask | (c0 ? N.filt_mask : 0u)) : 0u, e0 & 0x7fffffffu, v0, bad0);
  load_row(O, ok1 ? (N.kv_mask | (c1 ? N.filt_mask : 0u)) : 0u, e1 & 0x7fffffffu, v1, bad1);
  int64_t val0 = 0, val1 = 0;
  uint32_t g0 = 0, g1 = 0;
  const bool k0 = ok0 && eval_row(O, v0, bad0, c0, nr_grp, val0, g0);
  const bool k1 = ok1 && eval_row(O, v1, bad1, c1, nr_grp, val1, g1);
  cnt += (k0 ? 1u : 0u) + (k1 ? 1u : 0u);
  aggregate<GS>(G, k0, g0, val0, acc);
  if (nrows_avail > 32) aggregate<GS>(G, k1, g1, val1, acc);
}

constexpr uint32_t FT_QCAP = 32 * 32 + 64;  // one 32-word chunk + fewer than 64 pending rows

// Appends the set rows of one 32-word chunk (word w0 + lane of each lane,
// possible bits m, uncertain bits uw) to the warp queue (qn rows pending,
// warp-uniform), then drains full 64-row batches.  Queue entries are row ids
// with the uncertain flag in bit 31 (rows < 2^31).
template <bool CHK, int GS>
__device__ __forceinline__ void compact_chunk(const mb_op &O, const OpNeeds &N, uint32_t *queue, uint32_t &qn,
                                              uint64_t w0, uint32_t m, uint32_t uw, uint32_t nr_grp,
                                              const GrpCtx &G, int64_t &acc, uint64_t &cnt) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t pc = __popc(m);
  uint32_t incl = pc;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= (uint32_t)d) incl += y;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  if (total == 0) return;
  uint32_t off = qn + incl - pc;
  const uint32_t rowbase = (uint32_t)((w0 + lane) * 32);
  while (m) {
    const uint32_t b = __ffs(m) - 1;
    m &= m - 1;
    uint32_t e = rowbase + b;
    if (CHK && ((uw >> b) & 1u)) e |= 0x80000000u;
    queue[off++] = e;
  }
  qn += total;
  __syncwarp();
  while (qn >= 64) {  // drain from the end: the queue's order is irrelevant
    qn -= 64;
    drain64<CHK, GS>(O, N, queue + qn, 64, nr_grp, G, acc, cnt);
  }
  __syncwarp();
}

// The conjunctive chain on words w0 + k*32 + lane (k < V): every bitmap of the
// chain is loaded in batches of 8 independent coalesced loads, so a warp tile
// costs one memory round trip per 8 bitmaps (the interpreter's ANDM chain
// costs one per operand).
template <int V, bool CHK>
__device__ __forceinline__ void cnf_words(const DevPrg &P, uint64_t w0, uint32_t (&p)[V], uint32_t (&u)[V]) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t acc[V], cur[V], ce[V], unc[V];
#pragma unroll
  for (int k = 0; k < V; ++k) acc[k] = 0xffffffffu, cur[k] = ce[k] = unc[k] = 0;
  const uint32_t nb = P.ncnf;
  for (uint32_t b0 = 0; b0 < nb; b0 += 8) {
    uint32_t x[8][V];
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
      for (int k = 0; k < V; ++k) {
        const uint64_t w = w0 + k * 32 + lane;
        x[j][k] = (b0 + j < nb && w < P.nwords) ? __ldcs(P.cnf_ptr[b0 + j] + w) : 0u;
      }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (b0 + j >= nb) break;
      const uint32_t f = P.cnf_flag[b0 + j];
#pragma unroll
      for (int k = 0; k < V; ++k) {
        cur[k] |= x[j][k];
        if (f & CNF_EDGE) ce[k] |= x[j][k];
      }
      if (f & CNF_END) {
#pragma unroll
        for (int k = 0; k < V; ++k) {
          acc[k] &= (f & CNF_NEG) ? ~cur[k] : cur[k];
          if (CHK && !(f & CNF_NEG)) unc[k] |= ce[k];
          cur[k] = ce[k] = 0;
        }
      }
    }
  }
  const uint32_t tail = (uint32_t)(P.nrows & 31u);
#pragma unroll
  for (int k = 0; k < V; ++k) {
    const uint64_t w = w0 + k * 32 + lane;
    uint32_t m = w < P.nwords ? 0xffffffffu : 0u;
    if (tail && w + 1 == P.nwords) m = (1u << tail) - 1u;
    p[k] = acc[k] & m;
    u[k] = CHK ? (unc[k] & p[k]) : 0u;
  }
}

// Warp-independent fused kernel for conjunctive programs: each warp walks
// tiles of 32*V words on its own (no block barrier until the final flush):
// load the chain's words, compact 32-word chunks into its queue, drain.
template <int V, bool CHK, int GS>
__global__ void __launch_bounds__(FT_THREADS)
fused_warp_kernel(const __grid_constant__ DevPrg P, const __grid_constant__ mb_op O, OpNeeds N, uint32_t nr_grp,
                  uint32_t hcap, unsigned long long *__restrict__ out, unsigned long long *__restrict__ nqual) {
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ uint64_t red[64];
  const uint32_t warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const size_t gbytes = (grp_smem_bytes(GS, nr_grp, hcap) + 15) & ~(size_t)15;
  GrpCtx G = grp_init<GS>(smem, nr_grp, hcap, out);
  uint32_t *queue = reinterpret_cast<uint32_t *>(smem + gbytes) + (size_t)warp * FT_QCAP;
  __syncthreads();
  int64_t acc = 0;
  uint64_t cnt = 0;
  uint32_t qn = 0;
  constexpr uint32_t TW = 32 * V;
  const uint64_t ntiles = (P.nwords + TW - 1) / TW;
  for (uint64_t t = (uint64_t)blockIdx.x * nw + warp; t < ntiles; t += (uint64_t)gridDim.x * nw) {
    uint32_t p[V], u[V];
    cnf_words<V, CHK>(P, t * TW, p, u);
#pragma unroll
    for (int k = 0; k < V; ++k)
      compact_chunk<CHK, GS>(O, N, queue, qn, t * TW + k * 32, p[k], u[k], nr_grp, G, acc, cnt);
  }
  if (qn) drain64<CHK, GS>(O, N, queue, qn, nr_grp, G, acc, cnt);
  __syncthreads();
  grp_flush<GS>(G, nr_grp, acc, cnt, nqual, red);
}

// T = FT_THREADS * V words per CTA tile.
template <bool CHK, int GS>
__global__ void __launch_bounds__(FT_THREADS, 2)
fused_tma_kernel(const __grid_constant__ DevPrg P, const __grid_constant__ mb_op O, OpNeeds N, uint32_t nb,
                 uint32_t T, uint32_t nr_grp, uint32_t hcap, unsigned long long *__restrict__ out,
                 unsigned long long *__restrict__ nqual, uint32_t *errw) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ uint64_t red[64];
  __shared__ __align__(8) uint64_t bars[2];
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const size_t stage_words = (size_t)nb * T;
  uint32_t *stages = reinterpret_cast<uint32_t *>(smem);
  uint32_t *ptile = stages + 2 * stage_words;      // the program's possible words of the tile
  uint32_t *utile = ptile + T;                      // ... and uncertain words (CHK)
  uint8_t *gsm = reinterpret_cast<uint8_t *>(utile + (CHK ? T : 0));
  const size_t gbytes = (grp_smem_bytes(GS, nr_grp, hcap) + 15) & ~(size_t)15;
  GrpCtx G = grp_init<GS>(gsm, nr_grp, hcap, out);
  uint32_t *queue = reinterpret_cast<uint32_t *>(gsm + gbytes) + (size_t)warp * FT_QCAP;
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  __syncthreads();

  const uint64_t ntiles = (P.nwords + T - 1) / T;
  auto valid_words = [&](uint64_t t) -> uint32_t {
    const uint64_t r = P.nwords - t * T;
    return (uint32_t)(r < T ? r : T);
  };
  auto issue = [&](uint64_t t, int s) {
    const uint32_t cw = valid_words(t) & ~3u;  // whole 16-byte chunks
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&bars[s], cw * 4 * nb);
    if (cw)
      for (uint32_t b = 0; b < nb; ++b)
        bulk_g2s(stages + s * stage_words + (size_t)b * T, P.ptr[b] + t * T, cw * 4, &bars[s]);
  };
  if (tid == 0) {
    if ((uint64_t)blockIdx.x < ntiles) issue(blockIdx.x, 0);
    if ((uint64_t)blockIdx.x + gridDim.x < ntiles) issue(blockIdx.x + gridDim.x, 1);
  }

  int64_t acc = 0;
  uint64_t cnt = 0;
  uint32_t qn = 0;  // rows pending in this warp's queue (warp-uniform)
  uint32_t it = 0;
  const uint32_t nchunks = T / 32;
  for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
    const int s = it & 1;
    const uint32_t parity = (it >> 1) & 1u;
    const bool arrived = mbar_wait_bounded(&bars[s], parity, errw, MB_DEVERR_TMA_WAIT);
    if (!__syncthreads_and(arrived)) {
      if (tid == 0) mbar_wait_bounded(&bars[s], parity, nullptr, 0, 1u << 16);
      break;
    }
    TileView tv;
    tv.stage = stages + s * stage_words;
    tv.T = T;
    tv.valid = valid_words(t);
    tv.copied = tv.valid & ~3u;
    tv.w0 = t * T;
    if (tv.copied < T) {  // last tile: tail words by plain loads, the rest zero
      uint32_t *st = stages + s * stage_words;
      const uint32_t span = T - tv.copied;
      for (uint32_t i = tid; i < nb * span; i += FT_THREADS) {
        const uint32_t b = i / span, lw = tv.copied + i % span;
        st[(size_t)b * T + lw] = lw < tv.valid ? __ldg(P.ptr[b] + tv.w0 + lw) : 0u;
      }
      __syncthreads();
    }
    // phase A: the program over the staged tile, one word per lane per chunk
    for (uint32_t c = warp; c < nchunks; c += FT_WARPS) {
      const uint32_t w = c * 32 + lane;
      uint32_t p1, u1;
      if (P.cnf) {
        cnf_eval<CHK>(P, tv, w, p1, u1);
      } else {
        uint32_t lw[1] = {w}, p[1], u[1];
        vbp_eval_staged<1, CHK>(P, tv, lw, p, u);
        p1 = p[0], u1 = u[0];
      }
      ptile[w] = p1;
      if (CHK) utile[w] = u1;
    }
    __syncthreads();  // stage s consumed, ptile complete
    if (tid == 0 && t + 2ull * gridDim.x < ntiles) issue(t + 2ull * gridDim.x, s);
    // phase B: compaction into the warp queue; the op runs on full 64-row batches
    for (uint32_t c = warp; c < nchunks; c += FT_WARPS)
      compact_chunk<CHK, GS>(O, N, queue, qn, tv.w0 + c * 32, ptile[c * 32 + lane], CHK ? utile[c * 32 + lane] : 0u,
                             nr_grp, G, acc, cnt);
  }
  if (qn) drain64<CHK, GS>(O, N, queue, qn, nr_grp, G, acc, cnt);
  __syncthreads();
  grp_flush<GS>(G, nr_grp, acc, cnt, nqual, red);
}

// ------------------------------------------------------------------ host
constexpr size_t FT_STAGE_TARGET = 24 * 1024;  // bytes of one stage when the tile can shrink

template <bool CHK, int GS>
static mb_status launch_ft(const DevPrg &P, const mb_op &O, uint32_t nb, uint32_t T, uint32_t nr_grp,
                           uint32_t hcap, int64_t *out, uint64_t *nq, uint32_t cps, cudaStream_t st) {
  auto kern = fused_tma_kernel<CHK, GS>;
  const size_t smem = 2 * (size_t)nb * T * 4 + (size_t)T * 4 * (CHK ? 2 : 1) +
                      ((grp_smem_bytes(GS, nr_grp, hcap) + 15) & ~(size_t)15) + (size_t)FT_WARPS * FT_QCAP * 4;
  const DevInfo &di = dev_info();
  if (smem > (size_t)di.max_smem_optin) return fail(MB_ERR_INVALID, "fused: %zu bytes of shared memory", smem);
  MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, FT_THREADS, smem));
  if (occ < 1) return fail(MB_ERR_INVALID, "fused: kernel does not fit on an SM");
  if (cps && (int)cps < occ) occ = (int)cps;
  const uint64_t ntiles = (P.nwords + T - 1) / T;
  uint64_t grid = (uint64_t)di.sms * occ;
  if (grid > ntiles) grid = ntiles ? ntiles : 1;
  uint32_t *errw = device_error_word();
  if (!errw) return fail(MB_ERR_OOM, "fused: device error word");
  kern<<<(unsigned)grid, FT_THREADS, smem, st>>>(P, O, op_needs(O), nb, T, nr_grp, hcap,
                                                 reinterpret_cast<unsigned long long *>(out),
                                                 reinterpret_cast<unsigned long long *>(nq), errw);
  MB_LAUNCH_CHECK("fused_tma_kernel");
  return MB_OK;
}

template <bool CHK>
static mb_status ft_gs(int gs, const DevPrg &P, const mb_op &O, uint32_t nb, uint32_t T, uint32_t nr_grp,
                       uint32_t hcap, int64_t *out, uint64_t *nq, uint32_t cps, cudaStream_t st) {
  switch (gs) {
  case GS_SCALAR: return launch_ft<CHK, GS_SCALAR>(P, O, nb, T, nr_grp, hcap, out, nq, cps, st);
  case GS_SHARED: return launch_ft<CHK, GS_SHARED>(P, O, nb, T, nr_grp, hcap, out, nq, cps, st);
  case GS_GLOBAL: return launch_ft<CHK, GS_GLOBAL>(P, O, nb, T, nr_grp, hcap, out, nq, cps, st);
  default: return launch_ft<CHK, GS_HASH>(P, O, nb, T, nr_grp, hcap, out, nq, cps, st);
  }
}

// The staged kernel applies when every bitmap is 16-byte aligned (bulk
// copies), every op source is at most 4 bytes wide and the program reads at
// least one bitmap.
bool fused_tma_applies(const DevPrg &P, bool vec4, const mb_op &O) {
  uint32_t nb = 0;
  for (uint32_t c = 0; c < MB_MAXCOLS; ++c) nb += P.nmid[c] + P.nedge[c];
  if (!vec4 || nb == 0 || P.nrows == 0) return false;
  for (uint32_t s = 0; s < O.nsrc; ++s)
    if (O.src[s].width > 4) return false;
  return true;
}

static size_t ft_smem(uint32_t nb, uint32_t T, bool chk, int gs, uint32_t nr_grp, uint32_t hcap) {
  return 2 * (size_t)nb * T * 4 + (size_t)T * 4 * (chk ? 2 : 1) +
         ((grp_smem_bytes(gs, nr_grp, hcap) + 15) & ~(size_t)15) + (size_t)FT_WARPS * FT_QCAP * 4;
}

// V (words per thread of a tile; 0 = auto) sets the tile to 256 * V words:
// auto picks the widest tile whose stage stays near FT_STAGE_TARGET bytes;
// a tile that does not fit in shared memory shrinks.  Returns
// MB_ERR_UNSUPPORTED if even the narrowest tile does not fit.
mb_status fused_tma(const DevPrg &P, const mb_op &O, uint32_t nr_grp, int gs, uint32_t hcap, uint32_t V,
                    int64_t *out, uint64_t *nq, uint32_t cps, cudaStream_t st) {
  uint32_t nb = 0;
  for (uint32_t c = 0; c < MB_MAXCOLS; ++c) nb += P.nmid[c] + P.nedge[c];
  if (V == 0) V = nb * FT_THREADS * 4 * 4 <= FT_STAGE_TARGET ? 4 : nb * FT_THREADS * 2 * 4 <= FT_STAGE_TARGET ? 2 : 1;
  const size_t cap = (size_t)dev_info().max_smem_optin;
  while (V > 1 && ft_smem(nb, FT_THREADS * V, P.chk != 0, gs, nr_grp, hcap) > cap) V >>= 1;
  if (ft_smem(nb, FT_THREADS * V, P.chk != 0, gs, nr_grp, hcap) > cap)
    return fail(MB_ERR_UNSUPPORTED, "fused: %u bitmaps do not fit a staged tile", nb);
  const uint32_t T = FT_THREADS * V;
  return P.chk ? ft_gs<true>(gs, P, O, nb, T, nr_grp, hcap, out, nq, cps, st)
               : ft_gs<false>(gs, P, O, nb, T, nr_grp, hcap, out, nq, cps, st);
}

// ------------------------------------------------- warp-independent kernel
bool fused_warp_applies(const DevPrg &P, const mb_op &O) {
  if (!P.cnf || P.nrows == 0) return false;
  for (uint32_t s = 0; s < O.nsrc; ++s)
    if (O.src[s].width > 4) return false;
  return true;
}

template <int V, bool CHK, int GS>
static mb_status launch_fw(const DevPrg &P, const mb_op &O, uint32_t nr_grp, uint32_t hcap, int64_t *out,
                           uint64_t *nq, uint32_t warps, uint32_t cps, cudaStream_t st) {
  auto kern = fused_warp_kernel<V, CHK, GS>;
  const size_t smem = ((grp_smem_bytes(GS, nr_grp, hcap) + 15) & ~(size_t)15) + (size_t)warps * FT_QCAP * 4;
  const DevInfo &di = dev_info();
  if (smem > (size_t)di.max_smem_optin) return fail(MB_ERR_INVALID, "fused: %zu bytes of shared memory", smem);
  MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, (int)(warps * 32), smem));
  if (occ < 1) return fail(MB_ERR_INVALID, "fused: kernel does not fit on an SM");
  if (cps && (int)cps < occ) occ = (int)cps;
  const uint64_t ntiles = (P.nwords + 32 * V - 1) / (32 * V);
  uint64_t grid = (uint64_t)di.sms * occ;
  const uint64_t need = (ntiles + warps - 1) / warps;
  if (grid > need) grid = need ? need : 1;
  kern<<<(unsigned)grid, warps * 32, smem, st>>>(P, O, op_needs(O), nr_grp, hcap,
                                                 reinterpret_cast<unsigned long long *>(out),
                                                 reinterpret_cast<unsigned long long *>(nq));
  MB_LAUNCH_CHECK("fused_warp_kernel");
  return MB_OK;
}

template <int V, bool CHK>
static mb_status fw_gs(int gs, const DevPrg &P, const mb_op &O, uint32_t nr_grp, uint32_t hcap, int64_t *out,
                       uint64_t *nq, uint32_t warps, uint32_t cps, cudaStream_t st) {
  switch (gs) {
  case GS_SCALAR: return launch_fw<V, CHK, GS_SCALAR>(P, O, nr_grp, hcap, out, nq, warps, cps, st);
  case GS_SHARED: return launch_fw<V, CHK, GS_SHARED>(P, O, nr_grp, hcap, out, nq, warps, cps, st);
  case GS_GLOBAL: return launch_fw<V, CHK, GS_GLOBAL>(P, O, nr_grp, hcap, out, nq, warps, cps, st);
  default: return launch_fw<V, CHK, GS_HASH>(P, O, nr_grp, hcap, out, nq, warps, cps, st);
  }
}

mb_status fused_warp(const DevPrg &P, const mb_op &O, uint32_t nr_grp, int gs, uint32_t hcap, uint32_t V,
                     uint32_t warps, int64_t *out, uint64_t *nq, uint32_t cps, cudaStream_t st) {
  if (V == 0) V = 2;
  if (warps == 0 || warps > 8) warps = 8;  // FT_THREADS bounds the block
  const bool chk = P.chk != 0;
  if (V == 4) return chk ? fw_gs<4, true>(gs, P, O, nr_grp, hcap, out, nq, warps, cps, st)
                         : fw_gs<4, false>(gs, P, O, nr_grp, hcap, out, nq, warps, cps, st);
  if (V == 2) return chk ? fw_gs<2, true>(gs, P, O, nr_grp, hcap, out, nq, warps, cps, st)
                         : fw_gs<2, false>(gs, P, O, nr_grp, hcap, out, nq, warps, cps, st);
  return chk ? fw_gs<1, true>(gs, P, O, nr_grp, hcap, out, nq, warps, cps, st)
             : fw_gs<1, false>(gs, P, O, nr_grp, hcap, out, nq, warps, cps, st);
}

}  // namespace mb
