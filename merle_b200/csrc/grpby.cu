// grpby.cu - the query kernels: fused program -> compaction -> op -> group-by
// (mb_vprg_grpby), the no-index scan (mb_join_grpby) and the three
// materialised stages (mb_vprg_eval, mb_bitmap_to_rows, mb_rows_grpby).
//
// Reference kernels: vprg_grpby (primitive.cuh:340-445), grpby
// (primitive.cuh:16-48), abla::_stg1/_stg2/_stg3 (primitive_abla.cuh:262-394).
//
// B200 design of the fused kernel:
//  - Persistent grid (SMs x occupancy).  Work unit = one warp tile of 32*V
//    bitmap words (V = 4: 4096 rows); warps of a CTA take adjacent tiles.
//  - The program runs in registers (vbp.cuh) with 128-bit streaming loads.
//  - Compaction is per warp: popcounts, a 5-step shuffle scan, and the set
//    bits' row offsets (12 bits + the uncertain flag in bit 15) written to a
//    warp-private 16-bit list in shared memory.  No block barrier sits
//    between a warp's tiles, and every lane then takes one listed row per
//    round, so lanes stay busy at any selectivity (the reference switches to
//    a per-bit loop above nt*vt0 hits, primitive.cuh:373-397).
//  - Group-by: dense shared-memory int64 table (GS_SHARED), warp-aggregated
//    global atomics (GS_GLOBAL), a shared-memory hash table (GS_HASH), or a
//    register accumulator when there is one group (GS_SCALAR).
#include <string.h>
#include <mutex>
#include "common.cuh"
#include "opeval.cuh"
#include "vbp.cuh"

namespace mb {

// ------------------------------------------------------------ validation
mb_status flatten_prg(const mb_vprg *p, int chk, DevPrg *o, bool *vec4) {
  if (!p) return fail(MB_ERR_INVALID, "program is NULL");
  if (p->ncols > MB_MAXCOLS) return fail(MB_ERR_INVALID, "program: %u operands > %d", p->ncols, MB_MAXCOLS);
  memset(o, 0, sizeof(*o));
  o->nrows = p->factsz;
  o->nwords = (p->factsz + 31) / 32;
  o->chk = chk ? 1u : 0u;
  bool v4 = true;
  uint32_t np = 0;
  for (uint32_t c = 0; c < p->ncols; ++c) {
    const mb_col &col = p->cols[c];
    if (col.nmiddle > MB_MAXBINS) return fail(MB_ERR_INVALID, "operand %u: %u bins > %d", c, col.nmiddle, MB_MAXBINS);
    uint32_t ne = (col.leftmost ? 1 : 0) + (col.rightmost ? 1 : 0);
    if (np + col.nmiddle + ne > MB_MAXPTRS) return fail(MB_ERR_INVALID, "program: more than %d bitmaps", MB_MAXPTRS);
    if (col.nmiddle && !col.middle) return fail(MB_ERR_INVALID, "operand %u: middle array is NULL", c);
    o->off[c] = (uint8_t)np;
    o->nmid[c] = (uint8_t)col.nmiddle;
    o->nedge[c] = (uint8_t)ne;
    for (uint32_t k = 0; k < col.nmiddle; ++k) {
      if (!col.middle[k]) return fail(MB_ERR_INVALID, "operand %u: middle bin %u is NULL", c, k);
      o->ptr[np++] = col.middle[k];
    }
    if (col.leftmost) o->ptr[np++] = col.leftmost;
    if (col.rightmost) o->ptr[np++] = col.rightmost;
  }
  for (uint32_t i = 0; i < np; ++i)
    if (((uintptr_t)o->ptr[i] & 15) != 0) v4 = false;
  uint32_t n = 0;
  for (; n < MB_MAXNINSTR; ++n) {
    const mb_instr in = p->instrs[n];
    if (in.opcode == MB_END) break;
    if (in.opcode > MB_ORM) return fail(MB_ERR_INVALID, "instruction %u: bad opcode %u", n, in.opcode);
    if (in.dstreg >= MB_NREGS) return fail(MB_ERR_INVALID, "instruction %u: register %u >= %d", n, in.dstreg, MB_NREGS);
    if (in.opcode == MB_ANDM || in.opcode == MB_ORM) {
      if (in.src1 >= p->ncols) return fail(MB_ERR_INVALID, "instruction %u: operand %u >= ncols %u", n, in.src1, p->ncols);
    } else if (in.src1 >= MB_NREGS) {
      return fail(MB_ERR_INVALID, "instruction %u: register %u >= %d", n, in.src1, MB_NREGS);
    }
    o->ins[n] = in;
  }
  o->ninstr = n;
  *vec4 = v4;
  detect_cnf(o);
  return MB_OK;
}

// Recognises the conjunctive chain the planner emits (every conjunct a
// distinct operand; r2 and r3 never written):
//   first conjunct:  ORM r0,c            | ORM r1,c; NOT r0,r1    | NOT r0,r3 (all rows)
//   next conjuncts:  ANDM r0,c           | AND r1,r2; ORM r1,c; NOT r1,r1; AND r0,r1
// On every row the chain selects, its (possible, uncertain) result equals
// p = AND_c (m_c or ~m_c), u = (OR of the positive conjuncts' edge bins) & p,
// with m_c = middle | edge bins of operand c: a negated conjunct contributes
// no uncertain bit (its edge bits lie outside ~m_c), and the zero-word skip of
// ANDM only changes uncertain bits of unselected words (primitive.cuh:292).
void detect_cnf(DevPrg *o) {
  o->cnf = 0;
  o->cmask = 0;
  o->neg = 0;
  const uint32_t n = o->ninstr;
  auto is = [&](uint32_t i, uint8_t op, uint8_t d, int s) {
    return i < n && o->ins[i].opcode == op && o->ins[i].dstreg == d && (s < 0 || o->ins[i].src1 == (uint8_t)s);
  };
  uint32_t i = 0;
  uint8_t used = 0, neg = 0;
  auto add = [&](uint8_t c, bool ng) -> bool {
    if (c >= MB_MAXCOLS || (used >> c) & 1u) return false;
    used |= (uint8_t)(1u << c);
    if (ng) neg |= (uint8_t)(1u << c);
    return true;
  };
  if (is(i, MB_ORM, 0, -1)) {
    if (!add(o->ins[i].src1, false)) return;
    i += 1;
  } else if (is(i, MB_ORM, 1, -1) && is(i + 1, MB_NOT, 0, 1)) {
    if (!add(o->ins[i].src1, true)) return;
    i += 2;
  } else if (is(i, MB_NOT, 0, 3)) {
    i += 1;
  } else {
    return;
  }
  while (i < n) {
    if (is(i, MB_ANDM, 0, -1)) {
      if (!add(o->ins[i].src1, false)) return;
      i += 1;
    } else if (is(i, MB_AND, 1, 2) && is(i + 1, MB_ORM, 1, -1) && is(i + 2, MB_NOT, 1, 1) && is(i + 3, MB_AND, 0, 1)) {
      if (!add(o->ins[i + 1].src1, true)) return;
      i += 4;
    } else {
      return;
    }
  }
  // flatten the chain: bins of each conjunct, the last one flagged CNF_END
  uint32_t k = 0;
  for (uint32_t c = 0; c < MB_MAXCOLS; ++c) {
    if (!((used >> c) & 1u)) continue;
    const uint32_t nb = o->nmid[c] + o->nedge[c];
    for (uint32_t b = 0; b < nb; ++b, ++k) {
      o->cnf_ptr[k] = o->ptr[o->off[c] + b];
      uint8_t f = (uint8_t)((b >= o->nmid[c] ? CNF_EDGE : 0) | (b + 1 == nb ? CNF_END : 0) |
                            (((neg >> c) & 1u) ? CNF_NEG : 0));
      o->cnf_flag[k] = f;
    }
    if (nb == 0) return;  // a conjunct without bitmaps: keep the interpreter
  }
  o->ncnf = (uint8_t)k;
  o->cnf = 1;
  o->cmask = used;
  o->neg = neg;
}

static mb_status validate_op(const mb_op *op) {
  if (!op) return fail(MB_ERR_INVALID, "op is NULL");
  if (op->nsrc > MB_MAXSRC) return fail(MB_ERR_INVALID, "op: %u sources > %d", op->nsrc, MB_MAXSRC);
  for (uint32_t i = 0; i < op->nsrc; ++i) {
    const mb_src &s = op->src[i];
    if (!s.col) return fail(MB_ERR_INVALID, "op source %u: column is NULL", i);
    if (s.width != 1 && s.width != 2 && s.width != 4 && s.width != 8)
      return fail(MB_ERR_INVALID, "op source %u: width %u", i, s.width);
  }
  if (op->nclause > MB_MAXCLAUSE) return fail(MB_ERR_INVALID, "op: %u clauses > %d", op->nclause, MB_MAXCLAUSE);
  uint32_t nt = 0;
  for (uint32_t c = 0; c < op->nclause; ++c) nt += op->clause_len[c];
  if (nt > MB_MAXTERM) return fail(MB_ERR_INVALID, "op: %u terms > %d", nt, MB_MAXTERM);
  for (uint32_t t = 0; t < nt; ++t)
    if (op->terms[t].src >= op->nsrc) return fail(MB_ERR_INVALID, "op term %u: source %u", t, op->terms[t].src);
  if (op->nkey > MB_MAXKEY) return fail(MB_ERR_INVALID, "op: %u key fields > %d", op->nkey, MB_MAXKEY);
  for (uint32_t k = 0; k < op->nkey; ++k) {
    const mb_key &kk = op->keys[k];
    if (kk.src >= op->nsrc) return fail(MB_ERR_INVALID, "op key %u: source %u", k, kk.src);
    if (kk.xform > MB_X_YEAR) return fail(MB_ERR_INVALID, "op key %u: xform %u", k, kk.xform);
    if (kk.xform == MB_X_DIV && kk.div == 0) return fail(MB_ERR_INVALID, "op key %u: div 0", k);
  }
  if (op->vkind > MB_V_SUB) return fail(MB_ERR_INVALID, "op: value kind %u", op->vkind);
  if (op->vkind != MB_V_ONE && op->va >= op->nsrc) return fail(MB_ERR_INVALID, "op: value source %u", op->va);
  if ((op->vkind == MB_V_MUL || op->vkind == MB_V_SUB) && op->vb >= op->nsrc)
    return fail(MB_ERR_INVALID, "op: value source %u", op->vb);
  return MB_OK;
}

// ----------------------------------------------------------- fused kernel
template <int V>
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x) {
  const uint32_t lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= (uint32_t)d) x += y;
  }
  return x;
}

template <int V, bool CHK, int GS>
__global__ void __launch_bounds__(512)
vbp_grpby_kernel(const __grid_constant__ DevPrg P, const __grid_constant__ mb_op O, uint32_t nr_grp,
                 uint32_t hcap, unsigned long long *__restrict__ out, unsigned long long *__restrict__ nqual) {
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ uint64_t red[64];
  constexpr uint32_t WT_WORDS = 32 * V;  // words of one warp tile
  constexpr uint32_t WT_ROWS = WT_WORDS * 32;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const size_t gbytes = (grp_smem_bytes(GS, nr_grp, hcap) + 15) & ~(size_t)15;
  GrpCtx G = grp_init<GS>(smem, nr_grp, hcap, out);
  uint16_t *buf = reinterpret_cast<uint16_t *>(smem + gbytes) + (size_t)warp * WT_ROWS;
  __syncthreads();

  int64_t acc = 0;
  uint64_t cnt = 0;
  const uint64_t ntiles = (P.nwords + WT_WORDS - 1) / WT_WORDS;
  for (uint64_t t = (uint64_t)blockIdx.x * nw + warp; t < ntiles; t += (uint64_t)gridDim.x * nw) {
    const uint64_t w0 = t * WT_WORDS + lane * V;
    uint32_t p[V], u[V];
    vbp_eval<V, CHK>(P, w0, p, u);
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < V; ++k) c += __popc(p[k]);
    const uint32_t incl = warp_incl_scan<V>(c);
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0) continue;
    uint32_t off = incl - c;
#pragma unroll
    for (int k = 0; k < V; ++k) {
      uint32_t m = p[k];
      const uint32_t base = (lane * V + k) * 32;
      while (m) {
        const uint32_t b = __ffs(m) - 1;
        m &= m - 1;
        uint32_t e = base + b;
        if (CHK && ((u[k] >> b) & 1u)) e |= 0x8000u;
        buf[off++] = (uint16_t)e;
      }
    }
    __syncwarp();
    const uint32_t row0 = (uint32_t)(t * WT_ROWS);
    for (uint32_t base = 0; base < total; base += 32) {
      const uint32_t j = base + lane;
      bool kept = false;
      int64_t val = 0;
      uint32_t grp = 0;
      if (j < total) {
        const uint32_t e = buf[j];
        kept = op_eval(O, row0 + (e & 0x7fffu), CHK && (e & 0x8000u), nr_grp, val, grp);
      }
      cnt += kept ? 1u : 0u;
      aggregate<GS>(G, kept, grp, val, acc);
    }
    __syncwarp();
  }
  __syncthreads();
  grp_flush<GS>(G, nr_grp, acc, cnt, nqual, red);
}

// -------------------------------------------------------- no-index scan
// Clause c alone on one row, as op_eval evaluates it.
__device__ __forceinline__ bool clause_pass(const mb_op &O, uint32_t c, uint32_t t0, uint32_t row) {
  bool any = false;
  for (uint32_t k = 0; k < O.clause_len[c] && !any; ++k) {
    const mb_term &tm = O.terms[t0 + k];
    uint64_t v;
    any = src_value(O.src[tm.src], row, v) && v >= tm.lo && v < tm.hi;
  }
  return any;
}

constexpr uint32_t JQ = 160;  // rows a warp queues between the screen and the op (31 + a 128-row chunk)

// Every row through the op.  A row first meets one clause (`screen`, first
// term `t0`; none if screen >= nclause), one row per lane; the rows that pass
// queue per warp, and each full warp of them runs the rest of the op, so the
// lanes of its loads and branches are all live rows.  The result equals
// op_eval on every row (the screen is one of the op's own clauses).
// Four consecutive values of a fact column of SW-byte elements from one
// vector load (the column 16-byte aligned, rows r .. r+3 inside it, r a
// multiple of 4).
template <int SW>
__device__ __forceinline__ void load4(const void *col, uint64_t r, uint64_t (&v)[4]) {
  if (SW == 1) {
    const uint32_t w = __ldg(reinterpret_cast<const uint32_t *>(col) + r / 4);
#pragma unroll
    for (int j = 0; j < 4; ++j) v[j] = (w >> (8 * j)) & 0xffu;
  } else if (SW == 2) {
    const uint2 w = __ldg(reinterpret_cast<const uint2 *>(col) + r / 4);
    v[0] = w.x & 0xffffu, v[1] = w.x >> 16, v[2] = w.y & 0xffffu, v[3] = w.y >> 16;
  } else if (SW == 4) {
    const uint4 w = __ldg(reinterpret_cast<const uint4 *>(col) + r / 4);
    v[0] = w.x, v[1] = w.y, v[2] = w.z, v[3] = w.w;
  } else {
    const ulonglong2 a = __ldg(reinterpret_cast<const ulonglong2 *>(col) + r / 2),
                     b = __ldg(reinterpret_cast<const ulonglong2 *>(col) + r / 2 + 1);
    v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
  }
}

template <int GS, int SW>
__global__ void __launch_bounds__(256, 8)
join_grpby_kernel(uint64_t nrows, const __grid_constant__ mb_op O, uint32_t nr_grp, uint32_t hcap,
                  uint32_t grp_bytes, uint32_t screen, uint32_t t0, unsigned long long *__restrict__ out,
                  unsigned long long *__restrict__ nqual) {
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ uint64_t red[64];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  GrpCtx G = grp_init<GS>(smem, nr_grp, hcap, out);
  uint32_t *queue = reinterpret_cast<uint32_t *>(smem + grp_bytes) + (size_t)warp * JQ;
  __syncthreads();
  int64_t acc = 0;
  uint64_t cnt = 0;
  uint32_t qn = 0;
  const uint32_t lt = (1u << lane) - 1u;
  auto drain = [&](uint32_t m) {  // the last m (<= 32) queued rows through the op
    bool kept = false;
    int64_t val = 0;
    uint32_t grp = 0;
    if (lane < m) kept = op_eval(O, queue[qn - m + lane], true, nr_grp, val, grp, screen);
    cnt += kept ? 1u : 0u;
    aggregate<GS>(G, kept, grp, val, acc);
    qn -= m;
    __syncwarp();
  };
  const uint64_t nchunks = (nrows + 31) / 32;
  if (screen >= O.nclause) {  // no screen (or no room for the queues): every row through the op
    for (uint64_t ch = (uint64_t)blockIdx.x * nw + warp; ch < nchunks; ch += (uint64_t)gridDim.x * nw) {
      const uint64_t row = ch * 32 + lane;
      bool kept = false;
      int64_t val = 0;
      uint32_t grp = 0;
      if (row < nrows) kept = op_eval(O, (uint32_t)row, true, nr_grp, val, grp);
      cnt += kept ? 1u : 0u;
      aggregate<GS>(G, kept, grp, val, acc);
    }
  } else if (SW == 0) {
    for (uint64_t ch = (uint64_t)blockIdx.x * nw + warp; ch < nchunks; ch += (uint64_t)gridDim.x * nw) {
      const uint64_t row = ch * 32 + lane;
      const bool pass = row < nrows && clause_pass(O, screen, t0, (uint32_t)row);
      const uint32_t bal = __ballot_sync(0xffffffffu, pass);
      if (pass) queue[qn + __popc(bal & lt)] = (uint32_t)row;
      qn += __popc(bal);  // at most 31 + 32 < JQ
      __syncwarp();
      if (qn >= 32) drain(32);
    }
    if (qn) drain(qn);
  } else {
    // the screen is one range on a fact column of SW-byte elements: four rows
    // a lane from one vector load; 128-row chunks, the last one partly by
    // scalar loads
    const mb_term &tm = O.terms[t0];
    const void *col = O.src[tm.src].col;
    const uint64_t lo = tm.lo, hi = tm.hi, nch4 = (nrows + 127) / 128;
    for (uint64_t ch = (uint64_t)blockIdx.x * nw + warp; ch < nch4; ch += (uint64_t)gridDim.x * nw) {
      const uint64_t r = ch * 128 + 4 * lane;
      uint64_t v[4] = {0, 0, 0, 0};
      if (ch * 128 + 128 <= nrows) {
        load4<SW>(col, r, v);
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (r + j < nrows) v[j] = load_width(col, r + j, SW);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const bool pass = r + j < nrows && v[j] >= lo && v[j] < hi;
        const uint32_t bal = __ballot_sync(0xffffffffu, pass);
        if (pass) queue[qn + __popc(bal & lt)] = (uint32_t)(r + j);
        qn += __popc(bal);  // at most 31 + 128 < JQ
      }
      __syncwarp();
      while (qn >= 32) drain(32);
    }
    if (qn) drain(qn);
  }
  __syncthreads();
  grp_flush<GS>(G, nr_grp, acc, cnt, nqual, red);
}

// ------------------------------------------------ materialised stage 1
template <int V, bool CHK>
__global__ void __launch_bounds__(256)
vbp_eval_kernel(const __grid_constant__ DevPrg P, uint32_t *__restrict__ poss, uint32_t *__restrict__ unc,
                unsigned long long *__restrict__ pop) {
  __shared__ uint64_t red[64];
  uint64_t c = 0;
  const uint64_t nvec = (P.nwords + V - 1) / V;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nvec; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t w0 = i * V;
    uint32_t p[V], u[V];
    vbp_eval<V, CHK>(P, w0, p, u);
#pragma unroll
    for (int k = 0; k < V; ++k) {
      if (w0 + k < P.nwords) {
        poss[w0 + k] = p[k];
        if (unc) unc[w0 + k] = u[k];
        c += __popc(p[k]);
      }
    }
  }
  uint64_t z = 0;
  block_sum2(c, z, red);
  if (threadIdx.x == 0 && pop && c) atomicAdd(pop, (unsigned long long)c);
}

// ------------------------------------------------ materialised stage 2
// Row list in ascending order: per-segment counts, one-CTA exclusive scan,
// then each segment writes its rows at its offset.
constexpr uint32_t RL_THREADS = 256;
constexpr uint32_t RL_SEG_WORDS = RL_THREADS * 8;  // 2048 words per segment

__global__ void __launch_bounds__(RL_THREADS)
rows_count_kernel(const uint32_t *__restrict__ poss, uint64_t nrows, uint32_t *__restrict__ segcnt) {
  __shared__ uint64_t red[64];
  const uint64_t nwords = (nrows + 31) / 32;
  const uint64_t w0 = (uint64_t)blockIdx.x * RL_SEG_WORDS;
  uint64_t c = 0;
  const uint32_t tail = (uint32_t)(nrows & 31);
  for (uint32_t k = threadIdx.x; k < RL_SEG_WORDS; k += RL_THREADS) {
    const uint64_t w = w0 + k;
    if (w < nwords) {
      uint32_t m = poss[w];
      if (tail && w + 1 == nwords) m &= (1u << tail) - 1u;
      c += __popc(m);
    }
  }
  uint64_t z = 0;
  block_sum2(c, z, red);
  if (threadIdx.x == 0) segcnt[blockIdx.x] = (uint32_t)c;
}

// Exclusive scan of nseg counts in place (one CTA of 1024 threads); the total
// goes to *count.
__global__ void __launch_bounds__(1024)
rows_scan_kernel(uint32_t *__restrict__ seg, uint64_t nseg, unsigned long long *__restrict__ count) {
  __shared__ uint64_t part[1024];
  const uint64_t per = (nseg + 1023) / 1024;
  const uint64_t b = threadIdx.x * per, e = b + per < nseg ? b + per : nseg;
  uint64_t s = 0;
  for (uint64_t i = b; i < e; ++i) s += seg[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (uint32_t d = 1; d < 1024; d <<= 1) {  // Hillis-Steele inclusive scan
    uint64_t v = threadIdx.x >= d ? part[threadIdx.x - d] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  uint64_t run = part[threadIdx.x] - s;
  for (uint64_t i = b; i < e; ++i) {
    const uint32_t v = seg[i];
    seg[i] = (uint32_t)run;
    run += v;
  }
  if (threadIdx.x == 1023) *count = part[1023];
}

__global__ void __launch_bounds__(RL_THREADS)
rows_write_kernel(const uint32_t *__restrict__ poss, const uint32_t *__restrict__ unc, uint64_t nrows,
                  const uint32_t *__restrict__ segoff, uint32_t *__restrict__ rows) {
  __shared__ uint32_t wsum[RL_THREADS / 32];
  const uint64_t nwords = (nrows + 31) / 32;
  const uint32_t tail = (uint32_t)(nrows & 31);
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // thread t owns words w0 + t*8 .. +8 (contiguous, so row order is kept)
  const uint64_t w0 = (uint64_t)blockIdx.x * RL_SEG_WORDS + threadIdx.x * 8;
  uint32_t m[8], uu[8], c = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint64_t w = w0 + k;
    m[k] = w < nwords ? poss[w] : 0u;
    if (tail && w + 1 == nwords) m[k] &= (1u << tail) - 1u;
    uu[k] = (unc && w < nwords) ? unc[w] : 0u;
    c += __popc(m[k]);
  }
  uint32_t incl = c;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= (uint32_t)d) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  uint32_t before = 0;
  for (uint32_t w = 0; w < warp; ++w) before += wsum[w];
  uint64_t off = (uint64_t)segoff[blockIdx.x] + before + incl - c;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    uint32_t x = m[k];
    while (x) {
      const uint32_t b = __ffs(x) - 1;
      x &= x - 1;
      uint32_t r = (uint32_t)((w0 + k) * 32 + b);
      if ((uu[k] >> b) & 1u) r |= 0x80000000u;
      rows[off++] = r;
    }
  }
}

// ------------------------------------------------ materialised stage 3
template <int GS>
__global__ void __launch_bounds__(512)
rows_grpby_kernel(const uint32_t *__restrict__ rows, const unsigned long long *__restrict__ count, uint64_t capacity,
                  const __grid_constant__ mb_op O, uint32_t nr_grp, uint32_t hcap,
                  unsigned long long *__restrict__ out, unsigned long long *__restrict__ nqual) {
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ uint64_t red[64];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  GrpCtx G = grp_init<GS>(smem, nr_grp, hcap, out);
  __syncthreads();
  uint64_t n = *count;
  if (n > capacity) n = capacity;
  int64_t acc = 0;
  uint64_t cnt = 0;
  const uint64_t nchunks = (n + 31) / 32;
  for (uint64_t ch = (uint64_t)blockIdx.x * nw + warp; ch < nchunks; ch += (uint64_t)gridDim.x * nw) {
    const uint64_t i = ch * 32 + lane;
    bool kept = false;
    int64_t val = 0;
    uint32_t grp = 0;
    if (i < n) {
      const uint32_t r = __ldcs(rows + i);
      kept = op_eval(O, r & 0x7fffffffu, (r >> 31) != 0, nr_grp, val, grp);
    }
    cnt += kept ? 1u : 0u;
    aggregate<GS>(G, kept, grp, val, acc);
  }
  __syncthreads();
  grp_flush<GS>(G, nr_grp, acc, cnt, nqual, red);
}

__global__ void certain_kernel(uint32_t *__restrict__ p, const uint32_t *__restrict__ u, uint64_t W) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < W; i += (uint64_t)gridDim.x * blockDim.x)
    p[i] &= ~u[i];
}

mb_status certain_of(uint32_t *p, const uint32_t *u, uint64_t nrows, cudaStream_t st) {
  const uint64_t W = (nrows + 31) / 32;
  if (W == 0) return MB_OK;
  uint64_t grid = (W + 255) / 256, cap = (uint64_t)dev_info().sms * 8;
  certain_kernel<<<(unsigned)(grid < cap ? grid : cap), 256, 0, st>>>(p, u, W);
  MB_LAUNCH_CHECK("certain_kernel");
  return MB_OK;
}

// ------------------------------------------------------------------ host
constexpr uint32_t DEFAULT_HCAP = 4096;
constexpr uint32_t SHARED_MAX_GROUPS = 8192;

static int pick_gs(uint32_t nr_grp, uint32_t requested) {
  if (nr_grp == 1 && requested != MB_GRP_GLOBAL && requested != MB_GRP_HASH) return GS_SCALAR;
  switch (requested) {
  case MB_GRP_SHARED: return GS_SHARED;
  case MB_GRP_GLOBAL: return GS_GLOBAL;
  case MB_GRP_HASH: return GS_HASH;
  default: return nr_grp <= SHARED_MAX_GROUPS ? GS_SHARED : GS_GLOBAL;
  }
}

struct LaunchShape {
  unsigned grid, block;
  size_t smem;
};

template <typename K>
static mb_status shape_for(K kern, uint32_t warps, size_t smem, uint64_t units_per_warp_total, LaunchShape *ls,
                           uint32_t ctas_per_sm) {
  const DevInfo &di = dev_info();
  if (smem > (size_t)di.max_smem_optin)
    return fail(MB_ERR_INVALID, "launch needs %zu bytes of shared memory > %d", smem, di.max_smem_optin);
  MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, (int)(warps * 32), smem));
  if (occ < 1) return fail(MB_ERR_INVALID, "kernel does not fit on an SM (smem %zu)", smem);
  if (ctas_per_sm && (int)ctas_per_sm < occ) occ = (int)ctas_per_sm;
  uint64_t grid = (uint64_t)di.sms * occ;
  const uint64_t need = (units_per_warp_total + warps - 1) / warps;
  if (grid > need) grid = need ? need : 1;
  ls->grid = (unsigned)grid;
  ls->block = warps * 32;
  ls->smem = smem;
  return MB_OK;
}

template <int V, bool CHK, int GS>
static mb_status launch_fused(const DevPrg &P, const mb_op &O, uint32_t nr_grp, uint32_t hcap, int64_t *out,
                              uint64_t *nqual, uint32_t warps, uint32_t cps, cudaStream_t st) {
  auto kern = vbp_grpby_kernel<V, CHK, GS>;
  const size_t gbytes = (grp_smem_bytes(GS, nr_grp, hcap) + 15) & ~(size_t)15;
  const size_t smem = gbytes + (size_t)warps * (32 * V * 32) * 2;
  const uint64_t ntiles = (P.nwords + 32 * V - 1) / (32 * V);
  LaunchShape ls;
  MB_CHECK(shape_for(kern, warps, smem, ntiles, &ls, cps));
  kern<<<ls.grid, ls.block, ls.smem, st>>>(P, O, nr_grp, hcap, reinterpret_cast<unsigned long long *>(out),
                                           reinterpret_cast<unsigned long long *>(nqual));
  MB_LAUNCH_CHECK("vbp_grpby_kernel");
  return MB_OK;
}

template <int V, bool CHK>
static mb_status fused_gs(int gs, const DevPrg &P, const mb_op &O, uint32_t nr_grp, uint32_t hcap, int64_t *out,
                          uint64_t *nqual, uint32_t warps, uint32_t cps, cudaStream_t st) {
  switch (gs) {
  case GS_SCALAR: return launch_fused<V, CHK, GS_SCALAR>(P, O, nr_grp, hcap, out, nqual, warps, cps, st);
  case GS_SHARED: return launch_fused<V, CHK, GS_SHARED>(P, O, nr_grp, hcap, out, nqual, warps, cps, st);
  case GS_GLOBAL: return launch_fused<V, CHK, GS_GLOBAL>(P, O, nr_grp, hcap, out, nqual, warps, cps, st);
  default: return launch_fused<V, CHK, GS_HASH>(P, O, nr_grp, hcap, out, nqual, warps, cps, st);
  }
}

}  // namespace mb

using namespace mb;

namespace mb {
mb_status fused_grpby(const mb_vprg *p, const mb_op *op, uint32_t nr_grp, int64_t *out, uint64_t *nqual,
                      const mb_launch *launch, cudaStream_t st, bool zero) {
  if (!out || !nqual) return fail(MB_ERR_INVALID, "mb_vprg_grpby: NULL output");
  if (nr_grp == 0) return fail(MB_ERR_INVALID, "mb_vprg_grpby: nr_grp == 0");
  const int chk = !mb_vprg_is_nochk(p);
  DevPrg P;
  bool v4 = false;
  MB_CHECK(flatten_prg(p, chk, &P, &v4));
  MB_CHECK(validate_op(op));
  if (P.nrows >= (1ull << 32)) return fail(MB_ERR_INVALID, "mb_vprg_grpby: %llu rows >= 2^32", (unsigned long long)P.nrows);
  if (zero) {
    MB_CUDA(cudaMemsetAsync(out, 0, (size_t)nr_grp * sizeof(int64_t), st));
    MB_CUDA(cudaMemsetAsync(nqual, 0, sizeof(uint64_t), st));
  }
  if (P.nrows == 0) return MB_OK;
  mb_launch L = launch ? *launch : mb_launch{0, 0, 0, 0, 0};
  const int gs = pick_gs(nr_grp, L.grp_strategy);
  const uint32_t warps = L.warps_per_cta ? L.warps_per_cta : 8;
  if (warps > 16 || warps == 0) return fail(MB_ERR_INVALID, "mb_vprg_grpby: warps_per_cta %u", warps);
  if (L.words_per_lane != 0 && L.words_per_lane != 1 && L.words_per_lane != 2 && L.words_per_lane != 4)
    return fail(MB_ERR_INVALID, "mb_vprg_grpby: words_per_lane %u", L.words_per_lane);
  const uint32_t hcap = DEFAULT_HCAP;
  if (L.staging == MB_STAGE_AUTO && fused_warp_applies(P, *op))
    return fused_warp(P, *op, nr_grp, gs, hcap, L.words_per_lane, L.warps_per_cta, out, nqual, L.ctas_per_sm, st);
  if (L.staging == MB_STAGE_TMA && fused_tma_applies(P, v4, *op)) {
    const mb_status r = fused_tma(P, *op, nr_grp, gs, hcap, L.words_per_lane, out, nqual, L.ctas_per_sm, st);
    if (r != MB_ERR_UNSUPPORTED) return r;  // else: too many bitmaps to stage, load directly
  }
  uint32_t V = L.words_per_lane ? L.words_per_lane : 4;
  if (!v4) V = 1;  // unaligned bitmaps: scalar loads
  if (V == 4) return chk ? fused_gs<4, true>(gs, P, *op, nr_grp, hcap, out, nqual, warps, L.ctas_per_sm, st)
                         : fused_gs<4, false>(gs, P, *op, nr_grp, hcap, out, nqual, warps, L.ctas_per_sm, st);
  if (V == 2) return chk ? fused_gs<2, true>(gs, P, *op, nr_grp, hcap, out, nqual, warps, L.ctas_per_sm, st)
                         : fused_gs<2, false>(gs, P, *op, nr_grp, hcap, out, nqual, warps, L.ctas_per_sm, st);
  return chk ? fused_gs<1, true>(gs, P, *op, nr_grp, hcap, out, nqual, warps, L.ctas_per_sm, st)
             : fused_gs<1, false>(gs, P, *op, nr_grp, hcap, out, nqual, warps, L.ctas_per_sm, st);
}
}  // namespace mb

extern "C" mb_status mb_vprg_grpby(const mb_vprg *p, const mb_op *op, uint32_t nr_grp, int64_t *out,
                                   uint64_t *nqual, const mb_launch *launch, void *stream) {
  return fused_grpby(p, op, nr_grp, out, nqual, launch, as_stream(stream), true);
}

// The clause that screens rows in the no-index scan: the first whose terms
// read fact columns only (one load a row), else the first; nclause if none.
static uint32_t screen_clause(const mb_op &O, uint32_t *t0) {
  uint32_t t = 0, first_t = 0;
  for (uint32_t c = 0; c < O.nclause; ++c) {
    bool fact = true;
    for (uint32_t k = 0; k < O.clause_len[c]; ++k)
      if (O.src[O.terms[t + k].src].fk) fact = false;
    if (fact) {
      *t0 = t;
      return c;
    }
    t += O.clause_len[c];
  }
  *t0 = first_t;
  return 0;
}

template <int GS, int SW>
static mb_status launch_join_sw(uint64_t n, const mb_op &O, uint32_t nr_grp, uint32_t hcap, int64_t *out,
                                uint64_t *nqual, cudaStream_t st, uint32_t screen, uint32_t t0) {
  auto kern = join_grpby_kernel<GS, SW>;
  const uint32_t warps = 8;
  const size_t gb = (grp_smem_bytes(GS, nr_grp, hcap) + 15) & ~(size_t)15;
  // the row queues only where they cost no resident CTA (a large group
  // table in shared memory can leave no room for them)
  const size_t qbytes = (size_t)warps * JQ * 4;
  if (screen < O.nclause) {
    const size_t cap = (size_t)dev_info().max_smem_optin - 1024;  // room for the kernel's static shared memory
    int with = 0, without = 0;
    MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::min(cap, gb + qbytes)));
    if (gb + qbytes <= cap)
      MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&with, kern, (int)(warps * 32), gb + qbytes));
    MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&without, kern, (int)(warps * 32), gb));
    if (with < without) screen = O.nclause;
  }
  const size_t smem = gb + (screen < O.nclause ? qbytes : 0);
  LaunchShape ls;
  MB_CHECK(shape_for(kern, warps, smem, (n + 31) / 32, &ls, 0));
  kern<<<ls.grid, ls.block, ls.smem, st>>>(n, O, nr_grp, hcap, (uint32_t)gb, screen, t0,
                                           reinterpret_cast<unsigned long long *>(out),
                                           reinterpret_cast<unsigned long long *>(nqual));
  MB_LAUNCH_CHECK("join_grpby_kernel");
  return MB_OK;
}

// The screen's shape picks the kernel: one range on a 16-byte-aligned fact
// column screens four rows a lane (its width a template argument).
template <int GS>
static mb_status launch_join(uint64_t n, const mb_op &O, uint32_t nr_grp, uint32_t hcap, int64_t *out,
                             uint64_t *nqual, cudaStream_t st) {
  uint32_t t0 = 0;
  const uint32_t screen = screen_clause(O, &t0);
  uint32_t sw = 0;
  if (screen < O.nclause && O.clause_len[screen] == 1) {
    const mb_src &s = O.src[O.terms[t0].src];
    if (!s.fk && (reinterpret_cast<uintptr_t>(s.col) & 15) == 0) sw = s.width;
  }
  switch (sw) {
  case 1: return launch_join_sw<GS, 1>(n, O, nr_grp, hcap, out, nqual, st, screen, t0);
  case 2: return launch_join_sw<GS, 2>(n, O, nr_grp, hcap, out, nqual, st, screen, t0);
  case 4: return launch_join_sw<GS, 4>(n, O, nr_grp, hcap, out, nqual, st, screen, t0);
  case 8: return launch_join_sw<GS, 8>(n, O, nr_grp, hcap, out, nqual, st, screen, t0);
  default: return launch_join_sw<GS, 0>(n, O, nr_grp, hcap, out, nqual, st, screen, t0);
  }
}

extern "C" mb_status mb_join_grpby(uint64_t nrows, const mb_op *op, uint32_t nr_grp, int64_t *out,
                                   uint64_t *nqual, void *stream) {
  if (!out || !nqual) return fail(MB_ERR_INVALID, "mb_join_grpby: NULL output");
  if (nr_grp == 0) return fail(MB_ERR_INVALID, "mb_join_grpby: nr_grp == 0");
  MB_CHECK(validate_op(op));
  if (nrows >= (1ull << 32)) return fail(MB_ERR_INVALID, "mb_join_grpby: rows >= 2^32");
  cudaStream_t st = as_stream(stream);
  MB_CUDA(cudaMemsetAsync(out, 0, (size_t)nr_grp * sizeof(int64_t), st));
  MB_CUDA(cudaMemsetAsync(nqual, 0, sizeof(uint64_t), st));
  if (nrows == 0) return MB_OK;
  const int gs = pick_gs(nr_grp, MB_GRP_AUTO);
  switch (gs) {
  case GS_SCALAR: return launch_join<GS_SCALAR>(nrows, *op, nr_grp, DEFAULT_HCAP, out, nqual, st);
  case GS_SHARED: return launch_join<GS_SHARED>(nrows, *op, nr_grp, DEFAULT_HCAP, out, nqual, st);
  default: return launch_join<GS_GLOBAL>(nrows, *op, nr_grp, DEFAULT_HCAP, out, nqual, st);
  }
}

extern "C" mb_status mb_vprg_eval(const mb_vprg *p, int chk, uint32_t *possible, uint32_t *uncertain,
                                  uint64_t *popcount, void *stream) {
  if (!possible) return fail(MB_ERR_INVALID, "mb_vprg_eval: possible is NULL");
  DevPrg P;
  bool v4 = false;
  MB_CHECK(flatten_prg(p, chk, &P, &v4));
  if (((uintptr_t)possible & 15) || ((uintptr_t)uncertain & 15)) v4 = false;
  if (P.nrows == 0) return MB_OK;
  cudaStream_t st = as_stream(stream);
  const uint64_t nvec = v4 ? (P.nwords + 3) / 4 : P.nwords;
  uint64_t grid = (nvec + 255) / 256, cap = (uint64_t)dev_info().sms * 8;
  if (grid > cap) grid = cap;
  unsigned long long *pc = reinterpret_cast<unsigned long long *>(popcount);
  if (v4) {
    if (chk) vbp_eval_kernel<4, true><<<(unsigned)grid, 256, 0, st>>>(P, possible, uncertain, pc);
    else vbp_eval_kernel<4, false><<<(unsigned)grid, 256, 0, st>>>(P, possible, uncertain, pc);
  } else {
    if (chk) vbp_eval_kernel<1, true><<<(unsigned)grid, 256, 0, st>>>(P, possible, uncertain, pc);
    else vbp_eval_kernel<1, false><<<(unsigned)grid, 256, 0, st>>>(P, possible, uncertain, pc);
  }
  MB_LAUNCH_CHECK("vbp_eval_kernel");
  return MB_OK;
}

namespace mb {
// Segment-offset scratch of mb_bitmap_to_rows: one grow-only buffer per device.
static uint32_t *seg_scratch(uint64_t nseg) {
  static uint32_t *bufs[64] = {nullptr};
  static uint64_t caps[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return nullptr;
  if (caps[dev] < nseg) {
    if (bufs[dev]) cudaFree(bufs[dev]);
    bufs[dev] = nullptr;
    caps[dev] = 0;
    uint64_t cap = nseg < 4096 ? 4096 : nseg;
    if (cudaMalloc(&bufs[dev], cap * sizeof(uint32_t)) != cudaSuccess) return nullptr;
    caps[dev] = cap;
  }
  return bufs[dev];
}
}  // namespace mb

extern "C" mb_status mb_bitmap_to_rows(const uint32_t *possible, const uint32_t *uncertain, uint64_t nrows,
                                       uint32_t *rows, uint64_t *count, void *stream) {
  if (!possible || !rows || !count) return fail(MB_ERR_INVALID, "mb_bitmap_to_rows: NULL argument");
  if (nrows >= (1ull << 31)) return fail(MB_ERR_INVALID, "mb_bitmap_to_rows: row ids must be < 2^31");
  cudaStream_t st = as_stream(stream);
  if (nrows == 0) {
    MB_CUDA(cudaMemsetAsync(count, 0, sizeof(uint64_t), st));
    return MB_OK;
  }
  const uint64_t nwords = (nrows + 31) / 32;
  const uint64_t nseg = (nwords + RL_SEG_WORDS - 1) / RL_SEG_WORDS;
  uint32_t *seg = seg_scratch(nseg);
  if (!seg) return fail(MB_ERR_OOM, "mb_bitmap_to_rows: scratch allocation failed");
  rows_count_kernel<<<(unsigned)nseg, RL_THREADS, 0, st>>>(possible, nrows, seg);
  MB_LAUNCH_CHECK("rows_count_kernel");
  rows_scan_kernel<<<1, 1024, 0, st>>>(seg, nseg, reinterpret_cast<unsigned long long *>(count));
  MB_LAUNCH_CHECK("rows_scan_kernel");
  rows_write_kernel<<<(unsigned)nseg, RL_THREADS, 0, st>>>(possible, uncertain, nrows, seg, rows);
  MB_LAUNCH_CHECK("rows_write_kernel");
  return MB_OK;
}

template <int GS>
static mb_status launch_rows(const uint32_t *rows, const uint64_t *count, uint64_t cap, const mb_op &O,
                             uint32_t nr_grp, uint32_t hcap, int64_t *out, uint64_t *nqual, cudaStream_t st) {
  auto kern = rows_grpby_kernel<GS>;
  const uint32_t warps = 8;
  const size_t smem = (grp_smem_bytes(GS, nr_grp, hcap) + 15) & ~(size_t)15;
  LaunchShape ls;
  MB_CHECK(shape_for(kern, warps, smem, (cap + 31) / 32, &ls, 0));
  kern<<<ls.grid, ls.block, ls.smem, st>>>(rows, reinterpret_cast<const unsigned long long *>(count), cap, O,
                                           nr_grp, hcap, reinterpret_cast<unsigned long long *>(out),
                                           reinterpret_cast<unsigned long long *>(nqual));
  MB_LAUNCH_CHECK("rows_grpby_kernel");
  return MB_OK;
}

extern "C" mb_status mb_rows_grpby(const uint32_t *rows, const uint64_t *count, uint64_t capacity,
                                   const mb_op *op, uint32_t nr_grp, int64_t *out, uint64_t *nqual,
                                   void *stream) {
  if (!rows || !count || !out || !nqual) return fail(MB_ERR_INVALID, "mb_rows_grpby: NULL argument");
  if (nr_grp == 0) return fail(MB_ERR_INVALID, "mb_rows_grpby: nr_grp == 0");
  MB_CHECK(validate_op(op));
  cudaStream_t st = as_stream(stream);
  MB_CUDA(cudaMemsetAsync(out, 0, (size_t)nr_grp * sizeof(int64_t), st));
  MB_CUDA(cudaMemsetAsync(nqual, 0, sizeof(uint64_t), st));
  if (capacity == 0) return MB_OK;
  const int gs = pick_gs(nr_grp, MB_GRP_AUTO);
  switch (gs) {
  case GS_SCALAR: return launch_rows<GS_SCALAR>(rows, count, capacity, *op, nr_grp, DEFAULT_HCAP, out, nqual, st);
  case GS_SHARED: return launch_rows<GS_SHARED>(rows, count, capacity, *op, nr_grp, DEFAULT_HCAP, out, nqual, st);
  default: return launch_rows<GS_GLOBAL>(rows, count, capacity, *op, nr_grp, DEFAULT_HCAP, out, nqual, st);
  }
}

// ------------------------------------------- row list without allocation
// mb_bitmap_to_rows keeps its per-segment offsets in a library-allocated
// buffer.  This variant keeps them in a fixed array compiled into the
// library, for callers that must not allocate device memory.  The array is
// shared by every call on a device and keeps whatever the previous call left
// in it; the count kernel overwrites every entry the scan and write kernels
// later read, so nothing has to be cleared between calls.
namespace mb {
constexpr uint64_t NOALLOC_MAX_SEGMENTS = MB_NOALLOC_MAX_ROWS / (RL_SEG_WORDS * 32ull);
static __device__ __align__(256) uint32_t g_noalloc_seg[NOALLOC_MAX_SEGMENTS];

// Device address of g_noalloc_seg on the current device, looked up once per
// device.  The name g_noalloc_seg in host code is only a host-side handle,
// never a device address, so it is never passed to a kernel directly.
static mb_status noalloc_scratch(uint32_t **out) {
  static std::mutex mu;
  static uint32_t *addr[64] = {nullptr};
  int dev = 0;
  MB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(MB_ERR_INVALID, "mb_bitmap_to_rows_noalloc: device %d out of range", dev);
  std::lock_guard<std::mutex> lk(mu);
  if (!addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_seg);
    if (e != cudaSuccess) return cuda_fail(e, "mb_bitmap_to_rows_noalloc: cudaGetSymbolAddress");
    addr[dev] = static_cast<uint32_t *>(p);
  }
  *out = addr[dev];
  return MB_OK;
}
}  // namespace mb

extern "C" mb_status mb_bitmap_to_rows_noalloc(const uint32_t *possible, const uint32_t *uncertain,
                                               uint64_t nrows, uint32_t *rows, uint64_t *count, void *stream) {
  if (!possible || !rows || !count) return fail(MB_ERR_INVALID, "mb_bitmap_to_rows_noalloc: NULL argument");
  if (nrows > MB_NOALLOC_MAX_ROWS)
    return fail(MB_ERR_INVALID, "mb_bitmap_to_rows_noalloc: %llu rows exceed the fixed limit of %llu rows",
                (unsigned long long)nrows, (unsigned long long)MB_NOALLOC_MAX_ROWS);
  uint32_t *seg = nullptr;
  MB_CHECK(noalloc_scratch(&seg));
  cudaStream_t st = as_stream(stream);
  if (nrows == 0) {
    MB_CUDA(cudaMemsetAsync(count, 0, sizeof(uint64_t), st));
    return MB_OK;
  }
  const uint64_t nwords = (nrows + 31) / 32;
  const uint64_t nseg = (nwords + RL_SEG_WORDS - 1) / RL_SEG_WORDS;
  rows_count_kernel<<<(unsigned)nseg, RL_THREADS, 0, st>>>(possible, nrows, seg);
  MB_LAUNCH_CHECK("rows_count_kernel");
  rows_scan_kernel<<<1, 1024, 0, st>>>(seg, nseg, reinterpret_cast<unsigned long long *>(count));
  MB_LAUNCH_CHECK("rows_scan_kernel");
  rows_write_kernel<<<(unsigned)nseg, RL_THREADS, 0, st>>>(possible, uncertain, nrows, seg, rows);
  MB_LAUNCH_CHECK("rows_write_kernel");
  return MB_OK;
}

// ------------------------------------------------------- hash-join plan
// Crystal-style join plan (the reference's comparison system, crystal/src/ssb/q21.cu and
// its siblings: build a hash table per filtered dimension, then one pass over the fact rows
// probes them).  For every foreign key whose dimension attributes carry a predicate of their
// own (a clause all of whose terms read that dimension), the dimension rows passing those
// clauses go into an open-addressing table keyed by dimension key and carrying the
// attributes the op reads; the probe pass evaluates the fact-column clauses first, then looks
// each key up (a miss eliminates the row), then the remaining clauses, group key and value.
// Tables up to HJ_SMEM_MAX bytes are copied into every CTA's shared memory.  Results equal
// mb_join_grpby's on the same op.
namespace mb {

constexpr uint32_t HJ_MAXT = 4;                 // tables (distinct foreign keys) per op
constexpr uint32_t HJ_PAY = 3;                  // attributes one entry carries
constexpr uint32_t HJ_SMEM_MAX = 48 * 1024;     // per staged table
constexpr uint32_t HJ_SMEM_TOTAL = 128 * 1024;  // all staged tables

struct HjTable {
  const uint32_t *fk;
  uint64_t dimsz;
  uint4 *slots;       // {key, a0, a1, a2}; key HASH_EMPTY = free
  uint32_t mask;      // capacity - 1
  uint32_t npay;
  uint32_t pushed;    // clauses evaluated at the build
  uint32_t smem_off;  // byte offset of the staged copy, or ~0u
  uint32_t pay_src[HJ_PAY];
};

struct HjPlan {
  uint32_t ntab;
  HjTable tab[HJ_MAXT];
  int32_t src_tab[MB_MAXSRC];   // table carrying source s, -1: read directly
  uint32_t src_pay[MB_MAXSRC];  // its slot in the entry
  uint32_t fact_clauses;        // probe clauses that read fact columns only
  uint32_t late_clauses;        // the other probe clauses
  uint32_t term0[MB_MAXCLAUSE]; // first term of each clause
  uint32_t smem_tables;         // bytes of the staged tables (the row queues follow)
};

// Clauses `mask` on dimension row d of table t (sources read at index d).
__device__ __forceinline__ bool hj_dim_pass(const mb_op &O, const HjPlan &H, uint32_t mask, uint64_t d) {
  for (uint32_t c = 0; c < O.nclause; ++c) {
    if (!(mask >> c & 1u)) continue;
    bool any = false;
    for (uint32_t k = 0, t = H.term0[c]; k < O.clause_len[c] && !any; ++k, ++t) {
      const mb_term &tm = O.terms[t];
      const uint64_t v = load_width(O.src[tm.src].col, d, O.src[tm.src].width);
      any = v >= tm.lo && v < tm.hi;
    }
    if (!any) return false;
  }
  return true;
}

__global__ void hj_count_kernel(const __grid_constant__ mb_op O, const __grid_constant__ HjPlan H, uint32_t t,
                                unsigned long long *count) {
  const HjTable &T = H.tab[t];
  uint32_t c = 0;
  for (uint64_t d = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; d < T.dimsz; d += (uint64_t)gridDim.x * blockDim.x)
    c += hj_dim_pass(O, H, T.pushed, d) ? 1u : 0u;
  for (int o = 16; o; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count + t, (unsigned long long)c);
}

// Inserts the passing dimension rows of table t.  The walk from a key's hash
// slot ends within the table: it holds at most half as many rows as slots.
__global__ void hj_insert_kernel(const __grid_constant__ mb_op O, const __grid_constant__ HjPlan H, uint32_t t) {
  const HjTable &T = H.tab[t];
  for (uint64_t d = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; d < T.dimsz;
       d += (uint64_t)gridDim.x * blockDim.x) {
    if (!hj_dim_pass(O, H, T.pushed, d)) continue;
    uint32_t a[HJ_PAY] = {0, 0, 0};
    for (uint32_t j = 0; j < T.npay; ++j) {
      const mb_src &s = O.src[T.pay_src[j]];
      a[j] = (uint32_t)load_width(s.col, d, s.width);
    }
    uint32_t h = hash32((uint32_t)d) & T.mask;
    for (uint32_t p = 0; p <= T.mask; ++p, h = (h + 1) & T.mask)
      if (atomicCAS(&T.slots[h].x, HASH_EMPTY, (uint32_t)d) == HASH_EMPTY) {
        T.slots[h].y = a[0], T.slots[h].z = a[1], T.slots[h].w = a[2];
        break;
      }
  }
}

// Value of source s at `row`: a table's attribute, or a direct read (as
// src_value: false when a foreign key is out of its dimension).
__device__ __forceinline__ bool hj_value(const mb_op &O, const HjPlan &H, uint32_t s, uint32_t row,
                                         const uint32_t *got, uint64_t &v) {
  const int32_t t = H.src_tab[s];
  if (t >= 0) {
    v = got[t * HJ_PAY + H.src_pay[s]];
    return true;
  }
  return src_value(O.src[s], row, v);
}

__device__ __forceinline__ bool hj_clauses(const mb_op &O, const HjPlan &H, uint32_t mask, uint32_t row,
                                           const uint32_t *got) {
  for (uint32_t c = 0; c < O.nclause; ++c) {
    if (!(mask >> c & 1u)) continue;
    bool any = false;
    for (uint32_t k = 0, t = H.term0[c]; k < O.clause_len[c] && !any; ++k, ++t) {
      const mb_term &tm = O.terms[t];
      uint64_t v;
      any = hj_value(O, H, tm.src, row, got, v) && v >= tm.lo && v < tm.hi;
    }
    if (!any) return false;
  }
  return true;
}

// The op on a row whose fact-column clauses already passed.
__device__ __forceinline__ bool hj_row(const mb_op &O, const HjPlan &H, const uint4 *const *tabs, uint32_t row,
                                       uint32_t nr_grp, int64_t &value, uint32_t &group) {
  uint32_t got[HJ_MAXT * HJ_PAY];
  for (uint32_t t = 0; t < H.ntab; ++t) {
    const HjTable &T = H.tab[t];
    const uint32_t key = __ldg(T.fk + row);
    uint32_t h = hash32(key) & T.mask;
    const uint4 *tab = tabs[t];
    for (;;) {  // at least half the slots are free: the walk ends
      const uint4 e = tab[h];
      if (e.x == key) {
        got[t * HJ_PAY + 0] = e.y, got[t * HJ_PAY + 1] = e.z, got[t * HJ_PAY + 2] = e.w;
        break;
      }
      if (e.x == HASH_EMPTY) return false;
      h = (h + 1) & T.mask;
    }
  }
  if (!hj_clauses(O, H, H.late_clauses, row, got)) return false;
  uint32_t g = 0;
  for (uint32_t k = 0; k < O.nkey; ++k) {
    const mb_key &kk = O.keys[k];
    uint64_t v;
    if (!hj_value(O, H, kk.src, row, got, v)) return false;
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
    if (!hj_value(O, H, O.va, row, got, a)) return false;
    value = (int64_t)a;
    break;
  case MB_V_MUL:
    if (!hj_value(O, H, O.va, row, got, a) || !hj_value(O, H, O.vb, row, got, b)) return false;
    value = (int64_t)(a * b);
    break;
  default:
    if (!hj_value(O, H, O.va, row, got, a) || !hj_value(O, H, O.vb, row, got, b)) return false;
    value = (int64_t)a - (int64_t)b;
    break;
  }
  group = g;
  return true;
}

template <int GS, int SW>
__global__ void __launch_bounds__(SW ? 256 : 512, SW ? 4 : 1)
hj_probe_kernel(uint64_t nrows, const __grid_constant__ mb_op O, const __grid_constant__ HjPlan H, uint32_t nr_grp,
                uint32_t hcap, uint32_t grp_bytes, uint32_t t0, unsigned long long *__restrict__ out,
                unsigned long long *__restrict__ nqual) {
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ uint64_t red[64];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  GrpCtx G = grp_init<GS>(smem, nr_grp, hcap, out);
  const uint4 *tabs[HJ_MAXT];
  for (uint32_t t = 0; t < HJ_MAXT; ++t) {
    tabs[t] = nullptr;
    if (t >= H.ntab) continue;
    const HjTable &T = H.tab[t];
    if (T.smem_off == ~0u) {
      tabs[t] = T.slots;
      continue;
    }
    uint4 *dst = reinterpret_cast<uint4 *>(smem + grp_bytes + T.smem_off);
    for (uint32_t i = threadIdx.x; i <= T.mask; i += blockDim.x) dst[i] = T.slots[i];
    tabs[t] = dst;
  }
  __syncthreads();
  int64_t acc = 0;
  uint64_t cnt = 0;
  // as the no-index scan: the fact-column clauses screen the rows one per
  // lane, the rows that pass queue per warp and full warps of them probe
  uint32_t *queue = reinterpret_cast<uint32_t *>(smem + grp_bytes + H.smem_tables) + (size_t)warp * JQ;
  uint32_t qn = 0;
  const uint32_t lt = (1u << lane) - 1u;
  auto drain = [&](uint32_t m) {
    bool kept = false;
    int64_t val = 0;
    uint32_t grp = 0;
    if (lane < m) kept = hj_row(O, H, tabs, queue[qn - m + lane], nr_grp, val, grp);
    cnt += kept ? 1u : 0u;
    aggregate<GS>(G, kept, grp, val, acc);
    qn -= m;
    __syncwarp();
  };
  if (SW == 0) {
    const uint64_t nchunks = (nrows + 31) / 32;
    for (uint64_t ch = (uint64_t)blockIdx.x * nw + warp; ch < nchunks; ch += (uint64_t)gridDim.x * nw) {
      const uint64_t row = ch * 32 + lane;
      const bool pass = row < nrows && hj_clauses(O, H, H.fact_clauses, (uint32_t)row, nullptr);
      const uint32_t bal = __ballot_sync(0xffffffffu, pass);
      if (pass) queue[qn + __popc(bal & lt)] = (uint32_t)row;
      qn += __popc(bal);
      __syncwarp();
      if (qn >= 32) drain(32);
    }
  } else {
    // the fact clauses are one range on an aligned column: four rows a lane
    // from one vector load, as the no-index scan screens
    const mb_term &tm = O.terms[t0];
    const void *col = O.src[tm.src].col;
    const uint64_t lo = tm.lo, hi = tm.hi, nch4 = (nrows + 127) / 128;
    for (uint64_t ch = (uint64_t)blockIdx.x * nw + warp; ch < nch4; ch += (uint64_t)gridDim.x * nw) {
      const uint64_t r = ch * 128 + 4 * lane;
      uint64_t v[4] = {0, 0, 0, 0};
      if (ch * 128 + 128 <= nrows) {
        load4<SW>(col, r, v);
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (r + j < nrows) v[j] = load_width(col, r + j, SW);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const bool pass = r + j < nrows && v[j] >= lo && v[j] < hi;
        const uint32_t bal = __ballot_sync(0xffffffffu, pass);
        if (pass) queue[qn + __popc(bal & lt)] = (uint32_t)(r + j);
        qn += __popc(bal);  // at most 31 + 128 < JQ
      }
      __syncwarp();
      while (qn >= 32) drain(32);
    }
  }
  if (qn) drain(qn);
  __syncthreads();
  grp_flush<GS>(G, nr_grp, acc, cnt, nqual, red);
}

template <int GS, int SW>
static mb_status launch_hj_sw(uint64_t n, const mb_op &O, const HjPlan &H, uint32_t smem_tables, uint32_t nr_grp,
                              int64_t *out, uint64_t *nqual, cudaStream_t st, uint32_t t0);

// The probe's screen shape picks the kernel: the fact clauses one range on a
// 16-byte-aligned fact column screen four rows a lane.
template <int GS>
static mb_status launch_hj(uint64_t n, const mb_op &O, const HjPlan &H, uint32_t smem_tables, uint32_t nr_grp,
                           int64_t *out, uint64_t *nqual, cudaStream_t st) {
  uint32_t sw = 0, t0 = 0;
  const uint32_t fc = H.fact_clauses;
  if (fc && !(fc & (fc - 1))) {
    const uint32_t c = (uint32_t)__builtin_ctz(fc);
    if (O.clause_len[c] == 1) {
      t0 = H.term0[c];
      const mb_src &s = O.src[O.terms[t0].src];
      if (!s.fk && (reinterpret_cast<uintptr_t>(s.col) & 15) == 0) sw = s.width;
    }
  }
  switch (sw) {
  case 1: return launch_hj_sw<GS, 1>(n, O, H, smem_tables, nr_grp, out, nqual, st, t0);
  case 2: return launch_hj_sw<GS, 2>(n, O, H, smem_tables, nr_grp, out, nqual, st, t0);
  case 4: return launch_hj_sw<GS, 4>(n, O, H, smem_tables, nr_grp, out, nqual, st, t0);
  case 8: return launch_hj_sw<GS, 8>(n, O, H, smem_tables, nr_grp, out, nqual, st, t0);
  default: return launch_hj_sw<GS, 0>(n, O, H, smem_tables, nr_grp, out, nqual, st, t0);
  }
}

template <int GS, int SW>
static mb_status launch_hj_sw(uint64_t n, const mb_op &O, const HjPlan &H, uint32_t smem_tables, uint32_t nr_grp,
                              int64_t *out, uint64_t *nqual, cudaStream_t st, uint32_t t0) {
  auto kern = hj_probe_kernel<GS, SW>;
  const uint32_t warps = 8;
  const size_t grp_bytes = (grp_smem_bytes(GS, nr_grp, DEFAULT_HCAP) + 15) & ~(size_t)15;
  LaunchShape ls;
  MB_CHECK(shape_for(kern, warps, grp_bytes + smem_tables + (size_t)warps * JQ * 4, (n + 31) / 32, &ls, 0));
  kern<<<ls.grid, ls.block, ls.smem, st>>>(n, O, H, nr_grp, DEFAULT_HCAP, (uint32_t)grp_bytes, t0,
                                           reinterpret_cast<unsigned long long *>(out),
                                           reinterpret_cast<unsigned long long *>(nqual));
  MB_LAUNCH_CHECK("hj_probe_kernel");
  return MB_OK;
}

}  // namespace mb

extern "C" mb_status mb_hash_join_grpby(uint64_t nrows, const mb_op *op, uint32_t nr_grp, int64_t *out,
                                        uint64_t *nqual, void *stream) {
  using namespace mb;
  if (!out || !nqual) return fail(MB_ERR_INVALID, "mb_hash_join_grpby: NULL output");
  if (nr_grp == 0) return fail(MB_ERR_INVALID, "mb_hash_join_grpby: nr_grp == 0");
  MB_CHECK(validate_op(op));
  if (nrows >= (1ull << 32)) return fail(MB_ERR_INVALID, "mb_hash_join_grpby: rows >= 2^32");
  const mb_op &O = *op;
  HjPlan H;
  memset(&H, 0, sizeof(H));
  for (uint32_t s = 0; s < MB_MAXSRC; ++s) H.src_tab[s] = -1;
  uint32_t t0 = 0;
  for (uint32_t c = 0; c < O.nclause; ++c) H.term0[c] = t0, t0 += O.clause_len[c];
  // clauses whose terms all read one foreign key's dimension go into that key's table
  uint32_t pushed_any = 0;
  for (uint32_t c = 0; c < O.nclause; ++c) {
    const uint32_t *fk = nullptr;
    bool one = O.clause_len[c] > 0;
    for (uint32_t k = 0; k < O.clause_len[c]; ++k) {
      const mb_src &s = O.src[O.terms[H.term0[c] + k].src];
      if (!s.fk || s.dimsz == 0 || s.width > 4 || (fk && s.fk != fk)) one = false;
      fk = s.fk;
    }
    if (!one) continue;
    uint32_t t = 0;
    while (t < H.ntab && H.tab[t].fk != fk) ++t;
    if (t == H.ntab) {
      if (H.ntab == HJ_MAXT) continue;  // more keys than tables: probe this clause directly
      H.tab[t].fk = fk;
      H.tab[t].dimsz = ~0ull;
      ++H.ntab;
    }
    H.tab[t].pushed |= 1u << c;
    pushed_any |= 1u << c;
  }
  // each table carries every source on its key (the op may read them later)
  for (uint32_t t = 0; t < H.ntab; ++t) {
    HjTable &T = H.tab[t];
    for (uint32_t s = 0; s < O.nsrc; ++s) {
      if (O.src[s].fk != T.fk) continue;
      if (O.src[s].width > 4 || T.npay == HJ_PAY)
        return fail(MB_ERR_UNSUPPORTED, "mb_hash_join_grpby: more than %u attributes (or one over 4 bytes) on one key",
                    HJ_PAY);
      T.dimsz = std::min<uint64_t>(T.dimsz, O.src[s].dimsz ? O.src[s].dimsz : ~0ull);
      H.src_tab[s] = (int32_t)t;
      H.src_pay[s] = T.npay;
      T.pay_src[T.npay++] = s;
    }
  }
  for (uint32_t c = 0; c < O.nclause; ++c) {
    if (pushed_any >> c & 1u) continue;
    bool fact = true;
    for (uint32_t k = 0; k < O.clause_len[c]; ++k)
      if (O.src[O.terms[H.term0[c] + k].src].fk) fact = false;
    (fact ? H.fact_clauses : H.late_clauses) |= 1u << c;
  }
  cudaStream_t st = as_stream(stream);
  MB_CUDA(cudaMemsetAsync(out, 0, (size_t)nr_grp * sizeof(int64_t), st));
  MB_CUDA(cudaMemsetAsync(nqual, 0, sizeof(uint64_t), st));
  if (nrows == 0) return MB_OK;
  // build: count the passing dimension rows of every table (one wait), size
  // each table to a power of two >= 2 x its rows, insert
  uint64_t cnt[HJ_MAXT] = {0, 0, 0, 0};
  if (H.ntab) {
    Scratch sc(st);  // freed after the probe, in stream order
    unsigned long long *dcnt;
    MB_CHECK(sc.get(&dcnt, HJ_MAXT));
    MB_CUDA(cudaMemsetAsync(dcnt, 0, 8 * HJ_MAXT, st));
    for (uint32_t t = 0; t < H.ntab; ++t) {
      const unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(H.tab[t].dimsz, 256), (uint64_t)dev_info().sms * 8);
      hj_count_kernel<<<grid, 256, 0, st>>>(O, H, t, dcnt);
      MB_LAUNCH_CHECK("hj_count_kernel");
    }
    MB_CUDA(cudaMemcpyAsync(cnt, dcnt, 8 * HJ_MAXT, cudaMemcpyDeviceToHost, st));
    MB_CUDA(cudaStreamSynchronize(st));
    for (uint32_t t = 0; t < H.ntab; ++t)
      if (cnt[t] == 0) return MB_OK;  // a dimension with no passing row: nothing qualifies
    uint64_t off = 0, smem_tables = 0;
    uint64_t offs[HJ_MAXT];
    for (uint32_t t = 0; t < H.ntab; ++t) {
      if (cnt[t] > (1ull << 30))
        return fail(MB_ERR_UNSUPPORTED, "mb_hash_join_grpby: %llu dimension rows in one table (at most 2^30)",
                    (unsigned long long)cnt[t]);
      uint64_t capt = 64;
      while (capt < 2 * cnt[t]) capt <<= 1;
      H.tab[t].mask = (uint32_t)(capt - 1);
      offs[t] = off;
      off += capt * 16;
      H.tab[t].smem_off = ~0u;
      if (capt * 16 <= HJ_SMEM_MAX && smem_tables + capt * 16 <= HJ_SMEM_TOTAL) {
        H.tab[t].smem_off = (uint32_t)smem_tables;
        smem_tables += capt * 16;
      }
    }
    uint8_t *base;
    MB_CHECK(sc.get(&base, off));
    for (uint32_t t = 0; t < H.ntab; ++t) {
      H.tab[t].slots = reinterpret_cast<uint4 *>(base + offs[t]);
      MB_CUDA(cudaMemsetAsync(H.tab[t].slots, 0xff, (size_t)(H.tab[t].mask + 1) * 16, st));
    }
    for (uint32_t t = 0; t < H.ntab; ++t) {
      const unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(H.tab[t].dimsz, 256), (uint64_t)dev_info().sms * 8);
      hj_insert_kernel<<<grid, 256, 0, st>>>(O, H, t);
      MB_LAUNCH_CHECK("hj_insert_kernel");
    }
    H.smem_tables = (uint32_t)smem_tables;
    const int gs = pick_gs(nr_grp, MB_GRP_AUTO);
    mb_status r;
    switch (gs) {
    case GS_SCALAR: r = launch_hj<GS_SCALAR>(nrows, O, H, (uint32_t)smem_tables, nr_grp, out, nqual, st); break;
    case GS_SHARED: r = launch_hj<GS_SHARED>(nrows, O, H, (uint32_t)smem_tables, nr_grp, out, nqual, st); break;
    default: r = launch_hj<GS_GLOBAL>(nrows, O, H, (uint32_t)smem_tables, nr_grp, out, nqual, st); break;
    }
    return r;
  }
  // no table to build: the plain scan
  return mb_join_grpby(nrows, op, nr_grp, out, nqual, stream);
}
