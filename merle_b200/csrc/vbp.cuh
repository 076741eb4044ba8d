// vbp.cuh - device interpreter of the virtual bitmap program (VBP).
//
// Reference: struct vprg with nochk / chk (primitive.cuh:165-332).  The
// reference keeps its 3 (or 6) virtual registers per word in shared memory
// because the register index is only known at run time; here the program is
// uniform across the grid, so registers are plain variables selected by
// warp-uniform branches and never leave the register file.  Each lane
// evaluates V consecutive words (V = 4: one 128-bit load per bitmap), and the
// OR over an operand's bins issues its loads in batches of 8 so that each
// thread has up to 8 x 16 bytes in flight.
#pragma once
#include "common.cuh"

namespace mb {

// Flattened program, passed by value as a kernel parameter.
struct DevPrg {
  uint64_t nrows, nwords;
  uint32_t ninstr, chk;
  mb_instr ins[MB_MAXNINSTR];
  uint8_t off[MB_MAXCOLS];    // first pointer of operand c in ptr[]
  uint8_t nmid[MB_MAXCOLS];   // middle bins of operand c
  uint8_t nedge[MB_MAXCOLS];  // edge bins of operand c (after the middles)
  // Conjunctive form, when the program is a chain of conjuncts over distinct
  // operands (see flatten_prg): p = AND over operands of m_c or ~m_c (neg bit
  // c), u = OR of the edge bins of the positive operands, masked by p.
  uint8_t cnf;                // 1 if the conjunctive form applies
  uint8_t cmask;              // bit c: operand c is a conjunct
  uint8_t neg;                // bit c: operand c enters negated
  uint8_t ncnf;               // bitmaps in cnf_ptr
  uint8_t pad_[4];
  const uint32_t *ptr[MB_MAXPTRS];
  // The conjunctive chain flattened conjunct by conjunct: bitmap i of the
  // chain is cnf_ptr[i] with flags cnf_flag[i] (CNF_EDGE, CNF_END, CNF_NEG).
  const uint32_t *cnf_ptr[MB_MAXPTRS];
  uint8_t cnf_flag[MB_MAXPTRS];
};
enum { CNF_EDGE = 1, CNF_END = 2, CNF_NEG = 4 };

// Host: validates and flattens an mb_vprg.  vec4 = every bitmap pointer is
// 16-byte aligned (128-bit loads allowed).
mb_status flatten_prg(const mb_vprg *p, int chk, DevPrg *out, bool *vec4);
// Host: sets cnf / cmask / neg when the program is a conjunctive chain.
void detect_cnf(DevPrg *o);

template <int V>
__device__ __forceinline__ void vload(const uint32_t *p, uint64_t w0, uint64_t nwords, uint32_t (&o)[V]) {
  if (V == 4 && w0 + 4 <= nwords) {
    uint4 t = ld_stream4(p + w0);
    o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
  } else {
#pragma unroll
    for (int k = 0; k < V; ++k) o[k] = (w0 + k < nwords) ? __ldcs(p + w0 + k) : 0u;
  }
}

// OR of `cnt` bitmaps ptr[first .. first+cnt) at words [w0, w0+V).
template <int V>
__device__ __forceinline__ void or_bins(const DevPrg &P, int first, int cnt, uint64_t w0, uint32_t (&acc)[V]) {
#pragma unroll
  for (int k = 0; k < V; ++k) acc[k] = 0;
  int b = 0;
  for (; b + 8 <= cnt; b += 8) {
    uint32_t t[8][V];
#pragma unroll
    for (int j = 0; j < 8; ++j) vload<V>(P.ptr[first + b + j], w0, P.nwords, t[j]);
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
      for (int k = 0; k < V; ++k) acc[k] |= t[j][k];
  }
  for (; b + 2 <= cnt; b += 2) {
    uint32_t t0[V], t1[V];
    vload<V>(P.ptr[first + b], w0, P.nwords, t0);
    vload<V>(P.ptr[first + b + 1], w0, P.nwords, t1);
#pragma unroll
    for (int k = 0; k < V; ++k) acc[k] |= t0[k] | t1[k];
  }
  if (b < cnt) {
    uint32_t t0[V];
    vload<V>(P.ptr[first + b], w0, P.nwords, t0);
#pragma unroll
    for (int k = 0; k < V; ++k) acc[k] |= t0[k];
  }
}

template <int V>
struct Regs {
  uint32_t r[MB_NREGS][V];
};

// Copy register `idx` into `o` (idx is warp-uniform).
template <int V>
__device__ __forceinline__ void rget(const Regs<V> &R, uint32_t idx, uint32_t (&o)[V]) {
  switch (idx) {
  case 0: for (int k = 0; k < V; ++k) o[k] = R.r[0][k]; break;
  case 1: for (int k = 0; k < V; ++k) o[k] = R.r[1][k]; break;
  case 2: for (int k = 0; k < V; ++k) o[k] = R.r[2][k]; break;
  default: for (int k = 0; k < V; ++k) o[k] = R.r[3][k]; break;
  }
}
template <int V>
__device__ __forceinline__ void rset(Regs<V> &R, uint32_t idx, const uint32_t (&v)[V]) {
  switch (idx) {
  case 0: for (int k = 0; k < V; ++k) R.r[0][k] = v[k]; break;
  case 1: for (int k = 0; k < V; ++k) R.r[1][k] = v[k]; break;
  case 2: for (int k = 0; k < V; ++k) R.r[2][k] = v[k]; break;
  default: for (int k = 0; k < V; ++k) R.r[3][k] = v[k]; break;
  }
}

// Evaluates the program on words [w0, w0+V): possible bits in p, uncertain
// bits in u (CHK only).  Bits of rows >= nrows and words >= nwords are 0.
template <int V, bool CHK>
__device__ __forceinline__ void vbp_eval(const DevPrg &P, uint64_t w0, uint32_t (&p)[V], uint32_t (&u)[V]) {
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
#pragma unroll
      for (int k = 0; k < V; ++k) dp[k] &= sp[k];
      if (CHK) {
        rget(U, in.src1, su);
#pragma unroll
        for (int k = 0; k < V; ++k) du[k] = (du[k] | su[k]) & dp[k];
      }
      break;
    case MB_OR:
      rget(R, in.src1, sp);
      if (CHK) {
        rget(U, in.src1, su);
#pragma unroll
        for (int k = 0; k < V; ++k) du[k] = (du[k] & ~(sp[k] & ~su[k])) | (su[k] & ~dp[k]);
      }
#pragma unroll
      for (int k = 0; k < V; ++k) dp[k] |= sp[k];
      break;
    case MB_NOT:
      rget(R, in.src1, sp);
#pragma unroll
      for (int k = 0; k < V; ++k) dp[k] = ~sp[k];
      if (CHK && in.dstreg != in.src1) rget(U, in.src1, du);
      break;
    case MB_ANDM: {
      uint32_t any = 0;
#pragma unroll
      for (int k = 0; k < V; ++k) any |= dp[k];
      if (any == 0) break;  // all-zero destination: no loads (primitive.cuh:215,292)
      const int c = in.src1;
      uint32_t cm[V], ce[V];
      or_bins<V>(P, P.off[c], P.nmid[c], w0, cm);
      or_bins<V>(P, P.off[c] + P.nmid[c], P.nedge[c], w0, ce);
      if (CHK) {
#pragma unroll
        for (int k = 0; k < V; ++k) {
          // a zero destination word keeps its uncertain word (primitive.cuh:292)
          const uint32_t np = dp[k] & (ce[k] | cm[k]);
          du[k] = dp[k] ? ((du[k] | ce[k]) & np) : du[k];
          dp[k] = np;
        }
      } else {
#pragma unroll
        for (int k = 0; k < V; ++k) dp[k] &= (cm[k] | ce[k]);
      }
      break;
    }
    case MB_ORM: {
      const int c = in.src1;
      uint32_t cm[V], ce[V];
      or_bins<V>(P, P.off[c], P.nmid[c], w0, cm);
      or_bins<V>(P, P.off[c] + P.nmid[c], P.nedge[c], w0, ce);
      if (CHK) {
#pragma unroll
        for (int k = 0; k < V; ++k) du[k] = (du[k] & ~cm[k]) | (ce[k] & ~dp[k]);
      }
#pragma unroll
      for (int k = 0; k < V; ++k) dp[k] |= ce[k] | cm[k];
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
    const uint64_t w = w0 + k;
    uint32_t m = w < P.nwords ? 0xffffffffu : 0u;
    if (tail && w + 1 == P.nwords) m = (1u << tail) - 1u;
    p[k] = R.r[0][k] & m;
    u[k] = CHK ? (U.r[0][k] & m) : 0u;
  }
}

}  // namespace mb

namespace mb {
// The TMA-staged fused kernel (fused.cu).
bool fused_tma_applies(const DevPrg &P, bool vec4, const mb_op &O);
mb_status fused_tma(const DevPrg &P, const mb_op &O, uint32_t nr_grp, int gs, uint32_t hcap, uint32_t V,
                    int64_t *out, uint64_t *nq, uint32_t cps, cudaStream_t st);
}  // namespace mb

namespace mb {
// The warp-independent kernel for conjunctive programs (fused.cu).
bool fused_warp_applies(const DevPrg &P, const mb_op &O);
// Which op sources every row needs (keys, value) and which only uncertain
// rows need (filter terms).
struct OpNeeds {
  uint32_t kv_mask, filt_mask;
};
OpNeeds op_needs(const mb_op &O);
mb_status fused_warp(const DevPrg &P, const mb_op &O, uint32_t nr_grp, int gs, uint32_t hcap, uint32_t V,
                     uint32_t warps, int64_t *out, uint64_t *nq, uint32_t cps, cudaStream_t st);
}  // namespace mb
