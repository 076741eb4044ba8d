// refgpu.cu - test infrastructure: the reference's own GPU kernel for the
// fused query, vprg_grpby (primitive.cuh:340-445), with its SSB op functors
// s1op..s4op (ssb/lambdas.cuh:19-152), run on this machine's GPU over device
// columns and bitmaps the caller provides, so that the reference's kernel and
// this library's kernels can be compared on the same inputs and the same GPU.
// Compiled from the reference's headers by oracle/Makefile into
// oracle/_ref/librefgpu.so; only the tests load it.
//
// The launch and the timing loop are the reference's own (DOWORK,
// ssb/lambdas.cuh:154-243, cases 2 and 3): nt = 256 threads, vt = 3 words a
// thread without candidate checks, cp_vt = 2 with them, vt0 = 8, each of the
// `reps` repetitions a cudaMemset of the group array and one launch, the
// mean over the repetitions by CUDA events.  The group array lives in the
// kernel's static shared-memory union, so refgpu_query refuses a query whose
// group count does not fit it (the reference's SSB queries all do).
#include <cuda_runtime.h>
#include <stdint.h>
#include "primitive.cuh"
#include "ssb/lambdas.cuh"

namespace {
template <bool CHK, typename Op>
int run(const mybmpidx::vprg &p, uint32_t *out, uint32_t nr_grp, const Op &op, int reps, float *ms) {
  constexpr size_t vtx = CHK ? cp_vt : vt;
  constexpr size_t per_cta = nt * vtx * 32;  // rows a CTA covers
  constexpr size_t smem_words = (CHK ? 6 : 3) * nt * vtx;  // the union's idxbuf, the largest member
  if (nr_grp > smem_words) return 2;
  const unsigned grid = (unsigned)((p.factsz + per_cta - 1) / per_cta);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  // one untimed launch (module load), then the timed repetitions
  cudaMemset(out, 0, nr_grp * sizeof(uint32_t));
  mybmpidx::vprg_grpby<nt, vtx, vt0, CHK><<<grid, nt>>>(p, out, nr_grp, op);
  cudaEventRecord(a);
  for (int d = 0; d < reps; ++d) {
    cudaMemset(out, 0, nr_grp * sizeof(uint32_t));
    mybmpidx::vprg_grpby<nt, vtx, vt0, CHK><<<grid, nt>>>(p, out, nr_grp, op);
  }
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  cudaEventElapsedTime(ms, a, b);
  *ms /= reps;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

template <typename Op>
int run_any(const mybmpidx::vprg &p, uint32_t *out, uint32_t nr_grp, const Op &op, int reps, float *ms) {
  return p.is_nochk() ? run<false>(p, out, nr_grp, op, reps, ms) : run<true>(p, out, nr_grp, op, reps, ms);
}
}  // namespace

extern "C" {

// Device columns in the reference's ssb_schema widths (ssb/ssbdemo.h:41-49)
// and its dimension arrays (zero pad at key 0).
struct refgpu_cols {
  uint32_t *custkey, *partkey;
  uint16_t *orderdate;
  uint32_t *extendedprice, *revenue, *supplycost;
  uint8_t *quantity, *discount, *suppcity;
  uint8_t *custcity;
  uint16_t *partmfgr;
};

// One bitmap column of the program: up to 4 middle bins (the reference's
// MAXBIN_PERCOL) and the optional edge bins.
struct refgpu_col {
  uint32_t nmiddle;
  uint32_t *middle[4];
  uint32_t *leftmost, *rightmost;
};

// Query template tmpl (1..4) with the parameters p of s1op..s4op, over
// ncols program columns and ninstr (opcode, dst, src1, src2) instructions
// (primitive.cuh:169-187 numbering).  out: nr_grp device uint32 group sums.
// Returns 0, 1 for an argument outside the reference's limits, 2 for a group
// count above the kernel's shared-memory union, 3 for a CUDA error.
int refgpu_query(const refgpu_cols *c, uint32_t n, uint32_t tmpl, const uint32_t *p, const refgpu_col *cols,
                 uint32_t ncols, const uint8_t *instrs, uint32_t ninstr, uint32_t *out, uint32_t nr_grp, int reps,
                 float *ms) {
  using mybmpidx::vprg;
  if (ncols > mybmpidx::MAXCOLS || ninstr > mybmpidx::MAXNINSTR || tmpl < 1 || tmpl > 4 || reps < 1) return 1;
  vprg P{};
  P.factsz = n;
  for (uint32_t i = 0; i < ncols; ++i) {
    if (cols[i].nmiddle > mybmpidx::MAXBIN_PERCOL) return 1;
    for (uint32_t k = 0; k < cols[i].nmiddle; ++k) P.cols[i].middle[k] = cols[i].middle[k];
    P.cols[i].leftmost = cols[i].leftmost;
    P.cols[i].rightmost = cols[i].rightmost;
  }
  for (uint32_t i = 0; i < ninstr; ++i) {
    const uint8_t op = instrs[4 * i], d = instrs[4 * i + 1], s1 = instrs[4 * i + 2];
    if (op < vprg::AND || op > vprg::ORM || d > 2) return 1;
    if ((op == vprg::ANDM || op == vprg::ORM) ? s1 >= ncols : s1 > 2) return 1;
    P.instrs[i].opcode = (vprg::ops)op;
    P.instrs[i].dstreg = d;
    P.instrs[i].src1 = s1;
    P.instrs[i].src2 = instrs[4 * i + 3];
  }
  if (tmpl == 1) {
    s1op o;
    o.dateMin = (uint16_t)p[0], o.dateMax = (uint16_t)p[1], o.loOrderDate = c->orderdate;
    o.discntMin = (uint8_t)p[2], o.discntMax = (uint8_t)p[3], o.loDiscount = c->discount;
    o.qtyMin = (uint8_t)p[4], o.qtyMax = (uint8_t)p[5], o.loQuantity = c->quantity;
    o.extendedPrice = c->extendedprice;
    return run_any(P, out, nr_grp, o, reps, ms);
  }
  if (tmpl == 2) {
    s2op o;
    o.loPartKey = c->partkey, o.pMfgrMin = (uint16_t)p[0], o.pMfgrMax = (uint16_t)p[1], o.partMfgr = c->partmfgr;
    o.sCityMin = (uint8_t)p[2], o.sCityMax = (uint8_t)p[3], o.loSuppCity = c->suppcity;
    o.loOrderDate = c->orderdate, o.loRevenue = c->revenue;
    return run_any(P, out, nr_grp, o, reps, ms);
  }
  if (tmpl == 3) {
    s3op o;
    o.loCustKey = c->custkey, o.cCityMin = (uint8_t)p[0], o.cCityMax = (uint8_t)p[1], o.custCity = c->custcity;
    o.sCityMin = (uint8_t)p[2], o.sCityMax = (uint8_t)p[3], o.loSuppCity = c->suppcity;
    o.dateMin = (uint16_t)p[4], o.dateMax = (uint16_t)p[5], o.loOrderDate = c->orderdate;
    o.loRevenue = c->revenue;
    return run_any(P, out, nr_grp, o, reps, ms);
  }
  s4op o;
  o.loCustKey = c->custkey, o.loPartKey = c->partkey;
  o.cCityMin = (uint8_t)p[0], o.cCityMax = (uint8_t)p[1], o.custCity = c->custcity;
  o.sCityMin = (uint8_t)p[2], o.sCityMax = (uint8_t)p[3], o.loSuppCity = c->suppcity;
  o.pMfgrMin = (uint16_t)p[4], o.pMfgrMax = (uint16_t)p[5], o.partMfgr = c->partmfgr;
  o.dateMin = (uint16_t)p[6], o.dateMax = (uint16_t)p[7], o.loOrderDate = c->orderdate;
  o.loRevenue = c->revenue, o.loSupplyCost = c->supplycost;
  return run_any(P, out, nr_grp, o, reps, ms);
}

}  // extern "C"
