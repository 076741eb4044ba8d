// engine.cu - resident star schema, canonical bitmap index, rule planner and
// single-query execution (mb_engine_*).
//
// Reference: the SSB drivers (ssb/fixedlayout.cu:34-186 building programs
// from a fixed index with col::from_bin / from_bin2, ssb/bmpidx-create.cu
// building that index) and the op functors s1op..s4op (ssb/lambdas.cuh:19-152).
// The planner generalises from_bin/from_bin2 (bmpidx_create.cu:138-226):
//  - an exact multi-level cover (coarsest bins first, e.g. years then months),
//  - the complement of an exact cover taken with NOT when it needs fewer bins
//    (the reference's Q3 date trick, ssb/fixedlayout.cu:93-98),
//  - otherwise edge bins with the candidate check (leftmost / rightmost),
// choosing by the bytes each option reads.
#include <string.h>
#include <algorithm>
#include <memory>
#include <unordered_map>
#include "batch.cuh"
#include "engine.h"
#include "vbp.cuh"

namespace mb {

// ------------------------------------------------------------ lifetime
Engine::~Engine() {
  if (device >= 0) cudaSetDevice(device);
  for (void *p : allocs) cudaFree(p);
  allocs.clear();
  if (h_out) cudaFreeHost(h_out);
  if (h_nqual) cudaFreeHost(h_nqual);
  for (int i = 0; i < BQ_RING; ++i) {
    if (bq_host[i]) cudaFreeHost(bq_host[i]);
    if (bq_copied[i]) cudaEventDestroy(bq_copied[i]);
  }
  for (cudaEvent_t ev : qev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : marks)
    if (ev) cudaEventDestroy(ev);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (stream) cudaStreamDestroy(stream);
  if (pstream) cudaStreamDestroy(pstream);
}

mb_status Engine::alloc(void **p, size_t bytes) {
  MB_CUDA(cudaMalloc(p, bytes < 256 ? 256 : bytes));
  allocs.push_back(*p);
  return MB_OK;
}

static void free_one(std::vector<void *> &allocs, void *p);

void Engine::drop_index() {
  have_tuned = false;
  for (auto &c : idx)
    for (auto &l : c.levels) l.slab = nullptr;
  free_one(allocs, islab);
  islab = nullptr;
  free_bmaps();
  nbm = 0;
  indexed = false;
}

void Engine::free_bmaps() {
  for (void *&m : bmaps) {
    free_one(allocs, m);
    m = nullptr;
  }
}

static void free_one(std::vector<void *> &allocs, void *p) {
  if (!p) return;
  auto it = std::find(allocs.begin(), allocs.end(), p);
  if (it != allocs.end()) allocs.erase(it);
  cudaFree(p);
}

void Engine::free_star() {
  void **cols[] = {&custkey, &partkey, &suppkey, &orderdate, &quantity, &discount, &extendedprice,
                   &revenue, &supplycost, &suppcity};
  for (void **c : cols) {
    free_one(allocs, *c);
    *c = nullptr;
  }
  free_one(allocs, custcity);
  free_one(allocs, suppcity_dim);
  free_one(allocs, partmfgr);
  custcity = suppcity_dim = nullptr;
  partmfgr = nullptr;
  free_denorm();
  for (auto &c : idx)
    for (auto &l : c.levels) l.slab = nullptr;
  free_one(allocs, islab);
  islab = nullptr;
  free_bmaps();
  nbm = 0;
  for (auto &c : idx) c.levels.clear();
  indexed = false;
}

mb_status Engine::ensure_out(uint32_t n) {
  if (n <= out_cap) return MB_OK;
  uint32_t cap = std::max<uint32_t>(n, 8192);
  free_one(allocs, d_out);
  free_one(allocs, d_nqual);
  if (h_out) cudaFreeHost(h_out);
  if (h_nqual) cudaFreeHost(h_nqual);
  h_out = nullptr;
  h_nqual = nullptr;
  MB_CHECK(alloc((void **)&d_out, (size_t)cap * 8));
  MB_CHECK(alloc((void **)&d_nqual, 64 * 8));
  MB_CUDA(cudaMallocHost(&h_out, (size_t)cap * 8));
  MB_CUDA(cudaMallocHost(&h_nqual, 64 * 8));
  out_cap = cap;
  return MB_OK;
}

mb_status Engine::ensure_tmp(uint64_t words) {
  if (words <= tmp_words) return MB_OK;
  free_one(allocs, tmp_bits);
  tmp_bits = nullptr;
  MB_CHECK(alloc((void **)&tmp_bits, words * 4));
  tmp_words = words;
  return MB_OK;
}

mb_status Engine::ensure_rows(uint64_t n) {
  if (n <= rows_cap) return MB_OK;
  free_one(allocs, rows);
  rows = nullptr;
  MB_CHECK(alloc((void **)&rows, n * 4));
  rows_cap = n;
  return MB_OK;
}

uint32_t Engine::fact_width(const char *col) const {
  if (width4) return 4;
  if (!strcmp(col, "orderdate")) return 2;
  if (!strcmp(col, "quantity") || !strcmp(col, "discount") || !strcmp(col, "suppcity")) return 1;
  return 4;
}

// ------------------------------------------------------------ index layout
static std::vector<uint64_t> range_bounds(uint64_t lo, uint64_t hi, uint64_t step) {
  std::vector<uint64_t> b;
  for (uint64_t x = lo; x < hi; x += step) b.push_back(x);
  b.push_back(hi);
  return b;
}

static std::vector<uint64_t> year_bounds() { return {0, 366, 731, 1096, 1461, 1827, 2192, 2557}; }

static std::vector<uint64_t> month_bounds() {
  static const int dm[12] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
  std::vector<uint64_t> b;
  uint64_t d = 0;
  for (int y = 1992; y < 1999; ++y)
    for (int m = 0; m < 12; ++m) {
      b.push_back(d);
      d += dm[m] + ((m == 1 && y % 4 == 0) ? 1 : 0);
    }
  b.push_back(d);  // 2557 = 1999-01-01
  return b;
}

static mb_src fact_src(const void *col, uint32_t w) {
  mb_src s;
  memset(&s, 0, sizeof(s));
  s.col = col;
  s.width = w;
  return s;
}

static mb_src join_src(const void *dim, const void *fk, uint64_t dimsz, uint32_t w) {
  mb_src s;
  memset(&s, 0, sizeof(s));
  s.col = dim;
  s.fk = reinterpret_cast<const uint32_t *>(fk);
  s.dimsz = dimsz;
  s.width = w;
  return s;
}

mb_src Engine::ccity_src() const {
  return custcity_row ? fact_src(custcity_row, 1) : join_src(custcity, custkey, ncust + 1, 1);
}

mb_src Engine::mfgr_src() const {
  return partmfgr_row ? fact_src(partmfgr_row, 2) : join_src(partmfgr, partkey, npart + 1, 2);
}

void Engine::free_denorm() {
  free_one(allocs, custcity_row);
  free_one(allocs, partmfgr_row);
  custcity_row = nullptr;
  partmfgr_row = nullptr;
}

// custcity_row[r] = custcity[custkey[r]] and partmfgr_row[r] =
// partmfgr[partkey[r]], 0 where a key lies outside its dimension (counted in
// bad[0] / bad[1]).  Four rows a thread per step: one 16-byte load of each
// key column, eight dimension loads in flight, one 4-byte and one 8-byte
// store.
__global__ void denorm_kernel(const uint32_t *__restrict__ ck, const uint8_t *__restrict__ cdim, uint64_t csz,
                              const uint32_t *__restrict__ pk, const uint16_t *__restrict__ pdim, uint64_t psz,
                              uint8_t *__restrict__ cout, uint16_t *__restrict__ pout, uint64_t n,
                              unsigned long long *bad) {
  uint32_t bc = 0, bp = 0;
  const uint64_t n4 = n / 4, step = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (uint64_t i = g; i < n4; i += step) {
    const uint4 c = __ldcs(reinterpret_cast<const uint4 *>(ck) + i);
    const uint4 p = __ldcs(reinterpret_cast<const uint4 *>(pk) + i);
    const uint32_t cv[4] = {c.x, c.y, c.z, c.w}, pv[4] = {p.x, p.y, p.z, p.w};
    uint32_t co = 0, po[2] = {0, 0};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (cv[j] < csz) co |= (uint32_t)__ldg(cdim + cv[j]) << (8 * j);
      else ++bc;
      if (pv[j] < psz) po[j >> 1] |= (uint32_t)__ldg(pdim + pv[j]) << (16 * (j & 1));
      else ++bp;
    }
    reinterpret_cast<uint32_t *>(cout)[i] = co;
    reinterpret_cast<uint2 *>(pout)[i] = make_uint2(po[0], po[1]);
  }
  if (g < n - 4 * n4) {  // the last n % 4 rows
    const uint64_t r = 4 * n4 + g;
    const uint32_t c = ck[r], p = pk[r];
    cout[r] = c < csz ? cdim[c] : 0;
    pout[r] = p < psz ? pdim[p] : 0;
    bc += c >= csz;
    bp += p >= psz;
  }
  bc = __reduce_add_sync(0xffffffffu, bc);
  bp = __reduce_add_sync(0xffffffffu, bp);
  if ((threadIdx.x & 31) == 0) {
    if (bc) atomicAdd(bad, (unsigned long long)bc);
    if (bp) atomicAdd(bad + 1, (unsigned long long)bp);
  }
}

// The denormalised per-row columns (allocated by the caller), filled on
// stream st; d_bad (device, 2 counters) counts foreign keys outside their
// dimension.
mb_status Engine::enqueue_denorm(unsigned long long *d_bad, cudaStream_t st) {
  MB_CUDA(cudaMemsetAsync(d_bad, 0, 16, st));
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div(nrows, 1024), 148ull * 8));
  denorm_kernel<<<grid, 256, 0, st>>>(reinterpret_cast<const uint32_t *>(custkey), custcity, ncust + 1,
                                          reinterpret_cast<const uint32_t *>(partkey), partmfgr, npart + 1,
                                          custcity_row, partmfgr_row, nrows, d_bad);
  MB_LAUNCH_CHECK("denorm_kernel");
  return MB_OK;
}

// The denormalised columns, built and checked before returning; a foreign key
// outside its dimension leaves the probes in place instead.
mb_status Engine::build_denorm() {
  free_denorm();
  unsigned long long *d_bad = nullptr;
  MB_CHECK(alloc((void **)&d_bad, 16));
  MB_CHECK(alloc((void **)&custcity_row, nrows));
  MB_CHECK(alloc((void **)&partmfgr_row, nrows * 2));
  MB_CHECK(enqueue_denorm(d_bad, stream));
  unsigned long long bad[2] = {0, 0};
  MB_CUDA(cudaMemcpyAsync(bad, d_bad, 16, cudaMemcpyDeviceToHost, stream));
  MB_CUDA(cudaStreamSynchronize(stream));
  free_one(allocs, d_bad);
  if (bad[0] || bad[1]) free_denorm();
  return MB_OK;
}

mb_status Engine::setup_index_cols() {
  auto lv = [](std::vector<uint64_t> b) {
    Level l;
    l.bounds = std::move(b);
    return l;
  };
  IdxCol &d = idx[IC_DATE];
  d.name = "date";
  d.src = fact_src(orderdate, fact_width("orderdate"));
  d.dom_lo = 0, d.dom_hi = 2557;
  d.levels = {lv(year_bounds()), lv(month_bounds())};
  IdxCol &di = idx[IC_DISC];
  di.name = "discount";
  di.src = fact_src(discount, fact_width("discount"));
  di.dom_lo = 0, di.dom_hi = 11;
  di.levels = {lv(range_bounds(0, 11, 1))};
  IdxCol &q = idx[IC_QTY];
  q.name = "quantity";
  q.src = fact_src(quantity, fact_width("quantity"));
  q.dom_lo = 1, q.dom_hi = 51;
  q.levels = {lv(range_bounds(1, 51, 1))};
  IdxCol &cc = idx[IC_CCITY];
  cc.name = "custcity";
  cc.src = ccity_src();
  cc.dom_lo = 0, cc.dom_hi = 250;
  cc.levels = {lv(range_bounds(0, 250, 50)), lv(range_bounds(0, 250, 10))};
  IdxCol &sc = idx[IC_SCITY];
  sc.name = "suppcity";
  sc.src = fact_src(suppcity, fact_width("suppcity"));
  sc.dom_lo = 0, sc.dom_hi = 250;
  sc.levels = {lv(range_bounds(0, 250, 50)), lv(range_bounds(0, 250, 10))};
  IdxCol &m = idx[IC_MFGR];
  m.name = "partmfgr";
  m.src = mfgr_src();
  m.dom_lo = 0, m.dom_hi = 1000;
  m.levels = {lv(range_bounds(0, 1000, 200)), lv(range_bounds(0, 1000, 40))};
  // keep the levels of level_mask (bit i: the i-th level in column order)
  uint32_t bit = 0;
  for (auto &c : idx) {
    std::vector<Level> keep;
    for (auto &l : c.levels)
      if ((level_mask >> bit++) & 1u) keep.push_back(std::move(l));
    if (keep.empty()) return fail(MB_ERR_INVALID, "index: level mask 0x%x keeps no level of %s", level_mask, c.name);
    c.levels = std::move(keep);
  }
  return MB_OK;
}

// ------------------------------------------------------------ planner
// Level l's bin j starting exactly at x, or -1.
static int bin_at(const Level &L, uint64_t x) {
  auto it = std::lower_bound(L.bounds.begin(), L.bounds.end() - 1, x);
  if (it == L.bounds.end() - 1 || *it != x) return -1;
  return (int)(it - L.bounds.begin());
}

static const uint32_t *bin_ptr(const Level &L, int j, uint64_t stride) {
  return L.slab + (uint64_t)j * stride;
}

// Exact cover of [lo, hi) with the coarsest bins that fit (levels nest);
// with fine_only, with the finest level's bins alone.
static bool exact_cover(const IdxCol &c, uint64_t lo, uint64_t hi, uint64_t stride,
                        std::vector<const uint32_t *> &out, uint64_t &rows, bool fine_only = false) {
  uint64_t x = lo;
  while (x < hi) {
    bool found = false;
    for (size_t li = fine_only ? c.levels.size() - 1 : 0; li < c.levels.size(); ++li) {
      const Level &L = c.levels[li];
      int j = bin_at(L, x);
      if (j >= 0 && L.bounds[j + 1] <= hi) {
        out.push_back(bin_ptr(L, j, stride));
        rows += L.pop.empty() ? 0 : L.pop[j];
        x = L.bounds[j + 1];
        found = true;
        break;
      }
    }
    if (!found) return false;
  }
  return true;
}

Cover plan_cover(const IdxCol &c, uint64_t lo, uint64_t hi, uint64_t stride, int nchk_sources, uint64_t *cost_out,
                 uint32_t mode) {
  const bool fine = mode == MB_COVER_FINE, nocompl = mode == MB_COVER_NOCOMPL || fine, noedge = mode == MB_COVER_NOEDGE;
  Cover best;
  if (cost_out) *cost_out = 0;
  lo = std::max(lo, c.dom_lo);
  hi = std::min(hi, c.dom_hi);
  if (lo >= hi) {
    best.empty = true;
    return best;
  }
  if (lo == c.dom_lo && hi == c.dom_hi) {
    best.full = true;
    return best;
  }
  const uint64_t W = stride;  // bytes of one bitmap / 4 (padding is negligible)
  uint64_t best_cost = UINT64_MAX;
  // (a) exact direct cover
  {
    Cover cv;
    if (exact_cover(c, lo, hi, stride, cv.mid, cv.est_rows, fine)) {
      uint64_t cost = (uint64_t)cv.nb() * W * 4;
      if (cost < best_cost) best = cv, best_cost = cost;
    }
  }
  // (b) complement: NOT of the exact cover of [dom_lo, lo) u [hi, dom_hi)
  if (!nocompl) {
    Cover cv;
    uint64_t rows = 0;
    bool ok = true;
    if (c.dom_lo < lo) ok = exact_cover(c, c.dom_lo, lo, stride, cv.mid, rows);
    if (ok && hi < c.dom_hi) ok = exact_cover(c, hi, c.dom_hi, stride, cv.mid, rows);
    if (ok && !cv.mid.empty()) {
      cv.complement = true;
      uint64_t total = 0;
      for (uint64_t p : c.levels[0].pop) total += p;
      cv.est_rows = total > rows ? total - rows : 0;
      uint64_t cost = (uint64_t)cv.nb() * W * 4;
      if (cost < best_cost) best = cv, best_cost = cost;
    }
  }
  // (c) edge bins on the finest level around an exact inner cover (from_bin /
  // from_bin2 generalised); edge rows pay the candidate check
  {
    const Level &F = c.levels.back();
    const uint64_t *b = F.bounds.data();
    const int nb = (int)F.nbins();
    int l = (int)(std::upper_bound(b, b + nb + 1, lo) - b) - 1;      // bin holding lo
    int r = (int)(std::lower_bound(b, b + nb + 1, hi) - b) - 1;      // bin holding hi-1
    if (l >= 0 && r < nb && l <= r) {
      Cover cv;
      uint64_t ilo = b[l] == lo ? lo : b[l + 1];
      uint64_t ihi = b[r + 1] == hi ? hi : b[r];
      bool ok = true;
      if (l == r && (b[l] != lo || b[r + 1] != hi)) {
        cv.left = bin_ptr(F, l, stride);
        cv.edge_rows += F.pop.empty() ? 0 : F.pop[l];
      } else {
        if (b[l] != lo) {
          cv.left = bin_ptr(F, l, stride);
          cv.edge_rows += F.pop.empty() ? 0 : F.pop[l];
        }
        if (b[r + 1] != hi) {
          cv.right = bin_ptr(F, r, stride);
          cv.edge_rows += F.pop.empty() ? 0 : F.pop[r];
        }
        if (ilo < ihi) ok = exact_cover(c, ilo, ihi, stride, cv.mid, cv.est_rows, fine);
      }
      if (ok && cv.nb() > 0) {
        // the check gathers ~one 32-byte sector per filter source per edge row
        uint64_t cost = (uint64_t)cv.nb() * W * 4 + cv.edge_rows * 32ull * (uint64_t)nchk_sources;
        cv.est_rows += cv.edge_rows / 2;
        // without candidate checks, edges only where no exact cover exists
        if (noedge && best_cost != UINT64_MAX) cost = UINT64_MAX;
        if (cost < best_cost) best = cv, best_cost = cost;
      }
    }
  }
  if (cost_out) *cost_out = best_cost;
  return best;
}

// ------------------------------------------------------------ index-memory planner
// Cost in bytes of a workload's predicates under the levels of `mask` (the
// planner's cover costs), with the bin row counts of the built index.
static uint64_t workload_cost(const Engine &E, const std::vector<std::vector<Pred>> &preds, uint32_t mask,
                              bool *ok) {
  IdxCol cols[IC_N];
  uint32_t bit = 0;
  *ok = true;
  for (int c = 0; c < IC_N; ++c)
    cols[c].name = E.idx[c].name, cols[c].dom_lo = E.idx[c].dom_lo, cols[c].dom_hi = E.idx[c].dom_hi;
  // the engine's levels are the kept subset of the canonical list: walk the
  // canonical bits and pick the built levels in order
  for (int c = 0; c < IC_N; ++c) {
    const uint32_t nl = c == IC_DISC || c == IC_QTY ? 1u : 2u;  // canonical levels of the column
    uint32_t li = 0;
    for (uint32_t k = 0; k < nl; ++k, ++bit) {
      const bool built = (E.level_mask >> bit) & 1u;
      if (built && ((mask >> bit) & 1u)) cols[c].levels.push_back(E.idx[c].levels[li]);
      if (built) ++li;
    }
    if (cols[c].levels.empty()) *ok = false;
  }
  if (!*ok) return UINT64_MAX;
  uint64_t total = 0;
  for (const auto &ps : preds)
    for (const Pred &p : ps) {
      uint64_t cst = 0;
      plan_cover(cols[p.col], p.lo, p.hi, E.stride, 1, &cst);
      if (cst == UINT64_MAX) {
        *ok = false;
        return UINT64_MAX;
      }
      total += cst;
    }
  return total;
}

static uint64_t mask_bytes(const Engine &E, uint32_t mask) {
  static const uint32_t nbins[MB_INDEX_LEVELS] = {7, 84, 11, 50, 5, 25, 5, 25, 5, 25};
  uint64_t b = 0;
  for (uint32_t i = 0; i < MB_INDEX_LEVELS; ++i)
    if ((mask >> i) & 1u) b += (uint64_t)nbins[i] * E.stride * 4;
  return b;
}

uint32_t query_ngroups(const mb_query &q) {
  const uint32_t *p = q.p;
  auto years = [](uint32_t dmin, uint32_t dmax) -> uint32_t {
    if (dmax <= dmin) return 1;
    return date_to_year(dmax - 1) - date_to_year(dmin) + 1;
  };
  switch (q.tmpl) {
  case 1: return 1;
  case 2: return p[1] > p[0] ? 7 * (p[1] - p[0]) : 1;
  case 3: {
    uint32_t a = p[1] - p[0], b = p[3] - p[2];
    if (p[1] - p[0] >= 50) a = p[1] / 10 - p[0] / 10, b = p[3] / 10 - p[2] / 10;
    uint32_t g = a * b * years(p[4], p[5]);
    return g ? g : 1;
  }
  case 4: {
    uint32_t a = p[3] - p[2], b = p[5] - p[4];
    if (p[3] - p[2] >= 50) a = p[3] / 10 - p[2] / 10;
    if (p[5] - p[4] >= 200) b = p[5] / 40 - p[4] / 40;
    uint32_t g = a * b * years(p[6], p[7]);
    return g ? g : 1;
  }
  default: return 0;
  }
}

// The op functors s1op..s4op (ssb/lambdas.cuh:19-152) as mb_op.
struct OpB {
  mb_op o;
  uint32_t nt = 0;
  OpB() { memset(&o, 0, sizeof(o)); }
  uint32_t src(const mb_src &s) {
    o.src[o.nsrc] = s;
    return o.nsrc++;
  }
  void clause1(uint32_t s, uint64_t lo, uint64_t hi) {
    o.clause_len[o.nclause++] = 1;
    o.terms[nt].src = s, o.terms[nt].lo = lo, o.terms[nt].hi = hi;
    ++nt;
  }
  void key(uint32_t s, uint32_t xf, uint32_t div, uint32_t base, uint32_t mul) {
    mb_key &k = o.keys[o.nkey++];
    k.src = s, k.xform = xf, k.div = div, k.base = base, k.mul = mul;
  }
};

void ssb_build_op(const SsbSrc &S, const mb_query &q, mb_op &out) {
  OpB b;
  const uint32_t *p = q.p;
  if (q.tmpl == 1) {
    uint32_t sd = b.src(S.date), sdi = b.src(S.disc), sq = b.src(S.qty), se = b.src(S.eprice);
    b.clause1(sd, p[0], p[1]), b.clause1(sdi, p[2], p[3]), b.clause1(sq, p[4], p[5]);
    b.o.vkind = MB_V_MUL, b.o.va = se, b.o.vb = sdi;
  } else if (q.tmpl == 2) {
    uint32_t ss = b.src(S.scity), sm = b.src(S.mfgr), sd = b.src(S.date), sr = b.src(S.rev);
    b.clause1(ss, p[2], p[3]), b.clause1(sm, p[0], p[1]);
    b.key(sm, MB_X_ID, 1, p[0], 1);
    b.key(sd, MB_X_YEAR, 1, 0, p[1] - p[0]);
    b.o.vkind = MB_V_COL, b.o.va = sr;
  } else if (q.tmpl == 3) {
    uint32_t ss = b.src(S.scity), sd = b.src(S.date), sc = b.src(S.ccity), sr = b.src(S.rev);
    b.clause1(ss, p[2], p[3]), b.clause1(sd, p[4], p[5]), b.clause1(sc, p[0], p[1]);
    uint32_t cmn = p[0], cmx = p[1], smn = p[2], smx = p[3], xf = MB_X_ID, dv = 1;
    if (p[1] - p[0] >= 50) cmn /= 10, cmx /= 10, smn /= 10, smx /= 10, xf = MB_X_DIV, dv = 10;
    const uint32_t a = cmx - cmn, bb = smx - smn;
    b.key(sd, MB_X_YEAR, 1, date_to_year(p[4]), a * bb);
    b.key(sc, xf, dv, cmn, a);
    b.key(ss, xf, dv, smn, 1);
    b.o.vkind = MB_V_COL, b.o.va = sr;
  } else {
    uint32_t ss = b.src(S.scity), sd = b.src(S.date), sc = b.src(S.ccity), sm = b.src(S.mfgr), sr = b.src(S.rev);
    uint32_t sk = b.src(S.scost);
    b.clause1(ss, p[2], p[3]), b.clause1(sd, p[6], p[7]), b.clause1(sc, p[0], p[1]), b.clause1(sm, p[4], p[5]);
    uint32_t smn = p[2], smx = p[3], sxf = MB_X_ID, sdv = 1;
    if (p[3] - p[2] >= 50) smn /= 10, smx /= 10, sxf = MB_X_DIV, sdv = 10;
    uint32_t pmn = p[4], pmx = p[5], pxf = MB_X_ID, pdv = 1;
    if (p[5] - p[4] >= 200) pmn /= 40, pmx /= 40, pxf = MB_X_DIV, pdv = 40;
    const uint32_t a = smx - smn, bb = pmx - pmn;
    b.key(sd, MB_X_YEAR, 1, date_to_year(p[6]), a * bb);
    b.key(ss, sxf, sdv, smn, a);
    b.key(sm, pxf, pdv, pmn, 1);
    b.o.vkind = MB_V_SUB, b.o.va = sr, b.o.vb = sk;
  }
  out = b.o;
}

// joins: dimension attributes through their foreign keys even where the
// engine keeps denormalised copies (the hash-join plan builds its tables
// from the dimensions).
static void build_op(const Engine &E, const mb_query &q, mb_op &out, bool joins = false) {
  SsbSrc S;
  S.date = fact_src(E.orderdate, E.fact_width("orderdate"));
  S.disc = fact_src(E.discount, E.fact_width("discount"));
  S.qty = fact_src(E.quantity, E.fact_width("quantity"));
  S.eprice = fact_src(E.extendedprice, 4);
  S.rev = fact_src(E.revenue, 4);
  S.scost = fact_src(E.supplycost, 4);
  S.scity = fact_src(E.suppcity, E.fact_width("suppcity"));
  S.ccity = joins ? join_src(E.custcity, E.custkey, E.ncust + 1, 1) : E.ccity_src();
  S.mfgr = joins ? join_src(E.partmfgr, E.partkey, E.npart + 1, 2) : E.mfgr_src();
  ssb_build_op(S, q, out);
}

static void query_preds(const mb_query &q, std::vector<Pred> &preds) {
  const uint32_t *p = q.p;
  switch (q.tmpl) {
  case 1: preds = {{IC_DATE, p[0], p[1]}, {IC_DISC, p[2], p[3]}, {IC_QTY, p[4], p[5]}}; break;
  case 2: preds = {{IC_MFGR, p[0], p[1]}, {IC_SCITY, p[2], p[3]}}; break;
  case 3: preds = {{IC_CCITY, p[0], p[1]}, {IC_SCITY, p[2], p[3]}, {IC_DATE, p[4], p[5]}}; break;
  default: preds = {{IC_CCITY, p[0], p[1]}, {IC_SCITY, p[2], p[3]}, {IC_MFGR, p[4], p[5]}, {IC_DATE, p[6], p[7]}};
  }
}

mb_status lower_query(Engine &E, const mb_query &q, const mb_plan &plan, Lowered &L, bool stats) {
  if (q.tmpl < 1 || q.tmpl > 4) return fail(MB_ERR_INVALID, "query: template %u not in 1..4", q.tmpl);
  if (!E.indexed) return fail(MB_ERR_INVALID, "query: the engine has no index (mb_engine_build_index)");
  if (plan.kind > MB_PLAN_HASH) return fail(MB_ERR_INVALID, "query: plan kind %u", plan.kind);
  if (plan.cover > MB_COVER_FINE) return fail(MB_ERR_INVALID, "query: cover mode %u", plan.cover);
  L.reset();
  L.ngroups = query_ngroups(q);
  build_op(E, q, L.op, plan.kind == MB_PLAN_HASH);
  query_preds(q, L.preds);
  const int nchk = (int)L.op.nclause;
  L.covers.resize(L.preds.size());
  for (size_t i = 0; i < L.preds.size(); ++i) {
    const Pred &pr = L.preds[i];
    L.covers[i] = plan_cover(E.idx[pr.col], pr.lo, pr.hi, E.stride, nchk, nullptr, plan.cover);
    if (plan.cover != MB_COVER_RULE && L.covers[i].mid.size() > MB_MAXBINS)  // over the limit: the rule's cover
      L.covers[i] = plan_cover(E.idx[pr.col], pr.lo, pr.hi, E.stride, nchk);
    if (L.covers[i].empty) L.empty = true;
    if (stats) {
      // plan-independent canonical count: the fewer of direct and complement exact covers
      Cover d = plan_cover(E.idx[pr.col], pr.lo, pr.hi, E.stride, 1 << 20);  // edges priced out
      L.canonical_bitmaps += d.full || d.empty ? 0 : d.nb();
    }
  }
  // predicate order: most selective first (ANDM skips loads under zero words)
  std::vector<int> order;
  for (size_t i = 0; i < L.preds.size(); ++i)
    if (!L.covers[i].full) order.push_back((int)i);
  if (plan.order_mode == 0)
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return L.covers[a].est_rows < L.covers[b].est_rows; });
  mb_vprg &P = L.prg;
  memset(&P, 0, sizeof(P));
  P.factsz = E.nrows;
  for (int c = 0; c < MB_MAXCOLS; ++c) P.cols[c].middle = L.mids[c];
  uint32_t ni = 0, nc = 0;
  auto ins = [&](uint8_t op, uint8_t d, uint8_t s) {
    P.instrs[ni].opcode = op, P.instrs[ni].dstreg = d, P.instrs[ni].src1 = s, P.instrs[ni].src2 = 0;
    ++ni;
  };
  if (L.empty) return MB_OK;
  if (order.empty()) {  // every predicate is full: all rows (NOT of the zero register)
    ins(MB_NOT, 0, 3);
    return MB_OK;
  }
  bool first = true;
  for (int i : order) {
    const Cover &cv = L.covers[i];
    mb_col &col = P.cols[nc];
    if (cv.mid.size() > MB_MAXBINS) return fail(MB_ERR_INVALID, "query: predicate needs %zu bins", cv.mid.size());
    col.nmiddle = (uint32_t)cv.mid.size();
    for (size_t k = 0; k < cv.mid.size(); ++k) L.mids[nc][k] = cv.mid[k];
    col.leftmost = cv.left;
    col.rightmost = cv.right;
    L.col_pred[nc] = i;
    L.nbitmaps += cv.nb();
    L.chk |= cv.chk();
    if (!cv.complement) {
      ins(first ? MB_ORM : MB_ANDM, 0, (uint8_t)nc);
    } else if (first) {
      ins(MB_ORM, 1, (uint8_t)nc);
      ins(MB_NOT, 0, 1);
    } else {
      ins(MB_AND, 1, 2);  // r2 is never written: clears r1
      ins(MB_ORM, 1, (uint8_t)nc);
      ins(MB_NOT, 1, 1);
      ins(MB_AND, 0, 1);
    }
    first = false;
    ++nc;
  }
  P.ncols = nc;
  return MB_OK;
}

}  // namespace mb

using namespace mb;

// ------------------------------------------------------------------ C ABI
extern "C" mb_status mb_engine_create(int device, mb_engine **out) {
  if (!out) return fail(MB_ERR_INVALID, "mb_engine_create: out is NULL");
  *out = nullptr;
  int ndev = 0;
  MB_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(MB_ERR_INVALID, "mb_engine_create: device %d of %d", device, ndev);
  MB_CUDA(cudaSetDevice(device));
  mb_engine *e = new (std::nothrow) mb_engine();
  if (!e) return fail(MB_ERR_OOM, "mb_engine_create: host allocation");
  e->E.device = device;
  cudaError_t r = cudaStreamCreateWithFlags(&e->E.stream, cudaStreamNonBlocking);
  if (r == cudaSuccess) r = cudaEventCreate(&e->E.ev0);
  if (r == cudaSuccess) r = cudaEventCreate(&e->E.ev1);
  if (r != cudaSuccess) {
    delete e;
    return cuda_fail(r, "mb_engine_create");
  }
  *out = e;
  return MB_OK;
}

extern "C" mb_status mb_engine_destroy(mb_engine *e) {
  if (e) {
    cudaSetDevice(e->E.device);
    cudaStreamSynchronize(e->E.stream);
    delete e;
  }
  return MB_OK;
}

extern "C" mb_status mb_engine_gen_star(mb_engine *e, uint64_t seed, uint32_t k, uint64_t row0, uint64_t nrows,
                                        int width4) {
  if (!e || k == 0) return fail(MB_ERR_INVALID, "mb_engine_gen_star: engine NULL or k == 0");
  if (nrows >= (1ull << 31)) return fail(MB_ERR_INVALID, "mb_engine_gen_star: rows must be < 2^31");
  Engine &E = e->E;
  MB_CUDA(cudaSetDevice(E.device));
  E.free_star();
  E.nrows = nrows, E.k = k, E.width4 = width4 ? 1 : 0;
  E.stride = mb_bitmap_stride(nrows);
  uint32_t lg = 0;
  while ((2u << lg) <= k) ++lg;
  E.ncust = 30000ull * k, E.nsupp = 2000ull * k, E.npart = 200000ull * (1 + lg);
  const char *names[] = {"custkey", "partkey", "suppkey", "orderdate", "quantity", "discount",
                         "extendedprice", "revenue", "supplycost", "suppcity"};
  void **cols[] = {&E.custkey, &E.partkey, &E.suppkey, &E.orderdate, &E.quantity, &E.discount,
                   &E.extendedprice, &E.revenue, &E.supplycost, &E.suppcity};
  for (int i = 0; i < 10; ++i) MB_CHECK(E.alloc(cols[i], nrows * E.fact_width(names[i])));
  MB_CHECK(E.alloc((void **)&E.custcity, E.ncust + 1));
  MB_CHECK(E.alloc((void **)&E.suppcity_dim, E.nsupp + 1));
  MB_CHECK(E.alloc((void **)&E.partmfgr, (E.npart + 1) * 2));
  mb_star_cols sc = {E.custkey, E.partkey, E.suppkey, E.orderdate, E.quantity, E.discount,
                     E.extendedprice, E.revenue, E.supplycost, E.suppcity};
  MB_CHECK(mb_gen_star(seed, k, row0, nrows, E.width4, &sc, E.stream));
  MB_CHECK(mb_gen_star_dims(seed, k, E.custcity, E.suppcity_dim, E.partmfgr, E.stream));
  MB_CUDA(cudaStreamSynchronize(E.stream));
  return E.setup_index_cols();
}

extern "C" mb_status mb_engine_load_star(mb_engine *e, const mb_star_host *h) {
  if (!e || !h) return fail(MB_ERR_INVALID, "mb_engine_load_star: NULL argument");
  if (h->nrows >= (1ull << 31)) return fail(MB_ERR_INVALID, "mb_engine_load_star: rows must be < 2^31");
  Engine &E = e->E;
  MB_CUDA(cudaSetDevice(E.device));
  E.free_star();
  E.nrows = h->nrows, E.k = 0, E.width4 = 0;
  E.stride = mb_bitmap_stride(h->nrows);
  E.ncust = h->ncust ? h->ncust - 1 : 0, E.nsupp = h->nsupp ? h->nsupp - 1 : 0, E.npart = h->npart ? h->npart - 1 : 0;
  struct {
    void **d;
    const void *s;
    size_t bytes;
  } cp[] = {{&E.custkey, h->custkey, h->nrows * 4},          {&E.partkey, h->partkey, h->nrows * 4},
            {&E.orderdate, h->orderdate, h->nrows * 2},      {&E.extendedprice, h->extendedprice, h->nrows * 4},
            {&E.revenue, h->revenue, h->nrows * 4},          {&E.supplycost, h->supplycost, h->nrows * 4},
            {&E.quantity, h->quantity, h->nrows},            {&E.discount, h->discount, h->nrows},
            {&E.suppcity, h->suppcity, h->nrows},            {(void **)&E.custcity, h->custcity, h->ncust},
            {(void **)&E.partmfgr, h->partmfgr, h->npart * 2}};
  for (auto &c : cp) {
    if (!c.s) return fail(MB_ERR_INVALID, "mb_engine_load_star: a host column is NULL");
    MB_CHECK(E.alloc(c.d, c.bytes));
    MB_CUDA(cudaMemcpyAsync(*c.d, c.s, c.bytes, cudaMemcpyHostToDevice, E.stream));
  }
  MB_CUDA(cudaStreamSynchronize(E.stream));
  return E.setup_index_cols();
}

extern "C" mb_status mb_engine_build_index(mb_engine *e) { return mb_engine_build_index_ex(e, 0); }

extern "C" mb_status mb_engine_build_index_ex(mb_engine *e, uint32_t flags) {
  return mb_engine_build_index_levels(e, flags, MB_LEVELS_ALL);
}

extern "C" mb_status mb_engine_build_index_levels(mb_engine *e, uint32_t flags, uint32_t level_mask) {
  NvtxRange nvtx_("mb_engine_build_index");
  if (!e) return fail(MB_ERR_INVALID, "mb_engine_build_index: NULL engine");
  if (flags & ~MB_INDEX_PROBE_DIMS) return fail(MB_ERR_INVALID, "mb_engine_build_index_ex: flags 0x%x", flags);
  if (level_mask & ~MB_LEVELS_ALL) return fail(MB_ERR_INVALID, "mb_engine_build_index_levels: mask 0x%x", level_mask);
  Engine &E = e->E;
  E.level_mask = level_mask;
  if (!E.custkey) return fail(MB_ERR_INVALID, "mb_engine_build_index: no table");
  MB_CUDA(cudaSetDevice(E.device));
  E.drop_index();
  const bool denorm = !(flags & MB_INDEX_PROBE_DIMS);
  // every allocation first, so the timed build below is device work only
  unsigned long long *d_bad = nullptr;
  MB_CHECK(E.alloc((void **)&d_bad, 16));
  E.free_denorm();
  if (denorm) {
    MB_CHECK(E.alloc((void **)&E.custcity_row, E.nrows));
    MB_CHECK(E.alloc((void **)&E.partmfgr_row, E.nrows * 2));
  }
  MB_CHECK(E.setup_index_cols());  // sources: the denormalised columns filled below
  for (auto &c : E.idx)
    for (auto &l : c.levels) E.nbm += l.nbins();
  uint64_t *d_pop = nullptr;
  MB_CHECK(E.alloc((void **)&d_pop, (size_t)E.nbm * 8));
  MB_CHECK(E.alloc((void **)&E.islab, (size_t)E.nbm * E.stride * 4));
  const uint64_t nwords = (E.nrows + 31) / 32;

  MB_CUDA(cudaEventRecord(E.ev0, E.stream));
  MB_CUDA(cudaMemsetAsync(d_bad, 0, 16, E.stream));
  // only the padding words past each bitmap's end need clearing: the passes
  // write every word below it
  if (E.stride > nwords)
    MB_CUDA(cudaMemset2DAsync(E.islab + nwords, E.stride * 4, 0, (E.stride - nwords) * 4, E.nbm, E.stream));
  MB_CUDA(cudaMemsetAsync(d_pop, 0, (size_t)E.nbm * 8, E.stream));
  uint64_t first = 0;
  for (int ci = 0; ci < IC_N; ++ci) {
    IdxCol &c = E.idx[ci];
    std::vector<std::vector<uint64_t>> lo(c.levels.size()), hi(c.levels.size());
    std::vector<mb_level> lv(c.levels.size());
    for (size_t i = 0; i < c.levels.size(); ++i) {
      Level &l = c.levels[i];
      const uint32_t nb = l.nbins();
      l.slab = E.islab + first * E.stride;
      lo[i].assign(l.bounds.begin(), l.bounds.end() - 1);
      hi[i].assign(l.bounds.begin() + 1, l.bounds.end());
      memset(&lv[i], 0, sizeof(mb_level));
      lv[i].lo = lo[i].data(), lv[i].hi = hi[i].data(), lv[i].nbins = nb;
      lv[i].out = l.slab, lv[i].popcounts = d_pop + first;
      first += nb;
    }
    const bool dn = denorm && (ci == IC_CCITY || ci == IC_MFGR);
    if (!dn) {
      MB_CHECK(mb_bitmap_create_levels(&c.src, E.nrows, lv.data(), (uint32_t)lv.size(), E.stride, E.stream));
      continue;
    }
    // the column's levels through the foreign key; the same pass writes the
    // denormalised column and counts keys outside the dimension
    const mb_src js = ci == IC_CCITY ? join_src(E.custcity, E.custkey, E.ncust + 1, 1)
                                     : join_src(E.partmfgr, E.partkey, E.npart + 1, 2);
    void *dout = ci == IC_CCITY ? (void *)E.custcity_row : (void *)E.partmfgr_row;
    const mb_status st = bitmap_create_levels_join(&js, E.nrows, lv.data(), (uint32_t)lv.size(), E.stride,
                                                   E.stream, dout, d_bad + (ci == IC_CCITY ? 0 : 1));
    if (st == MB_OK) continue;
    if (st != MB_ERR_INVALID) return st;
    // the levels need more than one pass: denormalise first, then index the column
    MB_CHECK(E.enqueue_denorm(d_bad, E.stream));
    MB_CHECK(mb_bitmap_create_levels(&c.src, E.nrows, lv.data(), (uint32_t)lv.size(), E.stride, E.stream));
  }
  MB_CUDA(cudaEventRecord(E.ev1, E.stream));
  std::vector<uint64_t> pops(E.nbm);
  unsigned long long bad[2] = {0, 0};
  MB_CUDA(cudaMemcpyAsync(pops.data(), d_pop, (size_t)E.nbm * 8, cudaMemcpyDeviceToHost, E.stream));
  MB_CUDA(cudaMemcpyAsync(bad, d_bad, 16, cudaMemcpyDeviceToHost, E.stream));
  MB_CUDA(cudaStreamSynchronize(E.stream));
  MB_CHECK(check_device_error(E.stream));
  cudaEventElapsedTime(&E.index_build_ms, E.ev0, E.ev1);
  free_one(E.allocs, d_pop);
  free_one(E.allocs, d_bad);
  if (denorm && (bad[0] || bad[1])) {
    // a foreign key outside its dimension: the denormalised columns cannot
    // stand in for the probes; build over the probes instead
    return mb_engine_build_index_levels(e, flags | MB_INDEX_PROBE_DIMS, level_mask);
  }
  first = 0;
  for (auto &c : E.idx)
    for (auto &l : c.levels) {
      l.pop.assign(pops.begin() + first, pops.begin() + first + l.nbins());
      first += l.nbins();
    }
  E.indexed = true;
  return MB_OK;
}

extern "C" mb_status mb_engine_plan_index(mb_engine *e, const mb_query *qs, uint32_t n, uint64_t budget,
                                          uint32_t *level_mask, uint64_t *index_bytes, uint64_t *workload_bytes) {
  if (!e || (!qs && n) || !level_mask) return fail(MB_ERR_INVALID, "mb_engine_plan_index: NULL argument");
  Engine &E = e->E;
  if (!E.indexed) return fail(MB_ERR_INVALID, "mb_engine_plan_index: build an index first (its bin row counts)");
  std::vector<std::vector<Pred>> preds(n);
  for (uint32_t i = 0; i < n; ++i) {
    if (qs[i].tmpl < 1 || qs[i].tmpl > 4) return fail(MB_ERR_INVALID, "mb_engine_plan_index: template %u", qs[i].tmpl);
    query_preds(qs[i], preds[i]);
  }
  uint32_t mask = E.level_mask;
  bool ok = false;
  uint64_t cost = workload_cost(E, preds, mask, &ok);
  if (!ok) return fail(MB_ERR_INVALID, "mb_engine_plan_index: the built index cannot cover the workload");
  while (mask_bytes(E, mask) > budget) {
    int best = -1;
    double best_rate = 0;
    uint64_t best_cost = 0;
    for (uint32_t i = 0; i < MB_INDEX_LEVELS; ++i) {
      if (!((mask >> i) & 1u)) continue;
      bool ok2 = false;
      const uint64_t c2 = workload_cost(E, preds, mask & ~(1u << i), &ok2);
      if (!ok2) continue;
      const double rate = ((double)c2 - (double)cost) / (double)mask_bytes(E, 1u << i);
      if (best < 0 || rate < best_rate) best = (int)i, best_rate = rate, best_cost = c2;
    }
    if (best < 0)
      return fail(MB_ERR_INVALID, "mb_engine_plan_index: no level set fits %llu bytes", (unsigned long long)budget);
    mask &= ~(1u << best);
    cost = best_cost;
  }
  *level_mask = mask;
  if (index_bytes) *index_bytes = mask_bytes(E, mask);
  if (workload_bytes) *workload_bytes = cost;
  return MB_OK;
}

extern "C" mb_status mb_engine_get_info(mb_engine *e, mb_engine_info *o) {
  if (!e || !o) return fail(MB_ERR_INVALID, "mb_engine_get_info: NULL argument");
  Engine &E = e->E;
  memset(o, 0, sizeof(*o));
  o->nrows = E.nrows, o->k = E.k, o->width4 = E.width4;
  const char *names[] = {"custkey", "partkey", "suppkey", "orderdate", "quantity", "discount",
                         "extendedprice", "revenue", "supplycost", "suppcity"};
  for (const char *n : names) o->fact_bytes += E.nrows * E.fact_width(n);
  o->dim_bytes = (E.ncust + 1) + (E.nsupp + 1) + (E.npart + 1) * 2;
  for (auto &c : E.idx)
    for (auto &l : c.levels) {
      o->nbitmaps += l.nbins();
      if (E.indexed) o->index_bytes += (uint64_t)l.nbins() * E.stride * 4;
    }
  o->sms = (uint32_t)dev_info().sms;
  o->index_build_ms = E.index_build_ms;
  o->denorm = (E.custcity_row || E.partmfgr_row) ? 1u : 0u;
  o->denorm_bytes = (E.custcity_row ? E.nrows : 0) + (E.partmfgr_row ? E.nrows * 2 : 0);
  return MB_OK;
}

extern "C" uint32_t mb_query_ngroups(const mb_query *q) { return q ? query_ngroups(*q) : 0; }

extern "C" mb_status mb_engine_plan_rule(mb_engine *e, const mb_query *q, mb_plan *out) {
  if (!e || !q || !out) return fail(MB_ERR_INVALID, "mb_engine_plan_rule: NULL argument");
  memset(out, 0, sizeof(*out));
  out->kind = MB_PLAN_FUSED;
  out->order_mode = 0;
  out->launch.grp_strategy = MB_GRP_AUTO;
  return MB_OK;
}

namespace mb {
// Runs a lowered query on the engine stream; results stay on the device.
// Materialised predicates (plan.materialise, template order) are evaluated
// into a (certain, uncertain) bitmap pair first and read as one operand.
mb_status run_lowered(Engine &E, Lowered &L, const mb_plan &plan, int64_t *d_out, uint64_t *d_nq, bool zero) {
  cudaStream_t st = E.stream;
  if (L.empty) {
    if (!zero) return MB_OK;
    MB_CUDA(cudaMemsetAsync(d_out, 0, (size_t)L.ngroups * 8, st));
    MB_CUDA(cudaMemsetAsync(d_nq, 0, 8, st));
    return MB_OK;
  }
  if (plan.kind == MB_PLAN_SCAN) return mb_join_grpby(E.nrows, &L.op, L.ngroups, d_out, d_nq, st);
  if (plan.kind == MB_PLAN_HASH) return mb_hash_join_grpby(E.nrows, &L.op, L.ngroups, d_out, d_nq, st);
  // materialise predicates whose bit is set: their operand becomes one
  // (certain, uncertain) bitmap pair evaluated up front
  const uint64_t W = E.stride;
  uint32_t nmat = 0;
  for (uint32_t c = 0; c < L.prg.ncols; ++c)
    if (plan.materialise & (1u << L.col_pred[c])) ++nmat;
  if (plan.kind == MB_PLAN_MATERIALISED || nmat) MB_CHECK(E.ensure_tmp(W * (2 * nmat + 2)));
  uint32_t used = 0;
  for (uint32_t c = 0; c < L.prg.ncols && nmat; ++c) {
    if (!(plan.materialise & (1u << L.col_pred[c]))) continue;
    mb_col &col = L.prg.cols[c];
    mb_vprg one;
    memset(&one, 0, sizeof(one));
    one.factsz = E.nrows;
    one.ncols = 1;
    one.cols[0] = col;
    one.instrs[0].opcode = MB_ORM;
    const bool chk = col.leftmost || col.rightmost;
    uint32_t *pc = E.tmp_bits + W * used++, *pu = chk ? E.tmp_bits + W * used++ : nullptr;
    MB_CHECK(mb_vprg_eval(&one, chk ? 1 : 0, pc, pu, nullptr, st));
    if (chk) MB_CHECK(certain_of(pc, pu, E.nrows, st));
    L.mids[c][0] = pc;
    col.nmiddle = 1;
    col.leftmost = pu;
    col.rightmost = nullptr;
  }
  if (plan.kind == MB_PLAN_MATERIALISED) {
    uint32_t *poss = E.tmp_bits + W * used, *unc = E.tmp_bits + W * (used + 1);
    const int chk = !mb_vprg_is_nochk(&L.prg);
    MB_CHECK(mb_vprg_eval(&L.prg, chk, poss, chk ? unc : nullptr, nullptr, st));
    MB_CHECK(E.ensure_rows(E.nrows + 1));
    if (!E.d_rowcnt) MB_CHECK(E.alloc((void **)&E.d_rowcnt, 8));
    MB_CHECK(mb_bitmap_to_rows(poss, chk ? unc : nullptr, E.nrows, E.rows, E.d_rowcnt, st));
    return mb_rows_grpby(E.rows, E.d_rowcnt, E.rows_cap, &L.op, L.ngroups, d_out, d_nq, st);
  }
  return fused_grpby(&L.prg, &L.op, L.ngroups, d_out, d_nq, &plan.launch, st, zero);
}
}  // namespace mb

extern "C" mb_status mb_engine_query(mb_engine *e, const mb_query *q, const mb_plan *plan, int64_t *out_host,
                                     uint64_t *nqual_host, mb_query_stats *stats) {
  NvtxRange nvtx_("mb_engine_query");
  if (!e || !q || !out_host) return fail(MB_ERR_INVALID, "mb_engine_query: NULL argument");
  Engine &E = e->E;
  MB_CUDA(cudaSetDevice(E.device));
  mb_plan pl;
  if (plan) pl = *plan;
  else MB_CHECK(mb_engine_plan_rule(e, q, &pl));
  Lowered L;
  MB_CHECK(lower_query(E, *q, pl, L, stats != nullptr));
  MB_CHECK(E.ensure_out(L.ngroups));
  MB_CUDA(cudaEventRecord(E.ev0, E.stream));
  MB_CHECK(run_lowered(E, L, pl, E.d_out, E.d_nqual, true));
  MB_CUDA(cudaEventRecord(E.ev1, E.stream));
  MB_CUDA(cudaMemcpyAsync(E.h_out, E.d_out, (size_t)L.ngroups * 8, cudaMemcpyDeviceToHost, E.stream));
  MB_CUDA(cudaMemcpyAsync(E.h_nqual, E.d_nqual, 8, cudaMemcpyDeviceToHost, E.stream));
  MB_CUDA(cudaStreamSynchronize(E.stream));
  memcpy(out_host, E.h_out, (size_t)L.ngroups * 8);
  if (nqual_host) *nqual_host = E.h_nqual[0];
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    cudaEventElapsedTime(&stats->ms, E.ev0, E.ev1);
    stats->nbitmaps = L.nbitmaps;
    stats->chk = L.chk ? 1 : 0;
    stats->algo_bytes = L.canonical_bitmaps * mb_bitmap_words(E.nrows) * 4;
  }
  return MB_OK;
}

extern "C" uint64_t mb_queries_layout(const mb_query *qs, uint32_t n, uint64_t *offsets) {
  uint64_t off = 0;
  for (uint32_t i = 0; i < n; ++i) {
    if (offsets) offsets[i] = off;
    off += query_ngroups(qs[i]);
  }
  return off;
}

extern "C" mb_status mb_engine_enqueue(mb_engine *e, const mb_query *qs, uint32_t n, const mb_plan *plans,
                                       int64_t *out_dev, uint64_t *nqual_dev, int record_times) {
  NvtxRange nvtx_("mb_engine_enqueue");
  if (!e || (!qs && n) || !out_dev || !nqual_dev) return fail(MB_ERR_INVALID, "mb_engine_enqueue: NULL argument");
  Engine &E = e->E;
  MB_CUDA(cudaSetDevice(E.device));
  if (record_times) {
    while (E.qev.size() < 2ull * n) {
      cudaEvent_t ev;
      MB_CUDA(cudaEventCreate(&ev));
      E.qev.push_back(ev);
    }
  }
  E.qev_used = record_times ? n : 0;
  // one memset zeroes every query's outputs; the per-query events then
  // bracket the query kernels only
  const uint64_t total = mb_queries_layout(qs, n, nullptr);
  MB_CUDA(cudaMemsetAsync(out_dev, 0, total * 8, E.stream));
  MB_CUDA(cudaMemsetAsync(nqual_dev, 0, (size_t)n * 8, E.stream));
  uint64_t off = 0;
  Lowered L;
  for (uint32_t i = 0; i < n; ++i) {
    mb_plan pl;
    if (plans) pl = plans[i];
    else MB_CHECK(mb_engine_plan_rule(e, &qs[i], &pl));
    MB_CHECK(lower_query(E, qs[i], pl, L));
    if (record_times) MB_CUDA(cudaEventRecord(E.qev[2 * i], E.stream));
    MB_CHECK(run_lowered(E, L, pl, out_dev + off, nqual_dev + i, false));
    if (record_times) MB_CUDA(cudaEventRecord(E.qev[2 * i + 1], E.stream));
    off += L.ngroups;
  }
  return MB_OK;
}

extern "C" mb_status mb_engine_sync(mb_engine *e, float *times_ms, uint32_t n) {
  if (!e) return fail(MB_ERR_INVALID, "mb_engine_sync: NULL engine");
  Engine &E = e->E;
  MB_CUDA(cudaSetDevice(E.device));
  MB_CUDA(cudaStreamSynchronize(E.stream));
  if (times_ms) {
    if (n > E.qev_used) return fail(MB_ERR_INVALID, "mb_engine_sync: %u times requested, %u recorded", n, E.qev_used);
    for (uint32_t i = 0; i < n; ++i) MB_CUDA(cudaEventElapsedTime(&times_ms[i], E.qev[2 * i], E.qev[2 * i + 1]));
  }
  return MB_OK;
}

extern "C" mb_status mb_engine_mark(mb_engine *e, uint32_t idx) {
  if (!e || idx >= 8) return fail(MB_ERR_INVALID, "mb_engine_mark: engine NULL or marker >= 8");
  Engine &E = e->E;
  MB_CUDA(cudaSetDevice(E.device));
  if (!E.marks[idx]) MB_CUDA(cudaEventCreate(&E.marks[idx]));
  MB_CUDA(cudaEventRecord(E.marks[idx], E.stream));
  return MB_OK;
}

extern "C" mb_status mb_engine_marks_ms(mb_engine *e, uint32_t a, uint32_t b, float *ms) {
  if (!e || a >= 8 || b >= 8 || !ms) return fail(MB_ERR_INVALID, "mb_engine_marks_ms: bad argument");
  Engine &E = e->E;
  if (!E.marks[a] || !E.marks[b]) return fail(MB_ERR_INVALID, "mb_engine_marks_ms: marker not recorded");
  MB_CUDA(cudaEventSynchronize(E.marks[b]));
  MB_CUDA(cudaEventElapsedTime(ms, E.marks[a], E.marks[b]));
  return MB_OK;
}

extern "C" void *mb_engine_stream(mb_engine *e) { return e ? (void *)e->E.stream : nullptr; }

// ------------------------------------------------------------------ batches
namespace mb {

// Inclusive 32-bit form of a half-open 64-bit term [lo, hi) over values that
// fit 32 bits; an empty term becomes lo = 1, hi = 0.
static void term32(uint64_t lo, uint64_t hi, uint32_t &l, uint32_t &h) {
  if (lo >= hi || lo > 0xffffffffull) {
    l = 1, h = 0;
    return;
  }
  l = (uint32_t)lo;
  h = (uint32_t)((hi > 0x100000000ull ? 0x100000000ull : hi) - 1);
}

enum { BADD_OK = 0, BADD_FULL = 1, BADD_ALONE = 2 };

// Batch under construction: the staging header and its lookup tables.
struct BatchBuild {
  BatchHdr *h = nullptr;
  std::vector<uint8_t> used;  // slab rows the batch reads
  uint32_t nused = 0;
  std::vector<double> cost;   // estimated cost of each query (per bitmap word)
  std::vector<double> sel;    // estimated selected-row fraction of each query
  double src_weight[BS_MAX] = {};  // selected-row fraction reading each source

  void reset(BatchHdr *hh, const Engine &E) {
    h = hh;
    memset(h, 0, sizeof(*h));
    h->nrows = E.nrows;
    h->nwords = (E.nrows + 31) / 32;
    h->stride = E.stride;
    h->slab = E.islab;
    h->nslab = E.nbm;
    for (uint32_t q = 0; q < BQ_MAX; ++q) h->toff[q] = 0xffffffffu;
    used.assign(E.nbm, 0);
    nused = 0;
    cost.clear();
    sel.clear();
    for (double &w : src_weight) w = 0;
  }
};

// The staging of a set of slab rows: runs of rows, one tensor copy per run
// (the smallest gaps merged while there would be more than BCP_MAX copies).  Fills copy[] (BatchHdr packing) and, if stage_of is
// given, the stage row of every used slab row; returns the rows staged, or
// 0 if the set needs more than BU_MAX rows or BCP_MAX copies.
static uint32_t stage_plan(const std::vector<uint8_t> &used, uint32_t *copy, uint32_t *ncopy, uint16_t *stage_of) {
  std::vector<std::pair<uint32_t, uint32_t>> runs;  // [a, b)
  for (uint32_t r = 0; r < used.size(); ++r) {
    if (!used[r]) continue;
    if (!runs.empty() && r == runs.back().second) runs.back().second = r + 1;
    else runs.push_back({r, r + 1});
  }
  if (runs.empty()) runs.push_back({0, 1});  // no bitmap read: stage one row anyway
  uint32_t staged = 0;
  for (auto &r : runs) staged += r.second - r.first;
  // too many copies: merge the runs with the smallest gap
  while (runs.size() > BCP_MAX) {
    size_t bi = 0;
    for (size_t i = 1; i + 1 < runs.size(); ++i)
      if (runs[i + 1].first - runs[i].second < runs[bi + 1].first - runs[bi].second) bi = i;
    staged += runs[bi + 1].first - runs[bi].second;
    runs[bi].second = runs[bi + 1].second;
    runs.erase(runs.begin() + bi + 1);
  }
  if (staged > BU_MAX) return 0;
  uint32_t t = 0, c = 0;
  for (auto &r : runs) {
    const uint32_t h = r.second - r.first;
    if (stage_of)
      for (uint32_t x = r.first; x < r.second; ++x) stage_of[x] = (uint16_t)(t + x - r.first);
    if (copy) copy[c] = r.first | (t << 12) | ((h - 1) << 24);
    ++c;
    t += h;
  }
  if (ncopy) *ncopy = c;
  return staged;
}

// Row of the index slab holding bitmap p, or -1.
static int64_t slab_row(const BatchHdr &h, const uint32_t *p) {
  if (p < h.slab || p >= h.slab + (uint64_t)h.nslab * h.stride) return -1;
  const uint64_t off = (uint64_t)(p - h.slab);
  return off % h.stride ? -1 : (int64_t)(off / h.stride);
}

static bool same_src(const mb_src &a, const mb_src &b) {
  return a.col == b.col && a.fk == b.fk && a.width == b.width && a.dimsz == b.dimsz;
}

static int src_slot(const BatchHdr &h, const mb_src &s) {
  for (uint32_t i = 0; i < h.nsrc; ++i) {
    const BatchSrc &b = h.src[i];
    if (b.col == s.col && b.fk == s.fk && b.width == s.width && b.dimsz == (uint32_t)s.dimsz) return (int)i;
  }
  return -1;
}

// The op as the batch kernel's per-slot descriptor (batch.cuh); false if it
// is outside that form.
static bool slot_plan(const mb_op &O, uint32_t *d) {
  if (O.nsrc > BSLOT) return false;
  for (uint32_t s = 0; s < O.nsrc; ++s)
    if (O.src[s].width > 4 || O.src[s].width == 3 || O.src[s].dimsz > 0xffffffffull) return false;
  const OpNeeds N = op_needs(O);
  uint32_t termm = 0, keym = 0;
  uint32_t lo[BSLOT], hi[BSLOT];
  for (uint32_t s = 0; s < BSLOT; ++s) lo[s] = 0, hi[s] = 0xffffffffu;
  for (uint32_t c = 0; c < O.nclause; ++c) {
    if (O.clause_len[c] != 1) return false;  // OR clauses: single-query path
    const mb_term &t = O.terms[c];
    uint32_t l, h;
    term32(t.lo, t.hi, l, h);
    const uint32_t s = t.src;
    termm |= 1u << s;
    lo[s] = std::max(lo[s], l);
    hi[s] = std::min(hi[s], h);
  }
  for (uint32_t k = 0; k < O.nkey; ++k) {
    const mb_key &kk = O.keys[k];
    if ((keym >> kk.src) & 1u) return false;  // a source in two keys
    keym |= 1u << kk.src;
    uint32_t *sl = d + BQD_SLOT0 + BQD_SLOTW * kk.src;
    uint32_t sh = 0;
    if (kk.xform == MB_X_DIV || kk.xform == MB_X_ID) {  // an identity key divides by 1
      const uint32_t dv = kk.xform == MB_X_DIV ? kk.div : 1u;
      if (dv == 0) return false;
      const DivMagic m = div_magic(dv);
      for (uint32_t x : {0u, 1u, dv - 1, dv, dv + 1, 12345u, 0x7fffffffu, 0xfffffffeu, 0xffffffffu})
        if (div_by_magic(x, m.m, m.sh1, m.sh2) != x / dv) return false;
      sl[3] = m.m;
      sh = m.sh1 | (m.sh2 << 4);
    }
    sl[0] |= (kk.xform << 16) | (sh << 24);
    sl[4] = kk.base;
    sl[5] = kk.mul;
    sl[6] = kk.div;
  }
  for (uint32_t s = 0; s < O.nsrc; ++s) {
    uint32_t *sl = d + BQD_SLOT0 + BQD_SLOTW * s;
    sl[0] |= O.src[s].width << 8;
    if ((termm >> s) & 1u) {
      if (lo[s] > hi[s]) lo[s] = 1, hi[s] = 0;
      sl[1] = lo[s];
      sl[2] = hi[s];
    }
  }
  d[0] = O.nsrc | (O.vkind << 16) | (O.va << 20) | (O.vb << 24);
  d[5] = (N.kv_mask & 0xffu) | ((N.filt_mask & 0xffu) << 8) | (keym << 16) | (termm << 24);
  for (uint32_t s2 = 0; s2 < O.nsrc; ++s2)
    if (O.src[s2].fk) d[7] |= 1u << s2;
  // a compiled drain for this shape, if there is one
  const uint32_t va = O.vkind == MB_V_ONE ? 0 : O.va, vb = (O.vkind == MB_V_MUL || O.vkind == MB_V_SUB) ? O.vb : 0;
  uint32_t yearm = 0;
  for (uint32_t k = 0; k < O.nkey; ++k)
    if (O.keys[k].xform == MB_X_YEAR) yearm |= 1u << O.keys[k].src;
  for (uint32_t i = 0; i < BNSHAPE; ++i) {
    const BShape &b = BSHAPES[i];
    if (b.ns == O.nsrc && b.kv == (N.kv_mask & 0xffu) && b.filt == (N.filt_mask & 0xffu) && b.keym == keym &&
        b.yearm == yearm && b.vk == O.vkind && b.va == va && b.vb == vb && termm == b.filt) {
      d[6] = i + 1;
      break;
    }
  }
  return true;
}

// Adds a lowered query (its conjunctive program P) as the next query of the
// batch.  BADD_FULL: a limit of this launch is reached (flush and retry);
// BADD_ALONE: the batch kernel cannot run the query.
static int batch_add(BatchBuild &B, const Lowered &L, const DevPrg &P, uint64_t out_off, uint32_t nq_slot,
                     double sel) {
  BatchHdr &h = *B.h;
  const mb_op &O = L.op;
  if (!P.cnf) return BADD_ALONE;
  if (out_off + L.ngroups >= 0x80000000ull) return BADD_ALONE;
  uint32_t d[BQD_WORDS];
  memset(d, 0, sizeof(d));
  if (!slot_plan(O, d)) return BADD_ALONE;
  // the slab rows this query reads, added to the batch's
  std::vector<uint32_t> fresh;
  for (uint32_t i = 0; i < P.ncnf; ++i) {
    const int64_t r = slab_row(h, P.cnf_ptr[i]);
    if (r < 0) return BADD_ALONE;
    if (!B.used[r] && std::find(fresh.begin(), fresh.end(), (uint32_t)r) == fresh.end()) fresh.push_back((uint32_t)r);
  }
  uint32_t newsrc = 0;
  for (uint32_t s = 0; s < O.nsrc; ++s) {
    bool seen = src_slot(h, O.src[s]) >= 0;
    for (uint32_t t = 0; t < s && !seen; ++t) seen = same_src(O.src[t], O.src[s]);
    if (!seen) ++newsrc;
  }
  const uint32_t nch = P.ncnf;  // chain entries
  uint32_t ncj = 0;             // conjuncts, each of at most 255 middle and 15 edge bins
  for (uint32_t i = 0, nm = 0, ne = 0; i < P.ncnf; ++i) {
    if (P.cnf_flag[i] & CNF_EDGE) ++ne;
    else ++nm;
    if (nm > 0xff || ne > 0xf) return BADD_ALONE;
    if (P.cnf_flag[i] & CNF_END) ++ncj, nm = 0, ne = 0;
  }
  bool stages_ok = true;
  if (!fresh.empty()) {
    for (uint32_t r : fresh) B.used[r] = 1;
    stages_ok = stage_plan(B.used, nullptr, nullptr, nullptr) != 0;
    if (!stages_ok)
      for (uint32_t r : fresh) B.used[r] = 0;
  }
  if (newsrc > BS_MAX || nch > BC_MAX || ncj > BJ_MAX || (!stages_ok && B.nused == 0)) return BADD_ALONE;
  if (h.nq + 1 > BQ_MAX || !stages_ok || h.nsrc + newsrc > BS_MAX || h.nchain + nch > BC_MAX ||
      h.nconj + ncj > BJ_MAX) {
    if (stages_ok)
      for (uint32_t r : fresh) B.used[r] = 0;
    return BADD_FULL;
  }
  B.nused += (uint32_t)fresh.size();
  // commit
  const uint32_t q = h.nq++;
  const OpNeeds N = op_needs(O);
  for (uint32_t s = 0; s < O.nsrc; ++s) {
    int t = src_slot(h, O.src[s]);
    if (t < 0) {
      t = (int)h.nsrc++;
      BatchSrc &b = h.src[t];
      b.col = O.src[s].col;
      b.fk = O.src[s].fk;
      b.dimsz = (uint32_t)O.src[s].dimsz;
      b.width = O.src[s].width;
    }
    d[BQD_SLOT0 + BQD_SLOTW * s] |= (uint32_t)t;
    if ((N.kv_mask >> s) & 1u) B.src_weight[t] += sel;
  }
  d[0] |= (L.ngroups == 1 ? 1u : 0u) << 8;
  d[1] = L.ngroups;
  d[2] = (uint32_t)out_off;
  d[3] = nq_slot;
  // the program: per conjunct its middle bins then its edge bins in the
  // chain (slab rows, made stage rows by batch_finish) and one conjunct entry
  const uint32_t j0 = h.nconj;
  for (uint32_t i = 0; i < P.ncnf;) {
    uint32_t j = i;
    while (!(P.cnf_flag[j] & CNF_END)) ++j;  // [i, j] is one conjunct
    const uint32_t first = h.nchain;
    uint32_t nmid = 0, nedge = 0;
    for (uint32_t k = i; k <= j; ++k)
      if (!(P.cnf_flag[k] & CNF_EDGE)) h.chain[h.nchain++] = (uint16_t)slab_row(h, P.cnf_ptr[k]), ++nmid;
    for (uint32_t k = i; k <= j; ++k)
      if (P.cnf_flag[k] & CNF_EDGE) h.chain[h.nchain++] = (uint16_t)slab_row(h, P.cnf_ptr[k]), ++nedge;
    h.conj[h.nconj++] = first | (nmid << BJ_NMID_SHIFT) | (nedge << BJ_NEDGE_SHIFT) |
                        ((P.cnf_flag[j] & CNF_NEG) ? BJ_NEG : 0u);
    i = j + 1;
  }
  d[4] = j0 | ((h.nconj - j0) << 16);
  memcpy(h.Qd + (size_t)q * BQD_WORDS, d, sizeof(d));
  // cost per bitmap word of a tile: the chain entries and the ops of the
  // selected rows (a round of 32 rows costs about as much as 20 entries of a
  // word per lane)
  B.cost.push_back((double)P.ncnf + 2.0 + 600.0 * sel);
  B.sel.push_back(sel);
  return BADD_OK;
}

// Selected-row fraction of a lowered query: the product of its predicates'
// estimated fractions (bin popcounts, predicates taken as independent).
static double est_selectivity(const Engine &E, const Lowered &L) {
  if (E.nrows == 0) return 0;
  double f = 1;
  for (const Cover &c : L.covers)
    if (!c.full) f *= std::min(1.0, (double)c.est_rows / (double)E.nrows);
  return f;
}

// The most stages (up to smax) of shape c that fit in shared memory.
// Stages and chunk buffers of a launch shape: the larger buffer (1,024, then
// 256 rows a warp) that fits beside at least two stages (or the
// stages asked for, if fewer), the most stages (up to smax) beside it; else
// 256-row buffers and whatever number of stages fits.  (Larger buffers make
// fewer, fuller drain chunks: 1,024 rows and two stages measured 4 % faster
// than 256 rows and three stages on the 600M-row selectivity-spanning mix.)
static bool fit_stages(const BatchHdr &h, BatchCfg &c, uint32_t smax) {
  const size_t cap = (size_t)dev_info().max_smem_optin;
  const uint32_t smin = smax < 2 ? smax : 2u;
  for (uint32_t buf : {1024u, 256u})
    for (c.stages = smax; c.stages >= smin; --c.stages) {
      c.buf = buf;
      const size_t b = batch_smem(h, c);
      if (b && b <= cap) return true;
    }
  c.buf = 256;
  for (c.stages = smax; c.stages >= 1; --c.stages) {
    const size_t b = batch_smem(h, c);
    if (b && b <= cap) return true;
  }
  c.stages = 1;
  return false;
}

// The launch shape: the options given; for what they leave open, the widest
// tile (4, 2, then 1 words per lane) that keeps two stages in flight, and as
// many stages (up to 4) as fit.
static BatchCfg batch_cfg(const BatchHdr &h, const mb_batch_opts &o) {
  const uint32_t smax = o.stages ? o.stages : 4;
  std::vector<uint32_t> Vs;
  if (o.words_per_lane) Vs.push_back(o.words_per_lane);
  else Vs = {4u, 2u, 1u};
  BatchCfg one;  // the first shape with one stage, if none has two
  bool have_one = false;
  for (uint32_t V : Vs) {
    BatchCfg c;
    memset(&c, 0, sizeof(c));
    c.V = V;
    c.warps = o.warps ? std::min<uint32_t>(o.warps, BW_MAX) : 16;
    c.cps = o.ctas_per_sm;
    if (!fit_stages(h, c, smax)) continue;
    if (c.stages >= 2 || smax == 1) return c;
    if (!have_one) one = c, have_one = true;
  }
  if (have_one) return one;
  BatchCfg c;  // nothing fits: batch_scan reports the shape
  memset(&c, 0, sizeof(c));
  c.V = Vs.back();
  c.warps = o.warps ? std::min<uint32_t>(o.warps, BW_MAX) : 16;
  c.stages = 1;
  return c;
}

// Shared group tables: the multi-group queries whose estimated rows per CTA
// are many times their group count (so a flush of the table costs far less
// than the global atomics it saves), most rows first, while they fit in the
// shared memory the launch shape leaves (at most table_kb KB; 48 KB if 0).
static void batch_tables(BatchBuild &B, const mb_batch_opts &o, const BatchCfg &c) {
  BatchHdr &h = *B.h;
  const size_t cap = (size_t)dev_info().max_smem_optin;
  const size_t used = batch_smem(h, c);
  h.nstab = 0;
  if (!used || used >= cap) return;
  uint64_t slots = std::min<uint64_t>((cap - used) / 8 - 2, (o.table_kb ? o.table_kb : 48u) * 128ull);
  const double ctas = (double)dev_info().sms;
  std::vector<uint32_t> cand;
  for (uint32_t q = 0; q < h.nq; ++q) {
    const uint32_t ng = h.Qd[(size_t)q * BQD_WORDS + 1];
    if (ng > 1 && B.sel[q] * (double)h.nrows >= 8.0 * ctas * ng) cand.push_back(q);
  }
  std::stable_sort(cand.begin(), cand.end(), [&](uint32_t a, uint32_t b) { return B.sel[a] > B.sel[b]; });
  for (uint32_t q : cand) {
    const uint32_t ng = h.Qd[(size_t)q * BQD_WORDS + 1];
    if (h.nstab + ng > slots) continue;
    h.toff[q] = h.nstab;
    h.nstab += ng;
  }
}

// Completes a batch's header: the order of its queries, its staging copies
// (the chain's slab rows become stage rows), its L2 prefetches, its launch
// shape and its shared group tables.
static mb_status batch_finish(BatchBuild &B, const mb_batch_opts &o, BatchCfg *cfg) {
  BatchHdr &h = *B.h;
  std::vector<uint32_t> order(h.nq);
  for (uint32_t q = 0; q < h.nq; ++q) order[q] = q;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return B.cost[a] > B.cost[b]; });
  for (uint32_t i = 0; i < h.nq; ++i) h.order[i] = (uint8_t)order[i];
  std::vector<uint16_t> stage_of(h.nslab ? h.nslab : 1, 0xffffu);
  h.nu = stage_plan(B.used, h.copy, &h.ncopy, stage_of.data());
  if (h.nu == 0) return fail(MB_ERR_INVALID, "batch: staging plan over its limits");
  for (uint32_t i = 0; i < h.nchain; ++i) {
    const uint32_t r = h.chain[i];
    const uint16_t t = r < h.nslab ? stage_of[r] : 0xffffu;
    if (t >= h.nu) return fail(MB_ERR_INVALID, "batch: chain row %u not staged", r);
    h.chain[i] = t;
  }
  h.pf_mask = 0;
  for (uint32_t i = 0; i < h.nsrc; ++i) {
    const void *base = h.src[i].fk ? (const void *)h.src[i].fk : h.src[i].col;
    const bool aligned = ((uintptr_t)base & 15) == 0;
    const bool dense = o.prefetch == MB_PREFETCH_ALL || (o.prefetch == MB_PREFETCH_AUTO && B.src_weight[i] >= 0.02);
    if (aligned && dense && B.src_weight[i] > 0) h.pf_mask |= 1u << i;
  }
  h.nstab = 0;
  *cfg = batch_cfg(h, o);
  batch_tables(B, o, *cfg);
  return MB_OK;
}

// A planned enqueue: the batched launches (complete headers, host copies)
// and the queries that run alone on the plain path.
struct BatchPlanned {
  std::vector<std::unique_ptr<BatchHdr>> hdrs;
  std::vector<BatchCfg> cfgs;
  std::vector<uint32_t> alone;
  std::vector<mb_plan> alone_plan;  // the plan each query of `alone` runs with
  std::vector<double> sel;          // per query: estimated selected-row fraction (rule covers)
  std::vector<uint8_t> chk;         // per query: its covers have edge bins (uncertain rows)
  std::vector<uint64_t> offs;
  uint64_t total = 0;
};

// plans (optional, one per query): a fused plan puts its query in the batch
// with the plan's cover and order; any other kind runs the query alone on the
// plain path with that plan.  Without plans every query takes the rule plan.
static mb_status batch_plan(Engine &E, const mb_query *qs, uint32_t n, const mb_batch_opts &o, BatchPlanned &P,
                            const mb_plan *plans = nullptr) {
  P.offs.resize(n);
  P.total = mb_queries_layout(qs, n, P.offs.data());
  P.sel.assign(n, 0.0);
  P.chk.assign(n, 0);
  mb_plan pl;  // the rule plan
  memset(&pl, 0, sizeof(pl));
  pl.kind = MB_PLAN_FUSED;
  pl.launch.grp_strategy = MB_GRP_AUTO;
  BatchBuild B;
  auto fresh = [&]() -> mb_status {
    BatchHdr *h = new (std::nothrow) BatchHdr;
    if (!h) return fail(MB_ERR_OOM, "batch: host header");
    P.hdrs.emplace_back(h);
    B.reset(h, E);
    return MB_OK;
  };
  auto close = [&]() -> mb_status {
    if (B.h->nq == 0) {
      P.hdrs.pop_back();
      return MB_OK;
    }
    BatchCfg c;
    MB_CHECK(batch_finish(B, o, &c));
    P.cfgs.push_back(c);
    return MB_OK;
  };
  MB_CHECK(fresh());
  Lowered L;
  DevPrg D;
  for (uint32_t i = 0; i < n; ++i) {
    const mb_plan &qp = plans ? plans[i] : pl;
    if (qp.kind != MB_PLAN_FUSED) {
      P.alone.push_back(i);
      P.alone_plan.push_back(qp);
      continue;
    }
    mb_plan bp = pl;  // in the batch: the query's cover and predicate order
    bp.cover = qp.cover;
    bp.order_mode = qp.order_mode;
    MB_CHECK(lower_query(E, qs[i], bp, L));
    if (L.empty) continue;  // outputs stay zero
    bool v4 = false;
    MB_CHECK(flatten_prg(&L.prg, L.chk ? 1 : 0, &D, &v4));
    const double sel = est_selectivity(E, L);
    P.sel[i] = sel;
    P.chk[i] = L.chk ? 1 : 0;
    int r = batch_add(B, L, D, P.offs[i], i, sel);
    if (r == BADD_FULL) {
      MB_CHECK(close());
      MB_CHECK(fresh());
      r = batch_add(B, L, D, P.offs[i], i, sel);
    }
    if (r != BADD_OK) P.alone.push_back(i), P.alone_plan.push_back(pl);
  }
  return close();
}

// The slab's tensor maps for tile width T, in device memory (encoded once
// per index).
static mb_status batch_maps(Engine &E, uint32_t V, const void **out) {
  const int k = V == 6 ? 3 : V == 4 ? 2 : V == 2 ? 1 : 0;
  if (!E.bmaps[k]) {
    std::vector<uint8_t> host(BMAP_COUNT * BMAP_BYTES);
    MB_CHECK(batch_encode_maps(E.islab, E.stride, E.nbm, 32 * V, host.data()));
    void *d = nullptr;
    MB_CHECK(E.alloc(&d, host.size()));
    MB_CUDA(cudaMemcpy(d, host.data(), host.size(), cudaMemcpyHostToDevice));
    E.bmaps[k] = d;
  }
  *out = E.bmaps[k];
  return MB_OK;
}

static mb_status batch_staging(Engine &E, BatchHdr **out, uint32_t *slot);

static mb_status batch_opts_check(const mb_batch_opts &o, const char *who) {
  if ((o.words_per_lane && o.words_per_lane != 1 && o.words_per_lane != 2 && o.words_per_lane != 4 &&
       o.words_per_lane != 6) ||
      o.warps == 1 || o.warps > BW_MAX || o.stages > 4 || o.prefetch > MB_PREFETCH_ALL ||
      o.table_kb > 227)
    return fail(MB_ERR_INVALID, "%s: options out of range", who);
  return MB_OK;
}

// Enqueues a planned batch: zeroes the outputs, then per batched launch its
// header (copied through the pinned staging ring into the device header,
// or, with dev_hdrs, already resident there) and the scan; then the queries
// that run alone.
static mb_status batch_launch(Engine &E, const mb_query *qs, const BatchPlanned &P, int64_t *out, uint64_t *nq,
                              uint32_t n, BatchHdr *const *dev_hdrs) {
  MB_CUDA(cudaMemsetAsync(out, 0, P.total * 8, E.stream));
  MB_CUDA(cudaMemsetAsync(nq, 0, (size_t)n * 8, E.stream));
  for (size_t i = 0; i < P.hdrs.size(); ++i) {
    const BatchHdr &h = *P.hdrs[i];
    const void *maps = nullptr;
    MB_CHECK(batch_maps(E, P.cfgs[i].V, &maps));
    const BatchHdr *dh;
    if (dev_hdrs) {
      dh = dev_hdrs[i];
    } else {
      BatchHdr *st = nullptr;
      uint32_t slot = 0;
      MB_CHECK(batch_staging(E, &st, &slot));
      memcpy(st, &h, sizeof(BatchHdr));
      MB_CUDA(cudaMemcpyAsync(E.bq_dev, st, sizeof(BatchHdr), cudaMemcpyHostToDevice, E.stream));
      MB_CUDA(cudaEventRecord(E.bq_copied[slot], E.stream));
      dh = static_cast<const BatchHdr *>(E.bq_dev);
    }
    BatchCfg c = P.cfgs[i];
    if (E.test_stall) {
      c.skip_stage0 = 1;
      c.wait_tries = E.test_tries;
      --E.test_stall;
    }
    MB_CHECK(batch_scan(h, dh, c, maps, out, nq, E.stream));
  }
  if (!P.alone.empty()) {
    Lowered L;
    for (size_t k = 0; k < P.alone.size(); ++k) {
      const uint32_t i = P.alone[k];
      const mb_plan &pl = P.alone_plan[k];
      MB_CHECK(lower_query(E, qs[i], pl, L));
      MB_CHECK(run_lowered(E, L, pl, out + P.offs[i], nq + i, false));
    }
  }
  return MB_OK;
}

// The next staging header of the ring, once its previous copy is done.
static mb_status batch_staging(Engine &E, BatchHdr **out, uint32_t *slot) {
  if (!E.bq_dev) {
    for (int i = 0; i < Engine::BQ_RING; ++i) {
      MB_CUDA(cudaMallocHost(&E.bq_host[i], sizeof(BatchHdr)));
      MB_CUDA(cudaEventCreateWithFlags(&E.bq_copied[i], cudaEventDisableTiming));
    }
    MB_CHECK(E.alloc(&E.bq_dev, sizeof(BatchHdr)));
  }
  const uint32_t i = E.bq_next;
  E.bq_next = (E.bq_next + 1) % Engine::BQ_RING;
  MB_CUDA(cudaEventSynchronize(E.bq_copied[i]));  // an unrecorded event counts as complete
  *out = static_cast<BatchHdr *>(E.bq_host[i]);
  *slot = i;
  return MB_OK;
}

}  // namespace mb

namespace mb {
static mb_status batch_plan_learned(Engine &E, const mb_query *qs, uint32_t n, mb_batch_opts &o, uint32_t &cover,
                                    uint32_t &choice);
}

extern "C" mb_status mb_engine_enqueue_batch(mb_engine *e, const mb_query *qs, uint32_t n, const mb_batch_opts *opts,
                                             int64_t *out_dev, uint64_t *nqual_dev) {
  NvtxRange nvtx_("mb_engine_enqueue_batch");
  if (!e || (!qs && n) || !out_dev || !nqual_dev) return fail(MB_ERR_INVALID, "mb_engine_enqueue_batch: NULL argument");
  Engine &E = e->E;
  MB_CUDA(cudaSetDevice(E.device));
  mb_batch_opts o;
  std::vector<mb_plan> plans;
  if (opts) {
    o = *opts;
  } else if (E.batch_planner) {  // the learned batch plan: launch shape and covers
    uint32_t cover = 0, choice = 0;
    MB_CHECK(batch_plan_learned(E, qs, n, o, cover, choice));
    plans.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
      MB_CHECK(mb_engine_plan_rule(e, &qs[i], &plans[i]));
      plans[i].cover = cover;
    }
  } else if (E.have_tuned) {
    o = E.tuned;  // the autotuner's last choice
  } else {
    memset(&o, 0, sizeof(o));
  }
  MB_CHECK(batch_opts_check(o, "mb_engine_enqueue_batch"));
  BatchPlanned P;
  MB_CHECK(batch_plan(E, qs, n, o, P, plans.empty() ? nullptr : plans.data()));
  return batch_launch(E, qs, P, out_dev, nqual_dev, n, nullptr);
}

extern "C" mb_status mb_engine_enqueue_batch_plans(mb_engine *e, const mb_query *qs, const mb_plan *plans, uint32_t n,
                                                   const mb_batch_opts *opts, int64_t *out_dev, uint64_t *nqual_dev) {
  NvtxRange nvtx_("mb_engine_enqueue_batch_plans");
  if (!e || (!qs && n) || !out_dev || !nqual_dev) return fail(MB_ERR_INVALID, "mb_engine_enqueue_batch_plans: NULL argument");
  Engine &E = e->E;
  MB_CUDA(cudaSetDevice(E.device));
  mb_batch_opts o;
  if (opts) o = *opts;
  else if (E.have_tuned) o = E.tuned;
  else memset(&o, 0, sizeof(o));
  MB_CHECK(batch_opts_check(o, "mb_engine_enqueue_batch_plans"));
  BatchPlanned P;
  MB_CHECK(batch_plan(E, qs, n, o, P, plans));
  return batch_launch(E, qs, P, out_dev, nqual_dev, n, nullptr);
}

extern "C" mb_status mb_engine_batch_info(mb_engine *e, const mb_query *qs, uint32_t n, const mb_batch_opts *opts,
                                          mb_batch_launch_info *launches, uint32_t cap, uint32_t *nlaunches,
                                          uint32_t *nalone) {
  if (!e || (!qs && n) || (!launches && cap)) return fail(MB_ERR_INVALID, "mb_engine_batch_info: NULL argument");
  Engine &E = e->E;
  MB_CUDA(cudaSetDevice(E.device));
  mb_batch_opts o;
  if (opts) o = *opts;
  else if (E.have_tuned) o = E.tuned;  // the autotuner's last choice
  else memset(&o, 0, sizeof(o));
  MB_CHECK(batch_opts_check(o, "mb_engine_batch_info"));
  BatchPlanned P;
  MB_CHECK(batch_plan(E, qs, n, o, P));
  for (size_t i = 0; i < P.hdrs.size() && i < cap; ++i) {
    mb_batch_launch_info &l = launches[i];
    memset(&l, 0, sizeof(l));
    l.queries = P.hdrs[i]->nq;
    l.staged_rows = P.hdrs[i]->nu;
    l.copies = P.hdrs[i]->ncopy;
    l.words_per_lane = P.cfgs[i].V;
    l.warps = P.cfgs[i].warps;
    l.table_slots = P.hdrs[i]->nstab;
    l.chain_entries = P.hdrs[i]->nchain;
    l.stages = P.cfgs[i].stages;
  }
  if (nlaunches) *nlaunches = (uint32_t)P.hdrs.size();
  if (nalone) *nalone = (uint32_t)P.alone.size();
  return MB_OK;
}

extern "C" mb_status mb_engine_query_batch(mb_engine *e, const mb_query *qs, uint32_t n, const mb_batch_opts *opts,
                                           int64_t *out_host, uint64_t *nqual_host) {
  if (!e || (!qs && n) || !out_host) return fail(MB_ERR_INVALID, "mb_engine_query_batch: NULL argument");
  Engine &E = e->E;
  MB_CUDA(cudaSetDevice(E.device));
  const uint64_t total = mb_queries_layout(qs, n, nullptr);
  if (E.bout_cap < total + n) {
    free_one(E.allocs, E.bout);
    E.bout = nullptr;
    MB_CHECK(E.alloc((void **)&E.bout, (total + n) * 8));
    E.bout_cap = total + n;
  }
  MB_CHECK(mb_engine_enqueue_batch(e, qs, n, opts, E.bout, reinterpret_cast<uint64_t *>(E.bout + total)));
  MB_CUDA(cudaMemcpyAsync(out_host, E.bout, total * 8, cudaMemcpyDeviceToHost, E.stream));
  if (nqual_host) MB_CUDA(cudaMemcpyAsync(nqual_host, E.bout + total, (size_t)n * 8, cudaMemcpyDeviceToHost, E.stream));
  MB_CUDA(cudaStreamSynchronize(E.stream));
  const mb_status st = check_device_error(E.stream);
  if (st != MB_OK) {  // a launch gave up part way: its partial sums are not results
    memset(out_host, 0, total * 8);
    if (nqual_host) memset(nqual_host, 0, (size_t)n * 8);
  }
  return st;
}

extern "C" mb_status mb_engine_test_stall(mb_engine *e, uint32_t launches, uint32_t tries) {
  if (!e) return fail(MB_ERR_INVALID, "mb_engine_test_stall: NULL engine");
  e->E.test_stall = launches;
  e->E.test_tries = tries;
  return MB_OK;
}

// ------------------------------------------------------------ batch graphs
struct mb_batch_graph {
  mb_engine *e = nullptr;
  BatchHdr *dh = nullptr;  // the launches' descriptors, resident
  cudaGraph_t g = nullptr;
  cudaGraphExec_t x = nullptr;
};

extern "C" mb_status mb_batch_graph_destroy(mb_batch_graph *g) {
  if (!g) return MB_OK;
  cudaSetDevice(g->e->E.device);
  cudaStreamSynchronize(g->e->E.stream);
  if (g->x) cudaGraphExecDestroy(g->x);
  if (g->g) cudaGraphDestroy(g->g);
  if (g->dh) cudaFree(g->dh);
  delete g;
  return MB_OK;
}

extern "C" mb_status mb_batch_graph_create(mb_engine *e, const mb_query *qs, uint32_t n, const mb_batch_opts *opts,
                                           int64_t *out_dev, uint64_t *nqual_dev, mb_batch_graph **out) {
  return mb_batch_graph_create_plans(e, qs, nullptr, n, opts, out_dev, nqual_dev, out);
}

extern "C" mb_status mb_batch_graph_create_plans(mb_engine *e, const mb_query *qs, const mb_plan *plans, uint32_t n,
                                                 const mb_batch_opts *opts, int64_t *out_dev, uint64_t *nqual_dev,
                                                 mb_batch_graph **out) {
  if (!e || (!qs && n) || !out_dev || !nqual_dev || !out) return fail(MB_ERR_INVALID, "mb_batch_graph_create: NULL argument");
  *out = nullptr;
  Engine &E = e->E;
  MB_CUDA(cudaSetDevice(E.device));
  mb_batch_opts o;
  if (opts) o = *opts;
  else if (E.have_tuned) o = E.tuned;  // the autotuner's last choice
  else memset(&o, 0, sizeof(o));
  MB_CHECK(batch_opts_check(o, "mb_batch_graph_create"));
  BatchPlanned P;
  MB_CHECK(batch_plan(E, qs, n, o, P, plans));
  std::unique_ptr<mb_batch_graph, mb_status (*)(mb_batch_graph *)> G(new mb_batch_graph(), mb_batch_graph_destroy);
  G->e = e;
  const size_t nh = P.hdrs.size();
  std::vector<BatchHdr *> dptr(nh);
  if (nh) {
    MB_CUDA(cudaMalloc(&G->dh, nh * sizeof(BatchHdr)));
    for (size_t i = 0; i < nh; ++i) {
      dptr[i] = G->dh + i;
      MB_CUDA(cudaMemcpy(dptr[i], P.hdrs[i].get(), sizeof(BatchHdr), cudaMemcpyHostToDevice));
    }
  }
  if (!device_error_word()) return fail(MB_ERR_OOM, "mb_batch_graph_create: device error word");
  // one launch outside the capture makes every lazily allocated buffer
  // (tensor maps, plain-path scratch) exist before it
  MB_CHECK(batch_launch(E, qs, P, out_dev, nqual_dev, n, dptr.data()));
  MB_CUDA(cudaStreamSynchronize(E.stream));
  MB_CHECK(check_device_error(E.stream));
  MB_CUDA(cudaStreamBeginCapture(E.stream, cudaStreamCaptureModeRelaxed));
  const mb_status st = batch_launch(E, qs, P, out_dev, nqual_dev, n, dptr.data());
  const cudaError_t ce = cudaStreamEndCapture(E.stream, &G->g);
  MB_CHECK(st);
  MB_CUDA(ce);
  MB_CUDA(cudaGraphInstantiate(&G->x, G->g, 0));
  *out = G.release();
  return MB_OK;
}

extern "C" mb_status mb_batch_graph_launch(mb_batch_graph *g) {
  if (!g || !g->x) return fail(MB_ERR_INVALID, "mb_batch_graph_launch: NULL graph");
  MB_CUDA(cudaSetDevice(g->e->E.device));
  MB_CUDA(cudaGraphLaunch(g->x, g->e->E.stream));
  return MB_OK;
}

// ------------------------------------------------------------ autotuner
extern "C" mb_status mb_engine_tune_batch(mb_engine *e, const mb_query *qs, uint32_t n, uint32_t reps,
                                          mb_batch_opts *best, float *best_ms, uint32_t *tried) {
  NvtxRange nvtx_("mb_engine_tune_batch");
  if (!e || !qs || n == 0 || !best) return fail(MB_ERR_INVALID, "mb_engine_tune_batch: bad argument");
  Engine &E = e->E;
  MB_CUDA(cudaSetDevice(E.device));
  if (reps == 0) reps = 3;
  const uint64_t total = mb_queries_layout(qs, n, nullptr);
  if (E.bout_cap < total + n) {
    free_one(E.allocs, E.bout);
    E.bout = nullptr;
    MB_CHECK(E.alloc((void **)&E.bout, (total + n) * 8));
    E.bout_cap = total + n;
  }
  int64_t *out = E.bout;
  uint64_t *nq = reinterpret_cast<uint64_t *>(E.bout + total);
  uint32_t count = 0;
  std::vector<float> t(reps);
  auto time_of = [&](const mb_batch_opts &o, float *ms) -> mb_status {
    MB_CHECK(batch_opts_check(o, "mb_engine_tune_batch"));
    BatchPlanned P;
    MB_CHECK(batch_plan(E, qs, n, o, P));
    const mb_status w = batch_launch(E, qs, P, out, nq, n, nullptr);  // warm-up
    if (w == MB_ERR_UNSUPPORTED) {  // the shape does not fit on an SM: not a candidate
      MB_CUDA(cudaStreamSynchronize(E.stream));
      *ms = 1e30f;
      return MB_OK;
    }
    MB_CHECK(w);
    for (uint32_t r = 0; r < reps; ++r) {
      MB_CUDA(cudaEventRecord(E.ev0, E.stream));
      MB_CHECK(batch_launch(E, qs, P, out, nq, n, nullptr));
      MB_CUDA(cudaEventRecord(E.ev1, E.stream));
      MB_CUDA(cudaEventSynchronize(E.ev1));
      MB_CUDA(cudaEventElapsedTime(&t[r], E.ev0, E.ev1));
    }
    MB_CHECK(check_device_error(E.stream));
    std::sort(t.begin(), t.end());
    *ms = t[reps / 2];
    ++count;
    return MB_OK;
  };
  mb_batch_opts b;
  memset(&b, 0, sizeof(b));
  float bms = 1e30f;
  auto consider = [&](const mb_batch_opts &o) -> mb_status {
    float ms = 0;
    MB_CHECK(time_of(o, &ms));
    if (ms < bms) bms = ms, b = o;
    return MB_OK;
  };
  // tile width x warps
  for (uint32_t V : {6u, 4u, 2u, 1u})
    for (uint32_t w : {16u, 12u, 8u}) {
      mb_batch_opts o;
      memset(&o, 0, sizeof(o));
      o.words_per_lane = V;
      o.warps = w;
      MB_CHECK(consider(o));
    }
  // shared group tables: as large as fits, 16 KB, 1 KB
  const mb_batch_opts b1 = b;
  for (uint32_t kb : {16u, 1u}) {
    mb_batch_opts o = b1;
    o.table_kb = kb;
    MB_CHECK(consider(o));
  }
  // L2 prefetch of the payload
  const mb_batch_opts b2 = b;
  for (uint32_t pf : {(uint32_t)MB_PREFETCH_NONE, (uint32_t)MB_PREFETCH_ALL}) {
    mb_batch_opts o = b2;
    o.prefetch = pf;
    MB_CHECK(consider(o));
  }
  *best = b;
  E.tuned = b;
  E.have_tuned = true;
  if (best_ms) *best_ms = bms;
  if (tried) *tried = count;
  return MB_OK;
}

// ------------------------------------------------------------ learned planner
namespace mb {

// Popcounts of the program's possible and uncertain bits over its first nw
// words (the planner's 1% sample).
__global__ void sample_popc_kernel(const __grid_constant__ DevPrg P, uint64_t nw, unsigned long long *cnt) {
  unsigned long long pc = 0, uc = 0;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t p[1], u[1];
    vbp_eval<1, true>(P, w, p, u);
    pc += __popc(p[0]);
    uc += __popc(u[0]);
  }
  for (int o = 16; o; o >>= 1) {
    pc += __shfl_down_sync(0xffffffffu, pc, o);
    uc += __shfl_down_sync(0xffffffffu, uc, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (pc) atomicAdd(&cnt[0], pc);
    if (uc) atomicAdd(&cnt[1], uc);
  }
}

// The rule lowering of a query plus its per-predicate facts (template order).
struct QueryFacts {
  Lowered L;
  uint32_t npred = 0;
  double est[4] = {1, 1, 1, 1};  // estimated selected fraction per predicate
  bool full[4] = {}, comp[4] = {};
  uint32_t nb[4] = {}, ne[4] = {};
};

static mb_status query_facts(Engine &E, const mb_query &q, QueryFacts &F) {
  mb_plan pl;
  memset(&pl, 0, sizeof(pl));
  MB_CHECK(lower_query(E, q, pl, F.L));
  F.npred = (uint32_t)std::min<size_t>(4, F.L.preds.size());
  for (uint32_t i = 0; i < F.npred; ++i) {
    const Cover &c = F.L.covers[i];
    F.full[i] = c.full;
    F.comp[i] = c.complement;
    F.nb[i] = c.nb();
    F.ne[i] = (c.left ? 1 : 0) + (c.right ? 1 : 0);
    F.est[i] = c.full ? 1.0 : c.empty ? 0.0 : std::min(1.0, (double)c.est_rows / std::max<uint64_t>(1, E.nrows));
  }
  return MB_OK;
}

static float nlog10(double x, double floor_, double span) {  // log10 scaled into about [0, 1]
  return (float)((log10(std::max(x, floor_)) - log10(floor_)) / span);
}

// Features of n queries.  Each query's program is popcounted over the first
// 1% of the rows (its possible and uncertain bits): the sample passes of a
// chunk of queries are launched back to back and waited for once.
static constexpr uint32_t FEAT_CHUNK = 64;

static mb_status features_of(Engine &E, const mb_query *qs, uint32_t n, QueryFacts *F, float *x) {
  if (!E.d_feat) MB_CHECK(E.alloc((void **)&E.d_feat, 16 * FEAT_CHUNK));
  if (!E.pstream) MB_CUDA(cudaStreamCreateWithFlags(&E.pstream, cudaStreamNonBlocking));
  std::vector<unsigned long long> h(2 * FEAT_CHUNK);
  std::vector<uint64_t> sampled(FEAT_CHUNK);
  for (uint32_t c0 = 0; c0 < n; c0 += FEAT_CHUNK) {
    const uint32_t m = std::min(FEAT_CHUNK, n - c0);
    MB_CUDA(cudaMemsetAsync(E.d_feat, 0, 16 * m, E.pstream));
    for (uint32_t j = 0; j < m; ++j) {
      QueryFacts &Fi = F[c0 + j];
      MB_CHECK(query_facts(E, qs[c0 + j], Fi));
      sampled[j] = 0;
      if (Fi.L.empty || Fi.L.prg.ncols + Fi.L.prg.instrs[0].opcode == 0) continue;
      DevPrg P;
      bool v4 = false;
      MB_CHECK(flatten_prg(&Fi.L.prg, 1, &P, &v4));
      const uint64_t nw = std::max<uint64_t>(1, P.nwords / 100);
      const unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(nw, 256), 148ull * 4);
      sample_popc_kernel<<<grid, 256, 0, E.pstream>>>(P, nw, E.d_feat + 2 * j);
      MB_LAUNCH_CHECK("sample_popc_kernel");
      sampled[j] = nw;
    }
    MB_CUDA(cudaMemcpyAsync(h.data(), E.d_feat, 16 * m, cudaMemcpyDeviceToHost, E.pstream));
    MB_CUDA(cudaStreamSynchronize(E.pstream));
    for (uint32_t j = 0; j < m; ++j) {
      const QueryFacts &Fi = F[c0 + j];
      const mb_query &q = qs[c0 + j];
      float *f = x + (size_t)(c0 + j) * MB_PLAN_FEATURES;
      memset(f, 0, MB_PLAN_FEATURES * sizeof(float));
      if (q.tmpl >= 1 && q.tmpl <= 4) f[q.tmpl - 1] = 1.f;
      double sel = 1;
      for (uint32_t i = 0; i < Fi.npred; ++i) {
        float *g = f + 4 + 5 * i;
        g[0] = log2f(1.f + (float)Fi.nb[i]) / 6.f;
        g[1] = (float)Fi.ne[i] * 0.5f;
        g[2] = nlog10(Fi.est[i], 1e-7, 7.0);
        g[3] = Fi.comp[i] ? 1.f : 0.f;
        g[4] = Fi.full[i] ? 1.f : 0.f;
        sel *= Fi.est[i];
      }
      f[24] = nlog10(sel, 1e-9, 9.0);
      double ssel = 0, sunc = 0;
      if (sampled[j]) {
        const unsigned long long pc = h[2 * j], uc = h[2 * j + 1];
        const double rows = (double)std::min<uint64_t>(E.nrows, sampled[j] * 32);
        ssel = (double)pc / std::max(1.0, rows);
        sunc = pc ? (double)uc / (double)pc : 0.0;
      }
      f[25] = nlog10(ssel, 1e-7, 7.0);
      f[26] = (float)sunc;
      f[27] = log2f((float)std::max<uint32_t>(1, Fi.L.ngroups)) / 16.f;
      f[28] = 0.f;  // the table size is left out: trained at one size, planning at another must not extrapolate it
      f[29] = Fi.L.chk ? 1.f : 0.f;
      f[30] = (float)Fi.L.nbitmaps / 64.f;
      f[31] = 1.f;
    }
  }
  return MB_OK;
}

static void candidate_of(const QueryFacts &F, uint32_t idx, mb_plan &p) {
  memset(&p, 0, sizeof(p));
  p.kind = MB_PLAN_FUSED;
  p.launch.grp_strategy = MB_GRP_AUTO;
  int most = -1, least = -1;
  for (uint32_t i = 0; i < F.npred; ++i) {
    if (F.full[i]) continue;
    if (most < 0 || F.est[i] < F.est[most]) most = (int)i;
    if (least < 0 || F.est[i] > F.est[least]) least = (int)i;
  }
  switch (idx) {
  case 1: p.order_mode = 1; break;
  case 2: p.launch.words_per_lane = 4; break;
  case 3: p.launch.words_per_lane = 1; break;
  case 4:
    if (most >= 0) p.materialise = 1u << most;
    break;
  case 5:
    for (uint32_t i = 0; i < F.npred; ++i)
      if (!F.full[i] && (int)i != least) p.materialise |= 1u << i;
    break;
  case 6: p.kind = MB_PLAN_MATERIALISED; break;
  case 7: p.kind = MB_PLAN_SCAN; break;
  case 8:
    if (F.L.ngroups <= 4096) p.launch.grp_strategy = MB_GRP_SHARED;
    break;
  case 9: p.launch.grp_strategy = MB_GRP_GLOBAL; break;
  case 10: p.launch.grp_strategy = MB_GRP_HASH; break;
  case 11: p.launch.staging = MB_STAGE_TMA; break;
  // pairs of the single changes that were most often best on their own
  case 12: p.launch.words_per_lane = 4, p.launch.grp_strategy = MB_GRP_GLOBAL; break;
  case 13: p.launch.words_per_lane = 1, p.launch.grp_strategy = MB_GRP_GLOBAL; break;
  case 14: p.order_mode = 1, p.launch.words_per_lane = 4; break;
  case 15:
    p.launch.words_per_lane = 4;
    if (F.L.ngroups <= 4096) p.launch.grp_strategy = MB_GRP_SHARED;
    break;
  default: break;  // 0: the rule plan
  }
}

}  // namespace mb

extern "C" mb_status mb_engine_query_features(mb_engine *e, const mb_query *q, float *features) {
  if (!e || !q || !features) return fail(MB_ERR_INVALID, "mb_engine_query_features: NULL argument");
  Engine &E = e->E;
  MB_CUDA(cudaSetDevice(E.device));
  QueryFacts F;
  return features_of(E, q, 1, &F, features);
}

extern "C" mb_status mb_engine_plan_candidate(mb_engine *e, const mb_query *q, uint32_t idx, mb_plan *out) {
  if (!e || !q || !out) return fail(MB_ERR_INVALID, "mb_engine_plan_candidate: NULL argument");
  if (idx >= MB_PLAN_CANDIDATES) return fail(MB_ERR_INVALID, "mb_engine_plan_candidate: candidate %u", idx);
  QueryFacts F;
  MB_CHECK(query_facts(e->E, *q, F));
  candidate_of(F, idx, *out);
  return MB_OK;
}

extern "C" mb_status mb_engine_set_planner(mb_engine *e, mb_mlp *m) {
  if (!e) return fail(MB_ERR_INVALID, "mb_engine_set_planner: NULL engine");
  uint32_t in = 0, out = 0;
  if (m && (!mlp_shape(m, &in, &out) || in != MB_PLAN_FEATURES || out != MB_PLAN_CANDIDATES))
    return fail(MB_ERR_INVALID, "mb_engine_set_planner: the network maps %u features to %u plans, the engine needs "
                "%u to %u", in, out, MB_PLAN_FEATURES, MB_PLAN_CANDIDATES);
  e->E.planner = m;
  return MB_OK;
}

extern "C" mb_status mb_engine_plan_learned(mb_engine *e, const mb_query *qs, uint32_t n, mb_plan *plans,
                                           uint32_t *chosen) {
  NvtxRange nvtx_("mb_engine_plan_learned");
  if (!e || (n && (!qs || !plans))) return fail(MB_ERR_INVALID, "mb_engine_plan_learned: NULL argument");
  Engine &E = e->E;
  MB_CUDA(cudaSetDevice(E.device));
  std::vector<QueryFacts> F(n);
  std::vector<float> x((size_t)n * MB_PLAN_FEATURES);
  if (n) MB_CHECK(features_of(E, qs, n, F.data(), x.data()));
  std::vector<uint32_t> pick(n, 0);
  if (E.planner && n) {
    const uint32_t no = mb_mlp_nparams(E.planner) ? MB_PLAN_CANDIDATES : 0;
    std::vector<float> y((size_t)n * MB_PLAN_CANDIDATES);
    MB_CHECK(mb_mlp_forward(E.planner, x.data(), n, 1, y.data()));
    for (uint32_t i = 0; i < n; ++i) {
      const float *yi = &y[(size_t)i * MB_PLAN_CANDIDATES];
      uint32_t best = 0;
      for (uint32_t c = 1; c < no; ++c)
        if (yi[c] < yi[best]) best = c;
      pick[i] = best;
    }
  }
  for (uint32_t i = 0; i < n; ++i) {
    candidate_of(F[i], pick[i], plans[i]);
    if (chosen) chosen[i] = pick[i];
  }
  return MB_OK;
}

// ------------------------------------------------------------ learned batch planner
// A batch plan: the launch shape (words per lane x warps per CTA) and the
// cover every query of the batch takes.  Candidate c = cover * 9 + shape,
// shape = V index * 3 + warps index, V in {1, 2, 4}, warps in {8, 12, 16},
// cover in {MB_COVER_RULE, MB_COVER_NOEDGE}.
namespace mb {
static void batch_candidate_of(uint32_t idx, mb_batch_opts &o, uint32_t &cover) {
  static const uint32_t Vs[3] = {1, 2, 4}, Ws[3] = {8, 12, 16};
  memset(&o, 0, sizeof(o));
  const uint32_t shape = idx % 9;
  o.words_per_lane = Vs[shape / 3];
  o.warps = Ws[shape % 3];
  cover = idx / 9 == 0 ? MB_COVER_RULE : MB_COVER_NOEDGE;
}

// Features of a batch (planned with the rule, on the host): its size, the
// bitmaps it stages and reads per word, the stages each tile width leaves, its
// queries' estimated selectivities, group counts and templates.  The table
// size is left out, as for the single-query planner: the network is trained
// at one size and plans at another.
static mb_status batch_features_of(Engine &E, const mb_query *qs, uint32_t n, float *f) {
  memset(f, 0, MB_BATCH_FEATURES * sizeof(float));
  mb_batch_opts o;
  memset(&o, 0, sizeof(o));
  BatchPlanned P;
  MB_CHECK(batch_plan(E, qs, n, o, P));
  uint32_t staged = 0, nchain = 0, nconj = 0, nstab = 0;
  for (auto &h : P.hdrs) staged += h->nu, nchain += h->nchain, nconj += h->nconj, nstab += h->nstab;
  double ssel = 0, msel = 0, sg = 0, mg = 0, nmulti = 0, n3 = 0, n2 = 0, n1 = 0, nchk = 0;
  uint32_t tm[4] = {0, 0, 0, 0};
  for (uint32_t i = 0; i < n; ++i) {
    const double sl = P.sel[i];
    ssel += sl, msel = std::max(msel, sl);
    n3 += sl > 1e-3, n2 += sl > 1e-2, n1 += sl > 1e-1;
    const uint32_t ng = query_ngroups(qs[i]);
    sg += ng, mg = std::max<double>(mg, ng), nmulti += ng > 1;
    nchk += P.chk[i];
    if (qs[i].tmpl >= 1 && qs[i].tmpl <= 4) ++tm[qs[i].tmpl - 1];
  }
  const float fn = (float)std::max<uint32_t>(1, n);
  f[0] = log2f(1.f + (float)n) / 8.f;
  f[1] = (float)P.hdrs.size() / 4.f;
  f[2] = (float)P.alone.size() / fn;
  f[3] = (float)staged / 256.f;
  f[4] = log2f(1.f + (float)nchain) / 12.f;
  f[5] = log2f(1.f + (float)nconj) / 10.f;
  if (!P.hdrs.empty()) {
    const BatchHdr &h = *P.hdrs[0];
    static const uint32_t Vs[3] = {1, 2, 4};
    for (int k = 0; k < 3; ++k) {
      mb_batch_opts ov;
      memset(&ov, 0, sizeof(ov));
      ov.words_per_lane = Vs[k];
      const BatchCfg c = batch_cfg(h, ov);
      f[6 + k] = (float)c.stages / 4.f;
    }
  }
  f[9] = nlog10(ssel, 1e-7, 7.0);
  f[10] = nlog10(msel, 1e-7, 7.0);
  f[11] = (float)(n3 / fn), f[12] = (float)(n2 / fn), f[13] = (float)(n1 / fn);
  f[14] = log2f(1.f + (float)(ssel * 1024.0)) / 12.f;  // selected rows per 1024-row tile
  f[15] = log2f(1.f + (float)sg) / 16.f;
  f[16] = log2f(1.f + (float)mg) / 16.f;
  f[17] = (float)(nmulti / fn);
  for (int t = 0; t < 4; ++t) f[18 + t] = (float)tm[t] / fn;
  f[22] = (float)nstab / 6144.f;
  f[23] = (float)(nchk / fn);
  f[24] = (float)nchain / fn / 64.f;  // bitmaps a query reads per word
  f[31] = 1.f;
  return MB_OK;
}

// The learned batch plan of a query batch (the planner network's argmin),
// or the default (rule covers, the engine's launch shape) without a network.
static mb_status batch_plan_learned(Engine &E, const mb_query *qs, uint32_t n, mb_batch_opts &o, uint32_t &cover,
                                    uint32_t &choice) {
  memset(&o, 0, sizeof(o));
  cover = MB_COVER_RULE;
  choice = 0xffffffffu;
  if (!E.batch_planner || n == 0) return MB_OK;
  float x[MB_BATCH_FEATURES], y[MB_BATCH_CANDIDATES];
  MB_CHECK(batch_features_of(E, qs, n, x));
  MB_CHECK(mb_mlp_forward(E.batch_planner, x, 1, 1, y));
  uint32_t best = 0;
  for (uint32_t c = 1; c < MB_BATCH_CANDIDATES; ++c)
    if (y[c] < y[best]) best = c;
  batch_candidate_of(best, o, cover);
  choice = best;
  return MB_OK;
}
}  // namespace mb

extern "C" mb_status mb_engine_batch_features(mb_engine *e, const mb_query *qs, uint32_t n, float *features) {
  if (!e || (!qs && n) || !features) return fail(MB_ERR_INVALID, "mb_engine_batch_features: NULL argument");
  MB_CUDA(cudaSetDevice(e->E.device));
  return batch_features_of(e->E, qs, n, features);
}

extern "C" mb_status mb_engine_batch_candidate(uint32_t idx, mb_batch_opts *opts, uint32_t *cover) {
  if (!opts || !cover || idx >= MB_BATCH_CANDIDATES) return fail(MB_ERR_INVALID, "mb_engine_batch_candidate: bad argument");
  batch_candidate_of(idx, *opts, *cover);
  return MB_OK;
}

extern "C" mb_status mb_engine_set_batch_planner(mb_engine *e, mb_mlp *m) {
  if (!e) return fail(MB_ERR_INVALID, "mb_engine_set_batch_planner: NULL engine");
  if (m) {
    uint32_t in = 0, out = 0;
    if (!mlp_shape(m, &in, &out) || in != MB_BATCH_FEATURES || out != MB_BATCH_CANDIDATES)
      return fail(MB_ERR_INVALID, "mb_engine_set_batch_planner: the network maps %u features to %u outputs, not %u to %u",
                  in, out, MB_BATCH_FEATURES, MB_BATCH_CANDIDATES);
  }
  e->E.batch_planner = m;
  return MB_OK;
}

extern "C" mb_status mb_engine_plan_batch(mb_engine *e, const mb_query *qs, uint32_t n, mb_batch_opts *opts,
                                          uint32_t *cover, uint32_t *choice) {
  if (!e || (!qs && n) || !opts) return fail(MB_ERR_INVALID, "mb_engine_plan_batch: NULL argument");
  MB_CUDA(cudaSetDevice(e->E.device));
  uint32_t cv = 0, ch = 0;
  MB_CHECK(batch_plan_learned(e->E, qs, n, *opts, cv, ch));
  if (cover) *cover = cv;
  if (choice) *choice = ch;
  return MB_OK;
}

