// engine.h - internal C++ view of mb_engine: resident star schema, canonical
// bitmap index, the rule planner and query execution.
#pragma once
#include <memory>
#include <string>
#include <vector>
#include "common.cuh"

namespace mb {

// One partition of an indexed column's value domain into bins.
struct Level {
  std::vector<uint64_t> bounds;  // nbins + 1 ascending boundaries
  uint32_t *slab = nullptr;      // nbins bitmaps at `stride` words
  std::vector<uint64_t> pop;     // rows per bin
  uint32_t nbins() const { return (uint32_t)bounds.size() - 1; }
};

// An indexed column: its value source and levels, coarse to fine (every
// coarse boundary is also a fine boundary).
struct IdxCol {
  const char *name = "";
  mb_src src{};
  uint64_t dom_lo = 0, dom_hi = 0;
  std::vector<Level> levels;
};

enum { IC_DATE = 0, IC_DISC, IC_QTY, IC_CCITY, IC_SCITY, IC_MFGR, IC_N };

// A predicate lo <= value < hi on an indexed column.
struct Pred {
  int col;
  uint64_t lo, hi;
};

// The bitmaps that answer one predicate.
struct Cover {
  std::vector<const uint32_t *> mid;
  const uint32_t *left = nullptr, *right = nullptr;
  bool complement = false;  // the program takes NOT of the (exact) cover
  bool empty = false;       // no row qualifies
  bool full = false;        // every row qualifies: no operand needed
  uint64_t est_rows = 0;    // rows the predicate selects (from bin popcounts)
  uint64_t edge_rows = 0;   // rows in edge bins (candidate check)
  uint32_t nb() const { return (uint32_t)mid.size() + (left ? 1 : 0) + (right ? 1 : 0); }
  bool chk() const { return left || right; }
};

// A query lowered to the C ABI's program + op.
struct Lowered {
  mb_vprg prg{};
  const uint32_t *mids[MB_MAXCOLS][MB_MAXBINS] = {};
  mb_op op{};
  uint32_t ngroups = 1;
  bool empty = false;
  uint32_t nbitmaps = 0;
  bool chk = false;
  std::vector<Pred> preds;
  std::vector<Cover> covers;
  int col_pred[MB_MAXCOLS] = {};   // predicate (template order) of each program operand
  uint64_t canonical_bitmaps = 0;  // plan-independent: min(direct, complement) exact cover
  // Back to the state of a fresh Lowered for the fields lowering reads before
  // writing (prg, op and mids are rewritten in full, the vectors keep their
  // storage).
  void reset() {
    ngroups = 1;
    empty = false;
    nbitmaps = 0;
    chk = false;
    preds.clear();
    covers.clear();
    for (int &c : col_pred) c = 0;
    canonical_bitmaps = 0;
  }
};

struct Engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // star schema
  uint64_t nrows = 0, stride = 0;
  uint32_t k = 0, width4 = 0;
  uint64_t ncust = 0, nsupp = 0, npart = 0;  // without the pad key
  void *custkey = nullptr, *partkey = nullptr, *suppkey = nullptr, *orderdate = nullptr,
       *quantity = nullptr, *discount = nullptr, *extendedprice = nullptr, *revenue = nullptr,
       *supplycost = nullptr, *suppcity = nullptr;
  uint8_t *custcity = nullptr, *suppcity_dim = nullptr;
  uint16_t *partmfgr = nullptr;
  // Denormalised dimension attributes, one per fact row (custcity[custkey],
  // partmfgr[partkey]), built with the index: the ops and the index build
  // read them directly instead of probing through the foreign key.
  uint8_t *custcity_row = nullptr;
  uint16_t *partmfgr_row = nullptr;
  IdxCol idx[IC_N];
  // Every bitmap of the index in one slab, `stride` words apart (level by
  // level, bin by bin): the batched scan stages a tile of any run of them
  // with one 2-D tensor copy.
  uint32_t *islab = nullptr;
  uint32_t nbm = 0;  // bitmaps in the slab
  // Levels the index keeps (bit i: the i-th level in column order; the
  // canonical index has 10: date year/month, discount, quantity, customer
  // and supplier city region/nation, part mfgr/category).
  uint32_t level_mask = MB_LEVELS_ALL;
  void *bmaps[4] = {};  // the slab's tensor maps for tiles of 32, 64, 128, 192 words (device)
  bool indexed = false;
  float index_build_ms = 0;
  // query scratch
  int64_t *d_out = nullptr;
  uint64_t *d_nqual = nullptr;
  int64_t *h_out = nullptr;  // pinned
  uint64_t *h_nqual = nullptr;
  uint32_t out_cap = 0;
  uint32_t *tmp_bits = nullptr;  // materialisation / row-list scratch
  uint64_t tmp_words = 0;
  uint32_t *rows = nullptr;
  uint64_t rows_cap = 0;
  uint64_t *d_rowcnt = nullptr;  // row count of the materialised plan
  std::vector<void *> allocs;
  unsigned long long *d_feat = nullptr;  // the planner's sample popcounts, a pair per query
  // the planner's sample pass runs on its own stream: it reads only the index
  // slab, complete once indexed is set, and waiting for it must not wait for
  // queries in flight on the engine stream
  cudaStream_t pstream = nullptr;
  mb_mlp *planner = nullptr;             // borrowed (mb_engine_set_planner)
  mb_mlp *batch_planner = nullptr;       // borrowed (mb_engine_set_batch_planner)
  // batch descriptors: a ring of pinned host staging headers (each reusable
  // once its copy event completed) and the device copy
  static constexpr int BQ_RING = 4;
  void *bq_host[BQ_RING] = {}, *bq_dev = nullptr;
  cudaEvent_t bq_copied[BQ_RING] = {};
  uint32_t bq_next = 0;
  // the autotuner's last launch shape, used by batches enqueued without options
  mb_batch_opts tuned{};
  bool have_tuned = false;
  // tests of the bounded waits (mb_engine_test_stall): batched launches left
  // to stall, and their try limit
  uint32_t test_stall = 0, test_tries = 0;
  int64_t *bout = nullptr;  // device results of mb_engine_query_batch
  uint64_t bout_cap = 0;
  // timing: per-query event pairs of the last enqueue, and markers
  std::vector<cudaEvent_t> qev;
  uint32_t qev_used = 0;
  cudaEvent_t marks[8] = {};

  ~Engine();
  uint32_t fact_width(const char *col) const;
  mb_status ensure_out(uint32_t ngroups);
  mb_status ensure_tmp(uint64_t words);
  mb_status ensure_rows(uint64_t n);
  mb_status alloc(void **p, size_t bytes);
  void free_star();
  void free_denorm();
  void free_bmaps();
  void drop_index();  // frees the slab and its tensor maps; the levels keep their bounds
  mb_status setup_index_cols();
  // Customer city / part mfgr of a row: the denormalised column when built,
  // else a probe of the dimension through the foreign key.
  mb_src ccity_src() const;
  mb_src mfgr_src() const;
  mb_status build_denorm();
  mb_status enqueue_denorm(unsigned long long *d_bad, cudaStream_t st);
};

// The op functors s1op..s4op (ssb/lambdas.cuh:19-152) of a template query as
// an mb_op over the given sources (engine.cu).
struct SsbSrc {
  mb_src date, disc, qty, eprice, rev, scost, scity, ccity, mfgr;
};
void ssb_build_op(const SsbSrc &S, const mb_query &q, mb_op &out);

// The layer widths of a planner network (mlp.cu); false for NULL.
bool mlp_shape(const mb_mlp *m, uint32_t *in, uint32_t *out);

// Planner and lowering (engine.cu).
// The cheapest cover of [lo, hi) with c's levels; *cost_out (if given) = its
// cost in bytes (bitmap bytes + candidate-check sectors of its edge rows).
Cover plan_cover(const IdxCol &c, uint64_t lo, uint64_t hi, uint64_t W, int nchk_sources, uint64_t *cost_out = nullptr,
                 uint32_t mode = MB_COVER_RULE);
// stats: also count the plan-independent canonical bitmaps (query stats only)
mb_status lower_query(Engine &E, const mb_query &q, const mb_plan &plan, Lowered &L, bool stats = false);
uint32_t query_ngroups(const mb_query &q);
mb_status run_lowered(Engine &E, Lowered &L, const mb_plan &plan, int64_t *d_out, uint64_t *d_nq, bool zero);

// p &= ~u over the words of an nrows bitmap (grpby.cu).
mb_status certain_of(uint32_t *p, const uint32_t *u, uint64_t nrows, cudaStream_t st);
// mb_vprg_grpby with the output zeroing optional (grpby.cu).
mb_status fused_grpby(const mb_vprg *p, const mb_op *op, uint32_t nr_grp, int64_t *out, uint64_t *nqual,
                      const mb_launch *launch, cudaStream_t st, bool zero);

}  // namespace mb

struct mb_engine {
  mb::Engine E;
};
