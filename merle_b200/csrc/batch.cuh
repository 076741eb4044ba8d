// batch.cuh - the batched scan: one persistent launch evaluates a batch of
// conjunctive queries over the resident bitmap index and shares every HBM
// read between them.
//
// Per row tile (T = 32 * V words = 1024 * V rows) a CTA stages the tile of
// every DISTINCT bitmap the batch reads (the union: each word fetched from
// HBM once per batch instead of once per query) with a few 2-D tensor copies
// of runs of index-slab rows, and prefetches into L2 the tile's rows of the
// payload columns the batch's ops read densely.  Warps take the batch's
// queries off a counter, costliest first, evaluate each query's conjunctive
// chain on the staged words and run the query's op on its selected rows of
// the tile at once (batch.cu).
//
// The op of a batch query is its mb_op restated per source slot: the
// intersected bounds of the single-term clauses on the slot (re-checked for
// uncertain rows only), the slot's group-key transform (divisions by
// multiplication with a precomputed magic number), and the slots of the
// value.  Ops outside that form (a clause with several terms, a source in two
// keys, sources wider than 4 bytes) run through the single-query path.
#pragma once
#include "common.cuh"

namespace mb {

constexpr uint32_t BQ_MAX = 128;   // queries per launch
constexpr uint32_t BU_MAX = 256;   // bitmap rows staged per tile
constexpr uint32_t BCP_MAX = 48;   // tensor copies per tile
constexpr uint32_t BS_MAX = 16;    // distinct op sources per launch
constexpr uint32_t BC_MAX = 4096;  // chain entries (bins) per launch
constexpr uint32_t BJ_MAX = 1024;  // conjuncts per launch
constexpr uint32_t BW_MAX = 16;    // warps per CTA
constexpr uint32_t BSLOT = MB_MAXSRC;

// One op source of the batch: a column read by row or through a foreign key.
struct BatchSrc {
  const void *col;
  const uint32_t *fk;
  uint32_t dimsz;  // keys >= dimsz make the source invalid (0: unchecked)
  uint32_t width;  // 1, 2 or 4 bytes
};

// Query descriptor: BQD_WORDS 32-bit words.
//   [0] nslot | single group << 8 | vkind << 16 | va << 20 | vb << 24
//   [1] groups   [2] first output slot   [3] row-count slot
//   [4] first conjunct | conjuncts << 16
//   [5] kv mask | filt mask << 8 | key mask << 16 | term mask << 24 (bit s: slot s)
//   [6] compiled op shape (BSHAPES index + 1; 0: the generic drain)
//   [7] slots read through a foreign key (bit s)
//   slot s at 8 + 7 * s:
//     [0] source index | width << 8 | key xform << 16 | division shifts << 24
//     [1] term lo  [2] term hi (inclusive)  [3] division magic  [4] key base
//     [5] key multiplier  [6] divisor
enum : uint32_t { BQD_SLOT0 = 8, BQD_SLOTW = 7, BQD_WORDS = 8 + 7 * BSLOT };

// Op shapes with a compiled drain: which slots every row loads (kv), which
// only uncertain rows load (filt), which are group-key slots and which of
// those take the year of a date (the others divide by their divisor, 1 for
// an identity key, by the magic number of the descriptor), the value kind and
// its slots.  The engine's four query templates lower to these; any other op
// runs the generic drain.
struct BShape {
  uint32_t ns, kv, filt, keym, yearm, vk, va, vb;
};
constexpr BShape BSHAPES[] = {
    {4, 0x0a, 0x07, 0x00, 0x00, MB_V_MUL, 3, 1},  // tmpl 1
    {4, 0x0e, 0x03, 0x06, 0x04, MB_V_COL, 3, 0},  // tmpl 2
    {4, 0x0f, 0x07, 0x07, 0x02, MB_V_COL, 3, 0},  // tmpl 3
    {6, 0x3b, 0x0f, 0x0b, 0x02, MB_V_SUB, 4, 5},  // tmpl 4
};
constexpr uint32_t BNSHAPE = sizeof(BSHAPES) / sizeof(BSHAPES[0]);

struct BatchHdr {
  uint64_t nrows, nwords;
  uint64_t stride;       // words per slab row: a multiple of 32, >= nwords
  const uint32_t *slab;
  uint32_t nslab;        // rows of the slab
  uint32_t nu;           // rows staged per tile
  uint32_t nq, nsrc, nchain;
  uint32_t pf_mask;      // bit i: prefetch source i's row-indexed column into L2
  uint32_t ncopy;
  // The staging copies of a tile: slab rows [r0, r0 + h) to stage rows
  // [t0, t0 + h), packed r0 | t0 << 12 | (h - 1) << 24 (1 <= h <= 256).
  uint32_t copy[BCP_MAX];
  BatchSrc src[BS_MAX];
  uint32_t Qd[BQ_MAX * BQD_WORDS];
  uint16_t chain[BC_MAX];  // one entry per bin: its stage row (slab row while the batch is built)
  uint32_t conj[BJ_MAX];   // one entry per conjunct (BJ_*)
  uint32_t nconj;
  uint8_t order[BQ_MAX];   // the order in which warps take the queries (costliest first)
  // Group tables in shared memory: query q sums into slots [toff[q],
  // toff[q] + groups) of each CTA's table (0xffffffff: into the output
  // directly), nstab slots in all.
  uint32_t toff[BQ_MAX];
  uint32_t nstab;
};

// A query's conjunctive program: conjuncts, each the OR of its bins (edge
// bins also mark uncertain rows); the query is the AND of its conjuncts (of
// the complement of a negated one).  A conjunct entry gives its first chain
// entry, its middle bins and its edge bins (the middle ones first in the
// chain), and whether it is negated.
enum : uint32_t {
  BJ_FIRST = 0xfffu, BJ_NMID_SHIFT = 12, BJ_NEDGE_SHIFT = 20, BJ_NEG = 1u << 24
};  // first | nmid << 12 (8 bits) | nedge << 20 (4 bits) | negated

// Launch shape of the batched scan.
struct BatchCfg {
  uint32_t V;       // words per lane: tile = 32 * V words
  uint32_t warps;   // warps per CTA
  uint32_t stages;  // staged tiles in flight per CTA
  uint32_t cps;     // CTAs per SM (0: as many as fit)
  uint32_t wait_tries;   // try limit of a stage wait (0: 2^20, about a second)
  uint32_t skip_stage0;  // tests only: the first stage is armed and never filled, so its wait runs out
  uint32_t buf;          // rows of a worker warp's chunk buffer: 256 (or 0) or 1024
};

// Tensor maps of a bitmap slab for one tile width T (words): map h - 1 has
// a box of T words x h rows, h = 1..BU_MAX.  A staging copy of h rows uses
// map h - 1, so every run of rows is one copy.
constexpr uint32_t BMAP_COUNT = BU_MAX;
constexpr size_t BMAP_BYTES = 128;  // sizeof(CUtensorMap)
mb_status batch_encode_maps(const uint32_t *slab, uint64_t stride, uint32_t nslab, uint32_t T, void *host_maps);

// Launches the batched scan over the header at dh (device copy of h, which
// the host keeps for the sizes) with the slab's maps for T = 32 * cfg.V in
// device memory at maps; out / nqual are zeroed by the caller.
mb_status batch_scan(const BatchHdr &h, const BatchHdr *dh, const BatchCfg &cfg, const void *maps, int64_t *out,
                     uint64_t *nqual, cudaStream_t st);

// Shared-memory bytes of a launch (0 if the configuration is invalid).
size_t batch_smem(const BatchHdr &h, const BatchCfg &cfg);

}  // namespace mb
