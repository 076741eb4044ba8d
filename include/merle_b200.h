/*
 * merle_b200.h - C ABI of the B200 (sm_100a) fused bitmap-index query engine.
 *
 * The hot path this library implements is the reference's fused bitmap-index
 * query path:
 *   1. bitmap-index creation over fact columns (bmpidx_create.cu:14-136,
 *      kernels primitive.cuh:88-118);
 *   2. the virtual bitmap program (VBP) that combines predicate bitmaps with
 *      AND / OR / NOT / ANDM / ORM without materialising intermediates
 *      (primitive.cuh:165-338);
 *   3. the fused dimension join-probe plus group-by SUM (primitive.cuh:340-445
 *      driving the op functors of ssb/lambdas.cuh:19-152 and synth/synthdemo.cu:7-53).
 *
 * Conventions (all entry points):
 *  - Every function returns an mb_status; on failure mb_last_error() gives a
 *    thread-local message.  Nothing calls exit() and no kernel traps.
 *  - Pointers documented as "device" are CUDA device addresses; "host" are
 *    host addresses.  `stream` is a cudaStream_t passed as void* (NULL = legacy
 *    default stream).  Asynchronous calls return once the work is enqueued.
 *  - Bitmaps: bit i of 32-bit word w is row 32*w + i (LSB first), as the
 *    reference's __ballot_sync layout (primitive.cuh:96-98).  A bitmap over n
 *    rows has mb_bitmap_words(n) = ceil(n/32) words; bits of rows >= n are 0.
 *    Bitmaps produced by this library are padded to mb_bitmap_stride(n) words
 *    (a multiple of 32 words) and 256-byte aligned.
 *  - Group results are int64 sums (two's complement wrap), where the reference
 *    sums uint32 (primitive.cuh:395,444): (uint32)result equals the reference's
 *    value on the same inputs.
 */
#ifndef MERLE_B200_H
#define MERLE_B200_H
#include <stddef.h>
#include <stdint.h>

/* Symbols of the shared library are exported with default visibility; the
 * library is compiled with -fvisibility=hidden so nothing else leaks. */
#if defined(MB_BUILDING_LIBRARY) && defined(__GNUC__)
#define MB_API __attribute__((visibility("default")))
#else
#define MB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------- */
/* Status                                                                    */
/* ------------------------------------------------------------------------- */
typedef enum mb_status {
  MB_OK = 0,
  MB_ERR_INVALID = 1,     /* bad argument, limit exceeded, misaligned pointer */
  MB_ERR_OOM = 2,         /* device or host allocation failed */
  MB_ERR_CUDA = 3,        /* a CUDA runtime call or launch failed */
  MB_ERR_TIMEOUT = 4,     /* a bounded device-side wait ran out */
  MB_ERR_UNSUPPORTED = 5, /* feature not available in this build */
  MB_ERR_IO = 6,          /* file open / read / write failed */
  MB_ERR_REJECTED = 7,    /* serving: the request can never fit the admission budget */
  MB_ERR_CANCELLED = 8    /* serving: the request was cancelled before it launched */
} mb_status;

/* Thread-local message for the last failing call on this thread. */
MB_API const char *mb_last_error(void);
/* Library version string. */
MB_API const char *mb_version(void);

/* Words of a bitmap over n rows: ceil(n / 32) (bmpidx_create.cu:40). */
MB_API uint64_t mb_bitmap_words(uint64_t nrows);
/* Padded word stride this library uses between bitmaps of one slab. */
MB_API uint64_t mb_bitmap_stride(uint64_t nrows);

/* ------------------------------------------------------------------------- */
/* Limits (the reference's are MAXBIN_PERCOL=4, MAXCOLS=4, MAXNINSTR=6,      */
/* primitive.cuh:121; these are raised so that e.g. a 25-bin OR fits)       */
/* ------------------------------------------------------------------------- */
#define MB_MAXCOLS 8     /* memory operands of one program */
#define MB_MAXBINS 64    /* middle bins of one memory operand */
#define MB_MAXPTRS 128   /* all bitmaps of one program */
#define MB_MAXNINSTR 16  /* instructions of one program */
#define MB_NREGS 4       /* virtual registers (reference: 3) */
#define MB_MAXSRC 8      /* value sources of one op */
#define MB_MAXCLAUSE 6   /* AND-ed filter clauses of one op */
#define MB_MAXTERM 16    /* range terms over all clauses of one op */
#define MB_MAXKEY 4      /* group-key fields of one op */

/* ------------------------------------------------------------------------- */
/* Virtual bitmap program (primitive.cuh:135-198)                            */
/* ------------------------------------------------------------------------- */
/* Opcodes keep the reference's numbering (enum ops, primitive.cuh:169-173). */
typedef enum mb_opcode {
  MB_END = 0,  /* no more instructions */
  MB_AND = 1,  /* r[dst] &= r[src1] */
  MB_OR = 2,   /* r[dst] |= r[src1] */
  MB_NOT = 3,  /* r[dst] = ~r[src1] */
  MB_ANDM = 4, /* r[dst] &= OR of the bins of cols[src1] */
  MB_ORM = 5   /* r[dst] |= OR of the bins of cols[src1] */
} mb_opcode;

/* One instruction (struct vprg::instr, primitive.cuh:176-181). */
typedef struct mb_instr {
  uint8_t opcode, dstreg, src1, src2;
} mb_instr;

/* Bitmap index of one column restricted to a query range (struct col,
 * primitive.cuh:135-162): middle bins lie inside the range; leftmost and
 * rightmost are edge bins that need the candidate check. */
typedef struct mb_col {
  uint32_t nmiddle;                /* <= MB_MAXBINS */
  const uint32_t *const *middle;   /* host array of nmiddle device bitmaps */
  const uint32_t *leftmost;        /* device bitmap or NULL */
  const uint32_t *rightmost;       /* device bitmap or NULL */
} mb_col;

/* The program (struct vprg, primitive.cuh:165-198).  The result is r0.  The
 * instruction list ends at the first MB_END or after MB_MAXNINSTR. */
typedef struct mb_vprg {
  uint64_t factsz;                 /* rows */
  uint32_t ncols;                  /* memory operands in use */
  mb_col cols[MB_MAXCOLS];
  mb_instr instrs[MB_MAXNINSTR];
} mb_vprg;

/* 1 if no operand has an edge bin (vprg::is_nochk, primitive.cuh:190-195). */
MB_API int mb_vprg_is_nochk(const mb_vprg *p);

/* ------------------------------------------------------------------------- */
/* Query operator (the op functors of ssb/lambdas.cuh:19-152 and             */
/* synth/synthdemo.cu:7-53, restated declaratively so they cross a C ABI)    */
/* ------------------------------------------------------------------------- */
/* A value source: a fact column read at the row, or a dimension attribute
 * read through a foreign key: dim[fk[row]] (the join probe). */
typedef struct mb_src {
  const void *col;      /* device: fact column, or dimension array when fk != NULL */
  const uint32_t *fk;   /* device foreign-key fact column, or NULL */
  uint64_t dimsz;       /* fk != NULL and dimsz != 0: keys >= dimsz eliminate the row */
  uint32_t width;       /* element bytes: 1, 2, 4 or 8 (unsigned) */
  uint32_t pad_;
} mb_src;

/* Range term lo <= value < hi (all reference ranges are half-open). */
typedef struct mb_term {
  uint32_t src;
  uint32_t pad_;
  uint64_t lo, hi;
} mb_term;

/* Group-key field: mul * (xform(value) - base), summed over fields in uint32
 * arithmetic (the mixed-radix group indices of s2op..s4op). */
typedef enum mb_xform {
  MB_X_ID = 0,   /* value */
  MB_X_DIV = 1,  /* value / div (the /10 nation and /40 category scaling) */
  MB_X_YEAR = 2  /* ssbDateToYear(value) (ssb/ssbdemo.h:28-39) */
} mb_xform;

typedef struct mb_key {
  uint32_t src, xform, div, base, mul;
} mb_key;

typedef enum mb_vkind {
  MB_V_ONE = 0,  /* COUNT: value 1 */
  MB_V_COL = 1,  /* src[va] */
  MB_V_MUL = 2,  /* src[va] * src[vb] (int64, exact) */
  MB_V_SUB = 3   /* src[va] - src[vb] (int64, exact) */
} mb_vkind;

/* The operator applied to every selected row (op(row, chk) of
 * primitive.cuh:383-384,431-432).  When the row is uncertain (chk) all filter
 * clauses are re-evaluated: the row passes if every clause has a satisfied
 * term.  The group index is the key sum; indices >= nr_grp eliminate the row
 * (primitive.cuh:34,385,433). */
typedef struct mb_op {
  uint32_t nsrc;
  mb_src src[MB_MAXSRC];
  uint32_t nclause;
  uint32_t clause_len[MB_MAXCLAUSE];   /* terms of each clause, in order */
  mb_term terms[MB_MAXTERM];
  uint32_t nkey;
  mb_key keys[MB_MAXKEY];
  uint32_t vkind, va, vb;
  uint32_t pad_;
} mb_op;

/* ------------------------------------------------------------------------- */
/* Launch / plan knobs for the fused kernel                                  */
/* ------------------------------------------------------------------------- */
typedef enum mb_grp_strategy {
  MB_GRP_AUTO = 0,
  MB_GRP_SHARED = 1,  /* dense per-CTA shared-memory partial table */
  MB_GRP_GLOBAL = 2,  /* warp-aggregated atomics straight into global memory */
  MB_GRP_HASH = 3     /* per-CTA shared-memory hash table over (group, sum),
                         for large group domains that few rows touch */
} mb_grp_strategy;

typedef struct mb_launch {
  uint32_t grp_strategy;  /* mb_grp_strategy */
  uint32_t warps_per_cta; /* 0 = auto (4 / 8 / 16) */
  uint32_t ctas_per_sm;   /* 0 = auto (occupancy) */
  uint32_t words_per_lane;/* 0 = auto; 1, 2 or 4 bitmap words per lane */
  uint32_t staging;       /* mb_staging: how operand bitmaps reach the program */
} mb_launch;

typedef enum mb_staging {
  MB_STAGE_AUTO = 0,    /* conjunctive programs: warp-independent tiles with all
                           operand loads batched; others: MB_STAGE_DIRECT */
  MB_STAGE_DIRECT = 1,  /* the instruction interpreter with per-thread loads */
  MB_STAGE_TMA = 2      /* every operand tile staged in shared memory by TMA
                           bulk copies, double-buffered per CTA */
} mb_staging;

/* ------------------------------------------------------------------------- */
/* L2 kernels over raw device buffers                                        */
/* ------------------------------------------------------------------------- */

/* One pass over a column writes nbins bin bitmaps, bin j = [lo[j], hi[j])
 * (create_bin, bmpidx_create.cu:14-56, kernel primitive.cuh:102-118).  When
 * src->fk != NULL the value is dim[fk[row]] and keys >= dimsz give no bit
 * (bmpidx_create.cu:26-27).  out: device, nbins bitmaps at a stride of
 * `stride_words` words (>= mb_bitmap_words(n), multiple of 4); popcounts:
 * optional device uint64[nbins] (accumulated: zero it first), or NULL. */
MB_API mb_status mb_bitmap_create(const mb_src *src, uint64_t nrows, const uint64_t *lo,
                           const uint64_t *hi, uint32_t nbins, uint32_t *out,
                           uint64_t stride_words, uint64_t *popcounts, void *stream);

/* Several levels of bins from ONE pass over a column (a hierarchy such as the
 * years and months of a date, or the regions and nations of a city).  The
 * reference builds every level with its own create_bin pass
 * (bmpidx_create.cu:14-56, driven per level by ssb/bmpidx-create.cu:56-116);
 * here each row's bin in every level comes from one lookup, so the column is
 * read once.  Level l writes levels[l].nbins bitmaps (bin j = [lo[j], hi[j]))
 * to levels[l].out, `stride_words` apart, and accumulates their popcounts
 * into levels[l].popcounts (device uint64[nbins], or NULL).  src, nrows and
 * the stride as for mb_bitmap_create.  Levels with overlapping or unsorted
 * bins, 255 bins or more, or a value domain too wide for the one-pass lookup
 * run one mb_bitmap_create pass per level instead (same results). */
#define MB_MAXLEVELS 4
typedef struct mb_level {
  const uint64_t *lo, *hi; /* host: nbins bounds each */
  uint32_t nbins;
  uint32_t pad_;
  uint32_t *out;           /* device: nbins bitmaps, 16-byte aligned */
  uint64_t *popcounts;     /* device: nbins (accumulated), or NULL */
} mb_level;
MB_API mb_status mb_bitmap_create_levels(const mb_src *src, uint64_t nrows, const mb_level *levels,
                                         uint32_t nlevels, uint64_t stride_words, void *stream);

/* Materialised stage 1 (abla::_stg1, primitive_abla.cuh:262-288): runs the
 * program and writes the possible bitmap (and, when chk, the uncertain one).
 * chk selects vprg::chk vs vprg::nochk semantics.  popcount: optional device
 * uint64 (accumulated) of possible bits. */
MB_API mb_status mb_vprg_eval(const mb_vprg *p, int chk, uint32_t *possible,
                       uint32_t *uncertain, uint64_t *popcount, void *stream);

/* Materialised stage 2 (abla::_stg2, primitive_abla.cuh:290-354): bitmap to a
 * row-id list in ascending row order; uncertain rows carry bit 31
 * (primitive_abla.cuh:346).  count: device uint64, set (not accumulated).
 * rows: device, capacity >= popcount of `possible`. */
MB_API mb_status mb_bitmap_to_rows(const uint32_t *possible, const uint32_t *uncertain,
                            uint64_t nrows, uint32_t *rows, uint64_t *count,
                            void *stream);

/* No-allocation variant of mb_bitmap_to_rows.  It has no counterpart in the
 * reference.  Some callers cannot let a library allocate device memory during
 * a query: hosts that hand the whole device to their own memory pool (where a
 * cudaMalloc from a plugin fails or fragments the pool), and latency-critical
 * callers for whom the device-wide synchronisation that cudaMalloc and
 * cudaFree may cause is not acceptable.  This entry point calls no cudaMalloc,
 * cudaFree or other allocating routine: its only scratch (the per-segment row
 * offsets, one 32-bit word per 65,536 rows) is a fixed 64 KiB array compiled
 * into the library, which every device that loads the library holds until the
 * process exits.  The caller still provides `rows` and `count`.
 *  - Limit: nrows <= MB_NOALLOC_MAX_ROWS (2^30); larger inputs are rejected
 *    with MB_ERR_INVALID before any device work.
 *  - The first call on each device looks up the array's device address with
 *    that device current; make that first call before capturing the stream
 *    into a CUDA graph.  The address is kept for the life of the process: a
 *    cudaDeviceReset while the library is loaded is not supported (it would
 *    leave the kept address stale; mb_bitmap_to_rows keeps its scratch
 *    buffer the same way).
 *  - Every call on a device shares the one array.  Calls that may overlap on
 *    the GPU (different streams, or different host threads without ordering)
 *    race on it and corrupt each other's results; order them on one stream.
 * Output is identical to mb_bitmap_to_rows. */
#define MB_NOALLOC_MAX_ROWS 1073741824ull
MB_API mb_status mb_bitmap_to_rows_noalloc(const uint32_t *possible, const uint32_t *uncertain,
                                           uint64_t nrows, uint32_t *rows, uint64_t *count,
                                           void *stream);

/* Materialised stage 3 (abla::_stg3, primitive_abla.cuh:356-394): applies the
 * op to a row list and aggregates.  The row count is read on the device (no
 * host round trip, unlike primitive_abla.cuh:437).  out: device int64[nr_grp]
 * and qualifying-row count: device uint64; both overwritten. */
MB_API mb_status mb_rows_grpby(const uint32_t *rows, const uint64_t *count, uint64_t capacity,
                        const mb_op *op, uint32_t nr_grp, int64_t *out,
                        uint64_t *nqual, void *stream);

/* The fused kernel (vprg_grpby, primitive.cuh:340-445): program -> compaction
 * -> op -> group-by in one launch.  Uses the chk algebra iff the program has
 * edge bins.  out: device int64[nr_grp], nqual: device uint64 (rows
 * aggregated); both overwritten.  launch may be NULL (auto). */
MB_API mb_status mb_vprg_grpby(const mb_vprg *p, const mb_op *op, uint32_t nr_grp,
                        int64_t *out, uint64_t *nqual, const mb_launch *launch,
                        void *stream);

/* No-index plan (grpby, primitive.cuh:16-48): every row runs the op with the
 * candidate check on.  out / nqual as mb_vprg_grpby. */
MB_API mb_status mb_join_grpby(uint64_t nrows, const mb_op *op, uint32_t nr_grp,
                        int64_t *out, uint64_t *nqual, void *stream);

/* The same result through Crystal-style hash joins (the reference's comparison
 * system, crystal/src/ssb/q21.cu and siblings): for each foreign key whose
 * dimension attributes carry clauses of their own (every term of the clause
 * reads that key's dimension, whose size dimsz must be set), the dimension
 * rows passing them go into an open-addressing table keyed by dimension key
 * and carrying the op's attributes on that key (up to 3, each <= 4 bytes; up
 * to 4 keys); one pass over the fact rows then evaluates the fact-column
 * clauses, probes the tables (a miss eliminates the row) and aggregates.
 * Tables up to 48 KB are copied into each CTA's shared memory.  Waits for
 * the stream once (the table sizes).  An op without such clauses runs as
 * mb_join_grpby. */
MB_API mb_status mb_hash_join_grpby(uint64_t nrows, const mb_op *op, uint32_t nr_grp,
                                    int64_t *out, uint64_t *nqual, void *stream);

/* ------------------------------------------------------------------------- */
/* Host planning helpers of the reference's operator API                     */
/* ------------------------------------------------------------------------- */
/* col::from_bin (bmpidx_create.cu:138-163): maps [min, max) onto bins
 * bins[0..nbin) with bounds[0..nbin]: bins fully inside become middle bins,
 * partially covered end bins become leftmost / rightmost (candidate check).
 * An empty col (nmiddle 0, no edges) means the range is not coverable.
 * `mid_storage` (host, MB_MAXBINS entries) receives the middle pointers and
 * out->middle points into it.  Host-only: never dereferences the bitmaps.
 * Returns MB_ERR_INVALID if more than MB_MAXBINS middle bins are needed (the
 * reference silently overflows its 4-entry array, primitive.cuh:155). */
MB_API mb_status mb_col_from_bin(uint32_t nbin, const uint32_t *const *bins,
                                 const uint64_t *bounds, uint64_t min, uint64_t max,
                                 mb_col *out, const uint32_t **mid_storage);

/* col::from_bin2 (bmpidx_create.cu:165-173): coarse bins first; if they need a
 * candidate check, the fine bins instead. */
MB_API mb_status mb_col_from_bin2(uint32_t nc, const uint32_t *const *coarse,
                                  const uint64_t *cbounds, uint32_t nf,
                                  const uint32_t *const *fine, const uint64_t *fbounds,
                                  uint64_t min, uint64_t max, mb_col *out,
                                  const uint32_t **mid_storage);

/* struct recipe (primitive.cuh:448-474): per-query bitmaps for up to
 * MB_RECIPE_COLS predicates, built on the device from a column (fk == NULL,
 * create_select) or a dimension attribute through a foreign key (create_join,
 * keys >= dimsz give no bit; 0xffffffff = no check). */
#define MB_RECIPE_COLS 4
typedef struct mb_recipe {
  uint64_t factsz;
  uint32_t nbit[MB_RECIPE_COLS];          /* attribute bits: <=8, <=16, <=32, <=64 */
  uint32_t min[MB_RECIPE_COLS], max[MB_RECIPE_COLS], dimsz[MB_RECIPE_COLS];
  const uint32_t *fk[MB_RECIPE_COLS];     /* device */
  const void *attr[MB_RECIPE_COLS];       /* device; NULL = unused */
} mb_recipe;

typedef enum mb_recipe_kind {
  MB_RECIPE_PERFECT = 0, /* recipe::perfect, bmpidx_create.cu:228-239 */
  MB_RECIPE_MANY_OR = 1, /* recipe::many_or, bmpidx_create.cu:241-262 */
  MB_RECIPE_CANDCHK = 2  /* recipe::candchk, bmpidx_create.cu:264-316 */
} mb_recipe_kind;

/* A program owning its bitmaps (allocated here; free with mb_owned_vprg_release). */
typedef struct mb_owned_vprg {
  mb_vprg prg;
  const uint32_t *mid[MB_MAXCOLS][MB_MAXBINS]; /* storage of prg.cols[c].middle */
  uint32_t *owned[MB_MAXPTRS];                 /* device bitmaps to free */
  uint32_t nowned;
} mb_owned_vprg;

/* Builds the recipe's bitmaps (one mb_bitmap_create launch each, on `stream`)
 * and the program with `instrs` (MB_MAXNINSTR entries, END-terminated). */
MB_API mb_status mb_recipe_build(const mb_recipe *r, int kind, const mb_instr *instrs,
                                 mb_owned_vprg *out, void *stream);
/* Frees the bitmaps of a recipe-built program (vprg::release, primitive.cuh:186-189). */
MB_API mb_status mb_owned_vprg_release(mb_owned_vprg *p);

/* ------------------------------------------------------------------------- */
/* Synthetic data generation on the device (seeded, counter-based)           */
/* ------------------------------------------------------------------------- */
/* Flat 5-column int32 table a, b, c, d, e (any may be NULL), rows [row0, row0+n). */
MB_API mb_status mb_gen_flat(uint64_t seed, uint64_t row0, uint64_t n, int32_t *a, int32_t *b,
                      int32_t *c, int32_t *d, int32_t *e, void *stream);

/* Star schema fact columns for rows [row0, row0 + n) at scale k.  Each output
 * may be NULL.  width4 = 1: every fact column is 4 bytes (uint32); width4 = 0:
 * the reference's ssb_schema widths (ssb/ssbdemo.h:41-49): orderdate u16,
 * quantity/discount/suppcity u8, the rest u32. */
typedef struct mb_star_cols {
  void *custkey, *partkey, *suppkey, *orderdate, *quantity, *discount;
  void *extendedprice, *revenue, *supplycost, *suppcity;
} mb_star_cols;
MB_API mb_status mb_gen_star(uint64_t seed, uint32_t k, uint64_t row0, uint64_t n,
                      int width4, const mb_star_cols *out, void *stream);

/* Star schema dimension arrays, indexed by key with the zero pad at 0:
 * custcity (u8, ncust+1), suppcity (u8, nsupp+1), partmfgr (u16, npart+1). */
MB_API mb_status mb_gen_star_dims(uint64_t seed, uint32_t k, uint8_t *custcity,
                           uint8_t *suppcity, uint16_t *partmfgr, void *stream);

/* ------------------------------------------------------------------------- */
/* Engine: a resident star schema, its bitmap index, planners and queries    */
/* ------------------------------------------------------------------------- */
/* The engine keeps the fact columns, dimension arrays and the canonical
 * bitmap index resident in HBM of one device and runs queries of the four
 * star-schema templates (the SSB flights of ssb/cpuref.c:141-242, the op
 * functors s1op..s4op of ssb/lambdas.cuh:19-152).  Calls on one engine are
 * serialised by the caller; different engines are independent. */
typedef struct mb_engine mb_engine;

MB_API mb_status mb_engine_create(int device, mb_engine **out);
MB_API mb_status mb_engine_destroy(mb_engine *e);

/* Generates rows [row0, row0 + nrows) of the star schema at scale k on the
 * device (a row shard when several engines split one table); width4 = 1
 * stores every fact column in 4 bytes, 0 in the reference's ssb_schema widths. */
MB_API mb_status mb_engine_gen_star(mb_engine *e, uint64_t seed, uint32_t k, uint64_t row0,
                                    uint64_t nrows, int width4);

/* Copies a host star schema into the engine (ssb_load's host->device step,
 * ssb/cpuref.c:73-111).  Host columns in the reference's ssb_schema widths. */
typedef struct mb_star_host {
  uint64_t nrows, ncust, nsupp, npart;  /* dimension sizes include the pad key 0 */
  const uint32_t *custkey, *partkey;
  const uint16_t *orderdate;
  const uint32_t *extendedprice, *revenue, *supplycost;
  const uint8_t *quantity, *discount, *suppcity;
  const uint8_t *custcity;
  const uint16_t *partmfgr;
} mb_star_host;
MB_API mb_status mb_engine_load_star(mb_engine *e, const mb_star_host *h);

/* Builds the canonical index: date (7 years, 84 months), discount (11),
 * quantity (50), customer and supplier city (5 regions, 25 nations) and part
 * mfgr (5 mfgrs, 25 categories): 242 bitmaps, one column pass per level.
 * It also denormalises the customer city and part mfgr into one value per
 * fact row (custcity[custkey], partmfgr[partkey]: 3 bytes a row), which the
 * index build and the queries then read instead of probing the dimensions
 * through the foreign keys; a table with a foreign key outside its dimension
 * keeps the probes.  Results are the same either way. */
MB_API mb_status mb_engine_build_index(mb_engine *e);
#define MB_INDEX_PROBE_DIMS 1u  /* keep probing the dimensions (no denormalised columns) */
MB_API mb_status mb_engine_build_index_ex(mb_engine *e, uint32_t flags);

/* Index files, so an index need not be rebuilt between runs.  No
 * counterpart in the reference (whose on-disk state is the column files,
 * ssb/cpuref.c:8-27).  Layout, little-endian: "MBIX", version 1, table rows,
 * words per bitmap, bitmap count, level mask, then per kept level its bin
 * count, bin bounds (u64) and rows per bin (u64), then every bitmap of the
 * slab (stride words each), then an FNV-1a 64 hash of everything before it.
 * Saving needs a built index. */
MB_API mb_status mb_engine_save_index(mb_engine *e, const char *path);
/* Loads an index file written for this engine's table (same rows, same
 * levels; the caller vouches that the columns are the ones it was built
 * over).  flags as mb_engine_build_index_ex.  MB_ERR_IO on a file error or a
 * hash mismatch, MB_ERR_INVALID if the file does not fit the table. */
MB_API mb_status mb_engine_load_index(mb_engine *e, const char *path, uint32_t flags);

/* Column files in the reference's format (ssb/cpuref.c:8-27: a 4-byte
 * element-width header, then the n elements): one host array written to
 * path.  MB_ERR_IO on a file error. */
MB_API mb_status mb_write_column(const char *path, const void *host, uint64_t n, uint32_t width);
/* The engine's table as the reference's SSB column files in dir (the files
 * ssb_load reads: the nine fact columns in ssb_schema widths, custCity and
 * partMfgr with zero-filled custMktSegment, partName, partColor, partType,
 * partSize and partContainer of the same lengths), so the reference's own
 * drivers can run on data generated here.  The table must hold ssb_schema
 * widths or 4-byte columns whose values fit them. */
MB_API mb_status mb_engine_save_ssb(mb_engine *e, const char *dir);

typedef struct mb_engine_info {
  uint64_t nrows, fact_bytes, dim_bytes, index_bytes;
  uint32_t k, width4, nbitmaps, sms;
  float index_build_ms;
  uint32_t denorm;          /* 1 if the denormalised dimension columns are in use */
  uint64_t denorm_bytes;    /* their bytes */
} mb_engine_info;
MB_API mb_status mb_engine_get_info(mb_engine *e, mb_engine_info *out);

/* A query of one of the four templates; bounds are half-open [min, max).
 *  tmpl 1 (s1op): p = {dateMin, dateMax, discMin, discMax, qtyMin, qtyMax}
 *  tmpl 2 (s2op): p = {pMfgrMin, pMfgrMax, sCityMin, sCityMax}
 *  tmpl 3 (s3op): p = {cCityMin, cCityMax, sCityMin, sCityMax, dateMin, dateMax}
 *  tmpl 4 (s4op): p = {cCityMin, cCityMax, sCityMin, sCityMax, pMfgrMin,
 *                      pMfgrMax, dateMin, dateMax} */
typedef struct mb_query {
  uint32_t tmpl;
  uint32_t p[8];
} mb_query;

/* Group count of a query (the reference's NGRP_* formula, ssb/ssbdemo.h:79-87). */
MB_API uint32_t mb_query_ngroups(const mb_query *q);

/* The index-memory planner.  The canonical index has MB_INDEX_LEVELS
 * levels; bit i of a level mask keeps level i (column order: date year,
 * date month, discount, quantity, customer city region, customer city
 * nation, supplier city region, supplier city nation, part mfgr, part
 * category).  Every column keeps at least one level.  Generalises the
 * reference's hand-picked sparse / dense / balanced bin sets
 * (ssb/bmpidx-create.cu:120-215) into a choice under an HBM budget. */
#define MB_INDEX_LEVELS 10
#define MB_LEVELS_ALL 0x3ffu
/* Builds the index with the levels of level_mask (flags as above). */
MB_API mb_status mb_engine_build_index_levels(mb_engine *e, uint32_t flags, uint32_t level_mask);
/* Chooses the levels to keep within budget_bytes for a workload: starting
 * from every level, it drops the level whose loss raises the workload's
 * cost least per byte freed (cost = the planner's cover cost: bitmap bytes
 * read plus candidate-check bytes), until the index fits.  Needs a built
 * index (its bin row counts).  *level_mask receives the choice;
 * index_bytes / workload_bytes (may be NULL) its size and the workload's
 * estimated bytes.  MB_ERR_INVALID if no choice fits the budget. */
MB_API mb_status mb_engine_plan_index(mb_engine *e, const mb_query *qs, uint32_t n, uint64_t budget_bytes,
                                      uint32_t *level_mask, uint64_t *index_bytes, uint64_t *workload_bytes);


typedef enum mb_plan_kind {
  MB_PLAN_FUSED = 0,        /* virtual program + fused join-probe + group-by */
  MB_PLAN_SCAN = 1,         /* no index: every row through the op */
  MB_PLAN_MATERIALISED = 2, /* stage 1 -> row list -> stage 3 */
  MB_PLAN_HASH = 3          /* no index: Crystal-style hash joins (mb_hash_join_grpby) over the
                               dimensions, probed in one pass over the fact rows; waits once
                               per query for its table sizes */
} mb_plan_kind;

/* Per-query plan knobs.  The arithmetic never depends on them. */
/* How a predicate's range becomes bins (col::from_bin / from_bin2,
 * bmpidx_create.cu:138-226, generalised). */
typedef enum mb_cover {
  MB_COVER_RULE = 0,     /* the fewest bitmap bytes: an exact cover on the coarsest levels that fit,
                            the complement's, or an exact inner cover with checked edge bins */
  MB_COVER_NOEDGE = 1,   /* exact covers (direct or complement) where one exists: no candidate checks */
  MB_COVER_NOCOMPL = 2,  /* never the complement */
  MB_COVER_FINE = 3      /* the finest level's bins only, never the complement */
} mb_cover;

typedef struct mb_plan {
  uint32_t kind;            /* mb_plan_kind */
  uint32_t order_mode;      /* 0: most selective predicate first; 1: template order */
  uint32_t materialise;     /* bit i: predicate i is evaluated into a bitmap first */
  mb_launch launch;         /* group-by strategy and tile shape */
  uint32_t cover;           /* mb_cover, for every predicate */
} mb_plan;

typedef struct mb_query_stats {
  float ms;                 /* device time of the query's kernels */
  uint32_t nbitmaps;        /* bitmaps the program reads */
  uint32_t chk;             /* 1 if the program needs the candidate check */
  uint64_t algo_bytes;      /* canonical bitmap bytes + touched payload sectors */
} mb_query_stats;

/* Plans a query with the rule planner; plan may be NULL for the default. */
MB_API mb_status mb_engine_plan_rule(mb_engine *e, const mb_query *q, mb_plan *out);

/* Runs one query: results (int64[ngroups]) and the qualifying-row count
 * are copied to HOST memory before the call returns.  plan NULL = rule plan.
 * stats may be NULL. */
MB_API mb_status mb_engine_query(mb_engine *e, const mb_query *q, const mb_plan *plan,
                                 int64_t *out_host, uint64_t *nqual_host, mb_query_stats *stats);

/* Result layout of n queries: offsets[i] = sum of ngroups of queries < i;
 * returns the total group count. */
MB_API uint64_t mb_queries_layout(const mb_query *qs, uint32_t n, uint64_t *offsets);

/* Enqueues n queries on the engine stream, one launch sequence per query (the
 * plain path), without a host synchronisation.  Results go to DEVICE memory:
 * query i's group sums at out_dev + offsets[i] (mb_queries_layout), its row
 * count at nqual_dev[i].  plans: NULL = rule plan for every query.  With
 * record_times, each query's device time is kept for mb_engine_sync. */
MB_API mb_status mb_engine_enqueue(mb_engine *e, const mb_query *qs, uint32_t n,
                                   const mb_plan *plans, int64_t *out_dev, uint64_t *nqual_dev,
                                   int record_times);
/* Waits for the engine stream; times_ms (n floats of the last enqueue with
 * record_times, may be NULL) receives each query's device time. */
MB_API mb_status mb_engine_sync(mb_engine *e, float *times_ms, uint32_t n);

/* Device-time markers on the engine stream: mark records event `idx` (0..7);
 * marks_ms gives the device time between two recorded markers. */
MB_API mb_status mb_engine_mark(mb_engine *e, uint32_t idx);
MB_API mb_status mb_engine_marks_ms(mb_engine *e, uint32_t a, uint32_t b, float *ms);

/* The engine's stream (a cudaStream_t) for callers that order work after it. */
MB_API void *mb_engine_stream(mb_engine *e);

/* Batched execution: one persistent launch walks the rows once for a whole
 * batch of queries.  Per row tile it stages the union of the batch's bitmaps
 * in shared memory (each word read from HBM once per batch, not once per
 * query) and prefetches the tile's payload columns into L2; the selected rows
 * of all the batch's queries then share one row list per tile, so the ops run
 * on full warps and gather from the same lines.  No counterpart in the
 * reference, which runs one query per launch (ssb/fixedlayout.cu:34-186).
 * A launch takes up to MB_BATCH_MAX queries (and up to 256 distinct bitmaps);
 * longer batches are split.  A query the batch kernel cannot take (an op
 * source wider than 4 bytes, a clause of several terms) runs through the
 * single-query path on the same stream.  Each query's results equal what it
 * gets alone.  Results as mb_engine_enqueue (device memory, layout of
 * mb_queries_layout). */
#define MB_BATCH_MAX 128
typedef enum mb_prefetch {
  MB_PREFETCH_AUTO = 0,     /* the columns the batch's selected rows hit densely, into L2 */
  MB_PREFETCH_NONE = 1,     /* gathers straight from HBM */
  MB_PREFETCH_ALL = 2       /* every column an op reads for every selected row, into L2 */
} mb_prefetch;
typedef struct mb_batch_opts {
  uint32_t words_per_lane;  /* 1, 2, 4 or 6 (0 = the widest of 4, 2, 1 that keeps two stages in
                               flight): a tile is 1024 * words_per_lane rows */
  uint32_t warps;           /* warps per CTA, 2..16: one fills the stages, the others work (0 = 16) */
  uint32_t stages;          /* at most this many staged tiles in flight per CTA, 1..4
                               (0 = 4); fewer if they do not fit in shared memory */
  uint32_t ctas_per_sm;     /* 0 = occupancy */
  uint32_t prefetch;        /* mb_prefetch */
  uint32_t table_kb;        /* shared memory for per-CTA group tables of the queries with
                               many rows per group, at most this many KB (0 = up to 48) */
  uint32_t pad_[2];
} mb_batch_opts;
MB_API mb_status mb_engine_enqueue_batch(mb_engine *e, const mb_query *qs, uint32_t n,
                                         const mb_batch_opts *opts, int64_t *out_dev,
                                         uint64_t *nqual_dev);
/* The same with host buffers: results (layout of mb_queries_layout) are
 * copied to out_host / nqual_host (may be NULL), and the call returns when
 * they are there. */
MB_API mb_status mb_engine_query_batch(mb_engine *e, const mb_query *qs, uint32_t n,
                                       const mb_batch_opts *opts, int64_t *out_host,
                                       uint64_t *nqual_host);

/* For tests of the bounded device waits: the next `launches` batched-scan
 * launches of this engine arm their first staged tile without copying into
 * it, so the wait for that tile runs out after `tries` mbarrier tries
 * (0: the default limit, about a second).  The kernel records the wait
 * (code 1, MB_DEVERR_TMA_WAIT) and the block in the device error word, lets
 * its other copies land and exits; the call or the server then reports
 * MB_ERR_TIMEOUT (the results of that launch are not delivered) and the
 * engine carries on.  Nothing faults and nothing spins unbounded.  The
 * reference has no counterpart: it waits for its kernels without a limit
 * and exits on a launch error (ssb/lambdas.cuh:233-234). */
MB_API mb_status mb_engine_test_stall(mb_engine *e, uint32_t launches, uint32_t tries);

/* The batch with one plan per query: a fused plan (MB_PLAN_FUSED) puts its
 * query in the batched scan with the plan's cover (mb_cover) and predicate
 * order; any other kind runs the query alone on the plain path with that
 * plan.  Results as mb_engine_enqueue_batch.  No counterpart in the
 * reference (its queries run one at a time, ssb/lambdas.cuh:154-243). */
MB_API mb_status mb_engine_enqueue_batch_plans(mb_engine *e, const mb_query *qs, const mb_plan *plans,
                                               uint32_t n, const mb_batch_opts *opts, int64_t *out_dev,
                                               uint64_t *nqual_dev);

/* The launches a batch takes, planned on the host without GPU work: per
 * batched launch its queries, the bitmap rows it stages per tile, its
 * staging copies and its launch shape; *nalone = queries outside the batch
 * kernel's form (they run alone on the plain path). */
typedef struct mb_batch_launch_info {
  uint32_t queries, staged_rows, copies;
  uint32_t words_per_lane, warps, table_slots, stages;
  uint32_t chain_entries;   /* bitmap reads per 32-row word, over all queries */
  uint32_t pad_;
} mb_batch_launch_info;
MB_API mb_status mb_engine_batch_info(mb_engine *e, const mb_query *qs, uint32_t n,
                                      const mb_batch_opts *opts, mb_batch_launch_info *launches,
                                      uint32_t cap, uint32_t *nlaunches, uint32_t *nalone);

/* A batch captured once as a CUDA graph (its descriptors stay resident on
 * the device), replayed by mb_batch_graph_launch on the engine stream with
 * the same outputs: for a query mix that repeats, each replay is one graph
 * launch with no host planning or descriptor copy. */
typedef struct mb_batch_graph mb_batch_graph;
MB_API mb_status mb_batch_graph_create(mb_engine *e, const mb_query *qs, uint32_t n,
                                       const mb_batch_opts *opts, int64_t *out_dev,
                                       uint64_t *nqual_dev, mb_batch_graph **out);
/* The same with one plan per query (as mb_engine_enqueue_batch_plans). */
MB_API mb_status mb_batch_graph_create_plans(mb_engine *e, const mb_query *qs, const mb_plan *plans,
                                             uint32_t n, const mb_batch_opts *opts, int64_t *out_dev,
                                             uint64_t *nqual_dev, mb_batch_graph **out);
MB_API mb_status mb_batch_graph_launch(mb_batch_graph *g);
MB_API mb_status mb_batch_graph_destroy(mb_batch_graph *g);

/* Autotuner of the batched scan's launch shape for a query mix: times the
 * mix (median of reps launches, CUDA events on the engine stream) over tile
 * widths x warps, then drain warps, then L2 prefetch, each stage keeping the
 * best so far; *best receives the fastest options, *best_ms its time,
 * *tried the shapes timed.  The engine keeps the result: later batches
 * enqueued with opts == NULL use it (a new index forgets it). */
MB_API mb_status mb_engine_tune_batch(mb_engine *e, const mb_query *qs, uint32_t n, uint32_t reps,
                                      mb_batch_opts *best, float *best_ms, uint32_t *tried);

/* ------------------------------------------------------------------------
 * Learned planner.  No counterpart in the reference, whose programs come from
 * fixed rules (col::from_bin / from_bin2, bmpidx_create.cu:138-226).
 *
 * A 3-layer perceptron (in -> hidden -> hidden -> out, ReLU between), FP32
 * weights, trained on the GPU by the library's own forward, backward and Adam
 * kernels on timings the engine records; planning runs it in BF16.  It
 * predicts the log device time of each of MB_PLAN_CANDIDATES candidate plans
 * of a query from MB_PLAN_FEATURES features, and the engine runs the
 * candidate it predicts fastest.  Plans never change the arithmetic, so the
 * answers are the same under any plan. */
typedef struct mb_mlp mb_mlp;
typedef struct mb_mlp_config {
  uint32_t in, hidden, out;  /* layer widths */
  uint32_t seed;             /* initial weights (He-uniform from a counter hash) */
} mb_mlp_config;
typedef struct mb_mlp_train_opts {
  uint32_t epochs, batch;
  float lr, beta1, beta2;    /* Adam */
  uint32_t seed;             /* the order of the rows in each epoch */
} mb_mlp_train_opts;
MB_API mb_status mb_mlp_create(int device, const mb_mlp_config *cfg, mb_mlp **out);
MB_API mb_status mb_mlp_destroy(mb_mlp *m);
MB_API uint32_t mb_mlp_nparams(const mb_mlp *m);
/* Parameters, layer by layer: W1 [hidden x in], b1, W2 [hidden x hidden], b2,
 * W3 [out x hidden], b3 (row-major: W[j][i] weighs input i into output j). */
MB_API mb_status mb_mlp_get_params(mb_mlp *m, float *host);
MB_API mb_status mb_mlp_set_params(mb_mlp *m, const float *host);
/* y [n x out] for x [n x in] (host arrays); bf16 != 0 rounds weights and
 * activations to bfloat16 (FP32 accumulation). */
MB_API mb_status mb_mlp_forward(mb_mlp *m, const float *x_host, uint32_t n, int bf16, float *y_host);
/* Gradient of the masked mean squared error mean((y - t)^2 over mask != 0)
 * with respect to every parameter (layout of mb_mlp_get_params), and the
 * loss; for checking the backward kernels. */
MB_API mb_status mb_mlp_gradients(mb_mlp *m, const float *x, const float *t, const float *mask, uint32_t n,
                                  float *grad_host, float *loss);
/* Mini-batch Adam on (x, t, mask), all on the GPU; *final_loss = the mean
 * loss of the last epoch. */
MB_API mb_status mb_mlp_train(mb_mlp *m, const float *x, const float *t, const float *mask, uint32_t n,
                              const mb_mlp_train_opts *opts, float *final_loss);

#define MB_PLAN_FEATURES 32
#define MB_PLAN_CANDIDATES 16
/* A query's planner features (MB_PLAN_FEATURES floats): template, per
 * predicate its bins, edge bins and estimated selectivity (bin popcounts),
 * the popcount of the whole program on the first 1% of the rows (a GPU
 * pass), group-domain size, bitmap count (slot 28, once the table size, is
 * zero: planning must not depend on a size the network was not trained
 * over). */
MB_API mb_status mb_engine_query_features(mb_engine *e, const mb_query *q, float *features);
/* Candidate plan idx (0 = the rule plan) of a query: fused or materialised
 * predicates, predicate order, group-by strategy, tile width, staging, scan,
 * and four pairs of these (tile width with group-by strategy or order). */
MB_API mb_status mb_engine_plan_candidate(mb_engine *e, const mb_query *q, uint32_t idx, mb_plan *out);
/* The network the engine plans with (borrowed: it must outlive its use);
 * NULL returns to the rule planner.  It must map MB_PLAN_FEATURES inputs to
 * MB_PLAN_CANDIDATES outputs (MB_ERR_INVALID otherwise). */
MB_API mb_status mb_engine_set_planner(mb_engine *e, mb_mlp *m);
/* Plans n queries with the network (one BF16 forward pass for all of them):
 * plans[i] = the candidate with the least predicted time, chosen[i] its
 * index (may be NULL).  Without a network: the rule plan. */
MB_API mb_status mb_engine_plan_learned(mb_engine *e, const mb_query *qs, uint32_t n, mb_plan *plans,
                                        uint32_t *chosen);

/* The learned batch planner.  The reference plans every query alone with the
 * fixed rules of col::from_bin / from_bin2 (bmpidx_create.cu:138-226) and
 * runs it with a fixed launch shape (ssb/lambdas.cuh:13-15); a batch here is
 * planned as a whole: a second network of the mb_mlp kind maps
 * MB_BATCH_FEATURES features of a batch (planned with the rule, on the host)
 * to the predicted log device time of each of MB_BATCH_CANDIDATES batch plans
 * - a launch shape (words per lane in {1, 2, 4} x warps per CTA in {8, 12,
 * 16}) and the cover all its queries take (MB_COVER_RULE or
 * MB_COVER_NOEDGE): candidate c = cover * 9 + (V index * 3 + warps index).
 * Plans never change the arithmetic. */
#define MB_BATCH_FEATURES 32
#define MB_BATCH_CANDIDATES 18
MB_API mb_status mb_engine_batch_features(mb_engine *e, const mb_query *qs, uint32_t n, float *features);
/* The options and cover of batch candidate idx. */
MB_API mb_status mb_engine_batch_candidate(uint32_t idx, mb_batch_opts *opts, uint32_t *cover);
/* Sets (or clears, m = NULL) the batch planner network, borrowed: batches
 * enqueued without options then take its plan (the server's scan launches
 * among them).  The network must map MB_BATCH_FEATURES to MB_BATCH_CANDIDATES. */
MB_API mb_status mb_engine_set_batch_planner(mb_engine *e, mb_mlp *m);
/* The batch plan the planner picks (without a network: zero options, the
 * rule cover, *choice = 0xffffffff). */
MB_API mb_status mb_engine_plan_batch(mb_engine *e, const mb_query *qs, uint32_t n, mb_batch_opts *opts,
                                      uint32_t *cover, uint32_t *choice);

/* ------------------------------------------------------------------------
 * Serving loop.  No counterpart in the reference (its drivers run a fixed
 * list of queries once, ssb/ssbdemo.cu).
 *
 * A server owns a dispatcher thread over one engine whose columns and index
 * stay resident.  Requests queue on submission; whenever fewer than
 * max_inflight launches are on the GPU, the dispatcher launches every queued
 * request that fits (continuous batching: up to max_batch queries per
 * persistent batched-scan launch, or one query per launch in plain mode).
 * Admission: a request reserves its group table (8 bytes per group plus its
 * row count) and the intermediate bitmaps its plan writes; requests wait
 * while the reservations in flight would exceed mem_budget and are rejected
 * (MB_ERR_REJECTED) if theirs alone does.  Group tables live in a device
 * arena of mem_budget bytes and are copied back to the caller's buffer when
 * their launch completes.  While a server runs, its engine belongs to the
 * dispatcher thread: make no other call on that engine until
 * mb_server_destroy. */
typedef struct mb_server mb_server;
typedef enum mb_serve_mode {
  MB_SERVE_BATCHED = 0,     /* batched scan, up to max_batch queries per launch */
  MB_SERVE_PLAIN = 1        /* one query per launch sequence */
} mb_serve_mode;
typedef struct mb_server_opts {
  uint64_t mem_budget;      /* admission bytes and arena size (0 = 256 MiB) */
  uint32_t mode;            /* mb_serve_mode */
  uint32_t max_batch;       /* 1..MB_BATCH_MAX (0 = 64) */
  uint32_t max_inflight;    /* launches on the GPU at once, 1..8 (0 = 2) */
  uint32_t use_planner;     /* plain-path launches plan with the engine's learned planner
                               (mb_engine_set_planner) */
  uint32_t min_batch;       /* batched mode: fewer queued queries than this run on the plain
                               path, one query per launch (1 = always the batched scan); 0 = an
                               online cost model decides per launch: while the plain path keeps
                               up with the arrival rate, the scan only when it lowers the queued
                               queries' summed completion time; past that, the cheaper per query */
  uint32_t pad_;
  mb_batch_opts batch;      /* batched-scan launch shape */
} mb_server_opts;
typedef struct mb_request_info {
  int32_t status;           /* MB_OK, MB_ERR_REJECTED, MB_ERR_CANCELLED or the launch's error */
  uint32_t launch;          /* index of the launch that ran it */
  uint32_t batch_size;      /* queries in that launch */
  uint32_t plan;            /* candidate plan index (plain mode with the planner; else 0) */
  uint64_t nqual;           /* qualifying rows */
  double t_submit_us;       /* times since the server started */
  double t_launch_us;       /* the dispatcher enqueued its launch */
  double t_done_us;         /* its results were in the caller's buffer */
  float gpu_ms;             /* device time of its launch */
  float pad_;
} mb_request_info;
typedef struct mb_server_stats {
  uint64_t submitted, completed, rejected, cancelled, failed;
  uint64_t launches, launched_queries;
  uint64_t peak_reserved;   /* largest admission reservation in flight (bytes) */
  double gpu_ms;            /* sum of launch device times */
  uint64_t scan_launches;   /* launches that took the batched scan */
} mb_server_stats;
MB_API mb_status mb_server_create(mb_engine *e, const mb_server_opts *opts, mb_server **out);
/* Stops accepting requests, finishes the launches in flight (queued requests
 * complete as MB_ERR_CANCELLED) and joins the dispatcher. */
MB_API mb_status mb_server_destroy(mb_server *s);
/* Queues a query; out_host (mb_query_ngroups(q) int64 values) receives its
 * group sums.  *id identifies it for wait and cancel. */
MB_API mb_status mb_server_submit(mb_server *s, const mb_query *q, int64_t *out_host, uint64_t *id);
/* Cancels a request that has not launched yet (MB_ERR_INVALID if it has
 * launched or finished: its results arrive as usual). */
MB_API mb_status mb_server_cancel(mb_server *s, uint64_t id);
/* Waits up to timeout_ms (< 0: without limit) for a request, fills *info
 * and forgets the request.  MB_ERR_TIMEOUT if it is not done in time. */
MB_API mb_status mb_server_wait(mb_server *s, uint64_t id, int64_t timeout_ms, mb_request_info *info);
MB_API mb_status mb_server_get_stats(mb_server *s, mb_server_stats *out);
/* Open-loop load: submits qs[i] at Poisson arrival times of rate_qps (the
 * arrivals of mb_poisson_arrivals(seed, ...)), waits for every request and
 * fills out_host (layout of mb_queries_layout) and info[i]. */
MB_API mb_status mb_server_run_load(mb_server *s, const mb_query *qs, uint32_t n, double rate_qps, uint64_t seed,
                                    int64_t *out_host, mb_request_info *info);
/* Arrival times (microseconds from 0) of n Poisson arrivals at rate_qps:
 * exponential gaps by inversion of a counter-based uniform (SplitMix64 of
 * seed and i).  Host only. */
MB_API mb_status mb_poisson_arrivals(uint64_t seed, double rate_qps, uint32_t n, double *t_us);

/* Host-side fault injection for the serving loop (no GPU fault is made):
 * the next `count` launches fail their arena allocation (MB_ERR_OOM), fail
 * their enqueue as a CUDA error would (MB_ERR_CUDA), or are held on the host
 * for arg_us microseconds before they launch (a slow query). */
typedef enum mb_fault {
  MB_FAULT_NONE = 0,
  MB_FAULT_ALLOC = 1,
  MB_FAULT_LAUNCH = 2,
  MB_FAULT_SLOW = 3
} mb_fault;
MB_API mb_status mb_server_inject(mb_server *s, uint32_t fault, uint32_t count, uint32_t arg_us);

/* ------------------------------------------------------------------------
 * WAH compressed bitmaps: interop with the reference's compressed-bitmap
 * baseline (merle/wahGpu.cuh:5-44, merle/host/wahCpu.h, ssb/wah-demo.cu).
 *
 * A WAH stream cuts the rows into 31-bit groups: a literal word (bit 31 clear)
 * holds one group in bits 0..30; a fill word (bit 31 set) stands for a run of
 * all-0 (bit 30 clear) or all-1 (bit 30 set) groups, the run length in bits
 * 0..29 (merle/host/wahCpu.c:20-24).  Row 31g + j of group g is bit j
 * (MB_WAH_LSB, as the reference's loadArrayFile sets them,
 * merle/host/wahConv.c:85-87) or bit 30 - j (MB_WAH_MSB, as its simpleJoin and
 * dbjoinFlatWah build them, wahConv.c:142-144, wahGpuCmprs.cu:215-226).
 * Streams written here are canonical (maximal runs: wahCmprsCPU's output,
 * wahConv.c:36-57).  All pointers are device pointers except in
 * mb_wah_save / mb_wah_load; scratch is stream-ordered (cudaMallocAsync).
 *
 * A decoded stream is an ordinary bitmap of this library (stride
 * mb_bitmap_stride words, padding zeroed), so it can be a bin of any mb_col
 * operand of a virtual bitmap program: this is the compressed-operand hook
 * the reference declares but never defines (vprg::_cmprs_adapt_run,
 * primitive.cuh:334-337). */
typedef enum mb_wah_order { MB_WAH_LSB = 0, MB_WAH_MSB = 1 } mb_wah_order;
typedef enum mb_wah_opcode { MB_WAH_AND = 0, MB_WAH_OR = 1, MB_WAH_XOR = 2 } mb_wah_opcode;

/* Groups of n rows: ceil(n / 31) (the reference's decmprsNrWord). */
MB_API uint64_t mb_wah_groups(uint64_t nrows);
/* Compresses a bitmap of nrows rows (rows < 31 * (2^30 - 1)) into `wah`
 * (capacity words; mb_wah_groups(nrows) always suffice).  *nwords = the
 * stream's words.  wah NULL: a size query.  MB_ERR_INVALID if the stream does
 * not fit (nothing written, *nwords still set).  Waits for the stream once
 * (to learn the size); wahCompress / wahCmprsCPU (wahGpuCmprs.cu:172-198). */
MB_API mb_status mb_wah_encode(const uint32_t *bitmap, uint64_t nrows, uint32_t order, uint32_t *wah,
                               uint64_t capacity, uint64_t *nwords, void *stream);
/* Expands a stream into a bitmap of nrows rows (mb_bitmap_stride(nrows) words
 * written): groups past the stream and rows >= nrows are 0.  No host wait.
 * wahCntExcScan + wahDecomp (wahGpuCmprs.cu:6-14, 34-47). */
MB_API mb_status mb_wah_decode(const uint32_t *wah, uint64_t nwords, uint32_t order, uint64_t nrows,
                               uint32_t *bitmap, void *stream);
/* *ngroups = the groups a stream stands for (the sum of its run counts). */
MB_API mb_status mb_wah_ngroups(const uint32_t *wah, uint64_t nwords, uint64_t *ngroups, void *stream);
/* op (mb_wah_opcode) of two streams over ngroups groups (shorter streams are
 * extended with 0 groups) into a canonical stream; capacity and *nwords as in
 * mb_wah_encode.  The reference's wahAnd / wahOr / wahXor and their explicit
 * forms (wahGpu.cuh:11-30; wahAndCPU, wahCpu.c:27-79). */
MB_API mb_status mb_wah_op(uint32_t op, const uint32_t *a, uint64_t na, const uint32_t *b, uint64_t nb,
                           uint64_t ngroups, uint32_t *out, uint64_t capacity, uint64_t *nwords, void *stream);
/* The same with the method chosen: MB_WAH_EXPLICIT expands both streams,
 * combines the bitmaps and compresses the result (the reference's explicit
 * forms, wahAndExpl ...); MB_WAH_DIRECT cuts the runs of both streams at the
 * union of their word boundaries and combines each piece whole, never
 * expanding (wahAnd / wahOr / wahXor, merle/wahGpuDirect.cu); MB_WAH_AUTO
 * (mb_wah_op) takes the direct form when na + nb < ngroups / 8.  Both give
 * the same canonical stream. */
typedef enum mb_wah_method { MB_WAH_AUTO = 0, MB_WAH_EXPLICIT = 1, MB_WAH_DIRECT = 2 } mb_wah_method;
MB_API mb_status mb_wah_op_ex(uint32_t op, const uint32_t *a, uint64_t na, const uint32_t *b, uint64_t nb,
                              uint64_t ngroups, uint32_t method, uint32_t *out, uint64_t capacity,
                              uint64_t *nwords, void *stream);
/* The reference's WAH file (struct wahHost_s, wahCpu.h:10-15; read by
 * loadWahFile, wahConv.c:93-109): 24-byte header (has1Fill, magic 0x44f8a1ef,
 * cmprsNrWord, decmprsNrWord) then the words.  HOST buffers.  Load with
 * words NULL returns the sizes only; MB_ERR_IO on a bad magic or size. */
MB_API mb_status mb_wah_save(const char *path, const uint32_t *words, uint64_t nwords, uint64_t ngroups);
MB_API mb_status mb_wah_load(const char *path, uint32_t *words, uint64_t capacity, uint64_t *nwords,
                             uint64_t *ngroups);

#ifdef __cplusplus
} /* extern "C" */
#endif
#endif /* MERLE_B200_H */
