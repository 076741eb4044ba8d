/*
 * oracle.h - CPU restatement of the reference's fused bitmap-index query path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load this code, and only as the
 * checker.  The product library (merle_b200/libmerleb200.so) never links it.
 *
 * Parity is pinned two ways (tests/test_oracle.py):
 *  - against the reference's own CPU oracle ssb/cpuref.c (s1ref..s4ref,
 *    ssb_cpujoin) and synth/cpuref.c (synth_ref), compiled unmodified from the
 *    reference sources into oracle/_ref/ by oracle/Makefile;
 *  - against golden vectors produced by those reference functions and
 *    committed under tests/golden/ (tests/golden/make_golden.py).
 *
 * All descriptors are the public C ABI structs of include/merle_b200.h with
 * HOST pointers in place of device pointers.
 */
#ifndef MERLE_B200_ORACLE_H
#define MERLE_B200_ORACLE_H
#include "../include/merle_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* 1 if no operand has an edge bin (vprg::is_nochk, primitive.cuh:190-195). */
int orc_is_nochk(const mb_vprg *p);

/* Bin bitmaps of one column (bmpidx_create.cu:14-56; primitive.cuh:102-118). */
void orc_bitmap_create(const mb_src *src, uint64_t n, const uint64_t *lo,
                       const uint64_t *hi, uint32_t nbins, uint32_t *out,
                       uint64_t stride_words, uint64_t *popcounts);

/* Virtual bitmap program, nochk (primitive.cuh:201-252) or chk (:255-332);
 * bits of rows >= factsz are cleared in both outputs.  uncertain may be NULL. */
void orc_vprg_eval(const mb_vprg *p, int chk, uint32_t *possible, uint32_t *uncertain);

/* The op on one row (ssb/lambdas.cuh:19-152, synth/synthdemo.cu:7-53).
 * Returns 1 if the row is kept, with its value and group index. */
int orc_op_row(const mb_op *op, uint64_t row, int chk, uint32_t nr_grp,
               int64_t *value, uint32_t *group);

/* Fused plan (primitive.cuh:340-445): program, then the op over every possible
 * row, with chk = the row's uncertain bit. */
void orc_vprg_grpby(const mb_vprg *p, const mb_op *op, uint32_t nr_grp,
                    int64_t *out, uint64_t *nqual);

/* No-index plan (primitive.cuh:16-48): the op with chk on every row. */
void orc_join_grpby(uint64_t n, const mb_op *op, uint32_t nr_grp, int64_t *out,
                    uint64_t *nqual);

/* Bitmap to ascending row list, uncertain rows tagged with bit 31
 * (primitive_abla.cuh:290-354).  Returns the row count. */
uint64_t orc_bitmap_to_rows(const uint32_t *possible, const uint32_t *uncertain,
                            uint64_t n, uint32_t *rows);

/* Number of distinct 32-byte sectors of a column of `width`-byte elements that
 * hold at least one row set in `rowbits` (algorithmic gather bytes / 32). */
uint64_t orc_sector_count(const uint32_t *rowbits, uint64_t n, uint32_t width);

/* Generators (host restatement; values equal the device generator's). */
void orc_gen_flat(uint64_t seed, uint64_t row0, uint64_t n, int32_t *a, int32_t *b,
                  int32_t *c, int32_t *d, int32_t *e);
void orc_gen_star(uint64_t seed, uint32_t k, uint64_t row0, uint64_t n, int width4,
                  const mb_star_cols *out);
void orc_gen_star_dims(uint64_t seed, uint32_t k, uint8_t *custcity,
                       uint8_t *suppcity, uint16_t *partmfgr);

/* Direct restatements of the reference CPU loops with int64 sums
 * (ssb/cpuref.c:141-242) over ssb_schema-width columns. */
typedef struct orc_ssb {
  const uint32_t *loCustKey, *loPartKey;
  const uint16_t *loOrderDate;
  const uint32_t *loExtendedPrice, *loRevenue, *loSupplyCost;
  const uint8_t *loQuantity, *loDiscount, *loSuppCity;
  const uint8_t *custCity;
  const uint16_t *partMfgr;
} orc_ssb;

uint32_t orc_date_to_year(uint32_t date);
int64_t orc_s1(const orc_ssb *d, uint64_t n, uint32_t dateMin, uint32_t dateMax,
               uint32_t discntMin, uint32_t discntMax, uint32_t qtyMin, uint32_t qtyMax,
               uint64_t *nqual);
void orc_s2(const orc_ssb *d, uint64_t n, uint32_t pMfgrMin, uint32_t pMfgrMax,
            uint32_t sCityMin, uint32_t sCityMax, int64_t *out, uint32_t nr_grp,
            uint64_t *nqual);
void orc_s3(const orc_ssb *d, uint64_t n, uint32_t cCityMin, uint32_t cCityMax,
            uint32_t sCityMin, uint32_t sCityMax, uint32_t dateMin, uint32_t dateMax,
            int64_t *out, uint32_t nr_grp, uint64_t *nqual);
void orc_s4(const orc_ssb *d, uint64_t n, uint32_t cCityMin, uint32_t cCityMax,
            uint32_t sCityMin, uint32_t sCityMax, uint32_t pMfgrMin, uint32_t pMfgrMax,
            uint32_t dateMin, uint32_t dateMax, int64_t *out, uint32_t nr_grp,
            uint64_t *nqual);

/* Synthetic OR query (synth/cpuref.c:125-169) with 256 COUNT groups. */
void orc_synth(const void *a1, const void *a2, uint32_t bitwidth, const uint32_t *fk,
               const uint32_t *dimattr1, const uint8_t *dimattr2, uint64_t n,
               uint64_t fa1lo, uint64_t fa1hi, uint64_t fa2lo, uint64_t fa2hi,
               uint64_t da1lo, uint64_t da1hi, int64_t out[256], uint64_t *nqual);

/* Flat-table query: a in [alo,ahi) AND b in bset AND c in [clo,chi):
 * count and SUM(int64 e*d). */
int64_t orc_flat_query(const int32_t *a, const int32_t *b, const int32_t *c,
                       const int32_t *d, const int32_t *e, uint64_t n, int32_t alo,
                       int32_t ahi, const int32_t *bset, uint32_t nb, int32_t clo,
                       int32_t chi, uint64_t *count);

/* WAH (word-aligned hybrid) streams of the reference's compressed-bitmap
 * baseline (merle/host/wahCpu.h, merle/wahGpu.cuh).  order 0: row 31g + j of
 * group g at bit j; order 1: at bit 30 - j. */
uint64_t orc_wah_encode(const uint32_t *bitmap, uint64_t nrows, uint32_t order, uint32_t *out);
void orc_wah_decode(const uint32_t *wah, uint64_t nwords, uint32_t order, uint64_t nrows, uint32_t *bitmap,
                    uint64_t stride);
/* op 0 AND, 1 OR, 2 XOR over ngroups groups; returns the words written. */
uint64_t orc_wah_op(uint32_t op, const uint32_t *a, uint64_t na, const uint32_t *b, uint64_t nb,
                    uint64_t ngroups, uint32_t *out);

#ifdef __cplusplus
}
#endif
#endif
