/* merle_b200_legacy.h - the reference's own C entry points, exported by
 * libmerleb200.so with the same names, types and signatures, so a driver
 * written against them (the reference's main.c) links against this library
 * unchanged.
 *
 *   ssb/ssbdemo.h:10-97        -> ssb_* (star-schema benchmark)
 *   synth/synthdemo.h:15-64    -> synth_* and window_zipf
 *
 * Every computation runs on the GPU through the mb_* kernels of
 * merle_b200.h.  Differences from the reference, all on error paths or
 * out of scope:
 *   - a file or allocation failure returns 0 / NULL and prints one line to
 *     stderr instead of exit() or assert();
 *   - ssb_cpujoin and synth_ref compute their results on the GPU (the
 *     library has no CPU path; the reference's CPU code is the test oracle);
 *   - ssb_wah and synth_wah run the reference's WAH pipelines on this
 *     library's WAH kernels (mb_wah_*) and print "unavailable" in the RTScan
 *     column (an OptiX ray-tracing competitor, not available on this system);
 *   - results are the reference's uint32 values: the int64 sums of the
 *     mb_* kernels truncated to 32 bits (the reference's atomics wrap).
 * Struct layouts, enum values and the bin tables are the reference's,
 * because callers fill and read them. */
#ifndef MERLE_B200_LEGACY_H
#define MERLE_B200_LEGACY_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#include <vector_types.h> /* float2, float4 */

#include "merle_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- ssb/ssbdemo.h ---------------------------------------------------- */
enum {
  SSBDATE_920101 = 0,
  SSBDATE_930101 = 366,
  SSBDATE_940101 = 731,
  SSBDATE_940201 = 762,
  SSBDATE_940204 = 765,
  SSBDATE_940211 = 772,
  SSBDATE_940301 = 790,
  SSBDATE_940501 = 851,
  SSBDATE_940901 = 974,
  SSBDATE_950101 = 1096,
  SSBDATE_960101 = 1461,
  SSBDATE_970101 = 1827,
  SSBDATE_971201 = 2161,
  SSBDATE_980101 = 2192,
  SSBDATE_990101 = 2557,
};

/* Column set of the star schema (ssb/ssbdemo.h:41-49), host or device. */
struct ssb_schema {
  uint32_t *loCustKey, *loPartKey;
  uint16_t *loOrderDate;
  uint32_t *loExtendedPrice, *loRevenue, *loSupplyCost;
  uint8_t *loQuantity, *loDiscount, *loSuppCity;
  uint8_t *custMktSegment, *custCity;
  uint16_t *partName, *partMfgr;
  uint8_t *partColor, *partType, *partSize, *partContainer;
};

/* Reads <dir>/<column> files (4-byte element-width header, then the raw
 * array; ssb/cpuref.c:8-27) into host memory and, if dev != NULL, device
 * memory; returns the fact rows (ssb/cpuref.c:36-112), 0 on failure. */
MB_API size_t ssb_load(struct ssb_schema *host, struct ssb_schema *dev, const char *ssbDirname);
MB_API void ssb_free(struct ssb_schema *host, struct ssb_schema *dev);

/* The fixed bitmap index (ssb/ssbdemo.h:52-65): per column a coarse
 * ("Sparse") and a fine ("Dense") set of bins; the bitmaps of one set are one
 * device slab, [0] owning it. */
struct ssb_bmp {
  uint32_t *dateSparse[7], *dateDense[4];
  uint32_t *discntSparse[4], *discntDense[11];
  uint32_t *qtySparse[5], *qtyDense[10];
  uint32_t *mfgrSparse[5], *mfgrDense[5];
  uint32_t *sCitySparse[5], *sCityDense[3];
  uint32_t *cCitySparse[5], *cCityDense[3];
};
/* Builds every bin set with one column pass each (ssb/bmpidx-create.cu:120-215). */
MB_API void ssb_bmpcreate(const struct ssb_schema *host, const struct ssb_schema *dat, size_t factSz,
                          struct ssb_bmp *devOut);
MB_API void ssb_bmpfree(struct ssb_bmp *devOut);

/* Bin boundaries of the fixed index (ssb/bmpidx-create.cu:8-30). */
extern MB_API const uint64_t dateSpBin[8], dateDeBin[5], discntSpBin[5], discntDeBin[12], qtySpBin[6],
    qtyDeBin[11], mfgrSpBin[6], mfgrDeBin[6], sCitySpBin[6], sCityDeBin[4];

/* Group counts of the 13 SSB queries and their offsets in a result array
 * (ssb/ssbdemo.h:72-84). */
enum {
  NGRP_S11 = 1, NGRP_S12 = 1, NGRP_S13 = 1,
  NGRP_S21 = 280, NGRP_S22 = 56, NGRP_S23 = 7,
  NGRP_S31 = 150, NGRP_S32 = 600, NGRP_S33 = 96, NGRP_S34 = 16,
  NGRP_S41 = 350, NGRP_S42 = 100, NGRP_S43 = 800,
  SUMGRP_S1 = 3, SUMGRP_S2 = 3 + 280 + 56 + 7,
  SUMGRP_S3 = SUMGRP_S2 + 150 + 600 + 96 + 16,
  SUMGRP_ALL = SUMGRP_S3 + 350 + 100 + 800
};

/* The 13 queries over a HOST schema; a malloc'd array of SUMGRP_ALL + 1
 * uint32 results (ssb/cpuref.c:244-299).  Computed on the GPU here. */
MB_API uint32_t *ssb_cpujoin(const struct ssb_schema *dat, size_t factSz);
/* The 13 queries over the fixed index; a device array of 5 x SUMGRP_ALL
 * uint32: [0] the no-index join, [1] the fused kernel over the fine bins,
 * [2] the fused kernel with direct loads and global atomics, [3] the
 * materialised three-stage plan, [4] the fused kernel with TMA-staged
 * operands over the coarse bins (ssb/fixedlayout.cu:145-186). */
MB_API uint32_t *ssb_bmp_fixed(const struct ssb_schema *dat, struct ssb_bmp *bmp, size_t factSz);
/* The 13 queries over per-query recipe bitmaps; a device array of
 * 4 x SUMGRP_ALL uint32: [0] the join, [1] perfect, [2] many_or (aligned
 * bins), [3] candchk (misaligned bins) (ssb/controlled-demo.cu:98-129). */
MB_API uint32_t *ssb_bmp_control(const struct ssb_schema *dat, size_t factSz);
/* SUMGRP_ALL results of the fused (perfect recipes) and of the materialised
 * plan (ssb/ssbdemo.h:92-93). */
MB_API uint32_t *ssb_bmp_control_abl_fuse(const struct ssb_schema *dat, size_t factSz);
MB_API uint32_t *ssb_bmp_control_abl_nofuse(const struct ssb_schema *dat, size_t factSz);
MB_API void ssb_wah(const struct ssb_schema *host, const struct ssb_schema *dat, size_t factSz);
/* Load, index, run every path and compare with ssb_cpujoin
 * (ssb/cpuref.c:318-349); true if every result matches. */
MB_API bool ssb_demoall(const char *ssbDirname);

/* ---- synth/synthdemo.h ------------------------------------------------ */
/* SELECT count(*) FROM fact, dim WHERE fact.fk = dim.key AND
 * (fact.attr1 in [fa1lo, fa1hi) OR fact.attr2 in [fa2lo, fa2hi)) AND
 * dim.attr1 in [da1lo, da1hi) GROUP BY dim.attr2 (synth/synthdemo.h:9-24). */
struct synth_schema {
  uint32_t bitwidth; /* 8, 16, 32, 64 */
  void *factattr1, *factattr2;
  uint32_t *fkey;
  uint32_t *dimattr1;
  uint8_t *dimattr2;
};
/* Reads <dir>/{fk,a1,a2} and generates the dimension (synth/cpuref.c:44-101). */
MB_API size_t synth_load(struct synth_schema *host, struct synth_schema *dev, const char *synthDirname);
MB_API void synth_free(struct synth_schema *host, struct synth_schema *dev);
/* grpout: HOST, 256 counts (synth/cpuref.c:123-163).  Computed on the GPU here. */
MB_API void synth_ref(const struct synth_schema *host, size_t factsz, uint64_t fa1low, uint64_t fa1hi,
                      uint64_t fa2low, uint64_t fa2hi, uint64_t da1low, uint64_t da1hi, uint32_t grpout[256]);
/* grpout: DEVICE, 256 counts: the no-index join (synth/synthdemo.cu:67-78). */
MB_API void synth_join(const struct synth_schema *dev, size_t factsz, uint64_t fa1low, uint64_t fa1hi,
                       uint64_t fa2low, uint64_t fa2hi, uint64_t da1low, uint64_t da1hi, uint32_t grpout[256]);
/* ty < 0: the join; ty % 3 = 0, 1, 2: perfect / many_or / candchk recipe
 * bitmaps, fused (ty < 3) or materialised (ty >= 3).  Returns milliseconds:
 * x = the whole plan, or x, y, z = stages 1, 2, 3 (synth/synthdemo.cu:80-150).
 * grpout: DEVICE, 256 counts. */
MB_API float4 synth_bmp(const struct synth_schema *dat, uint32_t factsz, uint32_t fa1lo, uint32_t fa1hi,
                        uint32_t fa2lo, uint32_t fa2hi, uint32_t da1lo, uint32_t da1hi, uint32_t grpout[256],
                        int ty);
/* Milliseconds of the fused kernel at one and at four bitmap words per lane
 * on the perfect recipe; the two results must agree (synth/synthdemo.cu:152-204). */
MB_API float2 synth_method(const struct synth_schema *dat, uint32_t factsz, uint32_t fa1lo, uint32_t fa1hi,
                           uint32_t fa2lo, uint32_t fa2hi, uint32_t da1lo, uint32_t da1hi);
MB_API void synth_wah(const struct synth_schema *dat, uint32_t factsz, uint32_t fa1lo, uint32_t fa1hi,
                      uint32_t fa2lo, uint32_t fa2hi, uint32_t da1lo, uint32_t da1hi);
MB_API bool synth_demoall(const char *synthDirname);
/* P(value in [x, x + winsize)) for x < n under Zipf(skewness), values from 1
 * (synth/window_zipf.c:1-67); malloc'd. */
MB_API double *window_zipf(double skewness, size_t n, size_t winsize);

#ifdef __cplusplus
} /* extern "C" */
#endif
#endif /* MERLE_B200_LEGACY_H */
