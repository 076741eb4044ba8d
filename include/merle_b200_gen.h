/*
 * merle_b200_gen.h - seeded, counter-based synthetic data generator.
 *
 * Shared by the CUDA library (device + host) and by the CPU oracle so that both
 * see the same fact and dimension values for any (seed, column, row).  Every value
 * is a pure function of (seed, column id, row index): any row range can be
 * regenerated independently, on the CPU or on the GPU, in any order.
 *
 * Random stream: SplitMix64 (Steele, Lea, Flood, "Fast splittable pseudorandom
 * number generators", OOPSLA 2014): out_i = fmix(key + (i + 1) * golden) with the
 * stream key itself mixed from (seed, column id).
 *
 * Distributions (the synthetic star schema and the flat 5-column table):
 *  - uniform integers on an inclusive range use the high 32 random bits scaled by
 *    a 64-bit multiply (Lemire's multiply-shift without rejection);
 *  - Zipf(s = 1) over 64 values (P(v) proportional to 1/(v+1)) uses inverse-CDF
 *    thresholds floor(2^32 * H(k+1) / H(64)), computed exactly with rationals.
 *
 * The reference generators (ssb-dbgen-lite.c:16-190 with rand_r and an unpinned
 * time(NULL) seed, synth/onegen_zipf.py with unseeded numpy) are not reproducible;
 * this generator keeps their value encodings (city 0..249 with nation = city/10 and
 * region = city/50; mfgr code 0..999 with category = code/40, ssb-dbgen-lite.c:16-56)
 * and replaces their randomness.
 */
#ifndef MERLE_B200_GEN_H
#define MERLE_B200_GEN_H
#include <stdint.h>

#if defined(__CUDACC__)
#define MBG_FN static inline __host__ __device__
#else
#define MBG_FN static inline
#endif

#define MBG_GOLDEN 0x9E3779B97F4A7C15ULL

/* Column ids of the flat 5-column table (a, b, c, d, e). */
enum { MBG_COL_A = 1, MBG_COL_B = 2, MBG_COL_C = 3, MBG_COL_D = 4, MBG_COL_E = 5 };

/* Column ids of the star schema. */
enum {
  MBG_LO_DATE = 10, MBG_LO_CUSTKEY = 11, MBG_LO_SUPPKEY = 12, MBG_LO_PARTKEY = 13,
  MBG_LO_QUANTITY = 14, MBG_LO_DISCOUNT = 15, MBG_LO_SUPPLYCOST = 16,
  MBG_CUST_CITY = 20, MBG_SUPP_CITY = 21, MBG_PART_MFGR = 22, MBG_PART_PRICE = 23,
  MBG_CUST_MKTSEG = 24, MBG_PART_NAME = 25, MBG_PART_COLOR = 26, MBG_PART_TYPE = 27,
  MBG_PART_SIZE = 28, MBG_PART_CONTAINER = 29
};

/* Number of days in the date domain: seven years starting 1992-01-01. */
#define MBG_NDAYS 2556u

MBG_FN uint64_t mbg_fmix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

/* Key of the random stream of one column under one seed. */
MBG_FN uint64_t mbg_key(uint64_t seed, uint32_t col) {
  return mbg_fmix64(seed * MBG_GOLDEN + (uint64_t)col * 0xD1B54A32D192ED03ULL + 1u);
}

/* The i-th 64-bit random word of a stream. */
MBG_FN uint64_t mbg_rand(uint64_t key, uint64_t i) {
  return mbg_fmix64(key + (i + 1u) * MBG_GOLDEN);
}

/* Uniform integer on the inclusive range [lo, hi] (hi - lo < 2^32). */
MBG_FN uint32_t mbg_uniform(uint64_t r, uint32_t lo, uint32_t hi) {
  uint64_t span = (uint64_t)hi - (uint64_t)lo + 1u;
  return lo + (uint32_t)(((r >> 32) * span) >> 32);
}

/* Zipf(1) over {0..63}: thresholds floor(2^32 * H(k+1) / H(64)), k = 0..63, exact;
 * the value is the smallest v with u < threshold[v], u = high 32 random bits. */
#define MBG_ZIPF64_TABLE { \
  905368058ULL, 1358052087ULL, 1659841440ULL, 1886183454ULL, \
  2067257066ULL, 2218151742ULL, 2347490036ULL, 2460661044ULL, \
  2561257494ULL, 2651794300ULL, 2734100487ULL, 2809547826ULL, \
  2879191522ULL, 2943860669ULL, 3004218540ULL, 3060804044ULL, \
  3114060988ULL, 3164359214ULL, 3212010164ULL, 3257278567ULL, \
  3300391332ULL, 3341544425ULL, 3380908254ULL, 3418631923ULL, \
  3454846645ULL, 3489668494ULL, 3523200644ULL, 3555535217ULL, \
  3586754806ULL, 3616933741ULL, 3646139162ULL, 3674431914ULL, \
  3701867310ULL, 3728495782ULL, 3754363441ULL, 3779512554ULL, \
  3803981960ULL, 3827807436ULL, 3851022001ULL, 3873656203ULL, \
  3895738351ULL, 3917294733ULL, 3938349804ULL, 3958926351ULL, \
  3979045641ULL, 3998727555ULL, 4017990705ULL, 4036852540ULL, \
  4055329439ULL, 4073436800ULL, 4091189115ULL, 4108600039ULL, \
  4125682456ULL, 4142448531ULL, 4158909768ULL, 4175077055ULL, \
  4190960705ULL, 4206570499ULL, 4221915720ULL, 4237005188ULL, \
  4251847287ULL, 4266449998ULL, 4280820920ULL, 4294967296ULL, \
}
static const uint64_t mbg_zipf64_host[64] = MBG_ZIPF64_TABLE;
#if defined(__CUDACC__)
static __constant__ uint64_t mbg_zipf64_dev[64] = MBG_ZIPF64_TABLE;
#endif

MBG_FN uint32_t mbg_zipf64(uint64_t r) {
#if defined(__CUDA_ARCH__)
  const uint64_t *t = mbg_zipf64_dev;
#else
  const uint64_t *t = mbg_zipf64_host;
#endif
  uint64_t u = r >> 32;
  uint32_t lo = 0, hi = 63; /* answer in [lo, hi] */
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (u < t[mid]) hi = mid; else lo = mid + 1;
  }
  return lo;
}

/* ---- flat 5-column table (a, b, c, d, e), all int32 ---- */
MBG_FN int32_t mbg_flat_a(uint64_t seed, uint64_t i) { return (int32_t)mbg_uniform(mbg_rand(mbg_key(seed, MBG_COL_A), i), 0, 999); }
MBG_FN int32_t mbg_flat_b(uint64_t seed, uint64_t i) { return (int32_t)mbg_zipf64(mbg_rand(mbg_key(seed, MBG_COL_B), i)); }
MBG_FN int32_t mbg_flat_c(uint64_t seed, uint64_t i) { return (int32_t)mbg_uniform(mbg_rand(mbg_key(seed, MBG_COL_C), i), 1, 50); }
MBG_FN int32_t mbg_flat_d(uint64_t seed, uint64_t i) { return (int32_t)mbg_uniform(mbg_rand(mbg_key(seed, MBG_COL_D), i), 0, 10); }
MBG_FN int32_t mbg_flat_e(uint64_t seed, uint64_t i) { return (int32_t)mbg_uniform(mbg_rand(mbg_key(seed, MBG_COL_E), i), 90000, 10499999); }

/* ---- star schema sizes for scale k (6M fact rows per unit of k) ---- */
MBG_FN uint64_t mbg_star_ncust(uint32_t k) { return 30000ull * k; }
MBG_FN uint64_t mbg_star_nsupp(uint32_t k) { return 2000ull * k; }
MBG_FN uint64_t mbg_star_npart(uint32_t k) {
  uint32_t lg = 0;
  while ((2u << lg) <= k) ++lg; /* floor(log2 k) */
  return 200000ull * (1u + lg);
}

/* Dimension attributes; key 0 is the zero pad (keys are 1-based). */
MBG_FN uint32_t mbg_cust_city(uint64_t seed, uint64_t key) { return key ? mbg_uniform(mbg_rand(mbg_key(seed, MBG_CUST_CITY), key), 0, 249) : 0u; }
MBG_FN uint32_t mbg_supp_city(uint64_t seed, uint64_t key) { return key ? mbg_uniform(mbg_rand(mbg_key(seed, MBG_SUPP_CITY), key), 0, 249) : 0u; }
MBG_FN uint32_t mbg_part_mfgr(uint64_t seed, uint64_t key) { return key ? mbg_uniform(mbg_rand(mbg_key(seed, MBG_PART_MFGR), key), 0, 999) : 0u; }
MBG_FN uint32_t mbg_part_price(uint64_t seed, uint64_t key) { return key ? mbg_uniform(mbg_rand(mbg_key(seed, MBG_PART_PRICE), key), 90000, 110000) : 0u; }
/* Attributes that only the reference column-file layout carries. */
MBG_FN uint32_t mbg_cust_mktseg(uint64_t seed, uint64_t key) { return key ? mbg_uniform(mbg_rand(mbg_key(seed, MBG_CUST_MKTSEG), key), 0, 4) : 0u; }
MBG_FN uint32_t mbg_part_name(uint64_t seed, uint64_t key) { return key ? mbg_uniform(mbg_rand(mbg_key(seed, MBG_PART_NAME), key), 0, 8835) : 0u; }
MBG_FN uint32_t mbg_part_color(uint64_t seed, uint64_t key) { return key ? mbg_uniform(mbg_rand(mbg_key(seed, MBG_PART_COLOR), key), 0, 93) : 0u; }
MBG_FN uint32_t mbg_part_type(uint64_t seed, uint64_t key) { return key ? mbg_uniform(mbg_rand(mbg_key(seed, MBG_PART_TYPE), key), 0, 214) : 0u; }
MBG_FN uint32_t mbg_part_size(uint64_t seed, uint64_t key) { return key ? mbg_uniform(mbg_rand(mbg_key(seed, MBG_PART_SIZE), key), 0, 49) : 0u; }
MBG_FN uint32_t mbg_part_container(uint64_t seed, uint64_t key) { return key ? mbg_uniform(mbg_rand(mbg_key(seed, MBG_PART_CONTAINER), key), 0, 39) : 0u; }

/* Fact columns of row i. */
typedef struct mbg_lorow {
  uint32_t custkey, partkey, suppkey;
  uint32_t orderdate;
  uint32_t quantity, discount;
  uint32_t extendedprice, revenue, supplycost;
  uint32_t suppcity;
} mbg_lorow;

MBG_FN mbg_lorow mbg_star_row(uint64_t seed, uint32_t k, uint64_t i) {
  mbg_lorow r;
  r.orderdate = mbg_uniform(mbg_rand(mbg_key(seed, MBG_LO_DATE), i), 0, MBG_NDAYS - 1u);
  r.custkey = mbg_uniform(mbg_rand(mbg_key(seed, MBG_LO_CUSTKEY), i), 1, (uint32_t)mbg_star_ncust(k));
  r.suppkey = mbg_uniform(mbg_rand(mbg_key(seed, MBG_LO_SUPPKEY), i), 1, (uint32_t)mbg_star_nsupp(k));
  r.partkey = mbg_uniform(mbg_rand(mbg_key(seed, MBG_LO_PARTKEY), i), 1, (uint32_t)mbg_star_npart(k));
  r.quantity = mbg_uniform(mbg_rand(mbg_key(seed, MBG_LO_QUANTITY), i), 1, 50);
  r.discount = mbg_uniform(mbg_rand(mbg_key(seed, MBG_LO_DISCOUNT), i), 0, 10);
  r.supplycost = mbg_uniform(mbg_rand(mbg_key(seed, MBG_LO_SUPPLYCOST), i), 1, 100000);
  r.extendedprice = r.quantity * mbg_part_price(seed, r.partkey);
  r.revenue = r.extendedprice * (100u - r.discount) / 100u;
  r.suppcity = mbg_supp_city(seed, r.suppkey);
  return r;
}

#endif /* MERLE_B200_GEN_H */
