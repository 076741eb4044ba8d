/*
 * oracle.c - CPU restatement of the reference's fused bitmap-index query path.
 * TEST INFRASTRUCTURE ONLY (see oracle.h): the checker, never the product.
 *
 * Each function cites the reference code it restates.  Loops are scalar and
 * row-ordered on purpose: the point is to be obviously equal to the reference,
 * not fast.  OpenMP is used only for the embarrassingly parallel generators and
 * reductions whose result is order-independent (integer sums).
 */
#include "oracle.h"
#include "../include/merle_b200_gen.h"
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- values */

static uint64_t load_w(const void *p, uint64_t i, uint32_t width) {
  switch (width) {
  case 1: return ((const uint8_t *)p)[i];
  case 2: return ((const uint16_t *)p)[i];
  case 4: return ((const uint32_t *)p)[i];
  default: return ((const uint64_t *)p)[i];
  }
}

/* Reads src at row; returns 0 if a foreign key is out of range (dimsz). */
static int src_value(const mb_src *s, uint64_t row, uint64_t *v) {
  if (s->fk == NULL) {
    *v = load_w(s->col, row, s->width);
    return 1;
  }
  uint64_t key = s->fk[row];
  if (s->dimsz != 0 && key >= s->dimsz) return 0;
  *v = load_w(s->col, key, s->width);
  return 1;
}

uint32_t orc_date_to_year(uint32_t date) {
  /* ssbDateToYear, ssb/ssbdemo.h:28-39 (day 0 = 1992-01-01) */
  return date >= 2192 ? 6 : date >= 1827 ? 5 : date >= 1461 ? 4 :
         date >= 1096 ? 3 : date >= 731 ? 2 : date >= 366 ? 1 : 0;
}

/* ------------------------------------------------------- bitmap creation */

void orc_bitmap_create(const mb_src *src, uint64_t n, const uint64_t *lo,
                       const uint64_t *hi, uint32_t nbins, uint32_t *out,
                       uint64_t stride, uint64_t *popcounts) {
  /* bmpcreate<nt,vt,T,Fetch,Compar> (primitive.cuh:102-118) with the fetch and
   * compar lambdas of create_bin (bmpidx_create.cu:17-38): value in [min,max),
   * join keys >= dimsz compare as INT64_MAX, i.e. never inside a bin. */
  uint64_t W = (n + 31) / 32;
  for (uint32_t j = 0; j < nbins; ++j)
    memset(out + j * stride, 0, stride * sizeof(uint32_t));
  for (uint64_t i = 0; i < n; ++i) {
    uint64_t v;
    if (!src_value(src, i, &v)) continue;
    for (uint32_t j = 0; j < nbins; ++j)
      if (v >= lo[j] && v < hi[j]) out[j * stride + i / 32] |= 1u << (i % 32);
  }
  if (popcounts)
    for (uint32_t j = 0; j < nbins; ++j)
      for (uint64_t w = 0; w < W; ++w)
        popcounts[j] += (uint64_t)__builtin_popcount(out[j * stride + w]);
}

/* ------------------------------------------------ virtual bitmap program */

/* c' = OR of middle bins, u' = leftmost | rightmost (primitive.cuh:294-300) */
static void operand_words(const mb_col *c, uint64_t w, uint32_t *cert, uint32_t *unc) {
  uint32_t m = 0, e = 0;
  for (uint32_t k = 0; k < c->nmiddle; ++k) m |= c->middle[k][w];
  if (c->leftmost) e |= c->leftmost[w];
  if (c->rightmost) e |= c->rightmost[w];
  *cert = m;
  *unc = e;
}

static void eval_word(const mb_vprg *p, int chk, uint64_t w, uint32_t *po, uint32_t *uo) {
  uint32_t r[MB_NREGS] = {0}, u[MB_NREGS] = {0};
  for (int i = 0; i < MB_MAXNINSTR; ++i) {
    const mb_instr *in = &p->instrs[i];
    if (in->opcode == MB_END) break;
    uint32_t d = in->dstreg, s = in->src1;
    if (!chk) {
      /* vprg::nochk, primitive.cuh:201-252: edge bins OR in as certain */
      switch (in->opcode) {
      case MB_AND: r[d] &= r[s]; break;
      case MB_OR: r[d] |= r[s]; break;
      case MB_NOT: r[d] = ~r[s]; break;
      case MB_ANDM: {
        if (r[d] == 0) break; /* :215 */
        uint32_t c, e;
        operand_words(&p->cols[s], w, &c, &e);
        r[d] &= (c | e);
        break;
      }
      case MB_ORM: {
        uint32_t c, e;
        operand_words(&p->cols[s], w, &c, &e);
        r[d] |= (c | e);
        break;
      }
      }
    } else {
      /* vprg::chk, primitive.cuh:255-332: (possible, uncertain) pairs */
      switch (in->opcode) {
      case MB_AND:
        r[d] &= r[s];
        u[d] = (u[d] | u[s]) & r[d];
        break;
      case MB_OR: {
        uint32_t ps = r[s], pp = r[d], us = u[s], cs = ps & ~us;
        u[d] = (u[d] & ~cs) | (us & ~pp);
        r[d] = pp | ps;
        break;
      }
      case MB_NOT:
        r[d] = ~r[s];
        if (d != s) u[d] = u[s];
        break;
      case MB_ANDM: {
        if (r[d] == 0) break; /* :292, uncertain word left as is */
        uint32_t c, e;
        operand_words(&p->cols[s], w, &c, &e);
        r[d] &= (e | c);
        u[d] = (u[d] | e) & r[d];
        break;
      }
      case MB_ORM: {
        uint32_t c, e;
        operand_words(&p->cols[s], w, &c, &e);
        u[d] = (u[d] & ~c) | (e & ~r[d]);
        r[d] |= e | c;
        break;
      }
      }
    }
  }
  *po = r[0];
  *uo = chk ? u[0] : 0u;
}

static uint32_t tail_mask(uint64_t n, uint64_t w) {
  uint64_t W = (n + 31) / 32;
  if (w + 1 < W || (n % 32) == 0) return 0xffffffffu;
  return (1u << (n % 32)) - 1u;
}

void orc_vprg_eval(const mb_vprg *p, int chk, uint32_t *possible, uint32_t *uncertain) {
  uint64_t n = p->factsz, W = (n + 31) / 32;
  for (uint64_t w = 0; w < W; ++w) {
    uint32_t po, uo;
    eval_word(p, chk, w, &po, &uo);
    uint32_t m = tail_mask(n, w);
    possible[w] = po & m;
    if (uncertain) uncertain[w] = uo & m;
  }
}

/* -------------------------------------------------------------------- op */

int orc_op_row(const mb_op *op, uint64_t row, int chk, uint32_t nr_grp,
               int64_t *value, uint32_t *group) {
  /* Candidate check of uncertain rows: every clause needs one satisfied term
   * (s1op :27-33, s2op :49-56, s3op :74-84, s4op :116-133, synth _op :301-338). */
  if (chk) {
    uint32_t t = 0;
    for (uint32_t c = 0; c < op->nclause; ++c) {
      int any = 0;
      for (uint32_t k = 0; k < op->clause_len[c]; ++k, ++t) {
        const mb_term *tm = &op->terms[t];
        uint64_t v;
        if (!any && src_value(&op->src[tm->src], row, &v) && v >= tm->lo && v < tm->hi)
          any = 1;
      }
      if (!any) return 0;
    }
  }
  /* Dense group index: sum of mul * (xform(value) - base) in uint32
   * arithmetic (s2op :58, s3op :87-98, s4op :135-148). */
  uint32_t g = 0;
  for (uint32_t k = 0; k < op->nkey; ++k) {
    const mb_key *kk = &op->keys[k];
    uint64_t v;
    if (!src_value(&op->src[kk->src], row, &v)) return 0;
    uint32_t x = (uint32_t)v;
    if (kk->xform == MB_X_DIV) x = (uint32_t)(v / kk->div);
    else if (kk->xform == MB_X_YEAR) x = orc_date_to_year((uint32_t)v);
    g += kk->mul * (x - kk->base);
  }
  if (g >= nr_grp) return 0; /* primitive.cuh:34 */
  uint64_t a = 0, b = 0;
  switch (op->vkind) {
  case MB_V_ONE: *value = 1; break;
  case MB_V_COL:
    if (!src_value(&op->src[op->va], row, &a)) return 0;
    *value = (int64_t)a;
    break;
  case MB_V_MUL:
    if (!src_value(&op->src[op->va], row, &a) || !src_value(&op->src[op->vb], row, &b)) return 0;
    *value = (int64_t)(a * b);
    break;
  default: /* MB_V_SUB */
    if (!src_value(&op->src[op->va], row, &a) || !src_value(&op->src[op->vb], row, &b)) return 0;
    *value = (int64_t)a - (int64_t)b;
    break;
  }
  *group = g;
  return 1;
}

void orc_vprg_grpby(const mb_vprg *p, const mb_op *op, uint32_t nr_grp,
                    int64_t *out, uint64_t *nqual) {
  int chk = !orc_is_nochk(p);
  uint64_t n = p->factsz, W = (n + 31) / 32, cnt = 0;
  memset(out, 0, nr_grp * sizeof(int64_t));
  for (uint64_t w = 0; w < W; ++w) {
    uint32_t po, uo;
    eval_word(p, chk, w, &po, &uo);
    po &= tail_mask(n, w);
    while (po) {
      uint32_t b = (uint32_t)__builtin_ctz(po);
      po &= po - 1;
      int64_t v;
      uint32_t g;
      if (orc_op_row(op, w * 32 + b, chk && ((uo >> b) & 1u), nr_grp, &v, &g)) {
        out[g] = (int64_t)((uint64_t)out[g] + (uint64_t)v);
        ++cnt;
      }
    }
  }
  *nqual = cnt;
}

void orc_join_grpby(uint64_t n, const mb_op *op, uint32_t nr_grp, int64_t *out,
                    uint64_t *nqual) {
  uint64_t cnt = 0;
  memset(out, 0, nr_grp * sizeof(int64_t));
  for (uint64_t i = 0; i < n; ++i) {
    int64_t v;
    uint32_t g;
    if (orc_op_row(op, i, 1, nr_grp, &v, &g)) {
      out[g] = (int64_t)((uint64_t)out[g] + (uint64_t)v);
      ++cnt;
    }
  }
  *nqual = cnt;
}

uint64_t orc_bitmap_to_rows(const uint32_t *possible, const uint32_t *uncertain,
                            uint64_t n, uint32_t *rows) {
  uint64_t W = (n + 31) / 32, cnt = 0;
  for (uint64_t w = 0; w < W; ++w) {
    uint32_t m = possible[w] & tail_mask(n, w);
    while (m) {
      uint32_t b = (uint32_t)__builtin_ctz(m);
      m &= m - 1;
      uint32_t r = (uint32_t)(w * 32 + b);
      if (uncertain && ((uncertain[w] >> b) & 1u)) r |= 0x80000000u;
      rows[cnt++] = r;
    }
  }
  return cnt;
}

uint64_t orc_sector_count(const uint32_t *rowbits, uint64_t n, uint32_t width) {
  uint64_t rows_per_sector = 32 / width, cnt = 0;
  uint64_t nsec = (n + rows_per_sector - 1) / rows_per_sector;
  for (uint64_t s = 0; s < nsec; ++s) {
    uint64_t r0 = s * rows_per_sector, r1 = r0 + rows_per_sector;
    if (r1 > n) r1 = n;
    int hit = 0;
    for (uint64_t r = r0; r < r1 && !hit; ++r) hit = (rowbits[r / 32] >> (r % 32)) & 1u;
    cnt += (uint64_t)hit;
  }
  return cnt;
}

/* ------------------------------------------------------------ generators */

void orc_gen_flat(uint64_t seed, uint64_t row0, uint64_t n, int32_t *a, int32_t *b,
                  int32_t *c, int32_t *d, int32_t *e) {
#pragma omp parallel for schedule(static)
  for (uint64_t i = 0; i < n; ++i) {
    uint64_t r = row0 + i;
    if (a) a[i] = mbg_flat_a(seed, r);
    if (b) b[i] = mbg_flat_b(seed, r);
    if (c) c[i] = mbg_flat_c(seed, r);
    if (d) d[i] = mbg_flat_d(seed, r);
    if (e) e[i] = mbg_flat_e(seed, r);
  }
}

static void put(void *p, uint64_t i, uint32_t v, uint32_t width) {
  if (!p) return;
  if (width == 1) ((uint8_t *)p)[i] = (uint8_t)v;
  else if (width == 2) ((uint16_t *)p)[i] = (uint16_t)v;
  else ((uint32_t *)p)[i] = v;
}

void orc_gen_star(uint64_t seed, uint32_t k, uint64_t row0, uint64_t n, int width4,
                  const mb_star_cols *o) {
#pragma omp parallel for schedule(static)
  for (uint64_t i = 0; i < n; ++i) {
    mbg_lorow r = mbg_star_row(seed, k, row0 + i);
    put(o->custkey, i, r.custkey, 4);
    put(o->partkey, i, r.partkey, 4);
    put(o->suppkey, i, r.suppkey, 4);
    put(o->orderdate, i, r.orderdate, width4 ? 4 : 2);
    put(o->quantity, i, r.quantity, width4 ? 4 : 1);
    put(o->discount, i, r.discount, width4 ? 4 : 1);
    put(o->extendedprice, i, r.extendedprice, 4);
    put(o->revenue, i, r.revenue, 4);
    put(o->supplycost, i, r.supplycost, 4);
    put(o->suppcity, i, r.suppcity, width4 ? 4 : 1);
  }
}

void orc_gen_star_dims(uint64_t seed, uint32_t k, uint8_t *custcity, uint8_t *suppcity,
                       uint16_t *partmfgr) {
  uint64_t nc = mbg_star_ncust(k), ns = mbg_star_nsupp(k), np = mbg_star_npart(k);
  if (custcity) for (uint64_t i = 0; i <= nc; ++i) custcity[i] = (uint8_t)mbg_cust_city(seed, i);
  if (suppcity) for (uint64_t i = 0; i <= ns; ++i) suppcity[i] = (uint8_t)mbg_supp_city(seed, i);
  if (partmfgr) for (uint64_t i = 0; i <= np; ++i) partmfgr[i] = (uint16_t)mbg_part_mfgr(seed, i);
}

/* ------------------------------------- direct restatements (int64 sums) */

int64_t orc_s1(const orc_ssb *d, uint64_t n, uint32_t dateMin, uint32_t dateMax,
               uint32_t discntMin, uint32_t discntMax, uint32_t qtyMin, uint32_t qtyMax,
               uint64_t *nqual) {
  /* s1ref, ssb/cpuref.c:141-155 */
  int64_t res = 0;
  uint64_t cnt = 0;
  for (uint64_t i = 0; i < n; ++i) {
    if (d->loOrderDate[i] < dateMin || d->loOrderDate[i] >= dateMax) continue;
    if (d->loDiscount[i] < discntMin || d->loDiscount[i] >= discntMax) continue;
    if (d->loQuantity[i] < qtyMin || d->loQuantity[i] >= qtyMax) continue;
    res += (int64_t)d->loExtendedPrice[i] * (int64_t)d->loDiscount[i];
    ++cnt;
  }
  if (nqual) *nqual = cnt;
  return res;
}

void orc_s2(const orc_ssb *d, uint64_t n, uint32_t pMfgrMin, uint32_t pMfgrMax,
            uint32_t sCityMin, uint32_t sCityMax, int64_t *out, uint32_t nr_grp,
            uint64_t *nqual) {
  /* s2ref, ssb/cpuref.c:157-174 */
  uint64_t cnt = 0;
  memset(out, 0, nr_grp * sizeof(int64_t));
  for (uint64_t i = 0; i < n; ++i) {
    if (d->loSuppCity[i] < sCityMin || d->loSuppCity[i] >= sCityMax) continue;
    uint32_t mfgr = d->partMfgr[d->loPartKey[i]];
    if (mfgr < pMfgrMin || mfgr >= pMfgrMax) continue;
    uint32_t year = orc_date_to_year(d->loOrderDate[i]);
    uint32_t grp = (mfgr - pMfgrMin) + year * (pMfgrMax - pMfgrMin);
    if (grp >= nr_grp) continue;
    out[grp] += (int64_t)d->loRevenue[i];
    ++cnt;
  }
  if (nqual) *nqual = cnt;
}

void orc_s3(const orc_ssb *d, uint64_t n, uint32_t cCityMin, uint32_t cCityMax,
            uint32_t sCityMin, uint32_t sCityMax, uint32_t dateMin, uint32_t dateMax,
            int64_t *out, uint32_t nr_grp, uint64_t *nqual) {
  /* s3ref, ssb/cpuref.c:176-205 */
  uint64_t cnt = 0;
  memset(out, 0, nr_grp * sizeof(int64_t));
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t sCity = d->loSuppCity[i];
    if (sCity < sCityMin || sCity >= sCityMax) continue;
    uint32_t date = d->loOrderDate[i];
    if (date < dateMin || date >= dateMax) continue;
    uint32_t cCity = d->custCity[d->loCustKey[i]];
    if (cCity < cCityMin || cCity >= cCityMax) continue;
    uint32_t cmn = cCityMin, cmx = cCityMax, smn = sCityMin, smx = sCityMax;
    if (cCityMax - cCityMin >= 50) {
      cCity /= 10; cmn /= 10; cmx /= 10;
      sCity /= 10; smn /= 10; smx /= 10;
    }
    uint32_t year = orc_date_to_year(date), yearMin = orc_date_to_year(dateMin);
    uint32_t a = cmx - cmn, b = smx - smn;
    uint32_t grp = a * b * (year - yearMin) + a * (cCity - cmn) + (sCity - smn);
    if (grp >= nr_grp) continue;
    out[grp] += (int64_t)d->loRevenue[i];
    ++cnt;
  }
  if (nqual) *nqual = cnt;
}

void orc_s4(const orc_ssb *d, uint64_t n, uint32_t cCityMin, uint32_t cCityMax,
            uint32_t sCityMin, uint32_t sCityMax, uint32_t pMfgrMin, uint32_t pMfgrMax,
            uint32_t dateMin, uint32_t dateMax, int64_t *out, uint32_t nr_grp,
            uint64_t *nqual) {
  /* s4ref, ssb/cpuref.c:207-242 (value revenue - supplycost, signed here) */
  uint64_t cnt = 0;
  memset(out, 0, nr_grp * sizeof(int64_t));
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t sCity = d->loSuppCity[i];
    if (sCity < sCityMin || sCity >= sCityMax) continue;
    uint32_t date = d->loOrderDate[i];
    if (date < dateMin || date >= dateMax) continue;
    uint32_t cCity = d->custCity[d->loCustKey[i]];
    if (cCity < cCityMin || cCity >= cCityMax) continue;
    uint32_t pMfgr = d->partMfgr[d->loPartKey[i]];
    if (pMfgr < pMfgrMin || pMfgr >= pMfgrMax) continue;
    uint32_t smn = sCityMin, smx = sCityMax, pmn = pMfgrMin, pmx = pMfgrMax;
    if (sCityMax - sCityMin >= 50) { sCity /= 10; smn /= 10; smx /= 10; }
    if (pMfgrMax - pMfgrMin >= 200) { pMfgr /= 40; pmn /= 40; pmx /= 40; }
    uint32_t year = orc_date_to_year(date), yearMin = orc_date_to_year(dateMin);
    uint32_t a = smx - smn, b = pmx - pmn;
    uint32_t grp = a * b * (year - yearMin) + a * (sCity - smn) + (pMfgr - pmn);
    if (grp >= nr_grp) continue;
    out[grp] += (int64_t)d->loRevenue[i] - (int64_t)d->loSupplyCost[i];
    ++cnt;
  }
  if (nqual) *nqual = cnt;
}

void orc_synth(const void *a1, const void *a2, uint32_t bitwidth, const uint32_t *fk,
               const uint32_t *dimattr1, const uint8_t *dimattr2, uint64_t n,
               uint64_t fa1lo, uint64_t fa1hi, uint64_t fa2lo, uint64_t fa2hi,
               uint64_t da1lo, uint64_t da1hi, int64_t out[256], uint64_t *nqual) {
  /* synth_ref, synth/cpuref.c:125-169 */
  uint64_t cnt = 0;
  uint32_t w = bitwidth / 8;
  memset(out, 0, 256 * sizeof(int64_t));
  for (uint64_t i = 0; i < n; ++i) {
    uint64_t v1 = load_w(a1, i, w), v2 = load_w(a2, i, w);
    if (!((v1 >= fa1lo && v1 < fa1hi) || (v2 >= fa2lo && v2 < fa2hi))) continue;
    uint32_t key = fk[i];
    if (dimattr1[key] < da1lo || dimattr1[key] >= da1hi) continue;
    out[dimattr2[key]] += 1;
    ++cnt;
  }
  if (nqual) *nqual = cnt;
}

int64_t orc_flat_query(const int32_t *a, const int32_t *b, const int32_t *c,
                       const int32_t *d, const int32_t *e, uint64_t n, int32_t alo,
                       int32_t ahi, const int32_t *bset, uint32_t nb, int32_t clo,
                       int32_t chi, uint64_t *count) {
  /* Loop shape of s1ref (ssb/cpuref.c:141-155) with the OR-of-values
   * predicate of synth_ref (synth/cpuref.c:155-157). */
  int64_t sum = 0;
  uint64_t cnt = 0;
  for (uint64_t i = 0; i < n; ++i) {
    if (a[i] < alo || a[i] >= ahi) continue;
    int inb = 0;
    for (uint32_t k = 0; k < nb; ++k) inb |= (b[i] == bset[k]);
    if (!inb) continue;
    if (c[i] < clo || c[i] >= chi) continue;
    sum += (int64_t)e[i] * (int64_t)d[i];
    ++cnt;
  }
  *count = cnt;
  return sum;
}

int orc_is_nochk(const mb_vprg *p) {
  /* vprg::is_nochk, primitive.cuh:190-195 */
  for (uint32_t i = 0; i < p->ncols && i < MB_MAXCOLS; ++i)
    if (p->cols[i].leftmost || p->cols[i].rightmost) return 0;
  return 1;
}

/* ------------------------------------------------------- WAH interop */

/* 31-bit group g of a bitmap in this library's layout (row r is bit r % 32 of
 * word r / 32): rows 31g .. 31g + 30, row 31g + j at bit j (order 0, as
 * loadArrayFile sets bits, merle/host/wahConv.c:85-87) or at bit 30 - j
 * (order 1, as simpleJoin shifts them in, merle/host/wahConv.c:142-144,
 * and dbjoinFlatWah ballots them, merle/wahGpuCmprs.cu:215-226).
 * Rows >= nrows are 0. */
static uint32_t wah_group(const uint32_t *bm, uint64_t nrows, uint64_t g, uint32_t order) {
  uint32_t v = 0;
  for (uint32_t j = 0; j < 31; ++j) {
    uint64_t r = 31 * g + j;
    if (r >= nrows) break;
    if ((bm[r / 32] >> (r % 32)) & 1u) v |= 1u << (order ? 30 - j : j);
  }
  return v;
}

uint64_t orc_wah_encode(const uint32_t *bm, uint64_t nrows, uint32_t order, uint32_t *out) {
  /* wahCmprsCPU (merle/host/wahConv.c:36-57) over the groups: a group that is
   * neither 0 nor 0x7fffffff is a literal word; a maximal run of 0 groups is
   * 0x80000000 + run, a maximal run of 0x7fffffff groups 0xc0000000 + run. */
  uint64_t G = (nrows + 30) / 31, n = 0, g = 0;
  while (g < G) {
    uint32_t v = wah_group(bm, nrows, g, order);
    if (v != 0 && v != 0x7fffffffu) {
      out[n++] = v;
      ++g;
      continue;
    }
    uint64_t run = 0;
    while (g < G && wah_group(bm, nrows, g, order) == v) ++run, ++g;
    out[n++] = (v ? 0xc0000000u : 0x80000000u) + (uint32_t)run;
  }
  return n;
}

void orc_wah_decode(const uint32_t *wah, uint64_t nwords, uint32_t order, uint64_t nrows, uint32_t *bm,
                    uint64_t stride) {
  /* wahDecomp (merle/wahGpuCmprs.cu:34-47): word k expands to its group count
   * (a fill's 30-bit count, a literal's 1) of 31-bit groups, a fill to its
   * value repeated, a literal to its low 31 bits; the groups are then laid
   * out as rows.  Groups past the stream, rows >= nrows and the words up to
   * the stride are 0. */
  memset(bm, 0, stride * sizeof(uint32_t));
  uint64_t g = 0;
  for (uint64_t k = 0; k < nwords; ++k) {
    uint32_t w = wah[k];
    uint64_t cnt = (w & 0x80000000u) ? (w & 0x3fffffffu) : 1;
    uint32_t v = (w & 0x80000000u) ? ((w & 0x40000000u) ? 0x7fffffffu : 0u) : (w & 0x7fffffffu);
    if (v == 0) {
      g += cnt;
      continue;
    }
    for (uint64_t c = 0; c < cnt; ++c, ++g)
      for (uint32_t j = 0; j < 31; ++j) {
        uint64_t r = 31 * g + j;
        if (r >= nrows) return;
        if ((v >> (order ? 30 - j : j)) & 1u) bm[r / 32] |= 1u << (r % 32);
      }
  }
}

uint64_t orc_wah_op(uint32_t op, const uint32_t *a, uint64_t na, const uint32_t *b, uint64_t nb,
                    uint64_t ngroups, uint32_t *out) {
  /* The explicit operations wahAndExpl / wahOrExpl / wahXorExpl
   * (merle/wahGpuCmprs.cu:16-33) between the two decompressed streams, the
   * result compressed as wahCompress does (merle/wahGpuCmprs.cu:172-198,
   * the same words as wahCmprsCPU).  Streams shorter than ngroups groups are
   * extended with 0 groups. */
  uint64_t nrows = 31 * ngroups, W = (nrows + 31) / 32;
  uint32_t *x = (uint32_t *)calloc(W + 1, 4), *y = (uint32_t *)calloc(W + 1, 4);
  orc_wah_decode(a, na, 0, nrows, x, W + 1);
  orc_wah_decode(b, nb, 0, nrows, y, W + 1);
  for (uint64_t i = 0; i < W; ++i) x[i] = op == 0 ? x[i] & y[i] : op == 1 ? x[i] | y[i] : x[i] ^ y[i];
  uint64_t n = orc_wah_encode(x, nrows, 0, out);
  free(x);
  free(y);
  return n;
}
