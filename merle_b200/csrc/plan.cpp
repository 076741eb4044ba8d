// plan.cpp - host planning helpers of the reference's operator API:
// col::from_bin / from_bin2 (bmpidx_create.cu:138-226) and the per-query
// bitmap recipes (recipe::perfect / many_or / candchk, bmpidx_create.cu:228-316).
#include <string.h>
#include <algorithm>
#include "common.cuh"

using namespace mb;

extern "C" mb_status mb_col_from_bin(uint32_t nbin, const uint32_t *const *bins, const uint64_t *bounds,
                                     uint64_t min, uint64_t max, mb_col *out, const uint32_t **mid) {
  if (!out || !mid) return fail(MB_ERR_INVALID, "mb_col_from_bin: NULL output");
  memset(out, 0, sizeof(*out));
  out->middle = mid;
  if (nbin == 0 || min >= max || bounds[0] > min || bounds[nbin] < max) return MB_OK;  // empty col
  while (bounds[1] <= min) --nbin, ++bins, ++bounds;   // bins left of the range
  while (bounds[nbin - 1] >= max) --nbin;              // bins right of the range
  if (nbin == 1) {
    if (bounds[0] == min && bounds[1] == max) {
      mid[0] = bins[0];
      out->nmiddle = 1;
    } else {
      out->leftmost = bins[0];
    }
    return MB_OK;
  }
  if (bounds[0] != min) {
    out->leftmost = bins[0];
    ++bounds, ++bins, --nbin;
  }
  if (bounds[nbin] != max) out->rightmost = bins[--nbin];
  if (nbin > MB_MAXBINS) return fail(MB_ERR_INVALID, "mb_col_from_bin: %u middle bins > %d", nbin, MB_MAXBINS);
  for (uint32_t i = 0; i < nbin; ++i) mid[i] = bins[i];
  out->nmiddle = nbin;
  return MB_OK;
}

extern "C" mb_status mb_col_from_bin2(uint32_t nc, const uint32_t *const *coarse, const uint64_t *cb,
                                      uint32_t nf, const uint32_t *const *fine, const uint64_t *fb,
                                      uint64_t min, uint64_t max, mb_col *out, const uint32_t **mid) {
  MB_CHECK(mb_col_from_bin(nc, coarse, cb, min, max, out, mid));
  if (out->leftmost || out->rightmost) return mb_col_from_bin(nf, fine, fb, min, max, out, mid);
  return MB_OK;
}

static uint32_t width_of(uint32_t nbit) { return nbit <= 8 ? 1 : nbit <= 16 ? 2 : nbit <= 32 ? 4 : 8; }

// create_select / create_join (bmpidx_create.cu:58-136): one bitmap of rows
// whose value (or joined dimension value) lies in [min, max), uint32 bounds.
static mb_status create_bitmap(mb_owned_vprg *o, const mb_recipe *r, int i, uint32_t lo, uint32_t hi,
                               const uint32_t **slot, void *stream) {
  if (o->nowned >= MB_MAXPTRS) return fail(MB_ERR_INVALID, "recipe: too many bitmaps");
  const uint64_t words = mb_bitmap_stride(r->factsz);
  uint32_t *bm = nullptr;
  MB_CUDA(cudaMalloc(&bm, std::max<uint64_t>(words, 4) * sizeof(uint32_t)));
  o->owned[o->nowned++] = bm;
  MB_CUDA(cudaMemsetAsync(bm, 0, std::max<uint64_t>(words, 4) * sizeof(uint32_t), as_stream(stream)));
  mb_src s;
  memset(&s, 0, sizeof(s));
  s.width = width_of(r->nbit[i]);
  if (r->fk[i]) {
    s.col = r->attr[i];
    s.fk = r->fk[i];
    s.dimsz = r->dimsz[i] == 0xffffffffu ? 0 : r->dimsz[i];
  } else {
    s.col = r->attr[i];
  }
  const uint64_t l = lo, h = hi;
  MB_CHECK(mb_bitmap_create(&s, r->factsz, &l, &h, 1, bm, words, nullptr, stream));
  *slot = bm;
  return MB_OK;
}

extern "C" mb_status mb_owned_vprg_release(mb_owned_vprg *p) {
  if (!p) return MB_OK;
  for (uint32_t i = 0; i < p->nowned; ++i) cudaFree(p->owned[i]);
  p->nowned = 0;
  return MB_OK;
}

extern "C" mb_status mb_recipe_build(const mb_recipe *r, int kind, const mb_instr *instrs, mb_owned_vprg *o,
                                     void *stream) {
  if (!r || !instrs || !o) return fail(MB_ERR_INVALID, "mb_recipe_build: NULL argument");
  memset(o, 0, sizeof(*o));
  mb_vprg &p = o->prg;
  p.factsz = r->factsz;
  for (int i = 0; i < MB_MAXNINSTR; ++i) p.instrs[i] = instrs[i];
  for (int c = 0; c < MB_MAXCOLS; ++c) p.cols[c].middle = o->mid[c];
  uint32_t ncols = 0;
  for (int i = 0; i < MB_RECIPE_COLS; ++i)
    if (r->attr[i]) ncols = i + 1;
  p.ncols = ncols;
  mb_status st = MB_OK;
  auto add_mid = [&](int c, uint32_t lo, uint32_t hi) -> mb_status {
    mb_col &col = p.cols[c];
    MB_CHECK(create_bitmap(o, r, c, lo, hi, &o->mid[c][col.nmiddle], stream));
    ++col.nmiddle;
    return MB_OK;
  };
  auto set_edge = [&](int c, bool left, uint32_t lo, uint32_t hi) -> mb_status {
    const uint32_t *bm = nullptr;
    MB_CHECK(create_bitmap(o, r, c, lo, hi, &bm, stream));
    if (left) p.cols[c].leftmost = bm;
    else p.cols[c].rightmost = bm;
    return MB_OK;
  };
  // three aligned bins (recipe::many_or): [min,min+s), [min+s,min+2s), [min+2s,max)
  auto many = [&](int i) -> mb_status {
    const uint32_t step = (r->max[i] - r->min[i]) / 3;
    if (step == 0) return add_mid(i, r->min[i], r->max[i]);
    MB_CHECK(add_mid(i, r->min[i], r->min[i] + step));
    MB_CHECK(add_mid(i, r->min[i] + step, r->min[i] + 2 * step));
    return add_mid(i, r->min[i] + 2 * step, r->max[i]);
  };
  if (kind == MB_RECIPE_PERFECT) {
    for (int i = 0; i < MB_RECIPE_COLS && st == MB_OK; ++i)
      if (r->attr[i]) st = add_mid(i, r->min[i], r->max[i]);
  } else if (kind == MB_RECIPE_MANY_OR) {
    for (int i = 0; i < MB_RECIPE_COLS && st == MB_OK; ++i)
      if (r->attr[i]) st = many(i);
  } else if (kind == MB_RECIPE_CANDCHK) {
    do {
      // column 0: left edge bin widened by step/2 below min (needs the check)
      if (!r->attr[0]) break;
      uint32_t step = (r->max[0] - r->min[0]) / 3;
      if (step == 0) {
        if ((st = set_edge(0, true, r->min[0], r->max[0] + 1)) != MB_OK) break;
      } else {
        const uint32_t l = std::max(r->min[0], step / 2) - step / 2;
        if ((st = set_edge(0, true, l, r->min[0] + step)) != MB_OK) break;
        if ((st = add_mid(0, r->min[0] + step, r->min[0] + 2 * step)) != MB_OK) break;
        if ((st = add_mid(0, r->min[0] + 2 * step, r->max[0])) != MB_OK) break;
      }
      // column 1: right edge bin widened by step/2 above max
      if (!r->attr[1]) break;
      step = (r->max[1] - r->min[1]) / 3;
      if (step == 0) {
        if ((st = set_edge(1, false, r->min[1] - 1, r->max[1])) != MB_OK) break;
      } else {
        if ((st = set_edge(1, false, r->min[1] + 2 * step, r->max[1] + step / 2)) != MB_OK) break;
        if ((st = add_mid(1, r->min[1], r->min[1] + step)) != MB_OK) break;
        if ((st = add_mid(1, r->min[1] + step, r->min[1] + 2 * step)) != MB_OK) break;
      }
      // remaining columns as many_or, stopping at the first unused one
      for (int i = 2; i < MB_RECIPE_COLS && st == MB_OK; ++i) {
        if (!r->attr[i]) break;
        st = many(i);
      }
    } while (0);
  } else {
    st = fail(MB_ERR_INVALID, "mb_recipe_build: kind %d", kind);
  }
  if (st != MB_OK) {
    mb_owned_vprg_release(o);
    return st;
  }
  return MB_OK;
}
